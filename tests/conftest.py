import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_small.npz")
MESH_SETS = ("uniform", "clustered", "lattice")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def golden_set(g, name):
    pre = name + "/"
    return {k[len(pre):]: v for k, v in g.items() if k.startswith(pre)}


def split_visits(s):
    ends = np.cumsum(s["visit_len"])
    starts = ends - s["visit_len"]
    return [s["visits"][a:b] for a, b in zip(starts, ends)]


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference

    try:
        return Reference()
    except FileNotFoundError as e:
        pytest.skip(str(e))
