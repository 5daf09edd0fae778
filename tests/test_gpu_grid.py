"""The 3-D grid (src/dtfe.c:376-516, 658-735) in both precisions, through
the C ABI.

The FP64 grid equals the oracle cell for cell (tests/test_gpu_parity.py);
here the mixed grid (FP32 walk with guarded FP64, FP64 node values) is held
to the FP64 grid: the same tets crossed and every cell within 1e-5 relative,
zero cells zero in both, on the reference fixtures, a clustered mesh, and
with supersampling.
"""
import numpy as np
import pytest

from conftest import MESH_SETS, golden_set

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-5


@pytest.fixture(scope="module")
def sd():
    import sdtfe_b200

    return sdtfe_b200


def grid_err(got, want):
    assert np.array_equal(got == 0, want == 0), "zero cells differ"
    nz = want != 0
    return float(np.max(np.abs(got[nz] - want[nz]) / np.abs(want[nz]))) if nz.any() else 0.0


@pytest.mark.parametrize("name", MESH_SETS)
def test_mixed_grid_fixtures(golden, sd, name):
    s = golden_set(golden, name)
    with sd.Mesh(s["pos4"], s["tetra"], 1.0) as m:
        g64 = m.grid(8, 1.0, (0.5, 0.5, 0.5), 2, 20240611)
        st64 = m.last_stats()
        g32 = m.grid(8, 1.0, (0.5, 0.5, 0.5), 2, 20240611, precision=sd.DTFE_MIXED)
        st32 = m.last_stats()
    assert np.array_equal(g64, s["grid"])
    assert st32.visits == st64.visits and list(st32.status) == list(st64.status)
    assert grid_err(g32, g64) <= GRID_TOL


@pytest.fixture(scope="module")
def clustered(sd):
    from sdtfe_b200 import workloads

    pos4, _ = workloads.clustered_box(n=60000, seed=11, n_clusters=12, r_max=0.05)
    tetra = sd.triangulate(pos4)
    m = sd.Mesh(pos4, tetra, 1.0)
    yield m
    m.close()


@pytest.mark.parametrize("G,box,center,ss", [(64, 1.0, (0.5, 0.5, 0.5), 1),
                                             (48, 0.6, (0.45, 0.55, 0.5), 2),
                                             (33, 1.2, (0.5, 0.5, 0.5), 1)])
def test_mixed_grid_clustered(clustered, sd, G, box, center, ss):
    m = clustered
    g64 = m.grid(G, box, center, ss, 77)
    st64 = m.last_stats()
    g32 = m.grid(G, box, center, ss, 77, precision=sd.DTFE_MIXED)
    st32 = m.last_stats()
    assert st32.visits == st64.visits and list(st32.status) == list(st64.status)
    assert grid_err(g32, g64) <= GRID_TOL
    assert (g64 != 0).mean() > 0.3


def test_grid_device_accumulates(clustered, sd):
    import torch

    m = clustered
    G = 40
    want = m.grid(G, 1.0, (0.5, 0.5, 0.5), 1, 5, out=np.full((G, G, G), 2.5),
                  precision=sd.DTFE_MIXED)
    d = torch.full((G, G, G), 2.5, dtype=torch.float64, device="cuda")
    m.grid_device(G, 1.0, (0.5, 0.5, 0.5), 1, 5, d.data_ptr(), precision=sd.DTFE_MIXED)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), want)
