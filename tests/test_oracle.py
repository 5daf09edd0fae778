"""The oracle (C restatement) pinned against the reference's own outputs.

The golden fixtures were produced by the reference's C code compiled from its
sources (tests/golden/make_golden.py); every comparison here is bit-exact.
"""
import numpy as np
import pytest

from conftest import MESH_SETS, golden_set, split_visits


@pytest.mark.parametrize("name", MESH_SETS)
def test_precompute_matches_golden(golden, oracle, name):
    s = golden_set(golden, name)
    prep = oracle.prepare(s["pos4"], s["tetra"], 1.0)
    assert np.array_equal(prep["pos"][:, 3], s["density"])
    assert np.array_equal(prep["grad"], s["grad"])
    # forward faces: the reference's bitmap holds 4 face bits per word (one word per tet)
    words = s["bitmap"][: len(s["tetra"])]
    bits = ((words[:, None] >> np.arange(4)) & 1).reshape(-1).astype(np.uint8)
    assert np.array_equal(prep["flags"], bits)
    assert np.array_equal(prep["tri"][:, :7], s["tri"])
    assert np.array_equal(prep["adj"], np.bincount(s["tetra"][:, :4].ravel(), minlength=len(s["pos4"])))


@pytest.mark.parametrize("name", MESH_SETS)
def test_map_matches_golden(golden, oracle, name):
    s = golden_set(golden, name)
    prep = oracle.prepare(s["pos4"], s["tetra"], 1.0)
    m, rr, rc, rs = oracle.map(prep, 24, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 20240611, per_ray=True)
    assert np.array_equal(m, s["map"])
    assert np.array_equal(rr, s["ray_rho"])
    assert np.array_equal(rc, s["ray_crossed"])
    m2 = oracle.map(prep, 20, 0.6, 0.5, (0.45, 0.55, 0.5), 3, 0.05, 20240611 + 1)
    assert np.array_equal(m2, s["map2"])


@pytest.mark.parametrize("name", MESH_SETS)
def test_trace_visits_match_golden(golden, oracle, name):
    s = golden_set(golden, name)
    prep = oracle.prepare(s["pos4"], s["tetra"], 1.0)
    rho, crossed, status, visits = oracle.trace(prep, s["trace_x"], s["trace_y"], 0.0, 1.0,
                                                1.0 / 24, 20240611, max_record=4096)
    assert np.array_equal(rho, s["trace_rho"])
    assert np.array_equal(crossed, s["trace_crossed"])
    for i, v in enumerate(split_visits(s)):
        assert np.array_equal(visits[i, :crossed[i]], v), f"ray {i}"


@pytest.mark.parametrize("name", MESH_SETS)
def test_grid_matches_golden(golden, oracle, name):
    s = golden_set(golden, name)
    prep = oracle.prepare(s["pos4"], s["tetra"], 1.0)
    g, _ = oracle.grid(prep, 8, 1.0, (0.5, 0.5, 0.5), 2, 20240611)
    assert np.array_equal(g, s["grid"])


def test_lattice_exercises_degenerate_branches(golden, oracle):
    """Rays aimed at vertices of the jittered lattice hit zero Plücker signs."""
    s = golden_set(golden, "lattice")
    prep = oracle.prepare(s["pos4"], s["tetra"], 1.0)
    rho, crossed, status, _ = oracle.trace(prep, s["trace_x"], s["trace_y"], 0.0, 1.0, 1.0 / 24,
                                           20240611)
    # the vertex-aimed rays still produce the reference's integrals
    assert np.array_equal(rho, s["trace_rho"])
    assert (crossed[24:36] > 0).all()


def test_oracle_matches_live_reference(reference, oracle):
    """A fresh seeded mesh: restatement == reference compiled from its sources."""
    from oracle.oracle import delaunay_tetra, to_pos4

    rng = np.random.default_rng(99)
    pos4 = to_pos4(rng.random((1500, 3)))
    tetra = delaunay_tetra(pos4)
    po = oracle.prepare(pos4, tetra, 2.5)
    pr = reference.prepare(pos4, tetra, 2.5)
    assert np.array_equal(po["pos"], pr["pos"])
    assert np.array_equal(po["grad"], pr["grad"])
    assert np.array_equal(po["tri"][:, :7], pr["tri"][:, :7])
    mo = oracle.map(po, 32, 0.9, 0.8, (0.5, 0.5, 0.5), 5, 0.0, 77)
    mr = reference.map(pr, 32, 0.9, 0.8, (0.5, 0.5, 0.5), 5, 0.0, 77)
    assert np.array_equal(mo, mr)


def test_oracle_budget_stops_cyclic_links(golden, oracle):
    """Corrupt neighbour links (a 2-cycle) end with a budget status, not a hang."""
    s = golden_set(golden, "uniform")
    tet = s["tetra"].copy()
    prep = oracle.prepare(s["pos4"], tet, 1.0)
    # make every interior neighbour point back at tet 0 / 1 alternately
    bad = prep["tetra"].copy()
    inner = bad[:, 4:] >= 0
    bad[:, 4:][inner] = (np.arange(len(bad))[:, None].repeat(4, 1) % 2)[inner]
    prep["tetra"] = np.ascontiguousarray(bad)
    rho, crossed, status, _ = oracle.trace(prep, np.array([0.5]), np.array([0.5]), 0.0, 1.0, 0.04,
                                           1, max_visits=1000)
    assert status[0] in (2, 4)  # no exit face, or budget
    assert crossed[0] == 0
