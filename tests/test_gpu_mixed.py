"""Mixed-precision path (FP32 walk, guarded FP64) vs the FP64 path.

Integer outputs must be identical: the filtered FP32 sign tests fall back to
the reference's FP64 products whenever FP32 cannot decide, so every ray
visits the same tets, in the same order, with the same status.  The map
values may differ by FP32 rounding; the tolerance is a maximum relative error
of 1e-5 per pixel against the FP64 map, and the projected mass must agree.
"""
import numpy as np
import pytest

from conftest import MESH_SETS, golden_set

pytestmark = pytest.mark.gpu

MAX_REL = 1e-5


@pytest.fixture(scope="module")
def sd():
    import sdtfe_b200

    return sdtfe_b200


def rel_err(got, want):
    ok = np.abs(want) > 0
    assert np.array_equal(got == 0, want == 0), "zero pattern differs"
    r = np.abs(got - want)[ok] / np.abs(want[ok])
    return float(r.max()) if r.size else 0.0


@pytest.mark.parametrize("name", MESH_SETS)
def test_mixed_visits_identical_on_fixtures(golden, sd, name):
    s = golden_set(golden, name)
    with sd.Mesh(s["pos4"], s["tetra"], 1.0) as m:
        p64 = sd.map_params(24, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 20240611)
        p32 = sd.map_params(24, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 20240611,
                            precision=sd.DTFE_MIXED)
        r64, c64, s64, v64 = m.trace(p64, s["trace_x"], s["trace_y"], 0.0, 1.0, 1 / 24, 4096)
        r32, c32, s32, v32 = m.trace(p32, s["trace_x"], s["trace_y"], 0.0, 1.0, 1 / 24, 4096)
        assert np.array_equal(c32, c64)
        assert np.array_equal(s32, s64)
        assert np.array_equal(v32, v64)
        assert rel_err(r32, r64) <= MAX_REL
        m64, st64 = m.map(p64)
        m32, st32 = m.map(p32)
        assert st32.visits == st64.visits
        assert list(st32.status) == list(st64.status)
        assert rel_err(m32, m64) <= MAX_REL


@pytest.fixture(scope="module")
def clustered(sd):
    from sdtfe_b200 import workloads

    pos4, _ = workloads.clustered_box(n=60000, seed=41, n_clusters=10, r_max=0.02)
    tetra = sd.triangulate(pos4)
    m = sd.Mesh(pos4, tetra, 1.0)
    yield pos4, tetra, m
    m.close()


@pytest.mark.parametrize("G,S", [(128, 16), (96, 5)])
def test_mixed_map_error_and_topology(clustered, sd, G, S):
    pos4, tetra, m = clustered
    p64 = sd.map_params(G, 1.0, 1.0, (0.5, 0.5, 0.5), S, 0.0, 3)
    p32 = sd.map_params(G, 1.0, 1.0, (0.5, 0.5, 0.5), S, 0.0, 3, precision=sd.DTFE_MIXED)
    m64, st64 = m.map(p64)
    m32, st32 = m.map(p32)
    assert st32.visits == st64.visits
    assert list(st32.status) == list(st64.status)
    err = rel_err(m32, m64)
    assert err <= MAX_REL, err
    # projected mass: the whole unit box is mapped
    d = 1.0 / G
    assert abs(m32.sum() * d * d - m64.sum() * d * d) <= 1e-6 * m64.sum() * d * d


def test_mixed_rays_through_cluster_cores(clustered, sd):
    """Rays aimed at the densest vertices: near-degenerate Plücker products
    go to FP64 and the visit sequences still match."""
    pos4, tetra, m = clustered
    rho = m.density()
    top = np.argsort(rho)[-200:]
    xs, ys = pos4[top, 0] + 1e-9, pos4[top, 1] - 1e-9
    p64 = sd.map_params(8, 1.0, 1.0, (0.5, 0.5, 0.5), 1, 0.0, 9)
    p32 = sd.map_params(8, 1.0, 1.0, (0.5, 0.5, 0.5), 1, 0.0, 9, precision=sd.DTFE_MIXED)
    r64, c64, s64, v64 = m.trace(p64, xs, ys, 0.0, 1.0, 1 / 2048, 2048)
    r32, c32, s32, v32 = m.trace(p32, xs, ys, 0.0, 1.0, 1 / 2048, 2048)
    assert np.array_equal(s32, s64) and np.array_equal(c32, c64)
    assert np.array_equal(v32, v64)
    assert rel_err(r32, r64) <= MAX_REL


def test_mixed_on_float64_coordinates_uses_fp64_records(sd):
    """Coordinates that are not floats: the filter adds the records' rounding
    and the exact operands come from the FP64 records."""
    from sdtfe_b200 import workloads

    pos4, _ = workloads.uniform_box(n=8000, seed=12)
    tetra = sd.triangulate(pos4)
    with sd.Mesh(pos4, tetra, 1.0) as m:
        assert m.info().fp32_exact == 0
        p64 = sd.map_params(64, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 21)
        p32 = sd.map_params(64, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 21, precision=sd.DTFE_MIXED)
        m64, st64 = m.map(p64)
        m32, st32 = m.map(p32)
        assert st32.visits == st64.visits
        assert rel_err(m32, m64) <= MAX_REL


@pytest.mark.parametrize("axis", [1, 2])
def test_mixed_other_axes(clustered, sd, axis):
    pos4, tetra, m = clustered
    p64 = sd.map_params(64, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 8, axis=axis)
    p32 = sd.map_params(64, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 8, axis=axis,
                        precision=sd.DTFE_MIXED)
    m64, st64 = m.map(p64)
    m32, st32 = m.map(p32)
    assert st32.visits == st64.visits
    assert rel_err(m32, m64) <= MAX_REL


def test_mixed_sub_slab_guard(clustered, sd):
    """A slab that cuts through the cloud: midpoints near the slab planes are
    decided by the reference's FP64 midpoint."""
    pos4, tetra, m = clustered
    p64 = sd.map_params(64, 0.8, 0.3, (0.5, 0.5, 0.45), 6, 0.0, 10)
    p32 = sd.map_params(64, 0.8, 0.3, (0.5, 0.5, 0.45), 6, 0.0, 10, precision=sd.DTFE_MIXED)
    m64, _ = m.map(p64)
    m32, st32 = m.map(p32)
    assert rel_err(m32, m64) <= MAX_REL


def test_kernel_variants_identical_and_autotune(clustered, sd):
    """Every kernel variant computes the same rays in the same per-pixel order,
    so the maps are bit-identical; the autotuner times them all and keeps one."""
    pos4, tetra, m = clustered
    p32 = sd.map_params(96, 1.0, 1.0, (0.5, 0.5, 0.5), 8, 0.0, 4, precision=sd.DTFE_MIXED)
    first = None
    try:
        for v in range(sd.lib().dtfe_num_variants()):
            m.set_variant(v)
            got, st = m.map(p32)
            if first is None:
                first = got
            else:
                assert np.array_equal(got, first), f"variant {v}"
        best, table = m.autotune(p32)
        assert 0 <= best < len(table)
        assert all(t["ms"] > 0 for t in table)
        assert m.info().map_variant == best
        assert table[best]["ms"] == min(t["ms"] for t in table)
    finally:
        m.set_variant(-1)


def test_mixed_signed_field_mesh(clustered, sd):
    """A field mesh (column 3 is a field of either sign, as interpolate_field2grid
    uses): tets whose vertex values change sign or vanish cannot bound their FP32
    field value relative to itself and take the FP64 field value.  Pixel values
    can cross zero, so the error is measured against the map's largest value."""
    pos4, tetra, _ = clustered
    f4 = pos4.copy()
    f4[:, 3] = np.sin(9.0 * pos4[:, 0]) * np.cos(7.0 * pos4[:, 1]) + 0.3 * (pos4[:, 2] - 0.5)
    with sd.Mesh(f4, tetra, 1.0, sd.MESH_FIELD) as m:
        for axis in (0, 1):
            p64 = sd.map_params(80, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 31, axis=axis)
            p32 = sd.map_params(80, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 31, axis=axis,
                                precision=sd.DTFE_MIXED)
            m64, st64 = m.map(p64)
            m32, st32 = m.map(p32)
            assert st32.visits == st64.visits
            assert (m64 < 0).any() and (m64 > 0).any()
            assert np.max(np.abs(m32 - m64)) <= MAX_REL * np.max(np.abs(m64))


def test_mixed_first_tet_on_hull_slivers(sd):
    """A jittered lattice: flat tets along the hull faces, rays that start on
    them, zero-sign cases and perturbations; the mixed walk must still visit the
    FP64 path's tets and stay within tolerance."""
    rng = np.random.default_rng(44)
    g = (np.arange(14) + 0.5) / 14
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    lat = lat + rng.normal(scale=0.02 / 14, size=lat.shape)
    pos4 = np.zeros((len(lat), 4))
    pos4[:, :3] = lat.astype(np.float32)
    tetra = sd.triangulate(pos4)
    with sd.Mesh(pos4, tetra, 1.0) as m:
        p64 = sd.map_params(56, 1.0, 1.0, (0.5, 0.5, 0.5), 8, 0.0, 3)
        p32 = sd.map_params(56, 1.0, 1.0, (0.5, 0.5, 0.5), 8, 0.0, 3, precision=sd.DTFE_MIXED)
        m64, st64 = m.map(p64)
        m32, st32 = m.map(p32)
        assert st32.visits == st64.visits
        assert list(st32.status) == list(st64.status)
        assert rel_err(m32, m64) <= MAX_REL


def test_mixed_corrupt_links_end_like_fp64(golden, sd):
    """Neighbour links that do not point back (a 2-cycle): the per-entry-face
    records mark such neighbours, the general step follows the mesh rows, and
    the visit budget ends each ray with the FP64 path's status and count."""
    s = golden_set(golden, "uniform")
    tet = s["tetra"].copy()
    inner = tet[:, 4:] >= 0
    tet[:, 4:][inner] = (np.arange(len(tet))[:, None].repeat(4, 1) % 2)[inner]
    xs = np.linspace(0.2, 0.8, 9)
    ys = np.linspace(0.3, 0.7, 9)
    with sd.Mesh(s["pos4"], tet, 1.0) as m:
        p64 = sd.map_params(8, 1.0, 1.0, (0.5, 0.5, 0.5), 1, 0.0, 1, max_visits=500)
        p32 = sd.map_params(8, 1.0, 1.0, (0.5, 0.5, 0.5), 1, 0.0, 1, max_visits=500,
                            precision=sd.DTFE_MIXED)
        r64, c64, s64, _ = m.trace(p64, xs, ys, 0.0, 1.0, 0.04)
        r32, c32, s32, _ = m.trace(p32, xs, ys, 0.0, 1.0, 0.04)
    assert np.array_equal(s32, s64) and np.array_equal(c32, c64)
    assert (s32 != 0).all()


@pytest.mark.parametrize("G,S", [(1, 300), (5, 257), (3, 33)])
def test_more_samples_than_threads(golden, sd, oracle, G, S):
    """A pixel with more samples than a tile has threads (the tile walks them
    in several passes) and maps of one or a few pixels: FP64 equals the
    oracle, mixed stays within tolerance of FP64."""
    s = golden_set(golden, "clustered")
    prep = oracle.prepare(s["pos4"], s["tetra"], 1.0)
    want = oracle.map(prep, G, 0.5, 1.0, (0.5, 0.5, 0.5), S, 0.0, 61)
    with sd.Mesh(s["pos4"], s["tetra"], 1.0) as m:
        m64, st64 = m.map(sd.map_params(G, 0.5, 1.0, (0.5, 0.5, 0.5), S, 0.0, 61))
        m32, st32 = m.map(sd.map_params(G, 0.5, 1.0, (0.5, 0.5, 0.5), S, 0.0, 61,
                                        precision=sd.DTFE_MIXED))
    assert np.array_equal(m64, want)
    assert st64.rays == G * G * S and st32.visits == st64.visits
    assert rel_err(m32, m64) <= MAX_REL
