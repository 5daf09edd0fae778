"""FP64 GPU path vs the reference, through the C ABI.

Golden fixtures hold the reference's own outputs (compiled from its sources);
the oracle restates the same algorithm and covers sizes and settings the
fixtures do not.  The FP64 path repeats the reference's operations in order,
so every comparison here is exact equality (integers and doubles alike).
"""
import ctypes

import numpy as np
import pytest

from conftest import MESH_SETS, golden_set, split_visits

pytestmark = pytest.mark.gpu

SEED = 20240611


@pytest.fixture(scope="module")
def sd():
    import sdtfe_b200

    return sdtfe_b200


@pytest.fixture(scope="module", params=MESH_SETS)
def gmesh(request, golden, sd):
    s = golden_set(golden, request.param)
    m = sd.Mesh(s["pos4"], s["tetra"], 1.0)
    yield s, m
    m.close()


def test_density_gradients_adjacency_hull(gmesh):
    s, m = gmesh
    assert np.array_equal(m.density(), s["density"])
    assert np.array_equal(m.gradients(), s["grad"])
    assert np.array_equal(m.adjacency(),
                          np.bincount(s["tetra"][:, :4].ravel(), minlength=len(s["pos4"])))
    tri = m.hull(0)
    assert np.array_equal(tri[:, :7], s["tri"])


def test_map_fp64(gmesh, sd):
    s, m = gmesh
    p = sd.map_params(24, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, SEED)
    got, st = m.map(p)
    assert np.array_equal(got, s["map"])
    assert st.rays == 24 * 24 * 4
    assert st.visits == int(s["ray_crossed"].sum())
    p2 = sd.map_params(20, 0.6, 0.5, (0.45, 0.55, 0.5), 3, 0.05, SEED + 1)
    got2, _ = m.map(p2)
    assert np.array_equal(got2, s["map2"])


def test_map_accumulates(gmesh, sd):
    s, m = gmesh
    p = sd.map_params(24, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, SEED)
    base = np.full((24, 24), 3.25)
    got, _ = m.map(p, out=base.copy())
    assert np.array_equal(got, base + s["map"])


def test_map_fp64_tile_location(gmesh, sd):
    """One shared location walk per pixel tile (dtfe_set_location) leaves the
    FP64 maps equal to the reference's, lattice degeneracies included."""
    s, m = gmesh
    m.set_location(sd.LOCATE_TILE)
    try:
        got, _ = m.map(sd.map_params(24, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, SEED))
        assert np.array_equal(got, s["map"])
        got2, _ = m.map(sd.map_params(20, 0.6, 0.5, (0.45, 0.55, 0.5), 3, 0.05, SEED + 1))
        assert np.array_equal(got2, s["map2"])
    finally:
        m.set_location(sd.LOCATE_PER_RAY)


def test_trace_visits(gmesh, sd):
    s, m = gmesh
    p = sd.map_params(24, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, SEED)
    rho, crossed, status, visits = m.trace(p, s["trace_x"], s["trace_y"], 0.0, 1.0, 1.0 / 24,
                                           max_record=4096)
    assert np.array_equal(rho, s["trace_rho"])
    assert np.array_equal(crossed, s["trace_crossed"])
    for i, v in enumerate(split_visits(s)):
        assert np.array_equal(visits[i, :crossed[i]], v), f"ray {i}"


def test_grid(gmesh, sd):
    s, m = gmesh
    g = m.grid(8, 1.0, (0.5, 0.5, 0.5), 2, SEED)
    assert np.array_equal(g, s["grid"])


@pytest.fixture(scope="module")
def medium(sd, oracle):
    """20k clustered float32 points: bigger than the fixtures, still seconds on the CPU."""
    from sdtfe_b200 import workloads

    pos4, _ = workloads.clustered_box(n=20000, seed=31, n_clusters=8, r_max=0.05)
    tetra = sd.triangulate(pos4)
    prep = oracle.prepare(pos4, tetra, 0.75)
    m = sd.Mesh(pos4, tetra, 0.75)
    yield pos4, tetra, prep, m
    m.close()


def test_medium_precompute(medium):
    pos4, tetra, prep, m = medium
    assert np.array_equal(m.density(), prep["pos"][:, 3])
    assert np.array_equal(m.gradients(), prep["grad"])
    assert np.array_equal(m.adjacency(), prep["adj"])
    assert np.array_equal(m.hull(0)[:, :7], prep["tri"][:, :7])


@pytest.mark.parametrize("G,S,box,boxz,ds", [(64, 4, 1.0, 1.0, 0.0), (37, 3, 0.7, 0.4, 0.0),
                                            (50, 1, 1.2, 1.0, 0.05), (16, 33, 0.5, 1.0, 0.0)])
def test_medium_map_vs_oracle(medium, sd, oracle, G, S, box, boxz, ds):
    pos4, tetra, prep, m = medium
    c = (0.5, 0.48, 0.52)
    want, rr, rc, rs = oracle.map(prep, G, box, boxz, c, S, ds, 99, per_ray=True)
    got, st = m.map(sd.map_params(G, box, boxz, c, S, ds, 99))
    assert np.array_equal(got, want)
    assert st.visits == int(rc.sum())
    assert list(st.status) == [int((rs == k).sum()) for k in range(6)]


@pytest.mark.parametrize("G,S,box,c", [(64, 4, 1.0, (0.5, 0.48, 0.52)), (45, 3, 1.5, (0.5, 0.5, 0.5)),
                                       (33, 5, 0.4, (0.95, 0.05, 0.5)), (16, 33, 0.5, (0.3, 0.6, 0.5))])
def test_medium_tile_location_vs_oracle(medium, sd, oracle, G, S, box, c):
    """FP64 maps with tile-shared location against the oracle's walk from
    triangle 0 for every ray: maps, ray integrals, crossings and statuses
    equal, on windows inside the hull, around it and across its corner."""
    pos4, tetra, prep, m = medium
    want, rr, rc, rs = oracle.map(prep, G, box, 1.0, c, S, 0.0, 7, per_ray=True)
    m.set_location(sd.LOCATE_TILE)
    try:
        got, st, gr, gc, gs = m.map(sd.map_params(G, box, 1.0, c, S, 0.0, 7), per_ray=True)
    finally:
        m.set_location(sd.LOCATE_PER_RAY)
    assert np.array_equal(got, want)
    assert np.array_equal(gr, rr)
    assert np.array_equal(gc, rc)
    assert np.array_equal(gs, rs)
    if box > 1.0 or c[0] > 0.9:
        assert (rs == sd.RAY_MISS).any() and (rs == sd.RAY_OK).any()


def test_location_mode_rejected(medium, sd):
    pos4, tetra, prep, m = medium
    for bad in (-1, 2):
        with pytest.raises(sd.DTFEError):
            m.set_location(bad)


@pytest.mark.parametrize("axis", [1, 2])
def test_axis_projection_vs_oracle(medium, sd, oracle, axis):
    """Projection along x / y walks the same mesh in cyclically permuted
    coordinates; densities and gradients are the canonical ones, permuted."""
    pos4, tetra, prep, m = medium
    perm = {1: [1, 2, 0], 2: [2, 0, 1]}[axis]
    pp = dict(prep)
    pp["pos"] = np.ascontiguousarray(np.column_stack([prep["pos"][:, perm], prep["pos"][:, 3]]))
    pp["grad"] = np.ascontiguousarray(prep["grad"][:, perm])
    flags, _ = oracle.forward_faces(tetra, pp["pos"])
    pp["tri"] = oracle.hull_triangles(tetra, flags)
    center = (0.5, 0.45, 0.55)
    cp = tuple(np.array(center)[perm])
    want = oracle.map(pp, 40, 1.0, 1.0, cp, 4, 0.0, 5)
    got, _ = m.map(sd.map_params(40, 1.0, 1.0, center, 4, 0.0, 5, axis=axis))
    assert np.array_equal(got, want)
    assert np.array_equal(m.hull(axis)[:, :7], pp["tri"][:, :7])


def test_medium_grid_vs_oracle(medium, oracle):
    pos4, tetra, prep, m = medium
    want, _ = oracle.grid(prep, 12, 0.9, (0.5, 0.5, 0.5), 3, 4)
    got = m.grid(12, 0.9, (0.5, 0.5, 0.5), 3, 4)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("G,box,center", [(40, 1.0, (0.5, 0.5, 0.5)), (27, 1.3, (0.45, 0.5, 0.55))])
def test_medium_grid_one_node_per_cell_vs_oracle(medium, sd, oracle, G, box, center):
    """Supersampling 1 (one node per cell), onto a grid that already holds
    values: each cell receives its node with the reference's one rounding,
    cells outside the mesh keep theirs; both precisions cross the same tets."""
    pos4, tetra, prep, m = medium
    want, _ = oracle.grid(prep, G, box, center, 1, 9)
    got = m.grid(G, box, center, 1, 9)
    assert np.array_equal(got, want)
    base = np.random.default_rng(3).random((G, G, G)) + 1.0
    got = m.grid(G, box, center, 1, 9, out=base.copy())
    assert np.array_equal(got, base + want)
    st64 = m.last_stats()
    g32 = m.grid(G, box, center, 1, 9, out=base.copy(), precision=sd.DTFE_MIXED)
    assert m.last_stats().visits == st64.visits
    assert np.max(np.abs(g32 - got) / np.abs(got)) <= 1e-5


# --------------------------------------------------------------------------
# drop-in entry points of dtfe.h / triangulate.h
# --------------------------------------------------------------------------
def test_dropin_compute_density(golden, sd, oracle):
    s = golden_set(golden, "clustered")
    L = sd.lib()
    L.dtfe_set_seed(SEED)
    try:
        pd = s["pos4"].copy()
        pd[:, 3] = -1.0
        rho = np.zeros(24 * 24)
        L.compute_density(pd, len(pd), s["tetra"], len(s["tetra"]), 24, 1.0, 1.0, rho, 1.0, 0.5,
                          0.5, 0.5, 4, 0.0)
        assert np.array_equal(rho.reshape(24, 24), s["map"])
        assert np.array_equal(pd[:, 3], s["density"])  # column 3 overwritten in place
        assert np.array_equal(pd[:, :3], s["pos4"][:, :3])  # the positions untouched
        # the map is accumulated into, as the reference's rho[p] += ...
        pd[:, 3] = 0.0
        rho = np.full(24 * 24, 0.5)
        L.compute_density(pd, len(pd), s["tetra"], len(s["tetra"]), 24, 1.0, 1.0, rho, 1.0, 0.5,
                          0.5, 0.5, 4, 0.0)
        assert np.array_equal(rho.reshape(24, 24), 0.5 + s["map"])
    finally:
        L.dtfe_set_seed(0)


def test_dropin_precompute_functions(golden, sd, reference):
    s = golden_set(golden, "uniform")
    L = sd.lib()
    pd = s["pos4"].copy()
    pp = ctypes.c_void_p(pd.ctypes.data)
    L.pre_compute_vol(ctypes.byref(pp), len(pd), s["tetra"], len(s["tetra"]), 1.0)
    assert np.array_equal(pd[:, 3], s["density"])
    gp = L.gradients(s["tetra"], len(s["tetra"]), pd)
    g = np.ctypeslib.as_array(ctypes.cast(gp, ctypes.POINTER(ctypes.c_double)),
                              shape=(len(s["tetra"]) * 3,)).copy()
    ctypes.CDLL(None).free(ctypes.c_void_p(gp))
    assert np.array_equal(g.reshape(-1, 3), s["grad"])
    bm = reference.bitmap_words(len(s["tetra"]))
    n = L.find_forward_hull(s["tetra"], len(s["tetra"]), pd, len(pd), bm)
    assert n == len(s["tri"]) and np.array_equal(bm, s["bitmap"])
    tp = L.copy_fh_triangles(s["tetra"], len(s["tetra"]), pd, len(pd), n, bm)
    tri = np.ctypeslib.as_array(ctypes.cast(tp, ctypes.POINTER(ctypes.c_int)), shape=(n * 8,)).copy()
    ctypes.CDLL(None).free(ctypes.c_void_p(tp))
    assert np.array_equal(tri.reshape(-1, 8)[:, :7], s["tri"])


def test_dropin_3d(golden, sd, oracle):
    s = golden_set(golden, "lattice")
    L = sd.lib()
    L.dtfe_set_seed(SEED)
    try:
        pd = s["pos4"].copy()
        grid = np.zeros(8 ** 3)
        L.compute_3d_density(pd, len(pd), s["tetra"], len(s["tetra"]), 8, 1.0, grid, 1.0, 0.5, 0.5,
                             0.5, 2)
        assert np.array_equal(grid.reshape(8, 8, 8), s["grid"])
        assert np.array_equal(pd[:, 3], s["density"])
        # interpolate_to_3d_grid: column 3 is a user field, no density step
        field = s["pos4"].copy()
        field[:, 3] = np.sin(7 * field[:, 0]) + field[:, 1] ** 2
        prep = oracle.prepare(field, s["tetra"], 1.0)
        prep["pos"] = field.copy()
        prep["grad"] = oracle.gradients(s["tetra"], field)
        want, _ = oracle.grid(prep, 8, 1.0, (0.5, 0.5, 0.5), 2, SEED)
        grid2 = np.zeros(8 ** 3)
        L.interpolate_to_3d_grid(field.copy(), len(field), s["tetra"], len(s["tetra"]), 8, 1.0,
                                 grid2, 0.5, 0.5, 0.5, 2)
        assert np.array_equal(grid2.reshape(8, 8, 8), want)
    finally:
        L.dtfe_set_seed(0)


# --------------------------------------------------------------------------
# edge cases
# --------------------------------------------------------------------------
def test_minimal_mesh_and_rays_outside(sd, oracle):
    from oracle.oracle import delaunay_tetra, to_pos4

    pos4 = to_pos4(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.3, 0.3, 0.3]], float))
    tetra = delaunay_tetra(pos4)
    prep = oracle.prepare(pos4, tetra, 1.0)
    with sd.Mesh(pos4, tetra, 1.0) as m:
        assert np.array_equal(m.density(), prep["pos"][:, 3])
        # a 13 x 13 map (not a multiple of 4) over a box twice the hull: most rays miss
        want, _, rc, rs = oracle.map(prep, 13, 2.0, 2.0, (0.5, 0.5, 0.5), 2, 0.0, 3, per_ray=True)
        got, st = m.map(sd.map_params(13, 2.0, 2.0, (0.5, 0.5, 0.5), 2, 0.0, 3))
        assert np.array_equal(got, want)
        assert st.status[sd.RAY_MISS] == int((rs == 1).sum()) > 0


def test_hub_vertex_of_thousands_of_tets(sd, oracle):
    """One vertex in most tets of a ball (the centre of points on a sphere):
    its density is a sum over thousands of volumes, which the per-vertex sort
    must put in the reference's order for a bit-exact result."""
    from oracle.oracle import delaunay_tetra, to_pos4

    rng = np.random.default_rng(12)
    d = rng.normal(size=(3000, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pts = np.vstack([[0.5, 0.5, 0.5], 0.5 + 0.3 * d * (1 + 1e-3 * rng.random((3000, 1)))])
    pos4 = to_pos4(pts)
    tetra = delaunay_tetra(pos4)
    prep = oracle.prepare(pos4, tetra, 1.0)
    with sd.Mesh(pos4, tetra, 1.0) as m:
        adj = m.adjacency()
        assert adj[0] > 5000  # 5,734 of the 8,016 tets
        assert np.array_equal(adj, prep["adj"])
        assert np.array_equal(m.density(), prep["pos"][:, 3])
        want = oracle.map(prep, 20, 0.7, 0.7, (0.5, 0.5, 0.5), 3, 0.0, 21)
        got, _ = m.map(sd.map_params(20, 0.7, 0.7, (0.5, 0.5, 0.5), 3, 0.0, 21))
        assert np.array_equal(got, want)


def test_invalid_tetra_rejected_before_any_gather(sd):
    from oracle.oracle import to_pos4

    pos4 = to_pos4(np.random.default_rng(1).random((10, 3)))
    bad = np.array([[0, 1, 2, 99, -1, -1, -1, -1]], np.int32)
    with pytest.raises(sd.DTFEError) as e:
        sd.Mesh(pos4, bad)
    assert e.value.status == 4
    bad = np.array([[0, 1, 2, 3, -1, 7, -1, -1]], np.int32)
    with pytest.raises(sd.DTFEError):
        sd.Mesh(pos4, bad)


def test_cyclic_neighbour_links_end_with_budget(golden, sd, oracle):
    """Corrupt links make the walk cycle; the visit budget stops it with a
    status (checked against the oracle's identical budget logic)."""
    s = golden_set(golden, "uniform")
    tet = s["tetra"].copy()
    inner = tet[:, 4:] >= 0
    tet[:, 4:][inner] = (np.arange(len(tet))[:, None].repeat(4, 1) % 2)[inner]
    prep = oracle.prepare(s["pos4"], tet, 1.0)
    xs = np.linspace(0.2, 0.8, 9)
    ys = np.linspace(0.3, 0.7, 9)
    want = oracle.trace(prep, xs, ys, 0.0, 1.0, 0.04, 1, max_visits=500)
    with sd.Mesh(s["pos4"], tet, 1.0) as m:
        p = sd.map_params(8, 1.0, 1.0, (0.5, 0.5, 0.5), 1, 0.0, 1, max_visits=500)
        got = m.trace(p, xs, ys, 0.0, 1.0, 0.04)
    for a, b in zip(got[:3], want[:3]):
        assert np.array_equal(a, b)
    assert (got[2] != 0).all()


def test_bad_parameters_rejected(golden, sd):
    s = golden_set(golden, "uniform")
    with sd.Mesh(s["pos4"], s["tetra"], 1.0) as m:
        for kw in (dict(grid_dim=0), dict(n_samples=0), dict(box_len=0.0), dict(axis=3),
                   dict(precision=7)):
            args = dict(grid_dim=8, box_len=1.0, box_len_z=1.0, center=(0.5, 0.5, 0.5),
                        n_samples=2)
            args.update(kw)
            with pytest.raises(sd.DTFEError):
                m.map(sd.map_params(**args))
