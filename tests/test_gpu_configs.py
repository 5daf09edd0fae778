"""Parity at the benchmark configurations' own sizes, through the C ABI.

* Plain method, small (N = 32,768 float64 points uniform in the unit box, a
  256 x 256 z-projection, 4 samples per pixel, FP64): the GPU map, every ray's
  integral, crossing count and status, the densities, gradients and
  per-vertex adjacency counts equal the oracle's bit for bit; sampled rays
  visit the reference's own tets in the reference's order (its C, built from
  its sources, with the visit hook); the mixed path crosses the same tets with
  the same statuses within 1e-5.
* Clustered, the single-map recipe at a quarter of the points (262,144
  float32 points, half in 100 r^-2 clusters): a full-box 256 x 256 x 16 map
  equal to the oracle's bit for bit in FP64, its projected mass against the
  particle count, and a 256 x 256 x 16 window at the single map's own pixel
  size (1/2048) on the densest part of the box, mixed against FP64: the same
  crossings and statuses for every ray, map error <= 1e-5.

The reference itself (src/dtfe.c:554-654) draws its sample offsets from
rand(); the FP64 path and the oracle both draw them from the counter-based
generator with an explicit seed, so their maps can be compared exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 4242
MIXED_TOL = 1e-5  # the mixed path's bound on a map's relative error against FP64


@pytest.fixture(scope="module")
def sd():
    import sdtfe_b200

    return sdtfe_b200


def rel_err(got, want):
    nz = want != 0
    assert np.array_equal(got == 0, want == 0), "zero pixels differ"
    return float(np.max(np.abs(got[nz] - want[nz]) / np.abs(want[nz]))) if nz.any() else 0.0


# --------------------------------------------------------------------------
# plain method, small: 32,768 uniform float64 points, 256^2 x 4, FP64
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def config1(sd, oracle):
    from sdtfe_b200 import workloads

    pos4, spec = workloads.uniform_box()
    assert len(pos4) == 32768 and (spec.grid_dim, spec.n_samples) == (256, 4)
    tetra = sd.triangulate(pos4)
    prep = oracle.prepare(pos4, tetra, 1.0)
    m = sd.Mesh(pos4, tetra, 1.0)
    yield pos4, tetra, spec, prep, m
    m.close()


def _params(sd, spec, precision, seed=SEED):
    return sd.map_params(spec.grid_dim, spec.box_len, spec.box_len_z, spec.center, spec.n_samples,
                         0.0, seed, precision=precision)


def test_config1_precompute_bit_exact(config1):
    pos4, tetra, spec, prep, m = config1
    assert np.array_equal(m.density(), prep["pos"][:, 3])
    assert np.array_equal(m.gradients(), prep["grad"])
    assert np.array_equal(m.adjacency(), prep["adj"])
    assert np.array_equal(m.adjacency(), np.bincount(tetra[:, :4].ravel(), minlength=len(pos4)))
    assert np.array_equal(m.hull(0)[:, :7], prep["tri"][:, :7])


def test_config1_fp64_map_and_rays_bit_exact(config1, sd, oracle):
    pos4, tetra, spec, prep, m = config1
    want, rr, rc, rs = oracle.map(prep, spec.grid_dim, spec.box_len, spec.box_len_z, spec.center,
                                  spec.n_samples, 0.0, SEED, per_ray=True)
    got, st, gr, gc, gs = m.map(_params(sd, spec, sd.DTFE_FP64), per_ray=True)
    assert np.array_equal(got, want)
    assert np.array_equal(gr, rr)
    assert np.array_equal(gc, rc)
    assert np.array_equal(gs, rs)
    assert st.rays == spec.rays and st.visits == int(rc.sum())
    # uniform points fill the box: the projected mass is the particle count,
    # up to the Monte Carlo error of 4 samples per pixel
    mass = got.sum() * (spec.box_len / spec.grid_dim) ** 2
    assert abs(mass / len(pos4) - 1.0) < 2e-3


def test_config1_fp64_tile_location_bit_exact(config1, sd):
    """Config 1 with tile-shared location: the same map and rays as the
    reference's per-ray location walk."""
    pos4, tetra, spec, prep, m = config1
    want = m.map(_params(sd, spec, sd.DTFE_FP64), per_ray=True)
    m.set_location(sd.LOCATE_TILE)
    try:
        got = m.map(_params(sd, spec, sd.DTFE_FP64), per_ray=True)
    finally:
        m.set_location(sd.LOCATE_PER_RAY)
    for k in (0, 2, 3, 4):
        assert np.array_equal(got[k], want[k])
    assert got[1].visits == want[1].visits


def test_config1_mixed_same_crossings_within_tolerance(config1, sd):
    pos4, tetra, spec, prep, m = config1
    g64, s64, r64, c64, t64 = m.map(_params(sd, spec, sd.DTFE_FP64), per_ray=True)
    g32, s32, r32, c32, t32 = m.map(_params(sd, spec, sd.DTFE_MIXED), per_ray=True)
    assert np.array_equal(c32, c64)
    assert np.array_equal(t32, t64)
    assert s32.visits == s64.visits
    assert rel_err(g32, g64) <= MIXED_TOL


def test_config1_visit_sequences_vs_reference(config1, sd, reference):
    """200 rays at seeded positions: the reference's own walk (its C with the
    visit hook) against the FP64 and mixed walks, tet for tet."""
    pos4, tetra, spec, prep, m = config1
    rng = np.random.default_rng(SEED)
    xs = rng.uniform(0.0, 1.0, 200)
    ys = rng.uniform(0.0, 1.0, 200)
    dxy = spec.box_len / spec.grid_dim
    rp = reference.prepare(pos4, tetra, 1.0)
    rho, crossed, visits = reference.trace(rp, xs, ys, 0.0, 1.0, dxy, SEED, record_visits=True)
    assert (crossed > 0).sum() > 150
    for prec in (sd.DTFE_FP64, sd.DTFE_MIXED):
        p = _params(sd, spec, prec)
        grho, gcr, gst, gvis = m.trace(p, xs, ys, 0.0, 1.0, dxy, max_record=4096)
        assert np.array_equal(gcr, crossed)
        if prec == sd.DTFE_FP64:
            assert np.array_equal(grho, rho)
        else:
            ok = rho != 0
            assert np.max(np.abs(grho[ok] - rho[ok]) / np.abs(rho[ok])) <= MIXED_TOL
        for i, v in enumerate(visits):
            assert np.array_equal(gvis[i, :gcr[i]], v), f"ray {i}, precision {prec}"


# --------------------------------------------------------------------------
# clustered single-map recipe at 262,144 points
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def clustered(sd, oracle):
    from sdtfe_b200 import workloads

    pos4, _ = workloads.clustered_box(n=1 << 18)
    tetra = sd.triangulate(pos4)
    prep = oracle.prepare(pos4, tetra, 1.0)
    m = sd.Mesh(pos4, tetra, 1.0)
    yield pos4, tetra, prep, m
    m.close()


def test_clustered_full_box_fp64_bit_exact_and_mass(clustered, sd, oracle):
    pos4, tetra, prep, m = clustered
    G, S = 256, 16
    want = oracle.map(prep, G, 1.0, 1.0, (0.5, 0.5, 0.5), S, 0.0, SEED)
    got, st = m.map(sd.map_params(G, 1.0, 1.0, (0.5, 0.5, 0.5), S, 0.0, SEED))
    assert np.array_equal(got, want)
    mix, st32 = m.map(sd.map_params(G, 1.0, 1.0, (0.5, 0.5, 0.5), S, 0.0, SEED,
                                    precision=sd.DTFE_MIXED))
    assert st32.visits == st.visits and list(st32.status) == list(st.status)
    assert rel_err(mix, got) <= MIXED_TOL
    # DTFE conserves mass: the map's integral estimates the particle count
    # (here with the Monte Carlo error of 16 samples per pixel over clusters)
    px = (1.0 / G) ** 2
    assert abs(got.sum() * px / len(pos4) - 1.0) < 1e-2
    assert abs(mix.sum() / got.sum() - 1.0) < 1e-7


def test_clustered_fp64_tile_location_bit_exact(clustered, sd):
    """The clustered recipe at 512 x 512 x 16 (tiles along the hull's edges
    included): tile-shared location gives the per-ray walk's rays exactly."""
    pos4, tetra, prep, m = clustered
    p = sd.map_params(512, 1.0, 1.0, (0.5, 0.5, 0.5), 16, 0.0, SEED)
    want = m.map(p, per_ray=True)
    m.set_location(sd.LOCATE_TILE)
    try:
        got = m.map(p, per_ray=True)
    finally:
        m.set_location(sd.LOCATE_PER_RAY)
    for k in (0, 2, 3, 4):
        assert np.array_equal(got[k], want[k])
    assert list(got[1].status) == list(want[1].status)


def test_clustered_window_at_single_map_pixel_size(clustered, sd):
    """A 256 x 256 x 16 window at the 2048-pixel map's pixel size, centred on
    the densest pixel of a coarse map (a cluster core: the most slivers,
    FP64 fallbacks and short chords)."""
    pos4, tetra, prep, m = clustered
    coarse, _ = m.map(sd.map_params(64, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 7))
    row, col = np.unravel_index(np.argmax(coarse), coarse.shape)
    box = 256 / 2048
    c = (np.clip((col + 0.5) / 64, box / 2, 1 - box / 2),
         np.clip((row + 0.5) / 64, box / 2, 1 - box / 2), 0.5)
    kw = dict(grid_dim=256, box_len=box, box_len_z=1.0, center=c, n_samples=16, seed=SEED)
    g64, s64, r64, c64, t64 = m.map(sd.map_params(**kw), per_ray=True)
    g32, s32, r32, c32, t32 = m.map(sd.map_params(**kw, precision=sd.DTFE_MIXED), per_ray=True)
    assert np.array_equal(c32, c64)
    assert np.array_equal(t32, t64)
    # rays either cross the mesh or miss its hull (a window near the box's
    # edge reaches past the hull of the wrapped clusters)
    assert np.isin(t64, [sd.RAY_OK, sd.RAY_MISS]).all() and (t64 == sd.RAY_OK).mean() > 0.9
    assert rel_err(g32, g64) <= MIXED_TOL
    assert s32.fp64_fallbacks > 0


# --------------------------------------------------------------------------
# batched-cutouts recipe: a halo at the origin (r^-2 core) in [-1, 1]^3
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def halo(sd):
    from sdtfe_b200 import workloads

    pos4 = workloads.halo_cutout(200_000, 3007)
    m = sd.Mesh(pos4, sd.triangulate(pos4), 1.0)
    yield m
    m.close()


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_halo_cutout_mixed_against_fp64(halo, sd, axis):
    """A 200k-particle halo cutout (the batch configuration's recipe): tets
    from ~1e-5 in the core to ~0.1 in the background, crossings near z = 0
    where a large tet meets a small one.  Mixed against FP64 over the whole
    cutout: the same crossings and statuses, map error <= 1e-5."""
    kw = dict(grid_dim=256, box_len=2.0, box_len_z=2.0, center=(0.0, 0.0, 0.0), n_samples=8,
              seed=SEED, axis=axis)
    g64, s64 = halo.map(sd.map_params(**kw))
    g32, s32 = halo.map(sd.map_params(**kw, precision=sd.DTFE_MIXED))
    assert s32.visits == s64.visits and list(s32.status) == list(s64.status)
    assert rel_err(g32, g64) <= MIXED_TOL
    # and a 128^2 window on the core at 1/4096 of the box per pixel
    kw.update(grid_dim=128, box_len=2.0 / 32)
    g64, s64 = halo.map(sd.map_params(**kw))
    g32, s32 = halo.map(sd.map_params(**kw, precision=sd.DTFE_MIXED))
    assert s32.visits == s64.visits
    assert rel_err(g32, g64) <= MIXED_TOL
