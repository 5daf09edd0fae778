"""The pydtfe drop-in module: the reference's four functions with their
argument names, defaults, dtypes and errors (python/pydtfe.cpp:205-384).

The GPU tests reproduce each call's host preparation with the reference's own
C (convert_to_qhdata and shuffle_buff from oracle/_ref, driven by the same
srand() seed), triangulate with the same Qhull, and compare the module's
output with the oracle bit for bit."""
import ctypes
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "sdtfe_b200"))


@pytest.fixture(scope="module")
def pydtfe():
    import pydtfe as m  # the drop-in name, as the reference's users import it

    return m


def test_entry_points_bound_to_this_library(reference):
    """With the reference's libdtfe loaded globally first (the `reference`
    fixture does that), importing pydtfe must still bind the B200 library:
    checked in a subprocess that loads the reference before the module."""
    import subprocess

    code = ("import sys, numpy as np; sys.path[:0] = [%r, %r]\n"
            "from oracle.oracle import Reference; Reference()\n"
            "import pydtfe\n"
            "try:\n"
            "    pydtfe.compute_particle_density(np.random.rand(50, 3).astype(np.float32), 1.0)\n"
            "except RuntimeError as e:\n"
            "    print('gpu-error', e)\n"
            "print('launches', pydtfe.kernel_launches())\n") % (ROOT, os.path.join(ROOT, "sdtfe_b200"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    # without a GPU the library reports a CUDA error; with one it launches
    # kernels; the reference's CPU code would do neither
    assert "gpu-error" in out.stdout or "launches 0" not in out.stdout


def test_signatures_and_defaults(pydtfe):
    doc = pydtfe.compute_surface_density.__doc__
    for name in ("particle_pos", "center", "grid_dim", "sample_factor", "box_width", "box_depth",
                 "particle_mass", "mc_box_width", "mc_sample_count", "rotation_angle"):
        assert name in doc
    assert "supersampling" in pydtfe.compute_3d_density.__doc__
    assert "particle_value" in pydtfe.interpolate_field2grid.__doc__
    assert "particle_mass" in pydtfe.compute_particle_density.__doc__


def test_errors_match_the_reference(pydtfe):
    pos = np.random.default_rng(0).random((10, 3)).astype(np.float32)
    with pytest.raises(ValueError, match="incorrect shape"):
        pydtfe.compute_surface_density(pos[:, :2], [0, 0, 0], 8, 1.0, 1, 1, 1, 0, 1)
    with pytest.raises(ValueError, match="not enough particles"):
        pydtfe.compute_surface_density(pos[:4], [0, 0, 0], 8, 1.0, 1, 1, 1, 0, 1)
    with pytest.raises(ValueError, match="not enough particles"):
        pydtfe.compute_3d_density(pos, [0, 0, 0], 8, 0.3, 1, 1)
    with pytest.raises(ValueError, match="sample_factor"):
        pydtfe.interpolate_field2grid(pos, np.ones(10, np.float32), [0, 0, 0], 8, 0.5, 1)
    with pytest.raises(ValueError, match="different length"):
        pydtfe.interpolate_field2grid(pos, np.ones(9, np.float32), [0, 0, 0], 8, 1.0, 1)
    with pytest.raises(ValueError):
        pydtfe.set_precision("fp16")


def test_triangulate_backend_registered(pydtfe):
    """Importing the module registers SciPy's Qhull behind the C triangulate()."""
    from oracle.oracle import delaunay_tetra, to_pos4
    from sdtfe_b200 import lib

    L = lib()
    L.triangulate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                              ctypes.c_char_p]
    L.triangulate.restype = ctypes.c_void_p
    pos4 = to_pos4(np.random.default_rng(2).random((400, 3)))
    nt = ctypes.c_size_t(0)
    p = L.triangulate(pos4.ctypes.data, len(pos4), ctypes.byref(nt), b"qhull d Qz Qt Qbb")
    assert p
    got = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_int)),
                                shape=(nt.value, 8)).copy()
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    libc.free(p)
    assert np.array_equal(got, delaunay_tetra(pos4))


# --------------------------------------------------------------------------
# GPU: the module's results against the oracle on identically prepared input
# --------------------------------------------------------------------------
def _reference_prep(reference, pos, sample_factor, seed):
    """convert_to_qhdata + shuffle_buff exactly as the reference binding does."""
    libc = ctypes.CDLL(None)
    S = reference.stock
    soa = np.ascontiguousarray(pos.T.astype(np.float32))
    q = S.convert_to_qhdata(soa, len(pos))
    data = np.ctypeslib.as_array(ctypes.cast(q, ctypes.POINTER(ctypes.c_double)),
                                 shape=(len(pos), 4)).copy()
    reference.libc.free(ctypes.c_void_p(q))
    data[:, 3] = 0.0
    n_shuffle = int(np.float32(len(pos)) * np.float32(sample_factor))
    S.shuffle_buff.argtypes = [np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                               ctypes.c_int, ctypes.c_int]
    libc.srand(seed)
    S.shuffle_buff(data, len(pos), n_shuffle)
    return np.ascontiguousarray(data[:n_shuffle]), n_shuffle


@pytest.mark.gpu
@pytest.mark.parametrize("sample_factor", [1.0, 0.5])
def test_surface_density_bit_exact(pydtfe, reference, oracle, sample_factor):
    from oracle.oracle import delaunay_tetra

    pos = np.random.default_rng(3).random((3000, 3)).astype(np.float32)
    data, _ = _reference_prep(reference, pos, sample_factor, 4242)
    tetra = delaunay_tetra(data)
    prep = oracle.prepare(data, tetra, np.float32(2.0 / sample_factor))
    want = oracle.map(prep, 40, 1.0, 1.0, (0.5, 0.5, 0.5), 4, 0.0, 99)
    libc = ctypes.CDLL(None)
    libc.srand(4242)
    pydtfe.set_seed(99)
    launches = pydtfe.kernel_launches()
    try:
        got = pydtfe.compute_surface_density(pos, [0.5, 0.5, 0.5], 40, sample_factor, 1.0, 1.0,
                                             2.0, 0.0, 4)
    finally:
        pydtfe.set_seed(0)
    assert pydtfe.kernel_launches() > launches  # the GPU library did the work
    assert got.dtype == np.float64 and got.shape == (40, 40)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_particle_density_and_grids(pydtfe, reference, oracle):
    from oracle.oracle import delaunay_tetra, to_pos4

    pos = np.random.default_rng(5).random((2000, 3)).astype(np.float32)
    pos4 = to_pos4(pos.astype(np.float64))
    tetra = delaunay_tetra(pos4)
    prep = oracle.prepare(pos4, tetra, 1.5)
    launches = pydtfe.kernel_launches()
    rho = pydtfe.compute_particle_density(pos, 1.5)
    assert pydtfe.kernel_launches() > launches
    assert rho.dtype == np.float32 and np.array_equal(rho, prep["pos"][:, 3].astype(np.float32))
    # the 3-D grid (sample_factor 1: the reference shuffles with rand())
    data, _ = _reference_prep(reference, pos, 1.0, 17)
    t2 = delaunay_tetra(data)
    p2 = oracle.prepare(data, t2, 1.5)
    pydtfe.set_seed(5)
    try:
        libc = ctypes.CDLL(None)
        libc.srand(17)
        g = pydtfe.compute_3d_density(pos, [0.5, 0.5, 0.5], 10, 1.0, 1.0, 1.5, 2)
    finally:
        pydtfe.set_seed(0)
    want, _ = oracle.grid(p2, 10, 1.0, (0.5, 0.5, 0.5), 2, 5)
    assert g.shape == (10, 10, 10) and np.array_equal(g, want)
    # interpolate_field2grid: no shuffle, the field replaces the density column
    val = (pos[:, 0] * 3 + pos[:, 1]).astype(np.float32)
    f4 = pos4.copy()
    f4[:, 3] = val
    pf = dict(prep)
    pf["pos"] = f4
    pf["grad"] = oracle.gradients(tetra, f4)
    pydtfe.set_seed(6)
    try:
        gi = pydtfe.interpolate_field2grid(pos, val, [0.5, 0.5, 0.5], 8, 1.0, 1.0, 1)
    finally:
        pydtfe.set_seed(0)
    want_i, _ = oracle.grid(pf, 8, 1.0, (0.5, 0.5, 0.5), 1, 6)
    assert np.array_equal(gi, want_i)
