"""CPU-side checks of the C-ABI library: it loads, exports every function the
headers in include/ declare, and its host-side routines (input preparation,
face bitmap, the layout step of triangulate) match the reference bit for bit.
Nothing here launches a kernel."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_set


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        if os.path.basename(h) == "sdtfe_rng.h":  # header-only inline functions
            continue
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        src = re.sub(r"#[^\n]*", "", src)
        src = src.replace('extern "C" {', "").replace("}", "")
        for stmt in src.split(";"):
            stmt = " ".join(stmt.split())
            if not stmt or stmt.startswith("typedef") or "{" in stmt:
                continue
            m = re.match(r"^(?:extern \"C\" )?[\w\s\*]*?\b(\w+)\s*\(", stmt)
            if m and "static" not in stmt:
                names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_function():
    from sdtfe_b200 import lib

    L = lib()
    names = declared_functions()
    assert "compute_density" in names and "dtfe_mesh_create" in names and len(names) > 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_library_is_native_and_in_tree():
    from sdtfe_b200 import _lib

    assert os.path.dirname(_lib.LIB_PATH) == os.path.join(ROOT, "sdtfe_b200")
    assert os.path.exists(_lib.LIB_PATH)


def test_convert_rotate_shuffle_match_reference(golden):
    from sdtfe_b200 import lib

    L = lib()
    g = golden_set(golden, "prep")
    soa = np.ascontiguousarray(g["soa"])
    q = L.convert_to_qhdata(soa, soa.shape[1])
    arr = np.ctypeslib.as_array(ctypes.cast(q, ctypes.POINTER(ctypes.c_double)), shape=(200,)).copy()
    ctypes.CDLL(None).free(ctypes.c_void_p(q))
    arr = arr.reshape(50, 4)
    assert np.array_equal(arr, g["qhdata"])
    rot = arr.copy()
    L.rotate3d(rot, 50, np.array([0.3, 1.1, -2.0]), np.array([0.5, 0.4, 0.6]))
    assert np.array_equal(rot, g["rotated"])
    libc = ctypes.CDLL(None)
    libc.srand(12345)
    shuf = arr.copy()
    L.shuffle_buff(shuf, 50, 20)
    assert np.array_equal(shuf, g["shuffled"])


def test_bitmap_layout():
    from sdtfe_b200 import lib

    L = lib()
    L.set_bit.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.get_bit.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.clear_bit.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.delete_bitmap.argtypes = [ctypes.c_void_p]
    n_tet = 10
    bm = L.create_bitmap(n_tet * 4)
    words = np.ctypeslib.as_array(ctypes.cast(bm, ctypes.POINTER(ctypes.c_uint32)), shape=(n_tet + 1,))
    assert not words.any()
    L.set_bit(bm, 4 * 7 + 2)  # face 2 of tet 7
    L.set_bit(bm, 4 * 3 + 0)
    assert words[7] == 1 << 2 and words[3] == 1
    assert L.get_bit(bm, 30) == 1 and L.get_bit(bm, 31) == 0
    L.clear_bit(bm, 30)
    assert words[7] == 0
    L.delete_bitmap(bm)


def test_tetra_layout_matches_numpy_restatement():
    from scipy.spatial import Delaunay

    from oracle.oracle import qhull_to_tetra, to_pos4
    from sdtfe_b200 import tetra_from_cells

    rng = np.random.default_rng(5)
    pos4 = to_pos4(rng.random((2000, 3)))
    d = Delaunay(pos4[:, :3], qhull_options="Qt Qbb Qz")
    a = tetra_from_cells(pos4, d.simplices, d.neighbors)
    b = qhull_to_tetra(pos4, d.simplices, d.neighbors)
    assert np.array_equal(a, b)
    # every tet ends with (AB x AC) . AD <= 0 (src/triangulate.c:92-100)
    p = pos4[:, :3]
    A, B, C, D = (p[a[:, k]] for k in range(4))
    assert (np.einsum("ij,ij->i", np.cross(B - A, C - A), D - A) <= 0).all()


def test_triangulate_without_backend_returns_null(capfd):
    from sdtfe_b200 import lib

    L = lib()
    L.triangulate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                              ctypes.c_char_p]
    L.triangulate.restype = ctypes.c_void_p
    L.dtfe_set_triangulator(None, None)
    pos = np.zeros((8, 4))
    nf = ctypes.c_size_t(7)
    assert L.triangulate(pos.ctypes.data, 8, ctypes.byref(nf), b"qhull d Qz Qt Qbb") is None
    assert nf.value == 0
    assert "TRIANGULATION ERROR" in capfd.readouterr().err


def test_triangulate_with_registered_backend():
    """triangulate() calls the registered host Qhull and lays out its cells."""
    from scipy.spatial import Delaunay

    from oracle.oracle import qhull_to_tetra, to_pos4
    from sdtfe_b200 import lib

    L = lib()
    libc = ctypes.CDLL(None)
    libc.malloc.restype = ctypes.c_void_p
    libc.malloc.argtypes = [ctypes.c_size_t]
    L.triangulate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                              ctypes.c_char_p]
    L.triangulate.restype = ctypes.c_void_p
    FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                          ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p)
    seen = {}

    def backend(xyz4, n, options, simp, nbr, nt, user):
        pts = np.ctypeslib.as_array(ctypes.cast(xyz4, ctypes.POINTER(ctypes.c_double)),
                                    shape=(n, 4))[:, :3].copy()
        seen["options"] = options
        d = Delaunay(pts, qhull_options="Qt Qbb Qz")
        for arr, out in ((d.simplices, simp), (d.neighbors, nbr)):
            a = np.ascontiguousarray(arr, np.int32)
            p = libc.malloc(a.nbytes)
            ctypes.memmove(p, a.ctypes.data, a.nbytes)
            out[0] = p
        nt[0] = len(d.simplices)
        return 0

    cb = FN(backend)
    L.dtfe_set_triangulator.argtypes = [FN, ctypes.c_void_p]
    L.dtfe_set_triangulator(cb, None)
    try:
        rng = np.random.default_rng(8)
        pos4 = to_pos4(rng.random((300, 3)))
        nf = ctypes.c_size_t(0)
        ptr = L.triangulate(pos4.ctypes.data, 300, ctypes.byref(nf), b"qhull d Qz Qt Qbb")
        assert ptr and nf.value > 0
        got = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_int)),
                                    shape=(nf.value, 8)).copy()
        libc.free.argtypes = [ctypes.c_void_p]
        libc.free(ptr)
        d = Delaunay(pos4[:, :3], qhull_options="Qt Qbb Qz")
        assert np.array_equal(got, qhull_to_tetra(pos4, d.simplices, d.neighbors))
        assert seen["options"] == b"qhull d Qz Qt Qbb"
    finally:
        L.dtfe_set_triangulator.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.dtfe_set_triangulator(None, None)


def test_mesh_create_reports_cuda_failure_without_gpu():
    """On a machine without a usable GPU the handle API returns an error status
    (and never runs anything on the CPU instead)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from oracle.oracle import to_pos4
    from sdtfe_b200 import DTFEError, Mesh

    pos4 = to_pos4(np.random.default_rng(0).random((10, 3)))
    with pytest.raises(DTFEError):
        Mesh(pos4, np.zeros((1, 8), np.int32))


def test_triangulate_cache_answers_repeated_inputs_without_the_backend():
    """triangulate() keeps its results keyed by the exact input: a repeated
    input gets the same rows without a backend call; one changed coordinate
    or other options run the backend again; column 3 plays no part; a zero
    limit disables the cache."""
    from scipy.spatial import Delaunay

    from oracle.oracle import to_pos4
    from sdtfe_b200 import lib

    L = lib()
    libc = ctypes.CDLL(None)
    libc.malloc.restype = ctypes.c_void_p
    libc.malloc.argtypes = [ctypes.c_size_t]
    libc.free.argtypes = [ctypes.c_void_p]
    L.triangulate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                              ctypes.c_char_p]
    L.triangulate.restype = ctypes.c_void_p
    FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                          ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p)
    calls = [0]

    def backend(xyz4, n, options, simp, nbr, nt, user):
        calls[0] += 1
        pts = np.ctypeslib.as_array(ctypes.cast(xyz4, ctypes.POINTER(ctypes.c_double)),
                                    shape=(n, 4))[:, :3].copy()
        d = Delaunay(pts, qhull_options="Qt Qbb Qz")
        for arr, out in ((d.simplices, simp), (d.neighbors, nbr)):
            a = np.ascontiguousarray(arr, np.int32)
            p = libc.malloc(a.nbytes)
            ctypes.memmove(p, a.ctypes.data, a.nbytes)
            out[0] = p
        nt[0] = len(d.simplices)
        return 0

    def tri(pos4, options=b"qhull d Qz Qt Qbb"):
        nf = ctypes.c_size_t(0)
        ptr = L.triangulate(pos4.ctypes.data, len(pos4), ctypes.byref(nf), options)
        assert ptr and nf.value > 0
        rows = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_int)),
                                     shape=(nf.value, 8)).copy()
        libc.free(ptr)
        return rows

    def stats():
        h, m = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        e, b = ctypes.c_size_t(), ctypes.c_size_t()
        L.dtfe_triangulation_cache_stats(ctypes.byref(h), ctypes.byref(m), ctypes.byref(e),
                                         ctypes.byref(b))
        return h.value, m.value, e.value, b.value

    cb = FN(backend)
    L.dtfe_set_triangulator.argtypes = [FN, ctypes.c_void_p]
    L.dtfe_set_triangulator(cb, None)
    try:
        L.dtfe_set_triangulation_cache(0)  # start empty
        L.dtfe_set_triangulation_cache(64 << 20)
        h0, m0, _, _ = stats()
        pos4 = to_pos4(np.random.default_rng(9).random((400, 3)))
        first = tri(pos4)
        assert calls[0] == 1
        again = pos4.copy()
        again[:, 3] = 7.5  # column 3 is not part of the key
        assert np.array_equal(tri(again), first) and calls[0] == 1
        h, m, entries, nbytes = stats()
        assert (h - h0, m - m0, entries) == (1, 1, 1)
        assert nbytes == 400 * 3 * 8 + first.size * 4
        moved = pos4.copy()
        moved[17, 1] = np.nextafter(moved[17, 1], 2.0)
        tri(moved)
        assert calls[0] == 2
        tri(pos4, b"qhull d Qz Qt Qbb Pp")
        assert calls[0] == 3
        assert np.array_equal(tri(pos4), first) and calls[0] == 3
        L.dtfe_set_triangulation_cache(0)
        assert stats()[2] == 0
        assert np.array_equal(tri(pos4), first) and calls[0] == 4
    finally:
        L.dtfe_set_triangulation_cache(1024 << 20)
        L.dtfe_set_triangulator.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.dtfe_set_triangulator(None, None)


def test_write_rho_and_write_image(tmp_path):
    """The example driver's writers (src/io.c): write_rho writes the doubles
    raw; write_image writes a baseline palette TIFF of log(rho + 1) scaled to
    0..128 between the smallest positive and the largest value, and nothing
    for negative or NaN maps."""
    import struct

    from sdtfe_b200 import lib

    L = lib()
    L.write_rho.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
    L.write_rho.restype = ctypes.c_int
    L.write_image.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int]
    L.write_image.restype = None
    G = 5
    rho = np.zeros(G * G)
    rho[3:] = np.geomspace(0.5, 900.0, G * G - 3)
    rho[7] = 0.0
    p = ctypes.c_void_p(rho.ctypes.data)
    fn = str(tmp_path / "m.rho.bin").encode()
    assert L.write_rho(fn, ctypes.byref(p), G * G) == G * G
    assert np.array_equal(np.fromfile(fn.decode(), np.float64), rho)

    img = str(tmp_path / "m.rho.tiff").encode()
    L.write_image(img, rho.ctypes.data, G)
    b = open(img.decode(), "rb").read()
    assert b[:4] == b"II*\x00"
    ifd = struct.unpack_from("<I", b, 4)[0]
    n = struct.unpack_from("<H", b, ifd)[0]
    tags = {}
    for k in range(n):
        tag, typ, cnt, val = struct.unpack_from("<HHII", b, ifd + 2 + 12 * k)
        tags[tag] = (typ, cnt, val if typ == 4 or cnt > 1 else val & 0xFFFF)
    assert tags[256][2] == G and tags[257][2] == G and tags[258][2] == 8
    assert tags[259][2] == 1 and tags[262][2] == 3 and tags[277][2] == 1
    off, count = tags[273][2], tags[279][2]
    assert count == G * G
    pix = np.frombuffer(b, np.uint8, count, off)
    pos = rho > 0
    lo, hi = np.log(rho[pos].min() + 1.0), np.log(rho.max() + 1.0)
    want = np.zeros(G * G, np.uint8)
    want[pos] = (128.0 * (np.log(rho[pos] + 1.0) - lo) / (hi - lo)).astype(np.uint8)
    assert np.array_equal(pix, want)
    cmap = np.frombuffer(b, "<u2", 768, tags[320][2])
    x = np.arange(256) / 255.0
    for c, chan in zip((3.0, 2.0, 1.0), cmap.reshape(3, 256)):
        ref = np.floor(np.clip(1.5 - np.abs(4 * x - c), 0, 1) * 65535 + 0.5)
        assert np.array_equal(chan, ref.astype(np.uint16))

    for bad in (-1.0, np.nan):
        r2 = rho.copy()
        r2[4] = bad
        f2 = str(tmp_path / "bad.tiff").encode()
        L.write_image(f2, r2.ctypes.data, G)
        assert not (tmp_path / "bad.tiff").exists()


def write_positions(path, n, seed=3):
    """n float32 positions in the example driver's layout (x[n], y[n], z[n]),
    a Gaussian blob about the unit box's centre."""
    p = np.random.default_rng(seed).normal(0.5, 0.08, (n, 3)).astype(np.float32)
    np.ascontiguousarray(p.T).tofile(path)


def run_cli(tmp_path, n=3000, G=32, seed="7"):
    import os
    import subprocess

    write_positions(tmp_path / "pts.bin", n)
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sdtfe_b200",
                       "dtfe")
    env = dict(os.environ, SDTFE_SEED=seed)
    return subprocess.run([exe, "pts.bin", str(n), str(G), "0.5", "0.5", "0.5", "1", "1", "1",
                           "0", "4", "1"], cwd=tmp_path, env=env, capture_output=True, text=True,
                          timeout=300)


def test_cli_triangulates_through_the_registered_qhull(tmp_path):
    """The dtfe program reads the reference driver's arguments and file
    layout, and triangulates through the SciPy Qhull it registers (the map
    itself needs the GPU: without one the program stops there with an
    error)."""
    import torch

    r = run_cli(tmp_path)
    assert "Using prng seed: 7" in r.stdout
    assert "Done creating" in r.stdout, r.stdout + r.stderr
    if not torch.cuda.is_available():
        assert r.returncode != 0 and "compute_density failed" in r.stderr
