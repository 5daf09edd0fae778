"""Tile-shared point location (locate_region, sdtfe_b200/csrc/walk64.cuh).

The mixed maps walk the projected hull from triangle 0 once per tile, over the
rectangle that holds every sample position of the tile, for as long as each
edge test has one outcome for the whole rectangle; each ray then resumes its
own walk from there (src/dtfe.c:518-552).  Here the function is compiled for
the host and checked against the oracle's walk from triangle 0: every ray of
every tile must end in the same hull triangle with the same status, also
under small step budgets and on lattices whose points are collinear.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

KIND_RESUME, KIND_FOUND, KIND_MISS = 0, 1, 2
ORC_OK, ORC_MISS = 0, 1


def _nvcc():
    for p in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if p and os.path.exists(p):
            return p
    return None


@pytest.fixture(scope="module")
def lr():
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc is not available")
    src = os.path.join(ROOT, "tests", "locate_region_host.cu")
    out_dir = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "liblocate_region_host.so")
    hdr = os.path.join(ROOT, "sdtfe_b200", "csrc", "walk64.cuh")
    if not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(src),
                                                               os.path.getmtime(hdr)):
        subprocess.run([nvcc, "-O2", "-std=c++17", "-shared",
                        "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC,-ffp-contract=off",
                        "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(ROOT, "sdtfe_b200", "csrc"), src, "-o", out],
                       check=True)
    L = ctypes.CDLL(out)
    L.lr_set_triangles.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    L.lr_locate_region.argtypes = [ctypes.c_double] * 4 + [
        ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.lr_locate_region.restype = ctypes.c_int
    return L


def _meshes():
    from oracle.oracle import delaunay_tetra, to_pos4
    from sdtfe_b200 import workloads

    out = [("clustered", workloads.clustered_box(n=20000)[0]),
           ("halo", workloads.halo_cutout(20000, 3))]
    lat = workloads.perturbed_lattice(n_side=16)
    out.append(("jittered lattice", lat[0] if isinstance(lat, tuple) else lat))
    g = np.stack(np.meshgrid(np.arange(10.0), np.arange(10.0), np.arange(5.0), indexing="ij"),
                 -1).reshape(-1, 3) / 9.0
    out.append(("exact lattice", to_pos4(g)))
    return [(name, pos4, delaunay_tetra(pos4)) for name, pos4 in out]


@pytest.fixture(scope="module")
def meshes():
    return _meshes()


def _check_mesh(lr, oracle, pos4, tet, rng, n_tiles, per_tile, budget):
    prep = oracle.prepare(pos4, tet, 1.0)
    tri, pos = prep["tri"], prep["pos"]
    P = pos[:, :2]
    abc = np.ascontiguousarray(np.stack([P[tri[:, 0]], P[tri[:, 1]], P[tri[:, 2]]], 1).reshape(-1, 6))
    nb = np.ascontiguousarray(tri[:, [3, 4, 5, 6]].astype(np.int32))
    lr.lr_set_triangles(abc.ctypes.data, nb.ctypes.data, len(tri))
    # the oracle's walk then reports the final triangle instead of its tet
    tri_id = tri.astype(np.int32).copy()
    tri_id[:, 6] = np.arange(len(tri))
    tri_id = np.ascontiguousarray(tri_id)
    locate = oracle.lib.orc_locate
    st = ctypes.c_int()
    lo, hi = P.min(0), P.max(0)
    kinds = [0, 0, 0]
    bad = []
    for it in range(n_tiles):
        # a map as the library lays it out (src/dtfe.c:590-612): pixel size,
        # offsets, sample scale and shift, and one tile of TW x TH pixels
        G = int(rng.choice([16, 64, 256, 1024]))
        box = float((hi - lo).max() * rng.choice([0.5, 1.0, 1.3]))
        cx, cy = (float(v) for v in lo + (hi - lo) * rng.random(2))
        dxy = box / G
        delta = float(rng.choice([0.0, 3 * dxy]))
        scale = delta if delta > dxy else dxy
        soff = (delta - dxy) / 2.0 if delta > dxy else 0.0
        offx, offy = -(box / 2.0) + cx, -(box / 2.0) + cy
        TW, TH = (int(v) for v in rng.choice([1, 2, 4, 8], 2))
        tx0 = int(rng.integers(0, G)) // TW * TW
        ty0 = int(rng.integers(0, G)) // TH * TH
        c1, r1 = min(tx0 + TW, G) - 1, min(ty0 + TH, G) - 1
        # the rectangle exactly as tile_rect (walk32.cu) forms it
        xlo = tx0 * dxy + offx - soff
        xhi = (c1 * dxy + offx - soff) + scale
        ylo = ty0 * dxy + offy - soff
        yhi = (r1 * dxy + offy - soff) + scale
        start, steps = ctypes.c_int(), ctypes.c_int()
        kind = lr.lr_locate_region(xlo, xhi, ylo, yhi, budget, ctypes.byref(start),
                                   ctypes.byref(steps))
        kinds[kind] += 1
        for j in range(per_tile):
            col = int(rng.integers(tx0, c1 + 1))
            row = int(rng.integers(ty0, r1 + 1))
            u = (0.0, 1.0 - 2.0 ** -53)[j] if j < 2 else float(rng.random())
            v = float(rng.random()) if j >= 2 else u
            x = col * dxy + offx - soff
            y = row * dxy + offy - soff
            xt, yt = x + u * scale, y + v * scale
            want = (locate(tri_id, pos, 0, xt, yt, budget, ctypes.byref(st)), st.value)
            if kind == KIND_FOUND:
                got = (start.value, ORC_OK)
            elif kind == KIND_MISS:
                got = (-1, ORC_MISS)
            else:
                got = (locate(tri_id, pos, start.value, xt, yt, budget - steps.value,
                              ctypes.byref(st)), st.value)
            if got != want:
                bad.append((it, kind, start.value, steps.value, got, want))
    return kinds, bad


def test_tile_location_equals_the_walk_from_triangle_0(lr, oracle, meshes):
    rng = np.random.default_rng(7)
    for name, pos4, tet in meshes:
        kinds, bad = _check_mesh(lr, oracle, pos4, tet, rng, n_tiles=120, per_tile=12,
                                 budget=1 << 24)
        assert not bad, (name, bad[:3])
        assert kinds[KIND_RESUME] and kinds[KIND_FOUND], (name, kinds)


def test_tile_location_keeps_the_step_budget(lr, oracle, meshes):
    rng = np.random.default_rng(8)
    name, pos4, tet = meshes[0]
    for budget in (1, 2, 5, 9):
        kinds, bad = _check_mesh(lr, oracle, pos4, tet, rng, n_tiles=40, per_tile=8,
                                 budget=budget)
        assert not bad, (name, budget, bad[:3])


def test_tile_location_on_vertices_and_edges(lr, oracle, meshes):
    """Rectangles with corners exactly on lattice vertices (queries on edge
    lines, where s_q is exactly zero), zero-width rectangles, and queries at
    the corners and on the sides."""
    name, pos4, tet = meshes[3]  # the exact lattice
    prep = oracle.prepare(pos4, tet, 1.0)
    tri, pos = prep["tri"], prep["pos"]
    P = pos[:, :2]
    abc = np.ascontiguousarray(np.stack([P[tri[:, 0]], P[tri[:, 1]], P[tri[:, 2]]], 1).reshape(-1, 6))
    nb = np.ascontiguousarray(tri[:, [3, 4, 5, 6]].astype(np.int32))
    lr.lr_set_triangles(abc.ctypes.data, nb.ctypes.data, len(tri))
    tri_id = tri.astype(np.int32).copy()
    tri_id[:, 6] = np.arange(len(tri))
    tri_id = np.ascontiguousarray(tri_id)
    locate = oracle.lib.orc_locate
    st = ctypes.c_int()
    xs = np.unique(P[:, 0])
    ys = np.unique(P[:, 1])
    rng = np.random.default_rng(9)
    budget = 1 << 24
    bad = []
    n = 0
    for _ in range(300):
        i0, i1 = sorted(rng.integers(0, len(xs), 2))
        j0, j1 = sorted(rng.integers(0, len(ys), 2))
        if rng.random() < 0.3:
            i1 = i0  # zero width
        xlo, xhi, ylo, yhi = float(xs[i0]), float(xs[i1]), float(ys[j0]), float(ys[j1])
        start, steps = ctypes.c_int(), ctypes.c_int()
        kind = lr.lr_locate_region(xlo, xhi, ylo, yhi, budget, ctypes.byref(start),
                                   ctypes.byref(steps))
        for qx in (xlo, 0.5 * (xlo + xhi), xhi):
            for qy in (ylo, 0.5 * (ylo + yhi), yhi):
                want = (locate(tri_id, pos, 0, qx, qy, budget, ctypes.byref(st)), st.value)
                if kind == KIND_FOUND:
                    got = (start.value, ORC_OK)
                elif kind == KIND_MISS:
                    got = (-1, ORC_MISS)
                else:
                    got = (locate(tri_id, pos, start.value, qx, qy, budget - steps.value,
                                  ctypes.byref(st)), st.value)
                n += 1
                if got != want:
                    bad.append((xlo, xhi, ylo, yhi, qx, qy, kind, got, want))
    assert n > 2000 and not bad, bad[:3]
