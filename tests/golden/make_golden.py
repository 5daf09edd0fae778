"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's C code compiled from its sources (oracle/_ref, built by
`make -C oracle ref`) on small seeded meshes and stores its outputs:

  * densities (pre_compute_vol), gradients (gradients), forward-hull bitmap
    and hull triangles (find_forward_hull, copy_fh_triangles);
  * an explicit-offset surface map and its per-ray integrals and crossing
    counts (pt_loc_2d + shoot_3d_ray through oracle/ref_harness.c);
  * traced rays with their visited-tet sequences (the visit hook);
  * a 3-D grid (pt_loc_2d + evaluate_3d_ray_on_grid);
  * the host-prep utilities on a fixed input (convert_to_qhdata, rotate3d,
    shuffle_buff after srand(12345)).

The Delaunay cells come from SciPy's Qhull with the reference's options and
are stored in the fixture, so the tests never re-triangulate.

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference, delaunay_tetra, to_pos4  # noqa: E402

SEED = 20240611


def mesh_sets():
    rng = np.random.default_rng(7)
    sets = {}
    # uniform float64 points
    sets["uniform"] = to_pos4(rng.random((700, 3)))
    # clustered float32 points (r^-2 cluster + background), as the benchmark's
    c = rng.normal(size=(500, 3))
    c = 0.5 + (0.15 * rng.random(500))[:, None] * c / np.linalg.norm(c, axis=1)[:, None]
    p = np.concatenate([c, rng.random((300, 3))]).astype(np.float32).astype(np.float64)
    sets["clustered"] = to_pos4(p)
    # a slightly jittered lattice: many rays pass within ZERO of edges -> perturbations
    g = np.linspace(0.0, 1.0, 7)
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    lat = lat + rng.normal(scale=1e-3, size=lat.shape)
    sets["lattice"] = to_pos4(lat)
    return sets


def trace_points(pos4, tetra, rng, n_random=24):
    """Random rays plus rays aimed exactly at vertex (x, y) positions and
    edge midpoints, which force the degenerate branches."""
    xs = list(rng.random(n_random))
    ys = list(rng.random(n_random))
    for v in rng.choice(len(pos4), 12, replace=False):
        xs.append(pos4[v, 0])
        ys.append(pos4[v, 1])
    for t in rng.choice(len(tetra), 12, replace=False):
        a, b = tetra[t, 0], tetra[t, 1]
        xs.append(0.5 * (pos4[a, 0] + pos4[b, 0]))
        ys.append(0.5 * (pos4[a, 1] + pos4[b, 1]))
    return np.array(xs), np.array(ys)


def main():
    R = Reference()
    out = {}
    for name, pos4 in mesh_sets().items():
        tetra = delaunay_tetra(pos4)
        prep = R.prepare(pos4, tetra, 1.0)
        G, S = 24, 4
        box, cen = 1.0, (0.5, 0.5, 0.5)
        m, rr, rc = R.map(prep, G, box, box, cen, S, 0.0, SEED, per_ray=True)
        # a second map: sub-box, slab narrower than the cloud, MC box wider than a pixel
        m2 = R.map(prep, 20, 0.6, 0.5, (0.45, 0.55, 0.5), 3, 0.05, SEED + 1)
        rng = np.random.default_rng(3)
        xs, ys = trace_points(pos4, tetra, rng)
        tr_rho, tr_crossed, visits = R.trace(prep, xs, ys, 0.0, 1.0, 1.0 / G, SEED,
                                             record_visits=True)
        vlen = np.array([len(v) for v in visits], np.int32)
        vflat = np.concatenate(visits).astype(np.int32) if vlen.sum() else np.zeros(0, np.int32)
        grid = R.grid(prep, 8, 1.0, cen, 2, SEED)
        out.update({
            f"{name}/pos4": pos4, f"{name}/tetra": tetra,
            f"{name}/density": prep["pos"][:, 3], f"{name}/grad": prep["grad"],
            f"{name}/bitmap": prep["bitmap"], f"{name}/tri": prep["tri"][:, :7],
            f"{name}/map": m, f"{name}/ray_rho": rr, f"{name}/ray_crossed": rc,
            f"{name}/map2": m2,
            f"{name}/trace_x": xs, f"{name}/trace_y": ys, f"{name}/trace_rho": tr_rho,
            f"{name}/trace_crossed": tr_crossed, f"{name}/visit_len": vlen,
            f"{name}/visits": vflat, f"{name}/grid": grid,
        })
        print(f"{name}: n={len(pos4)} nt={len(tetra)} hull={len(prep['tri'])} "
              f"map mean={m.mean():.4g} crossed mean={rc.mean():.1f} "
              f"failed={(rc == 0).sum()} trace failed={(tr_crossed == 0).sum()}")
    # host-prep utilities
    rng = np.random.default_rng(11)
    soa = rng.random((3, 50)).astype(np.float32)
    S = R.stock
    q = S.convert_to_qhdata(np.ascontiguousarray(soa), 50)
    qd = np.ctypeslib.as_array(ctypes.cast(q, ctypes.POINTER(ctypes.c_double)), shape=(200,)).copy()
    R.libc.free(ctypes.c_void_p(q))
    qd = qd.reshape(50, 4)
    qd[:, 3] = 0.0  # the reference leaves column 3 uninitialised
    rot = qd.copy()
    S.rotate3d(rot, 50, np.array([0.3, 1.1, -2.0]), np.array([0.5, 0.4, 0.6]))
    libc = ctypes.CDLL(None)
    libc.srand(12345)
    shuf = qd.copy()
    S.shuffle_buff.argtypes = [np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                               ctypes.c_int, ctypes.c_int]
    S.shuffle_buff(shuf, 50, 20)
    out.update({"prep/soa": soa, "prep/qhdata": qd, "prep/rotated": rot, "prep/shuffled": shuf})
    np.savez_compressed(os.path.join(HERE, "reference_small.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_small.npz"))


if __name__ == "__main__":
    main()
