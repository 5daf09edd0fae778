"""ctypes front end of the parity checkers (test infrastructure only).

Two checkers, both CPU:

* ``Oracle`` wraps ``oracle/liboracle.so``, the C restatement of the reference
  algorithm (``oracle/dtfe_oracle.c``).
* ``Reference`` wraps the reference's own C compiled from its sources into
  ``oracle/_ref/`` by ``oracle/Makefile``: the stock build (``libdtfe_ref.so``,
  timed as the CPU baseline) and the explicit-offset harness build
  (``libdtfe_refh.so`` + the visit hook ``libdtfe_refhook.so``).

``qhull_to_tetra`` restates, in numpy, how the reference's ``triangulate``
(src/triangulate.c:63-175) lays out Qhull's Delaunay cells; the library has its
own C version of the same step that the tests compare against this one.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_u64 = ctypes.c_uint64

RAY_OK, RAY_MISS, RAY_NO_EXIT, RAY_PERTURB_MAX, RAY_BUDGET, RAY_LOC_BUDGET = range(6)
DEFAULT_MAX_VISITS = 1 << 26


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


# --------------------------------------------------------------------------
# triangulation boundary (host, Qhull)
# --------------------------------------------------------------------------
def qhull_to_tetra(pos4: np.ndarray, simplices: np.ndarray, neighbors: np.ndarray) -> np.ndarray:
    """Reference ``tetra_data`` rows from Qhull's cells.

    Neighbour k of a Qhull cell lies across the facet opposite vertex k, which
    is the reference's slot ``4+k`` (BDC, ACD, ADB, ABC).  Cells with
    (AB x AC) . AD > 0 get B and C swapped (src/triangulate.c:72-100), and with
    them the neighbours opposite B and C.  The orientation test repeats the
    reference's arithmetic order so that its decision is the same.
    """
    s = np.ascontiguousarray(simplices, dtype=np.int32)
    nb = np.ascontiguousarray(neighbors, dtype=np.int32)
    p = pos4[:, :3]
    a, b, c, d = (p[s[:, k]] for k in range(4))
    ab, ac, ad = b - a, c - a, d - a
    n0 = ab[:, 1] * ac[:, 2] - ab[:, 2] * ac[:, 1]
    n1 = ab[:, 2] * ac[:, 0] - ab[:, 0] * ac[:, 2]
    n2 = ab[:, 0] * ac[:, 1] - ab[:, 1] * ac[:, 0]
    temp = ((0.0 + n0 * ad[:, 0]) + n1 * ad[:, 1]) + n2 * ad[:, 2]
    flip = temp > 0
    out = np.empty((len(s), 8), dtype=np.int32)
    out[:, :4] = s
    out[:, 4:] = nb
    out[flip, 1], out[flip, 2] = s[flip, 2], s[flip, 1]
    out[flip, 5], out[flip, 6] = nb[flip, 2], nb[flip, 1]
    return out


def delaunay_tetra(pos4: np.ndarray) -> np.ndarray:
    """Delaunay tetrahedra of pos4[:, :3] with the reference's Qhull options."""
    from scipy.spatial import Delaunay

    tri = Delaunay(np.ascontiguousarray(pos4[:, :3]), qhull_options="Qt Qbb Qz")
    return qhull_to_tetra(pos4, tri.simplices, tri.neighbors)


def to_pos4(points: np.ndarray) -> np.ndarray:
    """(N, 3) positions -> the reference's (N, 4) float64 rows (src/utils.c:8-16)."""
    pos4 = np.zeros((len(points), 4), dtype=np.float64)
    pos4[:, :3] = points
    return pos4


# --------------------------------------------------------------------------
# the C restatement
# --------------------------------------------------------------------------
class Oracle:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = ctypes.CDLL(path)
        L.orc_density.argtypes = [_f64, _i, _i32, _i, ctypes.c_float, _vp]
        L.orc_gradients.argtypes = [_i32, _i, _f64, _f64]
        L.orc_forward_faces.argtypes = [_i32, _i, _f64, _u8]
        L.orc_forward_faces.restype = _i
        L.orc_hull_triangles.argtypes = [_i32, _i, _u8, _i32]
        L.orc_hull_triangles.restype = _i
        L.orc_locate.argtypes = [_i32, _f64, _i, _d, _d, _i, ctypes.POINTER(_i)]
        L.orc_locate.restype = _i
        L.orc_map.argtypes = [_f64, _i32, _f64, _i32, _i, _d, _d, _d, _d, _d, _i, _d, _u64, _i,
                              _f64, _vp, _vp, _vp]
        L.orc_trace.argtypes = [_f64, _i32, _f64, _i32, _i, _f64, _f64, _d, _d, _d, _u64, _i,
                                _f64, _i32, _i32, _vp, _i]
        L.orc_grid.argtypes = [_f64, _i32, _f64, _i32, _i, _d, _f64, _d, _d, _d, ctypes.c_uint,
                               _u64, _i, _vp]

    def density(self, pos4, tetra, p_mass):
        pos = np.array(pos4, dtype=np.float64, order="C", copy=True)
        adj = np.zeros(len(pos), dtype=np.int32)
        self.lib.orc_density(pos, len(pos), tetra, len(tetra), p_mass, _ptr(adj))
        return pos, adj

    def gradients(self, tetra, pos4):
        g = np.empty((len(tetra), 3), dtype=np.float64)
        self.lib.orc_gradients(tetra, len(tetra), pos4, g)
        return g

    def forward_faces(self, tetra, pos4):
        flags = np.zeros(len(tetra) * 4, dtype=np.uint8)
        n = self.lib.orc_forward_faces(tetra, len(tetra), pos4, flags)
        return flags, n

    def hull_triangles(self, tetra, flags):
        n = int(flags.sum())
        tri = np.empty((max(n, 1), 8), dtype=np.int32)
        self.lib.orc_hull_triangles(tetra, len(tetra), flags, tri)
        return tri[:n]

    def prepare(self, pos4, tetra, p_mass):
        """density -> gradients -> forward hull -> hull triangles."""
        pos, adj = self.density(pos4, tetra, p_mass)
        grad = self.gradients(tetra, pos)
        flags, _ = self.forward_faces(tetra, pos)
        tri = self.hull_triangles(tetra, flags)
        return dict(pos=pos, adj=adj, grad=grad, flags=flags, tri=tri, tetra=tetra)

    def map(self, prep, G, box_len, box_len_z, center, S, delta_sample, seed,
            max_visits=DEFAULT_MAX_VISITS, per_ray=False):
        m = np.zeros(G * G, dtype=np.float64)
        n_rays = G * G * S
        rr = np.zeros(n_rays, np.float64) if per_ray else None
        rc = np.zeros(n_rays, np.int32) if per_ray else None
        rs = np.zeros(n_rays, np.int32) if per_ray else None
        tri = prep["tri"] if len(prep["tri"]) else np.zeros((1, 8), np.int32)
        self.lib.orc_map(prep["pos"], prep["tetra"], prep["grad"], tri, G, box_len, box_len_z,
                         *center, S, delta_sample, seed, max_visits, m, _ptr(rr), _ptr(rc), _ptr(rs))
        m = m.reshape(G, G)
        return (m, rr, rc, rs) if per_ray else m

    def trace(self, prep, xs, ys, z0, lz, dxy, seed, max_visits=DEFAULT_MAX_VISITS, max_record=0):
        n = len(xs)
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        rho = np.zeros(n, np.float64)
        crossed = np.zeros(n, np.int32)
        status = np.zeros(n, np.int32)
        visits = np.full((n, max_record), -1, np.int32) if max_record else None
        self.lib.orc_trace(prep["pos"], prep["tetra"], prep["grad"], prep["tri"], n, xs, ys, z0, lz,
                           dxy, seed, max_visits, rho, crossed, status, _ptr(visits), max_record)
        return rho, crossed, status, visits

    def grid(self, prep, G, box_len, center, ss, seed, max_visits=DEFAULT_MAX_VISITS):
        g = np.zeros(G * G * G, np.float64)
        st = np.zeros(G * G, np.int32)
        self.lib.orc_grid(prep["pos"], prep["tetra"], prep["grad"], prep["tri"], G, box_len, g,
                          *center, ss, seed, max_visits, _ptr(st))
        return g.reshape(G, G, G), st


# --------------------------------------------------------------------------
# the reference itself, compiled from its sources into oracle/_ref
# --------------------------------------------------------------------------
class Reference:
    """The reference's C code.  ``stock`` is the unmodified build; ``harness``
    is the explicit-offset build with the visit hook interposed."""

    def __init__(self, stock_only=False):
        libs = ("libdtfe_ref.so",) if stock_only else ("libdtfe_ref.so", "libdtfe_refh.so",
                                                       "libdtfe_refhook.so")
        for f in libs:
            if not os.path.exists(os.path.join(REF_DIR, f)):
                raise FileNotFoundError(f"oracle/_ref/{f} missing: run `make -C oracle ref`")
        self.libc = ctypes.CDLL(None)
        self.libc.free.argtypes = [_vp]
        S = self.stock = ctypes.CDLL(os.path.join(REF_DIR, "libdtfe_ref.so"))
        self._bind(S)
        S.compute_density.argtypes = [_f64, _i, _i32, _i, _i, _d, _d, _f64, ctypes.c_float, _d, _d,
                                      _d, _i, _d]
        # the stock build's OpenMP runtime (libgomp, a dependency of the library)
        S.omp_set_num_threads.argtypes = [_i]
        S.omp_get_max_threads.restype = _i
        if stock_only:
            return
        S.compute_3d_density.argtypes = [_f64, _i, _i32, _i, _i, _d, _f64, ctypes.c_float, _d, _d,
                                         _d, ctypes.c_uint]
        S.interpolate_to_3d_grid.argtypes = [_f64, _i, _i32, _i, _i, _d, _f64, _d, _d, _d,
                                             ctypes.c_uint]
        S.rotate3d.argtypes = [_f64, ctypes.c_size_t, _f64, _f64]
        S.convert_to_qhdata.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                                        ctypes.c_size_t]
        S.convert_to_qhdata.restype = _vp
        # the hook must be global before the harness build is loaded
        self.hook = ctypes.CDLL(os.path.join(REF_DIR, "libdtfe_refhook.so"), mode=ctypes.RTLD_GLOBAL)
        H = self.harness = ctypes.CDLL(os.path.join(REF_DIR, "libdtfe_refh.so"),
                                       mode=ctypes.RTLD_GLOBAL)
        self._bind(H)
        H.refh_map.argtypes = [_f64, _i32, _f64, _i32, _i, _d, _d, _d, _d, _d, _i, _d, _u64, _f64,
                               _vp, _vp]
        self._on_ray = ctypes.CFUNCTYPE(None, _i)
        H.refh_trace.argtypes = [_f64, _i32, _f64, _i32, _i, _f64, _f64, _d, _d, _d, _u64, _f64,
                                 _i32, _vp]
        H.refh_grid.argtypes = [_f64, _i32, _f64, _i32, _i, _d, _f64, _d, _d, _d, ctypes.c_uint,
                                _u64]
        self.hook.refhook_begin.argtypes = [_f64, _i32, ctypes.c_long, _i32, _i]
        self.hook.refhook_end.restype = ctypes.c_long
        self.hook.refhook_ray.argtypes = [_i]
        self.hook.refhook_set_real.argtypes = [_vp]
        self.hook.refhook_set_real(ctypes.cast(H.rayTetraPlucker_full, _vp))

    @staticmethod
    def _bind(L):
        L.pre_compute_vol.argtypes = [ctypes.POINTER(_vp), _i, _i32, _i, ctypes.c_float]
        L.gradients.argtypes = [_i32, _i, _f64]
        L.gradients.restype = _vp
        L.find_forward_hull.argtypes = [_i32, _i, _f64, _i, _u32]
        L.find_forward_hull.restype = _i
        L.copy_fh_triangles.argtypes = [_i32, _i, _f64, _i, _i, _u32]
        L.copy_fh_triangles.restype = _vp
        L.pt_loc_2d.argtypes = [_i32, _f64, ctypes.POINTER(_i), _d, _d]
        L.pt_loc_2d.restype = _i

    def _take(self, ptr, count, dtype):
        ctype = ctypes.c_double if dtype == np.float64 else ctypes.c_int
        arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctype)), shape=(count,)).copy()
        self.libc.free(ptr)
        return arr

    # -- precompute, each on the stock build ---------------------------------
    def density(self, pos4, tetra, p_mass, lib=None):
        L = lib or self.stock
        pos = np.array(pos4, dtype=np.float64, order="C", copy=True)
        pp = _vp(pos.ctypes.data)
        L.pre_compute_vol(ctypes.byref(pp), len(pos), tetra, len(tetra), p_mass)
        return pos

    def gradients(self, tetra, pos4, lib=None):
        L = lib or self.stock
        p = L.gradients(tetra, len(tetra), pos4)
        return self._take(p, len(tetra) * 3, np.float64).reshape(-1, 3)

    @staticmethod
    def bitmap_words(n_tetra):
        # create_bitmap(n_tetra*4) allocates (n/BITS_PER_WORD)+1 words of 4 used bits
        return np.zeros(n_tetra * 4 // 4 + 1, dtype=np.uint32)

    def forward_hull(self, tetra, pos4, lib=None):
        L = lib or self.stock
        bm = self.bitmap_words(len(tetra))
        n = L.find_forward_hull(tetra, len(tetra), pos4, len(pos4), bm)
        return bm, n

    def hull_triangles(self, tetra, pos4, bitmap, n_tri, lib=None):
        L = lib or self.stock
        p = L.copy_fh_triangles(tetra, len(tetra), pos4, len(pos4), n_tri, bitmap)
        return self._take(p, n_tri * 8, np.int32).reshape(-1, 8)

    def prepare(self, pos4, tetra, p_mass, lib=None):
        pos = self.density(pos4, tetra, p_mass, lib)
        grad = self.gradients(tetra, pos, lib)
        bm, n = self.forward_hull(tetra, pos, lib)
        tri = self.hull_triangles(tetra, pos, bm, n, lib)
        return dict(pos=pos, grad=grad, bitmap=bm, tri=tri, tetra=tetra)

    # -- explicit-offset harness ---------------------------------------------
    def map(self, prep, G, box_len, box_len_z, center, S, delta_sample, seed, per_ray=False):
        m = np.zeros(G * G, np.float64)
        n_rays = G * G * S
        rr = np.zeros(n_rays, np.float64) if per_ray else None
        rc = np.zeros(n_rays, np.int32) if per_ray else None
        self.harness.refh_map(prep["pos"], prep["tetra"], prep["grad"], prep["tri"], G, box_len,
                              box_len_z, *center, S, delta_sample, seed, m, _ptr(rr), _ptr(rc))
        m = m.reshape(G, G)
        return (m, rr, rc) if per_ray else m

    def trace(self, prep, xs, ys, z0, lz, dxy, seed, record_visits=False, max_calls=None):
        """Per-ray integral and crossing count; with record_visits, also the
        sequence of visited tet indices per ray (list of int arrays)."""
        n = len(xs)
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        rho = np.zeros(n, np.float64)
        crossed = np.zeros(n, np.int32)
        cb = None
        if record_visits:
            cap = max_calls or (n * 4096)
            buf = np.zeros((cap, 4), np.int32)
            starts = np.zeros(n + 1, np.int32)
            self.hook.refhook_begin(prep["pos"], buf, cap, starts, n)
            cb = self._on_ray(lambda i: self.hook.refhook_ray(i))
        self.harness.refh_trace(prep["pos"], prep["tetra"], prep["grad"], prep["tri"], n, xs, ys,
                                z0, lz, dxy, seed, rho, crossed, ctypes.cast(cb, _vp) if cb else None)
        if not record_visits:
            return rho, crossed, None
        total = self.hook.refhook_end()
        if total >= cap:
            raise RuntimeError("visit log overflow")
        starts[n] = total
        lookup = {tuple(r): t for t, r in enumerate(prep["tetra"][:, :4].tolist())}
        visits = []
        for i in range(n):
            rows = buf[starts[i]:starts[i + 1]]
            seq = [lookup[tuple(r)] for r in rows.tolist()]
            dedup = [t for k, t in enumerate(seq) if k == 0 or t != seq[k - 1]]
            visits.append(np.array(dedup if crossed[i] > 0 else [], dtype=np.int32))
        return rho, crossed, visits

    def grid(self, prep, G, box_len, center, ss, seed):
        g = np.zeros(G * G * G, np.float64)
        self.harness.refh_grid(prep["pos"], prep["tetra"], prep["grad"], prep["tri"], G, box_len,
                               g, *center, ss, seed)
        return g.reshape(G, G, G)

    # -- the stock entry points (libc rand()) --------------------------------
    def set_threads(self, n):
        """Sets the OpenMP team size of the stock build's parallel regions and
        returns the size its runtime reports (omp_get_max_threads)."""
        self.stock.omp_set_num_threads(int(n))
        return int(self.stock.omp_get_max_threads())

    def compute_density(self, pos4, tetra, G, box_len, box_len_z, rho, p_mass, center, S,
                        delta_sample):
        self.stock.compute_density(pos4, len(pos4), tetra, len(tetra), G, box_len, box_len_z, rho,
                                   p_mass, *center, S, delta_sample)
        return rho
