"""ctypes bindings of libsdtfe_b200.so (the C ABI in include/sdtfe_b200.h).

Loading fails loudly when the shared library is missing: there is no CPU
fallback for anything in this package.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsdtfe_b200.so")

DTFE_FP64, DTFE_MIXED = 0, 1
AXIS_Z, AXIS_X, AXIS_Y = 0, 1, 2
MESH_FIELD, MESH_NO_FP64_REC, MESH_LAZY = 1, 2, 4
LOCATE_PER_RAY, LOCATE_TILE = 0, 1
RAY_OK, RAY_MISS, RAY_NO_EXIT, RAY_PERTURB_MAX, RAY_BUDGET, RAY_LOC_BUDGET = range(6)
N_RAY_STATUS = 6

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class MapParams(ctypes.Structure):
    _fields_ = [
        ("grid_dim", _i),
        ("box_len", _d),
        ("box_len_z", _d),
        ("center", _d * 3),
        ("n_samples", _i),
        ("delta_sample", _d),
        ("seed", ctypes.c_uint64),
        ("axis", _i),
        ("precision", _i),
        ("max_visits", _i),
    ]


class MapStats(ctypes.Structure):
    _fields_ = [
        ("rays", ctypes.c_ulonglong),
        ("visits", ctypes.c_ulonglong),
        ("status", ctypes.c_ulonglong * N_RAY_STATUS),
        ("fp64_fallbacks", ctypes.c_ulonglong),
        ("walk_ms", _d),
    ]

    def as_dict(self):
        return dict(rays=self.rays, visits=self.visits, status=list(self.status),
                    fp64_fallbacks=self.fp64_fallbacks, walk_ms=self.walk_ms)


class MeshInfo(ctypes.Structure):
    _fields_ = [
        ("n_particles", _i),
        ("n_tetra", _i),
        ("n_hull_tri", _i * 3),
        ("device_bytes", ctypes.c_size_t),
        ("fp32_exact", _i),
        ("map_variant", _i),
    ]


class Variant(ctypes.Structure):
    _fields_ = [("block", _i), ("min_blocks", _i), ("wide_tile", _i), ("ms", _d),
                ("rays_per_thread", _i)]


class BatchJob(ctypes.Structure):
    _fields_ = [("mesh", _vp), ("params", MapParams), ("d_map", _vp)]


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("device_budget", ctypes.c_size_t),
        ("max_active", _i),
        ("quantum_rays", ctypes.c_longlong),
        ("policy", _i),
        ("variant", _i),
    ]


class RequestInfo(ctypes.Structure):
    _fields_ = [
        ("status", _i),
        ("queue_ms", _d),
        ("latency_ms", _d),
        ("iterations", _i),
        ("stats", MapStats),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_ulonglong),
        ("completed", ctypes.c_ulonglong),
        ("failed", ctypes.c_ulonglong),
        ("iterations", ctypes.c_ulonglong),
        ("rays", ctypes.c_ulonglong),
        ("visits", ctypes.c_ulonglong),
        ("evictions", ctypes.c_ulonglong),
        ("budget", ctypes.c_size_t),
        ("in_use", ctypes.c_size_t),
        ("peak", ctypes.c_size_t),
        ("active", _i),
        ("queued", _i),
    ]


BATCH_GRAPH, BATCH_ZERO_MAPS = 1, 2
SERVE_FAIR, SERVE_FIFO = 0, 1
ERR_ADMISSION, ERR_TIMEOUT = 7, 8


class DTFEError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"status {status}: {msg}")
        self.status = status


_LIB = None


def lib() -> ctypes.CDLL:
    """The loaded library, with argtypes declared (loaded once)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C sdtfe_b200/csrc` "
                          "(or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    st = ctypes.c_int
    L.dtfe_last_error.restype = ctypes.c_char_p
    L.dtfe_mesh_create.argtypes = [_f64, _i, _i32, _i, ctypes.c_float, ctypes.c_uint,
                                   ctypes.POINTER(_vp)]
    L.dtfe_mesh_create.restype = st
    L.dtfe_mesh_destroy.argtypes = [_vp]
    L.dtfe_mesh_info.argtypes = [_vp, ctypes.POINTER(MeshInfo)]
    L.dtfe_mesh_sync.argtypes = [_vp]
    L.dtfe_mesh_density.argtypes = [_vp, _f64]
    L.dtfe_mesh_gradients.argtypes = [_vp, _f64]
    L.dtfe_mesh_adjacency.argtypes = [_vp, _i32]
    L.dtfe_mesh_hull.argtypes = [_vp, _i, _vp, ctypes.POINTER(_i)]
    L.dtfe_map.argtypes = [_vp, ctypes.POINTER(MapParams), _f64, ctypes.POINTER(MapStats)]
    L.dtfe_map_rays.argtypes = [_vp, ctypes.POINTER(MapParams), _f64, _f64, _i32, _i32,
                                ctypes.POINTER(MapStats)]
    L.dtfe_map_device.argtypes = [_vp, ctypes.POINTER(MapParams), _vp, _vp]
    L.dtfe_mesh_last_stats.argtypes = [_vp, ctypes.POINTER(MapStats)]
    L.dtfe_trace.argtypes = [_vp, ctypes.POINTER(MapParams), _i, _f64, _f64, _d, _d, _d, _f64,
                             _i32, _i32, _vp, _i]
    L.dtfe_grid.argtypes = [_vp, _i, _d, _d * 3, ctypes.c_uint, ctypes.c_uint64, _f64]
    L.dtfe_grid_ex.argtypes = [_vp, _i, _d, _d * 3, ctypes.c_uint, ctypes.c_uint64, _i, _f64]
    L.dtfe_grid_device.argtypes = [_vp, _i, _d, _d * 3, ctypes.c_uint, ctypes.c_uint64, _i, _vp,
                                   _vp]
    L.dtfe_set_triangulation_cache.argtypes = [ctypes.c_size_t]
    L.dtfe_set_triangulation_cache.restype = None
    L.dtfe_triangulation_cache_stats.argtypes = [ctypes.POINTER(ctypes.c_ulonglong),
                                                 ctypes.POINTER(ctypes.c_ulonglong),
                                                 ctypes.POINTER(ctypes.c_size_t),
                                                 ctypes.POINTER(ctypes.c_size_t)]
    L.dtfe_triangulation_cache_stats.restype = None
    L.dtfe_set_default_precision.argtypes = [_i]
    L.dtfe_set_seed.argtypes = [ctypes.c_uint64]
    L.dtfe_kernel_launches.restype = ctypes.c_ulonglong
    L.dtfe_autotune.argtypes = [_vp, ctypes.POINTER(MapParams), ctypes.POINTER(_i), _vp]
    L.dtfe_set_variant.argtypes = [_vp, _i]
    L.dtfe_set_location.argtypes = [_vp, _i]
    L.dtfe_trim_memory.argtypes = []
    L.dtfe_tetra_from_cells.argtypes = [_f64, _i32, _i32, ctypes.c_size_t, _i32]
    # batches and the serving loop
    L.dtfe_batch_create.argtypes = [ctypes.POINTER(BatchJob), _i, ctypes.c_uint, ctypes.POINTER(_vp)]
    L.dtfe_batch_launch.argtypes = [_vp, _vp]
    L.dtfe_batch_sync.argtypes = [_vp]
    L.dtfe_batch_stats.argtypes = [_vp, ctypes.POINTER(MapStats)]
    L.dtfe_batch_autotune.argtypes = [_vp, ctypes.POINTER(_i), _vp]
    L.dtfe_batch_set_variant.argtypes = [_vp, _i]
    L.dtfe_batch_info.argtypes = [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i),
                                  ctypes.POINTER(ctypes.c_longlong)]
    L.dtfe_batch_destroy.argtypes = [_vp]
    L.dtfe_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)]
    L.dtfe_server_add_mesh.argtypes = [_vp, _vp, ctypes.POINTER(_i)]
    L.dtfe_server_submit.argtypes = [_vp, _i, ctypes.POINTER(MapParams), _vp,
                                     ctypes.POINTER(ctypes.c_uint64)]
    L.dtfe_server_wait.argtypes = [_vp, ctypes.c_uint64, _i, ctypes.POINTER(RequestInfo)]
    L.dtfe_server_stats.argtypes = [_vp, ctypes.POINTER(ServerStats)]
    L.dtfe_server_destroy.argtypes = [_vp]
    # drop-ins
    L.compute_density.argtypes = [_f64, _i, _i32, _i, _i, _d, _d, _f64, ctypes.c_float, _d, _d,
                                  _d, _i, _d]
    L.compute_3d_density.argtypes = [_f64, _i, _i32, _i, _i, _d, _f64, ctypes.c_float, _d, _d,
                                     _d, ctypes.c_uint]
    L.interpolate_to_3d_grid.argtypes = [_f64, _i, _i32, _i, _i, _d, _f64, _d, _d, _d,
                                         ctypes.c_uint]
    L.pre_compute_vol.argtypes = [ctypes.POINTER(_vp), _i, _i32, _i, ctypes.c_float]
    L.gradients.argtypes = [_i32, _i, _f64]
    L.gradients.restype = _vp
    L.find_forward_hull.argtypes = [_i32, _i, _f64, _i,
                                    np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")]
    L.find_forward_hull.restype = _i
    L.copy_fh_triangles.argtypes = [_i32, _i, _f64, _i, _i,
                                    np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")]
    L.copy_fh_triangles.restype = _vp
    L.convert_to_qhdata.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                                    ctypes.c_size_t]
    L.convert_to_qhdata.restype = _vp
    L.rotate3d.argtypes = [_f64, ctypes.c_size_t, _f64, _f64]
    L.shuffle_buff.argtypes = [_f64, _i, _i]
    L.create_bitmap.argtypes = [_i]
    L.create_bitmap.restype = _vp
    _LIB = L
    return L


def _check(status):
    if status != 0:
        raise DTFEError(status, lib().dtfe_last_error().decode())


def tetra_from_cells(pos4: np.ndarray, simplices: np.ndarray, neighbors: np.ndarray) -> np.ndarray:
    """The library's C layout step of triangulate() (Qhull cells -> tetra_data)."""
    s = np.ascontiguousarray(simplices, np.int32)
    n = np.ascontiguousarray(neighbors, np.int32)
    out = np.empty((len(s), 8), np.int32)
    lib().dtfe_tetra_from_cells(np.ascontiguousarray(pos4, np.float64), s, n, len(s), out)
    return out


def trim_memory():
    """Return the device memory the library keeps for the next mesh to the system."""
    _check(lib().dtfe_trim_memory())


def triangulate(pos4: np.ndarray) -> np.ndarray:
    """Host Qhull (SciPy's build, options of src/main.c:160) + the library's layout step."""
    from scipy.spatial import Delaunay

    d = Delaunay(np.ascontiguousarray(pos4[:, :3]), qhull_options="Qt Qbb Qz")
    return tetra_from_cells(pos4, d.simplices, d.neighbors)


def map_params(grid_dim, box_len, box_len_z, center, n_samples, delta_sample=0.0, seed=1,
               axis=AXIS_Z, precision=DTFE_FP64, max_visits=0) -> MapParams:
    p = MapParams()
    p.grid_dim = grid_dim
    p.box_len = box_len
    p.box_len_z = box_len_z
    p.center[:] = list(center)
    p.n_samples = n_samples
    p.delta_sample = delta_sample
    p.seed = seed
    p.axis = axis
    p.precision = precision
    p.max_visits = max_visits
    return p


class Mesh:
    """A device-resident mesh (dtfe_mesh_t)."""

    def __init__(self, pos4: np.ndarray, tetra: np.ndarray, p_mass: float = 1.0, flags: int = 0):
        self.pos4 = np.ascontiguousarray(pos4, np.float64)
        self.tetra = np.ascontiguousarray(tetra, np.int32)
        h = _vp()
        _check(lib().dtfe_mesh_create(self.pos4, len(self.pos4), self.tetra, len(self.tetra),
                                      p_mass, flags, ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().dtfe_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self) -> MeshInfo:
        i = MeshInfo()
        _check(lib().dtfe_mesh_info(self.h, ctypes.byref(i)))
        return i

    def density(self) -> np.ndarray:
        out = np.empty(len(self.pos4), np.float64)
        _check(lib().dtfe_mesh_density(self.h, out))
        return out

    def gradients(self) -> np.ndarray:
        out = np.empty((len(self.tetra), 3), np.float64)
        _check(lib().dtfe_mesh_gradients(self.h, out))
        return out

    def adjacency(self) -> np.ndarray:
        out = np.empty(len(self.pos4), np.int32)
        _check(lib().dtfe_mesh_adjacency(self.h, out))
        return out

    def hull(self, axis=AXIS_Z) -> np.ndarray:
        n = _i()
        _check(lib().dtfe_mesh_hull(self.h, axis, None, ctypes.byref(n)))
        tri = np.empty((max(n.value, 1), 8), np.int32)
        _check(lib().dtfe_mesh_hull(self.h, axis, tri.ctypes.data_as(_vp), ctypes.byref(n)))
        return tri[:n.value]

    def map(self, params: MapParams, out: np.ndarray | None = None, per_ray: bool = False):
        """(map, MapStats); with per_ray, (map, stats, ray integrals, ray
        crossings, ray statuses), ray (row*G + col)*n_samples + sample."""
        G = params.grid_dim
        m = np.zeros((G, G), np.float64) if out is None else out
        st = MapStats()
        if not per_ray:
            _check(lib().dtfe_map(self.h, ctypes.byref(params), m.reshape(-1), ctypes.byref(st)))
            return m, st
        n = G * G * params.n_samples
        rr = np.zeros(n, np.float64)
        rc = np.zeros(n, np.int32)
        rs = np.zeros(n, np.int32)
        _check(lib().dtfe_map_rays(self.h, ctypes.byref(params), m.reshape(-1), rr, rc, rs,
                                   ctypes.byref(st)))
        return m, st, rr, rc, rs

    def map_device(self, params: MapParams, d_map_ptr: int, stream_ptr: int = 0):
        _check(lib().dtfe_map_device(self.h, ctypes.byref(params), _vp(d_map_ptr),
                                     _vp(stream_ptr) if stream_ptr else None))

    def autotune(self, params: MapParams):
        """Pick the fastest mixed-map kernel variant for maps like `params`.
        Returns (best index, list of per-variant dicts)."""
        n = lib().dtfe_num_variants()
        arr = (Variant * n)()
        best = _i()
        _check(lib().dtfe_autotune(self.h, ctypes.byref(params), ctypes.byref(best), arr))
        return best.value, [dict(block=v.block, min_blocks=v.min_blocks, wide_tile=v.wide_tile,
                                 rays_per_thread=v.rays_per_thread, ms=v.ms) for v in arr]

    def set_variant(self, variant: int):
        _check(lib().dtfe_set_variant(self.h, variant))

    def set_location(self, mode: int):
        """FP64 maps' point location: LOCATE_PER_RAY (the reference's walk from
        hull triangle 0 for every ray) or LOCATE_TILE (one shared walk per
        pixel tile, resumed per ray; bit-identical results)."""
        _check(lib().dtfe_set_location(self.h, mode))

    def last_stats(self) -> MapStats:
        st = MapStats()
        _check(lib().dtfe_mesh_last_stats(self.h, ctypes.byref(st)))
        return st

    def trace(self, params: MapParams, xs, ys, z0, lz, dxy, max_record=0):
        n = len(xs)
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        rho = np.zeros(n, np.float64)
        crossed = np.zeros(n, np.int32)
        status = np.zeros(n, np.int32)
        visits = np.full((n, max_record), -1, np.int32) if max_record else None
        _check(lib().dtfe_trace(self.h, ctypes.byref(params), n, xs, ys, z0, lz, dxy, rho, crossed,
                                status, visits.ctypes.data_as(_vp) if visits is not None else None,
                                max_record))
        return rho, crossed, status, visits

    def grid(self, G, box_len, center, ss, seed, out: np.ndarray | None = None,
             precision: int = DTFE_FP64) -> np.ndarray:
        g = np.zeros((G, G, G), np.float64) if out is None else out
        c = (_d * 3)(*center)
        _check(lib().dtfe_grid_ex(self.h, G, box_len, c, ss, seed, precision, g.reshape(-1)))
        return g

    def grid_device(self, G, box_len, center, ss, seed, d_grid_ptr: int,
                    precision: int = DTFE_FP64, stream_ptr: int = 0):
        c = (_d * 3)(*center)
        _check(lib().dtfe_grid_device(self.h, G, box_len, c, ss, seed, precision, _vp(d_grid_ptr),
                                      _vp(stream_ptr) if stream_ptr else None))


class Batch:
    """Maps of several meshes in one persistent launch (dtfe_batch_t).

    jobs: list of (Mesh, MapParams, device pointer of a grid_dim^2 float64 map)."""

    def __init__(self, jobs, flags: int = 0):
        self.meshes = [j[0] for j in jobs]  # keep the meshes alive
        arr = (BatchJob * len(jobs))()
        for k, (mesh, params, d_map) in enumerate(jobs):
            arr[k].mesh = mesh.h
            arr[k].params = params
            arr[k].d_map = d_map
        self.n = len(jobs)
        h = _vp()
        _check(lib().dtfe_batch_create(arr, len(jobs), flags, ctypes.byref(h)))
        self.h = h

    def launch(self, stream_ptr: int = 0):
        _check(lib().dtfe_batch_launch(self.h, _vp(stream_ptr) if stream_ptr else None))

    def sync(self):
        _check(lib().dtfe_batch_sync(self.h))

    def stats(self):
        arr = (MapStats * self.n)()
        _check(lib().dtfe_batch_stats(self.h, arr))
        return list(arr)

    def autotune(self):
        n = lib().dtfe_num_variants()
        arr = (Variant * n)()
        best = _i()
        _check(lib().dtfe_batch_autotune(self.h, ctypes.byref(best), arr))
        return best.value, [dict(block=v.block, min_blocks=v.min_blocks, wide_tile=v.wide_tile,
                                 rays_per_thread=v.rays_per_thread, ms=v.ms) for v in arr]

    def set_variant(self, v: int):
        _check(lib().dtfe_batch_set_variant(self.h, v))

    def info(self):
        g, b, t = _i(), _i(), ctypes.c_longlong()
        _check(lib().dtfe_batch_info(self.h, ctypes.byref(g), ctypes.byref(b), ctypes.byref(t)))
        return dict(grid=g.value, block=b.value, tiles=t.value)

    def close(self):
        if self.h:
            lib().dtfe_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving loop (dtfe_server_t): submit map requests, wait for them."""

    def __init__(self, device_budget: int = 0, max_active: int = 0, quantum_rays: int = 0,
                 policy: int = SERVE_FAIR, variant: int = -1):
        c = ServerConfig(device_budget, max_active, quantum_rays, policy, variant)
        h = _vp()
        _check(lib().dtfe_server_create(ctypes.byref(c), ctypes.byref(h)))
        self.h = h
        self.meshes = []
        self._maps = {}

    def add_mesh(self, mesh: Mesh) -> int:
        i = _i()
        _check(lib().dtfe_server_add_mesh(self.h, mesh.h, ctypes.byref(i)))
        self.meshes.append(mesh)
        return i.value

    def submit(self, mesh_id: int, params: MapParams, out: np.ndarray | None = None) -> int:
        G = params.grid_dim
        m = np.empty((G, G), np.float64) if out is None else out
        assert m.flags.c_contiguous and m.dtype == np.float64 and m.size == G * G
        rid = ctypes.c_uint64()
        _check(lib().dtfe_server_submit(self.h, mesh_id, ctypes.byref(params),
                                        m.ctypes.data_as(_vp), ctypes.byref(rid)))
        self._maps[rid.value] = m
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1):
        """(map, RequestInfo) of a finished request; raises DTFEError on failure or timeout."""
        info = RequestInfo()
        st = lib().dtfe_server_wait(self.h, rid, timeout_ms, ctypes.byref(info))
        if st == ERR_TIMEOUT:
            raise DTFEError(st, lib().dtfe_last_error().decode())
        m = self._maps.pop(rid, None)
        _check(st)
        return m, info

    def stats(self) -> ServerStats:
        s = ServerStats()
        _check(lib().dtfe_server_stats(self.h, ctypes.byref(s)))
        return s

    def close(self):
        if self.h:
            lib().dtfe_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
