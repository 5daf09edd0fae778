"""sdtfe_b200: SDTFE's density-estimation path on NVIDIA B200 (sm_100a).

The Delaunay mesh is built on the host (Qhull) and uploaded once; densities,
gradients, the projected hull and the Monte Carlo line-of-sight walk run as
CUDA kernels behind the C ABI of include/sdtfe_b200.h, which also exports the
reference's dtfe.h / triangulate.h / utils.h entry points.  This package holds
the host-side mirror of that interface (ctypes) and the synthetic workloads.
"""
from ._lib import (AXIS_X, AXIS_Y, AXIS_Z, BATCH_GRAPH, BATCH_ZERO_MAPS, DTFE_FP64, DTFE_MIXED,
                   ERR_ADMISSION, ERR_TIMEOUT, LOCATE_PER_RAY, LOCATE_TILE, MESH_FIELD, MESH_LAZY, MESH_NO_FP64_REC, RAY_BUDGET,
                   RAY_LOC_BUDGET, RAY_MISS, RAY_NO_EXIT, RAY_OK, RAY_PERTURB_MAX, SERVE_FAIR,
                   SERVE_FIFO, Batch, DTFEError, MapParams, MapStats, Mesh, Server, lib, map_params,
                   tetra_from_cells, triangulate, trim_memory)

__all__ = [
    "AXIS_X", "AXIS_Y", "AXIS_Z", "BATCH_GRAPH", "BATCH_ZERO_MAPS", "DTFE_FP64", "DTFE_MIXED",
    "ERR_ADMISSION", "ERR_TIMEOUT", "LOCATE_PER_RAY", "LOCATE_TILE", "MESH_FIELD", "MESH_LAZY", "MESH_NO_FP64_REC", "RAY_BUDGET",
    "RAY_LOC_BUDGET", "RAY_MISS", "RAY_NO_EXIT", "RAY_OK", "RAY_PERTURB_MAX", "SERVE_FAIR",
    "SERVE_FIFO", "Batch", "DTFEError", "MapParams", "MapStats", "Mesh", "Server", "lib",
    "map_params", "tetra_from_cells", "triangulate", "trim_memory",
]
