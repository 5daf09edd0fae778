// mesh.h - the device-resident mesh behind a dtfe_mesh_t handle.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "sdtfe_b200.h"
#include "walk64.cuh"
#include "walk32.cuh"

namespace sdtfe {

// thread-local last error (capi.cu)
dtfe_status_t set_error(dtfe_status_t s, const char* fmt, ...);

// process-wide count of kernels this library has launched (capi.cu)
void count_launch(unsigned n = 1);

#define SDTFE_CUDA(expr)                                                                  \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return ::sdtfe::set_error(e_ == cudaErrorMemoryAllocation ? DTFE_ERR_NOMEM           \
                                                                : DTFE_ERR_CUDA,          \
                                "%s:%d %s: %s", __FILE__, __LINE__, #expr,                 \
                                cudaGetErrorString(e_));                                  \
  } while (0)

#define SDTFE_TRY(expr)                 \
  do {                                  \
    dtfe_status_t s_ = (expr);          \
    if (s_ != DTFE_OK) return s_;       \
  } while (0)

// Counters of one map launch, in device memory.
enum StatSlot : int {
  kStatRays = 0,
  kStatVisits = 1,
  kStatStatus0 = 2,  // .. kStatStatus0 + DTFE_N_RAY_STATUS - 1
  kStatFallback = kStatStatus0 + DTFE_N_RAY_STATUS,
  kStatCount
};

struct AxisData {
  bool hull_built = false;
  int n_tri = 0;
  TriRec64* tri = nullptr;  // device, n_tri records
  int* tri_rows = nullptr;  // device, n_tri * 8 ints in the reference's tri_data layout
  signed char* tri_face = nullptr;  // device, n_tri: the tet face (0..3) under each triangle
  // walk records in this axis' projected frame (built on demand, per precision)
  TetRec64* rec64 = nullptr;
  TetRot32* rot32 = nullptr;  // 4 per tet (one per entry face): the mixed walk's records
};

struct Mesh {
  int n = 0, nt = 0;
  float p_mass = 0.f;
  unsigned flags = 0;
  bool fp32_exact = false;
  bool has_density = false;
  double coord_max = 0;     // largest |x|, |y|, |z| of any vertex (rounded up)
  cudaStream_t stream = nullptr;
  double4* pos = nullptr;   // (x, y, z, rho) in the original frame
  int4* rows = nullptr;     // 2 per tet: vertex ids, neighbour ids
  double* grad = nullptr;   // 3 per tet
  int* adj = nullptr;       // tets incident to each vertex
  double4* fld64 = nullptr; // per-tet FP64 field (k, grad) of the mixed 3-D grid (on demand)
  AxisData ax[3];
  unsigned long long* stats = nullptr;  // kStatCount counters of the last map
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timed = false;       // ev0/ev1 bracket the last walk launch
  int tune32 = -1;          // mixed-map kernel variant chosen by the autotuner (-1: default)
  int fp64_location = DTFE_LOCATE_PER_RAY;  // FP64 maps' point location (dtfe_locate_t)
  size_t bytes = 0;
};

// tricache.cc: triangulate()'s cache of results, keyed by the exact input.
// lookup returns a malloc'd copy of the rows (nullptr: not cached).
int* tri_cache_lookup(const double* xyz4, int n, const char* options, size_t* n_tetra);
void tri_cache_insert(const double* xyz4, int n, const char* options, const int* tetra,
                      size_t n_tetra);

// mesh.cu
dtfe_status_t mesh_upload(Mesh* m, const double* particle_data, int n, const int* tetra_data,
                          int nt, float p_mass, unsigned flags);
dtfe_status_t mesh_density(Mesh* m);
dtfe_status_t mesh_gradients(Mesh* m);
dtfe_status_t mesh_records(Mesh* m, int axis, bool want64, bool want32);
// the mixed 3-D grid's per-tet FP64 field (k_field64), built once on the mesh stream
dtfe_status_t mesh_field64(Mesh* m);
void mesh_drop_records(Mesh* m, int axis);
// device bytes of one axis' walk records: held now, and still to build for a
// map of the given precision
size_t mesh_record_bytes(const Mesh& m, int axis);
// returns the current device's cached, unused walk-record memory to the system
void mesh_trim_record_pool();
// per-call device scratch, stream-ordered on s from the walk-record pool
dtfe_status_t scratch_alloc_async(void** p, size_t bytes, cudaStream_t s);
void scratch_free_async(void* p, cudaStream_t s);
size_t mesh_missing_record_bytes(const Mesh& m, int axis, int precision);
// host_mask (optional) replaces the forward-face test with a caller's bitmap
// (one 32-bit word per tet, faces in bits 0..3)
dtfe_status_t mesh_hull(Mesh* m, int axis, const uint32_t* host_mask, int* count_out);
dtfe_status_t mesh_hull_mask(Mesh* m, int axis, uint32_t* host_mask_out, int* count_out);
void mesh_free(Mesh* m);

// Cyclic permutation of the projection axis: the walk sees (x', y', z').
__host__ __device__ inline void permute3(int axis, double x, double y, double z, double* px,
                                         double* py, double* pz) {
  if (axis == 1) {  // along x: (y, z, x)
    *px = y; *py = z; *pz = x;
  } else if (axis == 2) {  // along y: (z, x, y)
    *px = z; *py = x; *pz = y;
  } else {
    *px = x; *py = y; *pz = z;
  }
}

// capi.cu: parameter checks, and the records + hull a map of (axis,
// precision) reads, built on the mesh stream
dtfe_status_t check_params(const Mesh& m, const dtfe_map_params_t* p);
dtfe_status_t prepare_axis(Mesh& m, int axis, int precision);

// walk.cu / walk32.cu launchers
struct MapGeom {
  int axis;
  int G, S;
  double dxy, offx, offy, offz, lz, scale, soff, dist;
  uint64_t seed;
  int max_visits;
};
MapGeom map_geometry(const Mesh& m, const dtfe_map_params_t& p);
dtfe_status_t launch_map64(Mesh& m, const MapGeom& g, double* d_map, cudaStream_t s,
                           double* ray_rho, int* ray_crossed, int* ray_status);
dtfe_status_t launch_map32(Mesh& m, const MapGeom& g, double* d_map, cudaStream_t s,
                           double* ray_rho, int* ray_crossed, int* ray_status);
dtfe_status_t launch_trace64(Mesh& m, int axis, int n_rays, const double* d_x, const double* d_y,
                             double z0, double lz, double dxy, uint64_t seed, int max_visits,
                             double* d_rho, int* d_crossed, int* d_status, int* d_visits,
                             int max_record, cudaStream_t s);
dtfe_status_t launch_trace32(Mesh& m, int axis, int n_rays, const double* d_x, const double* d_y,
                             double z0, double lz, double dxy, uint64_t seed, int max_visits,
                             double* d_rho, int* d_crossed, int* d_status, int* d_visits,
                             int max_record, cudaStream_t s);
int num_map32_variants();
void map32_variant_info(int i, int* block, int* minb, int* wide, int* rpt);
dtfe_status_t launch_grid64(Mesh& m, int G, double box_len, const double center[3], unsigned ss,
                            uint64_t seed, int max_visits, double* d_grid, cudaStream_t s);
dtfe_status_t launch_grid32(Mesh& m, int G, double box_len, const double center[3], unsigned ss,
                            uint64_t seed, int max_visits, double* d_grid, cudaStream_t s);

// Batched maps (walk.cu, walk32.cu): one persistent launch walks the tiles of
// several maps, pulled from a device counter.  A map may be split into ranges
// of tiles that go to different launches (the serving loop does that).
struct BatchMap {
  Mesh* mesh;
  MapGeom g;
  double* d_map;              // the map, accumulated
  unsigned long long* stats;  // kStatCount device counters for this map
  int tile0 = 0;              // the range of the map's tiles this launch walks
  int count = -1;             // (-1: from tile0 to the end)
};
struct BatchPlan {
  int precision = DTFE_FP64;
  int variant = -1;           // mixed kernel variant (ignored for FP64)
  int n_jobs = 0;
  long long total_tiles = 0;
  size_t smem = 0;            // dynamic shared memory per block
  std::vector<unsigned char> jobs;  // the job table as the kernel reads it
};
// tiles of a whole map (the tile shape depends on precision and variant)
int map_tiles64(const MapGeom& g);
int map_tiles32(const MapGeom& g, int variant);
dtfe_status_t plan_batch64(const BatchMap* maps, int n, BatchPlan* plan);
dtfe_status_t plan_batch32(const BatchMap* maps, int n, int variant, BatchPlan* plan);
// blocks of a persistent launch: resident blocks per SM x SMs
dtfe_status_t batch_grid64(size_t smem, int* grid, int* block);
dtfe_status_t batch_grid32(int variant, size_t smem, int* grid, int* block);
// d_jobs holds plan.jobs; d_queue is a zeroed counter
dtfe_status_t launch_batch64(const BatchPlan& plan, const void* d_jobs, unsigned long long* d_queue,
                             int grid, cudaStream_t s);
// (mixed) d_loc: room for plan.total_tiles tile locations (kLocBytes each)
dtfe_status_t launch_batch32(const BatchPlan& plan, const void* d_jobs, unsigned long long* d_queue,
                             void* d_loc, int grid, cudaStream_t s);
// bytes of one tile's shared point-location result
constexpr size_t kLocBytes = 8;
int default_variant32();

}  // namespace sdtfe

// the object behind a dtfe_mesh_t handle
struct dtfe_mesh_s {
  sdtfe::Mesh m;
  std::mutex mu;  // one call at a time per handle
};
