/*
 * sdtfe_b200.h - device-resident DTFE meshes on NVIDIA B200 (sm_100a).
 *
 * The drop-in entry points of the reference (dtfe.h, triangulate.h, utils.h,
 * bitmap.h in this directory) are implemented on top of this handle API.  A
 * handle owns one Delaunay mesh in GPU memory: vertex positions and DTFE
 * densities, tet vertex/neighbour rows, per-tet gradients, the packed walk
 * records of each precision and the projected forward hull per projection
 * axis.  Every call returns a status; dtfe_last_error() gives the message of
 * the calling thread's last failure.
 *
 * Host pointers are plain C arrays in the reference layouts:
 *   particle_data  double[n*4]  (x, y, z, column 3 = density or field)
 *   tetra_data     int[nt*8]    (A, B, C, D, n_BDC, n_ACD, n_ADB, n_ABC)
 * Device pointers (the *_device calls) are CUDA global memory; a stream
 * argument of NULL means the handle's own stream.
 */
#ifndef SDTFE_B200_H
#define SDTFE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DTFE_OK = 0,
  DTFE_ERR_INVALID = 1,       /* bad argument                                   */
  DTFE_ERR_CUDA = 2,          /* CUDA runtime error                             */
  DTFE_ERR_NOMEM = 3,         /* device allocation failed                       */
  DTFE_ERR_MESH = 4,          /* index out of range in tetra_data               */
  DTFE_ERR_UNSUPPORTED = 5,   /* argument outside what this build implements   */
  DTFE_ERR_NO_TRIANGULATOR = 6, /* triangulate() called with no backend set     */
  DTFE_ERR_ADMISSION = 7,     /* request exceeds the serving memory budget      */
  DTFE_ERR_TIMEOUT = 8        /* dtfe_server_wait: the request is still running */
} dtfe_status_t;

/* arithmetic of the ray walk */
typedef enum {
  DTFE_FP64 = 0,  /* the reference's FP64 arithmetic, operation for operation */
  DTFE_MIXED = 1  /* FP32 walk, FP64 only where a filter says FP32 may be wrong */
} dtfe_precision_t;

/* projection axis; x and y project along a cyclic permutation of (x, y, z) */
typedef enum { DTFE_AXIS_Z = 0, DTFE_AXIS_X = 1, DTFE_AXIS_Y = 2 } dtfe_axis_t;

/* per-ray outcome (the reference prints a warning and drops the sample) */
typedef enum {
  DTFE_RAY_OK = 0,
  DTFE_RAY_MISS = 1,         /* outside the projected hull (src/dtfe.c:626)          */
  DTFE_RAY_NO_EXIT = 2,      /* no enter/leave face pair (src/dtfe.c:321-325,344-348) */
  DTFE_RAY_PERTURB_MAX = 3,  /* > PERTURB_MAX perturbations (src/dtfe.c:338-342)      */
  DTFE_RAY_BUDGET = 4,       /* visit budget exhausted (corrupt neighbour links)      */
  DTFE_RAY_LOC_BUDGET = 5    /* point location exceeded its step budget              */
} dtfe_ray_status_t;

#define DTFE_N_RAY_STATUS 6

typedef struct dtfe_mesh_s *dtfe_mesh_t;

/* Surface-density map: the arguments of compute_density (src/dtfe.h:27-29)
 * plus the explicit sample seed and the walk controls. */
typedef struct {
  int grid_dim;          /* map side G; map[row*G + col]                         */
  double box_len;        /* map width and height                                 */
  double box_len_z;      /* slab depth along the projection axis                 */
  double center[3];      /* in the original (x, y, z) frame                      */
  int n_samples;         /* Monte Carlo samples per pixel (1..1024)               */
  double delta_sample;   /* MC box width; the pixel width when smaller          */
  uint64_t seed;         /* sample offsets sdtfe_sample_u01(seed, pixel, sample) */
  int axis;              /* dtfe_axis_t                                          */
  int precision;         /* dtfe_precision_t                                     */
  int max_visits;        /* per-ray visit budget; <= 0 selects 2*n_tetra + 64     */
} dtfe_map_params_t;

typedef struct {
  unsigned long long rays;
  unsigned long long visits;                       /* tets crossed, summed over rays */
  unsigned long long status[DTFE_N_RAY_STATUS];    /* rays per dtfe_ray_status_t     */
  unsigned long long fp64_fallbacks;               /* MIXED: guarded FP64 re-tests   */
  double walk_ms;                 /* device time of the map's kernels (walk, and tile location) */
} dtfe_map_stats_t;

typedef struct {
  int n_particles;
  int n_tetra;
  int n_hull_tri[3];     /* forward-hull triangles per axis (-1: not built yet)  */
  size_t device_bytes;   /* device memory held by the handle                     */
  int fp32_exact;        /* 1 when every coordinate is exactly a float          */
  int map_variant;       /* mixed-map kernel variant in use (dtfe_autotune)      */
} dtfe_mesh_info_t;

/* One mixed-map kernel variant: threads per block, blocks per SM the register
 * budget allows, the pixel tile shape (0: square-ish, 1: row strip), and the
 * rays each thread walks per tile. */
typedef struct {
  int block;
  int min_blocks;
  int wide_tile;
  double ms;             /* autotuner timing on its window (0 if not timed)     */
  int rays_per_thread;   /* rays each thread walks per tile                      */
} dtfe_variant_t;

/* mesh flags */
#define DTFE_MESH_FIELD 1u       /* column 3 is a field: skip the density step      */
#define DTFE_MESH_NO_FP64_REC 2u /* keep no FP64 walk records (MIXED maps only)     */
#define DTFE_MESH_LAZY 4u        /* build no walk records or hull at creation: the
                                    first map (or the serving loop) builds what it
                                    needs; for meshes held in bulk                */

const char *dtfe_last_error(void);
void dtfe_clear_error(void); /* empty the calling thread's last-error message */
const char *dtfe_status_string(dtfe_status_t s);

/* Upload a mesh and build everything the walks need: densities, gradients, and
 * the z axis' hull and walk records for the default precision (other axes and
 * precisions are built on first use; with DTFE_MESH_LAZY the z axis' are too).
 * Unless DTFE_MESH_FIELD is set, column 3
 * of particle_data is ignored and replaced on the device by the DTFE density
 * 4*p_mass / (sum of adjacent |V|) (src/triangulate.c:183-225). */
dtfe_status_t dtfe_mesh_create(const double *particle_data, int n_particles,
                               const int *tetra_data, int n_tetra, float p_mass,
                               unsigned flags, dtfe_mesh_t *out);
/* Releases the mesh's device memory, stream-ordered on the handle's own
 * stream (no device-wide synchronisation), into a pool that keeps it for the
 * next mesh.  Work the caller enqueued on its own streams with the mesh
 * (dtfe_map_device, dtfe_grid_device, batches) must have finished first. */
dtfe_status_t dtfe_mesh_destroy(dtfe_mesh_t mesh);
/* Returns the current device's mesh memory that the pool keeps for reuse
 * (up to an eighth of the device, at most 16 GB, once meshes are destroyed)
 * to the system, for callers that need it elsewhere. */
dtfe_status_t dtfe_trim_memory(void);
dtfe_status_t dtfe_mesh_info(dtfe_mesh_t mesh, dtfe_mesh_info_t *info);
dtfe_status_t dtfe_mesh_sync(dtfe_mesh_t mesh);

/* downloads (host pointers) */
dtfe_status_t dtfe_mesh_density(dtfe_mesh_t mesh, double *rho /* n */);
dtfe_status_t dtfe_mesh_gradients(dtfe_mesh_t mesh, double *grad /* 3*nt */);
dtfe_status_t dtfe_mesh_adjacency(dtfe_mesh_t mesh, int *counts /* n */);
dtfe_status_t dtfe_mesh_hull(dtfe_mesh_t mesh, int axis, int *tri /* 8*n_tri or NULL */,
                             int *n_tri);

/* Map into a host array (accumulated: map[p] += value, as the reference does). */
dtfe_status_t dtfe_map(dtfe_mesh_t mesh, const dtfe_map_params_t *p, double *map,
                       dtfe_map_stats_t *stats);
/* dtfe_map, plus every ray's outcome in host arrays of grid_dim^2 * n_samples
 * entries, ray (row*G + col)*n_samples + sample: its integral (0 unless
 * DTFE_RAY_OK), its tet crossings (0 unless DTFE_RAY_OK) and its
 * dtfe_ray_status_t.  For parity checks of whole maps; the reference's
 * shoot_3d_ray returns the same two numbers per sample (src/dtfe.c:247-374,
 * 625-640). */
dtfe_status_t dtfe_map_rays(dtfe_mesh_t mesh, const dtfe_map_params_t *p, double *map,
                            double *ray_rho, int *ray_crossed, int *ray_status,
                            dtfe_map_stats_t *stats);
/* Map into device memory, asynchronous on `stream` (accumulated as above). */
dtfe_status_t dtfe_map_device(dtfe_mesh_t mesh, const dtfe_map_params_t *p, double *d_map,
                              void *stream);
/* Counters of the last map launched on this handle (synchronises). */
dtfe_status_t dtfe_mesh_last_stats(dtfe_mesh_t mesh, dtfe_map_stats_t *stats);

/* Rays at explicit positions (x[i], y[i]) in the projected frame of p->axis,
 * walked over the slab z0 .. z0+lz; ray id i keys the perturbation stream.
 * visits (optional) receives up to max_record tet indices per ray (-1 padded). */
dtfe_status_t dtfe_trace(dtfe_mesh_t mesh, const dtfe_map_params_t *p, int n_rays,
                         const double *x, const double *y, double z0, double lz,
                         double delta_xy, double *rho, int *crossed, int *status,
                         int *visits, int max_record);

/* 3-D grid of interpolate_to_3d_grid (src/dtfe.c:668-735) into a host array of
 * G^3 doubles, accumulated; grid[(i*G + j)*G + iz], i along x and j along y. */
dtfe_status_t dtfe_grid(dtfe_mesh_t mesh, int grid_dim, double box_len, const double center[3],
                        unsigned supersampling, uint64_t seed, double *grid);
/* The same grid with the walk's arithmetic chosen: DTFE_FP64 (dtfe_grid) or
 * DTFE_MIXED (FP32 walk, guarded FP64: the same tets crossed, each fine node
 * assigned to the FP64 path's tet, cells within 1e-5 relative of FP64). */
dtfe_status_t dtfe_grid_ex(dtfe_mesh_t mesh, int grid_dim, double box_len, const double center[3],
                           unsigned supersampling, uint64_t seed, int precision, double *grid);
/* Grid into device memory (G^3 doubles, accumulated), asynchronous on
 * `stream` (NULL: the handle's stream); dtfe_mesh_last_stats gives its
 * counters and kernel time. */
dtfe_status_t dtfe_grid_device(dtfe_mesh_t mesh, int grid_dim, double box_len,
                               const double center[3], unsigned supersampling, uint64_t seed,
                               int precision, double *d_grid, void *stream);

/* Autotuner for the mixed-precision map kernel: times every variant on a
 * central window of the map p describes (same pixel size and samples, about a
 * sixteenth of the pixels), keeps the fastest for this handle and returns its
 * index.  timings (optional) receives dtfe_num_variants() entries. */
int dtfe_num_variants(void);
dtfe_status_t dtfe_autotune(dtfe_mesh_t mesh, const dtfe_map_params_t *p, int *best,
                            dtfe_variant_t *timings);
/* Select a variant explicitly (-1: the built-in default). */
dtfe_status_t dtfe_set_variant(dtfe_mesh_t mesh, int variant);

/* Point location of FP64 maps (src/dtfe.c:518-552, restarted from hull
 * triangle 0 for every sample at src/dtfe.c:624).  PER_RAY, the default, is
 * the reference's walk for every ray.  TILE walks once per pixel tile, for the
 * rectangle holding all of the tile's samples, while every edge test has one
 * outcome for the whole rectangle; each ray resumes from where the rectangle
 * first straddled a test, with the steps already taken counted against its
 * budget.  Every ray then reaches exactly the tet and status of its own walk
 * (the maps, crossings and statuses are bit-identical), at a fraction of the
 * steps where the projected hull is large.  Mixed maps always locate by tile.
 * TILE needs fewer than 2^27 hull triangles (DTFE_ERR_UNSUPPORTED otherwise). */
typedef enum { DTFE_LOCATE_PER_RAY = 0, DTFE_LOCATE_TILE = 1 } dtfe_locate_t;
dtfe_status_t dtfe_set_location(dtfe_mesh_t mesh, int mode);

/* Defaults used by the drop-in entry points of dtfe.h. */
void dtfe_set_default_precision(int precision);
int dtfe_get_default_precision(void);
/* Fix the sample seed of the drop-in entry points; 0 restores the default,
 * which keys each call's samples with one value drawn from the C library's
 * rand(), so that srand() keeps its meaning. */
void dtfe_set_seed(uint64_t seed);

/* Per-vertex DTFE density with no device allocation (no counterpart in the
 * reference; it exists for callers that cannot allocate device memory mid-run:
 * code inside a framework's memory pool or arena, serving loops that cannot
 * afford the device-wide synchronisation of cudaMalloc/cudaFree, hosts that
 * forbid allocation after start-up).  Inputs and output are device pointers
 * in the reference layouts: d_particle_data (n*4 doubles, column 3 ignored),
 * d_tetra_data (nt*8 ints); d_rho receives n densities, bit-identical to
 * dtfe_mesh_density.  Temporaries live in one static 48 MiB device array;
 * sizes that do not fit (about 1.9M tets) are rejected with
 * DTFE_ERR_UNSUPPORTED.  The first call on each device sets the array up
 * (cudaGetSymbolAddress, with that device current); with CUDA's lazy module
 * loading that is also when the 48 MiB are reserved on the device, which
 * then holds them until the process exits.  So make one call per device at
 * start-up - a call with n_particles == 0 does the set-up alone - before a
 * memory pool takes the device's memory.  All
 * calls share the array, so calls that overlap on the GPU (other streams,
 * other host threads) race.  The call blocks: it reads a validation flag
 * back mid-call and returns after its work on `stream` (NULL: the default
 * stream), which it orders after the stream's earlier work, has finished;
 * so no call can be captured into a CUDA graph. */
dtfe_status_t dtfe_density_noalloc(const double *d_particle_data, int n_particles,
                                   const int *d_tetra_data, int n_tetra, float p_mass,
                                   double *d_rho, void *stream);

/* ---- Batched maps -----------------------------------------------------
 * Maps of many meshes (cutouts) in one persistent kernel launch: the blocks
 * pull pixel tiles of every map from one device counter, so maps of uneven
 * size share the GPU with no tail per map.  Each map's result is
 * bit-identical to dtfe_map_device with the same parameters.  No counterpart
 * in the reference, which maps one mesh per call (src/dtfe.c:554-654). */
typedef struct {
  dtfe_mesh_t mesh;
  dtfe_map_params_t params;  /* every job of a batch has the same precision    */
  double *d_map;             /* grid_dim^2 doubles on the device, accumulated  */
} dtfe_batch_job_t;

typedef struct dtfe_batch_s *dtfe_batch_t;

#define DTFE_BATCH_GRAPH 1u     /* capture the launch once in a CUDA graph and replay it */
#define DTFE_BATCH_ZERO_MAPS 2u /* zero every map before each launch                  */

/* Builds every job's records and hull (on the meshes' streams), plans the
 * tile queue and uploads the job table.  The meshes and maps must outlive
 * the batch, and the meshes take no other calls while its launches run. */
dtfe_status_t dtfe_batch_create(const dtfe_batch_job_t *jobs, int n_jobs, unsigned flags,
                                dtfe_batch_t *out);
/* One launch over all jobs, asynchronous on `stream` (NULL: the batch's own). */
dtfe_status_t dtfe_batch_launch(dtfe_batch_t batch, void *stream);
dtfe_status_t dtfe_batch_sync(dtfe_batch_t batch);
/* Counters of the last launch, per job (walk_ms: the whole launch). */
dtfe_status_t dtfe_batch_stats(dtfe_batch_t batch, dtfe_map_stats_t *per_job);
/* Mixed batches: time every kernel variant over the whole batch (maps are
 * zeroed afterwards) and keep the fastest. */
dtfe_status_t dtfe_batch_autotune(dtfe_batch_t batch, int *best, dtfe_variant_t *timings);
dtfe_status_t dtfe_batch_set_variant(dtfe_batch_t batch, int variant);
/* persistent grid: blocks, threads per block, tiles in the queue */
dtfe_status_t dtfe_batch_info(dtfe_batch_t batch, int *grid, int *block, long long *tiles);
dtfe_status_t dtfe_batch_destroy(dtfe_batch_t batch);

/* ---- Serving loop ------------------------------------------------------
 * A host thread that keeps many meshes resident and serves map requests as
 * they arrive, with continuous batching: every iteration is one persistent
 * launch over a slice of the tiles of every admitted request, so requests
 * that arrive while others run join the next iteration, and consecutive
 * iterations overlap on two streams.  Requests are admitted while a slot is
 * free and their map buffer plus any walk records they need fit the device
 * budget; records of idle (mesh, axis) pairs are evicted least recently used
 * first.  A request's map is the same alone and in any mix: every pixel is
 * formed by one block from its own samples, whatever else the launch holds. */
typedef struct dtfe_server_s *dtfe_server_t;

#define DTFE_SERVE_FAIR 0  /* each iteration splits its tiles evenly over requests */
#define DTFE_SERVE_FIFO 1  /* each iteration serves the oldest requests first      */

typedef struct {
  size_t device_budget;    /* bytes for walk records and maps (0: the free device
                              memory less a reserve of 5% (at least 2 GiB), plus the
                              records of the meshes as they are registered)      */
  int max_active;          /* requests on the GPU at once (0: 64)                     */
  long long quantum_rays;  /* rays per iteration launch under light load (0: 2^20);
                              with a backlog up to 8x this                           */
  int policy;              /* DTFE_SERVE_FAIR or DTFE_SERVE_FIFO                      */
  int variant;             /* mixed kernel variant (-1: default)                      */
} dtfe_server_config_t;

typedef struct {
  int status;              /* dtfe_status_t of the request                            */
  double queue_ms;         /* submit -> admitted                                      */
  double latency_ms;       /* submit -> map in the caller's buffer                    */
  int iterations;          /* launches that walked some of its tiles                  */
  dtfe_map_stats_t stats;  /* its rays, visits, statuses (walk_ms: 0)                 */
} dtfe_request_info_t;

typedef struct {
  unsigned long long submitted, completed, failed;
  unsigned long long iterations;     /* kernel launches of the loop                  */
  unsigned long long rays, visits;   /* of completed requests                        */
  unsigned long long evictions;      /* walk records dropped for memory              */
  size_t budget, in_use, peak;       /* device bytes under the budget                */
  int active, queued;                /* right now                                    */
} dtfe_server_stats_t;

dtfe_status_t dtfe_server_create(const dtfe_server_config_t *cfg, dtfe_server_t *out);
/* Registers a mesh (the caller keeps it; it must outlive the server and take
 * no other calls while registered).  Its current walk records count against
 * the budget and may be evicted. */
dtfe_status_t dtfe_server_add_mesh(dtfe_server_t server, dtfe_mesh_t mesh, int *mesh_id);
/* Queues one map of mesh `mesh_id`; the map (grid_dim^2 doubles, host
 * memory, overwritten) is written when the request completes. */
dtfe_status_t dtfe_server_submit(dtfe_server_t server, int mesh_id, const dtfe_map_params_t *p,
                                 double *map, uint64_t *request_id);
/* Waits up to timeout_ms (< 0: forever) for a request; DTFE_ERR_TIMEOUT if it
 * is still running.  A completed request's info can be read once. */
dtfe_status_t dtfe_server_wait(dtfe_server_t server, uint64_t request_id, int timeout_ms,
                               dtfe_request_info_t *info);
dtfe_status_t dtfe_server_stats(dtfe_server_t server, dtfe_server_stats_t *stats);
/* Finishes every queued request, then stops the loop and frees its memory. */
dtfe_status_t dtfe_server_destroy(dtfe_server_t server);

/* Number of CUDA kernels this library has launched in this process (all
 * handles); benchmarks read it before and after a timed region. */
unsigned long long dtfe_kernel_launches(void);

/* Host Qhull backend for triangulate(): returns Qhull's Delaunay cells as
 * simplices[nt*4] and neighbors[nt*4] (neighbour k opposite vertex k, -1 on
 * the hull), malloc'd; returns 0 on success. */
typedef int (*dtfe_triangulator_fn)(const double *xyz4, int n, const char *options,
                                    int **simplices, int **neighbors, size_t *n_tetra,
                                    void *user);
void dtfe_set_triangulator(dtfe_triangulator_fn fn, void *user);
/* triangulate() keeps its recent results, keyed by the exact input (the
 * count, the options and every x, y, z), and answers a repeated input with a
 * copy of the stored rows without running the backend: Qhull is deterministic
 * for one input order and option set, so the rows are the ones it would
 * return.  No counterpart in the reference, which triangulates on every call
 * (python/pydtfe.cpp:54, src/main.c:160).  max_bytes bounds the host memory
 * held (coordinates and rows; least recently used entries go first); 0
 * disables the cache and empties it.  The default limit is the
 * SDTFE_TRI_CACHE_MB environment variable, else 1024 MB. */
void dtfe_set_triangulation_cache(size_t max_bytes);
void dtfe_triangulation_cache_stats(unsigned long long *hits, unsigned long long *misses,
                                    size_t *entries, size_t *bytes);
/* The layout step of triangulate() (src/triangulate.c:63-175): Qhull cells to
 * tetra_data rows, swapping B and C (and their neighbours) where
 * (AB x AC) . AD > 0.  tetra_out holds nt*8 ints. */
void dtfe_tetra_from_cells(const double *particle_data, const int *simplices,
                           const int *neighbors, size_t n_tetra, int *tetra_out);

#ifdef __cplusplus
}
#endif
#endif /* SDTFE_B200_H */
