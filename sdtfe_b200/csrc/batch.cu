// batch.cu - many maps in one persistent launch (dtfe_batch_*).
//
// The reference maps one mesh per compute_density call, one OpenMP loop over
// 4x4-pixel tiles (src/dtfe.c:554-654).  A batch instead gives every map of
// the set (different meshes, sides, samples and axes) a range in one global
// tile queue; a persistent grid sized to the GPU's resident blocks pulls
// tiles from a device counter (k_batch32 / k_batch64), so small and large
// maps share the SMs and the launch has one tail instead of one per map.
// Tiles of expensive maps (more tets per ray) are queued first, which leaves
// the cheapest tiles for the tail.  The launch can be captured once in a CUDA
// graph: the counter reset, the optional map zeroing and the kernel replay
// as one graph launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "mesh.h"

using namespace sdtfe;

struct dtfe_batch_s {
  std::vector<dtfe_batch_job_t> jobs;  // in the caller's order
  std::vector<int> order;              // queue order: jobs by decreasing tile cost
  unsigned flags = 0;
  int precision = DTFE_FP64;
  int variant = -1;
  BatchPlan plan;
  int grid = 0, block = 0;
  void* d_jobs = nullptr;
  size_t d_jobs_bytes = 0;
  void* d_loc = nullptr;  // mixed: one tile location per queued tile
  size_t d_loc_bytes = 0;
  unsigned long long* d_queue = nullptr;
  unsigned long long* d_stats = nullptr;  // kStatCount per job, caller's order
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool launched = false;
};

namespace {

void drop_graph(dtfe_batch_s* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

void free_batch(dtfe_batch_s* b) {
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  if (b->d_jobs) cudaFree(b->d_jobs);
  if (b->d_loc) cudaFree(b->d_loc);
  if (b->d_queue) cudaFree(b->d_queue);
  if (b->d_stats) cudaFree(b->d_stats);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// (re)plans the queue for the current variant and uploads the job table
dtfe_status_t plan(dtfe_batch_s* b) {
  std::vector<BatchMap> maps(b->jobs.size());
  for (size_t k = 0; k < b->order.size(); ++k) {
    const int i = b->order[k];
    const dtfe_batch_job_t& j = b->jobs[i];
    BatchMap& bm = maps[k];
    bm.mesh = &j.mesh->m;
    bm.g = map_geometry(j.mesh->m, j.params);
    bm.d_map = j.d_map;
    bm.stats = b->d_stats + (size_t)i * kStatCount;
  }
  const int n = (int)maps.size();
  if (b->precision == DTFE_MIXED) {
    SDTFE_TRY(plan_batch32(maps.data(), n, b->variant, &b->plan));
    SDTFE_TRY(batch_grid32(b->plan.variant, b->plan.smem, &b->grid, &b->block));
  } else {
    SDTFE_TRY(plan_batch64(maps.data(), n, &b->plan));
    SDTFE_TRY(batch_grid64(b->plan.smem, &b->grid, &b->block));
  }
  const size_t bytes = b->plan.jobs.size();
  if (bytes > b->d_jobs_bytes) {
    if (b->d_jobs) SDTFE_CUDA(cudaFree(b->d_jobs));
    b->d_jobs = nullptr;
    SDTFE_CUDA(cudaMalloc(&b->d_jobs, bytes));
    b->d_jobs_bytes = bytes;
  }
  if (bytes)
    SDTFE_CUDA(cudaMemcpyAsync(b->d_jobs, b->plan.jobs.data(), bytes, cudaMemcpyHostToDevice,
                               b->stream));
  const size_t loc_bytes =
      b->precision == DTFE_MIXED ? kLocBytes * (size_t)b->plan.total_tiles : 0;
  if (loc_bytes > b->d_loc_bytes) {
    SDTFE_CUDA(cudaStreamSynchronize(b->stream));  // no launch still reads the old buffer
    if (b->d_loc) SDTFE_CUDA(cudaFree(b->d_loc));
    b->d_loc = nullptr;
    b->d_loc_bytes = 0;
    SDTFE_CUDA(cudaMalloc(&b->d_loc, loc_bytes));
    b->d_loc_bytes = loc_bytes;
  }
  SDTFE_CUDA(cudaStreamSynchronize(b->stream));  // the host table is reused by the next plan
  drop_graph(b);
  return DTFE_OK;
}

// counter reset, optional map zeroing, the kernel: what a launch (or its graph) holds
dtfe_status_t enqueue(dtfe_batch_s* b, cudaStream_t s) {
  SDTFE_CUDA(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned long long), s));
  SDTFE_CUDA(cudaMemsetAsync(b->d_stats, 0, sizeof(unsigned long long) * kStatCount * b->jobs.size(), s));
  if (b->flags & DTFE_BATCH_ZERO_MAPS)
    for (const auto& j : b->jobs)
      SDTFE_CUDA(cudaMemsetAsync(j.d_map, 0, sizeof(double) * (size_t)j.params.grid_dim * j.params.grid_dim, s));
  if (b->precision == DTFE_MIXED)
    return launch_batch32(b->plan, b->d_jobs, b->d_queue, b->d_loc, b->grid, s);
  return launch_batch64(b->plan, b->d_jobs, b->d_queue, b->grid, s);
}

dtfe_status_t launch(dtfe_batch_s* b, cudaStream_t s) {
  if (b->flags & DTFE_BATCH_GRAPH) {
    if (!b->exec) {
      // capture on the batch's own stream (the legacy stream cannot capture)
      SDTFE_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      const dtfe_status_t st = enqueue(b, b->stream);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (st != DTFE_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      SDTFE_CUDA(e);
      b->graph = g;
      SDTFE_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    SDTFE_CUDA(cudaEventRecord(b->ev0, s));
    SDTFE_CUDA(cudaGraphLaunch(b->exec, s));
    // the graph's kernel nodes: the mixed path's tile locations, then the walk
    count_launch(b->plan.n_jobs ? (b->precision == DTFE_MIXED ? 2 : 1) : 0);
  } else {
    SDTFE_CUDA(cudaEventRecord(b->ev0, s));
    SDTFE_TRY(enqueue(b, s));
  }
  SDTFE_CUDA(cudaEventRecord(b->ev1, s));
  b->launched = true;
  return DTFE_OK;
}

// cost of one tile of a job, for the queue order: rays per tile x tets crossed
// per ray, which grows as the cube root of the tet count
double tile_cost(const dtfe_batch_job_t& j) {
  return (double)j.params.n_samples * std::cbrt((double)j.mesh->m.nt + 1.0);
}

}  // namespace

extern "C" {

dtfe_status_t dtfe_batch_create(const dtfe_batch_job_t* jobs, int n_jobs, unsigned flags,
                                dtfe_batch_t* out) {
  if (!out) return set_error(DTFE_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (n_jobs < 1 || !jobs) return set_error(DTFE_ERR_INVALID, "a batch needs at least one job");
  const int prec = jobs[0].params.precision;
  for (int i = 0; i < n_jobs; ++i) {
    if (!jobs[i].mesh || !jobs[i].d_map) return set_error(DTFE_ERR_INVALID, "job %d: NULL mesh or map", i);
    if (jobs[i].params.precision != prec)
      return set_error(DTFE_ERR_INVALID, "job %d: every job of a batch has the same precision", i);
    Mesh& m = jobs[i].mesh->m;
    std::lock_guard<std::mutex> lk(jobs[i].mesh->mu);
    SDTFE_TRY(check_params(m, &jobs[i].params));
    SDTFE_TRY(prepare_axis(m, jobs[i].params.axis, prec));
    SDTFE_CUDA(cudaStreamSynchronize(m.stream));
  }
  auto* b = new (std::nothrow) dtfe_batch_s();
  if (!b) return set_error(DTFE_ERR_NOMEM, "host allocation failed");
  b->jobs.assign(jobs, jobs + n_jobs);
  b->flags = flags;
  b->precision = prec;
  b->order.resize(n_jobs);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
    return tile_cost(b->jobs[x]) > tile_cost(b->jobs[y]);
  });
  dtfe_status_t st = DTFE_OK;
  auto cuda = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && st == DTFE_OK)
      st = set_error(e == cudaErrorMemoryAllocation ? DTFE_ERR_NOMEM : DTFE_ERR_CUDA, "%s: %s", what,
                     cudaGetErrorString(e));
  };
  cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
  if (st == DTFE_OK) cuda(cudaEventCreate(&b->ev0), "event");
  if (st == DTFE_OK) cuda(cudaEventCreate(&b->ev1), "event");
  if (st == DTFE_OK) cuda(cudaMalloc(&b->d_queue, sizeof(unsigned long long)), "queue");
  if (st == DTFE_OK)
    cuda(cudaMalloc(&b->d_stats, sizeof(unsigned long long) * kStatCount * n_jobs), "stats");
  if (st == DTFE_OK) st = plan(b);
  if (st != DTFE_OK) {
    free_batch(b);
    return st;
  }
  *out = b;
  return DTFE_OK;
}

dtfe_status_t dtfe_batch_launch(dtfe_batch_t b, void* stream) {
  if (!b) return set_error(DTFE_ERR_INVALID, "NULL batch");
  return launch(b, stream ? static_cast<cudaStream_t>(stream) : b->stream);
}

dtfe_status_t dtfe_batch_sync(dtfe_batch_t b) {
  if (!b) return set_error(DTFE_ERR_INVALID, "NULL batch");
  if (b->launched) SDTFE_CUDA(cudaEventSynchronize(b->ev1));
  SDTFE_CUDA(cudaStreamSynchronize(b->stream));
  return DTFE_OK;
}

dtfe_status_t dtfe_batch_stats(dtfe_batch_t b, dtfe_map_stats_t* per_job) {
  if (!b || !per_job) return set_error(DTFE_ERR_INVALID, "NULL argument");
  SDTFE_TRY(dtfe_batch_sync(b));
  const size_t n = b->jobs.size();
  std::vector<unsigned long long> c(n * kStatCount);
  SDTFE_CUDA(cudaMemcpy(c.data(), b->d_stats, sizeof(unsigned long long) * c.size(),
                        cudaMemcpyDeviceToHost));
  float ms = 0.f;
  if (b->launched) SDTFE_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  for (size_t i = 0; i < n; ++i) {
    const unsigned long long* x = c.data() + i * kStatCount;
    dtfe_map_stats_t& s = per_job[i];
    memset(&s, 0, sizeof(s));
    s.rays = x[kStatRays];
    s.visits = x[kStatVisits];
    for (int k = 0; k < DTFE_N_RAY_STATUS; ++k) s.status[k] = x[kStatStatus0 + k];
    s.fp64_fallbacks = x[kStatFallback];
    s.walk_ms = ms;
  }
  return DTFE_OK;
}

dtfe_status_t dtfe_batch_set_variant(dtfe_batch_t b, int variant) {
  if (!b) return set_error(DTFE_ERR_INVALID, "NULL batch");
  if (variant < -1 || variant >= num_map32_variants())
    return set_error(DTFE_ERR_INVALID, "variant %d not in -1..%d", variant, num_map32_variants() - 1);
  if (b->precision != DTFE_MIXED) return DTFE_OK;  // one FP64 kernel
  SDTFE_TRY(dtfe_batch_sync(b));
  b->variant = variant;
  return plan(b);
}

dtfe_status_t dtfe_batch_autotune(dtfe_batch_t b, int* best, dtfe_variant_t* timings) {
  if (!b) return set_error(DTFE_ERR_INVALID, "NULL batch");
  const int nv = num_map32_variants();
  if (b->precision != DTFE_MIXED) {
    if (best) *best = -1;
    return DTFE_OK;
  }
  const unsigned flags = b->flags;
  b->flags = DTFE_BATCH_ZERO_MAPS;  // timing runs are not captured and leave zeroed maps
  int best_v = -1;
  float best_ms = 0.f;
  dtfe_status_t st = DTFE_OK;
  for (int v = 0; v < nv && st == DTFE_OK; ++v) {
    b->variant = v;
    st = plan(b);
    float ms_v = 0.f;
    for (int rep = 0; rep < 2 && st == DTFE_OK; ++rep) {  // the first run warms L2 and the TLBs
      st = launch(b, b->stream);
      if (st != DTFE_OK) break;
      cudaError_t e = cudaEventSynchronize(b->ev1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->ev0, b->ev1);
      if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "batch autotune: %s", cudaGetErrorString(e));
      ms_v = ms;
    }
    if (timings) {
      map32_variant_info(v, &timings[v].block, &timings[v].min_blocks, &timings[v].wide_tile,
                         &timings[v].rays_per_thread);
      timings[v].ms = ms_v;
    }
    if (st == DTFE_OK && (best_v < 0 || ms_v < best_ms)) {
      best_v = v;
      best_ms = ms_v;
    }
  }
  if (st == DTFE_OK) {
    for (const auto& j : b->jobs)
      cudaMemsetAsync(j.d_map, 0, sizeof(double) * (size_t)j.params.grid_dim * j.params.grid_dim,
                      b->stream);
    b->variant = best_v;
    st = plan(b);
  }
  b->flags = flags;
  b->launched = false;
  if (best) *best = best_v;
  return st;
}

dtfe_status_t dtfe_batch_info(dtfe_batch_t b, int* grid, int* block, long long* tiles) {
  if (!b) return set_error(DTFE_ERR_INVALID, "NULL batch");
  if (grid) *grid = b->grid;
  if (block) *block = b->block;
  if (tiles) *tiles = b->plan.total_tiles;
  return DTFE_OK;
}

dtfe_status_t dtfe_batch_destroy(dtfe_batch_t b) {
  if (b) free_batch(b);
  return DTFE_OK;
}

}  // extern "C"
