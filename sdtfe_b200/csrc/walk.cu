// walk.cu - FP64 surface-density map, explicit-ray trace and 3-D grid.
//
// Compiled with -fmad=false (see walk64.cuh).
//
// Map kernel: one block per tile of TW x TH pixels, one thread per
// (pixel, sample) ray, pixel-major so that the S rays of a pixel sit in
// neighbouring lanes (they cross nearly the same tets: coherent gathers).  Each
// thread locates its sample on the projected hull, walks it, and parks the
// integral in shared memory; one thread per pixel then adds the samples in
// sample order and divides by the successful count, which reproduces the
// reference's per-pixel sum order (src/dtfe.c:615-645).
#include <cstdio>
#include <cstring>

#include "mesh.h"

namespace sdtfe {

namespace {

struct MapArgs64 {
  const TetRec64* __restrict__ rec;
  const TriRec64* __restrict__ tri;
  int n_tri;
  double* __restrict__ map;
  int G, S, TW, TH, tiles_x;
  double dxy, offx, offy, offz, lz, scale, soff;
  WalkConf64 walk;
  int loc_budget;
  const int2* __restrict__ loc;  // per-tile shared locations, or nullptr: every ray walks from triangle 0
  unsigned long long* __restrict__ stats;
  double* __restrict__ ray_rho;
  int* __restrict__ ray_crossed;
  int* __restrict__ ray_status;
};

struct BatchJob64 {
  MapArgs64 args;
  long long first;  // first global tile of the job
  int tile0;        // the job's first tile within its map
  int count;
};

// warp-aggregated counters: one atomic per warp and counter
__device__ __forceinline__ void add_stats(unsigned long long* stats, bool active, int crossed,
                                          int status, int fallbacks) {
  const unsigned mask = __activemask();
  const unsigned r = __reduce_add_sync(mask, active ? 1u : 0u);
  const unsigned v = __reduce_add_sync(mask, active ? (unsigned)crossed : 0u);
  const unsigned fb = __reduce_add_sync(mask, active ? (unsigned)fallbacks : 0u);
  unsigned st[DTFE_N_RAY_STATUS];
#pragma unroll
  for (int k = 0; k < DTFE_N_RAY_STATUS; ++k)
    st[k] = __reduce_add_sync(mask, (active && status == k) ? 1u : 0u);
  const int leader = __ffs(mask) - 1;
  if ((int)(threadIdx.x & 31) == leader) {
    if (r) atomicAdd(stats + kStatRays, (unsigned long long)r);
    if (v) atomicAdd(stats + kStatVisits, (unsigned long long)v);
    if (fb) atomicAdd(stats + kStatFallback, (unsigned long long)fb);
#pragma unroll
    for (int k = 0; k < DTFE_N_RAY_STATUS; ++k)
      if (st[k]) atomicAdd(stats + kStatStatus0 + k, (unsigned long long)st[k]);
  }
}

// One tile of one map (TW x TH pixels x S samples) on the block's threads.
__device__ __forceinline__ void map_tile64(const MapArgs64& a, int tile, double* s_val,
                                           unsigned char* s_ok) {
  const int P = a.TW * a.TH;
  const int tx0 = (tile % a.tiles_x) * a.TW, ty0 = (tile / a.tiles_x) * a.TH;
  for (int t = threadIdx.x; t < P * a.S; t += blockDim.x) {
    const int lp = t / a.S, s = t % a.S;
    const int col = tx0 + lp % a.TW, row = ty0 + lp / a.TW;
    const bool active = col < a.G && row < a.G;
    double v = 0.0;
    int crossed = 0, status = kRayMiss;
    if (active) {
      const long long p = (long long)row * a.G + col;
      const double x = col * a.dxy + a.offx - a.soff;
      const double y = row * a.dxy + a.offy - a.soff;
      const double xt = x + sdtfe_sample_u01(a.walk.seed, (uint64_t)p, (uint32_t)s, 0) * a.scale;
      const double yt = y + sdtfe_sample_u01(a.walk.seed, (uint64_t)p, (uint32_t)s, 1) * a.scale;
      const uint64_t rid = (uint64_t)p * (uint64_t)a.S + (uint64_t)s;
      int ft = -1;
      if (a.loc) ft = locate_from_tile(a.tri, __ldg(a.loc + tile), xt, yt, a.loc_budget, &status);
      else if (a.n_tri > 0) ft = locate64(a.tri, 0, xt, yt, a.loc_budget, &status);
      if (ft >= 0) {
        SurfaceAcc64 acc{a.offz, a.offz + a.lz, 0.0};
        status = walk64(a.rec, ft, xt, yt, a.walk, rid, acc, &crossed, nullptr, 0);
        if (status == kRayOk) v = acc.rho;
      }
      if (a.ray_rho) {
        a.ray_rho[rid] = v;
        a.ray_crossed[rid] = crossed;
        a.ray_status[rid] = status;
      }
    }
    s_val[t] = v;
    s_ok[t] = crossed > 0;
    add_stats(a.stats, active, crossed, status, 0);
  }
  __syncthreads();
  for (int lp = threadIdx.x; lp < P; lp += blockDim.x) {
    const int col = tx0 + lp % a.TW, row = ty0 + lp / a.TW;
    if (col >= a.G || row >= a.G) continue;
    double total = 0.0;
    int n_avg = 0;
    for (int s = 0; s < a.S; ++s) {
      total += s_val[lp * a.S + s];
      n_avg += s_ok[lp * a.S + s];
    }
    a.map[(size_t)row * a.G + col] += n_avg > 0 ? total / n_avg : 0.0;
  }
}

__global__ void __launch_bounds__(256) k_map64(const MapArgs64 a) {
  extern __shared__ double s_val[];  // P*S doubles, then P*S bytes of success flags
  unsigned char* s_ok = reinterpret_cast<unsigned char*>(s_val + a.TW * a.TH * a.S);
  map_tile64(a, blockIdx.x, s_val, s_ok);
}

// Every tile's shared point location (tile_location), one thread per tile,
// before a map whose mesh asked for tile-shared location.
__global__ void __launch_bounds__(128) k_locate_map64(const MapArgs64 a, int n_tiles,
                                                      int2* __restrict__ loc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n_tiles) loc[t] = tile_location(a, t);
}

// Persistent batch over several maps (see k_batch32 in walk32.cu): thread 0
// claims the next tile while the block walks the current one.
__device__ __forceinline__ void claim_tile64(const BatchJob64* __restrict__ jobs, int n_jobs,
                                             unsigned long long* __restrict__ queue,
                                             long long* tile, int* job) {
  const long long t = (long long)atomicAdd(queue, 1ull);
  int lo = 0, hi = n_jobs - 1;  // last job whose first tile <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (__ldg(&jobs[mid].first) <= t) lo = mid;
    else hi = mid - 1;
  }
  *tile = t;
  *job = lo;
}

__global__ void __launch_bounds__(256) k_batch64(const BatchJob64* __restrict__ jobs, int n_jobs,
                                                 long long total_tiles,
                                                 unsigned long long* __restrict__ queue) {
  extern __shared__ double s_val[];
  __shared__ MapArgs64 s_args;
  __shared__ long long s_tile[2];
  __shared__ int s_job[2];
  if (threadIdx.x == 0) claim_tile64(jobs, n_jobs, queue, &s_tile[0], &s_job[0]);
  __syncthreads();
  int cur_job = -1;
  for (int it = 0;; ++it) {
    const int slot = it & 1;
    const long long tile = s_tile[slot];
    const int j = s_job[slot];
    if (tile >= total_tiles) break;
    if (threadIdx.x == 0) claim_tile64(jobs, n_jobs, queue, &s_tile[slot ^ 1], &s_job[slot ^ 1]);
    if (j != cur_job) {  // j is the same for the whole block
      const int* src = reinterpret_cast<const int*>(&jobs[j].args);
      int* dst = reinterpret_cast<int*>(&s_args);
      for (int k = threadIdx.x; k < (int)(sizeof(MapArgs64) / sizeof(int)); k += blockDim.x)
        dst[k] = src[k];
      cur_job = j;
      __syncthreads();
    }
    unsigned char* s_ok = reinterpret_cast<unsigned char*>(s_val + s_args.TW * s_args.TH * s_args.S);
    map_tile64(s_args, jobs[j].tile0 + (int)(tile - jobs[j].first), s_val, s_ok);
    __syncthreads();  // s_val, s_args and the claimed slot are reused next
  }
}

__global__ void __launch_bounds__(128) k_trace64(const TetRec64* __restrict__ rec,
                                                 const TriRec64* __restrict__ tri, int n_tri,
                                                 int n_rays, const double* __restrict__ xs,
                                                 const double* __restrict__ ys, double z0,
                                                 WalkConf64 walk, int loc_budget,
                                                 double* __restrict__ rho, int* __restrict__ crossed,
                                                 int* __restrict__ status, int* __restrict__ visits,
                                                 int max_record) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_rays) return;
  int st = kRayMiss, c = 0;
  double v = 0.0;
  const int ft = n_tri > 0 ? locate64(tri, 0, xs[i], ys[i], loc_budget, &st) : -1;
  if (ft >= 0) {
    SurfaceAcc64 acc{z0, z0 + walk.lz, 0.0};
    st = walk64(rec, ft, xs[i], ys[i], walk, (uint64_t)i, acc, &c,
                visits ? visits + (size_t)i * max_record : nullptr, max_record);
    if (st == kRayOk) v = acc.rho;
  }
  rho[i] = v;
  crossed[i] = c;
  status[i] = st;
}

// One thread per grid column (i, j); its ss^2 sub-rays run in (is, js) order
// and add into the column in walk order, as interpolate_to_3d_grid does
// (src/dtfe.c:710-729).  No two threads touch the same column.
__global__ void __launch_bounds__(128) k_grid64(const TetRec64* __restrict__ rec,
                                                const TriRec64* __restrict__ tri, int n_tri, int G,
                                                double dxy, double offx, double offy, double offz,
                                                double box_len, int ss, WalkConf64 walk,
                                                int loc_budget, double* __restrict__ grid,
                                                unsigned long long* __restrict__ stats) {
  int i, j;
  const bool active = grid_column(G, &i, &j);
  const long long cidx = (long long)i * G + j;
  int worst = kRayOk, visits = 0;
  if (active) {
    const double ds = dxy / ss;
    ColumnAcc64 acc;
    acc.col = grid + (size_t)cidx * G;
    acc.z0 = offz;
    const double dz = box_len / G;
    acc.dzs = dz / ss;
    acc.nzs = G * ss;
    acc.w = 1. / ((unsigned)ss * (unsigned)ss * (unsigned)ss);
    acc.ss = ss;
    for (int is = 0; is < ss; ++is)
      for (int js = 0; js < ss; ++js) {
        const double x = i * dxy + offx + is * ds + ds / 2.;
        const double y = j * dxy + offy + js * ds + ds / 2.;
        int st = kRayMiss, c = 0;
        const int ft = n_tri > 0 ? locate64(tri, 0, x, y, loc_budget, &st) : -1;
        if (ft >= 0) {
          const uint64_t rid = ((uint64_t)cidx * ss + (uint64_t)is) * ss + (uint64_t)js;
          st = walk64(rec, ft, x, y, walk, rid, acc, &c, nullptr, 0);
        }
        visits += c;
        if (st > worst) worst = st;
      }
  }
  add_stats(stats, active, visits, worst, 0);
}

}  // namespace

MapGeom map_geometry(const Mesh& m, const dtfe_map_params_t& p) {
  MapGeom g;
  g.axis = p.axis;
  g.G = p.grid_dim;
  g.S = p.n_samples;
  // src/dtfe.c:579-589, in the projected frame
  double cx, cy, cz;
  permute3(p.axis, p.center[0], p.center[1], p.center[2], &cx, &cy, &cz);
  g.dxy = p.box_len / p.grid_dim;
  g.offx = -(p.box_len / 2.0) + cx;
  g.offy = -(p.box_len / 2.0) + cy;
  g.offz = -(p.box_len_z / 2.0) + cz;
  g.lz = p.box_len_z;
  g.scale = p.delta_sample > g.dxy ? p.delta_sample : g.dxy;
  g.soff = p.delta_sample > g.dxy ? (p.delta_sample - g.dxy) / 2.0 : 0.0;
  const double max_dist = g.dxy / 2.0;  // src/dtfe.c:273-274
  g.dist = max_dist / kPerturbMax;
  g.seed = p.seed;
  long long mv = p.max_visits > 0 ? p.max_visits : 2LL * m.nt + 64;
  g.max_visits = (int)(mv > 0x7fffffff ? 0x7fffffff : mv);
  return g;
}

// tile of pixels per block: TW x TH pixels x S samples <= 256 threads
static void tile_shape(int S, int* TW, int* TH) {
  int P = 256 / S;
  if (P < 1) P = 1;
  int lg = 31 - __builtin_clz((unsigned)P);
  int tw = 1 << ((lg + 1) / 2);
  int th = P / tw;
  if (th < 1) th = 1;
  *TW = tw;
  *TH = th;
}

// The kernel arguments of one FP64 map; *tiles_y receives its rows of tiles.
static dtfe_status_t map_args64(Mesh& m, const MapGeom& g, double* d_map,
                                unsigned long long* stats, double* ray_rho, int* ray_crossed,
                                int* ray_status, MapArgs64* out, int* tiles_y) {
  const AxisData& A = m.ax[g.axis];
  if (!A.rec64 || !A.hull_built) return set_error(DTFE_ERR_INVALID, "FP64 map before its records");
  MapArgs64& a = *out;
  a.rec = A.rec64;
  a.tri = A.tri;
  a.n_tri = A.n_tri;
  a.map = d_map;
  a.G = g.G;
  a.S = g.S;
  tile_shape(g.S, &a.TW, &a.TH);
  a.tiles_x = (g.G + a.TW - 1) / a.TW;
  *tiles_y = (g.G + a.TH - 1) / a.TH;
  a.dxy = g.dxy;
  a.offx = g.offx;
  a.offy = g.offy;
  a.offz = g.offz;
  a.lz = g.lz;
  a.scale = g.scale;
  a.soff = g.soff;
  a.walk = WalkConf64{g.lz, g.dist, g.seed, g.max_visits};
  a.loc_budget = 4 * A.n_tri + 64;
  a.loc = nullptr;
  a.stats = stats;
  a.ray_rho = ray_rho;
  a.ray_crossed = ray_crossed;
  a.ray_status = ray_status;
  return DTFE_OK;
}

dtfe_status_t launch_map64(Mesh& m, const MapGeom& g, double* d_map, cudaStream_t s,
                           double* ray_rho, int* ray_crossed, int* ray_status) {
  MapArgs64 a;
  int tiles_y = 0;
  SDTFE_TRY(map_args64(m, g, d_map, m.stats, ray_rho, ray_crossed, ray_status, &a, &tiles_y));
  const int P = a.TW * a.TH;
  int threads = P * g.S;
  threads = threads > 256 ? 256 : ((threads + 31) / 32) * 32;
  const size_t smem = (size_t)P * g.S * (sizeof(double) + 1);
  if (smem > 48 * 1024)
    SDTFE_CUDA(cudaFuncSetAttribute(k_map64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long blocks = (long long)a.tiles_x * tiles_y;
  const bool tile_loc = m.fp64_location == DTFE_LOCATE_TILE && a.n_tri > 0;
  if (tile_loc && a.n_tri >= (1 << 27))
    return set_error(DTFE_ERR_UNSUPPORTED,
                     "tile-shared location over %d hull triangles (at most 2^27 - 1)", a.n_tri);
  SDTFE_CUDA(cudaMemsetAsync(m.stats, 0, sizeof(unsigned long long) * kStatCount, s));
  SDTFE_CUDA(cudaEventRecord(m.ev0, s));
  void* loc = nullptr;
  if (tile_loc) {
    SDTFE_TRY(scratch_alloc_async(&loc, kLocBytes * (size_t)blocks, s));
    k_locate_map64<<<(unsigned)((blocks + 127) / 128), 128, 0, s>>>(a, (int)blocks,
                                                                    static_cast<int2*>(loc));
    count_launch();
    a.loc = static_cast<const int2*>(loc);
  }
  k_map64<<<(unsigned)blocks, threads, smem, s>>>(a);
  count_launch();
  const cudaError_t e = cudaGetLastError();
  if (loc) scratch_free_async(loc, s);
  SDTFE_CUDA(e);
  SDTFE_CUDA(cudaEventRecord(m.ev1, s));
  m.timed = true;
  return DTFE_OK;
}

int map_tiles64(const MapGeom& g) {
  int TW, TH;
  tile_shape(g.S, &TW, &TH);
  return ((g.G + TW - 1) / TW) * ((g.G + TH - 1) / TH);
}

dtfe_status_t plan_batch64(const BatchMap* maps, int n, BatchPlan* plan) {
  plan->precision = DTFE_FP64;
  plan->variant = -1;
  plan->n_jobs = 0;
  plan->total_tiles = 0;
  plan->smem = 0;
  plan->jobs.assign(sizeof(BatchJob64) * (size_t)(n > 0 ? n : 0), 0);
  for (int i = 0; i < n; ++i) {
    const BatchMap& b = maps[i];
    BatchJob64 j;
    int tiles_y = 0;
    SDTFE_TRY(map_args64(*b.mesh, b.g, b.d_map, b.stats, nullptr, nullptr, nullptr, &j.args, &tiles_y));
    const long long tiles = (long long)j.args.tiles_x * tiles_y;
    const long long cnt = b.count < 0 ? tiles - b.tile0 : b.count;
    if (b.tile0 < 0 || cnt < 0 || b.tile0 + cnt > tiles)
      return set_error(DTFE_ERR_INVALID, "batch map %d: tiles [%d, %lld) outside the map's %lld", i,
                       b.tile0, b.tile0 + cnt, tiles);
    if (cnt == 0) continue;
    j.first = plan->total_tiles;
    j.tile0 = b.tile0;
    j.count = (int)cnt;
    memcpy(plan->jobs.data() + sizeof(BatchJob64) * plan->n_jobs, &j, sizeof(j));
    ++plan->n_jobs;
    plan->total_tiles += cnt;
    const size_t smem = (size_t)j.args.TW * j.args.TH * j.args.S * (sizeof(double) + 1);
    if (smem > plan->smem) plan->smem = smem;
  }
  plan->jobs.resize(sizeof(BatchJob64) * plan->n_jobs);
  return DTFE_OK;
}

dtfe_status_t batch_grid64(size_t smem, int* grid, int* block) {
  int dev = 0, sms = 0, per_sm = 0;
  SDTFE_CUDA(cudaGetDevice(&dev));
  SDTFE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (smem > 48 * 1024)
    SDTFE_CUDA(cudaFuncSetAttribute(k_batch64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  SDTFE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch64, 256, smem));
  if (per_sm < 1) return set_error(DTFE_ERR_UNSUPPORTED, "FP64 batch: %zu B of shared memory per block", smem);
  *grid = per_sm * sms;
  *block = 256;
  return DTFE_OK;
}

dtfe_status_t launch_batch64(const BatchPlan& plan, const void* d_jobs, unsigned long long* d_queue,
                             int grid, cudaStream_t s) {
  if (plan.n_jobs == 0) return DTFE_OK;
  if (plan.smem > 48 * 1024)
    SDTFE_CUDA(cudaFuncSetAttribute(k_batch64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem));
  k_batch64<<<grid, 256, plan.smem, s>>>(static_cast<const BatchJob64*>(d_jobs), plan.n_jobs,
                                         plan.total_tiles, d_queue);
  count_launch();
  SDTFE_CUDA(cudaGetLastError());
  return DTFE_OK;
}

dtfe_status_t launch_trace64(Mesh& m, int axis, int n_rays, const double* d_x, const double* d_y,
                             double z0, double lz, double dxy, uint64_t seed, int max_visits,
                             double* d_rho, int* d_crossed, int* d_status, int* d_visits,
                             int max_record, cudaStream_t s) {
  const AxisData& A = m.ax[axis];
  if (!A.rec64 || !A.hull_built) return set_error(DTFE_ERR_INVALID, "FP64 trace before its records");
  WalkConf64 w{lz, (dxy / 2.0) / kPerturbMax, seed, max_visits};
  if (n_rays > 0) {
    k_trace64<<<(n_rays + 127) / 128, 128, 0, s>>>(A.rec64, A.tri, A.n_tri, n_rays, d_x, d_y, z0, w,
                                                   4 * A.n_tri + 64, d_rho, d_crossed, d_status,
                                                   d_visits, max_record);
    count_launch();
  }
  SDTFE_CUDA(cudaGetLastError());
  return DTFE_OK;
}

dtfe_status_t launch_grid64(Mesh& m, int G, double box_len, const double center[3], unsigned ss,
                            uint64_t seed, int max_visits, double* d_grid, cudaStream_t s) {
  const AxisData& A = m.ax[DTFE_AXIS_Z];
  if (!A.rec64 || !A.hull_built) return set_error(DTFE_ERR_INVALID, "grid before its records");
  const double dxy = box_len / G;
  const double offx = -(box_len / 2.0) + center[0];
  const double offy = -(box_len / 2.0) + center[1];
  const double offz = -(box_len / 2.0) + center[2];
  WalkConf64 w{box_len, (dxy / 2.0) / kPerturbMax, seed, max_visits};
  SDTFE_CUDA(cudaMemsetAsync(m.stats, 0, sizeof(unsigned long long) * kStatCount, s));
  SDTFE_CUDA(cudaEventRecord(m.ev0, s));
  k_grid64<<<grid_blocks(G), 128, 0, s>>>(A.rec64, A.tri, A.n_tri, G, dxy, offx, offy, offz,
                                          box_len, (int)ss, w, 4 * A.n_tri + 64, d_grid, m.stats);
  count_launch();
  SDTFE_CUDA(cudaGetLastError());
  SDTFE_CUDA(cudaEventRecord(m.ev1, s));
  m.timed = true;
  return DTFE_OK;
}

}  // namespace sdtfe
