// capi.cu - the C ABI: the dtfe_mesh_* handle API of sdtfe_b200.h and, on
// top of it, the reference's dtfe.h / triangulate.h entry points.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <new>
#include <vector>

#include "dtfe.h"
#include "mesh.h"
#include "triangulate.h"

namespace sdtfe {

static thread_local char t_err[512] = "";

dtfe_status_t set_error(dtfe_status_t s, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
  return s;
}

static std::atomic<unsigned long long> g_launches{0};

void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace sdtfe

namespace sdtfe {

dtfe_status_t check_params(const Mesh& m, const dtfe_map_params_t* p) {
  if (!p) return set_error(DTFE_ERR_INVALID, "params is NULL");
  if (p->grid_dim < 1) return set_error(DTFE_ERR_INVALID, "grid_dim %d < 1", p->grid_dim);
  if ((long long)p->grid_dim * p->grid_dim > (1LL << 31))
    return set_error(DTFE_ERR_UNSUPPORTED, "grid_dim %d: more than 2^31 pixels", p->grid_dim);
  if (p->n_samples < 1 || p->n_samples > 16384)
    return set_error(DTFE_ERR_UNSUPPORTED, "n_samples %d not in 1..16384", p->n_samples);
  if (!(p->box_len > 0) || !(p->box_len_z > 0))
    return set_error(DTFE_ERR_INVALID, "box_len and box_len_z must be > 0");
  if (p->axis < 0 || p->axis > 2) return set_error(DTFE_ERR_INVALID, "axis %d not in 0..2", p->axis);
  if (p->precision != DTFE_FP64 && p->precision != DTFE_MIXED)
    return set_error(DTFE_ERR_INVALID, "precision %d unknown", p->precision);
  if (p->precision == DTFE_FP64 && (m.flags & DTFE_MESH_NO_FP64_REC))
    return set_error(DTFE_ERR_INVALID, "FP64 map on a mesh built with DTFE_MESH_NO_FP64_REC");
  if (!m.has_density) return set_error(DTFE_ERR_INVALID, "mesh has no density");
  return DTFE_OK;
}

// records + hull for the map's axis and precision, on the mesh stream
dtfe_status_t prepare_axis(Mesh& m, int axis, int precision) {
  if (!m.grad) SDTFE_TRY(mesh_gradients(&m));
  // the mixed walk reads FP64 records only when the coordinates are not floats
  const bool want64 = precision == DTFE_FP64 ||
                      (!m.fp32_exact && !(m.flags & DTFE_MESH_NO_FP64_REC));
  const bool want32 = precision == DTFE_MIXED;
  SDTFE_TRY(mesh_records(&m, axis, want64, want32));
  SDTFE_TRY(mesh_hull(&m, axis, nullptr, nullptr));
  return DTFE_OK;
}

}  // namespace sdtfe

using namespace sdtfe;

namespace {

int g_default_precision = -1;  // -1: read SDTFE_PRECISION once
uint64_t g_seed = 0;
dtfe_triangulator_fn g_tri_fn = nullptr;
void* g_tri_user = nullptr;

dtfe_status_t launch_map(Mesh& m, const dtfe_map_params_t* p, double* d_map, cudaStream_t s,
                         double* rr = nullptr, int* rc = nullptr, int* rs = nullptr) {
  const MapGeom g = map_geometry(m, *p);
  if (p->precision == DTFE_MIXED) return launch_map32(m, g, d_map, s, rr, rc, rs);
  return launch_map64(m, g, d_map, s, rr, rc, rs);
}

dtfe_status_t read_stats(Mesh& m, dtfe_map_stats_t* st) {
  unsigned long long c[kStatCount];
  SDTFE_CUDA(cudaMemcpy(c, m.stats, sizeof(c), cudaMemcpyDeviceToHost));
  memset(st, 0, sizeof(*st));
  st->rays = c[kStatRays];
  st->visits = c[kStatVisits];
  for (int k = 0; k < DTFE_N_RAY_STATUS; ++k) st->status[k] = c[kStatStatus0 + k];
  st->fp64_fallbacks = c[kStatFallback];
  float ms = 0.f;
  if (m.timed) SDTFE_CUDA(cudaEventElapsedTime(&ms, m.ev0, m.ev1));
  st->walk_ms = ms;
  return DTFE_OK;
}

uint64_t call_seed() {
  if (g_seed) return g_seed;
  // one draw from the C library stream keys this call's samples
  return ((uint64_t)(unsigned)rand() << 1) ^ 0x5bd1e995ULL;
}

void report(const char* fn) { fprintf(stderr, "sdtfe_b200: %s failed: %s\n", fn, dtfe_last_error()); }

}  // namespace

extern "C" {

const char* dtfe_last_error(void) { return t_err; }

void dtfe_clear_error(void) { t_err[0] = '\0'; }

const char* dtfe_status_string(dtfe_status_t s) {
  switch (s) {
    case DTFE_OK: return "ok";
    case DTFE_ERR_INVALID: return "invalid argument";
    case DTFE_ERR_CUDA: return "CUDA error";
    case DTFE_ERR_NOMEM: return "out of device memory";
    case DTFE_ERR_MESH: return "inconsistent mesh";
    case DTFE_ERR_UNSUPPORTED: return "unsupported";
    case DTFE_ERR_NO_TRIANGULATOR: return "no triangulator registered";
    case DTFE_ERR_ADMISSION: return "admission refused";
    case DTFE_ERR_TIMEOUT: return "timed out";
  }
  return "unknown";
}

void dtfe_set_default_precision(int precision) { g_default_precision = precision; }

int dtfe_get_default_precision(void) {
  if (g_default_precision < 0) {
    const char* e = getenv("SDTFE_PRECISION");
    g_default_precision = (e && (!strcmp(e, "mixed") || !strcmp(e, "1"))) ? DTFE_MIXED : DTFE_FP64;
  }
  return g_default_precision;
}

void dtfe_set_seed(uint64_t seed) { g_seed = seed; }

unsigned long long dtfe_kernel_launches(void) { return g_launches.load(); }

void dtfe_set_triangulator(dtfe_triangulator_fn fn, void* user) {
  g_tri_fn = fn;
  g_tri_user = user;
}

dtfe_status_t dtfe_mesh_create(const double* particle_data, int n_particles, const int* tetra_data,
                               int n_tetra, float p_mass, unsigned flags, dtfe_mesh_t* out) {
  if (!out) return set_error(DTFE_ERR_INVALID, "out is NULL");
  *out = nullptr;
  auto* h = new (std::nothrow) dtfe_mesh_s();
  if (!h) return set_error(DTFE_ERR_NOMEM, "host allocation failed");
  Mesh& m = h->m;
  dtfe_status_t s = mesh_upload(&m, particle_data, n_particles, tetra_data, n_tetra, p_mass, flags);
  if (s == DTFE_OK && !(flags & DTFE_MESH_FIELD)) s = mesh_density(&m);
  if (s == DTFE_OK) s = mesh_gradients(&m);
  if (s == DTFE_OK && !(flags & DTFE_MESH_LAZY)) {
    // the z-axis records and hull for the precision maps use by default
    const int prec = (flags & DTFE_MESH_NO_FP64_REC) ? DTFE_MIXED : dtfe_get_default_precision();
    s = prepare_axis(m, DTFE_AXIS_Z, prec);
  }
  if (s == DTFE_OK) {
    cudaError_t e = cudaStreamSynchronize(m.stream);
    if (e != cudaSuccess) s = set_error(DTFE_ERR_CUDA, "mesh build: %s", cudaGetErrorString(e));
  }
  if (s != DTFE_OK) {
    mesh_free(&m);
    delete h;
    return s;
  }
  *out = h;
  return DTFE_OK;
}

dtfe_status_t dtfe_mesh_destroy(dtfe_mesh_t h) {
  if (!h) return DTFE_OK;
  mesh_free(&h->m);
  delete h;
  return DTFE_OK;
}

dtfe_status_t dtfe_mesh_info(dtfe_mesh_t h, dtfe_mesh_info_t* info) {
  if (!h || !info) return set_error(DTFE_ERR_INVALID, "NULL argument");
  info->n_particles = h->m.n;
  info->n_tetra = h->m.nt;
  for (int a = 0; a < 3; ++a) info->n_hull_tri[a] = h->m.ax[a].hull_built ? h->m.ax[a].n_tri : -1;
  info->device_bytes = h->m.bytes;
  info->fp32_exact = h->m.fp32_exact ? 1 : 0;
  info->map_variant = h->m.tune32;
  return DTFE_OK;
}

dtfe_status_t dtfe_mesh_sync(dtfe_mesh_t h) {
  if (!h) return set_error(DTFE_ERR_INVALID, "NULL mesh");
  SDTFE_CUDA(cudaStreamSynchronize(h->m.stream));
  return DTFE_OK;
}

dtfe_status_t dtfe_mesh_density(dtfe_mesh_t h, double* rho) {
  if (!h || (!rho && h->m.n)) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  if (!m.n) return DTFE_OK;
  SDTFE_CUDA(cudaStreamSynchronize(m.stream));
  SDTFE_CUDA(cudaMemcpy2D(rho, sizeof(double), reinterpret_cast<const char*>(m.pos) + 3 * sizeof(double),
                          sizeof(double4), sizeof(double), m.n, cudaMemcpyDeviceToHost));
  return DTFE_OK;
}

dtfe_status_t dtfe_mesh_gradients(dtfe_mesh_t h, double* grad) {
  if (!h || (!grad && h->m.nt)) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  if (!m.grad) SDTFE_TRY(mesh_gradients(&m));
  SDTFE_CUDA(cudaStreamSynchronize(m.stream));
  if (m.nt) SDTFE_CUDA(cudaMemcpy(grad, m.grad, sizeof(double) * 3 * (size_t)m.nt, cudaMemcpyDeviceToHost));
  return DTFE_OK;
}

dtfe_status_t dtfe_mesh_adjacency(dtfe_mesh_t h, int* counts) {
  if (!h || (!counts && h->m.n)) return set_error(DTFE_ERR_INVALID, "NULL argument");
  if (!h->m.adj) return set_error(DTFE_ERR_INVALID, "mesh built with DTFE_MESH_FIELD has no adjacency counts");
  SDTFE_CUDA(cudaStreamSynchronize(h->m.stream));
  if (h->m.n) SDTFE_CUDA(cudaMemcpy(counts, h->m.adj, sizeof(int) * h->m.n, cudaMemcpyDeviceToHost));
  return DTFE_OK;
}

dtfe_status_t dtfe_mesh_hull(dtfe_mesh_t h, int axis, int* tri, int* n_tri) {
  if (!h || !n_tri) return set_error(DTFE_ERR_INVALID, "NULL argument");
  if (axis < 0 || axis > 2) return set_error(DTFE_ERR_INVALID, "axis %d not in 0..2", axis);
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  SDTFE_TRY(mesh_hull(&m, axis, nullptr, nullptr));
  SDTFE_CUDA(cudaStreamSynchronize(m.stream));
  *n_tri = m.ax[axis].n_tri;
  if (tri && m.ax[axis].n_tri)
    SDTFE_CUDA(cudaMemcpy(tri, m.ax[axis].tri_rows, sizeof(int) * 8 * (size_t)m.ax[axis].n_tri,
                          cudaMemcpyDeviceToHost));
  return DTFE_OK;
}

dtfe_status_t dtfe_map_device(dtfe_mesh_t h, const dtfe_map_params_t* p, double* d_map,
                              void* stream) {
  if (!h || !d_map) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  SDTFE_TRY(check_params(m, p));
  const AxisData& A = m.ax[p->axis];
  const bool ready = A.hull_built && (p->precision == DTFE_FP64 ? A.rec64 != nullptr
                                                                 : A.rot32 != nullptr &&
                                                                       (m.fp32_exact || A.rec64));
  cudaStream_t s = stream ? (cudaStream_t)stream : m.stream;
  if (!ready) {
    SDTFE_TRY(prepare_axis(m, p->axis, p->precision));
    if (s != m.stream) SDTFE_CUDA(cudaStreamSynchronize(m.stream));
  }
  return launch_map(m, p, d_map, s);
}

dtfe_status_t dtfe_trim_memory(void) {
  SDTFE_CUDA(cudaDeviceSynchronize());  // frees still in flight on any mesh stream
  mesh_trim_record_pool();
  return DTFE_OK;
}

int dtfe_num_variants(void) { return num_map32_variants(); }

dtfe_status_t dtfe_set_variant(dtfe_mesh_t h, int variant) {
  if (!h) return set_error(DTFE_ERR_INVALID, "NULL mesh");
  if (variant < -1 || variant >= num_map32_variants())
    return set_error(DTFE_ERR_INVALID, "variant %d not in -1..%d", variant, num_map32_variants() - 1);
  std::lock_guard<std::mutex> lk(h->mu);
  h->m.tune32 = variant;
  return DTFE_OK;
}

dtfe_status_t dtfe_set_location(dtfe_mesh_t h, int mode) {
  if (!h) return set_error(DTFE_ERR_INVALID, "NULL mesh");
  if (mode != DTFE_LOCATE_PER_RAY && mode != DTFE_LOCATE_TILE)
    return set_error(DTFE_ERR_INVALID, "location mode %d not 0 (per ray) or 1 (tile)", mode);
  std::lock_guard<std::mutex> lk(h->mu);
  h->m.fp64_location = mode;
  return DTFE_OK;
}

dtfe_status_t dtfe_autotune(dtfe_mesh_t h, const dtfe_map_params_t* p, int* best,
                            dtfe_variant_t* timings) {
  if (!h || !p) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  SDTFE_TRY(check_params(m, p));
  dtfe_map_params_t q = *p;
  q.precision = DTFE_MIXED;
  // central window: a quarter of the side, at the same pixel size
  q.grid_dim = p->grid_dim >= 128 ? p->grid_dim / 4 : p->grid_dim;
  q.box_len = p->box_len * q.grid_dim / p->grid_dim;
  SDTFE_TRY(prepare_axis(m, q.axis, q.precision));
  cudaStream_t s = m.stream;
  double* d_map = nullptr;
  const size_t bytes = sizeof(double) * (size_t)q.grid_dim * q.grid_dim;
  SDTFE_CUDA(cudaMallocAsync(&d_map, bytes, s));
  const int nv = num_map32_variants();
  int best_v = -1;
  float best_ms = 0.f;
  dtfe_status_t st = DTFE_OK;
  for (int v = 0; v < nv && st == DTFE_OK; ++v) {
    m.tune32 = v;
    float ms_v = 0.f;
    for (int rep = 0; rep < 3 && st == DTFE_OK; ++rep) {  // first run warms the caches
      st = launch_map(m, &q, d_map, s);
      if (st != DTFE_OK) break;
      cudaError_t e = cudaEventSynchronize(m.ev1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, m.ev0, m.ev1);
      if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
      if (rep == 1 || (rep == 2 && ms < ms_v)) ms_v = ms;
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
  cudaFreeAsync(d_map, s);
  m.tune32 = best_v;
  if (best) *best = best_v;
  return st;
}

dtfe_status_t dtfe_mesh_last_stats(dtfe_mesh_t h, dtfe_map_stats_t* st) {
  if (!h || !st) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  SDTFE_CUDA(cudaDeviceSynchronize());
  return read_stats(h->m, st);
}

extern "C++" {
namespace {

// A map into a host array, accumulated into as the reference does: the array
// is uploaded, the walk enqueued, while_walking() run on the host while the
// walk runs, and the array downloaded.  With the handle's lock held.
template <class F>
dtfe_status_t map_to_host(Mesh& m, const dtfe_map_params_t* p, double* map, F&& while_walking) {
  SDTFE_TRY(check_params(m, p));
  SDTFE_TRY(prepare_axis(m, p->axis, p->precision));
  cudaStream_t s = m.stream;
  const size_t bytes = sizeof(double) * (size_t)p->grid_dim * p->grid_dim;
  double* d_map = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&d_map, bytes, s));
  cudaError_t e = cudaMemcpyAsync(d_map, map, bytes, cudaMemcpyHostToDevice, s);
  dtfe_status_t st = e == cudaSuccess ? launch_map(m, p, d_map, s)
                                      : set_error(DTFE_ERR_CUDA, "map: %s", cudaGetErrorString(e));
  if (st == DTFE_OK) st = while_walking();
  if (st == DTFE_OK) {
    e = cudaMemcpyAsync(map, d_map, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "map: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(d_map, s);
  return st;
}

dtfe_status_t nothing_else() { return DTFE_OK; }

// Column 3 of the caller's particle array receives the densities, as
// pre_compute_vol does (src/triangulate.c:183-225).  The device's rows
// (x, y, z, rho) are the caller's rows with column 3 replaced, so they are
// copied back whole, on a stream of their own, while the walk enqueued before
// runs.  Returns when the copy is done.
dtfe_status_t copy_back_densities(Mesh& m, double* particle_data) {
  if (m.n == 0) return DTFE_OK;
  cudaStream_t side = nullptr;
  SDTFE_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  cudaError_t e = cudaMemcpyAsync(particle_data, m.pos, sizeof(double4) * (size_t)m.n,
                                  cudaMemcpyDeviceToHost, side);
  if (e == cudaSuccess) e = cudaStreamSynchronize(side);
  cudaStreamDestroy(side);
  SDTFE_CUDA(e);
  return DTFE_OK;
}

}  // namespace
}  // extern "C++"

dtfe_status_t dtfe_map(dtfe_mesh_t h, const dtfe_map_params_t* p, double* map,
                       dtfe_map_stats_t* stats) {
  if (!h || !map) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  dtfe_status_t st = map_to_host(m, p, map, nothing_else);
  if (st == DTFE_OK && stats) st = read_stats(m, stats);
  return st;
}

dtfe_status_t dtfe_map_rays(dtfe_mesh_t h, const dtfe_map_params_t* p, double* map,
                            double* ray_rho, int* ray_crossed, int* ray_status,
                            dtfe_map_stats_t* stats) {
  if (!h || !map || !ray_rho || !ray_crossed || !ray_status)
    return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  SDTFE_TRY(check_params(m, p));
  const size_t n_rays = (size_t)p->grid_dim * p->grid_dim * p->n_samples;
  if (n_rays > (size_t)1 << 31)
    return set_error(DTFE_ERR_UNSUPPORTED, "dtfe_map_rays: %zu rays (at most 2^31)", n_rays);
  SDTFE_TRY(prepare_axis(m, p->axis, p->precision));
  cudaStream_t s = m.stream;
  const size_t bytes = sizeof(double) * (size_t)p->grid_dim * p->grid_dim;
  void* d[4] = {nullptr, nullptr, nullptr, nullptr};  // map, rho, crossed, status
  const size_t sz[4] = {bytes, sizeof(double) * n_rays, sizeof(int) * n_rays, sizeof(int) * n_rays};
  void* host[4] = {map, ray_rho, ray_crossed, ray_status};
  dtfe_status_t st = DTFE_OK;
  for (int k = 0; k < 4 && st == DTFE_OK; ++k) {
    const cudaError_t e = cudaMallocAsync(&d[k], sz[k], s);
    if (e != cudaSuccess)
      st = set_error(e == cudaErrorMemoryAllocation ? DTFE_ERR_NOMEM : DTFE_ERR_CUDA,
                     "map_rays: %s", cudaGetErrorString(e));
  }
  if (st == DTFE_OK) {
    const cudaError_t e = cudaMemcpyAsync(d[0], map, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "map_rays: %s", cudaGetErrorString(e));
  }
  if (st == DTFE_OK)
    st = launch_map(m, p, static_cast<double*>(d[0]), s, static_cast<double*>(d[1]),
                    static_cast<int*>(d[2]), static_cast<int*>(d[3]));
  for (int k = 0; k < 4 && st == DTFE_OK; ++k) {
    const cudaError_t e = cudaMemcpyAsync(host[k], d[k], sz[k], cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "map_rays: %s", cudaGetErrorString(e));
  }
  if (st == DTFE_OK) {
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "map_rays: %s", cudaGetErrorString(e));
  }
  for (int k = 0; k < 4; ++k)
    if (d[k]) cudaFreeAsync(d[k], s);
  if (st == DTFE_OK && stats) st = read_stats(m, stats);
  return st;
}

dtfe_status_t dtfe_trace(dtfe_mesh_t h, const dtfe_map_params_t* p, int n_rays, const double* x,
                         const double* y, double z0, double lz, double delta_xy, double* rho,
                         int* crossed, int* status, int* visits, int max_record) {
  if (!h || !p || n_rays < 0 || (n_rays && (!x || !y || !rho || !crossed || !status)))
    return set_error(DTFE_ERR_INVALID, "NULL argument");
  if (visits && max_record < 1) return set_error(DTFE_ERR_INVALID, "max_record < 1");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  if (p->axis < 0 || p->axis > 2) return set_error(DTFE_ERR_INVALID, "axis %d not in 0..2", p->axis);
  SDTFE_TRY(prepare_axis(m, p->axis, p->precision));
  if (!n_rays) return DTFE_OK;
  cudaStream_t s = m.stream;
  const long long mv = p->max_visits > 0 ? p->max_visits : 2LL * m.nt + 64;
  const int max_visits = (int)(mv > 0x7fffffff ? 0x7fffffff : mv);
  double *dx, *dy, *dr;
  int *dc, *ds, *dv = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&dx, sizeof(double) * n_rays, s));
  SDTFE_CUDA(cudaMallocAsync(&dy, sizeof(double) * n_rays, s));
  SDTFE_CUDA(cudaMallocAsync(&dr, sizeof(double) * n_rays, s));
  SDTFE_CUDA(cudaMallocAsync(&dc, sizeof(int) * n_rays, s));
  SDTFE_CUDA(cudaMallocAsync(&ds, sizeof(int) * n_rays, s));
  const size_t vbytes = visits ? sizeof(int) * (size_t)n_rays * max_record : 0;
  if (visits) {
    SDTFE_CUDA(cudaMallocAsync(&dv, vbytes, s));
    SDTFE_CUDA(cudaMemsetAsync(dv, 0xff, vbytes, s));
  }
  SDTFE_CUDA(cudaMemcpyAsync(dx, x, sizeof(double) * n_rays, cudaMemcpyHostToDevice, s));
  SDTFE_CUDA(cudaMemcpyAsync(dy, y, sizeof(double) * n_rays, cudaMemcpyHostToDevice, s));
  dtfe_status_t st =
      p->precision == DTFE_MIXED
          ? launch_trace32(m, p->axis, n_rays, dx, dy, z0, lz, delta_xy, p->seed, max_visits, dr, dc, ds, dv,
                           max_record, s)
          : launch_trace64(m, p->axis, n_rays, dx, dy, z0, lz, delta_xy, p->seed, max_visits, dr, dc, ds, dv,
                           max_record, s);
  if (st == DTFE_OK) {
    cudaError_t e = cudaMemcpyAsync(rho, dr, sizeof(double) * n_rays, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(crossed, dc, sizeof(int) * n_rays, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, ds, sizeof(int) * n_rays, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && visits) e = cudaMemcpyAsync(visits, dv, vbytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "trace: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(dx, s);
  cudaFreeAsync(dy, s);
  cudaFreeAsync(dr, s);
  cudaFreeAsync(dc, s);
  cudaFreeAsync(ds, s);
  if (dv) cudaFreeAsync(dv, s);
  return st;
}

namespace {

dtfe_status_t check_grid(dtfe_mesh_t h, int G, double box_len, const double* center, unsigned ss,
                         int precision) {
  if (!h || !center) return set_error(DTFE_ERR_INVALID, "NULL argument");
  if (G < 1 || ss < 1) return set_error(DTFE_ERR_INVALID, "grid_dim and supersampling must be >= 1");
  if (!(box_len > 0)) return set_error(DTFE_ERR_INVALID, "box_len must be > 0");
  if ((double)G * G * G * sizeof(double) > 1e12)
    return set_error(DTFE_ERR_UNSUPPORTED, "grid_dim %d: grid larger than 1 TB", G);
  if (precision != DTFE_FP64 && precision != DTFE_MIXED)
    return set_error(DTFE_ERR_INVALID, "precision %d unknown", precision);
  if (precision == DTFE_FP64 && (h->m.flags & DTFE_MESH_NO_FP64_REC))
    return set_error(DTFE_ERR_INVALID, "FP64 grid on a mesh built with DTFE_MESH_NO_FP64_REC");
  return DTFE_OK;
}

// with h->mu held
dtfe_status_t launch_grid(Mesh& m, int G, double box_len, const double center[3], unsigned ss,
                          uint64_t seed, int precision, double* d, cudaStream_t s) {
  if (!m.has_density) return set_error(DTFE_ERR_INVALID, "mesh has no density");
  SDTFE_TRY(prepare_axis(m, DTFE_AXIS_Z, precision));
  if (precision == DTFE_MIXED) SDTFE_TRY(mesh_field64(&m));
  if (s != m.stream) SDTFE_CUDA(cudaStreamSynchronize(m.stream));  // records are built there
  const int max_visits = (int)((2LL * m.nt + 64) > 0x7fffffff ? 0x7fffffff : (2LL * m.nt + 64));
  if (precision == DTFE_MIXED) return launch_grid32(m, G, box_len, center, ss, seed, max_visits, d, s);
  return launch_grid64(m, G, box_len, center, ss, seed, max_visits, d, s);
}

}  // namespace

extern "C++" {
// The grid into a host array, accumulated into (src/dtfe.c:505-511), with
// while_walking() run on the host while the walk runs; as map_to_host.
template <class F>
dtfe_status_t grid_to_host(Mesh& m, int G, double box_len, const double center[3], unsigned ss,
                           uint64_t seed, int precision, double* grid, F&& while_walking) {
  cudaStream_t s = m.stream;
  const size_t bytes = sizeof(double) * (size_t)G * G * G;
  double* d = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&d, bytes, s));
  cudaError_t e = cudaMemcpyAsync(d, grid, bytes, cudaMemcpyHostToDevice, s);
  dtfe_status_t st = e == cudaSuccess ? launch_grid(m, G, box_len, center, ss, seed, precision, d, s)
                                      : set_error(DTFE_ERR_CUDA, "grid: %s", cudaGetErrorString(e));
  if (st == DTFE_OK) st = while_walking();
  if (st == DTFE_OK) {
    e = cudaMemcpyAsync(grid, d, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = set_error(DTFE_ERR_CUDA, "grid: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(d, s);
  return st;
}
}  // extern "C++"

dtfe_status_t dtfe_grid_ex(dtfe_mesh_t h, int G, double box_len, const double center[3],
                           unsigned ss, uint64_t seed, int precision, double* grid) {
  SDTFE_TRY(check_grid(h, G, box_len, center, ss, precision));
  if (!grid) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  return grid_to_host(h->m, G, box_len, center, ss, seed, precision, grid, nothing_else);
}

dtfe_status_t dtfe_grid(dtfe_mesh_t h, int G, double box_len, const double center[3],
                        unsigned ss, uint64_t seed, double* grid) {
  return dtfe_grid_ex(h, G, box_len, center, ss, seed, DTFE_FP64, grid);
}

dtfe_status_t dtfe_grid_device(dtfe_mesh_t h, int G, double box_len, const double center[3],
                               unsigned ss, uint64_t seed, int precision, double* d_grid,
                               void* stream) {
  SDTFE_TRY(check_grid(h, G, box_len, center, ss, precision));
  if (!d_grid) return set_error(DTFE_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(h->mu);
  Mesh& m = h->m;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : m.stream;
  return launch_grid(m, G, box_len, center, ss, seed, precision, d_grid, s);
}

// ---------------------------------------------------------------------------
// Drop-ins for src/dtfe.h and src/triangulate.h.

void compute_density(double* particle_data, int n_particles, int* tetra_data, int n_tetra,
                     int grid_dim, double box_len, double box_len_z, double* rho, float p_mass,
                     double center_x, double center_y, double center_z, const int n_mc_samp,
                     const double delta_sample) {
  dtfe_mesh_t h = nullptr;
  if (dtfe_mesh_create(particle_data, n_particles, tetra_data, n_tetra, p_mass, 0, &h) != DTFE_OK)
    return report("compute_density");
  dtfe_map_params_t p;
  memset(&p, 0, sizeof(p));
  p.grid_dim = grid_dim;
  p.box_len = box_len;
  p.box_len_z = box_len_z;
  p.center[0] = center_x;
  p.center[1] = center_y;
  p.center[2] = center_z;
  p.n_samples = n_mc_samp;
  p.delta_sample = delta_sample;
  p.seed = call_seed();
  p.axis = DTFE_AXIS_Z;
  p.precision = dtfe_get_default_precision();
  dtfe_status_t s;
  {
    std::lock_guard<std::mutex> lk(h->mu);
    s = map_to_host(h->m, &p, rho, [&] { return copy_back_densities(h->m, particle_data); });
  }
  if (s != DTFE_OK) report("compute_density");
  dtfe_mesh_destroy(h);
}

void interpolate_to_3d_grid(double* particle_data, int n_particles, int* tetra_data, int n_tetra,
                            int grid_dim, double box_len, double* grid, double center_x,
                            double center_y, double center_z, unsigned supersampling) {
  dtfe_mesh_t h = nullptr;
  if (dtfe_mesh_create(particle_data, n_particles, tetra_data, n_tetra, 0.f, DTFE_MESH_FIELD, &h) !=
      DTFE_OK)
    return report("interpolate_to_3d_grid");
  const double c[3] = {center_x, center_y, center_z};
  if (dtfe_grid_ex(h, grid_dim, box_len, c, supersampling, call_seed(),
                   dtfe_get_default_precision(), grid) != DTFE_OK)
    report("interpolate_to_3d_grid");
  dtfe_mesh_destroy(h);
}

void compute_3d_density(double* particle_data, int n_particles, int* tetra_data, int n_tetra,
                        int grid_dim, double box_len, double* rho, float p_mass, double center_x,
                        double center_y, double center_z, unsigned supersampling) {
  dtfe_mesh_t h = nullptr;
  if (dtfe_mesh_create(particle_data, n_particles, tetra_data, n_tetra, p_mass, 0, &h) != DTFE_OK)
    return report("compute_3d_density");
  const double c[3] = {center_x, center_y, center_z};
  const int precision = dtfe_get_default_precision();
  dtfe_status_t s = check_grid(h, grid_dim, box_len, c, supersampling, precision);
  if (s == DTFE_OK) {
    std::lock_guard<std::mutex> lk(h->mu);
    s = grid_to_host(h->m, grid_dim, box_len, c, supersampling, call_seed(), precision, rho,
                     [&] { return copy_back_densities(h->m, particle_data); });
  }
  if (s != DTFE_OK) report("compute_3d_density");
  dtfe_mesh_destroy(h);
}

// Density only: upload, volumes, CSR, densities, download into column 3.
void pre_compute_vol(double** particle_data, int n_particles, int* tetra_data, int n_tetra,
                     float p_mass) {
  if (!particle_data) return;
  Mesh m;
  dtfe_status_t s = mesh_upload(&m, *particle_data, n_particles, tetra_data, n_tetra, p_mass, 0);
  if (s == DTFE_OK) s = mesh_density(&m);
  if (s == DTFE_OK && n_particles) {
    cudaError_t e = cudaMemcpy2DAsync(*particle_data + 3, sizeof(double4),
                                      reinterpret_cast<const char*>(m.pos) + 3 * sizeof(double),
                                      sizeof(double4), sizeof(double), n_particles,
                                      cudaMemcpyDeviceToHost, m.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
    if (e != cudaSuccess) s = set_error(DTFE_ERR_CUDA, "pre_compute_vol: %s", cudaGetErrorString(e));
  }
  if (s != DTFE_OK) report("pre_compute_vol");
  mesh_free(&m);
}

// Gradients from the densities already in column 3 (the reference reads them
// from particle_data the same way).
double* gradients(int* tetra_data, int n_tetra, double* particle_data) {
  double* out = (double*)malloc(sizeof(double) * 3 * (size_t)(n_tetra > 0 ? n_tetra : 1));
  if (!out) return nullptr;
  // the reference signature carries no particle count: use the largest vertex id
  int n = 0;
  for (int t = 0; t < n_tetra; ++t)
    for (int k = 0; k < 4; ++k)
      if (tetra_data[8 * (size_t)t + k] + 1 > n) n = tetra_data[8 * (size_t)t + k] + 1;
  Mesh m;
  dtfe_status_t s = mesh_upload(&m, particle_data, n, tetra_data, n_tetra, 0.f, DTFE_MESH_FIELD);
  if (s == DTFE_OK) s = mesh_gradients(&m);
  if (s == DTFE_OK && n_tetra) {
    cudaError_t e = cudaMemcpyAsync(out, m.grad, sizeof(double) * 3 * (size_t)n_tetra,
                                    cudaMemcpyDeviceToHost, m.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
    if (e != cudaSuccess) s = set_error(DTFE_ERR_CUDA, "gradients: %s", cudaGetErrorString(e));
  }
  mesh_free(&m);
  if (s != DTFE_OK) {
    report("gradients");
    free(out);
    return nullptr;
  }
  return out;
}

int find_forward_hull(int* tetra_data, int n_tetra, double* particle_data, int n_particles,
                      word_t* bitmap) {
  Mesh m;
  int count = 0;
  std::vector<uint32_t> mask(n_tetra > 0 ? n_tetra : 0);
  dtfe_status_t s = mesh_upload(&m, particle_data, n_particles, tetra_data, n_tetra, 0.f,
                                DTFE_MESH_FIELD);
  if (s == DTFE_OK) s = mesh_hull_mask(&m, DTFE_AXIS_Z, mask.data(), &count);
  mesh_free(&m);
  if (s != DTFE_OK) {
    report("find_forward_hull");
    return 0;
  }
  for (int t = 0; t < n_tetra; ++t) bitmap[t] |= mask[t] & 0xFu;  // word t holds tet t's faces
  return count;
}

int* copy_fh_triangles(int* tetra_data, int n_tetra, double* particle_data, int n_particles,
                       int n_tri, word_t* bitmap) {
  int* out = (int*)malloc(sizeof(int) * 8 * (size_t)(n_tri > 0 ? n_tri : 1));
  if (!out) return nullptr;
  Mesh m;
  int count = 0;
  dtfe_status_t s = mesh_upload(&m, particle_data, n_particles, tetra_data, n_tetra, 0.f,
                                DTFE_MESH_FIELD);
  if (s == DTFE_OK) s = mesh_hull(&m, DTFE_AXIS_Z, bitmap, &count);
  if (s == DTFE_OK && count != n_tri)
    s = set_error(DTFE_ERR_INVALID, "bitmap holds %d faces, n_tri is %d", count, n_tri);
  if (s == DTFE_OK && count) {
    cudaError_t e = cudaMemcpyAsync(out, m.ax[0].tri_rows, sizeof(int) * 8 * (size_t)count,
                                    cudaMemcpyDeviceToHost, m.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m.stream);
    if (e != cudaSuccess) s = set_error(DTFE_ERR_CUDA, "copy_fh_triangles: %s", cudaGetErrorString(e));
  }
  mesh_free(&m);
  if (s != DTFE_OK) {
    report("copy_fh_triangles");
    free(out);
    return nullptr;
  }
  return out;
}

int* triangulate(double* particle_data, int n_particles, size_t* num_facets, const char* options) {
  if (num_facets) *num_facets = 0;
  size_t cached_nt = 0;
  if (particle_data && n_particles > 0) {
    if (int* hit = tri_cache_lookup(particle_data, n_particles, options, &cached_nt)) {
      if (num_facets) *num_facets = cached_nt;
      return hit;
    }
  }
  if (!g_tri_fn) {
    set_error(DTFE_ERR_NO_TRIANGULATOR, "no Qhull backend registered (dtfe_set_triangulator)");
    fprintf(stderr, "TRIANGULATION ERROR: %s\n", dtfe_last_error());
    return nullptr;
  }
  int *simp = nullptr, *nb = nullptr;
  size_t nt = 0;
  if (g_tri_fn(particle_data, n_particles, options, &simp, &nb, &nt, g_tri_user) != 0 || !simp || !nb) {
    free(simp);
    free(nb);
    set_error(DTFE_ERR_MESH, "triangulator failed");
    fprintf(stderr, "TRIANGULATION ERROR: %s\n", dtfe_last_error());
    return nullptr;
  }
  int* tetra = (int*)malloc(sizeof(int) * 8 * (nt ? nt : 1));
  if (tetra) dtfe_tetra_from_cells(particle_data, simp, nb, nt, tetra);
  free(simp);
  free(nb);
  if (tetra) tri_cache_insert(particle_data, n_particles, options, tetra, nt);
  if (tetra && num_facets) *num_facets = nt;
  return tetra;
}

}  // extern "C"
