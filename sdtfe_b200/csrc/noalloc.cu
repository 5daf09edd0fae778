// noalloc.cu - per-vertex DTFE density with no device allocation.
//
// Some callers cannot allocate device memory while they run this step, for
// example:
//   * code running inside a memory pool or arena that owns all device memory
//     (a framework allocator, a pre-sized serving process);
//   * real-time or serving loops where cudaMalloc/cudaFree, which synchronise
//     the whole device, would stall every other stream;
//   * hosts that forbid allocation after start-up.
// dtfe_density_noalloc serves them: the caller passes device inputs and a
// device output, and every temporary buffer lives in one file-scope
// __device__ array, g_density_scratch (kNoAllocScratchBytes, held on every GPU
// that loads this library until the process exits).
//
// The computation is the density build of mesh.cu: validation of the indices,
// per-tet |V| (src/triangulate.c:191-215), vertex->tet lists sorted by tet
// index, and rho = m*(1+3) / sum of adjacent volumes summed in increasing tet
// order (src/triangulate.c:216-224), so the result is bit-identical to
// dtfe_mesh_density and to the reference's pre_compute_vol.  Compiled with
// -fmad=false for the same reason as mesh.cu.
//
// Host code never touches g_density_scratch directly: its name is a host-side
// stand-in, not a device address.  The first call on each device sets the
// array up: it looks up the array's device address with cudaGetSymbolAddress
// (with that device current) and caches it.  With CUDA's lazy module loading
// that first call is also when the 48 MiB are reserved on the device, so a
// caller makes one call per device at start-up (n_particles == 0 does only the
// set-up), before its memory pool takes the device's memory and before any
// stream capture.  Each call waits on its stream twice (for the validation
// flag, and for its own work before it returns): it blocks the calling thread.
#include <cub/device/device_scan.cuh>

#include <cstring>
#include <mutex>

#include "mesh.h"

namespace sdtfe {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(48) << 20;  // 48 MiB
constexpr int kMaxDevices = 64;
constexpr int kBlk = 256;

__device__ __align__(256) unsigned char g_density_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

inline unsigned blocks_for(long long n) { return (unsigned)((n + kBlk - 1) / kBlk > 0 ? (n + kBlk - 1) / kBlk : 1); }

__global__ void k_na_validate(const int4* __restrict__ rows, int nt, int n, int* __restrict__ err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  if ((unsigned)v.x >= (unsigned)n || (unsigned)v.y >= (unsigned)n || (unsigned)v.z >= (unsigned)n ||
      (unsigned)v.w >= (unsigned)n)
    atomicOr(err, 1);
}

__global__ void k_na_volume_count(const double4* __restrict__ pos, const int4* __restrict__ rows,
                                  int nt, double* __restrict__ vol, int* __restrict__ cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  const double4 a = pos[v.x], b = pos[v.y], c = pos[v.z], d = pos[v.w];
  const double r0 = (a.x - d.x) * ((b.y - d.y) * (c.z - d.z) - (b.z - d.z) * (c.y - d.y));
  const double r1 = (a.y - d.y) * ((b.z - d.z) * (c.x - d.x) - (b.x - d.x) * (c.z - d.z));
  const double r2 = (a.z - d.z) * ((b.x - d.x) * (c.y - d.y) - (b.y - d.y) * (c.x - d.x));
  vol[t] = fabs((r0 + r1 + r2) / 6);
  atomicAdd(cnt + v.x, 1);
  atomicAdd(cnt + v.y, 1);
  atomicAdd(cnt + v.z, 1);
  atomicAdd(cnt + v.w, 1);
}

__global__ void k_na_fill(const int4* __restrict__ rows, int nt, const int* __restrict__ off,
                          int* __restrict__ cursor, int* __restrict__ idx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  idx[off[v.x] + atomicAdd(cursor + v.x, 1)] = t;
  idx[off[v.y] + atomicAdd(cursor + v.y, 1)] = t;
  idx[off[v.z] + atomicAdd(cursor + v.z, 1)] = t;
  idx[off[v.w] + atomicAdd(cursor + v.w, 1)] = t;
}

// sort each vertex's tets by index, then sum their volumes in that order
__global__ void k_na_density(const int* __restrict__ off, int* __restrict__ idx,
                             const double* __restrict__ vol, int n, double m4,
                             double* __restrict__ rho) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int b = off[v], e = off[v + 1];
  for (int i = b + 1; i < e; ++i) {
    const int key = idx[i];
    int j = i - 1;
    while (j >= b && idx[j] > key) {
      idx[j + 1] = idx[j];
      --j;
    }
    idx[j + 1] = key;
  }
  double s = 0;
  for (int i = b; i < e; ++i) s += vol[idx[i]];
  rho[v] = m4 / s;
}

// the scratch array's device address on the current device (looked up once)
dtfe_status_t scratch_base(unsigned char** base) {
  int dev = 0;
  SDTFE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(DTFE_ERR_UNSUPPORTED, "device %d", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    SDTFE_CUDA(cudaGetSymbolAddress(&p, g_density_scratch));
    g_scratch_ptr[dev] = p;
  }
  *base = static_cast<unsigned char*>(g_scratch_ptr[dev]);
  return DTFE_OK;
}

}  // namespace
}  // namespace sdtfe

using namespace sdtfe;

extern "C" dtfe_status_t dtfe_density_noalloc(const double* d_particle_data, int n_particles,
                                              const int* d_tetra_data, int n_tetra, float p_mass,
                                              double* d_rho, void* stream) {
  if (n_particles < 0 || n_tetra < 0) return set_error(DTFE_ERR_INVALID, "negative size");
  unsigned char* base = nullptr;
  if (n_particles == 0) return scratch_base(&base);  // set-up only (the start-up call)
  if (!d_particle_data || !d_rho || (n_tetra > 0 && !d_tetra_data))
    return set_error(DTFE_ERR_INVALID, "NULL device pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = n_particles, nt = n_tetra;
  // carve the scratch: error flag | vol | cnt (n+1) | off (n+1) | idx (4 nt) | scan temp;
  // the fixed part is checked first, in size_t, so that n + 1 below is an int
  const size_t o_vol = 256;
  const size_t o_cnt = align256(o_vol + sizeof(double) * (size_t)nt);
  const size_t o_off = align256(o_cnt + sizeof(int) * ((size_t)n + 1));
  const size_t o_idx = align256(o_off + sizeof(int) * ((size_t)n + 1));
  const size_t o_tmp = align256(o_idx + sizeof(int) * 4 * (size_t)nt);
  if (o_tmp > kNoAllocScratchBytes)
    return set_error(DTFE_ERR_UNSUPPORTED,
                     "dtfe_density_noalloc: %d particles and %d tets need over %zu bytes of "
                     "scratch; the static scratch holds %zu (about 1.9M tets)",
                     n, nt, o_tmp, kNoAllocScratchBytes);
  size_t scan_bytes = 0;
  SDTFE_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const int*)nullptr, (int*)nullptr,
                                           n + 1, s));
  const size_t need = align256(o_tmp + scan_bytes);
  if (need > kNoAllocScratchBytes)
    return set_error(DTFE_ERR_UNSUPPORTED,
                     "dtfe_density_noalloc: %d particles and %d tets need %zu bytes of scratch; "
                     "the static scratch holds %zu (about 1.9M tets)",
                     n, nt, need, kNoAllocScratchBytes);
  SDTFE_TRY(scratch_base(&base));
  int* err = reinterpret_cast<int*>(base);
  double* vol = reinterpret_cast<double*>(base + o_vol);
  int* cnt = reinterpret_cast<int*>(base + o_cnt);
  int* off = reinterpret_cast<int*>(base + o_off);
  int* idx = reinterpret_cast<int*>(base + o_idx);
  void* tmp = base + o_tmp;
  const double4* pos = reinterpret_cast<const double4*>(d_particle_data);
  const int4* rows = reinterpret_cast<const int4*>(d_tetra_data);

  // the array keeps the previous call's contents: clear what starts at zero
  SDTFE_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  SDTFE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)n + 1), s));
  if (nt) {
    k_na_validate<<<blocks_for(nt), kBlk, 0, s>>>(rows, nt, n, err);
    count_launch();
  }
  int h_err = 0;
  SDTFE_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  SDTFE_CUDA(cudaStreamSynchronize(s));
  if (h_err)
    return set_error(DTFE_ERR_MESH, "tetra_data holds a vertex id outside [0, %d)", n);
  if (nt) {
    k_na_volume_count<<<blocks_for(nt), kBlk, 0, s>>>(pos, rows, nt, vol, cnt);
    count_launch();
  }
  SDTFE_CUDA(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, cnt, off, n + 1, s));
  SDTFE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)n + 1), s));
  if (nt) {
    k_na_fill<<<blocks_for(nt), kBlk, 0, s>>>(rows, nt, off, cnt, idx);
    count_launch();
  }
  const double m4 = (double)(p_mass * 4);  // float product, as in the reference
  k_na_density<<<blocks_for(n), kBlk, 0, s>>>(off, idx, vol, n, m4, d_rho);
  count_launch();
  SDTFE_CUDA(cudaGetLastError());
  SDTFE_CUDA(cudaStreamSynchronize(s));
  return DTFE_OK;
}
