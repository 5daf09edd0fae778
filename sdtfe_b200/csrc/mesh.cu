// mesh.cu - builds the device-resident mesh: validation, per-tet volumes,
// vertex->tet CSR, DTFE densities, gradients, walk records and the projected
// forward hull with its edge adjacency.
//
// Compiled with -fmad=false: the volume, density and gradient arithmetic
// repeats the reference's FP64 operations in order (src/triangulate.c:183-316)
// and must not be contracted into fused multiply-adds.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "mesh.h"

namespace sdtfe {

namespace {

constexpr int kBlock = 256;

inline unsigned grid_for(long long n, int block = kBlock) {
  long long g = (n + block - 1) / block;
  return (unsigned)(g < 1 ? 1 : g);
}

// Every vertex id in [0, n), every neighbour id in [-1, nt).  Anything else
// would send a later gather out of bounds, so nothing runs until this passes.
__global__ void k_validate(const int4* __restrict__ rows, int nt, int n, int* __restrict__ err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  const int4 nb = rows[2 * (size_t)t + 1];
  const bool bad_v = (unsigned)v.x >= (unsigned)n || (unsigned)v.y >= (unsigned)n ||
                     (unsigned)v.z >= (unsigned)n || (unsigned)v.w >= (unsigned)n;
  auto bad_n = [nt](int k) { return k < -1 || k >= nt; };
  if (bad_v || bad_n(nb.x) || bad_n(nb.y) || bad_n(nb.z) || bad_n(nb.w)) atomicOr(err, 1);
}

// Whether every coordinate is exactly a float, and the largest coordinate
// magnitude (as float bits, rounded up; non-negative floats order as ints).
__global__ void k_fp32_exact(const double4* __restrict__ pos, int n, int* __restrict__ not_exact,
                             int* __restrict__ max_bits) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pos[i];
  if ((double)(float)p.x != p.x || (double)(float)p.y != p.y || (double)(float)p.z != p.z)
    atomicOr(not_exact, 1);
  const float mx = __double2float_ru(fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))));
  atomicMax(max_bits, __float_as_int(mx));
}

// a3 part 1: |det(A-D, B-D, C-D)|/6, the reference's expansion order
// (src/triangulate.c:191-215).
__global__ void k_volume(const double4* __restrict__ pos, const int4* __restrict__ rows, int nt,
                         double* __restrict__ vol) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  const double4 a = pos[v.x], b = pos[v.y], c = pos[v.z], d = pos[v.w];
  const double r0 = (a.x - d.x) * ((b.y - d.y) * (c.z - d.z) - (b.z - d.z) * (c.y - d.y));
  const double r1 = (a.y - d.y) * ((b.z - d.z) * (c.x - d.x) - (b.x - d.x) * (c.z - d.z));
  const double r2 = (a.z - d.z) * ((b.x - d.x) * (c.y - d.y) - (b.y - d.y) * (c.x - d.x));
  vol[t] = fabs((r0 + r1 + r2) / 6);
}

// CSR of (key -> value) pairs, built in three deterministic steps: integer
// counts, exclusive scan, fill.  The fill order inside a segment depends on
// atomic scheduling; segments that need an order are sorted afterwards.
__global__ void k_count_tet_vertices(const int4* __restrict__ rows, int nt, int* __restrict__ cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  atomicAdd(cnt + v.x, 1);
  atomicAdd(cnt + v.y, 1);
  atomicAdd(cnt + v.z, 1);
  atomicAdd(cnt + v.w, 1);
}

__global__ void k_fill_tet_vertices(const int4* __restrict__ rows, int nt,
                                    const int* __restrict__ off, int* __restrict__ cursor,
                                    int* __restrict__ idx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  idx[off[v.x] + atomicAdd(cursor + v.x, 1)] = t;
  idx[off[v.y] + atomicAdd(cursor + v.y, 1)] = t;
  idx[off[v.z] + atomicAdd(cursor + v.z, 1)] = t;
  idx[off[v.w] + atomicAdd(cursor + v.w, 1)] = t;
}

// Sort each vertex's tets by index, so that the density sum below adds the
// volumes in increasing tet order, the order of the reference's scatter loop
// (src/triangulate.c:190-221).  Shell sort over a diminishing gap sequence
// (Ciura's gaps, then x2.25): plain insertion sort for the usual ~27 tets of
// a vertex, and O(d^1.3) rather than O(d^2) for the rare hub vertex with
// hundreds or thousands of tets.  The tet ids of a segment are distinct, so
// the sorted order is unique.
__global__ void k_sort_segments(const int* __restrict__ off, int n, int* __restrict__ idx) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int b = off[v], d = off[v + 1] - b;
  int* a = idx + b;
  constexpr int kGaps[] = {1, 4, 10, 23, 57, 132, 301, 701, 1577, 3548, 7983, 17961, 40412};
  int g = 0;
  while (g + 1 < (int)(sizeof(kGaps) / sizeof(kGaps[0])) && kGaps[g + 1] < d) ++g;
  for (; g >= 0; --g) {
    const int gap = kGaps[g];
    for (int i = gap; i < d; ++i) {
      const int key = a[i];
      int j = i;
      while (j >= gap && a[j - gap] > key) {
        a[j] = a[j - gap];
        j -= gap;
      }
      a[j] = key;
    }
  }
}

// a3 part 2: rho_v = m*(1+3) / sum of adjacent volumes, the sum taken
// sequentially from 0 in increasing tet order (bit-identical to the
// reference's in-place scatter-add).  No float atomics.
__global__ void k_density(const int* __restrict__ off, const int* __restrict__ idx,
                          const double* __restrict__ vol, int n, double m4,
                          double4* __restrict__ pos, int* __restrict__ adj) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int b = off[v], e = off[v + 1];
  double s = 0;
  for (int i = b; i < e; ++i) s += vol[idx[i]];
  pos[v].w = m4 / s;
  adj[v] = e - b;
}

__device__ __forceinline__ double det3(double a, double b, double c, double d, double e, double f,
                                       double g, double h, double i) {
  return a * e * i + b * f * g + c * d * h - c * e * g - b * d * i - a * f * h;
}

// a4: gradient of the linear interpolant by Cramer's rule on
// [B-A; C-A; D-A] grad = [rB-rA; rC-rA; rD-rA] (src/triangulate.c:228-260).
__global__ void k_gradients(const double4* __restrict__ pos, const int4* __restrict__ rows, int nt,
                            double* __restrict__ grad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  const double4 a = pos[v.x], b = pos[v.y], c = pos[v.z], d = pos[v.w];
  const double xb = b.x - a.x, yb = b.y - a.y, zb = b.z - a.z;
  const double xc = c.x - a.x, yc = c.y - a.y, zc = c.z - a.z;
  const double xd = d.x - a.x, yd = d.y - a.y, zd = d.z - a.z;
  const double rb = b.w - a.w, rc = c.w - a.w, rd = d.w - a.w;
  const double den = det3(xb, yb, zb, xc, yc, zc, xd, yd, zd);
  grad[3 * (size_t)t + 0] = det3(rb, yb, zb, rc, yc, zc, rd, yd, zd) / den;
  grad[3 * (size_t)t + 1] = det3(xb, rb, zb, xc, rc, zc, xd, rd, zd) / den;
  grad[3 * (size_t)t + 2] = det3(xb, yb, rb, xc, yc, rc, xd, yd, rd) / den;
}

// Per-tet FP64 field of the mixed 3-D grid, the linear field of
// src/triangulate.c:233-260 from vertex A expanded once per tet: the value at
// (x, y, z) is k + gx x + gy y + gz z, k = rho_A - gx x_A - gy y_A - gz z_A.
__global__ void k_field64(const double4* __restrict__ pos, const int4* __restrict__ rows,
                          const double* __restrict__ grad, int nt, double4* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  const double4 a = pos[v.x];
  const double gx = grad[3 * (size_t)t], gy = grad[3 * (size_t)t + 1], gz = grad[3 * (size_t)t + 2];
  out[t] = make_double4(a.w - gx * a.x - gy * a.y - gz * a.z, gx, gy, gz);
}

// Walk records for projection axis `axis`: positions and gradient permuted
// cyclically, the neighbour links copied.  The FP64 record carries rho_A and
// the gradient (the reference's field form); the FP32 record carries the four
// vertex densities (the mixed walk's barycentric form of the same field).
__global__ void k_records(const double4* __restrict__ pos, const int4* __restrict__ rows,
                          const double* __restrict__ grad, int nt, int axis,
                          TetRec64* __restrict__ r64, TetRot32* __restrict__ rot) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  const int4 nb = rows[2 * (size_t)t + 1];
  double4 p[4] = {pos[v.x], pos[v.y], pos[v.z], pos[v.w]};
  double q[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) permute3(axis, p[k].x, p[k].y, p[k].z, &q[k][0], &q[k][1], &q[k][2]);
  double g[3];
  permute3(axis, grad[3 * (size_t)t + 0], grad[3 * (size_t)t + 1], grad[3 * (size_t)t + 2], &g[0],
           &g[1], &g[2]);
  if (r64) {
    TetRec64 r;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.xy[k] = make_double2(q[k][0], q[k][1]);
    r.zab = make_double2(q[0][2], q[1][2]);
    r.zcd = make_double2(q[2][2], q[3][2]);
    r.rg0 = make_double2(p[0].w, g[0]);
    r.rg1 = make_double2(g[1], g[2]);
    r.nb = nb;
    r.vid = v;
    r64[t] = r;
  }
  if (rot) {
    // the record of each neighbour as entered from this tet
    const int nbo[4] = {nb.x, nb.y, nb.z, nb.w};
    int nxt[4];
    float zmin = (float)q[0][2], zmax = zmin;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      zmin = fminf(zmin, (float)q[s][2]);
      zmax = fmaxf(zmax, (float)q[s][2]);
      const int n = nbo[s];
      if (n < 0) {
        nxt[s] = -1;
        continue;
      }
      const int4 m = rows[2 * (size_t)n + 1];
      const int f = m.x == t ? 0 : (m.y == t ? 1 : (m.z == t ? 2 : (m.w == t ? 3 : -1)));
      nxt[s] = f >= 0 ? 4 * n + f : INT_MIN;
    }
    // extent of the projection, over the float coordinates the walk reads
    float lo[2] = {(float)q[0][0], (float)q[0][1]}, hi[2] = {lo[0], lo[1]};
#pragma unroll
    for (int s = 1; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        lo[c] = fminf(lo[c], (float)q[s][c]);
        hi[c] = fmaxf(hi[c], (float)q[s][c]);
      }
    const float ext = __fmul_ru(fmaxf(__fsub_ru(hi[0], lo[0]), __fsub_ru(hi[1], lo[1])), 1.0000010f);
    // Condition of the FP32 field value rho3 + grad . (p - v3) at a point p
    // of the tet: the magnitudes summed over the least vertex value, a bound
    // on the field there (a convex combination of the vertex values).  Its
    // rounding is a few units of roundoff times this; above kFieldCond the
    // walk evaluates the tet in FP64 (slivers, whose gradient terms cancel,
    // and vertex values of mixed sign or zero).
    double rmin = fabs(p[0].w), rmax = rmin;
#pragma unroll
    for (int s = 1; s < 4; ++s) {
      rmin = fmin(rmin, fabs(p[s].w));
      rmax = fmax(rmax, fabs(p[s].w));
    }
    const double cond = (rmax + (fabs(g[0]) + fabs(g[1])) * (double)ext +
                         fabs(g[2]) * (double)(zmax - zmin)) / rmin;
    const int fp64_field = (cond <= kFieldCond) ? 0 : (int)0x80000000u;  // also NaN, rmin = 0
#pragma unroll
    for (int F = 0; F < 4; ++F) {
      const int s0 = rot_slot(F, 0), s1 = rot_slot(F, 1), s2 = rot_slot(F, 2), s3 = rot_slot(F, 3);
      TetRot32 r;
      r.xy01 = make_float4((float)q[s0][0], (float)q[s0][1], (float)q[s1][0], (float)q[s1][1]);
      r.xy23 = make_float4((float)q[s2][0], (float)q[s2][1], (float)q[s3][0], (float)q[s3][1]);
      r.z = make_float4((float)q[s0][2], (float)q[s1][2], (float)q[s2][2], (float)q[s3][2]);
      r.fld = make_float4((float)p[s3].w, (float)g[0], (float)g[1], (float)g[2]);
      r.nb = make_int4(nxt[s0], nxt[s1], nxt[s2], __float_as_int(ext) | fp64_field);
      rot[4 * (size_t)t + F] = r;
    }
  }
}

// a5: forward faces of the projected hull (src/triangulate.c:263-316): a face
// with no neighbour whose edge vectors t1, t2 (the reference's choice per
// face) have (t1 x t2)_z < 0 in the projected frame.  One 32-bit word per
// tet, faces in bits 0..3: the reference's bitmap layout.
__global__ void k_hull_mask(const double4* __restrict__ pos, const int4* __restrict__ rows, int nt,
                            int axis, uint32_t* __restrict__ mask, int* __restrict__ cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int4 v = rows[2 * (size_t)t];
  const int4 nb = rows[2 * (size_t)t + 1];
  const int vid[4] = {v.x, v.y, v.z, v.w};
  const int nbs[4] = {nb.x, nb.y, nb.z, nb.w};
  // (origin, t1 end, t2 end) per face BDC, ACD, ADB, ABC
  const int fo[4] = {1, 0, 0, 0}, f1[4] = {3, 2, 3, 1}, f2[4] = {2, 3, 1, 2};
  uint32_t m = 0;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if (nbs[f] != -1) continue;
    double ox, oy, oz, px, py, pz, qx, qy, qz;
    const double4 o = pos[vid[fo[f]]], p = pos[vid[f1[f]]], q = pos[vid[f2[f]]];
    permute3(axis, o.x, o.y, o.z, &ox, &oy, &oz);
    permute3(axis, p.x, p.y, p.z, &px, &py, &pz);
    permute3(axis, q.x, q.y, q.z, &qx, &qy, &qz);
    const double t1x = px - ox, t1y = py - oy, t2x = qx - ox, t2y = qy - oy;
    if (t1x * t2y - t1y * t2x < 0.0) m |= 1u << f;
  }
  mask[t] = m;
  cnt[t] = __popc(m & 0xFu);
}

// a6 part 1: emit hull triangles in (tet, face) order with the reference's
// corner order per face (src/triangulate.c:325-355).
__global__ void k_hull_emit(const int4* __restrict__ rows, int nt, const uint32_t* __restrict__ mask,
                            const int* __restrict__ off, int* __restrict__ tri_rows,
                            signed char* __restrict__ tri_face) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const uint32_t m = mask[t] & 0xFu;
  if (!m) return;
  const int4 v = rows[2 * (size_t)t];
  const int vid[4] = {v.x, v.y, v.z, v.w};
  const int ta[4] = {1, 0, 0, 0}, tb[4] = {3, 2, 3, 1}, tc[4] = {2, 3, 1, 2};
  int k = off[t];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if (!(m & (1u << f))) continue;
    tri_face[k] = (signed char)f;
    int* r = tri_rows + 8 * (size_t)k++;
    r[0] = vid[ta[f]];
    r[1] = vid[tb[f]];
    r[2] = vid[tc[f]];
    r[3] = r[4] = r[5] = -1;
    r[6] = t;
    r[7] = -1;
  }
}

__global__ void k_count_tri_vertices(const int* __restrict__ tri_rows, int n_tri,
                                     int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tri) return;
  for (int k = 0; k < 3; ++k) atomicAdd(cnt + tri_rows[8 * (size_t)i + k], 1);
}

__global__ void k_fill_tri_vertices(const int* __restrict__ tri_rows, int n_tri,
                                    const int* __restrict__ off, int* __restrict__ cursor,
                                    int* __restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tri) return;
  for (int k = 0; k < 3; ++k) {
    const int v = tri_rows[8 * (size_t)i + k];
    idx[off[v] + atomicAdd(cursor + v, 1)] = i;
  }
}

// a6 part 2: edge neighbours.  For the edge (p, q) of triangle i the
// neighbour is the largest j != i whose corners include both p and q: the
// result of the reference's all-pairs scan where the last match wins
// (src/triangulate.c:358-392), found here through the triangles incident to
// p.  Then the walk's triangle records.
__global__ void k_hull_adjacency(const double4* __restrict__ pos, int axis,
                                 int* __restrict__ tri_rows, int n_tri, const int* __restrict__ off,
                                 const int* __restrict__ idx, TriRec64* __restrict__ rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tri) return;
  int* r = tri_rows + 8 * (size_t)i;
  const int c[3] = {r[0], r[1], r[2]};
  // slot 3+CB: edge b-c; 3+AC: edge a-c; 3+BA: edge a-b
  const int ep[3] = {1, 0, 0}, eq[3] = {2, 2, 1};
  int nbr[3];
  for (int s = 0; s < 3; ++s) {
    const int p = c[ep[s]], q = c[eq[s]];
    int best = -1;
    for (int k = off[p]; k < off[p + 1]; ++k) {
      const int j = idx[k];
      if (j == i) continue;
      const int* rj = tri_rows + 8 * (size_t)j;
      if ((rj[0] == q || rj[1] == q || rj[2] == q) && j > best) best = j;
    }
    nbr[s] = best;
  }
  r[3] = nbr[0];
  r[4] = nbr[1];
  r[5] = nbr[2];
  double2 xy[3];
  for (int k = 0; k < 3; ++k) {
    const double4 pp = pos[c[k]];
    double x, y, z;
    permute3(axis, pp.x, pp.y, pp.z, &x, &y, &z);
    xy[k] = make_double2(x, y);
  }
  TriRec64 t;
  t.a = xy[0];
  t.b = xy[1];
  t.c = xy[2];
  t.nb = make_int4(nbr[0], nbr[1], nbr[2], r[6]);
  rec[i] = t;
}

// exclusive scan of n ints into out[0..n]; out[n] is the total
dtfe_status_t exclusive_scan(const int* in, int* out, int n, cudaStream_t s) {
  size_t tmp_bytes = 0;
  SDTFE_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, n + 1, s));
  void* tmp = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&tmp, tmp_bytes, s));
  cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, n + 1, s);
  cudaFreeAsync(tmp, s);
  SDTFE_CUDA(e);
  return DTFE_OK;
}

// The meshes' memory pool of each device (vertices, rows, gradients,
// adjacency, walk records, per-call scratch): stream-ordered allocation (no
// device-wide synchronisation when a mesh is built or destroyed, or records
// are built or dropped, while maps run), and freed memory kept for reuse up
// to an eighth of the device (at most 16 GB) instead of being unmapped and
// mapped again by every mesh.
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_record_pool[kMaxPoolDevices] = {};

dtfe_status_t record_pool(cudaMemPool_t* out) {
  int dev = 0;
  SDTFE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxPoolDevices) return set_error(DTFE_ERR_UNSUPPORTED, "device %d", dev);
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_record_pool[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    SDTFE_CUDA(cudaMemPoolCreate(&pool, &props));
    size_t fr = 0, total = 0;
    SDTFE_CUDA(cudaMemGetInfo(&fr, &total));
    uint64_t keep = std::min<uint64_t>(uint64_t(16) << 30, total / 8);
    SDTFE_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_record_pool[dev] = pool;
  }
  *out = g_record_pool[dev];
  return DTFE_OK;
}

}  // namespace

// Per-call device scratch, stream-ordered from the record pool (whose freed
// memory is kept for reuse, so a map's scratch costs no mapping).
dtfe_status_t scratch_alloc_async(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  cudaMemPool_t pool = nullptr;
  SDTFE_TRY(record_pool(&pool));
  SDTFE_CUDA(cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s));
  return DTFE_OK;
}

void scratch_free_async(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

void mesh_trim_record_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxPoolDevices) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (g_record_pool[dev]) cudaMemPoolTrimTo(g_record_pool[dev], 0);
}

namespace {

// stream-ordered allocation from the record pool, on the mesh stream
template <class T>
dtfe_status_t dmalloc_async(T** p, size_t count, Mesh* m) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaMemPool_t pool = nullptr;
  SDTFE_TRY(record_pool(&pool));
  SDTFE_CUDA(cudaMallocFromPoolAsync((void**)p, count * sizeof(T), pool, m->stream));
  m->bytes += count * sizeof(T);
  return DTFE_OK;
}

template <class T>
void dfree_async(T*& p, size_t count, Mesh* m) {
  if (p) {
    cudaFreeAsync(p, m->stream);
    m->bytes -= (count ? count : 1) * sizeof(T);
  }
  p = nullptr;
}

}  // namespace

dtfe_status_t mesh_upload(Mesh* m, const double* particle_data, int n, const int* tetra_data,
                          int nt, float p_mass, unsigned flags) {
  if (n < 0 || nt < 0 || (n > 0 && !particle_data) || (nt > 0 && !tetra_data))
    return set_error(DTFE_ERR_INVALID, "mesh_upload: bad sizes or null arrays");
  m->n = n;
  m->nt = nt;
  m->p_mass = p_mass;
  m->flags = flags;
  SDTFE_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  SDTFE_CUDA(cudaEventCreate(&m->ev0));
  SDTFE_CUDA(cudaEventCreate(&m->ev1));
  SDTFE_TRY(dmalloc_async(&m->pos, n, m));
  SDTFE_TRY(dmalloc_async(&m->rows, 2 * (size_t)nt, m));
  SDTFE_TRY(dmalloc_async(&m->stats, kStatCount, m));
  cudaStream_t s = m->stream;
  if (n) SDTFE_CUDA(cudaMemcpyAsync(m->pos, particle_data, sizeof(double4) * n, cudaMemcpyHostToDevice, s));
  if (nt) SDTFE_CUDA(cudaMemcpyAsync(m->rows, tetra_data, sizeof(int4) * 2 * (size_t)nt, cudaMemcpyHostToDevice, s));
  SDTFE_CUDA(cudaMemsetAsync(m->stats, 0, sizeof(unsigned long long) * kStatCount, s));
  int* d_flags = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&d_flags, 3 * sizeof(int), s));
  SDTFE_CUDA(cudaMemsetAsync(d_flags, 0, 3 * sizeof(int), s));
  if (nt) {
    k_validate<<<grid_for(nt), kBlock, 0, s>>>(m->rows, nt, n, d_flags);
    count_launch();
  }
  if (n) {
    k_fp32_exact<<<grid_for(n), kBlock, 0, s>>>(m->pos, n, d_flags + 1, d_flags + 2);
    count_launch();
  }
  int h_flags[3] = {0, 0, 0};
  SDTFE_CUDA(cudaMemcpyAsync(h_flags, d_flags, sizeof(h_flags), cudaMemcpyDeviceToHost, s));
  SDTFE_CUDA(cudaFreeAsync(d_flags, s));
  SDTFE_CUDA(cudaStreamSynchronize(s));
  SDTFE_CUDA(cudaGetLastError());
  m->fp32_exact = h_flags[1] == 0;
  {
    float mx;
    memcpy(&mx, &h_flags[2], sizeof mx);
    m->coord_max = (double)mx;
  }
  if (h_flags[0])
    return set_error(DTFE_ERR_MESH, "tetra_data holds a vertex id outside [0, %d) or a neighbour id outside [-1, %d)", n, nt);
  m->has_density = (flags & DTFE_MESH_FIELD) != 0;
  return DTFE_OK;
}

dtfe_status_t mesh_density(Mesh* m) {
  cudaStream_t s = m->stream;
  const int n = m->n, nt = m->nt;
  SDTFE_TRY(dmalloc_async(&m->adj, n, m));
  double* vol = nullptr;
  int *cnt = nullptr, *off = nullptr, *idx = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&vol, sizeof(double) * (nt ? nt : 1), s));
  SDTFE_CUDA(cudaMallocAsync(&cnt, sizeof(int) * (n + 1), s));
  SDTFE_CUDA(cudaMallocAsync(&off, sizeof(int) * (n + 1), s));
  SDTFE_CUDA(cudaMallocAsync(&idx, sizeof(int) * (4 * (size_t)nt + 1), s));
  SDTFE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (n + 1), s));
  if (nt) {
    k_volume<<<grid_for(nt), kBlock, 0, s>>>(m->pos, m->rows, nt, vol);
    count_launch();
    k_count_tet_vertices<<<grid_for(nt), kBlock, 0, s>>>(m->rows, nt, cnt);
    count_launch();
  }
  SDTFE_TRY(exclusive_scan(cnt, off, n, s));
  SDTFE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (n + 1), s));
  if (nt) {
    k_fill_tet_vertices<<<grid_for(nt), kBlock, 0, s>>>(m->rows, nt, off, cnt, idx);
    count_launch();
  }
  if (n) {
    k_sort_segments<<<grid_for(n), kBlock, 0, s>>>(off, n, idx);
    count_launch();
    // p_mass*(1+DIM) is a float product in the reference (float * int)
    const double m4 = (double)(m->p_mass * 4);
    k_density<<<grid_for(n), kBlock, 0, s>>>(off, idx, vol, n, m4, m->pos, m->adj);
    count_launch();
  }
  cudaFreeAsync(vol, s);
  cudaFreeAsync(cnt, s);
  cudaFreeAsync(off, s);
  cudaFreeAsync(idx, s);
  SDTFE_CUDA(cudaGetLastError());
  m->has_density = true;
  return DTFE_OK;
}

dtfe_status_t mesh_gradients(Mesh* m) {
  if (!m->grad) SDTFE_TRY(dmalloc_async(&m->grad, 3 * (size_t)m->nt, m));
  if (m->nt) {
    k_gradients<<<grid_for(m->nt), kBlock, 0, m->stream>>>(m->pos, m->rows, m->nt, m->grad);
    count_launch();
  }
  SDTFE_CUDA(cudaGetLastError());
  return DTFE_OK;
}

dtfe_status_t mesh_field64(Mesh* m) {
  if (m->fld64) return DTFE_OK;
  if (!m->grad) return set_error(DTFE_ERR_INVALID, "mesh_field64 before mesh_gradients");
  SDTFE_TRY(dmalloc_async(&m->fld64, m->nt, m));
  if (m->nt) {
    k_field64<<<grid_for(m->nt), kBlock, 0, m->stream>>>(m->pos, m->rows, m->grad, m->nt, m->fld64);
    count_launch();
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    dfree_async(m->fld64, m->nt, m);
    return set_error(DTFE_ERR_CUDA, "grid field: %s", cudaGetErrorString(e));
  }
  return DTFE_OK;
}

dtfe_status_t mesh_records(Mesh* m, int axis, bool want64, bool want32) {
  if (axis < 0 || axis > 2) return set_error(DTFE_ERR_INVALID, "axis %d not in 0..2", axis);
  if (!m->grad) return set_error(DTFE_ERR_INVALID, "mesh_records before mesh_gradients");
  AxisData& A = m->ax[axis];
  const bool need64 = want64 && !A.rec64, need32 = want32 && !A.rot32;
  if (!need64 && !need32) return DTFE_OK;
  // the mixed walk's records address 4*t + F in an int: up to 2^29 - 1 tets
  if (need32 && m->nt >= (1 << 29))
    return set_error(DTFE_ERR_UNSUPPORTED, "mixed maps of %d tets (at most 2^29 - 1)", m->nt);
  // all or nothing: a record array that exists has been built; stream-ordered
  // allocations, so that building records for one mesh does not stall the
  // device (the serving loop builds and drops them while maps run)
  dtfe_status_t st = DTFE_OK;
  if (need64) st = dmalloc_async(&A.rec64, m->nt, m);
  if (st == DTFE_OK && need32) st = dmalloc_async(&A.rot32, 4 * (size_t)m->nt, m);
  if (st == DTFE_OK && m->nt) {
    k_records<<<grid_for(m->nt), kBlock, 0, m->stream>>>(m->pos, m->rows, m->grad, m->nt, axis,
                                                         need64 ? A.rec64 : nullptr,
                                                         need32 ? A.rot32 : nullptr);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      st = set_error(DTFE_ERR_CUDA, "walk records: %s", cudaGetErrorString(e));
  }
  if (st != DTFE_OK) {
    if (need64) dfree_async(A.rec64, m->nt, m);
    if (need32) dfree_async(A.rot32, 4 * (size_t)m->nt, m);
    return st;
  }
  return DTFE_OK;
}

size_t mesh_record_bytes(const Mesh& m, int axis) {
  const AxisData& A = m.ax[axis];
  const size_t nt = (size_t)m.nt;
  return (A.rot32 ? 4 * sizeof(TetRot32) * nt : 0) + (A.rec64 ? sizeof(TetRec64) * nt : 0);
}

size_t mesh_missing_record_bytes(const Mesh& m, int axis, int precision) {
  const AxisData& A = m.ax[axis];
  const size_t nt = (size_t)m.nt;
  size_t b = 0;
  if (precision == DTFE_MIXED && !A.rot32) b += 4 * sizeof(TetRot32) * nt;
  // the mixed walk reads FP64 records only when the coordinates are not floats
  const bool want64 = precision == DTFE_FP64 ||
                      (!m.fp32_exact && !(m.flags & DTFE_MESH_NO_FP64_REC));
  if (want64 && !A.rec64) b += sizeof(TetRec64) * nt;
  return b;
}

// Frees one axis' walk records (the caller has no map of that axis in flight),
// ordered on the mesh stream.
void mesh_drop_records(Mesh* m, int axis) {
  if (axis < 0 || axis > 2) return;
  dfree_async(m->ax[axis].rec64, m->nt, m);
  dfree_async(m->ax[axis].rot32, 4 * (size_t)m->nt, m);
}

dtfe_status_t mesh_hull_mask(Mesh* m, int axis, uint32_t* host_mask_out, int* count_out) {
  cudaStream_t s = m->stream;
  const int nt = m->nt;
  uint32_t* mask = nullptr;
  int *cnt = nullptr, *off = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&mask, sizeof(uint32_t) * (nt ? nt : 1), s));
  SDTFE_CUDA(cudaMallocAsync(&cnt, sizeof(int) * (nt + 1), s));
  SDTFE_CUDA(cudaMallocAsync(&off, sizeof(int) * (nt + 1), s));
  if (nt) {
    k_hull_mask<<<grid_for(nt), kBlock, 0, s>>>(m->pos, m->rows, nt, axis, mask, cnt);
    count_launch();
  }
  SDTFE_TRY(exclusive_scan(cnt, off, nt, s));
  int total = 0;
  SDTFE_CUDA(cudaMemcpyAsync(&total, off + nt, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (host_mask_out && nt)
    SDTFE_CUDA(cudaMemcpyAsync(host_mask_out, mask, sizeof(uint32_t) * nt, cudaMemcpyDeviceToHost, s));
  SDTFE_CUDA(cudaStreamSynchronize(s));
  cudaFreeAsync(mask, s);
  cudaFreeAsync(cnt, s);
  cudaFreeAsync(off, s);
  *count_out = total;
  return DTFE_OK;
}

dtfe_status_t mesh_hull(Mesh* m, int axis, const uint32_t* host_mask, int* count_out) {
  if (axis < 0 || axis > 2) return set_error(DTFE_ERR_INVALID, "axis %d not in 0..2", axis);
  cudaStream_t s = m->stream;
  const int nt = m->nt, n = m->n;
  AxisData& A = m->ax[axis];
  if (A.hull_built && !host_mask) {
    if (count_out) *count_out = A.n_tri;
    return DTFE_OK;
  }
  uint32_t* mask = nullptr;
  int *cnt = nullptr, *off = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&mask, sizeof(uint32_t) * (nt ? nt : 1), s));
  SDTFE_CUDA(cudaMallocAsync(&cnt, sizeof(int) * (nt + 1), s));
  SDTFE_CUDA(cudaMallocAsync(&off, sizeof(int) * (nt + 1), s));
  if (host_mask) {
    // caller's bitmap: count its face bits on the device
    if (nt) SDTFE_CUDA(cudaMemcpyAsync(mask, host_mask, sizeof(uint32_t) * nt, cudaMemcpyHostToDevice, s));
    std::vector<int> hc(nt);
    for (int t = 0; t < nt; ++t) hc[t] = __builtin_popcount(host_mask[t] & 0xFu);
    if (nt) SDTFE_CUDA(cudaMemcpyAsync(cnt, hc.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s));
    SDTFE_CUDA(cudaStreamSynchronize(s));
  } else if (nt) {
    k_hull_mask<<<grid_for(nt), kBlock, 0, s>>>(m->pos, m->rows, nt, axis, mask, cnt);
    count_launch();
  }
  SDTFE_TRY(exclusive_scan(cnt, off, nt, s));
  int n_tri = 0;
  SDTFE_CUDA(cudaMemcpyAsync(&n_tri, off + nt, sizeof(int), cudaMemcpyDeviceToHost, s));
  SDTFE_CUDA(cudaStreamSynchronize(s));
  // replace the axis' triangles (the mesh stream is idle: synchronised above)
  dfree_async(A.tri, A.n_tri, m);
  dfree_async(A.tri_rows, 8 * (size_t)A.n_tri, m);
  dfree_async(A.tri_face, A.n_tri, m);
  SDTFE_TRY(dmalloc_async(&A.tri, n_tri, m));
  SDTFE_TRY(dmalloc_async(&A.tri_rows, 8 * (size_t)n_tri, m));
  SDTFE_TRY(dmalloc_async(&A.tri_face, n_tri, m));
  A.n_tri = n_tri;
  if (nt) {
    k_hull_emit<<<grid_for(nt), kBlock, 0, s>>>(m->rows, nt, mask, off, A.tri_rows, A.tri_face);
    count_launch();
  }
  // vertex -> hull triangle lists for the edge matching
  int *vcnt = nullptr, *voff = nullptr, *vidx = nullptr;
  SDTFE_CUDA(cudaMallocAsync(&vcnt, sizeof(int) * (n + 1), s));
  SDTFE_CUDA(cudaMallocAsync(&voff, sizeof(int) * (n + 1), s));
  SDTFE_CUDA(cudaMallocAsync(&vidx, sizeof(int) * (3 * (size_t)n_tri + 1), s));
  SDTFE_CUDA(cudaMemsetAsync(vcnt, 0, sizeof(int) * (n + 1), s));
  if (n_tri) {
    k_count_tri_vertices<<<grid_for(n_tri), kBlock, 0, s>>>(A.tri_rows, n_tri, vcnt);
    count_launch();
  }
  SDTFE_TRY(exclusive_scan(vcnt, voff, n, s));
  SDTFE_CUDA(cudaMemsetAsync(vcnt, 0, sizeof(int) * (n + 1), s));
  if (n_tri) {
    k_fill_tri_vertices<<<grid_for(n_tri), kBlock, 0, s>>>(A.tri_rows, n_tri, voff, vcnt, vidx);
    count_launch();
    k_hull_adjacency<<<grid_for(n_tri), kBlock, 0, s>>>(m->pos, axis, A.tri_rows, n_tri, voff, vidx, A.tri);
    count_launch();
  }
  cudaFreeAsync(vcnt, s);
  cudaFreeAsync(voff, s);
  cudaFreeAsync(vidx, s);
  cudaFreeAsync(mask, s);
  cudaFreeAsync(cnt, s);
  cudaFreeAsync(off, s);
  SDTFE_CUDA(cudaGetLastError());
  A.hull_built = !host_mask;
  if (count_out) *count_out = n_tri;
  return DTFE_OK;
}

void mesh_free(Mesh* m) {
  // every array returns to the pool stream-ordered on the mesh stream, which
  // is then synchronised (the caller's own streams are done with the mesh)
  for (auto& A : m->ax) {
    dfree_async(A.rec64, m->nt, m);
    dfree_async(A.rot32, 4 * (size_t)m->nt, m);
  }
  dfree_async(m->fld64, m->nt, m);
  dfree_async(m->pos, m->n, m);
  dfree_async(m->rows, 2 * (size_t)m->nt, m);
  dfree_async(m->grad, 3 * (size_t)m->nt, m);
  dfree_async(m->adj, m->n, m);
  dfree_async(m->stats, kStatCount, m);
  for (auto& A : m->ax) {
    dfree_async(A.tri, A.n_tri, m);
    dfree_async(A.tri_rows, 8 * (size_t)A.n_tri, m);
    dfree_async(A.tri_face, A.n_tri, m);
  }
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->stream) cudaStreamDestroy(m->stream);
  m->ev0 = m->ev1 = nullptr;
  m->stream = nullptr;
}

}  // namespace sdtfe
