// walk64.cuh - FP64 ray walk through a device-resident Delaunay mesh.
//
// The arithmetic here repeats the reference's FP64 operations in the same
// order (src/dtfe.c:19-374, 518-552), and the translation units that include
// this header are compiled with -fmad=false, so each product and sum is
// rounded on its own exactly as the reference's x86-64 build rounds it.  With
// the same mesh, the same sample positions and the same perturbation stream
// the walk therefore visits the same tets and returns the same doubles.
//
// Data layout (built by mesh.cu):
//   TetRec64  160 B per tet: the (x, y) and z of its four vertices in the
//             projected frame, rho_A, the gradient and the neighbour links.
//             One walk step reads one record: the next tet id and everything
//             the Plücker test and the integral need arrive together.
//   TriRec64   64 B per projected hull triangle: (x, y) of its corners, the
//             three edge neighbours and the tet under it.
#pragma once

#include <cstdint>

#include "sdtfe_rng.h"

namespace sdtfe {

// src/constants.h:6-8
constexpr double kZero = 1e4 * 2.220446049250313080847263336181640625e-16;
constexpr int kPerturbMax = 1000;

enum RayStatus : int {
  kRayOk = 0,
  kRayMiss = 1,
  kRayNoExit = 2,
  kRayPerturbMax = 3,
  kRayBudget = 4,
  kRayLocBudget = 5,
};

struct __align__(32) TetRec64 {
  double2 xy[4];  // vertices A..D in the projected frame
  double2 zab;    // (z_A, z_B)
  double2 zcd;    // (z_C, z_D)
  double2 rg0;    // (rho_A, grad_x)
  double2 rg1;    // (grad_y, grad_z)
  int4 nb;        // neighbours across faces BDC, ACD, ADB, ABC (-1: hull)
  int4 vid;       // vertex ids A..D
};
static_assert(sizeof(TetRec64) == 160, "TetRec64 layout");

struct __align__(16) TriRec64 {
  double2 a, b, c;  // projected corners
  int4 nb;          // (n_CB, n_AC, n_BA, tet)
};
static_assert(sizeof(TriRec64) == 64, "TriRec64 layout");

template <class T>
__device__ __forceinline__ T sel4(int k, T a, T b, T c, T d) {
  return k == 0 ? a : (k == 1 ? b : (k == 2 ? c : d));
}

__device__ __forceinline__ int sign_eps(double x) {
  return x > kZero ? 1 : (x < -kZero ? -1 : 0);
}

__device__ __forceinline__ int nb_at(const int4& n, int k) { return sel4(k, n.x, n.y, n.z, n.w); }

// ---------------------------------------------------------------------------
// a8: Plücker test for a ray along +z (src/dtfe.c:29-215).
//
// For the edge P->Q the permuted product with the ray (lz, -lz*oy, lz*ox) is
//   lz*(Px*Qy - Py*Qx) + (Px - Qx)*(-lz*oy) + (Py - Qy)*(lz*ox)
// (src/dtfe.c:24-26, 44-47).  Edges in side_t order: CB, AC, BA, DC, BD, DA.
struct Ray64 {
  double lz, m_oy, ox_l;  // lz, -lz*oy, lz*ox
};

__device__ __forceinline__ double edge_u64(const Ray64& r, double2 p, double2 q) {
  double v0 = p.x - q.x;
  double v1 = p.y - q.y;
  double v5 = p.x * q.y - p.y * q.x;
  return r.lz * v5 + v0 * r.m_oy + v1 * r.ox_l;
}

struct Hit64 {
  int enter, leave;
  bool ok, special;
};

// The four faces BDC, ACD, ADB, ABC each carry three signed edge terms; a face
// whose three edge signs are all zero is skipped, a face is entered when its
// signed terms are all >= 0 and left when all are <= 0 (the two are exclusive
// once the all-zero case is skipped).  The first entered and the first left
// face in that order are chosen; the test fails unless both exist.
__device__ __forceinline__ Hit64 plucker_faces(const int s[6]) {
  // signed sign terms per face (the reference's conditions, src/dtfe.c:66-213)
  const int f0a = -s[0], f0b = s[3], f0c = -s[4];   // BDC: -CB, +DC, -BD
  const int f1a = s[1], f1b = -s[3], f1c = -s[5];   // ACD: +AC, -DC, -DA
  const int f2a = s[5], f2b = s[4], f2c = -s[2];    // ADB: +DA, +BD, -BA
  const int f3a = s[2], f3b = s[0], f3c = -s[1];    // ABC: +BA, +CB, -AC
  auto live = [](int a, int b, int c) { return (a | b | c) != 0; };
  auto ent = [&](int a, int b, int c) { return live(a, b, c) && a >= 0 && b >= 0 && c >= 0; };
  auto lea = [&](int a, int b, int c) { return live(a, b, c) && a <= 0 && b <= 0 && c <= 0; };
  auto zer = [](int a, int b, int c) { return a == 0 || b == 0 || c == 0; };
  const bool e0 = ent(f0a, f0b, f0c), e1 = ent(f1a, f1b, f1c), e2 = ent(f2a, f2b, f2c),
             e3 = ent(f3a, f3b, f3c);
  const bool l0 = lea(f0a, f0b, f0c), l1 = lea(f1a, f1b, f1c), l2 = lea(f2a, f2b, f2c),
             l3 = lea(f3a, f3b, f3c);
  Hit64 h;
  h.enter = e0 ? 0 : (e1 ? 1 : (e2 ? 2 : (e3 ? 3 : -1)));
  h.leave = l0 ? 0 : (l1 ? 1 : (l2 ? 2 : (l3 ? 3 : -1)));
  h.ok = h.enter >= 0 && h.leave >= 0;
  const bool z0 = zer(f0a, f0b, f0c), z1 = zer(f1a, f1b, f1c), z2 = zer(f2a, f2b, f2c),
             z3 = zer(f3a, f3b, f3c);
  h.special = h.ok && (sel4(h.enter, z0, z1, z2, z3) || sel4(h.leave, z0, z1, z2, z3));
  return h;
}

// z of the point where the ray crosses face f: the face normaliser is summed
// in the reference's order, then ((1 - w1) - w2)*z0 + w1*z1 + w2*z2.
__device__ __forceinline__ double face_z64(int f, const double u[6], const double z[4]) {
  const double a0 = sel4(f, -u[0], u[1], u[5], u[2]);
  const double a1 = sel4(f, u[3], -u[3], u[4], u[0]);
  const double a2 = sel4(f, -u[4], -u[5], -u[2], -u[1]);
  const double w1n = sel4(f, -u[4], u[1], u[4], -u[1]);
  const double w2n = sel4(f, u[3], -u[3], -u[2], u[2]);
  const double z0 = sel4(f, z[3], z[2], z[1], z[0]);
  const double z1 = sel4(f, z[2], z[3], z[0], z[1]);
  const double z2 = sel4(f, z[1], z[0], z[3], z[2]);
  const double inv = 1.0 / (a0 + a1 + a2);
  const double w1 = w1n * inv;
  const double w2 = w2n * inv;
  return (1 - w1 - w2) * z0 + w1 * z1 + w2 * z2;
}

__device__ __forceinline__ Hit64 ray_tet64(const Ray64& r, const double2 xy[4], double u[6]) {
  u[0] = edge_u64(r, xy[2], xy[1]);  // CB
  u[1] = edge_u64(r, xy[2], xy[0]);  // AC
  u[2] = edge_u64(r, xy[1], xy[0]);  // BA
  u[3] = edge_u64(r, xy[2], xy[3]);  // DC
  u[4] = edge_u64(r, xy[1], xy[3]);  // BD
  u[5] = edge_u64(r, xy[3], xy[0]);  // DA
  int s[6];
#pragma unroll
  for (int e = 0; e < 6; ++e) s[e] = sign_eps(u[e]);
  return plucker_faces(s);
}

// ---------------------------------------------------------------------------
// a7: visibility walk on the projected hull, from triangle `start`
// (src/dtfe.c:518-552).  Returns the tet under the query point or -1.
// Returns the tet under the hull triangle containing (qx, qy); *tri_out (if
// given) receives the triangle.
__device__ __forceinline__ int locate64(const TriRec64* __restrict__ tri, int start, double qx,
                                        double qy, int max_steps, int* status,
                                        int* tri_out = nullptr) {
  int cur = start;
  int steps = 0;
  *status = kRayOk;
  do {
    if (++steps > max_steps) {
      *status = kRayLocBudget;
      return -1;
    }
    const TriRec64* t = tri + cur;
    const double2 a = __ldg(&t->a), b = __ldg(&t->b), c = __ldg(&t->c);
    const int4 nb = __ldg(&t->nb);
    double s_in, s_q;
    s_in = (c.x - a.x) * (b.y - a.y) - (c.y - a.y) * (b.x - a.x);
    s_q = (qx - a.x) * (b.y - a.y) - (qy - a.y) * (b.x - a.x);
    if (s_in * s_q < 0.0) {
      cur = nb.z;  // across a-b
      continue;
    }
    s_in = (a.x - b.x) * (c.y - b.y) - (a.y - b.y) * (c.x - b.x);
    s_q = (qx - b.x) * (c.y - b.y) - (qy - b.y) * (c.x - b.x);
    if (s_in * s_q < 0.0) {
      cur = nb.x;  // across b-c
      continue;
    }
    s_in = (b.x - c.x) * (a.y - c.y) - (b.y - c.y) * (a.x - c.x);
    s_q = (qx - c.x) * (a.y - c.y) - (qy - c.y) * (a.x - c.x);
    if (s_in * s_q < 0.0) {
      cur = nb.y;  // across c-a
      continue;
    }
    if (tri_out) *tri_out = cur;
    return nb.w;
  } while (cur != -1);
  *status = kRayMiss;
  return -1;
}

// One of locate64's edge tests (edge o->p, opposite vertex opp: s_in * s_q <
// 0) decided for every query point of the rectangle [xlo, xhi] x [ylo, yhi]
// at once: 1 when it holds for all of them, 0 when it fails for all, -1 when
// the outcome may differ inside.  s_in is the reference's own value.  The
// FP64 s_q = (qx - o.x) dy - (qy - o.y) dx (dy, dx the rounded edge
// differences) is within 3.0001 u M(q) of the linear form L(q) = (qx - o.x) dy
// - (qy - o.y) dx, M(q) = |qx - o.x| |dy| + |qy - o.y| |dx| (u = 2^-53; the
// operations are not contracted).  L and M take their extremes at the
// corners, so every s_q lies within 6.0002 u max M of the corners' FP64
// values; 16 u covers that and the rounding of the bound, and 2^-1000 any
// underflow.  The product s_in * s_q is then of one sign for all queries,
// and well clear of underflow to zero.
__host__ __device__ inline int edge_region(double2 o, double2 p, double2 opp, double xlo,
                                           double xhi, double ylo, double yhi) {
  const double s_in = (opp.x - o.x) * (p.y - o.y) - (opp.y - o.y) * (p.x - o.x);
  if (s_in == 0.0) return 0;  // the product is (signed) zero for every query
  const double dy = p.y - o.y, dx = p.x - o.x;
  const double qx[4] = {xlo, xhi, xlo, xhi}, qy[4] = {ylo, ylo, yhi, yhi};
  double lo = 0.0, hi = 0.0, mag = 0.0;
  for (int k = 0; k < 4; ++k) {
    const double tx = qx[k] - o.x, ty = qy[k] - o.y;
    const double s = tx * dy - ty * dx;
    lo = k == 0 ? s : (s < lo ? s : lo);
    hi = k == 0 ? s : (s > hi ? s : hi);
    const double m = (tx < 0.0 ? -tx : tx) * (dy < 0.0 ? -dy : dy) +
                     (ty < 0.0 ? -ty : ty) * (dx < 0.0 ? -dx : dx);
    mag = m > mag ? m : mag;
  }
  const double err = 16.0 * 0x1p-53 * mag + 0x1p-1000;
  const double a_in = s_in < 0.0 ? -s_in : s_in;
  if (lo > err) {  // s_q > 0 throughout
    if (a_in * (lo - err) < 0x1p-1000) return -1;
    return s_in < 0.0 ? 1 : 0;
  }
  if (hi < -err) {  // s_q < 0 throughout
    if (a_in * (-err - hi) < 0x1p-1000) return -1;
    return s_in > 0.0 ? 1 : 0;
  }
  return -1;
}

enum LocKind : int {
  kLocResume = 0,  // each query continues locate64 from *start with max_steps - *steps
  kLocFound = 1,   // every query's walk ends in triangle *start
  kLocMiss = 2,    // every query's walk leaves the hull
};

// The reference's location walk from triangle 0 (locate64), run once for a
// whole rectangle of query points while each edge test has one outcome for
// all of them.  Where the rectangle straddles a test, the walk stops and each
// query resumes it on its own at that triangle, with the steps taken so far
// counted against its budget: every query then makes exactly the moves, and
// ends with exactly the result, of its own walk from triangle 0.
__host__ __device__ inline int locate_region(const TriRec64* tri, double xlo, double xhi,
                                             double ylo, double yhi, int max_steps, int* start,
                                             int* steps_out) {
  int cur = 0, steps = 0;
  for (;;) {
    if (steps >= max_steps) break;  // each query's next step exceeds its budget
    const TriRec64& t = tri[cur];
    int nx = -1;
    int r = edge_region(t.a, t.b, t.c, xlo, xhi, ylo, yhi);  // edge a-b
    if (r == 1) {
      nx = t.nb.z;
    } else if (r == 0) {
      r = edge_region(t.b, t.c, t.a, xlo, xhi, ylo, yhi);  // edge b-c
      if (r == 1) {
        nx = t.nb.x;
      } else if (r == 0) {
        r = edge_region(t.c, t.a, t.b, xlo, xhi, ylo, yhi);  // edge c-a
        if (r == 1) {
          nx = t.nb.y;
        } else if (r == 0) {
          *start = cur;
          *steps_out = steps;
          return kLocFound;
        }
      }
    }
    if (r < 0) break;
    ++steps;
    if (nx == -1) {
      *start = -1;
      *steps_out = steps;
      return kLocMiss;
    }
    cur = nx;
  }
  *start = cur;
  *steps_out = steps;
  return kLocResume;
}

// The rectangle holding every sample position of a map tile (Args: the FP64
// or the mixed map's kernel arguments).  A ray's position is x(col) + u *
// scale with u in [0, 1), x(col) the expression below (the same as the
// rays'); each is monotone in col and u, so the tile's positions lie in
// [x(tx0), x(c1) + scale], and the same for y.
template <class Args>
__device__ __forceinline__ void tile_rect(const Args& a, int tile, double* xlo, double* xhi,
                                          double* ylo, double* yhi) {
  const int tx0 = (tile % a.tiles_x) * a.TW, ty0 = (tile / a.tiles_x) * a.TH;
  const int c1 = min(tx0 + a.TW, a.G) - 1, r1 = min(ty0 + a.TH, a.G) - 1;
  *xlo = tx0 * a.dxy + a.offx - a.soff;
  *xhi = (c1 * a.dxy + a.offx - a.soff) + a.scale;
  *ylo = ty0 * a.dxy + a.offy - a.soff;
  *yhi = (r1 * a.dxy + a.offy - a.soff) + a.scale;
}

// A tile's shared point location (locate_region), packed for the map kernel:
// (kind | steps << 2 as unsigned bits, start triangle).  steps <= loc_budget
// = 4 n_tri + 64 < 2^29 + 64 (the launchers cap n_tri below 2^27), so the
// packed value fits in 32 unsigned bits; it is unpacked with unsigned shifts.
template <class Args>
__device__ __forceinline__ int2 tile_location(const Args& a, int tile) {
  int kind = kLocMiss, start = -1, steps = 0;
  if (a.n_tri > 0) {
    double xlo, xhi, ylo, yhi;
    tile_rect(a, tile, &xlo, &xhi, &ylo, &yhi);
    kind = locate_region(a.tri, xlo, xhi, ylo, yhi, a.loc_budget, &start, &steps);
  }
  return make_int2((int)((unsigned)kind | ((unsigned)steps << 2)), start);
}

// One ray's point location from its tile's shared walk l (tile_location):
// where the tile's rectangle straddled a test, the ray resumes the walk from
// triangle 0 at that triangle with the steps already taken counted against
// its budget, so it reaches exactly the tet, triangle and status of its own
// locate64(tri, 0, ...).  A tile that left the hull leaves every ray a miss.
__device__ __forceinline__ int locate_from_tile(const TriRec64* __restrict__ tri, int2 l,
                                                double qx, double qy, int loc_budget,
                                                int* status, int* tri_out = nullptr) {
  const int lk = (int)((unsigned)l.x & 3u);
  if (lk == kLocFound) {
    if (tri_out) *tri_out = l.y;
    *status = kRayOk;
    return __ldg(&tri[l.y].nb.w);
  }
  if (lk == kLocResume)
    return locate64(tri, l.y, qx, qy, loc_budget - (int)((unsigned)l.x >> 2), status, tri_out);
  *status = kRayMiss;
  return -1;
}

// ---------------------------------------------------------------------------
// Accumulators: what a walk does with each crossed tet.

// a10: surface density, src/dtfe.c:356-369.  The chord midpoint must lie
// strictly inside (z0, z1); the linear field there times the chord length is
// added.
struct SurfaceAcc64 {
  double z0, z1;
  double rho;
  __device__ __forceinline__ void visit(double ox, double oy, const double2& xyA, double zA,
                                        double rhoA, double gx, double gy, double gz, double z_in,
                                        double z_out) {
    const double d = z_out - z_in;
    const double zm = d / 2 + z_in;
    if (zm > z0 && zm < z1) {
      const double fixed = rhoA + (gx * (ox - xyA.x)) + (gy * (oy - xyA.y)) - (gz * zA);
      rho += (fixed + gz * zm) * d;
    }
  }
};

// One node's value added into its grid cell, *cell += v, as a reduction
// performed at L2: the thread does not wait for the cell's old value.  Each
// grid column belongs to one thread, and one thread's reductions to one
// address are performed in its program order, so every cell receives exactly
// the additions, in the order and with the roundings, of the reference's
// loop (src/dtfe.c:505-511).
__device__ __forceinline__ void cell_add(double* cell, double v) { atomicAdd(cell, v); }

// This thread's grid column (i: x index, j: y index) in a launch of
// grid_blocks(G) blocks of 128 threads: a block covers 8 x 16 columns and
// each of its warps a 4 x 8 patch, so that a warp's columns are neighbours
// and cross many of the same tets.  False for the columns past the grid.
__device__ __forceinline__ bool grid_column(int G, int* i, int* j) {
  const int tiles_j = (G + 15) >> 4;
  const int ti = (int)blockIdx.x / tiles_j, tj = (int)blockIdx.x - ti * tiles_j;
  const int lane = (int)threadIdx.x & 31, wq = (int)threadIdx.x >> 5;
  *i = ti * 8 + (wq >> 1) * 4 + (lane >> 3);
  *j = tj * 16 + (wq & 1) * 8 + (lane & 7);
  return *i < G && *j < G;
}
inline unsigned grid_blocks(int G) { return (unsigned)(((G + 7) / 8) * ((G + 15) / 16)); }

// a12: 3-D column, src/dtfe.c:489-513.  The field is sampled at the fine z
// nodes inside the chord and added, with weight 1/ss^3, to the column cell.
struct ColumnAcc64 {
  double* col;
  double z0, dzs, w;
  int nzs, ss;
  __device__ __forceinline__ void visit(double ox, double oy, const double2& xyA, double zA,
                                        double rhoA, double gx, double gy, double gz, double z_in,
                                        double z_out) {
    int i0 = (int)ceil((z_in - z0 - dzs / 2.) / dzs);
    i0 = i0 < 0 ? 0 : i0;
    int i1 = (int)ceil((z_out - z0 - dzs / 2.) / dzs);
    i1 = i1 > nzs ? nzs : i1;
    if (i1 > i0) {
      const double fixed = rhoA + gx * (ox - xyA.x) + gy * (oy - xyA.y) - gz * zA;
      for (int is = i0; is < i1; ++is) {
        const int iz = (int)((unsigned)is / (unsigned)ss);
        const double zi = z0 + dzs * is + dzs / 2.;
        cell_add(col + iz, (fixed + gz * zi) * w);
      }
    }
  }
};

struct WalkConf64 {
  double lz;        // slab depth, the ray's direction length
  double dist;      // perturbation step (delta_xy/2)/PERTURB_MAX
  uint64_t seed;    // perturbation stream key
  int max_visits;   // visit budget
};

// ---------------------------------------------------------------------------
// a9 + a10: the tet walk (src/dtfe.c:247-374).  On failure *crossed_out stays 0
// and the status says why; column accumulators keep what they already added,
// as evaluate_3d_ray_on_grid does.  Starts as if it had just left
// a virtual tet through face 0 into `ft`; follows the neighbour across the
// leave face; turns around (swaps enter and leave) when that neighbour is the
// tet it came from; perturbs the ray towards a generator-chosen corner while
// a chosen face has a zero edge sign.
template <class Acc>
__device__ __forceinline__ int walk64(const TetRec64* __restrict__ R, int ft, double ox, double oy,
                                      const WalkConf64& W, uint64_t ray, Acc& acc, int* crossed_out,
                                      int* visits, int max_record) {
  *crossed_out = 0;
  if (ft < 0) return kRayMiss;
  Ray64 ry{W.lz, -W.lz * oy, W.lz * ox};
  uint64_t ctr = 0;
  int crossed = 0;
  int4 nb = make_int4(ft, -1, -1, -1);
  int leave = 0, enter = -1;
  int cur = ft, prev = -1;
  for (;;) {
    int nx = nb_at(nb, leave);
    if (nx == -1) break;
    if (nx == prev) {  // turn around
      const int t = enter;
      enter = leave;
      leave = t;
      nx = nb_at(nb, leave);
      if (nx == -1) break;
    }
    prev = cur;
    cur = nx;
    if (crossed >= W.max_visits) return kRayBudget;

    const TetRec64* rec = R + cur;
    double2 xy[4];
    xy[0] = __ldg(&rec->xy[0]);
    xy[1] = __ldg(&rec->xy[1]);
    xy[2] = __ldg(&rec->xy[2]);
    xy[3] = __ldg(&rec->xy[3]);
    const double2 zab = __ldg(&rec->zab), zcd = __ldg(&rec->zcd);
    const double2 rg0 = __ldg(&rec->rg0), rg1 = __ldg(&rec->rg1);
    nb = __ldg(&rec->nb);
    const double z[4] = {zab.x, zab.y, zcd.x, zcd.y};

    double u[6];
    Hit64 h = ray_tet64(ry, xy, u);
    if (!h.ok) return kRayNoExit;
    int np = 0;
    while (h.special) {  // src/dtfe.c:329-349, perturb_ray at :219-245
      const int r = sdtfe_rand31(W.seed, ray, ctr++) % 4;
      const double2 vr = sel4(r, xy[0], xy[1], xy[2], xy[3]);
      double dx = vr.x - ox;
      double dy = vr.y - oy;
      const double mag = sqrt(dx * dx + dy * dy);
      if (mag > W.dist) {
        dx = dx / mag;
        dy = dy / mag;
        dx = dx * W.dist;
        dy = dy * W.dist;
      }
      ox = ox + dx;
      oy = oy + dy;
      ry.m_oy = -W.lz * oy;
      ry.ox_l = W.lz * ox;
      if (++np > kPerturbMax) return kRayPerturbMax;
      h = ray_tet64(ry, xy, u);
      if (!h.ok) return kRayNoExit;
    }
    enter = h.enter;
    leave = h.leave;
    const double z_in = face_z64(enter, u, z);
    const double z_out = face_z64(leave, u, z);
    if (visits != nullptr && crossed < max_record) visits[crossed] = cur;
    ++crossed;
    acc.visit(ox, oy, xy[0], z[0], rg0.x, rg0.y, rg1.x, rg1.y, z_in, z_out);
  }
  *crossed_out = crossed;
  return kRayOk;
}

}  // namespace sdtfe
