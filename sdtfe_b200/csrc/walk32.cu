// walk32.cu - mixed-precision surface-density map: FP32 walk, guarded FP64.
//
// What stays exact.  The walk's topology (which faces the ray enters and
// leaves, when it perturbs, which tet comes next) depends only on the signs
// of six Plücker products per tet, thresholded at ZERO as the reference does
// (src/dtfe.c:19-21).  Each product is evaluated in FP32 from coordinates
// taken relative to the ray origin (the origin split into a float hi/lo
// pair) together with a bound on its FP32 error.  When every product clears
// the reference's threshold by more than that bound plus the reference's own
// FP64 rounding, all six reference signs are known and nonzero, and the
// reference's enter/leave rule follows from them.  Otherwise the tet is
// re-tested with the reference's FP64 products and operands and the general
// face rule (zero signs, perturbation) applies, exactly as in the FP64 walk.
// Every ray therefore visits the FP64 path's tets in the FP64 path's order.
//
// Two kinds of step.  A tet entered through a face shared with the previous
// tet takes the fast step on its record for that entry face (TetRot32): the
// entry face's vertices sit in fixed slots, so the six products, the exit
// face (closed form, proven equal to the reference's rule by static_assert),
// the exit crossing and the chord need no table and no data-dependent
// indexing beyond picking one of three exit faces.  Anything the fast step
// cannot decide exactly - an uncertain sign, a rule that does not enter
// through the known face, an ill-conditioned or hull crossing whose error
// would matter, a midpoint in the slab's guard band, a tet whose FP32 field
// value is not trusted - goes to the general step (mesh-order record, FP64
// where needed), which also takes the first tet of every ray.
//
// What is FP32.  The crossings and the field value.  The exit crossing's z is
// the apex z plus a barycentric offset (weights = the exit face's signed edge
// products over their sum; same sign, no cancellation), carried into the next
// tet as its entry, so consecutive chords share their interface exactly and
// the chord lengths telescope.  The chord's value is the reference's own
// formula (src/dtfe.c:363-368): the tet's linear field rho + grad.(p - v) at
// the point p of the ray line at the chord's midpoint, here from the apex.
// p is on the line, so an error in a crossing only moves a chord end shared
// with the neighbour, which the continuity of the linear field makes a
// second-order effect.  Tets whose FP32 field value could cancel badly
// (magnitudes over least vertex value above kFieldCond: slivers, extreme
// density contrast) are evaluated from the mesh's FP64 vertex, density and
// gradient in the general step.  Crossing positions and the ray's sum are
// FP64 (a float vertex z plus a float offset, added exactly).  The midpoint-
// in-slab test uses each crossing's error bound; inside that band the
// reference's FP64 midpoint decides.
//
// Compiled with -fmad=false like walk.cu: the sample positions and the point
// location it shares with the FP64 walk must round as the reference does;
// the FP32 arithmetic asks for fused multiply-adds explicitly.
#include <algorithm>
#include <cfloat>
#include <cstring>

#include "mesh.h"

namespace sdtfe {

namespace {

constexpr float kEps = 5.9604645e-08f;  // 2^-24, FP32 unit roundoff

// Error of one FP32 product u = px*qy - py*qx of relative coordinates, in
// units of kEps * dmax^2 (dmax: the tet's largest |relative coordinate|).
// Each relative coordinate (v - o_hi) - o_lo is within 2 kEps dmax (+ a term
// in kEps^2 |o| that e_coef covers) of v - o, which moves the product by at
// most 4 * 2 kEps dmax^2; rounding the product adds at most 4 kEps dmax^2
// (two products and a difference, each rounded once; 3 with a fused
// multiply-add).  16 covers the 12 with a margin.
constexpr float kProdErr = 16.f;

struct MixConf {
  double lz;          // slab depth (the reference's ray length)
  double z0d, z1d;    // slab bounds
  float z0, z1;       // slab bounds rounded to float (compared with a guard band)
  double thr;         // the reference's ZERO in units of lz
  double coord_max;   // largest vertex coordinate magnitude
  double coord_err;   // rounding of the float records (0 when they are exact)
  double dist;        // perturbation step
  uint64_t seed;
  int max_visits;
  const TetRec64* __restrict__ rec64;  // exact coordinates when the floats are not
  int exact32;                         // the float coordinates are the doubles
  const TetRot32* __restrict__ rot;    // records per entry face (NULL: general steps only)
  const signed char* __restrict__ tri_face;  // the tet face under each hull triangle
  const int4* __restrict__ rows;       // the mesh's tetra_data rows (vertex ids, neighbours)
  const double4* __restrict__ pos;     // vertices and their densities, original frame
  const double* __restrict__ grad;     // per-tet gradients, original frame
  int axis;                            // projection axis (frame permutation)
  // Chord midpoints inside (zlo_in, zhi_in) are surely inside the slab for
  // every tet of the mesh; others are tested against their own error bound.
  double zlo_in, zhi_in;
};

struct RayState {
  double ox, oy;     // ray origin (perturbed in place)
  float oxh, oxl, oyh, oyl;
  float thr_hi;      // the reference's threshold plus its own error, in units of lz
  float e_coef;      // error of the products per unit of the tet's largest |relative coordinate|
};

// Float hi/lo split of the origin and this ray's filter constants.  The
// reference's own FP64 error on a product is at most 8 roundings of
// magnitude <= 6*M^2*lz (M: largest coordinate or origin magnitude), i.e.
// 48*2^-53*M^2 in units of lz.  Beyond the relative error of the
// subtractions (kProdErr), a relative coordinate carries at most 3*eps^2*|o|
// from the split plus the records' rounding (e_abs); on a product that is at
// most 2*e_abs*(|px|+|py|+|qx|+|qy|) <= 8*e_abs*Dmax.
__device__ __forceinline__ void ray_setup(RayState& r, const MixConf& C) {
  r.oxh = (float)r.ox;
  r.oxl = (float)(r.ox - (double)r.oxh);
  r.oyh = (float)r.oy;
  r.oyl = (float)(r.oy - (double)r.oyh);
  const double M = fmax(C.coord_max, fmax(fabs(r.ox), fabs(r.oy)));
  const double ref_err = 32.0 * DBL_EPSILON * M * M + 1e-300;
  r.thr_hi = __double2float_ru((C.thr + ref_err) * (1.0 + 1e-5));
  const double eps = 5.9604644775390625e-08;
  const double e_abs = 4.0 * eps * eps * (fabs(r.ox) + fabs(r.oy)) + C.coord_err;
  r.e_coef = __double2float_ru(8.0 * 1.01 * e_abs) + FLT_MIN;
}

struct Verts32 {
  float x[4], y[4];  // absolute (projected frame)
  float z[4];
};

// The general step sees a tet in the mesh's own vertex order A..D: its record
// for entry face 3 (ABC) has exactly that slot order (rot_slot(3, k) = k), and
// the neighbours come from the mesh's tetra_data rows.
__device__ __forceinline__ const TetRot32* mesh_order(const TetRot32* __restrict__ R, int t) {
  return R + 4 * (size_t)t + 3;
}

__device__ __forceinline__ void load32(const TetRot32* __restrict__ R, const int4* __restrict__ rows,
                                       int t, Verts32& v, int4& nb) {
  const TetRot32* p = mesh_order(R, t);
  const float4 a = __ldg(&p->xy01), b = __ldg(&p->xy23), z = __ldg(&p->z);
  nb = __ldg(&rows[2 * (size_t)t + 1]);
  v.x[0] = a.x; v.y[0] = a.y; v.x[1] = a.z; v.y[1] = a.w;
  v.x[2] = b.x; v.y[2] = b.y; v.x[3] = b.z; v.y[3] = b.w;
  v.z[0] = z.x; v.z[1] = z.y; v.z[2] = z.z; v.z[3] = z.w;
}

// Exact double coordinates of vertex k of tet t, fetched from memory (the
// float record when its floats are the doubles, else the FP64 record).
__device__ __forceinline__ double2 xy64_at(const TetRot32* __restrict__ R32,
                                           const TetRec64* __restrict__ R64, int exact32, int t,
                                           int k) {
  if (exact32) {
    const TetRot32* p = mesh_order(R32, t);
    const float4 q = __ldg(k < 2 ? &p->xy01 : &p->xy23);
    return (k & 1) ? make_double2(q.z, q.w) : make_double2(q.x, q.y);
  }
  return __ldg(&R64[t].xy[k]);
}

__device__ __forceinline__ double z64_at(const TetRot32* __restrict__ R32,
                                         const TetRec64* __restrict__ R64, int exact32, int t,
                                         int k) {
  if (exact32) {
    const float4 z = __ldg(&mesh_order(R32, t)->z);
    return (double)sel4(k, z.x, z.y, z.z, z.w);
  }
  const double2 zz = __ldg(k < 2 ? &R64[t].zab : &R64[t].zcd);
  return (k & 1) ? zz.y : zz.x;
}

// The reference's FP64 product for edge P->Q, operands and order as in
// src/dtfe.c:24-26.
__device__ __forceinline__ double edge_u64_exact(double lz, double ox, double oy, double2 p,
                                                 double2 q) {
  const double v0 = __dsub_rn(p.x, q.x);
  const double v1 = __dsub_rn(p.y, q.y);
  const double v5 = __dsub_rn(__dmul_rn(p.x, q.y), __dmul_rn(p.y, q.x));
  const double m_oy = __dmul_rn(-lz, oy);
  const double ox_l = __dmul_rn(lz, ox);
  return __dadd_rn(__dadd_rn(__dmul_rn(lz, v5), __dmul_rn(v0, m_oy)), __dmul_rn(v1, ox_l));
}

// edges CB, AC, BA, DC, BD, DA as P -> Q vertex slots (inside unrolled loops)
#define SDTFE_EDGE_TABLES                       \
  constexpr int kEdgeP[6] = {2, 2, 1, 2, 1, 3}; \
  constexpr int kEdgeQ[6] = {1, 0, 0, 3, 3, 0};

// Slow path: the reference's six signs for tet t, packed 2 bits per edge
// (0: zero, 1: positive, 2: negative).
__device__ __noinline__ unsigned exact_signs(const TetRot32* __restrict__ R32,
                                             const TetRec64* __restrict__ R64, int exact32,
                                             double lz, int t, double ox, double oy) {
  SDTFE_EDGE_TABLES
  double2 xy[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) xy[k] = xy64_at(R32, R64, exact32, t, k);
  unsigned packed = 0;
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const int s = sign_eps(edge_u64_exact(lz, ox, oy, xy[kEdgeP[e]], xy[kEdgeQ[e]]));
    packed |= (unsigned)(s > 0 ? 1 : (s < 0 ? 2 : 0)) << (2 * e);
  }
  return packed;
}

// Face choice from six certain (nonzero) signs.  neg has bit e set when edge e
// (CB, AC, BA, DC, BD, DA) is negative; entry = enter | leave << 2 | ok << 4,
// the reference's first-entered / first-left rule (src/dtfe.c:66-213) with
// faces in the order BDC, ACD, ADB, ABC.
__host__ __device__ constexpr unsigned face_lut_entry(unsigned neg) {
  const bool e0 = (neg & 25u) == 17u, e1 = (neg & 42u) == 40u, e2 = (neg & 52u) == 4u,
             e3 = (neg & 7u) == 2u;
  const bool l0 = (neg & 25u) == 8u, l1 = (neg & 42u) == 2u, l2 = (neg & 52u) == 48u,
             l3 = (neg & 7u) == 5u;
  const int en = e0 ? 0 : (e1 ? 1 : (e2 ? 2 : (e3 ? 3 : -1)));
  const int le = l0 ? 0 : (l1 ? 1 : (l2 ? 2 : (l3 ? 3 : -1)));
  return (en >= 0 && le >= 0) ? ((unsigned)en | (unsigned)le << 2 | 16u) : 0u;
}

struct Hit32 {
  int enter, leave;
  bool ok, special;
};

// The filtered test of one tet.  u[] receives the FP32 products (units of lz).
__device__ __forceinline__ Hit32 tet_test(const TetRot32* __restrict__ R32, const MixConf& C,
                                          const RayState& r, int t, const Verts32& v, float u[6],
                                          float* bmax, const unsigned char* __restrict__ lut,
                                          int* fallbacks) {
  SDTFE_EDGE_TABLES
  float dx[4], dy[4];
  float dmax = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    dx[k] = __fsub_rn(__fsub_rn(v.x[k], r.oxh), r.oxl);
    dy[k] = __fsub_rn(__fsub_rn(v.y[k], r.oyh), r.oyl);
    dmax = fmaxf(dmax, fmaxf(fabsf(dx[k]), fabsf(dy[k])));
  }
  // one bound for the tet's six products: the FP32 error (kProdErr), the
  // records' rounding and the origin split (e_coef), and the reference's
  // threshold plus its own FP64 rounding (thr_hi)
  const float bound = __fmaf_ru(kProdErr * kEps * dmax, dmax, __fmaf_ru(r.e_coef, dmax, r.thr_hi));
  unsigned neg = 0, unc = 0;
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const float px = dx[kEdgeP[e]], py = dy[kEdgeP[e]], qx = dx[kEdgeQ[e]], qy = dy[kEdgeQ[e]];
    const float ue = __fsub_rn(__fmul_rn(px, qy), __fmul_rn(py, qx));
    unc |= (fabsf(ue) <= bound ? 1u : 0u) << e;
    neg |= (__float_as_uint(ue) >> 31) << e;
    u[e] = ue;
  }
  *bmax = bound;
  Hit32 h;
  if (unc == 0) {
    const unsigned ent = lut[neg];
    h.enter = (int)(ent & 3u);
    h.leave = (int)((ent >> 2) & 3u);
    h.ok = (ent & 16u) != 0;
    h.special = false;
    return h;
  }
  // some product is too close to the reference's threshold: the reference decides
  *fallbacks += __popc(unc);
  const unsigned pk = exact_signs(R32, C.rec64, C.exact32, C.lz, t, r.ox, r.oy);
  int s[6];
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const unsigned c = (pk >> (2 * e)) & 3u;
    s[e] = c == 1u ? 1 : (c == 2u ? -1 : 0);
  }
  const Hit64 g = plucker_faces(s);
  h.enter = g.enter;
  h.leave = g.leave;
  h.ok = g.ok;
  h.special = g.special;
  return h;
}

// Where the ray crosses face f (face f lies opposite vertex f): offset of the
// crossing's z from vertex A's z, and the field value there.  Each corner's
// weight is the signed term of the face edge opposite it over their sum.
// Returns a bound on the weights' error (three times the tet's product bound
// over |sum|): large for a face nearly parallel to the ray.
__device__ __forceinline__ float crossing(int f, const float u[6], float bmax, const Verts32& v,
                                          float* dz) {
  // u: CB=0, AC=1, BA=2, DC=3, BD=4, DA=5
  const float wa = sel4(f, 0.f, -u[3], u[4], u[0]);
  const float wb = sel4(f, u[3], 0.f, u[5], -u[1]);
  const float wc = sel4(f, -u[4], -u[5], 0.f, u[2]);
  const float wd = sel4(f, -u[0], u[1], -u[2], 0.f);
  const float den = wa + wb + wc + wd;
  const float r = __fdividef(1.f, den);
  const float zb = v.z[1] - v.z[0], zc = v.z[2] - v.z[0], zd = v.z[3] - v.z[0];
  *dz = r * __fmaf_rn(wd, zd, __fmaf_rn(wc, zc, wb * zb));
  return 3.f * bmax * fabsf(r);
}

// z of the crossing of face f of tet t, computed from the exact operands: the
// reference's FP64 point (face_z64).
// Used where a crossing is not shared with a neighbouring chord (the ray's
// entry into and exit from the mesh, a re-entry after a perturbation or a
// turn-around) and where the FP32 weights are ill-conditioned.
__device__ __noinline__ double exact_crossing(const TetRot32* __restrict__ R32,
                                               const TetRec64* __restrict__ R64, int exact32,
                                               double lz, int t, int f, double ox, double oy) {
  SDTFE_EDGE_TABLES
  double2 xy[4];
  double z[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    xy[k] = xy64_at(R32, R64, exact32, t, k);
    z[k] = z64_at(R32, R64, exact32, t, k);
  }
  double u[6];
#pragma unroll
  for (int e = 0; e < 6; ++e) u[e] = edge_u64_exact(lz, ox, oy, xy[kEdgeP[e]], xy[kEdgeQ[e]]);
  return face_z64(f, u, z);
}

// Weights' relative error above which a crossing is recomputed in FP64
// (2^-10).  With every weight's sign certified the FP32 crossing is a convex
// combination of the face's vertices, so it lies on the face whatever the
// error.  An interior crossing is shared by two chords, and the chord value
// at the midpoint on the ray line makes their sum stationary in it: an error
// delta <= tol * h (h: the face's height above the apex) leaves the second-
// order term (g1' - g2') delta^2 / 2, g' the field's slope along the ray in
// each tet (measured: map errors stay below 1.5e-6 against FP64).  Hull
// crossings and slab-band midpoints carry their bound (e_out) into their own
// tests.
// Nearly edge-on exit faces are the fast step's most common decline: on a
// clustered mesh 0.17 % of visits at 2^-12, 0.03 % at 2^-10.
constexpr float kCrossingTol = 9.765625e-4f;

// The reference's FP64 chord midpoint for the chosen faces (slab-test guard).
__device__ __noinline__ double midpoint64(const TetRot32* __restrict__ R32,
                                          const TetRec64* __restrict__ R64, int exact32, double lz,
                                          int t, int enter, int leave, double ox, double oy) {
  SDTFE_EDGE_TABLES
  double2 xy[4];
  double z[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    xy[k] = xy64_at(R32, R64, exact32, t, k);
    z[k] = z64_at(R32, R64, exact32, t, k);
  }
  double u[6];
#pragma unroll
  for (int e = 0; e < 6; ++e) u[e] = edge_u64_exact(lz, ox, oy, xy[kEdgeP[e]], xy[kEdgeQ[e]]);
  const double zi = face_z64(enter, u, z), zo = face_z64(leave, u, z);
  const double d = zo - zi;
  return d / 2 + zi;
}

// The reference's chord value (src/dtfe.c:363-368) in FP64: the tet's linear
// field rho_A + grad . (p - A) at the point of the ray line at height zmid,
// from the mesh's FP64 vertex, density and gradient.
__device__ __noinline__ double field64(const MixConf& C, int t, double ox, double oy, double zmid) {
  const int4 v = __ldg(&C.rows[2 * (size_t)t]);
  const double4 A = C.pos[v.x];
  double ax, ay, az, gx, gy, gz;
  permute3(C.axis, A.x, A.y, A.z, &ax, &ay, &az);
  permute3(C.axis, C.grad[3 * (size_t)t], C.grad[3 * (size_t)t + 1], C.grad[3 * (size_t)t + 2], &gx,
           &gy, &gz);
  return A.w + gx * (ox - ax) + gy * (oy - ay) + gz * (zmid - az);
}

// One chord's contribution: the field at its midpoint on the ray line times
// its length, when the midpoint lies in the slab (src/dtfe.c:356-369).  Crossing positions are
// doubles (a float vertex z plus a float offset, summed exactly), so the exit
// of one chord is bit-for-bit the entry of the next and the chord lengths
// telescope.  The slab test compares the float midpoint with a guard band;
// inside the band the reference's FP64 midpoint decides.
__device__ __forceinline__ double chord32(const TetRot32* __restrict__ R, const MixConf& C,
                                          const RayState& r, int t, int enter, int leave,
                                          double z_in, double z_out, float hz, float e_inout,
                                          int* fallbacks) {
  const double d = z_out - z_in;
  const double zmid = z_in + 0.5 * d;
  const float zm = (float)zmid;
  // float rounding of the midpoint plus the crossings' own error bounds
  const float guard = 64.f * kEps * (fabsf(zm) + hz) + e_inout;
  bool inside;
  if (fabsf(zm - C.z0) > guard && fabsf(zm - C.z1) > guard) {
    inside = zm > C.z0 && zm < C.z1;
  } else {
    const double zmd = midpoint64(R, C.rec64, C.exact32, C.lz, t, enter, leave, r.ox, r.oy);
    inside = zmd > C.z0d && zmd < C.z1d;
    ++*fallbacks;
  }
  if (!inside) return 0.0;
  ++*fallbacks;
  return field64(C, t, r.ox, r.oy, zmid) * d;
}

// The reference's rule seen from a rotated record: for entry face F and the
// sign bits of the rotated products (e01, e12, e20, a0, a1, a2 = u(0,1),
// u(1,2), u(2,0), u(3,0), u(3,1), u(3,2)), the rotated slot k (0..2) whose
// opposite face the ray leaves through, with bit 2 set, when the reference's
// rule (face_lut_entry on the products in the mesh's own edge order) enters
// through F; 0 otherwise.  A product of a reversed edge is the exact negative
// (the reference's formula is antisymmetric in its two vertices), so the
// mesh-order signs follow from the rotated ones.
__host__ __device__ constexpr unsigned rot_lut_entry(int F, unsigned neg_rot) {
  // rotated pair (p, q) -> product index j and reversal
  unsigned neg = 0;
  for (int e = 0; e < 6; ++e) {
    constexpr int P[6] = {2, 2, 1, 2, 1, 3}, Q[6] = {1, 0, 0, 3, 3, 0};  // kEdgeP / kEdgeQ
    const int p = rot_inv(F, P[e]), q = rot_inv(F, Q[e]);
    int j = 0;
    bool rev = false;
    if (p == 3 || q == 3) {  // apex edge: a_k = u(3, k)
      j = 3 + (p == 3 ? q : p);
      rev = q == 3;
    } else if ((p + 1) % 3 == q) {  // face edge in cyclic order: u(0,1), u(1,2), u(2,0)
      j = p;
    } else {
      j = q;
      rev = true;
    }
    neg |= (((neg_rot >> j) & 1u) ^ (rev ? 1u : 0u)) << e;
  }
  const unsigned ent = face_lut_entry(neg);
  if (!(ent & 16u)) return 0u;
  const int enter = (int)(ent & 3u), leave = (int)((ent >> 2) & 3u);
  if (enter != F || leave == F) return 0u;
  return (unsigned)rot_inv(F, leave) | 4u;
}

// The same rule in closed form, the same for every F (the four rotations
// list their faces with one orientation): the three entry-face products are
// negative, and the ray leaves through the face opposite the slot k with
// a(k+1) < 0 and a(k+2) > 0.
__host__ __device__ constexpr unsigned rot_exit_rule(unsigned neg_rot) {
  if ((neg_rot & 7u) != 7u) return 0u;
  const bool n0 = (neg_rot >> 3) & 1u, n1 = (neg_rot >> 4) & 1u, n2 = (neg_rot >> 5) & 1u;
  return (n1 && !n2) ? 4u : ((n2 && !n0) ? 5u : ((n0 && !n1) ? 6u : 0u));
}

constexpr bool exit_rule_is_the_reference_rule() {
  for (int F = 0; F < 4; ++F)
    for (unsigned v = 0; v < 64; ++v)
      if (rot_lut_entry(F, v) != rot_exit_rule(v)) return false;
  return true;
}
static_assert(exit_rule_is_the_reference_rule(), "fast-step exit rule differs from the reference's");

template <class T>
__device__ __forceinline__ T sel3(int k, T a, T b, T c) {
  return k == 0 ? a : (k == 1 ? b : c);
}

struct FastStep {
  double z_out;    // exit crossing
  float e_out;     // bound on the exit crossing's z error
  int next;        // record of the next tet; -1: the ray left the mesh here
};

// ---------------------------------------------------------------------------
// What a walk does with each crossed tet.  An accumulator provides
//   fast(...)        the fast step's chord, from the FP32 exit crossing and the
//                    record's field; false declines the step (nothing committed)
//   exact_exit(...)  whether the general step must recompute an FP32 exit
//                    crossing exactly before its chord
//   enter(z)         a ray's entry crossing was computed exactly
//   general(...)     the general step's chord (FP64 field values)
//   carry(leave)     the next tet is entered through this tet's leave face
//                    (true) or, after a turn-around, its enter face (false)

// Surface density (src/dtfe.c:356-369): the chord's value at its midpoint
// times its length, when the midpoint lies strictly inside the slab.
struct SurfaceAcc32 {
  double sum = 0.0;

  // The slab test compares the midpoint with a guard band (the crossings'
  // error bounds); inside the band the step declines and the reference's FP64
  // midpoint decides.  The chord value is the reference's own formula
  // (src/dtfe.c:363-368) from the apex: the tet's linear field
  // rho3 + grad . (p - v3) at the point p of the ray line at the chord's
  // midpoint.  p lies on the line, so errors of the crossings only move chord
  // ends, shared with the neighbours: they cancel to first order.
  // fld = (rho3, grad_x, grad_y, grad_z); (x3, y3) = v3 - origin.  An exit
  // through the hull (next == -1) is declined unless the error its FP32
  // crossing can add to the chord is below 1e-7 of the ray's integral: such a
  // crossing is not shared with a neighbouring chord, so its error does not
  // cancel.
  __device__ __forceinline__ bool fast(const MixConf& C, const RayState&, int, double z_in,
                                       float e_in, double z_out, float e_out, int next,
                                       const float4& f, float x3, float y3, float zw) {
    const double d = z_out - z_in;
    const double zm = z_in + 0.5 * d;
    bool inside = true;
    if (!(zm > C.zlo_in && zm < C.zhi_in)) {  // near a slab bound: this chord's own guard
      const float g = 64.f * kEps * fabsf((float)zm) + e_in + e_out;
      const float d0 = (float)(zm - C.z0d), d1 = (float)(zm - C.z1d);
      if (!(fabsf(d0) > g && fabsf(d1) > g)) return false;  // the reference's midpoint decides
      inside = d0 > 0.f && d1 < 0.f;
    }
    const float zr = (float)(zm - (double)zw);
    const float g = __fmaf_rn(f.w, zr, __fmaf_rn(-f.z, y3, __fmaf_rn(-f.y, x3, f.x)));
    const double contrib = inside ? (double)g * d : 0.0;
    if (next == -1 && inside) {
      // the exit crossing's z error times the field is not cancelled: at most
      // about 1.7e-7 of the ray's integral (5/3 e_out)
      if (!(fabsf(g) * e_out <= 1e-7f * (float)fabs(sum + contrib))) return false;
    }
    sum += contrib;
    return true;
  }
  __device__ __forceinline__ bool exact_exit(double, float) const { return false; }
  __device__ __forceinline__ void enter(double) {}
  __device__ __forceinline__ void carry(bool) {}
  __device__ __forceinline__ void general(const TetRot32* __restrict__ R, const MixConf& C,
                                          const RayState& r, int t, int enter, int leave,
                                          double z_in, double z_out, float hz, float e_inout,
                                          int* fallbacks) {
    sum += chord32(R, C, r, t, enter, leave, z_in, z_out, hz, e_inout, fallbacks);
  }
};

// One walk step on the record of (tet, entry face), for a ray whose entry
// crossing (z_in, f_in) was carried over from the previous tet.  Succeeds
// when the FP32 products decide all six reference signs, the reference's rule
// enters through the known face and the accumulator takes the chord
// (SurfaceAcc32: the midpoint is clear of the slab bounds); otherwise nothing
// is committed and the general step takes the tet.  The step also declines an
// ill-conditioned exit crossing; the general step computes it exactly.
template <class Acc>
__device__ __forceinline__ bool fast_step(const MixConf& C, const RayState& r, int ri,
                                          double z_in, float e_in, Acc& acc, FastStep* o) {
  const TetRot32* p = C.rot + ri;
  const float4 a = __ldg(&p->xy01), b = __ldg(&p->xy23), z = __ldg(&p->z), f = __ldg(&p->fld);
  const int4 nb = __ldg(&p->nb);
  const float x0 = __fsub_rn(__fsub_rn(a.x, r.oxh), r.oxl), y0 = __fsub_rn(__fsub_rn(a.y, r.oyh), r.oyl);
  const float x1 = __fsub_rn(__fsub_rn(a.z, r.oxh), r.oxl), y1 = __fsub_rn(__fsub_rn(a.w, r.oyh), r.oyl);
  const float x2 = __fsub_rn(__fsub_rn(b.x, r.oxh), r.oxl), y2 = __fsub_rn(__fsub_rn(b.y, r.oyh), r.oyl);
  const float x3 = __fsub_rn(__fsub_rn(b.z, r.oxh), r.oxl), y3 = __fsub_rn(__fsub_rn(b.w, r.oyh), r.oyl);
  // The line crossed the entry face (the previous step decided its signs), so
  // the origin lies in the tet's projection and no |relative coordinate|
  // exceeds the record's extent: the bound of tet_test with that for dmax.
  const float dmax = __int_as_float(nb.w & 0x7fffffff);
  const float bound = __fmaf_ru(kProdErr * kEps * dmax, dmax, __fmaf_ru(r.e_coef, dmax, r.thr_hi));
  const float e01 = __fmaf_rn(x0, y1, -__fmul_rn(y0, x1));
  const float e12 = __fmaf_rn(x1, y2, -__fmul_rn(y1, x2));
  const float e20 = __fmaf_rn(x2, y0, -__fmul_rn(y2, x0));
  const float a0 = __fmaf_rn(x3, y0, -__fmul_rn(y3, x0));
  const float a1 = __fmaf_rn(x3, y1, -__fmul_rn(y3, x1));
  const float a2 = __fmaf_rn(x3, y2, -__fmul_rn(y3, x2));
  const float umin = fminf(fminf(fminf(fabsf(e01), fabsf(e12)), fminf(fabsf(e20), fabsf(a0))),
                           fminf(fabsf(a1), fabsf(a2)));
  // every sign certain, and the reference's rule (rot_exit_rule) enters here;
  // sign-bit arithmetic, so that the only branch is the decline
  const unsigned n0 = __float_as_uint(a0) >> 31, n1 = __float_as_uint(a1) >> 31,
                 n2 = __float_as_uint(a2) >> 31;
  const unsigned k0 = n1 & ~n2, k1 = n2 & ~n0, k2 = n0 & ~n1;
  // (sign bit of nb.w: the tet's FP32 field value is not trusted)
  const unsigned ok = (__float_as_uint(e01) & __float_as_uint(e12) & __float_as_uint(e20) &
                       ~(unsigned)nb.w) >> 31 &
                      (k0 | k1 | k2) & (umin > bound ? 1u : 0u);
  if (!ok) return false;
  // The exit slot k is one-hot in (k0, k1, k2) (exactly one is set once ok
  // holds); every choice below picks by those bits with masks, so that lanes
  // leaving through different faces stay on one instruction stream.
  const unsigned m0 = 0u - k0, m1 = 0u - k1, m2 = 0u - k2;
  const auto pick = [m0, m1, m2](float a, float b, float c) {
    return __uint_as_float((__float_as_uint(a) & m0) | (__float_as_uint(b) & m1) |
                           (__float_as_uint(c) & m2));
  };
  const int next = (int)(((unsigned)nb.x & m0) | ((unsigned)nb.y & m1) | ((unsigned)nb.z & m2));
  if (next < -1) return false;  // a neighbour that does not list this tet
  // exit face: apex (slot 3) and slots i = k+1, j = k+2 (mod 3); the weight of
  // each corner is the product of the face edge opposite it
  const float w3 = pick(e12, e20, e01);
  const float wi = -pick(a2, a0, a1);
  const float wj = pick(a1, a2, a0);
  const float zi = pick(z.y, z.z, z.x), zj = pick(z.z, z.x, z.y);
  const float den = w3 + wi + wj;
  const float rr = __fdividef(1.f, den);
  const float cond = 3.f * bound * fabsf(rr);  // relative error of the weights
  const float hi = zi - z.w, hj = zj - z.w;
  if (!(cond <= kCrossingTol)) return false;  // ill-conditioned
  const float dzr = rr * __fmaf_rn(wj, hj, wi * hi);
  // z error: the weights' error over the face's height above the apex, plus
  // the rounding of the offset (the double sum with the apex z is exact).
  // The weights' error enters the offset's numerator and its denominator, so
  // the crossing is within 5/3 e_out (and the rounding) of the exact one; the
  // slab test compares the midpoint, whose error is at most half of
  // e_in + e_out times 5/3, with the whole of e_in + e_out.
  const float e_out = (cond + 8.f * kEps) * fmaxf(fabsf(hi), fabsf(hj));
  const double z_out = (double)z.w + (double)dzr;
  if (!acc.fast(C, r, ri >> 2, z_in, e_in, z_out, e_out, next, f, x3, y3, z.w)) return false;
  o->z_out = z_out;
  o->e_out = e_out;
  o->next = next;
  return true;
}

// Record of the neighbour across face m of tet t, as entered from t (-1: none).
__device__ __forceinline__ int rot_next(const MixConf& C, int t, int m) {
  if (!C.rot) return -1;
  const int G = m == 0 ? 1 : 0;  // a record of t whose entry face is not m
  const int4 nb = __ldg(&C.rot[4 * (size_t)t + G].nb);
  const int v = sel3(rot_inv(G, m), nb.x, nb.y, nb.z);
  return v >= 0 ? v : -1;
}

// 3-D grid column (src/dtfe.c:465-513): the tet's linear field is sampled at
// the fine z nodes inside each chord and added, with weight 1/ss^3, to the
// node's cell of the column.  Node k sits at z0 + dzs k + dzs/2; a chord
// [z_in, z_out] holds the nodes from the reference's index of z_in up to,
// not including, that of z_out (clamped to [0, nzs)).  Which chord a node
// belongs to must be the FP64 path's: the entry crossing is shared with the
// previous chord, so the index carried from there is used, and an FP32 exit
// crossing whose error band holds a node is recomputed exactly (the fast
// step declines; the general step asks for the exact crossing).  Nodes of
// the hull exit always use the exact crossing.  Node values are FP64: a
// point value has no neighbouring chord to cancel its error against, and the
// FP32 linear field loses up to the tet's density contrast in relative
// precision, so the fast step evaluates the per-tet FP64 field k_field64
// built (k + gx x + gy y + gz z) and the general step the reference's own
// expression from vertex A.
struct ColumnAcc32 {
  double* col;          // the column's cells (z fastest)
  const double4* __restrict__ fld;  // per-tet FP64 field (mesh_field64)
  double z0, dzs, inv_dzs, w;
  int nzs, ss;
  int i_in;             // index of the first node of the next chord (clamped to [-1, nzs + 1])
  int i_out;            // the general step's exit index

  // the reference's index expression (src/dtfe.c:493-496), kept in int range
  __device__ __forceinline__ int node_index(double z) const {
    const double t = ceil((z - z0 - dzs / 2.) / dzs);
    return (int)fmin(fmax(t, -1.0), (double)nzs + 1.0);
  }
  // True when a node with an index in [0, nzs) may lie on the other side of
  // an FP32 crossing z (error bound e, 5/3 e and the FP64 rounding covered
  // by 2e plus 64 ulps).  *t receives the node coordinate of z.
  __device__ __forceinline__ bool near_node(double z, float e, double* t) const {
    *t = (z - z0 - dzs / 2.) * inv_dzs;
    const double fl = floor(*t);
    const double band = (2.0 * (double)e + 64.0 * DBL_EPSILON * (fabs(z) + fabs(z0) + dzs)) * inv_dzs;
    return fl >= -1.0 && fl < (double)nzs && (*t - fl <= band || fl + 1.0 - *t <= band);
  }
  __device__ __forceinline__ bool fast(const MixConf&, const RayState& r, int t, double,
                                       float, double z_out, float e_out, int next, const float4&,
                                       float, float, float) {
    if (next < 0) return false;  // the hull exit: its crossing is computed exactly
    double tz;
    if (near_node(z_out, e_out, &tz)) return false;
    // away from the band tz's ceiling is the reference's index of z_out
    const int i1u = (int)fmin(fmax(ceil(tz), -1.0), (double)nzs + 1.0);
    const int i0 = i_in < 0 ? 0 : i_in, i1 = i1u > nzs ? nzs : i1u;
    if (i1 > i0) {
      const double2 kx = __ldg(reinterpret_cast<const double2*>(fld + t));
      const double2 yz = __ldg(reinterpret_cast<const double2*>(fld + t) + 1);
      const double base = kx.x + kx.y * r.ox + yz.x * r.oy;
      for (int is = i0; is < i1; ++is) {
        const int iz = (int)((unsigned)is / (unsigned)ss);
        const double zi = z0 + dzs * is + dzs / 2.;
        cell_add(col + iz, (base + yz.y * zi) * w);
      }
    }
    i_in = i1u;
    return true;
  }
  __device__ __forceinline__ bool exact_exit(double z_out, float e_out) const {
    double t;
    return near_node(z_out, e_out, &t);
  }
  __device__ __forceinline__ void enter(double z_in) { i_in = node_index(z_in); }
  __device__ __forceinline__ void carry(bool through_leave) {
    if (through_leave) i_in = i_out;  // else the enter face's index, already in i_in
  }
  __device__ __forceinline__ void general(const TetRot32* __restrict__, const MixConf& C,
                                          const RayState& r, int t, int, int, double, double z_out,
                                          float, float, int* fallbacks) {
    i_out = node_index(z_out);
    const int i0 = i_in < 0 ? 0 : i_in, i1 = i_out > nzs ? nzs : i_out;
    if (i1 <= i0) return;
    // the reference's FP64 value (src/dtfe.c:498-512), grid along z (no permutation)
    const int4 v = __ldg(&C.rows[2 * (size_t)t]);
    const double4 A = C.pos[v.x];
    const double gx = C.grad[3 * (size_t)t], gy = C.grad[3 * (size_t)t + 1],
                 gz = C.grad[3 * (size_t)t + 2];
    const double fixed = A.w + gx * (r.ox - A.x) + gy * (r.oy - A.y) - gz * A.z;
    for (int is = i0; is < i1; ++is) {
      const int iz = (int)((unsigned)is / (unsigned)ss);
      const double zi = z0 + dzs * is + dzs / 2.;
      cell_add(col + iz, (fixed + gz * zi) * w);
    }
    ++*fallbacks;
  }
};

// State of one ray between steps.
template <class Acc>
struct WalkState {
  RayState r;
  Acc acc;
  double z_in;
  float e_in;        // bound on z_in's error
  uint64_t ctr;      // perturbation draws so far
  int crossed, fallbacks, cur, prev, ri;
  bool carried;      // z_in holds the crossing of the face shared with prev
};

constexpr int kWalkOn = -1;  // general_step: the walk continues

// The general step on tet w.cur (src/dtfe.c:300-372): the mesh-order record,
// the filtered test with the reference's FP64 signs as fallback, perturbation,
// the chord, and the move through the leave face, or through the enter face
// when the leave face leads back to the previous tet (the reference's
// turn-around).  The crossing of the face passed through is carried on.
// Returns kWalkOn, or the ray's final status.  Kept out of line: it runs on
// about one step in a hundred and would otherwise crowd the fast loop's
// registers.
template <class Acc>
__device__ __noinline__ int general_step(const TetRot32* __restrict__ R, const MixConf& C,
                                         uint64_t ray, const unsigned char* __restrict__ lut,
                                         WalkState<Acc>& w, int* visits, int max_record) {
  RayState& r = w.r;
  const int cur = w.cur;
  int4 nb;
  Verts32 v;
  load32(R, C.rows, cur, v, nb);
  float u[6], bmax;
  Hit32 h = tet_test(R, C, r, cur, v, u, &bmax, lut, &w.fallbacks);
  if (!h.ok) return kRayNoExit;
  int np = 0;
  while (h.special) {  // FP64 perturbation, exactly as the reference (src/dtfe.c:219-245)
    const int k = sdtfe_rand31(C.seed, ray, w.ctr++) % 4;
    const double2 vk = xy64_at(R, C.rec64, C.exact32, cur, k);
    double dx = __dsub_rn(vk.x, r.ox);
    double dy = __dsub_rn(vk.y, r.oy);
    const double mag = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
    if (mag > C.dist) {
      dx = __ddiv_rn(dx, mag);
      dy = __ddiv_rn(dy, mag);
      dx = __dmul_rn(dx, C.dist);
      dy = __dmul_rn(dy, C.dist);
    }
    r.ox = __dadd_rn(r.ox, dx);
    r.oy = __dadd_rn(r.oy, dy);
    ray_setup(r, C);
    w.carried = false;  // the ray moved: this tet computes its own entry
    if (++np > kPerturbMax) return kRayPerturbMax;
    h = tet_test(R, C, r, cur, v, u, &bmax, lut, &w.fallbacks);
    if (!h.ok) return kRayNoExit;
  }
  const int enter = h.enter, leave = h.leave;
  if (visits != nullptr && w.crossed < max_record) visits[w.crossed] = cur;
  ++w.crossed;

  // entry crossing: carried over from the previous chord, or computed from
  // the exact operands where it is not shared (first tet, perturbation,
  // turn-around)
  if (!w.carried || nb_at(nb, enter) != w.prev) {
    w.z_in = exact_crossing(R, C.rec64, C.exact32, C.lz, cur, enter, r.ox, r.oy);
    w.e_in = 0.f;
    w.acc.enter(w.z_in);
    ++w.fallbacks;
  }
  // exit crossing: FP32 unless it leaves the mesh (not shared with a
  // neighbouring chord), is ill-conditioned, or the accumulator needs it exact
  float dzo, e_out = 0.f;
  double z_out;
  const float cond = crossing(leave, u, bmax, v, &dzo);
  const float hz = fmaxf(fmaxf(fabsf(v.z[1] - v.z[0]), fabsf(v.z[2] - v.z[0])),
                         fabsf(v.z[3] - v.z[0]));
  bool exact_out = nb_at(nb, leave) == -1 || !(cond <= kCrossingTol);
  if (!exact_out) {
    z_out = (double)v.z[0] + (double)dzo;
    e_out = (cond + 8.f * kEps) * hz;
    exact_out = w.acc.exact_exit(z_out, e_out);
  }
  if (exact_out) {
    z_out = exact_crossing(R, C.rec64, C.exact32, C.lz, cur, leave, r.ox, r.oy);
    e_out = 0.f;
    ++w.fallbacks;
  }
  w.acc.general(R, C, r, cur, enter, leave, w.z_in, z_out, hz, w.e_in + e_out, &w.fallbacks);

  // move on (src/dtfe.c:300-309)
  int m = leave;
  int nx = nb_at(nb, leave);
  if (nx == w.prev) {
    m = enter;
    nx = nb_at(nb, enter);
  }
  if (nx == -1) return kRayOk;
  if (m == leave) {
    w.z_in = z_out;
    w.e_in = e_out;
  }  // else the enter face's crossing, already in z_in
  w.acc.carry(m == leave);
  w.carried = true;
  w.ri = rot_next(C, cur, m);
  w.prev = cur;
  w.cur = nx;
  return kWalkOn;
}

// The mixed walk.  Same control flow as walk64 (src/dtfe.c:247-374); returns
// the status and the crossing count, and hands each crossed tet's chord to
// the accumulator.  A tet entered through a known face, with the crossing
// there in hand, takes the fast step on its record for that entry face; any
// tet the fast step declines takes the general step.  The first tet is
// entered through the hull triangle the sample was located in (ft_tri; its
// face is known from the hull build), at the exact crossing.
template <class Acc>
__device__ __forceinline__ int walk_mixed(const TetRot32* __restrict__ R, const MixConf& C, int ft,
                                          int ft_tri, double x, double y, uint64_t ray,
                                          const unsigned char* __restrict__ lut, Acc& acc,
                                          int* crossed_out, int* fallbacks_out, int* visits,
                                          int max_record) {
  *crossed_out = 0;
  *fallbacks_out = 0;
  if (ft < 0) return kRayMiss;
  RayState r;
  r.ox = x;
  r.oy = y;
  ray_setup(r, C);
  uint64_t ctr = 0;
  double z_in = 0.0;
  float e_in = 0.f;
  bool carried = false;
  int crossed = 0, fallbacks = 0;
  int cur = ft, prev = -1;
  int ri = -1;  // cur's record for its entry face (-1: general step)
  int status = kWalkOn;
  if (C.rot && ft_tri >= 0) {  // enter through the located hull face, exactly
    const int F = C.tri_face[ft_tri];
    z_in = exact_crossing(R, C.rec64, C.exact32, C.lz, ft, F, r.ox, r.oy);
    acc.enter(z_in);
    ++fallbacks;
    carried = true;
    ri = 4 * ft + F;
  }
  for (;;) {
    if (crossed >= C.max_visits) {
      status = kRayBudget;
      break;
    }
    if (ri >= 0) {
      FastStep o;
      if (fast_step(C, r, ri, z_in, e_in, acc, &o)) {
        if (visits != nullptr && crossed < max_record) visits[crossed] = cur;
        ++crossed;
        if (o.next < 0) {  // left the mesh
          status = kRayOk;
          break;
        }
        z_in = o.z_out;
        e_in = o.e_out;
        prev = cur;
        ri = o.next;
        cur = ri >> 2;
        continue;
      }
    }
    WalkState<Acc> w;
    w.r = r;
    w.acc = acc;
    w.z_in = z_in;
    w.e_in = e_in;
    w.ctr = ctr;
    w.crossed = crossed;
    w.fallbacks = fallbacks;
    w.cur = cur;
    w.prev = prev;
    w.ri = -1;
    // the first tet decides its own entry face (its exact crossing is recomputed)
    w.carried = carried && crossed > 0;
    status = general_step(R, C, ray, lut, w, visits, max_record);
    r = w.r;
    acc = w.acc;
    z_in = w.z_in;
    e_in = w.e_in;
    ctr = w.ctr;
    crossed = w.crossed;
    fallbacks = w.fallbacks;
    cur = w.cur;
    prev = w.prev;
    ri = w.ri;
    carried = w.carried;
    if (status != kWalkOn) break;
  }
  // as the reference (and walk64): a ray that fails reports no crossings, so
  // that the pixel mean leaves it out
  *crossed_out = status == kRayOk ? crossed : 0;
  *fallbacks_out = fallbacks;
  return status;
}

// The surface-density walk: the ray's integral in *rho_out (0 unless the
// ray's status is kRayOk).
__device__ __forceinline__ int walk32(const TetRot32* __restrict__ R, const MixConf& C, int ft,
                                      int ft_tri, double x, double y, uint64_t ray,
                                      const unsigned char* __restrict__ lut, double* rho_out,
                                      int* crossed_out, int* fallbacks_out, int* visits,
                                      int max_record) {
  SurfaceAcc32 acc;
  const int status = walk_mixed(R, C, ft, ft_tri, x, y, ray, lut, acc, crossed_out, fallbacks_out,
                                visits, max_record);
  *rho_out = status == kRayOk ? acc.sum : 0.0;
  return status;
}

// Shared-memory table of the general step: the face rule on 64 sign patterns.
constexpr int kLutBytes = 64;

__device__ __forceinline__ void fill_lut(unsigned char* lut) {
  for (int i = threadIdx.x; i < kLutBytes; i += blockDim.x) lut[i] = (unsigned char)face_lut_entry(i);
}

struct MapArgs32 {
  const TetRot32* __restrict__ rec;
  const TriRec64* __restrict__ tri;
  int n_tri;
  double* __restrict__ map;
  int G, S, TW, TH, tiles_x;
  double dxy, offx, offy, scale, soff;
  MixConf C;
  int loc_budget;
  unsigned long long* __restrict__ stats;
  double* __restrict__ ray_rho;
  int* __restrict__ ray_crossed;
  int* __restrict__ ray_status;
};

// One job of a batch launch: a range of one map's tiles.
struct BatchJob32 {
  MapArgs32 args;
  long long first;  // first global tile of the job
  int tile0;        // the job's first tile within its map
  int count;        // tiles of this job
};

__device__ __forceinline__ void add_stats32(unsigned long long* stats, bool active, int crossed,
                                            int status, int fallbacks) {
  const unsigned mask = __activemask();
  const unsigned rr = __reduce_add_sync(mask, active ? 1u : 0u);
  const unsigned vv = __reduce_add_sync(mask, active ? (unsigned)crossed : 0u);
  const unsigned fb = __reduce_add_sync(mask, active ? (unsigned)fallbacks : 0u);
  unsigned st[DTFE_N_RAY_STATUS];
#pragma unroll
  for (int k = 0; k < DTFE_N_RAY_STATUS; ++k)
    st[k] = __reduce_add_sync(mask, (active && status == k) ? 1u : 0u);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) {
    if (rr) atomicAdd(stats + kStatRays, (unsigned long long)rr);
    if (vv) atomicAdd(stats + kStatVisits, (unsigned long long)vv);
    if (fb) atomicAdd(stats + kStatFallback, (unsigned long long)fb);
#pragma unroll
    for (int k = 0; k < DTFE_N_RAY_STATUS; ++k)
      if (st[k]) atomicAdd(stats + kStatStatus0 + k, (unsigned long long)st[k]);
  }
}

// One tile of one map: TW x TH pixels x S samples on BLOCK threads, one ray
// per (pixel, sample), the S rays of a pixel in neighbouring lanes; the pixel
// means are formed in sample order from shared memory (src/dtfe.c:615-645).
// Point location (src/dtfe.c:518-552) starts from the tile's shared walk
// (*loc, from tile_location): a ray resumes the walk from triangle 0 where
// the tile's rectangle straddled a test, so it reaches exactly the triangle
// and status of its own walk.
template <int BLOCK>
__device__ __forceinline__ void map_tile32(const MapArgs32& a, int tile,
                                           const int2* __restrict__ loc,
                                           const unsigned char* __restrict__ lut, double* s_val,
                                           unsigned char* s_ok) {
  const int P = a.TW * a.TH;
  const int tx0 = (tile % a.tiles_x) * a.TW, ty0 = (tile / a.tiles_x) * a.TH;
  for (int t = threadIdx.x; t < P * a.S; t += BLOCK) {
    const int lp = t / a.S, s = t % a.S;
    const int col = tx0 + lp % a.TW, row = ty0 + lp / a.TW;
    const bool active = col < a.G && row < a.G;
    double v = 0.0;
    int crossed = 0, status = kRayMiss, fb = 0;
    if (active) {
      const long long p = (long long)row * a.G + col;
      const double x = col * a.dxy + a.offx - a.soff;
      const double y = row * a.dxy + a.offy - a.soff;
      const double xt = x + sdtfe_sample_u01(a.C.seed, (uint64_t)p, (uint32_t)s, 0) * a.scale;
      const double yt = y + sdtfe_sample_u01(a.C.seed, (uint64_t)p, (uint32_t)s, 1) * a.scale;
      const uint64_t rid = (uint64_t)p * (uint64_t)a.S + (uint64_t)s;
      int ft_tri = -1;
      int ft = locate_from_tile(a.tri, __ldg(loc), xt, yt, a.loc_budget, &status, &ft_tri);
      if (ft >= 0)
        status = walk32(a.rec, a.C, ft, ft_tri, xt, yt, rid, lut, &v, &crossed, &fb, nullptr, 0);
      if (status != kRayOk) v = 0.0;
      if (a.ray_rho) {
        a.ray_rho[rid] = v;
        a.ray_crossed[rid] = crossed;
        a.ray_status[rid] = status;
      }
    }
    s_val[t] = v;
    s_ok[t] = crossed > 0;
    add_stats32(a.stats, active, crossed, status, fb);
  }
  __syncthreads();
  for (int lp = threadIdx.x; lp < P; lp += BLOCK) {
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

// One block per tile.  BLOCK threads per block and MINB blocks per SM (the
// register budget) are compile-time; the autotuner picks among the
// instantiations.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_map32(const __grid_constant__ MapArgs32 a, const int2* __restrict__ loc) {
  extern __shared__ double s_val32[];  // P*S doubles, then P*S success bytes
  __shared__ unsigned char s_lut[kLutBytes];
  fill_lut(s_lut);
  __syncthreads();
  unsigned char* s_ok = reinterpret_cast<unsigned char*>(s_val32 + a.TW * a.TH * a.S);
  map_tile32<BLOCK>(a, blockIdx.x, loc + blockIdx.x, s_lut, s_val32, s_ok);
}

// Every tile's shared point location, one thread per tile, before the map
// kernel: the walk from triangle 0 runs once per tile, off the rays' path.
__global__ void __launch_bounds__(128) k_locate_map32(const __grid_constant__ MapArgs32 a,
                                                      int n_tiles, int2* __restrict__ loc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n_tiles) loc[t] = tile_location(a, t);
}

// Persistent batch: the blocks of one launch pull tiles from a device counter
// across every job of the batch (maps of different meshes, sides and sample
// counts), so uneven maps share the GPU without a tail per map.  Job j owns
// global tiles [first[j], first[j+1]) and maps them to its own tiles
// [tile0, tile0 + count).  The job table travels as the kernel's own
// parameter (up to kMaxJobsPerLaunch32 jobs; larger batches are launched in
// chunks): a tile's job is found by a binary search over the table with a
// block-uniform index, and the walk reads its job's fields from the constant
// bank as k_map32 reads its single map's, instead of holding them in
// registers.  Thread 0 claims the next tile while the block walks the current
// one, so the claim's latency is hidden.
constexpr int kMaxJobsPerLaunch32 = 96;
struct BatchTable32 {
  int n_jobs;
  long long total_tiles;
  BatchJob32 jobs[kMaxJobsPerLaunch32];
};
static_assert(sizeof(BatchTable32) <= 32764, "the job table must fit the kernel parameter space");

__device__ __forceinline__ int job_of(const BatchTable32& P, long long t) {
  int lo = 0, hi = P.n_jobs - 1;  // last job whose first tile <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (P.jobs[mid].first <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Every tile's shared point location, one thread per tile, before the batch
// kernel (loc indexed by global tile; jobs in device memory).
__global__ void __launch_bounds__(128) k_locate_batch32(const BatchJob32* __restrict__ jobs,
                                                        int n_jobs, long long total_tiles,
                                                        int2* __restrict__ loc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= total_tiles) return;
  int lo = 0, hi = n_jobs - 1;  // last job whose first tile <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (jobs[mid].first <= t) lo = mid;
    else hi = mid - 1;
  }
  loc[t] = tile_location(jobs[lo].args, jobs[lo].tile0 + (int)(t - jobs[lo].first));
}

template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_batch32(const __grid_constant__ BatchTable32 P, unsigned long long* __restrict__ queue,
              const int2* __restrict__ loc) {
  extern __shared__ double s_val32[];
  __shared__ unsigned char s_lut[kLutBytes];
  __shared__ long long s_tile[2];
  fill_lut(s_lut);
  if (threadIdx.x == 0) s_tile[0] = (long long)atomicAdd(queue, 1ull);
  __syncthreads();
  for (int it = 0;; ++it) {
    const int slot = it & 1;
    const long long tile = s_tile[slot];
    if (tile >= P.total_tiles) break;
    // the next claim goes to the other slot, read only after the end-of-tile barrier
    if (threadIdx.x == 0) s_tile[slot ^ 1] = (long long)atomicAdd(queue, 1ull);
    const int j = job_of(P, tile);
    const MapArgs32& a = P.jobs[j].args;
    unsigned char* s_ok = reinterpret_cast<unsigned char*>(s_val32 + a.TW * a.TH * a.S);
    map_tile32<BLOCK>(a, P.jobs[j].tile0 + (int)(tile - P.jobs[j].first), loc + tile, s_lut,
                      s_val32, s_ok);
    __syncthreads();  // s_val and the claimed slot are reused next
  }
}

__global__ void __launch_bounds__(128) k_trace32(const TetRot32* __restrict__ rec,
                                                 const TriRec64* __restrict__ tri, int n_tri,
                                                 int n_rays, const double* __restrict__ xs,
                                                 const double* __restrict__ ys,
                                                 const __grid_constant__ MixConf C,
                                                 int loc_budget, double* __restrict__ rho,
                                                 int* __restrict__ crossed,
                                                 int* __restrict__ status,
                                                 int* __restrict__ visits, int max_record) {
  __shared__ unsigned char s_lut[kLutBytes];
  fill_lut(s_lut);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_rays) return;
  int st = kRayMiss, c = 0, fb = 0;
  double v = 0.0;
  int ft_tri = -1;
  const int ft = n_tri > 0 ? locate64(tri, 0, xs[i], ys[i], loc_budget, &st, &ft_tri) : -1;
  if (ft >= 0)
    st = walk32(rec, C, ft, ft_tri, xs[i], ys[i], (uint64_t)i, s_lut, &v, &c, &fb,
                visits ? visits + (size_t)i * max_record : nullptr, max_record);
  rho[i] = st == kRayOk ? v : 0.0;
  crossed[i] = c;
  status[i] = st;
}

// 3-D grid (src/dtfe.c:658-735) on the mixed walk: one thread per column
// (i along x, j along y), its ss^2 sub-rays in (is, js) order at the
// reference's positions, each located on the projected hull from triangle 0
// and walked with ColumnAcc32.  No two threads touch the same column.
struct GridArgs32 {
  const TetRot32* __restrict__ rec;
  const TriRec64* __restrict__ tri;
  int n_tri, G, ss, loc_budget;
  double dxy, offx, offy;
  double z0, dzs, inv_dzs, w;
  MixConf C;
  const double4* __restrict__ fld;
  double* __restrict__ grid;
  unsigned long long* __restrict__ stats;
};

__global__ void __launch_bounds__(128) k_grid32(const __grid_constant__ GridArgs32 a) {
  __shared__ unsigned char s_lut[kLutBytes];
  fill_lut(s_lut);
  __syncthreads();
  int i, j;
  const bool active = grid_column(a.G, &i, &j);
  const long long cidx = (long long)i * a.G + j;
  int worst = kRayOk, visits = 0, fallbacks = 0;
  if (active) {
    const double ds = a.dxy / a.ss;
    ColumnAcc32 acc;
    acc.col = a.grid + (size_t)cidx * a.G;
    acc.fld = a.fld;
    acc.z0 = a.z0;
    acc.dzs = a.dzs;
    acc.inv_dzs = a.inv_dzs;
    acc.w = a.w;
    acc.nzs = a.G * a.ss;
    acc.ss = a.ss;
    acc.i_in = 0;
    acc.i_out = 0;
    for (int is = 0; is < a.ss; ++is)
      for (int js = 0; js < a.ss; ++js) {
        const double x = i * a.dxy + a.offx + is * ds + ds / 2.;
        const double y = j * a.dxy + a.offy + js * ds + ds / 2.;
        int st = kRayMiss, c = 0, fb = 0, ft_tri = -1;
        const int ft = a.n_tri > 0 ? locate64(a.tri, 0, x, y, a.loc_budget, &st, &ft_tri) : -1;
        if (ft >= 0) {
          const uint64_t rid = ((uint64_t)cidx * a.ss + (uint64_t)is) * a.ss + (uint64_t)js;
          st = walk_mixed(a.rec, a.C, ft, ft_tri, x, y, rid, s_lut, acc, &c, &fb, nullptr, 0);
        }
        visits += c;
        fallbacks += fb;
        if (st > worst) worst = st;
      }
  }
  add_stats32(a.stats, active, visits, worst, fallbacks);
}

MixConf mix_conf(const Mesh& m, int axis, double z0, double lz, double dist, uint64_t seed,
                 int max_visits) {
  MixConf C;
  C.lz = lz;
  C.z0d = z0;
  C.z1d = z0 + lz;
  C.z0 = (float)C.z0d;
  C.z1 = (float)C.z1d;
  C.thr = kZero / lz;
  C.coord_max = m.coord_max;
  C.coord_err = m.fp32_exact ? 0.0 : 5.9604644775390625e-08 * m.coord_max;
  C.dist = dist;
  C.seed = seed;
  C.max_visits = max_visits;
  C.rec64 = m.ax[axis].rec64;
  C.exact32 = m.fp32_exact ? 1 : 0;
  C.rot = m.ax[axis].rot32;
  C.tri_face = m.ax[axis].tri_face;
  C.rows = m.rows;
  C.pos = m.pos;
  C.grad = m.grad;
  C.axis = axis;
  // A midpoint from FP32-derived crossings is within tol * H of the
  // reference's (each crossing within tol times its tet's height, H a bound
  // on every height: the coordinates' range) plus float rounding of positions
  // of magnitude up to Z.
  const double H = 2.0 * m.coord_max;
  const double Z = fmax(fmax(fabs(C.z0d), fabs(C.z1d)), m.coord_max);
  const double G = 64.0 * 5.9604644775390625e-08 * (Z + H) + 2.0 * (double)kCrossingTol * H;
  C.zlo_in = C.z0d + G;
  C.zhi_in = C.z1d - G;
  return C;
}

// Pixels per block = threads / samples, laid out square-ish (wide = 0) or as
// a row strip (wide = 1).
void tile_shape32(int threads, int S, int wide, int* TW, int* TH) {
  int P = threads / S;
  if (P < 1) P = 1;
  if (wide) {
    *TW = P;
    *TH = 1;
    return;
  }
  const int lg = 31 - __builtin_clz((unsigned)P);
  const int tw = 1 << ((lg + 1) / 2);
  const int th = P / tw;
  *TW = tw;
  *TH = th < 1 ? 1 : th;
}

static_assert(sizeof(int2) == kLocBytes, "tile location layout");
typedef void (*MapKernel32)(const MapArgs32, const int2*);

// A kernel instantiation, its pixel-tile shape, and the rays each thread
// walks per tile (rpt): with rpt > 1 a tile holds rpt x block rays, and a
// lane that finishes a ray early starts its next one while the others walk,
// so the warp's ray-length tail and the end-of-tile barrier are paid once per
// rpt rays.
struct Variant32 {
  MapKernel32 kernel;
  int block, minb, wide, rpt;
};

const Variant32 kVariants32[] = {
    {k_map32<256, 2>, 256, 2, 0, 1}, {k_map32<256, 3>, 256, 3, 0, 1},
    {k_map32<256, 4>, 256, 4, 0, 1}, {k_map32<128, 4>, 128, 4, 0, 1},
    {k_map32<128, 6>, 128, 6, 0, 1}, {k_map32<256, 2>, 256, 2, 1, 1},
    {k_map32<256, 3>, 256, 3, 1, 1}, {k_map32<128, 8>, 128, 8, 0, 1},
    {k_map32<64, 16>, 64, 16, 0, 1}, {k_map32<32, 32>, 32, 32, 0, 1},
    {k_map32<128, 8>, 128, 8, 0, 2}, {k_map32<64, 16>, 64, 16, 0, 2},
    {k_map32<32, 32>, 32, 32, 0, 2}, {k_map32<128, 8>, 128, 8, 0, 4},
};
constexpr int kNumVariants32 = sizeof(kVariants32) / sizeof(kVariants32[0]);
constexpr int kDefaultVariant32 = 7;  // (128, 8): the usual winner on B200

typedef void (*BatchKernel32)(const BatchTable32, unsigned long long*, const int2*);
const BatchKernel32 kBatch32[] = {k_batch32<256, 2>, k_batch32<256, 3>, k_batch32<256, 4>,
                                  k_batch32<128, 4>, k_batch32<128, 6>, k_batch32<256, 2>,
                                  k_batch32<256, 3>, k_batch32<128, 8>, k_batch32<64, 16>,
                                  k_batch32<32, 32>, k_batch32<128, 8>, k_batch32<64, 16>,
                                  k_batch32<32, 32>, k_batch32<128, 8>};
static_assert(sizeof(kBatch32) / sizeof(kBatch32[0]) == kNumVariants32, "one batch kernel per variant");

// Checks that an axis has what the mixed walk reads.
dtfe_status_t check_mixed(const Mesh& m, int axis) {
  const AxisData& A = m.ax[axis];
  if (!A.rot32 || !A.hull_built) return set_error(DTFE_ERR_INVALID, "mixed walk without FP32 records");
  if (!m.fp32_exact && !A.rec64)
    return set_error(DTFE_ERR_INVALID, "coordinates are not floats and no FP64 records are kept");
  return DTFE_OK;
}

int pick_variant32(int v) { return (v >= 0 && v < kNumVariants32) ? v : kDefaultVariant32; }

// The kernel arguments of one mixed map; *tiles_y receives its rows of tiles.
dtfe_status_t map_args32(Mesh& m, const MapGeom& g, int vi, double* d_map,
                         unsigned long long* stats, double* ray_rho, int* ray_crossed,
                         int* ray_status, MapArgs32* out, int* tiles_y) {
  SDTFE_TRY(check_mixed(m, g.axis));
  const AxisData& A = m.ax[g.axis];
  const Variant32& V = kVariants32[vi];
  MapArgs32& a = *out;
  a.rec = A.rot32;
  a.tri = A.tri;
  a.n_tri = A.n_tri;
  a.map = d_map;
  a.G = g.G;
  a.S = g.S;
  tile_shape32(V.block * V.rpt, g.S, V.wide, &a.TW, &a.TH);
  a.tiles_x = (g.G + a.TW - 1) / a.TW;
  *tiles_y = (g.G + a.TH - 1) / a.TH;
  a.dxy = g.dxy;
  a.offx = g.offx;
  a.offy = g.offy;
  a.scale = g.scale;
  a.soff = g.soff;
  a.C = mix_conf(m, g.axis, g.offz, g.lz, g.dist, g.seed, g.max_visits);
  // the location walk's budget; tile_location packs its steps as unsigned steps << 2
  if (A.n_tri >= (1 << 27))
    return set_error(DTFE_ERR_UNSUPPORTED, "mixed maps over %d hull triangles (at most 2^27 - 1)",
                     A.n_tri);
  a.loc_budget = 4 * A.n_tri + 64;
  a.stats = stats;
  a.ray_rho = ray_rho;
  a.ray_crossed = ray_crossed;
  a.ray_status = ray_status;
  return DTFE_OK;
}

}  // namespace

dtfe_status_t launch_map32(Mesh& m, const MapGeom& g, double* d_map, cudaStream_t s,
                           double* ray_rho, int* ray_crossed, int* ray_status) {
  const int vi = pick_variant32(m.tune32);
  const Variant32& V = kVariants32[vi];
  MapArgs32 a;
  int tiles_y = 0;
  SDTFE_TRY(map_args32(m, g, vi, d_map, m.stats, ray_rho, ray_crossed, ray_status, &a, &tiles_y));
  const size_t smem = (size_t)a.TW * a.TH * g.S * (sizeof(double) + 1);
  if (smem > 40 * 1024)
    SDTFE_CUDA(cudaFuncSetAttribute(V.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long blocks = (long long)a.tiles_x * tiles_y;
  SDTFE_CUDA(cudaMemsetAsync(m.stats, 0, sizeof(unsigned long long) * kStatCount, s));
  SDTFE_CUDA(cudaEventRecord(m.ev0, s));
  void* loc = nullptr;  // each tile's shared point location
  SDTFE_TRY(scratch_alloc_async(&loc, kLocBytes * (size_t)blocks, s));
  k_locate_map32<<<(unsigned)((blocks + 127) / 128), 128, 0, s>>>(a, (int)blocks,
                                                                  static_cast<int2*>(loc));
  count_launch();
  V.kernel<<<(unsigned)blocks, V.block, smem, s>>>(a, static_cast<const int2*>(loc));
  count_launch();
  const cudaError_t e = cudaGetLastError();
  scratch_free_async(loc, s);
  SDTFE_CUDA(e);
  SDTFE_CUDA(cudaEventRecord(m.ev1, s));
  m.timed = true;
  return DTFE_OK;
}

dtfe_status_t launch_grid32(Mesh& m, int G, double box_len, const double center[3], unsigned ss,
                            uint64_t seed, int max_visits, double* d_grid, cudaStream_t s) {
  SDTFE_TRY(check_mixed(m, DTFE_AXIS_Z));
  const AxisData& A = m.ax[DTFE_AXIS_Z];
  if (A.n_tri >= (1 << 27))
    return set_error(DTFE_ERR_UNSUPPORTED, "grids over %d hull triangles (at most 2^27 - 1)", A.n_tri);
  if ((long long)G * ss > (1LL << 30))
    return set_error(DTFE_ERR_UNSUPPORTED, "grid_dim %d x supersampling %u: too many nodes", G, ss);
  GridArgs32 a;
  a.rec = A.rot32;
  a.tri = A.tri;
  a.n_tri = A.n_tri;
  a.G = G;
  a.ss = (int)ss;
  a.loc_budget = 4 * A.n_tri + 64;
  // src/dtfe.c:668-735 and :398-404: cell and node spacing, weight 1/ss^3
  a.dxy = box_len / G;
  a.offx = -(box_len / 2.0) + center[0];
  a.offy = -(box_len / 2.0) + center[1];
  a.z0 = -(box_len / 2.0) + center[2];
  const double dz = box_len / G;
  a.dzs = dz / ss;
  a.inv_dzs = 1.0 / a.dzs;
  a.w = 1. / ((unsigned)ss * (unsigned)ss * (unsigned)ss);
  a.C = mix_conf(m, DTFE_AXIS_Z, a.z0, box_len, (a.dxy / 2.0) / kPerturbMax, seed, max_visits);
  if (!m.fld64) return set_error(DTFE_ERR_INVALID, "mixed grid before its FP64 field");
  a.fld = m.fld64;
  a.grid = d_grid;
  a.stats = m.stats;
  SDTFE_CUDA(cudaMemsetAsync(m.stats, 0, sizeof(unsigned long long) * kStatCount, s));
  SDTFE_CUDA(cudaEventRecord(m.ev0, s));
  k_grid32<<<grid_blocks(G), 128, 0, s>>>(a);
  count_launch();
  SDTFE_CUDA(cudaGetLastError());
  SDTFE_CUDA(cudaEventRecord(m.ev1, s));
  m.timed = true;
  return DTFE_OK;
}

dtfe_status_t launch_trace32(Mesh& m, int axis, int n_rays, const double* d_x, const double* d_y,
                             double z0, double lz, double dxy, uint64_t seed, int max_visits,
                             double* d_rho, int* d_crossed, int* d_status, int* d_visits,
                             int max_record, cudaStream_t s) {
  SDTFE_TRY(check_mixed(m, axis));
  const AxisData& A = m.ax[axis];
  MixConf C = mix_conf(m, axis, z0, lz, (dxy / 2.0) / kPerturbMax, seed, max_visits);
  if (n_rays > 0) {
    k_trace32<<<(n_rays + 127) / 128, 128, 0, s>>>(A.rot32, A.tri, A.n_tri, n_rays, d_x, d_y, C,
                                                   4 * A.n_tri + 64, d_rho, d_crossed, d_status,
                                                   d_visits, max_record);
    count_launch();
  }
  SDTFE_CUDA(cudaGetLastError());
  return DTFE_OK;
}

}  // namespace sdtfe

namespace sdtfe {
int default_variant32() { return kDefaultVariant32; }

int map_tiles32(const MapGeom& g, int variant) {
  const Variant32& V = kVariants32[pick_variant32(variant)];
  int TW, TH;
  tile_shape32(V.block * V.rpt, g.S, V.wide, &TW, &TH);
  return ((g.G + TW - 1) / TW) * ((g.G + TH - 1) / TH);
}

dtfe_status_t plan_batch32(const BatchMap* maps, int n, int variant, BatchPlan* plan) {
  const int vi = pick_variant32(variant);
  plan->precision = DTFE_MIXED;
  plan->variant = vi;
  plan->n_jobs = 0;
  plan->total_tiles = 0;
  plan->smem = 0;
  plan->jobs.assign(sizeof(BatchJob32) * (size_t)(n > 0 ? n : 0), 0);
  for (int i = 0; i < n; ++i) {
    const BatchMap& b = maps[i];
    BatchJob32 j;
    int tiles_y = 0;
    SDTFE_TRY(map_args32(*b.mesh, b.g, vi, b.d_map, b.stats, nullptr, nullptr, nullptr, &j.args,
                         &tiles_y));
    const long long tiles = (long long)j.args.tiles_x * tiles_y;
    const long long cnt = b.count < 0 ? tiles - b.tile0 : b.count;
    if (b.tile0 < 0 || cnt < 0 || b.tile0 + cnt > tiles)
      return set_error(DTFE_ERR_INVALID, "batch map %d: tiles [%d, %lld) outside the map's %lld", i,
                       b.tile0, b.tile0 + cnt, tiles);
    if (cnt == 0) continue;
    j.first = plan->total_tiles;
    j.tile0 = b.tile0;
    j.count = (int)cnt;
    memcpy(plan->jobs.data() + sizeof(BatchJob32) * plan->n_jobs, &j, sizeof(j));
    ++plan->n_jobs;
    plan->total_tiles += cnt;
    const size_t smem = (size_t)j.args.TW * j.args.TH * j.args.S * (sizeof(double) + 1);
    if (smem > plan->smem) plan->smem = smem;
  }
  plan->jobs.resize(sizeof(BatchJob32) * plan->n_jobs);
  return DTFE_OK;
}

dtfe_status_t batch_grid32(int variant, size_t smem, int* grid, int* block) {
  const int vi = pick_variant32(variant);
  int dev = 0, sms = 0, per_sm = 0;
  SDTFE_CUDA(cudaGetDevice(&dev));
  SDTFE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (smem > 40 * 1024)
    SDTFE_CUDA(cudaFuncSetAttribute(kBatch32[vi], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  SDTFE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kBatch32[vi], kVariants32[vi].block,
                                                           smem));
  if (per_sm < 1)
    return set_error(DTFE_ERR_UNSUPPORTED, "mixed batch: %zu B of shared memory per block", smem);
  *grid = per_sm * sms;
  *block = kVariants32[vi].block;
  return DTFE_OK;
}

dtfe_status_t launch_batch32(const BatchPlan& plan, const void* d_jobs, unsigned long long* d_queue,
                             void* d_loc, int grid, cudaStream_t s) {
  if (plan.n_jobs == 0) return DTFE_OK;
  const int vi = pick_variant32(plan.variant);
  if (plan.smem > 40 * 1024)
    SDTFE_CUDA(cudaFuncSetAttribute(kBatch32[vi], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)plan.smem));
  const BatchJob32* jobs = static_cast<const BatchJob32*>(d_jobs);
  k_locate_batch32<<<(unsigned)((plan.total_tiles + 127) / 128), 128, 0, s>>>(
      jobs, plan.n_jobs, plan.total_tiles, static_cast<int2*>(d_loc));
  count_launch();
  // the job table as the kernel's parameter, kMaxJobsPerLaunch32 jobs per
  // launch; each chunk's tiles are renumbered from 0 and pull from the queue
  // counter, cleared before each chunk (the caller clears it for the first)
  const BatchJob32* host = reinterpret_cast<const BatchJob32*>(plan.jobs.data());
  static thread_local BatchTable32 P;  // about 30 KB: not on the stack
  for (int j0 = 0; j0 < plan.n_jobs; j0 += kMaxJobsPerLaunch32) {
    const int n = std::min(kMaxJobsPerLaunch32, plan.n_jobs - j0);
    const long long base = host[j0].first;
    const long long end = j0 + n < plan.n_jobs ? host[j0 + n].first : plan.total_tiles;
    P.n_jobs = n;
    P.total_tiles = end - base;
    for (int k = 0; k < n; ++k) {
      P.jobs[k] = host[j0 + k];
      P.jobs[k].first -= base;
    }
    if (j0 > 0) SDTFE_CUDA(cudaMemsetAsync(d_queue, 0, sizeof(unsigned long long), s));
    kBatch32[vi]<<<grid, kVariants32[vi].block, plan.smem, s>>>(
        P, d_queue, static_cast<const int2*>(d_loc) + base);
    count_launch();
  }
  SDTFE_CUDA(cudaGetLastError());
  return DTFE_OK;
}

int num_map32_variants() { return kNumVariants32; }
void map32_variant_info(int i, int* block, int* minb, int* wide, int* rpt) {
  *block = kVariants32[i].block;
  *minb = kVariants32[i].minb;
  *wide = kVariants32[i].wide;
  *rpt = kVariants32[i].rpt;
}
}  // namespace sdtfe
