/*
 * dtfe_oracle.c - CPU restatement of SDTFE's density-estimation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the GPU library is
 * compared against; nothing in the shipped library links, loads or calls it.
 * It is built into oracle/liboracle.so and used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU baseline.
 *
 * Every function restates one reference routine (paths relative to the
 * reference project root) and performs the floating-point operations in the
 * same order, so that its results are bit-identical to the reference on the
 * same inputs (x86-64 SSE2 double arithmetic without contraction).  The
 * restatement is pinned against the reference compiled from its own sources
 * (oracle/_ref, built by oracle/Makefile) and against tests/golden/.
 *
 * Layouts are the reference's:
 *   pos  double[n*4]   (x, y, z, rho)                      src/utils.c:8-16
 *   tet  int[nt*8]     (A, B, C, D, n_BDC, n_ACD, n_ADB, n_ABC)
 *                      neighbour slot 4+k lies across the face opposite k
 *                                                          src/triangulate.c:52,111-175
 *   grad double[nt*3]                                      src/triangulate.c:233-260
 *   tri  int[n_tri*8]  (a, b, c, n_CB, n_AC, n_BA, tet, -) src/triangulate.c:318-395
 *
 * Differences from the reference, all deliberate and listed here:
 *   - rand() is replaced by the counter-based generator of include/sdtfe_rng.h;
 *   - warnings are returned as per-ray status codes instead of stderr lines;
 *   - the two walks carry a visit budget and the point location a step budget,
 *     so a corrupt mesh ends with a status instead of looping.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "sdtfe_rng.h"

/* src/constants.h:6-8 */
#define ORC_ZERO (1e4 * DBL_EPSILON)
#define ORC_PERTURB_MAX 1000

/* vertex slots A..D and face slots (face k lies opposite vertex k) */
enum { VA = 0, VB = 1, VC = 2, VD = 3 };
enum { F_BDC = 0, F_ACD = 1, F_ADB = 2, F_ABC = 3 };
/* the six tetrahedron edges, in the reference's side_t order (src/constants.h:11) */
enum { E_CB = 0, E_AC = 1, E_BA = 2, E_DC = 3, E_BD = 4, E_DA = 5 };

/* per-ray status codes (same values as the library's DTFE_RAY_* codes) */
enum {
  ORC_RAY_OK = 0,
  ORC_RAY_MISS = 1,         /* sample falls outside the projected hull       */
  ORC_RAY_NO_EXIT = 2,      /* Plücker test found no enter/leave face pair   */
  ORC_RAY_PERTURB_MAX = 3,  /* more than PERTURB_MAX perturbations           */
  ORC_RAY_BUDGET = 4,       /* visit budget exhausted (corrupt neighbours)   */
  ORC_RAY_LOC_BUDGET = 5    /* point location did not settle                 */
};

static inline int orc_sign(double x) { return x > ORC_ZERO ? 1 : (x < -ORC_ZERO ? -1 : 0); }

/* ------------------------------------------------------------------------- */
/* a3: per-vertex density.  src/triangulate.c:183-225 (pre_compute_vol).      */
/* Volumes are scattered in increasing tet order, then rho = m*(1+3)/sum.      */
/* adj (optional) receives the number of tets incident to each vertex.         */
void orc_density(double *pos, int n, const int *tet, int nt, float p_mass, int *adj) {
  for (int i = 0; i < n; ++i) pos[i * 4 + 3] = 0;
  if (adj) memset(adj, 0, sizeof(int) * (size_t)n);
  for (int t = 0; t < nt; ++t) {
    const double *a = pos + 4 * (size_t)tet[t * 8 + VA];
    const double *b = pos + 4 * (size_t)tet[t * 8 + VB];
    const double *c = pos + 4 * (size_t)tet[t * 8 + VC];
    const double *d = pos + 4 * (size_t)tet[t * 8 + VD];
    /* determinant of (a-d, b-d, c-d) expanded along the first row, each
       factor formed from raw differences exactly as written at :191-213 */
    double r0 = (a[0] - d[0]) * ((b[1] - d[1]) * (c[2] - d[2]) - (b[2] - d[2]) * (c[1] - d[1]));
    double r1 = (a[1] - d[1]) * ((b[2] - d[2]) * (c[0] - d[0]) - (b[0] - d[0]) * (c[2] - d[2]));
    double r2 = (a[2] - d[2]) * ((b[0] - d[0]) * (c[1] - d[1]) - (b[1] - d[1]) * (c[0] - d[0]));
    double vol = fabs((r0 + r1 + r2) / 6);
    for (int k = 0; k < 4; ++k) {
      int v = tet[t * 8 + k];
      pos[4 * (size_t)v + 3] += vol;
      if (adj) adj[v] += 1;
    }
  }
  for (int i = 0; i < n; ++i) pos[i * 4 + 3] = p_mass * (1 + 3) / pos[i * 4 + 3];
}

/* ------------------------------------------------------------------------- */
/* a4: per-tet gradient by Cramer's rule.  src/triangulate.c:228-260.          */
static inline double det3(double a, double b, double c, double d, double e, double f, double g,
                          double h, double i) {
  /* six products summed left to right, as determ3x3 does */
  return a * e * i + b * f * g + c * d * h - c * e * g - b * d * i - a * f * h;
}

void orc_gradients(const int *tet, int nt, const double *pos, double *grad) {
  for (int t = 0; t < nt; ++t) {
    const double *a = pos + 4 * (size_t)tet[t * 8 + VA];
    const double *b = pos + 4 * (size_t)tet[t * 8 + VB];
    const double *c = pos + 4 * (size_t)tet[t * 8 + VC];
    const double *d = pos + 4 * (size_t)tet[t * 8 + VD];
    double xb = b[0] - a[0], yb = b[1] - a[1], zb = b[2] - a[2];
    double xc = c[0] - a[0], yc = c[1] - a[1], zc = c[2] - a[2];
    double xd = d[0] - a[0], yd = d[1] - a[1], zd = d[2] - a[2];
    double rb = b[3] - a[3], rc = c[3] - a[3], rd = d[3] - a[3];
    double den = det3(xb, yb, zb, xc, yc, zc, xd, yd, zd);
    grad[t * 3 + 0] = det3(rb, yb, zb, rc, yc, zc, rd, yd, zd) / den;
    grad[t * 3 + 1] = det3(xb, rb, zb, xc, rc, zc, xd, rd, zd) / den;
    grad[t * 3 + 2] = det3(xb, yb, rb, xc, yc, rc, xd, yd, rd) / den;
  }
}

/* ------------------------------------------------------------------------- */
/* a5: forward-hull faces.  src/triangulate.c:263-316.  A boundary face (no    */
/* neighbour) is forward when the z component of t1 x t2 is negative, with     */
/* (t1, t2) the two edge vectors the reference uses for that face.             */
/* flags[4*t+f] = 1 for forward faces; returns their number.                  */
static const int k_face_edge_vecs[4][3] = {
    /* origin, t1 end, t2 end */
    [F_BDC] = {VB, VD, VC},
    [F_ACD] = {VA, VC, VD},
    [F_ADB] = {VA, VD, VB},
    [F_ABC] = {VA, VB, VC},
};

int orc_forward_faces(const int *tet, int nt, const double *pos, unsigned char *flags) {
  int count = 0;
  for (int t = 0; t < nt; ++t) {
    for (int f = 0; f < 4; ++f) {
      flags[t * 4 + f] = 0;
      if (tet[t * 8 + 4 + f] != -1) continue;
      const double *o = pos + 4 * (size_t)tet[t * 8 + k_face_edge_vecs[f][0]];
      const double *p = pos + 4 * (size_t)tet[t * 8 + k_face_edge_vecs[f][1]];
      const double *q = pos + 4 * (size_t)tet[t * 8 + k_face_edge_vecs[f][2]];
      double t1x = p[0] - o[0], t1y = p[1] - o[1];
      double t2x = q[0] - o[0], t2y = q[1] - o[1];
      if (t1x * t2y - t1y * t2x < 0.0) {
        flags[t * 4 + f] = 1;
        ++count;
      }
    }
  }
  return count;
}

/* ------------------------------------------------------------------------- */
/* a6: projected hull triangles.  src/triangulate.c:318-395.  Triangles are    */
/* emitted in (tet, face) order; the vertex order per face is the reference's; */
/* neighbours are found by brute force over all pairs, the largest matching    */
/* index winning ("last match wins").                                          */
static const int k_tri_of_face[4][3] = {
    [F_BDC] = {VB, VD, VC},
    [F_ACD] = {VA, VC, VD},
    [F_ADB] = {VA, VD, VB},
    [F_ABC] = {VA, VB, VC},
};

int orc_hull_triangles(const int *tet, int nt, const unsigned char *flags, int *tri) {
  int nt2 = 0;
  for (int t = 0; t < nt; ++t)
    for (int f = 0; f < 4; ++f)
      if (flags[t * 4 + f]) {
        int *r = tri + 8 * (size_t)nt2;
        for (int k = 0; k < 3; ++k) r[k] = tet[t * 8 + k_tri_of_face[f][k]];
        r[3] = r[4] = r[5] = -1;
        r[6] = t;
        r[7] = -1;
        ++nt2;
      }
  for (int i = 0; i < nt2; ++i) {
    int *ri = tri + 8 * (size_t)i;
    for (int j = 0; j < nt2; ++j) {
      if (i == j) continue;
      const int *rj = tri + 8 * (size_t)j;
      int in_j[3];
      for (int k = 0; k < 3; ++k) in_j[k] = (ri[k] == rj[0]) || (ri[k] == rj[1]) || (ri[k] == rj[2]);
      if (in_j[0] && in_j[1]) ri[3 + 2] = j; /* edge a-b: slot 3+BA */
      if (in_j[0] && in_j[2]) ri[3 + 1] = j; /* edge a-c: slot 3+AC */
      if (in_j[1] && in_j[2]) ri[3 + 0] = j; /* edge b-c: slot 3+CB */
    }
  }
  return nt2;
}

/* ------------------------------------------------------------------------- */
/* a7: point location on the projected hull.  src/dtfe.c:518-552.  Visibility  */
/* walk from triangle `start`; each of the three edges is tested as            */
/* orient(edge, opposite vertex) * orient(edge, query) < 0.                    */
int orc_locate(const int *tri, const double *pos, int start, double qx, double qy, int max_steps,
               int *status) {
  int cur = start;
  int steps = 0;
  *status = ORC_RAY_OK;
  do {
    if (++steps > max_steps) {
      *status = ORC_RAY_LOC_BUDGET;
      return -1;
    }
    const int *r = tri + 8 * (size_t)cur;
    const double *a = pos + 4 * (size_t)r[0];
    const double *b = pos + 4 * (size_t)r[1];
    const double *c = pos + 4 * (size_t)r[2];
    double s_in, s_q;
    /* edge a-b, opposite c */
    s_in = (c[0] - a[0]) * (b[1] - a[1]) - (c[1] - a[1]) * (b[0] - a[0]);
    s_q = (qx - a[0]) * (b[1] - a[1]) - (qy - a[1]) * (b[0] - a[0]);
    if (s_in * s_q < 0.0) {
      cur = r[3 + 2];
      continue;
    }
    /* edge b-c, opposite a */
    s_in = (a[0] - b[0]) * (c[1] - b[1]) - (a[1] - b[1]) * (c[0] - b[0]);
    s_q = (qx - b[0]) * (c[1] - b[1]) - (qy - b[1]) * (c[0] - b[0]);
    if (s_in * s_q < 0.0) {
      cur = r[3 + 0];
      continue;
    }
    /* edge c-a, opposite b */
    s_in = (b[0] - c[0]) * (a[1] - c[1]) - (b[1] - c[1]) * (a[0] - c[0]);
    s_q = (qx - c[0]) * (a[1] - c[1]) - (qy - c[1]) * (a[0] - c[0]);
    if (s_in * s_q < 0.0) {
      cur = r[3 + 1];
      continue;
    }
    break;
  } while (cur != -1);
  if (cur == -1) {
    *status = ORC_RAY_MISS;
    return -1;
  }
  return tri[8 * (size_t)cur + 6];
}

/* ------------------------------------------------------------------------- */
/* a8: Plücker ray/tetrahedron test for a ray along +z.  src/dtfe.c:19-215.    */
/*                                                                            */
/* The ray's Plücker coordinates reduce to (lz, -lz*oy, lz*ox) on the three   */
/* components the permuted product touches (src/dtfe.c:24-26, 296-299).  The   */
/* edge P->Q contributes  lz*(Px*Qy - Py*Qx) + (Px-Qx)*(-lz*oy) + (Py-Qy)*(lz*ox).*/
typedef struct {
  double lz, m_oy, ox_l; /* lz, -lz*oy, lz*ox */
} orc_ray;

static const int k_edge_pq[6][2] = {
    [E_CB] = {VC, VB}, [E_AC] = {VC, VA}, [E_BA] = {VB, VA},
    [E_DC] = {VC, VD}, [E_BD] = {VB, VD}, [E_DA] = {VD, VA},
};

static inline double edge_u(const orc_ray *ry, const double *p, const double *q) {
  double v0 = p[0] - q[0];
  double v1 = p[1] - q[1];
  double v5 = p[0] * q[1] - p[1] * q[0];
  return ry->lz * v5 + v0 * ry->m_oy + v1 * ry->ox_l;
}

/* Per face: the three signed edge terms in the order the reference sums them
 * for the face's normaliser, the two barycentric weights (signed edge terms),
 * and the three face vertices the weights apply to: the crossing point is
 * ((1-w1)-w2)*P0 + w1*P1 + w2*P2.  A face is entered when all three signed
 * terms are >= 0 and left when all are <= 0. */
typedef struct {
  int e[3], s[3];
  int w1e, w1s, w2e, w2s;
  int p[3];
} orc_face;

static const orc_face k_faces[4] = {
    [F_BDC] = {{E_CB, E_DC, E_BD}, {-1, +1, -1}, E_BD, -1, E_DC, +1, {VD, VC, VB}},
    [F_ACD] = {{E_AC, E_DC, E_DA}, {+1, -1, -1}, E_AC, +1, E_DC, -1, {VC, VD, VA}},
    [F_ADB] = {{E_DA, E_BD, E_BA}, {+1, +1, -1}, E_BD, +1, E_BA, -1, {VB, VA, VD}},
    [F_ABC] = {{E_BA, E_CB, E_AC}, {+1, +1, -1}, E_AC, -1, E_BA, +1, {VA, VB, VC}},
};

/* Returns 1 when an enter and a leave face were both found.  Only the z of
 * the crossing points is produced (the x and y are never read by the walks). */
static int orc_ray_tet(const orc_ray *ry, const double *v[4], int *enter, int *leave, double *z_in,
                       double *z_out, int *special) {
  double u[6];
  int sg[6];
  for (int e = 0; e < 6; ++e) {
    u[e] = edge_u(ry, v[k_edge_pq[e][0]], v[k_edge_pq[e][1]]);
    sg[e] = orc_sign(u[e]);
  }
  *enter = -1;
  *leave = -1;
  *special = 0;
  int found = 0;
  for (int f = 0; f < 4; ++f) {
    const orc_face *F = &k_faces[f];
    if (sg[F->e[0]] == 0 && sg[F->e[1]] == 0 && sg[F->e[2]] == 0) continue;
    double t0 = F->s[0] * u[F->e[0]];
    double t1 = F->s[1] * u[F->e[1]];
    double t2 = F->s[2] * u[F->e[2]];
    double inv = 1.0 / (t0 + t1 + t2);
    int a = F->s[0] * sg[F->e[0]], b = F->s[1] * sg[F->e[1]], c = F->s[2] * sg[F->e[2]];
    int is_enter = (*enter == -1) && a >= 0 && b >= 0 && c >= 0;
    int is_leave = !is_enter && (*leave == -1) && a <= 0 && b <= 0 && c <= 0;
    if (!is_enter && !is_leave) continue;
    double w1 = (F->w1s * u[F->w1e]) * inv;
    double w2 = (F->w2s * u[F->w2e]) * inv;
    double z = (1 - w1 - w2) * v[F->p[0]][2] + w1 * v[F->p[1]][2] + w2 * v[F->p[2]][2];
    if (is_enter) {
      *enter = f;
      *z_in = z;
    } else {
      *leave = f;
      *z_out = z;
    }
    if (sg[F->e[0]] == 0 || sg[F->e[1]] == 0 || sg[F->e[2]] == 0) *special = 1;
    if (++found == 2) return 1;
  }
  return 0;
}

/* a9: move the ray origin towards a tet corner chosen by the generator.
 * src/dtfe.c:219-245. */
static void orc_perturb(double *ox, double *oy, const double *v[4], double max_dist, uint64_t seed,
                        uint64_t ray, uint64_t *ctr) {
  int r = sdtfe_rand31(seed, ray, (*ctr)++) % 4;
  double dx = v[r][0] - *ox;
  double dy = v[r][1] - *oy;
  double mag = sqrt(dx * dx + dy * dy);
  if (mag > max_dist) {
    dx = dx / mag;
    dy = dy / mag;
    dx = dx * max_dist;
    dy = dy * max_dist;
  }
  *ox = *ox + dx;
  *oy = *oy + dy;
}

/* ------------------------------------------------------------------------- */
/* a10 / a12: the tet walk along neighbour links, shared by the surface        */
/* integral (src/dtfe.c:247-374) and the 3-D column (src/dtfe.c:376-516).      */
typedef struct {
  /* surface mode */
  double rho;
  /* column mode (col != NULL): fine-z sampling */
  double *col;
  int nz;
  unsigned ss;
} orc_acc;

static int orc_walk(int ft, const int *tet, const double *grad, const double *pos, double x, double y,
                    double z0, double lz, double dxy, uint64_t seed, uint64_t ray, orc_acc *acc,
                    int *visits, int max_record, int max_visits, int *n_crossed) {
  const double max_dist = dxy / 2.0;
  const double dist = max_dist / ORC_PERTURB_MAX;
  double ox = x, oy = y;
  orc_ray ry = {lz, -lz * oy, lz * ox};
  uint64_t ctr = 0;
  int crossed = 0;
  *n_crossed = 0;
  if (ft == -1) return ORC_RAY_MISS;

  /* the column-mode constants of src/dtfe.c:398-404 */
  double dz = 0, dzs = 0, w = 0;
  int nzs = 0;
  if (acc->col) {
    dz = lz / acc->nz;
    dzs = dz / acc->ss;
    nzs = acc->nz * (int)acc->ss;
    w = 1. / (acc->ss * acc->ss * acc->ss);
  }

  /* the walk starts as if it had just left a virtual tet through face 0 */
  int nb[4] = {ft, -1, -1, -1};
  int leave = 0, enter = -1;
  int cur = ft, prev = -1;
  while (nb[leave] != -1) {
    if (nb[leave] == prev) { /* turn around: leave through the entry face */
      int t = enter;
      enter = leave;
      leave = t;
      if (nb[leave] == -1) break;
    }
    prev = cur;
    cur = nb[leave];
    if (crossed >= max_visits) {
      *n_crossed = 0;
      return ORC_RAY_BUDGET;
    }
    const int *row = tet + 8 * (size_t)cur;
    for (int k = 0; k < 4; ++k) nb[k] = row[4 + k];
    const double *v[4];
    for (int k = 0; k < 4; ++k) v[k] = pos + 4 * (size_t)row[k];

    double z_in = 0, z_out = 0;
    int special;
    if (!orc_ray_tet(&ry, v, &enter, &leave, &z_in, &z_out, &special)) {
      *n_crossed = 0;
      return ORC_RAY_NO_EXIT;
    }
    int np = 0;
    while (special) {
      orc_perturb(&ox, &oy, v, dist, seed, ray, &ctr);
      ry.m_oy = -lz * oy;
      ry.ox_l = lz * ox;
      if (++np > ORC_PERTURB_MAX) {
        *n_crossed = 0;
        return ORC_RAY_PERTURB_MAX;
      }
      if (!orc_ray_tet(&ry, v, &enter, &leave, &z_in, &z_out, &special)) {
        *n_crossed = 0;
        return ORC_RAY_NO_EXIT;
      }
    }
    if (visits && crossed < max_record) visits[crossed] = cur;
    ++crossed;

    const double *g = grad + 3 * (size_t)cur;
    if (!acc->col) {
      double d = z_out - z_in;
      double zm = d / 2 + z_in;
      if (zm > z0 && zm < z0 + lz) {
        double fixed = v[VA][3] + (g[0] * (ox - v[VA][0])) + (g[1] * (oy - v[VA][1])) - (g[2] * v[VA][2]);
        acc->rho += (fixed + g[2] * zm) * d;
      }
    } else {
      int i0 = (int)ceil((z_in - z0 - dzs / 2.) / dzs);
      i0 = i0 < 0 ? 0 : i0;
      int i1 = (int)ceil((z_out - z0 - dzs / 2.) / dzs);
      i1 = i1 > nzs ? nzs : i1;
      if (i1 > i0) {
        double fixed = v[VA][3] + g[0] * (ox - v[VA][0]) + g[1] * (oy - v[VA][1]) - g[2] * v[VA][2];
        for (int is = i0; is < i1; ++is) {
          int iz = is / (int)acc->ss;
          double zi = z0 + dzs * is + dzs / 2.;
          acc->col[iz] += (fixed + g[2] * zi) * w;
        }
      }
    }
  }
  *n_crossed = crossed;
  return ORC_RAY_OK;
}

/* Single surface ray from tet `ft` (the restatement of shoot_3d_ray).  Returns
 * the integral (0 on failure); crossed/status/visits as in the library. */
double orc_shoot(int ft, const int *tet, const double *grad, const double *pos, double x, double y,
                 double z0, double lz, double dxy, uint64_t seed, uint64_t ray, int *crossed,
                 int *status, int *visits, int max_record, int max_visits) {
  orc_acc acc = {0};
  int st = orc_walk(ft, tet, grad, pos, x, y, z0, lz, dxy, seed, ray, &acc, visits, max_record,
                    max_visits, crossed);
  *status = st;
  return st == ORC_RAY_OK ? acc.rho : 0.0;
}

/* ------------------------------------------------------------------------- */
/* a11: the Monte Carlo pixel loop of compute_density (src/dtfe.c:578-646)     */
/* with sample offsets from sdtfe_sample_u01.  map is accumulated (+=) in      */
/* row-major (row*G + col) order; ray_* (optional) are pixel*S + sample.       */
void orc_map(const double *pos, const int *tet, const double *grad, const int *tri, int G,
             double box_len, double box_len_z, double cx, double cy, double cz, int S,
             double delta_sample, uint64_t seed, int max_visits, double *map, double *ray_rho,
             int *ray_crossed, int *ray_status) {
  const double dxy = box_len / G;
  const double offx = -(box_len / 2.0) + cx;
  const double offy = -(box_len / 2.0) + cy;
  const double offz = -(box_len_z / 2.0) + cz;
  const double scale = delta_sample > dxy ? delta_sample : dxy;
  const double soff = delta_sample > dxy ? (delta_sample - dxy) / 2.0 : 0.0;
  const int loc_budget = 1 << 24;
  long long npix = (long long)G * G;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long p = 0; p < npix; ++p) {
    int col = (int)(p % G), row = (int)(p / G);
    double x = col * dxy + offx - soff;
    double y = row * dxy + offy - soff;
    double total = 0.0;
    int n_avg = S;
    for (int s = 0; s < S; ++s) {
      double xt = x + sdtfe_sample_u01(seed, (uint64_t)p, (uint32_t)s, 0) * scale;
      double yt = y + sdtfe_sample_u01(seed, (uint64_t)p, (uint32_t)s, 1) * scale;
      uint64_t rid = (uint64_t)p * (uint64_t)S + (uint64_t)s;
      int st;
      int ft = orc_locate(tri, pos, 0, xt, yt, loc_budget, &st);
      double v = 0.0;
      int crossed = 0;
      if (ft == -1) {
        --n_avg;
      } else {
        v = orc_shoot(ft, tet, grad, pos, xt, yt, offz, box_len_z, dxy, seed, rid, &crossed, &st,
                      NULL, 0, max_visits);
        total += v;
        if (crossed == 0) --n_avg;
      }
      if (ray_rho) ray_rho[rid] = v;
      if (ray_crossed) ray_crossed[rid] = crossed;
      if (ray_status) ray_status[rid] = st;
    }
    if (n_avg > 0) map[p] += total / n_avg;
    else map[p] += 0.0;
  }
}

/* Rays at explicit positions (x[i], y[i]); ray id i drives the perturbation. */
void orc_trace(const double *pos, const int *tet, const double *grad, const int *tri, int n_rays,
               const double *xs, const double *ys, double z0, double lz, double dxy, uint64_t seed,
               int max_visits, double *rho, int *crossed, int *status, int *visits, int max_record) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n_rays; ++i) {
    int st;
    int ft = orc_locate(tri, pos, 0, xs[i], ys[i], 1 << 24, &st);
    int c = 0;
    double v = 0.0;
    if (ft != -1)
      v = orc_shoot(ft, tet, grad, pos, xs[i], ys[i], z0, lz, dxy, seed, (uint64_t)i, &c, &st,
                    visits ? visits + (size_t)i * max_record : NULL, max_record, max_visits);
    rho[i] = v;
    crossed[i] = c;
    status[i] = st;
  }
}

/* ------------------------------------------------------------------------- */
/* a12: the 3-D grid of interpolate_to_3d_grid (src/dtfe.c:668-735).  Column   */
/* (i, j) sits at x index i, y index j; grid[(i*G + j)*G + iz] accumulates.     */
/* Ray id of sub-ray (is, js) of column (i, j) is ((i*G + j)*ss + is)*ss + js.  */
void orc_grid(const double *pos, const int *tet, const double *grad, const int *tri, int G,
              double box_len, double *grid, double cx, double cy, double cz, unsigned ss,
              uint64_t seed, int max_visits, int *col_status) {
  const double dxy = box_len / G;
  const double offx = -(box_len / 2.0) + cx;
  const double offy = -(box_len / 2.0) + cy;
  const double offz = -(box_len / 2.0) + cz;
  const double ds = dxy / ss;
  long long ncol = (long long)G * G;
#pragma omp parallel for schedule(dynamic, 4)
  for (long long cidx = 0; cidx < ncol; ++cidx) {
    int i = (int)(cidx / G), j = (int)(cidx % G);
    double *colp = grid + (size_t)cidx * G;
    int worst = ORC_RAY_OK;
    for (int is = 0; is < (int)ss; ++is)
      for (int js = 0; js < (int)ss; ++js) {
        double x = i * dxy + offx + is * ds + ds / 2.;
        double y = j * dxy + offy + js * ds + ds / 2.;
        int st;
        int ft = orc_locate(tri, pos, 0, x, y, 1 << 24, &st);
        uint64_t rid = ((uint64_t)cidx * ss + (uint64_t)is) * ss + (uint64_t)js;
        orc_acc acc = {0};
        acc.col = colp;
        acc.nz = G;
        acc.ss = ss;
        int crossed;
        if (ft != -1)
          st = orc_walk(ft, tet, grad, pos, x, y, offz, box_len, dxy, seed, rid, &acc, NULL, 0,
                        max_visits, &crossed);
        if (st > worst) worst = st;
      }
    if (col_status) col_status[cidx] = worst;
  }
}
