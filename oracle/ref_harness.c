/*
 * ref_harness.c - explicit-offset driver around the reference's own walk.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile links this file with the
 * reference's unmodified sources (src/dtfe.c, src/bitmap.c, src/utils.c and
 * the non-Qhull part of src/triangulate.c) into oracle/_ref/libdtfe_refh.so,
 * compiling them with -Drand=sdtfe_ref_rand so that the reference's
 * perturb_ray (src/dtfe.c:223) draws from the counter-based generator of
 * include/sdtfe_rng.h instead of the shared libc stream.
 *
 * The loops below restate only the pixel/sample bookkeeping of
 * compute_density (src/dtfe.c:607-646) and interpolate_to_3d_grid
 * (src/dtfe.c:710-729); every ray is located and walked by the reference's
 * exported pt_loc_2d (src/dtfe.c:518) and shoot_3d_ray (src/dtfe.c:247) /
 * evaluate_3d_ray_on_grid (src/dtfe.c:376).  The sample offsets come from
 * sdtfe_sample_u01, the same function the GPU library uses.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "sdtfe_rng.h"

/* reference entry points (src/dtfe.c) */
int pt_loc_2d(int *tri_data, double *particle_data, int *start_tri, double q_x, double q_y);
double shoot_3d_ray(int th_idx, int *tetra_data, double *nabla, double *particle_data, double x,
                    double y, double offset_z, double box_len_z, double delta_xy, int grid_dim,
                    int idx, int *tetra_crossed);
void evaluate_3d_ray_on_grid(int th_idx, int *tetra_data, double *nabla, double *particle_data,
                             double x, double y, double offset_z, double box_len_z, int nz,
                             double delta_xy, int *tetra_crossed, unsigned supersampling,
                             double *rho_vector);

/* the reference's rand() calls land here (see the -D in oracle/Makefile) */
static __thread uint64_t h_seed, h_ray, h_ctr;

int sdtfe_ref_rand(void) { return sdtfe_rand31(h_seed, h_ray, h_ctr++); }

static void begin_ray(uint64_t seed, uint64_t ray) {
  h_seed = seed;
  h_ray = ray;
  h_ctr = 0;
}

/* Map with sample offsets from sdtfe_sample_u01; same arguments and ray
 * numbering (pixel*S + sample) as the library's explicit-seed map. */
void refh_map(double *pos, int *tet, double *grad, int *tri, int G, double box_len,
              double box_len_z, double cx, double cy, double cz, int S, double delta_sample,
              uint64_t seed, double *map, double *ray_rho, int *ray_crossed) {
  const double dxy = box_len / G;
  const double offx = -(box_len / 2.0) + cx;
  const double offy = -(box_len / 2.0) + cy;
  const double offz = -(box_len_z / 2.0) + cz;
  const double scale = delta_sample > dxy ? delta_sample : dxy;
  const double soff = delta_sample > dxy ? (delta_sample - dxy) / 2.0 : 0.0;
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
      int start = 0;
      int ft = pt_loc_2d(tri, pos, &start, xt, yt);
      double v = 0.0;
      int crossed = 0;
      if (ft == -1) {
        --n_avg;
      } else {
        begin_ray(seed, rid);
        v = shoot_3d_ray(ft, tet, grad, pos, xt, yt, offz, box_len_z, dxy, G, (int)p, &crossed);
        total += v;
        if (crossed == 0) --n_avg;
      }
      if (ray_rho) ray_rho[rid] = v;
      if (ray_crossed) ray_crossed[rid] = crossed;
    }
    if (n_avg > 0) map[p] += total / n_avg;
    else map[p] += 0.0;
  }
}

/* Rays at explicit positions; ray i uses ray id i for the perturbation.
 * Single-threaded so that the visit hook sees one ray at a time. */
void refh_trace(double *pos, int *tet, double *grad, int *tri, int n_rays, const double *xs,
                const double *ys, double z0, double lz, double dxy, uint64_t seed, double *rho,
                int *crossed, void (*on_ray)(int)) {
  for (int i = 0; i < n_rays; ++i) {
    int start = 0;
    if (on_ray) on_ray(i);
    int ft = pt_loc_2d(tri, pos, &start, xs[i], ys[i]);
    int c = 0;
    double v = 0.0;
    if (ft != -1) {
      begin_ray(seed, (uint64_t)i);
      v = shoot_3d_ray(ft, tet, grad, pos, xs[i], ys[i], z0, lz, dxy, 0, i, &c);
    }
    rho[i] = v;
    crossed[i] = c;
  }
}

/* 3-D grid; sub-ray (is, js) of column (i, j) has ray id ((i*G+j)*ss+is)*ss+js. */
void refh_grid(double *pos, int *tet, double *grad, int *tri, int G, double box_len, double *grid,
               double cx, double cy, double cz, unsigned ss, uint64_t seed) {
  const double dxy = box_len / G;
  const double offx = -(box_len / 2.0) + cx;
  const double offy = -(box_len / 2.0) + cy;
  const double offz = -(box_len / 2.0) + cz;
  const double ds = dxy / ss;
  long long ncol = (long long)G * G;
#pragma omp parallel for schedule(dynamic, 4)
  for (long long cidx = 0; cidx < ncol; ++cidx) {
    int i = (int)(cidx / G), j = (int)(cidx % G);
    for (int is = 0; is < (int)ss; ++is)
      for (int js = 0; js < (int)ss; ++js) {
        double x = i * dxy + offx + is * ds + ds / 2.;
        double y = j * dxy + offy + js * ds + ds / 2.;
        int start = 0;
        int ft = pt_loc_2d(tri, pos, &start, x, y);
        int c;
        begin_ray(seed, ((uint64_t)cidx * ss + (uint64_t)is) * ss + (uint64_t)js);
        evaluate_3d_ray_on_grid(ft, tet, grad, pos, x, y, offz, box_len, G, dxy, &c, ss,
                                grid + (size_t)cidx * G);
      }
  }
}
