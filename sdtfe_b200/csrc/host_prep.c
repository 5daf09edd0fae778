/*
 * host_prep.c - host-side input preparation and the face bitmap, the parts of
 * the reference interface that stay on the CPU (as they do in the reference):
 * the data is on the host, the work is a single pass, and the results must
 * follow the C library's rand() stream and libm exactly.
 *
 *   convert_to_qhdata, shuffle_buff, rotate3d      src/utils.c:8-79
 *   set_bit, clear_bit, get_bit, create/delete     src/bitmap.c:1-33
 *   dtfe_tetra_from_cells                          src/triangulate.c:63-175
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bitmap.h"
#include "sdtfe_b200.h"
#include "utils.h"

/* ---- bitmap: 4 bits used per 32-bit word (sizeof(word_t)*sizeof(char)) --- */
enum { kBitsPerWord = 4 };

void set_bit(word_t *words, int n) { words[n / kBitsPerWord] |= (word_t)1 << (n % kBitsPerWord); }

void clear_bit(word_t *words, int n) { words[n / kBitsPerWord] &= ~((word_t)1 << (n % kBitsPerWord)); }

int get_bit(word_t *words, int n) { return (words[n / kBitsPerWord] >> (n % kBitsPerWord)) & 1u; }

word_t *create_bitmap(int n) { return (word_t *)calloc((size_t)(n / kBitsPerWord) + 1, sizeof(word_t)); }

void delete_bitmap(word_t *words) { free(words); }

/* ---- input preparation ---------------------------------------------------- */

/* (3, n) float SoA -> (n, 4) double rows; column 3 is set to 0 (the reference
 * leaves it uninitialised: it is overwritten later by the density or the
 * Qhull lift). */
double *convert_to_qhdata(const float *rm_buff, size_t n_data) {
  double *q = (double *)malloc(n_data * 4 * sizeof(double));
  if (!q) return NULL;
  for (size_t i = 0; i < n_data; ++i) {
    q[4 * i + 0] = (double)rm_buff[i];
    q[4 * i + 1] = (double)rm_buff[n_data + i];
    q[4 * i + 2] = (double)rm_buff[2 * n_data + i];
    q[4 * i + 3] = 0.0;
  }
  return q;
}

/* Subsample without replacement: for i = 1 .. n_shuffle-1 the row drawn from
 * [i, n) by rand() % (n - i) + i trades places with row i-1, so the first
 * n_shuffle-1 rows end up a random subset; the draw sequence is the
 * reference's, so the same srand() seed gives the same subset. */
void shuffle_buff(double *data, int n_particles_in_buff, int n_shuffle) {
  for (int i = 1; i < n_shuffle; ++i) {
    const int r = rand() % (n_particles_in_buff - i) + i;
    double row[4];
    memcpy(row, data + 4 * (size_t)r, sizeof row);
    memcpy(data + 4 * (size_t)r, data + 4 * (size_t)(i - 1), sizeof row);
    memcpy(data + 4 * (size_t)(i - 1), row, sizeof row);
  }
}

static void mat3_mul(double out[3][3], const double a[3][3], const double b[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += a[i][k] * b[k][j];
      out[i][j] = acc;
    }
}

/* Rotation R = Rx(t0) Ry(t1) Rz(t2) applied about `center`. */
void rotate3d(double *data, size_t n_particles, double theta[3], double center[3]) {
  const double c0 = cos(theta[0]), s0 = sin(theta[0]);
  const double c1 = cos(theta[1]), s1 = sin(theta[1]);
  const double c2 = cos(theta[2]), s2 = sin(theta[2]);
  const double rx[3][3] = {{1.0, 0.0, 0.0}, {0.0, c0, -s0}, {0.0, s0, c0}};
  const double ry[3][3] = {{c1, 0.0, s1}, {0.0, 1.0, 0.0}, {-s1, 0.0, c1}};
  const double rz[3][3] = {{c2, -s2, 0.0}, {s2, c2, 0.0}, {0.0, 0.0, 1.0}};
  double rxy[3][3], r[3][3];
  mat3_mul(rxy, rx, ry);
  mat3_mul(r, rxy, rz);
  for (size_t i = 0; i < n_particles; ++i) {
    double *p = data + 4 * i;
    const double x = p[0] - center[0], y = p[1] - center[1], z = p[2] - center[2];
    p[0] = x * r[0][0] + y * r[0][1] + z * r[0][2] + center[0];
    p[1] = x * r[1][0] + y * r[1][1] + z * r[1][2] + center[1];
    p[2] = x * r[2][0] + y * r[2][1] + z * r[2][2] + center[2];
  }
}

/* ---- the layout step of triangulate() --------------------------------------- */

/* Qhull cells -> tetra_data rows.  Neighbour k of a cell lies across the facet
 * opposite vertex k, i.e. the reference's slot 4+k.  A cell whose
 * (AB x AC) . AD is positive has B and C swapped, and with them the
 * neighbours opposite B and C, so every tet ends with (AB x AC) . AD <= 0;
 * the test sums the dot product from 0 in x, y, z order like the reference. */
void dtfe_tetra_from_cells(const double *particle_data, const int *simplices, const int *neighbors,
                           size_t n_tetra, int *tetra_out) {
  for (size_t t = 0; t < n_tetra; ++t) {
    const int *s = simplices + 4 * t;
    const int *nb = neighbors + 4 * t;
    const double *a = particle_data + 4 * (size_t)s[0];
    const double *b = particle_data + 4 * (size_t)s[1];
    const double *c = particle_data + 4 * (size_t)s[2];
    const double *d = particle_data + 4 * (size_t)s[3];
    double ab[3], ac[3], ad[3];
    for (int k = 0; k < 3; ++k) {
      ab[k] = b[k] - a[k];
      ac[k] = c[k] - a[k];
      ad[k] = d[k] - a[k];
    }
    const double nrm[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2],
                           ab[0] * ac[1] - ab[1] * ac[0]};
    double dot = 0;
    for (int k = 0; k < 3; ++k) dot += nrm[k] * ad[k];
    const int swap = dot > 0;
    int *row = tetra_out + 8 * t;
    row[0] = s[0];
    row[1] = swap ? s[2] : s[1];
    row[2] = swap ? s[1] : s[2];
    row[3] = s[3];
    row[4] = nb[0];
    row[5] = swap ? nb[2] : nb[1];
    row[6] = swap ? nb[1] : nb[2];
    row[7] = nb[3];
  }
}
