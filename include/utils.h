/*
 * utils.h - drop-in for the reference's src/utils.h:10-12 (host-side input
 * preparation, run on the CPU as in the reference).
 */
#ifndef SDTFE_UTILS_H
#define SDTFE_UTILS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* float SoA (3, n) -> malloc'd double (n, 4) rows, column 3 zero (src/utils.c:8-16) */
double *convert_to_qhdata(const float *rm_buff, size_t n_data);
/* rotation by Qx(t0) Qy(t1) Qz(t2) about center, rows (n, 4) (src/utils.c:33-79) */
void rotate3d(double *data, size_t n_particles, double theta[3], double center[3]);
/* partial Fisher-Yates with the C library rand() (src/utils.c:18-30) */
void shuffle_buff(double *data, int n_particles_in_buff, int n_shuffle);

#ifdef __cplusplus
}
#endif
#endif
