/*
 * triangulate.h - drop-in for the reference's src/triangulate.h:11-15.
 *
 * triangulate() keeps its signature; Qhull itself is not linked into this
 * library, so the Delaunay cells come from the host backend registered with
 * dtfe_set_triangulator() (the Python binding registers Qhull through SciPy),
 * and the result is laid out exactly as src/triangulate.c:63-175 does.  With no
 * backend registered it prints an error and returns NULL, the reference's own
 * failure value (src/triangulate.c:149-154).
 *
 * The other four run on the GPU and return the reference's layouts; buffers
 * returned by pointer are malloc'd and freed by the caller.
 */
#ifndef SDTFE_TRIANGULATE_H
#define SDTFE_TRIANGULATE_H

#include <stddef.h>
#include "bitmap.h"

#ifdef __cplusplus
extern "C" {
#endif

int *triangulate(double *particle_data, int n_particles, size_t *num_facets, const char *options);
void pre_compute_vol(double **particle_data, int n_particles, int *tetra_data, int n_tetra,
                     float p_mass);                                      /* :183-225 */
double *gradients(int *tetra_data, int n_tetra, double *particle_data); /* :233-260 */
int find_forward_hull(int *tetra_data, int n_tetra, double *particle_data, int n_particles,
                      word_t *bitmap);                                   /* :263-316 */
int *copy_fh_triangles(int *tetra_data, int n_tetra, double *particle_data, int n_particles,
                       int n_tri, word_t *bitmap);                       /* :318-395 */

#ifdef __cplusplus
}
#endif
#endif
