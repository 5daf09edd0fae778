/*
 * dtfe.h - drop-in for the reference's src/dtfe.h:13-21.  Same symbols and
 * signatures; the work runs on the GPU through the handle API of
 * sdtfe_b200.h.
 *
 * Conventions kept from the reference:
 *   - particle_data is (n_particles, 4) doubles; its column 3 is overwritten
 *     with the DTFE density (compute_density, compute_3d_density) exactly as
 *     pre_compute_vol does in place;
 *   - rho / grid are caller-allocated and ACCUMULATED (+=); callers zero them;
 *   - no return codes: failures are reported on stderr and through
 *     dtfe_last_error(), leaving the output untouched.
 * Differences:
 *   - Monte Carlo offsets come from the counter-based generator of
 *     sdtfe_rng.h keyed by one rand() draw per call (or dtfe_set_seed), so a
 *     map is reproducible for a given seed whatever the thread count;
 *   - any grid_dim >= 1 is accepted (the reference's 4x4 pixel tiling needs
 *     grid_dim % 4 == 0, src/dtfe.c:601-614);
 *   - the arithmetic of the walk follows dtfe_set_default_precision
 *     (DTFE_FP64 by default: the reference's FP64 operations in order).
 */
#ifndef SDTFE_DTFE_H
#define SDTFE_DTFE_H

#include <stdint.h>
#include "constants.h"
#include "bitmap.h"

#ifdef __cplusplus
extern "C" {
#endif

/* src/dtfe.h:13-15, src/dtfe.c:554-654 */
void compute_density(double *particle_data, int n_particles, int *tetra_data, int n_tetra,
                     int grid_dim, double box_len, double box_len_z, double *rho, float p_mass,
                     double center_x, double center_y, double center_z, const int n_mc_samp,
                     const double delta_sample);

/* src/dtfe.h:17-18, src/dtfe.c:668-735: column 3 of particle_data is the field */
void interpolate_to_3d_grid(double *particle_data, int n_particles, int *tetra_data, int n_tetra,
                            int grid_dim, double box_len, double *grid, double center_x,
                            double center_y, double center_z, unsigned supersampling);

/* src/dtfe.h:20-21, src/dtfe.c:658-665 */
void compute_3d_density(double *particle_data, int n_particles, int *tetra_data, int n_tetra,
                        int grid_dim, double box_len, double *rho, float p_mass, double center_x,
                        double center_y, double center_z, unsigned supersampling);

#ifdef __cplusplus
}
#endif
#endif
