/*
 * io.h - drop-in for the reference's src/io.h: the map writers of its example
 * driver (src/main.c:184-185).
 *
 * write_rho writes the map's doubles raw (src/io.c:89-95).  write_image
 * writes an 8-bit palette TIFF of log(rho + 1), scaled as src/io.c:13-47
 * does, with a Jet colour map; libtiff is not used: the file is a baseline
 * TIFF (one uncompressed strip) written directly.
 */
#ifndef SDTFE_IO_H
#define SDTFE_IO_H

#include <stdint.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum Read_Opt { POS, VEL, POSVEL } read_opt;

typedef struct fof_halo_properties {
  int32_t fof_halo_count;
  int64_t fof_halo_tag;
  float fof_halo_mass;
  float fof_halo_center_x;
  float fof_halo_center_y;
  float fof_halo_center_z;
  float fof_halo_mean_x;
  float fof_halo_mean_y;
  float fof_halo_mean_z;
  float fof_halo_mean_vx;
  float fof_halo_mean_vy;
  float fof_halo_mean_vz;
  float fof_halo_vel_disp;
  float redshift;
} fof_halo_properties;

typedef struct particle_data {
  float *x;
  float *y;
  float *z;
  float *vx;
  float *vy;
  float *vz;
} particle_data;

void write_image(char *file_name, double *rho, int grid_dim); /* src/io.c:13-85 */
int write_rho(char *fname, double **rho, int rho_size);       /* src/io.c:89-95 */

#ifdef __cplusplus
}
#endif
#endif
