// walk32.cu - mixed-precision surface-density map (FP32 walk, guarded FP64).
#include "mesh.h"

namespace sdtfe {

dtfe_status_t launch_map32(Mesh& m, const MapGeom& g, double* d_map, cudaStream_t s,
                           double* ray_rho, int* ray_crossed, int* ray_status) {
  (void)m; (void)g; (void)d_map; (void)s; (void)ray_rho; (void)ray_crossed; (void)ray_status;
  return set_error(DTFE_ERR_UNSUPPORTED, "mixed-precision map not built yet");
}

dtfe_status_t launch_trace32(Mesh& m, int n_rays, const double* d_x, const double* d_y, double z0,
                             double lz, double dxy, uint64_t seed, int max_visits, double* d_rho,
                             int* d_crossed, int* d_status, int* d_visits, int max_record,
                             cudaStream_t s) {
  (void)m; (void)n_rays; (void)d_x; (void)d_y; (void)z0; (void)lz; (void)dxy; (void)seed;
  (void)max_visits; (void)d_rho; (void)d_crossed; (void)d_status; (void)d_visits; (void)max_record;
  (void)s;
  return set_error(DTFE_ERR_UNSUPPORTED, "mixed-precision trace not built yet");
}

}  // namespace sdtfe
