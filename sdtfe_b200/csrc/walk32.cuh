// walk32.cuh - record layout of the mixed-precision walk.
#pragma once

#include <cstdint>

namespace sdtfe {

// 96 B per tet: everything one FP32 walk step reads, in six 16-byte words.
struct __align__(32) TetRec32 {
  float4 xyab;  // (x_A, y_A, x_B, y_B) in the projected frame
  float4 xycd;  // (x_C, y_C, x_D, y_D)
  float4 z;     // (z_A, z_B, z_C, z_D)
  float4 fld;   // (rho_A, rho_B, rho_C, rho_D): vertex densities (or field values)
  int4 nb;      // neighbours across faces BDC, ACD, ADB, ABC (-1: hull)
  int4 aux;     // vertex ids A..D
};
static_assert(sizeof(TetRec32) == 96, "TetRec32 layout");

}  // namespace sdtfe
