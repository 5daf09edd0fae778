// walk32.cuh - record layout of the mixed-precision walk.
#pragma once

#include <cstdint>

namespace sdtfe {

// 80 B per (tet, entry face), 4 per tet: the mixed walk's records.  Record
// 4*t + F is the tet seen by a ray that entered it through face F: slots 0..2
// hold face F's vertices (in the order the face is listed in: BDC, ACD, ADB,
// ABC), slot 3 the vertex opposite it.  The fast step reads one of these: the
// entry face is known, so every slot is fixed and only the exit face (opposite
// slot 0, 1 or 2) is chosen.  Record 4*t + 3 has the vertices in the mesh's
// own order A..D, which is how the general step reads a tet.
struct __align__(16) TetRot32 {
  float4 xy01;  // (x0, y0, x1, y1)
  float4 xy23;  // (x2, y2, x3, y3)
  float4 z;     // (z0, z1, z2, z3)
  float4 fld;   // (rho3, grad_x, grad_y, grad_z): the tet's linear field from the
                // apex, gradient in the projected frame
  int4 nb;      // x..z: record 4*n + F' of the neighbour n across the face opposite
                // slot 0..2, F' the face of n shared with this tet; -1 on the hull,
                // INT_MIN when n does not list this tet; w: the float bits of the
                // extent of the tet's projection (largest x or y difference of
                // two vertices, rounded up), a bound on |vertex - origin| for
                // any ray that crossed one of its faces, with the sign bit set
                // when the FP32 field value is not trusted (kFieldCond)
};
// largest field condition (magnitudes over least vertex value) the FP32
// field value is used for
constexpr double kFieldCond = 4096.0;
static_assert(sizeof(TetRot32) == 80, "TetRot32 layout");

// Original vertex slot of rotated slot k for entry face F, and its inverse;
// two bits per entry, one byte per F.
constexpr uint32_t kRotSlots = 0xE49C782Du;
constexpr uint32_t kRotInverse = 0xE4789C63u;
__host__ __device__ constexpr int rot_slot(int F, int k) { return (int)((kRotSlots >> (8 * F + 2 * k)) & 3u); }
__host__ __device__ constexpr int rot_inv(int F, int v) { return (int)((kRotInverse >> (8 * F + 2 * v)) & 3u); }

}  // namespace sdtfe
