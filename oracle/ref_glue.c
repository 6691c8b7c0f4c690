/* Exports the reference's header-only host helpers (src/core/lod.h,
 * src/core/mathx.h) as plain functions so the test suite can call the
 * reference's own code through ctypes.  Compiled against the reference tree
 * in place by oracle/Makefile; test infrastructure only. */
#include <stdint.h>

#include "core/lod.h"
#include "core/mathx.h"

uint32_t ref_lod_pick(float distance, float pixel_cone, float base_voxels, uint32_t nlevels) {
  return r3d_lod_pick(distance, pixel_cone, base_voxels, nlevels);
}

uint32_t ref_lod_fallback(uint32_t desired, uint32_t ordinal, uint32_t nlevels) {
  return r3d_lod_fallback(desired, ordinal, nlevels);
}

void ref_m3_ypr(float yaw, float pitch, float roll, float rows[9]) {
  r3d_m3 m = m3_ypr(yaw, pitch, roll);
  rows[0] = m.r0.x, rows[1] = m.r0.y, rows[2] = m.r0.z;
  rows[3] = m.r1.x, rows[4] = m.r1.y, rows[5] = m.r1.z;
  rows[6] = m.r2.x, rows[7] = m.r2.y, rows[8] = m.r2.z;
}
