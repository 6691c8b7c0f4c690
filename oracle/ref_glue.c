/* Exports the reference's header-only host helpers (src/core/lod.h,
 * src/core/mathx.h, and the layout math of the section modes in
 * src/core/slab.h, clip.h, vslab.h) as plain functions so the test suite
 * can call the reference's own code through ctypes.  Compiled against the reference tree
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

/* ---- the section modes' layout math (src/core/slab.h, clip.h, vslab.h) ---- */

#include "core/clip.h"
#include "core/slab.h"
#include "core/vslab.h"

/* slab layout: out = gx, gy, px, py, ovs, overview levels, then per
 * overview level k < 6: gx, gy, px, py (r3d_slab_ov_layout) */
int ref_slab_layout(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t wz, uint32_t out[30]) {
  r3d_slab_layout l;
  if (r3d_slab_layout_init(&l, nx, ny, nz, wz) != 0) return -1;
  out[0] = l.gx, out[1] = l.gy, out[2] = l.px, out[3] = l.py, out[4] = l.ovs;
  uint32_t n = r3d_slab_ov_levels(&l);
  out[5] = n;
  for (uint32_t k = 0; k < n && k < 6; k++) {
    r3d_slab_layout o;
    r3d_slab_ov_layout(&l, k, &o);
    out[6 + 4 * k] = o.gx, out[7 + 4 * k] = o.gy, out[8 + 4 * k] = o.px, out[9 + 4 * k] = o.py;
  }
  return 0;
}

/* clipmap origins over a focus sequence: r3d_clip_init at the first focus,
 * then per later focus each level recentred when r3d_clip_need_recenter
 * (the update loop of src/vk/vkclip.c:320-346); origins (n x 6 x 2) and
 * the ring depths (6) */
void ref_clip_sequence(uint64_t nx, uint64_t ny, uint64_t nz, uint32_t depth, uint32_t n,
                       const int64_t *focus, int64_t *origins, uint32_t wzl[6]) {
  r3d_clip c;
  r3d_clip_init(&c, nx, ny, nz, depth, focus[0], focus[1]);
  for (uint32_t f = 0; f < n; f++) {
    if (f)
      for (uint32_t l = 0; l < R3D_CLIP_LEVELS; l++)
        if (r3d_clip_need_recenter(&c, l, focus[2 * f], focus[2 * f + 1]))
          r3d_clip_recenter(&c, l, focus[2 * f], focus[2 * f + 1]);
    for (uint32_t l = 0; l < R3D_CLIP_LEVELS; l++) {
      origins[(f * 6 + l) * 2] = c.lv[l].ox;
      origins[(f * 6 + l) * 2 + 1] = c.lv[l].oy;
    }
  }
  for (uint32_t l = 0; l < R3D_CLIP_LEVELS; l++) wzl[l] = c.lv[l].wzl;
}

/* virtual-slab layout: out = px, wz, ntiles, gx[5], gy[5], base[5] */
int ref_vslab_layout(uint64_t nx, uint64_t ny, uint64_t nz, uint32_t W, uint32_t H, uint32_t D,
                     uint32_t margin, uint32_t out[18]) {
  r3d_vslab v;
  if (r3d_vslab_init_margin(&v, nx, ny, nz, W, H, D, margin) != 0) return -1;
  out[0] = v.px, out[1] = v.wz, out[2] = v.ntiles;
  for (uint32_t l = 0; l < R3D_VS_LEVELS; l++)
    out[3 + l] = v.lv[l].gx, out[8 + l] = v.lv[l].gy, out[13 + l] = v.lv[l].base;
  return 0;
}

void ref_vslab_ranges(uint64_t nx, uint64_t ny, uint64_t nz, uint32_t W, uint32_t H, uint32_t D,
                      uint32_t margin, int64_t o, int64_t z0, int64_t out[4]) {
  r3d_vslab v;
  if (r3d_vslab_init_margin(&v, nx, ny, nz, W, H, D, margin) != 0) return;
  r3d_vs_range(&v, 0, o, nx, W, &out[0], &out[1]);
  r3d_vs_zrange(&v, z0, &out[2], &out[3]);
}
