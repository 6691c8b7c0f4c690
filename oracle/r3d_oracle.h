/* CPU oracle for the volume raycast: test infrastructure, not product code.
 *
 * A plain-C restatement of render3d's raycast compute shader
 * (src/shaders/raycast.slang:117-295,409-416,457-495,505-1039 and
 * src/shaders/common.slang:44-61) plus the data the shader samples: mip chain,
 * 8^3 occupancy grid (src/vk/vkbackend.c:794-870,944-983), LOD brick pyramid
 * and page table (src/vk/vkbackend.c:4184-4206, tools/lodpack/main.c:203-230).
 *
 * Texture units are restated as exact FP32 arithmetic: clamp-to-edge
 * trilinear at texel centres, linear blending between mip floor(lod) and
 * floor(lod)+1, 1-D linear TF lookup at v*256-0.5, and round-to-nearest RGBA8
 * stores.  Every floating-point step is written out in a fixed order with
 * explicit fmaf and no contraction, so that the sm_100a kernels, which follow
 * the same arithmetic, reproduce it bit for bit.
 *
 * Only the test suite, the smoke check and the CPU baseline of the benchmark
 * use this code; the renderer library never links it. */
#ifndef R3D_ORACLE_H
#define R3D_ORACLE_H

#include <stdint.h>

#include "r3d_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_LEVELS 16

/* Cube volume with its mip chain (level 0 = the volume, x fastest). */
typedef struct orc_cube {
  uint32_t nlevels;
  uint32_t dim[ORC_MAX_LEVELS][3];
  const uint8_t *level[ORC_MAX_LEVELS];
  const uint8_t *occ; /* dilated 8^3 block maxima, x fastest */
  uint32_t odim[3];
} orc_cube;

/* Tiled slab (src/core/slab.h, raycast.slang:423-455): per level (0 base,
 * 1.. overview at scale 4 << (level - 1)) gx * gy tiles of (px + 2) x
 * (py + 2) x wz texels, tile k at tiles[level] + k * tile bytes; ring
 * layer s % wz holds world slice s.  z0 is the window start. */
typedef struct orc_slab {
  uint32_t wz, nlev, ovs, nx, ny, z0;
  uint32_t lev[8][4]; /* gx, gy, px, py */
  const uint8_t *tiles[8];
} orc_slab;

/* XY clipmap (src/core/clip.h, raycast.slang:357-408): level l is a
 * 2048 x 2048 x wzl[l] texture, ring layer ls % wzl[l] holding level
 * slice ls; ox, oy are the level origins (clip_orig), valid the level mask,
 * nx the volume width and z0 the window start. */
typedef struct orc_clip {
  uint32_t wzl[6];
  const uint8_t *lev[6];
  float ox[6], oy[6];
  uint32_t valid, nx, z0;
} orc_clip;

/* Virtual slab (src/core/vslab.h, raycast.slang:321-367): level l
 * (spacing 1, 4, 8, 16, 32; gx = 0 absent) has gx x gy tiles from tile
 * base[l] of the pool, each (px + 2)^2 texels by wz ring slices; table holds
 * four words per base tile (key, za, zb, 0).  Views carry the window origin
 * and grids in their frame parameters. */
typedef struct orc_vslab {
  uint32_t px, wz, ntiles;
  uint32_t gx[5], gy[5], base[5];
  uint8_t *tiles;
  uint32_t *table;
} orc_vslab;

/* Flattened segment (src/shaders/surfvol.comp, raycast.slang:515-638):
 * gw x gh grids of surface points (x, y, z, valid) and normals (x, y, z, -),
 * the baked W x H x L flattened volume (CT and overlay bytes per texel, x
 * fastest) and an optional mw x mh supervision mask. */
typedef struct orc_surf {
  const float *coords, *normals;
  uint32_t gw, gh;
  uint8_t *vol;
  uint32_t W, H, L;
  const uint8_t *mask;
  uint32_t mw, mh;
  /* live 2.5D ink prediction (NULL: none): pw x ph floats, texel (0, 0) at
   * grid coordinates (pg0u, pg0v), pppg texels per grid unit */
  const float *pred;
  uint32_t pw, ph;
  float pg0u, pg0v, pppg;
} orc_surf;

/* Brick cache.  LOD mode (brick_mode with the LOD flag): the page table in
 * render3d's word format and a pool of 128^3 slots (slot s at
 * pool + s * 128^3, x fastest).  Single-level mode (no LOD flag,
 * src/shaders/raycast.slang:163-180,800-822): page holds bpa^3 entries and
 * atlas is the (abpa * 128)^3 atlas texture with its 4 mips, its occ field
 * being the world-indexed (bpa * 16)^3 dilated occupancy grid. */
typedef struct orc_bricks {
  const uint32_t *page;
  uint32_t page_words;
  const uint8_t *pool;
  uint32_t nslots;
  const orc_cube *atlas;
  /* LOD mode: slot-parallel overlay atlases in the pool's layout (ink,
   * 3D ink, labels, registration; NULL when absent), sampled per
   * src/shaders/raycast.slang:45-115,872-914,1000-1014,1032-1036 */
  const uint8_t *ovl[4];
  /* slab views (slab_grid != 0) and clip views (clip_valid != 0) sample these */
  const orc_slab *slab;
  const orc_clip *clip;
  const orc_vslab *vslab; /* virtual-slab views (slab_grid bit 24) */
  const orc_surf *surf;   /* flattened-segment views (R3D_VIEW_SURF) */
} orc_bricks;

typedef struct orc_opts {
  float alpha_cutoff; /* front-to-back termination opacity; reference 0.98 */
  uint32_t quality;   /* R3D_QUALITY_FULL / R3D_QUALITY_FAST */
  int threads;        /* OpenMP threads over rows; <= 0: all */
} orc_opts;

/* Per-pixel auxiliary outputs (all nullable, img_w * img_h each). */
typedef struct orc_aux {
  uint32_t *steps;     /* loop iterations of the ray (heatmap counter) */
  uint32_t *mip_index; /* step index at which the MIP maximum was last raised */
  uint64_t total_steps; /* sum over rays (out) */
  uint32_t status;      /* bit 0: a page entry or slot was out of range */
} orc_aux;

/* Renders one view into the RGBA8 image (img_w x img_h, the view's rect at
 * view_org, already sanitized to lie inside the image).  The scene pointer
 * matching p->brick_mode must be non-NULL.  Returns 0 or -1 on bad input. */
int orc_render_view(const r3d_frame_params *p, const orc_cube *cube, const orc_bricks *bricks,
                    const uint8_t lut[256][4], const orc_opts *o, uint8_t *img, uint32_t img_w,
                    uint32_t img_h, orc_aux *aux);

/* Renders only the rays of the listed pixels (view-local thread coordinates,
 * 2 * n entries); colours go to out_rgba (4 * n), steps / mip_index to the
 * nullable arrays (n).  Used for sampled parity checks at full resolution. */
int orc_render_pixels(const r3d_frame_params *p, const orc_cube *cube, const orc_bricks *bricks,
                      const uint8_t lut[256][4], const orc_opts *o, const uint32_t *xy,
                      uint32_t n, uint8_t *out_rgba, uint32_t *steps, uint32_t *mip_index);

/* Differentiable emission-absorption render over an FP32 density grid
 * (n[0] x n[1] x n[2], x fastest) and an FP32 256x4 TF (see
 * r3d_oracle_diff.c).  orc_diff_forward32: FP32 RGB image (w*h*3) exactly as
 * the kernel computes it, and the per-ray step counts (nullable).
 * orc_diff_grad64: FP64 render (rgb64_out, nullable) and the gradients of
 * sum(dl_drgb * rgb) with respect to the voxels (g_dens), the LUT (g_lut,
 * 256*4) and the density scale (g_density), all accumulated (+=).
 * decisions32: contributing samples and termination as in the FP32 render
 * of (dec_dens, dec_lut), or of (dens, lut) when those are NULL. */
int orc_diff_forward32(const r3d_frame_params *pc, const float *dens, const uint32_t n[3],
                       const float *lut, float cutoff, float *rgb_out, uint32_t *steps_out,
                       int threads);
int orc_diff_grad64(const r3d_frame_params *pc, const float *dens, const uint32_t n[3],
                    const float *lut, float cutoff, const float *dl_drgb, int decisions32,
                    const float *dec_dens, const float *dec_lut, double *g_dens, double *g_lut,
                    double *g_density, double *rgb64_out, int threads);

/* CPU build of the shared log2 / exp2 / pow / x^24 (4 outputs per input). */
void orc_fmath_eval(const float *x, const float *y, float *out, uint32_t n);

/* Mip level sizes for a cube: level m is max(1, dim >> m); returns the level
 * count floor(log2(maxdim)) + 1 (src/vk/vkbackend.c:1517-1518). */
uint32_t orc_mip_levels(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t dims[][3]);

/* One 2x box reduction: dst = (sum of the 8 children + 4) / 8 with source
 * coordinates clamped to the source extent. */
void orc_downsample(const uint8_t *src, uint32_t sx, uint32_t sy, uint32_t sz, uint8_t *dst,
                    uint32_t dx, uint32_t dy, uint32_t dz);

/* 8^3 block maxima followed by 26-neighbour max dilation
 * (src/vk/vkbackend.c:794-870).  out holds ceil(n/8) per axis. */
void orc_occupancy(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint8_t *out);

/* LOD brick cache from a raw volume: level l is the (sum+4)/8 box pyramid
 * over the zero-padded brick grid, levels [0, nlev); a brick is resident when
 * its maximum is >= min_max.  Slots are assigned in (level, z, y, x) order.
 * Writes the page table (page_words = 64 + total bricks) and, if pool is not
 * NULL, the slot contents.  Returns the number of resident bricks, or -1. */
int64_t orc_build_lod_bricks(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz,
                             uint32_t nlev, uint32_t min_max, uint32_t *page,
                             uint32_t page_words, uint8_t *pool, uint64_t pool_slots);
uint32_t orc_lod_page_words(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t nlev);

/* Slot contents of an overlay atlas for an existing LOD page table: each
 * resident brick (level l, slot s) receives the same brick of the overlay
 * volume's level l -- the (sum+4)/8 box pyramid of orc_build_lod_bricks,
 * or with labels != 0 the level-0 voxel at (x, y, z) << l
 * (src/core/labelvol.c:172-196).  pool holds nslots * 128^3 bytes and is
 * written only at resident slots.  Returns 0, or -1 on bad input. */
int orc_build_lod_overlay(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz,
                          const uint32_t *page, uint32_t page_words, int labels, uint8_t *pool,
                          uint32_t nslots);

/* Slab layout of an nx x ny plane with ring depth wz (slab.h:42-62,
 * 122-135): per level gx, gy, px, py; returns the level count (base +
 * overview) and the overview scale, or 0 when the plane needs more than
 * 22 tiles per axis. */
uint32_t orc_slab_layout(uint32_t nx, uint32_t ny, uint32_t lev[8][4], uint32_t *ovs);
/* Tiles of every level for the window [z0, z0 + wz) of a volume, as the
 * reference assembles them (vkbackend.c:2128-2164,2280-2325); tiles[l]
 * must hold gx * gy * (px + 2) * (py + 2) * wz bytes of level l. */
void orc_slab_fill(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t wz,
                   uint32_t z0, uint8_t *const tiles[8]);

/* Clipmap level textures for the window from z0 with the given level
 * origins (vkclip.c:101-185, tools/mkpyramid): level 0 the volume, level 1
 * its truncating 2^3 box with coordinates clamped at full resolution,
 * levels 2..5 the tight truncating 2^3 box pyramid clamped at its own
 * extent; texel (tx, ty) is level voxel (ox / 2^l - 1 + tx, oy / 2^l - 1 +
 * ty); slices outside the volume are zero.  wzl[l] = max(depth_max / 2^l
 * + 3, 4); tex[l] holds 2048 * 2048 * wzl[l] bytes. */
void orc_clip_fill(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t depth_max,
                   uint32_t z0, const float orig[6][2], uint8_t *const tex[6]);

/* One virtual-slab fill (vkbackend.c:5985-6125): slices [zs0, zs0 + nz) of
 * base cell (cx, cy) into its base tile (texel (tx, ty) holds world voxel
 * (cx px - 1 + tx, cy px - 1 + ty) clamped up to 0, zero past the volume's
 * far edges), then each present pyramid level's strip (truncating 4x4 box
 * of the payload, then 2x2 boxes) into the tiles it overlaps, aprons
 * included (vkbackend.c:6032-6057).  Ring layer of slice z: z % wz. */
void orc_vslab_fill(orc_vslab *v, const uint8_t *vox, uint32_t nx, uint32_t ny, int64_t cx,
                    int64_t cy, int64_t zs0, uint32_t nz);

/* The bake of surfvol.comp:98-153 over the whole window: texel (x, y, l)
 * samples the LOD brick cache br (page, pool; ovl[ovl] into the second byte
 * when ovl >= 0) at surface(u, v) + normal(u, v) * (zoff0 + l - nback),
 * u = u0 + (x + 0.5) step, at the level of the xy pitch. */
void orc_surf_bake(orc_surf *sf, const orc_bricks *br, float u0, float v0, float step,
                   float zoff0, float sx, float sy, uint32_t nback, int ovl);

/* Single-level brick atlas from a cubic volume of edge bpa * 128: atlas
 * level 0 ((abpa * 128)^3, slot s at (s % abpa, s / abpa % abpa,
 * s / abpa^2) * 128, zeros where no brick sits) and the page table (bpa^3
 * words, slot | brick max << 24, or 0xFFFFFFFF).  slot_of[b] is brick b's
 * slot or 0xFFFFFFFF; NULL puts brick b in slot b (abpa == bpa).  Returns 1
 * when every brick sits in its own slot (identity layout), 0 otherwise, -1
 * on bad input.  Atlas mips come from orc_downsample
 * (src/vk/vkbackend.c:4236-4273,3241-3330). */
int orc_build_shard(const uint8_t *vox, uint32_t edge, uint32_t abpa, const uint32_t *slot_of,
                    uint32_t *page, uint8_t *atlas0);

/* World-indexed occupancy of a single-level atlas (src/shaders/occmax.comp,
 * occdilate.comp): block w of the (bpa * 16)^3 grid is the maximum of the
 * 8^3 atlas texels of its brick's slot (0 for absent bricks), followed by
 * 26-neighbour max dilation. */
void orc_shard_occupancy(const uint8_t *atlas0, uint32_t abpa, const uint32_t *page, uint32_t bpa,
                         uint8_t *out);

/* Host-side camera / TF helpers restated from src/core/camera.c:5-75,
 * src/core/transfer.c:5-50, src/core/lod.h:8-26 and src/core/mathx.h:34-43,
 * for checking the library's own versions against the reference. */
void orc_camera_basis(float yaw, float pitch, float fov_y, float aspect, float right[3],
                      float up[3], float fwd[3]);
void orc_orbit_pos(float yaw, float pitch, const float target[3], float dist, float pos[3]);
void orc_tf_build(const uint8_t *values, const uint8_t (*rgba)[4], uint32_t npts,
                  uint8_t lut[256][4]);
uint32_t orc_lod_pick(float distance, float pixel_cone, float base_voxels, uint32_t nlevels);
uint32_t orc_lod_fallback(uint32_t desired, uint32_t ordinal, uint32_t nlevels);
void orc_m3_ypr(float yaw, float pitch, float roll, float rows[3][3]);

/* The benchmark's inputs, restated here so that the CPU baseline needs
 * nothing from the library under test: the scripted orbit view
 * (src/main.c:3932-3946 with src/core/camera.c's basis) and the seeded
 * scroll phantom. */
void orc_orbit_view(r3d_frame_params *p, float ph, const float target[3], uint32_t w, uint32_t h,
                    float step_voxels, float density, float lod_bias, uint32_t mode,
                    uint32_t frame_index, float low_cut, const uint8_t lut[256][4]);
int orc_phantom(uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint64_t seed, int threads);

/* Post-decode display filter of n 128^3 slots in place (src/shaders/
 * postfilt.comp run by src/vk/vkbackend.c:3398-3466): mode low byte 1
 * median of 3^3, 2 median of 5^3, 3 max of 3^3, 4 max of 5^3, then the
 * unsharp pass when bit 8 is set; neighbourhoods clamp to the slot. */
void orc_postfilter(uint8_t *slots, uint32_t n, uint32_t mode, float amount);

#ifdef __cplusplus
}
#endif

#endif /* R3D_ORACLE_H */
