/* Host-side inputs of the raycast: camera basis, turntable orbit, volume
 * rotation, transfer-function LUTs and presets, the skip gate, the LOD
 * policy, the scripted benchmark orbit, and the seeded scroll phantom.
 *
 * These restate render3d's core helpers (src/core/camera.c:5-75,
 * src/core/mathx.h:34-43, src/core/transfer.c:5-50, src/core/lod.h:8-26,
 * src/main.c:1238-1242,3932-3946,6788-6824) under an r3d_host_ prefix so
 * that they link beside the reference's own core library without clashing.
 * With -ffp-contract=off they produce the same bits as the reference's. */
#ifndef R3D_HOST_H
#define R3D_HOST_H

#include <stdint.h>

#include "r3d_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct r3d_host_camera {
  float pos[3];
  float yaw, pitch, fov_y; /* radians; fov defaults to 60 degrees */
  float target[3];
  float dist;
} r3d_host_camera;

void r3d_host_camera_init(r3d_host_camera *c, const float pos[3]);
void r3d_host_camera_look(r3d_host_camera *c, float dyaw, float dpitch);
void r3d_host_camera_move(r3d_host_camera *c, const float local[3], float dist);
void r3d_host_camera_orbit_set(r3d_host_camera *c, const float target[3], float dist);
void r3d_host_camera_orbit_drag(r3d_host_camera *c, float dyaw, float dpitch);
void r3d_host_camera_orbit_zoom(r3d_host_camera *c, float factor);
/* right/up pre-scaled by tan(fov/2)*aspect and tan(fov/2). */
void r3d_host_camera_basis(const r3d_host_camera *c, float aspect, float right[3], float up[3],
                           float fwd[3]);
/* rows of R = Ry(yaw) Rx(pitch) Rz(roll) */
void r3d_host_m3_ypr(float yaw, float pitch, float roll, float rows[3][3]);

/* Piecewise-linear TF points -> LUT with render3d's integer lerp. */
void r3d_host_tf_build(const uint8_t *values, const uint8_t (*rgba)[4], uint32_t npts,
                       uint8_t lut[256][4]);
/* Presets 0 grey ramp, 1 scroll, 2 high-pass; returns idx, or the preset
 * count (3) when idx is out of range (lut untouched). */
uint32_t r3d_host_tf_preset(uint32_t idx, uint8_t lut[256][4]);
/* First value with nonzero alpha (255 if none). */
float r3d_host_tf_min_visible(const uint8_t lut[256][4]);
/* skip_gate = max(low_cut, tf_min_visible - 0.5) / 255. */
float r3d_host_skip_gate(float low_cut, const uint8_t lut[256][4]);

uint32_t r3d_host_lod_pick(float distance, float pixel_cone, float base_voxels,
                           uint32_t nlevels);
uint32_t r3d_host_lod_fallback(uint32_t desired, uint32_t ordinal, uint32_t nlevels);

/* View-cone LOD request of the brick streamer (src/vk/vkbackend.c:3082-3106,
 * 5416-5500): for every level but the coarsest, the bricks inside the
 * level's distance shell whose centre lies in the widened view cone
 * (half_tan * 1.15 + 1e-3) or near the eye, and whose desired level
 * (r3d_host_lod_pick of the centre distance) is that level.  Each one adds
 * its parent (priority 0) and itself (priority 1), both with its squared
 * distance; bricks whose maximum in page (the full pyramid's page table,
 * every brick present) is below max(gate * 255 + 0.5, 5) are left out, and
 * a brick is listed once (its first entry).  slice_depth > 0 limits z to
 * [slice_z0, slice_z0 + slice_depth).  mark (page_words bytes, zeroed by
 * the caller) records listed bricks.  Returns the number of candidates
 * written (at most cap), sorted by priority, then distance. */
typedef struct r3d_stream_cand {
  float d2;
  uint32_t brick;    /* page-table word index */
  uint32_t priority; /* 0: parent kept ahead of its children, 1: desired */
} r3d_stream_cand;
uint32_t r3d_host_stream_desired(const uint32_t *page, uint32_t page_words, const float eye[3],
                                 const float fwd[3], float half_tan, float pixel_cone,
                                 uint32_t slice_z0, uint32_t slice_depth, float gate,
                                 uint8_t *mark, r3d_stream_cand *out, uint32_t cap);
/* The multi-view collects (src/vk/vkbackend.c:5330-5414), appending to the
 * n candidates already in out with the same mark, gate and listing rules,
 * unsorted; each returns the new count.  _box: a volume-normalized box;
 * the level whose voxel pitch matches pixel_cone (floor(log2(max(pixel_cone
 * * max(shape), 1)))), coarsened one level at a time until the box holds at
 * most 2048 of its bricks; each brick of the box adds its parent
 * (priority 0, absent at the coarsest level) and itself (priority 1), with
 * the squared distance of its centre from the box's centre.  _point: the
 * brick of `level` (clamped to the coarsest) containing p, clamped to the
 * level's grid, after its parent; both at distance 0. */
uint32_t r3d_host_stream_box(const uint32_t *page, uint32_t page_words, const float lo[3],
                             const float hi[3], float pixel_cone, float gate, uint8_t *mark,
                             r3d_stream_cand *out, uint32_t cap, uint32_t n);
uint32_t r3d_host_stream_point(const uint32_t *page, uint32_t page_words, const float p[3],
                               uint32_t level, float gate, uint8_t *mark, r3d_stream_cand *out,
                               uint32_t cap, uint32_t n);
/* Sorts candidates by priority, then distance, then brick. */
void r3d_host_stream_sort(r3d_stream_cand *c, uint32_t n);

/* A CPU-sourced slot-parallel atlas (labels, registration; reference
 * r3d_label_src, src/render/render.h:80-101): gen(level, bx, by, bz) is a
 * cheap content generation of a brick (0: no content), fetch(...) fills
 * the brick's 128^3 bytes, x fastest. */
typedef struct r3d_brick_src {
  uint32_t (*gen)(void *user, uint32_t level, uint32_t bx, uint32_t by, uint32_t bz);
  void (*fetch)(void *user, uint32_t level, uint32_t bx, uint32_t by, uint32_t bz, uint8_t *out);
  void *user;
} r3d_brick_src;

/* Level and brick coordinates of page-table word b (b in a level's range). */
int r3d_host_brick_locate(const uint32_t *page, uint32_t b, uint32_t *level, uint32_t *bx,
                          uint32_t *by, uint32_t *bz);

/* One sync round of such an atlas (src/vk/vkbackend.c:4990-5060): slot s
 * holds brick slot_brick[s] (R3D_BRICK_ABSENT: free) and its atlas content
 * carries key keys[s] (0: zeros, else (brick + 1) << 32 | generation).
 * First the stale slots, whose key names another brick, are picked to be
 * zeroed (new key 0); only when there are none, the slots whose wanted key
 * (from src->gen of their brick; 0 when it returns 0) differs from theirs.
 * At most budget slots (0 or over 16: 16), in slot order.  Writes each
 * pick's slot, brick and new key; the caller fetches the bricks with a
 * nonzero key and zeroes the rest.  Returns the number picked. */
uint32_t r3d_host_atlas_pick(const uint32_t *page, const uint32_t *slot_brick, uint32_t nslots,
                             const uint64_t *keys, const r3d_brick_src *src, uint32_t budget,
                             uint32_t *sel_slot, uint32_t *sel_brick, uint64_t *sel_key);

/* Virtual slab: a W x H x D window anywhere in a volume, rendered from
 * world-anchored toroidal tile grids (src/core/vslab.h).  Level l has
 * spacing s = {1, 4, 8, 16, 32}[l] and cells of px * s voxels; cell (cx, cy)
 * lives in tile base + (cy mod gy) * gx + (cx mod gx), each tile
 * (px + 2)^2 texels (one-texel apron) by a ring of wz = D + 2 + 2 z_margin
 * slices, world slice z in layer z mod wz.  gx = 0 marks an absent level. */
#define R3D_VS_LEVELS 5u
typedef struct r3d_vslab_layout {
  uint64_t nx, ny, nz;      /* volume */
  uint32_t W, H, D;         /* visible window */
  uint32_t px, wz, z_margin;
  int64_t x0, y0, z0;       /* window origin; -1 before the first frame */
  uint32_t s[R3D_VS_LEVELS], gx[R3D_VS_LEVELS], gy[R3D_VS_LEVELS], base[R3D_VS_LEVELS];
  uint32_t ntiles;
} r3d_vslab_layout;
/* Layout of a window (vslab.h:55-105): payload px = max(W, H) / 8 rounded
 * up to 32 in [64, 2016], shrunk while one tile ring exceeds 3 GiB; per
 * level ceil(W / cell) (+2 where the axis can move) tiles per axis, pyramid
 * levels only while max(W, H) / s >= 1024.  -1 for a window that does not
 * fit (W or H < 64 or beyond the volume, D < 2 or > 2044, ring > 2046 or
 * deeper than the volume). */
int r3d_host_vslab_init(r3d_vslab_layout *v, uint64_t nx, uint64_t ny, uint64_t nz, uint32_t W,
                        uint32_t H, uint32_t D, uint32_t z_margin);
/* Resident z range [a, b) for a visible window at z0: the margin around it,
 * shifted inside the volume (vslab.h:113-125). */
void r3d_host_vslab_zrange(const r3d_vslab_layout *v, int64_t z0, int64_t *a, int64_t *b);
/* Cells [c0, c1] of level l covering [o, o + span) on an axis of n voxels,
 * clamped to the volume (vslab.h:129-139). */
void r3d_host_vslab_range(const r3d_vslab_layout *v, uint32_t l, int64_t o, uint64_t n,
                          uint32_t span, int64_t *c0, int64_t *c1);

/* Ledger entry of one base tile: the cell it holds (INT64_MIN: none) and
 * the slices [za, zb) of that cell its ring holds. */
typedef struct r3d_vslab_cell {
  int64_t cx, cy, za, zb;
} r3d_vslab_cell;
/* One fill: slices [zs0, zs0 + nz) of base cell (cx, cy), and the pyramid
 * texels derived from them. */
typedef struct r3d_vslab_job {
  int64_t cx, cy, zs0;
  uint32_t nz, prio;
} r3d_vslab_job;
/* One frame of the virtual slab (src/vk/vkbackend.c:6390-6620): the window
 * follows the focus (origin fx - W/2, fy - H/2 snapped down to 16 and kept
 * in the volume; z0 kept in [0, nz - D]), then the base cells under it are
 * listed with the slices they miss: the visible span [z0, z0 + D + 2) first
 * (priority 0, completing a partial span without rewriting what is held),
 * then the z margin in 16-slice steps, the direction of travel first;
 * sorted by priority, then squared cell distance from the window centre.
 * When the window moved in x or y, the cells one column / row beyond it in
 * the direction of motion follow (whole resident range), where the
 * straddle tile can host them.  At most budget jobs are written (and at
 * most cap); the layout's origin becomes the frame's.  Returns the number
 * of jobs. */
uint32_t r3d_host_vslab_plan(r3d_vslab_layout *v, const r3d_vslab_cell *cells, double fx,
                             double fy, int64_t z0, uint32_t budget, r3d_vslab_job *jobs,
                             uint32_t cap);
/* Records a finished job in the ledger (vkbackend.c:6408-6430): a new cell
 * takes the job's slices, a held one grows by them, and the range is
 * clamped to the resident range of the window at z0.  Returns the base
 * slot. */
uint32_t r3d_host_vslab_apply(const r3d_vslab_layout *v, r3d_vslab_cell *cells,
                              const r3d_vslab_job *j, int64_t z0);
/* Validity key of cell (cx, cy) (vslab.h:146-150). */
uint32_t r3d_host_vslab_key(int64_t cx, int64_t cy);

/* A view of the scripted "orbit" benchmark at phase ph in [0,1): yaw = 2 pi ph,
 * pitch = 0.5 sin(4 pi ph), distance 2 around target (src/main.c:3932-3946),
 * identity volume transform, viewport w x h.  Other fields: step_voxels,
 * density, lod_bias as given, max_mip 10, threshold / skip_gate from
 * low_cut and the LUT. */
void r3d_host_orbit_view(r3d_frame_params *p, float ph, const float target[3], uint32_t w,
                         uint32_t h, float step_voxels, float density, float lod_bias,
                         uint32_t mode, uint32_t frame_index, float low_cut,
                         const uint8_t lut[256][4]);

/* Seeded scroll phantom: papyrus sheets along an Archimedean spiral about
 * the z axis through the volume centre, r(theta) = r0 + pitch*theta/(2 pi).
 * A voxel is papyrus when its radial distance to the nearest wrap is below
 * sheet_half and r0 <= r < radius.  Papyrus ~ N(in_mean, in_sd), air
 * ~ N(air_mean, air_sd), plus N(0, noise_sd), rounded and clamped to u8.
 * Normals come from splitmix64 of (seed, voxel index) through Box-Muller,
 * so every voxel is independent of the thread count. */
typedef struct r3d_phantom_desc {
  uint64_t seed;
  float pitch, radius, r0, sheet_half;
  float in_mean, in_sd, air_mean, air_sd, noise_sd;
} r3d_phantom_desc;

/* The configuration used for a volume of edge n: pitch 14 and radius 110
 * at 256, pitch 18 and radius 110/256 of the edge above 256. */
void r3d_host_phantom_default(uint32_t n, uint64_t seed, r3d_phantom_desc *d);
int r3d_host_phantom(uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz,
                     const r3d_phantom_desc *d, int threads);

/* The same construction generated on the context's device into device
 * memory vox (nx*ny*nz); synchronizes.  CUDA's double-precision log / sin /
 * cos replace glibc's, so rare voxels on a rounding or sheet boundary may
 * differ from r3d_host_phantom's. */
struct r3d_cuda_ctx;
int r3d_cuda_phantom(struct r3d_cuda_ctx *ctx, const r3d_phantom_desc *d, uint32_t nx,
                     uint32_t ny, uint32_t nz, uint8_t *vox, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* R3D_HOST_H */
