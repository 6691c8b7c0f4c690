/* Plain-data types shared by the renderer's host code and the sm_100a raycast
 * library.  `r3d_frame_params` is the per-view parameter block render3d's
 * host code fills every frame; its byte layout is the reference's
 * (src/render/render_types.h:47-94, mirrored by FrameParams in
 * src/shaders/common.slang:5-42) so that existing callers drop in unchanged.
 * The static_assert below and the offset test in the test suite pin it. */
#ifndef R3D_TYPES_H
#define R3D_TYPES_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Render modes (reference src/render/render_types.h:25-33). */
enum {
  R3D_MODE_FULL = 0,    /* front-to-back compositing with gradient shading */
  R3D_MODE_MIP = 1,     /* maximum-intensity projection */
  R3D_MODE_DEPTH = 2,   /* first-hit depth */
  R3D_MODE_HEATMAP = 3, /* per-ray step count */
  R3D_MODE_RAYDIR = 4,  /* ray direction as colour (wiring check) */
  R3D_MODE_FLAT = 5,    /* compositing without shading */
  R3D_MODE_COUNT = 6,
};

/* Gradient quality (reference src/render/render_types.h:35-39). */
enum {
  R3D_QUALITY_FULL = 0, /* six-tap central differences */
  R3D_QUALITY_FAST = 1, /* four-tap tetrahedral differences */
  R3D_QUALITY_COUNT = 2,
};

typedef struct r3d_volume_desc {
  uint32_t nx, ny, nz;
  uint32_t brick_dim; /* always 128 */
  float voxel_um;
} r3d_volume_desc;

/* One view.  Field order, types and padding are fixed by the reference
 * (248 bytes; every float[3] is followed by a scalar so the block matches a
 * std140 float3+float pair). */
typedef struct r3d_frame_params {
  float cam_origin[3];
  float step_voxels; /* march step in voxels */
  float cam_right[3]; /* camera right, pre-scaled by tan(fov/2) * aspect */
  float density;      /* opacity scale (MIP: brightness scale) */
  float cam_up[3];    /* camera up, pre-scaled by tan(fov/2) */
  float lod_bias;
  float cam_forward[3];
  float max_mip; /* cube path: highest mip level the march may use */
  uint32_t viewport[2];
  uint32_t mode;
  uint32_t frame_index; /* jitter seed */
  float threshold;      /* low-cut: samples below it are void */
  /* window fields of the tiled slab (slab_grid: gx | gy << 8 | ovs << 16),
   * the virtual slab (slab_grid: gx | gy << 6 | 1 << 24; brick_mode packs
   * its pyramid grids), the clipmap and flattened-segment views (slab_grid:
   * layers behind the surface); r3d_cuda_*_params fill them */
  uint32_t slab_grid;
  uint32_t slab_wz;
  float slab_z0; /* bricks: slab near face / crop-box z origin, voxels */
  float slab_nx, slab_ny;
  float slab_px, slab_py; /* bricks: crop-box x/y extents, voxels */
  uint32_t slab_depth;    /* bricks: slab thickness in voxels (0 = off) */
  /* clipmap: valid level mask (non-zero selects the clipmap) and origins */
  uint32_t clip_valid;
  float clip_orig[6][2];
  /* model transform: p_volume = R^T (p_world - t - c) + c, c = extent / 2;
   * vol_rN holds row N of R */
  float vol_r0[3];
  float vol_tx;
  float vol_r1[3];
  float vol_ty;
  float vol_r2[3];
  float vol_tz;
  /* 0 = cube; LOD bricks: abpa | nlev << 8 | 0x20000;
   * flat bricks: bpa | abpa << 8 | (identity ? 0x10000 : 0) */
  uint32_t brick_mode;
  float skip_gate; /* samples below it are invisible under the current TF */
  float slab_x0, slab_y0; /* bricks: crop-box origin x/y, voxels */
  uint32_t view_org;      /* output pixel origin, x | y << 16 */
  uint32_t view_flags;    /* R3D_VIEW_* bits */
  float overlay_gain;     /* overlay tint strength */
  uint32_t overlay_flags;
} r3d_frame_params;

#ifdef __cplusplus
static_assert(sizeof(r3d_frame_params) == 248, "r3d_frame_params is 248 bytes");
#else
_Static_assert(sizeof(r3d_frame_params) == 248, "r3d_frame_params is 248 bytes");
#endif

/* view_flags bits (reference src/render/render_types.h:96-105). */
#define R3D_VIEW_ORTHO 1u    /* parallel rays; cam_right/up = half extents */
#define R3D_VIEW_SURF 2u     /* flattened-segment view (r3d_cuda_surfvol_*) */
#define R3D_VIEW_OBLIQUE 4u  /* bricks slab clipped along the ray */
#define R3D_VIEW_STRETCH 8u  /* surf view: flattening-distortion heatmap */
#define R3D_VIEW_CROP 16u    /* bricks: clip to the crop box */
#define R3D_VIEW_HALF 32u    /* one ray per 2x2 pixel block */
#define R3D_VIEW_AXIS(a) ((uint32_t)(a) << 8) /* bricks slab axis 0=z 1=x 2=y */
#define R3D_MAX_VIEWS 4u

/* brick_mode encodings (reference src/vk/vkbackend.c:4511-4517). */
#define R3D_BRICK_LOD_FLAG 0x20000u
#define R3D_BRICK_IDENTITY_FLAG 0x10000u
#define R3D_BRICK_PAGE_HEADER 64u
#define R3D_BRICK_ABSENT 0xFFFFFFFFu
#define R3D_BRICK_EDGE 128u

/* Per-frame timing, reference src/render/render_types.h:107-119; the GPU
 * zones come from CUDA events recorded around the raycast launches. */
typedef struct r3d_frame_stats {
  uint64_t gpu_ns;
  uint64_t gpu_raycast_ns;
  uint64_t gpu_blit_ns; /* always 0: there is no present blit */
  uint64_t gpu_gui_ns;  /* always 0: no GUI pass */
  uint32_t panes_drawn;
  uint64_t cpu_wait_ns;
  uint64_t cpu_acquire_ns;
  uint64_t cpu_record_ns;
  uint64_t cpu_submit_ns;
} r3d_frame_stats;

#ifdef __cplusplus
}
#endif

#endif /* R3D_TYPES_H */
