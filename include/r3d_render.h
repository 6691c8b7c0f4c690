/* Headless subset of render3d's render-backend interface
 * (reference src/render/render.h), implemented on the sm_100a raycast
 * library.  Same names, argument meaning and return convention: 0 on
 * success, nonzero on failure with a message on stderr.  The renderer keeps
 * its offscreen RGBA8 image in device memory; r3d_read_frame copies it out.
 *
 * Implemented: r3d_create / r3d_destroy (headless only), r3d_upload_volume,
 * r3d_set_transfer, r3d_set_quality, r3d_frame, r3d_frame_views,
 * r3d_read_frame, r3d_bricks_params / _extent / _shape / _end.  The brick
 * cache is built from a raw volume (r3d_bricks_begin_volume) instead of
 * from a compressed c5d shard tree, whose codec is not part of this
 * library.  Everything else in render.h (slab, clipmap, streaming,
 * overlays, surface views, GUI) is not provided. */
#ifndef R3D_RENDER_H
#define R3D_RENDER_H

#include <stdbool.h>
#include <stdint.h>

#include "r3d_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct SDL_Window SDL_Window; /* only NULL is accepted */
typedef struct r3d_renderer r3d_renderer;

/* Same fields as the reference's r3d_config
 * (src/render/render_types.h:11-22); headless must be true. */
typedef struct r3d_config {
  bool validate;
  bool vsync;
  const char *spv_dir;
  uint64_t gpu_budget_bytes;
  bool headless;
  uint32_t headless_w, headless_h; /* offscreen image size */
} r3d_config;

int r3d_create(SDL_Window *win, const r3d_config *cfg, r3d_renderer **out);
void r3d_destroy(r3d_renderer *r);

int r3d_upload_volume(r3d_renderer *r, const r3d_volume_desc *d, const uint8_t *voxels);
int r3d_set_transfer(r3d_renderer *r, const uint8_t rgba[256][4]);
void r3d_set_quality(r3d_renderer *r, uint32_t quality);

/* Builds the LOD brick cache (nlev levels; bricks with maximum < min_max
 * are left non-resident) from a raw u8 volume on the device. */
int r3d_bricks_begin_volume(r3d_renderer *r, const r3d_volume_desc *d, const uint8_t *voxels,
                            uint32_t nlev, uint32_t min_max);
/* Single-level bricks (a shard of edge = bpa * 128, the non-LOD bricks mode
 * of r3d_bricks_begin, reference src/render/render.h:44-50): with
 * pool_bpa == 0 or >= bpa the whole shard is resident in the identity
 * layout, as in the reference when the volume fits the pool.  A smaller
 * pool needs the streaming residency pump, which is not built: -1. */
int r3d_bricks_begin_shard(r3d_renderer *r, const uint8_t *voxels, uint32_t edge,
                           uint32_t pool_bpa);
int r3d_bricks_end(r3d_renderer *r);
void r3d_bricks_params(const r3d_renderer *r, r3d_frame_params *p);
void r3d_bricks_extent(const r3d_renderer *r, float extent[3]);
void r3d_bricks_shape(const r3d_renderer *r, uint32_t shape[3]);

int r3d_frame(r3d_renderer *r, const r3d_frame_params *p, r3d_frame_stats *st);
/* nviews 1..R3D_MAX_VIEWS, each into its view_org rect of the offscreen. */
int r3d_frame_views(r3d_renderer *r, const r3d_frame_params *views, uint32_t nviews,
                    r3d_frame_stats *st);
/* rgba NULL: query the size only. */
int r3d_read_frame(r3d_renderer *r, uint8_t *rgba, uint32_t *w, uint32_t *h);

/* Termination opacity for compositing modes (default 0.98). */
int r3d_set_alpha_cutoff(r3d_renderer *r, float cutoff);
/* The underlying raycast context (for r3d_cuda_* calls). */
struct r3d_cuda_ctx *r3d_renderer_cuda(r3d_renderer *r);

#ifdef __cplusplus
}
#endif

#endif /* R3D_RENDER_H */
