/* Headless subset of render3d's render-backend interface
 * (reference src/render/render.h), implemented on the sm_100a raycast
 * library.  Same names, argument meaning and return convention: 0 on
 * success, nonzero on failure with a message on stderr.  The renderer keeps
 * its offscreen RGBA8 image in device memory; r3d_read_frame copies it out.
 *
 * Implemented with the reference's signatures: r3d_create / r3d_destroy
 * (headless only), r3d_upload_volume, r3d_set_transfer, r3d_set_quality,
 * r3d_frame, r3d_frame_views, r3d_read_frame, r3d_bricks_params / _extent /
 * _shape / _end, the tiled slab (r3d_slab_init / _window / _params),
 * r3d_clip_frame, r3d_bricks_stream / _get_stats / _flush, r3d_vslab_frame
 * / _get / _resident_pending, and the flattened-segment calls (r3d_surf_*,
 * r3d_surfvol_*, r3d_surfmask*, r3d_max_dim3d).  Where the reference reads
 * a compressed c5d tree, a shard band or a Zarr cache from disk, the data
 * arrives as a raw u8 volume instead (r3d_bricks_begin_volume,
 * r3d_bricks_begin_stream, r3d_clip_begin_volume, r3d_vslab_begin_volume,
 * r3d_bricks_overlay_volume): the c5d codec, the shard store and network
 * ingest are not part of this library.  The GUI calls are not provided. */
#ifndef R3D_RENDER_H
#define R3D_RENDER_H

#include <stdbool.h>
#include <stddef.h>
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

/* A raw volume held by the caller (reference src/core/volume.h:14-19). */
typedef struct r3d_volume {
  const uint8_t *voxels; /* nx * ny * nz bytes, x fastest */
  uint32_t nx, ny, nz;
  size_t nbytes;
  float voxel_um;
} r3d_volume;

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
 * pool is refused (-1): a volume larger than the pool streams as an LOD
 * cache (r3d_bricks_begin_stream). */
int r3d_bricks_begin_shard(r3d_renderer *r, const uint8_t *voxels, uint32_t edge,
                           uint32_t pool_bpa);
int r3d_bricks_end(r3d_renderer *r);
void r3d_bricks_params(const r3d_renderer *r, r3d_frame_params *p);
void r3d_bricks_extent(const r3d_renderer *r, float extent[3]);
void r3d_bricks_shape(const r3d_renderer *r, uint32_t shape[3]);

/* Tiled slab (render.h:22-33): init records the window, the first window
 * call builds the tiles from src (held on the device from then on; a
 * different src rebuilds them) and later calls scroll to start slice z0
 * (clamped to [0, nz - wz]).  _params fills the view's slab fields. */
typedef struct r3d_slab_desc {
  uint32_t nx, ny, nz; /* source dims */
  uint32_t wz;         /* ring depth (window slices) */
} r3d_slab_desc;
int r3d_slab_init(r3d_renderer *r, const r3d_slab_desc *d);
int r3d_slab_window(r3d_renderer *r, const r3d_volume *src, uint32_t z0);
void r3d_slab_params(const r3d_renderer *r, r3d_frame_params *p);

/* Clipmap (render.h:35-41) over a raw volume instead of a shard band and
 * its pyramid files; r3d_clip_frame recentres, refills and writes the view's
 * clip fields before r3d_frame, as in the reference. */
int r3d_clip_begin_volume(r3d_renderer *r, const r3d_volume *src, uint32_t depth_max);
int r3d_clip_frame(r3d_renderer *r, double fx, double fy, uint64_t z0, r3d_frame_params *p);

/* Streamed LOD brick cache (render.h:44-50,116-160): the whole pyramid of
 * a raw volume in pinned host memory, nslots device slots (the coarsest
 * level stays resident); r3d_bricks_stream runs one pump update before
 * r3d_frame with the reference's arguments. */
int r3d_bricks_begin_stream(r3d_renderer *r, const r3d_volume_desc *d, const uint8_t *voxels,
                            uint32_t nlev, uint32_t nslots);
void r3d_bricks_stream(r3d_renderer *r, const float eye[3], const float fwd[3], float half_tan,
                       float pixel_cone, uint32_t slice_z0, uint32_t slice_depth, float gate,
                       uint32_t budget);
/* Multi-view pump (render.h:128-139): begin (false: not streaming), any
 * number of box / point collects, then submit. */
bool r3d_bricks_stream_begin(r3d_renderer *r);
void r3d_bricks_stream_box(r3d_renderer *r, const float lo[3], const float hi[3],
                           float pixel_cone, float gate);
void r3d_bricks_stream_point(r3d_renderer *r, const float p[3], uint32_t level, float gate);
void r3d_bricks_stream_submit(r3d_renderer *r, uint32_t budget);
/* Same fields as the reference's r3d_bricks_stats; the warm-tier, decode
 * and network fields stay 0 (the warm tier holds decoded bricks). */
typedef struct r3d_bricks_stats {
  uint32_t nb, hot, hot_cap;
  uint32_t warm_bricks;
  uint64_t warm_bytes, warm_cap;
  uint32_t inflight;
  uint64_t decoded, jobs, stream_ns;
  uint32_t failures;
  uint32_t nlevels, lod_wanted[8];
  uint64_t lod_requests[8];
  uint32_t net_pending;
  uint64_t net_fetched, net_encoded;
} r3d_bricks_stats;
void r3d_bricks_get_stats(r3d_renderer *r, r3d_bricks_stats *st);
void r3d_bricks_flush(r3d_renderer *r);

/* Overlay atlas `which` (0 ink, 1 3D ink, 2 labels, 3 registration) of the
 * LOD cache from a raw volume of the cache's shape (render.h:51-101 read
 * c5d trees and label sources instead). */
/* CPU-sourced atlases (render.h:74-97): labels (overlay_flags bit 3) and
 * registration (bit 4).  gen() is polled per resident slot on each sync;
 * fetch() fills a 128^3 brick only when gen changed.  _regatlas_sync runs
 * its round within the call; _regatlas_detach drops the source before the
 * caller destroys it and keeps the atlas for a later re-attach. */
typedef struct r3d_label_src {
  uint32_t (*gen)(void *user, uint32_t level, uint32_t bx, uint32_t by, uint32_t bz);
  void (*fetch)(void *user, uint32_t level, uint32_t bx, uint32_t by, uint32_t bz,
                uint8_t *out);
  void *user;
} r3d_label_src;
int r3d_bricks_labels(r3d_renderer *r, const r3d_label_src *src);
void r3d_bricks_labels_sync(r3d_renderer *r, uint32_t budget);
int r3d_bricks_regatlas(r3d_renderer *r, const r3d_label_src *src);
void r3d_bricks_regatlas_sync(r3d_renderer *r, uint32_t budget);
void r3d_bricks_regatlas_detach(r3d_renderer *r);
/* Post-decode display filter (render.h:62-73): the mode, amount and target
 * bits of r3d_cuda_bricks_postfilter, for bricks built, streamed in or
 * loaded as overlays from now on; _refilter re-streams the resident bricks
 * of a streamed cache through it (a resident cache is filtered when built). */
void r3d_bricks_postfilter(r3d_renderer *r, uint32_t mode, float amount, uint32_t targets);
void r3d_bricks_refilter(r3d_renderer *r);
int r3d_bricks_overlay_volume(r3d_renderer *r, uint32_t which, const r3d_volume_desc *d,
                              const uint8_t *voxels);

/* Virtual slab (render.h:161-184) over a raw volume of the descriptor's
 * dims instead of a Zarr cache: cache_dir, shard_url and the decoded
 * prefetch fields are ignored.  r3d_vslab_frame fills the frame's cells
 * (at most budget) before it returns. */
typedef struct r3d_vslab_desc {
  uint32_t nx, ny, nz;
  uint32_t W, H, D;
  const char *cache_dir;
  const char *shard_url;
  uint32_t z_prefetch;
  uint32_t prefetch_slots;
  uint32_t prefetch_threads;
} r3d_vslab_desc;
int r3d_vslab_begin_volume(r3d_renderer *r, const r3d_vslab_desc *d, const uint8_t *voxels);
void r3d_vslab_frame(r3d_renderer *r, double fx, double fy, int64_t z0, uint32_t budget,
                     r3d_frame_params *p);
void r3d_vslab_get(const r3d_renderer *r, int64_t o[3], uint32_t *pending);
uint32_t r3d_vslab_resident_pending(const r3d_renderer *r);

/* Flattened-segment views (render.h:193-238).  _surfvol_window bakes only
 * when the window changed, and bakes the whole window; _surfvol_visible is
 * accepted and has no effect. */
int r3d_surf_begin(r3d_renderer *r, uint32_t w, uint32_t h, const float *coords_rgba,
                   const float *normals_rgba);
int r3d_surf_swap(r3d_renderer *r, uint32_t w, uint32_t h, const float *coords_rgba,
                  const float *normals_rgba, float sx, float sy);
int r3d_surfvol_begin(r3d_renderer *r, uint32_t w, uint32_t h, uint32_t layers,
                      uint32_t nback, float sx, float sy);
void r3d_surfvol_window(r3d_renderer *r, double u0, double v0, float step, float zoff0);
void r3d_surfvol_visible(r3d_renderer *r, uint32_t x0, uint32_t y0, uint32_t z0, uint32_t x1,
                         uint32_t y1, uint32_t z1);
void r3d_surfvol_mark(r3d_renderer *r);
/* Live 2.5D ink prediction: w x h probabilities, texel (0, 0) at grid
 * coordinates (g0u, g0v), px_per_grid texels per grid unit; re-bakes. */
int r3d_surfvol_inkpred(r3d_renderer *r, const float *pred, uint32_t w, uint32_t h, float g0u,
                        float g0v, float px_per_grid);
void r3d_surfvol_inkpred_clear(r3d_renderer *r);
/* The bake's overlay byte: none unless the ink atlas is loaded and
 * _overlay_enable is on; then the registration atlas while _regtap is on,
 * else the 3D ink atlas when loaded, else the ink atlas. */
void r3d_surfvol_overlay_enable(r3d_renderer *r, bool enable);
void r3d_surfvol_regtap(r3d_renderer *r, bool on);
void r3d_surfvol_params(const r3d_renderer *r, r3d_frame_params *p);
int r3d_surfmask(r3d_renderer *r, const uint8_t *m, uint32_t w, uint32_t h);
void r3d_surfmask_clear(r3d_renderer *r);
uint32_t r3d_max_dim3d(const r3d_renderer *r);

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
