/* Headless render3d render-backend interface (r3d_render.h) on the sm_100a
 * raycast library.  Mirrors the reference's Vulkan backend entry points
 * (src/vk/vkbackend.c: r3d_create :985, r3d_upload_volume :1508,
 * r3d_set_transfer :2069, r3d_frame_views :6801, r3d_read_frame :7337):
 * the offscreen RGBA8 image lives in device memory, each view is one
 * raycast launch into its rect, frames are paced two in flight, and the GPU
 * raycast time of a frame is reported two frames later, as the reference's
 * timestamp queries are.  A frame of one view covering the whole image is
 * drawn as row bands, each on its own stream so that they run
 * concurrently (a band waiting for the previous one would pay its slowest
 * block); r3d_read_frame then copies each band to the host as soon as it is
 * done, so the copy of a frame overlaps its rendering. */
#include "r3d_render.h"

#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "r3d_cuda.h"

#define FRAMES_IN_FLIGHT 2
#define BANDS 3

struct r3d_renderer {
  r3d_cuda_ctx *ctx;
  uint32_t w, h;
  uint8_t *offscreen; /* device, w*h*4 */
  int bricks;
  uint32_t brick_mode;
  uint32_t shape[3];
  uint32_t slot;
  cudaEvent_t ev_begin[FRAMES_IN_FLIGHT], ev_end[FRAMES_IN_FLIGHT];
  int ev_used[FRAMES_IN_FLIGHT];
  /* banded frames: the render streams of bands 1.. (band 0 runs on the
   * context's stream), the copy stream, one event per band and the image
   * image rows of band k, [band_row[k], band_end[k]) */
  cudaStream_t band_stream[BANDS - 1], copy_stream;
  cudaEvent_t band_ev[BANDS];
  uint32_t nbands; /* bands of the last frame; 0: drawn whole */
  uint32_t band_row[BANDS], band_end[BANDS];
  /* section modes and flattened views driven through this interface */
  r3d_slab_desc slab;        /* from r3d_slab_init (wz 0: none) */
  const uint8_t *slab_src;   /* the volume the tiles were built from */
  int streaming;
  r3d_stream_stats stream_last;
  uint64_t stream_uploaded;
  uint32_t surf_w, surf_h, surf_l, surf_nback; /* surfvol window */
  int surf_baked;
  float surf_win[4]; /* u0, v0, step, zoff0 of the last bake */
  /* overlay atlases loaded (bit k: atlas k) and the flattened bake's pick */
  uint32_t ovl_loaded;
  int sv_use_overlay, sv_regtap, sv_pick;
  /* pane cache (vkbackend.c:7066-7159): the layout hash of the last
   * multi-view frame, each pane's input hash when it was last drawn, and
   * the scene generation, bumped by every call that changes what a view
   * samples; R3D_NO_PANE_CACHE=1 turns the cache off */
  uint64_t layout_key, pane_key[R3D_MAX_VIEWS], scene_gen;
  int pane_cache_off;
};

/* FNV-1a step over a 64-bit word, as the reference's pane hashes fold it */
static uint64_t fnv(uint64_t k, uint64_t v) { return (k ^ v) * 1099511628211ull; }

/* The scene (volume, caches, TF, quality, cutoff, sections, atlases) changed:
 * cached panes must be drawn again. */
static void touched(r3d_renderer *r) {
  if (r) r->scene_gen++;
}

static uint64_t now_ns(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (uint64_t)ts.tv_sec * 1000000000ull + (uint64_t)ts.tv_nsec;
}

static int report(r3d_renderer *r, const char *what, int rc) {
  if (rc != 0)
    fprintf(stderr, "r3d: %s failed (%d): %s\n", what, rc,
            r && r->ctx ? r3d_cuda_last_error(r->ctx) : "");
  return rc;
}

/* The atlas the flattened bake writes into G (vkbackend.c:1815-1822,7033):
 * none unless the ink atlas is loaded and r3d_surfvol_overlay_enable is
 * on; then the registration atlas while its tap is on, else the 3D ink
 * atlas when loaded, else the ink atlas.  Re-bakes when the pick changes. */
static void surf_pick(r3d_renderer *r) {
  if (!r->surf_w) return;
  int which = -1;
  if ((r->ovl_loaded & 1u) && r->sv_use_overlay)
    which = r->sv_regtap && (r->ovl_loaded & 8u) ? 3 : (r->ovl_loaded & 2u) ? 1 : 0;
  if (which == r->sv_pick) return;
  if (report(r, "surfvol_overlay", r3d_cuda_surfvol_overlay(r->ctx, which)) == 0) r->sv_pick = which;
}

int r3d_create(SDL_Window *win, const r3d_config *cfg, r3d_renderer **out) {
  if (!out) return -1;
  *out = NULL;
  if (win || !cfg || !cfg->headless || !cfg->headless_w || !cfg->headless_h ||
      cfg->headless_w > 65535u || cfg->headless_h > 65535u) {
    fprintf(stderr, "r3d: only headless renderers with a nonzero size are supported\n");
    return -1;
  }
  r3d_renderer *r = calloc(1, sizeof *r);
  if (!r) return -1;
  r->w = cfg->headless_w;
  r->h = cfg->headless_h;
  const char *pc = getenv("R3D_NO_PANE_CACHE");
  r->pane_cache_off = pc && *pc == '1';
  int dev = 0;
  cudaGetDevice(&dev);
  if (r3d_cuda_create(dev, &r->ctx) != R3D_OK) {
    fprintf(stderr, "r3d: no CUDA device\n");
    free(r);
    return -1;
  }
  if (cudaMalloc((void **)&r->offscreen, (size_t)r->w * r->h * 4) != cudaSuccess ||
      cudaMemset(r->offscreen, 0, (size_t)r->w * r->h * 4) != cudaSuccess) {
    fprintf(stderr, "r3d: offscreen allocation failed\n");
    r3d_destroy(r);
    return -1;
  }
  for (int i = 0; i < FRAMES_IN_FLIGHT; i++)
    if (cudaEventCreate(&r->ev_begin[i]) != cudaSuccess ||
        cudaEventCreate(&r->ev_end[i]) != cudaSuccess) {
      r3d_destroy(r);
      return -1;
    }
  if (cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    r3d_destroy(r);
    return -1;
  }
  for (int i = 0; i < BANDS - 1; i++)
    if (cudaStreamCreateWithFlags(&r->band_stream[i], cudaStreamNonBlocking) != cudaSuccess) {
      r3d_destroy(r);
      return -1;
    }
  for (int i = 0; i < BANDS; i++)
    if (cudaEventCreateWithFlags(&r->band_ev[i], cudaEventDisableTiming) != cudaSuccess) {
      r3d_destroy(r);
      return -1;
    }
  *out = r;
  return 0;
}

void r3d_destroy(r3d_renderer *r) {
  if (!r) return;
  if (r->ctx) cudaStreamSynchronize((cudaStream_t)r3d_cuda_stream(r->ctx));
  for (int i = 0; i < BANDS - 1; i++)
    if (r->band_stream[i]) cudaStreamSynchronize(r->band_stream[i]);
  if (r->copy_stream) cudaStreamSynchronize(r->copy_stream);
  for (int i = 0; i < FRAMES_IN_FLIGHT; i++) {
    if (r->ev_begin[i]) cudaEventDestroy(r->ev_begin[i]);
    if (r->ev_end[i]) cudaEventDestroy(r->ev_end[i]);
  }
  for (int i = 0; i < BANDS; i++)
    if (r->band_ev[i]) cudaEventDestroy(r->band_ev[i]);
  for (int i = 0; i < BANDS - 1; i++)
    if (r->band_stream[i]) cudaStreamDestroy(r->band_stream[i]);
  if (r->copy_stream) cudaStreamDestroy(r->copy_stream);
  cudaFree(r->offscreen);
  r3d_cuda_destroy(r->ctx);
  free(r);
}

int r3d_upload_volume(r3d_renderer *r, const r3d_volume_desc *d, const uint8_t *voxels) {
  if (!r) return -1;
  touched(r);
  return report(r, "upload_volume", r3d_cuda_upload_volume(r->ctx, d, voxels));
}

int r3d_set_transfer(r3d_renderer *r, const uint8_t rgba[256][4]) {
  if (!r) return -1;
  touched(r);
  return report(r, "set_transfer", r3d_cuda_set_transfer(r->ctx, rgba));
}

void r3d_set_quality(r3d_renderer *r, uint32_t quality) {
  touched(r);
  if (r) report(r, "set_quality", r3d_cuda_set_quality(r->ctx, quality));
}

int r3d_set_alpha_cutoff(r3d_renderer *r, float cutoff) {
  if (!r) return -1;
  touched(r);
  return report(r, "set_alpha_cutoff", r3d_cuda_set_alpha_cutoff(r->ctx, cutoff));
}

struct r3d_cuda_ctx *r3d_renderer_cuda(r3d_renderer *r) { return r ? r->ctx : NULL; }

int r3d_bricks_begin_volume(r3d_renderer *r, const r3d_volume_desc *d, const uint8_t *voxels,
                            uint32_t nlev, uint32_t min_max) {
  if (!r) return -1;
  touched(r);
  int rc = r3d_cuda_bricks_build(r->ctx, d, voxels, nlev, min_max);
  if (rc != R3D_OK) return report(r, "bricks_begin_volume", rc);
  r->bricks = 1;
  r->ovl_loaded = 0;
  r->brick_mode = r3d_cuda_brick_mode(r->ctx);
  r3d_cuda_bricks_info(r->ctx, NULL, NULL, r->shape, NULL);
  return 0;
}

int r3d_bricks_begin_shard(r3d_renderer *r, const uint8_t *voxels, uint32_t edge,
                           uint32_t pool_bpa) {
  if (!r) return -1;
  touched(r);
  if (pool_bpa && pool_bpa < edge / 128u) {
    fprintf(stderr, "r3d: bricks_begin_shard: a single-level shard is resident whole; a pool "
                    "smaller than the volume streams as an LOD cache (r3d_bricks_begin_stream)\n");
    return -1;
  }
  int rc = r3d_cuda_shard_build(r->ctx, edge, voxels, edge / 128u, NULL);
  if (rc != R3D_OK) return report(r, "bricks_begin_shard", rc);
  r->bricks = 1;
  r->ovl_loaded = 0;
  r->brick_mode = r3d_cuda_shard_mode(r->ctx);
  r->shape[0] = r->shape[1] = r->shape[2] = edge;
  return 0;
}

int r3d_bricks_end(r3d_renderer *r) {
  if (!r) return -1;
  touched(r);
  r->bricks = 0;
  r->brick_mode = 0;
  r->ovl_loaded = 0;
  return 0;
}

void r3d_bricks_params(const r3d_renderer *r, r3d_frame_params *p) {
  if (r && p) p->brick_mode = r->bricks ? r->brick_mode : 0u;
}

/* volume box in renderer units: shape / max(shape) (src/shaders/raycast.slang:305-309) */
void r3d_bricks_extent(const r3d_renderer *r, float extent[3]) {
  if (!r || !extent) return;
  if (!r->bricks) {
    extent[0] = extent[1] = extent[2] = 1.0f;
    return;
  }
  uint32_t md = r->shape[0];
  if (r->shape[1] > md) md = r->shape[1];
  if (r->shape[2] > md) md = r->shape[2];
  for (int a = 0; a < 3; a++) extent[a] = (float)r->shape[a] / (float)md;
}

void r3d_bricks_shape(const r3d_renderer *r, uint32_t shape[3]) {
  if (!r || !shape) return;
  memcpy(shape, r->shape, sizeof r->shape);
}

int r3d_frame(r3d_renderer *r, const r3d_frame_params *p, r3d_frame_stats *st) {
  return r3d_frame_views(r, p, 1, st);
}

int r3d_frame_views(r3d_renderer *r, const r3d_frame_params *views, uint32_t nviews,
                    r3d_frame_stats *st) {
  if (!r || !views || !nviews || nviews > R3D_MAX_VIEWS) return -1;
  if (st) memset(st, 0, sizeof *st);
  cudaStream_t stream = (cudaStream_t)r3d_cuda_stream(r->ctx);
  uint32_t slot = r->slot;
  uint64_t t0 = now_ns();
  /* pacing: wait for this slot's previous frame, then read its GPU time */
  if (r->ev_used[slot]) {
    if (cudaEventSynchronize(r->ev_end[slot]) != cudaSuccess) return -1;
    float ms = 0.0f;
    if (st && cudaEventElapsedTime(&ms, r->ev_begin[slot], r->ev_end[slot]) == cudaSuccess) {
      st->gpu_ns = (uint64_t)((double)ms * 1e6);
      st->gpu_raycast_ns = st->gpu_ns;
    }
  }
  if (st) st->cpu_wait_ns = now_ns() - t0;
  t0 = now_ns();
  if (cudaEventRecord(r->ev_begin[slot], stream) != cudaSuccess) return -1;
  const r3d_frame_params *v = views;
  const int whole = nviews == 1u && !(v->view_flags & R3D_VIEW_SURF) && v->view_org == 0u &&
                    (v->viewport[0] == 0u || v->viewport[0] == r->w) &&
                    (v->viewport[1] == 0u || v->viewport[1] == r->h) && r->h >= 256u;
  r->nbands = 0;
  uint32_t drawn = 0;
  if (whole) {
    /* row bands (multiples of 8 dispatch rows), band k > 0 on band stream
     * k - 1, which starts after this frame's begin event; the context's
     * stream then waits for every band */
    const int half = (v->view_flags & R3D_VIEW_HALF) != 0u;
    const uint32_t gh = half ? (r->h + 1u) / 2u : r->h;
    const uint32_t rb = ((gh + BANDS - 1u) / BANDS + 7u) / 8u * 8u;
    /* the band holding the middle row is drawn first, then the others in
     * row order: the kernels take a band's rows by their distance from the
     * view's middle row, so the frame's long rays start first and its last
     * band (and last copy) holds short ones */
    uint32_t lo[BANDS], hi[BANDS], order[BANDS], nb = 0, mid = 0, n = 0;
    for (uint32_t r0 = 0; r0 < gh && nb < BANDS; r0 += rb, nb++) {
      lo[nb] = r0;
      hi[nb] = r0 + rb < gh ? r0 + rb : gh;
      if (lo[nb] <= gh / 2u && gh / 2u < hi[nb]) mid = nb;
    }
    order[n++] = mid;
    for (uint32_t b = 0; b < nb; b++)
      if (b != mid) order[n++] = b;
    uint32_t k = 0;
    for (; k < nb; k++) {
      const uint32_t r0 = lo[order[k]], r1 = hi[order[k]];
      cudaStream_t s = k ? r->band_stream[k - 1] : stream;
      if (k && cudaStreamWaitEvent(s, r->ev_begin[slot], 0) != cudaSuccess) return -1;
      int rc = r3d_cuda_raycast_rows(r->ctx, v, r->offscreen, r->w, r->h, r0, r1, s);
      if (rc != R3D_OK) return report(r, "frame", rc);
      if (cudaEventRecord(r->band_ev[k], s) != cudaSuccess) return -1;
      r->band_row[k] = half ? 2u * r0 : r0;
      r->band_end[k] = half ? (2u * r1 < r->h ? 2u * r1 : r->h) : r1;
    }
    for (uint32_t j = 1; j < k; j++)
      if (cudaStreamWaitEvent(stream, r->band_ev[j], 0) != cudaSuccess) return -1;
    r->nbands = k;
    drawn = nviews;
  } else if (nviews == 1u && v->view_org == 0u) {
    /* one view at the origin draws every pixel of its region each frame
     * (the reference's region-upscale path: no clear, no pane cache) */
    int rc = r3d_cuda_raycast_fwd(r->ctx, views, nviews, r->offscreen, r->w, r->h, NULL, stream);
    if (rc != R3D_OK) return report(r, "frame", rc);
    drawn = 1;
  } else {
    /* pane cache (vkbackend.c:7066-7159): a frame of several views, or of
     * one view away from the origin, keeps the offscreen between frames;
     * the regions no view covers are cleared only when the layout changes,
     * and a view is drawn only when its parameters (all but the jitter
     * seed frame_index) or the scene changed since it was drawn; with
     * R3D_NO_PANE_CACHE=1 every view is drawn and the offscreen cleared
     * each frame */
    const int cache = !r->pane_cache_off;
    uint64_t lay = 1469598103934665603ull ^ nviews;
    for (uint32_t k = 0; k < nviews; k++) {
      lay = fnv(lay, views[k].view_org);
      lay = fnv(lay, views[k].viewport[0]);
      lay = fnv(lay, views[k].viewport[1]);
    }
    lay = fnv(fnv(lay, r->w), r->h);
    if (lay != r->layout_key || !cache) {
      static const uint8_t clear[4] = {13, 13, 15, 255}; /* (0.05, 0.05, 0.06, 1) */
      int rc = r3d_cuda_fill_rgba(r->ctx, r->offscreen, (size_t)r->w * r->h, clear, stream);
      if (rc != R3D_OK) return report(r, "frame", rc);
      r->layout_key = lay;
      memset(r->pane_key, 0, sizeof r->pane_key);
    }
    r3d_frame_params todo[R3D_MAX_VIEWS];
    for (uint32_t k = 0; k < nviews; k++) {
      if (cache) {
        r3d_frame_params hp = views[k];
        hp.frame_index = 0;
        const uint8_t *hb = (const uint8_t *)&hp;
        uint64_t key = 1469598103934665603ull;
        for (size_t i = 0; i < sizeof hp; i++) key = fnv(key, hb[i]);
        key = fnv(key, r->scene_gen);
        if (key == 0) key = 1;
        if (r->pane_key[k] == key) continue; /* unchanged: keep its pixels */
        r->pane_key[k] = key;
      }
      todo[drawn++] = views[k];
    }
    if (drawn) {
      int rc = r3d_cuda_raycast_fwd(r->ctx, todo, drawn, r->offscreen, r->w, r->h, NULL, stream);
      if (rc != R3D_OK) {
        memset(r->pane_key, 0, sizeof r->pane_key); /* nothing drawn is cached */
        return report(r, "frame", rc);
      }
    }
  }
  if (cudaEventRecord(r->ev_end[slot], stream) != cudaSuccess) return -1;
  r->ev_used[slot] = 1;
  if (st) {
    st->cpu_record_ns = now_ns() - t0;
    st->panes_drawn = drawn;
  }
  r->slot = (slot + 1u) % FRAMES_IN_FLIGHT;
  return 0;
}

int r3d_read_frame(r3d_renderer *r, uint8_t *rgba, uint32_t *w, uint32_t *h) {
  if (!r || !w || !h) return -1;
  *w = r->w;
  *h = r->h;
  if (!rgba) return 0;
  cudaStream_t stream = (cudaStream_t)r3d_cuda_stream(r->ctx);
  if (r->nbands) {
    /* each band as soon as it is drawn, on the copy stream */
    const size_t row = (size_t)r->w * 4u;
    for (uint32_t k = 0; k < r->nbands; k++) {
      const size_t off = r->band_row[k] * row, n = (r->band_end[k] - r->band_row[k]) * row;
      if (cudaStreamWaitEvent(r->copy_stream, r->band_ev[k], 0) != cudaSuccess ||
          (n && cudaMemcpyAsync(rgba + off, r->offscreen + off, n, cudaMemcpyDeviceToHost,
                                r->copy_stream) != cudaSuccess)) {
        fprintf(stderr, "r3d: read_frame copy failed\n");
        return -1;
      }
    }
    if (cudaStreamSynchronize(r->copy_stream) != cudaSuccess) {
      fprintf(stderr, "r3d: read_frame copy failed\n");
      return -1;
    }
    return 0;
  }
  if (cudaMemcpyAsync(rgba, r->offscreen, (size_t)r->w * r->h * 4, cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    fprintf(stderr, "r3d: read_frame copy failed\n");
    return -1;
  }
  return 0;
}

/* ---- tiled slab (render.h:22-33) ---- */

int r3d_slab_init(r3d_renderer *r, const r3d_slab_desc *d) {
  touched(r);
  if (!r || !d || !d->nx || !d->ny || !d->nz || d->wz < 4u || d->wz > d->nz) return -1;
  r->slab = *d;
  r->slab_src = NULL;
  return 0;
}

int r3d_slab_window(r3d_renderer *r, const r3d_volume *src, uint32_t z0) {
  touched(r);
  if (!r || !r->slab.wz || !src || !src->voxels || src->nx != r->slab.nx ||
      src->ny != r->slab.ny || src->nz != r->slab.nz)
    return -1;
  const uint32_t zmax = r->slab.nz - r->slab.wz;
  if (z0 > zmax) z0 = zmax;
  if (src->voxels != r->slab_src) {
    r3d_volume_desc d = {src->nx, src->ny, src->nz, 128u, 1.0f};
    int rc = r3d_cuda_slab_build(r->ctx, &d, src->voxels, r->slab.wz, z0);
    if (rc != R3D_OK) return report(r, "slab_window", rc);
    r->slab_src = src->voxels;
    return 0;
  }
  return report(r, "slab_window", r3d_cuda_slab_window(r->ctx, z0));
}

void r3d_slab_params(const r3d_renderer *r, r3d_frame_params *p) {
  if (r && p) r3d_cuda_slab_params(r->ctx, p);
}

/* ---- clipmap (render.h:35-41) ---- */

int r3d_clip_begin_volume(r3d_renderer *r, const r3d_volume *src, uint32_t depth_max) {
  touched(r);
  if (!r || !src || !src->voxels) return -1;
  r3d_volume_desc d = {src->nx, src->ny, src->nz, 128u, 1.0f};
  return report(r, "clip_begin", r3d_cuda_clip_build(r->ctx, &d, src->voxels, depth_max));
}

int r3d_clip_frame(r3d_renderer *r, double fx, double fy, uint64_t z0, r3d_frame_params *p) {
  touched(r);
  if (!r) return -1;
  return report(r, "clip_frame", r3d_cuda_clip_frame(r->ctx, fx, fy, z0, p));
}

/* ---- streamed LOD cache (render.h:116-160) ---- */

int r3d_bricks_begin_stream(r3d_renderer *r, const r3d_volume_desc *d, const uint8_t *voxels,
                            uint32_t nlev, uint32_t nslots) {
  touched(r);
  if (!r) return -1;
  int rc = r3d_cuda_stream_begin(r->ctx, d, voxels, nlev, nslots);
  if (rc != R3D_OK) return report(r, "bricks_begin_stream", rc);
  r->bricks = 1;
  r->ovl_loaded = 0;
  r->streaming = 1;
  r->stream_uploaded = 0;
  memset(&r->stream_last, 0, sizeof r->stream_last);
  r->brick_mode = r3d_cuda_brick_mode(r->ctx);
  r3d_cuda_bricks_info(r->ctx, NULL, NULL, r->shape, NULL);
  return 0;
}

void r3d_bricks_stream(r3d_renderer *r, const float eye[3], const float fwd[3], float half_tan,
                       float pixel_cone, uint32_t slice_z0, uint32_t slice_depth, float gate,
                       uint32_t budget) {
  if (!r || !r->streaming || !eye || !fwd) return;
  r3d_stream_view v;
  memcpy(v.eye, eye, sizeof v.eye);
  memcpy(v.fwd, fwd, sizeof v.fwd);
  v.half_tan = half_tan;
  v.pixel_cone = pixel_cone;
  v.slice_z0 = slice_z0;
  v.slice_depth = slice_depth;
  v.gate = gate;
  v.budget = budget;
  r3d_stream_stats st;
  if (report(r, "bricks_stream", r3d_cuda_stream_update(r->ctx, &v, &st)) == 0) {
    r->stream_last = st;
    r->stream_uploaded += st.uploaded;
    if (st.uploaded) touched(r); /* views sample the new bricks */
  }
}

/* The multi-view pump: the reference's begin returns false while a decode
 * batch is in flight; uploads here finish within _submit, so a frame can
 * always be opened while streaming. */
bool r3d_bricks_stream_begin(r3d_renderer *r) {
  if (!r || !r->streaming) return false;
  return report(r, "bricks_stream_begin", r3d_cuda_stream_collect_begin(r->ctx)) == 0;
}

void r3d_bricks_stream_box(r3d_renderer *r, const float lo[3], const float hi[3],
                           float pixel_cone, float gate) {
  if (r && r->streaming)
    report(r, "bricks_stream_box", r3d_cuda_stream_collect_box(r->ctx, lo, hi, pixel_cone, gate));
}

void r3d_bricks_stream_point(r3d_renderer *r, const float p[3], uint32_t level, float gate) {
  if (r && r->streaming)
    report(r, "bricks_stream_point", r3d_cuda_stream_collect_point(r->ctx, p, level, gate));
}

void r3d_bricks_stream_submit(r3d_renderer *r, uint32_t budget) {
  if (!r || !r->streaming) return;
  r3d_stream_stats st;
  if (report(r, "bricks_stream_submit", r3d_cuda_stream_submit(r->ctx, budget, &st)) == 0) {
    r->stream_last = st;
    r->stream_uploaded += st.uploaded;
    if (st.uploaded) touched(r); /* views sample the new bricks */
  }
}

void r3d_bricks_get_stats(r3d_renderer *r, r3d_bricks_stats *st) {
  if (!r || !st) return;
  memset(st, 0, sizeof *st);
  if (!r->bricks) return;
  uint32_t nslots = 0, nlev = 0, shape[3] = {0, 0, 0};
  r3d_cuda_bricks_info(r->ctx, NULL, &nslots, shape, &nlev);
  st->nlevels = nlev;
  st->hot_cap = nslots;
  st->hot = r->streaming ? r->stream_last.resident : nslots;
  st->inflight = r->streaming ? r->stream_last.uploaded : 0u;
  st->decoded = r->stream_uploaded;
  uint32_t nb = 0;
  for (uint32_t l = 0; l < nlev && l < 16u; l++) {
    uint32_t s = 128u << l, b = 1u;
    for (int a = 0; a < 3; a++) b *= (shape[a] + s - 1u) / s;
    nb += b;
  }
  st->nb = nb;
}

void r3d_bricks_flush(r3d_renderer *r) {
  if (r) cudaStreamSynchronize((cudaStream_t)r3d_cuda_stream(r->ctx));
}

/* ---- CPU-sourced atlases: labels (2), registration (3) ---- */

static int atlas_attach(r3d_renderer *r, uint32_t which, const r3d_label_src *src,
                        const char *what) {
  if (!r || !r->bricks || !src || !src->gen || !src->fetch) return -1;
  const r3d_brick_src s = {src->gen, src->fetch, src->user};
  int rc = report(r, what, r3d_cuda_bricks_atlas_attach(r->ctx, which, &s));
  if (rc == 0) r->ovl_loaded |= 1u << which;
  return rc;
}

int r3d_bricks_labels(r3d_renderer *r, const r3d_label_src *src) {
  touched(r);
  return atlas_attach(r, 2u, src, "bricks_labels");
}

void r3d_bricks_labels_sync(r3d_renderer *r, uint32_t budget) {
  touched(r);
  if (r) report(r, "bricks_labels_sync", r3d_cuda_bricks_atlas_sync(r->ctx, 2u, budget, NULL));
}

int r3d_bricks_regatlas(r3d_renderer *r, const r3d_label_src *src) {
  touched(r);
  return atlas_attach(r, 3u, src, "bricks_regatlas");
}

/* the reference syncs the registration atlas on a worker thread and this
 * call only observes it; here the round runs within the call (the
 * reference's own fallback when the worker is missing) */
void r3d_bricks_regatlas_sync(r3d_renderer *r, uint32_t budget) {
  touched(r);
  if (!r) return;
  uint32_t n = 0;
  if (report(r, "bricks_regatlas_sync", r3d_cuda_bricks_atlas_sync(r->ctx, 3u, budget, &n)) == 0 &&
      n && r->sv_pick == 3)
    r3d_surfvol_mark(r); /* the flattened bake taps this atlas */
}

void r3d_bricks_regatlas_detach(r3d_renderer *r) {
  touched(r);
  if (r) r3d_cuda_bricks_atlas_detach(r->ctx, 3u);
}

void r3d_bricks_postfilter(r3d_renderer *r, uint32_t mode, float amount, uint32_t targets) {
  touched(r);
  if (r) report(r, "bricks_postfilter", r3d_cuda_bricks_postfilter(r->ctx, mode, amount, targets));
}

void r3d_bricks_refilter(r3d_renderer *r) {
  touched(r);
  /* a no-op without a streamed LOD cache, as the reference's without one */
  if (r && r->streaming) report(r, "bricks_refilter", r3d_cuda_bricks_refilter(r->ctx));
}

int r3d_bricks_overlay_volume(r3d_renderer *r, uint32_t which, const r3d_volume_desc *d,
                              const uint8_t *voxels) {
  touched(r);
  if (!r) return -1;
  int rc = r3d_cuda_bricks_overlay_build(r->ctx, which, d, voxels);
  if (rc != R3D_OK) return report(r, "bricks_overlay", rc);
  r->ovl_loaded |= 1u << which;
  surf_pick(r);
  return 0;
}

/* ---- virtual slab (render.h:161-184) ---- */

int r3d_vslab_begin_volume(r3d_renderer *r, const r3d_vslab_desc *d, const uint8_t *voxels) {
  touched(r);
  if (!r || !d || !voxels) return -1;
  r3d_volume_desc vd = {d->nx, d->ny, d->nz, 128u, 1.0f};
  return report(r, "vslab_begin",
                r3d_cuda_vslab_begin(r->ctx, &vd, voxels, d->W, d->H, d->D, d->z_prefetch));
}

void r3d_vslab_frame(r3d_renderer *r, double fx, double fy, int64_t z0, uint32_t budget,
                     r3d_frame_params *p) {
  touched(r);
  if (r) report(r, "vslab_frame", r3d_cuda_vslab_frame(r->ctx, fx, fy, z0, budget, p, NULL));
}

/* origin and the window cells still missing their visible slices */
static uint32_t vslab_pending(const r3d_renderer *r, int64_t o[3]) {
  r3d_vslab_layout v;
  if (r3d_cuda_vslab_layout(r->ctx, &v) != R3D_OK) return 0;
  if (o) o[0] = v.x0, o[1] = v.y0, o[2] = v.z0;
  r3d_vslab_stats st;
  /* a zero-budget frame at the current origin moves nothing and fills
   * nothing; it only reports */
  if (v.x0 < 0 ||
      r3d_cuda_vslab_frame(r->ctx, (double)v.x0 + v.W / 2, (double)v.y0 + v.H / 2, v.z0, 0u, NULL,
                           &st) != R3D_OK)
    return 0;
  return st.pending;
}

void r3d_vslab_get(const r3d_renderer *r, int64_t o[3], uint32_t *pending) {
  if (!r) return;
  const uint32_t n = vslab_pending(r, o);
  if (pending) *pending = n;
}

uint32_t r3d_vslab_resident_pending(const r3d_renderer *r) {
  return r ? vslab_pending(r, NULL) : 0u;
}

/* ---- flattened-segment views (render.h:193-238) ---- */

int r3d_surf_begin(r3d_renderer *r, uint32_t w, uint32_t h, const float *coords_rgba,
                   const float *normals_rgba) {
  touched(r);
  if (!r) return -1;
  return report(r, "surf_begin", r3d_cuda_surf_begin(r->ctx, w, h, coords_rgba, normals_rgba));
}

int r3d_surf_swap(r3d_renderer *r, uint32_t w, uint32_t h, const float *coords_rgba,
                  const float *normals_rgba, float sx, float sy) {
  touched(r);
  if (!r || !r->surf_w) return -1;
  /* new grids, the window re-made with the new scale: the next _window
   * call bakes everything, as in the reference */
  int rc = r3d_cuda_surf_begin(r->ctx, w, h, coords_rgba, normals_rgba);
  if (rc == R3D_OK)
    rc = r3d_cuda_surfvol_begin(r->ctx, r->surf_w, r->surf_h, r->surf_l, r->surf_nback, sx, sy);
  r->surf_baked = 0;
  return report(r, "surf_swap", rc);
}

int r3d_surfvol_begin(r3d_renderer *r, uint32_t w, uint32_t h, uint32_t layers,
                      uint32_t nback, float sx, float sy) {
  touched(r);
  if (!r) return -1;
  int rc = r3d_cuda_surfvol_begin(r->ctx, w, h, layers, nback, sx, sy);
  if (rc != R3D_OK) return report(r, "surfvol_begin", rc);
  r->surf_w = w, r->surf_h = h, r->surf_l = layers, r->surf_nback = nback;
  r->surf_baked = 0;
  r->sv_pick = -2; /* the context's pick is unknown: set it again */
  surf_pick(r);
  return 0;
}

void r3d_surfvol_window(r3d_renderer *r, double u0, double v0, float step, float zoff0) {
  if (!r || !r->surf_w) return;
  const float w[4] = {(float)u0, (float)v0, step, zoff0};
  if (r->surf_baked && !memcmp(w, r->surf_win, sizeof w)) return; /* unchanged */
  touched(r); /* the flattened view samples fresh texels */
  if (report(r, "surfvol_window", r3d_cuda_surfvol_window(r->ctx, u0, v0, step, zoff0)) == 0) {
    memcpy(r->surf_win, w, sizeof w);
    r->surf_baked = 1;
  }
}

void r3d_surfvol_visible(r3d_renderer *r, uint32_t x0, uint32_t y0, uint32_t z0, uint32_t x1,
                         uint32_t y1, uint32_t z1) {
  (void)r, (void)x0, (void)y0, (void)z0, (void)x1, (void)y1, (void)z1;
}

void r3d_surfvol_mark(r3d_renderer *r) {
  touched(r);
  if (r) report(r, "surfvol_mark", r3d_cuda_surfvol_mark(r->ctx));
}

void r3d_surfvol_overlay_enable(r3d_renderer *r, bool enable) {
  touched(r);
  if (!r) return;
  r->sv_use_overlay = enable;
  surf_pick(r);
}

void r3d_surfvol_regtap(r3d_renderer *r, bool on) {
  touched(r);
  /* vkbackend.c:5154-5169: a no-op without a surface volume, or to turn
   * the tap on without a registration atlas */
  if (!r || !r->surf_w || (on && !(r->ovl_loaded & 8u))) return;
  r->sv_regtap = on;
  surf_pick(r);
}

int r3d_surfvol_inkpred(r3d_renderer *r, const float *pred, uint32_t w, uint32_t h, float g0u,
                        float g0v, float px_per_grid) {
  touched(r);
  if (!r || !r->surf_w || !pred || !w || !h) return -1;
  return report(r, "surfvol_inkpred",
                r3d_cuda_surfvol_inkpred(r->ctx, pred, w, h, g0u, g0v, px_per_grid));
}

void r3d_surfvol_inkpred_clear(r3d_renderer *r) {
  touched(r);
  if (r && r->surf_w)
    report(r, "surfvol_inkpred_clear", r3d_cuda_surfvol_inkpred(r->ctx, NULL, 0, 0, 0, 0, 0));
}

void r3d_surfvol_params(const r3d_renderer *r, r3d_frame_params *p) {
  if (r && p) r3d_cuda_surfvol_params(r->ctx, p);
}

int r3d_surfmask(r3d_renderer *r, const uint8_t *m, uint32_t w, uint32_t h) {
  touched(r);
  if (!r || !m || !w || !h) return -1;
  return report(r, "surfmask", r3d_cuda_surfmask(r->ctx, m, w, h));
}

void r3d_surfmask_clear(r3d_renderer *r) {
  touched(r);
  if (r) report(r, "surfmask_clear", r3d_cuda_surfmask(r->ctx, NULL, 0, 0));
}

/* the largest surf window side to request: r3d_cuda_surfvol_begin takes up
 * to 2048 layers (and 16384 texels a side) */
uint32_t r3d_max_dim3d(const r3d_renderer *r) { return r ? 2048u : 0u; }
