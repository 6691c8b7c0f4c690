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
   * rows of band k, [band_row[k], band_row[k + 1]) */
  cudaStream_t band_stream[BANDS - 1], copy_stream;
  cudaEvent_t band_ev[BANDS];
  uint32_t nbands; /* bands of the last frame; 0: drawn whole */
  uint32_t band_row[BANDS + 1];
};

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
  return report(r, "upload_volume", r3d_cuda_upload_volume(r->ctx, d, voxels));
}

int r3d_set_transfer(r3d_renderer *r, const uint8_t rgba[256][4]) {
  if (!r) return -1;
  return report(r, "set_transfer", r3d_cuda_set_transfer(r->ctx, rgba));
}

void r3d_set_quality(r3d_renderer *r, uint32_t quality) {
  if (r) report(r, "set_quality", r3d_cuda_set_quality(r->ctx, quality));
}

int r3d_set_alpha_cutoff(r3d_renderer *r, float cutoff) {
  if (!r) return -1;
  return report(r, "set_alpha_cutoff", r3d_cuda_set_alpha_cutoff(r->ctx, cutoff));
}

struct r3d_cuda_ctx *r3d_renderer_cuda(r3d_renderer *r) { return r ? r->ctx : NULL; }

int r3d_bricks_begin_volume(r3d_renderer *r, const r3d_volume_desc *d, const uint8_t *voxels,
                            uint32_t nlev, uint32_t min_max) {
  if (!r) return -1;
  int rc = r3d_cuda_bricks_build(r->ctx, d, voxels, nlev, min_max);
  if (rc != R3D_OK) return report(r, "bricks_begin_volume", rc);
  r->bricks = 1;
  r->brick_mode = r3d_cuda_brick_mode(r->ctx);
  r3d_cuda_bricks_info(r->ctx, NULL, NULL, r->shape, NULL);
  return 0;
}

int r3d_bricks_begin_shard(r3d_renderer *r, const uint8_t *voxels, uint32_t edge,
                           uint32_t pool_bpa) {
  if (!r) return -1;
  if (pool_bpa && pool_bpa < edge / 128u) {
    fprintf(stderr, "r3d: bricks_begin_shard: a pool smaller than the shard needs streaming "
                    "residency, which is not available\n");
    return -1;
  }
  int rc = r3d_cuda_shard_build(r->ctx, edge, voxels, edge / 128u, NULL);
  if (rc != R3D_OK) return report(r, "bricks_begin_shard", rc);
  r->bricks = 1;
  r->brick_mode = r3d_cuda_shard_mode(r->ctx);
  r->shape[0] = r->shape[1] = r->shape[2] = edge;
  return 0;
}

int r3d_bricks_end(r3d_renderer *r) {
  if (!r) return -1;
  r->bricks = 0;
  r->brick_mode = 0;
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
  if (whole) {
    /* row bands (multiples of 8 dispatch rows), band k > 0 on band stream
     * k - 1, which starts after this frame's begin event; the context's
     * stream then waits for every band */
    const int half = (v->view_flags & R3D_VIEW_HALF) != 0u;
    const uint32_t gh = half ? (r->h + 1u) / 2u : r->h;
    const uint32_t rb = ((gh + BANDS - 1u) / BANDS + 7u) / 8u * 8u;
    uint32_t k = 0;
    for (uint32_t r0 = 0; r0 < gh && k < BANDS; r0 += rb, k++) {
      const uint32_t r1 = r0 + rb < gh ? r0 + rb : gh;
      cudaStream_t s = k ? r->band_stream[k - 1] : stream;
      if (k && cudaStreamWaitEvent(s, r->ev_begin[slot], 0) != cudaSuccess) return -1;
      int rc = r3d_cuda_raycast_rows(r->ctx, v, r->offscreen, r->w, r->h, r0, r1, s);
      if (rc != R3D_OK) return report(r, "frame", rc);
      if (cudaEventRecord(r->band_ev[k], s) != cudaSuccess) return -1;
      r->band_row[k] = half ? 2u * r0 : r0;
      r->band_row[k + 1] = half ? (2u * r1 < r->h ? 2u * r1 : r->h) : r1;
    }
    for (uint32_t j = 1; j < k; j++)
      if (cudaStreamWaitEvent(stream, r->band_ev[j], 0) != cudaSuccess) return -1;
    r->nbands = k;
  } else {
    int rc = r3d_cuda_raycast_fwd(r->ctx, views, nviews, r->offscreen, r->w, r->h, NULL, stream);
    if (rc != R3D_OK) return report(r, "frame", rc);
  }
  if (cudaEventRecord(r->ev_end[slot], stream) != cudaSuccess) return -1;
  r->ev_used[slot] = 1;
  if (st) {
    st->cpu_record_ns = now_ns() - t0;
    st->panes_drawn = nviews;
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
      const size_t off = r->band_row[k] * row, n = (r->band_row[k + 1] - r->band_row[k]) * row;
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
