// Batched raycast of many views of uneven size: a plan with a device-
// resident view table, launched as persistent queue-draining kernels (or one
// grid per view), capturable into a CUDA graph, and an autotuner over the
// launch schedules.
#include <string.h>

#include <vector>

#include "r3d_internal.h"

using namespace r3d;

struct r3d_cuda_batch {
  r3d_cuda_ctx *ctx = nullptr;
  uint32_t n = 0;
  std::vector<r3d_frame_params> pcs;  // sanitized views
  std::vector<uint8_t *> imgs;
  // the contexts whose scenes the requests sample, and each request's
  std::vector<uint32_t> scene_of;
  r3d_cuda_ctx *scenes[kMaxScenes] = {};
  uint32_t nscenes = 0;
  r3d_cuda_schedule sched = {1u, 16u, 0u, 1u, 0u, 0u, 0u};
  // lane refill (batches of one scene): per tile shape, device view tables
  // (views grouped by path and mode)
  DevView *dviews[3] = {nullptr, nullptr, nullptr};
  uint32_t *queue = nullptr;  // [0, 64): refill counters; [64, 192): whole-tile counters
  uint32_t ngroups = 0;
  uint32_t gkey[kMaxBatchViews], gstart[kMaxBatchViews + 1];
  uint32_t ntiles[3][kMaxBatchViews];
  // whole tiles: host view tables grouped by path, mode and quality across
  // scenes, numbered in 8x4 tiles
  std::vector<DevView> tviews;
  uint32_t tgroups = 0;
  uint32_t tkey[kMaxBatchViews], tstart[kMaxBatchViews + 1], tntiles[kMaxBatchViews];
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static int batch_fail(r3d_cuda_batch *b, int code, const char *msg) {
  return fail(b ? b->ctx : nullptr, code, "%s", msg);
}

extern "C" int r3d_cuda_batch_create_scenes(r3d_cuda_ctx *c, const r3d_cuda_scene_request *reqs,
                                            uint32_t n, r3d_cuda_batch **out) {
  if (!c || !reqs || !out || !n || n > kMaxBatchViews)
    return fail(c, R3D_E_INVALID, "batch_create: 1..%u requests", kMaxBatchViews);
  *out = nullptr;
  cudaSetDevice(c->device);
  r3d_cuda_batch *b = new (std::nothrow) r3d_cuda_batch();
  if (!b) return R3D_E_NOMEM;
  b->ctx = c;
  b->n = n;
  for (uint32_t i = 0; i < n; i++) {
    const r3d_frame_params &v = reqs[i].view;
    r3d_cuda_ctx *sc = reqs[i].scene ? reqs[i].scene : c;
    uint32_t k = 0;
    while (k < b->nscenes && b->scenes[k] != sc) k++;
    if (k == b->nscenes) {
      if (b->nscenes == kMaxScenes || sc->device != c->device) {
        delete b;
        return fail(c, R3D_E_INVALID, "batch_create: request %u: at most %u scenes, all on the "
                                      "batch's device", i, kMaxScenes);
      }
      b->scenes[b->nscenes++] = sc;
    }
    if (!reqs[i].rgba || !v.viewport[0] || !v.viewport[1] || v.view_org) {
      delete b;
      return fail(c, R3D_E_INVALID, "batch_create: request %u needs an image, a viewport and "
                                    "view_org 0", i);
    }
    if (!is_device_ptr(reqs[i].rgba)) {
      delete b;
      return fail(c, R3D_E_INVALID, "batch_create: request %u image is not device memory", i);
    }
    r3d_frame_params pc;
    int rc = prepare_view(sc, v, v.viewport[0], v.viewport[1], pc);
    if (rc < 0 && sc != c) rc = fail(c, rc, "batch_create: request %u: %s", i, sc->err.c_str());
    if (rc >= 0 && ((v.overlay_flags & kOvlAtlases) || (v.view_flags & R3D_VIEW_SURF)))
      rc = fail(c, R3D_E_UNSUPPORTED, "batch: request %u: overlay and surface views render "
                                      "through r3d_cuda_raycast_fwd", i);
    if (rc < 0) {
      delete b;
      return rc;
    }
    b->pcs.push_back(pc);
    b->imgs.push_back(reqs[i].rgba);
    b->scene_of.push_back(k);
  }
  // whole tiles: group by (path, mode, quality) across scenes, request order
  // inside a group, 8x4 tiles numbered per group
  {
    uint32_t gof[kMaxBatchViews], cnt[kMaxBatchViews];
    for (uint32_t i = 0; i < n; i++) {
      const uint32_t fast = b->scenes[b->scene_of[i]]->quality == R3D_QUALITY_FAST;
      const uint32_t key = ((uint32_t)path_of_view(b->pcs[i]) * 8u + b->pcs[i].mode) * 2u + fast;
      uint32_t g = 0;
      while (g < b->tgroups && b->tkey[g] != key) g++;
      if (g == b->tgroups) {
        b->tkey[b->tgroups] = key;
        cnt[b->tgroups++] = 0;
      }
      gof[i] = g;
      cnt[g]++;
    }
    b->tstart[0] = 0;
    for (uint32_t g = 0; g < b->tgroups; g++) b->tstart[g + 1] = b->tstart[g] + cnt[g];
    uint32_t fill[kMaxBatchViews] = {0};
    b->tviews.resize(n);
    for (uint32_t g = 0; g < b->tgroups; g++) b->tntiles[g] = 0;
    for (uint32_t i = 0; i < n; i++) {
      const uint32_t g = gof[i];
      DevView &d = b->tviews[b->tstart[g] + fill[g]++];
      memset(&d, 0, sizeof d);
      d.pc = b->pcs[i];
      d.img = (uchar4 *)b->imgs[i];
      d.stride = b->pcs[i].viewport[0];
      d.scene = b->scene_of[i];
      d.tile_begin = b->tntiles[g];
      b->tntiles[g] += view_tiles(d, 0u);
    }
  }
  cudaError_t e = cudaMalloc(&b->queue, sizeof(uint32_t) * 3 * kMaxBatchViews);
  if (e == cudaSuccess) e = cudaMemset(b->queue, 0, sizeof(uint32_t) * 3 * kMaxBatchViews);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();  // the counters are zero before any launch
  if (e == cudaSuccess && b->nscenes == 1u) {
    // lane refill: group by (path, mode), keep request order inside a group
    uint32_t order[kMaxBatchViews], gcount[kMaxBatchViews], group_of[kMaxBatchViews];
    for (uint32_t i = 0; i < n; i++) {
      uint32_t key = (uint32_t)path_of_view(b->pcs[i]) * 8u | b->pcs[i].mode, g = 0;
      while (g < b->ngroups && b->gkey[g] != key) g++;
      if (g == b->ngroups) {
        b->gkey[b->ngroups] = key;
        gcount[b->ngroups++] = 0;
      }
      group_of[i] = g;
      gcount[g]++;
    }
    b->gstart[0] = 0;
    for (uint32_t g = 0; g < b->ngroups; g++) b->gstart[g + 1] = b->gstart[g] + gcount[g];
    uint32_t fill[kMaxBatchViews] = {0};
    for (uint32_t i = 0; i < n; i++) order[b->gstart[group_of[i]] + fill[group_of[i]]++] = i;
    std::vector<DevView> hv(n);
    for (uint32_t shape = 0; shape < 3 && e == cudaSuccess; shape++) {
      e = cudaMalloc(&b->dviews[shape], sizeof(DevView) * n);
      if (e != cudaSuccess) break;
      for (uint32_t g = 0; g < b->ngroups; g++) {
        uint32_t tiles = 0;
        for (uint32_t j = b->gstart[g]; j < b->gstart[g + 1]; j++) {
          const uint32_t i = order[j];
          DevView &d = hv[j];
          memset(&d, 0, sizeof d);
          d.pc = b->pcs[i];
          d.img = (uchar4 *)b->imgs[i];
          d.stride = b->pcs[i].viewport[0];
          d.tile_begin = tiles;
          tiles += view_tiles(d, shape);
        }
        b->ntiles[shape][g] = tiles;
      }
      e = copy_sync(c->stream, b->dviews[shape], hv.data(), sizeof(DevView) * n);
    }
  }
  if (e != cudaSuccess) {
    r3d_cuda_batch_destroy(b);
    return cuda_fail(c, e, "batch_create");
  }
  if (b->nscenes > 1u) b->sched.persistent = 2u;  // lane refill drains one scene
  *out = b;
  return R3D_OK;
}

extern "C" int r3d_cuda_batch_create(r3d_cuda_ctx *c, const r3d_cuda_request *reqs, uint32_t n,
                                     r3d_cuda_batch **out) {
  if (!c || !reqs || !out || !n || n > kMaxBatchViews)
    return fail(c, R3D_E_INVALID, "batch_create: 1..%u requests", kMaxBatchViews);
  r3d_cuda_scene_request rs[kMaxBatchViews];
  for (uint32_t i = 0; i < n; i++) rs[i] = {reqs[i].view, reqs[i].rgba, nullptr};
  return r3d_cuda_batch_create_scenes(c, rs, n, out);
}

extern "C" void r3d_cuda_batch_destroy(r3d_cuda_batch *b) {
  if (!b) return;
  if (b->ctx) cudaSetDevice(b->ctx->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto &d : b->dviews) cudaFree(d);
  cudaFree(b->queue);
  delete b;
}

extern "C" int r3d_cuda_batch_set_schedule(r3d_cuda_batch *b, const r3d_cuda_schedule *sc) {
  if (b && sc && sc->persistent == 1u && b->nscenes > 1u)
    return batch_fail(b, R3D_E_UNSUPPORTED, "batch_set_schedule: lane refill needs a batch of "
                                            "one scene");
  if (!b || !sc || sc->persistent > 3u || sc->staging > 1u || sc->refill_min < 1u || sc->refill_min > 32u ||
      sc->tile_shape > 2u || (sc->unroll != 1u && sc->unroll != 2u) || sc->shade_group > 32u || sc->blocks_per_sm > 32u)
    return batch_fail(b, R3D_E_INVALID, "batch_set_schedule: bad schedule");
  b->sched = *sc;
  b->sched.persistent = resolved_persistent(*sc, b->n);  // a batch's view count is fixed
  return R3D_OK;
}

extern "C" int r3d_cuda_batch_get_schedule(const r3d_cuda_batch *b, r3d_cuda_schedule *sc) {
  if (!b || !sc) return R3D_E_INVALID;
  *sc = b->sched;
  return R3D_OK;
}

extern "C" int r3d_cuda_batch_launch(r3d_cuda_batch *b, unsigned long long *total_steps,
                                     void *stream) {
  if (!b) return R3D_E_INVALID;
  r3d_cuda_ctx *c = b->ctx;
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const r3d_cuda_schedule &sc = b->sched;
  if (!sc.persistent) {
    for (uint32_t i = 0; i < b->n; i++) {
      r3d_cuda_ctx *s = b->scenes[b->scene_of[i]];
      const r3d_cuda_schedule keep = s->sched;
      s->sched.shade_group = sc.shade_group;
      cudaError_t e = launch_view(s, b->pcs[i], b->imgs[i], b->pcs[i].viewport[0], nullptr,
                                  nullptr, total_steps, nullptr, st);
      s->sched = keep;
      if (e != cudaSuccess) return cuda_fail(c, e, "batch_launch: grid");
    }
    return R3D_OK;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  if (sc.persistent == 2u) {  // whole tiles: one launch per group, every scene
    DevScene scenes[kMaxScenes];
    const uchar4 *luts[kMaxScenes];
    for (uint32_t k = 0; k < b->nscenes; k++) {
      scenes[k] = b->scenes[k]->scene();
      luts[k] = b->scenes[k]->lut;
    }
    for (uint32_t g = 0; g < b->tgroups; g++) {
      TilesLaunch T;
      memset(&T, 0, sizeof T);
      T.views = b->tviews.data() + b->tstart[g];
      T.nviews = b->tstart[g + 1] - b->tstart[g];
      T.ntiles = b->tntiles[g];
      T.scenes = scenes;
      T.luts = luts;
      T.nscenes = b->nscenes;
      T.queue = b->queue + kMaxBatchViews + 2 * g;
      T.total = total_steps;
      T.blocks = sc.blocks_per_sm * (uint32_t)sms;
      T.fast = (b->tkey[g] & 1u) != 0u;
      T.mode = (b->tkey[g] >> 1) & 7u;
      T.path = (int)(b->tkey[g] >> 4);
      cudaError_t e = launch_tiles(T, st);
      if (e != cudaSuccess) return cuda_fail(c, e, "batch_launch: whole tiles");
    }
    return R3D_OK;
  }
  if (b->nscenes > 1u)
    return batch_fail(b, R3D_E_UNSUPPORTED, "batch_launch: lane refill needs one scene");
  R3D_CUDA_TRY(c, cudaMemsetAsync(b->queue, 0, sizeof(uint32_t) * b->ngroups, st));
  const DevScene s = c->scene();
  for (uint32_t g = 0; g < b->ngroups; g++) {
    PersistLaunch L;
    memset(&L, 0, sizeof L);
    const uint32_t shape = sc.tile_shape;
    L.views = b->dviews[shape] + b->gstart[g];
    L.nviews = b->gstart[g + 1] - b->gstart[g];
    L.ntiles = b->ntiles[shape][g];
    L.lut = c->lut;
    L.queue = b->queue + g;
    L.refill_min = sc.refill_min;
    L.shape = shape;
    L.unroll = sc.unroll;
    L.total = total_steps;
    L.mode = b->gkey[g] & 7u;
    L.fast = c->quality == R3D_QUALITY_FAST;
    L.path = (int)(b->gkey[g] >> 3);
    int per_sm = sc.blocks_per_sm
                     ? (int)sc.blocks_per_sm
                     : persist_blocks_per_sm(L.path, L.mode, L.fast, L.unroll);
    uint32_t want = (uint32_t)per_sm * (uint32_t)sms;
    uint32_t cap = (L.ntiles + 3u) / 4u;
    L.blocks = want < cap ? want : (cap ? cap : 1u);
    cudaError_t e = launch_persist(L, s, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "batch_launch: persistent");
  }
  return R3D_OK;
}

extern "C" int r3d_cuda_batch_capture(r3d_cuda_batch *b, unsigned long long *total_steps,
                                      void *stream) {
  if (!b) return R3D_E_INVALID;
  r3d_cuda_ctx *c = b->ctx;
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  R3D_CUDA_TRY(c, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int rc = r3d_cuda_batch_launch(b, total_steps, st);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(st, &g);
  if (rc != R3D_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "batch_capture: end capture");
  b->graph = g;
  R3D_CUDA_TRY(c, cudaGraphInstantiate(&b->exec, g, 0));
  R3D_CUDA_TRY(c, cudaGraphLaunch(b->exec, st));
  return R3D_OK;
}

extern "C" int r3d_cuda_batch_replay(r3d_cuda_batch *b, void *stream) {
  if (!b || !b->exec) return batch_fail(b, R3D_E_STATE, "batch_replay: nothing captured");
  r3d_cuda_ctx *c = b->ctx;
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  R3D_CUDA_TRY(c, cudaGraphLaunch(b->exec, st));
  return R3D_OK;
}

extern "C" int r3d_cuda_batch_autotune(r3d_cuda_batch *b, uint32_t reps, r3d_cuda_schedule *best,
                                       float *best_ms) {
  if (!b || !reps) return R3D_E_INVALID;
  r3d_cuda_ctx *c = b->ctx;
  cudaSetDevice(c->device);
  cudaStream_t st = c->stream;
  std::vector<r3d_cuda_schedule> cands;
  for (uint32_t shade : {0u, 4u, 8u, 16u}) cands.push_back({0u, 16u, 0u, 1u, 0u, shade, 0u});
  if (b->nscenes == 1u)  // lane refill drains one scene
    for (uint32_t shape = 0; shape < 3; shape++)
      for (uint32_t refill : {8u, 16u, 24u})
        for (uint32_t unroll : {1u, 2u}) cands.push_back({1u, refill, shape, unroll, 0u, 0u, 0u});
  cands.push_back({2u, 16u, 0u, 1u, 0u, 0u, 0u});  // whole 8x4 tiles from one queue
  const r3d_cuda_schedule keep = b->sched;
  float bms = 1e30f;
  r3d_cuda_schedule bsc = keep;
  cudaEvent_t e0, e1;
  R3D_CUDA_TRY(c, cudaEventCreate(&e0));
  R3D_CUDA_TRY(c, cudaEventCreate(&e1));
  int rc = R3D_OK;
  for (const r3d_cuda_schedule &sc : cands) {
    b->sched = sc;
    if ((rc = r3d_cuda_batch_launch(b, nullptr, st)) != R3D_OK) break;  // warm-up
    cudaEventRecord(e0, st);
    for (uint32_t r = 0; r < reps && rc == R3D_OK; r++) rc = r3d_cuda_batch_launch(b, nullptr, st);
    cudaEventRecord(e1, st);
    if (rc != R3D_OK) break;
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      rc = cuda_fail(c, e, "batch_autotune");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= (float)reps;
    if (ms < bms) {
      bms = ms;
      bsc = sc;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->sched = rc == R3D_OK ? bsc : keep;
  if (rc != R3D_OK) return rc;
  if (best) *best = bsc;
  if (best_ms) *best_ms = bms;
  return R3D_OK;
}
