// Forward raycast that allocates no device memory per call.
//
// Some callers cannot let a library call cudaMalloc while they render: host
// applications that hand the renderer a fixed device-memory budget at start-
// up and forbid allocation afterwards, and real-time render threads for
// which an allocation (which can synchronize the device) is a frame hitch.
// For them this entry point runs the persistent queue-draining kernel with
// its per-call scratch -- the table of views and the tile counters -- in a
// fixed array of device memory that is part of the library itself, instead
// of buffers owned by the context.  The caller passes the views and a
// device output image; the scene (volume or brick cache, TF) is the one
// already loaded into the context.
#include <string.h>

#include <algorithm>
#include <atomic>

#include "r3d_internal.h"

namespace {

// Per-call scratch of every call on every device: up to kNoallocViews view
// records followed by two tile counters per view.  Each GPU that loads the
// library holds these bytes until the process exits.
constexpr uint32_t kNoallocViews = r3d::kMaxBatchViews;  // 64
constexpr size_t kTableBytes = sizeof(r3d::DevView) * kNoallocViews;
constexpr size_t kScratchBytes = 32768;  // 32 KiB
static_assert(kTableBytes + 2 * kNoallocViews * sizeof(uint32_t) <= kScratchBytes,
              "scratch too small for the view table");
static_assert(sizeof(r3d::DevView) % 4u == 0u, "view records are copied as words");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch for each device (the host-side symbol is not a
// device address).  Looked up by the first call on a device, with that
// device current; concurrent first calls store the same value.  A
// cudaDeviceReset reloads the module, so this cache (and the entry point)
// must not be used across one.
constexpr int kMaxDevices = 64;
static std::atomic<void *> g_scratch_dev[kMaxDevices];

// The view records of one call, passed by value as the table writer's launch
// parameters (at most 8 views, 2.3 KiB, per launch): the kernel reads no
// host buffer after the call returns.
constexpr uint32_t kChunkViews = 8;
struct TableChunk {
  r3d::DevView v[kChunkViews];
};

// Writes n (<= 8) view records at dst and, when nq > 0, zeroes the first nq
// tile counters of the call.
__global__ void k_noalloc_table(r3d::DevView *__restrict__ dst, uint32_t n,
                                uint32_t *__restrict__ queue, uint32_t nq,
                                const __grid_constant__ TableChunk t) {
  const uint32_t *src = reinterpret_cast<const uint32_t *>(t.v);
  uint32_t *d = reinterpret_cast<uint32_t *>(dst);
  const uint32_t words = n * (uint32_t)(sizeof(r3d::DevView) / 4u);
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) d[i] = src[i];
  for (uint32_t i = threadIdx.x; i < nq; i += blockDim.x) queue[i] = 0u;
}

}  // namespace

using namespace r3d;

extern "C" int r3d_cuda_raycast_fwd_noalloc(r3d_cuda_ctx *c, const r3d_frame_params *views,
                                            uint32_t nviews, uint8_t *rgba_out, uint32_t out_w,
                                            uint32_t out_h, void *stream) {
  if (!c || !views || !nviews || !rgba_out || !out_w || !out_h || out_w > 65535u ||
      out_h > 65535u)
    return fail(c, R3D_E_INVALID, "raycast_fwd_noalloc: bad arguments");
  if (nviews > kNoallocViews)
    return fail(c, R3D_E_INVALID,
                "raycast_fwd_noalloc: %u views, at most %u fit the %zu-byte scratch", nviews,
                kNoallocViews, kScratchBytes);
  if (c->device < 0 || c->device >= kMaxDevices)
    return fail(c, R3D_E_INVALID, "raycast_fwd_noalloc: device %d", c->device);
  R3D_CUDA_TRY(c, cudaSetDevice(c->device));
  if (!is_device_ptr(rgba_out))
    return fail(c, R3D_E_INVALID, "raycast_fwd_noalloc: the image must be device memory");
  void *base = g_scratch_dev[c->device].load(std::memory_order_acquire);
  if (!base) {  // once per device, with that device current
    cudaError_t e = cudaGetSymbolAddress(&base, g_scratch);
    if (e != cudaSuccess || !base) return cuda_fail(c, e, "raycast_fwd_noalloc: scratch address");
    g_scratch_dev[c->device].store(base, std::memory_order_release);
  }
  DevView *table = (DevView *)base;
  uint32_t *queue = (uint32_t *)((unsigned char *)base + kTableBytes);
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const r3d_cuda_schedule &sc = c->sched;

  r3d_frame_params pcs[kNoallocViews];
  int render[kNoallocViews];
  for (uint32_t v = 0; v < nviews; v++) {
    render[v] = prepare_view(c, views[v], out_w, out_h, pcs[v]);
    if (render[v] < 0) return render[v];
    if ((views[v].overlay_flags & kOvlAtlases) || (views[v].view_flags & R3D_VIEW_SURF))
      return fail(c, R3D_E_UNSUPPORTED,
                  "raycast_fwd_noalloc: overlay and surface views are not supported");
  }
  // views sharing a sampling path and mode form one launch
  TableChunk chunk[kNoallocViews / kChunkViews];
  DevView *hv = &chunk[0].v[0];
  uint32_t order[kNoallocViews], group_of[kNoallocViews], gkey[kNoallocViews];
  uint32_t gcount[kNoallocViews], gstart[kNoallocViews + 1], ngroups = 0, n = 0;
  for (uint32_t v = 0; v < nviews; v++) {
    if (!render[v]) continue;
    uint32_t key = (uint32_t)path_of_view(pcs[v]) * 8u | pcs[v].mode, g = 0;
    while (g < ngroups && gkey[g] != key) g++;
    if (g == ngroups) {
      gkey[ngroups] = key;
      gcount[ngroups++] = 0;
    }
    group_of[n] = g;
    order[n++] = v;
    gcount[g]++;
  }
  if (!n) return R3D_OK;
  const uint32_t persistent = resolved_persistent(sc, n);
  gstart[0] = 0;
  for (uint32_t g = 0; g < ngroups; g++) gstart[g + 1] = gstart[g] + gcount[g];
  uint32_t fill[kNoallocViews] = {0}, ntiles[kNoallocViews] = {0};
  for (uint32_t i = 0; i < n; i++) {
    uint32_t g = group_of[i], slot = gstart[g] + fill[g]++;
    DevView &d = hv[slot];
    memset(&d, 0, sizeof d);
    d.pc = pcs[order[i]];
    d.img = (uchar4 *)rgba_out;
    d.stride = out_w;
    d.tile_begin = ntiles[g];
    ntiles[g] += view_tiles(d, persistent == 2u ? 0u : sc.tile_shape);
  }
  // the table and this call's zeroed counters, written on the stream ahead
  // of the raycast launches (a call queued behind an earlier one on the
  // same stream overwrites the scratch only once that one has finished)
  for (uint32_t k = 0; k * kChunkViews < n; k++) {
    const uint32_t m = std::min(kChunkViews, n - k * kChunkViews);
    k_noalloc_table<<<1, 128, 0, st>>>(table + k * kChunkViews, m, queue, k ? 0u : 2u * ngroups,
                                       chunk[k]);
    R3D_CUDA_TRY(c, cudaGetLastError());
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const DevScene s = c->scene();
  for (uint32_t g = 0; g < ngroups; g++) {
    cudaError_t e;
    if (persistent == 2u) {  // whole tiles: the views travel as launch parameters
      TilesLaunch T;
      memset(&T, 0, sizeof T);
      T.views = hv + gstart[g];
      T.nviews = gcount[g];
      T.ntiles = ntiles[g];
      T.scenes = &s;
      T.luts = &c->lut;
      T.nscenes = 1u;
      T.queue = queue + 2 * g;
      T.blocks = sc.blocks_per_sm * (uint32_t)sms;
      T.mode = gkey[g] & 7u;
      T.fast = c->quality == R3D_QUALITY_FAST;
      T.path = (int)(gkey[g] >> 3);
      e = launch_tiles(T, st);
      if (e != cudaSuccess) return cuda_fail(c, e, "raycast_fwd_noalloc: launch");
      continue;
    }
    PersistLaunch L;
    memset(&L, 0, sizeof L);
    L.views = table + gstart[g];
    L.nviews = gcount[g];
    L.ntiles = ntiles[g];
    L.lut = c->lut;
    L.queue = queue + 2 * g;
    L.refill_min = sc.refill_min;
    L.shape = sc.tile_shape;
    L.unroll = sc.unroll;
    L.mode = gkey[g] & 7u;
    L.fast = c->quality == R3D_QUALITY_FAST;
    L.path = (int)(gkey[g] >> 3);
    const int per_sm = sc.blocks_per_sm
                           ? (int)sc.blocks_per_sm
                           : persist_blocks_per_sm(L.path, L.mode, L.fast, L.unroll);
    uint32_t want = (uint32_t)per_sm * (uint32_t)sms;
    uint32_t cap = (L.ntiles + 3u) / 4u;
    L.blocks = want < cap ? want : (cap ? cap : 1u);
    e = launch_persist(L, s, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "raycast_fwd_noalloc: launch");
  }
  return R3D_OK;
}
