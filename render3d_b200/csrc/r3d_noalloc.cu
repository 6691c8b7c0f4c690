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

#include "r3d_internal.h"

namespace {

// Per-call scratch of every call on every device: up to kNoallocViews view
// records followed by one tile counter per view.  Each GPU that loads the
// library holds these bytes until the process exits.
constexpr uint32_t kNoallocViews = r3d::kMaxBatchViews;  // 64
constexpr size_t kTableBytes = sizeof(r3d::DevView) * kNoallocViews;
constexpr size_t kScratchBytes = 32768;  // 32 KiB
static_assert(kTableBytes + kNoallocViews * sizeof(uint32_t) <= kScratchBytes,
              "scratch too small for the view table");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch for each device (the host-side symbol is not a
// device address).  Filled on the first call on a device.
constexpr int kMaxDevices = 64;
static void *g_scratch_dev[kMaxDevices];

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
  if (!g_scratch_dev[c->device]) {  // once per device, with that device current
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(c, e, "raycast_fwd_noalloc: scratch address");
    g_scratch_dev[c->device] = p;
  }
  DevView *table = (DevView *)g_scratch_dev[c->device];
  uint32_t *queue = (uint32_t *)((unsigned char *)g_scratch_dev[c->device] + kTableBytes);
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;

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
  DevView hv[kNoallocViews];
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
  gstart[0] = 0;
  for (uint32_t g = 0; g < ngroups; g++) gstart[g + 1] = gstart[g] + gcount[g];
  const uint32_t shape = 0u;  // 8x4 tiles
  uint32_t fill[kNoallocViews] = {0}, ntiles[kNoallocViews] = {0};
  for (uint32_t i = 0; i < n; i++) {
    uint32_t g = group_of[i], slot = gstart[g] + fill[g]++;
    DevView &d = hv[slot];
    memset(&d, 0, sizeof d);
    d.pc = pcs[order[i]];
    d.img = (uchar4 *)rgba_out;
    d.stride = out_w;
    d.tile_begin = ntiles[g];
    ntiles[g] += view_tiles(d, shape);
  }
  // from pageable host memory the copy is staged before the call returns,
  // so hv may go out of scope; the counters of this call start at zero
  R3D_CUDA_TRY(c, cudaMemcpyAsync(table, hv, sizeof(DevView) * n, cudaMemcpyHostToDevice, st));
  R3D_CUDA_TRY(c, cudaMemsetAsync(queue, 0, sizeof(uint32_t) * ngroups, st));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const DevScene s = c->scene();
  for (uint32_t g = 0; g < ngroups; g++) {
    PersistLaunch L;
    memset(&L, 0, sizeof L);
    L.views = table + gstart[g];
    L.nviews = gcount[g];
    L.ntiles = ntiles[g];
    L.lut = c->lut;
    L.queue = queue + g;
    L.refill_min = 16u;
    L.shape = shape;
    L.unroll = 1u;
    L.mode = gkey[g] & 7u;
    L.fast = c->quality == R3D_QUALITY_FAST;
    L.path = (int)(gkey[g] >> 3);
    uint32_t want =
        (uint32_t)persist_blocks_per_sm(L.path, L.mode, L.fast, 1u) * (uint32_t)sms;
    uint32_t cap = (L.ntiles + 3u) / 4u;
    L.blocks = want < cap ? want : (cap ? cap : 1u);
    cudaError_t e = launch_persist(L, s, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "raycast_fwd_noalloc: launch");
  }
  return R3D_OK;
}
