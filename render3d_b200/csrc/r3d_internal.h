// Internal state of a raycast context (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "r3d_cuda.h"
#include "r3d_march.cuh"
#include "r3d_persist.h"

struct r3d_cuda_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;

  // cube volume: all mip levels in one allocation, then the occupancy grid
  uint8_t *cube_buf = nullptr;
  size_t cube_bytes = 0;
  bool have_cube = false;
  r3d::DevCube cube{};

  // LOD brick cache
  uint32_t *page = nullptr;
  uint8_t *pool = nullptr;
  uint8_t *bmax = nullptr;  // per-slot dilated 8^3 block maxima (4096 B/slot)
  uint32_t *quad = nullptr;  // per-slot quad words (DevBricks::quad)
  uint32_t *ovl_quad[4] = {nullptr, nullptr, nullptr, nullptr};  // overlay atlases
  // CPU-sourced atlases: the attached source, each slot's content key and
  // the staging slots (pinned host and device) of one sync round
  r3d_brick_src ovl_src[4] = {};
  bool ovl_src_on[4] = {false, false, false, false};
  std::vector<uint64_t> ovl_key[4];
  uint8_t *ovl_stage = nullptr, *ovl_stage_dev = nullptr;
  uint32_t page_words = 0;
  uint32_t nslots = 0;
  uint32_t abpa = 0;
  uint32_t shape[3] = {0, 0, 0};
  bool have_bricks = false;
  r3d::DevBricks br{};

  // streaming LOD cache: every brick of the pyramid in pinned host memory
  // (store, indexed by its slot in the full build; store_page is that
  // build's page table), a pool of nslots device slots, the host shadow of
  // the device page table and the LRU state
  bool streaming = false;
  bool defer_tables = false;  // a brick build whose pool is about to be replaced
  uint8_t *store = nullptr;
  std::vector<uint32_t> store_page, slot_brick, slot_use, brick_slot;
  uint32_t *page_shadow = nullptr;
  uint32_t *stream_jobs = nullptr;  // device: slots filled by one update
  uint32_t stream_frame = 0;
  cudaEvent_t page_ev = nullptr;
  // the request set of an open collect (one frame's views), and the
  // bricks it lists (page_words bytes)
  bool stream_open = false;
  // post-decode display filter (mode word, sharpen amount, target bits:
  // 0 CT, 1 ink atlas, 2 3D ink atlas) and its scratch slots
  uint32_t pf_mode = 0, pf_targets = 1;
  float pf_amount = 0.0f;
  uint8_t *pf_scratch = nullptr;
  std::vector<r3d_stream_cand> stream_cand;
  std::vector<uint8_t> stream_mark;

  // tiled slab: tiles of every level in one buffer, the source volume and
  // per-level overview planes for 16 slices (fill scratch)
  uint8_t *slab_buf = nullptr, *slab_src = nullptr, *slab_planes = nullptr;
  uint32_t slab_dims[3] = {0, 0, 0};
  uint32_t slab_ovn[r3d::kSlabLevels][2] = {};
  size_t slab_plane_off[r3d::kSlabLevels] = {};
  uint32_t slab_win = 0;
  bool have_slab = false;
  r3d::DevSlab sl{};

  // XY clipmap: the source volume, its tight 2^3 box pyramid (levels 2..5),
  // the level textures, their origins and the level slice each ring layer
  // holds (-1: none)
  uint8_t *clip_src = nullptr, *clip_pyr = nullptr, *clip_tex = nullptr;
  size_t clip_pyr_off[r3d::kClipLevels] = {};
  uint32_t clip_pyr_dim[r3d::kClipLevels][3] = {};
  uint32_t clip_dims[3] = {0, 0, 0};
  uint32_t clip_depth = 0;
  int64_t clip_org[r3d::kClipLevels][2] = {};
  std::vector<int64_t> clip_layer[r3d::kClipLevels];
  bool have_clip = false;
  r3d::DevClip cl{};

  // virtual slab: the source volume, the tile pool, the validity table
  // (device and its host copy), the ledger of the base tiles and scratch for
  // one fill's pyramid strips
  uint8_t *vs_src = nullptr, *vs_tiles = nullptr, *vs_strip = nullptr;
  uint32_t *vs_table = nullptr;
  std::vector<uint32_t> vs_table_host;
  std::vector<r3d_vslab_cell> vs_cells;
  std::vector<r3d_vslab_job> vs_jobs;
  r3d_vslab_layout vsl{};
  size_t vs_strip_off[r3d::kVsLevels] = {};
  bool have_vslab = false;
  r3d::DevVslab vs{};

  // flattened-segment views: the segment grids (xyz + valid, normals), the
  // baked flattened volume (W x H x L texels of CT, overlay) and its window,
  // the supervision mask
  float4 *surf_coords = nullptr, *surf_normals = nullptr;
  uint32_t surf_gw = 0, surf_gh = 0;
  uint8_t *sv_vol = nullptr, *surf_mask = nullptr;
  uint32_t surf_mw = 0, surf_mh = 0;
  uint32_t sv_W = 0, sv_H = 0, sv_L = 0, sv_nback = 0;
  float sv_sx = 0.0f, sv_sy = 0.0f, sv_u0 = 0.0f, sv_v0 = 0.0f, sv_step = 0.0f, sv_zoff0 = 0.0f;
  int sv_ovl = -1;  // overlay atlas baked into G (-1: none)
  // live 2.5D ink prediction baked into G over every layer (null: none)
  float *sv_pred = nullptr;
  uint32_t sv_pw = 0, sv_ph = 0;
  float sv_pg0u = 0.0f, sv_pg0v = 0.0f, sv_pppg = 0.0f;
  bool sv_baked = false;

  // single-level brick atlas: 4 mip levels, then the world-indexed
  // occupancy grid, in one allocation; page table of bpa^3 entries
  uint8_t *shard_buf = nullptr;
  uint32_t *shard_page = nullptr;
  bool have_shard = false;
  r3d::DevShard sh{};

  // transfer function
  uchar4 *lut = nullptr;
  uint8_t lut_host[256][4];
  float tf_zero_t = -1.0f;

  uint32_t *slot_bits = nullptr;  // r3d_cuda_set_slot_trace
  uint32_t quality = R3D_QUALITY_FULL;
  float alpha_cutoff = 0.98f;
  uint32_t *status = nullptr;

  // device staging for host-pointer outputs
  uint8_t *img = nullptr;
  size_t img_cap = 0;
  uint32_t *aux_buf = nullptr;
  size_t aux_cap = 0;
  unsigned long long *total = nullptr;  // R3D_COUNTERS + 1 device counters

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timed = false;

  // fixed-point gradient accumulators of the deterministic adjoint
  unsigned long long *diff_q = nullptr;
  size_t diff_q_bytes = 0;
  // quad grid of the differentiable render (float4 per voxel) and the
  // density buffer it was last built from
  void *diff_quad = nullptr;
  size_t diff_quad_bytes = 0;
  const float *quad_src = nullptr;

  // tape of the last training forward (r3d_cuda_diff_forward_tape): per
  // ray up to 64 contributing samples (float2) and their count, and the
  // arguments it was recorded for
  void *tape = nullptr;
  uint32_t *tape_n = nullptr;
  size_t tape_rays = 0;
  bool tape_valid = false;
  r3d_frame_params tape_views[64];
  uint32_t tape_nviews = 0;
  const float *tape_density = nullptr, *tape_lut = nullptr;
  uint32_t tape_dims[3] = {0, 0, 0};
  float tape_cutoff = 0.0f;

  // forward scheduling and the view-table ring of persistent launches:
  // slot k holds one call's views (pinned host copy + device copy) and its
  // tile counters; ring_ev[k] completes once the slot's upload has run
  r3d_cuda_schedule sched = {3u, 16u, 0u, 1u, 0u, 0u, 0u};
  static constexpr int kRing = 4;
  r3d::DevView *ring_host = nullptr;
  r3d::DevView *ring_dev = nullptr;
  uint32_t *ring_queue = nullptr;
  cudaEvent_t ring_ev[kRing] = {};
  bool ring_used[kRing] = {};
  int ring_next = 0;

  r3d::DevScene scene() const;
};

namespace r3d {

int fail(r3d_cuda_ctx *c, int code, const char *fmt, ...);
int cuda_fail(r3d_cuda_ctx *c, cudaError_t e, const char *what);
bool is_device_ptr(const void *p);

// A copy in either direction (host or device source) ordered on stream s and
// complete on return.  Uploads go through here rather than cudaMemcpy on the
// legacy stream: the context's stream is non-blocking, so a device-to-device
// or staged pageable cudaMemcpy is not ordered before its kernels.
inline cudaError_t copy_sync(cudaStream_t s, void *dst, const void *src, size_t n) {
  cudaError_t e = cudaMemcpyAsync(dst, src, n, cudaMemcpyDefault, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

// The schedule a call with nrender renderable views runs under.  persistent
// = 3 (automatic) is whole tiles for two or more views and one thread per
// ray for one: a grid launch per view leaves the SMs idle between small
// views (1080p split into 4/16/64 views: 2.0x/6.2x/19.6x slower than whole
// tiles on a B200), while a single 1080p view is 10 % faster as a grid.
inline uint32_t resolved_persistent(const r3d_cuda_schedule &sc, uint32_t nrender) {
  return sc.persistent == 3u ? (nrender > 1u ? 2u : 0u) : sc.persistent;
}

// Dispatch rows [row0, row1) of a view (half-resolution views: rows of the
// halved grid); row0 is rounded down to a block row.
struct Rows {
  uint32_t row0 = 0u, row1 = 0xffffffffu;
};

// The forward launch of one sampling path (each defined in its own object).
template <int PATH>
cudaError_t launch_path(const r3d_frame_params &pc, const DevScene &s, bool fast,
                        const uchar4 *lut, uint8_t *img, uint32_t out_w, uint32_t *steps,
                        uint32_t *mip, unsigned long long *total, unsigned long long *cnt,
                        uint32_t shade, const Rows &rows, cudaStream_t st);

// Flattened-segment view (view_flags R3D_VIEW_SURF) into a device image.
cudaError_t launch_surf(const r3d_cuda_ctx *c, const r3d_frame_params &pc, uint8_t *img,
                        uint32_t out_w, uint32_t *steps, uint32_t *mip, cudaStream_t st);

// The TMA-staged kernel (r3d_staged.cu): whether a view can use it, and its
// launch into a device image.
bool staged_supported(const r3d_cuda_ctx *c, const r3d_frame_params &pc);
cudaError_t launch_staged(const r3d_cuda_ctx *c, const r3d_frame_params &pc, uint8_t *img,
                          uint32_t out_w, unsigned long long *total, cudaStream_t st);

// Forward launch of one sanitized view into a device image.
cudaError_t launch_view(const r3d_cuda_ctx *c, const r3d_frame_params &pc, uint8_t *img,
                        uint32_t out_w, uint32_t *steps, uint32_t *mip_index,
                        unsigned long long *total, unsigned long long *counters,
                        cudaStream_t stream, const Rows &rows = Rows());

}  // namespace r3d

// (Re)allocates and fills the per-slot block-maximum and quad tables of the
// context's slot pool (dropping its overlays); atlas bricks per axis of a
// pool of nslots slots.
int build_blockmax(r3d_cuda_ctx *c);
// Drops the streaming state (host store, shadows, LRU).
void stream_reset(r3d_cuda_ctx *c);
// The display filter: whether it changes target t (0 CT, 1 ink atlas, 2 3D
// ink atlas), and filtering n slots in place on the context's stream, of a
// linear pool of 128^3 slots (atlas_bpa 0) or of a single-level atlas of
// atlas_bpa^3 slots.
bool postfilter_on(const r3d_cuda_ctx *c, uint32_t target);
int postfilter_slots(r3d_cuda_ctx *c, uint32_t target, uint8_t *pool, const uint32_t *slots,
                     uint32_t n, uint32_t atlas_bpa = 0u);
void postfilter_reset(r3d_cuda_ctx *c);
// Frees the tiled slab / the clipmap.
void slab_reset(r3d_cuda_ctx *c);
void clip_reset(r3d_cuda_ctx *c);
void vslab_reset(r3d_cuda_ctx *c);
void surf_reset(r3d_cuda_ctx *c);
uint32_t atlas_bpa(uint32_t nslots);

// Validates one view and clips its rect to the image (1: render, 0: empty
// rect, < 0: error code).
int prepare_view(r3d_cuda_ctx *c, const r3d_frame_params &in, uint32_t out_w, uint32_t out_h,
                 r3d_frame_params &pc);

#define R3D_CUDA_TRY(ctx, expr)                                  \
  do {                                                           \
    cudaError_t e_ = (expr);                                     \
    if (e_ != cudaSuccess) return r3d::cuda_fail(ctx, e_, #expr); \
  } while (0)
