// Persistent, queue-draining raycast launch (r3d_persist.cu).
#pragma once

#include "r3d_march.cuh"

namespace r3d {

constexpr uint32_t kMaxBatchViews = 64;

// One view of a persistent launch.
struct DevView {
  r3d_frame_params pc;  // sanitized view
  uchar4 *img;          // image the view's rect is written into
  uint32_t stride;      // pixels per image row
  uint32_t grid_w, grid_h;  // dispatch grid (half-resolution views: halved)
  uint32_t sup_x;       // 8x8-tile supertiles per grid row
  uint32_t tile_begin;  // index of the view's first tile in the launch
  uint32_t scene;       // whole-tile launches: index of the view's scene
  ElideCounts el;       // whole-tile launches: the view's elision counts
};

struct PersistLaunch {
  const DevView *views;  // device array
  uint32_t nviews;       // <= kMaxBatchViews
  uint32_t ntiles;
  const uchar4 *lut;
  // lane refill (tiles false): one tile counter, zero at launch.  Whole
  // tiles (tiles true): the tile counter and a counter of retired warps,
  // zero at launch; the last warp to retire sets both back to zero.
  uint32_t *queue;
  uint32_t refill_min, shape, unroll;
  uint32_t *steps, *mip;
  unsigned long long *total, *counters;
  uint32_t blocks;
  uint32_t mode;
  bool fast;
  int path;  // a Path
};

// Tile geometry for a tile shape (0: 8x4, 1: 16x2, 2: 32x1).
__host__ __device__ inline uint32_t tile_w_of(uint32_t shape) { return shape == 0u ? 8u : (shape == 1u ? 16u : 32u); }

// Fills grid_w/h, sup_x and the view's tile count (64 per supertile).
inline uint32_t view_tiles(DevView &v, uint32_t shape) {
  const bool half = (v.pc.view_flags & R3D_VIEW_HALF) != 0u;
  v.grid_w = half ? (v.pc.viewport[0] + 1u) / 2u : v.pc.viewport[0];
  v.grid_h = half ? (v.pc.viewport[1] + 1u) / 2u : v.pc.viewport[1];
  const uint32_t tw = tile_w_of(shape), th = 32u / tw;
  const uint32_t tx = (v.grid_w + tw - 1u) / tw, ty = (v.grid_h + th - 1u) / th;
  v.sup_x = (tx + 7u) / 8u;
  const uint32_t sup_y = (ty + 7u) / 8u;
  return v.sup_x * sup_y * 64u;
}

// A whole-tile launch: warps take whole 8x4 tiles (shape 0 numbering) of
// views that may sample different scenes.  The views and scenes are host
// copies passed to the kernel by value as its launch parameters.
constexpr uint32_t kMaxScenes = 4;
struct TilesLaunch {
  const DevView *views;  // host array; DevView::scene indexes scenes
  uint32_t nviews;       // <= kMaxBatchViews
  uint32_t ntiles;
  const DevScene *scenes;  // host array of nscenes (<= kMaxScenes)
  const uchar4 *const *luts;  // per scene
  uint32_t nscenes;
  // the tile counter and a counter of retired warps, zero at launch; the
  // last warp to retire sets both back to zero
  uint32_t *queue;
  uint32_t *steps, *mip;
  unsigned long long *total, *counters;
  uint32_t blocks;  // 0: the occupancy limit on every SM
  uint32_t mode;
  bool fast;
  int path;
};

cudaError_t launch_persist(const PersistLaunch &L, const DevScene &s, cudaStream_t st);
cudaError_t launch_tiles(const TilesLaunch &L, cudaStream_t st);
template <int PATH>
cudaError_t tiles_path(const TilesLaunch &L, cudaStream_t st);
int persist_blocks_per_sm(int path, uint32_t mode, bool fast, uint32_t unroll);
// Per-path halves of the two above (each defined in its own object).
template <int PATH>
cudaError_t persist_path(const PersistLaunch &L, const DevScene &s, cudaStream_t st);
template <int PATH>
int persist_occupancy(uint32_t mode, bool fast, uint32_t unroll);

}  // namespace r3d
