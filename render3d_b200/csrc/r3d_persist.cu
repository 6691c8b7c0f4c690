// Persistent raycast kernel: resident warps drain a queue of ray tiles.
//
// A one-thread-per-ray launch leaves lanes idle once their rays end (early
// termination, background pixels) and SM slots idle while blocks wait for
// their slowest warp.  Here every warp keeps its lanes busy: when at least
// `refill_min` lanes are idle, it claims rays from its pending tile and, when
// that is used up, pulls the next tile from a global counter (one atomic per
// 32 rays).  Tiles are 32 dispatch threads (8x4, 16x2 or 32x1), ordered in
// 8x8-tile supertiles, Morton order inside.  A launch may cover many views of
// different sizes (the batched path): their tiles are numbered consecutively
// and the per-view march constants sit in shared memory.
//
// Per-ray arithmetic is the same ray_begin / ray_step / ray_end as the
// one-ray-per-thread kernel, so results are bit-identical to it and to the
// CPU oracle; only the order in which rays are processed changes.
#include <string.h>

#include "r3d_internal.h"
#include "r3d_persist.h"

// Resident 128-thread blocks per SM the whole-tile kernel's registers are
// bounded for: as the one-thread-per-ray kernels (8 for the plain LOD-brick
// kernels, 9 for their MIP, 7 elsewhere), except the LOD-brick FULL kernel
// (R3D_TILES_FULL_BLOCKS).
#ifndef R3D_TILES_FULL_BLOCKS
#define R3D_TILES_FULL_BLOCKS 8
#endif
#define R3D_TILES_BOUNDS                                                                   \
  __launch_bounds__(128, (PATH == PATH_LOD_BRICKS && !COUNT && MODE != R3D_MODE_HEATMAP)    \
                             ? (MODE == R3D_MODE_MIP     ? 9                                \
                                : MODE == R3D_MODE_FULL ? R3D_TILES_FULL_BLOCKS            \
                                                        : 8)                               \
                             : 7)

namespace r3d {

constexpr uint32_t kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// mask without its lowest n set bits
__device__ __forceinline__ uint32_t drop_low_bits(uint32_t mask, uint32_t n) {
  if (n == 0u) return mask;
  uint32_t p = __fns(mask, 0u, (int)n);
  return p >= 31u ? 0u : mask & (~0u << (p + 1u));
}

// dispatch-thread coordinates of ray k (0..31) of tile `tile` of a view
__host__ __device__ __forceinline__ void tile_ray(const DevView &v, uint32_t tile, uint32_t k,
                                         uint32_t shape, uint32_t &tx, uint32_t &ty) {
  const uint32_t tile_w = tile_w_of(shape);
  const uint32_t tile_h = 32u / tile_w;
  const uint32_t sup = tile >> 6, local = tile & 63u;
  const uint32_t lx = (local & 1u) | ((local >> 1) & 2u) | ((local >> 2) & 4u);
  const uint32_t ly = ((local >> 1) & 1u) | ((local >> 2) & 2u) | ((local >> 3) & 4u);
  // supertile rows from the view's middle outwards (c, c - 1, c + 1, ...;
  // each in [0, sup_y) once): the long rays start first (a 1080p view
  // drained alone 4 % faster, 4 to 64 views of a frame unchanged)
  const uint32_t sup_y = ((v.grid_h + tile_h - 1u) / tile_h + 7u) / 8u;
  const uint32_t sx = sup % v.sup_x, si = sup / v.sup_x, sc = sup_y / 2u, sd = (si + 1u) / 2u;
  const uint32_t sy = (si & 1u) ? sc - sd : sc + sd;
  const uint32_t tcx = sx * 8u + lx, tcy = sy * 8u + ly;  // tile coordinates
  // within the tile: Morton order of the 32 rays for 8x4, row-major else
  uint32_t ix, iy;
  if (tile_w == 8u) {
    ix = (k & 1u) | ((k >> 1) & 2u) | ((k >> 2) & 4u);
    iy = ((k >> 1) & 1u) | ((k >> 2) & 2u);
  } else {
    ix = k % tile_w;
    iy = k / tile_w;
  }
  tx = tcx * tile_w + ix;
  ty = tcy * tile_h + iy;
}

// mask of the rays of a tile that fall inside the view's dispatch grid
// (lane k tests ray k)
__device__ __forceinline__ uint32_t tile_valid(const DevView &v, uint32_t tile, uint32_t shape,
                                               uint32_t lane) {
  uint32_t tx, ty;
  tile_ray(v, tile, lane, shape, tx, ty);
  return __ballot_sync(0xffffffffu, tx < v.grid_w && ty < v.grid_h);
}

template <int MODE>
__device__ __forceinline__ void store_ray(const DevView &v, uint32_t px, uint32_t py,
                                          const RayResult &r, uint32_t *steps_out,
                                          uint32_t *mip_out) {
  const uchar4 col = make_uchar4(unorm8(r.rgb[0]), unorm8(r.rgb[1]), unorm8(r.rgb[2]), 255);
  const r3d_frame_params &pc = v.pc;
  const bool half = (pc.view_flags & R3D_VIEW_HALF) != 0u;
  const uint32_t vw = pc.viewport[0], vh = pc.viewport[1];
  const uint32_t ox = pc.view_org & 0xffffu, oy = pc.view_org >> 16;
  const uint32_t n = half ? 4u : 1u;
  for (uint32_t k = 0; k < n; k++) {
    uint32_t ax = px + (k & 1u), ay = py + (k >> 1);
    if (ax >= vw || ay >= vh) continue;
    size_t i = (size_t)(oy + ay) * v.stride + (ox + ax);
    v.img[i] = col;
    if (steps_out) steps_out[i] = r.steps;
    if (mip_out) mip_out[i] = r.mip_index;
  }
}

template <int PATH, int MODE, bool FAST, bool COUNT, int UNROLL>
__global__ void __launch_bounds__(128) k_raycast_persist(
    const DevView *__restrict__ views, uint32_t nviews, const __grid_constant__ DevScene s,
    const uchar4 *__restrict__ lut, uint32_t *__restrict__ queue, uint32_t ntiles,
    uint32_t refill_min, uint32_t shape, uint32_t *__restrict__ steps_out,
    uint32_t *__restrict__ mip_out, unsigned long long *__restrict__ total,
    unsigned long long *__restrict__ counters) {
  __shared__ float4 tf[256];
  __shared__ ViewConst vcs[kMaxBatchViews];
  for (uint32_t i = threadIdx.x; i < 256u; i += blockDim.x) {
    uchar4 u = lut[i];
    tf[i] = make_float4((float)u.x, (float)u.y, (float)u.z, (float)u.w);
  }
  for (uint32_t i = threadIdx.x; i < nviews; i += blockDim.x)
    vcs[i] = view_const<PATH>(views[i].pc, s, elide_counts(views[i].pc, s.tf_zero_t));
  __syncthreads();

  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt = lanemask_lt();
  RayState st;
  bool active = false;
  uint32_t my_view = 0, my_px = 0, my_py = 0;
  uint32_t pend_tile = 0, pend_view = 0, avail = 0;  // warp-uniform
  bool exhausted = false;
  uint32_t acc_steps = 0, acc_tf = 0, acc_grad = 0, acc_walk = 0;

  while (true) {
    uint32_t idle = __ballot_sync(kFull, !active);
    // refill rounds: assign rays to idle lanes until enough are busy
    while (!exhausted && idle != 0u && (__popc(idle) >= (int)refill_min || idle == kFull)) {
      if (avail == 0u) {
        uint32_t t0 = 0;
        if (lane == 0) t0 = atomicAdd(queue, 1u);
        t0 = __shfl_sync(kFull, t0, 0);
        if (t0 >= ntiles) {
          exhausted = true;
          break;
        }
        // view of global tile t0 (views are few: linear scan)
        uint32_t vi = 0;
        while (vi + 1u < nviews && views[vi + 1u].tile_begin <= t0) vi++;
        pend_view = vi;
        pend_tile = t0 - views[vi].tile_begin;
        avail = tile_valid(views[vi], pend_tile, shape, lane);
        continue;
      }
      const uint32_t n = min((uint32_t)__popc(idle), (uint32_t)__popc(avail));
      const bool mine = ((idle >> lane) & 1u) != 0u;
      const uint32_t rank = (uint32_t)__popc(idle & lt);
      if (mine && rank < n) {
        const uint32_t k = __fns(avail, 0u, (int)rank + 1);
        const DevView &v = views[pend_view];
        uint32_t tx, ty;
        tile_ray(v, pend_tile, k, shape, tx, ty);
        const bool half = (v.pc.view_flags & R3D_VIEW_HALF) != 0u;
        const uint32_t px = half ? tx * 2u : tx, py = half ? ty * 2u : ty;
        RayResult r;
        if (ray_begin<PATH, MODE>(v.pc, s, vcs[pend_view], px, py, st, r)) {
          active = true;
          my_view = pend_view;
          my_px = px;
          my_py = py;
        } else {
          store_ray<MODE>(v, px, py, r, steps_out, mip_out);
        }
      }
      idle = drop_low_bits(idle, n);
      avail = drop_low_bits(avail, n);
      idle = __ballot_sync(kFull, !active);
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;
    }
    if (active) {
      const ViewConst &vc = vcs[my_view];
#pragma unroll
      for (int u = 0; u < UNROLL; u++) {
        Pending pend;
        if (ray_step<PATH, MODE, FAST, COUNT>(s, vc, tf, st, pend) == kStepDone) {
          RayResult r;
          ray_end<MODE>(vc, st, r);
          store_ray<MODE>(views[my_view], my_px, my_py, r, steps_out, mip_out);
          acc_steps += r.steps;
          if (COUNT) {
            acc_tf += r.n_tf;
            acc_grad += r.n_grad;
            acc_walk += r.n_walk;
          }
          active = false;
          break;
        }
      }
    }
  }
  if (total) {
    uint32_t sum = acc_steps;
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
    if (lane == 0 && sum) atomicAdd(total, (unsigned long long)sum);
  }
  if (COUNT) {
    uint32_t v4[4] = {acc_steps, acc_tf, acc_grad, acc_walk};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t sum = v4[k];
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
      if (lane == 0 && sum) atomicAdd(counters + k, (unsigned long long)sum);
    }
  }
}

// The views and scenes of a whole-tile launch, held in its launch
// parameters (constant memory): N = 1 for a launch of one view, else up to
// 64 views; NS scenes (1, or up to 4 when the views sample several).
template <uint32_t N>
struct TileViews {
  DevView v[N];
  uint32_t n;
};
template <uint32_t NS>
struct TileScenes {
  DevScene s[NS];
  const uchar4 *lut[NS];
  uint32_t n;
};

// Whole-tile queue: each warp takes an 8x4 ray tile from the queue, marches
// its 32 rays to the end exactly as the one-thread-per-ray kernel does (no
// per-step warp votes; the view's parameters and its scene in constant
// memory), stores them and takes the next tile.  Warps never wait for each
// other, so an SM slot freed by a warp whose rays ended early is refilled
// at once, and the tail of a launch over many views is one tile long.
template <int PATH, int MODE, bool FAST, bool COUNT, uint32_t N, uint32_t NS>
__global__ void R3D_TILES_BOUNDS k_raycast_tiles(
    const __grid_constant__ TileViews<N> tv, const __grid_constant__ TileScenes<NS> sc,
    uint32_t *__restrict__ queue, uint32_t ntiles, uint32_t nwarps,
    uint32_t *__restrict__ steps_out, uint32_t *__restrict__ mip_out,
    unsigned long long *__restrict__ total, unsigned long long *__restrict__ counters) {
  __shared__ float4 tf[NS][256];
  for (uint32_t k = 0; k < (NS > 1 ? sc.n : 1u); k++)
    for (uint32_t i = threadIdx.x; i < 256u; i += blockDim.x) {
      const uchar4 u = sc.lut[k][i];
      tf[k][i] = make_float4((float)u.x, (float)u.y, (float)u.z, (float)u.w);
    }
  __syncthreads();
  uint32_t vi = 0;
  while (true) {
    uint32_t t = 0;
    if ((threadIdx.x & 31u) == 0u) t = atomicAdd(queue, 1u);
    t = __shfl_sync(kFull, t, 0);
    if (t >= ntiles) break;
    // tiles are taken in order, so the view index only moves forward
    if (N > 1)
      while (vi + 1u < tv.n && tv.v[vi + 1u].tile_begin <= t) vi++;
    const DevView &v = tv.v[N > 1 ? vi : 0u];
    const uint32_t si = NS > 1 ? v.scene : 0u;
    const DevScene &s = sc.s[si];
    const bool half = (v.pc.view_flags & R3D_VIEW_HALF) != 0u;
    RayResult r;
    r.steps = r.n_tf = r.n_grad = r.n_walk = 0u;
    {
      uint32_t tx, ty;
      tile_ray(v, t - v.tile_begin, threadIdx.x & 31u, 0u, tx, ty);
      const bool inside = tx < v.grid_w && ty < v.grid_h;
      const uint32_t px = half ? tx * 2u : tx, py = half ? ty * 2u : ty;
      const ViewConst vc = view_const<PATH>(v.pc, s, v.el);
      march_warp<PATH, MODE, FAST, COUNT>(v.pc, s, vc, tf[si], px, py, inside, r);
    }
    // the ray's pixel again, from the tile index: recomputed after the march
    // (an opaque copy of t stops the compiler from keeping it live across)
    uint32_t t2;
    asm volatile("mov.u32 %0, %1;" : "=r"(t2) : "r"(t));
    uint32_t tx, ty;
    tile_ray(v, t2 - v.tile_begin, threadIdx.x & 31u, 0u, tx, ty);
    if (tx < v.grid_w && ty < v.grid_h)
      store_ray<MODE>(v, half ? tx * 2u : tx, half ? ty * 2u : ty, r, steps_out, mip_out);
    // work counters per tile: one atomic per 32 rays, nothing kept live
    // across the march
    if (total) {
      uint32_t sum = r.steps;
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
      if ((threadIdx.x & 31u) == 0u && sum) atomicAdd(total, (unsigned long long)sum);
    }
    if (COUNT) {
      uint32_t v4[4] = {r.steps, r.n_tf, r.n_grad, r.n_walk};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        uint32_t sum = v4[k];
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
        if ((threadIdx.x & 31u) == 0u && sum) atomicAdd(counters + k, (unsigned long long)sum);
      }
    }
  }
  // the last warp to retire resets the counters for the next launch: every
  // other warp took its last tile before it counted itself out
  if ((threadIdx.x & 31u) == 0u) {
    __threadfence();
    if (atomicAdd(queue + 1, 1u) == nwarps - 1u) {
      atomicExch(queue, 0u);
      atomicExch(queue + 1, 0u);
    }
  }
}

template <int PATH, int MODE, bool FAST, bool COUNT, uint32_t N, uint32_t NS>
static cudaError_t launch_tn(const TilesLaunch &L, cudaStream_t st) {
  auto kern = k_raycast_tiles<PATH, MODE, FAST, COUNT, N, NS>;
  uint32_t blocks = L.blocks;
  if (!blocks) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 128, 0);
    if (e != cudaSuccess) return e;
    blocks = (uint32_t)(per > 0 ? per : 1) * (uint32_t)sms;
  }
  const uint32_t cap = (L.ntiles + 3u) / 4u;  // no more warps than tiles
  blocks = blocks < cap ? blocks : (cap ? cap : 1u);
  TileViews<N> tv;
  memcpy(tv.v, L.views, sizeof(DevView) * L.nviews);
  tv.n = L.nviews;
  for (uint32_t i = 0; i < L.nviews; i++)
    tv.v[i].el = elide_counts(tv.v[i].pc, L.scenes[L.nscenes > 1u ? tv.v[i].scene : 0u].tf_zero_t);
  TileScenes<NS> sc;
  for (uint32_t k = 0; k < L.nscenes; k++) {
    sc.s[k] = L.scenes[k];
    sc.lut[k] = L.luts[k];
  }
  sc.n = L.nscenes;
  kern<<<blocks, 128, 0, st>>>(tv, sc, L.queue, L.ntiles, blocks * 4u, L.steps, L.mip, L.total,
                               L.counters);
  return cudaGetLastError();
}

template <int PATH, int MODE, bool FAST, bool COUNT>
static cudaError_t launch_tt(const TilesLaunch &L, cudaStream_t st) {
  if (L.nscenes > 1u) return launch_tn<PATH, MODE, FAST, COUNT, kMaxBatchViews, kMaxScenes>(L, st);
  if (L.nviews == 1u) return launch_tn<PATH, MODE, FAST, COUNT, 1, 1>(L, st);
  return launch_tn<PATH, MODE, FAST, COUNT, kMaxBatchViews, 1>(L, st);
}

template <int PATH, int MODE, bool FAST>
static cudaError_t launch_tc(const TilesLaunch &L, cudaStream_t st) {
  return L.counters ? launch_tt<PATH, MODE, FAST, true>(L, st)
                    : launch_tt<PATH, MODE, FAST, false>(L, st);
}

template <int PATH>
static cudaError_t launch_tm(const TilesLaunch &L, cudaStream_t st) {
  switch (L.mode) {
    case R3D_MODE_FULL:
      return L.fast ? launch_tc<PATH, R3D_MODE_FULL, true>(L, st)
                    : launch_tc<PATH, R3D_MODE_FULL, false>(L, st);
    case R3D_MODE_MIP: return launch_tc<PATH, R3D_MODE_MIP, false>(L, st);
    case R3D_MODE_DEPTH: return launch_tc<PATH, R3D_MODE_DEPTH, false>(L, st);
    case R3D_MODE_HEATMAP: return launch_tc<PATH, R3D_MODE_HEATMAP, false>(L, st);
    case R3D_MODE_RAYDIR: return launch_tc<PATH, R3D_MODE_RAYDIR, false>(L, st);
    default: return launch_tc<PATH, R3D_MODE_FLAT, false>(L, st);
  }
}

template <int PATH, int MODE, bool FAST, bool COUNT, int UNROLL>
static cudaError_t launch_pt(const PersistLaunch &L, const DevScene &s, cudaStream_t st) {
  k_raycast_persist<PATH, MODE, FAST, COUNT, UNROLL><<<L.blocks, 128, 0, st>>>(
      L.views, L.nviews, s, L.lut, L.queue, L.ntiles, L.refill_min, L.shape, L.steps, L.mip,
      L.total, L.counters);
  return cudaGetLastError();
}

template <int PATH, int MODE, bool FAST, bool COUNT>
static cudaError_t launch_pu(const PersistLaunch &L, const DevScene &s, cudaStream_t st) {
  return L.unroll == 2 ? launch_pt<PATH, MODE, FAST, COUNT, 2>(L, s, st)
                       : launch_pt<PATH, MODE, FAST, COUNT, 1>(L, s, st);
}

template <int PATH, int MODE, bool FAST>
static cudaError_t launch_pc(const PersistLaunch &L, const DevScene &s, cudaStream_t st) {
  return L.counters ? launch_pu<PATH, MODE, FAST, true>(L, s, st)
                    : launch_pu<PATH, MODE, FAST, false>(L, s, st);
}

template <int PATH>
static cudaError_t launch_pm(const PersistLaunch &L, const DevScene &s, cudaStream_t st) {
  switch (L.mode) {
    case R3D_MODE_FULL:
      return L.fast ? launch_pc<PATH, R3D_MODE_FULL, true>(L, s, st)
                    : launch_pc<PATH, R3D_MODE_FULL, false>(L, s, st);
    case R3D_MODE_MIP: return launch_pc<PATH, R3D_MODE_MIP, false>(L, s, st);
    case R3D_MODE_DEPTH: return launch_pc<PATH, R3D_MODE_DEPTH, false>(L, s, st);
    case R3D_MODE_HEATMAP: return launch_pc<PATH, R3D_MODE_HEATMAP, false>(L, s, st);
    case R3D_MODE_RAYDIR: return launch_pc<PATH, R3D_MODE_RAYDIR, false>(L, s, st);
    default: return launch_pc<PATH, R3D_MODE_FLAT, false>(L, s, st);
  }
}

#ifdef R3D_FWD_PATH
// Compiled once per sampling path (R3D_FWD_PATH = 0..5), as the forward
// kernels are.
template <>
cudaError_t persist_path<R3D_FWD_PATH>(const PersistLaunch &L, const DevScene &s,
                                       cudaStream_t st) {
  return launch_pm<R3D_FWD_PATH>(L, s, st);
}

template <>
cudaError_t tiles_path<R3D_FWD_PATH>(const TilesLaunch &L, cudaStream_t st) {
  return launch_tm<R3D_FWD_PATH>(L, st);
}

template <>
int persist_occupancy<R3D_FWD_PATH>(uint32_t mode, bool fast, uint32_t unroll) {
  // occupancy of the instantiation that persist_path picks
  constexpr int P = R3D_FWD_PATH;
  int n = 0;
  cudaError_t e;
  if (P == PATH_LOD_BRICKS && (mode != R3D_MODE_FULL || fast))
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &n, k_raycast_persist<P, R3D_MODE_MIP, false, false, 1>, 128, 0);
  else if (P == PATH_LOD_BRICKS && unroll == 2)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &n, k_raycast_persist<P, R3D_MODE_FULL, false, false, 2>, 128, 0);
  else
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &n, k_raycast_persist<P, R3D_MODE_FULL, false, false, 1>, 128, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 4;
  }
  return n > 0 ? n : 1;
}
#else
cudaError_t launch_persist(const PersistLaunch &L, const DevScene &s, cudaStream_t st) {
  switch (L.path) {
    case PATH_VSLAB: return persist_path<PATH_VSLAB>(L, s, st);
    case PATH_CLIP: return persist_path<PATH_CLIP>(L, s, st);
    case PATH_SLAB: return persist_path<PATH_SLAB>(L, s, st);
    case PATH_LOD_BRICKS: return persist_path<PATH_LOD_BRICKS>(L, s, st);
    case PATH_SHARD: return persist_path<PATH_SHARD>(L, s, st);
    default: return persist_path<PATH_CUBE>(L, s, st);
  }
}

cudaError_t launch_tiles(const TilesLaunch &L, cudaStream_t st) {
  switch (L.path) {
    case PATH_VSLAB: return tiles_path<PATH_VSLAB>(L, st);
    case PATH_CLIP: return tiles_path<PATH_CLIP>(L, st);
    case PATH_SLAB: return tiles_path<PATH_SLAB>(L, st);
    case PATH_LOD_BRICKS: return tiles_path<PATH_LOD_BRICKS>(L, st);
    case PATH_SHARD: return tiles_path<PATH_SHARD>(L, st);
    default: return tiles_path<PATH_CUBE>(L, st);
  }
}

int persist_blocks_per_sm(int path, uint32_t mode, bool fast, uint32_t unroll) {
  switch (path) {
    case PATH_VSLAB: return persist_occupancy<PATH_VSLAB>(mode, fast, unroll);
    case PATH_CLIP: return persist_occupancy<PATH_CLIP>(mode, fast, unroll);
    case PATH_SLAB: return persist_occupancy<PATH_SLAB>(mode, fast, unroll);
    case PATH_LOD_BRICKS: return persist_occupancy<PATH_LOD_BRICKS>(mode, fast, unroll);
    case PATH_SHARD: return persist_occupancy<PATH_SHARD>(mode, fast, unroll);
    default: return persist_occupancy<PATH_CUBE>(mode, fast, unroll);
  }
}
#endif

}  // namespace r3d
