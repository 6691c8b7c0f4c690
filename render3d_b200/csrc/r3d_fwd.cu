// Forward raycast kernels: one thread per ray; each warp covers an 8x4 tile
// of dispatch threads (4x8 for LOD-brick FULL and FLAT views in 4-warp
// blocks) whose lanes follow a Morton (Z-order) curve, so a warp's rays stay
// spatially compact and share cache lines; a block holds 1, 2 or 4 warp
// tiles.  Mode, sampling path and gradient quality are template parameters
// (the reference specializes its shader per path for the same reason:
// src/shaders/raycast.slang:127-130).
#include "r3d_internal.h"

// Minimum resident 128-thread blocks per SM the register allocator targets
// (0: no target).  The plain LOD-brick kernels (no overlay atlases, counters
// or parked shading, not the step heatmap) get one block more, MIP two, all
// without spills: 1080p FULL runs 2 % faster at 64 registers and MIP 5 %
// at 56, while the overlay and shard kernels lose 14 % and 4 % and the
// heatmap 3 % at 8 blocks, and FULL spills at 9.
#ifndef R3D_FWD_MIN_BLOCKS
#define R3D_FWD_MIN_BLOCKS 7
#endif
// Warps per block: 1, 2 or 4 8x4 warp tiles.
#ifndef R3D_FWD_WARPS
#define R3D_FWD_WARPS 4
#endif
#if R3D_FWD_MIN_BLOCKS > 0
#define R3D_FWD_BOUNDS                                                                     \
  __launch_bounds__(R3D_FWD_WARPS * 32,                                                    \
                    (R3D_FWD_MIN_BLOCKS + (PATH == PATH_LOD_BRICKS && !OVL && !COUNT &&    \
                                                   !DEFER && MODE != R3D_MODE_HEATMAP            \
                                               ? (MODE == R3D_MODE_MIP ? 2 : 1)                  \
                                               : 0)) * 4 / R3D_FWD_WARPS)
#else
#define R3D_FWD_BOUNDS __launch_bounds__(R3D_FWD_WARPS * 32)
#endif

namespace r3d {

constexpr uint32_t kFwdWarps = R3D_FWD_WARPS;
constexpr uint32_t kBlockW = kFwdWarps >= 2 ? 16u : 8u;  // dispatch threads per block, x
constexpr uint32_t kBlockH = kFwdWarps == 4 ? 8u : 4u;   // and y
static_assert(kFwdWarps == 1 || kFwdWarps == 2 || kFwdWarps == 4, "1, 2 or 4 warps");

// DEFER (FULL mode): gradient shading is the long branch of a step and
// usually only one or two lanes of a warp need it at once.  A lane that
// reaches a shaded sample parks it (ray_step returns kStepShade); the warp
// shades the parked samples together once at least shade_min lanes are
// waiting or every live lane is, so the branch runs with more lanes active.
// Rays are independent, so each ray's arithmetic and result are unchanged.
template <int PATH, int MODE, bool FAST, bool COUNT, bool DEFER, bool OVL = false>
__global__ void R3D_FWD_BOUNDS k_raycast(const __grid_constant__ r3d_frame_params pc,
                                         const __grid_constant__ DevScene s,
                                         const uchar4 *__restrict__ lut,
                                         uchar4 *__restrict__ img, uint32_t out_w,
                                         uint32_t *__restrict__ steps_out,
                                         uint32_t *__restrict__ mip_out,
                                         unsigned long long *__restrict__ total,
                                         unsigned long long *__restrict__ counters,
                                         uint32_t shade_min, uint32_t row0) {
  __shared__ float4 tf[256];
  for (uint32_t i = threadIdx.x; i < 256u; i += blockDim.x) {
    uchar4 u = lut[i];
    tf[i] = make_float4((float)u.x, (float)u.y, (float)u.z, (float)u.w);
  }
  __syncthreads();
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  // Lane bits interleave x and y.  Compositing LOD-brick views take 4x8
  // warp tiles, four side by side (1080p FULL 1 % faster than 8x4, same
  // images); MIP and the other paths keep 8x4 tiles in a 2x2 arrangement.
  constexpr bool kTall = kFwdWarps == 4u && PATH == PATH_LOD_BRICKS &&
                         (MODE == R3D_MODE_FULL || MODE == R3D_MODE_FLAT);
  const uint32_t lx = kTall ? (lane & 1u) | ((lane >> 1) & 2u)
                            : (lane & 1u) | ((lane >> 1) & 2u) | ((lane >> 2) & 4u);
  const uint32_t ly = kTall ? ((lane >> 1) & 1u) | ((lane >> 2) & 6u)
                            : ((lane >> 1) & 1u) | ((lane >> 2) & 2u);
  // LOD-brick MIP views take their blocks in strips 32 blocks wide, the
  // rows of a strip in turn (1080p MIP 0.8 % faster than row order; the
  // compositing views lose with strips)
  constexpr uint32_t kStrip = PATH == PATH_LOD_BRICKS && MODE == R3D_MODE_MIP ? 32u : 0u;
  constexpr bool kMidRows =
      kFwdWarps == 4u && (MODE == R3D_MODE_FULL || MODE == R3D_MODE_FLAT) &&
      (PATH == PATH_LOD_BRICKS || PATH == PATH_SHARD || PATH == PATH_CUBE);
  uint32_t bx = blockIdx.x, by = blockIdx.y;
  if (kStrip) {
    const uint32_t nby = gridDim.y, lin = blockIdx.y * gridDim.x + blockIdx.x;
    const uint32_t strip = lin / (kStrip * nby), within = lin - strip * (kStrip * nby);
    const uint32_t sw = min(kStrip, gridDim.x - strip * kStrip);
    bx = strip * kStrip + within % sw;
    by = within / sw;
  } else if (kMidRows) {
    // block rows by their distance from the view's middle row c (c, c - 1,
    // c + 1, ..., then the longer side's rest; a band of rows off the
    // middle runs from its edge nearest it): the long rays through the
    // volume start first and the frame's tail holds the short ones (1080p
    // LOD FULL and FLAT 3.5 % faster than row order, the cube's FULL 6 %,
    // the identity shard's 2.5 %).  Every index stays in [0, gridDim.y)
    // and each row is taken once.
    const uint32_t nby = gridDim.y, i = blockIdx.y;
    const uint32_t gh = (pc.view_flags & R3D_VIEW_HALF) ? (pc.viewport[1] + 1u) / 2u
                                                         : pc.viewport[1];
    const int c0 = (int)(gh / 2u / kBlockH) - (int)(row0 / kBlockH);
    const uint32_t c = (uint32_t)min(max(c0, 0), (int)nby - 1);
    const uint32_t below = c, above = nby - 1u - c, m = min(below, above);
    if (i <= 2u * m)
      by = (i & 1u) ? c - (i + 1u) / 2u : c + i / 2u;
    else
      by = below > above ? c - (i - m) : c + (i - m);
  }
  const uint32_t tx = bx * kBlockW + (kTall ? warp * 4u : (warp & 1u) * 8u) + lx;
  const uint32_t ty = row0 + by * kBlockH + (kTall ? 0u : (warp >> 1) * 4u) + ly;
  const bool half = (pc.view_flags & R3D_VIEW_HALF) != 0u;
  const uint32_t px = half ? tx * 2u : tx, py = half ? ty * 2u : ty;
  const uint32_t vw = pc.viewport[0], vh = pc.viewport[1];
  uint32_t my_steps = 0, my_tf = 0, my_grad = 0, my_walk = 0;
  const bool inside = px < vw && py < vh;
  const ViewConst vc = view_const<PATH>(pc, s);
  RayResult r;
  if (DEFER) {
    RayState st;
    Pending pend;
    bool active = inside && ray_begin<PATH, MODE>(pc, s, vc, px, py, st, r);
    const bool marched = active;
    bool parked = false;
    while (true) {
      if (__ballot_sync(0xffffffffu, active) == 0u) break;
      if (active && !parked) {
        const int rs = ray_step<PATH, MODE, FAST, COUNT, true>(s, vc, tf, st, pend);
        if (rs == kStepDone)
          active = false;
        else if (rs == kStepShade)
          parked = true;
      }
      const uint32_t need = __ballot_sync(0xffffffffu, parked);
      if (need != 0u) {
        const uint32_t live = __ballot_sync(0xffffffffu, active);
        if ((uint32_t)__popc(need) >= shade_min || need == live) {
          if (parked) {
            parked = false;
            if (!composite_sample<PATH, MODE, FAST, COUNT>(s, vc, st, pend)) active = false;
          }
        }
      }
    }
    if (marched) ray_end<MODE>(vc, st, r);
  } else {
    march_warp<PATH, MODE, FAST, COUNT, OVL>(pc, s, vc, tf, px, py, inside, r);
  }
  if (inside) {
    my_tf = r.n_tf;
    my_grad = r.n_grad;
    my_walk = r.n_walk;
    const uchar4 col = make_uchar4(unorm8(r.rgb[0]), unorm8(r.rgb[1]), unorm8(r.rgb[2]), 255);
    const uint32_t ox = pc.view_org & 0xffffu, oy = pc.view_org >> 16;
    const uint32_t n = half ? 4u : 1u;
    for (uint32_t k = 0; k < n; k++) {
      uint32_t ax = px + (k & 1u), ay = py + (k >> 1);
      if (ax >= vw || ay >= vh) continue;
      size_t i = (size_t)(oy + ay) * out_w + (ox + ax);
      img[i] = col;
      if (steps_out) steps_out[i] = r.steps;
      if (mip_out) mip_out[i] = r.mip_index;
    }
    my_steps = r.steps;
  }
  if (total) {
    uint32_t sum = my_steps;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0 && sum) atomicAdd(total, (unsigned long long)sum);
  }
  if (COUNT) {
    uint32_t v[4] = {my_steps, my_tf, my_grad, my_walk};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t sum = v[k];
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0 && sum) atomicAdd(counters + k, (unsigned long long)sum);
    }
  }
}

template <int PATH, int MODE, bool FAST>
static cudaError_t launch_t(const r3d_frame_params &pc, const DevScene &s, const uchar4 *lut,
                            uint8_t *img, uint32_t out_w, uint32_t *steps, uint32_t *mip,
                            unsigned long long *total, unsigned long long *counters,
                            uint32_t shade, const Rows &rows, cudaStream_t stream) {
  const bool half = (pc.view_flags & R3D_VIEW_HALF) != 0u;
  uint32_t gw = half ? (pc.viewport[0] + 1u) / 2u : pc.viewport[0];
  uint32_t gh = half ? (pc.viewport[1] + 1u) / 2u : pc.viewport[1];
  // dispatch rows [row0, row1) of the view; row0 starts a block row
  const uint32_t row0 = rows.row0 / kBlockH * kBlockH, row1 = min(rows.row1, gh);
  if (row0 >= row1) return cudaSuccess;
  dim3 grid((gw + kBlockW - 1u) / kBlockW, (row1 - row0 + kBlockH - 1u) / kBlockH);
  const uint32_t threads = kFwdWarps * 32u;
  constexpr bool kDeferable = MODE == R3D_MODE_FULL;
  // overlay atlases: LOD bricks in the compositing and MIP modes
  constexpr bool kOvl = PATH == PATH_LOD_BRICKS &&
                        (MODE == R3D_MODE_FULL || MODE == R3D_MODE_FLAT || MODE == R3D_MODE_MIP);
  if constexpr (kOvl) {
    if (pc.overlay_flags & kOvlAtlases) {
      if (counters)
        k_raycast<PATH, MODE, FAST, true, false, true><<<grid, threads, 0, stream>>>(
            pc, s, lut, (uchar4 *)img, out_w, steps, mip, total, counters, 0u, row0);
      else
        k_raycast<PATH, MODE, FAST, false, false, true><<<grid, threads, 0, stream>>>(
            pc, s, lut, (uchar4 *)img, out_w, steps, mip, total, nullptr, 0u, row0);
      return cudaGetLastError();
    }
  }
  if (kDeferable && shade) {
    if (counters)
      k_raycast<PATH, MODE, FAST, true, kDeferable><<<grid, threads, 0, stream>>>(
          pc, s, lut, (uchar4 *)img, out_w, steps, mip, total, counters, shade, row0);
    else
      k_raycast<PATH, MODE, FAST, false, kDeferable><<<grid, threads, 0, stream>>>(
          pc, s, lut, (uchar4 *)img, out_w, steps, mip, total, nullptr, shade, row0);
  } else if (counters) {
    k_raycast<PATH, MODE, FAST, true, false><<<grid, threads, 0, stream>>>(
        pc, s, lut, (uchar4 *)img, out_w, steps, mip, total, counters, 0u, row0);
  } else {
    k_raycast<PATH, MODE, FAST, false, false><<<grid, threads, 0, stream>>>(
        pc, s, lut, (uchar4 *)img, out_w, steps, mip, total, nullptr, 0u, row0);
  }
  return cudaGetLastError();
}

template <int PATH>
static cudaError_t launch_p(const r3d_frame_params &pc, const DevScene &s, bool fast,
                            const uchar4 *lut, uint8_t *img, uint32_t out_w, uint32_t *steps,
                            uint32_t *mip, unsigned long long *total,
                            unsigned long long *cnt, uint32_t shade, const Rows &rows,
                            cudaStream_t st) {
  switch (pc.mode) {
    case R3D_MODE_FULL:
      return fast ? launch_t<PATH, R3D_MODE_FULL, true>(pc, s, lut, img, out_w, steps, mip, total, cnt, shade, rows, st)
                  : launch_t<PATH, R3D_MODE_FULL, false>(pc, s, lut, img, out_w, steps, mip,
                                                         total, cnt, shade, rows, st);
    case R3D_MODE_MIP:
      return launch_t<PATH, R3D_MODE_MIP, false>(pc, s, lut, img, out_w, steps, mip, total, cnt, shade, rows, st);
    case R3D_MODE_DEPTH:
      return launch_t<PATH, R3D_MODE_DEPTH, false>(pc, s, lut, img, out_w, steps, mip, total, cnt, shade, rows, st);
    case R3D_MODE_HEATMAP:
      return launch_t<PATH, R3D_MODE_HEATMAP, false>(pc, s, lut, img, out_w, steps, mip, total, cnt, shade, rows, st);
    case R3D_MODE_RAYDIR:
      return launch_t<PATH, R3D_MODE_RAYDIR, false>(pc, s, lut, img, out_w, steps, mip, total, cnt, shade, rows, st);
    default:
      return launch_t<PATH, R3D_MODE_FLAT, false>(pc, s, lut, img, out_w, steps, mip, total, cnt, shade, rows, st);
  }
}

#ifdef R3D_FWD_PATH
// The build compiles this file once per sampling path (R3D_FWD_PATH = 0..5)
// so that the paths' kernels compile in parallel; each object defines its
// path's entry.
template <>
cudaError_t launch_path<R3D_FWD_PATH>(const r3d_frame_params &pc, const DevScene &s, bool fast,
                                      const uchar4 *lut, uint8_t *img, uint32_t out_w,
                                      uint32_t *steps, uint32_t *mip, unsigned long long *total,
                                      unsigned long long *cnt, uint32_t shade, const Rows &rows,
                                      cudaStream_t st) {
  return launch_p<R3D_FWD_PATH>(pc, s, fast, lut, img, out_w, steps, mip, total, cnt, shade, rows,
                                st);
}
#else
}  // namespace r3d

extern "C" void r3d_cuda_elide_counts(const r3d_frame_params *p, float tf_zero_t,
                                      uint32_t out[2]) {
  const r3d::ElideCounts e = r3d::elide_counts(*p, tf_zero_t);
  out[0] = e.n_void;
  out[1] = e.n_dec;
}

namespace r3d {

cudaError_t launch_view(const r3d_cuda_ctx *c, const r3d_frame_params &pc, uint8_t *img,
                        uint32_t out_w, uint32_t *steps, uint32_t *mip_index,
                        unsigned long long *total, unsigned long long *counters,
                        cudaStream_t stream, const Rows &rows) {
  if (pc.view_flags & R3D_VIEW_SURF)
    return launch_surf(c, pc, img, out_w, steps, mip_index, stream);
  if (c->sched.staging && !steps && !mip_index && !counters && rows.row0 == 0u &&
      rows.row1 == 0xffffffffu && staged_supported(c, pc))
    return launch_staged(c, pc, img, out_w, total, stream);
  DevScene s = c->scene();
  s.el = elide_counts(pc, s.tf_zero_t);
  const bool fast = c->quality == R3D_QUALITY_FAST;
  // shade_group 0 picks the path's default: grouped shading pays where a
  // gradient tap is a whole section lookup (tiled slab, clipmap, virtual
  // slab: 13-31 % faster frames at 16) and costs where it is a fetch inside
  // the cached brick (LOD bricks, cube: 1.7x slower frames)
  const int path = path_of_view(pc);
  const uint32_t shade = c->sched.shade_group ? c->sched.shade_group
                         : (path == PATH_SLAB || path == PATH_CLIP || path == PATH_VSLAB) ? 16u
                                                                                          : 0u;
#define R3D_PATH_CASE(P)                                                                   \
  case P:                                                                                  \
    return launch_path<P>(pc, s, fast, c->lut, img, out_w, steps, mip_index, total, counters, \
                          shade, rows, stream)
  switch (path) {
    R3D_PATH_CASE(PATH_VSLAB);
    R3D_PATH_CASE(PATH_CLIP);
    R3D_PATH_CASE(PATH_SLAB);
    R3D_PATH_CASE(PATH_LOD_BRICKS);
    R3D_PATH_CASE(PATH_SHARD);
    default:
      return launch_path<PATH_CUBE>(pc, s, fast, c->lut, img, out_w, steps, mip_index, total,
                                    counters, shade, rows, stream);
  }
#undef R3D_PATH_CASE
}
#endif

}  // namespace r3d
