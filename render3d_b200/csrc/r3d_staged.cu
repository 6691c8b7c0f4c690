// TMA-staged raycast of the LOD brick path: each block marches one 8x8
// Morton tile of rays (two 8x4 warps) in lock step and stages, with a
// tensor copy (cp.async.bulk.tensor), the part of a slot its samples are in:
// a box of 32 x 17 x 17 texels of the u8 slot pool in shared memory.  Each
// step, the block looks at where its rays will sample next; when fewer
// than half of those samples lie in the staged box, one thread issues the
// copy of a box around the first ray outside it and the block waits for it
// on an mbarrier.  A sample whose 2x2x2 texels are in the box reads them
// from shared memory, any other from the quad pool, with the same texels
// and the same lerps either way, so images are bit-identical to the one-
// thread-per-ray kernel's (raycast.slang:284-288 is the fetch it replaces).
//
// The copy never multicasts and its tensor map covers only this GPU's own
// slot pool.  Every wait is bounded: a wait that runs out sets
// R3D_STATUS_WAIT, turns staging off for the block and falls back to the
// quad pool.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "r3d_internal.h"

namespace r3d {

constexpr uint32_t kStageThreads = 64;
constexpr uint32_t kWaitLimit = 1u << 20;  // try_wait polls before giving up (well under a second)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Polls the barrier's phase `parity` at most kWaitLimit times; true once
// that phase has completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One box of the slot pool into shared memory: x is a multiple of 16 texels
// (16 bytes), z counts planes over all slots (slot * 128 + z).
__device__ __forceinline__ void tma_load_box(uint8_t *dst, const CUtensorMap *tm, int x, int y,
                                             int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Where the ray's next step samples (slot, base texel), read-only, when the
// step's brick is the cached one; false otherwise (ended, a page walk or an
// absent brick).  The staging decision only; the step itself decides
// everything again.
template <int MODE>
__device__ __forceinline__ bool peek_fetch(const DevScene &s, const ViewConst &vc,
                                           const RayState &st, uint32_t &slot, SlotCoord &q) {
  constexpr uint32_t budget = MODE == R3D_MODE_FULL ? 192u : 256u;
  if (!(st.t < st.tf_ && st.steps < budget)) return false;
  const float t = st.t;
  int desired = st.lc.desired;
  if (vc.lod_on) {
    if (!(t >= st.lod_tlo && t < st.lod_thi)) {
      const float lod = clamp_(r3d_log2f(lod_y(vc, t)) + vc.lod_bias, 0.0f, vc.max_lod);
      desired = (int)clamp_(floorf(lod), 0.0f, (float)((int)s.br.nlev - 1));
    }
  } else {
    desired = 0;
  }
  const float3 p = make_float3(fmaf(t, st.dir.x, st.ro.x), fmaf(t, st.dir.y, st.ro.y),
                               fmaf(t, st.dir.z, st.ro.z));
  BrickCtx b;
  if (!lod_cache_hit(s, p, desired, st.lc, b) || !b.ok) return false;
  slot = b.slot;
  q = slot_coord(b.bl);
  return true;
}

template <int MODE, bool FAST>
__global__ void __launch_bounds__(kStageThreads, 16)
    k_raycast_staged(const __grid_constant__ r3d_frame_params pc,
                     const __grid_constant__ DevScene s, const uchar4 *__restrict__ lut,
                     uchar4 *__restrict__ img, uint32_t out_w,
                     unsigned long long *__restrict__ total,
                     const __grid_constant__ CUtensorMap tm) {
  __shared__ float4 tf[256];
  __shared__ __align__(128) uint8_t box[kBoxBytes];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int sh_slot, sh_bx, sh_by, sh_bz, sh_on, sh_pick;
  const uint32_t tid = threadIdx.x;
  for (uint32_t i = tid; i < 256u; i += kStageThreads) {
    const uchar4 u = lut[i];
    tf[i] = make_float4((float)u.x, (float)u.y, (float)u.z, (float)u.w);
  }
  if (tid == 0) {
    mbar_init(&bar, 1u);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    sh_slot = -1;
    sh_bx = sh_by = sh_bz = 0;
    sh_on = 1;
  }
  __syncthreads();
  // an 8x8 Morton tile: warp w takes rows 4w..4w+3, lanes in Morton order
  const uint32_t lane = tid & 31u, warp = tid >> 5;
  const uint32_t tx = blockIdx.x * 8u + ((lane & 1u) | ((lane >> 1) & 2u) | ((lane >> 2) & 4u));
  const uint32_t ty = blockIdx.y * 8u + warp * 4u + (((lane >> 1) & 1u) | ((lane >> 2) & 2u));
  const bool half = (pc.view_flags & R3D_VIEW_HALF) != 0u;
  const uint32_t px = half ? tx * 2u : tx, py = half ? ty * 2u : ty;
  const uint32_t vw = pc.viewport[0], vh = pc.viewport[1];
  const bool inside = px < vw && py < vh;
  const ViewConst vc = view_const<PATH_LOD_BRICKS>(pc, s);
  RayResult r;
  RayState st;
  Pending pend;
  ShadeBuf sbuf;
  sbuf.n = 0;
  constexpr bool kLater = MODE == R3D_MODE_FULL && R3D_SHADE_LATER;
  bool active = inside && ray_begin<PATH_LOD_BRICKS, MODE>(pc, s, vc, px, py, st, r);
  const bool marched = active;
  uint32_t phase = 0;
  bool waited_out = false;
  while (__syncthreads_or(active)) {
    // the block's next samples against the staged box
    uint32_t rslot = 0;
    SlotCoord rq;
    const bool req = active && sh_on && peek_fetch<MODE>(s, vc, st, rslot, rq);
    const StageBox cur = {box, sh_slot, sh_bx, sh_by, sh_bz};
    const bool in = req && box_has(cur, rslot, rq);
    const int nreq = __syncthreads_count(req);
    const int nin = __syncthreads_count(in);
    if (nreq > 0 && 2 * nin <= nreq) {  // uniform: every thread sees the same counts
      if (tid == 0) sh_pick = (int)kStageThreads;
      __syncthreads();
      if (req && !in) atomicMin(&sh_pick, (int)tid);
      __syncthreads();
      if ((int)tid == sh_pick) {  // a box around this ray's sample, x on 16 texels
        sh_slot = (int)rslot;
        sh_bx = min(max((int)rq.x0 - 8, 0), 96) & ~15;
        sh_by = min(max((int)rq.y0 - 8, 0), 111);
        sh_bz = min(max((int)rq.z0 - 8, 0), 111);
      }
      __syncthreads();
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(&bar, kBoxBytes);
        tma_load_box(box, &tm, sh_bx, sh_by, sh_slot * 128 + sh_bz, &bar);
      }
      const bool ok = mbar_wait(&bar, phase);
      phase ^= 1u;
      if (!ok) {  // stop staging; nothing reads the box again
        waited_out = true;
        sh_on = 0;
        sh_slot = -1;
        if (tid == 0) atomicOr(s.status, R3D_STATUS_WAIT);
      }
      __syncthreads();
    }
    if (active) {
      const StageBox sb = {box, sh_slot, sh_bx, sh_by, sh_bz};
      if (ray_step<PATH_LOD_BRICKS, MODE, FAST, false, false, false, kLater, true>(
              s, vc, tf, st, pend, &sbuf, &sb) == kStepDone)
        active = false;
    }
  }
  if (marched) {
    if (kLater) shade_flush<PATH_LOD_BRICKS, MODE, FAST, false>(s, vc, tf, st, sbuf);
    ray_end<MODE>(vc, st, r);
  }
  uint32_t my_steps = 0;
  if (inside) {
    const uchar4 col = make_uchar4(unorm8(r.rgb[0]), unorm8(r.rgb[1]), unorm8(r.rgb[2]), 255);
    const uint32_t ox = pc.view_org & 0xffffu, oy = pc.view_org >> 16;
    const uint32_t n = half ? 4u : 1u;
    for (uint32_t k = 0; k < n; k++) {
      const uint32_t ax = px + (k & 1u), ay = py + (k >> 1);
      if (ax >= vw || ay >= vh) continue;
      img[(size_t)(oy + ay) * out_w + (ox + ax)] = col;
    }
    my_steps = r.steps;
  }
  if (total) {
    uint32_t sum = my_steps;
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0 && sum) atomicAdd(total, (unsigned long long)sum);
  }
  // a copy that outlived its wait must land before the block's shared
  // memory goes away: one more bounded wait on the same phase
  if (waited_out) mbar_wait(&bar, phase ^ 1u);
}

// The CUDA driver API's tensor-map encoder, looked up once through the runtime.
static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    else
      cudaGetLastError();
  }
  return fn;
}

bool staged_supported(const r3d_cuda_ctx *c, const r3d_frame_params &pc) {
  return c->have_bricks && c->pool && c->nslots && path_of_view(pc) == PATH_LOD_BRICKS &&
         !(pc.overlay_flags & kOvlAtlases) &&
         (pc.mode == R3D_MODE_FULL || pc.mode == R3D_MODE_MIP);
}

cudaError_t launch_staged(const r3d_cuda_ctx *c, const r3d_frame_params &pc, uint8_t *img,
                          uint32_t out_w, unsigned long long *total, cudaStream_t st) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encoder();
  if (!enc) return cudaErrorNotSupported;
  // the u8 slot pool as a 128 x 128 x (128 * nslots) tensor, x fastest;
  // boxes of 32 x 17 x 17 texels (32-byte rows: a multiple of 16 bytes)
  CUtensorMap tm;
  const cuuint64_t dims[3] = {128u, 128u, 128ull * c->nslots};
  const cuuint64_t strides[2] = {128u, 128u * 128u};
  const cuuint32_t boxd[3] = {kBoxX, kBoxY, kBoxZ};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void *)c->pool, dims, strides, boxd, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  const bool half = (pc.view_flags & R3D_VIEW_HALF) != 0u;
  const uint32_t gw = half ? (pc.viewport[0] + 1u) / 2u : pc.viewport[0];
  const uint32_t gh = half ? (pc.viewport[1] + 1u) / 2u : pc.viewport[1];
  const dim3 grid((gw + 7u) / 8u, (gh + 7u) / 8u);
  DevScene s = c->scene();
  s.el = elide_counts(pc, s.tf_zero_t);
  const bool fast = c->quality == R3D_QUALITY_FAST;
  if (pc.mode == R3D_MODE_MIP)
    k_raycast_staged<R3D_MODE_MIP, false><<<grid, kStageThreads, 0, st>>>(
        pc, s, c->lut, (uchar4 *)img, out_w, total, tm);
  else if (fast)
    k_raycast_staged<R3D_MODE_FULL, true><<<grid, kStageThreads, 0, st>>>(
        pc, s, c->lut, (uchar4 *)img, out_w, total, tm);
  else
    k_raycast_staged<R3D_MODE_FULL, false><<<grid, kStageThreads, 0, st>>>(
        pc, s, c->lut, (uchar4 *)img, out_w, total, tm);
  return cudaGetLastError();
}

}  // namespace r3d
