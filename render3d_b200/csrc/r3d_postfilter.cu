// Post-decode 3D display filter over 128^3 brick slots (reference
// src/shaders/postfilt.comp, src/vk/vkbackend.c:3396-3466,4863-4906): a
// brick is filtered once when it lands in a slot, so every view sees the
// filtered volume.  Filters, each over the voxel's neighbourhood clamped to
// its slot:
//   median of 3^3 (the 14th smallest of 27 bytes), median of 5^3 (the 63rd
//   of 125), max of 3^3, max of 5^3, and unsharp: centre + amount *
//   (centre - mean of 3^3), clamped to [0, 1], with the mean summed in the
//   shader's order (z, then y, then x) over byte / 255 floats.
// Mode word (r3d_bricks_postfilter): low byte 1 median 3^3, 2 median 5^3,
// 3 max 3^3, 4 max 5^3 (other values: none); bit 8 adds the unsharp pass
// after it.
//
// Kernel shape: one CTA per 32 x 8 x 8 output tile of one slot, its halo
// staged in shared memory with the slot clamp applied at load.  A thread
// owns one x column of the tile and walks z.  The neighbourhood's rows are
// gathered from shared memory as packed bytes (two aligned words and a
// funnel shift per row), so the medians are exact rank selections done
// four bytes at a time: eight rounds of a bit-serial search, each counting
// the bytes below a candidate with __vsetltu4.  Max pools are separable
// (k_maxpool).  Results are bit-identical to the shader's sort / histogram
// formulation for bytes, which the oracle restates directly.
#include <string.h>

#include "r3d_internal.h"

namespace r3d {

constexpr uint32_t kSlot = 128u, kSlotBytes = kSlot * kSlot * kSlot;
constexpr uint32_t kPfWave = 64u;            // slots per launch (scratch of 128 MiB)
constexpr int kTX = 32, kTY = 8, kTZ = 8;    // output tile
constexpr int kRowWords = 10;                // a halo row: slot x0 - 4 .. x0 + 35
constexpr int kRowBytes = 4 * kRowWords;

enum PfOp { kMedian = 0, kSharpen = 1 };

struct PfLayout {
  uint32_t abpa;  // 0: a linear pool; else an atlas of abpa^3 slots
};

struct PfJobs {
  uint32_t src[kPfWave], dst[kPfWave];  // slot index of each job (in src / dst buffers)
  PfLayout src_l, dst_l;
};

// Texel (x, y, z) of slot s: a linear pool (abpa 0: slot s at s * 128^3, x
// fastest) or a single-level atlas of abpa^3 slots ((abpa * 128)^3 texels,
// slot s at (s mod abpa, s / abpa mod abpa, s / abpa^2) * 128).
__device__ __forceinline__ size_t slot_texel(const PfLayout &l, uint32_t s, uint32_t x, uint32_t y,
                                             uint32_t z) {
  if (!l.abpa) return (size_t)s * kSlotBytes + ((size_t)z * kSlot + y) * kSlot + x;
  const size_t a = (size_t)l.abpa * kSlot;
  const size_t sx = (s % l.abpa) * kSlot, sy = ((s / l.abpa) % l.abpa) * kSlot,
               sz = (s / (l.abpa * l.abpa)) * kSlot;
  return ((sz + z) * a + sy + y) * a + sx + x;
}

// Stages the tile's halo rows (z0 - R .. z0 + 8 + R, y likewise) as aligned
// words of slot x x0 - 4 .. x0 + 35, the slot clamp applied: clamped y and
// z rows, and at the x edges the edge byte repeated through the word
// outside the slot.  Output x of the tile sits at row byte x + 4.
template <int R>
__device__ __forceinline__ void load_tile(uint8_t (*t)[kTY + 2 * R][kRowBytes], const uint8_t *src,
                                          const PfLayout &l, uint32_t slot, uint32_t x0, uint32_t y0,
                                          uint32_t z0) {
  constexpr int TY = kTY + 2 * R, TZ = kTZ + 2 * R, kWords = TZ * TY * kRowWords;
  constexpr int kIters = (kWords + 255) / 256;  // blocks of 256 threads
  uint32_t w[kIters];
  // every load in flight before the first shared store
#pragma unroll
  for (int it = 0; it < kIters; it++) {
    const uint32_t i = threadIdx.x + 256u * it;
    if (i >= (uint32_t)kWords) break;
    const uint32_t row = i / kRowWords, wi = i % kRowWords;
    const int ly = (int)(row % TY), lz = (int)(row / TY);
    const int gy = min(max((int)y0 + ly - R, 0), 127), gz = min(max((int)z0 + lz - R, 0), 127);
    const int gw = (int)(x0 >> 2) - 1 + (int)wi;  // -1 .. 32
    const uint32_t *g = reinterpret_cast<const uint32_t *>(src + slot_texel(l, slot, 0, gy, gz));
    w[it] = __ldg(g + min(max(gw, 0), 31));
  }
#pragma unroll
  for (int it = 0; it < kIters; it++) {
    const uint32_t i = threadIdx.x + 256u * it;
    if (i >= (uint32_t)kWords) break;
    const uint32_t row = i / kRowWords, wi = i % kRowWords;
    const int gw = (int)(x0 >> 2) - 1 + (int)wi;
    uint32_t v = w[it];
    if (gw < 0) v = (v & 0xFFu) * 0x01010101u;
    if (gw > 31) v = (v >> 24) * 0x01010101u;
    reinterpret_cast<uint32_t *>(&t[row / TY][row % TY][0])[wi] = v;
  }
}

// the rank-th smallest byte (0-based) of the bytes packed in w (pad bytes
// 0xFF are never counted below a candidate)
template <int NW>
__device__ __forceinline__ uint32_t rank_select(const uint32_t (&w)[NW], uint32_t rank) {
  uint32_t res = 0;
#pragma unroll
  for (int bit = 7; bit >= 0; bit--) {
    const uint32_t cand = res | (1u << bit), cb = cand * 0x01010101u;
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < NW; i++) acc += __vsetltu4(w[i], cb);  // per byte: 1 if below
    if (((acc * 0x01010101u) >> 24) <= rank) res = cand;    // bytes summed (< 256)
  }
  return res;
}

template <int R, int OP>
__global__ void __launch_bounds__(256) k_postfilter(const uint8_t *__restrict__ src,
                                                    uint8_t *__restrict__ dst,
                                                    const __grid_constant__ PfJobs jobs,
                                                    float amount) {
  constexpr int TY = kTY + 2 * R, TZ = kTZ + 2 * R;
  __shared__ __align__(16) uint8_t t[TZ][TY][kRowBytes];
  __shared__ float lut[256];
  const uint32_t tid = threadIdx.x, j = blockIdx.y;
  const uint32_t x0 = (blockIdx.x & 3u) * kTX, y0 = ((blockIdx.x >> 2) & 15u) * kTY,
                 z0 = (blockIdx.x >> 6) * kTZ;
  load_tile<R>(t, src, jobs.src_l, jobs.src[j], x0, y0, z0);
  if (OP == kSharpen) lut[tid] = (float)tid / 255.0f;  // texelFetch of an R8 texel
  __syncthreads();
  const uint32_t x = tid & 31u, y = tid >> 5;
  uint8_t *d = dst + slot_texel(jobs.dst_l, jobs.dst[j], x0 + x, y0 + y, z0);
  const size_t zstride = jobs.dst_l.abpa ? (size_t)jobs.dst_l.abpa * kSlot * jobs.dst_l.abpa * kSlot
                                         : (size_t)kSlot * kSlot;
  // the window of output x starts at row byte x + 4 - R
  const uint32_t xb = x + 4u - (uint32_t)R, xa = xb & ~3u, sh = 8u * (xb & 3u);
#pragma unroll 1
  for (int z = 0; z < kTZ; z++) {
    uint32_t out;
    if (OP == kSharpen) {
      float sum = 0.0f;
      for (int dz = 0; dz < 3; dz++)
        for (int dy = 0; dy < 3; dy++)
          for (int dx = 0; dx < 3; dx++) sum += lut[t[z + dz][y + dy][xb + dx]];
      const float center = lut[t[z + 1][y + 1][xb + 1]];
      const float v = fminf(fmaxf(center + amount * (center - sum / 27.0f), 0.0f), 1.0f);
      out = (uint32_t)(int)fmaf(v, 255.0f, 0.5f);
    } else if (R == 1) {
      // 9 rows of 3 bytes, one word each (fourth byte: a pad)
      uint32_t w[9];
#pragma unroll
      for (int r = 0; r < 9; r++) {
        const uint32_t *row = reinterpret_cast<const uint32_t *>(&t[z + r / 3][y + r % 3][xa]);
        const uint32_t a = __funnelshift_r(row[0], row[1], sh);
        w[r] = a | 0xFF000000u;
      }
      out = rank_select<9>(w, 13u);
    } else {
      // 25 rows of 5 bytes: the first four of each row in one word, the
      // fifth bytes packed four to a word (7 words, 3 pad bytes)
      uint32_t w[32];
#pragma unroll
      for (int r = 0; r < 25; r++) {
        const uint32_t *row = reinterpret_cast<const uint32_t *>(&t[z + r / 5][y + r % 5][xa]);
        const uint32_t r0 = row[0], r1 = row[1];
        w[r] = __funnelshift_r(r0, r1, sh);
        const uint32_t fifth = (r1 >> sh) & 0xFFu;
        if (r % 4 == 0)
          w[25 + r / 4] = fifth | 0xFFFFFF00u;
        else
          w[25 + r / 4] = (w[25 + r / 4] & ~(0xFFu << (8 * (r % 4)))) | (fifth << (8 * (r % 4)));
      }
      out = rank_select<32>(w, 62u);
    }
    d[(size_t)z * zstride] = (uint8_t)out;
  }
}

// Max pools, separable: the window is a box and the slot clamp acts per
// axis, so the max of the box is the max over z of the max over y of the
// max over x.  Three passes through shared memory, four bytes a word: x
// (halo rows -> 32-wide rows), y, then z straight to the slot.
template <int R>
__global__ void __launch_bounds__(256) k_maxpool(const uint8_t *__restrict__ src,
                                                 uint8_t *__restrict__ dst,
                                                 const __grid_constant__ PfJobs jobs, float) {
  constexpr int TY = kTY + 2 * R, TZ = kTZ + 2 * R;
  __shared__ __align__(16) uint8_t t[TZ][TY][kRowBytes];
  __shared__ __align__(16) uint32_t mx[TZ][TY][kTX / 4];  // max over x
  __shared__ __align__(16) uint32_t my[TZ][kTY][kTX / 4];  // then over y
  const uint32_t tid = threadIdx.x, j = blockIdx.y;
  const uint32_t x0 = (blockIdx.x & 3u) * kTX, y0 = ((blockIdx.x >> 2) & 15u) * kTY,
                 z0 = (blockIdx.x >> 6) * kTZ;
  load_tile<R>(t, src, jobs.src_l, jobs.src[j], x0, y0, z0);
  __syncthreads();
  // x: the 4 outputs of word g sit in row word g + 1; their windows reach R
  // bytes into words g and g + 2
  for (uint32_t i = tid; i < (uint32_t)(TZ * TY * (kTX / 4)); i += 256u) {
    const uint32_t g = i % (kTX / 4), ly = (i / (kTX / 4)) % TY, lz = i / ((kTX / 4) * TY);
    const uint32_t *row = reinterpret_cast<const uint32_t *>(&t[lz][ly][0]);
    const uint32_t w0 = row[g], w1 = row[g + 1], w2 = row[g + 2];
    uint32_t m = w1;
#pragma unroll
    for (int k = 1; k <= R; k++)
      m = __vmaxu4(m, __vmaxu4(__funnelshift_r(w0, w1, 32 - 8 * k), __funnelshift_r(w1, w2, 8 * k)));
    mx[lz][ly][g] = m;
  }
  __syncthreads();
  for (uint32_t i = tid; i < (uint32_t)(TZ * kTY * (kTX / 4)); i += 256u) {
    const uint32_t g = i % (kTX / 4), y = (i / (kTX / 4)) % kTY, lz = i / ((kTX / 4) * kTY);
    uint32_t m = mx[lz][y][g];
#pragma unroll
    for (int k = 1; k <= 2 * R; k++) m = __vmaxu4(m, mx[lz][y + k][g]);
    my[lz][y][g] = m;
  }
  __syncthreads();
  for (uint32_t i = tid; i < (uint32_t)(kTZ * kTY * (kTX / 4)); i += 256u) {
    const uint32_t g = i % (kTX / 4), y = (i / (kTX / 4)) % kTY, z = i / ((kTX / 4) * kTY);
    uint32_t m = my[z][y][g];
#pragma unroll
    for (int k = 1; k <= 2 * R; k++) m = __vmaxu4(m, my[z + k][y][g]);
    *reinterpret_cast<uint32_t *>(dst + slot_texel(jobs.dst_l, jobs.dst[j], x0 + 4u * g, y0 + y, z0 + z)) = m;
  }
}

using PfKernel = void (*)(const uint8_t *, uint8_t *, const PfJobs, float);

// Slot copies between layouts, 16 bytes a thread (one CTA per 128 x 8 x 8
// block of a slot).
__global__ void __launch_bounds__(256) k_slot_copy(const uint8_t *__restrict__ src,
                                                   uint8_t *__restrict__ dst,
                                                   const __grid_constant__ PfJobs jobs) {
  const uint32_t j = blockIdx.y, tid = threadIdx.x;
  const uint32_t y0 = (blockIdx.x & 15u) * 8u, z0 = (blockIdx.x >> 4) * 8u;
#pragma unroll
  for (int it = 0; it < 2; it++) {
    const uint32_t i = tid + 256u * it;  // 512 chunks of 16 bytes: 8 per row, 8 x 8 rows
    const uint32_t x = (i & 7u) * 16u, y = y0 + ((i >> 3) & 7u), z = z0 + (i >> 6);
    *reinterpret_cast<uint4 *>(dst + slot_texel(jobs.dst_l, jobs.dst[j], x, y, z)) =
        *reinterpret_cast<const uint4 *>(src + slot_texel(jobs.src_l, jobs.src[j], x, y, z));
  }
}


// the kernel of a primary filter id (1 median 3^3, 2 median 5^3, 3 max 3^3,
// 4 max 5^3), or null
static PfKernel primary_kernel(uint32_t prim) {
  switch (prim) {
    case 1: return k_postfilter<1, kMedian>;
    case 2: return k_postfilter<2, kMedian>;
    case 3: return k_maxpool<1>;
    case 4: return k_maxpool<2>;
    default: return nullptr;
  }
}

}  // namespace r3d

using namespace r3d;

void postfilter_reset(r3d_cuda_ctx *c) {
  cudaFree(c->pf_scratch);
  c->pf_scratch = nullptr;
}

bool postfilter_on(const r3d_cuda_ctx *c, uint32_t target) {
  if (!((c->pf_targets >> target) & 1u)) return false;
  return primary_kernel(c->pf_mode & 0xFFu) != nullptr || (c->pf_mode & 0x100u);
}

int postfilter_slots(r3d_cuda_ctx *c, uint32_t target, uint8_t *pool, const uint32_t *slots,
                     uint32_t n, uint32_t atlas_bpa) {
  if (!n || !postfilter_on(c, target)) return R3D_OK;
  const PfKernel prim = primary_kernel(c->pf_mode & 0xFFu);
  const bool sharpen = (c->pf_mode & 0x100u) != 0;
  if (!c->pf_scratch) R3D_CUDA_TRY(c, cudaMalloc(&c->pf_scratch, (size_t)kPfWave * kSlotBytes));
  cudaStream_t st = c->stream;
  const dim3 grid(4u * 16u * 16u, 1u);
  for (uint32_t w0 = 0; w0 < n; w0 += kPfWave) {
    const uint32_t wn = min(n - w0, kPfWave);
    PfJobs to_scratch, back;
    to_scratch.src_l = back.dst_l = PfLayout{atlas_bpa};
    to_scratch.dst_l = back.src_l = PfLayout{0u};
    for (uint32_t i = 0; i < wn; i++) {
      to_scratch.src[i] = back.dst[i] = slots[w0 + i];
      to_scratch.dst[i] = back.src[i] = i;
    }
    const dim3 g(grid.x, wn);
    // median / max first, so that the sharpen sees despeckled data
    // (vkbackend.c:3398-3418); two passes end back in the slots, one pass
    // is copied back
    if (prim) prim<<<g, 256, 0, st>>>(pool, c->pf_scratch, to_scratch, c->pf_amount);
    if (sharpen)
      k_postfilter<1, kSharpen><<<g, 256, 0, st>>>(prim ? c->pf_scratch : pool,
                                                   prim ? pool : c->pf_scratch,
                                                   prim ? back : to_scratch, c->pf_amount);
    R3D_CUDA_TRY(c, cudaGetLastError());
    if (!(prim && sharpen)) k_slot_copy<<<dim3(16u * 16u, wn), 256, 0, st>>>(c->pf_scratch, pool, back);
    R3D_CUDA_TRY(c, cudaGetLastError());
  }
  return R3D_OK;
}

extern "C" {

int r3d_cuda_bricks_postfilter(r3d_cuda_ctx *c, uint32_t mode, float amount, uint32_t targets) {
  if (!c) return R3D_E_INVALID;
  if (!(amount == amount)) return fail(c, R3D_E_INVALID, "bricks_postfilter: amount is NaN");
  c->pf_mode = mode;
  c->pf_amount = amount;
  c->pf_targets = targets ? targets : 1u;  // 0: the CT volume
  return R3D_OK;
}

}  // extern "C"
