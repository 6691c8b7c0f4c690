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
// the bytes below a candidate with __vsetltu4.  Max pools fold the same
// words with __vmaxu4.  Results are bit-identical to the shader's sort /
// histogram formulation for bytes, which the oracle restates directly.
#include <string.h>

#include "r3d_internal.h"

namespace r3d {

constexpr uint32_t kSlot = 128u, kSlotBytes = kSlot * kSlot * kSlot;
constexpr uint32_t kPfWave = 64u;            // slots per launch (scratch of 128 MiB)
constexpr int kTX = 32, kTY = 8, kTZ = 8;    // output tile
constexpr int kRowBytes = 36;                // 32 + 2 * 2 halo, a multiple of 4

enum PfOp { kMedian = 0, kMax = 1, kSharpen = 2 };

struct PfJobs {
  uint32_t src[kPfWave], dst[kPfWave];  // slot index of each job (in src / dst buffers)
};

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

template <int NW>
__device__ __forceinline__ uint32_t max_bytes(const uint32_t (&w)[NW]) {
  uint32_t m = w[0];
#pragma unroll
  for (int i = 1; i < NW; i++) m = __vmaxu4(m, w[i]);
  m = __vmaxu4(m, m >> 16);
  m = __vmaxu4(m, m >> 8);
  return m & 0xFFu;
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
  const uint8_t *s = src + (size_t)jobs.src[j] * kSlotBytes;
  // halo rows, the slot clamp applied here (columns past the 32 + 2R used
  // ones are clamped copies too, so every byte read below is initialized)
  for (uint32_t i = tid; i < (uint32_t)(TZ * TY * kRowBytes); i += 256u) {
    const int lx = (int)(i % kRowBytes), ly = (int)((i / kRowBytes) % TY), lz = (int)(i / (kRowBytes * TY));
    const int gx = min(max((int)x0 + lx - R, 0), 127), gy = min(max((int)y0 + ly - R, 0), 127),
              gz = min(max((int)z0 + lz - R, 0), 127);
    t[lz][ly][lx] = __ldg(s + ((size_t)gz * kSlot + gy) * kSlot + gx);
  }
  if (OP == kSharpen) lut[tid] = (float)tid / 255.0f;  // texelFetch of an R8 texel
  __syncthreads();
  const uint32_t x = tid & 31u, y = tid >> 5;
  uint8_t *d = dst + (size_t)jobs.dst[j] * kSlotBytes + ((size_t)z0 * kSlot + y0 + y) * kSlot + x0 + x;
  const uint32_t xa = x & ~3u, sh = 8u * (x & 3u);
#pragma unroll 1
  for (int z = 0; z < kTZ; z++) {
    uint32_t out;
    if (OP == kSharpen) {
      float sum = 0.0f;
      for (int dz = 0; dz < 3; dz++)
        for (int dy = 0; dy < 3; dy++)
          for (int dx = 0; dx < 3; dx++) sum += lut[t[z + dz][y + dy][x + dx]];
      const float center = lut[t[z + 1][y + 1][x + 1]];
      const float v = fminf(fmaxf(center + amount * (center - sum / 27.0f), 0.0f), 1.0f);
      out = (uint32_t)(int)fmaf(v, 255.0f, 0.5f);
    } else if (R == 1) {
      // 9 rows of 3 bytes, one word each (fourth byte: a pad)
      uint32_t w[9];
#pragma unroll
      for (int r = 0; r < 9; r++) {
        const uint32_t *row = reinterpret_cast<const uint32_t *>(&t[z + r / 3][y + r % 3][xa]);
        const uint32_t a = __funnelshift_r(row[0], row[1], sh);
        w[r] = OP == kMedian ? (a | 0xFF000000u) : (a & 0x00FFFFFFu);
      }
      out = OP == kMedian ? rank_select<9>(w, 13u) : max_bytes<9>(w);
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
          w[25 + r / 4] = fifth | (OP == kMedian ? 0xFFFFFF00u : 0u);
        else
          w[25 + r / 4] = (w[25 + r / 4] & ~(0xFFu << (8 * (r % 4)))) | (fifth << (8 * (r % 4)));
      }
      out = OP == kMedian ? rank_select<32>(w, 62u) : max_bytes<32>(w);
    }
    d[(size_t)z * kSlot * kSlot] = (uint8_t)out;
  }
}

using PfKernel = void (*)(const uint8_t *, uint8_t *, const PfJobs, float);

// the kernel of a primary filter id (1 median 3^3, 2 median 5^3, 3 max 3^3,
// 4 max 5^3), or null
static PfKernel primary_kernel(uint32_t prim) {
  switch (prim) {
    case 1: return k_postfilter<1, kMedian>;
    case 2: return k_postfilter<2, kMedian>;
    case 3: return k_postfilter<1, kMax>;
    case 4: return k_postfilter<2, kMax>;
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
                     uint32_t n) {
  if (!n || !postfilter_on(c, target)) return R3D_OK;
  const PfKernel prim = primary_kernel(c->pf_mode & 0xFFu);
  const bool sharpen = (c->pf_mode & 0x100u) != 0;
  if (!c->pf_scratch) R3D_CUDA_TRY(c, cudaMalloc(&c->pf_scratch, (size_t)kPfWave * kSlotBytes));
  cudaStream_t st = c->stream;
  const dim3 grid(4u * 16u * 16u, 1u);
  for (uint32_t w0 = 0; w0 < n; w0 += kPfWave) {
    const uint32_t wn = min(n - w0, kPfWave);
    PfJobs to_scratch, back;
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
    if (!(prim && sharpen))
      for (uint32_t i = 0; i < wn; i++)
        R3D_CUDA_TRY(c, cudaMemcpyAsync(pool + (size_t)slots[w0 + i] * kSlotBytes,
                                        c->pf_scratch + (size_t)i * kSlotBytes, kSlotBytes,
                                        cudaMemcpyDeviceToDevice, st));
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
