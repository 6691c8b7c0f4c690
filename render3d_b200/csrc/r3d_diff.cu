// Differentiable emission-absorption raycast: forward and adjoint.
//
// The render is render3d's compositing without shading (FLAT mode,
// src/shaders/raycast.slang:894-1017) over an FP32 density grid and an FP32
// 256x4 transfer function: ray setup of the cube path, trilinear density at
// texel centres (level 0, clamp to edge, no empty-space skip), TF lookup at
// v*256-0.5, alpha clamped to [0, 1], opacity correction
// a = 1 - (1 - alpha)^(density * step * lod_step), samples with a <= 0.003
// ignored, front-to-back compositing with termination at the cutoff, then
// the background.  The forward kernel writes an FP32 RGB image per view;
// its arithmetic equals the CPU oracle's bit for bit.  A sample whose
// density falls in the TF's leading run of zero-alpha texels (both texels
// alpha 0) has opacity exactly 0; it is skipped before the TF lookup.
//
// The adjoint kernel (one thread per ray) returns the gradients of
// L = sum(dL/drgb * rgb) with respect to every voxel, every LUT entry and the
// density scale.  It first marches the ray forward, keeping a checkpoint
// (position and accumulated opacity) every K samples in local memory, the
// number of contributing samples of each K-sample segment, and the last 64
// contributing samples.  It then walks the segments with contributions from
// last to first: a segment whose samples are still among the remembered ones
// uses them, any other is recomputed from its checkpoint; the samples are
// visited in reverse with the colour behind them S (S <- a c + (1 - a) S,
// starting from the background).  Transmittance is never divided out, which
// would be unstable as alpha approaches 1.
//
// Gradients: voxel contributions are summed per trilinear cell in registers
// while consecutive samples stay in one cell, then flushed with global
// atomics; LUT contributions go to a per-block shared-memory table flushed
// once per block; the density-scale gradient is reduced per warp.  Atomic
// mode adds FP32 (order-dependent rounding).  Deterministic mode adds
// fixed-point integers (value * 2^32, rounded, in int64; mod 2^64 as two
// 32-bit words in the shared table): integer addition is associative, so
// the result is identical for any execution order.
#include <string.h>

#include "r3d_internal.h"

namespace r3d {

constexpr double kFix = 4294967296.0;  // 2^32, deterministic fixed point

struct DiffView {
  r3d_frame_params pc;
  unsigned long long out_off;  // first float of the view's RGB image
  uint32_t pad[2];
};

struct DiffGrid {
  const float *dens;
  // per voxel (x, y, z): the densities at (x, y), (x1, y), (x, y1), (x1, y1)
  // of its z plane, x1 = min(x + 1, nx - 1) and y1 likewise, so that a
  // trilinear sample reads two float4 instead of eight floats
  const float4 *quad;
  const uint32_t *zc;  // the TF's first texel with alpha not 0 (256: none)
  uint32_t n[3];
  uint32_t nmax;
  const float *lut;  // 256 x 4
  float cutoff;
};

struct DiffRay {
  float ro[3], dir[3];
  float t0, tf, dt, span;
  bool hit;
};

// ray setup of the cube path (raycast.slang:640-748)
__device__ __forceinline__ void diff_setup(const r3d_frame_params &pc, const DiffGrid &g,
                                           uint32_t px, uint32_t py, DiffRay &r) {
  const bool ortho = (pc.view_flags & R3D_VIEW_ORTHO) != 0u;
  float ux = ((float)px + 0.5f) / (float)pc.viewport[0];
  float uy = ((float)py + 0.5f) / (float)pc.viewport[1];
  float nx = ux * 2.0f - 1.0f, ny = 1.0f - uy * 2.0f;
  float3 fw = make_float3(pc.cam_forward[0], pc.cam_forward[1], pc.cam_forward[2]);
  float3 rt = make_float3(pc.cam_right[0], pc.cam_right[1], pc.cam_right[2]);
  float3 up = make_float3(pc.cam_up[0], pc.cam_up[1], pc.cam_up[2]);
  float3 d = ortho ? fw
                   : make_float3(fmaf(ny, up.x, fmaf(nx, rt.x, fw.x)),
                                 fmaf(ny, up.y, fmaf(nx, rt.y, fw.y)),
                                 fmaf(ny, up.z, fmaf(nx, rt.z, fw.z)));
  d = norm3(d);
  float3 o = make_float3(pc.cam_origin[0], pc.cam_origin[1], pc.cam_origin[2]);
  if (ortho)
    o = make_float3(fmaf(ny, up.x, fmaf(nx, rt.x, o.x)), fmaf(ny, up.y, fmaf(nx, rt.y, o.y)),
                    fmaf(ny, up.z, fmaf(nx, rt.z, o.z)));
  const float c = 0.5f;
  float q[3] = {(o.x - pc.vol_tx) - c, (o.y - pc.vol_ty) - c, (o.z - pc.vol_tz) - c};
  float dv[3] = {d.x, d.y, d.z};
  const float *r0 = pc.vol_r0, *r1 = pc.vol_r1, *r2 = pc.vol_r2;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    r.ro[a] = fmaf(r2[a], q[2], fmaf(r1[a], q[1], r0[a] * q[0])) + c;
    r.dir[a] = fmaf(r2[a], dv[2], fmaf(r1[a], dv[1], r0[a] * dv[0]));
  }
  float tmn[3], tmx[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float iv = 1.0f / r.dir[a];
    float t0 = (0.0f - r.ro[a]) * iv, t1 = (1.0f - r.ro[a]) * iv;
    tmn[a] = fminf(t0, t1);
    tmx[a] = fmaxf(t0, t1);
  }
  float tn = fmaxf(fmaxf(fmaxf(tmn[0], tmn[1]), tmn[2]), 0.0f);
  float tf = fminf(fminf(fminf(tmx[0], tmx[1]), tmx[2]), 1e30f);
  r.hit = !(tn >= tf);
  float voxel = 1.0f / (float)g.nmax;
  r.dt = pc.step_voxels * voxel;
  r.t0 = fmaf(hash12(px, py, pc.frame_index), r.dt, tn);
  r.tf = tf;
  r.span = fmaxf((tf - tn) / (4096.0f * r.dt), 1.0f);
}


// One sample: density, TF, opacity.  Fills the trilinear cell for scatters.
struct DiffSample {
  float v, tt, f, s[4], alpha, a;
  uint32_t i0, i1;
  uint32_t base, sx, sy, sz;  // corner (x0,y0,z0) and strides to x1/y1/z1 (0 at edges)
  float fx, fy, fz;
};

// The trilinear cell of the sample at t: corner, strides, fractions.
__device__ __forceinline__ void diff_cell(const DiffGrid &g, const DiffRay &r, float t,
                                          DiffSample &o) {
  float p[3] = {fmaf(t, r.dir[0], r.ro[0]), fmaf(t, r.dir[1], r.ro[1]),
                fmaf(t, r.dir[2], r.ro[2])};
  uint32_t i0[3];
  float fr[3];
  bool up[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float tc = clamp_(fmaf(p[a], (float)g.n[a], -0.5f), 0.0f, (float)(g.n[a] - 1u));
    i0[a] = (uint32_t)tc;
    fr[a] = tc - (float)i0[a];
    up[a] = i0[a] + 1u < g.n[a];
  }
  const uint32_t nx = g.n[0], nxy = g.n[0] * g.n[1];
  o.base = i0[0] + i0[1] * nx + i0[2] * nxy;
  o.sx = up[0] ? 1u : 0u;
  o.sy = up[1] ? nx : 0u;
  o.sz = up[2] ? nxy : 0u;
  o.fx = fr[0];
  o.fy = fr[1];
  o.fz = fr[2];
}

__device__ __forceinline__ void diff_sample(const DiffGrid &g, const DiffRay &r, float t,
                                            DiffSample &o) {
  diff_cell(g, r, t, o);
  const float4 q0 = __ldg(g.quad + o.base), q1 = __ldg(g.quad + o.base + o.sz);
  const float c00 = lerp_(q0.x, q0.y, o.fx), c10 = lerp_(q0.z, q0.w, o.fx);
  const float c01 = lerp_(q1.x, q1.y, o.fx), c11 = lerp_(q1.z, q1.w, o.fx);
  o.v = lerp_(lerp_(c00, c10, o.fy), lerp_(c01, c11, o.fy), o.fz);
}

// TF coordinate, texels and colour of a sample (FP32, as the oracle)
__device__ __forceinline__ void diff_tf_color(const float4 *lut, DiffSample &o) {
  o.tt = clamp_(fmaf(o.v, 256.0f, -0.5f), 0.0f, 255.0f);
  o.i0 = (uint32_t)o.tt;
  o.i1 = min(o.i0 + 1u, 255u);
  o.f = o.tt - (float)o.i0;
  const float4 l0 = lut[o.i0], l1 = lut[o.i1];
  o.s[0] = lerp_(l0.x, l1.x, o.f);
  o.s[1] = lerp_(l0.y, l1.y, o.f);
  o.s[2] = lerp_(l0.z, l1.z, o.f);
  o.s[3] = lerp_(l0.w, l1.w, o.f);
  o.alpha = clamp_(o.s[3], 0.0f, 1.0f);
}

// TF and opacity of a sample
__device__ __forceinline__ void diff_tf(const float4 *lut, float k, DiffSample &o) {
  diff_tf_color(lut, o);
  o.a = 1.0f - r3d_powf(1.0f - o.alpha, k);
}

// True when both TF texels of density v have alpha 0 (z = the first texel
// whose alpha is not 0): then alpha = lerp(0, 0, f) = 0, the opacity is
// 1 - 1^k = 0 and the sample cannot contribute.
__device__ __forceinline__ bool diff_clear(float v, uint32_t z) {
  const uint32_t i0 = (uint32_t)clamp_(fmaf(v, 256.0f, -0.5f), 0.0f, 255.0f);
  return min(i0 + 1u, 255u) < z;
}

// The quad grid of DiffGrid::quad from the density grid.
__global__ void k_diff_quads(const float *__restrict__ d, uint32_t nx, uint32_t ny, uint32_t nz,
                             float4 *__restrict__ q) {
  const size_t n = (size_t)nx * ny * nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i % nx), y = (uint32_t)((i / nx) % ny);
    const size_t dx = x + 1u < nx ? 1u : 0u, dy = y + 1u < ny ? nx : 0u;
    q[i] = make_float4(__ldg(d + i), __ldg(d + i + dx), __ldg(d + i + dy), __ldg(d + i + dy + dx));
  }
}

// DiffGrid::zc from the TF (one block).
__global__ void k_diff_tf_clear(const float *__restrict__ lut, uint32_t *__restrict__ zc) {
  __shared__ uint32_t z;
  if (threadIdx.x == 0) z = 256u;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < 256u; i += blockDim.x)
    if (__ldg(lut + 4u * i + 3u) != 0.0f) atomicMin(&z, i);
  __syncthreads();
  if (threadIdx.x == 0) *zc = z;
}

// Tape of a training forward: per ray, the first kTape contributing samples
// and their count.  An entry holds t, the accumulated opacity before the
// sample, and the sample's density and opacity (x, y, z, w), so that the
// backward needs neither the density fetch nor the opacity's power again.
// A backward over the same views and scene walks these in reverse instead
// of marching the ray again; rays with more contributions take the
// checkpoint path.
constexpr uint32_t kTape = 64;
using TapeEntry = float4;

template <bool TAPE>
__global__ void __launch_bounds__(128) k_diff_fwd(const DiffView *__restrict__ views,
                                                  const __grid_constant__ DiffGrid g,
                                                  float *__restrict__ rgb,
                                                  unsigned long long *__restrict__ total,
                                                  TapeEntry *__restrict__ tape,
                                                  uint32_t *__restrict__ tape_n) {
  const float4 *lut = (const float4 *)g.lut;
  const uint32_t zc = __ldg(g.zc);
  const DiffView &vw = views[blockIdx.z];
  const r3d_frame_params &pc = vw.pc;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u +
                      ((lane & 1u) | ((lane >> 1) & 2u) | ((lane >> 2) & 4u));
  const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (((lane >> 1) & 1u) | ((lane >> 2) & 2u));
  uint32_t steps = 0;
  if (px < pc.viewport[0] && py < pc.viewport[1]) {
    const size_t ray = vw.out_off / 3u + (size_t)py * pc.viewport[0] + px;
    DiffRay r;
    diff_setup(pc, g, px, py, r);
    float acc_r = 0.0f, acc_g = 0.0f, acc_b = 0.0f, acc_a = 0.0f;
    uint32_t nc = 0;
    if (r.hit) {
      const float k = (pc.density * pc.step_voxels) * r.span;
      float t = r.t0;
      while (t < r.tf && steps < 4096u) {
        steps++;
        DiffSample s;
        diff_sample(g, r, t, s);
        if (!(s.v < pc.threshold) && !diff_clear(s.v, zc)) {
          diff_tf(lut, k, s);
          if (s.a > 0.003f) {
            if (TAPE && nc < kTape) tape[ray * kTape + nc] = make_float4(t, acc_a, s.v, s.a);
            nc++;
            float w = (1.0f - acc_a) * s.a;
            acc_r = fmaf(w, s.s[0], acc_r);
            acc_g = fmaf(w, s.s[1], acc_g);
            acc_b = fmaf(w, s.s[2], acc_b);
            acc_a = acc_a + w;
            if (acc_a >= g.cutoff) break;
          }
        }
        t = fmaf(r.dt, r.span, t);
      }
    }
    if (TAPE) tape_n[ray] = nc;
    float tr = 1.0f - acc_a;
    float *o = rgb + vw.out_off + ((size_t)py * pc.viewport[0] + px) * 3u;
    o[0] = fmaf(tr, 0.02f, acc_r);
    o[1] = fmaf(tr, 0.02f, acc_g);
    o[2] = fmaf(tr, 0.03f, acc_b);
  }
  if (total) {
    uint32_t sum = steps;
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
    if (lane == 0 && sum) atomicAdd(total, (unsigned long long)sum);
  }
}

// x * 2^32 rounded to the nearest int64: the product is exact in FP32 (a
// power-of-two scale), so converting it directly equals converting
// (double)x * 2^32
__device__ __forceinline__ long long fix32(float x) {
  return __float2ll_rn(x * 4294967296.0f);
}

// voxel gradient sink: FP32 atomics or 2^32 fixed point
template <bool DET>
__device__ __forceinline__ void vox_add(float *gf, unsigned long long *gq, uint32_t i, float x) {
  if (x == 0.0f) return;
  if (DET)
    atomicAdd(gq + i, (unsigned long long)fix32(x));
  else
    atomicAdd(gf + i, x);
}

// The block's LUT-gradient table in shared memory.  Deterministic sums are
// kept mod 2^64 as two 32-bit words per entry: the low word takes the low
// half of each addend, and a carry out of it goes to the high word with the
// high half, so that every update is two native 32-bit shared atomics.
struct LutGrad {
  union {
    uint32_t w[2048];  // deterministic: low words w[i], high words w[1024 + i]
    float f[1024];     // FP32 atomics
  };
};

template <bool DET>
__device__ __forceinline__ void lut_add(LutGrad &lg, uint32_t i, float x) {
  if (DET) {
    const long long q = fix32(x);
    if (!q) return;
    const uint32_t ql = (uint32_t)q, qh = (uint32_t)((unsigned long long)q >> 32);
    const uint32_t old = atomicAdd(&lg.w[i], ql);
    const uint32_t h = qh + (old + ql < old ? 1u : 0u);
    if (h) atomicAdd(&lg.w[1024u + i], h);
  } else {
    atomicAdd(&lg.f[i], x);
  }
}

template <bool DET>
__device__ __forceinline__ void lut_clear(LutGrad &lg) {
  for (uint32_t i = threadIdx.x; i < 1024u; i += blockDim.x) {
    if (DET) {
      lg.w[i] = 0u;
      lg.w[1024u + i] = 0u;
    } else {
      lg.f[i] = 0.0f;
    }
  }
}

template <bool DET>
__device__ __forceinline__ void lut_flush(const LutGrad &lg, float *g_lut,
                                          unsigned long long *q_lut) {
  for (uint32_t i = threadIdx.x; i < 1024u; i += blockDim.x) {
    if (DET) {
      const unsigned long long q = ((unsigned long long)lg.w[1024u + i] << 32) | lg.w[i];
      if (q) atomicAdd(q_lut + i, q);
    } else {
      if (lg.f[i] != 0.0f) atomicAdd(g_lut + i, lg.f[i]);
    }
  }
}

constexpr int kRing = 64;  // contributing samples remembered by the forward sweep

// State of one ray's reverse sweep: the colour behind the current sample,
// the trilinear cell whose voxel gradients are being summed, and the
// density-scale gradient.
struct BwdRay {
  float gr, gg, gb;  // dL/drgb of the pixel
  float k, kstep;
  float S_r, S_g, S_b;
  uint32_t cell, csx, csy, csz;
  float cw[8];
  float g_density;
};

template <bool DET>
__device__ __forceinline__ void bwd_flush(BwdRay &b, float *g_dens, unsigned long long *q_dens) {
  if (b.cell == 0xffffffffu) return;
#pragma unroll
  for (int c = 0; c < 8; c++)
    vox_add<DET>(g_dens, q_dens,
                 b.cell + ((c & 1) ? b.csx : 0u) + ((c & 2) ? b.csy : 0u) + ((c & 4) ? b.csz : 0u),
                 b.cw[c]);
}

// Adjoint of one contributing sample s (density, TF and opacity filled) with
// accumulated opacity acc_a before it, visited in reverse order (suffix
// colour S <- a c + (1 - a) S).
template <bool DET>
__device__ __forceinline__ void bwd_contrib(const float4 *lut, const DiffSample &s, float acc_a,
                                            BwdRay &b, LutGrad &lg, float *g_dens,
                                            unsigned long long *q_dens) {
  const float tprev = 1.0f - acc_a;
  const float dc_r = b.gr * tprev * s.a, dc_g = b.gg * tprev * s.a, dc_b = b.gb * tprev * s.a;
  const float da = b.gr * tprev * (s.s[0] - b.S_r) + b.gg * tprev * (s.s[1] - b.S_g) +
                   b.gb * tprev * (s.s[2] - b.S_b);
  b.S_r = fmaf(s.a, s.s[0] - b.S_r, b.S_r);
  b.S_g = fmaf(s.a, s.s[1] - b.S_g, b.S_g);
  b.S_b = fmaf(s.a, s.s[2] - b.S_b, b.S_b);
  float dalpha = 0.0f;
  const bool alpha_free = s.s[3] > 0.0f && s.s[3] < 1.0f;  // implies alpha < 1
  if (s.alpha < 1.0f) {
    const float x = 1.0f - s.alpha, l2 = r3d_log2f(x);
    if (alpha_free) {  // r3d_powf(x, k - 1) with the logarithm shared (x > 0 here)
      const float y = b.k - 1.0f;
      dalpha = da * b.k * (y == 0.0f || x == 1.0f ? 1.0f : r3d_exp2f(y * l2));
    }
    b.g_density += da * (-(1.0f - s.a) * (l2 * 0.693147181f)) * b.kstep;
  }
  const float ds[4] = {dc_r, dc_g, dc_b, dalpha};
  const float lf0 = 1.0f - s.f;
  const float4 l0 = lut[s.i0];
  const float4 l1 = lut[s.i1];
  const float dl[4] = {l1.x - l0.x, l1.y - l0.y, l1.z - l0.z, l1.w - l0.w};
  float dvv = 0.0f;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    lut_add<DET>(lg, s.i0 * 4u + c, ds[c] * lf0);
    lut_add<DET>(lg, s.i1 * 4u + c, ds[c] * s.f);
    dvv = fmaf(ds[c], dl[c], dvv);
  }
  const bool tt_free = s.tt > 0.0f && s.tt < 255.0f;
  const float dv = tt_free ? dvv * 256.0f : 0.0f;
  // trilinear scatter, aggregated per cell
  if (s.base != b.cell || s.sx != b.csx || s.sy != b.csy || s.sz != b.csz) {
    bwd_flush<DET>(b, g_dens, q_dens);
    b.cell = s.base;
    b.csx = s.sx;
    b.csy = s.sy;
    b.csz = s.sz;
#pragma unroll
    for (int c = 0; c < 8; c++) b.cw[c] = 0.0f;
  }
  const float wx[2] = {1.0f - s.fx, s.fx}, wy[2] = {1.0f - s.fy, s.fy},
              wz[2] = {1.0f - s.fz, s.fz};
#pragma unroll
  for (int c = 0; c < 8; c++)
    b.cw[c] = fmaf(dv, (wx[c & 1] * wy[(c >> 1) & 1]) * wz[c >> 2], b.cw[c]);
}

// The adjoint of the contributing sample at t, recomputed from the grid.
template <bool DET>
__device__ __forceinline__ void bwd_sample(const DiffGrid &g, const float4 *lut, const DiffRay &r,
                                           float t, float acc_a, BwdRay &b, LutGrad &lg,
                                           float *g_dens, unsigned long long *q_dens) {
  DiffSample s;
  diff_sample(g, r, t, s);
  diff_tf(lut, b.k, s);
  bwd_contrib<DET>(lut, s, acc_a, b, lg, g_dens, q_dens);
}

template <int K, bool DET>
__global__ void __launch_bounds__(128) k_diff_bwd(const DiffView *__restrict__ views,
                                                  const __grid_constant__ DiffGrid g,
                                                  const float *__restrict__ dl_drgb,
                                                  float *__restrict__ g_dens,
                                                  unsigned long long *__restrict__ q_dens,
                                                  float *__restrict__ g_lut,
                                                  unsigned long long *__restrict__ q_lut,
                                                  float *__restrict__ g_scale,
                                                  unsigned long long *__restrict__ q_scale,
                                                  const TapeEntry *__restrict__ tape,
                                                  const uint32_t *__restrict__ tape_n) {
  constexpr int kMaxCk = (4096 + K - 1) / K;
  __shared__ LutGrad lg;
  lut_clear<DET>(lg);
  __syncthreads();
  const float4 *lut = (const float4 *)g.lut;
  const uint32_t zc = __ldg(g.zc);

  const DiffView &vw = views[blockIdx.z];
  const r3d_frame_params &pc = vw.pc;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u +
                      ((lane & 1u) | ((lane >> 1) & 2u) | ((lane >> 2) & 4u));
  const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (((lane >> 1) & 1u) | ((lane >> 2) & 2u));
  BwdRay b;
  b.g_density = 0.0f;
  if (px < pc.viewport[0] && py < pc.viewport[1]) {
    const size_t ray = vw.out_off / 3u + (size_t)py * pc.viewport[0] + px;
    DiffRay r;
    diff_setup(pc, g, px, py, r);
    const float *gp = dl_drgb + vw.out_off + ((size_t)py * pc.viewport[0] + px) * 3u;
    b.gr = gp[0];
    b.gg = gp[1];
    b.gb = gp[2];
    b.k = (pc.density * pc.step_voxels) * r.span;
    b.kstep = pc.step_voxels * r.span;
    b.S_r = 0.02f;
    b.S_g = 0.02f;
    b.S_b = 0.03f;
    b.cell = 0xffffffffu;
    b.csx = b.csy = b.csz = 0u;
#pragma unroll
    for (int c = 0; c < 8; c++) b.cw[c] = 0.0f;
    const uint32_t ntape = tape ? tape_n[ray] : 0xffffffffu;
    if (r.hit && (b.gr != 0.0f || b.gg != 0.0f || b.gb != 0.0f)) {
      if (ntape <= kTape) {  // every contribution is on the tape
        for (int i = (int)ntape - 1; i >= 0; i--) {
          const float4 e = __ldg(tape + ray * kTape + i);
          DiffSample s;
          diff_cell(g, r, e.x, s);
          s.v = e.z;
          diff_tf_color(lut, s);
          s.a = e.w;
          bwd_contrib<DET>(lut, s, e.y, b, lg, g_dens, q_dens);
        }
      } else {
        // forward sweep: checkpoints (t, accumulated opacity) before steps
        // 1, K+1, 2K+1, ..., the number of contributing samples of each
        // segment, and the last kRing contributing samples themselves
        float ck_t[kMaxCk], ck_a[kMaxCk];
        uint8_t ck_n[kMaxCk];
        float ring_t[kRing], ring_a[kRing];
        uint32_t nsteps = 0, ncontrib = 0;
        {
          float t = r.t0, acc_a = 0.0f;
          while (t < r.tf && nsteps < 4096u) {
            if (nsteps % K == 0u) {
              ck_t[nsteps / K] = t;
              ck_a[nsteps / K] = acc_a;
              ck_n[nsteps / K] = 0;
            }
            nsteps++;
            DiffSample s;
            bool stop = false;
            bool live;
            diff_sample(g, r, t, s);
            live = !(s.v < pc.threshold) && !diff_clear(s.v, zc);
            if (live) {
              diff_tf(lut, b.k, s);
              if (s.a > 0.003f) {
                ring_t[ncontrib % kRing] = t;
                ring_a[ncontrib % kRing] = acc_a;
                ncontrib++;
                ck_n[(nsteps - 1u) / K]++;
                acc_a = acc_a + (1.0f - acc_a) * s.a;
                stop = acc_a >= g.cutoff;
              }
            }
            if (stop) break;
            t = fmaf(r.dt, r.span, t);
          }
        }
        // reverse sweep over segments with contributions
        float seg_t[K], seg_a[K];
        const int nck = (int)((nsteps + K - 1) / K);
        uint32_t end = ncontrib;  // contributions of segments < j: [0, end)
        for (int j = nck - 1; j >= 0; j--) {
          const uint32_t nj = ck_n[j];
          if (nj == 0u) continue;
          const uint32_t start = end - nj;
          const bool in_ring = ncontrib - start <= (uint32_t)kRing;
          int nseg = 0;
          if (in_ring) {  // the segment's samples are still in the ring
            for (uint32_t i = start; i < end; i++) {
              seg_t[nseg] = ring_t[i % kRing];
              seg_a[nseg] = ring_a[i % kRing];
              nseg++;
            }
          } else {  // recompute segment j from its checkpoint
            float t = ck_t[j], acc_a = ck_a[j];
            const uint32_t s_end = min(nsteps, (uint32_t)(j + 1) * K);
            for (uint32_t st = (uint32_t)j * K; st < s_end; st++) {
              DiffSample s;
              bool live;
              diff_sample(g, r, t, s);
              live = !(s.v < pc.threshold) && !diff_clear(s.v, zc);
              if (live) {
                diff_tf(lut, b.k, s);
                if (s.a > 0.003f) {
                  seg_t[nseg] = t;
                  seg_a[nseg] = acc_a;
                  nseg++;
                  acc_a = acc_a + (1.0f - acc_a) * s.a;
                }
              }
              t = fmaf(r.dt, r.span, t);
            }
          }
          end = start;
          for (int i = nseg - 1; i >= 0; i--)
            bwd_sample<DET>(g, lut, r, seg_t[i], seg_a[i], b, lg, g_dens, q_dens);
        }
      }
      bwd_flush<DET>(b, g_dens, q_dens);
    }
  }
  // density scale: warp reduction, one global add per warp
  float gs = b.g_density;
  if (DET) {
    long long q = fix32(gs);
    for (int off = 16; off > 0; off >>= 1) q += __shfl_xor_sync(0xffffffffu, q, off);
    if (lane == 0 && q) atomicAdd(q_scale, (unsigned long long)q);
  } else {
    for (int off = 16; off > 0; off >>= 1) gs += __shfl_xor_sync(0xffffffffu, gs, off);
    if (lane == 0 && gs != 0.0f) atomicAdd(g_scale, gs);
  }
  __syncthreads();
  lut_flush<DET>(lg, g_lut, q_lut);
}

static unsigned grid_blocks(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b < 148u * 32u ? (b ? b : 1) : 148u * 32u);
}

// fixed point -> float
__global__ void k_fix_to_float(const unsigned long long *__restrict__ q, float *__restrict__ out,
                               size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)((double)(long long)q[i] / kFix);
}

}  // namespace r3d

using namespace r3d;

// Validates the grid and views, uploads the view table; returns the grid
// descriptor and total output floats.
static int diff_prepare(r3d_cuda_ctx *c, const r3d_cuda_diff_scene *sc,
                        const r3d_frame_params *views, uint32_t nviews, DiffGrid &g,
                        DiffView *&dviews, uint32_t &maxw, uint32_t &maxh, size_t &nfloats,
                        cudaStream_t st) {
  if (!sc || !sc->density || !sc->lut || !sc->nx || !sc->ny || !sc->nz || !views || !nviews ||
      nviews > kMaxBatchViews)
    return fail(c, R3D_E_INVALID, "diff: bad arguments");
  if ((uint64_t)sc->nx * sc->ny * sc->nz >= (1ull << 32))
    return fail(c, R3D_E_INVALID, "diff: grid too large for 32-bit voxel indices");
  g.dens = sc->density;
  g.n[0] = sc->nx;
  g.n[1] = sc->ny;
  g.n[2] = sc->nz;
  g.nmax = max(sc->nx, max(sc->ny, sc->nz));
  g.lut = sc->lut;
  g.cutoff = c->alpha_cutoff;
  const int k = c->ring_next;
  c->ring_next = (k + 1) % r3d_cuda_ctx::kRing;
  if (c->ring_used[k]) R3D_CUDA_TRY(c, cudaEventSynchronize(c->ring_ev[k]));
  static_assert(sizeof(DiffView) <= sizeof(DevView), "ring slot size");
  DiffView *hv = (DiffView *)(c->ring_host + (size_t)k * kMaxBatchViews);
  dviews = (DiffView *)(c->ring_dev + (size_t)k * kMaxBatchViews);
  maxw = maxh = 0;
  nfloats = 0;
  for (uint32_t v = 0; v < nviews; v++) {
    const r3d_frame_params &p = views[v];
    if (!p.viewport[0] || !p.viewport[1] || p.viewport[0] > 16384u || p.viewport[1] > 16384u)
      return fail(c, R3D_E_INVALID, "diff: view %u needs an explicit viewport", v);
    if (p.brick_mode || p.slab_grid || p.clip_valid || p.overlay_flags ||
        (p.view_flags & ~R3D_VIEW_ORTHO))
      return fail(c, R3D_E_UNSUPPORTED, "diff: view %u uses a feature the differentiable "
                                        "render does not have", v);
    if (!(p.step_voxels > 0.0f)) return fail(c, R3D_E_INVALID, "diff: step_voxels");
    memset(&hv[v], 0, sizeof hv[v]);
    hv[v].pc = p;
    hv[v].out_off = nfloats;
    nfloats += (size_t)p.viewport[0] * p.viewport[1] * 3u;
    maxw = max(maxw, p.viewport[0]);
    maxh = max(maxh, p.viewport[1]);
  }
  R3D_CUDA_TRY(c, cudaMemcpyAsync(dviews, hv, sizeof(DiffView) * nviews, cudaMemcpyHostToDevice,
                                  st));
  R3D_CUDA_TRY(c, cudaEventRecord(c->ring_ev[k], st));
  c->ring_used[k] = true;
  return R3D_OK;
}

// Fills g.quad: the context's quad grid, rebuilt from the density unless
// `reuse` and it was last built from this density buffer.
static int diff_quads(r3d_cuda_ctx *c, const r3d_cuda_diff_scene *sc, DiffGrid &g, bool reuse,
                      cudaStream_t st) {
  const size_t nvox = (size_t)sc->nx * sc->ny * sc->nz;
  const size_t need = nvox * sizeof(float4) + 256u;  // the quads, then DiffGrid::zc
  if (c->diff_quad_bytes < need) {  // grow; earlier work on the old buffer must finish first
    R3D_CUDA_TRY(c, cudaDeviceSynchronize());
    cudaFree(c->diff_quad);
    c->diff_quad = nullptr;
    c->diff_quad_bytes = 0;
    c->quad_src = nullptr;
    R3D_CUDA_TRY(c, cudaMalloc(&c->diff_quad, need));
    c->diff_quad_bytes = need;
  }
  g.quad = (const float4 *)c->diff_quad;
  uint32_t *zc = (uint32_t *)((char *)c->diff_quad + nvox * sizeof(float4));
  g.zc = zc;
  // the TF may change between calls that share the density
  k_diff_tf_clear<<<1, 256, 0, st>>>(sc->lut, zc);
  R3D_CUDA_TRY(c, cudaGetLastError());
  if (reuse && c->quad_src == sc->density) return R3D_OK;
  k_diff_quads<<<grid_blocks(nvox), 256, 0, st>>>(sc->density, sc->nx, sc->ny, sc->nz,
                                                  (float4 *)c->diff_quad);
  R3D_CUDA_TRY(c, cudaGetLastError());
  c->quad_src = sc->density;
  return R3D_OK;
}

// Identity of a tape: the views, the scene's buffers and sizes and the
// cutoff of the forward that wrote it.
static bool tape_matches(const r3d_cuda_ctx *c, const r3d_cuda_diff_scene *sc,
                         const r3d_frame_params *views, uint32_t nviews) {
  return c->tape_valid && c->tape_nviews == nviews && c->tape_density == sc->density &&
         c->tape_lut == sc->lut && c->tape_dims[0] == sc->nx && c->tape_dims[1] == sc->ny &&
         c->tape_dims[2] == sc->nz && c->tape_cutoff == c->alpha_cutoff &&
         memcmp(c->tape_views, views, sizeof(r3d_frame_params) * nviews) == 0;
}

static int diff_forward(r3d_cuda_ctx *c, const r3d_cuda_diff_scene *sc,
                        const r3d_frame_params *views, uint32_t nviews, float *rgb_out,
                        unsigned long long *total_steps, void *stream, bool tape) {
  if (!c || !rgb_out) return fail(c, R3D_E_INVALID, "diff_forward: bad arguments");
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  if (!is_device_ptr(rgb_out)) return fail(c, R3D_E_INVALID, "diff_forward: rgb_out not device");
  DiffGrid g;
  DiffView *dv;
  uint32_t mw, mh;
  size_t nf;
  int rc = diff_prepare(c, sc, views, nviews, g, dv, mw, mh, nf, st);
  if (rc != R3D_OK) return rc;
  rc = diff_quads(c, sc, g, false, st);
  if (rc != R3D_OK) return rc;
  TapeEntry *tp = nullptr;
  uint32_t *tn = nullptr;
  if (tape) {
    const size_t rays = nf / 3u;
    c->tape_valid = false;
    if (c->tape_rays < rays) {  // grow; earlier work on the old buffers must finish first
      R3D_CUDA_TRY(c, cudaDeviceSynchronize());
      cudaFree(c->tape);
      cudaFree(c->tape_n);
      c->tape = nullptr;
      c->tape_n = nullptr;
      c->tape_rays = 0;
      R3D_CUDA_TRY(c, cudaMalloc(&c->tape, rays * kTape * sizeof(TapeEntry)));
      R3D_CUDA_TRY(c, cudaMalloc(&c->tape_n, rays * sizeof(uint32_t)));
      c->tape_rays = rays;
    }
    tp = (TapeEntry *)c->tape;
    tn = c->tape_n;
  }
  R3D_CUDA_TRY(c, cudaEventRecord(c->ev0, st));
  dim3 grid((mw + 15u) / 16u, (mh + 7u) / 8u, nviews);
  if (tape)
    k_diff_fwd<true><<<grid, 128, 0, st>>>(dv, g, rgb_out, total_steps, tp, tn);
  else
    k_diff_fwd<false><<<grid, 128, 0, st>>>(dv, g, rgb_out, total_steps, nullptr, nullptr);
  R3D_CUDA_TRY(c, cudaGetLastError());
  R3D_CUDA_TRY(c, cudaEventRecord(c->ev1, st));
  c->timed = true;
  if (tape) {
    memcpy(c->tape_views, views, sizeof(r3d_frame_params) * nviews);
    c->tape_nviews = nviews;
    c->tape_density = sc->density;
    c->tape_lut = sc->lut;
    c->tape_dims[0] = sc->nx;
    c->tape_dims[1] = sc->ny;
    c->tape_dims[2] = sc->nz;
    c->tape_cutoff = c->alpha_cutoff;
    c->tape_valid = true;
  }
  return R3D_OK;
}

extern "C" int r3d_cuda_diff_forward(r3d_cuda_ctx *c, const r3d_cuda_diff_scene *sc,
                                     const r3d_frame_params *views, uint32_t nviews,
                                     float *rgb_out, unsigned long long *total_steps,
                                     void *stream) {
  return diff_forward(c, sc, views, nviews, rgb_out, total_steps, stream, false);
}

extern "C" int r3d_cuda_diff_forward_tape(r3d_cuda_ctx *c, const r3d_cuda_diff_scene *sc,
                                          const r3d_frame_params *views, uint32_t nviews,
                                          float *rgb_out, unsigned long long *total_steps,
                                          void *stream) {
  return diff_forward(c, sc, views, nviews, rgb_out, total_steps, stream, true);
}

template <int K, bool DET>
static cudaError_t launch_bwd(dim3 grid, cudaStream_t st, const DiffView *dv, const DiffGrid &g,
                              const float *dl, float *gd, unsigned long long *qd, float *gl,
                              unsigned long long *ql, float *gs, unsigned long long *qs,
                              const TapeEntry *tp, const uint32_t *tn) {
  k_diff_bwd<K, DET><<<grid, 128, 0, st>>>(dv, g, dl, gd, qd, gl, ql, gs, qs, tp, tn);
  return cudaGetLastError();
}

extern "C" int r3d_cuda_raycast_bwd(r3d_cuda_ctx *c, const r3d_cuda_diff_scene *sc,
                                    const r3d_frame_params *views, uint32_t nviews,
                                    const float *dl_drgb, const r3d_cuda_grads *out,
                                    uint32_t ckpt_k, int deterministic, void *stream) {
  if (!c || !dl_drgb || !out || !out->density || !out->lut || !out->density_scale)
    return fail(c, R3D_E_INVALID, "raycast_bwd: bad arguments");
  if (ckpt_k != 32u && ckpt_k != 64u && ckpt_k != 128u)
    return fail(c, R3D_E_INVALID, "raycast_bwd: checkpoint interval %u not 32, 64 or 128",
                ckpt_k);
  if (deterministic & ~(int)(R3D_BWD_DETERMINISTIC | R3D_BWD_TAPE))
    return fail(c, R3D_E_INVALID, "raycast_bwd: unknown flags 0x%x", deterministic);
  const bool det = (deterministic & (int)R3D_BWD_DETERMINISTIC) != 0;
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  DiffGrid g;
  DiffView *dv;
  uint32_t mw, mh;
  size_t nf;
  int rc = diff_prepare(c, sc, views, nviews, g, dv, mw, mh, nf, st);
  if (rc != R3D_OK) return rc;
  const size_t nvox = (size_t)sc->nx * sc->ny * sc->nz;
  unsigned long long *qd = nullptr, *ql = nullptr, *qs = nullptr;
  if (det) {
    const size_t need = (nvox + 1024u + 1u) * sizeof(unsigned long long);
    if (c->diff_q_bytes < need) {
      cudaFree(c->diff_q);
      c->diff_q = nullptr;
      c->diff_q_bytes = 0;
      R3D_CUDA_TRY(c, cudaMalloc(&c->diff_q, need));
      c->diff_q_bytes = need;
    }
    qd = c->diff_q;
    ql = qd + nvox;
    qs = ql + 1024;
    R3D_CUDA_TRY(c, cudaMemsetAsync(c->diff_q, 0, need, st));
  } else {
    R3D_CUDA_TRY(c, cudaMemsetAsync(out->density, 0, nvox * sizeof(float), st));
    R3D_CUDA_TRY(c, cudaMemsetAsync(out->lut, 0, 1024 * sizeof(float), st));
    R3D_CUDA_TRY(c, cudaMemsetAsync(out->density_scale, 0, sizeof(float), st));
  }
  // the tape of the matching training forward, when asked for
  const bool use_tape = (deterministic & (int)R3D_BWD_TAPE) != 0;
  if (use_tape && !tape_matches(c, sc, views, nviews))
    return fail(c, R3D_E_STATE, "raycast_bwd: no tape of a training forward over these views "
                                "and this scene");
  const TapeEntry *tp = use_tape ? (const TapeEntry *)c->tape : nullptr;
  const uint32_t *tn = use_tape ? c->tape_n : nullptr;
  // the tape's forward built the quads from this (unchanged) density
  rc = diff_quads(c, sc, g, use_tape, st);
  if (rc != R3D_OK) return rc;
  R3D_CUDA_TRY(c, cudaEventRecord(c->ev0, st));
  dim3 grid((mw + 15u) / 16u, (mh + 7u) / 8u, nviews);
  cudaError_t e;
  float *gd = out->density, *gl = out->lut, *gs = out->density_scale;
  if (det) {
    e = ckpt_k == 32u ? launch_bwd<32, true>(grid, st, dv, g, dl_drgb, gd, qd, gl, ql, gs, qs, tp, tn)
        : ckpt_k == 64u ? launch_bwd<64, true>(grid, st, dv, g, dl_drgb, gd, qd, gl, ql, gs, qs, tp, tn)
                        : launch_bwd<128, true>(grid, st, dv, g, dl_drgb, gd, qd, gl, ql, gs, qs, tp, tn);
  } else {
    e = ckpt_k == 32u ? launch_bwd<32, false>(grid, st, dv, g, dl_drgb, gd, qd, gl, ql, gs, qs, tp, tn)
        : ckpt_k == 64u ? launch_bwd<64, false>(grid, st, dv, g, dl_drgb, gd, qd, gl, ql, gs, qs, tp, tn)
                        : launch_bwd<128, false>(grid, st, dv, g, dl_drgb, gd, qd, gl, ql, gs, qs, tp, tn);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "raycast_bwd: launch");
  if (det) {
    k_fix_to_float<<<grid_blocks(nvox), 256, 0, st>>>(qd, gd, nvox);
    k_fix_to_float<<<4, 256, 0, st>>>(ql, gl, 1024);
    k_fix_to_float<<<1, 32, 0, st>>>(qs, gs, 1);
    R3D_CUDA_TRY(c, cudaGetLastError());
  }
  R3D_CUDA_TRY(c, cudaEventRecord(c->ev1, st));
  c->timed = true;
  return R3D_OK;
}
