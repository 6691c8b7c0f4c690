// XY clipmap: 6 nested octaves around a focus, each one 2048^2 texture with
// a z ring of level slices (render3d's clip mode: src/core/clip.h,
// src/vk/vkclip.c:101-215,318-346,428-453, tools/mkpyramid/main.c).  The
// reference decodes level 0 and 1 from the shard store and reads levels
// 2..5 from a precomputed 2^3 box pyramid; here the volume and that pyramid
// live on the device and a kernel fills the ring layers a focus or window
// change needs.
#include <string.h>

#include <algorithm>
#include <vector>

#include "r3d_internal.h"

namespace r3d {

constexpr uint32_t kClipTex = 2048u, kClipPayload = 2046u, kClipSnap = 16u;

// Tight 2^3 box with truncation (mkpyramid down2): dst (sx/2, sy/2, sz/2).
__global__ void k_clip_down2(const uint8_t *__restrict__ src, uint32_t sx, uint32_t sy,
                             uint8_t *__restrict__ dst, uint32_t dx, uint32_t dy, uint32_t dz) {
  const size_t n = (size_t)dx * dy * dz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i % dx), y = (uint32_t)((i / dx) % dy), z = (uint32_t)(i / dx / dy);
    const uint8_t *s0 = src + ((size_t)(2u * z) * sy + 2u * y) * sx + 2u * x;
    const uint8_t *s1 = s0 + sx, *s2 = s0 + (size_t)sx * sy, *s3 = s2 + sx;
    const uint32_t v = s0[0] + s0[1] + s1[0] + s1[1] + s2[0] + s2[1] + s3[0] + s3[1];
    dst[i] = (uint8_t)(v / 8u);
  }
}

// One ring layer of level l holding level slice ls (vkclip.c:101-185):
// level 0 is the volume, level 1 the 2^3 box (truncating) of the volume with
// coordinates clamped at full resolution, levels 2.. the pyramid clamped at
// their own extent; texel (tx, ty) is level voxel (vx0 + tx, vy0 + ty);
// slices outside the volume are zero.
__global__ void k_clip_fill(const uint8_t *__restrict__ vol, uint32_t nx, uint32_t ny, uint32_t nz,
                            const uint8_t *__restrict__ pyr, uint32_t lx, uint32_t ly,
                            uint32_t lz, uint32_t l, int64_t vx0, int64_t vy0, int64_t ls,
                            uint8_t *__restrict__ layer) {
  const size_t n = (size_t)kClipTex * kClipTex;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int64_t tx = (int64_t)(i % kClipTex), ty = (int64_t)(i / kClipTex);
    uint32_t v = 0;
    if (l == 0u) {
      if (ls >= 0 && ls < (int64_t)nz) {
        const int64_t x = min(max(vx0 + tx, (int64_t)0), (int64_t)nx - 1);
        const int64_t y = min(max(vy0 + ty, (int64_t)0), (int64_t)ny - 1);
        v = vol[((size_t)ls * ny + (size_t)y) * nx + (size_t)x];
      }
    } else if (l == 1u) {
      uint32_t sum = 0;
      for (int k = 0; k < 8; k++) {
        const int64_t z = 2 * ls + (k >> 2);
        if (z < 0 || z >= (int64_t)nz) continue;
        const int64_t x = min(max(2 * (vx0 + tx) + (k & 1), (int64_t)0), (int64_t)nx - 1);
        const int64_t y = min(max(2 * (vy0 + ty) + ((k >> 1) & 1), (int64_t)0), (int64_t)ny - 1);
        sum += vol[((size_t)z * ny + (size_t)y) * nx + (size_t)x];
      }
      v = sum / 8u;
    } else if (ls >= 0 && ls < (int64_t)lz && lx && ly) {
      const int64_t x = min(max(vx0 + tx, (int64_t)0), (int64_t)lx - 1);
      const int64_t y = min(max(vy0 + ty, (int64_t)0), (int64_t)ly - 1);
      v = pyr[((size_t)ls * ly + (size_t)y) * lx + (size_t)x];
    }
    layer[i] = (uint8_t)v;
  }
}

static int64_t clip_snap(int64_t v, int64_t q) {  // clip.h:33-37
  return v >= 0 ? v / q * q : -((-v + q - 1) / q) * q;
}

}  // namespace r3d

using namespace r3d;

void clip_reset(r3d_cuda_ctx *c) {
  cudaFree(c->clip_src);
  cudaFree(c->clip_pyr);
  cudaFree(c->clip_tex);
  c->clip_src = c->clip_pyr = c->clip_tex = nullptr;
  for (int l = 0; l < kClipLevels; l++) c->clip_layer[l].clear();
  c->have_clip = false;
}

extern "C" {

int r3d_cuda_clip_build(r3d_cuda_ctx *c, const r3d_volume_desc *d, const uint8_t *voxels,
                        uint32_t depth_max) {
  if (!c || !d || !voxels || !d->nx || !d->ny || !d->nz || !depth_max)
    return fail(c, R3D_E_INVALID, "clip_build: bad arguments");
  const uint32_t nx = d->nx, ny = d->ny, nz = d->nz;
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  clip_reset(c);
  DevClip cl;
  memset(&cl, 0, sizeof cl);
  size_t tex = 0, pyr = 0;
  uint32_t pd[3] = {nx, ny, nz};
  for (int l = 0; l < kClipLevels; l++) {
    // ring of depth_max / 2^l level slices plus 2 apron slices, at least 4
    // (clip.h:72-75)
    cl.wzl[l] = std::max(depth_max / (1u << l) + 3u, 4u);
    if (cl.wzl[l] > 64u)
      return fail(c, R3D_E_INVALID, "clip_build: depth %u needs a %u-slice ring", depth_max,
                  cl.wzl[l]);
    tex += (size_t)kClipTex * kClipTex * cl.wzl[l];
    for (int a = 0; a < 3; a++) pd[a] >>= (l ? 1 : 0);
    if (l >= 2) {  // tight pyramid levels nx >> l (mkpyramid)
      c->clip_pyr_off[l] = pyr;
      memcpy(c->clip_pyr_dim[l], pd, sizeof pd);
      pyr += (size_t)pd[0] * pd[1] * pd[2];
    } else if (l == 1) {
      memcpy(c->clip_pyr_dim[1], pd, sizeof pd);
    }
  }
  const size_t vbytes = (size_t)nx * ny * nz;
  const size_t l1 = (size_t)c->clip_pyr_dim[1][0] * c->clip_pyr_dim[1][1] * c->clip_pyr_dim[1][2];
  uint8_t *half = nullptr;
  cudaError_t e = cudaMalloc(&c->clip_src, vbytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->clip_pyr, pyr ? pyr : 1u);
  if (e == cudaSuccess) e = cudaMalloc(&c->clip_tex, tex);
  if (e == cudaSuccess) e = cudaMalloc(&half, l1 ? l1 : 1u);
  if (e == cudaSuccess) e = copy_sync(c->stream, c->clip_src, voxels, vbytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->clip_tex, 0, tex, c->stream);
  if (e == cudaSuccess && l1) {  // down2 chain: volume -> half -> levels 2..5
    const uint32_t *h = c->clip_pyr_dim[1];
    k_clip_down2<<<4096, 256, 0, c->stream>>>(c->clip_src, nx, ny, half, h[0], h[1], h[2]);
    const uint8_t *prev = half;
    uint32_t px = h[0], py = h[1];
    for (int l = 2; l < kClipLevels; l++) {
      const uint32_t *q = c->clip_pyr_dim[l];
      if (q[0] && q[1] && q[2])
        k_clip_down2<<<4096, 256, 0, c->stream>>>(prev, px, py, c->clip_pyr + c->clip_pyr_off[l],
                                                  q[0], q[1], q[2]);
      prev = c->clip_pyr + c->clip_pyr_off[l];
      px = q[0];
      py = q[1];
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(half);
  if (e != cudaSuccess) {
    clip_reset(c);
    return cuda_fail(c, e, "clip_build");
  }
  size_t off = 0;
  for (int l = 0; l < kClipLevels; l++) {
    cl.lev[l] = c->clip_tex + off;
    off += (size_t)kClipTex * kClipTex * cl.wzl[l];
    c->clip_layer[l].assign(cl.wzl[l], -1);
    c->clip_org[l][0] = c->clip_org[l][1] = INT64_MIN;  // not centred yet
  }
  cl.nx = (float)nx;
  c->clip_dims[0] = nx;
  c->clip_dims[1] = ny;
  c->clip_dims[2] = nz;
  c->clip_depth = depth_max;
  c->cl = cl;
  c->have_clip = true;
  return R3D_OK;
}

int r3d_cuda_clip_frame(r3d_cuda_ctx *c, double fx, double fy, uint64_t z0, r3d_frame_params *p) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_clip) return fail(c, R3D_E_STATE, "clip_frame: no clipmap");
  cudaSetDevice(c->device);
  const int64_t nx = c->clip_dims[0], ny = c->clip_dims[1];
  const int64_t ifx = (int64_t)fx, ify = (int64_t)fy;
  for (int l = 0; l < kClipLevels; l++) {
    const int64_t s = (int64_t)1 << l, cov = (int64_t)kClipPayload * s;
    int64_t &ox = c->clip_org[l][0], &oy = c->clip_org[l][1];
    // recentre when the focus drifted beyond a quarter of the coverage
    // (clip.h:46-64,92-103)
    bool recentre = ox == INT64_MIN;
    if (!recentre && !(cov >= nx && cov >= ny)) {
      const int64_t cx = ox + cov / 2, cy = oy + cov / 2;
      const int64_t dx = ifx > cx ? ifx - cx : cx - ifx, dy = ify > cy ? ify - cy : cy - ify;
      recentre = dx > cov / 4 || dy > cov / 4;
    }
    if (recentre) {
      const int64_t snap = (int64_t)kClipSnap * s;
      int64_t x = clip_snap(ifx - cov / 2, snap), y = clip_snap(ify - cov / 2, snap);
      if (x < 0) x = 0;
      if (y < 0) y = 0;
      if (x + cov > nx) x = clip_snap(nx - cov, snap);
      if (y + cov > ny) y = clip_snap(ny - cov, snap);
      if (x < 0) x = 0;
      if (y < 0) y = 0;
      if (x != ox || y != oy)
        std::fill(c->clip_layer[l].begin(), c->clip_layer[l].end(), (int64_t)-1);
      ox = x;
      oy = y;
    }
    // the ring layers of level slices [z0 >> l, (z0 >> l) + wzl)
    const uint32_t wzl = c->cl.wzl[l];
    const int64_t ls0 = (int64_t)(z0 >> l);
    const uint32_t *q = c->clip_pyr_dim[l];
    const uint8_t *pyr = l >= 2 ? c->clip_pyr + c->clip_pyr_off[l] : nullptr;
    for (uint32_t k = 0; k < wzl; k++) {
      const int64_t ls = ls0 + k;
      const uint32_t layer = (uint32_t)(ls % wzl);
      if (c->clip_layer[l][layer] == ls) continue;
      k_clip_fill<<<4096, 256, 0, c->stream>>>(
          c->clip_src, c->clip_dims[0], c->clip_dims[1], c->clip_dims[2], pyr, q[0], q[1], q[2],
          (uint32_t)l, ox / s - 1, oy / s - 1, ls,
          const_cast<uint8_t *>(c->cl.lev[l]) + (size_t)layer * kClipTex * kClipTex);
      c->clip_layer[l][layer] = ls;
    }
    c->cl.ox[l] = (float)ox;
    c->cl.oy[l] = (float)oy;
  }
  R3D_CUDA_TRY(c, cudaGetLastError());
  c->cl.valid = (1u << kClipLevels) - 1u;
  c->cl.z0 = (float)z0;
  if (p) r3d_cuda_clip_params(c, p);
  return R3D_OK;
}

void r3d_cuda_clip_params(const r3d_cuda_ctx *c, r3d_frame_params *p) {
  if (!c || !p || !c->have_clip) return;
  p->slab_nx = (float)c->clip_dims[0];
  p->slab_ny = (float)c->clip_dims[1];
  p->slab_z0 = c->cl.z0;
  p->slab_wz = c->clip_depth;
  p->slab_depth = c->clip_depth;
  for (int l = 0; l < kClipLevels; l++) {
    p->clip_orig[l][0] = c->cl.ox[l];
    p->clip_orig[l][1] = c->cl.oy[l];
  }
  p->clip_valid = c->cl.valid;
  p->slab_grid = 0u;
  p->brick_mode = 0u;
}

int r3d_cuda_clip_read(r3d_cuda_ctx *c, uint32_t level, uint32_t layer, uint8_t *out) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_clip) return fail(c, R3D_E_STATE, "clip_read: no clipmap");
  if (level >= (uint32_t)kClipLevels || layer >= c->cl.wzl[level])
    return fail(c, R3D_E_INVALID, "clip_read: level %u layer %u", level, layer);
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  R3D_CUDA_TRY(c, cudaMemcpy(out, c->cl.lev[level] + (size_t)layer * kClipTex * kClipTex,
                             (size_t)kClipTex * kClipTex, cudaMemcpyDeviceToHost));
  return R3D_OK;
}

}  // extern "C"
