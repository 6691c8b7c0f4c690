// Tiled slab: a wide, thin window of a volume as a grid of apron-padded
// tiles with a z ring, plus the overview pyramid (render3d's slab mode:
// src/core/slab.h, src/vk/vkbackend.c:2128-2164,2172-2335).  The reference
// assembles each tile slice on the host and uploads it; here the source
// volume stays on the device and kernels cut the overview planes and the
// tile slices of the ring layers that a window move needs.
#include <string.h>

#include <algorithm>
#include <vector>

#include "r3d_internal.h"

namespace r3d {

// Layout of one slab level (r3d_slab_layout_init_cap with the 2048 tile
// cap, slab.h:42-62): tiles per axis and uniform payload.
struct SlabLayout {
  uint32_t nx, ny, gx, gy, px, py;
};

static bool slab_layout(uint32_t nx, uint32_t ny, SlabLayout &l) {
  const uint32_t maxp = 2048u - 2u;
  l.nx = nx;
  l.ny = ny;
  l.gx = (nx + maxp - 1u) / maxp;
  l.gy = (ny + maxp - 1u) / maxp;
  if (l.gx > 22u || l.gy > 22u) return false;
  l.px = (nx + l.gx - 1u) / l.gx;
  l.py = (ny + l.gy - 1u) / l.gy;
  return true;
}

// One downsampled plane per slice: dst (dx x dy) averages the n x n blocks
// of src (sx x sy), clipped at the far edges, truncating
// (vkbackend.c:2128-2144).  Grid: (.., slices).
__global__ void k_slab_down(const uint8_t *__restrict__ src, uint32_t sx, uint32_t sy,
                            size_t src_stride, uint8_t *__restrict__ dst, uint32_t dx, uint32_t dy,
                            size_t dst_stride, uint32_t n) {
  const uint8_t *s = src + (size_t)blockIdx.y * src_stride;
  uint8_t *d = dst + (size_t)blockIdx.y * dst_stride;
  const size_t total = (size_t)dx * dy;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i % dx), y = (uint32_t)(i / dx);
    const uint32_t x0 = x * n, x1 = min(x0 + n, sx), y0 = y * n, y1 = min(y0 + n, sy);
    uint32_t sum = 0;
    for (uint32_t yy = y0; yy < y1; yy++)
      for (uint32_t xx = x0; xx < x1; xx++) sum += s[(size_t)yy * sx + xx];
    d[i] = (uint8_t)(sum / ((y1 - y0) * (x1 - x0)));
  }
}

// Tile slices of one level for a run of slices: texel (tx, ty) of tile
// (i, j) in ring layer (s % wz) is plane[s][row(j, ty)][col(i, tx)] with
// the apron rows and columns clamped to the plane (slab.h:82-95,
// vkbackend.c:2148-2164).  Grid: (.., slices).
__global__ void k_slab_tiles(const uint8_t *__restrict__ plane, size_t plane_stride,
                             uint32_t nx, uint32_t ny, uint32_t gx, uint32_t gy, uint32_t px,
                             uint32_t py, uint32_t wz, uint32_t s0, uint8_t *__restrict__ tiles) {
  const uint32_t s = s0 + blockIdx.y, layer = s % wz;
  const uint8_t *p = plane + (size_t)blockIdx.y * plane_stride;
  const uint32_t tw = px + 2u, th = py + 2u;
  const size_t tile_bytes = (size_t)tw * th * wz;
  const size_t total = (size_t)gx * gy * tw * th;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t tx = (uint32_t)(i % tw), ty = (uint32_t)((i / tw) % th);
    const uint32_t k = (uint32_t)(i / ((size_t)tw * th));
    const uint32_t ti = k % gx, tj = k / gx;
    const int64_t cx = min(max((int64_t)ti * px - 1 + tx, (int64_t)0), (int64_t)nx - 1);
    const int64_t cy = min(max((int64_t)tj * py - 1 + ty, (int64_t)0), (int64_t)ny - 1);
    tiles[(size_t)k * tile_bytes + (size_t)layer * tw * th + (size_t)ty * tw + tx] =
        p[(size_t)cy * nx + (size_t)cx];
  }
}

static unsigned slab_grid1(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b < 4096u ? (b ? b : 1) : 4096u);
}

// Fills ring layers of world slices [s0, s1).
static int slab_fill(r3d_cuda_ctx *c, uint32_t s0, uint32_t s1) {
  cudaStream_t st = c->stream;
  const DevSlab &sl = c->sl;
  const uint32_t nx = c->slab_dims[0], ny = c->slab_dims[1];
  const size_t plane = (size_t)nx * ny;
  for (uint32_t a = s0; a < s1; a += 16u) {  // 16 slices at a time
    const uint32_t n = std::min(16u, s1 - a);
    const uint8_t *src = c->slab_src + (size_t)a * plane;
    const DevSlabLevel &b = sl.lev[0];
    k_slab_tiles<<<dim3(slab_grid1((size_t)b.gx * b.gy * (b.px + 2u) * (b.py + 2u)), n), 256, 0,
                   st>>>(src, plane, nx, ny, b.gx, b.gy, b.px, b.py, sl.wz, a,
                         c->slab_buf + b.off);
    const uint8_t *prev = src;
    uint32_t pnx = nx, pny = ny;
    size_t pstride = plane;
    for (uint32_t lev = 1; lev < sl.nlev; lev++) {
      const uint32_t f = lev == 1u ? 4u : 2u;  // 4x from the slice, then 2x chains
      const uint32_t onx = c->slab_ovn[lev][0], ony = c->slab_ovn[lev][1];
      uint8_t *dst = c->slab_planes + c->slab_plane_off[lev];
      k_slab_down<<<dim3(slab_grid1((size_t)onx * ony), n), 256, 0, st>>>(
          prev, pnx, pny, pstride, dst, onx, ony, (size_t)onx * ony, f);
      const DevSlabLevel &L = sl.lev[lev];
      k_slab_tiles<<<dim3(slab_grid1((size_t)L.gx * L.gy * (L.px + 2u) * (L.py + 2u)), n), 256,
                     0, st>>>(dst, (size_t)onx * ony, onx, ony, L.gx, L.gy, L.px, L.py, sl.wz, a,
                              c->slab_buf + L.off);
      prev = dst;
      pnx = onx;
      pny = ony;
      pstride = (size_t)onx * ony;
    }
    R3D_CUDA_TRY(c, cudaGetLastError());
  }
  return R3D_OK;
}

}  // namespace r3d

using namespace r3d;

void slab_reset(r3d_cuda_ctx *c) {
  cudaFree(c->slab_buf);
  cudaFree(c->slab_src);
  cudaFree(c->slab_planes);
  c->slab_buf = nullptr;
  c->slab_src = nullptr;
  c->slab_planes = nullptr;
  c->have_slab = false;
}

extern "C" {

int r3d_cuda_slab_build(r3d_cuda_ctx *c, const r3d_volume_desc *d, const uint8_t *voxels,
                        uint32_t wz, uint32_t z0) {
  if (!c || !d || !voxels || !d->nx || !d->ny || !d->nz)
    return fail(c, R3D_E_INVALID, "slab_build: bad arguments");
  const uint32_t nx = d->nx, ny = d->ny, nz = d->nz;
  if (wz < 4u || wz > nz) return fail(c, R3D_E_INVALID, "slab_build: ring depth %u", wz);
  SlabLayout base;
  if (!slab_layout(nx, ny, base))
    return fail(c, R3D_E_INVALID, "slab_build: %ux%u needs more than 22 tiles per axis", nx, ny);
  // overview scale: the whole composite in <= 2046-texel tiles (slab.h:57-61)
  uint32_t ovs = 4u;
  while ((nx + ovs - 1u) / ovs > 2046u || (ny + ovs - 1u) / ovs > 2046u) ovs <<= 1;
  if (ovs > 255u) return fail(c, R3D_E_INVALID, "slab_build: overview scale %u", ovs);
  uint32_t nov = 1u;  // levels 4 << lev up to ovs (slab.h:122-129)
  for (uint32_t s = 4u; s < ovs; s <<= 1) nov++;
  if (nov + 1u > (uint32_t)kSlabLevels) return fail(c, R3D_E_INVALID, "slab_build: levels");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  slab_reset(c);
  DevSlab sl;
  memset(&sl, 0, sizeof sl);
  sl.wz = wz;
  sl.nlev = nov + 1u;
  sl.ovs = ovs;
  sl.nx = (float)nx;
  sl.ny = (float)ny;
  sl.px = (float)base.px;
  sl.py = (float)base.py;
  // the overview branch's per-level constants, in the shader's float
  // expressions (raycast.slang:430-446)
  sl.nov = (int)(r3d_log2f((float)ovs) + 0.5f) - 1;
  for (int k = 0; k < sl.nov && k < kSlabLevels; k++) {
    const float sc = (float)(4 << k);
    const float vnx = ceilf(sl.nx / sc), vny = ceilf(sl.ny / sc);
    const float gxl = ceilf(vnx / 2046.0f), gyl = ceilf(vny / 2046.0f);
    sl.ov[k][0] = gxl;
    sl.ov[k][1] = gyl;
    sl.ov[k][2] = ceilf(vnx / gxl);
    sl.ov[k][3] = ceilf(vny / gyl);
  }
  size_t off = 0, planes = 0;
  for (uint32_t lev = 0; lev < sl.nlev; lev++) {
    SlabLayout l = base;
    if (lev) {
      const uint32_t s = 4u << (lev - 1u);
      slab_layout((nx + s - 1u) / s, (ny + s - 1u) / s, l);
      c->slab_ovn[lev][0] = l.nx;
      c->slab_ovn[lev][1] = l.ny;
      c->slab_plane_off[lev] = planes;
      planes += (size_t)l.nx * l.ny * 16u;  // 16 slices per fill batch
    }
    sl.lev[lev] = {l.gx, l.gy, l.px, l.py, off};
    off += (size_t)l.gx * l.gy * (l.px + 2u) * (l.py + 2u) * wz;
  }
  const size_t vbytes = (size_t)nx * ny * nz;
  cudaError_t e = cudaMalloc(&c->slab_buf, off);
  if (e == cudaSuccess) e = cudaMalloc(&c->slab_src, vbytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->slab_planes, planes ? planes : 1u);
  if (e == cudaSuccess) e = copy_sync(c->stream, c->slab_src, voxels, vbytes);
  if (e != cudaSuccess) {
    slab_reset(c);
    return cuda_fail(c, e, "slab_build");
  }
  sl.pool = c->slab_buf;
  c->slab_dims[0] = nx;
  c->slab_dims[1] = ny;
  c->slab_dims[2] = nz;
  c->sl = sl;
  const uint32_t z = std::min(z0, nz - wz);
  c->sl.z0 = (float)z;
  int rc = slab_fill(c, z, z + wz);
  if (rc == R3D_OK) R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (rc != R3D_OK) {
    slab_reset(c);
    return rc;
  }
  c->slab_win = z;
  c->have_slab = true;
  return R3D_OK;
}

int r3d_cuda_slab_window(r3d_cuda_ctx *c, uint32_t z0) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_slab) return fail(c, R3D_E_STATE, "slab_window: no slab");
  cudaSetDevice(c->device);
  const uint32_t wz = c->sl.wz, z = std::min(z0, c->slab_dims[2] - wz);
  // slices entering the window (slab.h:100-121); frames queued on the
  // context's stream finish before the layers they read are refilled
  const int64_t d = (int64_t)z - (int64_t)c->slab_win;
  uint32_t s0, s1;
  if (d >= (int64_t)wz || d <= -(int64_t)wz) {
    s0 = z;
    s1 = z + wz;
  } else if (d > 0) {
    s0 = c->slab_win + wz;
    s1 = z + wz;
  } else if (d < 0) {
    s0 = z;
    s1 = c->slab_win;
  } else {
    return R3D_OK;
  }
  int rc = slab_fill(c, s0, s1);
  if (rc != R3D_OK) return rc;
  c->slab_win = z;
  c->sl.z0 = (float)z;
  return R3D_OK;
}

void r3d_cuda_slab_params(const r3d_cuda_ctx *c, r3d_frame_params *p) {
  if (!c || !p || !c->have_slab) return;
  p->slab_grid = c->sl.lev[0].gx | (c->sl.lev[0].gy << 8) | (c->sl.ovs << 16);
  p->slab_wz = c->sl.wz;
  p->slab_z0 = c->sl.z0;
  p->slab_nx = c->sl.nx;
  p->slab_ny = c->sl.ny;
  p->slab_px = c->sl.px;
  p->slab_py = c->sl.py;
  p->slab_depth = c->sl.wz - 2u;  // the maximum; a view may lower it
  p->brick_mode = 0u;
}

int r3d_cuda_slab_read(r3d_cuda_ctx *c, uint32_t level, uint32_t tile, uint8_t *out,
                       uint32_t dims[3]) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_slab) return fail(c, R3D_E_STATE, "slab_read: no slab");
  if (level >= c->sl.nlev) return fail(c, R3D_E_INVALID, "slab_read: level %u", level);
  const DevSlabLevel &L = c->sl.lev[level];
  if (tile >= L.gx * L.gy) return fail(c, R3D_E_INVALID, "slab_read: tile %u", tile);
  const uint32_t dd[3] = {L.px + 2u, L.py + 2u, c->sl.wz};
  if (dims) memcpy(dims, dd, sizeof dd);
  if (out) {
    cudaSetDevice(c->device);
    R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    const size_t bytes = (size_t)dd[0] * dd[1] * dd[2];
    R3D_CUDA_TRY(c, cudaMemcpy(out, c->slab_buf + L.off + (size_t)tile * bytes, bytes,
                               cudaMemcpyDeviceToHost));
  }
  return R3D_OK;
}

}  // extern "C"
