// Virtual slab: a W x H x D window anywhere in a volume, rendered from
// world-anchored toroidal tile grids (render3d's vslab mode: src/core/vslab.h,
// src/vk/vkbackend.c:5675-6660).  The reference decodes cells from its shard
// store on a worker thread and uploads them layer by layer; here the volume
// lives on the device, a frame's fills run as kernels on the context's
// stream ahead of the frames that read them, and the validity table is
// published right after.  The fill writes the texels the reference's
// vs_fill / vs_scatter_depth write: the base tile with its one-texel apron
// (duplicated at the volume's near edges, zero past its far edges), and the
// pyramid strips (a 4x4 box of the payload, then 2x2 boxes, truncating)
// scattered into the up to four pyramid tiles they overlap, aprons included.
#include <string.h>

#include <algorithm>
#include <vector>

#include "r3d_internal.h"

namespace r3d {

// Base tile of cell (cx, cy): texel (tx, ty) of world slice zs0 + k holds
// world voxel (cx * px - 1 + tx, cy * px - 1 + ty), clamped up to 0 and zero
// past the volume (vkbackend.c:6089-6111,5992-6010).
__global__ void k_vs_base(const uint8_t *__restrict__ vol, uint32_t nx, uint32_t ny,
                          uint32_t px, int64_t cx, int64_t cy, int64_t zs0, uint32_t nz,
                          uint32_t wz, uint8_t *__restrict__ tile) {
  const uint32_t T = px + 2u;
  const size_t plane = (size_t)T * T, n = plane * nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t tx = (uint32_t)(i % T), ty = (uint32_t)((i / T) % T), k = (uint32_t)(i / plane);
    const int64_t wx = cx * (int64_t)px - 1 + tx, wy = cy * (int64_t)px - 1 + ty;
    const int64_t z = zs0 + k;
    uint8_t v = 0;
    if (wx < (int64_t)nx && wy < (int64_t)ny)
      v = vol[((size_t)z * ny + (size_t)max(wy, (int64_t)0)) * nx + (size_t)max(wx, (int64_t)0)];
    tile[(size_t)(z % wz) * plane + (size_t)ty * T + tx] = v;
  }
}

// Pyramid level 1 strip of a cell: the truncating 4x4 box of its payload
// (vkbackend.c:5682-5696,6118-6121), n = px / 4 texels a side, per slice.
__global__ void k_vs_down4(const uint8_t *__restrict__ vol, uint32_t nx, uint32_t ny,
                           uint32_t px, int64_t cx, int64_t cy, int64_t zs0, uint32_t nz,
                           uint8_t *__restrict__ strip) {
  const uint32_t n = px / 4u;
  const size_t plane = (size_t)n * n, total = plane * nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i % n), y = (uint32_t)((i / n) % n), k = (uint32_t)(i / plane);
    const int64_t z = zs0 + k;
    uint32_t sum = 0;
    for (uint32_t yy = 0; yy < 4u; yy++) {
      const int64_t wy = cy * (int64_t)px + 4u * y + yy;
      if (wy >= (int64_t)ny) continue;
      const uint8_t *row = vol + ((size_t)z * ny + (size_t)wy) * nx;
      for (uint32_t xx = 0; xx < 4u; xx++) {
        const int64_t wx = cx * (int64_t)px + 4u * x + xx;
        if (wx < (int64_t)nx) sum += row[wx];
      }
    }
    strip[i] = (uint8_t)(sum / 16u);
  }
}

// Next pyramid strip: truncating 2x2 box of the previous one (n a side).
__global__ void k_vs_down2(const uint8_t *__restrict__ src, uint32_t n, uint32_t nz,
                           uint8_t *__restrict__ dst) {
  const uint32_t h = n / 2u;
  const size_t plane = (size_t)h * h, total = plane * nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i % h), y = (uint32_t)((i / h) % h), k = (uint32_t)(i / plane);
    const uint8_t *s = src + (size_t)k * n * n + (size_t)(2u * y) * n + 2u * x;
    dst[i] = (uint8_t)((s[0] + s[1] + s[n] + s[n + 1]) / 4u);
  }
}

// Scatters a level strip (n x n texels at level texel (t0x, t0y)) into the
// level's tiles it overlaps (vkbackend.c:6032-6057): tile (p, q) holds level
// texels [p * px - 1, p * px + px + 1) of each axis at texel t - p * px + 1;
// tiles p in [max(0, (t0 - 1) / px), (t0 + n) / px].
__global__ void k_vs_scatter(const uint8_t *__restrict__ strip, uint32_t n, uint32_t nz,
                             int64_t t0x, int64_t t0y, uint32_t px, uint32_t gx, uint32_t gy,
                             uint32_t base, int64_t zs0, uint32_t wz, uint8_t *__restrict__ pool) {
  const uint32_t T = px + 2u;
  const size_t tplane = (size_t)T * T, tbytes = tplane * wz;
  const size_t plane = (size_t)n * n, total = plane * nz;
  const int64_t P = px;
  int64_t p0x = (t0x - 1) / P, p0y = (t0y - 1) / P;  // truncating, as the reference's
  if (p0x < 0) p0x = 0;
  if (p0y < 0) p0y = 0;
  const int64_t p1x = (t0x + n) / P, p1y = (t0y + n) / P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i % n), y = (uint32_t)((i / n) % n), k = (uint32_t)(i / plane);
    const int64_t tx = t0x + x, ty = t0y + y;
    const uint8_t v = strip[i];
    const size_t layer = (size_t)((zs0 + k) % wz) * tplane;
    for (int64_t q = ty / P - 1; q <= ty / P + 1; q++) {
      if (q < p0y || q > p1y || ty < q * P - 1 || ty >= q * P + P + 1) continue;
      for (int64_t p = tx / P - 1; p <= tx / P + 1; p++) {
        if (p < p0x || p > p1x || tx < p * P - 1 || tx >= p * P + P + 1) continue;
        const uint32_t tile = base + (uint32_t)(q % gy) * gx + (uint32_t)(p % gx);
        pool[(size_t)tile * tbytes + layer + (size_t)(ty - q * P + 1) * T + (tx - p * P + 1)] = v;
      }
    }
  }
}

static unsigned grid_for(size_t n) {
  return (unsigned)std::min<size_t>((n + 255) / 256, 148u * 16u);
}

// One fill job on the context's stream.
static cudaError_t vs_fill(r3d_cuda_ctx *c, const r3d_vslab_job &j) {
  if (!j.nz) return cudaSuccess;
  const r3d_vslab_layout &v = c->vsl;
  const uint32_t nx = (uint32_t)v.nx, ny = (uint32_t)v.ny, P = v.px, T = P + 2u;
  const size_t tbytes = (size_t)T * T * v.wz;
  const uint32_t slot =
      (uint32_t)(j.cy % v.gy[0]) * v.gx[0] + (uint32_t)(j.cx % v.gx[0]);
  cudaStream_t st = c->stream;
  k_vs_base<<<grid_for((size_t)T * T * j.nz), 256, 0, st>>>(
      c->vs_src, nx, ny, P, j.cx, j.cy, j.zs0, j.nz, v.wz,
      c->vs_tiles + (size_t)(v.base[0] + slot) * tbytes);
  if (v.gx[1]) {
    uint32_t n = P / 4u;
    k_vs_down4<<<grid_for((size_t)n * n * j.nz), 256, 0, st>>>(c->vs_src, nx, ny, P, j.cx, j.cy,
                                                               j.zs0, j.nz,
                                                               c->vs_strip + c->vs_strip_off[1]);
    for (uint32_t l = 2; l < R3D_VS_LEVELS && v.gx[l]; l++) {
      k_vs_down2<<<grid_for((size_t)(n / 2u) * (n / 2u) * j.nz), 256, 0, st>>>(
          c->vs_strip + c->vs_strip_off[l - 1], n, j.nz, c->vs_strip + c->vs_strip_off[l]);
      n /= 2u;
    }
    for (uint32_t l = 1; l < R3D_VS_LEVELS && v.gx[l]; l++) {
      const uint32_t m = P / v.s[l];
      k_vs_scatter<<<grid_for((size_t)m * m * j.nz), 256, 0, st>>>(
          c->vs_strip + c->vs_strip_off[l], m, j.nz, j.cx * (int64_t)m, j.cy * (int64_t)m, P,
          v.gx[l], v.gy[l], v.base[l], j.zs0, v.wz, c->vs_tiles);
    }
  }
  return cudaGetLastError();
}

}  // namespace r3d

using namespace r3d;

void vslab_reset(r3d_cuda_ctx *c) {
  cudaFree(c->vs_src);
  cudaFree(c->vs_tiles);
  cudaFree(c->vs_strip);
  cudaFree(c->vs_table);
  c->vs_src = c->vs_tiles = c->vs_strip = nullptr;
  c->vs_table = nullptr;
  c->vs_table_host.clear();
  c->vs_cells.clear();
  c->vs_jobs.clear();
  c->have_vslab = false;
  c->vs = DevVslab{};
}

extern "C" {

int r3d_cuda_vslab_begin(r3d_cuda_ctx *c, const r3d_volume_desc *d, const uint8_t *voxels,
                         uint32_t W, uint32_t H, uint32_t D, uint32_t z_margin) {
  if (!c || !d || !voxels || !d->nx || !d->ny || !d->nz)
    return fail(c, R3D_E_INVALID, "vslab_begin: bad arguments");
  r3d_vslab_layout v;
  if (r3d_host_vslab_init(&v, d->nx, d->ny, d->nz, W, H, D, z_margin) != 0)
    return fail(c, R3D_E_INVALID, "vslab_begin: bad %ux%ux%u window (margin %u) for %ux%ux%u",
                W, H, D, z_margin, d->nx, d->ny, d->nz);
  if (v.gx[0] > 63u || v.gy[0] > 63u)
    return fail(c, R3D_E_INVALID, "vslab_begin: %ux%u base tiles exceed slab_grid", v.gx[0],
                v.gy[0]);
  for (uint32_t l = 1; l < R3D_VS_LEVELS; l++)
    if (v.gx[l] > 15u || v.gy[l] > 15u)
      return fail(c, R3D_E_INVALID, "vslab_begin: level %u grid exceeds brick_mode", l);
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  vslab_reset(c);
  const size_t T = v.px + 2u, tbytes = T * T * v.wz;
  const size_t vbytes = (size_t)d->nx * d->ny * d->nz;
  size_t strip = 0;
  for (uint32_t l = 1; l < R3D_VS_LEVELS; l++) {
    const size_t n = v.px / v.s[l];
    c->vs_strip_off[l] = strip;
    strip += (n * n * v.wz + 255u) & ~(size_t)255u;
  }
  const uint32_t nslot = v.gx[0] * v.gy[0];
  cudaError_t e = cudaMalloc(&c->vs_src, vbytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->vs_tiles, tbytes * v.ntiles);
  if (e == cudaSuccess) e = cudaMalloc(&c->vs_strip, strip);
  if (e == cudaSuccess) e = cudaMalloc(&c->vs_table, (size_t)nslot * 16u);
  if (e == cudaSuccess) e = copy_sync(c->stream, c->vs_src, voxels, vbytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->vs_tiles, 0, tbytes * v.ntiles, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->vs_table, 0, (size_t)nslot * 16u, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    vslab_reset(c);
    return cuda_fail(c, e, "vslab_begin");
  }
  c->vsl = v;
  c->vs_cells.assign(nslot, r3d_vslab_cell{INT64_MIN, INT64_MIN, 0, 0});
  c->vs_table_host.assign((size_t)nslot * 4u, 0u);
  DevVslab dv{};
  dv.tiles = c->vs_tiles;
  dv.table = c->vs_table;
  dv.tile_bytes = tbytes;
  dv.px = v.px;
  dv.wz = v.wz;
  for (uint32_t l = 0; l < R3D_VS_LEVELS; l++) {
    dv.gx[l] = v.gx[l];
    dv.gy[l] = v.gy[l];
    dv.base[l] = v.base[l];
  }
  dv.nx = (float)v.W;
  c->vs = dv;
  c->have_vslab = true;
  return R3D_OK;
}

int r3d_cuda_vslab_frame(r3d_cuda_ctx *c, double fx, double fy, int64_t z0, uint32_t budget,
                         r3d_frame_params *p, r3d_vslab_stats *st) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_vslab) return fail(c, R3D_E_STATE, "vslab_frame: no virtual slab");
  cudaSetDevice(c->device);
  r3d_vslab_layout &v = c->vsl;
  c->vs_jobs.resize(64u + 48u);
  const uint32_t nj = r3d_host_vslab_plan(&v, c->vs_cells.data(), fx, fy, z0, budget,
                                          c->vs_jobs.data(), (uint32_t)c->vs_jobs.size());
  c->vs_jobs.resize(nj);
  uint32_t slices = 0;
  for (uint32_t k = 0; k < nj; k++) {
    const r3d_vslab_job &j = c->vs_jobs[k];
    R3D_CUDA_TRY(c, vs_fill(c, j));
    slices += j.nz;
    const uint32_t slot = r3d_host_vslab_apply(&v, c->vs_cells.data(), &j, v.z0);
    const r3d_vslab_cell &cell = c->vs_cells[slot];
    uint32_t *w = &c->vs_table_host[(size_t)slot * 4u];
    w[0] = r3d_host_vslab_key(cell.cx, cell.cy);
    w[1] = (uint32_t)cell.za;
    w[2] = (uint32_t)cell.zb;
  }
  // publish the table after the fills, in stream order (a pageable copy is
  // staged before this returns, so the host copy may change right after)
  if (nj)
    R3D_CUDA_TRY(c, cudaMemcpyAsync(c->vs_table, c->vs_table_host.data(),
                                    c->vs_table_host.size() * 4u, cudaMemcpyHostToDevice,
                                    c->stream));
  c->vs.x0 = (float)v.x0;
  c->vs.y0 = (float)v.y0;
  c->vs.z0 = (float)v.z0;
  if (st) {
    int64_t c0x, c1x, c0y, c1y;
    r3d_host_vslab_range(&v, 0, v.x0, v.nx, v.W, &c0x, &c1x);
    r3d_host_vslab_range(&v, 0, v.y0, v.ny, v.H, &c0y, &c1y);
    int64_t vis_end = v.z0 + (int64_t)v.D + 2;
    if (vis_end > (int64_t)v.nz) vis_end = (int64_t)v.nz;
    uint32_t pending = 0;
    for (int64_t cy = c0y; cy <= c1y; cy++)
      for (int64_t cx = c0x; cx <= c1x; cx++) {
        const r3d_vslab_cell &cell =
            c->vs_cells[(uint32_t)(cy % v.gy[0]) * v.gx[0] + (uint32_t)(cx % v.gx[0])];
        pending += !(cell.cx == cx && cell.cy == cy && cell.za <= v.z0 && cell.zb >= vis_end);
      }
    st->jobs = nj;
    st->slices = slices;
    st->pending = pending;
    st->pad = 0;
    st->origin[0] = v.x0;
    st->origin[1] = v.y0;
    st->origin[2] = v.z0;
  }
  if (p) r3d_cuda_vslab_params(c, p);
  return R3D_OK;
}

void r3d_cuda_vslab_params(const r3d_cuda_ctx *c, r3d_frame_params *p) {
  if (!c || !p || !c->have_vslab) return;
  const r3d_vslab_layout &v = c->vsl;
  // vkbackend.c:6628-6645
  p->slab_grid = v.gx[0] | (v.gy[0] << 6) | kVslabGrid;
  uint32_t bm = 0;
  for (uint32_t l = 1; l < R3D_VS_LEVELS; l++) bm |= (v.gx[l] | (v.gy[l] << 4)) << ((l - 1u) * 8u);
  p->brick_mode = bm;
  p->slab_wz = v.wz;
  p->slab_z0 = (float)(v.z0 < 0 ? 0 : v.z0);
  p->slab_nx = (float)v.W;
  p->slab_ny = (float)v.H;
  p->slab_px = (float)v.px;
  p->slab_py = (float)v.px;
  p->slab_depth = v.D;
  p->slab_x0 = (float)(v.x0 < 0 ? 0 : v.x0);
  p->slab_y0 = (float)(v.y0 < 0 ? 0 : v.y0);
  p->clip_valid = 0u;
}

int r3d_cuda_vslab_layout(const r3d_cuda_ctx *c, r3d_vslab_layout *out) {
  if (!c || !out) return R3D_E_INVALID;
  if (!c->have_vslab) return R3D_E_STATE;
  *out = c->vsl;
  return R3D_OK;
}

int r3d_cuda_vslab_read(r3d_cuda_ctx *c, uint32_t tile, uint8_t *out) {
  if (!c || !out) return R3D_E_INVALID;
  if (!c->have_vslab) return fail(c, R3D_E_STATE, "vslab_read: no virtual slab");
  if (tile >= c->vsl.ntiles) return fail(c, R3D_E_INVALID, "vslab_read: tile %u", tile);
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const size_t tb = c->vs.tile_bytes;
  R3D_CUDA_TRY(c, cudaMemcpy(out, c->vs_tiles + (size_t)tile * tb, tb, cudaMemcpyDeviceToHost));
  return R3D_OK;
}

int r3d_cuda_vslab_table(r3d_cuda_ctx *c, uint32_t *out) {
  if (!c || !out) return R3D_E_INVALID;
  if (!c->have_vslab) return fail(c, R3D_E_STATE, "vslab_table: no virtual slab");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  R3D_CUDA_TRY(c, cudaMemcpy(out, c->vs_table, c->vs_table_host.size() * 4u,
                             cudaMemcpyDeviceToHost));
  return R3D_OK;
}

}  // extern "C"
