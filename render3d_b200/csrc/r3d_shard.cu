// Single-level brick atlas (render3d's bricks mode without the LOD flag):
// builder and read-back.  The reference decodes a c5s shard into a 3-D
// atlas texture, blits 4 mips per slot and max-reduces each resident slot
// into a world-indexed occupancy grid that is then dilated
// (src/vk/vkbackend.c:3241-3330,4060-4075,4236-4273;
// src/shaders/occmax.comp, occdilate.comp).  Here the shard arrives as a raw
// volume, and the same atlas, mips, occupancy and page table are built on
// the device.
#include <string.h>

#include <vector>

#include "r3d_internal.h"

namespace r3d {

// Atlas level 0: slot s holds brick brick_of[s] of the volume (edge e,
// bpa bricks per axis), or zeros.  One thread per 16 atlas bytes; both
// sides are 16-byte aligned because e and 128 are multiples of 16.
__global__ void k_shard_place(const uint8_t *__restrict__ vol, uint32_t e, uint32_t bpa,
                              const uint32_t *__restrict__ brick_of, uint32_t abpa,
                              uint8_t *__restrict__ atlas) {
  const uint32_t a = abpa * 128u, row16 = a / 16u;
  const size_t n = (size_t)a * a * row16;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i % row16) * 16u;
    const uint32_t y = (uint32_t)((i / row16) % a), z = (uint32_t)(i / row16 / a);
    const uint32_t s = ((z >> 7) * abpa + (y >> 7)) * abpa + (x >> 7);
    const uint32_t b = brick_of[s];
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (b != R3D_BRICK_ABSENT) {
      const uint32_t bx = b % bpa, by = (b / bpa) % bpa, bz = b / (bpa * bpa);
      const size_t src = ((size_t)(bz * 128u + (z & 127u)) * e + (by * 128u + (y & 127u))) * e +
                         bx * 128u + (x & 127u);
      v = __ldg(reinterpret_cast<const uint4 *>(vol + src));
    }
    reinterpret_cast<uint4 *>(atlas)[i] = v;
  }
}

// World-indexed raw occupancy (occmax.comp): block w of the (bpa * 16)^3
// grid is the maximum of the 8^3 atlas texels of its brick's slot, or 0 when
// the brick is not resident.
__global__ void k_shard_occ_raw(const uint8_t *__restrict__ atlas, uint32_t abpa,
                                const uint32_t *__restrict__ slot_of, uint32_t bpa,
                                uint8_t *__restrict__ raw) {
  const uint32_t od = bpa * 16u, a = abpa * 128u;
  const size_t n = (size_t)od * od * od;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t wx = (uint32_t)(i % od), wy = (uint32_t)((i / od) % od),
                   wz = (uint32_t)(i / od / od);
    const uint32_t s = slot_of[((wz >> 4) * bpa + (wy >> 4)) * bpa + (wx >> 4)];
    uint32_t m = 0;
    if (s != R3D_BRICK_ABSENT) {
      const uint32_t x0 = (s % abpa) * 128u + (wx & 15u) * 8u;
      const uint32_t y0 = ((s / abpa) % abpa) * 128u + (wy & 15u) * 8u;
      const uint32_t z0 = (s / (abpa * abpa)) * 128u + (wz & 15u) * 8u;
      for (uint32_t z = z0; z < z0 + 8u; z++)
        for (uint32_t y = y0; y < y0 + 8u; y++) {
          const uint2 r =
              __ldg(reinterpret_cast<const uint2 *>(atlas + ((size_t)z * a + y) * a + x0));
          const uint32_t w0 = __vmaxu4(r.x, r.y);
          m = max(m, max(max(w0 & 0xffu, (w0 >> 8) & 0xffu), max((w0 >> 16) & 0xffu, w0 >> 24)));
        }
    }
    raw[i] = (uint8_t)m;
  }
}

// Defined in r3d_ctx.cu.
__global__ void k_downsample_clamp(const uint8_t *__restrict__ src, uint32_t sx, uint32_t sy,
                                   uint32_t sz, uint8_t *__restrict__ dst, uint32_t dx,
                                   uint32_t dy, uint32_t dz);
__global__ void k_occ_dilate(const uint8_t *__restrict__ raw, uint8_t *__restrict__ dil,
                             uint32_t ox, uint32_t oy, uint32_t oz);
__global__ void k_brick_max(const uint8_t *__restrict__ lev, uint32_t ex, uint32_t ey,
                            uint32_t ez, uint32_t bdx, uint32_t bdy, uint32_t *__restrict__ out);

static unsigned shard_grid(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b < 148u * 64u ? (b ? b : 1) : 148u * 64u);
}

}  // namespace r3d

using namespace r3d;

extern "C" {

int r3d_cuda_shard_build(r3d_cuda_ctx *c, uint32_t edge, const uint8_t *voxels, uint32_t abpa,
                         const uint32_t *slot_of) {
  if (!c || !voxels) return fail(c, R3D_E_INVALID, "shard_build: bad arguments");
  if (!edge || edge % 128u || edge / 128u > 255u)
    return fail(c, R3D_E_INVALID, "shard_build: edge %u is not 128 * (1..255)", edge);
  const uint32_t bpa = edge / 128u, nb = bpa * bpa * bpa;
  if (!abpa || abpa > bpa)
    return fail(c, R3D_E_INVALID, "shard_build: abpa %u not in [1, %u]", abpa, bpa);
  if (!slot_of && abpa != bpa)
    return fail(c, R3D_E_INVALID, "shard_build: slot_of is required when abpa < bpa");
  const uint32_t ns = abpa * abpa * abpa;
  std::vector<uint32_t> slot(nb), brick(ns, R3D_BRICK_ABSENT);
  bool identity = abpa == bpa;
  for (uint32_t b = 0; b < nb; b++) {
    const uint32_t s = slot_of ? slot_of[b] : b;
    slot[b] = s;
    identity = identity && s == b;
    if (s == R3D_BRICK_ABSENT) continue;
    if (s >= ns) return fail(c, R3D_E_INVALID, "shard_build: brick %u -> slot %u >= %u", b, s, ns);
    if (brick[s] != R3D_BRICK_ABSENT)
      return fail(c, R3D_E_INVALID, "shard_build: slot %u holds bricks %u and %u", s, brick[s], b);
    brick[s] = b;
  }
  cudaSetDevice(c->device);
  const uint32_t a = abpa * 128u, od = bpa * 16u;
  DevShard h;
  memset(&h, 0, sizeof h);
  h.atlas.nlevels = 4u;
  h.atlas.maxdim = a;
  size_t off[5];
  off[0] = 0;
  for (uint32_t m = 0; m < 4u; m++) {
    for (int k = 0; k < 3; k++) h.atlas.dim[m][k] = a >> m;
    const size_t b = (size_t)(a >> m) * (a >> m) * (a >> m);
    off[m + 1] = off[m] + ((b + 255) & ~(size_t)255);
  }
  for (int k = 0; k < 3; k++) h.atlas.odim[k] = od;
  const size_t onb = (size_t)od * od * od;
  const size_t total = off[4] + ((onb + 255) & ~(size_t)255);
  const size_t vbytes = (size_t)edge * edge * edge;

  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  uint8_t *buf = nullptr, *vtmp = nullptr;
  uint32_t *dslot = nullptr, *dbrick = nullptr, *dmax = nullptr, *dpage = nullptr;
  const bool dev_in = is_device_ptr(voxels) && ((uintptr_t)voxels & 15u) == 0u;
  cudaError_t e = cudaMalloc(&buf, total + onb);
  if (e == cudaSuccess) e = cudaMalloc(&dslot, sizeof(uint32_t) * nb);
  if (e == cudaSuccess) e = cudaMalloc(&dbrick, sizeof(uint32_t) * ns);
  if (e == cudaSuccess) e = cudaMalloc(&dmax, sizeof(uint32_t) * nb);
  if (e == cudaSuccess) e = cudaMalloc(&dpage, sizeof(uint32_t) * nb);
  if (e == cudaSuccess && !dev_in) e = cudaMalloc(&vtmp, vbytes);
  const uint8_t *vol = dev_in ? voxels : vtmp;
  if (e == cudaSuccess && !dev_in)
    e = cudaMemcpyAsync(vtmp, voxels, vbytes, cudaMemcpyDefault, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dslot, slot.data(), sizeof(uint32_t) * nb, cudaMemcpyHostToDevice,
                        c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dbrick, brick.data(), sizeof(uint32_t) * ns, cudaMemcpyHostToDevice,
                        c->stream);
  std::vector<uint32_t> maxv(nb);
  if (e == cudaSuccess) {
    k_shard_place<<<shard_grid((size_t)a * a * a / 16u), 256, 0, c->stream>>>(vol, edge, bpa,
                                                                             dbrick, abpa, buf);
    // the display filter on the placed slots, before the mips and the
    // occupancy derived from them (page maxima stay the source bricks')
    if (postfilter_on(c, 0u)) {
      std::vector<uint32_t> used;
      for (uint32_t s = 0; s < ns; s++)
        if (brick[s] != R3D_BRICK_ABSENT) used.push_back(s);
      const int frc = postfilter_slots(c, 0u, buf, used.data(), (uint32_t)used.size(), abpa);
      if (frc != R3D_OK) {
        cudaStreamSynchronize(c->stream);
        cudaFree(vtmp);
        cudaFree(dslot);
        cudaFree(dbrick);
        cudaFree(dmax);
        cudaFree(dpage);
        cudaFree(buf);
        return frc;
      }
    }
    k_brick_max<<<nb, 256, 0, c->stream>>>(vol, edge, edge, edge, bpa, bpa, dmax);
    for (uint32_t m = 1; m < 4u; m++) {
      const uint32_t s = a >> (m - 1), d = a >> m;
      k_downsample_clamp<<<shard_grid((size_t)d * d * d), 256, 0, c->stream>>>(
          buf + off[m - 1], s, s, s, buf + off[m], d, d, d);
    }
    k_shard_occ_raw<<<shard_grid(onb), 256, 0, c->stream>>>(buf, abpa, dslot, bpa, buf + total);
    k_occ_dilate<<<shard_grid(onb), 256, 0, c->stream>>>(buf + total, buf + off[4], od, od, od);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(maxv.data(), dmax, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost,
                        c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  std::vector<uint32_t> page(nb);
  for (uint32_t b = 0; b < nb; b++)
    page[b] = slot[b] == R3D_BRICK_ABSENT ? R3D_BRICK_ABSENT : slot[b] | (maxv[b] << 24);
  if (e == cudaSuccess)
    e = copy_sync(c->stream, dpage, page.data(), sizeof(uint32_t) * nb);
  cudaFree(vtmp);
  cudaFree(dslot);
  cudaFree(dbrick);
  cudaFree(dmax);
  if (e != cudaSuccess) {
    cudaFree(buf);
    cudaFree(dpage);
    return cuda_fail(c, e, "shard_build");
  }
  for (uint32_t m = 0; m < 4u; m++) h.atlas.lev[m] = buf + off[m];
  h.atlas.occ = buf + off[4];
  h.page = dpage;
  h.bpa = bpa;
  h.abpa = abpa;
  h.n = (float)edge;
  h.inv_adim = 1.0f / ((float)abpa * 128.0f);  // raycast.slang:758
  h.identity = identity ? 1u : 0u;
  cudaFree(c->shard_buf);
  cudaFree(c->shard_page);
  c->shard_buf = buf;
  c->shard_page = dpage;
  c->sh = h;
  c->have_shard = true;
  return R3D_OK;
}

uint32_t r3d_cuda_shard_mode(const r3d_cuda_ctx *c) {
  if (!c || !c->have_shard) return 0u;
  return c->sh.bpa | (c->sh.abpa << 8) | (c->sh.identity ? R3D_BRICK_IDENTITY_FLAG : 0u);
}

int r3d_cuda_shard_read(r3d_cuda_ctx *c, int level, uint32_t *page, uint8_t *out,
                        uint32_t dims[3]) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_shard) return fail(c, R3D_E_STATE, "shard_read: no atlas");
  if (level < -1 || level > 3) return fail(c, R3D_E_INVALID, "shard_read: level %d", level);
  const DevCube &a = c->sh.atlas;
  const uint8_t *src = level < 0 ? a.occ : a.lev[level];
  const uint32_t *d = level < 0 ? a.odim : a.dim[level];
  if (dims) memcpy(dims, d, sizeof(uint32_t) * 3);
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const uint32_t nb = c->sh.bpa * c->sh.bpa * c->sh.bpa;
  if (page)
    R3D_CUDA_TRY(c, cudaMemcpy(page, c->sh.page, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost));
  if (out)
    R3D_CUDA_TRY(c, cudaMemcpy(out, src, (size_t)d[0] * d[1] * d[2], cudaMemcpyDeviceToHost));
  return R3D_OK;
}

}  // extern "C"
