// Slot-parallel overlay atlases of the LOD brick cache: ink (surface
// predictions), 3D ink, paint labels and a registered second scan.  In the
// reference each is a texture with the CT atlas's slot layout, filled
// whenever a CT brick lands in a slot (src/render/render.h:51-101,
// src/vk/vkbackend.c bricks overlay paths) and sampled by the raycast at
// the CT sample's slot coordinate (src/shaders/raycast.slang:45-115,
// 872-914,1000-1014,1032-1036).  Here an overlay is given either as slot
// contents in the CT pool's order or as a raw volume of the CT volume's
// shape, from which the same LOD bricks are cut; it is stored in the quad
// form of the CT pool.
#include <string.h>

#include <vector>

#include "r3d_internal.h"

namespace r3d {

// Defined in r3d_ctx.cu.
__global__ void k_downsample_zero(const uint8_t *__restrict__ src, uint32_t sx, uint32_t sy,
                                  uint32_t sz, uint8_t *__restrict__ dst, uint32_t dx,
                                  uint32_t dy, uint32_t dz);
__global__ void k_brick_copy(const uint8_t *__restrict__ lev, uint32_t ex, uint32_t ey,
                             uint32_t ez, uint32_t bdx, uint32_t bdy,
                             const uint32_t *__restrict__ src_brick,
                             const uint32_t *__restrict__ dst_slot, uint8_t *__restrict__ pool);
__global__ void k_slot_quads(const uint8_t *__restrict__ pool, uint32_t *__restrict__ quad,
                             size_t n);

// Level l of a label volume: the level-0 voxel at (x, y, z) << l, zero
// outside the volume (coarse label bricks stride-sample the paint grid,
// src/core/labelvol.c:172-196).
__global__ void k_label_stride(const uint8_t *__restrict__ vol, uint32_t nx, uint32_t ny,
                               uint32_t nz, uint32_t l, uint8_t *__restrict__ dst, uint32_t dx,
                               uint32_t dy, uint32_t dz) {
  const size_t n = (size_t)dx * dy * dz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t x = (uint64_t)(i % dx) << l, y = (uint64_t)((i / dx) % dy) << l,
                   z = (uint64_t)(i / dx / dy) << l;
    dst[i] = x < nx && y < ny && z < nz ? vol[(z * ny + y) * nx + x] : 0;
  }
}

// Byte 0 of every quad word: the atlas's own texels.
__global__ void k_quad_texels(const uint32_t *__restrict__ quad, uint8_t *__restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (uint8_t)(quad[i] & 0xFFu);
}

static unsigned ovl_grid(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b < 148u * 64u ? (b ? b : 1) : 148u * 64u);
}

// Converts a byte pool (device) into overlay atlas `which`.
static int overlay_quads(r3d_cuda_ctx *c, uint32_t which, const uint8_t *pool) {
  const size_t n = (size_t)(c->nslots ? c->nslots : 1u) * (128u * 128u * 128u);
  uint32_t *q = nullptr;
  R3D_CUDA_TRY(c, cudaMalloc(&q, n * sizeof(uint32_t)));
  if (c->nslots) k_slot_quads<<<ovl_grid(n), 256, 0, c->stream>>>(pool, q, n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    cudaFree(q);
    return cuda_fail(c, e, "bricks_overlay");
  }
  cudaFree(c->ovl_quad[which]);
  c->ovl_quad[which] = q;
  c->br.ovl[which] = q;
  if (c->ovl_src_on[which]) c->ovl_key[which].assign(c->nslots, UINT64_MAX);  // replaced content
  return R3D_OK;
}

// overlay_quads through the display filter when it targets the atlas (ink:
// target 1, 3D ink: 2); a pool the context does not own is filtered in a
// copy.
static int set_overlay(r3d_cuda_ctx *c, uint32_t which, const uint8_t *pool, bool owned) {
  if (which >= 2u || !c->nslots || !postfilter_on(c, which + 1u)) return overlay_quads(c, which, pool);
  const size_t n = (size_t)c->nslots * (128u * 128u * 128u);
  uint8_t *f = owned ? const_cast<uint8_t *>(pool) : nullptr;
  if (!owned) {
    R3D_CUDA_TRY(c, cudaMalloc(&f, n));
    cudaError_t e = cudaMemcpyAsync(f, pool, n, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) {
      cudaFree(f);
      return cuda_fail(c, e, "bricks_overlay: filter copy");
    }
  }
  std::vector<uint32_t> all(c->nslots);
  for (uint32_t s = 0; s < c->nslots; s++) all[s] = s;
  int rc = postfilter_slots(c, which + 1u, f, all.data(), c->nslots);
  if (rc == R3D_OK) rc = overlay_quads(c, which, f);  // synchronizes the stream
  if (!owned) {
    cudaStreamSynchronize(c->stream);
    cudaFree(f);
  }
  return rc;
}

}  // namespace r3d

using namespace r3d;

extern "C" {

int r3d_cuda_bricks_overlay_load(r3d_cuda_ctx *c, uint32_t which, const uint8_t *slots) {
  if (!c || which > 3u) return fail(c, R3D_E_INVALID, "bricks_overlay_load: bad arguments");
  if (!c->have_bricks) return fail(c, R3D_E_STATE, "bricks_overlay_load: no brick cache");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (!slots) {
    cudaFree(c->ovl_quad[which]);
    c->ovl_quad[which] = nullptr;
    c->br.ovl[which] = nullptr;
    return R3D_OK;
  }
  const size_t bytes = (size_t)c->nslots * (128u * 128u * 128u);
  if (is_device_ptr(slots)) return set_overlay(c, which, slots, false);
  uint8_t *tmp = nullptr;
  R3D_CUDA_TRY(c, cudaMalloc(&tmp, bytes ? bytes : 1u));
  cudaError_t e = copy_sync(c->stream, tmp, slots, bytes);
  int rc = e == cudaSuccess ? set_overlay(c, which, tmp, true) : cuda_fail(c, e, "bricks_overlay_load");
  cudaFree(tmp);
  return rc;
}

// ---- CPU-sourced atlases (vkbackend.c:4908-5150) ----

static constexpr uint32_t kAtlasBatch = 16u, kSlotTexels = 128u * 128u * 128u;

int r3d_cuda_bricks_atlas_attach(r3d_cuda_ctx *c, uint32_t which, const r3d_brick_src *src) {
  if (!c || which > 3u || !src || !src->gen || !src->fetch)
    return fail(c, R3D_E_INVALID, "bricks_atlas_attach: atlas 0..3 and a gen and fetch callback");
  if (!c->have_bricks) return fail(c, R3D_E_STATE, "bricks_atlas_attach: no brick cache");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (!c->ovl_stage) {
    R3D_CUDA_TRY(c, cudaMallocHost(&c->ovl_stage, (size_t)kAtlasBatch * kSlotTexels));
    R3D_CUDA_TRY(c, cudaMalloc(&c->ovl_stage_dev, (size_t)kAtlasBatch * kSlotTexels));
  }
  uint64_t key0 = UINT64_MAX;  // content of unknown bricks: zeroed first
  if (!c->ovl_quad[which]) {   // a cleared atlas
    const size_t n = (size_t)(c->nslots ? c->nslots : 1u) * kSlotTexels;
    uint32_t *q = nullptr;
    R3D_CUDA_TRY(c, cudaMalloc(&q, n * sizeof(uint32_t)));
    cudaError_t e = cudaMemsetAsync(q, 0, n * sizeof(uint32_t), c->stream);
    if (e != cudaSuccess) {
      cudaFree(q);
      return cuda_fail(c, e, "bricks_atlas_attach");
    }
    c->ovl_quad[which] = q;
    c->br.ovl[which] = q;
    key0 = 0;
  }
  c->ovl_key[which].assign(c->nslots, key0);
  c->ovl_src[which] = *src;
  c->ovl_src_on[which] = true;
  return R3D_OK;
}

int r3d_cuda_bricks_atlas_detach(r3d_cuda_ctx *c, uint32_t which) {
  if (!c || which > 3u) return fail(c, R3D_E_INVALID, "bricks_atlas_detach: atlas 0..3");
  c->ovl_src_on[which] = false;  // the atlas and its keys stay for a re-attach
  c->ovl_src[which] = r3d_brick_src{};
  return R3D_OK;
}

int r3d_cuda_bricks_atlas_sync(r3d_cuda_ctx *c, uint32_t which, uint32_t budget, uint32_t *synced) {
  if (synced) *synced = 0;
  if (!c || which > 3u) return fail(c, R3D_E_INVALID, "bricks_atlas_sync: atlas 0..3");
  if (!c->ovl_src_on[which] || !c->have_bricks) return R3D_OK;
  cudaSetDevice(c->device);
  // which brick each slot holds: the pump's table, or the page table of a
  // resident cache
  std::vector<uint32_t> page, sb;
  const uint32_t *hpage, *slot_brick;
  if (c->streaming) {
    hpage = c->store_page.data();
    slot_brick = c->slot_brick.data();
  } else {
    page.resize(c->page_words);
    R3D_CUDA_TRY(c, copy_sync(c->stream, page.data(), c->page, page.size() * 4u));
    sb.assign(c->nslots, R3D_BRICK_ABSENT);
    for (uint32_t b = R3D_BRICK_PAGE_HEADER; b < c->page_words; b++)
      if (page[b] != R3D_BRICK_ABSENT && (page[b] & 0xFFFFFFu) < c->nslots) sb[page[b] & 0xFFFFFFu] = b;
    hpage = page.data();
    slot_brick = sb.data();
  }
  uint32_t sel[kAtlasBatch], selb[kAtlasBatch];
  uint64_t key[kAtlasBatch];
  const uint32_t n = r3d_host_atlas_pick(hpage, slot_brick, c->nslots, c->ovl_key[which].data(),
                                         &c->ovl_src[which], budget, sel, selb, key);
  if (!n) return R3D_OK;
  // the staging slots of the previous round are free once the stream is
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  for (uint32_t i = 0; i < n; i++) {
    uint8_t *dst = c->ovl_stage + (size_t)i * kSlotTexels;
    uint32_t l, bx, by, bz;
    if (key[i] && r3d_host_brick_locate(hpage, selb[i], &l, &bx, &by, &bz) == 0)
      c->ovl_src[which].fetch(c->ovl_src[which].user, l, bx, by, bz, dst);
    else
      memset(dst, 0, kSlotTexels);
  }
  R3D_CUDA_TRY(c, cudaMemcpyAsync(c->ovl_stage_dev, c->ovl_stage, (size_t)n * kSlotTexels,
                                  cudaMemcpyHostToDevice, c->stream));
  for (uint32_t i = 0; i < n; i++)  // that slot's overlay words
    k_slot_quads<<<ovl_grid(kSlotTexels), 256, 0, c->stream>>>(
        c->ovl_stage_dev + (size_t)i * kSlotTexels, c->ovl_quad[which] + (size_t)sel[i] * kSlotTexels,
        kSlotTexels);
  R3D_CUDA_TRY(c, cudaGetLastError());
  for (uint32_t i = 0; i < n; i++) c->ovl_key[which][sel[i]] = key[i];
  if (synced) *synced = n;
  return R3D_OK;
}

int r3d_cuda_bricks_overlay_read(r3d_cuda_ctx *c, uint32_t which, uint8_t *slots) {
  if (!c || which > 3u || !slots) return fail(c, R3D_E_INVALID, "bricks_overlay_read: bad arguments");
  if (!c->ovl_quad[which]) return fail(c, R3D_E_STATE, "bricks_overlay_read: atlas %u is not loaded", which);
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->nslots * (128u * 128u * 128u);
  if (!n) return R3D_OK;
  uint8_t *tmp = nullptr;
  R3D_CUDA_TRY(c, cudaMalloc(&tmp, n));
  k_quad_texels<<<ovl_grid(n), 256, 0, c->stream>>>(c->ovl_quad[which], tmp, n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(slots, tmp, n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(tmp);
  return e == cudaSuccess ? R3D_OK : cuda_fail(c, e, "bricks_overlay_read");
}

int r3d_cuda_bricks_overlay_build(r3d_cuda_ctx *c, uint32_t which, const r3d_volume_desc *d,
                                  const uint8_t *voxels) {
  if (!c || which > 3u || !d || !voxels)
    return fail(c, R3D_E_INVALID, "bricks_overlay_build: bad arguments");
  if (!c->have_bricks) return fail(c, R3D_E_STATE, "bricks_overlay_build: no brick cache");
  if (d->nx != c->shape[0] || d->ny != c->shape[1] || d->nz != c->shape[2])
    return fail(c, R3D_E_INVALID, "bricks_overlay_build: %ux%ux%u is not the cache's %ux%ux%u",
                d->nx, d->ny, d->nz, c->shape[0], c->shape[1], c->shape[2]);
  cudaSetDevice(c->device);
  cudaStream_t st = c->stream;
  R3D_CUDA_TRY(c, cudaStreamSynchronize(st));
  const DevBricks &br = c->br;
  const uint32_t nlev = br.nlev, nx = d->nx, ny = d->ny, nz = d->nz;
  // level extents as the CT pyramid's: level 0 the volume, level l >= 1 the
  // zero-padded brick grid
  uint32_t E[16][3];
  size_t lev_off[16] = {0}, lev_total = 0;
  for (uint32_t l = 0; l < nlev; l++) {
    const uint32_t n3[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) E[l][a] = l == 0 ? n3[a] : br.bd[l][a] * 128u;
    lev_off[l] = lev_total;
    lev_total += ((size_t)E[l][0] * E[l][1] * E[l][2] + 255) & ~(size_t)255;
  }
  // resident bricks of every level and their slots, from the page table
  std::vector<uint32_t> page(c->page_words);
  R3D_CUDA_TRY(c, cudaMemcpy(page.data(), c->page, page.size() * 4, cudaMemcpyDeviceToHost));
  std::vector<uint32_t> jobs_src, jobs_dst, lvl_count(nlev, 0);
  for (uint32_t l = 0; l < nlev; l++) {
    const uint32_t nb = br.bd[l][0] * br.bd[l][1] * br.bd[l][2];
    for (uint32_t bi = 0; bi < nb; bi++) {
      const uint32_t e = page[br.off[l] + bi];
      if (e == R3D_BRICK_ABSENT || (e & 0xFFFFFFu) >= c->nslots) continue;
      jobs_src.push_back(bi);
      jobs_dst.push_back(e & 0xFFFFFFu);
      lvl_count[l]++;
    }
  }
  const size_t nj = jobs_src.size();
  const size_t pool_bytes = (size_t)(c->nslots ? c->nslots : 1u) * (128u * 128u * 128u);
  uint8_t *lev = nullptr, *pool = nullptr;
  uint32_t *jobs = nullptr;
  cudaError_t e = cudaMalloc(&lev, lev_total);
  if (e == cudaSuccess) e = cudaMalloc(&pool, pool_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&jobs, (nj ? nj : 1u) * 8);
  if (e == cudaSuccess) e = cudaMemsetAsync(pool, 0, pool_bytes, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(lev, voxels, (size_t)nx * ny * nz, cudaMemcpyDefault, st);
  for (uint32_t l = 1; l < nlev && e == cudaSuccess; l++) {
    const size_t n = (size_t)E[l][0] * E[l][1] * E[l][2];
    if (which == 2u)  // labels: stride sampling, never blended
      k_label_stride<<<ovl_grid(n), 256, 0, st>>>(lev, nx, ny, nz, l, lev + lev_off[l], E[l][0],
                                                   E[l][1], E[l][2]);
    else  // the CT's (sum+4)/8 box pyramid
      k_downsample_zero<<<ovl_grid(n), 256, 0, st>>>(lev + lev_off[l - 1], E[l - 1][0],
                                                     E[l - 1][1], E[l - 1][2], lev + lev_off[l],
                                                     E[l][0], E[l][1], E[l][2]);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && nj) {
    e = cudaMemcpyAsync(jobs, jobs_src.data(), nj * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(jobs + nj, jobs_dst.data(), nj * 4, cudaMemcpyHostToDevice, st);
  }
  size_t joff = 0;
  for (uint32_t l = 0; l < nlev && e == cudaSuccess; l++) {
    for (uint32_t j0 = 0; j0 < lvl_count[l] && e == cudaSuccess; j0 += 65535u) {
      const uint32_t n = min(lvl_count[l] - j0, 65535u);
      k_brick_copy<<<dim3(128, n), 256, 0, st>>>(lev + lev_off[l], E[l][0], E[l][1], E[l][2],
                                                 br.bd[l][0], br.bd[l][1], jobs + joff + j0,
                                                 jobs + nj + joff + j0, pool);
      e = cudaGetLastError();
    }
    joff += lvl_count[l];
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  int rc = e == cudaSuccess ? set_overlay(c, which, pool, true) : cuda_fail(c, e, "bricks_overlay_build");
  cudaFree(lev);
  cudaFree(pool);
  cudaFree(jobs);
  return rc;
}

}  // extern "C"
