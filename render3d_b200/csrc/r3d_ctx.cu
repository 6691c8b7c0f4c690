// C-ABI entry points: context, scene uploads and device-side builders (mip
// chain, occupancy grid, LOD brick pyramid and page table), forward raycast.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "r3d_internal.h"

namespace r3d {

int fail(r3d_cuda_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

int cuda_fail(r3d_cuda_ctx *c, cudaError_t e, const char *what) {
  return fail(c, e == cudaErrorMemoryAllocation ? R3D_E_NOMEM : R3D_E_CUDA, "%s: %s (%s)", what,
              cudaGetErrorName(e), cudaGetErrorString(e));
}

bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// ------------------------------------------------------------- builders

// 2x box reduction with clamped source coordinates: (sum + 4) / 8
__global__ void k_downsample_clamp(const uint8_t *__restrict__ src, uint32_t sx, uint32_t sy,
                                   uint32_t sz, uint8_t *__restrict__ dst, uint32_t dx,
                                   uint32_t dy, uint32_t dz) {
  size_t n = (size_t)dx * dy * dz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t x = (uint32_t)(i % dx), y = (uint32_t)((i / dx) % dy), z = (uint32_t)(i / dx / dy);
    uint32_t sum = 4u;
#pragma unroll
    for (uint32_t k = 0; k < 8u; k++) {
      uint32_t xx = min(2u * x + (k & 1u), sx - 1u), yy = min(2u * y + ((k >> 1) & 1u), sy - 1u),
               zz = min(2u * z + (k >> 2), sz - 1u);
      sum += src[((size_t)zz * sy + yy) * sx + xx];
    }
    dst[i] = (uint8_t)(sum >> 3);
  }
}

// 2x box reduction reading zeros outside the source extent (brick pyramid)
__global__ void k_downsample_zero(const uint8_t *__restrict__ src, uint32_t sx, uint32_t sy,
                                  uint32_t sz, uint8_t *__restrict__ dst, uint32_t dx,
                                  uint32_t dy, uint32_t dz) {
  size_t n = (size_t)dx * dy * dz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t x = (uint32_t)(i % dx), y = (uint32_t)((i / dx) % dy), z = (uint32_t)(i / dx / dy);
    uint32_t sum = 4u;
#pragma unroll
    for (uint32_t k = 0; k < 8u; k++) {
      uint32_t xx = 2u * x + (k & 1u), yy = 2u * y + ((k >> 1) & 1u), zz = 2u * z + (k >> 2);
      if (xx < sx && yy < sy && zz < sz) sum += src[((size_t)zz * sy + yy) * sx + xx];
    }
    dst[i] = (uint8_t)(sum >> 3);
  }
}

// 8^3 block maxima (src/vk/vkbackend.c:794-824)
__global__ void k_occ_raw(const uint8_t *__restrict__ vox, uint32_t nx, uint32_t ny, uint32_t nz,
                          uint8_t *__restrict__ raw, uint32_t ox, uint32_t oy, uint32_t oz) {
  size_t n = (size_t)ox * oy * oz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t bx = (uint32_t)(i % ox), by = (uint32_t)((i / ox) % oy), bz = (uint32_t)(i / ox / oy);
    uint32_t m = 0;
    for (uint32_t z = bz * 8u; z < min(bz * 8u + 8u, nz); z++)
      for (uint32_t y = by * 8u; y < min(by * 8u + 8u, ny); y++) {
        const uint8_t *row = vox + ((size_t)z * ny + y) * nx;
        for (uint32_t x = bx * 8u; x < min(bx * 8u + 8u, nx); x++) m = max(m, (uint32_t)row[x]);
      }
    raw[i] = (uint8_t)m;
  }
}

// 26-neighbour max dilation (src/vk/vkbackend.c:845-860)
__global__ void k_occ_dilate(const uint8_t *__restrict__ raw, uint8_t *__restrict__ dil,
                             uint32_t ox, uint32_t oy, uint32_t oz) {
  size_t n = (size_t)ox * oy * oz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    int x = (int)(i % ox), y = (int)((i / ox) % oy), z = (int)(i / ox / oy);
    uint32_t m = 0;
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int zz = z + dz, yy = y + dy, xx = x + dx;
          if (zz < 0 || yy < 0 || xx < 0 || zz >= (int)oz || yy >= (int)oy || xx >= (int)ox)
            continue;
          m = max(m, (uint32_t)raw[((size_t)zz * oy + yy) * ox + xx]);
        }
    dil[i] = (uint8_t)m;
  }
}

// Maximum of each 128^3 brick of a level (zero outside the level's extent).
// One block per brick.
__global__ void k_brick_max(const uint8_t *__restrict__ lev, uint32_t ex, uint32_t ey,
                            uint32_t ez, uint32_t bdx, uint32_t bdy, uint32_t *__restrict__ out) {
  uint32_t bi = blockIdx.x;
  uint32_t bx = bi % bdx, by = (bi / bdx) % bdy, bz = bi / bdx / bdy;
  uint32_t m = 0;
  for (uint32_t r = threadIdx.x; r < 128u * 128u; r += blockDim.x) {
    uint32_t y = by * 128u + (r & 127u), z = bz * 128u + (r >> 7);
    if (y >= ey || z >= ez) continue;
    const uint8_t *row = lev + ((size_t)z * ey + y) * ex;
    uint32_t x0 = bx * 128u, x1 = min(x0 + 128u, ex);
    for (uint32_t x = x0; x < x1; x++) m = max(m, (uint32_t)row[x]);
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ uint32_t wm[32];
  if ((threadIdx.x & 31u) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t r = 0;
    for (uint32_t w = 0; w < blockDim.x / 32u; w++) r = max(r, wm[w]);
    out[bi] = r;
  }
}

// Copies bricks into their slots: job j copies brick src_brick[j] (linear
// index in the level's brick grid) into slot dst_slot[j]; zero outside the
// level's extent.  Grid: (128 z-slices, jobs).
__global__ void k_brick_copy(const uint8_t *__restrict__ lev, uint32_t ex, uint32_t ey,
                             uint32_t ez, uint32_t bdx, uint32_t bdy,
                             const uint32_t *__restrict__ src_brick,
                             const uint32_t *__restrict__ dst_slot, uint8_t *__restrict__ pool) {
  uint32_t j = blockIdx.y, zl = blockIdx.x;
  uint32_t bi = src_brick[j];
  uint32_t bx = bi % bdx, by = (bi / bdx) % bdy, bz = bi / bdx / bdy;
  uint8_t *dst = pool + (size_t)dst_slot[j] * (128u * 128u * 128u) + (size_t)zl * 16384u;
  uint32_t z = bz * 128u + zl;
  for (uint32_t r = threadIdx.x; r < 128u * 128u; r += blockDim.x) {
    uint32_t yl = r >> 7, xl = r & 127u;
    uint32_t y = by * 128u + yl, x = bx * 128u + xl;
    uint8_t v = 0;
    if (x < ex && y < ey && z < ez) v = lev[((size_t)z * ey + y) * ex + x];
    dst[r] = v;
  }
}

// Per-slot table of dilated 8^3 block maxima: entry (bz, by, bx) of slot s
// is the max over voxels [8b, min(8b+8, 127)] on each axis.  One block per
// slot, one thread per table entry.
__global__ void k_slot_blockmax(const uint8_t *__restrict__ pool, uint8_t *__restrict__ out) {
  const uint8_t *g = pool + (size_t)blockIdx.x * (128u * 128u * 128u);
  for (uint32_t e = threadIdx.x; e < 4096u; e += blockDim.x) {
    uint32_t bx = e & 15u, by = (e >> 4) & 15u, bz = e >> 8;
    uint32_t m = 0;
    for (uint32_t z = bz * 8u; z <= min(bz * 8u + 8u, 127u); z++)
      for (uint32_t y = by * 8u; y <= min(by * 8u + 8u, 127u); y++) {
        const uint8_t *row = g + ((size_t)z << 14) + ((size_t)y << 7);
        for (uint32_t x = bx * 8u; x <= min(bx * 8u + 8u, 127u); x++)
          m = max(m, (uint32_t)row[x]);
      }
    out[(size_t)blockIdx.x * 4096u + e] = (uint8_t)m;
  }
}

// Quad words of every slot (DevBricks::quad); one thread per texel.
__global__ void k_slot_quads(const uint8_t *__restrict__ pool, uint32_t *__restrict__ quad,
                             size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(i & 127u), y = (uint32_t)((i >> 7) & 127u);
    const size_t dx = x < 127u ? 1u : 0u, dy = y < 127u ? 128u : 0u;
    quad[i] = (uint32_t)pool[i] | ((uint32_t)pool[i + dx] << 8) | ((uint32_t)pool[i + dy] << 16) |
              ((uint32_t)pool[i + dy + dx] << 24);
  }
}

static unsigned grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b < 148u * 64u ? (b ? b : 1) : 148u * 64u);
}

}  // namespace r3d

using namespace r3d;

r3d::DevScene r3d_cuda_ctx::scene() const {
  DevScene s;
  memset(&s, 0, sizeof s);
  s.cube = cube;
  s.br = br;
  s.sh = sh;
  s.sl = sl;
  s.cl = cl;
  s.vs = vs;
  s.status = status;
  s.alpha_cutoff = alpha_cutoff;
  s.tf_zero_t = tf_zero_t;
  s.slot_bits = slot_bits;
  return s;
}

extern "C" {

int r3d_cuda_create(int device, r3d_cuda_ctx **out) {
  if (!out) return R3D_E_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return R3D_E_CUDA;
  }
  r3d_cuda_ctx *c = new (std::nothrow) r3d_cuda_ctx();
  if (!c) return R3D_E_NOMEM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->status, sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->lut, 256 * sizeof(uchar4)) != cudaSuccess ||
      cudaMalloc(&c->total, (R3D_COUNTERS + 1) * sizeof(unsigned long long)) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaMallocHost(&c->ring_host, sizeof(DevView) * kMaxBatchViews * r3d_cuda_ctx::kRing) !=
          cudaSuccess ||
      cudaMalloc(&c->ring_dev, sizeof(DevView) * kMaxBatchViews * r3d_cuda_ctx::kRing) !=
          cudaSuccess ||
      cudaMalloc(&c->ring_queue, sizeof(uint32_t) * 2 * kMaxBatchViews * r3d_cuda_ctx::kRing) !=
          cudaSuccess) {
    cudaGetLastError();
    r3d_cuda_destroy(c);
    return R3D_E_CUDA;
  }
  if (cudaMemsetAsync(c->status, 0, sizeof(uint32_t), c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    cudaGetLastError();
    r3d_cuda_destroy(c);
    return R3D_E_CUDA;
  }
  for (int k = 0; k < r3d_cuda_ctx::kRing; k++)
    if (cudaEventCreateWithFlags(&c->ring_ev[k], cudaEventDisableTiming) != cudaSuccess) {
      r3d_cuda_destroy(c);
      return R3D_E_CUDA;
    }
  // default transfer function: grey ramp with alpha = value
  // (src/vk/vkbackend.c:1100-1114)
  uint8_t ramp[256][4];
  for (int i = 0; i < 256; i++) ramp[i][0] = ramp[i][1] = ramp[i][2] = ramp[i][3] = (uint8_t)i;
  if (r3d_cuda_set_transfer(c, ramp) != R3D_OK) {
    r3d_cuda_destroy(c);
    return R3D_E_CUDA;
  }
  *out = c;
  return R3D_OK;
}

void r3d_cuda_destroy(r3d_cuda_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->cube_buf);
  cudaFree(c->page);
  cudaFree(c->pool);
  cudaFree(c->bmax);
  cudaFree(c->quad);
  for (int i = 0; i < 4; i++) cudaFree(c->ovl_quad[i]);
  cudaFreeHost(c->ovl_stage);
  cudaFree(c->ovl_stage_dev);
  cudaFree(c->shard_buf);
  cudaFree(c->shard_page);
  cudaFree(c->lut);
  cudaFree(c->status);
  cudaFree(c->img);
  cudaFree(c->aux_buf);
  cudaFree(c->total);
  stream_reset(c);
  slab_reset(c);
  clip_reset(c);
  vslab_reset(c);
  surf_reset(c);
  postfilter_reset(c);
  if (c->page_ev) cudaEventDestroy(c->page_ev);
  cudaFree(c->diff_q);
  cudaFree(c->tape);
  cudaFree(c->diff_quad);
  cudaFree(c->tape_n);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (int k = 0; k < r3d_cuda_ctx::kRing; k++)
    if (c->ring_ev[k]) cudaEventDestroy(c->ring_ev[k]);
  cudaFreeHost(c->ring_host);
  cudaFree(c->ring_dev);
  cudaFree(c->ring_queue);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char *r3d_cuda_last_error(const r3d_cuda_ctx *c) { return c ? c->err.c_str() : "no ctx"; }

void *r3d_cuda_stream(r3d_cuda_ctx *c) { return c ? (void *)c->stream : nullptr; }

int r3d_cuda_status(r3d_cuda_ctx *c, uint32_t *bits, int clear) {
  if (!c) return R3D_E_INVALID;
  cudaSetDevice(c->device);
  uint32_t v = 0;
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  R3D_CUDA_TRY(c, cudaMemcpy(&v, c->status, 4, cudaMemcpyDeviceToHost));
  if (clear) R3D_CUDA_TRY(c, cudaMemsetAsync(c->status, 0, 4, c->stream));
  if (bits) *bits = v;
  return R3D_OK;
}

int r3d_cuda_upload_volume(r3d_cuda_ctx *c, const r3d_volume_desc *d, const uint8_t *voxels) {
  if (!c || !d || !voxels || !d->nx || !d->ny || !d->nz)
    return fail(c, R3D_E_INVALID, "upload_volume: bad arguments");
  cudaSetDevice(c->device);
  uint32_t nx = d->nx, ny = d->ny, nz = d->nz;
  uint32_t maxdim = max(nx, max(ny, nz));
  if (maxdim > 65535u) return fail(c, R3D_E_INVALID, "upload_volume: dimension > 65535");
  uint32_t mips = 1;
  while ((maxdim >> mips) >= 1u && mips < 16u) mips++;
  DevCube cube;
  memset(&cube, 0, sizeof cube);
  cube.nlevels = mips;
  cube.maxdim = maxdim;
  size_t off[17];
  off[0] = 0;
  for (uint32_t m = 0; m < mips; m++) {
    cube.dim[m][0] = nx >> m ? nx >> m : 1u;
    cube.dim[m][1] = ny >> m ? ny >> m : 1u;
    cube.dim[m][2] = nz >> m ? nz >> m : 1u;
    size_t b = (size_t)cube.dim[m][0] * cube.dim[m][1] * cube.dim[m][2];
    off[m + 1] = off[m] + ((b + 255) & ~(size_t)255);
  }
  for (int a = 0; a < 3; a++) cube.odim[a] = ((a == 0 ? nx : a == 1 ? ny : nz) + 7u) / 8u;
  size_t onb = (size_t)cube.odim[0] * cube.odim[1] * cube.odim[2];
  size_t total = off[mips] + ((onb + 255) & ~(size_t)255);
  uint8_t *buf = nullptr, *raw = nullptr;
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  cudaError_t e = cudaMalloc(&buf, total + onb);
  if (e != cudaSuccess) return cuda_fail(c, e, "upload_volume: cudaMalloc");
  raw = buf + total;
  e = cudaMemcpyAsync(buf, voxels, (size_t)nx * ny * nz, cudaMemcpyDefault, c->stream);
  for (uint32_t m = 1; m < mips && e == cudaSuccess; m++) {
    size_t n = (size_t)cube.dim[m][0] * cube.dim[m][1] * cube.dim[m][2];
    k_downsample_clamp<<<grid_for(n), 256, 0, c->stream>>>(
        buf + off[m - 1], cube.dim[m - 1][0], cube.dim[m - 1][1], cube.dim[m - 1][2], buf + off[m],
        cube.dim[m][0], cube.dim[m][1], cube.dim[m][2]);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_occ_raw<<<grid_for(onb), 256, 0, c->stream>>>(buf, nx, ny, nz, raw, cube.odim[0],
                                                    cube.odim[1], cube.odim[2]);
    k_occ_dilate<<<grid_for(onb), 256, 0, c->stream>>>(raw, buf + off[mips], cube.odim[0],
                                                       cube.odim[1], cube.odim[2]);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    cudaFree(buf);
    return cuda_fail(c, e, "upload_volume");
  }
  for (uint32_t m = 0; m < mips; m++) cube.lev[m] = buf + off[m];
  cube.occ = buf + off[mips];
  cudaFree(c->cube_buf);
  c->cube_buf = buf;
  c->cube_bytes = total;
  c->have_cube = true;
  c->cube = cube;
  return R3D_OK;
}

int r3d_cuda_set_transfer(r3d_cuda_ctx *c, const uint8_t rgba[256][4]) {
  if (!c || !rgba) return fail(c, R3D_E_INVALID, "set_transfer: bad arguments");
  cudaSetDevice(c->device);
  memcpy(c->lut_host, rgba, sizeof c->lut_host);
  int imin = 256;
  for (int i = 0; i < 256; i++)
    if (rgba[i][3]) {
      imin = i;
      break;
    }
  // TF coordinate t < imin - 1 interpolates two zero-alpha texels
  c->tf_zero_t = (float)(imin - 1);
  R3D_CUDA_TRY(c, cudaMemcpyAsync(c->lut, c->lut_host, sizeof c->lut_host, cudaMemcpyHostToDevice,
                                  c->stream));
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return R3D_OK;
}

int r3d_cuda_set_quality(r3d_cuda_ctx *c, uint32_t quality) {
  if (!c || quality >= R3D_QUALITY_COUNT) return fail(c, R3D_E_INVALID, "set_quality: %u", quality);
  c->quality = quality;
  return R3D_OK;
}

int r3d_cuda_set_slot_trace(r3d_cuda_ctx *c, uint32_t *bits) {
  if (!c) return R3D_E_INVALID;
  if (bits && !is_device_ptr(bits)) return fail(c, R3D_E_INVALID, "set_slot_trace: not device");
  c->slot_bits = bits;
  return R3D_OK;
}

int r3d_cuda_set_alpha_cutoff(r3d_cuda_ctx *c, float cutoff) {
  if (!c || !(cutoff > 0.0f && cutoff <= 1.0f))
    return fail(c, R3D_E_INVALID, "set_alpha_cutoff: %g not in (0, 1]", (double)cutoff);
  c->alpha_cutoff = cutoff;
  return R3D_OK;
}

}  // extern "C"

// Validates a LOD page-table header and decodes it into the kernel's form.
static int decode_header(r3d_cuda_ctx *c, const uint32_t *page, uint32_t words, uint32_t nslots,
                         DevBricks &b) {
  memset(&b, 0, sizeof b);
  if (words < R3D_BRICK_PAGE_HEADER) return fail(c, R3D_E_INVALID, "page table < 64 words");
  uint32_t nlev = page[0];
  if (nlev < 1u || nlev > 15u) return fail(c, R3D_E_INVALID, "page header: %u levels", nlev);
  if (!page[1] || !page[2] || !page[3] || page[1] > 65535u || page[2] > 65535u ||
      page[3] > 65535u)
    return fail(c, R3D_E_INVALID, "page header: bad base shape");
  b.nlev = nlev;
  for (int a = 0; a < 3; a++) b.bs[a] = (float)page[1 + a];
  b.md = fmaxf(b.bs[0], fmaxf(b.bs[1], b.bs[2]));
  for (int a = 0; a < 3; a++) b.bs_hi[a] = fmaxf(b.bs[a] - 0.001f, 0.0f);
  for (uint32_t l = 0; l < nlev; l++) {
    uint32_t off = page[4 + 4 * l], packed = page[5 + 4 * l], scale = page[6 + 4 * l];
    uint32_t bd[3] = {packed & 1023u, (packed >> 10) & 1023u, packed >> 20};
    if (!scale || (scale & (scale - 1u)) || scale > (1u << 20))
      return fail(c, R3D_E_INVALID, "page header: level %u scale %u not a power of two", l, scale);
    if (!bd[0] || !bd[1] || !bd[2] || bd[2] > 1023u)
      return fail(c, R3D_E_INVALID, "page header: level %u empty brick grid", l);
    uint64_t end = (uint64_t)off + (uint64_t)bd[0] * bd[1] * bd[2];
    if (off < R3D_BRICK_PAGE_HEADER || end > words)
      return fail(c, R3D_E_INVALID, "page header: level %u entries out of range", l);
    b.off[l] = off;
    b.scale[l] = scale;
    b.inv_scale[l] = 1.0f / (float)scale;
    for (int a = 0; a < 3; a++) b.bd[l][a] = bd[a];
  }
  b.page_words = words;
  b.nslots = nslots;
  return R3D_OK;
}

// (Re)builds the block-maximum table of the context's slot pool.
int build_blockmax(r3d_cuda_ctx *c) {
  if (c->defer_tables) return R3D_OK;
  cudaFree(c->bmax);
  c->bmax = nullptr;
  size_t n = (size_t)(c->nslots ? c->nslots : 1u) * 4096u;
  R3D_CUDA_TRY(c, cudaMalloc(&c->bmax, n));
  R3D_CUDA_TRY(c, cudaMemsetAsync(c->bmax, 0, n, c->stream));
  cudaFree(c->quad);
  c->quad = nullptr;
  for (int i = 0; i < 4; i++) {  // overlays follow the old slot assignment
    cudaFree(c->ovl_quad[i]);
    c->ovl_quad[i] = nullptr;
    c->br.ovl[i] = nullptr;
    c->ovl_src_on[i] = false;  // a new cache detaches CPU-sourced atlases
    c->ovl_key[i].clear();
  }
  const size_t nq = (size_t)(c->nslots ? c->nslots : 1u) * (128u * 128u * 128u);
  R3D_CUDA_TRY(c, cudaMalloc(&c->quad, nq * sizeof(uint32_t)));
  if (c->nslots) {
    k_slot_blockmax<<<c->nslots, 256, 0, c->stream>>>(c->pool, c->bmax);
    k_slot_quads<<<grid_for(nq), 256, 0, c->stream>>>(c->pool, c->quad, nq);
    R3D_CUDA_TRY(c, cudaGetLastError());
  }
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->br.bmax = c->bmax;
  c->br.quad = c->quad;
  return R3D_OK;
}

uint32_t atlas_bpa(uint32_t nslots) {
  uint32_t a = 1;
  while ((uint64_t)a * a * a < nslots) a++;
  return a;
}

extern "C" {

int r3d_cuda_bricks_build(r3d_cuda_ctx *c, const r3d_volume_desc *d, const uint8_t *voxels,
                          uint32_t nlev, uint32_t min_max) {
  if (!c || !d || !voxels || !d->nx || !d->ny || !d->nz || nlev < 1u || nlev > 15u)
    return fail(c, R3D_E_INVALID, "bricks_build: bad arguments");
  uint32_t nx = d->nx, ny = d->ny, nz = d->nz;
  if (max(nx, max(ny, nz)) > 65535u) return fail(c, R3D_E_INVALID, "bricks_build: too large");
  cudaSetDevice(c->device);
  stream_reset(c);
  cudaStream_t st = c->stream;
  R3D_CUDA_TRY(c, cudaStreamSynchronize(st));
  // level extents: level 0 is the volume itself, level l >= 1 the zero-
  // padded brick grid 128 * ceil(ceil(n / 2^l) / 128)
  uint32_t E[16][3], bd[16][3];
  size_t lev_off[16] = {0}, lev_total = 0;
  uint32_t nb_total = 0;
  for (uint32_t l = 0; l < nlev; l++) {
    uint32_t n3[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) {
      uint32_t dl = (n3[a] + (1u << l) - 1u) >> l;
      bd[l][a] = (dl + 127u) / 128u;
      E[l][a] = l == 0 ? n3[a] : bd[l][a] * 128u;
    }
    if (bd[l][0] > 1023u || bd[l][1] > 1023u || bd[l][2] > 1023u)
      return fail(c, R3D_E_INVALID, "bricks_build: brick grid too large");
    lev_off[l] = lev_total;
    lev_total += ((size_t)E[l][0] * E[l][1] * E[l][2] + 255) & ~(size_t)255;
    nb_total += bd[l][0] * bd[l][1] * bd[l][2];
  }
  uint32_t words = R3D_BRICK_PAGE_HEADER + nb_total;
  uint8_t *lev = nullptr;
  uint32_t *dmax = nullptr, *jobs = nullptr;
  uint8_t *pool = nullptr;
  uint32_t *page = nullptr;
  std::vector<uint32_t> hmax(nb_total), hpage(words, R3D_BRICK_ABSENT);
  std::vector<uint32_t> src_brick, dst_slot;
  int rc = R3D_OK;
  cudaError_t e = cudaMalloc(&lev, lev_total);
  if (e == cudaSuccess) e = cudaMalloc(&dmax, (size_t)nb_total * 4);
  if (e != cudaSuccess) {
    rc = cuda_fail(c, e, "bricks_build: cudaMalloc levels");
    goto out;
  }
  e = cudaMemcpyAsync(lev, voxels, (size_t)nx * ny * nz, cudaMemcpyDefault, st);
  for (uint32_t l = 1; l < nlev && e == cudaSuccess; l++) {
    size_t n = (size_t)E[l][0] * E[l][1] * E[l][2];
    k_downsample_zero<<<grid_for(n), 256, 0, st>>>(lev + lev_off[l - 1], E[l - 1][0], E[l - 1][1],
                                                   E[l - 1][2], lev + lev_off[l], E[l][0], E[l][1],
                                                   E[l][2]);
    e = cudaGetLastError();
  }
  {
    uint32_t moff = 0;
    for (uint32_t l = 0; l < nlev && e == cudaSuccess; l++) {
      uint32_t nb = bd[l][0] * bd[l][1] * bd[l][2];
      k_brick_max<<<nb, 256, 0, st>>>(lev + lev_off[l], E[l][0], E[l][1], E[l][2], bd[l][0],
                                      bd[l][1], dmax + moff);
      e = cudaGetLastError();
      moff += nb;
    }
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hmax.data(), dmax, (size_t)nb_total * 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    rc = cuda_fail(c, e, "bricks_build: pyramid");
    goto out;
  }
  {
    // page table in render3d's format (src/vk/vkbackend.c:4184-4206)
    memset(hpage.data(), 0, R3D_BRICK_PAGE_HEADER * 4);
    hpage[0] = nlev;
    hpage[1] = nx;
    hpage[2] = ny;
    hpage[3] = nz;
    uint32_t off = 0, slot = 0;
    for (uint32_t l = 0; l < nlev; l++) {
      uint32_t nb = bd[l][0] * bd[l][1] * bd[l][2];
      hpage[4 + 4 * l] = R3D_BRICK_PAGE_HEADER + off;
      hpage[5 + 4 * l] = bd[l][0] | (bd[l][1] << 10) | (bd[l][2] << 20);
      hpage[6 + 4 * l] = 1u << l;
      for (uint32_t bi = 0; bi < nb; bi++) {
        uint32_t m = hmax[off + bi];
        if (m >= min_max) {
          hpage[R3D_BRICK_PAGE_HEADER + off + bi] = slot | (m << 24);
          slot++;
        }
      }
      off += nb;
    }
    if (slot >= (1u << 24)) {
      rc = fail(c, R3D_E_INVALID, "bricks_build: %u slots exceed the 24-bit slot field", slot);
      goto out;
    }
    uint32_t nslots = slot;
    size_t pool_bytes = (size_t)(nslots ? nslots : 1u) * (128u * 128u * 128u);
    e = cudaMalloc(&pool, pool_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&page, (size_t)words * 4);
    if (e == cudaSuccess) e = cudaMalloc(&jobs, (size_t)(nslots ? nslots : 1u) * 8);
    if (e != cudaSuccess) {
      rc = cuda_fail(c, e, "bricks_build: cudaMalloc pool");
      goto out;
    }
    off = 0;
    uint32_t joff = 0;
    std::vector<uint32_t> hj;
    hj.reserve((size_t)nslots * 2);
    std::vector<uint32_t> lvl_count(nlev, 0);
    for (uint32_t l = 0; l < nlev; l++) {
      uint32_t nb = bd[l][0] * bd[l][1] * bd[l][2];
      for (uint32_t bi = 0; bi < nb; bi++) {
        uint32_t en = hpage[R3D_BRICK_PAGE_HEADER + off + bi];
        if (en != R3D_BRICK_ABSENT) {
          src_brick.push_back(bi);
          dst_slot.push_back(en & 0xFFFFFFu);
          lvl_count[l]++;
        }
      }
      off += nb;
    }
    if (nslots) {
      e = cudaMemcpyAsync(jobs, src_brick.data(), (size_t)nslots * 4, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(jobs + nslots, dst_slot.data(), (size_t)nslots * 4,
                            cudaMemcpyHostToDevice, st);
    }
    for (uint32_t l = 0; l < nlev && e == cudaSuccess; l++) {
      uint32_t n = lvl_count[l];
      if (!n) continue;
      for (uint32_t j0 = 0; j0 < n && e == cudaSuccess; j0 += 65535u) {
        uint32_t nj = min(n - j0, 65535u);
        k_brick_copy<<<dim3(128, nj), 256, 0, st>>>(lev + lev_off[l], E[l][0], E[l][1], E[l][2],
                                                    bd[l][0], bd[l][1], jobs + joff + j0,
                                                    jobs + nslots + joff + j0, pool);
        e = cudaGetLastError();
      }
      joff += n;
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(page, hpage.data(), (size_t)words * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      rc = cuda_fail(c, e, "bricks_build: slot copy");
      goto out;
    }
    DevBricks b;
    rc = decode_header(c, hpage.data(), words, nslots, b);
    if (rc != R3D_OK) goto out;
    b.page = page;
    b.pool = pool;
    cudaFree(c->page);
    cudaFree(c->pool);
    c->page = page;
    c->pool = pool;
    page = nullptr;
    pool = nullptr;
    c->page_words = words;
    c->nslots = nslots;
    c->abpa = atlas_bpa(nslots);
    c->shape[0] = nx;
    c->shape[1] = ny;
    c->shape[2] = nz;
    c->br = b;
    c->have_bricks = false;
    // the display filter, before the tables that derive from the slots (a
    // build whose pool becomes a streaming store stays unfiltered: its
    // bricks are filtered when uploaded)
    if (!c->defer_tables && postfilter_on(c, 0u)) {
      std::vector<uint32_t> all(nslots);
      for (uint32_t s = 0; s < nslots; s++) all[s] = s;
      rc = postfilter_slots(c, 0u, c->pool, all.data(), nslots);
      if (rc != R3D_OK) goto out;
    }
    rc = build_blockmax(c);
    if (rc != R3D_OK) goto out;
    c->have_bricks = true;
  }
out:
  cudaFree(lev);
  cudaFree(dmax);
  cudaFree(jobs);
  cudaFree(pool);
  cudaFree(page);
  return rc;
}

int r3d_cuda_bricks_load(r3d_cuda_ctx *c, const uint32_t *page, uint32_t page_words,
                         const uint8_t *slots, uint32_t nslots) {
  if (!c || !page || (!slots && nslots)) return fail(c, R3D_E_INVALID, "bricks_load: bad args");
  if (nslots >= (1u << 24)) return fail(c, R3D_E_INVALID, "bricks_load: too many slots");
  stream_reset(c);
  DevBricks b;
  int rc = decode_header(c, page, page_words, nslots, b);
  if (rc != R3D_OK) return rc;
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  uint32_t *dpage = nullptr;
  uint8_t *dpool = nullptr;
  size_t pool_bytes = (size_t)(nslots ? nslots : 1u) * (128u * 128u * 128u);
  cudaError_t e = cudaMalloc(&dpage, (size_t)page_words * 4);
  if (e == cudaSuccess) e = cudaMalloc(&dpool, pool_bytes);
  if (e == cudaSuccess) e = copy_sync(c->stream, dpage, page, (size_t)page_words * 4);
  if (e == cudaSuccess && nslots)
    e = copy_sync(c->stream, dpool, slots, (size_t)nslots * (128u * 128u * 128u));
  if (e != cudaSuccess) {
    cudaFree(dpage);
    cudaFree(dpool);
    return cuda_fail(c, e, "bricks_load");
  }
  b.page = dpage;
  b.pool = dpool;
  cudaFree(c->page);
  cudaFree(c->pool);
  c->page = dpage;
  c->pool = dpool;
  c->page_words = page_words;
  c->nslots = nslots;
  c->abpa = atlas_bpa(nslots);
  c->shape[0] = page[1];
  c->shape[1] = page[2];
  c->shape[2] = page[3];
  c->br = b;
  c->have_bricks = false;
  rc = build_blockmax(c);
  if (rc != R3D_OK) return rc;
  c->have_bricks = true;
  return R3D_OK;
}

uint32_t r3d_cuda_brick_mode(const r3d_cuda_ctx *c) {
  if (!c || !c->have_bricks) return 0u;
  return c->abpa | (c->br.nlev << 8) | R3D_BRICK_LOD_FLAG;
}

int r3d_cuda_bricks_info(const r3d_cuda_ctx *c, uint32_t *page_words, uint32_t *nslots,
                         uint32_t shape[3], uint32_t *nlev) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_bricks) return R3D_E_STATE;
  if (page_words) *page_words = c->page_words;
  if (nslots) *nslots = c->nslots;
  if (shape) memcpy(shape, c->shape, sizeof c->shape);
  if (nlev) *nlev = c->br.nlev;
  return R3D_OK;
}

int r3d_cuda_bricks_read(r3d_cuda_ctx *c, uint32_t *page, uint8_t *slots) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_bricks) return fail(c, R3D_E_STATE, "bricks_read: no bricks");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (page) R3D_CUDA_TRY(c, cudaMemcpy(page, c->page, (size_t)c->page_words * 4, cudaMemcpyDefault));
  if (slots && c->nslots)
    R3D_CUDA_TRY(c, cudaMemcpy(slots, c->pool, (size_t)c->nslots * (128u * 128u * 128u),
                               cudaMemcpyDefault));
  return R3D_OK;
}

int r3d_cuda_cube_read(r3d_cuda_ctx *c, int level, uint8_t *out, uint32_t dims[3]) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_cube) return fail(c, R3D_E_STATE, "cube_read: no volume");
  const DevCube &cb = c->cube;
  const uint8_t *src;
  uint32_t d[3];
  if (level < 0) {
    src = cb.occ;
    memcpy(d, cb.odim, sizeof d);
  } else {
    if ((uint32_t)level >= cb.nlevels) return fail(c, R3D_E_INVALID, "cube_read: level");
    src = cb.lev[level];
    memcpy(d, cb.dim[level], sizeof d);
  }
  if (dims) memcpy(dims, d, sizeof d);
  if (out) {
    cudaSetDevice(c->device);
    R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    R3D_CUDA_TRY(c, cudaMemcpy(out, src, (size_t)d[0] * d[1] * d[2], cudaMemcpyDefault));
  }
  return R3D_OK;
}

}  // extern "C"

// The view's rectangle clipped to the image (src/vk/vkbackend.c:6871-6900):
// 1 to render, 0 when nothing of it is inside.
static int view_rect(const r3d_frame_params &in, uint32_t out_w, uint32_t out_h,
                     r3d_frame_params &pc) {
  uint32_t ox = in.view_org & 0xffffu, oy = (in.view_org >> 16) & 0xffffu;
  uint32_t vw = in.viewport[0] ? in.viewport[0] : out_w;
  uint32_t vh = in.viewport[1] ? in.viewport[1] : out_h;
  bool ok = ox < out_w && oy < out_h;
  if (ok) {
    vw = min(vw, out_w - ox);
    vh = min(vh, out_h - oy);
    ok = vw && vh;
  }
  pc.view_org = ox | (oy << 16);
  pc.viewport[0] = ok ? vw : 0u;
  pc.viewport[1] = ok ? vh : 0u;
  return ok ? 1 : 0;
}

// Validates and sanitizes one view against the image.  Returns 1 to render,
// 0 to skip, < 0 error.
int prepare_view(r3d_cuda_ctx *c, const r3d_frame_params &in, uint32_t out_w,
                        uint32_t out_h, r3d_frame_params &pc) {
  pc = in;
  if (in.mode >= R3D_MODE_COUNT) return fail(c, R3D_E_INVALID, "view: mode %u", in.mode);
  if (in.view_flags & R3D_VIEW_SURF) {  // flattened segment: the view must describe the window
    if (!c->sv_vol || !c->sv_baked)
      return fail(c, R3D_E_STATE, "view: no baked surface volume (r3d_cuda_surfvol_window)");
    r3d_frame_params ref = in;
    r3d_cuda_surfvol_params(c, &ref);
    if (in.slab_x0 != ref.slab_x0 || in.slab_y0 != ref.slab_y0 || in.slab_px != ref.slab_px ||
        in.slab_nx != ref.slab_nx || in.slab_ny != ref.slab_ny || in.slab_wz != ref.slab_wz ||
        in.slab_grid != ref.slab_grid || in.max_mip != ref.max_mip ||
        in.vol_tx != ref.vol_tx || in.vol_ty != ref.vol_ty)
      return fail(c, R3D_E_INVALID, "view: surface parameters do not match the baked window "
                                    "(r3d_cuda_surfvol_params)");
    if (!(in.step_voxels > 0.0f)) return fail(c, R3D_E_INVALID, "view: step_voxels must be > 0");
    return view_rect(in, out_w, out_h, pc);
  }
  if (in.clip_valid) {  // clipmap: the view must describe the loaded levels
    if (!c->have_clip) return fail(c, R3D_E_STATE, "view: no clipmap loaded");
    r3d_frame_params ref;
    memset(&ref, 0, sizeof ref);
    r3d_cuda_clip_params(c, &ref);
    if (in.clip_valid != ref.clip_valid || in.slab_z0 != ref.slab_z0 ||
        in.slab_nx != ref.slab_nx || in.slab_ny != ref.slab_ny || in.slab_wz != ref.slab_wz ||
        memcmp(in.clip_orig, ref.clip_orig, sizeof ref.clip_orig) || in.brick_mode ||
        in.slab_grid)
      return fail(c, R3D_E_INVALID, "view: clipmap parameters do not match the loaded levels "
                                    "(r3d_cuda_clip_params)");
    if (in.slab_depth < 1u || in.slab_depth > in.slab_wz)
      return fail(c, R3D_E_INVALID, "view: slab_depth %u not in [1, %u]", in.slab_depth,
                  in.slab_wz);
    if (in.overlay_flags & kOvlAtlases)
      return fail(c, R3D_E_UNSUPPORTED, "view: overlay atlases need the LOD brick cache");
  } else if (in.slab_grid & kVslabGrid) {  // virtual slab: the view must describe the window
    if (!c->have_vslab) return fail(c, R3D_E_STATE, "view: no virtual slab loaded");
    r3d_frame_params ref;
    memset(&ref, 0, sizeof ref);
    r3d_cuda_vslab_params(c, &ref);
    if (in.slab_grid != ref.slab_grid || in.brick_mode != ref.brick_mode ||
        in.slab_wz != ref.slab_wz || in.slab_z0 != ref.slab_z0 || in.slab_nx != ref.slab_nx ||
        in.slab_ny != ref.slab_ny || in.slab_px != ref.slab_px || in.slab_py != ref.slab_py ||
        in.slab_x0 != ref.slab_x0 || in.slab_y0 != ref.slab_y0)
      return fail(c, R3D_E_INVALID, "view: virtual-slab parameters do not match the loaded "
                                    "window (r3d_cuda_vslab_params)");
    if (in.slab_depth < 1u || in.slab_depth > c->vsl.D)
      return fail(c, R3D_E_INVALID, "view: slab_depth %u not in [1, %u]", in.slab_depth,
                  c->vsl.D);
    if (in.overlay_flags & kOvlAtlases)
      return fail(c, R3D_E_UNSUPPORTED, "view: overlay atlases need the LOD brick cache");
  } else if (in.slab_grid) {  // tiled slab: the view must describe the loaded window
    if (!c->have_slab) return fail(c, R3D_E_STATE, "view: no slab loaded");
    r3d_frame_params ref;
    memset(&ref, 0, sizeof ref);
    r3d_cuda_slab_params(c, &ref);
    if (in.slab_grid != ref.slab_grid || in.slab_wz != ref.slab_wz ||
        in.slab_z0 != ref.slab_z0 || in.slab_nx != ref.slab_nx || in.slab_ny != ref.slab_ny ||
        in.slab_px != ref.slab_px || in.slab_py != ref.slab_py || in.brick_mode)
      return fail(c, R3D_E_INVALID, "view: slab parameters do not match the loaded window "
                                    "(r3d_cuda_slab_params)");
    if (in.slab_depth < 1u || in.slab_depth > in.slab_wz - 1u)
      return fail(c, R3D_E_INVALID, "view: slab_depth %u not in [1, %u]", in.slab_depth,
                  in.slab_wz - 1u);
    if (in.overlay_flags & kOvlAtlases)
      return fail(c, R3D_E_UNSUPPORTED, "view: overlay atlases need the LOD brick cache");
  }
  if (in.overlay_flags & kOvlAtlases) {
    if (!(in.brick_mode & R3D_BRICK_LOD_FLAG))
      return fail(c, R3D_E_UNSUPPORTED, "view: overlay atlases need the LOD brick cache");
    static const char *names[4] = {"ink", "3D ink", "labels", "registration"};
    const uint32_t bit[4] = {kOvlInk, kOvlInk3d, kOvlLabels, kOvlReg};
    for (int i = 0; i < 4; i++)
      if ((in.overlay_flags & bit[i]) && !c->ovl_quad[i])
        return fail(c, R3D_E_STATE, "view: overlay atlas '%s' is not loaded", names[i]);
  }
  if (!(in.max_mip >= 0.0f)) return fail(c, R3D_E_INVALID, "view: max_mip must be >= 0");
  if (!(in.step_voxels > 0.0f)) return fail(c, R3D_E_INVALID, "view: step_voxels must be > 0");
  if (in.slab_grid & kVslabGrid) {
    // brick_mode holds the pyramid grids (checked above)
  } else if (in.brick_mode & R3D_BRICK_LOD_FLAG) {
    if (!c->have_bricks) return fail(c, R3D_E_STATE, "view: no brick cache loaded");
  } else if (in.brick_mode) {
    if (!c->have_shard) return fail(c, R3D_E_STATE, "view: no single-level brick atlas loaded");
    if (in.brick_mode != r3d_cuda_shard_mode(c))
      return fail(c, R3D_E_INVALID, "view: brick_mode 0x%x does not match the atlas (0x%x)",
                  in.brick_mode, r3d_cuda_shard_mode(c));
  } else if (!in.slab_grid && !in.clip_valid && !c->have_cube) {
    return fail(c, R3D_E_STATE, "view: no volume uploaded");
  }
  return view_rect(in, out_w, out_h, pc);
}

// Persistent launches for the renderable views of one call: views sharing a
// sampling path and mode go into one launch (template parameters of the
// kernel), in order of first appearance.
static int launch_views_persistent(r3d_cuda_ctx *c, uint32_t persistent,
                                   const r3d_frame_params *pcs, const int *render,
                                   uint32_t nviews, uint8_t *const *imgs,
                                   const uint32_t *strides, uint32_t *steps, uint32_t *mip,
                                   unsigned long long *total, unsigned long long *counters,
                                   cudaStream_t st) {
  const int k = c->ring_next;
  c->ring_next = (k + 1) % r3d_cuda_ctx::kRing;
  if (c->ring_used[k]) R3D_CUDA_TRY(c, cudaEventSynchronize(c->ring_ev[k]));
  DevView *hv = c->ring_host + (size_t)k * kMaxBatchViews;
  DevView *dv = c->ring_dev + (size_t)k * kMaxBatchViews;
  uint32_t *queue = c->ring_queue + (size_t)k * 2 * kMaxBatchViews;  // two words per group
  const r3d_cuda_schedule &sc = c->sched;
  // group views by (path, mode)
  uint32_t order[64], group_of[64], ngroups = 0, gkey[64], gstart[65], gcount[64];
  uint32_t n = 0;
  for (uint32_t v = 0; v < nviews; v++) {
    if (!render[v]) continue;
    uint32_t key = (uint32_t)path_of_view(pcs[v]) * 8u | pcs[v].mode;
    uint32_t g = 0;
    while (g < ngroups && gkey[g] != key) g++;
    if (g == ngroups) {
      gkey[ngroups] = key;
      gcount[ngroups] = 0;
      ngroups++;
    }
    group_of[n] = g;
    order[n++] = v;
    gcount[g]++;
  }
  if (!n) return R3D_OK;
  gstart[0] = 0;
  for (uint32_t g = 0; g < ngroups; g++) gstart[g + 1] = gstart[g] + gcount[g];
  uint32_t fill[64] = {0}, ntiles[64] = {0};
  for (uint32_t i = 0; i < n; i++) {
    uint32_t g = group_of[i], slot = gstart[g] + fill[g]++;
    DevView &d = hv[slot];
    memset(&d, 0, sizeof d);
    d.pc = pcs[order[i]];
    d.img = (uchar4 *)imgs[order[i]];
    d.stride = strides[order[i]];
    d.tile_begin = ntiles[g];
    ntiles[g] += view_tiles(d, persistent == 2u ? 0u : sc.tile_shape);
  }
  R3D_CUDA_TRY(c, cudaMemcpyAsync(dv, hv, sizeof(DevView) * n, cudaMemcpyHostToDevice, st));
  R3D_CUDA_TRY(c, cudaEventRecord(c->ring_ev[k], st));
  c->ring_used[k] = true;
  R3D_CUDA_TRY(c, cudaMemsetAsync(queue, 0, sizeof(uint32_t) * 2 * ngroups, st));
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
  const DevScene s = c->scene();
  if (persistent == 2u) {  // whole tiles, the views as launch parameters
    for (uint32_t g = 0; g < ngroups; g++) {
      TilesLaunch T;
      memset(&T, 0, sizeof T);
      T.views = hv + gstart[g];
      T.nviews = gcount[g];
      T.ntiles = ntiles[g];
      T.scenes = &s;
      T.luts = &c->lut;
      T.nscenes = 1u;
      T.queue = queue + 2 * g;
      T.steps = steps;
      T.mip = mip;
      T.total = total;
      T.counters = counters;
      T.blocks = sc.blocks_per_sm * (uint32_t)dev_sms;
      T.mode = gkey[g] & 7u;
      T.fast = c->quality == R3D_QUALITY_FAST;
      T.path = (int)(gkey[g] >> 3);
      cudaError_t e = launch_tiles(T, st);
      if (e != cudaSuccess) return cuda_fail(c, e, "raycast_fwd: whole-tile launch");
    }
    return R3D_OK;
  }
  for (uint32_t g = 0; g < ngroups; g++) {
    PersistLaunch L;
    memset(&L, 0, sizeof L);
    L.views = dv + gstart[g];
    L.nviews = gcount[g];
    L.ntiles = ntiles[g];
    L.lut = c->lut;
    L.queue = queue + 2 * g;
    L.refill_min = sc.refill_min;
    L.shape = sc.tile_shape;
    L.unroll = sc.unroll;
    L.steps = steps;
    L.mip = mip;
    L.total = total;
    L.counters = counters;
    L.mode = gkey[g] & 7u;
    L.fast = c->quality == R3D_QUALITY_FAST;
    L.path = (int)(gkey[g] >> 3);
    int per_sm = sc.blocks_per_sm
                     ? (int)sc.blocks_per_sm
                     : persist_blocks_per_sm(L.path, L.mode, L.fast, L.unroll);
    // no more blocks than there are tiles for their warps
    uint32_t want = (uint32_t)per_sm * (uint32_t)dev_sms;
    uint32_t cap = (L.ntiles + 3u) / 4u;
    L.blocks = want < cap ? want : (cap ? cap : 1u);
    cudaError_t e = launch_persist(L, s, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "raycast_fwd: persistent launch");
  }
  return R3D_OK;
}

// One colour into every pixel of an RGBA8 image (grid-stride).
__global__ void k_fill_rgba(uchar4 *__restrict__ img, size_t npix, uchar4 col) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix;
       i += (size_t)gridDim.x * blockDim.x)
    img[i] = col;
}

extern "C" {

int r3d_cuda_set_schedule(r3d_cuda_ctx *c, const r3d_cuda_schedule *sc) {
  if (!c || !sc || sc->persistent > 3u || sc->staging > 1u || sc->refill_min < 1u || sc->refill_min > 32u ||
      sc->tile_shape > 2u || (sc->unroll != 1u && sc->unroll != 2u) || sc->shade_group > 32u ||
      sc->blocks_per_sm > 32u)
    return fail(c, R3D_E_INVALID, "set_schedule: bad schedule");
  c->sched = *sc;
  return R3D_OK;
}

int r3d_cuda_get_schedule(const r3d_cuda_ctx *c, r3d_cuda_schedule *sc) {
  if (!c || !sc) return R3D_E_INVALID;
  *sc = c->sched;
  return R3D_OK;
}

int r3d_cuda_raycast_rows(r3d_cuda_ctx *c, const r3d_frame_params *view, uint8_t *rgba_out,
                          uint32_t out_w, uint32_t out_h, uint32_t row0, uint32_t row1,
                          void *stream) {
  if (!c || !view || !rgba_out || !out_w || !out_h || out_w > 65535u || out_h > 65535u)
    return fail(c, R3D_E_INVALID, "raycast_rows: bad arguments");
  if (!is_device_ptr(rgba_out))
    return fail(c, R3D_E_INVALID, "raycast_rows: the image must be device memory");
  if (view->view_flags & R3D_VIEW_SURF)
    return fail(c, R3D_E_UNSUPPORTED, "raycast_rows: surface views render whole");
  cudaSetDevice(c->device);
  r3d_frame_params pc;
  const int rc = prepare_view(c, *view, out_w, out_h, pc);
  if (rc <= 0) return rc;
  Rows rows;
  rows.row0 = row0;
  rows.row1 = row1;
  R3D_CUDA_TRY(c, launch_view(c, pc, rgba_out, out_w, nullptr, nullptr, nullptr, nullptr,
                              stream ? (cudaStream_t)stream : c->stream, rows));
  return R3D_OK;
}

int r3d_cuda_raycast_fwd(r3d_cuda_ctx *c, const r3d_frame_params *views, uint32_t nviews,
                         uint8_t *rgba_out, uint32_t out_w, uint32_t out_h,
                         const r3d_cuda_aux *aux, void *stream) {
  if (!c || !views || !nviews || nviews > 64u || !rgba_out || !out_w || !out_h ||
      out_w > 65535u || out_h > 65535u)
    return fail(c, R3D_E_INVALID, "raycast_fwd: bad arguments");
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  r3d_frame_params pcs[64];
  int render[64];
  for (uint32_t v = 0; v < nviews; v++) {
    render[v] = prepare_view(c, views[v], out_w, out_h, pcs[v]);
    if (render[v] < 0) return render[v];
  }
  bool host = !is_device_ptr(rgba_out);
  size_t npix = (size_t)out_w * out_h;
  uint8_t *img = rgba_out;
  uint32_t *steps = aux ? aux->steps : nullptr, *mip = aux ? aux->mip_index : nullptr;
  unsigned long long *total = aux ? aux->total_steps : nullptr;
  unsigned long long *counters = aux ? aux->counters : nullptr;
  if (host) {
    if (c->img_cap < npix * 4) {
      cudaFree(c->img);
      c->img = nullptr;
      c->img_cap = 0;
      R3D_CUDA_TRY(c, cudaMalloc(&c->img, npix * 4));
      c->img_cap = npix * 4;
    }
    img = c->img;
    // pixels outside every view keep the caller's contents
    R3D_CUDA_TRY(c, cudaMemcpyAsync(img, rgba_out, npix * 4, cudaMemcpyHostToDevice, st));
    if (steps || mip) {
      if (c->aux_cap < npix * 2) {
        cudaFree(c->aux_buf);
        c->aux_buf = nullptr;
        c->aux_cap = 0;
        R3D_CUDA_TRY(c, cudaMalloc(&c->aux_buf, npix * 2 * 4));
        c->aux_cap = npix * 2;
      }
      steps = steps ? c->aux_buf : nullptr;
      mip = mip ? c->aux_buf + npix : nullptr;
      if (steps)
        R3D_CUDA_TRY(c, cudaMemcpyAsync(steps, aux->steps, npix * 4, cudaMemcpyHostToDevice, st));
      if (mip)
        R3D_CUDA_TRY(c,
                     cudaMemcpyAsync(mip, aux->mip_index, npix * 4, cudaMemcpyHostToDevice, st));
    }
    if (total || counters) {
      R3D_CUDA_TRY(c, cudaMemsetAsync(c->total, 0, (R3D_COUNTERS + 1) * 8, st));
      total = total ? c->total : nullptr;
      counters = counters ? c->total + 1 : nullptr;
    }
  }
  R3D_CUDA_TRY(c, cudaEventRecord(c->ev0, st));
  // views with overlay atlases and flattened-segment views render through
  // their own grid kernels
  bool any_ovl = false;
  for (uint32_t v = 0; v < nviews; v++)
    any_ovl = any_ovl || (render[v] && ((pcs[v].overlay_flags & kOvlAtlases) ||
                                        (pcs[v].view_flags & R3D_VIEW_SURF)));
  uint32_t nrender = 0;
  for (uint32_t v = 0; v < nviews; v++) nrender += render[v] ? 1u : 0u;
  const uint32_t persistent = resolved_persistent(c->sched, nrender);
  if (persistent && !any_ovl) {
    uint8_t *imgs[64];
    uint32_t strides[64];
    for (uint32_t v = 0; v < nviews; v++) {
      imgs[v] = img;
      strides[v] = out_w;
    }
    int rc = launch_views_persistent(c, persistent, pcs, render, nviews, imgs, strides, steps,
                                     mip, total, counters, st);
    if (rc != R3D_OK) return rc;
  } else {
    for (uint32_t v = 0; v < nviews; v++) {
      if (!render[v]) continue;
      cudaError_t e = launch_view(c, pcs[v], img, out_w, steps, mip, total, counters, st);
      if (e != cudaSuccess) return cuda_fail(c, e, "raycast_fwd: launch");
    }
  }
  R3D_CUDA_TRY(c, cudaEventRecord(c->ev1, st));
  c->timed = true;
  if (host) {
    R3D_CUDA_TRY(c, cudaMemcpyAsync(rgba_out, img, npix * 4, cudaMemcpyDeviceToHost, st));
    if (steps)
      R3D_CUDA_TRY(c, cudaMemcpyAsync(aux->steps, steps, npix * 4, cudaMemcpyDeviceToHost, st));
    if (mip)
      R3D_CUDA_TRY(c, cudaMemcpyAsync(aux->mip_index, mip, npix * 4, cudaMemcpyDeviceToHost, st));
    unsigned long long tsum[R3D_COUNTERS + 1] = {0};
    if (total || counters)
      R3D_CUDA_TRY(c, cudaMemcpyAsync(tsum, c->total, sizeof tsum, cudaMemcpyDeviceToHost, st));
    R3D_CUDA_TRY(c, cudaStreamSynchronize(st));
    if (total) *aux->total_steps += tsum[0];
    if (counters)
      for (int k = 0; k < R3D_COUNTERS; k++) aux->counters[k] += tsum[1 + k];
  }
  return R3D_OK;
}

int r3d_cuda_fill_rgba(r3d_cuda_ctx *c, uint8_t *img, size_t npix, const uint8_t rgba[4],
                       void *stream) {
  if (!c || !img || !rgba) return fail(c, R3D_E_INVALID, "fill_rgba: bad arguments");
  if (!npix) return R3D_OK;
  R3D_CUDA_TRY(c, cudaSetDevice(c->device));
  if (!is_device_ptr(img)) return fail(c, R3D_E_INVALID, "fill_rgba: the image must be device memory");
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const uchar4 col = make_uchar4(rgba[0], rgba[1], rgba[2], rgba[3]);
  const uint32_t blocks = (uint32_t)std::min<size_t>((npix + 255u) / 256u, 148u * 16u);
  k_fill_rgba<<<blocks, 256, 0, st>>>((uchar4 *)img, npix, col);
  R3D_CUDA_TRY(c, cudaGetLastError());
  return R3D_OK;
}

int r3d_cuda_raycast_batch(r3d_cuda_ctx *c, const r3d_cuda_request *reqs, uint32_t n,
                           unsigned long long *total_steps, void *stream) {
  if (!c || !reqs || !n || n > kMaxBatchViews)
    return fail(c, R3D_E_INVALID, "raycast_batch: 1..%u requests", kMaxBatchViews);
  R3D_CUDA_TRY(c, cudaSetDevice(c->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  r3d_frame_params pcs[kMaxBatchViews];
  int render[kMaxBatchViews];
  uint8_t *imgs[kMaxBatchViews];
  uint32_t strides[kMaxBatchViews];
  bool any_ovl = false;
  for (uint32_t i = 0; i < n; i++) {
    const r3d_frame_params &v = reqs[i].view;
    if (!reqs[i].rgba || !v.viewport[0] || !v.viewport[1] || v.view_org)
      return fail(c, R3D_E_INVALID, "raycast_batch: request %u needs an image, a viewport and "
                                    "view_org 0", i);
    if (!is_device_ptr(reqs[i].rgba))
      return fail(c, R3D_E_INVALID, "raycast_batch: request %u image is not device memory", i);
    render[i] = prepare_view(c, v, v.viewport[0], v.viewport[1], pcs[i]);
    if (render[i] < 0) return render[i];
    imgs[i] = reqs[i].rgba;
    strides[i] = pcs[i].viewport[0];
    any_ovl = any_ovl || (pcs[i].overlay_flags & kOvlAtlases) || (pcs[i].view_flags & R3D_VIEW_SURF);
  }
  uint32_t nrender = 0;
  for (uint32_t i = 0; i < n; i++) nrender += render[i] ? 1u : 0u;
  const uint32_t persistent = resolved_persistent(c->sched, nrender);
  if (persistent && !any_ovl)
    return launch_views_persistent(c, persistent, pcs, render, n, imgs, strides, nullptr,
                                   nullptr, total_steps, nullptr, st);
  for (uint32_t i = 0; i < n; i++) {
    if (!render[i]) continue;
    cudaError_t e = launch_view(c, pcs[i], imgs[i], strides[i], nullptr, nullptr, total_steps,
                                nullptr, st);
    if (e != cudaSuccess) return cuda_fail(c, e, "raycast_batch: launch");
  }
  return R3D_OK;
}

int r3d_cuda_last_kernel_ns(r3d_cuda_ctx *c, uint64_t *ns) {
  if (!c || !ns) return R3D_E_INVALID;
  if (!c->timed) return fail(c, R3D_E_STATE, "last_kernel_ns: nothing timed");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaEventSynchronize(c->ev1));
  float ms = 0.0f;
  R3D_CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  *ns = (uint64_t)((double)ms * 1e6);
  return R3D_OK;
}

}  // extern "C"

