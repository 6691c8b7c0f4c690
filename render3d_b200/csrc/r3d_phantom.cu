// Seeded scroll phantom generated on the device (same construction as
// r3d_host_phantom: Archimedean spiral sheets about the z axis, normals from
// splitmix64 of (seed, voxel index) through Box-Muller), for volumes too
// large to generate quickly on the host.  The transcendentals are CUDA's
// double-precision ones, so a voxel whose value falls within rounding of a
// .5 boundary, or on a sheet edge, can differ from the host generator's.
#include "r3d_host.h"
#include "r3d_internal.h"

namespace r3d {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__global__ void k_phantom_mask(uint32_t nx, uint32_t ny, r3d_phantom_desc d,
                               uint8_t *__restrict__ mask) {
  const double two_pi = 6.283185307179586;
  size_t n = (size_t)nx * ny;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t x = (uint32_t)(i % nx), y = (uint32_t)(i / nx);
    double dx = x + 0.5 - 0.5 * nx, dy = y + 0.5 - 0.5 * ny;
    double r = sqrt(dx * dx + dy * dy);
    double th = atan2(dy, dx);
    if (th < 0.0) th += two_pi;
    double m = fmod(r - d.r0 - d.pitch * th / two_pi, (double)d.pitch);
    if (m < 0.0) m += d.pitch;
    double dist = m < d.pitch - m ? m : d.pitch - m;
    mask[i] = dist < d.sheet_half && r >= d.r0 && r < d.radius;
  }
}

__global__ void k_phantom(uint32_t nx, uint32_t ny, uint32_t nz, r3d_phantom_desc d,
                          const uint8_t *__restrict__ mask, uint8_t *__restrict__ vox) {
  const double two_pi = 6.283185307179586;
  const size_t n = (size_t)nx * ny * nz, slice = (size_t)nx * ny;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n;
       idx += (size_t)gridDim.x * blockDim.x) {
    uint64_t h1 = splitmix64(d.seed ^ ((uint64_t)idx * 2u));
    uint64_t h2 = splitmix64(d.seed ^ ((uint64_t)idx * 2u + 1u));
    double u1 = ((double)(h1 >> 11) + 1.0) * 0x1.0p-53;
    double u2 = (double)(h2 >> 11) * 0x1.0p-53;
    double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincos(two_pi * u2, &s, &c);
    int pap = mask[idx % slice];
    double mean = pap ? d.in_mean : d.air_mean, sd = pap ? d.in_sd : d.air_sd;
    double v = floor(mean + sd * (rad * c) + d.noise_sd * (rad * s) + 0.5);
    vox[idx] = (uint8_t)(v < 0.0 ? 0.0 : (v > 255.0 ? 255.0 : v));
  }
}

}  // namespace r3d

extern "C" int r3d_cuda_phantom(r3d_cuda_ctx *c, const r3d_phantom_desc *d, uint32_t nx,
                                uint32_t ny, uint32_t nz, uint8_t *vox, void *stream) {
  if (!c || !d || !vox || !nx || !ny || !nz || !(d->pitch > 0.0f))
    return r3d::fail(c, R3D_E_INVALID, "phantom: bad arguments");
  cudaSetDevice(c->device);
  if (!r3d::is_device_ptr(vox)) return r3d::fail(c, R3D_E_INVALID, "phantom: vox not device");
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  uint8_t *mask = nullptr;
  R3D_CUDA_TRY(c, cudaMallocAsync(&mask, (size_t)nx * ny, st));
  r3d::k_phantom_mask<<<1024, 256, 0, st>>>(nx, ny, *d, mask);
  r3d::k_phantom<<<148 * 16, 256, 0, st>>>(nx, ny, nz, *d, mask, vox);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(mask, st);
  if (e != cudaSuccess) return r3d::cuda_fail(c, e, "phantom: launch");
  R3D_CUDA_TRY(c, cudaStreamSynchronize(st));
  return R3D_OK;
}
