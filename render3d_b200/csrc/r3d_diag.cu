// Diagnostic entry point: evaluates the raycast's log2 / exp2 / pow on the
// device so tests can check them bit for bit against the CPU build.
#include "r3d_internal.h"

namespace r3d {

__global__ void k_fmath(const float *__restrict__ x, const float *__restrict__ y,
                        float *__restrict__ out, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[4 * i + 0] = r3d_log2f(x[i]);
  out[4 * i + 1] = r3d_exp2f(x[i]);
  out[4 * i + 2] = r3d_powf(x[i], y[i]);
  out[4 * i + 3] = r3d_powi24f(x[i]);
}

}  // namespace r3d

extern "C" int r3d_cuda_fmath_eval(r3d_cuda_ctx *c, const float *x, const float *y, float *out,
                                   uint32_t n) {
  if (!c || !x || !y || !out || !n) return R3D_E_INVALID;
  cudaSetDevice(c->device);
  float *d = nullptr;
  size_t b = (size_t)n * 4;
  R3D_CUDA_TRY(c, cudaMalloc(&d, b * 6));
  cudaError_t e = cudaMemcpyAsync(d, x, b, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + n, y, b, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    r3d::k_fmath<<<(n + 255) / 256, 256, 0, c->stream>>>(d, d + n, d + 2 * (size_t)n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d + 2 * (size_t)n, b * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return r3d::cuda_fail(c, e, "fmath_eval");
  return R3D_OK;
}
