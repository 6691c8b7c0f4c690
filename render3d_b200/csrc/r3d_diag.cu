// Diagnostic entry points: the raycast's log2 / exp2 / pow evaluated on the
// device (so tests can check them bit for bit against the CPU build), and
// an L2-resident read probe whose bandwidth is the denominator of the
// raycast's L2 roofline.
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

// Reads a buffer that fits in L2 `passes` times through L2 (ld.global.cg:
// no L1 allocation), 16 bytes per thread per load, and keeps a checksum so
// the loads are not removed.  Block b starts its sweep at a different
// offset so that every L2 slice serves every pass.
__global__ void k_l2_read(const uint4 *__restrict__ buf, size_t n16, uint32_t passes,
                          uint32_t *__restrict__ sink) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t start = ((size_t)blockIdx.x * 977u * blockDim.x) % n16;
  uint32_t acc = 0;
  for (uint32_t p = 0; p < passes; p++)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += stride) {
      size_t j = i + start;
      if (j >= n16) j -= n16;
      const uint4 v = __ldcg(buf + j);
      acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
  if (acc == 0x9e3779b9u) sink[0] = acc;  // practically never taken
}

}  // namespace r3d

extern "C" int r3d_cuda_l2_read_probe(r3d_cuda_ctx *c, size_t bytes, uint32_t passes, float *gbs) {
  if (!c || !gbs || bytes < (1u << 20) || !passes) return R3D_E_INVALID;
  R3D_CUDA_TRY(c, cudaSetDevice(c->device));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const size_t n16 = bytes / 16u;
  uint4 *buf = nullptr;
  R3D_CUDA_TRY(c, cudaMalloc(&buf, n16 * 16u + 256u));
  uint32_t *sink = (uint32_t *)(buf + n16);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMemsetAsync(buf, 1, n16 * 16u, c->stream);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const uint32_t blocks = (uint32_t)sms * 8u;
  if (e == cudaSuccess) {  // warm: the buffer becomes L2 resident
    r3d::k_l2_read<<<blocks, 256, 0, c->stream>>>(buf, n16, 2u, sink);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
  if (e == cudaSuccess) {
    r3d::k_l2_read<<<blocks, 256, 0, c->stream>>>(buf, n16, passes, sink);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  if (e != cudaSuccess) return r3d::cuda_fail(c, e, "l2_read_probe");
  *gbs = (float)((double)n16 * 16.0 * passes / (ms * 1e-3) / 1e9);
  return R3D_OK;
}

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
