/* Project-written log2 / exp2 / pow for the raycast, compiled identically
 * for the CPU (C, gcc) and the GPU (CUDA, nvcc).
 *
 * The raycast's early-termination step counts and MIP indices depend on the
 * ray-cone LOD (log2, exp2) and the opacity correction (pow) of every sample,
 * so the CPU restatement and the sm_100a kernels must produce the same bits
 * for them.  Library transcendentals differ between glibc and CUDA; these do
 * not, because they use only IEEE-754 correctly rounded operations (+ - * /,
 * fmaf, exponent bit manipulation), evaluated in a fixed order.
 * Callers must compile without floating-point contraction
 * (gcc -ffp-contract=off, nvcc -fmad=false); every fused multiply-add
 * below is an explicit fmaf.
 *
 * Methods (textbook, coefficients are exact series terms, not fitted):
 *  - log2: x = m * 2^e with m in [sqrt(1/2), sqrt(2)];
 *          ln m = 2 atanh(s), s = (m - 1) / (m + 1), |s| <= 0.1716, using the
 *          odd series 2 (s + s^3/3 + s^5/5 + s^7/7 + s^9/9) (Abramowitz &
 *          Stegun 4.1.28); truncation error < 3e-9 relative.
 *  - exp2: x = n + f with n = rint(x) (round-half-even, by the 1.5*2^23
 *          shift), |f| <= 1/2; 2^f = e^(f ln 2) by its
 *          Taylor series to degree 7 (truncation < 8e-9 relative); 2^n is
 *          applied by building the exponent field (two factors so that
 *          subnormal results round once).
 *  - pow:  x^y = exp2(y log2 x) for x >= 0.
 *  - powi24: x^24 by repeated squaring (the specular exponent).
 * Accuracy against glibc in double precision is checked by the test suite
 * (a few ulp), and the GPU build is checked bit-for-bit against the CPU
 * build on the device. */
#ifndef R3D_FMATH_H
#define R3D_FMATH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define R3D_FM_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#define R3D_FM_HD static inline
#endif

R3D_FM_HD uint32_t r3d_f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}

R3D_FM_HD float r3d_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

#define R3D_FM_INF r3d_u2f(0x7f800000u)
#define R3D_FM_NAN r3d_u2f(0x7fc00000u)

/* log2 for finite or infinite x; x == 0 -> -inf, x < 0 -> NaN. */
R3D_FM_HD float r3d_log2f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -R3D_FM_INF : R3D_FM_NAN;
  if (!(x < R3D_FM_INF)) return x;
  uint32_t b = r3d_f2u(x);
  int e = 0;
  if (b < 0x00800000u) { /* subnormal: scale into the normal range */
    x = x * 8388608.0f;  /* 2^23, exact */
    b = r3d_f2u(x);
    e = -23;
  }
  e += (int)(b >> 23) - 127;
  float m = r3d_u2f((b & 0x007fffffu) | 0x3f800000u); /* [1, 2) */
  if (m > 1.41421356f) {
    m = m * 0.5f; /* exact */
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = fmaf(s2, 0.111111111f, 0.142857143f); /* 1/9, 1/7 */
  p = fmaf(s2, p, 0.2f);
  p = fmaf(s2, p, 0.333333333f);
  p = fmaf(s2, p, 1.0f);
  float r = (s * 2.88539008f) * p; /* 2 / ln 2 */
  return (float)e + r;
}

/* 2^x; NaN -> NaN, x >= 128 -> inf, x < -151 -> 0. */
R3D_FM_HD float r3d_exp2f(float x) {
  if (x != x) return x;
  if (x >= 128.0f) return R3D_FM_INF;
  if (x < -151.0f) return 0.0f;
  /* n = rint(x): adding 1.5 * 2^23 rounds to the nearest even integer,
   * which then sits in the low mantissa bits of big */
  float big = x + 12582912.0f;
  float n = big - 12582912.0f;
  float f = x - n; /* exact, |f| <= 0.5 */
  float p = fmaf(f, 1.52527338e-05f, 1.54035304e-04f);
  p = fmaf(f, p, 1.33335581e-03f);
  p = fmaf(f, p, 9.61812911e-03f);
  p = fmaf(f, p, 5.55041087e-02f);
  p = fmaf(f, p, 2.40226507e-01f);
  p = fmaf(f, p, 6.93147181e-01f);
  p = fmaf(f, p, 1.0f);
  int ni = (int)(r3d_f2u(big) - 0x4B400000u);
  if (ni >= -126 && ni <= 127) return p * r3d_u2f((uint32_t)(ni + 127) << 23);
  /* split the scale so a subnormal result is rounded exactly once */
  int n1 = ni / 2, n2 = ni - n1;
  float a = p * r3d_u2f((uint32_t)(n1 + 127) << 23);
  return a * r3d_u2f((uint32_t)(n2 + 127) << 23);
}

/* x^y for x >= 0 (the only use here): 0^y = 0 for y > 0, x^0 = 1. */
R3D_FM_HD float r3d_powf(float x, float y) {
  if (y == 0.0f || x == 1.0f) return 1.0f;
  if (x == 0.0f) return y > 0.0f ? 0.0f : R3D_FM_INF;
  return r3d_exp2f(y * r3d_log2f(x));
}

/* x^24 by squaring: x^24 = (((x^3)^2)^2)^2. */
R3D_FM_HD float r3d_powi24f(float x) {
  float x2 = x * x;
  float x3 = x2 * x;
  float x6 = x3 * x3;
  float x12 = x6 * x6;
  return x12 * x12;
}

#endif /* R3D_FMATH_H */
