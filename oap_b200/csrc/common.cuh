// Shared helpers for the oapb200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "oapb200.h"

#define OAPB_CUDA_TRY(expr)                                  \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return OAPB_ERR_CUDA;             \
  } while (0)

#define OAPB_LAUNCH_CHECK()                                  \
  do {                                                       \
    cudaError_t _e = cudaGetLastError();                     \
    if (_e != cudaSuccess) return OAPB_ERR_CUDA;             \
  } while (0)

namespace oapb {

constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

// ---------------------------------------------------------------- complex --
struct cplx {
  double re, im;
};

__host__ __device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx conj(cplx a) { return {a.re, -a.im}; }
__host__ __device__ __forceinline__ double abs2(cplx a) { return a.re * a.re + a.im * a.im; }
__host__ __device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
__host__ __device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  // Smith's algorithm
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  } else {
    double r = b.re / b.im, d = b.re * r + b.im;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
  }
}
__host__ __device__ __forceinline__ cplx csqrt_(cplx z) {
  double r = hypot(z.re, z.im);
  if (r == 0) return {0, 0};
  double t = sqrt(0.5 * (r + fabs(z.re)));
  if (z.re >= 0) return {t, z.im / (2 * t)};
  return {fabs(z.im) / (2 * t), z.im >= 0 ? t : -t};
}

// Unitary rotation G = [p q; -conj(q) conj(p)], p = conj(x)/r, q = conj(y)/r,
// so G [x; y] = [r; 0] with r = sqrt(|x|^2 + |y|^2) > 0.  For real inputs
// this is the reference's c = x / r, s = y / r (CuQRProcedures_GR.h:80-101).
__device__ __forceinline__ void givens(cplx x, cplx y, cplx& p, cplx& q) {
  double r2 = x.re * x.re + x.im * x.im + y.re * y.re + y.im * y.im;
  if (r2 == 0) {
    p = {1, 0};
    q = {0, 0};
    return;
  }
  double s = 1.0;
  if (!(r2 < 1e300) || r2 < 1e-290) {
    // rescale by the largest component so the sum of squares stays finite
    s = fmax(fmax(fabs(x.re), fabs(x.im)), fmax(fabs(y.re), fabs(y.im)));
    const double is = 1.0 / s;
    x = is * x;
    y = is * y;
    r2 = x.re * x.re + x.im * x.im + y.re * y.re + y.im * y.im;
  }
  const double ir = rsqrt(r2);  // 1 / r of the (rescaled) pair
  p = {x.re * ir, -x.im * ir};
  q = {y.re * ir, -y.im * ir};
}

// FP32 complex (the working type of the FP32 small dense eigensolver)
struct cplxf {
  float re, im;
};
__host__ __device__ __forceinline__ cplxf operator+(cplxf a, cplxf b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplxf operator-(cplxf a, cplxf b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplxf operator-(cplxf a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ cplxf operator*(cplxf a, cplxf b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplxf operator*(float s, cplxf a) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplxf conj(cplxf a) { return {a.re, -a.im}; }
__host__ __device__ __forceinline__ float abs2(cplxf a) { return a.re * a.re + a.im * a.im; }
__host__ __device__ __forceinline__ float cabs_(cplxf a) { return hypotf(a.re, a.im); }
__host__ __device__ __forceinline__ cplxf cdiv(cplxf a, cplxf b) {
  if (fabsf(b.re) >= fabsf(b.im)) {
    float r = b.im / b.re, d = b.re + b.im * r;
    return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  } else {
    float r = b.re / b.im, d = b.re * r + b.im;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
  }
}
__host__ __device__ __forceinline__ cplxf csqrt_(cplxf z) {
  float r = hypotf(z.re, z.im);
  if (r == 0) return {0, 0};
  float t = sqrtf(0.5f * (r + fabsf(z.re)));
  if (z.re >= 0) return {t, z.im / (2 * t)};
  return {fabsf(z.im) / (2 * t), z.im >= 0 ? t : -t};
}
__device__ __forceinline__ void givens(cplxf x, cplxf y, cplxf& p, cplxf& q) {
  float r2 = x.re * x.re + x.im * x.im + y.re * y.re + y.im * y.im;
  if (r2 == 0) {
    p = {1, 0};
    q = {0, 0};
    return;
  }
  if (!(r2 < 1e36f) || r2 < 1e-36f) {
    const float s = fmaxf(fmaxf(fabsf(x.re), fabsf(x.im)), fmaxf(fabsf(y.re), fabsf(y.im)));
    const float is = 1.0f / s;
    x = is * x;
    y = is * y;
    r2 = x.re * x.re + x.im * x.im + y.re * y.re + y.im * y.im;
  }
  const float ir = rsqrtf(r2);
  p = {x.re * ir, -x.im * ir};
  q = {y.re * ir, -y.im * ir};
}

// conversions between the FP64 storage type and a working type
template <typename Cx>
__host__ __device__ __forceinline__ Cx cx_from(cplx v);
template <>
__host__ __device__ __forceinline__ cplx cx_from<cplx>(cplx v) { return v; }
template <>
__host__ __device__ __forceinline__ cplxf cx_from<cplxf>(cplx v) { return {(float)v.re, (float)v.im}; }
__host__ __device__ __forceinline__ cplx cx_to(cplx v) { return v; }
__host__ __device__ __forceinline__ cplx cx_to(cplxf v) { return {(double)v.re, (double)v.im}; }

// ------------------------------------------------------------ warp reduce --
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic U[-1, 1) start vector: splitmix64 of (seed, index).  The
// same function is restated on the host side of the tests.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ double uniform_pm1(uint64_t seed, uint64_t i) {
  uint64_t h = splitmix64(seed * 0x100000001B3ull + i);
  return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

inline int grid_for(long work, int per_block, int cap = kNumSMs * 16) {
  long g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

}  // namespace oapb
