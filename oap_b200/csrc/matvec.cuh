// Dense operator application on the reference layout (row-major split re/im
// planes).  These are the HBM-bound hot kernels of the solver:
//
//   y = A x      (k_matvec)          bytes = 2 * sizeof(T) * n^2 (complex)
//   Y = A X      (k_block_matvec)    same bytes, `nrhs` right-hand sides
//
// k_matvec: a CTA of 8 warps owns a tile of R consecutive rows; warp w
// streams columns [w n/8, (w+1) n/8) of those R rows with 16-byte loads
// (float4 / double2, cache-streaming so A does not evict x from L1), lane
// partials are reduced with shuffles, then across warps in shared memory.
// x is read through the read-only path and reused R times per load.  The
// grid is persistent (a multiple of the SM count) and strides over tiles.
#pragma once

#include "common.cuh"

namespace oapb {

template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int N = 4;
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int N = 2;
};

__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_ro(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double2 ld_ro(const double2* p) { return __ldg(p); }

template <typename T>
struct Lanes;
template <>
struct Lanes<float> {
  __device__ static __forceinline__ float at(const float4& v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
  }
};
template <>
struct Lanes<double> {
  __device__ static __forceinline__ double at(const double2& v, int i) { return i == 0 ? v.x : v.y; }
};

constexpr int kMvWarps = 8;
constexpr int kMvThreads = kMvWarps * 32;

// Vectorised path.  Requires n % (8 * VW) == 0 and 16-byte aligned planes.
// Accumulation type: T for the per-lane partial sums (FP32 arithmetic is the
// point of the mixed form), double across lanes / warps; y is FP64.
template <typename T, bool CPLX, int R>
__global__ void __launch_bounds__(kMvThreads)
k_matvec(const T* __restrict__ Are, const T* __restrict__ Aim, int n,
         const T* __restrict__ xre, const T* __restrict__ xim,
         double* __restrict__ yre, double* __restrict__ yim, int ntiles) {
  using V = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::N;
  __shared__ double red[kMvWarps][R][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cw = n / kMvWarps;              // columns per warp
  const int c0 = warp * cw;
  const int nv = cw / VW;                   // vectors per warp row segment
  const V* xr = reinterpret_cast<const V*>(xre + c0);
  const V* xi = CPLX ? reinterpret_cast<const V*>(xim + c0) : nullptr;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long r0 = (long)tile * R;
    T accr[R], acci[R];
#pragma unroll
    for (int q = 0; q < R; ++q) { accr[q] = 0; acci[q] = 0; }
    const V* ar[R];
    const V* ai[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      ar[q] = reinterpret_cast<const V*>(Are + (r0 + q) * n + c0);
      ai[q] = CPLX ? reinterpret_cast<const V*>(Aim + (r0 + q) * n + c0) : nullptr;
    }
#pragma unroll 2
    for (int v = lane; v < nv; v += 32) {
      V xv = ld_ro(xr + v);
      V xiv;
      if (CPLX) xiv = ld_ro(xi + v);
      V a[R], b[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        a[q] = ld_stream(ar[q] + v);
        if (CPLX) b[q] = ld_stream(ai[q] + v);
      }
#pragma unroll
      for (int q = 0; q < R; ++q) {
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          T are_ = Lanes<T>::at(a[q], e), xr_ = Lanes<T>::at(xv, e);
          if (CPLX) {
            T aim_ = Lanes<T>::at(b[q], e), xi_ = Lanes<T>::at(xiv, e);
            accr[q] = fma(are_, xr_, accr[q]);
            accr[q] = fma(-aim_, xi_, accr[q]);
            acci[q] = fma(are_, xi_, acci[q]);
            acci[q] = fma(aim_, xr_, acci[q]);
          } else {
            accr[q] = fma(are_, xr_, accr[q]);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      double sr = warp_sum((double)accr[q]);
      double si = CPLX ? warp_sum((double)acci[q]) : 0.0;
      if (lane == 0) {
        red[warp][q][0] = sr;
        red[warp][q][1] = si;
      }
    }
    __syncthreads();
    if (threadIdx.x < R) {
      const int q = threadIdx.x;
      double sr = 0, si = 0;
#pragma unroll
      for (int w = 0; w < kMvWarps; ++w) {
        sr += red[w][q][0];
        si += red[w][q][1];
      }
      yre[r0 + q] = sr;
      if (CPLX) yim[r0 + q] = si;
    }
    __syncthreads();
  }
}

// Generic path for any n: one warp per row, scalar loads, FP64 accumulation
// of T products.
template <typename T, bool CPLX>
__global__ void k_matvec_scalar(const T* __restrict__ Are, const T* __restrict__ Aim,
                                int nrows, int ncols, const T* __restrict__ xre,
                                const T* __restrict__ xim, double* __restrict__ yre,
                                double* __restrict__ yim) {
  const int lane = threadIdx.x & 31;
  const long warps = (long)gridDim.x * (blockDim.x >> 5);
  for (long r = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nrows; r += warps) {
    double sr = 0, si = 0;
    for (int c = lane; c < ncols; c += 32) {
      double a = (double)Are[r * ncols + c], x = (double)xre[c];
      if (CPLX) {
        double b = (double)Aim[r * ncols + c], y = (double)xim[c];
        sr += a * x - b * y;
        si += a * y + b * x;
      } else {
        sr += a * x;
      }
    }
    sr = warp_sum(sr);
    if (CPLX) si = warp_sum(si);
    if (lane == 0) {
      yre[r] = sr;
      if (CPLX) yim[r] = si;
    }
  }
}

// Launch variants of k_matvec: rows per CTA (R) and grid (persistent,
// 148 x resident CTAs, or one CTA per row tile).  Variant 0 is the default
// policy; an autotuner may pick another by timing them on the operator.
constexpr int kMvVariants = 6;
__host__ __device__ inline int mv_rows(int variant) { return variant % 3 == 0 ? 4 : variant % 3 == 1 ? 2 : 8; }
__host__ __device__ inline bool mv_persistent(int variant) { return variant < 3; }

template <typename T, bool CPLX, int R>
cudaError_t launch_matvec_r(const T* Are, const T* Aim, int ncols, const T* xre, const T* xim, double* yre,
                            double* yim, int ntiles, bool persistent, cudaStream_t s) {
  static int occ = 0;  // per instantiation
  if (occ == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_matvec<T, CPLX, R>, kMvThreads, 0);
    if (occ < 1) occ = 1;
  }
  int grid = persistent ? kNumSMs * occ : ntiles;
  if (grid > ntiles) grid = ntiles;
  k_matvec<T, CPLX, R><<<grid, kMvThreads, 0, s>>>(Are, Aim, ncols, xre, xim, yre, yim, ntiles);
  return cudaGetLastError();
}

// Host launcher: y (FP64) = A (T) x (T).  Returns a CUDA error code.
template <typename T>
cudaError_t launch_matvec(const T* Are, const T* Aim, int nrows, int ncols,
                          const T* xre, const T* xim, double* yre, double* yim,
                          cudaStream_t s, int variant = 0) {
  constexpr int VW = Vec16<T>::N;
  const bool cplx = Aim != nullptr;
  const bool aligned =
      nrows == ncols && ncols % (kMvWarps * VW) == 0 &&
      ((uintptr_t)Are % 16 == 0) && ((uintptr_t)xre % 16 == 0) &&
      (!cplx || (((uintptr_t)Aim % 16 == 0) && ((uintptr_t)xim % 16 == 0)));
  if (variant < 0 || variant >= kMvVariants) variant = 0;
  const int R = mv_rows(variant);
  if (aligned && nrows % R == 0 && ncols >= 256) {
    const int ntiles = nrows / R;
    const bool pers = mv_persistent(variant);
    switch (R * (cplx ? -1 : 1)) {
      case 2: return launch_matvec_r<T, false, 2>(Are, nullptr, ncols, xre, nullptr, yre, nullptr, ntiles, pers, s);
      case 4: return launch_matvec_r<T, false, 4>(Are, nullptr, ncols, xre, nullptr, yre, nullptr, ntiles, pers, s);
      case 8: return launch_matvec_r<T, false, 8>(Are, nullptr, ncols, xre, nullptr, yre, nullptr, ntiles, pers, s);
      case -2: return launch_matvec_r<T, true, 2>(Are, Aim, ncols, xre, xim, yre, yim, ntiles, pers, s);
      case -4: return launch_matvec_r<T, true, 4>(Are, Aim, ncols, xre, xim, yre, yim, ntiles, pers, s);
      default: return launch_matvec_r<T, true, 8>(Are, Aim, ncols, xre, xim, yre, yim, ntiles, pers, s);
    }
  } else {
    int grid = grid_for((long)nrows * 32, 256, kNumSMs * 8);
    if (cplx)
      k_matvec_scalar<T, true><<<grid, 256, 0, s>>>(Are, Aim, nrows, ncols, xre, xim, yre, yim);
    else
      k_matvec_scalar<T, false><<<grid, 256, 0, s>>>(Are, nullptr, nrows, ncols, xre, nullptr, yre, nullptr);
  }
  return cudaGetLastError();
}

}  // namespace oapb
