// Block (multi-vector) FP64 kernels: the refinement and verification passes
// of the solver apply the FP64 operator to `b` vectors at once, reading A
// from HBM once per pass instead of once per vector.
//
//   k_block_matvec   W = A X        A row-major split planes (reference
//                                   layout, FP64 or FP32); X, W
//                                   vector-contiguous FP64, b <= 32; split
//                                   over K, partials summed by k_split_reduce
//   k_block_dot      part = X^H Y   per row chunk (b1 x b2)
//   k_block_reduce   G = sum of chunk partials
//   k_block_update   Out = Base - X C   (C column-major b1 x b2)
//   k_colnorm2       per-column ||Y_q||^2 partials
//   k_chol_inv       one warp: G = R^H R (Cholesky), Rinv = R^-1
#pragma once

#include "common.cuh"

namespace oapb {

constexpr int kBmRows = 64;   // rows per CTA tile
constexpr int kBmTM = 4;      // rows per thread
constexpr int kBmTQ = 4;      // right-hand sides per thread
constexpr int kBmMaxB = 32;
constexpr int kBmThreads = 128;

// Partial products of W = A X over one K split: CTA (tile, split) computes
// rows [64 tile, 64 tile + 64) over columns [k0, k1) and writes the FP64
// partial to Wp[split][q][row].  T is the operator's element type (double
// for the FP64 pass, float for the FP32 pass; X is converted to T when it is
// staged); the per-thread accumulators are T.  Thread layout: 16 row groups
// of kBmTM rows x QB / kBmTQ groups of right-hand sides.
template <typename T, bool CPLX>
__global__ void __launch_bounds__(kBmThreads)
k_block_matvec(const T* __restrict__ Are, const T* __restrict__ Aim, int n, const double* __restrict__ Xre,
               const double* __restrict__ Xim, int b, int ksplit, double* __restrict__ Wp) {
  constexpr int BK = 128 / sizeof(T);
  __shared__ T as_re[kBmRows][BK + 1];
  __shared__ T as_im[CPLX ? kBmRows : 1][BK + 1];
  __shared__ T xs_re[BK][kBmMaxB];
  __shared__ T xs_im[CPLX ? BK : 1][kBmMaxB];
  const int QB = ((b + kBmTQ - 1) / kBmTQ) * kBmTQ;
  const int nqg = QB / kBmTQ;
  const int t = threadIdx.x;
  const int rg = t % (kBmRows / kBmTM), qg = t / (kBmRows / kBmTM);
  const bool active = qg < nqg;
  const long r0 = (long)blockIdx.x * kBmRows;
  const long kb = (long)blockIdx.y * ksplit;
  const long ke = min((long)n, kb + ksplit);
  T accr[kBmTM][kBmTQ], acci[kBmTM][kBmTQ];
#pragma unroll
  for (int i = 0; i < kBmTM; ++i)
#pragma unroll
    for (int q = 0; q < kBmTQ; ++q) accr[i][q] = acci[i][q] = 0;
  for (long k0 = kb; k0 < ke; k0 += BK) {
    __syncthreads();
#pragma unroll 4
    for (int e = t; e < kBmRows * BK; e += kBmThreads) {
      const int rr = e / BK, kk = e % BK;
      const long r = r0 + rr, c = k0 + kk;
      const bool in = r < n && c < ke;
      as_re[rr][kk] = in ? __ldcs(Are + r * n + c) : T(0);
      if (CPLX) as_im[rr][kk] = in ? __ldcs(Aim + r * n + c) : T(0);
    }
    for (int e = t; e < BK * QB; e += kBmThreads) {
      const int kk = e % BK, q = e / BK;
      const long c = k0 + kk;
      const bool in = q < b && c < ke;
      xs_re[kk][q] = in ? (T)Xre[(long)q * n + c] : T(0);
      if (CPLX) xs_im[kk][q] = in ? (T)Xim[(long)q * n + c] : T(0);
    }
    __syncthreads();
    if (active) {
#pragma unroll 8
      for (int kk = 0; kk < BK; ++kk) {
        T ar[kBmTM], ai[kBmTM], xr[kBmTQ], xi[kBmTQ];
#pragma unroll
        for (int i = 0; i < kBmTM; ++i) {
          ar[i] = as_re[rg * kBmTM + i][kk];
          ai[i] = CPLX ? as_im[rg * kBmTM + i][kk] : T(0);
        }
#pragma unroll
        for (int q = 0; q < kBmTQ; ++q) {
          xr[q] = xs_re[kk][qg * kBmTQ + q];
          xi[q] = CPLX ? xs_im[kk][qg * kBmTQ + q] : T(0);
        }
#pragma unroll
        for (int i = 0; i < kBmTM; ++i)
#pragma unroll
          for (int q = 0; q < kBmTQ; ++q) {
            accr[i][q] = fma(ar[i], xr[q], accr[i][q]);
            if (CPLX) {
              acci[i][q] = fma(ar[i], xi[q], acci[i][q]);
              accr[i][q] = fma(-ai[i], xi[q], accr[i][q]);
              acci[i][q] = fma(ai[i], xr[q], acci[i][q]);
            }
          }
      }
    }
  }
  if (active) {
    double* wr = Wp + (long)blockIdx.y * 2 * b * n;
    double* wi = wr + (long)b * n;
#pragma unroll
    for (int i = 0; i < kBmTM; ++i) {
      const long r = r0 + rg * kBmTM + i;
#pragma unroll
      for (int q = 0; q < kBmTQ; ++q) {
        const int qq = qg * kBmTQ + q;
        if (r < n && qq < b) {
          wr[(long)qq * n + r] = (double)accr[i][q];
          if (CPLX) wi[(long)qq * n + r] = (double)acci[i][q];
        }
      }
    }
  }
}

// W[q][r] = sum over splits of Wp[s][q][r]
template <bool CPLX>
__global__ void k_split_reduce(const double* __restrict__ Wp, int nsplit, int b, int n, double* Wre, double* Wim) {
  const long len = (long)b * n;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x) {
    double a = 0, c = 0;
    for (int s = 0; s < nsplit; ++s) {
      a += Wp[(long)s * 2 * len + e];
      if (CPLX) c += Wp[(long)s * 2 * len + len + e];
    }
    Wre[e] = a;
    if (CPLX) Wim[e] = c;
  }
}

constexpr int kDotChunk = 32;

// part[blk][i + j * b1] = sum_{r in chunk} conj(X_i[r]) Y_j[r]
template <bool CPLX>
__global__ void k_block_dot(const double* __restrict__ Xre, const double* __restrict__ Xim, int b1,
                            const double* __restrict__ Yre, const double* __restrict__ Yim, int b2, int n,
                            cplx* part) {
  __shared__ double xr[kBmMaxB][kDotChunk], xi[kBmMaxB][kDotChunk];
  __shared__ double yr[kBmMaxB][kDotChunk], yi[kBmMaxB][kDotChunk];
  const long r0 = (long)blockIdx.x * kDotChunk;
  for (int e = threadIdx.x; e < kBmMaxB * kDotChunk; e += blockDim.x) {
    const int q = e / kDotChunk, rr = e % kDotChunk;
    const long r = r0 + rr;
    const bool in = r < n;
    xr[q][rr] = (in && q < b1) ? Xre[(long)q * n + r] : 0.0;
    xi[q][rr] = (in && q < b1 && CPLX) ? Xim[(long)q * n + r] : 0.0;
    yr[q][rr] = (in && q < b2) ? Yre[(long)q * n + r] : 0.0;
    yi[q][rr] = (in && q < b2 && CPLX) ? Yim[(long)q * n + r] : 0.0;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < b1 * b2; p += blockDim.x) {
    const int i = p % b1, j = p / b1;
    double sr = 0, si = 0;
    for (int rr = 0; rr < kDotChunk; ++rr) {
      const double a = xr[i][rr], bb = xi[i][rr], c = yr[j][rr], d = yi[j][rr];
      sr += a * c + bb * d;
      si += a * d - bb * c;
    }
    part[(long)blockIdx.x * b1 * b2 + p] = cplx{sr, si};
  }
}

__global__ void k_block_reduce(const cplx* part, int nblk, int cnt, cplx* out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < cnt; p += gridDim.x * blockDim.x) {
    double a = 0, b = 0;
    for (int c = 0; c < nblk; ++c) {
      cplx v = part[(long)c * cnt + p];
      a += v.re;
      b += v.im;
    }
    out[p] = cplx{a, b};
  }
}

// Out_j = Base_j - sum_i X_i C[i + j ldc]  (Base may be null: Out = -X C, or
// with negate = 0: Out = X C)
template <bool CPLX>
__global__ void k_block_update(const double* __restrict__ Xre, const double* __restrict__ Xim, int b1,
                               const cplx* __restrict__ Cm, int ldc, int b2, const double* Bre, const double* Bim,
                               int negate, int n, double* Ore, double* Oim) {
  __shared__ cplx cs[kBmMaxB * kBmMaxB];
  for (int e = threadIdx.x; e < b1 * b2; e += blockDim.x) cs[e] = Cm[(e % b1) + (long)(e / b1) * ldc];
  __syncthreads();
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
    cplx xv[kBmMaxB];
    for (int i = 0; i < b1; ++i) xv[i] = cplx{Xre[(long)i * n + r], CPLX ? Xim[(long)i * n + r] : 0.0};
    for (int j = 0; j < b2; ++j) {
      cplx acc = {0, 0};
      for (int i = 0; i < b1; ++i) acc = acc + xv[i] * cs[i + j * b1];
      cplx o;
      if (Bre) o = cplx{Bre[(long)j * n + r], CPLX ? Bim[(long)j * n + r] : 0.0} - acc;
      else o = negate ? -acc : acc;
      Ore[(long)j * n + r] = o.re;
      if (CPLX) Oim[(long)j * n + r] = o.im;
    }
  }
}

// part[blk * b + q] = sum over the block's rows of |Y_q[r]|^2
template <bool CPLX>
__global__ void k_colnorm2(const double* __restrict__ Yre, const double* __restrict__ Yim, int b, int n,
                           double* part) {
  __shared__ double red[kBmMaxB][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = 0; q < b; ++q) {
    double s = 0;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
      double a = Yre[(long)q * n + r];
      s += a * a;
      if (CPLX) {
        double c = Yim[(long)q * n + r];
        s += c * c;
      }
    }
    s = warp_sum(s);
    if (lane == 0) red[q][warp] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < b; q += blockDim.x) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[q][w];
    part[(long)blockIdx.x * b + q] = s;
  }
}

// One warp: Cholesky G = R^H R of a b x b Hermitian positive definite matrix
// (column-major), then Rinv = R^-1 (upper triangular).  status bit 2 when a
// pivot is not positive.
__global__ void k_chol_inv(const cplx* G, int b, cplx* Rinv, int* status) {
  __shared__ cplx R[kBmMaxB * kBmMaxB];
  __shared__ cplx Ri[kBmMaxB * kBmMaxB];
  const int lane = threadIdx.x;
  for (int e = lane; e < b * b; e += 32) {
    R[e] = cplx{0, 0};
    Ri[e] = cplx{0, 0};
  }
  __syncwarp();
  // R[i][j] (i <= j) column-major at i + j b
  for (int j = 0; j < b; ++j) {
    // R[i][j] = (G[i][j] - sum_{p<i} conj(R[p][i]) R[p][j]) / R[i][i], i < j
    for (int i = 0; i < j; ++i) {
      cplx acc = {0, 0};
      for (int p = lane; p < i; p += 32) acc = acc + conj(R[p + i * b]) * R[p + j * b];
      acc.re = warp_sum(acc.re);
      acc.im = warp_sum(acc.im);
      if (lane == 0) R[i + j * b] = cdiv(G[i + j * b] - acc, R[i + i * b]);
      __syncwarp();
    }
    double d = 0;
    for (int p = lane; p < j; p += 32) d += abs2(R[p + j * b]);
    d = warp_sum(d);
    const double piv = G[j + j * b].re - d;
    if (lane == 0) {
      if (!(piv > 0)) {
        atomicOr(status, 4);
        R[j + j * b] = cplx{1e-300, 0};
      } else {
        R[j + j * b] = cplx{sqrt(piv), 0};
      }
    }
    __syncwarp();
  }
  // inverse of upper-triangular R: column j of Ri solves R x = e_j
  for (int j = lane; j < b; j += 32) {
    for (int i = j; i >= 0; --i) {
      cplx acc = (i == j) ? cplx{1, 0} : cplx{0, 0};
      for (int p = i + 1; p <= j; ++p) acc = acc - R[i + p * b] * Ri[p + j * b];
      Ri[i + j * b] = cdiv(acc, R[i + i * b]);
    }
  }
  __syncwarp();
  for (int e = lane; e < b * b; e += 32) Rinv[e] = Ri[e];
}

}  // namespace oapb
