// Block (multi-vector) FP64 kernels: the refinement and verification passes
// of the solver apply the FP64 operator to `b` vectors at once, reading A
// from HBM once per pass instead of once per vector.
//
//   k_block_matvec   W = A X        A row-major split planes (reference
//                                   layout, FP64 or FP32); X, W
//                                   vector-contiguous FP64, b <= 32; split
//                                   over K, partials summed by k_split_reduce
//   k_block_dot      part = X^H Y   per row chunk (b1 x b2)
//   k_block_reduce   G = sum of chunk partials (optionally followed by the
//                    Cholesky inverse in the last block to finish)
//   k_block_update   Out = Base - X C   (C column-major b1 x b2; X + Y with an addend Y)
//   k_colnorm2       per-column ||Y_q||^2 partials
//   k_chol_inv       one warp: G = R^H R (Cholesky), Rinv = R^-1
#pragma once

#include "common.cuh"
#include "matvec.cuh"

namespace oapb {
// The kernels below may be launched as programmatic dependents of the
// kernel before them in the stream: they wait for it to complete (and its
// memory to be visible) before touching global memory; a no-op otherwise.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
}  // namespace oapb

namespace oapb {

constexpr int kBmRows = 128;  // rows per CTA tile
constexpr int kBmTM = 4;      // rows per thread
constexpr int kBmTQ = 4;      // right-hand sides per thread
constexpr int kBmMaxB = 32;
constexpr int kBmThreads = 256;

__device__ __forceinline__ void mkvec(const float (&t)[4], float4& v) { v = make_float4(t[0], t[1], t[2], t[3]); }
__device__ __forceinline__ void mkvec(const double (&t)[2], double2& v) { v = make_double2(t[0], t[1]); }

template <typename T>
struct Quad;  // four consecutive T in shared memory
template <>
struct Quad<float> {
  __device__ static __forceinline__ void ld(const float* p, float (&v)[4]) {
    float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  }
};
template <>
struct Quad<double> {
  __device__ static __forceinline__ void ld(const double* p, double (&v)[4]) {
    double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
};

// Partial products of W = A X over one K split: CTA (tile, split) computes
// rows [128 tile, 128 tile + 128) over columns [k0, k1) and writes the FP64
// partial to Wp[split][plane][q][row].  T is the operator's element type
// (double for the FP64 pass, float for the FP32 pass; X is converted to T
// when it is staged); the per-thread accumulators are T.
//
// A tiles are read with 16-byte coalesced loads (8 lanes per 128-byte row
// segment), prefetched into registers one tile ahead, and stored transposed
// ([k][row]) in shared memory with the row index XOR-swizzled by the
// 16-byte column group, so both the transposing stores and the 4-row vector
// reads are free of bank conflicts.  Thread (rg, qg) owns rows 4 rg .. 4 rg + 3
// and right-hand sides 4 qg .. 4 qg + 3: per k it reads 4 + 4 A values and
// 4 + 4 X values (broadcast across the warp) for 16 complex FMAs.
template <typename T, bool CPLX>
__global__ void __launch_bounds__(kBmThreads)
k_block_matvec(const T* __restrict__ Are, const T* __restrict__ Aim, int n, const double* __restrict__ Xre,
               const double* __restrict__ Xim, int b, int ksplit, double* __restrict__ Wp, int vec_ok) {
  using V = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::N;            // T per 16-byte vector
  constexpr int BK = 128 / sizeof(T);        // k per tile: one 128-byte row segment
  constexpr int VPR = BK / VW;               // vectors per row segment (8)
  constexpr int NV = kBmRows * VPR / kBmThreads;  // vectors per thread per plane (4)
  constexpr int NP = CPLX ? 2 : 1;
  __shared__ __align__(16) T As[NP][BK][kBmRows];
  __shared__ __align__(16) T Xs[NP][kBmMaxB][BK + 1];
  const int QB = ((b + kBmTQ - 1) / kBmTQ) * kBmTQ;
  const int t = threadIdx.x;
  const int rg = t % (kBmRows / kBmTM), qg = t / (kBmRows / kBmTM);
  const bool active = qg * kBmTQ < QB;
  const long r0 = (long)blockIdx.x * kBmRows;
  const long kb = (long)blockIdx.y * ksplit;
  const long ke = min((long)n, kb + ksplit);
  const T* planes[2] = {Are, Aim};
  const bool full_rows = r0 + kBmRows <= n;

  constexpr int NX = (BK * kBmMaxB + kBmThreads - 1) / kBmThreads;  // X values per thread per plane
  V pre[NP][NV];
  T xpre[NP][NX];
  auto fetch_x = [&](long k0) {
#pragma unroll
    for (int u = 0; u < NX; ++u) {
      const int e = t + u * kBmThreads;
      const int kk = e % BK, q = e / BK;
      const long c = k0 + kk;
      const bool in = q < b && c < ke;
      xpre[0][u] = in ? (T)Xre[(long)q * n + c] : T(0);
      if (CPLX) xpre[NP - 1][u] = in ? (T)Xim[(long)q * n + c] : T(0);
    }
  };
  auto fetch = [&](long k0) {
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        const int c = t + i * kBmThreads;
        const int row = c / VPR, kq = c % VPR;
        const long r = r0 + row, col = k0 + (long)kq * VW;
        if (vec_ok && (full_rows || r < n) && col + VW <= ke) {
          pre[p][i] = __ldcs(reinterpret_cast<const V*>(planes[p] + r * n + col));
        } else {
          T tmp[VW];
#pragma unroll
          for (int e = 0; e < VW; ++e) tmp[e] = (r < n && col + e < ke) ? planes[p][r * n + col + e] : T(0);
          mkvec(tmp, pre[p][i]);
        }
      }
  };

  T accr[kBmTM][kBmTQ], acci[kBmTM][kBmTQ];
#pragma unroll
  for (int i = 0; i < kBmTM; ++i)
#pragma unroll
    for (int q = 0; q < kBmTQ; ++q) accr[i][q] = acci[i][q] = 0;

  if (kb < ke) {
    fetch(kb);
    fetch_x(kb);
  }
  for (long k0 = kb; k0 < ke; k0 += BK) {
    __syncthreads();
    // registers -> shared (transposed, swizzled)
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        const int c = t + i * kBmThreads;
        const int row = c / VPR, kq = c % VPR;
        const int prow = row ^ ((kq & 7) << 2);
        const T* v = reinterpret_cast<const T*>(&pre[p][i]);
#pragma unroll
        for (int e = 0; e < VW; ++e) As[p][kq * VW + e][prow] = v[e];
      }
#pragma unroll
    for (int u = 0; u < NX; ++u) {
      const int e = t + u * kBmThreads;
      const int kk = e % BK, q = e / BK;
      if (q < kBmMaxB) {
        Xs[0][q][kk] = xpre[0][u];
        if (CPLX) Xs[NP - 1][q][kk] = xpre[NP - 1][u];
      }
    }
    __syncthreads();
    if (k0 + BK < ke) {  // next tiles in flight during the math
      fetch(k0 + BK);
      fetch_x(k0 + BK);
    }
    if (active) {
#pragma unroll 4
      for (int kk = 0; kk < BK; ++kk) {
        const int prow = (rg * kBmTM) ^ (((kk / VW) & 7) << 2);
        T ar[4], ai[4], xr[4], xi[4];
        Quad<T>::ld(&As[0][kk][prow], ar);
        if (CPLX) Quad<T>::ld(&As[NP - 1][kk][prow], ai);
#pragma unroll
        for (int q = 0; q < 4; ++q) {   // same address across the warp: broadcast
          xr[q] = Xs[0][qg * kBmTQ + q][kk];
          if (CPLX) xi[q] = Xs[NP - 1][qg * kBmTQ + q][kk];
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
constexpr int kDotBlocks = 2 * kNumSMs;

// part[blk][i + j * b1] = sum over the block's row chunks of conj(X_i[r]) Y_j[r]
// (chunks blk, blk + gridDim.x, ...; every thread owns a 2 x 2 tile of entries)
template <bool CPLX>
__global__ void __launch_bounds__(256) k_block_dot(const double* __restrict__ Xre, const double* __restrict__ Xim,
                                                   int b1, const double* __restrict__ Yre,
                                                   const double* __restrict__ Yim, int b2, int n, cplx* part) {
  __shared__ double xr[kBmMaxB][kDotChunk + 1], xi[kBmMaxB][kDotChunk + 1];
  __shared__ double yr[kBmMaxB][kDotChunk + 1], yi[kBmMaxB][kDotChunk + 1];
  if (blockDim.x != 256) return;  // the staging below assumes 256 threads
  pdl_wait();
  const int cnt = b1 * b2;
  // 2 x 2 tiles over (b1 rounded up to even) x (b2 rounded up to even):
  // at most 16 x 16 = 256 tiles for b <= 32
  const int tb1 = (b1 + 1) / 2, tb2 = (b2 + 1) / 2;
  const bool tile = (int)threadIdx.x < tb1 * tb2;
  const int i0 = tile ? 2 * ((int)threadIdx.x % tb1) : 0, j0 = tile ? 2 * ((int)threadIdx.x / tb1) : 0;
  double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
  const long nchunks = (n + kDotChunk - 1) / kDotChunk;
  // 256 threads: each stages kDotPer elements of every plane, loaded into
  // registers before the barrier (they overlap the previous chunk's products)
  constexpr int kDotPer = kBmMaxB * kDotChunk / 256;
  for (long ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const long r0 = ch * kDotChunk;
    double vxr[kDotPer], vxi[kDotPer], vyr[kDotPer], vyi[kDotPer];
#pragma unroll
    for (int u = 0; u < kDotPer; ++u) {
      const int e = threadIdx.x + u * 256;
      const int q = e / kDotChunk, rr = e % kDotChunk;
      const long r = r0 + rr;
      const bool in = r < n;
      vxr[u] = (in && q < b1) ? Xre[(long)q * n + r] : 0.0;
      vxi[u] = (in && q < b1 && CPLX) ? Xim[(long)q * n + r] : 0.0;
      vyr[u] = (in && q < b2) ? Yre[(long)q * n + r] : 0.0;
      vyi[u] = (in && q < b2 && CPLX) ? Yim[(long)q * n + r] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kDotPer; ++u) {
      const int e = threadIdx.x + u * 256;
      const int q = e / kDotChunk, rr = e % kDotChunk;
      xr[q][rr] = vxr[u];
      xi[q][rr] = vxi[u];
      yr[q][rr] = vyr[u];
      yi[q][rr] = vyi[u];
    }
    __syncthreads();
    // thread = 2 x 2 tile of entries (rows i0, i0 + 1 of X, j0, j0 + 1 of Y):
    // each staged value feeds two products; per entry the chunk's rows are
    // summed in order and the chunk sum added to the running sum
    if (tile) {
      double sr[4] = {0, 0, 0, 0}, si[4] = {0, 0, 0, 0};
#pragma unroll 4
      for (int rr = 0; rr < kDotChunk; ++rr) {
        const double a0 = xr[i0][rr], b0 = xi[i0][rr], a1 = xr[i0 + 1][rr], b1v = xi[i0 + 1][rr];
        const double c0 = yr[j0][rr], d0 = yi[j0][rr], c1 = yr[j0 + 1][rr], d1 = yi[j0 + 1][rr];
        sr[0] += a0 * c0 + b0 * d0;
        si[0] += a0 * d0 - b0 * c0;
        sr[1] += a1 * c0 + b1v * d0;
        si[1] += a1 * d0 - b1v * c0;
        sr[2] += a0 * c1 + b0 * d1;
        si[2] += a0 * d1 - b0 * c1;
        sr[3] += a1 * c1 + b1v * d1;
        si[3] += a1 * d1 - b1v * c1;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        ar[u] += sr[u];
        ai[u] += si[u];
      }
    }
  }
  if (tile) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + (u & 1), j = j0 + (u >> 1);
      if (i < b1 && j < b2) part[(long)blockIdx.x * cnt + i + j * b1] = cplx{ar[u], ai[u]};
    }
  }
}

// One warp: Cholesky G = R^H R of a b x b Hermitian positive definite matrix
// (column-major, b <= 32), then Rinv = R^-1 (upper triangular).  status bit
// 2 when a pivot is not positive.
// Right-looking factorization with lane j owning column j: per step k the
// lanes scale row k and update their own trailing column entries, reading
// row k by broadcast; shared arrays use an odd leading dimension, so the
// per-lane column accesses are conflict-free.  The inverse is one back
// substitution per lane (column j of R^-1).
constexpr int kCholLD = kBmMaxB + 1;
struct CholSmem {
  cplx R[kBmMaxB * kCholLD];
  cplx X[kBmMaxB * kCholLD];
  double rd[kBmMaxB];  // 1 / R[j][j]
};

// one full warp (lane = 0..31); sm in shared memory
__device__ void warp_chol_inv(const cplx* G, int b, cplx* Rinv, int* status, CholSmem& sm, int lane) {
  constexpr int LD = kCholLD;
  cplx* R = sm.R;
  cplx* X = sm.X;
  double* rd = sm.rd;
  const int j = lane;
  const bool own = j < b;
  for (int e = lane; e < b * b; e += 32) {  // L2 loads: G may come from other blocks of the caller
    const double* gp = reinterpret_cast<const double*>(G + e);
    R[e % b + (e / b) * LD] = cplx{__ldcg(gp), __ldcg(gp + 1)};
  }
  __syncwarp();
  for (int k = 0; k < b; ++k) {
    const double piv = R[k + k * LD].re;
    const double rkk = piv > 0 ? sqrt(piv) : 1e-300;
    const double inv = 1.0 / rkk;
    if (lane == 0 && !(piv > 0)) atomicOr(status, 4);
    cplx rkj = {0, 0};
    if (own && j >= k) {
      rkj = (j == k) ? cplx{rkk, 0} : inv * R[k + j * LD];
      R[k + j * LD] = rkj;
    }
    if (lane == k) rd[k] = inv;
    __syncwarp();
    if (own && j > k)
      for (int i = k + 1; i <= j; ++i) R[i + j * LD] = R[i + j * LD] - conj(R[k + i * LD]) * rkj;
    __syncwarp();
  }
  // column j of R^-1: x_j = 1 / R[j][j]; x_i = -(sum_{p>i} R[i][p] x_p) / R[i][i]
  for (int i = b - 1; i >= 0; --i) {
    cplx a0 = {0, 0}, a1 = {0, 0};
    if (own && i < j) {
      int p = i + 1;
      for (; p + 1 <= j; p += 2) {
        a0 = a0 + R[i + p * LD] * X[p + j * LD];
        a1 = a1 + R[i + (p + 1) * LD] * X[p + 1 + j * LD];
      }
      if (p <= j) a0 = a0 + R[i + p * LD] * X[p + j * LD];
    }
    if (own && i <= j) X[i + j * LD] = (i == j) ? cplx{rd[i], 0} : (-rd[i]) * (a0 + a1);
  }
  __syncwarp();
  for (int e = lane; e < b * b; e += 32) {
    const int r = e % b, c = e / b;
    Rinv[e] = r <= c ? X[r + c * LD] : cplx{0, 0};
  }
}

// barrier of the nthr threads (whole warps, from thread 0) that run
// block_chol_inv: named barrier 1, so the rest of the block may have left
__device__ __forceinline__ void chol_bar(int nthr) { asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory"); }

// The same with nthr threads of a block (whole warps, tid = 0 .. nthr - 1,
// all calling), by symmetric Gaussian elimination on [G | I]: step k takes
// the pivot d_k = M[k][k] and, for every row i > k, subtracts
// conj(M[k][i]) / d_k times row k from the upper-triangular part of row i
// and from the entries of the augmented part left of the diagonal (the
// multiplier M[i][k] of the Hermitian trailing matrix is conj(M[k][i])).
// Row k is read and rows below it are written, so one barrier per step
// suffices; every updated entry has a thread of its own when nthr >= (b - 1)
// b.  At the end the augmented part holds L^-1 of G = L D L^H (unit lower
// triangular), so R = D^1/2 L^H and Rinv = L^-H D^-1/2:
// Rinv[r][c] = conj(L^-1[c][r]) / sqrt(d_c), r <= c.
__device__ void block_chol_inv(const cplx* G, int b, cplx* Rinv, int* status, CholSmem& sm, int tid, int nthr) {
  constexpr int LD = kCholLD;
  cplx* M = sm.R;  // left part: M[i + c LD], upper triangle in use
  cplx* L = sm.X;  // augmented part: L[i + c LD] = L^-1[i][c]
  double* rd = sm.rd;
  for (int e = tid; e < b * b; e += nthr) {  // L2 loads: G may come from other blocks of the caller
    const double* gp = reinterpret_cast<const double*>(G + e);
    const int r = e % b, c = e / b;
    M[r + c * LD] = cplx{__ldcg(gp), __ldcg(gp + 1)};
    L[r + c * LD] = cplx{r == c ? 1.0 : 0.0, 0.0};
  }
  chol_bar(nthr);
  for (int k = 0; k + 1 < b; ++k) {
    const double piv = M[k + k * LD].re;
    const double inv = 1.0 / (piv > 0 ? piv : 1e-300);
    const int t = b - k - 1;
    for (int e = tid; e < t * b; e += nthr) {
      const int i = k + 1 + e / b, c = e % b;
      const cplx mi = inv * conj(M[k + i * LD]);  // M[i][k] / d_k
      if (c >= i)
        M[i + c * LD] = M[i + c * LD] - mi * M[k + c * LD];
      else if (c <= k)
        L[i + c * LD] = L[i + c * LD] - mi * L[k + c * LD];
    }
    chol_bar(nthr);
  }
  for (int j = tid; j < b; j += nthr) {
    const double piv = M[j + j * LD].re;
    if (!(piv > 0)) atomicOr(status, 4);
    rd[j] = rsqrt(piv > 0 ? piv : 1e-300);
  }
  chol_bar(nthr);
  for (int e = tid; e < b * b; e += nthr) {
    const int r = e % b, c = e / b;
    Rinv[e] = r <= c ? rd[c] * conj(L[c + r * LD]) : cplx{0, 0};
  }
}

__global__ void __launch_bounds__(32) k_chol_inv(const cplx* G, int b, cplx* Rinv, int* status) {
  __shared__ CholSmem sm;
  warp_chol_inv(G, b, Rinv, status, sm, threadIdx.x);
}

// Tinv = T^-1 of a general p x p complex T (column-major, p <= kBmMaxB) by
// Gauss-Jordan elimination with partial pivoting on one warp: [T | I] is
// reduced to [I | T^-1], lane l owning columns l and l + 32 of the
// augmented matrix.  A zero pivot sets bit 8 of *status (Tinv undefined).
__global__ void __launch_bounds__(32) k_small_inv(const cplx* __restrict__ T, int p, cplx* Tinv, int* status) {
  constexpr int LD = kBmMaxB + 1;
  __shared__ cplx M[2 * kBmMaxB * LD];  // column c at M + c LD
  __shared__ cplx fk[kBmMaxB];
  pdl_wait();
  const int lane = threadIdx.x;
  if (p < 1 || p > kBmMaxB) return;
  for (int e = lane; e < p * p; e += 32) M[(e % p) + (e / p) * LD] = T[e];
  for (int e = lane; e < p * p; e += 32) M[(e % p) + (p + e / p) * LD] = cplx{(e % p) == (e / p) ? 1.0 : 0.0, 0.0};
  __syncwarp();
  for (int k = 0; k < p; ++k) {
    // pivot row: the largest |M[i][k]|, i >= k (lowest index on ties)
    double best = -1;
    int bi = k;
    for (int i = k + lane; i < p; i += 32) {
      const double v = fabs(M[i + k * LD].re) + fabs(M[i + k * LD].im);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (!(best > 0)) {
      if (lane == 0) atomicOr(status, 8);
      return;
    }
    // swap rows k and bi, scale row k by 1 / pivot
    const cplx inv = cdiv(cplx{1, 0}, M[bi + k * LD]);
    for (int c = lane; c < 2 * p; c += 32) {
      const cplx t = M[bi + c * LD];
      M[bi + c * LD] = M[k + c * LD];
      M[k + c * LD] = inv * t;
    }
    __syncwarp();
    for (int i = lane; i < p; i += 32) fk[i] = M[i + k * LD];
    __syncwarp();
    // eliminate column k from every other row
    for (int c = lane; c < 2 * p; c += 32) {
      const cplx mk = M[k + c * LD];
      for (int i = 0; i < p; ++i)
        if (i != k) M[i + c * LD] = M[i + c * LD] - fk[i] * mk;
    }
    __syncwarp();
  }
  for (int e = lane; e < p * p; e += 32) Tinv[e] = M[(e % p) + (p + e / p) * LD];
}

// G[p] = sum_c part[c][p] (block order, deterministic): 32 entries per
// block along x, the partials split over 32 rows of threads, four
// independent sums per thread.  With Rinv set, the last block to finish
// (counter *done, reset on exit) forms Rinv = R^-1 of the Cholesky factor
// G = R^H R on one warp.
__global__ void __launch_bounds__(1024) k_block_reduce(const cplx* __restrict__ part, int nblk, int cnt, cplx* G,
                                                       unsigned* done, int b, cplx* Rinv, int* status) {
  union Smem {
    struct {
      double sr[32][33], si[32][33];
    } r;
    CholSmem chol;
  };
  __shared__ Smem sm;
  __shared__ bool last;
  auto& sr = sm.r.sr;
  auto& si = sm.r.si;
  if (blockDim.x != 32 || blockDim.y != 32) return;  // the layout below assumes 32 x 32
  pdl_wait();
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int p = blockIdx.x * 32 + tx;
  double a[4] = {0, 0, 0, 0}, c4[4] = {0, 0, 0, 0};
  if (p < cnt) {
    int c = ty;
    for (; c + 96 < nblk; c += 128) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const cplx v = part[(long)(c + 32 * u) * cnt + p];
        a[u] += v.re;
        c4[u] += v.im;
      }
    }
    for (; c < nblk; c += 32) {
      const cplx v = part[(long)c * cnt + p];
      a[0] += v.re;
      c4[0] += v.im;
    }
  }
  sr[ty][tx] = (a[0] + a[1]) + (a[2] + a[3]);
  si[ty][tx] = (c4[0] + c4[1]) + (c4[2] + c4[3]);
  __syncthreads();
  if (ty == 0 && p < cnt) {
    double x = 0, y = 0;
    for (int r = 0; r < 32; ++r) {
      x += sr[r][tx];
      y += si[r][tx];
    }
    G[p] = cplx{x, y};
  }
  if (!Rinv) return;
  __threadfence();
  __syncthreads();
  if (tx == 0 && ty == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the factor and its inverse on the warps that give every entry of a
  // step's update a thread of its own ((b - 1) b of them)
  const int nthr = ((b - 1) * b + 31) / 32 * 32 < 32 ? 32 : ((b - 1) * b + 31) / 32 * 32;
  if (ty * 32 + tx >= nthr) return;
  block_chol_inv(G, b, Rinv, status, sm.chol, ty * 32 + tx, nthr);
  if (tx == 0 && ty == 0) *done = 0;
}

// Out_j = Base_j - sum_i X_i C[i + j ldc]  (Base may be null: Out = -X C, or
// with negate = 0: Out = X C).  A block stages kUpRows rows of X (all b1
// vectors) in shared memory; thread (row, g) forms the outputs j = g, g + 4,
// ... of its row.  Out may alias Base (each element is read and written by
// one thread) and X (rows are staged before any output is written).
constexpr int kUpRows = 64;
constexpr int kUpGroups = 4;  // 256 threads
template <bool CPLX>
__global__ void __launch_bounds__(256) k_block_update(const double* __restrict__ Xre, const double* __restrict__ Xim,
                                                      int b1, const cplx* __restrict__ Cm, int ldc, int b2,
                                                      const double* Bre, const double* Bim, int negate, int n,
                                                      double* Ore, double* Oim, const double* __restrict__ Yre = nullptr,
                                                      const double* __restrict__ Yim = nullptr) {
  __shared__ cplx cs[kBmMaxB * kBmMaxB];
  __shared__ double xs_r[kBmMaxB][kUpRows], xs_i[CPLX ? kBmMaxB : 1][kUpRows];
  if (blockDim.x != 256) return;  // the staging below assumes 256 threads
  pdl_wait();
  for (int e = threadIdx.x; e < b1 * b2; e += blockDim.x) cs[e] = Cm[(e % b1) + (long)(e / b1) * ldc];
  const int rr = threadIdx.x % kUpRows, g = threadIdx.x / kUpRows;
  const long nblk = (n + kUpRows - 1) / kUpRows;
  // 256 threads: each stages kUpPer rows x vectors, loaded into registers
  // before the barrier
  constexpr int kUpPer = kBmMaxB * kUpRows / 256;
  for (long blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const long r0 = blk * kUpRows;
    double vr[kUpPer], vi[kUpPer];
#pragma unroll
    for (int u = 0; u < kUpPer; ++u) {
      const int e = threadIdx.x + u * 256;
      const int i = e / kUpRows, q = e % kUpRows;
      const long r = r0 + q;
      const bool in = i < b1 && r < n;
      vr[u] = in ? Xre[(long)i * n + r] + (Yre ? Yre[(long)i * n + r] : 0.0) : 0.0;
      vi[u] = (CPLX && in) ? Xim[(long)i * n + r] + (Yim ? Yim[(long)i * n + r] : 0.0) : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kUpPer; ++u) {
      const int e = threadIdx.x + u * 256;
      const int i = e / kUpRows, q = e % kUpRows;
      if (i < b1) {
        xs_r[i][q] = vr[u];
        if (CPLX) xs_i[i][q] = vi[u];
      }
    }
    __syncthreads();
    const long r = r0 + rr;
    if (r < n) {
      for (int j = g; j < b2; j += kUpGroups) {
        cplx acc = {0, 0};
        for (int i = 0; i < b1; ++i) acc = acc + cplx{xs_r[i][rr], CPLX ? xs_i[i][rr] : 0.0} * cs[i + j * b1];
        cplx o;
        if (Bre) o = cplx{Bre[(long)j * n + r], CPLX ? Bim[(long)j * n + r] : 0.0} - acc;
        else o = negate ? -acc : acc;
        Ore[(long)j * n + r] = o.re;
        if (CPLX) Oim[(long)j * n + r] = o.im;
      }
    }
  }
}

// part[blk * b + q] = sum over the block's rows of |Y_q[r]|^2
template <bool CPLX>
__global__ void k_colnorm2(const double* __restrict__ Yre, const double* __restrict__ Yim, int b, int n,
                           double* part) {
  __shared__ double red[kBmMaxB][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  pdl_wait();
  // every vector's loads of a row issued together (static register index),
  // each vector summed over the rows in the same order as one at a time
  double s[kBmMaxB];
#pragma unroll
  for (int q = 0; q < kBmMaxB; ++q) s[q] = 0;
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < kBmMaxB; ++q)
      if (q < b) {
        const double a = Yre[(long)q * n + r];
        s[q] += a * a;
        if (CPLX) {
          const double c = Yim[(long)q * n + r];
          s[q] += c * c;
        }
      }
  }
#pragma unroll
  for (int q = 0; q < kBmMaxB; ++q)
    if (q < b) {
      const double t = warp_sum(s[q]);
      if (lane == 0) red[q][warp] = t;
    }
  __syncthreads();
  for (int q = threadIdx.x; q < b; q += blockDim.x) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[q][w];
    part[(long)blockIdx.x * b + q] = s;
  }
}


}  // namespace oapb
