// Implicitly restarted Arnoldi (CuHArnoldi, ArnoldiPackage/ArnoldiProcedures.cpp)
// resident on one B200.
//
// Layout in HBM (per solver handle):
//   V      (m + 1) Krylov vectors of n, FP64, vector-contiguous split planes
//          (the reference stores the basis row-major with stride m,
//          oapGenericArnoldiApi.h:348-352; here vector j is one contiguous
//          run so every pass over the basis is coalesced)
//   f, w   residual and operator output, FP64 split planes
//   x32    FP32 copy of the current basis vector (mixed form)
//   A32    FP32 copy of the dense operator (mixed form), reference layout
//   H, Q   m x m complex, column-major; partial-sum buffers of the Gram-Schmidt
//
// One Arnoldi step j (executeArnoldiFactorization, ArnoldiProcedures.cpp:407-461):
//   k_normalize   v_j = f / ||f||, H[j][j-1] = ||f||          (no host sync)
//   matvec        w = A v_j                                  (HBM-bound)
//   k_gs_project  partial V^H w per row chunk
//   k_gs_reduce   h = sum of partials
//   k_gs_update   f = w - V h, partial ||f||^2
//   k_gs_finalize ||f||, ||h||, DGKS decision ||f|| < rho ||h||
//   (the same four kernels again for the DGKS pass; they return at once
//    when the device flag says the pass is not needed)
// After the m-th column one warp computes the Schur form, Ritz pairs,
// estimates and the exact-shift restart (k_hess); V <- V Q and the Sorensen
// residual update follow.  The host reads one small status block per
// restart.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <new>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "block.cuh"
#include "blockdmma.cuh"
#include "blocki8.cuh"
#include "blocktc.cuh"
#include "common.cuh"
#include "gramop.cuh"
#include "hess.cuh"
#include "matio.cuh"
#include "matvec.cuh"
#include "streamk.cuh"

namespace oapb {

constexpr int kGsThreads = 256;
constexpr int kUpdThreads = 256;

// ------------------------------------------------------------ vector kernels
__global__ void k_init_vector(double* fre, double* fim, int n, uint64_t seed, int mode) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    if (mode == OAPB_INIT_RANDOM) {
      fre[i] = uniform_pm1(seed, (uint64_t)i);
      if (fim) fim[i] = uniform_pm1(seed ^ 0x5851F42D4C957F2Dull, (uint64_t)i);
    } else {
      fre[i] = (i == 0) ? 1.0 : 0.0;
      if (fim) fim[i] = 0.0;
    }
  }
}

// part[b] = sum |x|^2 over block b's grid-stride share
__global__ void k_sumsq_partial(const double* __restrict__ xre, const double* __restrict__ xim, long n,
                                double* part) {
  double s = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double a = xre[i];
    s += a * a;
    if (xim) {
      double b = xim[i];
      s += b * b;
    }
  }
  __shared__ double red[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
  }
}

__device__ __forceinline__ double block_sum(const double* part, int np) {
  // executed by one full block; returns the sum to every thread
  __shared__ double red[32];
  __shared__ double out;
  double s = 0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) out = s;
  }
  __syncthreads();
  return out;
}

__global__ void k_set_fnorm(const double* part, int np, DevState* st) {
  double s = block_sum(part, np);
  if (threadIdx.x == 0) st->fnorm2 = s;
}

// v_j = f / ||f|| (FP64 into V, FP32 copy for the mixed matvec);
// H[j][j-1] = ||f|| (j > 0).
template <bool CPLX>
__global__ void k_normalize(const double* __restrict__ fre, const double* __restrict__ fim, int n,
                            const DevState* st, double* vre, double* vim, float* x32re, float* x32im, cplx* H,
                            int m, int j, DevState* wst) {
  const double beta = sqrt(st->fnorm2);
  const double inv = beta > 0 ? 1.0 / beta : 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double a = fre[i] * inv;
    vre[i] = a;
    if (x32re) x32re[i] = (float)a;
    if (CPLX) {
      double b = fim[i] * inv;
      vim[i] = b;
      if (x32im) x32im[i] = (float)b;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (j > 0) H[j + (long)(j - 1) * m] = cplx{st->brk ? 0.0 : beta, 0};
    if (!(beta > 0) || isinf(beta)) wst->status |= isfinite(beta) ? 1 : 4;
  }
}

// Invariant-subspace breakdown at the start of step j (j >= 1): when
// ||f|| <= 1e-12 ||A v_{j-1}||, f is replaced by a seeded random vector made
// orthogonal to v_0..v_{j-1} (two modified Gram-Schmidt sweeps) and the step
// records H[j][j-1] = 0, as ARPACK's getv0 restart does.  One CTA; returns
// at once when there is no breakdown.
template <bool CPLX>
__global__ void __launch_bounds__(1024)
k_breakdown_fix(const double* __restrict__ Vre, const double* __restrict__ Vim, int n, int j, double* fre,
                double* fim, DevState* st, uint64_t seed) {
  const double f2 = st->fnorm2, scale2 = st->hnorm2 + st->fnorm2;
  if (threadIdx.x == 0) st->brk = 0;
  if (!(f2 <= 1e-24 * scale2)) return;
  __shared__ double red[2][32];
  __shared__ double dot[2];
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    fre[i] = uniform_pm1(seed, (uint64_t)i);
    if (CPLX) fim[i] = uniform_pm1(seed ^ 0x5851F42D4C957F2Dull, (uint64_t)i);
  }
  __syncthreads();
  for (int sweep = 0; sweep < 2; ++sweep) {
    for (int v = 0; v < j; ++v) {
      const double* vr = Vre + (long)v * n;
      const double* vi = CPLX ? Vim + (long)v * n : nullptr;
      double sr = 0, si = 0;
      for (long i = threadIdx.x; i < n; i += blockDim.x) {
        double a = vr[i], x = fre[i];
        if (CPLX) {
          double b = vi[i], y = fim[i];
          sr += a * x + b * y;
          si += a * y - b * x;
        } else {
          sr += a * x;
        }
      }
      sr = warp_sum(sr);
      si = warp_sum(si);
      if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = sr;
        red[1][threadIdx.x >> 5] = si;
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        double a = threadIdx.x < (blockDim.x >> 5) ? red[0][threadIdx.x] : 0.0;
        double b = threadIdx.x < (blockDim.x >> 5) ? red[1][threadIdx.x] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        if (threadIdx.x == 0) {
          dot[0] = a;
          dot[1] = b;
        }
      }
      __syncthreads();
      const double cr = dot[0], ci = dot[1];
      for (long i = threadIdx.x; i < n; i += blockDim.x) {
        double a = vr[i];
        if (CPLX) {
          double b = vi[i];
          fre[i] -= a * cr - b * ci;
          fim[i] -= a * ci + b * cr;
        } else {
          fre[i] -= a * cr;
        }
      }
      __syncthreads();
    }
  }
  double s2 = 0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s2 += fre[i] * fre[i] + (CPLX ? fim[i] * fim[i] : 0.0);
  s2 = warp_sum(s2);
  if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = s2;
  __syncthreads();
  if (threadIdx.x < 32) {
    double a = threadIdx.x < (blockDim.x >> 5) ? red[0][threadIdx.x] : 0.0;
    a = warp_sum(a);
    if (threadIdx.x == 0) {
      st->fnorm2 = a;
      st->brk = 1;
      st->brk_count += 1;
    }
  }
}

// Partial projections: part[b * ldp + i] = sum_{r in chunk b} conj(V_i[r]) x[r]
// for i < nvec.  Warp w of the block handles vectors i = w, w + 8, ...
template <bool CPLX>
__global__ void __launch_bounds__(kGsThreads)
k_gs_project(const double* __restrict__ Vre, const double* __restrict__ Vim, int n, int nvec,
             const double* __restrict__ xre, const double* __restrict__ xim, int chunk, cplx* part, int ldp,
             const DevState* st, int gated) {
  if (gated && !st->dgks) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long r0 = (long)blockIdx.x * chunk;
  const long r1 = min((long)n, r0 + chunk);
  for (int i = warp; i < nvec; i += kGsThreads / 32) {
    const double* vr = Vre + (long)i * n;
    const double* vi = CPLX ? Vim + (long)i * n : nullptr;
    double sr = 0, si = 0;
    for (long r = r0 + lane; r < r1; r += 32) {
      double a = vr[r], x = xre[r];
      if (CPLX) {
        double b = vi[r], y = xim[r];
        sr += a * x + b * y;   // conj(v) * x
        si += a * y - b * x;
      } else {
        sr += a * x;
      }
    }
    sr = warp_sum(sr);
    if (CPLX) si = warp_sum(si);
    if (lane == 0) part[(long)blockIdx.x * ldp + i] = cplx{sr, si};
  }
}

// coef[i] = sum_b part[b][i]   (one block)
__global__ void k_gs_reduce(const cplx* part, int nblk, int ldp, int nvec, cplx* coef, const DevState* st,
                            int gated) {
  if (gated && !st->dgks) return;
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
    double a = 0, b = 0;
    for (int c = 0; c < nblk; ++c) {
      cplx v = part[(long)c * ldp + i];
      a += v.re;
      b += v.im;
    }
    coef[i] = cplx{a, b};
  }
}

// f = src - sum_i V_i coef[i]; fpart[b] = block's share of ||f||^2
template <bool CPLX>
__global__ void __launch_bounds__(kUpdThreads)
k_gs_update(const double* __restrict__ Vre, const double* __restrict__ Vim, int n, int nvec, const cplx* coef,
            const double* srcre, const double* srcim, double* fre, double* fim, double* fpart,
            const DevState* st, int gated) {
  if (gated && !st->dgks) return;
  __shared__ cplx c[kMaxM + 1];
  for (int i = threadIdx.x; i < nvec; i += blockDim.x) c[i] = coef[i];
  __syncthreads();
  double s = 0;
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
    double ar = srcre[r], ai = CPLX ? srcim[r] : 0.0;
    for (int i = 0; i < nvec; ++i) {
      double vr = Vre[(long)i * n + r];
      if (CPLX) {
        double vi = Vim[(long)i * n + r];
        ar -= vr * c[i].re - vi * c[i].im;
        ai -= vr * c[i].im + vi * c[i].re;
      } else {
        ar -= vr * c[i].re;
      }
    }
    fre[r] = ar;
    if (CPLX) fim[r] = ai;
    s += ar * ar + ai * ai;
  }
  __shared__ double red[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) fpart[blockIdx.x] = s;
  }
}

// pass 0: decide DGKS (||f|| < rho ||h||), write H[:, j] = h when no second
// pass is needed.  pass 1: h += s, write H[:, j].  Zeroes H below the column.
__global__ void k_gs_finalize(const double* fpart, int np, cplx* h, const cplx* s, cplx* H, int m, int j,
                              double rho, DevState* st, int pass, int real_basis) {
  if (pass == 1 && !st->dgks) return;
  const double f2 = block_sum(fpart, np);
  const int nvec = j + 1;
  if (pass == 0) {
    __shared__ double hn;
    if (threadIdx.x == 0) {
      double a = 0;
      for (int i = 0; i < nvec; ++i) a += abs2(h[i]);
      hn = a;
    }
    __syncthreads();
    const int dg = sqrt(f2) < rho * sqrt(hn);
    if (threadIdx.x == 0) {
      st->dgks = dg;
      st->hnorm2 = hn;
      st->fnorm2 = f2;
    }
    if (!dg)
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        cplx v = i < nvec ? h[i] : cplx{0, 0};
        if (real_basis) v.im = 0;
        H[i + (long)j * m] = v;
      }
  } else {
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      cplx v = i < nvec ? h[i] + s[i] : cplx{0, 0};
      if (real_basis) v.im = 0;
      H[i + (long)j * m] = v;
    }
    if (threadIdx.x == 0) {
      st->fnorm2 = f2;
      st->dgks_count += 1;
    }
  }
}

// out_j = sum_{i < nin} V_i C[i + j * ldc] for j < nout (V vector-contiguous,
// C column-major complex).  8 output columns per pass over V.
template <bool CPLX>
__global__ void k_vq(const double* __restrict__ Vre, const double* __restrict__ Vim, int n, int nin,
                     const cplx* __restrict__ C, int ldc, int nout, double* outre, double* outim) {
  extern __shared__ cplx cs[];
  for (int t = threadIdx.x; t < nin * nout; t += blockDim.x) cs[t] = C[(t % nin) + (long)(t / nin) * ldc];
  __syncthreads();
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
    for (int j0 = 0; j0 < nout; j0 += 8) {
      cplx acc[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[q] = {0, 0};
      const int jn = min(8, nout - j0);
      for (int i = 0; i < nin; ++i) {
        cplx v = {Vre[(long)i * n + r], CPLX ? Vim[(long)i * n + r] : 0.0};
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < jn) acc[q] = acc[q] + v * cs[i + (j0 + q) * nin];
      }
      for (int q = 0; q < jn; ++q) {
        outre[(long)(j0 + q) * n + r] = acc[q].re;
        if (CPLX) outim[(long)(j0 + q) * n + r] = acc[q].im;
      }
    }
  }
}

// f = vk * beta_hat + f * sigma  (iram_fVplusfq, oapGenericArnoldiApi.h:73-102,
// with Sorensen's indices)
template <bool CPLX>
__global__ void k_restart_f(const double* __restrict__ vkre, const double* __restrict__ vkim, double* fre,
                            double* fim, int n, const DevState* st) {
  const cplx b = st->beta_hat, s = st->sigma;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    cplx v = {vkre[i], CPLX ? vkim[i] : 0.0};
    cplx f = {fre[i], CPLX ? fim[i] : 0.0};
    cplx o = v * b + f * s;
    fre[i] = o.re;
    if (CPLX) fim[i] = o.im;
  }
}

// y = x * alpha - y  (used for residuals r = A x - lambda x, alpha = lambda)
template <bool CPLX>
__global__ void k_axmy(const double* __restrict__ xre, const double* __restrict__ xim, cplx alpha, double* yre,
                       double* yim, int n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    cplx x = {xre[i], CPLX ? xim[i] : 0.0};
    cplx y = {yre[i], CPLX ? yim[i] : 0.0};
    cplx o = y - alpha * x;
    yre[i] = o.re;
    if (CPLX) yim[i] = o.im;
  }
}

template <typename T>
__global__ void k_to_f32(const double* __restrict__ src, T* dst, long len) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x)
    dst[i] = (T)src[i];
}

// row-major (reference layout) n x k matrix from k vector-contiguous vectors
// the inverse: row-major n x k (column q = vector q) -> vector-major planes
__global__ void k_rowmajor_to_vectors(const double* __restrict__ ire, const double* __restrict__ iim, int n, int k,
                                      double* xre, double* xim) {
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < (long)n * k; t += (long)gridDim.x * blockDim.x) {
    const long q = t / n, r = t % n;
    xre[t] = ire[r * k + q];
    if (xim) xim[t] = iim ? iim[r * k + q] : 0.0;
  }
}

__global__ void k_vectors_to_rowmajor(const double* __restrict__ xre, const double* __restrict__ xim, int n, int k,
                                      double* ore, double* oim) {
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < (long)n * k; t += (long)gridDim.x * blockDim.x) {
    long r = t / k, q = t % k;
    if (ore) ore[t] = xre[q * n + r];
    if (oim) oim[t] = xim ? xim[q * n + r] : 0.0;
  }
}

}  // namespace oapb

using namespace oapb;

struct oapb_arnoldi {
  oapb_arnoldi_config cfg;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool is_c = false;
  int n = 0, m = 0, k = 0;
  // operator
  const double* a64re = nullptr;
  const double* a64im = nullptr;
  double* own64re = nullptr;   // library-owned FP64 copy (host-input solves)
  double* own64im = nullptr;
  double* hvre = nullptr;      // row-major eigenvectors staged for the host (n x k each)
  double* hvim = nullptr;
  float* a32re = nullptr;
  float* a32im = nullptr;
  bool fp32_ready = false;   // a32 holds the current operator (built on first use)
  bool mixed_ready = false;  // the mixed form's operator data (BF16 planes or FP32 copy) is current
  oapb_matvec_fn cb = nullptr;
  void* cb_user = nullptr;
  // single-vector matvec launch variants (autotuned per operator shape)
  int mv64 = 0, mv32 = 0;
  // implicit Gram operator A = X X^T (FP32 images, rows = n)
  const float* gX = nullptr;
  int gcols = 0;
  double* gws = nullptr;
  GramStream* gS = nullptr;  // the same operator with X in host memory (column blocks)
  // vectors
  double *Vre = nullptr, *Vim = nullptr;
  double *Xre = nullptr, *Xim = nullptr;   // Ritz vectors / restart scratch (m vectors)
  // the device holds a complete m-step factorization (V, H, f) of the
  // plain restart loop: after a plain solve, or loaded from a checkpoint
  bool ckpt_ready = false;
  double *fre = nullptr, *fim = nullptr, *wre = nullptr, *wim = nullptr;
  float *x32re = nullptr, *x32im = nullptr;
  double *v0re = nullptr, *v0im = nullptr;
  bool have_v0 = false;
  std::vector<double> start_shifts;
  // small
  cplx *H = nullptr, *Qs = nullptr, *ritz = nullptr, *Y = nullptr, *h = nullptr, *s = nullptr, *part = nullptr,
       *hws = nullptr;
  double *est = nullptr, *fpart = nullptr;
  int* order = nullptr;
  DevState* st = nullptr;
  int nchunk = 0, chunk = 0, nupd = 0;
  // block (multi-vector) buffers: X, W, R, E of up to kBmMaxB vectors each
  static constexpr int kBlocks = 6;
  double *Bre[kBlocks] = {}, *Bim[kBlocks] = {};
  cplx* Tinv = nullptr;   // T^-1 of the refinement's projected operator (kBmMaxB^2)
  int* ntflag = nullptr;  // [0] the near-triangular eigensolver delivered, [1] its pairs' acceptance (device words)
  std::vector<oapb_trace_rec> trace;  // convergence checks of the last solve
  cplx *bpart = nullptr, *G = nullptr, *G2 = nullptr, *Rinv = nullptr, *bY = nullptr, *bQ = nullptr, *bH = nullptr;
  cplx *britz = nullptr;
  double *best = nullptr, *bnorm = nullptr;
  int *border = nullptr, *bstatus = nullptr;
  DevState* bst = nullptr;
  int ndot = 0, nnorm = 0;
  unsigned* bdone = nullptr;  // arrival counter of k_block_reduce (self-resetting)
  // the FP32-class phase's Rayleigh-Ritz checks run on a second stream while
  // the main stream takes the next power: own Gram scratch, pinned outputs
  cudaStream_t s2 = nullptr;
  cudaEvent_t ev_w = nullptr, ev_chk = nullptr;
  // a check is in flight on s2: the tensor-core passes leave one SM to it
  // (their CTAs hold most of an SM's shared memory, so a check kernel that
  // holds an SM would otherwise hold back one CTA of the pass)
  bool side_busy = false;
  cplx* bpart2 = nullptr;
  unsigned* bdone2 = nullptr;
  unsigned char* hpin = nullptr;  // pinned: norm partials, Ritz values, DevState, tcerr
  int nvec_hess = 0;
  double* Wp = nullptr;   // split-K partials of the block matvec
  double* wdm = nullptr;  // stream-K partials of the tensor-core passes
  DmmaPlan dplan{};
  bool have_dmma = false;
  int nsplit = 1, ksplit = 0;
  // tensor-core FP32-class block pass: BF16 hi / lo operator planes
  __nv_bfloat16* abf = nullptr;   // 4 planes (2 for a real operator) of n x kp
  __nv_bfloat16* xbf = nullptr;   // B operand scratch, 2 x 64 x kp
  int kp = 0;
  int* tcerr = nullptr;
  bool have_tc = false;
  // FP64-class block pass on the integer tensor cores: int8 operator slices
  // (row scales), vector-slice scratch and its scales
  int8_t* ai8 = nullptr;
  double* ai8s = nullptr;
  int8_t* xi8 = nullptr;
  double* xi8s = nullptr;
  bool have_i8 = false;
  // ||A - hi||_F^2 of the BF16 hi planes (device, summed by the split) and
  // its host copy as ||A - hi||_F (read once per operator; < 0: not read)
  double* bf16err2 = nullptr;
  double bf16_err = -1;
  size_t hess_smem = 0;
  oapb_arnoldi_stats stats{};
  std::vector<cudaEvent_t> ev_pool;   // profiling events (pairs)
  size_t ev_used = 0;
  std::vector<int> ev_kind;           // per pair: 0 matvec, 1 block matvec; +2 if FP32
  std::vector<int> ev_b;
  // last solve outputs (host)
  std::vector<cplx> evals;
};

static int ensure_fp32_copy(oapb_arnoldi* a);

namespace {

int launch_check() { return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA; }

template <typename P>
int dalloc(P** p, size_t bytes) {
  if (cudaMalloc((void**)p, bytes) != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return OAPB_ERR_NOMEM;
  }
  return OAPB_OK;
}

int grid_n(long n) { return grid_for(n, 256, kNumSMs * 8); }
// k_block_update: one block per kUpRows rows
int grid_up(long n) { return grid_for(n, kUpRows, kNumSMs * 8); }

// Profiling: an event pair around one launch on the solver stream.
// kind 0: single-vector dense matvec, 1: block matvec
struct Timed {
  cudaEvent_t e0, e1;
  int kind, fp32, b;
};

bool prof_begin(oapb_arnoldi* a, Timed& t) {
  if (!a->cfg.profile) return false;
  while (a->ev_pool.size() < a->ev_used + 2) {
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return false;
    a->ev_pool.push_back(ev);
  }
  t.e0 = a->ev_pool[a->ev_used];
  t.e1 = a->ev_pool[a->ev_used + 1];
  a->ev_used += 2;
  a->ev_kind.push_back(t.kind + 2 * t.fp32);
  a->ev_b.push_back(t.b);
  cudaEventRecord(t.e0, a->stream);
  return true;
}
void prof_end(oapb_arnoldi* a, Timed& t) { cudaEventRecord(t.e1, a->stream); }
// a pair of events for a pass kernel alone (kind 6 + pass: 0 FP64-class,
// 1 split, 2 BF16), recorded by the launch function; nullptr without profile
const cudaEvent_t* prof_kernel_pair(oapb_arnoldi* a, int pass) {
  if (!a->cfg.profile) return nullptr;
  while (a->ev_pool.size() < a->ev_used + 2) {
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
    a->ev_pool.push_back(ev);
  }
  const cudaEvent_t* e = &a->ev_pool[a->ev_used];
  a->ev_used += 2;
  a->ev_kind.push_back(6 + pass);
  a->ev_b.push_back(0);
  return e;
}

// f <- ||f||^2 into st->fnorm2
int set_fnorm(oapb_arnoldi* a) {
  const int nb = a->nupd;
  ++a->stats.kernel_launches;
  k_sumsq_partial<<<nb, 256, 0, a->stream>>>(a->fre, a->is_c ? a->fim : nullptr, a->n, a->fpart);
  ++a->stats.kernel_launches;
  k_set_fnorm<<<1, 256, 0, a->stream>>>(a->fpart, nb, a->st);
  return launch_check();
}

// w = A x (x = basis vector j, FP64; x32 its FP32 copy)
int apply_op(oapb_arnoldi* a, const double* xre, const double* xim, double* yre, double* yim, bool fp32,
             int type) {
  cudaStream_t s = a->stream;
  const int n = a->n;
  if (a->cb) {
    oapb_mat w = {1u, (uint32_t)n, yre, a->is_c ? yim : nullptr, OAPB_F64};
    oapb_mat v = {1u, (uint32_t)n, (void*)xre, a->is_c ? (void*)xim : nullptr, OAPB_F64};
    int rc = a->cb(&w, &v, a->cb_user, type, (void*)s);
    return rc == 0 ? OAPB_OK : OAPB_ERR_CALLBACK;
  }
  if (a->gX) {
    a->stats.kernel_launches += 3;
    return launch_gram_apply(a->gX, n, a->gcols, xre, yre, a->gws, s);
  }
  if (a->gS) {
    a->stats.kernel_launches += 3 * (uint64_t)gram_stream_blocks(a->gS);
    return gram_stream_apply(a->gS, xre, yre, s);
  }
  Timed tm{nullptr, nullptr, 0, fp32 ? 1 : 0, 1};
  const bool prof = prof_begin(a, tm);
  cudaError_t e;
  ++a->stats.kernel_launches;
  if (fp32)
    e = launch_matvec<float>(a->a32re, a->is_c ? a->a32im : nullptr, n, n, a->x32re, a->is_c ? a->x32im : nullptr,
                             yre, a->is_c ? yim : nullptr, s, a->mv32);
  else
    e = launch_matvec<double>(a->a64re, a->is_c ? a->a64im : nullptr, n, n, xre, a->is_c ? xim : nullptr, yre,
                              a->is_c ? yim : nullptr, s, a->mv64);
  if (prof) prof_end(a, tm);
  if (fp32) a->stats.matvec_fp32++;
  return e == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

template <bool C>
int gs_pass(oapb_arnoldi* a, int j, const double* srcre, const double* srcim, cplx* coef, int gated) {
  cudaStream_t s = a->stream;
  const int n = a->n, nvec = j + 1;
  ++a->stats.kernel_launches;
  k_gs_project<C><<<a->nchunk, kGsThreads, 0, s>>>(a->Vre, a->Vim, n, nvec, srcre, srcim, a->chunk, a->part,
                                                    a->m + 1, a->st, gated);
  ++a->stats.kernel_launches;
  k_gs_reduce<<<1, 128, 0, s>>>(a->part, a->nchunk, a->m + 1, nvec, coef, a->st, gated);
  ++a->stats.kernel_launches;
  k_gs_update<C><<<a->nupd, kUpdThreads, 0, s>>>(a->Vre, a->Vim, n, nvec, coef, srcre, srcim, a->fre, a->fim,
                                                 a->fpart, a->st, gated);
  return launch_check();
}

template <bool C>
int arnoldi_step(oapb_arnoldi* a, int j, bool fp32) {
  cudaStream_t s = a->stream;
  const int n = a->n, m = a->m;
  double* vre = a->Vre + (long)j * n;
  double* vim = C ? a->Vim + (long)j * n : nullptr;
  if (j > 0) ++a->stats.kernel_launches;
  if (j > 0)
    k_breakdown_fix<C><<<1, 1024, 0, s>>>(a->Vre, a->Vim, n, j, a->fre, a->fim, a->st,
                                          a->cfg.seed * 7919ull + (uint64_t)(a->stats.restarts * 1024 + j));
  ++a->stats.kernel_launches;
  k_normalize<C><<<grid_n(n), 256, 0, s>>>(a->fre, a->fim, n, a->st, vre, vim, fp32 ? a->x32re : nullptr,
                                           fp32 ? a->x32im : nullptr, a->H, m, j, a->st);
  int rc = launch_check();
  if (rc) return rc;
  rc = apply_op(a, vre, vim, a->wre, a->wim, fp32, OAPB_TYPE_WV);
  if (rc) return rc;
  a->stats.matvecs++;
  if ((rc = gs_pass<C>(a, j, a->wre, a->wim, a->h, 0))) return rc;
  ++a->stats.kernel_launches;
  k_gs_finalize<<<1, 256, 0, s>>>(a->fpart, a->nupd, a->h, a->s, a->H, m, j, a->cfg.rho, a->st, 0, !C);
  if ((rc = gs_pass<C>(a, j, a->fre, a->fim, a->s, 1))) return rc;
  ++a->stats.kernel_launches;
  k_gs_finalize<<<1, 256, 0, s>>>(a->fpart, a->nupd, a->h, a->s, a->H, m, j, a->cfg.rho, a->st, 1, !C);
  return launch_check();
}

int hess(oapb_arnoldi* a, int do_shift, double tol) {
  HessArgs h;
  h.Hin = a->H;
  h.Hout = a->H;
  h.Qout = a->Qs;
  h.ritz = a->ritz;
  h.Y = a->Y;
  h.est = a->est;
  h.order = a->order;
  h.st = a->st;
  h.gws = a->hess_smem ? nullptr : a->hws;
  h.m = a->m;
  h.k = a->k;
  h.nvec = a->nvec_hess;
  h.which = a->cfg.sort;
  h.do_shift = do_shift;
  h.real_shifts = !a->is_c;
  h.dense = 0;
  h.use_beta = 1;
  h.tol = tol;
  h.beta = 0;
  ++a->stats.kernel_launches;
  launch_dependent(k_hess, dim3(1), dim3(hess_threads(h.m)), a->hess_smem, a->stream, h);
  return launch_check();
}

template <bool C>
int restart(oapb_arnoldi* a) {
  cudaStream_t s = a->stream;
  const int n = a->n, m = a->m, k = a->k;
  // X[0..k] = V Q[:, 0..k]
  const size_t shm = sizeof(cplx) * m * (k + 1);
  ++a->stats.kernel_launches;
  k_vq<C><<<grid_n(n), 256, shm, s>>>(a->Vre, a->Vim, n, m, a->Qs, m, k + 1, a->Xre, a->Xim);
  ++a->stats.kernel_launches;
  k_restart_f<C><<<grid_n(n), 256, 0, s>>>(a->Xre + (long)k * n, C ? a->Xim + (long)k * n : nullptr, a->fre,
                                           a->fim, n, a->st);
  if (cudaMemcpyAsync(a->Vre, a->Xre, sizeof(double) * k * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if (C && cudaMemcpyAsync(a->Vim, a->Xim, sizeof(double) * k * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  int rc = launch_check();
  if (rc) return rc;
  return set_fnorm(a);
}

int read_state(oapb_arnoldi* a, DevState* h) {
  if (cudaMemcpyAsync(h, a->st, sizeof(DevState), cudaMemcpyDeviceToHost, a->stream) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  return OAPB_OK;
}

// One IRAM run until the Ritz estimates reach `tol` or the restart budget
// is spent.  Returns OAPB_OK / OAPB_NOT_CONVERGED / error.
template <bool C>
int iram(oapb_arnoldi* a, bool fp32, double tol, unsigned max_restarts, int start) {
  DevState hs;
  for (unsigned r = 0;; ++r) {
    for (int j = start; j < a->m; ++j) {
      int rc = arnoldi_step<C>(a, j, fp32);
      if (rc) return rc;
    }
    const int do_shift = r < max_restarts;
    int rc = hess(a, do_shift, tol);
    if (rc) return rc;
    if ((rc = read_state(a, &hs))) return rc;
    if (hs.status & 4) return OAPB_ERR_NONFINITE;
    if (hs.status & 1) return OAPB_ERR_BREAKDOWN;
    if (hs.status & 2) return OAPB_ERR_TIMEOUT;
    a->stats.dgks_passes = hs.dgks_count;
    a->stats.symtri = (uint32_t)hs.symtri;
    if (hs.converged) return OAPB_OK;
    if (!do_shift) return OAPB_NOT_CONVERGED;
    if ((rc = restart<C>(a))) return rc;
    a->stats.restarts++;
    start = a->k;
  }
}

template <bool C>
int ritz_vectors(oapb_arnoldi* a, int nv) {
  const int n = a->n, m = a->m;
  const size_t shm = sizeof(cplx) * m * nv;
  ++a->stats.kernel_launches;
  k_vq<C><<<grid_n(n), 256, shm, a->stream>>>(a->Vre, a->Vim, n, m, a->Y, m, nv, a->Xre, a->Xim);
  return launch_check();
}

// ---------------------------------------------------------------- blocks --
// pinned check outputs: norm partials (kBmMaxB x nnorm), Ritz values
// (kBmMaxB), DevState, the tensor-core error word
size_t pin_norm_off(const oapb_arnoldi*) { return 0; }
size_t pin_ritz_off(const oapb_arnoldi* a) { return (sizeof(double) * kBmMaxB * (size_t)a->nnorm + 63) & ~(size_t)63; }
size_t pin_st_off(const oapb_arnoldi* a) { return pin_ritz_off(a) + ((sizeof(cplx) * kBmMaxB + 63) & ~(size_t)63); }
size_t pin_err_off(const oapb_arnoldi* a) { return pin_st_off(a) + ((sizeof(DevState) + 63) & ~(size_t)63); }
size_t pin_nt_off(const oapb_arnoldi* a) { return pin_err_off(a) + 64; }
size_t pin_e2_off(const oapb_arnoldi* a) { return pin_nt_off(a) + 64; }
size_t pin_bytes(const oapb_arnoldi* a) { return pin_e2_off(a) + 64; }

int alloc_blocks(oapb_arnoldi* a) {
  if (a->Bre[0]) return OAPB_OK;
  const size_t vb = sizeof(double) * (size_t)a->n * kBmMaxB;
  int rc = OAPB_OK;
  for (int i = 0; i < oapb_arnoldi::kBlocks; ++i) {
    rc |= dalloc(&a->Bre[i], vb);
    if (a->is_c) rc |= dalloc(&a->Bim[i], vb);
  }
  a->ndot = (a->n + kDotChunk - 1) / kDotChunk;
  if (a->ndot > kDotBlocks) a->ndot = kDotBlocks;
  {
    const long tiles = (a->n + kBmRows - 1) / kBmRows;
    long sp = (6L * kNumSMs + tiles - 1) / tiles;
    if (sp < 1) sp = 1;
    if (sp > 8) sp = 8;
    long ks = (a->n + sp - 1) / sp;
    ks = ((ks + 63) / 64) * 64;  // a multiple of the 64-wide tensor-core K chunk
    a->ksplit = (int)ks;
    a->nsplit = (int)((a->n + ks - 1) / ks);
    rc |= dalloc(&a->Wp, sizeof(double) * 2 * (size_t)kBmMaxB * a->n * a->nsplit);
  }
  if (!a->cb && !a->gX && !a->gS) {  // stream-K partials of the tensor-core passes (FP64 DMMA and split-BF16)
    size_t need = btc_workspace(a->n, (a->n + 127) / 128 * 128);
    need = std::max(need, i8_workspace(a->n, (a->n + 127) / 128 * 128));
    if (dmma_plan(a->n, &a->dplan)) {
      need = std::max(need, dmma_workspace(a->dplan));
      a->have_dmma = true;
    }
    rc |= dalloc(&a->wdm, sizeof(double) * need);
  }
  a->nnorm = grid_for(a->n, 256, kNumSMs * 2);
  const size_t bb = sizeof(cplx) * kBmMaxB * kBmMaxB;
  rc |= dalloc(&a->bpart, bb * (size_t)a->ndot);
  rc |= dalloc(&a->bdone, sizeof(unsigned));
  if (a->bdone && cudaMemset(a->bdone, 0, sizeof(unsigned)) != cudaSuccess) rc |= OAPB_ERR_CUDA;
  rc |= dalloc(&a->G, bb);
  rc |= dalloc(&a->G2, bb);
  rc |= dalloc(&a->Rinv, bb);
  rc |= dalloc(&a->bY, bb);
  rc |= dalloc(&a->bQ, bb);
  rc |= dalloc(&a->bH, bb);
  rc |= dalloc(&a->britz, sizeof(cplx) * kBmMaxB);
  rc |= dalloc(&a->Tinv, bb);
  rc |= dalloc(&a->ntflag, 2 * sizeof(int));
  if (a->ntflag) {  // delivered = 0, ok = 1 (k_eig_near_tri_finish sets ok again after each use)
    const int init[2] = {0, 1};
    if (cudaMemcpy(a->ntflag, init, sizeof(init), cudaMemcpyHostToDevice) != cudaSuccess) rc |= OAPB_ERR_CUDA;
  }
  rc |= dalloc(&a->best, sizeof(double) * kBmMaxB);
  rc |= dalloc(&a->bnorm, sizeof(double) * kBmMaxB * (size_t)a->nnorm);
  rc |= dalloc(&a->border, sizeof(int) * kBmMaxB);
  rc |= dalloc(&a->bstatus, sizeof(int));
  rc |= dalloc(&a->bst, sizeof(DevState));
  rc |= dalloc(&a->bpart2, bb * (size_t)a->ndot);
  rc |= dalloc(&a->bdone2, sizeof(unsigned));
  if (a->bdone2 && cudaMemset(a->bdone2, 0, sizeof(unsigned)) != cudaSuccess) rc |= OAPB_ERR_CUDA;
  if (cudaMallocHost((void**)&a->hpin, pin_bytes(a)) != cudaSuccess) {
    a->hpin = nullptr;
    cudaGetLastError();
    rc |= OAPB_ERR_NOMEM;
  }
  return rc ? OAPB_ERR_NOMEM : OAPB_OK;
}

// G (b1 x b2, column-major) = X^H Y
template <bool C>
void block_gram(oapb_arnoldi* a, const double* xr, const double* xi, int b1, const double* yr, const double* yi,
                int b2, cplx* G) {
  a->stats.kernel_launches += 2;
  launch_dependent(k_block_dot<C>, dim3(a->ndot), dim3(256), 0, a->stream, xr, xi, b1, yr, yi, b2, a->n, a->bpart);
  launch_dependent(k_block_reduce, dim3((b1 * b2 + 31) / 32), dim3(32, 32), 0, a->stream, a->bpart, a->ndot, b1 * b2,
                   G, a->bdone, 0, nullptr, nullptr);
}

// W = A X (b vectors); FP32-class operator copy when fp32, else FP64.
// bf16 (with fp32): on the tensor cores, the BF16 hi planes alone.
// smallest residual goal the FP64-class int8-slice pass serves
constexpr double kI8MinTolerance = 1e-12;

// OAPB_SIDE_SM_RESERVE=0 turns the SM left to an overlapped check off (for
// A/B timing); on by default
static bool side_sm_reserve() {
  static const int v = [] {
    const char* e = getenv("OAPB_SIDE_SM_RESERVE");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return v != 0;
}

template <bool C>
int block_apply(oapb_arnoldi* a, const double* xr, const double* xi, int b, double* wr, double* wi,
                bool fp32 = false, bool bf16 = false, bool coarse = false) {
  if (a->cb || a->gX || a->gS) {
    for (int q = 0; q < b; ++q) {
      int rc = apply_op(a, xr + (long)q * a->n, C ? xi + (long)q * a->n : nullptr, wr + (long)q * a->n,
                        C ? wi + (long)q * a->n : nullptr, false, OAPB_TYPE_EIGENVECTOR);
      if (rc) return rc;
    }
    return OAPB_OK;
  }
  const int tiles = (a->n + kBmRows - 1) / kBmRows;
  dim3 grid(tiles, a->nsplit);
  a->stats.kernel_launches += 2;
  const bool tcp = fp32 && a->have_tc && a->cfg.tensor_cores;
  if (fp32 && !tcp) {  // the CUDA-core FP32 pass reads the FP32 copy
    const int rc = ensure_fp32_copy(a);
    if (rc) return rc;
  }
  Timed tm{nullptr, nullptr, 1, fp32 ? (tcp && bf16 ? 2 : 1) : 0, b};
  const bool prof = prof_begin(a, tm);
  if (tcp) {
    BtcOperator op{a->abf, a->abf + (size_t)a->n * a->kp, C ? a->abf + 2 * (size_t)a->n * a->kp : nullptr,
                   C ? a->abf + 3 * (size_t)a->n * a->kp : nullptr, a->n, a->kp};
    const int ctas = (a->side_busy && side_sm_reserve()) ? kNumSMs - 1 : kNumSMs;
    const cudaEvent_t* kev = prof ? prof_kernel_pair(a, bf16 ? 2 : 1) : nullptr;
    int rc = launch_block_matvec_tc(op, xr, xi, b, wr, wi, a->xbf, a->xbf + 64 * (size_t)a->kp, a->wdm,
                                    a->tcerr, a->stream, bf16, bf16 && coarse, ctas, kev);
    if (bf16) a->stats.block_bf16++;
    if (prof) prof_end(a, tm);
    if (rc) return rc;
    a->stats.block_matvecs++;
    return launch_check();
  }
  // the int8-slice pass certifies residuals to about 2^-42 of the row scale:
  // tighter goals keep the FP64 DMMA pass
  if (!fp32 && a->have_i8 && a->mixed_ready && a->cfg.tensor_cores && b <= i8_max_vectors(C) &&
      a->cfg.tolerance >= kI8MinTolerance) {
    const I8Operator op{a->ai8, a->ai8s, a->n, a->kp, C};
    const cudaEvent_t* kev = prof ? prof_kernel_pair(a, 0) : nullptr;
    int rc = launch_block_matvec_i8(op, xr, xi, b, wr, wi, a->xi8, a->xi8s, a->wdm, a->tcerr, a->stream, kev);
    if (prof) prof_end(a, tm);
    if (rc) return rc;
    a->stats.block_matvecs++;
    a->stats.block_i8++;
    return launch_check();
  }
  if (!fp32 && a->have_dmma && a->cfg.tensor_cores) {
    const uintptr_t al64 = (uintptr_t)a->a64re | (uintptr_t)(C ? (const void*)a->a64im : nullptr) | (uintptr_t)xr |
                           (uintptr_t)(C ? (const void*)xi : nullptr);
    if (al64 % 16 == 0) {
      int rc = launch_block_matvec_dmma(a->a64re, C ? a->a64im : nullptr, a->n, xr, xi, b, wr, wi, a->dplan, a->wdm,
                                        a->stream);
      if (prof) prof_end(a, tm);
      if (rc) return rc;
      a->stats.block_matvecs++;
      return launch_check();
    }
  }
  const uintptr_t al = fp32 ? ((uintptr_t)a->a32re | (uintptr_t)(C ? (const void*)a->a32im : nullptr))
                            : ((uintptr_t)a->a64re | (uintptr_t)(C ? (const void*)a->a64im : nullptr));
  const int vec_ok = (al % 16 == 0) && (a->n % 4 == 0);
  if (fp32)
    k_block_matvec<float, C><<<grid, kBmThreads, 0, a->stream>>>(a->a32re, a->a32im, a->n, xr, xi, b, a->ksplit,
                                                                a->Wp, vec_ok);
  else
    k_block_matvec<double, C><<<grid, kBmThreads, 0, a->stream>>>(a->a64re, a->a64im, a->n, xr, xi, b, a->ksplit,
                                                                 a->Wp, vec_ok);
  if (prof) prof_end(a, tm);
  k_split_reduce<C><<<grid_n((long)b * a->n), 256, 0, a->stream>>>(a->Wp, a->nsplit, b, a->n, wr, wi);
  a->stats.block_matvecs++;
  return launch_check();
}

// host copy of the column norms ||Y_q|| for q < b (synchronises)
template <bool C>
int col_norms(oapb_arnoldi* a, const double* yr, const double* yi, int b, double* out) {
  ++a->stats.kernel_launches;
  launch_dependent(k_colnorm2<C>, dim3(a->nnorm), dim3(256), 0, a->stream, yr, yi, b, a->n, a->bnorm);
  std::vector<double> h((size_t)b * a->nnorm);
  if (cudaMemcpyAsync(h.data(), a->bnorm, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, a->stream) !=
      cudaSuccess)
    return OAPB_ERR_CUDA;
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  for (int q = 0; q < b; ++q) {
    double s = 0;
    for (int blk = 0; blk < a->nnorm; ++blk) s += h[(size_t)blk * b + q];
    out[q] = sqrt(s);
  }
  return OAPB_OK;
}

// X <- orthonormal basis of span(Win) by two CholeskyQR passes (Win is kept)
template <bool C>
int cholqr2(oapb_arnoldi* a, const double* wr, const double* wi, int b, double* xr, double* xi, double* tr,
            double* ti, int passes = 2) {
  const double* sr = wr;
  const double* si = wi;
  for (int pass = 0; pass < passes; ++pass) {
    double* dr = pass + 1 < passes ? tr : xr;
    double* di = pass + 1 < passes ? ti : xi;
    // Gram matrix, then (last reduce block) its Cholesky factor and R^-1
    a->stats.kernel_launches += 3;
    launch_dependent(k_block_dot<C>, dim3(a->ndot), dim3(256), 0, a->stream, sr, si, b, sr, si, b, a->n, a->bpart);
    launch_dependent(k_block_reduce, dim3((b * b + 31) / 32), dim3(32, 32), 0, a->stream, a->bpart, a->ndot, b * b,
                     a->G2, a->bdone, b, a->Rinv, a->bstatus);
    launch_dependent(k_block_update<C>, dim3(grid_up(a->n)), dim3(256), 0, a->stream, sr, si, b, a->Rinv, b, b, nullptr, nullptr, 0, a->n, dr, di, nullptr, nullptr);
    sr = dr;
    si = di;
  }
  return launch_check();
}

// small dense eigenproblem of the b x b matrix G on one warp (Hessenberg
// reduction + Schur + eigenvectors of the first nv values in sort order);
// fp32: FP32 working arithmetic (the FP32-class phase's checks)
// near_tri (FP64, b <= 32): G is nearly upper triangular (the Rayleigh
// quotient of orthonormalised Ritz vectors): inverse iteration per pair
// first, the Schur path only when that does not deliver.
int small_eig(oapb_arnoldi* a, const cplx* G, int b, int kk, int nv, bool fp32 = false, bool near_tri = false) {
  HessArgs h;
  h.Hin = G;
  h.Hout = a->bH;
  h.Qout = a->bQ;
  h.ritz = a->britz;
  h.Y = a->bY;
  h.est = a->best;
  h.order = a->border;
  h.st = a->bst;
  h.gws = nullptr;
  h.m = b;
  h.k = kk;
  h.nvec = nv;
  h.which = a->cfg.sort;
  h.do_shift = 0;
  h.real_shifts = 0;
  h.dense = 1;
  h.use_beta = 0;
  h.tol = 0;
  h.beta = 0;
  ++a->stats.kernel_launches;
  if (near_tri && !fp32 && b <= 32 && a->ntflag) {
    // one CTA per pair (V, th in the unused bQ / bH scratch), then the
    // acceptance and ordering; ntflag[0] = delivered, ntflag[1] = ok
    a->stats.kernel_launches += 2;
    launch_dependent(k_eig_near_tri, dim3(b), dim3(32), nt_smem_bytes(b), a->stream, (const cplx*)G, b, a->bQ,
                     a->bH, a->ntflag + 1);
    launch_dependent(k_eig_near_tri_finish, dim3(1), dim3(32), 0, a->stream, b, (int)a->cfg.sort,
                     (const cplx*)a->bQ, (const cplx*)a->bH, a->ntflag + 1, a->britz, a->bY, a->border, a->ntflag);
    h.skip = a->ntflag;
  }
  if (fp32)
    launch_dependent(k_hess_f32, dim3(1), dim3(hess_threads(b)), sizeof(cplxf) * hess_ws_cplx(b), a->stream, h);
  else
    launch_dependent(k_hess, dim3(1), dim3(hess_threads(b)), sizeof(cplx) * hess_ws_cplx(b), a->stream, h);
  return launch_check();
}

// Rayleigh-Ritz check of the block X (b vectors) with W = A X, enqueued on
// stream cs: G = X^H W, R = W - X G, the eigenpairs (theta, S) of G, E = R S
// (kk columns), the column-norm partials of E, the Ritz values, the small
// eigensolver's state and the tensor-core error word copied to pinned host
// memory; a->ev_chk is recorded on cs.  With cs != a->stream the check uses
// the second Gram scratch, so that the main stream may run cholqr2 and the
// next pass meanwhile (they read X and W and write neither).
template <bool C>
int check_enqueue(oapb_arnoldi* a, cudaStream_t cs, const double* X, const double* Xi, const double* W,
                  const double* Wi, double* R, double* Ri, double* E, double* Ei, int b, int kk, int nv, bool fp32,
                  bool near_tri = false) {
  const int n = a->n;
  const bool side = cs != a->stream;
  cudaStream_t s0 = a->stream;
  cplx* bp0 = a->bpart;
  unsigned* bd0 = a->bdone;
  a->stream = cs;
  if (side) {
    a->bpart = a->bpart2;
    a->bdone = a->bdone2;
  }
  block_gram<C>(a, X, Xi, b, W, Wi, b, a->G);
  a->stats.kernel_launches += 3;
  launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, cs, X, Xi, b, a->G, b, b, W, Wi, 1, n, R, Ri, nullptr, nullptr);
  int rc = small_eig(a, a->G, b, kk, nv, fp32, near_tri);
  if (!rc) {
    launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, cs, R, Ri, b, a->bY, b, kk, nullptr, nullptr, 0, n, E, Ei, nullptr, nullptr);
    launch_dependent(k_colnorm2<C>, dim3(a->nnorm), dim3(256), 0, cs, E, Ei, kk, n, a->bnorm);
    rc = launch_check();
  }
  a->stream = s0;
  a->bpart = bp0;
  a->bdone = bd0;
  if (rc) return rc;
  unsigned char* hp = a->hpin;
  if (cudaMemcpyAsync(hp + pin_norm_off(a), a->bnorm, sizeof(double) * kk * (size_t)a->nnorm, cudaMemcpyDeviceToHost,
                      cs) != cudaSuccess ||
      cudaMemcpyAsync(hp + pin_ritz_off(a), a->britz, sizeof(cplx) * b, cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
      cudaMemcpyAsync(hp + pin_st_off(a), a->bst, sizeof(DevState), cudaMemcpyDeviceToHost, cs) != cudaSuccess)
    return OAPB_ERR_CUDA;
  *(int*)(hp + pin_err_off(a)) = 0;
  if (a->tcerr &&
      cudaMemcpyAsync(hp + pin_err_off(a), a->tcerr, sizeof(int), cudaMemcpyDeviceToHost, cs) != cudaSuccess)
    return OAPB_ERR_CUDA;
  *(int*)(hp + pin_nt_off(a)) = 0;
  if (near_tri && b <= 32 &&
      cudaMemcpyAsync(hp + pin_nt_off(a), a->ntflag, sizeof(int), cudaMemcpyDeviceToHost, cs) != cudaSuccess)
    return OAPB_ERR_CUDA;
  a->side_busy = side;
  *(double*)(hp + pin_e2_off(a)) = -1;  // the BF16 rounding energy rides along until known
  if (a->bf16_err < 0 && a->bf16err2 &&
      cudaMemcpyAsync(hp + pin_e2_off(a), a->bf16err2, sizeof(double), cudaMemcpyDeviceToHost, cs) != cudaSuccess)
    return OAPB_ERR_CUDA;
  return cudaEventRecord(a->ev_chk, cs) == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

// wait for the enqueued check: Ritz values (b) and residual norms ||E_q|| (kk)
int check_collect(oapb_arnoldi* a, int b, int kk, cplx* th, double* norms) {
  a->side_busy = false;
  if (cudaEventSynchronize(a->ev_chk) != cudaSuccess) return OAPB_ERR_CUDA;
  const unsigned char* hp = a->hpin;
  const double* part = (const double*)(hp + pin_norm_off(a));
  for (int q = 0; q < kk; ++q) {
    double s = 0;
    for (int blk = 0; blk < a->nnorm; ++blk) s += part[(size_t)blk * kk + q];
    norms[q] = sqrt(s);
  }
  memcpy(th, hp + pin_ritz_off(a), sizeof(cplx) * b);
  DevState bs;
  memcpy(&bs, hp + pin_st_off(a), sizeof(DevState));
  const int tcerr = *(const int*)(hp + pin_err_off(a));
  if (*(const int*)(hp + pin_nt_off(a))) a->stats.eig_fast++;
  const double e2 = *(const double*)(hp + pin_e2_off(a));
  if (a->bf16_err < 0 && e2 >= 0) a->bf16_err = sqrt(e2);
  return ((bs.status & 2) || tcerr) ? OAPB_ERR_TIMEOUT : OAPB_OK;
}

// second stream and events of the overlapped checks (created once)
int ensure_side_stream(oapb_arnoldi* a) {
  if (a->s2) return OAPB_OK;
  if (cudaEventCreateWithFlags(&a->ev_w, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->ev_chk, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&a->s2, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return OAPB_ERR_CUDA;
  }
  return OAPB_OK;
}

constexpr int kSlow = 100;   // subspace(): convergence too slow for the iteration budget
constexpr int kMixedMinN = 8192;
// The chosen form for small dense operators: the whole restart loop of one
// problem in one CTA (the batched kernel's solver with a batch of one), with
// no launch or host round trip per Arnoldi step.  Up to n = 2048 and
// hdim = 32 (the batched kernel's limits).
constexpr int kOnchipMaxN = 2048;
constexpr int kOnchipMaxM = 32;
// BF16 operator passes (tensor cores only).  In the FP32-class subspace
// iteration: the powers taken while the block is still far from the wanted
// subspace (before the first check, then while the residual extrapolated
// from the last check stays above kBf16Until), never the pass right before
// a check, so that their rounding (about 2^-8 of the block) is damped by
// FP32-class powers before any residual is measured.  In the refinement's
// fixed point: the leading sweeps, as many as leave the last sweeps on the
// FP32-class operator to contract the BF16 error (bf16_sweep_error, at most
// kBf16Err) to the correction's goal.
constexpr double kBf16Until = 0.02;
constexpr double kBf16Err = 4e-3;
// Goal of the FP32-class phase, the hand-over to the refinement: one outer
// refinement step leaves about 5e-6 (the FP32-class accuracy of the
// correction) of the residual it starts from, so from 5e-6 a single step
// reaches 1e-10 with margin; the FP32-class floor itself lies near 1e-6.
constexpr double kFp32Goal = 5e-6;

// Block subspace iteration with Rayleigh-Ritz on b vectors:
//   W = A X; G = X^H W; R = W - X G; G = S diag(theta) S^-1;
//   residual_q = ||R s_q|| / (max |theta| ||s_q||);  X <- orth(W)
// The start block is a->Xre (orthonormalised here) or, with from_bx, the
// current block buffer.  fp32 selects the FP32 operator copy; that phase
// stops at `tol` or when the residuals stop falling (the FP32 floor).
// Returns OAPB_OK (goal met: Ritz vectors in a->Xre, values in a->evals),
// kSlow when the observed rate cannot reach the goal within the budget,
// OAPB_NOT_CONVERGED or an error.
// fp32 phase: one CholeskyQR pass per iteration (the FP32 operator's
// rounding dominates), hand-over of the first `b_next` Ritz vectors in
// a->Xre; the observed per-iteration contraction goes to *rate_out.
// FP64 phase: two passes; the first `skip` iterations carry no check.
template <bool C>
int subspace(oapb_arnoldi* a, int b, bool fp32, double tol, unsigned max_it, double* res_out, bool from_bx,
             int b_next = 0, double* rate_out = nullptr, int skip = 0, double* floor_out = nullptr,
             std::vector<cplx>* ritz_out = nullptr) {
  const int passes = fp32 ? 1 : 2;
  const int n = a->n, kk = a->k;
  double *X = a->Bre[0], *W = a->Bre[1], *R = a->Bre[2], *E = a->Bre[3];
  double *Xi = a->Bim[0], *Wi = a->Bim[1], *Ri = a->Bim[2], *Ei = a->Bim[3];
  double *Xn = a->Bre[4], *Wn = a->Bre[5], *Xni = a->Bim[4], *Wni = a->Bim[5];  // the overlapped next power
  if (cudaMemsetAsync(a->bstatus, 0, sizeof(int), a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  if (cudaMemsetAsync(a->bst, 0, sizeof(DevState), a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  int rc = OAPB_OK;
  if (fp32 && (rc = ensure_side_stream(a))) return rc;
  // the FP32 phase starts from a zero-mean uniform random block (condition
  // number near 1): one CholeskyQR pass is orthonormal to rounding
  if (!from_bx && (rc = cholqr2<C>(a, a->Xre, a->Xim, b, X, Xi, E, Ei, passes))) return rc;
  const int nv = (fp32 && b_next > kk) ? b_next : kk;
  std::vector<double> norms(kk), hist;
  std::vector<int> hist_it;
  std::vector<cplx> th(b);
  // In the FP32 phase the first Rayleigh-Ritz checks carry no decision:
  // from a random block the wanted directions need several powers before
  // the residuals mean anything, so the first check is at iteration 6 (after
  // five BF16 powers and one FP32-class one), the second two later, and from
  // then on at the iteration the observed contraction predicts for the goal
  // (each check costs a small dense eigensolve and a host synchronisation).
  unsigned next_check = 6;
  // FP32 phase: CholeskyQR only where the block's columns could drift
  // apart by more than 1e3 since the last one (growth per iteration = the
  // spread |theta|max / |theta|min of the last Rayleigh-Ritz values, known
  // from the first check on) and always right before a check; otherwise the
  // next pass takes W itself (the span is what the iteration carries).
  double growth = 0, drift = 1;
  // FP32 phase: a check that is not expected to meet the goal runs on the
  // second stream while the main stream orthonormalises W and takes the
  // next power into (Xn, Wn); `pre` marks an iteration whose W is there.
  bool pre = false;
  for (unsigned it = 0; it < max_it; ++it) {
    bool bf16 = false;
    if (fp32 && !from_bx && it + 1 < next_check) {
      const size_t h = hist.size();
      double est = 1.0;  // before the first check: a random block
      if (h) {
        const double r = h >= 2 ? pow(hist[h - 1] / hist[h - 2], 1.0 / (hist_it[h - 1] - hist_it[h - 2])) : 0.5;
        est = hist[h - 1] * pow(r < 1.0 ? r : 1.0, (double)((int)it - hist_it[h - 1]));
      }
      bf16 = est >= kBf16Until;
    }
    // (the BF16 powers of a block still far from the subspace round X to
    // BF16 too: its 2^-8 is as far below that distance as the operator's)
    if (!pre && (rc = block_apply<C>(a, X, Xi, b, W, Wi, fp32, bf16, bf16))) return rc;
    pre = false;
    const bool check = fp32 ? (it >= next_check || it + 1 == max_it)
                            : ((int)it >= skip || it + 1 == max_it);
    if (!check) {
      const bool before_check = it + 1 >= next_check || it + 2 == max_it;
      if (fp32 && growth > 0 && !before_check && drift * growth <= 1e3) {
        drift *= growth;
        std::swap(X, W);
        if (C) std::swap(Xi, Wi);
        continue;
      }
      drift = 1;
      if ((rc = cholqr2<C>(a, W, Wi, b, X, Xi, E, Ei, passes))) return rc;
      continue;
    }
    // overlap unless this check is predicted to meet the goal
    bool overlap = fp32 && it + 1 < max_it && hist.size() < 2;
    if (fp32 && it + 1 < max_it && hist.size() >= 2) {
      const size_t h = hist.size();
      const double r = pow(hist[h - 1] / hist[h - 2], 1.0 / (hist_it[h - 1] - hist_it[h - 2]));
      overlap = !(r < 1.0 && hist[h - 1] * pow(r, (double)((int)it - hist_it[h - 1])) <= 1.5 * tol);
    }
    const uint32_t passes_now = a->stats.block_matvecs, bf16_now = a->stats.block_bf16;
    if (overlap) {
      if (cudaEventRecord(a->ev_w, a->stream) != cudaSuccess || cudaStreamWaitEvent(a->s2, a->ev_w, 0) != cudaSuccess)
        return OAPB_ERR_CUDA;
    }
    if ((rc = check_enqueue<C>(a, overlap ? a->s2 : a->stream, X, Xi, W, Wi, R, Ri, E, Ei, b, kk, nv, fp32)))
      return rc;
    if (overlap) {  // X' = orth(W), W' = A X' meanwhile
      if ((rc = cholqr2<C>(a, W, Wi, b, Xn, Xni, E, Ei, 1))) return rc;
      if ((rc = block_apply<C>(a, Xn, Xni, b, Wn, Wni, true, false))) return rc;
    }
    if ((rc = check_collect(a, b, kk, th.data(), norms.data()))) return rc;
    double scale = 0;
    for (int q = 0; q < kk; ++q) scale = fmax(scale, cabs_(th[q]));
    if (scale == 0) scale = 1;
    {
      double tmin = 1e300, tmax = 0;
      for (int q = 0; q < b; ++q) {
        tmin = fmin(tmin, cabs_(th[q]));
        tmax = fmax(tmax, cabs_(th[q]));
      }
      growth = tmin > 0 ? tmax / tmin : 0;
      drift = 1;
    }
    double mx = 0;
    for (int q = 0; q < kk; ++q) {
      res_out[q] = norms[q] / scale;
      mx = fmax(mx, res_out[q]);
    }
    hist.push_back(mx);
    hist_it.push_back((int)it);
    a->stats.refine_iterations++;
    a->trace.push_back({fp32 ? 1 : 2, (int)it, passes_now, bf16_now, mx});
    const bool done = mx <= tol;
    bool stop = done;
    if (fp32) {
      unsigned step = 2;
      const size_t h = hist.size();
      if (h >= 2 && !done) {
        const double r2 = pow(mx / hist[h - 2], 1.0 / (hist_it[h - 1] - hist_it[h - 2]));
        if (r2 > 0 && r2 < 0.9) {
          // the iteration the observed contraction predicts for the goal: a
          // check that comes one iteration early costs a Rayleigh-Ritz step
          // and a host synchronisation, about as much as one pass more
          const double need = log(tol / mx) / log(r2);
          step = need < 1.1 ? 1u : (unsigned)ceil(need - 0.1);
          if (step > 6) step = 6;
        }
      }
      next_check = it + step;
    }
    if (!done && hist.size() >= 3) {
      const size_t h = hist.size();
      const double r0 = hist[h - 3], r1 = mx;
      const int span = hist_it[h - 1] - hist_it[h - 3];
      const double rate = (r0 > 0 && r1 > 0 && span > 0) ? pow(r1 / r0, 1.0 / span) : 1.0;  // per iteration
      // the contraction of the iteration, not the stagnation at the FP32 floor
      if (rate_out && (*rate_out <= 0 || rate < *rate_out)) *rate_out = rate;
      if (fp32 && mx < 1e-4 && rate > 0.75) stop = true;  // FP32 floor reached
      if (!stop) {
        const double need = rate < 1.0 ? log(tol / mx) / log(rate) : 1e30;
        if (rate > 0.92 || need > (double)(max_it - it - 1)) return kSlow;
      }
    }
    if (stop || it + 1 == max_it) {
      if (fp32) {  // the FP32 operator's residuals are not the goal: always hand over
        // hand the first b_next Ritz vectors X s_q to the FP64 phase
        const int bn = b_next > kk ? b_next : b;
        a->stats.kernel_launches += 1;
        if (bn == b) {
          if ((rc = cholqr2<C>(a, W, Wi, b, a->Xre, a->Xim, E, Ei, 1))) return rc;
        } else {
          launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, X, Xi, b, a->bY, b, bn, nullptr, nullptr, 0, n, a->Xre, a->Xim, nullptr, nullptr);
        }
        if (floor_out) *floor_out = mx;
        if (ritz_out) *ritz_out = th;
        return launch_check();
      }
      a->stats.kernel_launches += 1;
      launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, X, Xi, b, a->bY, b, kk, nullptr, nullptr, 0, n, a->Xre, a->Xim, nullptr, nullptr);
      a->evals.assign(th.begin(), th.begin() + kk);
      if ((rc = launch_check())) return rc;
      return done ? OAPB_OK : OAPB_NOT_CONVERGED;
    }
    if (overlap) {  // the next power is there: X <- orth(W), W <- A X
      std::swap(X, Xn);
      std::swap(W, Wn);
      std::swap(Xi, Xni);
      std::swap(Wi, Wni);
      pre = true;
      continue;
    }
    if ((rc = cholqr2<C>(a, W, Wi, b, X, Xi, E, Ei, passes))) return rc;
  }
  return OAPB_NOT_CONVERGED;
}

// Out = X + Y (b vectors)
__global__ void k_block_add(const double* __restrict__ xr, const double* __restrict__ xi, const double* __restrict__ yr,
                            const double* __restrict__ yi, int b, int n, double* outr, double* outi) {
  pdl_wait();
  const long len = (long)b * n;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x) {
    outr[e] = xr[e] + yr[e];
    outi[e] = xi[e] + yi[e];
  }
}

// Relative error a BF16 sweep of the refinement leaves in the correction:
// ||A - hi||_2 / min |theta|, with ||A - hi||_2 estimated from the rounding
// energy the split summed as 2 ||A - hi||_F / sqrt(n) (rounding errors act
// like independent random entries, whose matrix has that norm), clamped to
// [kBf16Err / 16, kBf16Err].
static double bf16_sweep_error(oapb_arnoldi* a, const std::vector<cplx>& th) {
  if (a->bf16_err < 0 && a->bf16err2) {
    double e2 = -1;
    if (cudaMemcpyAsync(&e2, a->bf16err2, sizeof(double), cudaMemcpyDeviceToHost, a->stream) == cudaSuccess &&
        cudaStreamSynchronize(a->stream) == cudaSuccess && e2 >= 0)
      a->bf16_err = sqrt(e2);
  }
  double tmin = 1e300;
  for (const cplx& t : th) tmin = fmin(tmin, cabs_(t));
  if (!(a->bf16_err >= 0) || !(tmin > 0) || tmin >= 1e300) return kBf16Err;
  const double e = 2.0 * a->bf16_err / sqrt((double)a->n) / tmin;
  return e < kBf16Err / 16 ? kBf16Err / 16 : (e > kBf16Err ? kBf16Err : e);
}

// FP64-anchored refinement of the wanted invariant subspace (complex
// operator, largest-magnitude wanted set, p = k vectors from a->Xre).
// Outer step: W = A X on the FP64 operator, T = X^H W, R = W - X T.  From
// the second step on, Rayleigh-Ritz T S = S Theta checks the pairs, which
// are accepted when every ||R s_q|| / (max |theta| ||s_q||) <= tol; the
// first step starts from the FP32-class phase's residual res0 (Ritz values
// th0) and takes no check.  The correction D (orthogonal to X) of the
// projected Sylvester equation
//     P A D - D T = -R,   P = I - X X^H,
// is computed by the fixed point D <- (P A D + R) T^-1 on the FP32-class
// operator (contraction about rho = |theta_{k+1}| / |theta_k|; T^-1 by
// Gauss-Jordan on one warp) and X <- orth(X + D).  The outer iteration
// converges quadratically, so the FP64 operator is applied about twice per
// solve; the FP32-class operator's rounding enters only through the small
// correction.  Returns OAPB_OK, kSlow (no quadratic progress) or an error.
template <bool C>
int refine(oapb_arnoldi* a, double tol, double rho, double res0, const std::vector<cplx>& th0, double* res_out,
           int max_outer = 3) {
  const int n = a->n, p = a->k;
  double *X = a->Bre[0], *W = a->Bre[1], *R = a->Bre[2], *E = a->Bre[3], *D = a->Bre[4], *Tm = a->Bre[5];
  double *Xi = a->Bim[0], *Wi = a->Bim[1], *Ri = a->Bim[2], *Ei = a->Bim[3], *Di = a->Bim[4], *Tmi = a->Bim[5];
  if ((int)th0.size() < p || !(res0 > 0)) return kSlow;
  if (cudaMemsetAsync(a->bstatus, 0, sizeof(int), a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  if (cudaMemsetAsync(a->bst, 0, sizeof(DevState), a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  int rc = cholqr2<C>(a, a->Xre, a->Xim, p, X, Xi, Tm, Tmi, 2);
  if (rc) return rc;
  std::vector<double> norms(p);
  std::vector<cplx> th(th0.begin(), th0.begin() + p);
  double prev = res0;
  const long len = (long)p * n;
  for (int outer = 0; outer < max_outer; ++outer) {
    if ((rc = block_apply<C>(a, X, Xi, p, W, Wi, false))) return rc;
    double mx = res0;
    if (outer == 0) {  // T and R only
      block_gram<C>(a, X, Xi, p, W, Wi, p, a->G);
      ++a->stats.kernel_launches;
      launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, X, Xi, p, a->G, p, p, W, Wi, 1, n, R, Ri, nullptr, nullptr);
    } else {
      const uint32_t passes_now = a->stats.block_matvecs, bf16_now = a->stats.block_bf16;
      if ((rc = check_enqueue<C>(a, a->stream, X, Xi, W, Wi, R, Ri, E, Ei, p, p, p, false, true))) return rc;
      if ((rc = check_collect(a, p, p, th.data(), norms.data()))) return rc;
      a->stats.refine_iterations++;
      double scale = 0;
      for (int q = 0; q < p; ++q) scale = fmax(scale, cabs_(th[q]));
      if (scale == 0) return kSlow;
      mx = 0;
      for (int q = 0; q < p; ++q) {
        res_out[q] = norms[q] / scale;
        mx = fmax(mx, res_out[q]);
      }
      a->trace.push_back({3, outer, passes_now, bf16_now, mx});
      if (mx <= tol) {  // Ritz vectors X S
        ++a->stats.kernel_launches;
        launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, X, Xi, p, a->bY, p, p, nullptr, nullptr, 0, n, a->Xre, a->Xim, nullptr, nullptr);
        a->evals.assign(th.begin(), th.end());
        return launch_check();
      }
      if (!(mx == mx) || mx > 1e-2 * prev) return kSlow;
      prev = mx;
    }
    // inner fixed point on the FP32-class operator, for a truncation error
    // of 3 % of the goal (the correction's FP32-class rounding, about 5e-6 of
    // the starting residual, dominates the result); the observed contraction
    // of non-normal problems is slower than rho, so the count assumes at
    // least 0.3 per sweep: a contraction up to 0.37 still leaves the
    // truncation below a third of the goal, and a shortfall costs one more
    // outer step, not the result
    const double rho_eff = rho > 0.3 ? rho : 0.3;
    int J = (int)ceil(log(0.03 * tol / mx) / log(rho_eff));
    if (J < 2) J = 2;
    if (J > 30) J = 30;
    // leading sweeps on the BF16 planes: the last Jf contract their error
    const int Jf = (int)ceil(log(0.03 * tol / mx / bf16_sweep_error(a, th)) / log(rho_eff));
    const int Jb = J - Jf > 0 ? J - Jf : 0;
    a->stats.kernel_launches += 2;
    launch_dependent(k_small_inv, dim3(1), dim3(32), 0, a->stream, (const cplx*)a->G, p, a->Tinv, a->bstatus);
    // D = R T^-1 (the first sweep from D = 0)
    launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, R, Ri, p, a->Tinv, p, p, nullptr, nullptr, 0, n, D, Di, nullptr, nullptr);
    // Components of D inside span(X) do not move the subspace; between
    // projections they grow at most like |theta_1| / |theta_p| per
    // iteration, so project when that growth would pass 4x, and last.
    double tmax = 0, tmin = 1e300;
    for (int q = 0; q < p; ++q) {
      tmax = fmax(tmax, cabs_(th[q]));
      tmin = fmin(tmin, cabs_(th[q]));
    }
    const double spread = tmin > 0 ? tmax / tmin : 1e300;
    int every = spread > 1.0 + 1e-12 ? (int)floor(log(4.0) / log(spread)) : J;
    if (every < 1) every = 1;
    for (int j = 0; j < J; ++j) {
      // BF16 sweeps before the last one also round D to BF16 (coarse): an
      // error a sweep leaves is damped by every later sweep, so only the last
      // BF16 sweep's, contracted by the Jf that follow, reaches the result
      if ((rc = block_apply<C>(a, D, Di, p, W, Wi, true, j < Jb, j + 1 < Jb))) return rc;
      if ((j + 1) % every == 0 || j + 1 == J) {
        block_gram<C>(a, X, Xi, p, W, Wi, p, a->G2);
        a->stats.kernel_launches++;
        launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, X, Xi, p, a->G2, p, p, W, Wi, 1, n, W, Wi, nullptr, nullptr);
      }
      // D = (P A D + R) T^-1
      a->stats.kernel_launches++;
      launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, W, Wi, p, a->Tinv, p, p, nullptr, nullptr, 0, n, D, Di, R, Ri);
    }
    // X <- orth(X + D): X is orthonormal and D orthogonal to it, so X + D is
    // conditioned like 1 + ||D|| and one CholeskyQR pass is orthonormal to
    // rounding (a diverging D is rejected by the next step's check)
    a->stats.kernel_launches++;
    launch_dependent(k_block_add, dim3(grid_n(len)), dim3(256), 0, a->stream, (const double*)X, (const double*)Xi,
                     (const double*)D, (const double*)Di, p, n, R, Ri);
    if ((rc = cholqr2<C>(a, R, Ri, p, X, Xi, Tm, Tmi, 1))) return rc;
  }
  return kSlow;
}

// FP64 residuals of the k Ritz pairs in a->Xre with values a->evals, one
// block pass per group of kBmMaxB vectors.
template <bool C>
int verify(oapb_arnoldi* a, double scale, double* out) {
  const int n = a->n, kk = a->k;
  std::vector<cplx> diag((size_t)kBmMaxB * kBmMaxB);
  for (int q0 = 0; q0 < kk; q0 += kBmMaxB) {
    const int b = kk - q0 < kBmMaxB ? kk - q0 : kBmMaxB;
    const double* xr = a->Xre + (long)q0 * n;
    const double* xi = C ? a->Xim + (long)q0 * n : nullptr;
    int rc = block_apply<C>(a, xr, xi, b, a->Bre[1], a->Bim[1]);
    if (rc) return rc;
    for (auto& d : diag) d = cplx{0, 0};
    for (int q = 0; q < b; ++q) diag[q + q * b] = a->evals[q0 + q];
    if (cudaMemcpyAsync(a->G, diag.data(), sizeof(cplx) * b * b, cudaMemcpyHostToDevice, a->stream) != cudaSuccess)
      return OAPB_ERR_CUDA;
    ++a->stats.kernel_launches;
    launch_dependent(k_block_update<C>, dim3(grid_up(n)), dim3(256), 0, a->stream, xr, xi, b, a->G, b, b, a->Bre[1], a->Bim[1], 1, n, a->Bre[2], a->Bim[2], nullptr, nullptr);
    std::vector<double> rn(b), xn(b);
    if ((rc = col_norms<C>(a, a->Bre[2], a->Bim[2], b, rn.data()))) return rc;
    if ((rc = col_norms<C>(a, xr, xi, b, xn.data()))) return rc;
    for (int q = 0; q < b; ++q) out[q0 + q] = rn[q] / (scale * (xn[q] > 0 ? xn[q] : 1));
  }
  return OAPB_OK;
}

__global__ void k_init_block(double* xre, double* xim, int b, int n, uint64_t seed) {
  const long len = (long)b * n;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x) {
    xre[e] = uniform_pm1(seed ^ 0xA0761D6478BD642Full, (uint64_t)e);
    if (xim) xim[e] = uniform_pm1(seed ^ 0xE7037ED1A0B428DBull, (uint64_t)e);
  }
}

// f = w - s f (start-vector shift filter)
template <bool CPLX>
__global__ void k_shift_filter(const double* __restrict__ wre, const double* __restrict__ wim, double s, double* fre,
                               double* fim, int n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    fre[i] = wre[i] - s * fre[i];
    if (CPLX) fim[i] = wim[i] - s * fim[i];
  }
}

// Fresh start of the Krylov factorization: f = start vector, H = 0.
template <bool C>
int iram_start(oapb_arnoldi* a, bool user_start = true) {
  cudaStream_t s = a->stream;
  const int n = a->n, m = a->m;
  if (cudaMemsetAsync(a->st, 0, sizeof(DevState), s) != cudaSuccess) return OAPB_ERR_CUDA;
  if (cudaMemsetAsync(a->H, 0, sizeof(cplx) * m * m, s) != cudaSuccess) return OAPB_ERR_CUDA;
  if (a->cfg.init == OAPB_INIT_USER && user_start) {
    if (!a->have_v0) return OAPB_ERR_ARG;
    cudaMemcpyAsync(a->fre, a->v0re, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
    if (C) cudaMemcpyAsync(a->fim, a->v0im, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
    // shift filter: f <- prod_i (A - s_i I) f
    for (double sh : a->start_shifts) {
      int rc = apply_op(a, a->fre, C ? a->fim : nullptr, a->wre, C ? a->wim : nullptr, false, OAPB_TYPE_WV);
      if (rc) return rc;
      a->stats.matvecs++;
      a->stats.kernel_launches++;
      k_shift_filter<C><<<grid_n(n), 256, 0, s>>>(a->wre, a->wim, sh, a->fre, a->fim, n);
    }
  } else {
    a->stats.kernel_launches++;
    const int mode = a->cfg.init == OAPB_INIT_USER ? OAPB_INIT_RANDOM : a->cfg.init;
    k_init_vector<<<grid_n(n), 256, 0, s>>>(a->fre, C ? a->fim : nullptr, n, a->cfg.seed, mode);
  }
  return set_fnorm(a);
}

// Ritz vectors and FP64 verification after the plain restart loop ended
// with status st; V, H, f stay a complete factorization (checkpointable).
template <bool C>
int finish_plain(oapb_arnoldi* a, int st, double* r) {
  if (st != OAPB_OK && st != OAPB_NOT_CONVERGED) return st;
  a->ckpt_ready = true;
  int rc = ritz_vectors<C>(a, a->k);
  if (rc) return rc;
  std::vector<cplx> th(a->m);
  DevState hs;
  if (cudaMemcpyAsync(th.data(), a->ritz, sizeof(cplx) * a->m, cudaMemcpyDeviceToHost, a->stream) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if ((rc = read_state(a, &hs))) return rc;
  a->evals.assign(th.begin(), th.begin() + a->k);
  return verify<C>(a, hs.scale, r);
}

// The plain FP64 GPU Arnoldi: IRAM to the goal, Ritz vectors, FP64
// verification of every wanted pair in one block pass.
template <bool C>
int solve_plain(oapb_arnoldi* a, double* r) {
  a->nvec_hess = a->k;
  int rc = iram_start<C>(a);
  if (rc) return rc;
  int st = iram<C>(a, false, a->cfg.tolerance, a->cfg.max_restarts, 0);
  if (st == OAPB_NOT_CONVERGED && a->cfg.init == OAPB_INIT_USER && a->cfg.fallback_random) {
    // the warm start did not reach the goal: the random-start method decides
    a->stats.fallbacks++;
    if ((rc = iram_start<C>(a, false))) return rc;
    st = iram<C>(a, false, a->cfg.tolerance, a->cfg.max_restarts, 0);
  }
  return finish_plain<C>(a, st, r);
}

// Continue the plain restart loop from the factorization a checkpoint
// restored (oapb_arnoldi_load): Schur form and shifts of the restored H
// first, then restarts as in solve_plain, with a fresh restart budget.
template <bool C>
int resume_plain(oapb_arnoldi* a, double* r) {
  a->nvec_hess = a->k;
  if (cudaMemsetAsync(a->st, 0, sizeof(DevState), a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  int rc = set_fnorm(a);
  if (rc) return rc;
  const int st = iram<C>(a, false, a->cfg.tolerance, a->cfg.max_restarts, a->m);
  return finish_plain<C>(a, st, r);
}

// The mixed form: (1) FP32 block subspace iteration from a seeded random
// block down to the FP32 floor, (2) FP64 block subspace iteration to the
// goal.  When the spectrum makes subspace iteration too slow, (3) FP32 IRAM
// followed by the FP64 refinement of its Ritz vectors, and finally (4) the
// plain FP64 IRAM.
template <bool C>
int solve_mixed(oapb_arnoldi* a, double* r) {
  const int n = a->n, m = a->m, k = a->k;
  const double tol = a->cfg.tolerance;
  // FP32 phase on k + 4 vectors, FP64 phase on the first k + 2 Ritz vectors
  int b = k + 4;
  if (b > kBmMaxB) b = kBmMaxB;
  if (b > n) b = n;
  int b64 = k + 2 < b ? k + 2 : b;
  a->stats.kernel_launches++;
  k_init_block<<<grid_n((long)b * n), 256, 0, a->stream>>>(a->Xre, C ? a->Xim : nullptr, b, n, a->cfg.seed);
  double rate = 0.0, floor1 = 1e-6;
  std::vector<double> r1(k);
  std::vector<cplx> th32;
  int st = subspace<C>(a, b, true, tol > kFp32Goal ? tol : kFp32Goal, 60, r1.data(), false, b64, &rate, 0, &floor1,
                       &th32);
  if (st == OAPB_OK && C && a->cfg.sort == 0 && a->cfg.refine && (int)th32.size() > k && cabs_(th32[k - 1]) > 0) {
    // largest-magnitude wanted set: the correction contracts by |theta_{k+1}| / |theta_k|
    const double rho = cabs_(th32[k]) / cabs_(th32[k - 1]);
    if (rho < 0.6) {
      const int rs = refine<C>(a, tol, rho, floor1, th32, r);
      if (rs == OAPB_OK) return OAPB_OK;
      if (rs != kSlow) return rs;
      a->stats.fallbacks++;
    }
  }
  if (st == OAPB_OK) {
    // the FP32 phase measured the contraction per iteration: the FP64 phase
    // cannot meet the goal before about log(tol / floor) / log(rate) passes
    int skip = 0;
    if (rate > 0 && rate < 0.9 && floor1 > tol) skip = (int)(log(tol / floor1) / log(rate)) - 1;
    if (skip < 0) skip = 0;
    if (skip > 12) skip = 12;
    st = subspace<C>(a, b64, false, tol, 30, r, false, 0, nullptr, skip);
    if (st == OAPB_OK) return OAPB_OK;
  }
  if (st != OAPB_OK && st != kSlow && st != OAPB_NOT_CONVERGED) return st;
  // (3) Krylov phase on the FP32 operator
  int bi = k + (m - k < 4 ? m - k : 4);
  if (bi > kBmMaxB) bi = kBmMaxB;
  a->nvec_hess = bi;
  int rc = ensure_fp32_copy(a);
  if (rc) return rc;
  if ((rc = iram_start<C>(a))) return rc;
  st = iram<C>(a, true, tol > 1e-7 ? tol : 1e-7, a->cfg.max_restarts, 0);
  if (st != OAPB_OK && st != OAPB_NOT_CONVERGED) return st;
  if ((rc = ritz_vectors<C>(a, bi))) return rc;
  st = subspace<C>(a, bi, false, tol, 40, r, false);
  if (st == OAPB_OK) return OAPB_OK;
  if (st != kSlow && st != OAPB_NOT_CONVERGED) return st;
  // (4)
  return solve_plain<C>(a, r);
}

// The chosen form below kMixedMinN: the FP64 restart loop on one CTA
// (oapb_arnoldi_solve_batched with one problem).  Ritz vectors land in
// a->Xre (vector-major) like the multi-kernel path's, so the outputs,
// test_outcome and the host-buffer solve read them the same way.
template <bool C>
int solve_onchip(oapb_arnoldi* a, double* r) {
  const int n = a->n, k = a->k;
  oapb_arnoldi_config cfg = a->cfg;
  cfg.hdim = (uint32_t)a->m;
  oapb_batch_problem p;
  p.n = (uint32_t)n;
  p.re = a->a64re;
  p.im = C ? a->a64im : nullptr;
  p.eigvec_re = a->Bre[3];  // row-major n x k scratch (a block buffer holds n x 32)
  p.eigvec_im = C ? a->Bim[3] : nullptr;
  std::vector<double> er(k), ei(k), rs(k);
  int32_t st = 0;
  oapb_batch_stats bs;
  const int rc = oapb_arnoldi_solve_batched(&cfg, &p, 1, er.data(), ei.data(), rs.data(), &st, &bs, (void*)a->stream);
  if (rc != OAPB_OK && rc != OAPB_NOT_CONVERGED) return rc;
  if (st != OAPB_OK && st != OAPB_NOT_CONVERGED) return st;
  a->stats.kernel_launches += 2;
  k_rowmajor_to_vectors<<<grid_for((long)n * k, 256, kNumSMs * 8), 256, 0, a->stream>>>(
      a->Bre[3], C ? a->Bim[3] : nullptr, n, k, a->Xre, C ? a->Xim : nullptr);
  if (cudaGetLastError() != cudaSuccess) return OAPB_ERR_CUDA;
  a->evals.resize(k);
  for (int q = 0; q < k; ++q) {
    a->evals[q] = cplx{er[q], C ? ei[q] : 0.0};
    r[q] = rs[q];
  }
  a->stats.matvecs = (uint32_t)bs.matvecs;
  a->stats.restarts = (uint32_t)bs.restarts;
  a->stats.onchip = 1;
  return st;
}

template <bool C>
int solve_impl(oapb_arnoldi* a, double* eig_re, double* eig_im, double* res, bool resume = false) {
  const int k = a->k;
  // The mixed form needs the dense operator and the block kernels (k <= 32),
  // and pays off only when the operator pass is HBM-bound: below n = 8192
  // (at most 1 GiB of complex FP64 operator) a pass is a few tens of
  // microseconds and the single-vector FP64 restart loop is faster.
  const bool mixed = a->cfg.precision == OAPB_PREC_MIXED && !a->cb && !a->gX && !a->gS && k <= kBmMaxB && a->mixed_ready &&
                     a->n >= kMixedMinN;
  if (!resume) a->stats.restarts = 0;  // a resumed solve continues the saved count
  a->stats.matvecs = 0;
  a->stats.block_matvecs = 0;
  a->stats.block_bf16 = 0;
  a->stats.block_i8 = 0;
  a->stats.eig_fast = 0;
  a->stats.refine_iterations = 0;
  a->trace.clear();
  a->stats.dgks_passes = 0;
  a->stats.fallbacks = 0;
  int rc = alloc_blocks(a);
  if (rc) return rc;
  std::vector<double> r(k);
  a->ckpt_ready = false;
  a->stats.onchip = 0;
  const bool onchip = !resume && !mixed && a->cfg.precision == OAPB_PREC_MIXED && !a->cb && !a->gX && !a->gS &&
                      a->a64re && a->n <= kOnchipMaxN && a->m <= kOnchipMaxM && a->cfg.init == OAPB_INIT_RANDOM &&
                      a->start_shifts.empty();
  int st = resume ? resume_plain<C>(a, r.data())
           : mixed ? solve_mixed<C>(a, r.data())
           : onchip ? solve_onchip<C>(a, r.data())
                    : solve_plain<C>(a, r.data());
  if (st != OAPB_OK && st != OAPB_NOT_CONVERGED) return st;
  double mx = 0;
  bool finite = true;
  for (int q = 0; q < k; ++q) {
    if (eig_re) eig_re[q] = a->evals[q].re;
    if (eig_im) eig_im[q] = a->evals[q].im;
    if (res) res[q] = r[q];
    // a NaN residual (or eigenvalue) never counts as converged
    if (!std::isfinite(r[q]) || !std::isfinite(a->evals[q].re) || !std::isfinite(a->evals[q].im)) finite = false;
    mx = r[q] > mx ? r[q] : mx;
  }
  a->stats.max_residual = finite ? mx : NAN;
  a->stats.converged = finite && mx <= a->cfg.tolerance;
  if (!finite) return OAPB_ERR_NONFINITE;
  return a->stats.converged ? OAPB_OK : OAPB_NOT_CONVERGED;
}

// drop the host-X Gram operator (its copies finish first)
void drop_gram_stream(oapb_arnoldi* a) {
  if (a->gS) {
    cudaStreamSynchronize(a->stream);
    gram_stream_destroy(a->gS);
    a->gS = nullptr;
  }
}

void free_all(oapb_arnoldi* a) {
  drop_gram_stream(a);
  void* ps[] = {a->own64re, a->own64im, a->hvre, a->hvim, a->a32re, a->a32im, a->Vre, a->Vim, a->Xre, a->Xim, a->fre,
                a->fim, a->wre, a->wim, a->x32re, a->x32im, a->v0re, a->v0im, a->H, a->Qs, a->ritz,
                a->Y, a->h, a->s, a->part, a->hws, a->est, a->fpart, a->order, a->st};
  for (void* p : ps)
    if (p) cudaFree(p);
  void* bs[] = {a->abf, a->xbf, a->tcerr, a->Wp, a->wdm, a->bpart, a->bdone, a->gws, a->G, a->G2, a->Rinv, a->bY, a->bQ, a->bH, a->britz, a->best, a->bnorm, a->border,
                a->bstatus, a->bst, a->bpart2, a->bdone2, a->Tinv, a->ntflag,
                a->bf16err2, a->ai8, a->ai8s, a->xi8, a->xi8s};
  for (void* p : bs)
    if (p) cudaFree(p);
  for (int i = 0; i < oapb_arnoldi::kBlocks; ++i) {
    if (a->Bre[i]) cudaFree(a->Bre[i]);
    if (a->Bim[i]) cudaFree(a->Bim[i]);
  }
  if (a->hpin) cudaFreeHost(a->hpin);
  if (a->ev_w) cudaEventDestroy(a->ev_w);
  if (a->ev_chk) cudaEventDestroy(a->ev_chk);
  if (a->s2) cudaStreamDestroy(a->s2);
}

}  // namespace

// Launch autotuner of the single-vector operator pass (replaces the
// reference's fixed launch mapping, utils::mapper::SetThreadsBlocks,
// oapUtils/ThreadsMapper.cpp:36-74): every k_matvec variant (rows per CTA,
// persistent or one CTA per row tile) runs once to warm up and three times
// timed with CUDA events on the handle's stream; the fastest is kept per
// (device, n, element type, complex) for the life of the process.
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune;

template <typename T>
int tune_matvec(oapb_arnoldi* a, const T* Are, const T* Aim, const T* xre, const T* xim) {
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, a->n, (int)sizeof(T), a->is_c ? 1 : 0);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return 0;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return 0;
  }
  int best = 0;
  float best_ms = 1e30f;
  for (int v = 0; v < kMvVariants; ++v) {
    if (launch_matvec<T>(Are, Aim, a->n, a->n, xre, xim, a->wre, a->is_c ? a->wim : nullptr, a->stream, v) !=
        cudaSuccess)
      continue;
    cudaEventRecord(e0, a->stream);
    for (int r = 0; r < 3; ++r)
      launch_matvec<T>(Are, Aim, a->n, a->n, xre, xim, a->wre, a->is_c ? a->wim : nullptr, a->stream, v);
    cudaEventRecord(e1, a->stream);
    float ms = 0;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) continue;
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  return best;
}
}  // namespace

extern "C" {

void oapb_arnoldi_config_default(oapb_arnoldi_config* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->sort = OAPB_SORT_LARGEST_VALUES;
  c->precision = OAPB_PREC_FP64;
  c->init = OAPB_INIT_RANDOM;
  c->max_restarts = 300;
  c->tolerance = 1e-10;
  c->rho = 1.0 / 3.14;
  c->seed = 1;
  c->tensor_cores = 1;
  c->refine = 1;
  c->autotune = 1;
}

int oapb_arnoldi_create(oapb_arnoldi** out, const oapb_arnoldi_config* cfg, void* stream) {
  if (!out || !cfg) return OAPB_ERR_ARG;
  *out = nullptr;
  const int n = (int)cfg->n, m = (int)cfg->hdim, k = (int)cfg->wanted;
  if (n < 2 || m < 2 || k < 1 || k >= m || m > n || m > kMaxM || cfg->sort < 0 || cfg->sort > 5) return OAPB_ERR_ARG;
  if (!(cfg->tolerance > 0)) return OAPB_ERR_ARG;
  oapb_arnoldi* a = new (std::nothrow) oapb_arnoldi();
  if (!a) return OAPB_ERR_NOMEM;
  a->cfg = *cfg;
  a->n = n;
  a->m = m;
  a->k = k;
  a->is_c = cfg->is_complex != 0;
  // NULL selects the legacy default stream, like every other call
  a->stream = (cudaStream_t)stream;
  const size_t vb = sizeof(double) * (size_t)n;
  a->chunk = 128;
  a->nchunk = (n + a->chunk - 1) / a->chunk;
  if (a->nchunk > 2 * kNumSMs) {
    a->nchunk = 2 * kNumSMs;
    a->chunk = (n + a->nchunk - 1) / a->nchunk;
  }
  a->nupd = grid_for(n, kUpdThreads, kNumSMs * 4);
  int rc = OAPB_OK;
  const bool C = a->is_c;
  rc |= dalloc(&a->Vre, vb * (m + 1));
  if (C) rc |= dalloc(&a->Vim, vb * (m + 1));
  const int nx = (m + 1) > kBmMaxB ? (m + 1) : kBmMaxB;  // Ritz / start blocks
  rc |= dalloc(&a->Xre, vb * nx);
  if (C) rc |= dalloc(&a->Xim, vb * nx);
  rc |= dalloc(&a->fre, vb);
  rc |= dalloc(&a->wre, vb);
  if (C) rc |= dalloc(&a->fim, vb);
  if (C) rc |= dalloc(&a->wim, vb);
  rc |= dalloc(&a->H, sizeof(cplx) * m * m);
  rc |= dalloc(&a->Qs, sizeof(cplx) * m * m);
  rc |= dalloc(&a->ritz, sizeof(cplx) * m);
  rc |= dalloc(&a->Y, sizeof(cplx) * m * m);
  rc |= dalloc(&a->h, sizeof(cplx) * (m + 1));
  rc |= dalloc(&a->s, sizeof(cplx) * (m + 1));
  rc |= dalloc(&a->part, sizeof(cplx) * (size_t)a->nchunk * (m + 1));
  rc |= dalloc(&a->est, sizeof(double) * m);
  rc |= dalloc(&a->fpart, sizeof(double) * (a->nupd > 1024 ? a->nupd : 1024));
  rc |= dalloc(&a->order, sizeof(int) * m);
  rc |= dalloc(&a->st, sizeof(DevState));
  const size_t hb = sizeof(cplx) * hess_ws_cplx(m);
  const size_t hb_block = sizeof(cplx) * hess_ws_cplx(kBmMaxB);  // small_eig of the block methods
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t static_smem =
      kMaxM * (sizeof(cplx) + sizeof(double) + sizeof(int)) + sizeof(HessShared<cplx, kHessWarps>) + 1024;
  if (hb + static_smem <= (size_t)optin) {
    a->hess_smem = hb;
  } else {
    rc |= dalloc(&a->hws, hb);
  }
  {
    const size_t attr = std::max(a->hess_smem, hb_block);
    if (attr > 48 * 1024 &&
        cudaFuncSetAttribute(k_hess, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)attr) != cudaSuccess)
      rc |= OAPB_ERR_CUDA;
  }
  const size_t vqb = sizeof(cplx) * (size_t)m * m;
  if (vqb > 48 * 1024) {
    cudaFuncSetAttribute(k_vq<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vqb);
    cudaFuncSetAttribute(k_vq<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vqb);
  }
  if (rc != OAPB_OK) {
    free_all(a);
    if (a->own_stream) cudaStreamDestroy(a->stream);
    delete a;
    return (rc & OAPB_ERR_NOMEM) ? OAPB_ERR_NOMEM : OAPB_ERR_CUDA;
  }
  *out = a;
  return OAPB_OK;
}

int oapb_arnoldi_destroy(oapb_arnoldi* a) {
  if (!a) return OAPB_ERR_ARG;
  cudaStreamSynchronize(a->stream);
  if (a->s2) cudaStreamSynchronize(a->s2);
  for (cudaEvent_t e : a->ev_pool) cudaEventDestroy(e);
  free_all(a);
  if (a->own_stream) cudaStreamDestroy(a->stream);
  delete a;
  return OAPB_OK;
}

}  // extern "C"

// BF16 hi / lo planes of the tensor-core passes: buffers (first call), then
// the split of rows row0 .. row0 + rows - 1 of both operator planes
static int build_tc_planes(oapb_arnoldi* a, long row0, long rows) {
  a->kp = (a->n + 127) / 128 * 128;
  const size_t plane = (size_t)a->n * a->kp;
  const int np = a->is_c ? 4 : 2;
  if (!a->abf && dalloc(&a->abf, sizeof(__nv_bfloat16) * plane * np)) return OAPB_ERR_NOMEM;
  if (!a->xbf && dalloc(&a->xbf, sizeof(__nv_bfloat16) * 2 * 64 * (size_t)a->kp)) return OAPB_ERR_NOMEM;
  if (!a->tcerr) {
    if (dalloc(&a->tcerr, sizeof(int))) return OAPB_ERR_NOMEM;
    if (cudaMemsetAsync(a->tcerr, 0, sizeof(int), a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  }
  if (!a->bf16err2 && dalloc(&a->bf16err2, sizeof(double))) return OAPB_ERR_NOMEM;
  if (row0 == 0) {  // a new operator: its BF16 rounding energy from zero
    if (cudaMemsetAsync(a->bf16err2, 0, sizeof(double), a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
    a->bf16_err = -1;
  }
  a->stats.kernel_launches += np / 2;
  // int8 slices of the FP64-class pass (optional: without the memory the
  // FP64 pass stays on the FP64 tensor cores)
  if (row0 == 0) {
    a->have_i8 = false;
    if (!a->ai8 && (dalloc(&a->ai8, i8_operator_bytes(a->n, a->kp, a->is_c)) ||
                    dalloc(&a->ai8s, sizeof(double) * a->n) || dalloc(&a->xi8, i8_block_bytes(a->kp)) ||
                    dalloc(&a->xi8s, sizeof(double) * kI8ScaleDoubles))) {
      for (void** p : {(void**)&a->ai8, (void**)&a->ai8s, (void**)&a->xi8, (void**)&a->xi8s})
        if (*p) {
          cudaFree(*p);
          *p = nullptr;
        }
      cudaGetLastError();
    }
  }
  if (a->ai8) {
    ++a->stats.kernel_launches;
    if (split_operator_i8(a->a64re, a->is_c ? a->a64im : nullptr, a->n, a->kp, a->ai8, a->ai8s, a->stream, row0,
                          rows))
      return OAPB_ERR_CUDA;
    a->have_i8 = true;
  }
  if (split_operator_bf16(a->a64re, a->n, a->kp, a->abf, a->abf + plane, a->stream, row0, rows, a->bf16err2))
    return OAPB_ERR_CUDA;
  if (a->is_c && split_operator_bf16(a->a64im, a->n, a->kp, a->abf + 2 * plane, a->abf + 3 * plane, a->stream, row0,
                                     rows, a->bf16err2))
    return OAPB_ERR_CUDA;
  a->have_tc = true;
  return OAPB_OK;
}

// FP32 copy of the operator for the CUDA-core passes (tensor_cores = 0) and
// the FP32 restart loop, built when first needed (it is not on the
// tensor-core path), with the launch variant of its single-vector pass
static int ensure_fp32_copy(oapb_arnoldi* a) {
  if (a->fp32_ready) return OAPB_OK;
  const long nn = (long)a->n * a->n;
  if (!a->a32re && dalloc(&a->a32re, sizeof(float) * nn)) return OAPB_ERR_NOMEM;
  if (a->is_c && !a->a32im && dalloc(&a->a32im, sizeof(float) * nn)) return OAPB_ERR_NOMEM;
  if (!a->x32re && dalloc(&a->x32re, sizeof(float) * a->n)) return OAPB_ERR_NOMEM;
  if (a->is_c && !a->x32im && dalloc(&a->x32im, sizeof(float) * a->n)) return OAPB_ERR_NOMEM;
  const int g = kNumSMs * 8;
  ++a->stats.kernel_launches;
  k_to_f32<float><<<g, 256, 0, a->stream>>>(a->a64re, a->a32re, nn);
  if (a->is_c) {
    ++a->stats.kernel_launches;
    k_to_f32<float><<<g, 256, 0, a->stream>>>(a->a64im, a->a32im, nn);
  }
  if (launch_check()) return OAPB_ERR_CUDA;
  if (a->cfg.autotune == 1) {
    if (cudaMemsetAsync(a->x32re, 0, sizeof(float) * a->n, a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
    if (a->is_c && cudaMemsetAsync(a->x32im, 0, sizeof(float) * a->n, a->stream) != cudaSuccess)
      return OAPB_ERR_CUDA;
    a->mv32 = tune_matvec<float>(a, a->a32re, a->a32im, a->x32re, a->is_c ? a->x32im : nullptr);
  }
  a->fp32_ready = true;
  return OAPB_OK;
}

// the mixed form's operator data for the operator now set
static int make_mixed(oapb_arnoldi* a) {
  const int rc = a->cfg.tensor_cores ? build_tc_planes(a, 0, a->n) : ensure_fp32_copy(a);
  if (rc) return rc;
  a->mixed_ready = true;
  return OAPB_OK;
}

// launch variants of the FP64 single-vector pass (forced or autotuned)
static int tune_operator(oapb_arnoldi* a) {
  if (a->cfg.autotune >= 2 && a->cfg.autotune < 2 + kMvVariants) {  // a forced variant
    a->mv64 = a->mv32 = a->cfg.autotune - 2;
  } else if (a->cfg.autotune == 1) {
    // x: the residual buffers (zeroed), y: the work vector
    if (cudaMemsetAsync(a->fre, 0, sizeof(double) * a->n, a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
    if (a->is_c && cudaMemsetAsync(a->fim, 0, sizeof(double) * a->n, a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
    a->mv64 = tune_matvec<double>(a, a->a64re, a->a64im, a->fre, a->is_c ? a->fim : nullptr);
  }
  a->stats.matvec_variant = (uint32_t)a->mv64;
  return OAPB_OK;
}

extern "C" {

int oapb_arnoldi_set_dense_operator(oapb_arnoldi* a, const oapb_mat* A) {
  if (!a || !A || A->dtype != OAPB_F64 || !A->re) return OAPB_ERR_ARG;
  if (A->columns != (uint32_t)a->n || A->rows != (uint32_t)a->n) return OAPB_ERR_ARG;
  if ((A->im != nullptr) != a->is_c) return OAPB_ERR_ARG;
  a->a64re = (const double*)A->re;
  a->a64im = (const double*)A->im;
  a->cb = nullptr;
  a->gX = nullptr;
  drop_gram_stream(a);
  a->fp32_ready = false;
  a->mixed_ready = false;
  if (a->cfg.precision == OAPB_PREC_MIXED) {
    const int rc = make_mixed(a);
    if (rc) return rc;
  }
  return tune_operator(a);
}

int oapb_arnoldi_set_callback(oapb_arnoldi* a, oapb_matvec_fn fn, void* user) {
  if (!a || !fn) return OAPB_ERR_ARG;
  a->cb = fn;
  a->cb_user = user;
  a->gX = nullptr;
  drop_gram_stream(a);
  return OAPB_OK;
}

int oapb_arnoldi_set_gram_operator(oapb_arnoldi* a, const float* X, uint32_t rows, uint32_t cols) {
  if (!a || !X || a->is_c || rows != (uint32_t)a->n || cols < 1) return OAPB_ERR_ARG;
  if (cols % 4 == 0 && ((uintptr_t)X & 15)) return OAPB_ERR_ARG;
  if (a->gws && a->gcols != (int)cols) {
    cudaFree(a->gws);
    a->gws = nullptr;
  }
  if (!a->gws && dalloc(&a->gws, sizeof(double) * gram_op_workspace(a->n, (int)cols))) return OAPB_ERR_NOMEM;
  a->gX = X;
  a->gcols = (int)cols;
  a->cb = nullptr;
  drop_gram_stream(a);
  return OAPB_OK;
}

int oapb_arnoldi_set_gram_operator_host(oapb_arnoldi* a, const float* X, uint32_t rows, uint32_t cols,
                                        uint32_t block_cols, uint64_t resident_bytes) {
  if (!a || !X || a->is_c || rows != (uint32_t)a->n || cols < 1 || block_cols < 1) return OAPB_ERR_ARG;
  drop_gram_stream(a);
  GramStream* g = nullptr;
  const int rc = gram_stream_create(X, (int)rows, (int)cols, (int)block_cols, resident_bytes, a->stream, &g);
  if (rc) return rc;
  a->gS = g;
  a->gX = nullptr;
  a->cb = nullptr;
  return OAPB_OK;
}

int oapb_arnoldi_gram_stream_info(const oapb_arnoldi* a, uint32_t* blocks, uint32_t* resident_blocks,
                                  uint64_t* streamed_bytes) {
  if (!a || !a->gS) return OAPB_ERR_ARG;
  if (blocks) *blocks = (uint32_t)gram_stream_blocks(a->gS);
  if (resident_blocks) *resident_blocks = (uint32_t)gram_stream_resident_blocks(a->gS);
  if (streamed_bytes) *streamed_bytes = gram_stream_bytes(a->gS);
  return OAPB_OK;
}

int oapb_arnoldi_set_start_vector(oapb_arnoldi* a, const double* re, const double* im) {
  if (!a || !re || (a->is_c && !im)) return OAPB_ERR_ARG;
  const size_t vb = sizeof(double) * a->n;
  if (!a->v0re && dalloc(&a->v0re, vb)) return OAPB_ERR_NOMEM;
  if (a->is_c && !a->v0im && dalloc(&a->v0im, vb)) return OAPB_ERR_NOMEM;
  if (cudaMemcpyAsync(a->v0re, re, vb, cudaMemcpyDefault, a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  if (a->is_c && cudaMemcpyAsync(a->v0im, im, vb, cudaMemcpyDefault, a->stream) != cudaSuccess)
    return OAPB_ERR_CUDA;
  a->have_v0 = true;
  return OAPB_OK;
}

int oapb_arnoldi_set_start_shifts(oapb_arnoldi* a, const double* shifts, uint32_t count) {
  if (!a || count > 64 || (count && !shifts)) return OAPB_ERR_ARG;
  a->start_shifts.assign(shifts, shifts + count);
  return OAPB_OK;
}

static int solve_entry(oapb_arnoldi* a, double* eig_re, double* eig_im, double* residuals, const oapb_mat* evecs,
                       bool resume);

int oapb_arnoldi_solve(oapb_arnoldi* a, double* eig_re, double* eig_im, double* residuals,
                       const oapb_mat* evecs) {
  return solve_entry(a, eig_re, eig_im, residuals, evecs, false);
}

int oapb_arnoldi_resume(oapb_arnoldi* a, double* eig_re, double* eig_im, double* residuals,
                        const oapb_mat* evecs) {
  if (!a || !a->ckpt_ready) return OAPB_ERR_ARG;
  return solve_entry(a, eig_re, eig_im, residuals, evecs, true);
}

// ------------------------------------------------------------ checkpoint --
// File: one buffer in the reference's matrix format (matio.cuh) holding four
// matrices: a header (1 column x 8 rows: format 1, n, m, k, complex,
// restarts, matvecs, sort), V (m columns x n rows, the reference's basis
// layout: column j = Krylov vector j), H (m x m, row-major (c, r) = H[r][c])
// and f (1 column x n rows).
int oapb_arnoldi_save(oapb_arnoldi* a, const char* path) {
  if (!a || !path || !a->ckpt_ready) return OAPB_ERR_ARG;
  const int n = a->n, m = a->m;
  cudaStream_t s = a->stream;
  std::vector<double> vre((size_t)n * m), vim(a->is_c ? (size_t)n * m : 0), fre(n), fim(a->is_c ? n : 0);
  std::vector<cplx> H((size_t)m * m);
  bool ok = cudaMemcpyAsync(vre.data(), a->Vre, sizeof(double) * n * m, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
            cudaMemcpyAsync(fre.data(), a->fre, sizeof(double) * n, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
            cudaMemcpyAsync(H.data(), a->H, sizeof(cplx) * m * m, cudaMemcpyDeviceToHost, s) == cudaSuccess;
  if (a->is_c)
    ok = ok && cudaMemcpyAsync(vim.data(), a->Vim, sizeof(double) * n * m, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(fim.data(), a->fim, sizeof(double) * n, cudaMemcpyDeviceToHost, s) == cudaSuccess;
  if (!ok || cudaStreamSynchronize(s) != cudaSuccess) return OAPB_ERR_CUDA;
  std::vector<char> payload;
  HostMat hd;
  hd.columns = 1;
  hd.rows = 8;
  hd.re = {1.0, (double)n, (double)m, (double)a->k, a->is_c ? 1.0 : 0.0, (double)a->stats.restarts,
           (double)a->stats.matvecs, (double)a->cfg.sort};
  matio_append(payload, hd);
  HostMat V;
  V.columns = m;
  V.rows = n;
  V.has_im = a->is_c;
  V.re.resize((size_t)n * m);
  if (a->is_c) V.im.resize((size_t)n * m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < n; ++i) {
      V.re[(size_t)j + (size_t)i * m] = vre[(size_t)j * n + i];
      if (a->is_c) V.im[(size_t)j + (size_t)i * m] = vim[(size_t)j * n + i];
    }
  matio_append(payload, V);
  HostMat Hm;
  Hm.columns = Hm.rows = m;
  Hm.has_im = true;
  Hm.re.resize((size_t)m * m);
  Hm.im.resize((size_t)m * m);
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < m; ++r) {
      Hm.re[(size_t)c + (size_t)r * m] = H[(size_t)r + (size_t)c * m].re;
      Hm.im[(size_t)c + (size_t)r * m] = H[(size_t)r + (size_t)c * m].im;
    }
  matio_append(payload, Hm);
  HostMat F;
  F.columns = 1;
  F.rows = n;
  F.has_im = a->is_c;
  F.re = fre;
  F.im = fim;
  matio_append(payload, F);
  return matio_write_file(path, payload);
}

int oapb_arnoldi_load(oapb_arnoldi* a, const char* path) {
  if (!a || !path) return OAPB_ERR_ARG;
  std::vector<char> payload;
  int rc = matio_read_file(path, &payload);
  if (rc) return rc;
  size_t off = 0;
  HostMat hd, V, Hm, F;
  if (!matio_parse(payload, off, &hd) || !matio_parse(payload, off, &V) || !matio_parse(payload, off, &Hm) ||
      !matio_parse(payload, off, &F))
    return OAPB_ERR_ARG;
  const int n = a->n, m = a->m;
  if (hd.re.size() != 8 || hd.re[0] != 1.0 || hd.re[1] != n || hd.re[2] != m || hd.re[3] != a->k ||
      (hd.re[4] != 0.0) != a->is_c)
    return OAPB_ERR_ARG;
  if (V.columns != (uint32_t)m || V.rows != (uint32_t)n || Hm.columns != (uint32_t)m || Hm.rows != (uint32_t)m ||
      F.columns != 1 || F.rows != (uint32_t)n || !V.has_re || !Hm.has_re || !F.has_re ||
      (a->is_c && (!V.has_im || !F.has_im)))
    return OAPB_ERR_ARG;
  std::vector<double> vre((size_t)n * m), vim(a->is_c ? (size_t)n * m : 0);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < n; ++i) {
      vre[(size_t)j * n + i] = V.re[(size_t)j + (size_t)i * m];
      if (a->is_c) vim[(size_t)j * n + i] = V.im[(size_t)j + (size_t)i * m];
    }
  std::vector<cplx> H((size_t)m * m);
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < m; ++r)
      H[(size_t)r + (size_t)c * m] =
          cplx{Hm.re[(size_t)c + (size_t)r * m], Hm.has_im ? Hm.im[(size_t)c + (size_t)r * m] : 0.0};
  cudaStream_t s = a->stream;
  bool ok = cudaMemcpyAsync(a->Vre, vre.data(), sizeof(double) * n * m, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(a->fre, F.re.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(a->H, H.data(), sizeof(cplx) * m * m, cudaMemcpyHostToDevice, s) == cudaSuccess;
  if (a->is_c)
    ok = ok && cudaMemcpyAsync(a->Vim, vim.data(), sizeof(double) * n * m, cudaMemcpyHostToDevice, s) == cudaSuccess &&
         cudaMemcpyAsync(a->fim, F.im.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s) == cudaSuccess;
  if (!ok || cudaStreamSynchronize(s) != cudaSuccess) return OAPB_ERR_CUDA;
  a->stats.restarts = (uint32_t)hd.re[5];
  a->ckpt_ready = true;
  return OAPB_OK;
}

static int solve_entry(oapb_arnoldi* a, double* eig_re, double* eig_im, double* residuals, const oapb_mat* evecs,
                       bool resume) {
  if (!a) return OAPB_ERR_ARG;
  if (!a->cb && !a->gX && !a->gS && !a->a64re) return OAPB_ERR_ARG;
  if (evecs && (evecs->columns != (uint32_t)a->k || evecs->rows != (uint32_t)a->n || evecs->dtype != OAPB_F64 ||
                !evecs->re))
    return OAPB_ERR_ARG;
  auto t0 = std::chrono::steady_clock::now();
  a->ev_used = 0;
  a->stats.matvec_fp32 = 0;
  int st = a->is_c ? solve_impl<true>(a, eig_re, eig_im, residuals, resume)
                   : solve_impl<false>(a, eig_re, eig_im, residuals, resume);
  if ((st == OAPB_OK || st == OAPB_NOT_CONVERGED) && evecs) {
    const long nk = (long)a->n * a->k;
    ++a->stats.kernel_launches;
    k_vectors_to_rowmajor<<<grid_for(nk, 256, kNumSMs * 8), 256, 0, a->stream>>>(
        a->Xre, a->is_c ? a->Xim : nullptr, a->n, a->k, (double*)evecs->re, (double*)evecs->im);
    if (launch_check()) return OAPB_ERR_CUDA;
    if (cudaStreamSynchronize(a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  }
  a->stats.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  a->stats.matvec_seconds = 0;
  a->stats.matvec_timed = 0;
  a->stats.block_seconds = 0;
  a->stats.block_timed = 0;
  a->stats.block_fp32_seconds = 0;
  a->stats.block_fp32_timed = 0;
  a->stats.block_bf16_seconds = 0;
  a->stats.block_bf16_timed = 0;
  for (int p = 0; p < 3; ++p) {
    a->stats.pass_kernel_seconds[p] = 0;
    a->stats.pass_kernel_timed[p] = 0;
  }
  if (a->ev_used) {
    cudaStreamSynchronize(a->stream);
    for (size_t i = 0; i + 1 < a->ev_used; i += 2) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, a->ev_pool[i], a->ev_pool[i + 1]) != cudaSuccess) continue;
      const int kind = a->ev_kind[i / 2];
      if (kind >= 6) {
        a->stats.pass_kernel_seconds[kind - 6] += ms * 1e-3;
        a->stats.pass_kernel_timed[kind - 6]++;
      } else if (kind == 0 || kind == 2) {
        a->stats.matvec_seconds += ms * 1e-3;
        a->stats.matvec_timed++;
      } else if (kind == 1) {
        a->stats.block_seconds += ms * 1e-3;
        a->stats.block_timed++;
      } else if (kind == 5) {
        a->stats.block_bf16_seconds += ms * 1e-3;
        a->stats.block_bf16_timed++;
      } else {
        a->stats.block_fp32_seconds += ms * 1e-3;
        a->stats.block_fp32_timed++;
        a->stats.block_fp32_width = a->ev_b[i / 2];
      }
    }
  }
  a->ev_kind.clear();
  a->ev_b.clear();
  return st;
}

int oapb_arnoldi_solve_host(oapb_arnoldi* a, const double* hre, const double* him, double* eig_re, double* eig_im,
                            double* residuals, double* vre, double* vim) {
  if (!a || !hre || (a->is_c && !him)) return OAPB_ERR_ARG;
  const size_t bytes = sizeof(double) * (size_t)a->n * a->n;
  if (!a->own64re && dalloc(&a->own64re, bytes)) return OAPB_ERR_NOMEM;
  if (a->is_c && !a->own64im && dalloc(&a->own64im, bytes)) return OAPB_ERR_NOMEM;
  int rc = OAPB_OK;
  if (a->cfg.precision == OAPB_PREC_MIXED && a->cfg.tensor_cores) {
    // The host -> device copy in row blocks on the second stream; the BF16
    // split of each block runs on the solver stream while the next block
    // crosses the bus.
    if ((rc = ensure_side_stream(a))) return rc;
    a->a64re = a->own64re;
    a->a64im = a->is_c ? a->own64im : nullptr;
    a->cb = nullptr;
    a->gX = nullptr;
    drop_gram_stream(a);
    a->fp32_ready = false;
    a->mixed_ready = false;
    // the previous solve's work on the solver stream precedes the copies
    if (cudaEventRecord(a->ev_w, a->stream) != cudaSuccess || cudaStreamWaitEvent(a->s2, a->ev_w, 0) != cudaSuccess)
      return OAPB_ERR_CUDA;
    constexpr int kChunks = 8;
    const long rows = (a->n + kChunks - 1) / kChunks;
    for (long r0 = 0; r0 < a->n; r0 += rows) {
      const long nr = r0 + rows <= a->n ? rows : a->n - r0;
      const size_t off = (size_t)r0 * a->n, cb = sizeof(double) * (size_t)nr * a->n;
      if (cudaMemcpyAsync(a->own64re + off, hre + off, cb, cudaMemcpyHostToDevice, a->s2) != cudaSuccess)
        return OAPB_ERR_CUDA;
      if (a->is_c && cudaMemcpyAsync(a->own64im + off, him + off, cb, cudaMemcpyHostToDevice, a->s2) != cudaSuccess)
        return OAPB_ERR_CUDA;
      if (cudaEventRecord(a->ev_chk, a->s2) != cudaSuccess || cudaStreamWaitEvent(a->stream, a->ev_chk, 0) != cudaSuccess)
        return OAPB_ERR_CUDA;
      if ((rc = build_tc_planes(a, r0, nr))) return rc;
    }
    a->mixed_ready = true;
    if ((rc = tune_operator(a))) return rc;
  } else {
    if (cudaMemcpyAsync(a->own64re, hre, bytes, cudaMemcpyHostToDevice, a->stream) != cudaSuccess)
      return OAPB_ERR_CUDA;
    if (a->is_c && cudaMemcpyAsync(a->own64im, him, bytes, cudaMemcpyHostToDevice, a->stream) != cudaSuccess)
      return OAPB_ERR_CUDA;
    oapb_mat A = {(uint32_t)a->n, (uint32_t)a->n, a->own64re, a->is_c ? a->own64im : nullptr, OAPB_F64};
    if ((rc = oapb_arnoldi_set_dense_operator(a, &A))) return rc;
  }
  int st = oapb_arnoldi_solve(a, eig_re, eig_im, residuals, nullptr);
  if (st != OAPB_OK && st != OAPB_NOT_CONVERGED) return st;
  if (vre || vim) {
    // staging buffers kept with the handle (a free would synchronise the
    // device on every call)
    const long nk = (long)a->n * a->k;
    if (!a->hvre && dalloc(&a->hvre, sizeof(double) * nk)) return OAPB_ERR_NOMEM;
    if (a->is_c && !a->hvim && dalloc(&a->hvim, sizeof(double) * nk)) return OAPB_ERR_NOMEM;
    ++a->stats.kernel_launches;
    k_vectors_to_rowmajor<<<grid_for(nk, 256, kNumSMs * 8), 256, 0, a->stream>>>(
        a->Xre, a->is_c ? a->Xim : nullptr, a->n, a->k, a->hvre, a->is_c ? a->hvim : nullptr);
    if (vre && cudaMemcpyAsync(vre, a->hvre, sizeof(double) * nk, cudaMemcpyDeviceToHost, a->stream) != cudaSuccess)
      return OAPB_ERR_CUDA;
    if (vim && a->is_c &&
        cudaMemcpyAsync(vim, a->hvim, sizeof(double) * nk, cudaMemcpyDeviceToHost, a->stream) != cudaSuccess)
      return OAPB_ERR_CUDA;
    if (cudaStreamSynchronize(a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  }
  return st;
}

int oapb_arnoldi_apply_block(oapb_arnoldi* a, const double* xre, const double* xim, uint32_t b, double* wre,
                             double* wim, int32_t precision) {
  if (!a || !xre || !wre || b == 0 || b > (uint32_t)kBmMaxB || a->cb || !a->a64re) return OAPB_ERR_ARG;
  if (a->is_c && (!xim || !wim)) return OAPB_ERR_ARG;
  if (precision != OAPB_PREC_FP64 && precision != OAPB_PREC_MIXED && precision != OAPB_PASS_BF16 &&
      precision != OAPB_PASS_BF16_COARSE)
    return OAPB_ERR_ARG;
  const bool fp32 = precision != OAPB_PREC_FP64;
  const bool coarse = precision == OAPB_PASS_BF16_COARSE;
  const bool bf16 = precision == OAPB_PASS_BF16 || coarse;
  if (fp32 && !a->mixed_ready) return OAPB_ERR_ARG;
  int rc = alloc_blocks(a);
  if (rc) return rc;
  rc = a->is_c ? block_apply<true>(a, xre, xim, (int)b, wre, wim, fp32, bf16, coarse)
               : block_apply<false>(a, xre, nullptr, (int)b, wre, nullptr, fp32, bf16, coarse);
  if (rc) return rc;
  int tcerr = 0;
  if (a->tcerr && cudaMemcpyAsync(&tcerr, a->tcerr, sizeof(int), cudaMemcpyDeviceToHost, a->stream) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return OAPB_ERR_CUDA;
  return tcerr ? OAPB_ERR_TIMEOUT : OAPB_OK;
}

int oapb_arnoldi_get_stats(const oapb_arnoldi* a, oapb_arnoldi_stats* out) {
  if (!a || !out) return OAPB_ERR_ARG;
  *out = a->stats;
  return OAPB_OK;
}

int oapb_arnoldi_set_profile(oapb_arnoldi* a, int32_t on) {
  if (!a) return OAPB_ERR_ARG;
  a->cfg.profile = on != 0;
  return OAPB_OK;
}

int oapb_arnoldi_get_trace(const oapb_arnoldi* a, oapb_trace_rec* out, uint32_t cap, uint32_t* count) {
  if (!a || !count || (cap && !out)) return OAPB_ERR_ARG;
  *count = (uint32_t)a->trace.size();
  for (uint32_t i = 0; i < cap && i < *count; ++i) out[i] = a->trace[i];
  return OAPB_OK;
}

int oapb_arnoldi_test_outcome(oapb_arnoldi* a, uint32_t index, double* out) {
  if (!a || !out || index >= (uint32_t)a->k || a->evals.empty()) return OAPB_ERR_ARG;
  std::vector<double> r(a->k);
  double scale = 0;
  for (auto& e : a->evals) scale = fmax(scale, cabs_(e));
  if (scale == 0) scale = 1;
  int rc = a->is_c ? verify<true>(a, scale, r.data()) : verify<false>(a, scale, r.data());
  if (rc) return rc;
  *out = r[index];
  return OAPB_OK;
}

}  // extern "C"
