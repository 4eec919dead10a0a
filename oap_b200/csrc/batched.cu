// Batched implicitly restarted Arnoldi: thousands of independent small
// eigenproblems (n up to 2048, hdim up to 32) in ONE persistent launch.
//
// Reference: IEigenCalculator::calculate (oap2dt3dDevice/IEigenCalculator.cpp:56-70)
// and CuHArnoldi::execute (ArnoldiPackage/ArnoldiProcedures.cpp:129-140)
// solve one problem per call, driven from the host.  Here every CTA
// (256 threads) pulls the next problem from an atomic queue ordered by
// decreasing n (largest first, for load balance over uneven sizes) and runs
// the whole restart loop on the device: Arnoldi steps with CGS + DGKS
// (rho rule), the one-warp Schur / exact-shift restart (hess_core), the
// in-place V <- V Q, Sorensen's residual update, Ritz vectors and the FP64
// residual of every wanted pair.  There are no host round trips between
// restarts, so no per-restart launch or graph replay exists at all.
//
// Shared memory per CTA: the current vector x, w and f (n complex each), H,
// the Schur workspaces T and Z, Q, Y (m x m complex each) and small arrays.
// The Krylov basis V ((hdim + 1) x n complex) lives in a global workspace
// slot owned by the CTA (L2-resident).
#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "hess.cuh"

namespace oapb {

// launch variants (oapb_batch_stats.variant; the autotuner picks one per
// (device, largest n, hdim, wanted, complex)): threads per CTA and the
// resident CTAs per SM the register budget is compiled for (more CTAs per SM
// keep more problems in flight; fewer registers per thread move the
// restart's small arrays to local memory)
constexpr int kBtVariants = 5;
constexpr int kBtThreadsOf[kBtVariants] = {256, 128, 256, 128, 64};
constexpr int kBtMinBlocksOf[kBtVariants] = {1, 2, 2, 4, 8};
constexpr int kBtMaxM = 32;
constexpr int kBtMaxN = 2048;

struct BatchDesc {
  int n;
  int index;  // position in the caller's array (outputs)
  const double* re;
  const double* im;
  double* vre;
  double* vim;
};

struct BatchArgs {
  const BatchDesc* desc;  // sorted by decreasing n
  int count;
  int* counter;
  int mcap, k, which, max_restarts;
  double tol, rho;
  uint64_t seed;
  double* vws;      // per-CTA basis slots: 2 planes x (mcap + 1) x nmax
  int nmax;
  double* ev_re;    // count x k
  double* ev_im;
  double* res;      // count x k
  int* status;      // count
  unsigned long long* matvecs;
  unsigned long long* restarts;
  unsigned long long* op_bytes;  // operator bytes the matvecs read (8 n^2 real, 16 n^2 complex each)
};

struct BatchSmem {
  double *xr, *xi, *wr, *wi, *fr, *fi;
  cplx *H, *T, *Z, *Q, *Y, *ritz, *h, *s, *u;
  double *est, *key, *red;
  int* ord;
  int* order;
  DevState* st;
};

__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline size_t batch_smem_bytes(int nmax, int m) {
  size_t b = 0;
  b += 6 * (size_t)nmax * sizeof(double);  // x, w, f (re / im)
  b += 3 * (size_t)m * m * sizeof(cplx);   // H, Q, Y
  b += (2 * (size_t)m + 2) * sizeof(cplx); // Q tail: rotation list while Q is hess_core scratch
  b += 2 * (size_t)hess_ld(m) * m * sizeof(cplx);  // T, Z
  b += 4 * (size_t)(m + 1) * sizeof(cplx); // ritz, h, s, u
  b += 2 * (size_t)(m + 1) * sizeof(double) + 64 * sizeof(double);
  b += 2 * (size_t)(m + 1) * sizeof(int) + sizeof(DevState) + 16 * 16;
  return b;
}

__device__ BatchSmem carve(char* base, int nmax, int m) {
  BatchSmem S;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    char* p = base + o;
    o += (bytes + 15) & ~(size_t)15;
    return p;
  };
  S.xr = (double*)take(sizeof(double) * nmax);
  S.xi = (double*)take(sizeof(double) * nmax);
  S.wr = (double*)take(sizeof(double) * nmax);
  S.wi = (double*)take(sizeof(double) * nmax);
  S.fr = (double*)take(sizeof(double) * nmax);
  S.fi = (double*)take(sizeof(double) * nmax);
  S.H = (cplx*)take(sizeof(cplx) * m * m);
  S.T = (cplx*)take(sizeof(cplx) * hess_ld(m) * m);
  S.Z = (cplx*)take(sizeof(cplx) * hess_ld(m) * m);
  S.Q = (cplx*)take(sizeof(cplx) * ((size_t)m * m + 2 * m + 2));
  S.Y = (cplx*)take(sizeof(cplx) * m * m);
  S.ritz = (cplx*)take(sizeof(cplx) * (m + 1));
  S.h = (cplx*)take(sizeof(cplx) * (m + 1));
  S.s = (cplx*)take(sizeof(cplx) * (m + 1));
  S.u = (cplx*)take(sizeof(cplx) * (m + 1));
  S.est = (double*)take(sizeof(double) * (m + 1));
  S.key = (double*)take(sizeof(double) * (m + 1));
  S.red = (double*)take(sizeof(double) * 64);
  S.ord = (int*)take(sizeof(int) * (m + 1));
  S.order = (int*)take(sizeof(int) * (m + 1));
  S.st = (DevState*)take(sizeof(DevState));
  return S;
}

// Sum of (a, b) over the CTA of NT threads; every thread gets the result.
template <int NT>
__device__ __forceinline__ cplx cta_sum2(double a, double b, double* red) {
  a = warp_sum(a);
  b = warp_sum(b);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) {
    red[w] = a;
    red[32 + w] = b;
  }
  __syncthreads();
  double ra = 0, rb = 0;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) {
    ra += red[i];
    rb += red[32 + i];
  }
  return cplx{ra, rb};
}

// w = A x  (A row-major n x n; warps over rows, lanes over columns)
// w = A x for one problem (A row-major split planes in global memory, x in
// shared memory): warp w takes kMvRows rows at a time, the lanes stride the
// columns; the loads of all its rows are issued together (the operator
// streams from HBM, so the bytes a CTA keeps in flight set its rate), each
// row summed per lane in column order and then across the warp.
constexpr int kMvRows = 4;
template <bool C, int NT>
__device__ void cta_matvec(const double* __restrict__ Are, const double* __restrict__ Aim, int n, const double* xr,
                           const double* xi, double* wr, double* wi) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int r0 = kMvRows * w; r0 < n; r0 += kMvRows * (NT / 32)) {
    double sr[kMvRows], si[kMvRows];
#pragma unroll
    for (int q = 0; q < kMvRows; ++q) sr[q] = si[q] = 0.0;
    const int nr = (n - r0) < kMvRows ? (n - r0) : kMvRows;
#pragma unroll 4
    for (int c = l; c < n; c += 32) {
      const double x0 = xr[c], x1 = C ? xi[c] : 0.0;
#pragma unroll
      for (int q = 0; q < kMvRows; ++q) {
        if (q < nr) {
          const long idx = (long)(r0 + q) * n + c;
          const double a = __ldcs(Are + idx);
          if (C) {
            const double b = __ldcs(Aim + idx);
            sr[q] += a * x0 - b * x1;
            si[q] += a * x1 + b * x0;
          } else {
            sr[q] += a * x0;
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kMvRows; ++q) {
      const double a = warp_sum(sr[q]);
      const double b = C ? warp_sum(si[q]) : 0.0;
      if (l == 0 && q < nr) {
        wr[r0 + q] = a;
        if (C) wi[r0 + q] = b;
      }
    }
  }
}

// coef[i] = sum_r conj(V_i[r]) src[r], i < nvec (warps over vectors)
template <bool C, int NT>
__device__ void cta_project(const double* Vr, const double* Vi, int n, int nvec, const double* srcr,
                            const double* srci, cplx* coef) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int i = w; i < nvec; i += NT / 32) {
    const double* vr = Vr + (long)i * n;
    const double* vi = C ? Vi + (long)i * n : nullptr;
    double a = 0, b = 0;
    for (int r = l; r < n; r += 32) {
      const double p = vr[r], x = srcr[r];
      if (C) {
        const double q = vi[r], y = srci[r];
        a += p * x + q * y;
        b += p * y - q * x;
      } else {
        a += p * x;
      }
    }
    a = warp_sum(a);
    b = C ? warp_sum(b) : 0.0;
    if (l == 0) coef[i] = cplx{a, b};
  }
}

// dst = src - V coef; returns ||dst||^2 (CTA-wide)
template <bool C, int NT>
__device__ double cta_update(const double* Vr, const double* Vi, int n, int nvec, const cplx* coef,
                             const double* srcr, const double* srci, double* dstr, double* dsti, double* red) {
  double s2 = 0;
  for (int r = threadIdx.x; r < n; r += NT) {
    double a = srcr[r], b = C ? srci[r] : 0.0;
    for (int i = 0; i < nvec; ++i) {
      const double p = Vr[(long)i * n + r];
      if (C) {
        const double q = Vi[(long)i * n + r];
        a -= p * coef[i].re - q * coef[i].im;
        b -= p * coef[i].im + q * coef[i].re;
      } else {
        a -= p * coef[i].re;
      }
    }
    dstr[r] = a;
    if (C) dsti[r] = b;
    s2 += a * a + b * b;
  }
  return cta_sum2<NT>(s2, 0.0, red).re;
}

template <bool C, int NT>
__device__ void solve_one(const BatchArgs& A, const BatchDesc& P, int slot, const BatchSmem& S) {
  const int n = P.n;
  const int m = n < A.mcap ? n : A.mcap;
  const int k = A.k;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* Vr = A.vws + (size_t)slot * 2 * (A.mcap + 1) * A.nmax;
  double* Vi = Vr + (size_t)(A.mcap + 1) * A.nmax;
  const uint64_t pseed = A.seed * 0x9E3779B97F4A7C15ull + (uint64_t)P.index * 0xD1B54A32D192ED03ull;
  unsigned long long matvecs = 0, restarts = 0;
  int status = OAPB_OK;
  if (m <= k || m < 2) status = OAPB_ERR_ARG;

  // start vector
  double s2 = 0;
  for (int r = tid; r < n; r += NT) {
    S.fr[r] = uniform_pm1(pseed, r);
    if (C) S.fi[r] = uniform_pm1(pseed ^ 0x5851F42D4C957F2Dull, r);
    s2 += S.fr[r] * S.fr[r] + (C ? S.fi[r] * S.fi[r] : 0.0);
  }
  double fnorm2 = cta_sum2<NT>(s2, 0, S.red).re, hnorm2 = 0;
  for (int e = tid; e < m * m; e += NT) S.H[e] = cplx{0, 0};
  if (tid == 0) {
    S.st->status = 0;
    S.st->converged = 0;
    S.st->symtri = 0;
  }
  __syncthreads();
  int start = 0;
  for (int rs = 0; status == OAPB_OK; ++rs) {
    for (int j = start; j < m; ++j) {
      // invariant-subspace breakdown: new random direction orthogonal to V
      bool brk = false;
      if (j > 0 && fnorm2 <= 1e-24 * (hnorm2 + fnorm2)) {
        brk = true;
        const uint64_t bs = pseed ^ (0xBF58476D1CE4E5B9ull * (uint64_t)(rs * 64 + j + 1));
        for (int r = tid; r < n; r += NT) {
          S.fr[r] = uniform_pm1(bs, r);
          if (C) S.fi[r] = uniform_pm1(bs ^ 0x5851F42D4C957F2Dull, r);
        }
        __syncthreads();
        for (int sweep = 0; sweep < 2; ++sweep) {
          cta_project<C, NT>(Vr, Vi, n, j, S.fr, S.fi, S.s);
          __syncthreads();
          fnorm2 = cta_update<C, NT>(Vr, Vi, n, j, S.s, S.fr, S.fi, S.fr, S.fi, S.red);
        }
      }
      const double beta = sqrt(fnorm2);
      const double inv = beta > 0 ? 1.0 / beta : 0.0;
      double* vj = Vr + (long)j * n;
      double* vji = Vi + (long)j * n;
      for (int r = tid; r < n; r += NT) {
        const double a = S.fr[r] * inv;
        S.xr[r] = a;
        vj[r] = a;
        if (C) {
          const double b = S.fi[r] * inv;
          S.xi[r] = b;
          vji[r] = b;
        }
      }
      if (tid == 0 && j > 0) S.H[j + (j - 1) * m] = cplx{brk ? 0.0 : beta, 0};
      __syncthreads();
      cta_matvec<C, NT>(P.re, P.im, n, S.xr, S.xi, S.wr, S.wi);
      ++matvecs;
      __syncthreads();
      cta_project<C, NT>(Vr, Vi, n, j + 1, S.wr, S.wi, S.h);
      __syncthreads();
      fnorm2 = cta_update<C, NT>(Vr, Vi, n, j + 1, S.h, S.wr, S.wi, S.fr, S.fi, S.red);
      double h2 = 0;
      for (int i = 0; i <= j; ++i) h2 += abs2(S.h[i]);
      hnorm2 = h2;
      if (sqrt(fnorm2) < A.rho * sqrt(hnorm2)) {  // DGKS (ArnoldiProcedures.cpp:446-456)
        cta_project<C, NT>(Vr, Vi, n, j + 1, S.fr, S.fi, S.s);
        __syncthreads();
        fnorm2 = cta_update<C, NT>(Vr, Vi, n, j + 1, S.s, S.fr, S.fi, S.fr, S.fi, S.red);
        if (tid <= j) S.h[tid] = S.h[tid] + S.s[tid];
        __syncthreads();
      }
      for (int i = tid; i < m; i += NT) {
        cplx v = i <= j ? S.h[i] : cplx{0, 0};
        if (!C) v.im = 0;
        S.H[i + j * m] = v;
      }
      __syncthreads();
    }
    // Schur form, Ritz pairs, estimates and (if not converged) exact shifts
    const int do_shift = rs < A.max_restarts;
    if (tid == 0) S.st->fnorm2 = fnorm2;
    __syncthreads();
    if (warp == 0) {
      HessArgs h;
      h.Hin = S.H;
      h.Hout = S.H;
      h.Qout = S.Q;
      h.ritz = S.ritz;
      h.Y = S.Y;
      h.est = S.est;
      h.order = S.order;
      h.st = S.st;
      h.gws = nullptr;
      h.m = m;
      h.k = k;
      h.nvec = k;
      h.which = A.which;
      h.do_shift = do_shift;
      h.real_shifts = !C;
      h.dense = 0;
      h.use_beta = 1;
      h.tol = A.tol;
      h.beta = 0;
      // Q is written only at the end of hess_core: until then it is the
      // rotation list and eigenvector scratch (2 m + 2 + m k <= m^2 + 2 m + 2)
      hess_core(h, S.T, S.Z, S.u, S.key, S.ord, S.Q, lane);
    }
    __syncthreads();
    if (S.st->status & 2) {
      status = OAPB_ERR_TIMEOUT;
      break;
    }
    if (S.st->converged) break;
    if (!do_shift) {
      status = OAPB_NOT_CONVERGED;
      break;
    }
    // V[0..k] <- V Q[:, 0..k] in place (each thread owns whole rows r)
    for (int r = tid; r < n; r += NT) {
      cplx out[kBtMaxM + 1];
      for (int q = 0; q <= k; ++q) out[q] = cplx{0, 0};
      for (int i = 0; i < m; ++i) {
        const cplx v = {Vr[(long)i * n + r], C ? Vi[(long)i * n + r] : 0.0};
        for (int q = 0; q <= k; ++q) out[q] = out[q] + v * S.Q[i + q * m];
      }
      for (int q = 0; q <= k; ++q) {
        Vr[(long)q * n + r] = out[q].re;
        if (C) Vi[(long)q * n + r] = out[q].im;
      }
      // f = v_k beta_hat + f sigma (Sorensen)
      const cplx f = {S.fr[r], C ? S.fi[r] : 0.0};
      const cplx nf = out[k] * S.st->beta_hat + f * S.st->sigma;
      S.fr[r] = nf.re;
      if (C) S.fi[r] = nf.im;
    }
    double a2 = 0;
    for (int r = tid; r < n; r += NT) a2 += S.fr[r] * S.fr[r] + (C ? S.fi[r] * S.fi[r] : 0.0);
    fnorm2 = cta_sum2<NT>(a2, 0, S.red).re;
    ++restarts;
    start = k;
  }
  // Ritz vectors x_q = V y_q (q < k) in place, then FP64 residuals
  double scale = 0;
  for (int q = 0; q < k; ++q) scale = fmax(scale, cabs_(S.ritz[q]));
  if (scale == 0) scale = 1;
  if (status == OAPB_OK || status == OAPB_NOT_CONVERGED) {
    for (int r = tid; r < n; r += NT) {
      cplx out[kBtMaxM];
      for (int q = 0; q < k; ++q) out[q] = cplx{0, 0};
      for (int i = 0; i < m; ++i) {
        const cplx v = {Vr[(long)i * n + r], C ? Vi[(long)i * n + r] : 0.0};
        for (int q = 0; q < k; ++q) out[q] = out[q] + v * S.Y[i + q * m];
      }
      for (int q = 0; q < k; ++q) {
        Vr[(long)q * n + r] = out[q].re;
        if (C) Vi[(long)q * n + r] = out[q].im;
      }
    }
    __syncthreads();
    bool all_ok = true;
    for (int q = 0; q < k; ++q) {
      const double* xr = Vr + (long)q * n;
      const double* xi = Vi + (long)q * n;
      for (int r = tid; r < n; r += NT) {
        S.xr[r] = xr[r];
        if (C) S.xi[r] = xi[r];
      }
      __syncthreads();
      cta_matvec<C, NT>(P.re, P.im, n, S.xr, S.xi, S.wr, S.wi);
      ++matvecs;
      __syncthreads();
      const cplx lam = S.ritz[q];
      double e2 = 0, x2 = 0;
      for (int r = tid; r < n; r += NT) {
        const cplx x = {S.xr[r], C ? S.xi[r] : 0.0};
        const cplx w = cplx{S.wr[r], C ? S.wi[r] : 0.0} - lam * x;
        e2 += abs2(w);
        x2 += abs2(x);
        if (P.vre) P.vre[(long)r * k + q] = x.re;
        if (P.vim) P.vim[(long)r * k + q] = x.im;
      }
      const cplx sums = cta_sum2<NT>(e2, x2, S.red);
      const double rr = sqrt(sums.re) / (scale * (sums.im > 0 ? sqrt(sums.im) : 1.0));
      if (tid == 0) {
        A.ev_re[(long)P.index * k + q] = lam.re;
        A.ev_im[(long)P.index * k + q] = lam.im;
        A.res[(long)P.index * k + q] = rr;
      }
      if (!(rr <= A.tol)) all_ok = false;
    }
    if (status == OAPB_OK && !all_ok) status = OAPB_NOT_CONVERGED;
  }
  if (tid == 0) {
    A.status[P.index] = status;
    atomicAdd(A.matvecs, matvecs);
    atomicAdd(A.restarts, restarts);
    atomicAdd(A.op_bytes, matvecs * (unsigned long long)(C ? 16 : 8) * (unsigned long long)n * n);
  }
  __syncthreads();
}

template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_batched_iram(BatchArgs A) {
  extern __shared__ __align__(16) char bsm[];
  __shared__ int next;
  const int mcap = A.mcap;
  const BatchSmem S = carve(bsm, A.nmax, mcap);
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(A.counter, 1);
    __syncthreads();
    const int t = next;
    __syncthreads();
    if (t >= A.count) break;
    const BatchDesc P = A.desc[t];
    if (P.n < 2 || P.n > A.nmax) {
      if (threadIdx.x == 0) A.status[P.index] = OAPB_ERR_ARG;
      continue;
    }
    // per-problem hdim: the carve uses mcap; hess_core indexes with m = min(n, mcap)
    if (P.im)
      solve_one<true, NT>(A, P, blockIdx.x, S);
    else
      solve_one<false, NT>(A, P, blockIdx.x, S);
  }
}

const void* batched_kernel(int v) {
  switch (v) {
    case 1: return (const void*)k_batched_iram<128, 2>;
    case 2: return (const void*)k_batched_iram<256, 2>;
    case 3: return (const void*)k_batched_iram<128, 4>;
    case 4: return (const void*)k_batched_iram<64, 8>;
    default: return (const void*)k_batched_iram<256, 1>;
  }
}

cudaError_t launch_batched(int v, int grid, size_t smem, cudaStream_t s, const BatchArgs& A) {
  switch (v) {
    case 1: k_batched_iram<128, 2><<<grid, 128, smem, s>>>(A); break;
    case 2: k_batched_iram<256, 2><<<grid, 256, smem, s>>>(A); break;
    case 3: k_batched_iram<128, 4><<<grid, 128, smem, s>>>(A); break;
    case 4: k_batched_iram<64, 8><<<grid, 64, smem, s>>>(A); break;
    default: k_batched_iram<256, 1><<<grid, 256, smem, s>>>(A); break;
  }
  return cudaGetLastError();
}

// The autotuner's choice per (device, largest n, hdim, wanted, complex):
// the variant whose launch on a sample of the batch took the least device
// time (replaces the fixed launch shapes of utils::mapper::SetThreadsBlocks,
// oapUtils/ThreadsMapper.cpp:36-74).
struct BatchKey {
  int dev, nmax, mcap, k, cplx;
  bool operator<(const BatchKey& o) const {
    return std::tie(dev, nmax, mcap, k, cplx) < std::tie(o.dev, o.nmax, o.mcap, o.k, o.cplx);
  }
};
std::mutex g_bt_mutex;
std::map<BatchKey, int> g_bt_choice;

bool tuned_variant(const BatchKey& key, int* v) {
  std::lock_guard<std::mutex> lock(g_bt_mutex);
  auto it = g_bt_choice.find(key);
  if (it == g_bt_choice.end()) return false;
  *v = it->second;
  return true;
}

void remember_variant(const BatchKey& key, int v) {
  std::lock_guard<std::mutex> lock(g_bt_mutex);
  g_bt_choice[key] = v;
}

// Time every variant on an evenly strided sample of the size-sorted batch
// (one wave of the default variant's grid) with CUDA events; the sample's
// outputs land in the batch's output slots and are overwritten by the full
// launch that follows.  dsample: device room for the sample's descriptors.
int tune_batched(BatchArgs A, const std::vector<BatchDesc>& d, const int* grids, size_t smem, cudaStream_t s,
                 char* dsample, int* best) {
  const int count = (int)d.size();
  const int ns = std::min(count, grids[0]);
  std::vector<BatchDesc> sample(ns);
  for (int i = 0; i < ns; ++i) sample[i] = d[(long)i * count / ns];
  if (cudaMemcpyAsync(dsample, sample.data(), sizeof(BatchDesc) * ns, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  A.desc = (const BatchDesc*)dsample;
  A.count = ns;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return OAPB_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return OAPB_ERR_CUDA;
  }
  int rc = OAPB_OK;
  float best_ms = 0;
  *best = 0;
  for (int v = 0; v < kBtVariants && !rc; ++v) {
    if (cudaMemsetAsync((void*)A.counter, 0, 4 * sizeof(unsigned long long), s) != cudaSuccess ||
        cudaEventRecord(e0, s) != cudaSuccess ||
        launch_batched(v, std::min(grids[v], ns), smem, s, A) != cudaSuccess ||
        cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (v == 0 || ms < best_ms) {
      best_ms = ms;
      *best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // namespace oapb

using namespace oapb;

extern "C" {

int oapb_arnoldi_solve_batched(const oapb_arnoldi_config* cfg, const oapb_batch_problem* problems, uint32_t count,
                               double* eig_re, double* eig_im, double* residuals, int32_t* status,
                               oapb_batch_stats* stats, void* stream) {
  if (!cfg || !problems || count == 0 || !eig_re || !eig_im || !residuals || !status) return OAPB_ERR_ARG;
  const int mcap = (int)cfg->hdim, k = (int)cfg->wanted;
  if (mcap < 2 || mcap > kBtMaxM || k < 1 || k >= mcap || cfg->sort < 0 || cfg->sort > 5) return OAPB_ERR_ARG;
  if (cfg->autotune >= 2 && cfg->autotune >= 2 + kBtVariants) return OAPB_ERR_ARG;
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<BatchDesc> d(count);
  int nmax = 0;
  bool any_complex = false;
  for (uint32_t i = 0; i < count; ++i) {
    const oapb_batch_problem& p = problems[i];
    if (p.n < 2 || p.n > (uint32_t)kBtMaxN || !p.re || p.n <= (uint32_t)k) return OAPB_ERR_ARG;
    d[i] = BatchDesc{(int)p.n, (int)i, p.re, p.im, p.eigvec_re, p.eigvec_im};
    nmax = std::max(nmax, (int)p.n);
    any_complex |= p.im != nullptr;
  }
  // largest first: the atomic queue then balances uneven sizes
  std::stable_sort(d.begin(), d.end(), [](const BatchDesc& a, const BatchDesc& b) { return a.n > b.n; });
  nmax = (nmax + 1) & ~1;
  const size_t smem = batch_smem_bytes(nmax, mcap);
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem + 1024 > (size_t)optin) return OAPB_ERR_ARG;
  // the persistent grid of every launch variant (resident CTAs x SMs)
  int grids[kBtVariants];
  int gmax = 0;
  for (int v = 0; v < kBtVariants; ++v) {
    const void* kern = batched_kernel(v);
    OAPB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    OAPB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kBtThreadsOf[v], smem));
    grids[v] = std::min(kNumSMs * occ, (int)count);
    gmax = std::max(gmax, grids[v]);
  }
  if (grids[0] < 1) return OAPB_ERR_ARG;

  // one device allocation for descriptors (the batch, then a tuning sample),
  // counters, outputs and the basis slots
  const size_t vws = sizeof(double) * 2 * (size_t)(mcap + 1) * nmax * gmax;
  const size_t nout = (size_t)count * k;
  size_t off_desc = 0, off_cnt = align16(off_desc + sizeof(BatchDesc) * 2 * (size_t)count);
  size_t off_out = align16(off_cnt + 4 * sizeof(unsigned long long));
  size_t off_res = align16(off_out + 2 * sizeof(double) * nout);
  size_t off_st = align16(off_res + sizeof(double) * nout);
  size_t off_v = (off_st + sizeof(int) * count + 255) & ~(size_t)255;
  const size_t total = off_v + vws;
  char* buf = nullptr;
  if (cudaMallocAsync((void**)&buf, total, s) != cudaSuccess) {
    cudaGetLastError();
    return OAPB_ERR_NOMEM;
  }
  int rc = OAPB_OK;
  int variant = 0;
  do {
    if (cudaMemcpyAsync(buf + off_desc, d.data(), sizeof(BatchDesc) * count, cudaMemcpyHostToDevice, s) !=
        cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    BatchArgs A;
    A.desc = (const BatchDesc*)(buf + off_desc);
    A.count = (int)count;
    A.counter = (int*)(buf + off_cnt);
    A.matvecs = (unsigned long long*)(buf + off_cnt) + 1;
    A.restarts = (unsigned long long*)(buf + off_cnt) + 2;
    A.op_bytes = (unsigned long long*)(buf + off_cnt) + 3;
    A.mcap = mcap;
    A.k = k;
    A.which = cfg->sort;
    A.max_restarts = (int)cfg->max_restarts;
    A.tol = cfg->tolerance;
    A.rho = cfg->rho;
    A.seed = cfg->seed;
    A.vws = (double*)(buf + off_v);
    A.nmax = nmax;
    A.ev_re = (double*)(buf + off_out);
    A.ev_im = A.ev_re + nout;
    A.res = (double*)(buf + off_res);
    A.status = (int*)(buf + off_st);
    // launch variant: forced, cached, or timed on a sample of the batch
    if (cfg->autotune >= 2) {
      variant = cfg->autotune - 2;
    } else if (cfg->autotune == 1) {
      const BatchKey key{dev, nmax, mcap, k, any_complex ? 1 : 0};
      if (!tuned_variant(key, &variant)) {
        rc = tune_batched(A, d, grids, smem, s, buf + off_desc + sizeof(BatchDesc) * count, &variant);
        if (rc) break;
        remember_variant(key, variant);
      }
    }
    A.count = (int)count;
    A.desc = (const BatchDesc*)(buf + off_desc);
    if (cudaMemsetAsync(buf + off_cnt, 0, 4 * sizeof(unsigned long long), s) != cudaSuccess ||
        launch_batched(variant, grids[variant], smem, s, A) != cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    unsigned long long ctr[4];
    if (cudaMemcpyAsync(eig_re, A.ev_re, sizeof(double) * nout, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(eig_im, A.ev_im, sizeof(double) * nout, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(residuals, A.res, sizeof(double) * nout, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(status, A.status, sizeof(int) * count, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(ctr, buf + off_cnt, sizeof(ctr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    if (stats) {
      stats->problems = count;
      stats->converged = 0;
      for (uint32_t i = 0; i < count; ++i) stats->converged += status[i] == OAPB_OK;
      stats->matvecs = ctr[1];
      stats->restarts = ctr[2];
      stats->operator_bytes = ctr[3];
      stats->ctas = (uint32_t)grids[variant];
      stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      stats->variant = (uint32_t)variant;
      stats->threads = (uint32_t)kBtThreadsOf[variant];
    }
  } while (0);
  cudaFreeAsync(buf, s);
  if (rc == OAPB_OK) {
    for (uint32_t i = 0; i < count; ++i)
      if (status[i] != OAPB_OK) return OAPB_NOT_CONVERGED;
  }
  return rc;
}

}  // extern "C"
