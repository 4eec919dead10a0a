// Small dense kernels of the restart loop, one warp, FP64 complex.
//
// k_hess works on the m x m upper Hessenberg H of the Arnoldi factorization
// (column-major, m <= kMaxM):
//   1. complex Schur form T = Z^H H Z by single-shift QR sweeps (Givens
//      bulge chasing, Wilkinson shifts, deflation at
//      |T[i][i-1]| <= eps (|T[i-1][i-1]| + |T[i][i]|)), the restatement of
//      calculateTriangularHEigens (ArnoldiProcedures.cpp:341-349) with a
//      shifted, deflating iteration instead of the reference's unshifted one;
//   2. Ritz values = diag(T), sorted by the ArnUtils order
//      (ArnoldiUtils.cpp:24-50); wanted = first k (getWanted,
//      ArnoldiProcedures.cpp:381-398);
//   3. eigenvectors y_q = Z u_q of the wanted values (back substitution on
//      T) and Ritz estimates beta |e_m^T y_q|;
//   4. if not converged: exact shifts with the unwanted values
//      (iram_shiftedQRIterations, oapGenericArnoldiApi.h:186-222) on H,
//      Q accumulating the rotations, H compressed to its leading k x k block.
// With `dense` set the input is a general matrix, first reduced to
// Hessenberg form by Householder reflectors accumulated into Z.
//
// Every loop is bounded (30 m sweeps for the Schur form); hitting the bound
// sets bit 1 of DevState::status and the kernel returns.
#pragma once

#include "common.cuh"

namespace oapb {

constexpr int kMaxM = 256;

struct DevState {
  double fnorm2;    // ||f||^2 of the current residual vector
  double hnorm2;
  int dgks;         // second Gram-Schmidt pass needed for the current column
  int converged;
  int status;       // bit 0: breakdown (||f|| = 0), bit 1: Schur sweep limit
  int dgks_count;
  int brk;          // the current basis vector replaces a zero residual (H[j][j-1] = 0)
  int brk_count;
  double scale;     // max |theta| over the wanted set
  double maxest;    // max relative Ritz estimate of the wanted set
  cplx beta_hat;    // H[k][k-1] after the shifts
  cplx sigma;       // Q[m-1][k-1]
};

struct HessArgs {
  const cplx* Hin;  // m x m column-major input
  cplx* Hout;       // compressed H after the shifts (may alias Hin)
  cplx* Qout;       // accumulated shift rotations (m x m)
  cplx* ritz;       // m Ritz values in sort order
  cplx* Y;          // k eigenvectors of H (column q at Y + q m)
  double* est;      // k relative Ritz estimates
  int* order;       // m sort order (indices into diag(T))
  DevState* st;
  cplx* gws;        // global workspace (2 m^2) when shared memory is too small
  int m, k, nvec, which, do_shift, real_shifts, dense, use_beta;
  double tol;
  double beta;      // used when use_beta == 0 (dense mode: residual norms come separately)
};

#define TT_(i, j) T[(i) + (long)(j) * m]
#define ZZ_(i, j) Z[(i) + (long)(j) * m]

__device__ __forceinline__ double sort_key(cplx v, int which) {
  switch (which) {
    case 0: return -(v.re * v.re + v.im * v.im);
    case 1: return -v.re;
    case 2: return -v.im;
    case 3: return v.re * v.re + v.im * v.im;
    case 4: return v.re;
    default: return v.im;
  }
}

// One single-shift QR sweep on the active window [l, h] of Hessenberg T,
// applied to whole rows / columns; Z <- Z G^H for every rotation.
static __device__ void warp_sweep(cplx* T, cplx* Z, int m, int l, int h, cplx mu, int lane) {
  for (int k = l; k < h; ++k) {
    cplx x, y;
    if (k == l) {
      x = TT_(l, l) - mu;
      y = TT_(l + 1, l);
    } else {
      x = TT_(k, k - 1);
      y = TT_(k + 1, k - 1);
    }
    cplx p, q;
    givens(x, y, p, q);
    __syncwarp();
    const int j0 = k > 0 ? k - 1 : 0;
    for (int j = j0 + lane; j < m; j += 32) {
      cplx a = TT_(k, j), b = TT_(k + 1, j);
      TT_(k, j) = p * a + q * b;
      TT_(k + 1, j) = (-conj(q)) * a + conj(p) * b;
    }
    __syncwarp();
    const int ihi = (k + 2 < h) ? k + 2 : h;
    for (int i = lane; i <= ihi; i += 32) {
      cplx a = TT_(i, k), b = TT_(i, k + 1);
      TT_(i, k) = a * conj(p) + b * conj(q);
      TT_(i, k + 1) = (-a) * q + b * p;
    }
    if (Z)
      for (int i = lane; i < m; i += 32) {
        cplx a = ZZ_(i, k), b = ZZ_(i, k + 1);
        ZZ_(i, k) = a * conj(p) + b * conj(q);
        ZZ_(i, k + 1) = (-a) * q + b * p;
      }
    __syncwarp();
    if (k > l && lane == 0) TT_(k + 1, k - 1) = cplx{0, 0};
    __syncwarp();
  }
}

// |re| + |im| (LAPACK's CABS1): the deflation test only needs a norm-equivalent
__device__ __forceinline__ double cabs1(cplx a) { return fabs(a.re) + fabs(a.im); }

__device__ __forceinline__ bool negligible(const cplx* T, int m, int l) {
  const double eps = 2.220446049250313e-16;
  double s = cabs1(TT_(l - 1, l - 1)) + cabs1(TT_(l, l));
  if (s == 0) s = 1e-300;
  return cabs1(TT_(l, l - 1)) <= eps * s;
}

// Householder reduction of dense T to Hessenberg form, Z accumulating.
static __device__ void warp_hessenberg(cplx* T, cplx* Z, cplx* v, int m, int lane) {
  for (int k = 0; k + 2 < m; ++k) {
    double s = 0;
    for (int i = k + 1 + lane; i < m; i += 32) s += abs2(TT_(i, k));
    s = warp_sum(s);
    double a = sqrt(s);
    if (a == 0) continue;
    cplx x0 = TT_(k + 1, k);
    double ax0 = cabs_(x0);
    cplx ph = ax0 > 0 ? cplx{x0.re / ax0, x0.im / ax0} : cplx{1, 0};
    for (int i = lane; i < m; i += 32) v[i] = (i > k) ? TT_(i, k) : cplx{0, 0};
    __syncwarp();
    if (lane == 0) v[k + 1] = v[k + 1] + a * ph;
    __syncwarp();
    double vv = 0;
    for (int i = k + 1 + lane; i < m; i += 32) vv += abs2(v[i]);
    vv = warp_sum(vv);
    const double f = 2.0 / vv;
    // T <- P T : column j
    for (int j = lane; j < m; j += 32) {
      cplx d = {0, 0};
      for (int i = k + 1; i < m; ++i) d = d + conj(v[i]) * TT_(i, j);
      d = f * d;
      for (int i = k + 1; i < m; ++i) TT_(i, j) = TT_(i, j) - d * v[i];
    }
    __syncwarp();
    // T <- T P, Z <- Z P : row i
    for (int i = lane; i < m; i += 32) {
      cplx d = {0, 0}, e = {0, 0};
      for (int j = k + 1; j < m; ++j) {
        d = d + TT_(i, j) * v[j];
        e = e + ZZ_(i, j) * v[j];
      }
      d = f * d;
      e = f * e;
      for (int j = k + 1; j < m; ++j) {
        TT_(i, j) = TT_(i, j) - d * conj(v[j]);
        ZZ_(i, j) = ZZ_(i, j) - e * conj(v[j]);
      }
    }
    __syncwarp();
    for (int i = k + 2 + lane; i < m; i += 32) TT_(i, k) = cplx{0, 0};
    __syncwarp();
  }
}

// Complex Schur form in place; returns false when the sweep budget ran out.
static __device__ bool warp_schur(cplx* T, cplx* Z, int m, int lane) {
  int h = m - 1, its = 0, total = 0;
  while (h > 0) {
    int l = h;
    while (l > 0 && !negligible(T, m, l)) --l;
    __syncwarp();
    if (l > 0 && lane == 0) TT_(l, l - 1) = cplx{0, 0};
    __syncwarp();
    if (l == h) {
      --h;
      its = 0;
      continue;
    }
    if (++total > 30 * m) return false;
    cplx a = TT_(h - 1, h - 1), b = TT_(h - 1, h), c = TT_(h, h - 1), d = TT_(h, h);
    cplx mu;
    if (its > 0 && its % 10 == 0) {
      mu = d + cplx{cabs_(c), 0};
    } else {
      cplx tr2 = 0.5 * (a + d);
      cplx amd = 0.5 * (a - d);
      cplx disc = csqrt_(amd * amd + b * c);
      cplx m1 = tr2 + disc, m2 = tr2 - disc;
      mu = cabs_(m1 - d) < cabs_(m2 - d) ? m1 : m2;
    }
    warp_sweep(T, Z, m, l, h, mu, lane);
    ++its;
  }
  __syncwarp();
  return true;
}

// The body of k_hess for one warp (lane = 0..31 of the calling warp), with
// its workspaces passed in: T, Z (m x m each), u (m), key (m), ord (m).
// Callable from any kernel by one full warp; the outputs in `a` may point
// to shared or global memory.
static __device__ void hess_core(const HessArgs& a, cplx* T, cplx* Z, cplx* u, double* key, int* ord, int lane) {
  const int m = a.m, k = a.k;
  const long mm = (long)m * m;
  DevState* st = a.st;

  for (long i = lane; i < mm; i += 32) {
    T[i] = a.Hin[i];
    Z[i] = (i % m == i / m) ? cplx{1, 0} : cplx{0, 0};
  }
  __syncwarp();
  if (a.dense) warp_hessenberg(T, Z, u, m, lane);
  if (!warp_schur(T, Z, m, lane)) {
    if (lane == 0) { st->status |= 2; st->converged = 0; }
    return;
  }
  // sort order of diag(T)
  for (int i = lane; i < m; i += 32) {
    double kv = sort_key(TT_(i, i), a.which);
    key[i] = (kv != kv) ? INFINITY : kv;  // NaN sorts last; ranks stay a permutation
  }
  __syncwarp();
  for (int i = lane; i < m; i += 32) {
    int r = 0;
    for (int j = 0; j < m; ++j) r += (key[j] < key[i]) || (key[j] == key[i] && j < i);
    ord[r] = i;
  }
  __syncwarp();
  for (int q = lane; q < m; q += 32) {
    a.order[q] = ord[q];
    a.ritz[q] = TT_(ord[q], ord[q]);
  }
  double scale = 0;
  for (int q = 0; q < k; ++q) scale = fmax(scale, cabs_(TT_(ord[q], ord[q])));
  if (scale == 0) scale = 1;
  double tnorm = 0;
  for (int i = 0; i < m; ++i) tnorm = fmax(tnorm, cabs_(TT_(i, i)));
  const double small = 2.220446049250313e-16 * (tnorm > 0 ? tnorm : 1.0);
  const double beta = a.use_beta ? sqrt(st->fnorm2) : a.beta;

  // eigenvectors of the first nvec Ritz values (the wanted k and optional
  // guard vectors) and the estimates of the wanted ones
  double maxest = 0;
  const int nvec = a.nvec > k ? (a.nvec < m ? a.nvec : m) : k;
  for (int q = 0; q < nvec; ++q) {
    const int idx = ord[q];
    const cplx lam = TT_(idx, idx);
    for (int i = lane; i < m; i += 32) u[i] = (i == idx) ? cplx{1, 0} : cplx{0, 0};
    __syncwarp();
    for (int i = idx - 1; i >= 0; --i) {
      cplx acc = {0, 0};
      for (int j = i + 1 + lane; j <= idx; j += 32) acc = acc + TT_(i, j) * u[j];
      acc.re = warp_sum(acc.re);
      acc.im = warp_sum(acc.im);
      cplx den = TT_(i, i) - lam;
      if (cabs_(den) < small) den = cplx{small, 0};
      if (lane == 0) {
        cplx ui = -cdiv(acc, den);
        u[i] = ui;
      }
      __syncwarp();
      if (cabs_(u[i]) > 1e150) {  // rescale to avoid overflow
        for (int j = i + lane; j <= idx; j += 32) u[j] = 1e-150 * u[j];
        __syncwarp();
      }
    }
    double nrm = 0;
    cplx ylast = {0, 0};
    for (int r = lane; r < m; r += 32) {
      cplx y = {0, 0};
      for (int j = 0; j <= idx; ++j) y = y + ZZ_(r, j) * u[j];
      a.Y[(long)q * m + r] = y;
      nrm += abs2(y);
      if (r == m - 1) ylast = y;
    }
    nrm = sqrt(warp_sum(nrm));
    ylast.re = warp_sum(ylast.re);
    ylast.im = warp_sum(ylast.im);
    __syncwarp();
    const double inv = nrm > 0 ? 1.0 / nrm : 0.0;
    for (int r = lane; r < m; r += 32) a.Y[(long)q * m + r] = inv * a.Y[(long)q * m + r];
    const double e = beta * cabs_(ylast) * inv / scale;
    if (lane == 0) a.est[q] = e;
    if (q < k) maxest = fmax(maxest, e);
    __syncwarp();
  }
  const int conv = maxest <= a.tol;
  if (lane == 0) {
    st->converged = conv;
    st->scale = scale;
    st->maxest = maxest;
  }
  if (conv || !a.do_shift) return;

  // exact shifts on H with the unwanted Ritz values (kept in u[] before T
  // is reloaded with H)
  __syncwarp();
  for (int q = lane; q < m; q += 32) u[q] = TT_(ord[q], ord[q]);
  __syncwarp();
  for (long i = lane; i < mm; i += 32) {
    T[i] = a.Hin[i];
    Z[i] = (i % m == i / m) ? cplx{1, 0} : cplx{0, 0};
  }
  __syncwarp();
  for (int q = k; q < m; ++q) {
    cplx mu = u[q];
    if (a.real_shifts) mu.im = 0;
    int hb = m - 1;
    while (hb > 0) {
      int l = hb;
      while (l > 0 && !negligible(T, m, l)) --l;
      __syncwarp();
      if (l > 0 && lane == 0) TT_(l, l - 1) = cplx{0, 0};
      __syncwarp();
      if (l < hb) warp_sweep(T, Z, m, l, hb, mu, lane);
      hb = l - 1;
    }
  }
  __syncwarp();
  if (lane == 0) {
    st->beta_hat = TT_(k, k - 1);
    st->sigma = ZZ_(m - 1, k - 1);
  }
  for (long i = lane; i < mm; i += 32) {
    const int r = i % m, c = i / m;
    a.Hout[i] = (r < k && c < k) ? T[i] : cplx{0, 0};
    a.Qout[i] = Z[i];
  }
}

static __global__ void __launch_bounds__(32) k_hess(HessArgs a) {
  extern __shared__ cplx sws[];
  __shared__ cplx u[kMaxM];
  __shared__ double key[kMaxM];
  __shared__ int ord[kMaxM];
  cplx* T = a.gws ? a.gws : sws;
  hess_core(a, T, T + (long)a.m * a.m, u, key, ord, threadIdx.x);
}

#undef TT_
#undef ZZ_

}  // namespace oapb
