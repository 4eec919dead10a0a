// Small dense kernels of the restart loop and of the block methods' checks,
// FP64 complex (FP32 working arithmetic in k_hess_f32).
//
// k_hess works on the m x m upper Hessenberg H of the Arnoldi factorization
// (column-major, m <= kMaxM):
//   1. complex Schur form T = Z^H H Z by single-shift QR sweeps (Givens
//      bulge chasing, Wilkinson shifts, deflation at
//      |T[i][i-1]| <= eps (|T[i-1][i-1]| + |T[i][i]|)), the restatement of
//      calculateTriangularHEigens (ArnoldiProcedures.cpp:341-349) with a
//      shifted, deflating iteration instead of the reference's unshifted
//      one; for a Hermitian H (a Hermitian or real symmetric operator) the
//      implicit symmetric tridiagonal QR instead;
//   2. Ritz values = diag(T), sorted by the ArnUtils order
//      (ArnoldiUtils.cpp:24-50); wanted = first k (getWanted,
//      ArnoldiProcedures.cpp:381-398);
//   3. eigenvectors y_q = Z u_q of the wanted values (back substitution on
//      T) and Ritz estimates beta |e_m^T y_q|;
//   4. if not converged: exact shifts with the unwanted values
//      (iram_shiftedQRIterations, oapGenericArnoldiApi.h:186-222) on H,
//      Q accumulating the rotations, H compressed to its leading k x k block.
// With `dense` set the input is a general matrix, first reduced to
// Hessenberg form by Householder reflectors accumulated into Z.  The input
// is scaled by a power of two (exact) so that the rotations need no
// overflow branches.
//
// Work layout: T and Z are column-major with an odd leading dimension
// hess_ld(m), so a lane-per-column access (row rotations) and a
// lane-per-row access (column rotations) are both free of bank conflicts.
// A QR sweep runs its chain of rotations in registers (the 2 x 2 window and
// the bulge, one shuffle per rotation) while the lanes apply each row
// rotation to their columns; the column rotations of the sweep, and those on
// Z, are applied after the chain (each lane the whole sequence to its
// rows).  The eigenvector back substitutions run one lane per eigenvector
// (T read by broadcast).  The sweeps run on one warp; for m <= 32 the kernel
// has four warps, which share the Householder reduction and the product
// Y = Z U.
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
  int status;       // bit 0: breakdown (||f|| = 0), bit 1: Schur sweep limit, bit 2: ||f|| not finite
  int dgks_count;
  int brk;          // the current basis vector replaces a zero residual (H[j][j-1] = 0)
  int brk_count;
  double scale;     // max |theta| over the wanted set
  double maxest;    // max relative Ritz estimate of the wanted set
  cplx beta_hat;    // H[k][k-1] after the shifts
  cplx sigma;       // Q[m-1][k-1]
  int symtri;       // eigensolves that took the Hermitian tridiagonal path
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
  cplx* gws;        // global workspace (hess_ws_cplx(m)) when shared memory is too small
  int m, k, nvec, which, do_shift, real_shifts, dense, use_beta;
  double tol;
  double beta;      // used when use_beta == 0 (dense mode: residual norms come separately)
  const int* skip = nullptr;  // k_hess: when set and *skip != 0, return at once (another solver delivered)
};

// leading dimension of the T / Z work arrays (odd)
__host__ __device__ __forceinline__ int hess_ld(int m) { return m | 1; }
// scratch (rotation list and eigenvector columns), in cplx
__host__ __device__ __forceinline__ size_t hess_scratch_cplx(int m) { return (size_t)m * 32 + 2 * (size_t)m + 2; }
// whole k_hess workspace: T, Z and the scratch
__host__ __device__ __forceinline__ size_t hess_ws_cplx(int m) {
  return 2 * (size_t)hess_ld(m) * m + hess_scratch_cplx(m);
}

// precision constants of the working type
template <typename R>
struct HessK;
template <>
struct HessK<double> {
  static constexpr double eps = 2.220446049250313e-16, tiny = 1e-300, big = 1e150, unbig = 1e-150;
  static constexpr double tiny2 = 1e-280;  // |x|^2 + |y|^2 of a negligible pair (prescaled matrix)
};
template <>
struct HessK<float> {
  static constexpr float eps = 1.1920929e-7f, tiny = 1e-37f, big = 1e15f, unbig = 1e-15f;  // big^2 stays finite
  static constexpr float tiny2 = 1e-36f;
};

__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float rsqrt_t(float a) { return rsqrtf(a); }
__device__ __forceinline__ double rsqrt_t(double a) { return rsqrt(a); }
__device__ __forceinline__ float sqrt_t(float a) { return sqrtf(a); }
__device__ __forceinline__ float abs_t(float a) { return fabsf(a); }
__device__ __forceinline__ double abs_t(double a) { return fabs(a); }
__device__ __forceinline__ double sqrt_t(double a) { return sqrt(a); }

// a b + c with fused multiply-adds
template <typename Cx>
__device__ __forceinline__ Cx cfma(Cx a, Cx b, Cx c) {
  return {fma_t(a.re, b.re, fma_t(-a.im, b.im, c.re)), fma_t(a.re, b.im, fma_t(a.im, b.re, c.im))};
}
// a b + c d
template <typename Cx>
__device__ __forceinline__ Cx cfma2(Cx a, Cx b, Cx c, Cx d) {
  return cfma(a, b, c * d);
}

// The rotation of givens() (p x + q y = sqrt(|x|^2 + |y|^2), p = conj(x) / r,
// q = conj(y) / r) for entries of a matrix that hess_core has scaled to a
// largest entry in [1, 2): the sum of squares cannot overflow, and a pair
// whose squares sum below tiny2 (far below the working precision relative
// to the matrix) gives the identity.  No branch: the sweep's rotation chain
// stays one straight block of instructions.
template <typename Cx>
__device__ __forceinline__ void givens_s(Cx x, Cx y, Cx& p, Cx& q) {
  using R = decltype(Cx::re);
  const R r2 = fma_t(x.re, x.re, fma_t(x.im, x.im, fma_t(y.re, y.re, y.im * y.im)));
  const bool ok = r2 > HessK<R>::tiny2;
  const R ir = rsqrt_t(ok ? r2 : R(1));
  p = ok ? Cx{x.re * ir, -x.im * ir} : Cx{1, 0};
  q = ok ? Cx{y.re * ir, -y.im * ir} : Cx{0, 0};
}

// principal square root of z (prescaled entries: |z| stays far inside the
// range), re >= 0
template <typename Cx>
__device__ __forceinline__ Cx csqrt_s(Cx z) {
  using R = decltype(Cx::re);
  const R r = sqrt_t(abs2(z));
  const R u = R(0.5) * (r + abs_t(z.re));
  const R iu = rsqrt_t(u > 0 ? u : R(1));
  const R t = u > 0 ? u * iu : R(0), hh = u > 0 ? R(0.5) * z.im * iu : R(0);  // sqrt(u), im / (2 sqrt(u))
  return z.re >= 0 ? Cx{t, hh} : Cx{abs_t(hh), z.im >= 0 ? t : -t};
}

__device__ __forceinline__ double warp_sum_t(double v) { return warp_sum(v); }
__device__ __forceinline__ float warp_sum_t(float v) { return warp_sumf(v); }

#define TT_(i, j) T[(i) + (j) * ld]
#define ZZ_(i, j) Z[(i) + (j) * ld]

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

// |re| + |im| (LAPACK's CABS1): the deflation test only needs a norm-equivalent
__device__ __forceinline__ double cabs1(cplx a) { return fabs(a.re) + fabs(a.im); }
__device__ __forceinline__ float cabs1(cplxf a) { return fabsf(a.re) + fabsf(a.im); }

template <typename Cx>
__device__ __forceinline__ bool negligible(const Cx* T, int ld, int l) {
  using R = decltype(Cx::re);
  R s = cabs1(TT_(l - 1, l - 1)) + cabs1(TT_(l, l));
  if (s == 0) s = HessK<R>::tiny;
  return cabs1(TT_(l, l - 1)) <= HessK<R>::eps * s;
}

__device__ __forceinline__ cplx shfl_c(cplx v, int src) {
  return cplx{__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}
__device__ __forceinline__ cplxf shfl_c(cplxf v, int src) {
  return cplxf{__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}

// The largest l in [1, h] with T[l][l-1] negligible, else 0 (all lanes).
template <typename Cx>
static __device__ int find_split(const Cx* T, int ld, int h, int lane) {
  for (int base = h; base >= 1; base -= 32) {
    const int l = base - lane;
    const bool f = l >= 1 && negligible(T, ld, l);
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (bal) return base - (__ffs(bal) - 1);
  }
  return 0;
}

// One single-shift QR sweep on the active window [l, h] of Hessenberg T,
// applied to whole rows / columns of T (the final T is G T G^H with G =
// G_{h-1} ... G_l); Z <- Z G_l^H ... G_{h-1}^H.  rot: 2 m cplx of scratch.
// T must be prescaled (hess_core): the rotations come from givens_s.
//
// The rotations form a dependent chain: rotation k needs the bulge pair
// left by rotation k - 1.  That chain runs in registers: every lane carries
// the 2 x 2 window T[k..k+1][k..k+1] and the bulge through the algebra of
// one rotation on both sides, and the one entry of the window that earlier
// rotations reach from outside it, T[k][k+1], comes from the lane that owns
// column k + 1.  The matrix itself is updated off the chain: while the chain
// runs, lane c applies each row rotation to column c (its row-k entry carried
// in a register, the row-(k+1) entry read once), and after the chain one
// lane per row applies all column rotations to its row of T and of Z.  Left
// and right rotations commute, so the result is G T G^H as in the
// interleaved sweep; the entries below the subdiagonal that the interleaved
// sweep never fills come out of this order at rounding level and are set
// to zero.  The loop over rotations l .. h-2 has no branch (the last
// rotation, which has no next window, is peeled): a single warp issues it
// as one straight block, so the row updates fill the chain's latency.
// NT: columns per lane (c = lane + 32 t, t < NT); m <= 32 NT.  WZ: Z is
// updated (Z non-null).
template <typename Cx, int NT, bool WZ>
static __device__ __forceinline__ void warp_sweep_nt(Cx* T, Cx* Z, int m, int ld, int l, int h, Cx mu, Cx* rot,
                                                     int lane) {
  const int nt = (m + 31) >> 5;
  const Cx zero = {0, 0};
  Cx carry[NT], b[NT];
  bool own[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int c = lane + 32 * t;
    own[t] = t < nt && c >= l && c < m;
    carry[t] = own[t] ? TT_(l, c) : zero;
    b[t] = own[t] ? TT_(l + 1, c) : zero;
  }
  Cx D = TT_(l, l), E = TT_(l, l + 1), F = TT_(l + 1, l), G = TT_(l + 1, l + 1);
  Cx x = D - mu, y = F;
  int k = l;
  for (; k + 1 < h; ++k) {
    // inputs of this step from rows k + 1, k + 2 (not written before it)
    Cx bn[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) bn[t] = own[t] ? TT_(k + 2, lane + 32 * t) : zero;
    const Cx s2 = TT_(k + 2, k + 1), g2 = TT_(k + 2, k + 2), t2 = TT_(k + 1, k + 2);
    // row k's entry of column k + 2 before this rotation
    const int c2 = k + 2;
    Cx e = carry[0];
#pragma unroll
    for (int t = 1; t < NT; ++t)
      if (t == (c2 >> 5)) e = carry[t];
    const Cx epre = shfl_c(e, c2 & 31);
    Cx p, q;
    givens_s(x, y, p, q);
    rot[2 * k] = p;  // every lane stores the same values
    rot[2 * k + 1] = q;
    const Cx pc = conj(p), qc = conj(q), nqc = -qc;
    // the window through rotation k on both sides, then the next one
    const Cx F1 = cfma2(nqc, D, pc, F), G1 = cfma2(nqc, E, pc, G);
    x = cfma2(F1, pc, G1, qc);   // T[k+1][k]
    y = s2 * qc;                 // T[k+2][k], the bulge
    D = cfma2(-F1, q, G1, p);    // T[k+1][k+1]
    F = s2 * p;                  // T[k+2][k+1]
    G = g2;                      // T[k+2][k+2]
    E = cfma2(nqc, epre, pc, t2);  // T[k+1][k+2] after row rotation k
    // row rotation k on the lanes' columns (rows k, k + 1)
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      if (own[t]) {
        TT_(k, lane + 32 * t) = cfma2(p, carry[t], q, b[t]);
        carry[t] = cfma2(nqc, carry[t], pc, b[t]);
      }
      b[t] = bn[t];
    }
  }
  {  // rotation h - 1
    Cx p, q;
    givens_s(x, y, p, q);
    rot[2 * k] = p;
    rot[2 * k + 1] = q;
    const Cx pc = conj(p), nqc = -conj(q);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      if (own[t]) {
        TT_(k, lane + 32 * t) = cfma2(p, carry[t], q, b[t]);
        TT_(h, lane + 32 * t) = cfma2(nqc, carry[t], pc, b[t]);
      }
    }
  }
  __syncwarp();
  // column rotations l .. h-1 on rows 0 .. h of T and on every row of Z (one
  // lane per row); the entries below the subdiagonal of the window (rows
  // i >= k + 2 of column k) are set to zero.  Rows below h hold zeros in
  // these columns: their T stores are skipped.
  for (int i = lane; i < m; i += 32) {
    const bool trow = i <= h;
    Cx c = TT_(i, l);
    Cx cz = WZ ? ZZ_(i, l) : zero;
    for (int kk = l; kk < h; ++kk) {
      const Cx p = rot[2 * kk], q = rot[2 * kk + 1], pc = conj(p), qc = conj(q);
      const Cx nb = TT_(i, kk + 1);
      const Cx tk = cfma2(c, pc, nb, qc);
      if (trow) TT_(i, kk) = kk + 2 <= i ? zero : tk;
      c = cfma2(-c, q, nb, p);
      if (WZ) {
        const Cx z1 = ZZ_(i, kk + 1);
        ZZ_(i, kk) = cfma2(cz, pc, z1, qc);
        cz = cfma2(-cz, q, z1, p);
      }
    }
    if (trow) TT_(i, h) = c;
    if (WZ) ZZ_(i, h) = cz;
  }
  __syncwarp();
}

// the carries stay in registers when their count is fixed by m's range
template <typename Cx, bool WZ>
static __device__ void warp_sweep_z(Cx* T, Cx* Z, int m, int ld, int l, int h, Cx mu, Cx* rot, int lane) {
  if (m <= 32)
    warp_sweep_nt<Cx, 1, WZ>(T, Z, m, ld, l, h, mu, rot, lane);
  else if (m <= 64)
    warp_sweep_nt<Cx, 2, WZ>(T, Z, m, ld, l, h, mu, rot, lane);
  else if (m <= 128)
    warp_sweep_nt<Cx, 4, WZ>(T, Z, m, ld, l, h, mu, rot, lane);
  else
    warp_sweep_nt<Cx, kMaxM / 32, WZ>(T, Z, m, ld, l, h, mu, rot, lane);
}
template <typename Cx>
static __device__ void warp_sweep(Cx* T, Cx* Z, int m, int ld, int l, int h, Cx mu, Cx* rot, int lane) {
  if (Z)
    warp_sweep_z<Cx, true>(T, Z, m, ld, l, h, mu, rot, lane);
  else
    warp_sweep_z<Cx, false>(T, Z, m, ld, l, h, mu, rot, lane);
}

// Householder reduction of dense T to Hessenberg form, Z accumulating.
template <typename Cx>
static __device__ void warp_hessenberg(Cx* T, Cx* Z, Cx* v, int m, int ld, int lane) {
  using R = decltype(Cx::re);
  for (int k = 0; k + 2 < m; ++k) {
    R s = 0;
    for (int i = k + 1 + lane; i < m; i += 32) s += abs2(TT_(i, k));
    s = warp_sum_t(s);
    R a = sqrt(s);
    if (a == 0) continue;
    Cx x0 = TT_(k + 1, k);
    R ax0 = cabs_(x0);
    Cx ph = ax0 > 0 ? Cx{x0.re / ax0, x0.im / ax0} : Cx{1, 0};
    for (int i = lane; i < m; i += 32) v[i] = (i > k) ? TT_(i, k) : Cx{0, 0};
    __syncwarp();
    if (lane == 0) v[k + 1] = v[k + 1] + a * ph;
    __syncwarp();
    R vv = 0;
    for (int i = k + 1 + lane; i < m; i += 32) vv += abs2(v[i]);
    vv = warp_sum_t(vv);
    const R f = R(2) / vv;
    // T <- P T : column j (two partial sums break the dependency chain)
    for (int j = lane; j < m; j += 32) {
      Cx d0 = {0, 0}, d1 = {0, 0};
      int i = k + 1;
      for (; i + 1 < m; i += 2) {
        d0 = d0 + conj(v[i]) * TT_(i, j);
        d1 = d1 + conj(v[i + 1]) * TT_(i + 1, j);
      }
      if (i < m) d0 = d0 + conj(v[i]) * TT_(i, j);
      const Cx d = f * (d0 + d1);
      for (i = k + 1; i < m; ++i) TT_(i, j) = TT_(i, j) - d * v[i];
    }
    __syncwarp();
    // T <- T P, Z <- Z P : row i
    for (int i = lane; i < m; i += 32) {
      Cx d0 = {0, 0}, d1 = {0, 0}, e0 = {0, 0}, e1 = {0, 0};
      int j = k + 1;
      for (; j + 1 < m; j += 2) {
        d0 = d0 + TT_(i, j) * v[j];
        d1 = d1 + TT_(i, j + 1) * v[j + 1];
        e0 = e0 + ZZ_(i, j) * v[j];
        e1 = e1 + ZZ_(i, j + 1) * v[j + 1];
      }
      if (j < m) {
        d0 = d0 + TT_(i, j) * v[j];
        e0 = e0 + ZZ_(i, j) * v[j];
      }
      const Cx d = f * (d0 + d1), e = f * (e0 + e1);
      for (j = k + 1; j < m; ++j) {
        TT_(i, j) = TT_(i, j) - d * conj(v[j]);
        ZZ_(i, j) = ZZ_(i, j) - e * conj(v[j]);
      }
    }
    __syncwarp();
    for (int i = k + 2 + lane; i < m; i += 32) TT_(i, k) = Cx{0, 0};
    __syncwarp();
  }
}

// barrier of the NW warps of a multi-warp small eigensolver (named barrier
// 1: the rest of a block may use barrier 0)
__device__ __forceinline__ void hess_bar(int nthr) { asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory"); }

// The Householder reduction on NW warps (m <= 32, all NW warps calling;
// warp 0 forms each reflector): per step, P T has one lane per column and
// the rows split over the warps (partial sums v^H T summed through shared
// memory), T P and Z P one lane per row and the columns split over the
// warps.  part: 2 NW x 32 entries of shared scratch; v: 32; fs: 1.
template <typename Cx, int NW>
static __device__ void block_hessenberg32(Cx* T, Cx* Z, Cx* v, Cx* part, decltype(Cx::re)* fs, int m, int ld,
                                          int warp, int lane) {
  using R = decltype(Cx::re);
  constexpr int nthr = NW * 32;
  const Cx zero = {0, 0};
  Cx* pa = part;            // NW x 32: P T partials, then T P partials
  Cx* pz = part + NW * 32;  // NW x 32: Z P partials
  for (int k = 0; k + 2 < m; ++k) {
    hess_bar(nthr);  // the previous step's updates are in place
    if (warp == 0) {
      const Cx xi = (lane > k && lane < m) ? TT_(lane, k) : zero;
      const R s = warp_sum_t(abs2(xi));
      const Cx x0 = shfl_c(xi, k + 1);
      R f = 0;
      Cx vi = xi;
      if (s > 0) {
        const R a = sqrt_t(s), ax0 = sqrt_t(abs2(x0));
        const Cx ph = ax0 > 0 ? Cx{x0.re / ax0, x0.im / ax0} : Cx{1, 0};
        if (lane == k + 1) vi = xi + a * ph;
        f = R(1) / (a * (a + ax0));  // 2 / |v|^2
      }
      v[lane] = vi;  // zero outside rows k + 1 .. m - 1
      if (lane == 0) *fs = f;
    }
    hess_bar(nthr);
    const R f = *fs;
    if (f == 0) continue;  // column k is reduced already (the same for every warp)
    // P T: lane j = column (j >= k), this warp's rows of k + 1 .. m - 1
    const int nr = m - k - 1, cr = (nr + NW - 1) / NW;
    const int i0 = k + 1 + warp * cr, i1 = i0 + cr < m ? i0 + cr : m;
    const bool colj = lane >= k && lane < m;
    {
      Cx w0 = zero, w1 = zero;
      if (colj) {
        int i = i0;
        for (; i + 1 < i1; i += 2) {
          w0 = cfma(conj(v[i]), TT_(i, lane), w0);
          w1 = cfma(conj(v[i + 1]), TT_(i + 1, lane), w1);
        }
        if (i < i1) w0 = cfma(conj(v[i]), TT_(i, lane), w0);
      }
      pa[warp * 32 + lane] = w0 + w1;
    }
    hess_bar(nthr);
    {
      Cx w = pa[lane];
#pragma unroll
      for (int u = 1; u < NW; ++u) w = w + pa[u * 32 + lane];
      w = f * w;
      if (colj)
        for (int i = i0; i < i1; ++i) TT_(i, lane) = (lane == k && i >= k + 2) ? zero : cfma(-v[i], w, TT_(i, lane));
    }
    hess_bar(nthr);
    // T P, Z P: lane i = row, this warp's columns of k + 1 .. m - 1
    const int j0 = k + 1 + warp * cr, j1 = j0 + cr < m ? j0 + cr : m;
    const bool rowi = lane < m;
    {
      Cx y0 = zero, y1 = zero;
      if (rowi)
        for (int j = j0; j < j1; ++j) {
          y0 = cfma(TT_(lane, j), v[j], y0);
          y1 = cfma(ZZ_(lane, j), v[j], y1);
        }
      pa[warp * 32 + lane] = y0;
      pz[warp * 32 + lane] = y1;
    }
    hess_bar(nthr);
    {
      Cx y = pa[lane], yz = pz[lane];
#pragma unroll
      for (int u = 1; u < NW; ++u) {
        y = y + pa[u * 32 + lane];
        yz = yz + pz[u * 32 + lane];
      }
      y = f * y;
      yz = f * yz;
      if (rowi)
        for (int j = j0; j < j1; ++j) {
          TT_(lane, j) = cfma(-y, conj(v[j]), TT_(lane, j));
          ZZ_(lane, j) = cfma(-yz, conj(v[j]), ZZ_(lane, j));
        }
    }
  }
  hess_bar(nthr);
}

// Complex Schur form in place; returns false when the sweep budget ran out.
template <typename Cx>
static __device__ bool warp_schur(Cx* T, Cx* Z, int m, int ld, Cx* rot, int lane) {
  using R = decltype(Cx::re);
  int h = m - 1, its = 0, total = 0;
  while (h > 0) {
    const int l = find_split(T, ld, h, lane);
    if (l > 0 && lane == 0) TT_(l, l - 1) = Cx{0, 0};
    __syncwarp();
    if (l == h) {
      --h;
      its = 0;
      continue;
    }
    if (++total > 30 * m) return false;
    // Wilkinson shift: the eigenvalue of the trailing 2 x 2 nearer d
    // (prescaled entries: squared moduli stay in range); every tenth sweep
    // of a window an exceptional shift d + |c|
    const Cx a = TT_(h - 1, h - 1), b = TT_(h - 1, h), c = TT_(h, h - 1), d = TT_(h, h);
    const Cx tr2 = R(0.5) * (a + d), amd = R(0.5) * (a - d);
    const Cx disc = csqrt_s(cfma(amd, amd, b * c));
    const Cx m1 = tr2 + disc, m2 = tr2 - disc;
    Cx mu = abs2(m1 - d) < abs2(m2 - d) ? m1 : m2;
    if (its > 0 && its % 10 == 0) mu = d + Cx{sqrt_t(abs2(c)), 0};
    warp_sweep(T, Z, m, ld, l, h, mu, rot, lane);
    ++its;
  }
  __syncwarp();
  return true;
}

// Hermitian tridiagonal path (the restart loop of a Hermitian operator,
// real symmetric included, whose Hessenberg matrix is Hermitian tridiagonal
// to rounding): with the diagonal unitary D of phases D_0 = 1, D_{i+1} =
// D_i e_i / |e_i| (e_i = H[i+1][i]), H = D T' D^H where T' is real
// symmetric tridiagonal with diagonal Re H[i][i] and off-diagonal |e_i|.
// d (m) and e (m - 1) of T' are real in shared memory; Z starts as D and
// accumulates the real rotations, so Z = D Q' holds the eigenvectors of H
// (and the exact shifts' Q for the restart, with T' after the shifts as the
// new H).  The implicit QR step with shift mu on the window [l, h] (Golub &
// Van Loan, Matrix Computations, Alg. 8.3.2) runs its rotation chain on
// lane 0 and records the rotations (c, s) in cs; every lane then applies
// them to one row of Z (Z <- Z G^T).  The rotation of the pair (x, y) is
// c = x / r, s = y / r (the entries are prescaled, so r^2 stays in range; a
// pair below tiny2 gives the identity).

// true when T (prescaled: largest entry in [1, 2), m x m) is Hermitian to
// rtol: the Arnoldi matrix of a Hermitian operator, whose entries beyond the
// tridiagonal band and whose departure from Hermitian symmetry come from the
// basis's loss of orthogonality (about 4e-13 of max |H| for a real n = 256
// operator with eigenvalues over three decades); they are dropped, which
// moves the Ritz values by as much, so rtol is a tenth of the residual goal
// (every result is verified against the operator)
template <typename Cx>
static __device__ bool warp_is_hermitian(const Cx* T, int m, int ld, double rtol, int lane) {
  using R = decltype(Cx::re);
  const R tol = (R)rtol;
  int bad = 0;
  for (int e = lane; e < m * m; e += 32) {
    const int r = e % m, c = e / m;
    const Cx a = TT_(r, c), b = TT_(c, r);
    if (!(abs_t(a.re - b.re) <= tol && abs_t(a.im + b.im) <= tol)) bad = 1;
  }
  return !__any_sync(0xffffffffu, bad);
}

template <typename R>
static __device__ void symtri_step(R* d, R* e, R* cs, int l, int h, R mu) {  // one lane
  R x = d[l] - mu, y = e[l];
  for (int k = l; k < h; ++k) {
    const R r2 = x * x + y * y;
    const bool ok = r2 > HessK<R>::tiny2;
    const R ir = rsqrt_t(ok ? r2 : R(1));
    const R c = ok ? x * ir : R(1), s = ok ? y * ir : R(0);
    if (k > l) e[k - 1] = ok ? r2 * ir : x;
    const R dk = d[k], dk1 = d[k + 1], ek = e[k];
    const R t1 = c * dk + s * ek, t2 = c * ek + s * dk1;
    const R t3 = c * ek - s * dk, t4 = c * dk1 - s * ek;
    d[k] = c * t1 + s * t2;
    e[k] = c * t2 - s * t1;
    d[k + 1] = c * t4 - s * t3;
    cs[2 * k] = c;
    cs[2 * k + 1] = s;
    if (k + 1 < h) {  // the bulge at (k + 2, k)
      x = e[k];
      y = s * e[k + 1];
      e[k + 1] = c * e[k + 1];
    }
  }
}

// Z <- Z G_l^T ... G_{h-1}^T, one lane per row
template <typename Cx>
static __device__ void symtri_apply_z(Cx* Z, const decltype(Cx::re)* cs, int m, int ld, int l, int h, int lane) {
  for (int i = lane; i < m; i += 32) {
    Cx zc = ZZ_(i, l);
    for (int k = l; k < h; ++k) {
      const auto c = cs[2 * k], s = cs[2 * k + 1];
      const Cx z1 = ZZ_(i, k + 1);
      ZZ_(i, k) = Cx{c * zc.re + s * z1.re, c * zc.im + s * z1.im};
      zc = Cx{c * z1.re - s * zc.re, c * z1.im - s * zc.im};
    }
    ZZ_(i, h) = zc;
  }
}

// the largest l in [1, h] with e[l-1] negligible, else 0 (all lanes)
template <typename R>
static __device__ int symtri_split(const R* d, const R* e, int h, int lane) {
  for (int base = h; base >= 1; base -= 32) {
    const int l = base - lane;
    const bool f = l >= 1 && abs_t(e[l - 1]) <= HessK<R>::eps * (abs_t(d[l - 1]) + abs_t(d[l]));
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (bal) return base - (__ffs(bal) - 1);
  }
  return 0;
}

// T (m x m, Hermitian tridiagonal) -> d, e of T'; Z (the identity on
// entry) <- D, the phases
template <typename Cx>
static __device__ void symtri_load(const Cx* T, Cx* Z, int m, int ld, decltype(Cx::re)* d, decltype(Cx::re)* e,
                                   int lane) {
  using R = decltype(Cx::re);
  for (int i = lane; i < m; i += 32) {
    d[i] = TT_(i, i).re;
    if (i + 1 < m) e[i] = sqrt_t(abs2(TT_(i + 1, i)));
  }
  __syncwarp();
  if (lane == 0) {
    Cx ph = {1, 0};
    for (int i = 0; i + 1 < m; ++i) {
      const Cx sub = TT_(i + 1, i);
      const R a = e[i];
      if (a > 0) ph = ph * Cx{sub.re / a, sub.im / a};
      ZZ_(i + 1, i + 1) = ph;
    }
  }
  __syncwarp();
}
template <typename Cx>
static __device__ void symtri_store(Cx* T, int m, int ld, const decltype(Cx::re)* d, const decltype(Cx::re)* e,
                                    int lane) {
  __syncwarp();
  for (int x = lane; x < m * m; x += 32) {
    const int r = x % m, c = x / m;
    using R = decltype(Cx::re);
    const R v = r == c ? d[r] : (r == c + 1 ? e[c] : (c == r + 1 ? e[r] : R(0)));
    TT_(r, c) = Cx{v, 0};
  }
  __syncwarp();
}

// Eigen-decomposition of the symmetric tridiagonal (d, e): d becomes the
// eigenvalues, Z accumulates the rotations; false when the sweep budget ran
// out.
template <typename Cx>
static __device__ bool warp_symtri_eig(decltype(Cx::re)* d, decltype(Cx::re)* e, decltype(Cx::re)* cs, Cx* Z, int m,
                                       int ld, int lane) {
  using R = decltype(Cx::re);
  int h = m - 1, its = 0, total = 0;
  while (h > 0) {
    const int l = symtri_split(d, e, h, lane);
    __syncwarp();
    if (l > 0 && lane == 0) e[l - 1] = 0;
    __syncwarp();
    if (l == h) {
      --h;
      its = 0;
      continue;
    }
    if (++total > 30 * m) return false;
    if (lane == 0) {
      // Wilkinson shift: the eigenvalue of the trailing 2 x 2 nearer d[h];
      // every tenth step of a window an exceptional shift d[h] + |e[h-1]|
      const R a = d[h - 1], c = d[h], b = e[h - 1];
      const R del = R(0.5) * (a - c);
      const R den = del + (del >= 0 ? R(1) : R(-1)) * sqrt_t(del * del + b * b);
      R mu = den != 0 ? c - b * b / den : c;
      if (its > 0 && its % 10 == 0) mu = c + abs_t(b);
      symtri_step(d, e, cs, l, h, mu);
    }
    __syncwarp();
    symtri_apply_z(Z, cs, m, ld, l, h, lane);
    __syncwarp();
    ++its;
  }
  return true;
}

// Eigenvectors y_q = Z u_q (q < nvec) of the upper triangular T for the
// diagonal entries ord[q]: u by back substitution, one lane per eigenvector
// (columns of U in the scratch, stride min(32, nvec)), then Y = Z U one
// lane per row.  The back substitution divides through |den|^2 (one real
// reciprocal per step; T is prescaled, so |den|^2 >= small^2 stays in
// range).  warp_backsub: one warp, the U columns of eigenvectors
// q0 .. q0 + 31.
template <typename Cx>
static __device__ void warp_backsub(const Cx* T, int m, int ld, const int* ord, int nvec, int q0, double small_d,
                                    Cx* U, int lane) {
  using R = decltype(Cx::re);
  const R small = (R)small_d, small2 = small * small;
  const Cx zero = {0, 0};
  const int W = nvec < 32 ? nvec : 32;
  const int q = q0 + lane;
  const bool act = lane < W && q < nvec;
  const int idx = act ? ord[q] : 0;
  const Cx lam = TT_(idx, idx);
  if (lane < W)
    for (int i = 0; i < m; ++i) U[i * W + lane] = (act && i == idx) ? Cx{1, 0} : zero;
  for (int i = m - 2; i >= 0; --i) {
    Cx a0 = zero, a1 = zero;
    if (lane < W) {
      int j = i + 1;
      for (; j + 1 < m; j += 2) {
        a0 = cfma(TT_(i, j), U[j * W + lane], a0);
        a1 = cfma(TT_(i, j + 1), U[(j + 1) * W + lane], a1);
      }
      if (j < m) a0 = cfma(TT_(i, j), U[j * W + lane], a0);
    }
    if (act && i < idx) {
      Cx den = TT_(i, i) - lam;
      R d2 = abs2(den);
      if (d2 < small2) {
        den = Cx{small, 0};
        d2 = small2;
      }
      const Cx ui = (-R(1) / d2) * ((a0 + a1) * conj(den));
      U[i * W + lane] = ui;
      if (cabs1(ui) > HessK<R>::big)  // rescale this column to avoid overflow
        for (int j = i; j <= idx; ++j) U[j * W + lane] = HessK<R>::unbig * U[j * W + lane];
    }
  }
}

// Y[:, q] = Z U[:, q - q0] normalised, and the estimates beta |y_q[m-1]| /
// (scale ||y_q||), for the eigenvectors q0 + c with c < nq in this warp's
// share: for m <= 32, chunks of eight columns c0 = 8 (part + nparts t), one
// lane per row, their norms summed by interleaved butterflies.  Returns the
// largest estimate over q < k of the share.
template <typename Cx>
static __device__ double warp_zu(const Cx* Z, int m, int ld, const Cx* U, int W, int q0, int nq, int k, double beta,
                                 double scale, cplx* Y, double* est, int part, int nparts, int lane) {
  using R = decltype(Cx::re);
  const Cx zero = {0, 0};
  double maxest = 0;
  if (m <= 32) {
    constexpr int CH = 8;
    const bool rin = lane < m;
    for (int c0 = CH * part; c0 < nq; c0 += CH * nparts) {
      Cx y[CH];
#pragma unroll
      for (int c = 0; c < CH; ++c) y[c] = zero;
      for (int j = 0; j < m; ++j) {
        const Cx z = rin ? ZZ_(lane, j) : zero;
#pragma unroll
        for (int c = 0; c < CH; ++c) y[c] = cfma(z, U[j * W + (c0 + c < nq ? c0 + c : c0)], y[c]);
      }
      R n2[CH];
      Cx yl[CH];
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        n2[c] = abs2(y[c]);
        yl[c] = shfl_c(y[c], m - 1);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < CH; ++c) n2[c] += __shfl_xor_sync(0xffffffffu, n2[c], o);
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        const int qq = q0 + c0 + c;
        if (c0 + c < nq) {
          const R nrm = sqrt_t(n2[c]);
          const R inv = nrm > 0 ? R(1) / nrm : R(0);
          if (rin) Y[(long)qq * m + lane] = cx_to(inv * y[c]);
          const double e = beta * (double)sqrt_t(abs2(yl[c])) * (double)inv / scale;
          if (lane == 0) est[qq] = e;
          if (qq < k) maxest = fmax(maxest, e);
        }
      }
    }
    return maxest;
  }
  for (int c = part; c < nq; c += nparts) {
    const int qq = q0 + c;
    Cx yv[kMaxM / 32];
    R nrm = 0;
    Cx ylast = zero;
#pragma unroll
    for (int t = 0; t < kMaxM / 32; ++t) {
      const int r = lane + 32 * t;
      yv[t] = zero;
      if (r < m) {
        Cx s0 = zero, s1 = zero;
        int j = 0;
        for (; j + 1 < m; j += 2) {
          s0 = cfma(ZZ_(r, j), U[j * W + c], s0);
          s1 = cfma(ZZ_(r, j + 1), U[(j + 1) * W + c], s1);
        }
        if (j < m) s0 = cfma(ZZ_(r, j), U[j * W + c], s0);
        yv[t] = s0 + s1;
        nrm += abs2(yv[t]);
        if (r == m - 1) ylast = yv[t];
      }
    }
    nrm = sqrt(warp_sum_t(nrm));
    ylast.re = warp_sum_t(ylast.re);
    ylast.im = warp_sum_t(ylast.im);
    const R inv = nrm > 0 ? R(1) / nrm : R(0);
#pragma unroll
    for (int t = 0; t < kMaxM / 32; ++t) {
      const int r = lane + 32 * t;
      if (r < m) Y[(long)qq * m + r] = cx_to(inv * yv[t]);
    }
    const double e = beta * (double)cabs_(ylast) * (double)inv / scale;
    if (lane == 0) est[qq] = e;
    if (qq < k) maxest = fmax(maxest, e);
  }
  return maxest;
}

// Shared scratch of the multi-warp (NW > 1) hess_core beyond its workspaces.
template <typename Cx, int NW>
struct HessShared {
  Cx v[32];
  Cx part[2 * NW * 32];
  decltype(Cx::re) f;
  double mx[NW];
  double scale;
  int ok;
};

// The body of k_hess on NW warps (tid = 0 .. 32 NW - 1 of the calling
// threads), with its workspaces passed in: T, Z (leading dimension
// hess_ld(m), m columns each), u (m), key (m), ord (m), scratch
// (hess_scratch_cplx(m)); hs (NW > 1 only): shared scratch.  Callable from
// any kernel by one full warp (NW = 1) or by NW full warps when m <= 32; the
// outputs in `a` may point to shared or global memory.  With NW > 1 the
// Householder reduction and the product Y = Z U run on all warps, the Schur
// sweeps, the sort and the back substitutions on warp 0; the other warps
// return before the exact shifts.
template <typename Cx, int NW = 1>
static __device__ void hess_core(const HessArgs& a, Cx* T, Cx* Z, Cx* u, double* key, int* ord, Cx* scratch,
                                 int tid, HessShared<Cx, NW>* hs = nullptr) {
  using R = decltype(Cx::re);
  constexpr int nthr = NW * 32;
  const int lane = tid & 31, warp = tid >> 5;
  const int m = a.m, k = a.k, ld = hess_ld(m);
  const long mm = (long)m * m;
  DevState* st = a.st;
  Cx* rot = scratch;           // 2 m
  Cx* U = scratch + 2 * m + 2; // m x 32

  // T = sig H with sig a power of two that puts the largest |re| or |im| of
  // H in [1, 2): exact, and the Schur sweeps' rotations and shifts then need
  // no overflow / underflow branches (givens_s, csqrt_s).  Values leave
  // hess_core unscaled (times isig).  (Every warp finds the same maximum.)
  double mx = 0;
  for (long i = lane; i < mm; i += 32) mx = fmax(mx, fmax(fabs(a.Hin[i].re), fabs(a.Hin[i].im)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  int ex = 0;
  if (mx > 0 && mx <= 1.7e308) frexp(mx, &ex);  // mx = f 2^ex, f in [0.5, 1)
  ex = ex > 1000 ? 1000 : (ex < -1000 ? -1000 : ex);
  const double sig = ldexp(1.0, 1 - ex), isig = ldexp(1.0, ex - 1);
  for (long i = tid; i < mm; i += nthr) {
    const int r = (int)(i % m), c = (int)(i / m);
    TT_(r, c) = cx_from<Cx>(sig * a.Hin[i]);
    ZZ_(r, c) = (r == c) ? Cx{1, 0} : Cx{0, 0};
  }
  if constexpr (NW > 1) {
    hess_bar(nthr);
    if (a.dense) block_hessenberg32<Cx, NW>(T, Z, hs->v, hs->part, &hs->f, m, ld, warp, lane);
  } else {
    __syncwarp();
    if (a.dense) warp_hessenberg(T, Z, u, m, ld, lane);
  }
  const int nvec = a.nvec > k ? (a.nvec < m ? a.nvec : m) : k;
  const int W = nvec < 32 ? nvec : 32;
  double scale = 0, small = 0;
  const double beta = a.use_beta ? sqrt(st->fnorm2) : a.beta;
  // Hermitian Hessenberg input: the tridiagonal path (d, e in the
  // eigenvector scratch, the rotations in rot)
  R* sd = reinterpret_cast<R*>(U);
  R* se = sd + m;
  R* scs = reinterpret_cast<R*>(rot);
  bool sym = false;
  if (warp == 0) {
    sym = !a.dense && a.tol > 0 && warp_is_hermitian(T, m, ld, 0.1 * a.tol, lane);
    if (sym && lane == 0) st->symtri += 1;
    bool ok;
    if (sym) {
      symtri_load(T, Z, m, ld, sd, se, lane);
      ok = warp_symtri_eig(sd, se, scs, Z, m, ld, lane);
      if (ok) {
        for (int i = lane; i + 1 < m; i += 32) se[i] = 0;
        symtri_store(T, m, ld, sd, se, lane);
      }
    } else {
      ok = warp_schur(T, Z, m, ld, rot, lane);
    }
    if (!ok && lane == 0) {
      st->status |= 2;
      st->converged = 0;
    }
    if constexpr (NW > 1) {
      if (lane == 0) hs->ok = ok;
    }
    if (ok) {
      // sort order of diag(T)
      for (int i = lane; i < m; i += 32) {
        double kv = sort_key(cx_to(TT_(i, i)), a.which);
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
        a.ritz[q] = isig * cx_to(TT_(ord[q], ord[q]));
      }
      // max |theta| over the wanted set, unscaled
      for (int q = 0; q < k; ++q) scale = fmax(scale, (double)cabs_(TT_(ord[q], ord[q])));
      scale *= isig;
      if (scale == 0) scale = 1;
      double tnorm = 0;
      for (int i = lane; i < m; i += 32) tnorm = fmax(tnorm, (double)cabs_(TT_(i, i)));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tnorm = fmax(tnorm, __shfl_xor_sync(0xffffffffu, tnorm, o));
      small = (double)HessK<R>::eps * (tnorm > 0 ? tnorm : 1.0);
      warp_backsub(T, m, ld, ord, nvec, 0, small, U, lane);
      if constexpr (NW > 1) {
        if (lane == 0) hs->scale = scale;
      }
    }
    __syncwarp();
  }
  double maxest = 0;
  if constexpr (NW > 1) {
    // eigenvectors of the first nvec Ritz values (the wanted k and optional
    // guard vectors; nvec <= m <= 32) on all warps
    hess_bar(nthr);
    if (!hs->ok) return;
    scale = hs->scale;
    const double me = warp_zu(Z, m, ld, U, W, 0, nvec, k, beta, scale, a.Y, a.est, warp, NW, lane);
    if (lane == 0) hs->mx[warp] = me;
    hess_bar(nthr);
    if (warp != 0) return;
    for (int w = 0; w < NW; ++w) maxest = fmax(maxest, hs->mx[w]);
  } else {
    if (scale == 0) return;  // the Schur sweeps ran out (status set)
    for (int q0 = 0; q0 < nvec; q0 += 32) {
      if (q0 > 0) {
        warp_backsub(T, m, ld, ord, nvec, q0, small, U, lane);
        __syncwarp();
      }
      const int nq = (nvec - q0) < W ? (nvec - q0) : W;
      maxest = fmax(maxest, warp_zu(Z, m, ld, U, W, q0, nq, k, beta, scale, a.Y, a.est, 0, 1, lane));
      __syncwarp();
    }
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
    const int r = (int)(i % m), c = (int)(i / m);
    TT_(r, c) = cx_from<Cx>(sig * a.Hin[i]);
    ZZ_(r, c) = (r == c) ? Cx{1, 0} : Cx{0, 0};
  }
  __syncwarp();
  if (sym) {  // the same exact shifts as implicit symmetric tridiagonal steps
    symtri_load(T, Z, m, ld, sd, se, lane);
    for (int q = k; q < m; ++q) {
      const R mu = u[q].re;
      int hb = m - 1;
      while (hb > 0) {
        const int l = symtri_split(sd, se, hb, lane);
        __syncwarp();
        if (l > 0 && lane == 0) se[l - 1] = 0;
        __syncwarp();
        if (l < hb) {
          if (lane == 0) symtri_step(sd, se, scs, l, hb, mu);
          __syncwarp();
          symtri_apply_z(Z, scs, m, ld, l, hb, lane);
          __syncwarp();
        }
        hb = l - 1;
      }
    }
    symtri_store(T, m, ld, sd, se, lane);
  } else {
    for (int q = k; q < m; ++q) {
      Cx mu = u[q];
      if (a.real_shifts) mu.im = 0;
      int hb = m - 1;
      while (hb > 0) {
        const int l = find_split(T, ld, hb, lane);
        if (l > 0 && lane == 0) TT_(l, l - 1) = Cx{0, 0};
        __syncwarp();
        if (l < hb) warp_sweep(T, Z, m, ld, l, hb, mu, rot, lane);
        hb = l - 1;
      }
    }
  }
  __syncwarp();
  if (lane == 0) {
    st->beta_hat = isig * cx_to(TT_(k, k - 1));
    st->sigma = cx_to(ZZ_(m - 1, k - 1));
  }
  for (long i = lane; i < mm; i += 32) {
    const int r = (int)(i % m), c = (int)(i / m);
    a.Hout[i] = (r < k && c < k) ? isig * cx_to(TT_(r, c)) : cplx{0, 0};
    a.Qout[i] = cx_to(ZZ_(r, c));
  }
}

// warps of k_hess / k_hess_f32 for m <= 32 (one warp above)
constexpr int kHessWarps = 4;
__host__ __device__ inline int hess_threads(int m) { return m <= 32 ? 32 * kHessWarps : 32; }

// dynamic shared memory (or a.gws): T, Z, scratch of the working type Cx;
// launched with hess_threads(m) threads
template <typename Cx>
static __device__ void hess_kernel_body(const HessArgs& a, unsigned char* dyn) {
  __shared__ Cx u[kMaxM];
  __shared__ double key[kMaxM];
  __shared__ int ord[kMaxM];
  __shared__ HessShared<Cx, kHessWarps> hs;
  Cx* T = a.gws ? reinterpret_cast<Cx*>(a.gws) : reinterpret_cast<Cx*>(dyn);
  const size_t tz = (size_t)hess_ld(a.m) * a.m;
  if (blockDim.x == 32 * kHessWarps && a.m <= 32)
    hess_core<Cx, kHessWarps>(a, T, T + tz, u, key, ord, T + 2 * tz, threadIdx.x, &hs);
  else if (threadIdx.x < 32)
    hess_core<Cx, 1>(a, T, T + tz, u, key, ord, T + 2 * tz, threadIdx.x);
}

// FP64 working arithmetic (the restart loop and the refinement)
static __global__ void __launch_bounds__(32 * kHessWarps) k_hess(HessArgs a) {
  extern __shared__ __align__(16) unsigned char hess_dyn[];
  asm volatile("griddepcontrol.wait;" ::: "memory");  // dependent launch
  if (a.skip && *(volatile const int*)a.skip) return;
  hess_kernel_body<cplx>(a, hess_dyn);
}

// FP32 working arithmetic, FP64 inputs and outputs: the Rayleigh-Ritz checks
// of the FP32-class phase (whose Ritz vectors are FP32-accurate at best);
// dynamic shared memory hess_ws_cplx(m) * sizeof(cplxf)
static __global__ void __launch_bounds__(32 * kHessWarps) k_hess_f32(HessArgs a) {
  extern __shared__ __align__(16) unsigned char hess_dyn[];
  asm volatile("griddepcontrol.wait;" ::: "memory");  // dependent launch
  hess_kernel_body<cplxf>(a, hess_dyn);
}

#undef TT_
#undef ZZ_

// Eigenpairs of a nearly upper-triangular T (m x m complex, column-major,
// m <= 32): the Rayleigh quotient of an orthonormalised basis of Ritz vectors
// ordered like their values, whose strictly lower part is of the size of the
// Ritz vectors' errors.  k_eig_near_tri: one CTA of one warp per pair q
// (grid m, each pair on its own SM): Rayleigh quotient iteration from v =
// e_q, sigma = T(q,q) (LU with partial pivoting of T - sigma I, a zero pivot
// replaced by eps ||T||_F; v <- (T - sigma I)^-1 v normalised; sigma <- v^H
// T v), at most kNtIters steps, until ||T v - sigma v|| <= 16 eps ||T||_F;
// the pair goes to the scratch (V column q at V + q m, th[q]) and ok[0] is
// cleared when its residual is above 64 eps ||T||_F.  k_eig_near_tri_finish
// (one warp, after it): accepted when ok[0] is set and the values are
// pairwise apart by more than 1e-9 max |theta|; then ritz / Y / order are
// written in the ArnUtils order of `which` (as k_hess writes them, Y column
// q at Y + q m, unit 2-norm) and *delivered = 1; otherwise *delivered = 0
// and nothing else is written (k_hess follows with skip = delivered).
// ok[0] is set again for the next call (it must hold 1 before the first).
constexpr int kNtIters = 4;
__host__ __device__ inline int nt_ld(int m) { return m + 1; }
// dynamic shared memory of k_eig_near_tri: T, M (m x LD), x, t, the pivots'
// reciprocals (m each), pivot rows
__host__ __device__ inline size_t nt_smem_bytes(int m) {
  return sizeof(cplx) * (2 * (size_t)m * nt_ld(m) + 3 * (size_t)m) + sizeof(int) * (size_t)m;
}

static __global__ void __launch_bounds__(32) k_eig_near_tri(const cplx* __restrict__ Tin, int m, cplx* V, cplx* th,
                                                            int* ok) {
  extern __shared__ __align__(16) unsigned char nt_dyn[];
  asm volatile("griddepcontrol.wait;" ::: "memory");  // dependent launch
  const int LD = nt_ld(m);
  cplx* T = reinterpret_cast<cplx*>(nt_dyn);  // m x LD
  cplx* M = T + (size_t)m * LD;               // m x LD
  cplx* x = M + (size_t)m * LD;               // m
  cplx* t = x + m;                            // m
  cplx* dinv = t + m;                         // m: reciprocals of U's diagonal
  int* pv = reinterpret_cast<int*>(dinv + m); // m
  const int lane = threadIdx.x, q = blockIdx.x;
  if (m < 1 || m > 32 || q >= m) return;
  // T scaled by the power of two that puts its largest |re| or |im| in
  // [1, 2) (exact): the pivots' squared moduli below stay in range; the
  // value is unscaled on output
  double mx = 0;
  for (int e = lane; e < m * m; e += 32) mx = fmax(mx, fmax(fabs(Tin[e].re), fabs(Tin[e].im)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  int ex = 0;
  if (mx > 0 && mx <= 1.7e308) frexp(mx, &ex);
  ex = ex > 1000 ? 1000 : (ex < -1000 ? -1000 : ex);
  const double sig = ldexp(1.0, 1 - ex), isig = ldexp(1.0, ex - 1);
  for (int e = lane; e < m * m; e += 32) T[(e % m) + (e / m) * LD] = sig * Tin[e];
  __syncwarp();
  double fro = 0;
  for (int e = lane; e < m * m; e += 32) fro += abs2(T[(e % m) + (e / m) * LD]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, o);
  fro = sqrt(fro);
  const double eps = 2.220446049250313e-16;
  const double tiny = eps * (fro > 0 ? fro : 1.0);
  {
    cplx sigma = T[q + q * LD], thq = {0, 0};
    double rq = 1e300;
    for (int i = lane; i < m; i += 32) x[i] = cplx{i == q ? 1.0 : 0.0, 0.0};
    __syncwarp();
    for (int itr = 0; itr < kNtIters && !(rq <= 16 * eps * fro); ++itr) {
      for (int e = lane; e < m * m; e += 32) {
        const int r = e % m, c = e / m;
        M[r + c * LD] = T[r + c * LD] - (r == c ? sigma : cplx{0, 0});
      }
      __syncwarp();
      // LU with partial pivoting, lane = column
      for (int k = 0; k < m; ++k) {
        double best = -1;
        int bi = k;
        for (int i = k + lane; i < m; i += 32) {
          const double v = abs2(M[i + k * LD]);
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
        if (lane == 0) pv[k] = bi;
        for (int c = lane; c < m; c += 32) {  // swap rows k and bi
          const cplx tmp = M[k + c * LD];
          M[k + c * LD] = M[bi + c * LD];
          M[bi + c * LD] = tmp;
        }
        __syncwarp();
        // the pivot (a zero one replaced by tiny) and its reciprocal
        // conj(p) / |p|^2, kept for the back substitution
        cplx pk = M[k + k * LD];
        double p2 = abs2(pk);
        if (!(p2 >= tiny * tiny)) {
          pk = cplx{tiny, 0};
          p2 = tiny * tiny;
        }
        const cplx inv = (1.0 / p2) * conj(pk);
        __syncwarp();
        if (lane == 0) {
          M[k + k * LD] = pk;
          dinv[k] = inv;
        }
        for (int i = k + 1 + lane; i < m; i += 32) M[i + k * LD] = M[i + k * LD] * inv;  // multipliers
        __syncwarp();
        for (int c = k + 1 + lane; c < m; c += 32) {
          const cplx ukc = M[k + c * LD];
          for (int i = k + 1; i < m; ++i) M[i + c * LD] = M[i + c * LD] - M[i + k * LD] * ukc;
        }
        __syncwarp();
      }
      // x <- (T - sigma I)^-1 x, normalised: lane i holds x_i; the row
      // swaps, then L y = P b and U x = y column by column (one shuffle of
      // the finished entry per column)
      cplx xv = lane < m ? x[lane] : cplx{0, 0};
      for (int k = 0; k < m; ++k) {
        const int r = pv[k];
        const cplx xk = shfl_c(xv, k), xr = shfl_c(xv, r);
        if (lane == k) xv = xr;
        else if (lane == r) xv = xk;
      }
      for (int j = 0; j + 1 < m; ++j) {
        const cplx xj = shfl_c(xv, j);
        if (lane > j && lane < m) xv = xv - M[lane + j * LD] * xj;
      }
      for (int i = m - 1; i >= 0; --i) {
        if (lane == i) xv = xv * dinv[i];
        const cplx xi = shfl_c(xv, i);
        if (lane < i) xv = xv - M[lane + i * LD] * xi;
      }
      double nrm = abs2(xv);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
      nrm = sqrt(nrm);
      const double sc = nrm > 0 ? 1.0 / nrm : 0.0;
      if (lane < m) x[lane] = sc * xv;
      __syncwarp();
      // Rayleigh quotient (the next shift) and residual ||T x - theta x||
      for (int i = lane; i < m; i += 32) {
        cplx acc = {0, 0};
        for (int j = 0; j < m; ++j) acc = acc + T[i + j * LD] * x[j];
        t[i] = acc;
      }
      __syncwarp();
      thq = cplx{0, 0};
      for (int i = lane; i < m; i += 32) thq = thq + conj(x[i]) * t[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        thq.re += __shfl_xor_sync(0xffffffffu, thq.re, o);
        thq.im += __shfl_xor_sync(0xffffffffu, thq.im, o);
      }
      double r2 = 0;
      for (int i = lane; i < m; i += 32) r2 += abs2(t[i] - thq * x[i]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
      rq = sqrt(r2);
      sigma = thq;
    }
    for (int i = lane; i < m; i += 32) V[i + (size_t)q * m] = x[i];
    if (lane == 0) {
      th[q] = isig * thq;
      if (!(rq <= 64 * eps * fro)) ok[0] = 0;
    }
  }
}

static __global__ void __launch_bounds__(32) k_eig_near_tri_finish(int m, int which, const cplx* __restrict__ V,
                                                                   const cplx* __restrict__ th, int* ok, cplx* ritz,
                                                                   cplx* Y, int* order, int* delivered) {
  __shared__ double key[32];
  __shared__ int ord[32];
  asm volatile("griddepcontrol.wait;" ::: "memory");  // dependent launch
  const int lane = threadIdx.x;
  if (m < 1 || m > 32) return;
  // distinct values, then the ArnUtils order
  double tmax = 0;
  for (int q = lane; q < m; q += 32) tmax = fmax(tmax, cabs_(th[q]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) tmax = fmax(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
  int bad = 0;
  for (int e = lane; e < m * m; e += 32) {
    const int q = e % m, r = e / m;
    if (q < r && !(cabs_(th[q] - th[r]) > 1e-9 * tmax)) bad = 1;
  }
  bad = __any_sync(0xffffffffu, bad);
  for (int i = lane; i < m; i += 32) {
    const double kv = sort_key(th[i], which);
    key[i] = (kv != kv) ? INFINITY : kv;
  }
  __syncwarp();
  for (int i = lane; i < m; i += 32) {
    int r = 0;
    for (int j = 0; j < m; ++j) r += (key[j] < key[i]) || (key[j] == key[i] && j < i);
    ord[r] = i;
  }
  __syncwarp();
  const int good = ok[0] && !bad;
  __syncwarp();
  if (lane == 0) {
    *delivered = good;
    ok[0] = 1;
  }
  if (!good) return;
  for (int q = lane; q < m; q += 32) {
    ritz[q] = th[ord[q]];
    order[q] = ord[q];
  }
  for (int e = lane; e < m * m; e += 32) {
    const int i = e % m, q = e / m;
    Y[i + (size_t)q * m] = V[i + (size_t)ord[q] * m];
  }
}

}  // namespace oapb
