// Operator surface of oap::CuProceduresApi (oapMatrixCuda/CuProceduresApi.h)
// on device FP64 planes in the reference layout.
//
// Each entry validates the handles on the host (dims, present planes) and
// launches one kernel (two for the reductions).  Unlike the reference:
//  - element-wise kernels index the whole grid, so add / substract are
//    correct for any size (CuAdditionProcedures.h:33-53 indexes threadIdx
//    only and is wrong past one block);
//  - multiplyConstant is a complex scale (the reference scales each plane by
//    its own part, CuMultiplicationProcedures.h:56-69);
//  - reductions finish on the device (two-stage, deterministic order) and
//    return one value, instead of copying per-block partials to the host.
#include <stdio.h>

#include "common.cuh"
#include "matvec.cuh"

namespace oapb {

static inline bool ok_mat(const oapb_mat* m) {
  return m && m->columns > 0 && m->rows > 0 && m->dtype == OAPB_F64 && (m->re || m->im);
}
static inline long numel(const oapb_mat* m) { return (long)m->columns * m->rows; }
static inline const double* RE(const oapb_mat* m) { return (const double*)m->re; }
static inline const double* IM(const oapb_mat* m) { return (const double*)m->im; }
static inline double* WRE(const oapb_mat* m) { return (double*)m->re; }
static inline double* WIM(const oapb_mat* m) { return (double*)m->im; }

__device__ __forceinline__ cplx ldc(const double* re, const double* im, long i) {
  return {re ? re[i] : 0.0, im ? im[i] : 0.0};
}
__device__ __forceinline__ void stc(double* re, double* im, long i, cplx v) {
  if (re) re[i] = v.re;
  if (im) im[i] = v.im;
}

// ------------------------------------------------------------ GEMM (FP64) --
// C (M x N) = A (M x K) B (K x N), all row-major, complex via optional planes.
constexpr int GT = 16;
__global__ void k_gemm(const double* __restrict__ are, const double* __restrict__ aim,
                       const double* __restrict__ bre, const double* __restrict__ bim,
                       double* cre, double* cim, int M, int N, int K) {
  __shared__ cplx As[GT][GT + 1];
  __shared__ cplx Bs[GT][GT + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int row = blockIdx.y * GT + ty, col = blockIdx.x * GT + tx;
  cplx acc = {0, 0};
  for (int k0 = 0; k0 < K; k0 += GT) {
    int ka = k0 + tx, kb = k0 + ty;
    As[ty][tx] = (row < M && ka < K) ? ldc(are, aim, (long)row * K + ka) : cplx{0, 0};
    Bs[ty][tx] = (kb < K && col < N) ? ldc(bre, bim, (long)kb * N + col) : cplx{0, 0};
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GT; ++kk) acc = acc + As[ty][kk] * Bs[kk][tx];
    __syncthreads();
  }
  if (row < M && col < N) stc(cre, cim, (long)row * N + col, acc);
}

// ------------------------------------------------------------- transpose --
constexpr int TT = 32;
__global__ void k_transpose(const double* __restrict__ ire, const double* __restrict__ iim,
                            double* ore, double* oim, int cols, int rows, int conjugate) {
  __shared__ cplx t[TT][TT + 1];
  int x = blockIdx.x * TT + threadIdx.x, y0 = blockIdx.y * TT;
  for (int j = threadIdx.y; j < TT; j += blockDim.y) {
    int y = y0 + j;
    if (x < cols && y < rows) t[j][threadIdx.x] = ldc(ire, iim, (long)y * cols + x);
  }
  __syncthreads();
  // out is rows x cols transposed: out[x][y], out has `rows` columns
  int ox = y0 + threadIdx.x;
  for (int j = threadIdx.y; j < TT; j += blockDim.y) {
    int oy = blockIdx.x * TT + j;
    if (ox < rows && oy < cols) {
      cplx v = t[threadIdx.x][j];
      if (conjugate) v.im = -v.im;
      stc(ore, oim, (long)oy * rows + ox, v);
    }
  }
}

// ------------------------------------------------------------ reductions --
constexpr int RB = 256;
constexpr int RMaxBlocks = 1024;
// mode 0: partial sum |x|^2 -> part[b].x; mode 1: sum re, sum im -> part[b]
__global__ void k_reduce_partial(const double* __restrict__ re, const double* __restrict__ im,
                                 long len, int mode, double2* part) {
  double a = 0, b = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x) {
    double r = re ? re[i] : 0.0, m = im ? im[i] : 0.0;
    if (mode == 0) a += r * r + m * m;
    else { a += r; b += m; }
  }
  __shared__ double sa[RB / 32], sb[RB / 32];
  a = warp_sum(a);
  b = warp_sum(b);
  if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = a; sb[threadIdx.x >> 5] = b; }
  __syncthreads();
  if (threadIdx.x < 32) {
    a = threadIdx.x < RB / 32 ? sa[threadIdx.x] : 0;
    b = threadIdx.x < RB / 32 ? sb[threadIdx.x] : 0;
    a = warp_sum(a);
    b = warp_sum(b);
    if (threadIdx.x == 0) part[blockIdx.x] = make_double2(a, b);
  }
}
__global__ void k_reduce_final(const double2* part, int nparts, int mode, double2* out) {
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) { a += part[i].x; b += part[i].y; }
  __shared__ double sa[RB / 32], sb[RB / 32];
  a = warp_sum(a);
  b = warp_sum(b);
  if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = a; sb[threadIdx.x >> 5] = b; }
  __syncthreads();
  if (threadIdx.x < 32) {
    a = threadIdx.x < RB / 32 ? sa[threadIdx.x] : 0;
    b = threadIdx.x < RB / 32 ? sb[threadIdx.x] : 0;
    a = warp_sum(a);
    b = warp_sum(b);
    if (threadIdx.x == 0) *out = make_double2(mode == 0 ? sqrt(a) : a, b);
  }
}

// ------------------------------------------------------------ element-wise --
// op 0: out = a + b; 1: out = a - b; 2: out = a * s (complex s);
// 3: identity; 4: diagonal s; 5: zero
__global__ void k_elementwise(int op, const double* __restrict__ are, const double* __restrict__ aim,
                              const double* __restrict__ bre, const double* __restrict__ bim,
                              double* ore, double* oim, int cols, long len, double sre, double sim) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x) {
    cplx v;
    switch (op) {
      case 0: v = ldc(are, aim, i) + ldc(bre, bim, i); break;
      case 1: v = ldc(are, aim, i) - ldc(bre, bim, i); break;
      case 2: v = ldc(are, aim, i) * cplx{sre, sim}; break;
      case 3: v = (i / cols == i % cols) ? cplx{1, 0} : cplx{0, 0}; break;
      case 4: v = (i / cols == i % cols) ? cplx{sre, sim} : cplx{0, 0}; break;
      default: v = {0, 0}; break;
    }
    stc(ore, oim, i, v);
  }
}

__global__ void k_tensor(const double* __restrict__ p0re, const double* __restrict__ p0im, int c0,
                         const double* __restrict__ p1re, const double* __restrict__ p1im, int c1, int r1,
                         double* ore, double* oim, int oc, long len) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x) {
    long y = i / oc, x = i % oc;
    cplx v0 = ldc(p0re, p0im, (y / r1) * c0 + x / c1);
    cplx v1 = ldc(p1re, p1im, (y % r1) * c1 + x % c1);
    stc(ore, oim, i, v0 * v1);
  }
}

// V[r][column] = v[r] (dir 0) or v[r] = V[r][column] (dir 1), r < length
__global__ void k_vector_copy(double* Vre, double* Vim, int Vcols, int column, double* vre,
                              double* vim, int vcols, int length, int dir) {
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < length; r += (long)gridDim.x * blockDim.x) {
    long iV = r * Vcols + column, iv = r * vcols;
    if (dir == 0) {
      if (Vre && vre) Vre[iV] = vre[iv];
      if (Vim && vim) Vim[iV] = vim[iv];
    } else {
      if (Vre && vre) vre[iv] = Vre[iV];
      if (Vim && vim) vim[iv] = Vim[iV];
    }
  }
}

__global__ void k_is_upper(const double* __restrict__ re, const double* __restrict__ im, int n,
                           double tol, int* out) {
  int bad = 0;
  for (int c = threadIdx.x; c + 1 < n; c += blockDim.x) {
    long i = (long)(c + 1) * n + c;
    if (re && !(-tol < re[i] && re[i] < tol)) bad = 1;
    if (im && !(-tol < im[i] && im[i] < tol)) bad = 1;
  }
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) *out = !bad;
}

// --------------------------------------------------------- Givens QR (CTA) --
// One CTA; R and Q (n x n complex, row-major) live in `ws` (shared memory
// when they fit, else global scratch).  Rotation order of the reference:
// column fa, rows fb = n-1 .. fa+1 (CuQRProcedures_GR.h:123-140); a rotation
// is skipped when the current R[fb][fa] is exactly zero.
__device__ void qr_givens_cta(cplx* R, cplx* Q, int n) {
  __shared__ cplx pq[2];
  for (int fa = 0; fa < n; ++fa) {
    for (int fb = n - 1; fb > fa; --fb) {
      __syncthreads();
      cplx y = R[(long)fb * n + fa];
      if (y.re == 0 && y.im == 0) continue;  // uniform: all threads read the same value
      if (threadIdx.x == 0) {
        cplx p, q;
        givens(R[(long)fa * n + fa], y, p, q);
        pq[0] = p;
        pq[1] = q;
      }
      __syncthreads();
      const cplx p = pq[0], q = pq[1];
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        cplx a = R[(long)fa * n + j], b = R[(long)fb * n + j];
        R[(long)fa * n + j] = p * a + q * b;
        R[(long)fb * n + j] = (-conj(q)) * a + conj(p) * b;
        cplx u = Q[(long)j * n + fa], w = Q[(long)j * n + fb];
        Q[(long)j * n + fa] = u * conj(p) + w * conj(q);
        Q[(long)j * n + fb] = (-u) * q + w * p;
      }
      __syncthreads();
      if (threadIdx.x == 0) R[(long)fb * n + fa] = {0, 0};
    }
  }
  __syncthreads();
}

__global__ void k_qr_givens(const double* __restrict__ are, const double* __restrict__ aim,
                            double* qre, double* qim, double* rre, double* rim, int n, cplx* gws) {
  extern __shared__ cplx sws[];
  cplx* ws = gws ? gws : sws;
  cplx* R = ws;
  cplx* Q = ws + (long)n * n;
  for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) {
    R[i] = ldc(are, aim, i);
    Q[i] = (i / n == i % n) ? cplx{1, 0} : cplx{0, 0};
  }
  __syncthreads();
  qr_givens_cta(R, Q, n);
  for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) {
    stc(qre, qim, i, Q[i]);
    stc(rre, rim, i, R[i]);
  }
}

// Unshifted QR iteration (oapGenericArnoldiApi.h:268-296): H <- R Q,
// Qacc <- Q Qacc, until the first subdiagonal is within tol or `count`
// iterations.  ws holds H, R, Q, Qacc, tmp (5 n^2).
__global__ void k_calc_triangular_h(double* hre, double* him, double* qre, double* qim, int n,
                                    int count, double tol, cplx* gws, unsigned* iters) {
  extern __shared__ cplx sws[];
  cplx* ws = gws ? gws : sws;
  const long nn = (long)n * n;
  cplx *R = ws, *Q = ws + nn, *Qa = ws + 2 * nn, *Tm = ws + 3 * nn;
  __shared__ int done;
  for (long i = threadIdx.x; i < nn; i += blockDim.x) {
    R[i] = ldc(hre, him, i);
    Qa[i] = (i / n == i % n) ? cplx{1, 0} : cplx{0, 0};
  }
  __syncthreads();
  int it = 0;
  for (; it < count; ++it) {
    if (threadIdx.x == 0) {
      int up = 1;
      for (int c = 0; c + 1 < n; ++c) {
        cplx v = R[(long)(c + 1) * n + c];
        if (!(-tol < v.re && v.re < tol)) up = 0;
        if (him && !(-tol < v.im && v.im < tol)) up = 0;
      }
      done = up;
    }
    __syncthreads();
    if (done) break;
    for (long i = threadIdx.x; i < nn; i += blockDim.x) Q[i] = (i / n == i % n) ? cplx{1, 0} : cplx{0, 0};
    __syncthreads();
    qr_givens_cta(R, Q, n);   // R now triangular, H = Q R
    // H <- R Q  (into Tm), Qacc <- Q Qacc
    for (long i = threadIdx.x; i < nn; i += blockDim.x) {
      int r = i / n, c = i % n;
      cplx a = {0, 0}, b = {0, 0};
      for (int k = 0; k < n; ++k) {
        a = a + R[(long)r * n + k] * Q[(long)k * n + c];
        b = b + Q[(long)r * n + k] * Qa[(long)k * n + c];
      }
      Tm[i] = a;
      Tm[nn + i] = b;  // uses the slot after Tm (5th n^2)
    }
    __syncthreads();
    for (long i = threadIdx.x; i < nn; i += blockDim.x) {
      R[i] = Tm[i];
      Qa[i] = Tm[nn + i];
    }
    __syncthreads();
  }
  for (long i = threadIdx.x; i < nn; i += blockDim.x) {
    stc(hre, him, i, R[i]);
    stc(qre, qim, i, Qa[i]);
  }
  if (threadIdx.x == 0 && iters) *iters = it;
}

// Householder QR (real), CuQRProcedures_HT.h:63-131 restated in FP64.
__global__ void k_qr_householder(const double* __restrict__ a, double* q, double* r, int n, double* gws) {
  extern __shared__ double dws[];
  double* ws = gws ? gws : dws;
  double *R = ws, *Q = ws + (long)n * n, *v = ws + 2L * n * n;
  __shared__ double sh_s, sh_vv;
  for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) {
    R[i] = a[i];
    Q[i] = (i / n == i % n) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x == 0) {
      double s = 0;
      for (int i = k; i < n; ++i) s += R[(long)i * n + k] * R[(long)i * n + k];
      sh_s = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) v[i] = i < k ? 0.0 : R[(long)i * n + k];
    __syncthreads();
    if (threadIdx.x == 0) {
      double x = R[(long)k * n + k];
      v[k] += (x < 0 ? -1.0 : 1.0) * sqrt(sh_s);
      double vv = 0;
      for (int i = k; i < n; ++i) vv += v[i] * v[i];
      sh_vv = vv;
    }
    __syncthreads();
    const double vv = sh_vv;
    if (vv != 0) {
      for (int j = threadIdx.x; j < n; j += blockDim.x) {  // R <- P R, column j
        double d = 0;
        for (int i = k; i < n; ++i) d += v[i] * R[(long)i * n + j];
        d *= 2.0 / vv;
        for (int i = k; i < n; ++i) R[(long)i * n + j] -= d * v[i];
      }
      for (int i = threadIdx.x; i < n; i += blockDim.x) {  // Q <- Q P, row i
        double d = 0;
        for (int c = k; c < n; ++c) d += Q[(long)i * n + c] * v[c];
        d *= 2.0 / vv;
        for (int c = k; c < n; ++c) Q[(long)i * n + c] -= d * v[c];
      }
    }
    __syncthreads();
  }
  for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) {
    q[i] = Q[i];
    r[i] = R[i];
  }
}

static size_t g_smem_limit = 0;
static size_t smem_limit() {
  if (!g_smem_limit) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    g_smem_limit = v > 0 ? (size_t)v : 48 * 1024;
  }
  return g_smem_limit;
}

// Workspace of a one-CTA kernel: shared memory when it fits, else
// stream-ordered global scratch (freed after the launch on the same stream).
struct Scratch {
  void* g = nullptr;
  size_t shm = 0;
};
static int prep_ws(const void* kernel, size_t bytes, cudaStream_t s, Scratch& w) {
  if (bytes + 1024 <= smem_limit()) {
    w.shm = bytes;
    if (bytes > 48 * 1024)
      OAPB_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  } else {
    OAPB_CUDA_TRY(cudaMallocAsync(&w.g, bytes, s));
  }
  return OAPB_OK;
}
static int finish_ws(Scratch& w, cudaStream_t s) {
  cudaError_t e = cudaGetLastError();
  if (w.g) cudaFreeAsync(w.g, s);
  return e == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

}  // namespace oapb

using namespace oapb;

#define STREAM(s) ((cudaStream_t)(s))

extern "C" {

const char* oapb_status_string(int st) {
  switch (st) {
    case OAPB_OK: return "ok";
    case OAPB_ERR_ARG: return "invalid argument";
    case OAPB_ERR_CUDA: return "CUDA error";
    case OAPB_NOT_CONVERGED: return "not converged";
    case OAPB_ERR_TIMEOUT: return "device loop gave up";
    case OAPB_ERR_BOUNDS: return "device bounds check";
    case OAPB_ERR_CALLBACK: return "user callback failed";
    case OAPB_ERR_NOMEM: return "out of device memory";
    case OAPB_ERR_BREAKDOWN: return "Krylov breakdown";
    case OAPB_ERR_NONFINITE: return "non-finite value (NaN or infinity) in the solve";
  }
  return "unknown status";
}

int oapb_api_version(void) { return OAPB_API_VERSION; }

int oapb_dot_product(const oapb_mat* out, const oapb_mat* a, const oapb_mat* b, void* stream) {
  if (!ok_mat(out) || !ok_mat(a) || !ok_mat(b)) return OAPB_ERR_ARG;
  const int M = out->rows, N = out->columns, K = a->columns;
  if (a->rows != (uint32_t)M || b->columns != (uint32_t)N || b->rows != (uint32_t)K) return OAPB_ERR_ARG;
  cudaStream_t s = STREAM(stream);
  // matrix-vector product with full planes: the coalesced GEMV
  const bool ac = a->im != nullptr, bc = b->im != nullptr, oc = out->im != nullptr;
  if (N == 1 && a->re && b->re && out->re && ac == bc && ac == oc && M >= 256) {
    OAPB_CUDA_TRY(launch_matvec<double>(RE(a), IM(a), M, K, RE(b), IM(b), WRE(out), WIM(out), s));
    return OAPB_OK;
  }
  dim3 blk(GT, GT), grd((N + GT - 1) / GT, (M + GT - 1) / GT);
  k_gemm<<<grd, blk, 0, s>>>(RE(a), IM(a), RE(b), IM(b), WRE(out), WIM(out), M, N, K);
  OAPB_LAUNCH_CHECK();
  return OAPB_OK;
}

static int transpose_impl(const oapb_mat* out, const oapb_mat* in, int conj, void* stream) {
  if (!ok_mat(out) || !ok_mat(in)) return OAPB_ERR_ARG;
  if (out->columns != in->rows || out->rows != in->columns) return OAPB_ERR_ARG;
  dim3 blk(TT, 8), grd((in->columns + TT - 1) / TT, (in->rows + TT - 1) / TT);
  k_transpose<<<grd, blk, 0, STREAM(stream)>>>(RE(in), IM(in), WRE(out), WIM(out), in->columns, in->rows, conj);
  OAPB_LAUNCH_CHECK();
  return OAPB_OK;
}
int oapb_transpose(const oapb_mat* out, const oapb_mat* in, void* stream) { return transpose_impl(out, in, 0, stream); }
int oapb_conjugate_transpose(const oapb_mat* out, const oapb_mat* in, void* stream) {
  return transpose_impl(out, in, 1, stream);
}

static int reduce_impl(const oapb_mat* m, int mode, double* a, double* b, void* stream) {
  if (!ok_mat(m)) return OAPB_ERR_ARG;
  cudaStream_t s = STREAM(stream);
  const long len = numel(m);
  const int nb = grid_for(len, RB, RMaxBlocks);
  double2* buf = nullptr;
  OAPB_CUDA_TRY(cudaMallocAsync(&buf, sizeof(double2) * (nb + 1), s));
  k_reduce_partial<<<nb, RB, 0, s>>>(RE(m), IM(m), len, mode, buf + 1);
  k_reduce_final<<<1, RB, 0, s>>>(buf + 1, nb, mode, buf);
  double2 h;
  cudaError_t e = cudaMemcpyAsync(&h, buf, sizeof(double2), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(buf, s);
  if (e != cudaSuccess) return OAPB_ERR_CUDA;
  OAPB_CUDA_TRY(cudaStreamSynchronize(s));
  if (a) *a = h.x;
  if (b) *b = h.y;
  return OAPB_OK;
}
int oapb_magnitude(double* out, const oapb_mat* v, void* stream) {
  if (!out) return OAPB_ERR_ARG;
  return reduce_impl(v, 0, out, nullptr, stream);
}
int oapb_sum(double* re, double* im, const oapb_mat* m, void* stream) {
  if (!re) return OAPB_ERR_ARG;
  double b = 0;
  int st = reduce_impl(m, 1, re, &b, stream);
  if (im) *im = b;
  return st;
}

int oapb_tensor_product(const oapb_mat* out, const oapb_mat* p0, const oapb_mat* p1, void* stream) {
  if (!ok_mat(out) || !ok_mat(p0) || !ok_mat(p1)) return OAPB_ERR_ARG;
  if (out->columns != p0->columns * p1->columns || out->rows != p0->rows * p1->rows) return OAPB_ERR_ARG;
  const long len = numel(out);
  k_tensor<<<grid_for(len, 256), 256, 0, STREAM(stream)>>>(RE(p0), IM(p0), p0->columns, RE(p1), IM(p1),
                                                           p1->columns, p1->rows, WRE(out), WIM(out),
                                                           out->columns, len);
  OAPB_LAUNCH_CHECK();
  return OAPB_OK;
}

static int ew(int op, const oapb_mat* out, const oapb_mat* a, const oapb_mat* b, double sre, double sim,
              void* stream) {
  if (!ok_mat(out)) return OAPB_ERR_ARG;
  if (a && (!ok_mat(a) || numel(a) != numel(out))) return OAPB_ERR_ARG;
  if (b && (!ok_mat(b) || numel(b) != numel(out))) return OAPB_ERR_ARG;
  const long len = numel(out);
  k_elementwise<<<grid_for(len, 256), 256, 0, STREAM(stream)>>>(
      op, a ? RE(a) : nullptr, a ? IM(a) : nullptr, b ? RE(b) : nullptr, b ? IM(b) : nullptr, WRE(out),
      WIM(out), out->columns, len, sre, sim);
  OAPB_LAUNCH_CHECK();
  return OAPB_OK;
}
int oapb_add(const oapb_mat* o, const oapb_mat* a, const oapb_mat* b, void* s) { return ew(0, o, a, b, 0, 0, s); }
int oapb_substract(const oapb_mat* o, const oapb_mat* a, const oapb_mat* b, void* s) {
  return ew(1, o, a, b, 0, 0, s);
}
int oapb_multiply_re_constant(const oapb_mat* v, const oapb_mat* f, double re, void* s) {
  if (!f) return OAPB_ERR_ARG;
  return ew(2, v, f, nullptr, re, 0, s);
}
int oapb_multiply_constant(const oapb_mat* v, const oapb_mat* f, double re, double im, void* s) {
  if (!f) return OAPB_ERR_ARG;
  return ew(2, v, f, nullptr, re, im, s);
}
int oapb_set_identity(const oapb_mat* m, void* s) {
  if (!ok_mat(m) || m->columns != m->rows) return OAPB_ERR_ARG;
  return ew(3, m, nullptr, nullptr, 0, 0, s);
}
int oapb_set_diagonal(const oapb_mat* m, double re, double im, void* s) {
  if (!ok_mat(m) || m->columns != m->rows) return OAPB_ERR_ARG;
  return ew(4, m, nullptr, nullptr, re, im, s);
}
int oapb_set_zero_matrix(const oapb_mat* m, void* s) { return ew(5, m, nullptr, nullptr, 0, 0, s); }

static int vec_copy(const oapb_mat* V, uint32_t column, const oapb_mat* v, uint32_t length, int dir,
                    void* stream) {
  if (!ok_mat(V) || !ok_mat(v)) return OAPB_ERR_ARG;
  if (column >= V->columns || length > V->rows || length > v->rows) return OAPB_ERR_ARG;
  if (length == 0) return OAPB_OK;
  k_vector_copy<<<grid_for(length, 256), 256, 0, STREAM(stream)>>>(WRE(V), WIM(V), V->columns, column, WRE(v),
                                                                   WIM(v), v->columns, length, dir);
  OAPB_LAUNCH_CHECK();
  return OAPB_OK;
}
int oapb_set_vector(const oapb_mat* V, uint32_t column, const oapb_mat* v, uint32_t length, void* s) {
  return vec_copy(V, column, v, length, 0, s);
}
int oapb_get_vector(const oapb_mat* v, uint32_t length, const oapb_mat* V, uint32_t column, void* s) {
  return vec_copy(V, column, v, length, 1, s);
}

int oapb_is_upper_triangular(int* out, const oapb_mat* m, double tol, void* stream) {
  if (!out || !ok_mat(m) || m->columns != m->rows) return OAPB_ERR_ARG;
  cudaStream_t s = STREAM(stream);
  int* d = nullptr;
  OAPB_CUDA_TRY(cudaMallocAsync(&d, sizeof(int), s));
  k_is_upper<<<1, 256, 0, s>>>(RE(m), IM(m), m->columns, tol, d);
  cudaError_t e = cudaMemcpyAsync(out, d, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(d, s);
  if (e != cudaSuccess) return OAPB_ERR_CUDA;
  OAPB_CUDA_TRY(cudaStreamSynchronize(s));
  return OAPB_OK;
}

static bool same_square(const oapb_mat* a, const oapb_mat* b) {
  return ok_mat(a) && ok_mat(b) && a->columns == a->rows && b->columns == a->columns && b->rows == a->rows;
}

int oapb_qr_givens(const oapb_mat* Q, const oapb_mat* R, const oapb_mat* A, void* stream) {
  if (!same_square(A, Q) || !same_square(A, R)) return OAPB_ERR_ARG;
  cudaStream_t s = STREAM(stream);
  const int n = A->columns;
  Scratch w;
  int st = prep_ws((const void*)k_qr_givens, 2 * sizeof(cplx) * n * n, s, w);
  if (st) return st;
  k_qr_givens<<<1, 256, w.shm, s>>>(RE(A), IM(A), WRE(Q), WIM(Q), WRE(R), WIM(R), n, (cplx*)w.g);
  return finish_ws(w, s);
}

int oapb_qr_householder(const oapb_mat* Q, const oapb_mat* R, const oapb_mat* A, void* stream) {
  if (!same_square(A, Q) || !same_square(A, R) || !A->re || !Q->re || !R->re) return OAPB_ERR_ARG;
  cudaStream_t s = STREAM(stream);
  const int n = A->columns;
  Scratch w;
  int st = prep_ws((const void*)k_qr_householder, sizeof(double) * (2L * n * n + n), s, w);
  if (st) return st;
  k_qr_householder<<<1, 256, w.shm, s>>>(RE(A), WRE(Q), WRE(R), n, (double*)w.g);
  st = finish_ws(w, s);
  if (st) return st;
  // the Householder path is real; clear imaginary outputs if present
  if (Q->im) OAPB_CUDA_TRY(cudaMemsetAsync(Q->im, 0, sizeof(double) * n * n, s));
  if (R->im) OAPB_CUDA_TRY(cudaMemsetAsync(R->im, 0, sizeof(double) * n * n, s));
  return OAPB_OK;
}

int oapb_calc_triangular_h(const oapb_mat* H, const oapb_mat* Q, uint32_t max_iterations, uint32_t* iterations,
                           void* stream) {
  if (!same_square(H, Q)) return OAPB_ERR_ARG;
  cudaStream_t s = STREAM(stream);
  const int n = H->columns;
  unsigned* d = nullptr;
  OAPB_CUDA_TRY(cudaMallocAsync(&d, sizeof(unsigned), s));
  Scratch w;
  int st = prep_ws((const void*)k_calc_triangular_h, 5 * sizeof(cplx) * n * n, s, w);
  if (st) return st;
  k_calc_triangular_h<<<1, 256, w.shm, s>>>(WRE(H), WIM(H), WRE(Q), WIM(Q), n, (int)max_iterations, 1e-3,
                                            (cplx*)w.g, d);
  st = finish_ws(w, s);
  unsigned h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(d, s);
  if (st) return st;
  if (e != cudaSuccess) return OAPB_ERR_CUDA;
  OAPB_CUDA_TRY(cudaStreamSynchronize(s));
  if (iterations) *iterations = h;
  return OAPB_OK;
}

}  // extern "C"
