// Implicit Gram operator: A v = X (X^T v) for FP32 images X (rows samples x
// cols pixels, row-major), the operator of the reference's image
// application (oap2dt3dDevice/MainAPExecutor.cpp:42-127 builds the Gram
// X X^T, or row blocks of it, on every multiplication through
// SquareMatrixApi::getDeviceMatrix / getDeviceSubMatrix,
// oapMatrixCuda/SquareMatrixApi.cpp:143-181).  Here A is never formed: two
// HBM-bound passes over X per multiplication,
//   t = X^T v   (k_gram_xt: a thread owns 4 consecutive pixels and streams a
//               slice of rows with 16-byte loads; v[r] is a broadcast; the
//               row slices' partials are summed by k_gram_reduce),
//   w = X t     (k_gram_x: one warp per row, 16-byte loads, t L2-resident),
// FP32 pixels times FP64 vectors accumulated in FP64: the result is the
// product with the exact Gram matrix of the FP32 images.
#include "common.cuh"
#include "gramop.cuh"

namespace oapb {

constexpr int kGxThreads = 256;
constexpr int kGxCols = kGxThreads * 4;  // pixels per block

__global__ void __launch_bounds__(kGxThreads) k_gram_xt(const float* __restrict__ X, int rows, int cols,
                                                       const double* __restrict__ v, int rows_per_split,
                                                       double* __restrict__ part) {
  const long c = ((long)blockIdx.x * kGxThreads + threadIdx.x) * 4;
  const int r0 = blockIdx.y * rows_per_split;
  const int r1 = min(rows, r0 + rows_per_split);
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  if (c < cols) {
    if ((cols & 3) == 0) {
      for (int r = r0; r < r1; ++r) {
        const float4 x = __ldcs(reinterpret_cast<const float4*>(X + (long)r * cols + c));
        const double vr = v[r];
        a0 = fma((double)x.x, vr, a0);
        a1 = fma((double)x.y, vr, a1);
        a2 = fma((double)x.z, vr, a2);
        a3 = fma((double)x.w, vr, a3);
      }
    } else {
      for (int r = r0; r < r1; ++r) {
        const float* xr = X + (long)r * cols;
        const double vr = v[r];
        a0 = fma((double)xr[c], vr, a0);
        if (c + 1 < cols) a1 = fma((double)xr[c + 1], vr, a1);
        if (c + 2 < cols) a2 = fma((double)xr[c + 2], vr, a2);
        if (c + 3 < cols) a3 = fma((double)xr[c + 3], vr, a3);
      }
    }
    double* p = part + (long)blockIdx.y * cols + c;
    p[0] = a0;
    if (c + 1 < cols) p[1] = a1;
    if (c + 2 < cols) p[2] = a2;
    if (c + 3 < cols) p[3] = a3;
  }
}

// t[c] = sum over the row splits (stored after the partials)
__global__ void k_gram_reduce(const double* __restrict__ part, int nsplit, int cols, double* __restrict__ t) {
  for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += (long)gridDim.x * blockDim.x) {
    double s = 0;
    for (int k = 0; k < nsplit; ++k) s += part[(long)k * cols + c];
    t[c] = s;
  }
}

__global__ void __launch_bounds__(256) k_gram_x(const float* __restrict__ X, int rows, int cols,
                                               const double* __restrict__ t, double* __restrict__ w) {
  const int lane = threadIdx.x & 31;
  const long warps = (long)gridDim.x * (blockDim.x >> 5);
  for (long r = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
    const float* xr = X + r * cols;
    double a0 = 0, a1 = 0;
    if ((cols & 3) == 0) {
      for (int q = lane; q < cols / 4; q += 32) {
        const float4 x = __ldcs(reinterpret_cast<const float4*>(xr) + q);
        const double2 t0 = *reinterpret_cast<const double2*>(t + 4 * q);
        const double2 t1 = *reinterpret_cast<const double2*>(t + 4 * q + 2);
        a0 = fma((double)x.x, t0.x, a0);
        a1 = fma((double)x.y, t0.y, a1);
        a0 = fma((double)x.z, t1.x, a0);
        a1 = fma((double)x.w, t1.y, a1);
      }
    } else {
      for (int c = lane; c < cols; c += 32) a0 = fma((double)xr[c], t[c], a0);
    }
    const double s = warp_sum(a0 + a1);
    if (lane == 0) w[r] = s;
  }
}

int gram_op_splits(int rows, int cols) {
  const int tiles = (cols + kGxCols - 1) / kGxCols;
  int s = (4 * kNumSMs + tiles - 1) / tiles;
  if (s > 64) s = 64;
  if (s > rows) s = rows;
  return s < 1 ? 1 : s;
}

size_t gram_op_workspace(int rows, int cols) { return ((size_t)gram_op_splits(rows, cols) + 1) * cols; }

int launch_gram_apply(const float* X, int rows, int cols, const double* v, double* w, double* ws, cudaStream_t s) {
  if (!X || !v || !w || !ws || rows < 1 || cols < 1) return OAPB_ERR_ARG;
  if ((cols & 3) == 0 && ((uintptr_t)X & 15)) return OAPB_ERR_ARG;
  const int ns = gram_op_splits(rows, cols);
  const int rps = (rows + ns - 1) / ns;
  double* t = ws + (size_t)ns * cols;
  k_gram_xt<<<dim3((cols + kGxCols - 1) / kGxCols, ns), kGxThreads, 0, s>>>(X, rows, cols, v, rps, ws);
  k_gram_reduce<<<grid_for(cols, 256, kNumSMs * 4), 256, 0, s>>>(ws, ns, cols, t);
  k_gram_x<<<grid_for((long)rows * 32, 256, kNumSMs * 8), 256, 0, s>>>(X, rows, cols, t, w);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

}  // namespace oapb
