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
//
// For X in host memory (larger than HBM, as the reference's application
// reads its image folders block by block, MainAPExecutor.cpp:59-100,
// RecToSquareApi.cpp:71-141) the operator runs on column (pixel) blocks:
// A v = sum_c X_c (X_c^T v), so one application reads X exactly once.  The
// first blocks that fit the caller's device budget stay resident; the rest
// stream through two device buffers, the host-to-device copy of the next
// block (on its own stream) overlapping the two passes over the current one.
#include <algorithm>
#include <new>

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
                                               const double* __restrict__ t, double* __restrict__ w,
                                               int accumulate) {
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
    if (lane == 0) w[r] = accumulate ? w[r] + s : s;
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

int launch_gram_apply(const float* X, int rows, int cols, const double* v, double* w, double* ws, cudaStream_t s,
                      bool accumulate) {
  if (!X || !v || !w || !ws || rows < 1 || cols < 1) return OAPB_ERR_ARG;
  if ((cols & 3) == 0 && ((uintptr_t)X & 15)) return OAPB_ERR_ARG;
  const int ns = gram_op_splits(rows, cols);
  const int rps = (rows + ns - 1) / ns;
  double* t = ws + (size_t)ns * cols;
  k_gram_xt<<<dim3((cols + kGxCols - 1) / kGxCols, ns), kGxThreads, 0, s>>>(X, rows, cols, v, rps, ws);
  k_gram_reduce<<<grid_for(cols, 256, kNumSMs * 4), 256, 0, s>>>(ws, ns, cols, t);
  k_gram_x<<<grid_for((long)rows * 32, 256, kNumSMs * 8), 256, 0, s>>>(X, rows, cols, t, w, accumulate ? 1 : 0);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

// ------------------------------------------------------------ host X --
struct GramStream {
  const float* hX = nullptr;  // host, rows x cols row-major
  int rows = 0, cols = 0, bc = 0, nb = 0, resident = 0;
  float* dres = nullptr;      // resident blocks, each rows x bc (the last may be narrower)
  float* dbuf[2] = {nullptr, nullptr};
  double* ws = nullptr;       // gram_op_workspace(rows, bc)
  cudaStream_t cs = nullptr;  // copy stream
  cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
  unsigned long long streamed_bytes = 0;
};

static int block_width(const GramStream* g, int c) { return std::min(g->bc, g->cols - c * g->bc); }

void gram_stream_destroy(GramStream* g) {
  if (!g) return;
  if (g->cs) cudaStreamSynchronize(g->cs);
  for (int i = 0; i < 2; ++i) {
    if (g->dbuf[i]) cudaFree(g->dbuf[i]);
    if (g->copied[i]) cudaEventDestroy(g->copied[i]);
    if (g->consumed[i]) cudaEventDestroy(g->consumed[i]);
  }
  if (g->dres) cudaFree(g->dres);
  if (g->ws) cudaFree(g->ws);
  if (g->cs) cudaStreamDestroy(g->cs);
  delete g;
}

int gram_stream_create(const float* hX, int rows, int cols, int block_cols, unsigned long long resident_bytes,
                       cudaStream_t s, GramStream** out) {
  if (!hX || rows < 1 || cols < 1 || block_cols < 1 || !out) return OAPB_ERR_ARG;
  GramStream* g = new (std::nothrow) GramStream();
  if (!g) return OAPB_ERR_NOMEM;
  g->hX = hX;
  g->rows = rows;
  g->cols = cols;
  g->bc = std::min(cols, (block_cols + 3) / 4 * 4);  // 16-byte rows for the vector loads
  g->nb = (cols + g->bc - 1) / g->bc;
  const size_t block_bytes = sizeof(float) * (size_t)rows * g->bc;
  g->resident = (int)std::min<unsigned long long>((unsigned long long)g->nb, resident_bytes / block_bytes);
  int rc = OAPB_OK;
  do {
    if (cudaMalloc(&g->ws, sizeof(double) * gram_op_workspace(rows, g->bc)) != cudaSuccess) {
      rc = OAPB_ERR_NOMEM;
      break;
    }
    if (g->resident > 0 && cudaMalloc(&g->dres, block_bytes * g->resident) != cudaSuccess) {
      rc = OAPB_ERR_NOMEM;
      break;
    }
    if (g->resident < g->nb) {
      for (int i = 0; i < 2 && !rc; ++i) {
        if (cudaMalloc(&g->dbuf[i], block_bytes) != cudaSuccess) rc = OAPB_ERR_NOMEM;
        else if (cudaEventCreateWithFlags(&g->copied[i], cudaEventDisableTiming) != cudaSuccess ||
                 cudaEventCreateWithFlags(&g->consumed[i], cudaEventDisableTiming) != cudaSuccess)
          rc = OAPB_ERR_CUDA;
      }
      if (!rc && cudaStreamCreateWithFlags(&g->cs, cudaStreamNonBlocking) != cudaSuccess) rc = OAPB_ERR_CUDA;
      if (rc) break;
    }
    // the resident blocks, copied once
    for (int c = 0; c < g->resident; ++c) {
      const int w = block_width(g, c);
      if (cudaMemcpy2DAsync(g->dres + (size_t)c * rows * g->bc, sizeof(float) * w, hX + (size_t)c * g->bc,
                            sizeof(float) * cols, sizeof(float) * w, rows, cudaMemcpyHostToDevice, s) !=
          cudaSuccess) {
        rc = OAPB_ERR_CUDA;
        break;
      }
    }
  } while (0);
  if (rc) {
    cudaGetLastError();
    gram_stream_destroy(g);
    return rc;
  }
  *out = g;
  return OAPB_OK;
}

int gram_stream_apply(GramStream* g, const double* v, double* w, cudaStream_t s) {
  int slot = 0;
  for (int c = 0; c < g->nb; ++c) {
    const int wc = block_width(g, c);
    const float* Xc;
    bool streamed = c >= g->resident;
    if (!streamed) {
      Xc = g->dres + (size_t)c * g->rows * g->bc;
    } else {
      // the slot's previous block has been read; then copy this block into it
      if (cudaStreamWaitEvent(g->cs, g->consumed[slot], 0) != cudaSuccess ||
          cudaMemcpy2DAsync(g->dbuf[slot], sizeof(float) * wc, g->hX + (size_t)c * g->bc, sizeof(float) * g->cols,
                            sizeof(float) * wc, g->rows, cudaMemcpyHostToDevice, g->cs) != cudaSuccess ||
          cudaEventRecord(g->copied[slot], g->cs) != cudaSuccess ||
          cudaStreamWaitEvent(s, g->copied[slot], 0) != cudaSuccess)
        return OAPB_ERR_CUDA;
      g->streamed_bytes += sizeof(float) * (unsigned long long)wc * g->rows;
      Xc = g->dbuf[slot];
    }
    const int rc = launch_gram_apply(Xc, g->rows, wc, v, w, g->ws, s, c > 0);
    if (rc) return rc;
    if (streamed) {
      if (cudaEventRecord(g->consumed[slot], s) != cudaSuccess) return OAPB_ERR_CUDA;
      slot ^= 1;
    }
  }
  return OAPB_OK;
}

unsigned long long gram_stream_bytes(const GramStream* g) { return g ? g->streamed_bytes : 0; }
int gram_stream_resident_blocks(const GramStream* g) { return g ? g->resident : 0; }
int gram_stream_blocks(const GramStream* g) { return g ? g->nb : 0; }

}  // namespace oapb
