// Gram operator build A = X X^T on the 5th-generation tensor cores.
//
// Reference: SquareMatrixApi::getDeviceMatrix (oapMatrixCuda/SquareMatrixApi.cpp:143-156)
// forms the Gram matrix with a naive FP64 dotProduct(out, X, X^T) and the
// image application rebuilds it on every matvec (oap2dt3dDevice/MainAPExecutor.cpp:53-55).
// Here it is built once: X (rows x cols, FP32, row-major, e.g. samples x
// pixels) is split into BF16 hi + lo parts (hi = bf16(x), lo = bf16(x - hi)),
// and every 128 x 256 output tile accumulates
//     hi hi^T + hi lo^T + lo hi^T
// in FP32 in tensor memory with tcgen05.mma (kind::f16, both operands
// K-major in 128-byte-swizzled shared memory, filled by cp.async, two
// stages).  Only tiles touching the upper triangle are computed; the
// epilogue writes each (i <= j) element and its mirror.
//
// Algorithmic work: 2 rows^2 cols flops (one product, counted once).
#include <stdio.h>

#include <vector>

#include "common.cuh"
#include "tc.cuh"

namespace oapb {

constexpr int kGmM = 128;   // tile rows (A operand)
constexpr int kGmN = 256;   // tile columns (B operand)
constexpr int kGmK = 64;    // BF16 per 128-byte row segment
constexpr int kGmThreads = 128;
constexpr uint32_t kGmStageBytes = (2 * kGmM + 2 * kGmN) * 128;  // Ahi, Alo, Bhi, Blo
constexpr uint32_t kGmSmem = 2 * kGmStageBytes + 1024;           // + alignment slack
constexpr uint64_t kGmWaitNs = 2000000000ull;                    // 2 s per wait

// hi / lo split into zero-padded (rows_p x cols_p) BF16 arrays
__global__ void k_split_bf16(const float* __restrict__ X, int rows, int cols, int rows_p, int cols_p,
                             __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
  const long total = (long)rows_p * cols_p;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long r = e / cols_p, c = e % cols_p;
    const float x = (r < rows && c < cols) ? X[r * cols + c] : 0.0f;
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi[e] = h;
    lo[e] = __float2bfloat16_rn(x - __bfloat162float(h));
  }
}

struct GramArgs {
  const __nv_bfloat16* hi;
  const __nv_bfloat16* lo;
  int rows, cols_p;        // cols_p % 64 == 0; rows of hi / lo padded to a multiple of 256
  const int2* tiles;       // (row tile, column tile)
  float* C;                // rows x rows
  double* C64;             // optional FP64 copy
  int* err;
};

__global__ void __launch_bounds__(kGmThreads, 1) k_gram_tc(GramArgs g) {
  extern __shared__ __align__(1024) uint8_t gsm_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t* gsm = (uint8_t*)(((uintptr_t)gsm_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = tc::smem_u32(gsm);
  const int2 tile = g.tiles[blockIdx.x];
  const long i0 = (long)tile.x * kGmM, j0 = (long)tile.y * kGmN;
  const int niter = g.cols_p / kGmK;

  if (warp == 0) tc::tmem_alloc(&tmem_slot, kGmN);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
    tc::fence_mbar_init();
    abort_flag = 0;
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;
  constexpr uint32_t idesc = tc::idesc_bf16_f32(kGmM, kGmN);

  // stage s: Ahi at s*stage, Alo +16K, Bhi +32K, Blo +64K
  auto load_stage = [&](int it, int s) {
    const uint32_t st = sbase + s * kGmStageBytes;
    const long k0 = (long)it * kGmK;
    // A: 2 x 1024 chunks, B: 2 x 2048 chunks of 16 bytes
    for (int c = tid; c < 2 * kGmM * 8; c += kGmThreads) {
      const int part = c / (kGmM * 8), q = c % (kGmM * 8);
      const int r = q >> 3, ch = q & 7;
      const __nv_bfloat16* src = (part ? g.lo : g.hi) + (i0 + r) * (long)g.cols_p + k0 + ch * 8;
      tc::cp_async16(st + part * (kGmM * 128) + tc::sw128(r, ch), src);
    }
    for (int c = tid; c < 2 * kGmN * 8; c += kGmThreads) {
      const int part = c / (kGmN * 8), q = c % (kGmN * 8);
      const int r = q >> 3, ch = q & 7;
      const __nv_bfloat16* src = (part ? g.lo : g.hi) + (j0 + r) * (long)g.cols_p + k0 + ch * 8;
      tc::cp_async16(st + 2 * kGmM * 128 + part * (kGmN * 128) + tc::sw128(r, ch), src);
    }
    tc::cp_async_commit();
  };

  bool ok = true;
  load_stage(0, 0);
  for (int it = 0; it < niter; ++it) {
    const int s = it & 1;
    if (it + 1 < niter) {
      const int s1 = (it + 1) & 1;
      if (it >= 1) {
        // the MMAs of iteration it - 1 read stage s1: wait for their commit
        if (!tc::mbar_wait(&bar[s1], ((it - 1) >> 1) & 1, kGmWaitNs)) {
          atomicOr(&abort_flag, 1);
        }
      }
      __syncthreads();
      if (abort_flag) {
        ok = false;
        break;
      }
      load_stage(it + 1, s1);
      tc::cp_async_wait<1>();
    } else {
      tc::cp_async_wait<0>();
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::tc_fence_after();
      const uint32_t st = sbase + s * kGmStageBytes;
      const uint64_t ahi = tc::sdesc_k_sw128(st), alo = tc::sdesc_k_sw128(st + kGmM * 128);
      const uint64_t bhi = tc::sdesc_k_sw128(st + 2 * kGmM * 128);
      const uint64_t blo = tc::sdesc_k_sw128(st + 2 * kGmM * 128 + kGmN * 128);
#pragma unroll
      for (int kk = 0; kk < kGmK / 16; ++kk) {
        const uint64_t off = (uint64_t)(kk * 32) >> 4;  // 32 bytes per K=16 step
        tc::mma_bf16(tmem, ahi + off, bhi + off, idesc, (it > 0 || kk > 0) ? 1u : 0u);
        tc::mma_bf16(tmem, ahi + off, blo + off, idesc, 1u);
        tc::mma_bf16(tmem, alo + off, bhi + off, idesc, 1u);
      }
      tc::commit(&bar[s]);
    }
  }
  // all MMAs done before reading the accumulator
  if (ok && niter > 0) {
    const int last = niter - 1;
    if (!tc::mbar_wait(&bar[last & 1], (last >> 1) & 1, kGmWaitNs)) atomicOr(&abort_flag, 2);
  }
  tc::cp_async_wait<0>();
  __syncthreads();
  tc::tc_fence_after();
  if (!abort_flag) {
    const long i = i0 + warp * 32 + lane;
#pragma unroll 1
    for (int cc = 0; cc < kGmN / 32; ++cc) {
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + cc * 32, v);
      if (i < g.rows) {
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          const long j = j0 + cc * 32 + q;
          if (j < g.rows && i <= j) {
            g.C[i * g.rows + j] = v[q];
            if (i != j) g.C[j * g.rows + i] = v[q];
            if (g.C64) {
              g.C64[i * g.rows + j] = (double)v[q];
              if (i != j) g.C64[j * g.rows + i] = (double)v[q];
            }
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicOr(g.err, abort_flag);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kGmN);
}

}  // namespace oapb

using namespace oapb;

extern "C" {

int oapb_gram_build(const float* X, uint32_t rows, uint32_t cols, float* A, double* A64, void* stream) {
  if (!X || !A || rows == 0 || cols == 0) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int rows_p = (int)((rows + kGmN - 1) / kGmN) * kGmN;
  const int cols_p = (int)((cols + kGmK - 1) / kGmK) * kGmK;
  // tiles touching the upper triangle
  std::vector<int2> tiles;
  for (int r = 0; r * kGmM < (int)rows; ++r)
    for (int c = 0; c * kGmN < (int)rows; ++c)
      if (r * kGmM <= c * kGmN + kGmN - 1) tiles.push_back(make_int2(r, c));
  const size_t half = (size_t)rows_p * cols_p;
  const size_t bytes = 2 * half * sizeof(__nv_bfloat16) + tiles.size() * sizeof(int2) + 256;
  char* buf = nullptr;
  if (cudaMallocAsync((void**)&buf, bytes, s) != cudaSuccess) {
    cudaGetLastError();
    return OAPB_ERR_NOMEM;
  }
  __nv_bfloat16* hi = (__nv_bfloat16*)buf;
  __nv_bfloat16* lo = hi + half;
  int2* dtiles = (int2*)(lo + half);
  int* err = (int*)(dtiles + tiles.size());
  int rc = OAPB_OK;
  do {
    if (cudaMemcpyAsync(dtiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    k_split_bf16<<<kNumSMs * 8, 256, 0, s>>>(X, (int)rows, (int)cols, rows_p, cols_p, hi, lo);
    if (cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGmSmem) !=
        cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    GramArgs g{hi, lo, (int)rows, cols_p, dtiles, A, A64, err};
    k_gram_tc<<<(unsigned)tiles.size(), kGmThreads, kGmSmem, s>>>(g);
    if (cudaGetLastError() != cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    int herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    if (herr) rc = OAPB_ERR_TIMEOUT;
  } while (0);
  cudaFreeAsync(buf, s);
  return rc;
}

}  // extern "C"
