// FP32-class block operator pass on the 5th-generation tensor cores:
//   W (b vectors) = A X,  A complex (or real) n x n in the reference layout.
//
// The operator is stored once as BF16 hi / lo planes (hi = bf16(a),
// lo = bf16(a - hi): 2 x 2 bytes per element, the footprint of FP32) and X
// is split the same way into B = [X_re | X_im] (N = 2 QB columns, QB = b
// rounded up to 8; real operators use B = [X] only).  Per 64-wide K chunk
// the CTA accumulates in tensor memory
//     D1 += Ar_hi B_hi^T + Ar_hi B_lo^T + Ar_lo B_hi^T
//     D2 += Ai_hi B_hi^T + Ai_hi B_lo^T + Ai_lo B_hi^T
// (tcgen05.mma kind::f16, M = 128, both operands K-major in 128-byte
// swizzled shared memory filled by cp.async, two stages), and the epilogue
// forms W_re = D1[:, :QB] - D2[:, QB:], W_im = D1[:, QB:] + D2[:, :QB] as
// FP64 split-K partials (summed by k_split_reduce).  The pass is HBM-bound:
// 8 n^2 bytes of operator per pass, read once.
#include <vector>

#include "blocktc.cuh"
#include "common.cuh"
#include "tc.cuh"

namespace oapb {

constexpr int kBtcM = 128;
constexpr int kBtcK = 64;
constexpr int kBtcThreads = 128;
constexpr uint64_t kBtcWaitNs = 2000000000ull;

// X (FP64 planes, b vectors of n) -> B operand hi / lo (rows: q for re,
// QB + q for im; K = n padded to kp), zero rows / columns beyond b / n
__global__ void k_split_block_bf16(const double* __restrict__ xr, const double* __restrict__ xi, int b, int QB,
                                   int nrows, int n, int kp, __nv_bfloat16* hi, __nv_bfloat16* lo) {
  const long total = (long)nrows * kp;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int row = (int)(e / kp);
    const long c = e % kp;
    float v = 0.f;
    if (c < n) {
      if (row < b) v = (float)xr[(long)row * n + c];
      else if (xi && row >= QB && row < QB + b) v = (float)xi[(long)(row - QB) * n + c];
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[e] = h;
    lo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

// A (FP64 plane, n x n) -> hi / lo BF16 planes (n x kp, zero-padded columns)
__global__ void k_split_operator_bf16(const double* __restrict__ a, int n, int kp, __nv_bfloat16* hi,
                                      __nv_bfloat16* lo) {
  const long total = (long)n * kp;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long r = e / kp, c = e % kp;
    const float v = c < n ? (float)a[r * n + c] : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[e] = h;
    lo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct BtcArgs {
  const __nv_bfloat16 *arh, *arl, *aih, *ail;  // operator planes, n x kp
  const __nv_bfloat16 *bh, *bl;                // B operand, N x kp
  int n, kp, b, QB, N, ksplit;                 // N = QB (real) or 2 QB (complex)
  double* Wp;                                  // nsplit x 2 x b x n partials
  int* err;
};

template <bool CPLX>
__global__ void __launch_bounds__(kBtcThreads, 1) k_block_matvec_tc(BtcArgs g) {
  extern __shared__ __align__(1024) uint8_t bsm_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  constexpr int NA = CPLX ? 4 : 2;  // operator tiles per stage
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t* sm = (uint8_t*)(((uintptr_t)bsm_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = tc::smem_u32(sm);
  const int N = g.N;
  const uint32_t a_tile = kBtcM * 128, b_tile = (uint32_t)N * 128;
  const uint32_t stage_bytes = ((NA * a_tile + 2 * b_tile) + 1023) & ~1023u;
  const long i0 = (long)blockIdx.x * kBtcM;
  const long kb = (long)blockIdx.y * g.ksplit;
  const long ke = min((long)g.kp, kb + g.ksplit);
  const int niter = (int)((ke - kb) / kBtcK);
  const __nv_bfloat16* ap[4] = {g.arh, g.arl, g.aih, g.ail};

  if (warp == 0) tc::tmem_alloc(&tmem_slot, 128);
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
  const uint32_t idesc = tc::idesc_bf16_f32(kBtcM, N);

  auto load_stage = [&](int it, int s) {
    const uint32_t st = sbase + s * stage_bytes;
    const long k0 = kb + (long)it * kBtcK;
    for (int c = tid; c < NA * kBtcM * 8; c += kBtcThreads) {
      const int part = c / (kBtcM * 8), q = c % (kBtcM * 8);
      const int r = q >> 3, ch = q & 7;
      const long row = i0 + r;
      const __nv_bfloat16* src = ap[part] + (row < g.n ? row : 0) * (long)g.kp + k0 + ch * 8;
      tc::cp_async16(st + part * a_tile + tc::sw128(r, ch), src);
    }
    for (int c = tid; c < 2 * N * 8; c += kBtcThreads) {
      const int part = c / (N * 8), q = c % (N * 8);
      const int r = q >> 3, ch = q & 7;
      const __nv_bfloat16* src = (part ? g.bl : g.bh) + (long)r * g.kp + k0 + ch * 8;
      tc::cp_async16(st + NA * a_tile + part * b_tile + tc::sw128(r, ch), src);
    }
    tc::cp_async_commit();
  };

  bool ok = niter > 0;
  if (ok) load_stage(0, 0);
  for (int it = 0; ok && it < niter; ++it) {
    const int s = it & 1;
    if (it + 1 < niter) {
      const int s1 = (it + 1) & 1;
      if (it >= 1 && !tc::mbar_wait(&bar[s1], ((it - 1) >> 1) & 1, kBtcWaitNs)) atomicOr(&abort_flag, 1);
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
      const uint32_t st = sbase + s * stage_bytes;
      const uint64_t bh = tc::sdesc_k_sw128(st + NA * a_tile), bl = tc::sdesc_k_sw128(st + NA * a_tile + b_tile);
#pragma unroll
      for (int kk = 0; kk < kBtcK / 16; ++kk) {
        const uint64_t off = (uint64_t)(kk * 32) >> 4;
        const uint32_t first = (it > 0 || kk > 0) ? 1u : 0u;
#pragma unroll
        for (int p = 0; p < NA / 2; ++p) {  // p = 0: real plane -> D1, p = 1: imaginary plane -> D2
          const uint64_t ah = tc::sdesc_k_sw128(st + (2 * p) * a_tile) + off;
          const uint64_t al = tc::sdesc_k_sw128(st + (2 * p + 1) * a_tile) + off;
          const uint32_t d = tmem + p * 64;
          tc::mma_bf16(d, ah, bh + off, idesc, first);
          tc::mma_bf16(d, ah, bl + off, idesc, 1u);
          tc::mma_bf16(d, al, bh + off, idesc, 1u);
        }
      }
      tc::commit(&bar[s]);
    }
  }
  if (ok) {
    const int last = niter - 1;
    if (!tc::mbar_wait(&bar[last & 1], (last >> 1) & 1, kBtcWaitNs)) atomicOr(&abort_flag, 2);
  }
  tc::cp_async_wait<0>();
  __syncthreads();
  tc::tc_fence_after();
  if (ok && !abort_flag) {
    const long row = i0 + warp * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
    float d1[64], d2[64];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      if (c * 16 < N) {
        tmem_ld16(tl + c * 16, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) d1[c * 16 + j] = v[j];
        if (CPLX) {
          tmem_ld16(tl + 64 + c * 16, v);
#pragma unroll
          for (int j = 0; j < 16; ++j) d2[c * 16 + j] = v[j];
        }
      }
    }
    if (row < g.n) {
      double* wr = g.Wp + (long)blockIdx.y * 2 * g.b * g.n;
      double* wi = wr + (long)g.b * g.n;
      for (int q = 0; q < g.b; ++q) {
        if (CPLX) {
          wr[(long)q * g.n + row] = (double)d1[q] - (double)d2[g.QB + q];
          wi[(long)q * g.n + row] = (double)d1[g.QB + q] + (double)d2[q];
        } else {
          wr[(long)q * g.n + row] = (double)d1[q];
        }
      }
    }
  } else if (tid == 0) {
    atomicOr(g.err, abort_flag | (ok ? 0 : 4));
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

size_t block_tc_smem(int N, bool cplx) {
  const int NA = cplx ? 4 : 2;
  const size_t stage = ((size_t)(NA * kBtcM * 128 + 2 * N * 128) + 1023) & ~(size_t)1023;
  return 2 * stage + 1024;
}

int split_operator_bf16(const double* a, int n, int kp, __nv_bfloat16* hi, __nv_bfloat16* lo, cudaStream_t s) {
  k_split_operator_bf16<<<kNumSMs * 8, 256, 0, s>>>(a, n, kp, hi, lo);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

// W partials (nsplit x 2 x b x n) of A X on the tensor cores; xbh / xbl:
// scratch for the split block (2 x 64 x kp BF16 each).
int launch_block_matvec_tc(const BtcOperator& op, const double* xr, const double* xi, int b, double* Wp,
                           int nsplit, int ksplit, __nv_bfloat16* xbh, __nv_bfloat16* xbl, int* err,
                           cudaStream_t s) {
  const bool cplx = op.aih != nullptr;
  if (b < 1 || b > 32 || ksplit % kBtcK != 0) return OAPB_ERR_ARG;
  const int QB = (b + 7) / 8 * 8;
  int N = cplx ? 2 * QB : QB;
  if (N % 16) N += 8;  // M = 128 needs N % 16 == 0
  k_split_block_bf16<<<kNumSMs * 4, 256, 0, s>>>(xr, cplx ? xi : nullptr, b, QB, N, op.n, op.kp, xbh, xbl);
  const size_t smem = block_tc_smem(N, cplx);
  BtcArgs g{op.arh, op.arl, op.aih, op.ail, xbh, xbl, op.n, op.kp, b, QB, N, ksplit, Wp, err};
  dim3 grid((op.n + kBtcM - 1) / kBtcM, nsplit);
  if (cplx) {
    if (cudaFuncSetAttribute(k_block_matvec_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return OAPB_ERR_CUDA;
    k_block_matvec_tc<true><<<grid, kBtcThreads, smem, s>>>(g);
  } else {
    if (cudaFuncSetAttribute(k_block_matvec_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return OAPB_ERR_CUDA;
    k_block_matvec_tc<false><<<grid, kBtcThreads, smem, s>>>(g);
  }
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

}  // namespace oapb
