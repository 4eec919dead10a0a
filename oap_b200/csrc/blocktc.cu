// FP32-class block operator pass on the 5th-generation tensor cores:
//   W (b vectors) = A X,  A complex (or real) n x n in the reference layout.
//
// The operator is stored once as BF16 hi / lo planes (hi = bf16(a),
// lo = bf16(a - hi): 2 x 2 bytes per element, the footprint of FP32) and X
// is split the same way into B = [X_re | X_im] (N = 2 QB columns, QB = b
// rounded up to 8; real operators use B = [X] only).  Per 64-wide K chunk
// of a 128-row tile the CTA accumulates in tensor memory
//     D1 += Ar_hi B_hi^T + Ar_hi B_lo^T + Ar_lo B_hi^T
//     D2 += Ai_hi B_hi^T + Ai_hi B_lo^T + Ai_lo B_hi^T
// (tcgen05.mma kind::f16, M = 128, both operands K-major, 128-byte
// swizzle), and the epilogue forms W_re = D1[:, :QB] - D2[:, QB:],
// W_im = D1[:, QB:] + D2[:, :QB] in FP64.
//
// The BF16 variant (LO = false) reads the hi planes only and drops the
// A_lo terms: 4 n^2 bytes per pass (complex), products within 2^-8 of
// |A| |X| instead of about 2^-16, for the passes whose rounding a later
// FP32-class pass removes (the first powers of a subspace iteration, the
// first sweeps of a contracting fixed point).  Its coarse form (XLO =
// false) also drops X's lo part, for the first powers (a block still far
// from the wanted subspace) and the fixed point's sweeps before its last
// BF16 one (their errors are damped by the sweeps that follow): one B tile
// per K chunk instead of two, half the MMAs, and fewer bytes through the
// shared-memory fill.
//
// The kernel is persistent and stream-K scheduled (streamk.cuh): one CTA
// per SM walks an equal share of the (tile, K chunk) iterations.  Warps are
// specialised:
//   warp 0      TMA producer: per stage one cp.async.bulk.tensor load per
//               operator plane and per B plane, completion counted on the
//               stage's `full` mbarrier;
//   warp 1      MMA issuer (one lane) and TMEM owner; tcgen05.commit frees
//               the stage (`empty`) and, at the end of a tile segment,
//               hands the accumulator to the epilogue (`accf`);
//   warps 2-5   epilogue: TMEM -> registers -> FP64 tile partial, then
//               release the accumulator (`acce`).
// Two accumulator buffers in TMEM let the epilogue of one segment overlap
// the MMAs of the next.  A segment is at most kBtcSub K chunks of one tile;
// the epilogue adds the segments of a tile in FP64 registers and stores
// the tile's partial once.  The pass is HBM-bound: 8 n^2 bytes of operator per
// pass (complex), read once.  Every wait is bounded; a timeout sets *err.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>
#include <vector>

#include "blocktc.cuh"
#include "common.cuh"
#include "streamk.cuh"
#include "tc.cuh"

namespace oapb {

constexpr int kBtcM = 128;
constexpr int kBtcK = 64;
constexpr int kBtcThreads = 192;
constexpr uint64_t kBtcWaitNs = 2000000000ull;
constexpr size_t kBtcSmemBudget = 220 * 1024;
// K chunks accumulated in FP32 (TMEM) before the epilogue adds the
// sub-partial in FP64: 2048 columns, which keeps the FP32 accumulation
// error of a pass independent of n.
constexpr int kBtcSub = 32;

// X (FP64 planes, b vectors of n) -> B operand hi / lo (rows: q for re,
// QB + q for im; K = n padded to kp), zero rows / columns beyond b / n.
// Grid (column blocks, nrows): row blockIdx.y, four consecutive columns per
// thread, stored as 8-byte packs (kp is a multiple of 128).
__global__ void k_split_block_bf16(const double* __restrict__ xr, const double* __restrict__ xi, int b, int QB,
                                   int nrows, int n, int kp, __nv_bfloat16* hi, __nv_bfloat16* lo) {
  // launched as a dependent of whatever wrote X (or last read hi / lo)
  tc::griddep_wait();
  const int row = blockIdx.y;
  if (row >= nrows) return;
  const double* src = row < b ? xr + (long)row * n
                              : ((xi && row >= QB && row < QB + b) ? xi + (long)(row - QB) * n : nullptr);
  __nv_bfloat16* hrow = hi + (long)row * kp;
  __nv_bfloat16* lrow = lo + (long)row * kp;
  for (long c0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 4; c0 < kp;
       c0 += (long)gridDim.x * blockDim.x * 4) {
    __align__(8) __nv_bfloat16 h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long c = c0 + u;
      const float v = (src && c < n) ? (float)src[c] : 0.f;
      h[u] = __float2bfloat16_rn(v);
      l[u] = __float2bfloat16_rn(v - __bfloat162float(h[u]));
    }
    *reinterpret_cast<uint2*>(hrow + c0) = *reinterpret_cast<const uint2*>(h);
    *reinterpret_cast<uint2*>(lrow + c0) = *reinterpret_cast<const uint2*>(l);
  }
}

// A (FP64 plane, n x n) -> hi / lo BF16 planes (n x kp, zero-padded
// columns); with err2 set, adds sum (a - hi)^2 (the squared Frobenius norm
// of the BF16 planes' rounding) to *err2
__global__ void __launch_bounds__(256) k_split_operator_bf16(const double* __restrict__ a, int n, int kp, long row0,
                                                             long rows, __nv_bfloat16* hi, __nv_bfloat16* lo,
                                                             double* err2) {
  __shared__ double red[8];
  const long total = rows * kp;
  double acc = 0;
  for (long e0 = (long)blockIdx.x * blockDim.x + threadIdx.x; e0 < total; e0 += (long)gridDim.x * blockDim.x) {
    const long e = row0 * kp + e0;
    const long r = e / kp, c = e % kp;
    const double ad = c < n ? a[r * n + c] : 0.0;
    const float v = (float)ad;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[e] = h;
    lo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
    const double d = ad - (double)__bfloat162float(h);
    acc += d * d;
  }
  if (!err2) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(err2, t);
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

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}
// 2-D tiled TMA load (no multicast) into this CTA's shared memory
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(tc::smem_u32(bar))
      : "memory");
}

struct BtcArgs {
  CUtensorMap tm[6];  // ar_hi, ar_lo, ai_hi, ai_lo, b_hi, b_lo
  double* ws;         // stream-K tile partials
  int* err;
  SkGrid grid;
  int n, b, QB, N, stages;
  uint32_t stage_bytes;
};

// the FP64 sums of one row of a tile (slot = tile - first tile of the CTA)
template <bool CPLX, int QB>
__device__ __forceinline__ void btc_store_partial(const BtcArgs& g, long slot, int row, const double (&s1)[QB],
                                                  const double (&s2)[CPLX ? QB : 1]) {
  constexpr int NP = CPLX ? 2 : 1;
  double* out = g.ws + ((size_t)blockIdx.x * g.grid.slots + slot) * (size_t)NP * g.b * kSkRows + row;
#pragma unroll
  for (int q = 0; q < QB; ++q) {
    if (q < g.b) {
      out[(size_t)q * kSkRows] = s1[q];
      if (CPLX) out[((size_t)g.b + q) * kSkRows] = s2[q];
    }
  }
}

// wait for `parity` of `bar`; gives up after the time limit or when another
// role has already given up (*abort set)
__device__ __forceinline__ bool btc_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  const uint64_t t0 = tc::globaltimer();
  while (!tc::mbar_try_wait(bar, parity)) {
    if (*abort || tc::globaltimer() - t0 > kBtcWaitNs) {
      *abort = 1;
      return false;
    }
  }
  return true;
}

// Epilogue (warps 2-5).  Per tile segment the accumulator columns of this
// thread's row leave TMEM 16 at a time and are added in FP64 to running
// sums held in registers (QB is a compile-time constant, so every index is
// static); a tile's sums are stored to its stream-K partial once, when the
// CTA's share of the tile ends, so no global load waits in the loop.
template <bool CPLX, int QB, int KSUB>
__device__ __forceinline__ void btc_epilogue(const BtcArgs& g, uint32_t tmem, uint64_t* accf, uint64_t* acce,
                                             volatile int* abort, long it0, long it1, long kch, long first_tile,
                                             int warp, int lane) {
  constexpr int NP = CPLX ? 2 : 1;
  constexpr int NCH = (NP * QB + 15) / 16;  // 16-column TMEM loads per accumulator
  const int wq = warp & 3;                  // TMEM lane quarter of this warp
  const int row = wq * 32 + lane;
  double s1[QB], s2[CPLX ? QB : 1];
  long cur = -1, seg = 0;
  bool ok = true;
  for (long it = it0; it < it1; ++seg) {
    const long tile = it / kch, kc = it % kch;
    long kc_end = (kc / KSUB + 1) * KSUB;
    if (kc_end > kch) kc_end = kch;
    it = min(it1, tile * kch + kc_end);
    const int buf = (int)(seg & 1);
    if (!btc_wait(&accf[buf], (uint32_t)((seg / 2) & 1), abort)) {
      ok = false;
      break;
    }
    tc::tc_fence_after();
    if (tile != cur) {
      if (cur >= 0) btc_store_partial<CPLX, QB>(g, cur - first_tile, row, s1, s2);
      cur = tile;
#pragma unroll
      for (int q = 0; q < QB; ++q) {
        s1[q] = 0;
        if (CPLX) s2[q] = 0;
      }
    }
    const uint32_t tl = tmem + ((uint32_t)(wq * 32) << 16) + buf * 128;
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
      float v[16];
      tmem_ld16(tl + c * 16, v);  // D1 = A_re B^T: W_re += [:, q], W_im += [:, QB + q]
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int col = c * 16 + j;
        if (col < QB)
          s1[col] += (double)v[j];
        else if (CPLX && col < 2 * QB)
          s2[col - QB] += (double)v[j];
      }
      if (CPLX) {
        tmem_ld16(tl + 64 + c * 16, v);  // D2 = A_im B^T: W_im += [:, q], W_re -= [:, QB + q]
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = c * 16 + j;
          if (col < QB)
            s2[col] += (double)v[j];
          else if (col < 2 * QB)
            s1[col - QB] -= (double)v[j];
        }
      }
    }
    tc::tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(&acce[buf]);
  }
  if (ok && cur >= 0) btc_store_partial<CPLX, QB>(g, cur - first_tile, row, s1, s2);
}

template <bool CPLX, bool LO, bool XLO>
__global__ void __launch_bounds__(kBtcThreads, 1) k_block_matvec_tc(const __grid_constant__ BtcArgs g) {
  extern __shared__ __align__(1024) uint8_t bsm_raw[];
  constexpr int kMaxStages = 4;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], accf[2], acce[2], done;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  constexpr int NPL = CPLX ? 2 : 1;         // operator planes (re, im)
  constexpr int NR = LO ? 2 : 1;            // parts per plane (hi [, lo])
  constexpr int KH = LO ? 1 : 2;            // 64-column K chunks per stage
  constexpr int NA = NPL * NR * KH;         // operator tiles per stage, index (p * NR + r) * KH + h
  constexpr int NB = XLO ? 2 : 1;           // B parts per K chunk (hi [, lo])
  constexpr int KSUB = kBtcSub / KH;        // stages per FP32 segment
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t* sm = (uint8_t*)(((uintptr_t)bsm_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = tc::smem_u32(sm);
  const int N = g.N, S = g.stages;
  const uint32_t a_tile = kBtcM * 128, b_tile = (uint32_t)N * 128;
  const long total = g.grid.total, kch = g.grid.kchunks;
  const long it0 = sk_begin(blockIdx.x, total, gridDim.x), it1 = sk_begin(blockIdx.x + 1, total, gridDim.x);
  const long first_tile = it0 / kch;

  if (warp == 1) tc::tmem_alloc(&tmem_slot, 256);
  if (tid == 0) {
    for (int i = 0; i < S; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&accf[i], 1);
      tc::mbar_init(&acce[i], 4);
    }
    tc::mbar_init(&done, 1);
    tc::fence_mbar_init();
    abort_flag = 0;
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;
  // launched as a dependent of the B-operand split: set-up above overlaps
  // its tail; nothing below may read B before it has completed
  tc::griddep_wait();

  if (warp == 0) {
    // ---------------------------------------------------------- producer --
    if (lane == 0) {
      const uint32_t tx = NA * a_tile + NB * KH * b_tile;
      long it = it0;
      for (; it < it1; ++it) {
        const long i = it - it0;
        const int s = (int)(i % S);
        if (i >= S && !btc_wait(&empty[s], (uint32_t)((i / S - 1) & 1), &abort_flag)) break;
        const uint32_t st = sbase + s * g.stage_bytes;
        const int x = (int)((it % kch) * kBtcK * KH), y = (int)((it / kch) * kBtcM);
        mbar_expect_tx(&full[s], tx);
#pragma unroll
        for (int p = 0; p < NPL; ++p)
#pragma unroll
          for (int r = 0; r < NR; ++r)
#pragma unroll
            for (int h = 0; h < KH; ++h)
              tma_load_2d(st + ((p * NR + r) * KH + h) * a_tile, &g.tm[2 * p + r], x + h * kBtcK, y, &full[s]);
#pragma unroll
        for (int h = 0; h < KH; ++h) {
          tma_load_2d(st + NA * a_tile + h * b_tile, &g.tm[4], x + h * kBtcK, 0, &full[s]);
          if (XLO) tma_load_2d(st + NA * a_tile + (KH + h) * b_tile, &g.tm[5], x + h * kBtcK, 0, &full[s]);
        }
      }
      // no copy may still be landing in shared memory when the CTA exits:
      // wait for the last stage loads issued (already consumed normally)
      for (long j = (it - S > it0 ? it - S : it0); j < it; ++j) {
        const long i = j - it0;
        tc::mbar_wait(&full[i % S], (uint32_t)((i / S) & 1), kBtcWaitNs);
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------------- MMA --
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_bf16_f32(kBtcM, N);
      long seg = 0;
      bool ok = true;
      for (long it = it0; ok && it < it1; ++it) {
        const long i = it - it0;
        const int s = (int)(i % S);
        const long kc = it % kch;
        const bool seg_first = it == it0 || kc % KSUB == 0;
        const int buf = (int)(seg & 1);
        if (seg_first && seg >= 2 && !btc_wait(&acce[buf], (uint32_t)((seg / 2 - 1) & 1), &abort_flag)) break;
        if (!btc_wait(&full[s], (uint32_t)((i / S) & 1), &abort_flag)) break;
        tc::tc_fence_after();
        const uint32_t st = sbase + s * g.stage_bytes;
#pragma unroll
        for (int h = 0; h < KH; ++h) {
          const uint64_t bh = tc::sdesc_k_sw128(st + NA * a_tile + h * b_tile);
          const uint64_t bl = XLO ? tc::sdesc_k_sw128(st + NA * a_tile + (KH + h) * b_tile) : 0;
#pragma unroll
          for (int kk = 0; kk < kBtcK / 16; ++kk) {
            const uint64_t off = (uint64_t)(kk * 32) >> 4;
            const uint32_t acc0 = (seg_first && h == 0 && kk == 0) ? 0u : 1u;
#pragma unroll
            for (int p = 0; p < NPL; ++p) {  // p = 0: real plane -> D1, p = 1: imaginary plane -> D2
              const uint64_t ah = tc::sdesc_k_sw128(st + (p * NR * KH + h) * a_tile) + off;
              const uint32_t d = tmem + buf * 128 + p * 64;
              tc::mma_bf16(d, ah, bh + off, idesc, acc0);
              if (XLO) tc::mma_bf16(d, ah, bl + off, idesc, 1u);
              if (LO) {
                const uint64_t al = tc::sdesc_k_sw128(st + ((p * NR + 1) * KH + h) * a_tile) + off;
                tc::mma_bf16(d, al, bh + off, idesc, 1u);
              }
            }
          }
        }
        tc::commit(&empty[s]);
        if (it + 1 == it1 || (kc + 1) % KSUB == 0 || kc + 1 == kch) {
          tc::commit(&accf[buf]);
          ++seg;
        }
      }
      // every MMA issued so far has completed once `done` flips
      tc::commit(&done);
      if (!tc::mbar_wait(&done, 0, kBtcWaitNs)) abort_flag = 1;
    }
  } else {
    // ---------------------------------------------------------- epilogue --
    switch (g.QB) {
      case 8:
        btc_epilogue<CPLX, 8, KSUB>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
        break;
      case 16:
        btc_epilogue<CPLX, 16, KSUB>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
        break;
      case 24:
        btc_epilogue<CPLX, 24, KSUB>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
        break;
      default:
        btc_epilogue<CPLX, 32, KSUB>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
        break;
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::griddep_launch();  // the stream-K reduction may launch (it waits for this grid to complete)
  if (abort_flag && tid == 0) atomicOr(g.err, 1);
  if (warp == 1) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 256);
  }
}

static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// BF16 row-major plane (rows x kp, row stride kp), box 64 x box_rows, 128-byte swizzle
static bool make_tmap(CUtensorMap* m, const __nv_bfloat16* base, int kp, int rows, int box_rows) {
  auto enc = tmap_encoder();
  if (!enc || ((uintptr_t)base % 16) || kp % kBtcK) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kp * sizeof(__nv_bfloat16)};
  cuuint32_t box[2] = {(cuuint32_t)kBtcK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// one stage: lo -> 1 K chunk of hi + lo planes; else 2 K chunks of the hi
// planes; the B operand's hi (and with xlo its lo) tile per K chunk
static size_t btc_stage_bytes(int N, bool cplx, bool lo, bool xlo) {
  const int KH = lo ? 1 : 2;
  const int NA = (cplx ? 2 : 1) * (lo ? 2 : 1) * KH;
  return ((size_t)(NA * kBtcM * 128 + (xlo ? 2 : 1) * KH * N * 128) + 1023) & ~(size_t)1023;
}

int split_operator_bf16(const double* a, int n, int kp, __nv_bfloat16* hi, __nv_bfloat16* lo, cudaStream_t s,
                        long row0, long rows, double* err2) {
  if (rows < 0) rows = n - row0;
  if (row0 < 0 || row0 + rows > n) return OAPB_ERR_ARG;
  if (rows == 0) return OAPB_OK;
  k_split_operator_bf16<<<kNumSMs * 8, 256, 0, s>>>(a, n, kp, row0, rows, hi, lo, err2);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

// stream-K grid over (tile, stage) iterations of kh K chunks each
static SkGrid btc_grid(int n, int kp, int kh, int ctas = kNumSMs) {
  return sk_grid((n + kBtcM - 1) / kBtcM, kp / (kBtcK * kh), ctas);
}

size_t btc_workspace(int n, int kp) {
  size_t w = 0;
  for (int kh = 1; kh <= 2; ++kh)
    for (int c = kNumSMs - 1; c <= kNumSMs; ++c) {
      const size_t x = sk_workspace(btc_grid(n, kp, kh, c));
      w = x > w ? x : w;
    }
  return w;
}

int launch_block_matvec_tc(const BtcOperator& op, const double* xr, const double* xi, int b, double* wr,
                           double* wi, __nv_bfloat16* xbh, __nv_bfloat16* xbl, double* ws, int* err,
                           cudaStream_t s, bool bf16_only, bool x_hi_only, int ctas, const cudaEvent_t* kev) {
  const bool cplx = op.aih != nullptr;
  const int kh = bf16_only ? 2 : 1;
  if (b < 1 || b > 32 || op.kp % (kBtcK * kh) != 0 || (cplx && (!xi || !wi))) return OAPB_ERR_ARG;
  if (ctas < kNumSMs - 1 || ctas > kNumSMs) return OAPB_ERR_ARG;  // the workspace covers these grids
  const int QB = (b + 7) / 8 * 8;
  int N = cplx ? 2 * QB : QB;
  if (N % 16) N += 8;  // M = 128 needs N % 16 == 0
  if (launch_dependent(k_split_block_bf16, dim3((op.kp + 1023) / 1024, N), dim3(256), 0, s, xr, cplx ? xi : nullptr, b,
                       QB, N, op.n, op.kp, xbh, xbl) != cudaSuccess)
    return OAPB_ERR_CUDA;
  BtcArgs g;
  const __nv_bfloat16* planes[4] = {op.arh, op.arl, cplx ? op.aih : op.arh, cplx ? op.ail : op.arl};
  for (int p = 0; p < 4; ++p)
    if (!make_tmap(&g.tm[p], planes[p], op.kp, op.n, kBtcM)) return OAPB_ERR_CUDA;
  if (!make_tmap(&g.tm[4], xbh, op.kp, N, N) || !make_tmap(&g.tm[5], xbl, op.kp, N, N)) return OAPB_ERR_CUDA;
  g.ws = ws;
  g.err = err;
  g.grid = btc_grid(op.n, op.kp, kh, ctas);
  g.n = op.n;
  g.b = b;
  g.QB = QB;
  g.N = N;
  const bool xlo = !(bf16_only && x_hi_only);
  const size_t stage = btc_stage_bytes(N, cplx, !bf16_only, xlo);
  g.stage_bytes = (uint32_t)stage;
  g.stages = (int)(kBtcSmemBudget / stage);
  if (g.stages > 4) g.stages = 4;
  if (g.stages < 2) return OAPB_ERR_ARG;
  const size_t smem = g.stages * stage + 1024;
  auto kern = bf16_only ? (xlo ? (cplx ? k_block_matvec_tc<true, false, true> : k_block_matvec_tc<false, false, true>)
                              : (cplx ? k_block_matvec_tc<true, false, false> : k_block_matvec_tc<false, false, false>))
                        : (cplx ? k_block_matvec_tc<true, true, true> : k_block_matvec_tc<false, true, true>);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if (kev) cudaEventRecord(kev[0], s);
  if (launch_dependent(kern, dim3(g.grid.grid), dim3(kBtcThreads), smem, s, g) != cudaSuccess) return OAPB_ERR_CUDA;
  if (kev) cudaEventRecord(kev[1], s);
  if (cplx)
    launch_sk_reduce<true>(ws, g.grid, op.n, b, wr, wi, s);
  else
    launch_sk_reduce<false>(ws, g.grid, op.n, b, wr, nullptr, s);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

}  // namespace oapb
