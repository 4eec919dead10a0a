// FP64-class block operator pass on the integer tensor cores:
//   W (b vectors) = A X,  A complex (or real) n x n, to about 2^-43 of each
//   row's scale: the refinement's residual pass of the mixed form.
//
// Exact integer products in place of FP64 arithmetic (the splitting idea of
// Ozaki, Ogita, Oishi and Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59, 2012, with int8 slices):
//   row r of both operator planes is scaled by its power of two 2^e_r and
//   cut into 6 signed 7-bit slices, a = 2^e_r sum_i a_i 2^-7i (|a_1| <= 127,
//   |a_i| <= 64 after it: round to nearest), built once per operator;
//   vector q likewise into 7 slices below 2^f_q, per pass.
// Every slice product a_i x_j is exact in int32.  The pass forms
//   acc_o = sum over i + j = o of  A_i X_j^T      (o = 2 .. 8, 27 products)
// in tensor memory (tcgen05.mma kind::i8, M = 128, both operands K-major,
// 64-byte swizzle) and the epilogue adds 2^-7o acc_o in FP64, times
// 2^(e_r + f_q).  Dropped: slice products of order 9 and above and the
// slicing remainders, below 2^-43 of the row scale times |x|_1 plus 2^-50
// of the vector scale times |row|_1.  |acc_o| stays below 32640 per K
// column and plane, so a segment of at most 16384 K columns cannot
// overflow int32.
//
// Per 64-wide K chunk of a 128-row tile the CTA loads 6 slices x planes of
// A (8 KB each) and the 7 x N-row B block, and issues per plane and operator
// slice i one MMA of N (7 - i) columns over B's slices 0 .. 6 - i into the
// accumulators of orders i .. 6 (TMEM columns p 7N + o N): the column range
// of every order the slice contributes to is contiguous.
//
// The pass reads 6 bytes per operator element and plane (FP64: 8) and is
// HBM-bound: the integer tensor cores do 27 x 2 x 128 x N x 64 MACs per 96
// KB chunk and are busy about 40 % of the time the chunk takes to arrive.  Stream-K
// scheduled, warp-specialised (warp 0 TMA, warp 1 MMA issuer and TMEM owner,
// warps 2-5 epilogue), every wait bounded; a timeout sets *err.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "blocki8.cuh"
#include "common.cuh"
#include "streamk.cuh"
#include "tc.cuh"

namespace oapb {
namespace {

constexpr int kI8M = 128;               // operator rows per tile (MMA M)
constexpr int kI8K = 64;                // K columns (bytes) per chunk
constexpr int kI8Threads = 192;
constexpr int kI8Orders = 7;            // accumulators per plane: slice orders 2 .. 8
constexpr int kI8Sub = 256;             // K chunks per accumulation segment (16384 columns)
constexpr uint64_t kI8WaitNs = 2000000000ull;
constexpr size_t kI8SmemBudget = 225 * 1024;
constexpr uint32_t kI8ATile = kI8M * kI8K;  // bytes of one operator slice tile

// Slices of v (|v| <= 127/128) into n signed 7-bit digits, round to nearest:
// v = sum_i out[i] 2^-7(i+1) + remainder, |remainder| <= 2^-(7n+1).
template <int NS>
__device__ __forceinline__ void slice_value(double v, int (&out)[NS]) {
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    v *= 128.0;
    const double t = rint(v);
    out[i] = (int)t;
    v -= t;
  }
}

// the power of two 2^e with m 2^-e <= 127/128 (e = 0 for m = 0)
__device__ __forceinline__ int scale_exponent(double m) {
  if (!(m > 0.0)) return 0;
  int e;
  const double f = frexp(m, &e);  // m = f 2^e, f in [0.5, 1)
  if (f > 127.0 / 128.0) ++e;
  return e;
}

__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
  __syncthreads();
  return m;
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) |
         ((uint32_t)(d & 0xff) << 24);
}

// One block per operator row: the row scale of both planes, then the 6
// slices of 4 consecutive columns per thread (one 32-bit store per slice).
template <bool CPLX>
__global__ void __launch_bounds__(256) k_split_operator_i8(const double* __restrict__ are,
                                                           const double* __restrict__ aim, int n, int kp, long row0,
                                                           int8_t* __restrict__ sl, double* __restrict__ rscale) {
  __shared__ double red[8];
  const long r = row0 + blockIdx.x;
  const double* pr = are + r * n;
  const double* pi = CPLX ? aim + r * n : nullptr;
  double m = 0.0;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    m = fmax(m, fabs(pr[c]));
    if (CPLX) m = fmax(m, fabs(pi[c]));
  }
  m = block_max(m, red);
  const int e = scale_exponent(m);
  if (threadIdx.x == 0) rscale[r] = ldexp(1.0, e);
  const double inv = ldexp(1.0, -e);
  const size_t plane = (size_t)n * kp;
  for (int c4 = threadIdx.x; c4 < kp / 4; c4 += blockDim.x) {
#pragma unroll
    for (int p = 0; p < (CPLX ? 2 : 1); ++p) {
      const double* src = p == 0 ? pr : pi;
      int d[4][kI8SlicesA];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int c = 4 * c4 + t;
        slice_value<kI8SlicesA>(c < n ? src[c] * inv : 0.0, d[t]);
      }
#pragma unroll
      for (int i = 0; i < kI8SlicesA; ++i)
        *reinterpret_cast<uint32_t*>(sl + (p * kI8SlicesA + i) * plane + (size_t)r * kp + 4 * c4) =
            pack4(d[0][i], d[1][i], d[2][i], d[3][i]);
    }
  }
}

constexpr int kI8MaxBlocks = 148;  // blocks of the vector maximum pass (partials per vector)
constexpr int kI8SplitCols = 1024;  // columns of one block of the vector split

// Partial maxima of |x| over both planes of the b vectors: block k covers a
// contiguous column range and writes part[k * 32 + q]; warp w takes the
// vectors w, w + 8, ... (shuffle reductions, no block barrier).
__global__ void __launch_bounds__(256) k_block_absmax_i8(const double* __restrict__ xr,
                                                         const double* __restrict__ xi, int b, int n,
                                                         double* __restrict__ part) {
  tc::griddep_wait();  // launched as a dependent of whatever wrote X
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const long per = ((long)n + gridDim.x - 1) / gridDim.x;
  const long c0 = (long)blockIdx.x * per, c1 = min((long)n, c0 + per);
  for (int q = warp; q < b; q += nw) {
    const double* pr = xr + (long)q * n;
    const double* pi = xi ? xi + (long)q * n : nullptr;
    double m = 0.0;
    for (long c = c0 + lane; c < c1; c += 32) {
      m = fmax(m, fabs(pr[c]));
      if (pi) m = fmax(m, fabs(pi[c]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) part[blockIdx.x * 32 + q] = m;
  }
}

// Block (q, k): vector q's scale from the partial maxima (written by the
// blocks k = 0), then the 7 slices of columns k 1024 .. k 1024 + 1023 into
// B rows j N + q (re) and j N + QB + q (im); vectors q >= b give zero rows
// (the padding of B up to N rows).
__global__ void __launch_bounds__(256) k_split_block_i8(const double* __restrict__ xr, const double* __restrict__ xi,
                                                        int b, int QB, int N, int n, int kp,
                                                        const double* __restrict__ part, int nparts,
                                                        int8_t* __restrict__ xs, double* __restrict__ xscale) {
  __shared__ double red[8];
  tc::griddep_wait();  // launched as a dependent of the maximum pass
  const int q = blockIdx.x;
  const bool live = q < b;
  double m = 0.0;
  if (live)
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) m = fmax(m, part[k * 32 + q]);
  m = block_max(m, red);
  const int e = scale_exponent(m);
  if (threadIdx.x == 0 && live && blockIdx.y == 0) xscale[q] = ldexp(1.0, e);
  const double inv = ldexp(1.0, -e);
  const double* pr = live ? xr + (long)q * n : nullptr;
  const double* pi = (live && xi) ? xi + (long)q * n : nullptr;
  const int nrow = xi ? 2 : 1;
  const int c4end = min(kp / 4, (int)(blockIdx.y + 1) * (kI8SplitCols / 4));
  for (int c4 = blockIdx.y * (kI8SplitCols / 4) + threadIdx.x; c4 < c4end; c4 += blockDim.x) {
    for (int h = 0; h < nrow; ++h) {
      const double* src = h == 0 ? pr : pi;
      const int row = h == 0 ? q : QB + q;
      int d[4][kI8SlicesX];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int c = 4 * c4 + t;
        slice_value<kI8SlicesX>((live && c < n) ? src[c] * inv : 0.0, d[t]);
      }
#pragma unroll
      for (int j = 0; j < kI8SlicesX; ++j)
        *reinterpret_cast<uint32_t*>(xs + ((size_t)j * N + row) * kp + 4 * c4) =
            pack4(d[0][j], d[1][j], d[2][j], d[3][j]);
    }
  }
}

// zero B rows beyond the vectors (real operators: rows QB .. N - 1)
__global__ void k_zero_rows_i8(int r0, int r1, int N, int kp, int8_t* __restrict__ xs) {
  tc::griddep_wait();
  const long per = (long)(r1 - r0) * kp / 4, total = per * kI8SlicesX;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long j = e / per, w = e % per;
    *reinterpret_cast<uint32_t*>(xs + ((size_t)j * N + r0) * kp + 4 * w) = 0u;
  }
}

__device__ __forceinline__ void i8_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void i8_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}
// tiled TMA loads (no multicast) into this CTA's shared memory
__device__ __forceinline__ void i8_tma_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(tc::smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void i8_tma_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(tc::smem_u32(bar))
      : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, signed int8 inputs, int32 accumulation.
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Instruction descriptor: s8 x s8 -> s32 (c_format 2, a / b format 1 =
// signed), both operands K-major.
__host__ __device__ constexpr uint32_t idesc_s8_s32(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Shared-memory descriptor of a K-major tile with 64-byte rows, 64-byte
// swizzle (layout type 4), 8-row groups 512 bytes apart; base 512-byte aligned.
__device__ __forceinline__ uint64_t sdesc_k_sw64(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

struct I8Args {
  CUtensorMap ta;  // operator slices: kp x n x (planes x 6), box 64 x 128 x 1
  CUtensorMap tb;  // vector slices: kp x 7N, box 64 x 7N
  const double* rscale;
  const double* xscale;
  double* ws;
  int* err;
  SkGrid grid;
  int n, b, QB, N, stages;
  uint32_t stage_bytes;
};

__device__ __forceinline__ bool i8_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  const uint64_t t0 = tc::globaltimer();
  while (!tc::mbar_try_wait(bar, parity)) {
    if (*abort || tc::globaltimer() - t0 > kI8WaitNs) {
      *abort = 1;
      return false;
    }
  }
  return true;
}

// the scaled FP64 sums of one row of a tile (slot = tile - first tile of the CTA)
template <bool CPLX, int QB>
__device__ __forceinline__ void i8_store_partial(const I8Args& g, long tile, long slot, int row,
                                                 const double (&s1)[QB], const double (&s2)[CPLX ? QB : 1]) {
  constexpr int NP = CPLX ? 2 : 1;
  const long grow = tile * kI8M + row;
  const double rs = grow < g.n ? g.rscale[grow] : 0.0;
  double* out = g.ws + ((size_t)blockIdx.x * g.grid.slots + slot) * (size_t)NP * g.b * kSkRows + row;
#pragma unroll
  for (int q = 0; q < QB; ++q) {
    if (q < g.b) {
      const double sc = rs * g.xscale[q];
      out[(size_t)q * kSkRows] = s1[q] * sc;
      if (CPLX) out[((size_t)g.b + q) * kSkRows] = s2[q] * sc;
    }
  }
}

// B rows (N) of the pass for QB vector slots: [re | im] for a complex
// operator, rounded up to a multiple of 16 (M = 128 needs N % 16 == 0)
template <bool CPLX, int QB>
__host__ __device__ constexpr int i8_rows() {
  return CPLX ? 2 * QB : (QB + 15) / 16 * 16;
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (no wait)
__device__ __forceinline__ void i8_tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

// Epilogue (warps 2-5): per segment, the 7 order accumulators of each plane
// leave TMEM (one wait per order) and are added in FP64, scaled by 2^-7o,
// to the row's running sums (D1 = A_re B^T: W_re += [:, q], W_im += [:, QB + q];
// D2 = A_im B^T: W_im += [:, q], W_re -= [:, QB + q]).  QB is a compile-time
// constant, so every register index is static.
template <bool CPLX, int QB>
__device__ __forceinline__ void i8_epilogue(const I8Args& g, uint32_t tmem, uint64_t* accf, uint64_t* acce,
                                            volatile int* abort, long it0, long it1, long kch, long first_tile,
                                            int warp, int lane) {
  constexpr int N = i8_rows<CPLX, QB>();
  constexpr int NCH = N / 16;
  constexpr int NPL = CPLX ? 2 : 1;
  const int wq = warp & 3;
  const int row = wq * 32 + lane;
  double s1[QB], s2[CPLX ? QB : 1];
  long cur = -1, seg = 0;
  bool ok = true;
  for (long it = it0; it < it1; ++seg) {
    const long tile = it / kch, kc = it % kch;
    long kc_end = (kc / kI8Sub + 1) * kI8Sub;
    if (kc_end > kch) kc_end = kch;
    it = min(it1, tile * kch + kc_end);
    if (!i8_wait(accf, (uint32_t)(seg & 1), abort)) {
      ok = false;
      break;
    }
    tc::tc_fence_after();
    if (tile != cur) {
      if (cur >= 0) i8_store_partial<CPLX, QB>(g, cur, cur - first_tile, row, s1, s2);
      cur = tile;
#pragma unroll
      for (int q = 0; q < QB; ++q) {
        s1[q] = 0;
        if (CPLX) s2[q] = 0;
      }
    }
    const uint32_t tl = tmem + ((uint32_t)(wq * 32) << 16);
#pragma unroll 1
    for (int o = 0; o < kI8Orders; ++o) {
      const double sc = ldexp(1.0, -7 * (o + 2));
      uint32_t v[NPL][NCH][16];
#pragma unroll
      for (int p = 0; p < NPL; ++p)
#pragma unroll
        for (int c = 0; c < NCH; ++c) i8_tmem_ld16(tl + (uint32_t)(p * kI8Orders * N + o * N + c * 16), v[p][c]);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int c = 0; c < NCH; ++c)
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = c * 16 + j;
          const double d1 = (double)(int)v[0][c][j] * sc;
          if (col < QB)
            s1[col] += d1;
          else if (CPLX && col < 2 * QB)
            s2[col - QB] += d1;
          if constexpr (CPLX) {
            const double d2 = (double)(int)v[NPL - 1][c][j] * sc;
            if (col < QB)
              s2[col] += d2;
            else if (col < 2 * QB)
              s1[col - QB] -= d2;
          }
        }
    }
    tc::tc_fence_before();
    __syncwarp();
    if (lane == 0) i8_arrive(acce);
  }
  if (ok && cur >= 0) i8_store_partial<CPLX, QB>(g, cur, cur - first_tile, row, s1, s2);
}

template <bool CPLX>
__global__ void __launch_bounds__(kI8Threads, 1) k_block_matvec_i8(const __grid_constant__ I8Args g) {
  extern __shared__ __align__(1024) uint8_t ism_raw[];
  constexpr int kMaxStages = 4;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], accf[1], acce[1], done;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  constexpr int NPL = CPLX ? 2 : 1;
  constexpr int NA = NPL * kI8SlicesA;  // operator tiles per stage, index p * 6 + i
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t* sm = (uint8_t*)(((uintptr_t)ism_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = tc::smem_u32(sm);
  const int N = g.N, S = g.stages;
  const uint32_t tcols = (uint32_t)(NPL * kI8Orders * N) <= 128 ? 128u : (NPL * kI8Orders * N <= 256 ? 256u : 512u);
  const long total = g.grid.total, kch = g.grid.kchunks;
  const long it0 = sk_begin(blockIdx.x, total, gridDim.x), it1 = sk_begin(blockIdx.x + 1, total, gridDim.x);
  const long first_tile = it0 / kch;

  if (warp == 1) tc::tmem_alloc(&tmem_slot, tcols);
  if (tid == 0) {
    for (int i = 0; i < S; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    tc::mbar_init(&accf[0], 1);
    tc::mbar_init(&acce[0], 4);
    tc::mbar_init(&done, 1);
    tc::fence_mbar_init();
    abort_flag = 0;
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;
  // launched as a dependent of the vector split: nothing below may read B
  // (or the scales) before it has completed
  tc::griddep_wait();

  if (warp == 0) {
    // ---------------------------------------------------------- producer --
    if (lane == 0) {
      const uint32_t b_bytes = (uint32_t)(kI8SlicesX * N * kI8K);
      const uint32_t tx = NA * kI8ATile + b_bytes;
      long it = it0;
      for (; it < it1; ++it) {
        const long i = it - it0;
        const int s = (int)(i % S);
        if (i >= S && !i8_wait(&empty[s], (uint32_t)((i / S - 1) & 1), &abort_flag)) break;
        const uint32_t st = sbase + s * g.stage_bytes;
        const int x = (int)((it % kch) * kI8K), y = (int)((it / kch) * kI8M);
        i8_expect_tx(&full[s], tx);
#pragma unroll
        for (int t = 0; t < NA; ++t) i8_tma_3d(st + t * kI8ATile, &g.ta, x, y, t, &full[s]);
        i8_tma_2d(st + NA * kI8ATile, &g.tb, x, 0, &full[s]);
      }
      // no copy may still be landing in shared memory when the CTA exits
      for (long j = (it - S > it0 ? it - S : it0); j < it; ++j) {
        const long i = j - it0;
        tc::mbar_wait(&full[i % S], (uint32_t)((i / S) & 1), kI8WaitNs);
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------------- MMA --
    if (lane == 0) {
      long seg = 0;
      for (long it = it0; it < it1; ++it) {
        const long i = it - it0;
        const int s = (int)(i % S);
        const long kc = it % kch;
        const bool seg_first = it == it0 || kc % kI8Sub == 0;
        if (seg_first && seg >= 1 && !i8_wait(acce, (uint32_t)((seg - 1) & 1), &abort_flag)) break;
        if (!i8_wait(&full[s], (uint32_t)((i / S) & 1), &abort_flag)) break;
        tc::tc_fence_after();
        const uint32_t st = sbase + s * g.stage_bytes;
        const uint64_t bd = sdesc_k_sw64(st + NA * kI8ATile);
#pragma unroll
        for (int p = 0; p < NPL; ++p) {
#pragma unroll
          for (int sa = 0; sa < kI8SlicesA; ++sa) {
            // operator slice sa times vector slices 0 .. 6 - sa: orders sa .. 6
            const uint32_t idesc = idesc_s8_s32(kI8M, N * (kI8SlicesX - sa));
            const uint32_t d = tmem + (uint32_t)(p * kI8Orders * N + sa * N);
            const uint64_t ad = sdesc_k_sw64(st + (p * kI8SlicesA + sa) * kI8ATile);
#pragma unroll
            for (int kk = 0; kk < kI8K / 32; ++kk) {
              const uint64_t off = (uint64_t)(kk * 32) >> 4;
              const uint32_t acc = (seg_first && sa == 0 && kk == 0) ? 0u : 1u;
              mma_i8(d, ad + off, bd + off, idesc, acc);
            }
          }
        }
        tc::commit(&empty[s]);
        if (it + 1 == it1 || (kc + 1) % kI8Sub == 0 || kc + 1 == kch) {
          tc::commit(accf);
          ++seg;
        }
      }
      tc::commit(&done);
      if (!tc::mbar_wait(&done, 0, kI8WaitNs)) abort_flag = 1;
    }
  } else {
    // ---------------------------------------------------------- epilogue --
    if (g.QB == 8) {
      i8_epilogue<CPLX, 8>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
    } else if (g.QB == 16) {
      i8_epilogue<CPLX, 16>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
    } else if constexpr (!CPLX) {
      if (g.QB == 24)
        i8_epilogue<CPLX, 24>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
      else
        i8_epilogue<CPLX, 32>(g, tmem, accf, acce, &abort_flag, it0, it1, kch, first_tile, warp, lane);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::griddep_launch();  // the stream-K reduction may launch (it waits for this grid to complete)
  if (abort_flag && tid == 0) atomicOr(g.err, 1);
  if (warp == 1) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, tcols);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 i8_encoder() {
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

// int8 row-major slices (kp bytes a row, rows x depth), box 64 x box_rows x 1, 64-byte swizzle
bool make_tmap_i8(CUtensorMap* m, const int8_t* base, int kp, int rows, int depth, int box_rows) {
  auto enc = i8_encoder();
  if (!enc || ((uintptr_t)base % 16) || kp % kI8K || box_rows < 1 || box_rows > 256) return false;
  const cuuint32_t rank = depth > 1 ? 3 : 2;
  cuuint64_t dims[3] = {(cuuint64_t)kp, (cuuint64_t)rows, (cuuint64_t)depth};
  cuuint64_t strides[2] = {(cuuint64_t)kp, (cuuint64_t)kp * rows};
  cuuint32_t box[3] = {(cuuint32_t)kI8K, (cuuint32_t)box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, rank, (void*)base, dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

SkGrid i8_grid(int n, int kp) { return sk_grid((n + kI8M - 1) / kI8M, kp / kI8K, kNumSMs); }

}  // namespace

int split_operator_i8(const double* are, const double* aim, int n, int kp, int8_t* slices, double* rscale,
                      cudaStream_t s, long row0, long rows) {
  if (rows < 0) rows = n - row0;
  if (row0 < 0 || row0 + rows > n || kp % 128 || kp < n) return OAPB_ERR_ARG;
  if (rows == 0) return OAPB_OK;
  if (aim)
    k_split_operator_i8<true><<<(unsigned)rows, 256, 0, s>>>(are, aim, n, kp, row0, slices, rscale);
  else
    k_split_operator_i8<false><<<(unsigned)rows, 256, 0, s>>>(are, nullptr, n, kp, row0, slices, rscale);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

size_t i8_workspace(int n, int kp) { return sk_workspace(i8_grid(n, kp)); }

int launch_block_matvec_i8(const I8Operator& op, const double* xr, const double* xi, int b, double* wr, double* wi,
                           int8_t* xs, double* xscale, double* ws, int* err, cudaStream_t s, const cudaEvent_t* kev) {
  const bool cplx = op.cplx;
  if (b < 1 || b > i8_max_vectors(cplx) || op.kp % 128 || (cplx && (!xi || !wi))) return OAPB_ERR_ARG;
  const int QB = (b + 7) / 8 * 8;
  const int N = cplx ? 2 * QB : (QB + 15) / 16 * 16;  // i8_rows<cplx, QB>()
  // vector maxima (partials), then the vector slices (rows beyond the
  // vectors zeroed: the real case's N > QB)
  const int nparts = op.n < kI8MaxBlocks ? op.n : kI8MaxBlocks;
  double* part = xscale + kI8BlockScales;
  if (launch_dependent(k_block_absmax_i8, dim3(nparts), dim3(256), 0, s, xr, cplx ? xi : nullptr, b, op.n, part) !=
      cudaSuccess)
    return OAPB_ERR_CUDA;
  if (launch_dependent(k_split_block_i8, dim3(QB, (op.kp + kI8SplitCols - 1) / kI8SplitCols), dim3(256), 0, s, xr,
                       cplx ? xi : nullptr, b, QB, N, op.n, op.kp, (const double*)part, nparts, xs,
                       xscale) != cudaSuccess)
    return OAPB_ERR_CUDA;
  const int used = cplx ? 2 * QB : QB;
  if (used < N && launch_dependent(k_zero_rows_i8, dim3(kNumSMs), dim3(256), 0, s, used, N, N, op.kp, xs) !=
                      cudaSuccess)
    return OAPB_ERR_CUDA;
  I8Args g;
  const int planes = (cplx ? 2 : 1) * kI8SlicesA;
  if (!make_tmap_i8(&g.ta, op.slices, op.kp, op.n, planes, kI8M)) return OAPB_ERR_CUDA;
  if (!make_tmap_i8(&g.tb, xs, op.kp, kI8SlicesX * N, 1, kI8SlicesX * N)) return OAPB_ERR_CUDA;
  g.rscale = op.rscale;
  g.xscale = xscale;
  g.ws = ws;
  g.err = err;
  g.grid = i8_grid(op.n, op.kp);
  g.n = op.n;
  g.b = b;
  g.QB = QB;
  g.N = N;
  const size_t stage = ((size_t)planes * kI8ATile + (size_t)kI8SlicesX * N * kI8K + 1023) & ~(size_t)1023;
  g.stage_bytes = (uint32_t)stage;
  g.stages = (int)(kI8SmemBudget / stage);
  if (g.stages > 4) g.stages = 4;
  if (g.stages < 2) return OAPB_ERR_ARG;
  const size_t smem = g.stages * stage + 1024;
  auto kern = cplx ? k_block_matvec_i8<true> : k_block_matvec_i8<false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if (kev) cudaEventRecord(kev[0], s);
  if (launch_dependent(kern, dim3(g.grid.grid), dim3(kI8Threads), smem, s, g) != cudaSuccess) return OAPB_ERR_CUDA;
  if (kev) cudaEventRecord(kev[1], s);
  if (cplx)
    launch_sk_reduce<true>(ws, g.grid, op.n, b, wr, wi, s);
  else
    launch_sk_reduce<false>(ws, g.grid, op.n, b, wr, nullptr, s);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

}  // namespace oapb
