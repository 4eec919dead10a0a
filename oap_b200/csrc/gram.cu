// Gram operator build A = X X^T on the 5th-generation tensor cores.
//
// Reference: SquareMatrixApi::getDeviceMatrix (oapMatrixCuda/SquareMatrixApi.cpp:143-156)
// forms the Gram matrix with a naive FP64 dotProduct(out, X, X^T) and the
// image application rebuilds it on every matvec (oap2dt3dDevice/MainAPExecutor.cpp:53-55).
// Here it is built once: X (rows x cols, FP32, row-major, e.g. samples x
// pixels) is split into BF16 hi + lo parts (hi = bf16(x), lo = bf16(x - hi)),
// and every 128 x 256 output tile accumulates
//     hi hi^T + hi lo^T + lo hi^T
// in FP32 in tensor memory with tcgen05.mma (kind::f16, M = 128, N = 256,
// both operands K-major).  Only tiles touching the upper triangle are
// computed; a second kernel writes each (i <= j) element and its mirror.
//
// k_gram_tc walks (tile, 32-column K chunk) iterations in contiguous CTA
// shares; it is launched with one CTA per tile (one resident per SM), so the
// CTAs of a wave read the same K chunks at the same time and the operands
// come from L2.  With fewer CTAs than tiles (stream-K) each CTA's share is
// at least one tile long, so a tile is split between at most two CTAs: the
// part that starts at the tile's first chunk goes to slot 0 of the tile's
// FP32 partials, the rest to slot 1, and k_gram_finish adds the slots in
// that order (deterministic).  Warps are specialised:
//   warp 0      TMA producer: per stage 4 tiled loads (A hi / lo: 128 rows,
//               B hi / lo: 256 rows, 32 columns = 64 bytes, 64-byte swizzle)
//               completing on the stage's `full` mbarrier; 4 stages of 48 KB;
//   warp 1      MMA issuer (one lane) and TMEM owner: 3 products per K=16
//               step into one of two 256-column FP32 accumulators;
//               tcgen05.commit frees the stage (`empty`) and hands a finished
//               segment to the epilogue (`accf`);
//   warps 2-5   epilogue: TMEM -> registers -> the segment's FP32 partial
//               (column-major, coalesced), then release the accumulator
//               (`acce`), so the next segment's MMAs overlap the drain.
// Every wait is bounded (2 s); a timeout sets the error word (OAPB_ERR_TIMEOUT).
//
// Algorithmic work: 2 rows^2 cols flops (one product, counted once).
#include <stdio.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "tc.cuh"
#include "tma.cuh"

namespace oapb {

constexpr int kGmM = 128;   // tile rows (A operand)
constexpr int kGmN = 256;   // tile columns (B operand)
constexpr int kGmK = 32;    // BF16 per 64-byte row segment (one stage)
constexpr int kGmStages = 4;
constexpr int kGmThreads = 192;
constexpr uint32_t kGmATile = kGmM * kGmK * 2;                 // 8 KB
constexpr uint32_t kGmBTile = kGmN * kGmK * 2;                 // 16 KB
constexpr uint32_t kGmStageBytes = 2 * kGmATile + 2 * kGmBTile;  // Ahi, Alo, Bhi, Blo: 48 KB
constexpr uint32_t kGmSmem = kGmStages * kGmStageBytes + 1024;  // + alignment slack
constexpr uint64_t kGmWaitNs = 2000000000ull;                   // 2 s per wait
constexpr int kGmTileElems = kGmM * kGmN;

// hi / lo split into zero-padded (rows_p x cols_p) BF16 arrays: block row
// blockIdx.y, four consecutive elements per thread (a 16-byte load when the
// row allows it, 8-byte stores)
__global__ void k_split_bf16(const float* __restrict__ X, int rows, int cols, int rows_p, int cols_p,
                             __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
  const bool vec = (cols & 3) == 0 && ((uintptr_t)X & 15) == 0;
  for (int r = blockIdx.y; r < rows_p; r += gridDim.y) {
    const float* xr = X + (long)r * cols;
    __nv_bfloat16* hr = hi + (long)r * cols_p;
    __nv_bfloat16* lr = lo + (long)r * cols_p;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) * 4; c < cols_p; c += gridDim.x * blockDim.x * 4) {
      float v[4];
      if (r < rows && vec && c + 3 < cols) {
        const float4 x4 = __ldcs(reinterpret_cast<const float4*>(xr + c));
        v[0] = x4.x, v[1] = x4.y, v[2] = x4.z, v[3] = x4.w;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = (r < rows && c + j < cols) ? xr[c + j] : 0.0f;
      }
      __align__(8) __nv_bfloat16 h[4], l[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        h[j] = __float2bfloat16_rn(v[j]);
        l[j] = __float2bfloat16_rn(v[j] - __bfloat162float(h[j]));
      }
      // cols_p is a multiple of 32: the four outputs are in the row and 8-byte aligned
      *reinterpret_cast<uint2*>(hr + c) = *reinterpret_cast<const uint2*>(h);
      *reinterpret_cast<uint2*>(lr + c) = *reinterpret_cast<const uint2*>(l);
    }
  }
}

// The build's workspace (BF16 planes, partials, tile list) comes from a
// stream-ordered pool owned by the library, one per device, that keeps freed
// memory for the next build instead of returning it to the driver at every
// synchronisation (a 1 GiB workspace mapped anew per call took several
// milliseconds).  oapb_gram_trim releases what it holds.
static std::mutex g_gram_pool_mutex;
static cudaMemPool_t g_gram_pool[64] = {};

static cudaMemPool_t gram_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_gram_pool_mutex);
  if (!g_gram_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    g_gram_pool[dev] = p;
  }
  return g_gram_pool[dev];
}

struct GramArgs {
  CUtensorMap ahi, alo, bhi, blo;  // the hi / lo planes with A (128-row) and B (256-row) boxes
  const int4* tiles;               // (row tile, column tile, split, 0)
  float* ws;                       // FP32 partials: tile x 2 slots x (256 columns x 128 rows)
  int* err;
  long total;                      // tiles x K chunks
  int kch;                         // K chunks per tile
  int ctas;
};

// Shared-memory descriptor of a K-major tile with 64-byte rows (32 BF16),
// 64-byte swizzle (layout type 4), 8-row groups 512 bytes apart.
__device__ __forceinline__ uint64_t gm_sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

__global__ void __launch_bounds__(kGmThreads, 1) k_gram_tc(const __grid_constant__ GramArgs g) {
  extern __shared__ __align__(1024) uint8_t gsm_raw[];
  __shared__ __align__(8) uint64_t full[kGmStages], empty[kGmStages], accf[2], acce[2], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t* gsm = (uint8_t*)(((uintptr_t)gsm_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = tc::smem_u32(gsm);
  const long it0 = (long)blockIdx.x * g.total / g.ctas, it1 = (long)(blockIdx.x + 1) * g.total / g.ctas;
  const int kch = g.kch;

  if (warp == 1) tc::tmem_alloc(&tmem_slot, 512);
  if (tid == 0) {
    for (int i = 0; i < kGmStages; ++i) {
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

  if (warp == 0) {
    // ---------------------------------------------------------- producer --
    if (lane == 0) {
      long it = it0;
      for (; it < it1; ++it) {
        const long i = it - it0;
        const int s = (int)(i % kGmStages);
        if (i >= kGmStages && !tma::wait(&empty[s], (uint32_t)((i / kGmStages - 1) & 1), &abort_flag, kGmWaitNs))
          break;
        const int4 t = g.tiles[it / kch];
        const int x = (int)(it % kch) * kGmK;
        const uint32_t st = sbase + s * kGmStageBytes;
        tma::expect_tx(&full[s], kGmStageBytes);
        tma::load_2d(st, &g.ahi, x, t.x * kGmM, &full[s]);
        tma::load_2d(st + kGmATile, &g.alo, x, t.x * kGmM, &full[s]);
        tma::load_2d(st + 2 * kGmATile, &g.bhi, x, t.y * kGmN, &full[s]);
        tma::load_2d(st + 2 * kGmATile + kGmBTile, &g.blo, x, t.y * kGmN, &full[s]);
      }
      // no copy may still be landing in shared memory when the CTA exits
      for (long j = (it - kGmStages > it0 ? it - kGmStages : it0); j < it; ++j) {
        const long i = j - it0;
        tc::mbar_wait(&full[i % kGmStages], (uint32_t)((i / kGmStages) & 1), kGmWaitNs);
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------------- MMA --
    if (lane == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(kGmM, kGmN);
      long seg = 0;
      for (long it = it0; it < it1; ++it) {
        const long i = it - it0;
        const int s = (int)(i % kGmStages);
        const long kc = it % kch;
        const bool seg_first = it == it0 || kc == 0;
        const int buf = (int)(seg & 1);
        if (seg_first && seg >= 2 && !tma::wait(&acce[buf], (uint32_t)((seg / 2 - 1) & 1), &abort_flag, kGmWaitNs))
          break;
        if (!tma::wait(&full[s], (uint32_t)((i / kGmStages) & 1), &abort_flag, kGmWaitNs)) break;
        tc::tc_fence_after();
        const uint32_t st = sbase + s * kGmStageBytes;
        const uint64_t ahi = gm_sdesc(st), alo = gm_sdesc(st + kGmATile);
        const uint64_t bhi = gm_sdesc(st + 2 * kGmATile), blo = gm_sdesc(st + 2 * kGmATile + kGmBTile);
        const uint32_t d = tmem + buf * kGmN;
#pragma unroll
        for (int kk = 0; kk < kGmK / 16; ++kk) {
          const uint64_t off = (uint64_t)(kk * 32) >> 4;  // 32 bytes per K = 16 step
          tc::mma_bf16(d, ahi + off, bhi + off, idesc, (seg_first && kk == 0) ? 0u : 1u);
          tc::mma_bf16(d, ahi + off, blo + off, idesc, 1u);
          tc::mma_bf16(d, alo + off, bhi + off, idesc, 1u);
        }
        tc::commit(&empty[s]);
        if (it + 1 == it1 || kc + 1 == kch) {
          tc::commit(&accf[buf]);
          ++seg;
        }
      }
      // every MMA issued so far has completed once `done` flips
      tc::commit(&done);
      if (!tc::mbar_wait(&done, 0, kGmWaitNs)) abort_flag = 1;
    }
  } else {
    // ---------------------------------------------------------- epilogue --
    const int wq = warp & 3;  // TMEM lane quarter of this warp
    const int row = wq * 32 + lane;
    long seg = 0;
    for (long it = it0; it < it1; ++seg) {
      const long tile = it / kch;
      const long seg_end = (tile + 1) * kch < it1 ? (tile + 1) * kch : it1;
      const int slot = it == tile * kch ? 0 : 1;
      const int buf = (int)(seg & 1);
      if (!tma::wait(&accf[buf], (uint32_t)((seg / 2) & 1), &abort_flag, kGmWaitNs)) break;
      tc::tc_fence_after();
      float* out = g.ws + ((size_t)tile * 2 + slot) * kGmTileElems + row;
#pragma unroll 1
      for (int cc = 0; cc < kGmN / 32; ++cc) {
        float v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(wq * 32) << 16) + buf * kGmN + cc * 32, v);
#pragma unroll
        for (int q = 0; q < 32; ++q) out[(size_t)(cc * 32 + q) * kGmM] = v[q];
      }
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tma::arrive(&acce[buf]);
      it = seg_end;
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (abort_flag && tid == 0) atomicOr(g.err, 1);
  if (warp == 1) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 512);
  }
}

// A (and its FP64 copy) from the tile partials: one block per 32 x 32 piece
// of a tile; element (i, j), i <= j, and its mirror (j, i).  The piece goes
// through shared memory so both the direct and the mirrored rows are
// written with consecutive lanes on consecutive columns.
__global__ void k_gram_finish(const float* __restrict__ ws, const int4* __restrict__ tiles, int rows, float* C,
                              double* C64) {
  __shared__ float t[32][33];
  const int tile = blockIdx.x / 32, piece = blockIdx.x % 32;
  const int a = piece / 8, b = piece % 8;  // 32-row strip a of 4, 32-column strip b of 8
  const int4 T = tiles[tile];
  const long i0 = (long)T.x * kGmM + a * 32, j0 = (long)T.y * kGmN + b * 32;
  if (i0 > j0 + 31) return;  // every element below the diagonal
  const float* s0 = ws + (size_t)tile * 2 * kGmTileElems;
  const float* s1 = s0 + kGmTileElems;
  const int r = threadIdx.x, cy = threadIdx.y;
  for (int c = cy; c < 32; c += 8) {
    const size_t idx = (size_t)(b * 32 + c) * kGmM + a * 32 + r;
    float v = s0[idx];
    if (T.z) v += s1[idx];
    t[c][r] = v;
  }
  __syncthreads();
  for (int rr = cy; rr < 32; rr += 8) {  // direct: row i0 + rr, lanes over columns
    const long i = i0 + rr, j = j0 + r;
    if (i < rows && j < rows && i <= j) {
      const float v = t[r][rr];
      C[i * rows + j] = v;
      if (C64) C64[i * rows + j] = (double)v;
    }
  }
  for (int cc = cy; cc < 32; cc += 8) {  // mirror: row j0 + cc, lanes over columns i
    const long j = j0 + cc, i = i0 + r;
    if (i < rows && j < rows && i < j) {
      const float v = t[cc][r];
      C[j * rows + i] = v;
      if (C64) C64[j * rows + i] = (double)v;
    }
  }
}

}  // namespace oapb

using namespace oapb;

extern "C" {

int oapb_gram_build(const float* X, uint32_t rows, uint32_t cols, float* A, double* A64, void* stream) {
  if (!X || !A || rows == 0 || cols == 0) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int rows_p = (int)((rows + kGmN - 1) / kGmN) * kGmN;
  const int cols_p = (int)((cols + kGmK - 1) / kGmK) * kGmK;
  const int kch = cols_p / kGmK;
  // tiles touching the upper triangle, and the stream-K split of
  // (tile, K chunk) iterations over at most one CTA per SM
  std::vector<int4> tiles;
  for (int r = 0; r * kGmM < (int)rows; ++r)
    for (int c = 0; c * kGmN < (int)rows; ++c)
      if (r * kGmM <= c * kGmN + kGmN - 1) tiles.push_back(make_int4(r, c, 0, 0));
  const long ntiles = (long)tiles.size();
  // one CTA per tile, resident one per SM, so the CTAs of a wave stream K
  // in step and read each operand chunk from L2 (a stream-K split over
  // min(tiles, SMs) CTAs left them at scattered K offsets: 4.7 GB of DRAM
  // reads for 256 MB of operands at 4096 x 16384); the split machinery below
  // stays for grids of fewer CTAs than tiles
  const int ctas = (int)ntiles;
  const long total = ntiles * kch;
  // with at least one tile per CTA a tile meets at most two CTAs: it is
  // split when the CTA holding its first chunk ends inside it (never with
  // one CTA per tile)
  for (long t = 0; t < ntiles; ++t) {
    const long first = t * kch;
    long b = (first * ctas) / total;  // the CTA whose [b total / ctas, (b + 1) total / ctas) holds `first`
    while (b > 0 && b * total / ctas > first) --b;
    while ((b + 1) * total / ctas <= first) ++b;
    tiles[t].z = (b + 1) * total / ctas < first + kch ? 1 : 0;
  }
  const size_t half = (size_t)rows_p * cols_p;
  const size_t ws_elems = (size_t)ntiles * 2 * kGmTileElems;
  const size_t bytes = 2 * half * sizeof(__nv_bfloat16) + ws_elems * sizeof(float) + tiles.size() * sizeof(int4) + 256;
  char* buf = nullptr;
  cudaMemPool_t pool = gram_pool();
  if (!pool || cudaMallocFromPoolAsync((void**)&buf, bytes, pool, s) != cudaSuccess) {
    cudaGetLastError();
    return OAPB_ERR_NOMEM;
  }
  __nv_bfloat16* hi = (__nv_bfloat16*)buf;
  __nv_bfloat16* lo = hi + half;
  float* ws = (float*)(lo + half);
  int4* dtiles = (int4*)(ws + ws_elems);
  int* err = (int*)(dtiles + tiles.size());
  int rc = OAPB_OK;
  do {
    GramArgs g;
    if (!tma::map_bf16(&g.ahi, hi, cols_p, rows_p, kGmK, kGmM, CU_TENSOR_MAP_SWIZZLE_64B) ||
        !tma::map_bf16(&g.alo, lo, cols_p, rows_p, kGmK, kGmM, CU_TENSOR_MAP_SWIZZLE_64B) ||
        !tma::map_bf16(&g.bhi, hi, cols_p, rows_p, kGmK, kGmN, CU_TENSOR_MAP_SWIZZLE_64B) ||
        !tma::map_bf16(&g.blo, lo, cols_p, rows_p, kGmK, kGmN, CU_TENSOR_MAP_SWIZZLE_64B)) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    if (cudaMemcpyAsync(dtiles, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    {
      const int bx = (int)std::min<long>((cols_p / 4 + 255) / 256, 16);
      k_split_bf16<<<dim3(bx, std::min(rows_p, 65535)), 256, 0, s>>>(X, (int)rows, (int)cols, rows_p, cols_p, hi, lo);
    }
    if (cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGmSmem) !=
        cudaSuccess) {
      rc = OAPB_ERR_CUDA;
      break;
    }
    g.tiles = dtiles;
    g.ws = ws;
    g.err = err;
    g.total = total;
    g.kch = kch;
    g.ctas = ctas;
    k_gram_tc<<<(unsigned)ctas, kGmThreads, kGmSmem, s>>>(g);
    k_gram_finish<<<(unsigned)(ntiles * 32), dim3(32, 8), 0, s>>>(ws, dtiles, (int)rows, A, A64);
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

int oapb_gram_trim(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return OAPB_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_gram_pool_mutex);
  if (g_gram_pool[dev] && cudaMemPoolTrimTo(g_gram_pool[dev], 0) != cudaSuccess) return OAPB_ERR_CUDA;
  return OAPB_OK;
}

}  // extern "C"
