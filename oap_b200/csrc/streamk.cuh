// Stream-K decomposition of a block operator pass over 128-row tiles.
//
// A pass is tiles x kchunks iterations.  A persistent grid of G CTAs splits
// the iteration range into G contiguous, equal shares (CTA c owns
// [sk_begin(c), sk_begin(c + 1))), so every SM gets the same work whatever
// the tile count.  A CTA writes one FP64 partial per tile it touches into
// slot (tile - first tile of the CTA); k_sk_reduce sums the partials of a
// tile in CTA order, so the result is deterministic.
//
// Partial layout: ws[((c * slots + slot) * planes * b + plane * b + q) * 128 + row].
#pragma once

#include <utility>

#include "common.cuh"

namespace oapb {

constexpr int kSkRows = 128;

struct SkGrid {
  long tiles, kchunks, total;
  int grid, slots;
};

// first iteration of CTA c
__host__ __device__ inline long sk_begin(long c, long total, int G) { return c * total / G; }
// CTA owning iteration it: the largest c with sk_begin(c) <= it
__host__ __device__ inline long sk_owner(long it, long total, int G) { return ((it + 1) * G + total - 1) / total - 1; }

inline SkGrid sk_grid(long tiles, long kchunks, long ctas) {
  SkGrid p;
  p.tiles = tiles;
  p.kchunks = kchunks;
  p.total = tiles * kchunks;
  if (p.total <= 0) {  // nothing to do (no grid, no workspace)
    p.grid = p.slots = 0;
    return p;
  }
  const long G = ctas < p.total ? ctas : p.total;
  p.grid = (int)G;
  // tiles one CTA can touch: its share spans at most ceil(share / kchunks) + 1
  const long share = (p.total + G - 1) / G;
  p.slots = (int)((share + p.kchunks - 1) / p.kchunks + 1);
  return p;
}

// doubles of partial workspace for b <= 32 vectors, two planes
inline size_t sk_workspace(const SkGrid& p) { return (size_t)p.grid * p.slots * 2 * 32 * kSkRows; }

// W[plane][q][row] = sum of the partials of the row's tile; block (tile,
// group of kSkCols output columns pq = plane * b + q), one thread per row of
// the tile: the owners of the tile are found once, then each owner's
// partials of the group are independent loads
constexpr int kSkCols = 8;
template <bool CPLX>
__global__ void __launch_bounds__(kSkRows) k_sk_reduce(const double* __restrict__ ws, SkGrid p, int n, int b,
                                                       double* wr, double* wi) {
  constexpr int NP = CPLX ? 2 : 1;
  // launched as a dependent of the pass that wrote the partials
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const long tile = blockIdx.x;
  const int pq0 = blockIdx.y * kSkCols, npq = NP * b;
  const long row = tile * kSkRows + threadIdx.x;
  if (row >= n) return;
  const long ilo = tile * p.kchunks;
  const long ihi = min(p.total, ilo + p.kchunks) - 1;
  const long c0 = sk_owner(ilo, p.total, p.grid), c1 = sk_owner(ihi, p.total, p.grid);
  double s[kSkCols];
#pragma unroll
  for (int j = 0; j < kSkCols; ++j) s[j] = 0.0;
  for (long c = c0; c <= c1; ++c) {
    const long slot = tile - sk_begin(c, p.total, p.grid) / p.kchunks;
    const double* src = ws + (((size_t)c * p.slots + slot) * npq + pq0) * kSkRows + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kSkCols; ++j)
      if (pq0 + j < npq) s[j] += src[(size_t)j * kSkRows];
  }
#pragma unroll
  for (int j = 0; j < kSkCols; ++j) {
    const int pq = pq0 + j;
    if (pq < npq) {
      const int q = pq % b, plane = pq / b;
      (plane == 0 ? wr : wi)[(long)q * n + row] = s[j];
    }
  }
}

// Launch with programmatic stream serialization: the kernel may start before
// the preceding grid in the stream completes and must griddepcontrol.wait
// before it reads that grid's output.
template <typename... P, typename... A>
inline cudaError_t launch_dependent(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                    A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

template <bool CPLX>
inline void launch_sk_reduce(const double* ws, const SkGrid& p, int n, int b, double* wr, double* wi,
                             cudaStream_t s) {
  const int npq = (CPLX ? 2 : 1) * b;
  launch_dependent(k_sk_reduce<CPLX>, dim3((unsigned)p.tiles, (npq + kSkCols - 1) / kSkCols), dim3(kSkRows), 0, s,
                   ws, p, n, b, wr, wi);
}

}  // namespace oapb
