// FP64 block operator pass W = A X on the FP64 tensor cores.
//
// Each iteration stages a 128 x 16 tile of every operator plane and the
// 16-wide slice of X in shared memory (cp.async, three stages; two CTAs per
// SM up to 32 output columns).  Warp w owns
// operator rows 16 w .. 16 w + 15 of the tile and all N output columns:
//   complex: B1 = [X_re | X_im] (N = 2 b columns), B2 = [-X_im | X_re], so
//            C = A_re B1 + A_im B2 = [W_re | W_im] in one accumulator;
//   real:    C = A_re X (N = b).
// Both products run as mma.sync.m16n8k16.f64 over n-tiles of 8 columns with
// FP64 accumulation (the same rounding class as the FP64 CUDA-core pass).
// B2 is not stored: its fragment is read from the B1 row of the permuted
// column, negated where the column is an X_im column.
//
// Shared layout per stage:
//   A plane: 128 rows x 128 bytes, 16-byte chunk c of row r at chunk
//            c ^ (r & 7) (a fragment read is two wavefronts, the minimum
//            for 256 bytes);
//   X:       NT x 8 rows (B1 columns) x 16 doubles, swizzled the same way;
//            rows beyond N are zero and never written.
#include "blockdmma.cuh"
#include "common.cuh"
#include "streamk.cuh"

namespace oapb {

constexpr int kDmM = 128;        // operator rows per tile
constexpr int kDmK = 16;         // columns per iteration (one 128-byte row segment)
constexpr int kDmStages = 3;
constexpr int kDmThreads = 256;  // 8 warps x 16 rows
constexpr int kDmXStride = kDmK; // doubles per staged X row (swizzled like the operator rows)

__host__ __device__ inline size_t dmma_stage_doubles(int np, int nt) {
  return (size_t)np * kDmM * kDmK + (size_t)nt * 8 * kDmXStride;
}

__device__ __forceinline__ void cp_async16_zfill(uint32_t saddr, const void* g, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(g), "r"(bytes) : "memory");
}
__device__ __forceinline__ void dcommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void dwait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// C += A B over k = 16: the k = 4 fragments of four consecutive K chunks
// (a[2c], a[2c + 1] and b[c] of chunk c), one instruction
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// C += A B over k = 8: the k = 4 fragments of two consecutive K chunks (a0,
// a1 and b0 of chunk 0, a2, a3 and b1 of chunk 1), one instruction
__device__ __forceinline__ void dmma8(double (&c)[4], double a0, double a1, double a2, double a3, double b0,
                                      double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

struct DmArgs {
  const double* are;
  const double* aim;
  const double* xr;
  const double* xi;
  double* ws;
  int n, b, N, NT;
  long tiles, kchunks, total;
  int slots;
};

// 16-byte chunk c (0..3) of operator row r inside a staged plane, in doubles
__device__ __forceinline__ int dm_aoff(int r, int c) { return r * kDmK + ((c ^ (r & 7)) << 1); }

template <bool CPLX, int NT>
__global__ void __launch_bounds__(kDmThreads, (NT <= 6 ? 2 : 1)) k_block_matvec_dmma(DmArgs g) {
  constexpr int NP = CPLX ? 2 : 1;
  extern __shared__ __align__(128) double dsm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gq = lane >> 2, tq = lane & 3;  // fragment group / thread-in-group
  const int n = g.n, b = g.b, N = g.N;
  const size_t stage_d = dmma_stage_doubles(NP, NT);
  const long it0 = sk_begin(blockIdx.x, g.total, gridDim.x);
  const long it1 = sk_begin(blockIdx.x + 1, g.total, gridDim.x);
  const long first_tile = it0 / g.kchunks;

  // zero the X pad rows of every stage once (cp.async never writes them)
  for (int s = 0; s < kDmStages; ++s) {
    double* xs = dsm + s * stage_d + (size_t)NP * kDmM * kDmK;
    for (int e = tid; e < (NT * 8 - N) * kDmXStride; e += kDmThreads) xs[N * kDmXStride + e] = 0.0;
  }
  // dependent launch: the operand blocks are the previous kernel's output
  asm volatile("griddepcontrol.wait;" ::: "memory");

  auto load = [&](long it, int stage) {
    const long tile = it / g.kchunks;
    const long k0 = (it % g.kchunks) * kDmK;
    double* base = dsm + stage * stage_d;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(base);
    // operator planes: 128 rows x 4 chunks per plane
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const double* pl = p == 0 ? g.are : g.aim;
#pragma unroll
      for (int u = 0; u < kDmM * (kDmK / 2) / kDmThreads; ++u) {
        const int e = tid + u * kDmThreads;
        const int r = e / (kDmK / 2), ch = e % (kDmK / 2);
        const long row = tile * kDmM + r, col = k0 + 2 * ch;
        const bool ok = row < n && col < n;
        const double* src = ok ? pl + row * n + col : pl;
        const uint32_t dst = sbase + (uint32_t)((p * kDmM * kDmK + dm_aoff(r, ch)) * 8);
        cp_async16_zfill(dst, src, ok ? 16 : 0);
      }
    }
    // X slice: N rows x 4 chunks
    const uint32_t xbase = sbase + (uint32_t)(NP * kDmM * kDmK * 8);
    for (int e = tid; e < N * (kDmK / 2); e += kDmThreads) {
      const int r = e / (kDmK / 2), ch = e % (kDmK / 2);
      const long col = k0 + 2 * ch;
      const double* pl = (CPLX && r >= b) ? g.xi + (long)(r - b) * n : g.xr + (long)r * n;
      const bool ok = col < n;
      cp_async16_zfill(xbase + (uint32_t)(dm_aoff(r, ch) * 8), ok ? pl + col : pl, ok ? 16 : 0);
    }
  };

  // per-lane B2 row / sign of n-tile j (B1 row is the column j * 8 + gq)
  int r2[NT];
  double sg[NT];
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    const int c = j * 8 + gq;
    if (CPLX && c < 2 * b) {
      r2[j] = c < b ? c + b : c - b;
      sg[j] = c < b ? -1.0 : 1.0;
    } else {
      r2[j] = c;
      sg[j] = 1.0;
    }
  }

  double acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;

  auto flush = [&](long tile) {
    const int slot = (int)(tile - first_tile);
    double* out = g.ws + ((size_t)blockIdx.x * g.slots + slot) * (size_t)NP * b * kDmM;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int row = warp * 16 + gq + (e >> 1) * 8;
        const int col = j * 8 + 2 * tq + (e & 1);
        if (col < N) {
          const int plane = col < b ? 0 : 1;
          const int q = col - plane * b;
          out[((size_t)plane * b + q) * kDmM + row] = acc[j][e];
        }
        acc[j][e] = 0.0;
      }
    }
  };

#pragma unroll
  for (int s = 0; s < kDmStages - 1; ++s) {
    if (it0 + s < it1) load(it0 + s, s);
    dcommit();
  }
  for (long it = it0; it < it1; ++it) {
    dwait<kDmStages - 2>();
    __syncthreads();
    {
      const long nx = it + kDmStages - 1;
      if (nx < it1) load(nx, (int)((nx - it0) % kDmStages));
      dcommit();
    }
    const double* base = dsm + (size_t)((it - it0) % kDmStages) * stage_d;
    const double* xs = base + (size_t)NP * kDmM * kDmK;
    const int ra = warp * 16 + gq;  // rows ra and ra + 8 share the swizzle
    // the stage's 16 columns as one m16n8k16 per plane and n-tile: the
    // k = 4 fragments of the four K chunks (A rows ra, ra + 8; B row kk)
    static_assert(kDmK == 16, "one k = 16 MMA per stage");
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      double a[8];
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4) {
        const int kk = c4 * 4 + tq;
        const int off = p * kDmM * kDmK + dm_aoff(ra, kk >> 1) + (kk & 1);
        a[2 * c4] = base[off];
        a[2 * c4 + 1] = base[off + 8 * kDmK];
      }
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        double bv[4];
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
          const int kk = c4 * 4 + tq;
          bv[c4] = p == 0 ? xs[dm_aoff(j * 8 + gq, kk >> 1) + (kk & 1)]
                          : sg[j] * xs[dm_aoff(r2[j], kk >> 1) + (kk & 1)];
        }
        dmma16(acc[j], a, bv);
      }
    }
    if ((it + 1) % g.kchunks == 0 || it + 1 == it1) flush(it / g.kchunks);
  }
  dwait<0>();
}

// grid of `ctas` CTAs over the iterations of an n x n operator
static DmmaPlan dmma_grid(int n, long ctas) {
  const SkGrid k = sk_grid((n + kDmM - 1) / kDmM, (n + kDmK - 1) / kDmK, ctas);
  DmmaPlan p;
  p.n = n;
  p.tiles = k.tiles;
  p.kchunks = k.kchunks;
  p.total = k.total;
  p.grid = k.grid;
  p.slots = k.slots;
  return p;
}

bool dmma_plan(int n, DmmaPlan* p) {
  if (n < 2 || n % 2) return false;
  *p = dmma_grid(n, kNumSMs);
  return true;
}

// workspace for either occupancy (one or two CTAs per SM)
size_t dmma_workspace(const DmmaPlan& p) {
  size_t best = 0;
  for (long occ = 1; occ <= 2; ++occ) {
    const DmmaPlan q = dmma_grid(p.n, kNumSMs * occ);
    const size_t need = (size_t)q.grid * q.slots * 2 * 32 * kDmM;
    if (need > best) best = need;
  }
  return best;
}

template <bool CPLX, int NT>
static int dmma_launch(const DmArgs& g0, int n, double* wr, double* wi, cudaStream_t s) {
  auto kern = k_block_matvec_dmma<CPLX, NT>;
  const size_t smem = dmma_stage_doubles(CPLX ? 2 : 1, NT) * kDmStages * sizeof(double);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return OAPB_ERR_CUDA;
  int occ = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kDmThreads, smem) != cudaSuccess || occ < 1)
    return OAPB_ERR_CUDA;
  if (occ > 2) occ = 2;
  const DmmaPlan p = dmma_grid(n, (long)kNumSMs * occ);
  DmArgs g = g0;
  g.tiles = p.tiles;
  g.kchunks = p.kchunks;
  g.total = p.total;
  g.slots = p.slots;
  launch_dependent(kern, dim3(p.grid), dim3(kDmThreads), smem, s, g);
  const SkGrid sg{p.tiles, p.kchunks, p.total, p.grid, p.slots};
  launch_sk_reduce<CPLX>(g.ws, sg, n, g.b, wr, wi, s);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

int launch_block_matvec_dmma(const double* Are, const double* Aim, int n, const double* xr, const double* xi,
                             int b, double* wr, double* wi, const DmmaPlan& p, double* ws, cudaStream_t s) {
  const bool cplx = Aim != nullptr;
  if (b < 1 || b > 32 || (cplx && (!xi || !wi))) return OAPB_ERR_ARG;
  (void)p;
  DmArgs g{Are, Aim, xr, xi, ws, n, b, cplx ? 2 * b : b, 0, 0, 0, 0, 0};
  g.NT = (g.N + 7) / 8;
  if (cplx) {
    switch (g.NT) {
      case 1: return dmma_launch<true, 1>(g, n, wr, wi, s);
      case 2: return dmma_launch<true, 2>(g, n, wr, wi, s);
      case 3: return dmma_launch<true, 3>(g, n, wr, wi, s);
      case 4: return dmma_launch<true, 4>(g, n, wr, wi, s);
      case 5: return dmma_launch<true, 5>(g, n, wr, wi, s);
      case 6: return dmma_launch<true, 6>(g, n, wr, wi, s);
      case 7: return dmma_launch<true, 7>(g, n, wr, wi, s);
      default: return dmma_launch<true, 8>(g, n, wr, wi, s);
    }
  }
  switch (g.NT) {
    case 1: return dmma_launch<false, 1>(g, n, wr, nullptr, s);
    case 2: return dmma_launch<false, 2>(g, n, wr, nullptr, s);
    case 3: return dmma_launch<false, 3>(g, n, wr, nullptr, s);
    default: return dmma_launch<false, 4>(g, n, wr, nullptr, s);
  }
}

}  // namespace oapb
