// Tensor-memory-accelerator (TMA) helpers for this GPU's own memory: the
// driver's tensor-map encoder and 2-D tiled loads into this CTA's shared
// memory with completion counted on an mbarrier.  No load here uses cluster
// multicast.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>

#include "tc.cuh"

namespace oapb {
namespace tma {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on libcuda); nullptr when unavailable.
inline PFN_cuTensorMapEncodeTiled_v12000 encoder() {
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

// Row-major BF16 matrix (rows x cols, row stride cols elements), box of
// box_cols x box_rows elements with the given swizzle.  The base must be
// 16-byte aligned and a row a multiple of 16 bytes.
inline bool map_bf16(CUtensorMap* m, const void* base, long cols, long rows, int box_cols, int box_rows,
                     CUtensorMapSwizzle swz) {
  auto enc = encoder();
  if (!enc || ((uintptr_t)base % 16) || (cols * 2) % 16) return false;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

// 2-D tiled load (no multicast) of the box at element coordinates (x, y)
// into this CTA's shared memory at `dst`; x * element size must be a
// multiple of 16 bytes.
__device__ __forceinline__ void load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(tc::smem_u32(bar))
      : "memory");
}

// Wait for `parity` of `bar`; gives up after `limit_ns` or as soon as another
// role has given up (*abort set), and then sets *abort.
__device__ __forceinline__ bool wait(uint64_t* bar, uint32_t parity, volatile int* abort, uint64_t limit_ns) {
  const uint64_t t0 = tc::globaltimer();
  while (!tc::mbar_try_wait(bar, parity)) {
    if (*abort || tc::globaltimer() - t0 > limit_ns) {
      *abort = 1;
      return false;
    }
  }
  return true;
}

}  // namespace tma
}  // namespace oapb
