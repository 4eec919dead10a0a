// Self-test of the bounded device-side wait that every tensor-core kernel of
// the library uses (tc::mbar_wait: a %globaltimer-limited try_wait loop on a
// shared-memory mbarrier).
//
// One CTA initialises an mbarrier that expects one arrival and, in the
// "expire" mode, waits on it with no arrival at all: the wait runs out after
// `limit_us`, the kernel records that and returns, and the context stays
// usable.  In the "arrive" mode the same thread arrives first, so the wait
// must succeed at once.  The reference has no counterpart (its kernels never
// wait on device-side conditions; its host aborts on any CUDA error,
// oapCuda/KernelExecutor.h:34-41).
#include "common.cuh"
#include "tc.cuh"

namespace oapb {

// result word of the last self-test launch: 1 = the wait completed, 2 = it
// ran out (read back with cudaMemcpyFromSymbolAsync; nothing is allocated)
static __device__ int g_selftest_word;

__global__ void k_selftest_wait(uint64_t limit_ns, int arrive) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  tc::mbar_init(&bar, 1);
  tc::fence_mbar_init();
  if (arrive) {
    uint64_t state;
    asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(tc::smem_u32(&bar)) : "memory");
    (void)state;
  }
  const bool ok = tc::mbar_wait(&bar, 0, limit_ns);
  g_selftest_word = ok ? 1 : 2;
}

}  // namespace oapb

using namespace oapb;

extern "C" int oapb_selftest_bounded_wait(uint32_t limit_us, int32_t arrive, int32_t* timed_out, void* stream) {
  if (!timed_out || limit_us == 0 || limit_us > 1000000u) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int zero = 0;
  if (cudaMemcpyToSymbolAsync(g_selftest_word, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  k_selftest_wait<<<1, 32, 0, s>>>((uint64_t)limit_us * 1000ull, arrive ? 1 : 0);
  if (cudaGetLastError() != cudaSuccess) return OAPB_ERR_CUDA;
  int word = 0;
  if (cudaMemcpyFromSymbolAsync(&word, g_selftest_word, sizeof(int), 0, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return OAPB_ERR_CUDA;
  if (word != 1 && word != 2) return OAPB_ERR_CUDA;
  *timed_out = word == 2;
  return word == 2 ? OAPB_ERR_TIMEOUT : OAPB_OK;
}
