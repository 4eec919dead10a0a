// Givens QR without any device allocation.
//
// Some callers cannot allocate device memory: code that runs while a CUDA
// graph is being captured on a stream that forbids allocations, code inside
// an allocator callback or a memory-pool hook, and embedders whose memory
// budget is fixed at start-up.  oapb_qr_givens may allocate a global
// workspace (cudaMallocAsync) when the matrix does not fit in shared
// memory; this variant never does: its workspace is the file-scope array
// below, 2 x 128 x 128 complex FP64 values (512 KiB), which every GPU that
// loads the library holds until the process exits.  It accepts n <= 128.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (once per device, with that device current); make
// that first call before any stream capture.  The looked-up address stays
// cached for the life of the process: after cudaDeviceReset (or any reset of
// the device's primary context) the library's module is loaded again and
// the cached address no longer names the array, so do not call this entry
// point on a device after resetting it.  All calls share the array:
// calls whose kernels overlap on the GPU (different streams, or different
// host threads on one device) race on it and must be serialised by the
// caller.  The kernel overwrites the whole workspace it uses before reading
// it, so nothing has to be cleared between calls.

#include "common.cuh"

namespace oapb {

constexpr int kNoAllocMaxN = 128;

// R and Q of the one-CTA Givens QR kernel (column-independent layout of
// k_qr_givens: R then Q, n x n complex each).
static __device__ __align__(256) cplx g_qr_scratch[2 * kNoAllocMaxN * kNoAllocMaxN];

// defined in ops.cu
__global__ void k_qr_givens(const double* __restrict__ are, const double* __restrict__ aim, double* qre,
                            double* qim, double* rre, double* rim, int n, cplx* gws);

namespace {
// Device address of g_qr_scratch in the current context, looked up on every
// call (the lookup allocates nothing, and a cached address would not survive
// a reset of the context).
int scratch_address(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_qr_scratch) != cudaSuccess || !p) return OAPB_ERR_CUDA;
  *out = p;
  return OAPB_OK;
}
}  // namespace

}  // namespace oapb

using namespace oapb;

extern "C" int oapb_qr_givens_noalloc(const oapb_mat* Q, const oapb_mat* R, const oapb_mat* A, void* stream) {
  if (!Q || !R || !A) return OAPB_ERR_ARG;
  const oapb_mat* ms[3] = {Q, R, A};
  for (const oapb_mat* m : ms)
    if (m->columns == 0 || m->columns != m->rows || m->columns != A->columns || m->dtype != OAPB_F64 ||
        (!m->re && !m->im))
      return OAPB_ERR_ARG;
  const int n = (int)A->columns;
  if (n > kNoAllocMaxN) return OAPB_ERR_ARG;  // beyond the static workspace
  void* ws = nullptr;
  int rc = scratch_address(&ws);
  if (rc) return rc;
  k_qr_givens<<<1, 256, 0, (cudaStream_t)stream>>>((const double*)A->re, (const double*)A->im, (double*)Q->re,
                                                   (double*)Q->im, (double*)R->re, (double*)R->im, n, (cplx*)ws);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}
