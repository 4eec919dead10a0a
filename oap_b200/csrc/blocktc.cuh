// Host interface of the tensor-core block operator pass (blocktc.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>

#include "common.cuh"

namespace oapb {

// Operator stored as BF16 hi / lo planes, n x kp (kp = n rounded up to 128,
// zero-padded columns); aih / ail are NULL for a real operator.
struct BtcOperator {
  const __nv_bfloat16 *arh, *arl, *aih, *ail;
  int n, kp;
};

// hi / lo BF16 planes of one FP64 operator plane (rows row0 .. row0 + rows - 1;
// rows < 0: to the last row); err2 (optional) accumulates sum (a - hi)^2
int split_operator_bf16(const double* a, int n, int kp, __nv_bfloat16* hi, __nv_bfloat16* lo, cudaStream_t s,
                        long row0 = 0, long rows = -1, double* err2 = nullptr);

// Doubles of stream-K partial workspace for an n x n operator (b <= 32),
// for a grid of any CTA count from kNumSMs - 1 to kNumSMs.
size_t btc_workspace(int n, int kp);

// W (planes wr / wi, vector q at offset q n) = A X for b <= 32 vectors (X
// vector-contiguous FP64).  xbh / xbl hold 64 x kp BF16 each (the split
// block); ws: btc_workspace() doubles; *err receives timeout bits.
// bf16_only: the operator's hi planes only (half the bytes, BF16 accuracy);
// x_hi_only (with bf16_only): X rounded to BF16 as well (its lo part unused).
// ctas: stream-K CTAs (kNumSMs - 1 leaves one SM to kernels of another
// stream; every CTA holds most of its SM's shared memory).  kev (optional,
// two events): recorded right before and after the pass kernel alone
// (profiling; breaks the dependent-launch overlap with the kernels around it).
int launch_block_matvec_tc(const BtcOperator& op, const double* xr, const double* xi, int b, double* wr,
                           double* wi, __nv_bfloat16* xbh, __nv_bfloat16* xbl, double* ws, int* err,
                           cudaStream_t s, bool bf16_only = false, bool x_hi_only = false, int ctas = kNumSMs,
                           const cudaEvent_t* kev = nullptr);

}  // namespace oapb
