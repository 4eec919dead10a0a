// Implicit Gram operator A v = X (X^T v) on FP32 images X (rows samples x
// cols pixels, row-major) without forming A.
#pragma once

#include <cuda_runtime.h>

namespace oapb {

// row splits of the X^T v pass and the partial buffer it needs (doubles)
int gram_op_splits(int rows, int cols);
size_t gram_op_workspace(int rows, int cols);

// w = X (X^T v); v, w: rows FP64 values; ws: gram_op_workspace() doubles
int launch_gram_apply(const float* X, int rows, int cols, const double* v, double* w, double* ws, cudaStream_t s);

}  // namespace oapb
