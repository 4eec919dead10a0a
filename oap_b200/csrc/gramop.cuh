// Implicit Gram operator A v = X (X^T v) on FP32 images X (rows samples x
// cols pixels, row-major) without forming A.
#pragma once

#include <cuda_runtime.h>

namespace oapb {

// row splits of the X^T v pass and the partial buffer it needs (doubles)
int gram_op_splits(int rows, int cols);
size_t gram_op_workspace(int rows, int cols);

// w = X (X^T v) (accumulate: w += X (X^T v)); v, w: rows FP64 values; ws:
// gram_op_workspace() doubles
int launch_gram_apply(const float* X, int rows, int cols, const double* v, double* w, double* ws, cudaStream_t s,
                      bool accumulate = false);

// X in host memory, applied by column blocks of block_cols pixels: the
// blocks that fit resident_bytes are copied to the device once, the others
// stream through two device buffers on every application (the copy of the
// next block overlapping the products of the current one).  hX must stay
// valid while the operator is in use.
struct GramStream;
int gram_stream_create(const float* hX, int rows, int cols, int block_cols, unsigned long long resident_bytes,
                       cudaStream_t s, GramStream** out);
void gram_stream_destroy(GramStream* g);
// w = sum_c X_c (X_c^T v), ordered on stream s
int gram_stream_apply(GramStream* g, const double* v, double* w, cudaStream_t s);
unsigned long long gram_stream_bytes(const GramStream* g);  // host-to-device bytes streamed so far
int gram_stream_resident_blocks(const GramStream* g);
int gram_stream_blocks(const GramStream* g);

}  // namespace oapb
