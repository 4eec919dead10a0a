// Host interface of the FP64-class block operator pass on the integer
// tensor cores (blocki8.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace oapb {

constexpr int kI8SlicesA = 6;  // operator slices (7 bits each below a power-of-two row scale)
constexpr int kI8SlicesX = 7;  // vector slices (7 bits each below a power-of-two vector scale)

// Operator as int8 slices: slice i of plane p (0 = re, 1 = im) is the n x kp
// matrix at slices + (p * kI8SlicesA + i) n kp (kp = n rounded up to 128,
// zero-padded columns); rscale[r] = 2^e_r, the power of two above row r of
// both planes.  cplx = false: plane 0 only.
struct I8Operator {
  const int8_t* slices;
  const double* rscale;
  int n, kp;
  bool cplx;
};

// Bytes of the sliced operator of an n x n (complex: two-plane) operator.
inline size_t i8_operator_bytes(int n, int kp, bool cplx) {
  return (size_t)(cplx ? 2 : 1) * kI8SlicesA * (size_t)n * kp;
}
// Bytes of the vector-slice scratch (b <= 32 vectors) and doubles of its
// scales (kI8BlockScales) followed by the partial maxima of the scale pass.
inline size_t i8_block_bytes(int kp) { return (size_t)kI8SlicesX * 64 * kp; }
constexpr int kI8BlockScales = 64;
constexpr int kI8ScaleDoubles = kI8BlockScales + 148 * 32;

// Slices of rows row0 .. row0 + rows - 1 (rows < 0: to the last row) of the
// FP64 operator (aim NULL for a real operator).
int split_operator_i8(const double* are, const double* aim, int n, int kp, int8_t* slices, double* rscale,
                      cudaStream_t s, long row0 = 0, long rows = -1);

// Largest b the pass takes (complex / real operator).
inline int i8_max_vectors(bool cplx) { return cplx ? 16 : 32; }

// Doubles of stream-K partial workspace for an n x n operator.
size_t i8_workspace(int n, int kp);

// W (planes wr / wi, vector q at offset q n) = A X for b <= i8_max_vectors
// vectors (X vector-contiguous FP64).  xs: i8_block_bytes(kp) bytes, xscale:
// kI8ScaleDoubles doubles, ws: i8_workspace() doubles; *err receives
// timeout bits.  kev (optional, two events): recorded right before and after
// the pass kernel alone (profiling; breaks the dependent-launch overlap with
// the kernels around it).
int launch_block_matvec_i8(const I8Operator& op, const double* xr, const double* xi, int b, double* wr, double* wi,
                           int8_t* xs, double* xscale, double* ws, int* err, cudaStream_t s,
                           const cudaEvent_t* kev = nullptr);

}  // namespace oapb
