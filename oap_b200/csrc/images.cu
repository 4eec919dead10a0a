// Image ingestion: decoded RGB8 images -> the FP32 data matrix of the Gram
// operators, on the device.  The reference's DataLoader puts image i in
// column i of an FP64 pixels x images matrix (oapAppUtils/DataLoader.cpp:
// 47-66, 150-169) with every pixel packed as r << 16 | g << 8 | b and
// divided by 0xFFFFFF (Image::convertRgbToFloatt, oapAppUtils/Image.cpp:
// 155-180).  Here the same values go to X (images x pixels, row-major FP32),
// the layout oapb_gram_build and oapb_arnoldi_set_gram_operator take (the
// reference matrix transposed).
#include <cuda_runtime.h>

#include "common.cuh"
#include "oapb200.h"

namespace oapb {

__global__ void k_rgb_to_x(const uint8_t* __restrict__ rgb, long total, float* __restrict__ X) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const uint8_t* p = rgb + 3 * e;
    const uint32_t packed = ((uint32_t)p[0] << 16) | ((uint32_t)p[1] << 8) | (uint32_t)p[2];
    X[e] = (float)((double)packed / 16777215.0);
  }
}

}  // namespace oapb

using namespace oapb;

extern "C" int oapb_images_to_matrix(const uint8_t* rgb, int32_t rgb_on_host, uint32_t count, uint32_t pixels,
                                     float* X, void* stream) {
  if (!rgb || !X || count == 0 || pixels == 0) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const long total = (long)count * pixels;
  const uint8_t* src = rgb;
  uint8_t* staged = nullptr;
  if (rgb_on_host) {
    if (cudaMallocAsync((void**)&staged, 3 * (size_t)total, s) != cudaSuccess) return OAPB_ERR_NOMEM;
    if (cudaMemcpyAsync(staged, rgb, 3 * (size_t)total, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      cudaFreeAsync(staged, s);
      return OAPB_ERR_CUDA;
    }
    src = staged;
  }
  k_rgb_to_x<<<grid_for(total, 256, kNumSMs * 16), 256, 0, s>>>(src, total, X);
  const bool ok = cudaGetLastError() == cudaSuccess;
  if (staged) cudaFreeAsync(staged, s);
  if (!ok) return OAPB_ERR_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}
