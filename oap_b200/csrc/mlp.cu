// Warm-start network and parametric operators.
//
// 1. oapb_param_operators: A(theta_p) = A0 + sum_i theta_p[i] B_i for a batch
//    of parameter vectors (each basis element read once, written P times).
// 2. A dense MLP with BF16 weights and activations and FP32 accumulation:
//    forward, backward (data and weight gradients) and an Adam step on FP32
//    master weights, all on the device.  Each layer's outputs pass through
//    one of the reference's activations (oapNeuralHost/oapLayerStructure.h:
//    32-38, applied by activateFunc / derivativeFunc,
//    oapGenericNeuralApi.h:43-120): LINEAR, SIGMOID, TANH or SIN; by
//    default tanh hidden layers and a linear output.
//    The network maps an operator's parameters theta to a warm-start vector
//    and a shift set for the Arnoldi method.  Nearest reference analogue:
//    the generic forward / back-propagation of the neural library
//    (oapNeuralHost/oapGenericNeuralApi.h:195-360) over CuProceduresApi ops
//    (dotProduct, tensorProduct, sum).
//
// Every layer product is one kernel: C[M x N] = sum_k A(m, k) B(n, k) with
// strided BF16 operands (the forward product, the data gradient and the
// weight gradient differ only in strides), 32 x 32 output tiles, FP32
// accumulation, optional bias + activation epilogue (the pre-activation
// kept for SIN, whose derivative needs it) and a BF16 copy of the output.
#include <cuda_bf16.h>
#include <math.h>

#include <new>
#include <vector>

#include "common.cuh"
#include "matio.cuh"

namespace oapb {

// ------------------------------------------------------ parametric operator
__global__ void k_param_operators(const double* __restrict__ A0, const double* const* __restrict__ Bs, int nparams,
                                  const double* __restrict__ theta, int P, long nn, double* __restrict__ out) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (long)gridDim.x * blockDim.x) {
    double base = A0[e];
    double b[32];
    for (int i = 0; i < nparams; ++i) b[i] = Bs[i][e];
    for (int p = 0; p < P; ++p) {
      double v = base;
      for (int i = 0; i < nparams; ++i) v += theta[(long)p * nparams + i] * b[i];
      out[(long)p * nn + e] = v;
    }
  }
}

// ------------------------------------------------------------ layer GEMM --
constexpr int kLT = 32;  // output tile
constexpr int kLK = 16;  // k chunk

// activation of a layer's outputs (oapb_activation) and its derivative from
// the pre-activation z and the output h
__device__ __forceinline__ float act_f(float z, int act) {
  switch (act) {
    case OAPB_ACT_SIGMOID: return 1.f / (1.f + expf(-z));
    case OAPB_ACT_TANH: return tanhf(z);
    case OAPB_ACT_SIN: return sinf(z);
    default: return z;
  }
}
__device__ __forceinline__ float act_df(float z, float h, int act) {
  switch (act) {
    case OAPB_ACT_SIGMOID: return h * (1.f - h);
    case OAPB_ACT_TANH: return 1.f - h * h;
    case OAPB_ACT_SIN: return cosf(z);
    default: return 1.f;
  }
}

// C[m][n] (ldc) = sum_k A[m*sam + k*sak] * B[n*sbn + k*sbk]; with EPI:
// z = C + bias[n] (kept in Z when given), C = act(z)
template <bool EPI>
__global__ void __launch_bounds__(256) k_layer_gemm(const __nv_bfloat16* __restrict__ A, long sam, long sak,
                                                    const __nv_bfloat16* __restrict__ Bm, long sbn, long sbk, int M,
                                                    int N, int K, const float* __restrict__ bias, int act, float* C,
                                                    float* Z, __nv_bfloat16* Cb, int ldc) {
  __shared__ float As[kLK][kLT + 1];
  __shared__ float Bsm[kLK][kLT + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads, 2 x 2 outputs each
  const int m0 = blockIdx.y * kLT, n0 = blockIdx.x * kLT;
  float acc[2][2] = {{0, 0}, {0, 0}};
  for (int k0 = 0; k0 < K; k0 += kLK) {
    for (int e = threadIdx.x; e < kLK * kLT; e += 256) {
      const int kk = e / kLT, j = e % kLT;
      const int m = m0 + j, n = n0 + j, k = k0 + kk;
      As[kk][j] = (m < M && k < K) ? __bfloat162float(A[m * sam + k * sak]) : 0.f;
      Bsm[kk][j] = (n < N && k < K) ? __bfloat162float(Bm[n * sbn + k * sbk]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kLK; ++kk) {
      const float a0 = As[kk][ty * 2], a1 = As[kk][ty * 2 + 1];
      const float b0 = Bsm[kk][tx * 2], b1 = Bsm[kk][tx * 2 + 1];
      acc[0][0] = fmaf(a0, b0, acc[0][0]);
      acc[0][1] = fmaf(a0, b1, acc[0][1]);
      acc[1][0] = fmaf(a1, b0, acc[1][0]);
      acc[1][1] = fmaf(a1, b1, acc[1][1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int m = m0 + ty * 2 + i, n = n0 + tx * 2 + j;
      if (m < M && n < N) {
        float v = acc[i][j];
        if (EPI) {
          v += bias[n];
          if (Z) Z[(long)m * ldc + n] = v;
          v = act_f(v, act);
        }
        if (C) C[(long)m * ldc + n] = v;
        if (Cb) Cb[(long)m * ldc + n] = __float2bfloat16_rn(v);
      }
    }
}

// dY = (Y - T) / B (FP32, and BF16 for the backward products when given);
// loss partial sums
__global__ void k_mse_grad(const float* Y, const float* T, int B, long len, __nv_bfloat16* dYb, float* dYf,
                           double* loss) {
  double s = 0;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x) {
    const float d = Y[e] - T[e];
    s += (double)d * d;
    const float g = d / (float)B;
    if (dYb) dYb[e] = __float2bfloat16_rn(g);
    if (dYf) dYf[e] = g;
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, 0.5 * s / B);
}

// dZ = dH * act'(z) (from the output h, or the pre-activation z for SIN),
// FP32 and BF16 out
__global__ void k_act_grad(const float* dH, const float* H, const float* Z, int act, long len,
                           __nv_bfloat16* dZb, float* dZf) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x) {
    const float g = dH[e] * act_df(Z ? Z[e] : 0.f, H[e], act);
    dZb[e] = __float2bfloat16_rn(g);
    if (dZf) dZf[e] = g;
  }
}

// db[n] = sum_b dZ[b][n]
__global__ void k_bias_grad(const float* dZ, int B, int N, float* db) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    float s = 0;
    for (int b = 0; b < B; ++b) s += dZ[(long)b * N + n];
    db[n] = s;
  }
}

// Adam on FP32 masters; BF16 working copy refreshed
__global__ void k_adam(float* w, const float* g, float* m1, float* m2, long len, float lr, float b1, float b2,
                       float eps, float c1, float c2, __nv_bfloat16* wb) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x) {
    const float gg = g[e];
    const float a = b1 * m1[e] + (1.f - b1) * gg;
    const float v = b2 * m2[e] + (1.f - b2) * gg * gg;
    m1[e] = a;
    m2[e] = v;
    const float nw = w[e] - lr * (a / c1) / (sqrtf(v / c2) + eps);
    w[e] = nw;
    if (wb) wb[e] = __float2bfloat16_rn(nw);
  }
}

__global__ void k_to_bf16(const float* x, long len, __nv_bfloat16* y) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x)
    y[e] = __float2bfloat16_rn(x[e]);
}

__global__ void k_init_uniform(float* w, long len, float scale, uint64_t seed) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (long)gridDim.x * blockDim.x)
    w[e] = (float)(scale * uniform_pm1(seed, (uint64_t)e));
}

}  // namespace oapb

using namespace oapb;

struct oapb_mlp {
  int nl = 0;                 // layers
  std::vector<int> sz;        // nl + 1 sizes
  std::vector<long> woff, boff;
  long nparam = 0;
  float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;  // FP32 [all weights | all biases]
  __nv_bfloat16* wb = nullptr;                                     // BF16 copy of the weights
  int step = 0;
  std::vector<int> act;                // activation of each layer's outputs (oapb_activation)
  // activations for the last forward (capacity batch)
  int cap = 0;
  std::vector<float*> hf;              // FP32 activations per layer output (nl)
  std::vector<float*> zf;              // FP32 pre-activations per layer output (nl)
  std::vector<__nv_bfloat16*> hb;      // BF16 activations: input + per layer
  float *dA = nullptr, *dB2 = nullptr; // FP32 gradient scratch (cap x max size)
  __nv_bfloat16 *dAb = nullptr;
  double* loss = nullptr;
};

namespace {

int g_mlp_free_acts(oapb_mlp* h) {
  for (auto p : h->hf) cudaFree(p);
  for (auto p : h->hb) cudaFree(p);
  for (auto p : h->zf) cudaFree(p);
  h->hf.clear();
  h->hb.clear();
  h->zf.clear();
  if (h->dA) cudaFree(h->dA);
  if (h->dB2) cudaFree(h->dB2);
  if (h->dAb) cudaFree(h->dAb);
  h->dA = h->dB2 = nullptr;
  h->dAb = nullptr;
  h->cap = 0;
  return OAPB_OK;
}

int ensure_acts(oapb_mlp* h, int batch) {
  if (batch <= h->cap) return OAPB_OK;
  g_mlp_free_acts(h);
  int mx = 0;
  for (int s : h->sz) mx = s > mx ? s : mx;
  h->hb.resize(h->nl + 1, nullptr);
  h->hf.resize(h->nl, nullptr);
  h->zf.resize(h->nl, nullptr);
  for (int l = 0; l <= h->nl; ++l)
    if (cudaMalloc(&h->hb[l], sizeof(__nv_bfloat16) * (size_t)batch * h->sz[l]) != cudaSuccess) return OAPB_ERR_NOMEM;
  for (int l = 0; l < h->nl; ++l)
    if (cudaMalloc(&h->hf[l], sizeof(float) * (size_t)batch * h->sz[l + 1]) != cudaSuccess ||
        cudaMalloc(&h->zf[l], sizeof(float) * (size_t)batch * h->sz[l + 1]) != cudaSuccess)
      return OAPB_ERR_NOMEM;
  if (cudaMalloc(&h->dA, sizeof(float) * (size_t)batch * mx) != cudaSuccess ||
      cudaMalloc(&h->dB2, sizeof(float) * (size_t)batch * mx) != cudaSuccess ||
      cudaMalloc(&h->dAb, sizeof(__nv_bfloat16) * (size_t)batch * mx) != cudaSuccess)
    return OAPB_ERR_NOMEM;
  h->cap = batch;
  return OAPB_OK;
}

void layer_gemm(bool epi, int act, const __nv_bfloat16* A, long sam, long sak, const __nv_bfloat16* Bm, long sbn,
                long sbk, int M, int N, int K, const float* bias, float* C, float* Z, __nv_bfloat16* Cb, int ldc,
                cudaStream_t s) {
  dim3 grid((N + kLT - 1) / kLT, (M + kLT - 1) / kLT);
  if (epi)
    k_layer_gemm<true><<<grid, 256, 0, s>>>(A, sam, sak, Bm, sbn, sbk, M, N, K, bias, act, C, Z, Cb, ldc);
  else
    k_layer_gemm<false><<<grid, 256, 0, s>>>(A, sam, sak, Bm, sbn, sbk, M, N, K, bias, act, C, Z, Cb, ldc);
}

int forward_impl(oapb_mlp* h, const float* x, int B, cudaStream_t s) {
  int rc = ensure_acts(h, B);
  if (rc) return rc;
  const long n0 = (long)B * h->sz[0];
  k_to_bf16<<<grid_for(n0, 256), 256, 0, s>>>(x, n0, h->hb[0]);
  for (int l = 0; l < h->nl; ++l) {
    const int in = h->sz[l], out = h->sz[l + 1];
    const __nv_bfloat16* W = h->wb + h->woff[l];
    const float* bias = h->w + h->boff[l];
    layer_gemm(true, h->act[l], h->hb[l], in, 1, W, in, 1, B, out, in, bias, h->hf[l],
               h->act[l] == OAPB_ACT_SIN ? h->zf[l] : nullptr, h->hb[l + 1], out, s);
  }
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

}  // namespace

extern "C" {

int oapb_param_operators(const double* A0, const double* const* B, uint32_t nparams, const double* theta,
                         uint32_t count, uint32_t n, double* out, void* stream) {
  if (!A0 || !B || !theta || !out || nparams == 0 || nparams > 32 || count == 0 || n == 0) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const double** dB = nullptr;
  if (cudaMallocAsync((void**)&dB, sizeof(double*) * nparams, s) != cudaSuccess) return OAPB_ERR_NOMEM;
  int rc = OAPB_OK;
  if (cudaMemcpyAsync(dB, B, sizeof(double*) * nparams, cudaMemcpyHostToDevice, s) != cudaSuccess) rc = OAPB_ERR_CUDA;
  if (!rc) {
    const long nn = (long)n * n;
    k_param_operators<<<grid_for(nn, 256, kNumSMs * 8), 256, 0, s>>>(A0, dB, (int)nparams, theta, (int)count, nn,
                                                                      out);
    if (cudaGetLastError() != cudaSuccess) rc = OAPB_ERR_CUDA;
  }
  cudaFreeAsync(dB, s);
  return rc;
}

int oapb_mlp_create(oapb_mlp** out, const uint32_t* sizes, uint32_t nlayers, uint64_t seed) {
  if (!out || !sizes || nlayers < 1 || nlayers > 8) return OAPB_ERR_ARG;
  oapb_mlp* h = new (std::nothrow) oapb_mlp();
  if (!h) return OAPB_ERR_NOMEM;
  h->nl = (int)nlayers;
  for (uint32_t i = 0; i <= nlayers; ++i) {
    if (sizes[i] == 0) {
      delete h;
      return OAPB_ERR_ARG;
    }
    h->sz.push_back((int)sizes[i]);
  }
  long off = 0;
  for (int l = 0; l < h->nl; ++l) {
    h->woff.push_back(off);
    off += (long)h->sz[l] * h->sz[l + 1];
  }
  const long nw = off;
  for (int l = 0; l < h->nl; ++l) {
    h->boff.push_back(off);
    off += h->sz[l + 1];
  }
  h->nparam = off;
  h->act.assign(h->nl, OAPB_ACT_TANH);
  h->act[h->nl - 1] = OAPB_ACT_LINEAR;
  const size_t fb = sizeof(float) * (size_t)off;
  if (cudaMalloc(&h->w, fb) != cudaSuccess || cudaMalloc(&h->g, fb) != cudaSuccess ||
      cudaMalloc(&h->m1, fb) != cudaSuccess || cudaMalloc(&h->m2, fb) != cudaSuccess ||
      cudaMalloc(&h->wb, sizeof(__nv_bfloat16) * (size_t)off) != cudaSuccess ||
      cudaMalloc(&h->loss, sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return OAPB_ERR_NOMEM;
  }
  cudaMemset(h->m1, 0, fb);
  cudaMemset(h->m2, 0, fb);
  cudaMemset(h->g, 0, fb);
  // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases
  for (int l = 0; l < h->nl; ++l) {
    const long len = (long)h->sz[l] * h->sz[l + 1];
    k_init_uniform<<<grid_for(len, 256), 256>>>(h->w + h->woff[l], len, 1.0f / sqrtf((float)h->sz[l]),
                                                 seed * 1315423911ull + l);
  }
  cudaMemset(h->w + nw, 0, sizeof(float) * (size_t)(off - nw));
  k_to_bf16<<<grid_for(off, 256), 256>>>(h->w, off, h->wb);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    delete h;
    return OAPB_ERR_CUDA;
  }
  *out = h;
  return OAPB_OK;
}

int oapb_mlp_destroy(oapb_mlp* h) {
  if (!h) return OAPB_ERR_ARG;
  cudaDeviceSynchronize();
  g_mlp_free_acts(h);
  cudaFree(h->w);
  cudaFree(h->g);
  cudaFree(h->m1);
  cudaFree(h->m2);
  cudaFree(h->wb);
  cudaFree(h->loss);
  delete h;
  return OAPB_OK;
}

uint64_t oapb_mlp_num_params(const oapb_mlp* h) { return h ? (uint64_t)h->nparam : 0; }

int oapb_mlp_forward(oapb_mlp* h, const float* x, uint32_t batch, float* y, void* stream) {
  if (!h || !x || batch == 0) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = forward_impl(h, x, (int)batch, s);
  if (rc) return rc;
  if (y && cudaMemcpyAsync(y, h->hf[h->nl - 1], sizeof(float) * (size_t)batch * h->sz[h->nl],
                           cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  return OAPB_OK;
}

// Forward + backward of loss = 1/(2B) sum (y - target)^2; gradients (FP32,
// same packing as the parameters) stay in the handle.  *loss_out (host,
// may be NULL) receives the loss (synchronises the stream).
int oapb_mlp_backward(oapb_mlp* h, const float* x, const float* target, uint32_t batch, double* loss_out,
                      void* stream) {
  if (!h || !x || !target || batch == 0) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int B = (int)batch;
  int rc = forward_impl(h, x, B, s);
  if (rc) return rc;
  if (cudaMemsetAsync(h->loss, 0, sizeof(double), s) != cudaSuccess) return OAPB_ERR_CUDA;
  const int L = h->nl;
  const long lenY = (long)B * h->sz[L];
  // dZ of the output layer into dAb (BF16) / dA (FP32): dY itself for a
  // linear output, else dY through the activation's derivative
  if (h->act[L - 1] == OAPB_ACT_LINEAR) {
    k_mse_grad<<<grid_for(lenY, 256), 256, 0, s>>>(h->hf[L - 1], target, B, lenY, h->dAb, h->dA, h->loss);
  } else {
    k_mse_grad<<<grid_for(lenY, 256), 256, 0, s>>>(h->hf[L - 1], target, B, lenY, nullptr, h->dB2, h->loss);
    k_act_grad<<<grid_for(lenY, 256), 256, 0, s>>>(h->dB2, h->hf[L - 1], h->zf[L - 1], h->act[L - 1], lenY, h->dAb,
                                                    h->dA);
  }
  for (int l = L - 1; l >= 0; --l) {
    const int in = h->sz[l], out = h->sz[l + 1];
    // dZ (B x out) in dAb / dA; weight gradient dW[o][i] = sum_b dZ[b][o] X[b][i]
    layer_gemm(false, 0, h->dAb, 1, out, h->hb[l], 1, in, out, in, B, nullptr, h->g + h->woff[l], nullptr, nullptr,
               in, s);
    k_bias_grad<<<grid_for(out, 256), 256, 0, s>>>(h->dA, B, out, h->g + h->boff[l]);
    if (l == 0) break;
    // data gradient dX[b][i] = sum_o dZ[b][o] W[o][i], then through layer
    // l - 1's activation
    const __nv_bfloat16* W = h->wb + h->woff[l];
    layer_gemm(false, 0, h->dAb, out, 1, W, 1, in, B, in, out, nullptr, h->dB2, nullptr, nullptr, in, s);
    k_act_grad<<<grid_for((long)B * in, 256), 256, 0, s>>>(h->dB2, h->hf[l - 1], h->zf[l - 1], h->act[l - 1],
                                                            (long)B * in, h->dAb, h->dA);
  }
  if (cudaGetLastError() != cudaSuccess) return OAPB_ERR_CUDA;
  if (loss_out) {
    if (cudaMemcpyAsync(loss_out, h->loss, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return OAPB_ERR_CUDA;
  }
  return OAPB_OK;
}

int oapb_mlp_adam_step(oapb_mlp* h, float lr, void* stream) {
  if (!h || !(lr > 0)) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  h->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)h->step), c2 = 1.f - powf(b2, (float)h->step);
  k_adam<<<grid_for(h->nparam, 256), 256, 0, s>>>(h->w, h->g, h->m1, h->m2, h->nparam, lr, b1, b2, 1e-8f, c1, c2,
                                                   h->wb);
  return cudaGetLastError() == cudaSuccess ? OAPB_OK : OAPB_ERR_CUDA;
}

// which: 0 parameters (FP32 masters), 1 gradients; dst/src device or host
int oapb_mlp_copy(oapb_mlp* h, int which, float* dst, void* stream) {
  if (!h || !dst || which < 0 || which > 1) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(dst, which ? h->g : h->w, sizeof(float) * (size_t)h->nparam, cudaMemcpyDefault, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  return OAPB_OK;
}

int oapb_mlp_set_params(oapb_mlp* h, const float* src, void* stream) {
  if (!h || !src) return OAPB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(h->w, src, sizeof(float) * (size_t)h->nparam, cudaMemcpyDefault, s) != cudaSuccess)
    return OAPB_ERR_CUDA;
  k_to_bf16<<<grid_for(h->nparam, 256), 256, 0, s>>>(h->w, h->nparam, h->wb);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return OAPB_ERR_CUDA;
  return OAPB_OK;
}

int oapb_mlp_set_activations(oapb_mlp* h, const int32_t* acts, uint32_t count) {
  if (!h || !acts || count != (uint32_t)h->nl) return OAPB_ERR_ARG;
  for (uint32_t l = 0; l < count; ++l)
    if (acts[l] < OAPB_ACT_LINEAR || acts[l] > OAPB_ACT_SIN) return OAPB_ERR_ARG;
  for (uint32_t l = 0; l < count; ++l) h->act[l] = acts[l];
  return OAPB_OK;
}

int oapb_mlp_get_activations(const oapb_mlp* h, int32_t* acts, uint32_t count) {
  if (!h || !acts || count != (uint32_t)h->nl) return OAPB_ERR_ARG;
  for (uint32_t l = 0; l < count; ++l) acts[l] = h->act[l];
  return OAPB_OK;
}

uint32_t oapb_mlp_num_layers(const oapb_mlp* h, uint32_t* sizes) {
  if (!h) return 0;
  if (sizes)
    for (int i = 0; i <= h->nl; ++i) sizes[i] = (uint32_t)h->sz[i];
  return (uint32_t)h->nl;
}

// File (the reference's matrix format, matio.cuh): sizes (1 column x
// nlayers + 1 rows), then per layer its weights (in columns x out rows) and
// biases (1 column x out rows), FP64 values of the FP32 master weights, and
// last the layers' activations (1 column x nlayers rows, oapb_activation
// values; a file without it loads with the default activations).
int oapb_mlp_save(oapb_mlp* h, const char* path) {
  if (!h || !path) return OAPB_ERR_ARG;
  std::vector<float> p((size_t)h->nparam);
  int rc = oapb_mlp_copy(h, 0, p.data(), nullptr);
  if (rc) return rc;
  std::vector<char> payload;
  HostMat sz;
  sz.columns = 1;
  sz.rows = (uint32_t)(h->nl + 1);
  for (int v : h->sz) sz.re.push_back((double)v);
  matio_append(payload, sz);
  for (int l = 0; l < h->nl; ++l) {
    HostMat W, bv;
    W.columns = (uint32_t)h->sz[l];
    W.rows = (uint32_t)h->sz[l + 1];
    W.re.assign(p.begin() + h->woff[l], p.begin() + h->woff[l] + (long)W.columns * W.rows);
    bv.columns = 1;
    bv.rows = W.rows;
    bv.re.assign(p.begin() + h->boff[l], p.begin() + h->boff[l] + W.rows);
    matio_append(payload, W);
    matio_append(payload, bv);
  }
  HostMat acts;
  acts.columns = 1;
  acts.rows = (uint32_t)h->nl;
  for (int a : h->act) acts.re.push_back((double)a);
  matio_append(payload, acts);
  return matio_write_file(path, payload);
}

int oapb_mlp_load(oapb_mlp** out, const char* path, uint64_t seed) {
  if (!out || !path) return OAPB_ERR_ARG;
  std::vector<char> payload;
  int rc = matio_read_file(path, &payload);
  if (rc) return rc;
  size_t off = 0;
  HostMat sz;
  if (!matio_parse(payload, off, &sz) || sz.columns != 1 || sz.rows < 2 || sz.rows > 9) return OAPB_ERR_ARG;
  std::vector<uint32_t> sizes;
  for (double v : sz.re) {
    if (!(v >= 1 && v < 1e9)) return OAPB_ERR_ARG;
    sizes.push_back((uint32_t)v);
  }
  const int nl = (int)sizes.size() - 1;
  std::vector<HostMat> Ws(nl), bs(nl);
  for (int l = 0; l < nl; ++l) {
    if (!matio_parse(payload, off, &Ws[l]) || !matio_parse(payload, off, &bs[l])) return OAPB_ERR_ARG;
    if (Ws[l].columns != sizes[l] || Ws[l].rows != sizes[l + 1] || bs[l].columns != 1 || bs[l].rows != sizes[l + 1])
      return OAPB_ERR_ARG;
  }
  std::vector<int32_t> acts;
  HostMat am;
  if (off < payload.size()) {
    if (!matio_parse(payload, off, &am) || am.columns != 1 || am.rows != (uint32_t)nl) return OAPB_ERR_ARG;
    for (double v : am.re) {
      if (!(v >= OAPB_ACT_LINEAR && v <= OAPB_ACT_SIN) || v != (double)(int)v) return OAPB_ERR_ARG;
      acts.push_back((int32_t)v);
    }
  }
  oapb_mlp* h = nullptr;
  if ((rc = oapb_mlp_create(&h, sizes.data(), (uint32_t)nl, seed))) return rc;
  if (!acts.empty()) oapb_mlp_set_activations(h, acts.data(), (uint32_t)nl);
  std::vector<float> p((size_t)h->nparam);
  for (int l = 0; l < nl; ++l) {
    for (size_t e = 0; e < Ws[l].re.size(); ++e) p[h->woff[l] + e] = (float)Ws[l].re[e];
    for (size_t e = 0; e < bs[l].re.size(); ++e) p[h->boff[l] + e] = (float)bs[l].re[e];
  }
  if ((rc = oapb_mlp_set_params(h, p.data(), nullptr))) {
    oapb_mlp_destroy(h);
    return rc;
  }
  *out = h;
  return OAPB_OK;
}

}  // extern "C"
