// Test of the C++ face (include/oapb200.hpp), written like a caller of the
// reference's oap::CuProceduresApi and CuHArnoldiCallback would write it.
//   shim_test cpu   argument checks and error conversion (no GPU needed)
//   shim_test gpu   operator surface, QRGR, dense and callback solves on cuda:0
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "oapb200.hpp"

static int failures = 0;
#define EXPECT(c)                                             \
  do {                                                        \
    if (!(c)) {                                               \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      ++failures;                                             \
    }                                                         \
  } while (0)

typedef std::complex<double> cd;

static int cpu_tests() {
  EXPECT(oapb_api_version() == OAPB_API_VERSION);
  // a wanted count >= hdim is rejected before any device work
  oapb::CuHArnoldiCallback arnoldi;
  oapb::Matrix A{8, 8, nullptr, nullptr, OAPB_F64};
  arnoldi.setMatrix(&A);
  bool threw = false;
  try {
    arnoldi.execute(4, 4, oapb::MatrixInfo(true, false, 8, 8));
  } catch (const oapb::Error& e) {
    threw = e.status() == OAPB_ERR_ARG;
  }
  EXPECT(threw);
  // operator surface: NULL planes are an argument error, not a crash
  oapb::CuProceduresApi api;
  threw = false;
  try {
    api.dotProduct(&A, &A, &A);
  } catch (const oapb::Error& e) {
    threw = e.status() == OAPB_ERR_ARG;
  }
  EXPECT(threw);
  // Network: the reference's four activations are accepted, anything else
  // (and an empty layer) is an argument error
  oapb::Network net;
  net.createLayer(4);
  net.createLayer(8, oapb::Activation::SIGMOID);
  net.createLayer(8, oapb::Activation::SIN);
  threw = false;
  try {
    net.createLayer(8, static_cast<oapb::Activation>(7));
  } catch (const oapb::Error& e) {
    threw = e.status() == OAPB_ERR_ARG;
  }
  EXPECT(threw);
  threw = false;
  try {
    net.createLayer(0, oapb::Activation::TANH);
  } catch (const oapb::Error& e) {
    threw = e.status() == OAPB_ERR_ARG;
  }
  EXPECT(threw);
  EXPECT(net.getLayersCount() == 3);
  return failures;
}

struct DevMat {
  oapb::Matrix m{};
  DevMat(uint32_t c, uint32_t r, bool cplx) {
    m.columns = c;
    m.rows = r;
    m.dtype = OAPB_F64;
    cudaMalloc(&m.re, sizeof(double) * c * r);
    cudaMemset(m.re, 0, sizeof(double) * c * r);
    if (cplx) {
      cudaMalloc(&m.im, sizeof(double) * c * r);
      cudaMemset(m.im, 0, sizeof(double) * c * r);
    }
  }
  ~DevMat() {
    cudaFree(m.re);
    if (m.im) cudaFree(m.im);
  }
  void upload(const std::vector<cd>& h) {
    std::vector<double> re(h.size()), im(h.size());
    for (size_t i = 0; i < h.size(); ++i) {
      re[i] = h[i].real();
      im[i] = h[i].imag();
    }
    cudaMemcpy(m.re, re.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice);
    if (m.im) cudaMemcpy(m.im, im.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice);
  }
  std::vector<cd> download() const {
    const size_t n = (size_t)m.columns * m.rows;
    std::vector<double> re(n), im(n, 0.0);
    cudaMemcpy(re.data(), m.re, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (m.im) cudaMemcpy(im.data(), m.im, sizeof(double) * n, cudaMemcpyDeviceToHost);
    std::vector<cd> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = cd(re[i], im[i]);
    return h;
  }
};

// the user operator of the callback solve: w = A v through the api it is given
static void multiply(oapb::Matrix* w, oapb::Matrix* v, oapb::CuProceduresApi& api, void* user,
                     oapb::VecMultiplicationType) {
  api.dotProduct(w, static_cast<oapb::Matrix*>(user), v);
}

static int gpu_tests() {
  const int n = 400, k = 4, m = 24;
  std::mt19937_64 rng(3);
  std::normal_distribution<double> nd;
  // upper triangular A (row-major, element (c, r) at c + r n): the eigenvalues
  // are its diagonal, 10, 9.5, 9, ... far from the rest (|x| <= 1)
  std::vector<cd> A(n * n, 0.0);
  std::vector<cd> lam(n);
  for (int r = 0; r < n; ++r) {
    lam[r] = r < 8 ? cd(10.0 - 0.5 * r, 0.25 * (r % 3)) : cd(0.9 * std::cos(r), 0.9 * std::sin(r));
    for (int c = r; c < n; ++c) A[c + r * n] = c == r ? lam[r] : cd(0.02 * nd(rng), 0.02 * nd(rng));
  }
  DevMat dA(n, n, true);
  dA.upload(A);

  // operator surface: w = A v, magnitude
  oapb::CuProceduresApi api;
  DevMat v(1, n, true), w(1, n, true);
  std::vector<cd> hv(n);
  for (auto& x : hv) x = cd(nd(rng), nd(rng));
  v.upload(hv);
  api.dotProduct(&w.m, &dA.m, &v.m);
  std::vector<cd> hw = w.download();
  double err = 0, nrm = 0;
  for (int r = 0; r < n; ++r) {
    cd s = 0;
    for (int c = 0; c < n; ++c) s += A[c + r * n] * hv[c];
    err = std::max(err, std::abs(s - hw[r]));
    nrm += std::norm(hw[r]);
  }
  EXPECT(err < 1e-12);
  double mag = 0;
  api.magnitude(mag, &w.m);
  EXPECT(std::fabs(mag - std::sqrt(nrm)) < 1e-10 * std::sqrt(nrm));

  // QRGR on a 16 x 16 block: Q R = H
  const int q = 16;
  std::vector<cd> H(q * q);
  for (auto& x : H) x = cd(nd(rng), 0.0);
  DevMat dH(q, q, false), dQ(q, q, false), dR(q, q, false);
  dH.upload(H);
  api.QRGR(&dQ.m, &dR.m, &dH.m);
  std::vector<cd> Q = dQ.download(), R = dR.download();
  double qr = 0;
  for (int r = 0; r < q; ++r)
    for (int c = 0; c < q; ++c) {
      cd s = 0;
      for (int t = 0; t < q; ++t) s += Q[t + r * q] * R[c + t * q];
      qr = std::max(qr, std::abs(s - H[c + r * q]));
    }
  EXPECT(qr < 1e-12);

  // dense solve (CuHArnoldiDefault::setMatrix) and callback solve
  // (CuHArnoldiCallback::setCallback) agree with the planted spectrum
  for (int mode = 0; mode < 2; ++mode) {
    oapb::CuHArnoldiCallback arnoldi;
    std::vector<double> re(k), im(k);
    DevMat vecs(k, n, true);
    arnoldi.setRho(1. / 3.14);
    arnoldi.setSortType(oapb::ArnUtils::SortLargestValues);
    arnoldi.setCheckTolerance(1e-10);
    arnoldi.setOutputsEigenvalues(re.data(), im.data());
    arnoldi.setOutputsEigenvectors(&vecs.m);
    if (mode == 0) arnoldi.setMatrix(&dA.m);
    else arnoldi.setCallback(multiply, &dA.m);
    arnoldi.execute(m, k, oapb::MatrixInfo(true, true, n, n));
    EXPECT(arnoldi.converged());
    for (int i = 0; i < k; ++i) {
      EXPECT(std::abs(cd(re[i], im[i]) - lam[i]) < 1e-9 * std::abs(lam[i]));
      EXPECT(arnoldi.residuals()[i] <= 1e-10);
      EXPECT(arnoldi.testOutcome(i) <= 1e-10);
    }
    EXPECT(arnoldi.trace().empty());  // the plain restart loop records no block-phase checks
    std::printf("mode %d: lambda_1 = %.12f%+.12fi, residual %.2e\n", mode, re[0], im[0], arnoldi.residuals()[0]);
  }
  // Network (oapNetwork.h names): learn y = M x on 256 samples, save, load
  {
    const int ni = 6, no = 3, S = 256;
    std::vector<float> X(S * ni), Y(S * no), M(no * ni);
    for (auto& v : M) v = (float)(0.3 * nd(rng));
    for (int s = 0; s < S; ++s) {
      for (int i = 0; i < ni; ++i) X[s * ni + i] = (float)nd(rng);
      for (int o = 0; o < no; ++o) {
        float acc = 0;
        for (int i = 0; i < ni; ++i) acc += M[o * ni + i] * X[s * ni + i];
        Y[s * no + o] = acc;
      }
    }
    float *dX, *dY, *dOut1, *dOut2;
    cudaMalloc(&dX, sizeof(float) * X.size());
    cudaMalloc(&dY, sizeof(float) * Y.size());
    cudaMalloc(&dOut1, sizeof(float) * Y.size());
    cudaMalloc(&dOut2, sizeof(float) * Y.size());
    cudaMemcpy(dX, X.data(), sizeof(float) * X.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(dY, Y.data(), sizeof(float) * Y.size(), cudaMemcpyHostToDevice);
    oapb::Network net(7);
    net.createLayer(ni);
    net.createLayer(32, oapb::Activation::TANH);
    net.createLayer(no, oapb::Activation::LINEAR);
    net.setLearningRate(3e-3);
    net.train(dX, dY, S);
    const double first = net.calculateMSE();
    for (int step = 0; step < 400; ++step) net.train(dX, dY, S);
    const double last = net.calculateMSE();
    std::printf("network mse %.4g -> %.4g\n", first, last);
    EXPECT(last < 0.1 * first);
    EXPECT(net.getLayersCount() == 3);
    net.setInputs(dX, S);
    net.forwardPropagation(dOut1);
    net.save("/tmp/oapb_shim_network.bin");
    oapb::Network* back = oapb::Network::load("/tmp/oapb_shim_network.bin");
    back->setInputs(dX, S);
    back->forwardPropagation(dOut2);
    std::vector<float> o1(Y.size()), o2(Y.size());
    cudaMemcpy(o1.data(), dOut1, sizeof(float) * o1.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(o2.data(), dOut2, sizeof(float) * o2.size(), cudaMemcpyDeviceToHost);
    EXPECT(o1 == o2);
    delete back;
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dOut1);
    cudaFree(dOut2);
  }
  return failures;
}

int main(int argc, char** argv) {
  const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
  const int f = gpu ? gpu_tests() : cpu_tests();
  std::printf("%s: %d failures\n", gpu ? "gpu" : "cpu", f);
  return f == 0 ? 0 : 1;
}
