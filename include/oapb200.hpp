/*
 * oapb200.hpp - C++ face of liboapb200 with the reference's class and method
 * names, header-only, over the C ABI of oapb200.h.
 *
 * A caller of oap's operator surface and Arnoldi solver keeps its call sites:
 *   oap::CuProceduresApi (oapMatrixCuda/CuProceduresApi.h:45-421)
 *       -> oapb::CuProceduresApi, same method names and argument order;
 *   CuHArnoldiCallback / CuHArnoldiDefault
 *     (ArnoldiPackage/ArnoldiProceduresImpl.h:25-78, ArnoldiProcedures.h:33-62)
 *       -> oapb::CuHArnoldiCallback (setters, setCallback / setMatrix,
 *          execute(hdim, wanted, MatrixInfo), testOutcome);
 *   math::MatrixInfo (oapMatrix/MatrixInfo.h:31) -> oapb::MatrixInfo;
 *   ArnUtils::Sort* (ArnoldiPackage/ArnoldiUtils.h:60-72) -> oapb::ArnUtils.
 * Differences a caller sees: a matrix is the host handle oapb_mat (columns,
 * rows, device re / im planes) instead of a device math::Matrix*; errors
 * throw oapb::Error (the reference aborts); eigenvectors come back as one
 * n x wanted device matrix of Ritz vectors.
 */
#ifndef OAPB200_HPP
#define OAPB200_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "oapb200.h"

namespace oapb {

typedef double floatt;
typedef unsigned int uint;
typedef oapb_mat Matrix;

/* A non-OK status of the C ABI. */
class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& where)
      : std::runtime_error(where + ": " + oapb_status_string(status)), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int status, const char* where) {
  if (status != OAPB_OK) throw Error(status, where);
}

/* oap::VecMultiplicationType (ArnoldiPackage/oapGenericArnoldiApi.h:38-42). */
enum class VecMultiplicationType { TYPE_EIGENVECTOR = OAPB_TYPE_EIGENVECTOR, TYPE_WV = OAPB_TYPE_WV };

/* ArnUtils sort orders (ArnoldiUtils.h:60-72) as the solver's enumeration. */
namespace ArnUtils {
typedef oapb_sort SortType;
const SortType SortLargestValues = OAPB_SORT_LARGEST_VALUES;
const SortType SortLargestReValues = OAPB_SORT_LARGEST_RE;
const SortType SortLargestImValues = OAPB_SORT_LARGEST_IM;
const SortType SortSmallestValues = OAPB_SORT_SMALLEST_VALUES;
const SortType SortSmallestReValues = OAPB_SORT_SMALLEST_RE;
const SortType SortSmallestImValues = OAPB_SORT_SMALLEST_IM;
}  // namespace ArnUtils

/* math::MatrixInfo(isRe, isIm, columns, rows) (oapMatrix/MatrixInfo.h:31). */
struct MatrixInfo {
  bool isRe = true, isIm = false;
  uint columns = 0, rows = 0;
  MatrixInfo() {}
  MatrixInfo(bool re, bool im, uint c, uint r) : isRe(re), isIm(im), columns(c), rows(r) {}
};

/* oap::CuProceduresApi: every call runs on the stream given at construction
 * (NULL: the legacy default stream). */
class CuProceduresApi {
 public:
  explicit CuProceduresApi(void* stream = nullptr) : stream_(stream) {}
  CuProceduresApi(const CuProceduresApi&) = delete;
  CuProceduresApi& operator=(const CuProceduresApi&) = delete;

  void* stream() const { return stream_; }

  void dotProduct(Matrix* output, Matrix* params0, Matrix* params1) {
    check(oapb_dot_product(output, params0, params1, stream_), "dotProduct");
  }
  void transpose(Matrix* output, Matrix* params0) { check(oapb_transpose(output, params0, stream_), "transpose"); }
  void conjugateTranspose(Matrix* output, Matrix* params0) {
    check(oapb_conjugate_transpose(output, params0, stream_), "conjugateTranspose");
  }
  void tensorProduct(Matrix* output, Matrix* params0, Matrix* params1) {
    check(oapb_tensor_product(output, params0, params1, stream_), "tensorProduct");
  }
  void add(Matrix* output, Matrix* params0, Matrix* params1) {
    check(oapb_add(output, params0, params1, stream_), "add");
  }
  void substract(Matrix* output, Matrix* params0, Matrix* params1) {
    check(oapb_substract(output, params0, params1, stream_), "substract");
  }
  void setVector(Matrix* output, uint column, Matrix* params0, uint length) {
    check(oapb_set_vector(output, column, params0, length, stream_), "setVector");
  }
  void getVector(Matrix* vector, uint length, Matrix* matrix, uint column) {
    check(oapb_get_vector(vector, length, matrix, column, stream_), "getVector");
  }
  void getVector(Matrix* vector, Matrix* matrix, uint column) { getVector(vector, vector->rows, matrix, column); }
  void magnitude(floatt& output, Matrix* params0) { check(oapb_magnitude(&output, params0, stream_), "magnitude"); }
  void sum(floatt& reoutput, floatt& imoutput, Matrix* matrix) {
    check(oapb_sum(&reoutput, &imoutput, matrix, stream_), "sum");
  }
  void sum(floatt& reoutput, Matrix* matrix) {
    floatt im = 0;
    sum(reoutput, im, matrix);
  }
  void multiplyReConstant(Matrix* v, Matrix* f, floatt re) {
    check(oapb_multiply_re_constant(v, f, re, stream_), "multiplyReConstant");
  }
  void multiplyConstant(Matrix* v, Matrix* f, floatt re, floatt im) {
    check(oapb_multiply_constant(v, f, re, im, stream_), "multiplyConstant");
  }
  void setDiagonal(Matrix* matrix, floatt re, floatt im) {
    check(oapb_set_diagonal(matrix, re, im, stream_), "setDiagonal");
  }
  void setIdentity(Matrix* matrix) { check(oapb_set_identity(matrix, stream_), "setIdentity"); }
  void setZeroMatrix(Matrix* matrix) { check(oapb_set_zero_matrix(matrix, stream_), "setZeroMatrix"); }
  /* QRGR(Q, R, H, R1, Q1, G, GT): the four auxiliary matrices are not needed. */
  void QRGR(Matrix* Q, Matrix* R, Matrix* H, Matrix* = nullptr, Matrix* = nullptr, Matrix* = nullptr,
            Matrix* = nullptr) {
    check(oapb_qr_givens(Q, R, H, stream_), "QRGR");
  }
  /* QRHT(Q, R, A, V, VT, P, VVT): the auxiliary matrices are not needed. */
  void QRHT(Matrix* Q, Matrix* R, Matrix* A, Matrix* = nullptr, Matrix* = nullptr, Matrix* = nullptr,
            Matrix* = nullptr) {
    check(oapb_qr_householder(Q, R, A, stream_), "QRHT");
  }
  /* the reference's fixed 1e-3 sub-diagonal gate */
  bool isUpperTriangular(Matrix* matrix) {
    int out = 0;
    check(oapb_is_upper_triangular(&out, matrix, 1e-3, stream_), "isUpperTriangular");
    return out != 0;
  }
  /* calcTriangularH: unshifted QR iteration to the 1e-3 gate (600 steps). */
  uint calcTriangularH(Matrix* H, Matrix* Q, uint maxIterations = 600) {
    uint32_t it = 0;
    check(oapb_calc_triangular_h(H, Q, maxIterations, &it, stream_), "calcTriangularH");
    return it;
  }

 private:
  void* stream_;
};

/* CuHArnoldiCallback (user operator through setCallback) and
 * CuHArnoldiDefault (dense operator through setMatrix) in one class. */
class CuHArnoldiCallback {
 public:
  typedef void (*MultiplyFunc)(Matrix* w, Matrix* v, CuProceduresApi& api, void* userData,
                               VecMultiplicationType mt);

  explicit CuHArnoldiCallback(void* stream = nullptr) : api_(stream), stream_(stream) {
    oapb_arnoldi_config_default(&cfg_);
  }
  ~CuHArnoldiCallback() {
    if (h_) oapb_arnoldi_destroy(h_);
  }
  CuHArnoldiCallback(const CuHArnoldiCallback&) = delete;
  CuHArnoldiCallback& operator=(const CuHArnoldiCallback&) = delete;

  void setRho(floatt rho = 1. / 3.14) { cfg_.rho = rho; }
  void setSortType(ArnUtils::SortType sortType) { cfg_.sort = sortType; }
  /* residual goal ||A x - l x|| / (|l_1| ||x||) (the reference has no residual goal) */
  void setCheckTolerance(floatt tolerance) { cfg_.tolerance = tolerance; }
  /* restart budget */
  void setCheckCounts(uint count) { cfg_.max_restarts = count; }
  void setPrecision(oapb_precision precision) { cfg_.precision = precision; }
  void setSeed(uint64_t seed) { cfg_.seed = seed; }
  void setOutputsEigenvalues(floatt* reoevalues, floatt* imoevalues) {
    re_ = reoevalues;
    im_ = imoevalues;
  }
  /* n x wanted device matrix (column q = eigenvector q) */
  void setOutputsEigenvectors(Matrix* oevectors) { vectors_ = oevectors; }
  void setCallback(MultiplyFunc multiplyFunc, void* userData) {
    fn_ = multiplyFunc;
    user_ = userData;
    A_ = nullptr;
  }
  /* CuHArnoldiDefault::setMatrix: a dense n x n device operator */
  void setMatrix(Matrix* A) {
    A_ = A;
    fn_ = nullptr;
  }

  /* CuHArnoldi::execute(hdim, wantedCount, matrixInfo) */
  void execute(uint hdim, uint wantedCount, const MatrixInfo& matrixInfo) {
    if (h_) {
      oapb_arnoldi_destroy(h_);
      h_ = nullptr;
    }
    cfg_.n = matrixInfo.rows;
    cfg_.hdim = hdim;
    cfg_.wanted = wantedCount;
    cfg_.is_complex = matrixInfo.isIm ? 1 : 0;
    check(oapb_arnoldi_create(&h_, &cfg_, stream_), "CuHArnoldi::execute (create)");
    if (A_) {
      check(oapb_arnoldi_set_dense_operator(h_, A_), "CuHArnoldiDefault::setMatrix");
    } else if (fn_) {
      check(oapb_arnoldi_set_callback(h_, &CuHArnoldiCallback::bridge, this), "CuHArnoldiCallback::setCallback");
    } else {
      throw Error(OAPB_ERR_ARG, "CuHArnoldi::execute: no operator (setCallback or setMatrix)");
    }
    residuals_.assign(wantedCount, 0.0);
    const int st = oapb_arnoldi_solve(h_, re_, im_, residuals_.data(), vectors_);
    if (st != OAPB_OK && st != OAPB_NOT_CONVERGED) throw Error(st, "CuHArnoldi::execute");
    converged_ = st == OAPB_OK;
  }

  /* CuHArnoldi::testOutcome(index): relative residual of pair `index` */
  floatt testOutcome(size_t index) {
    double out = 0;
    check(oapb_arnoldi_test_outcome(h_, (uint32_t)index, &out), "testOutcome");
    return out;
  }

  bool converged() const { return converged_; }
  const std::vector<floatt>& residuals() const { return residuals_; }
  oapb_arnoldi_stats stats() const {
    oapb_arnoldi_stats s{};
    if (h_) oapb_arnoldi_get_stats(h_, &s);
    return s;
  }
  // convergence checks of the last execute (the data behind the reference's
  // per-step logInfo printouts, ArnoldiPackage/ArnoldiProcedures.cpp:391-395, 539)
  std::vector<oapb_trace_rec> trace() const {
    std::vector<oapb_trace_rec> t;
    uint32_t n = 0;
    if (!h_ || oapb_arnoldi_get_trace(h_, nullptr, 0, &n) != OAPB_OK) return t;
    t.resize(n);
    if (n && oapb_arnoldi_get_trace(h_, t.data(), n, &n) != OAPB_OK) t.clear();
    return t;
  }
  CuProceduresApi& api() { return api_; }

 private:
  // the user's operator runs on the solver's stream (the api handed to it
  // is bound to that stream)
  static int bridge(const oapb_mat* w, const oapb_mat* v, void* user, int type, void* stream) {
    CuHArnoldiCallback* self = static_cast<CuHArnoldiCallback*>(user);
    oapb_mat wm = *w, vm = *v;
    CuProceduresApi api(stream);
    try {
      self->fn_(&wm, &vm, api, self->user_, static_cast<VecMultiplicationType>(type));
    } catch (...) {
      return 1;  // the solve ends with OAPB_ERR_CALLBACK
    }
    return 0;
  }

  CuProceduresApi api_;
  void* stream_;
  oapb_arnoldi_config cfg_{};
  oapb_arnoldi* h_ = nullptr;
  MultiplyFunc fn_ = nullptr;
  void* user_ = nullptr;
  Matrix* A_ = nullptr;
  floatt* re_ = nullptr;
  floatt* im_ = nullptr;
  Matrix* vectors_ = nullptr;
  std::vector<floatt> residuals_;
  bool converged_ = false;
};

/* Network (oapNeuralDevice/oapNetwork.h:27-124) over the library's BF16
 * network: createLayer per layer (the first is the input layer, whose
 * activation is not used) with the reference's activations, inputs /
 * expected outputs as device FP32 samples x features, forwardPropagation /
 * backPropagation / updateWeights (Adam with the learning rate), train =
 * the three in one call, the MSE of the last backPropagation, save / load
 * in the reference's matrix file format. */
/* oapNeuralHost/oapLayerStructure.h:32-38, the same order (= oapb_activation). */
enum class Activation { LINEAR = OAPB_ACT_LINEAR, SIGMOID = OAPB_ACT_SIGMOID, TANH = OAPB_ACT_TANH, SIN = OAPB_ACT_SIN };

class Network {
 public:
  explicit Network(uint64_t seed = 1) : seed_(seed) {}
  ~Network() {
    if (h_) oapb_mlp_destroy(h_);
  }
  Network(const Network&) = delete;
  Network& operator=(const Network&) = delete;

  /* Layer* createLayer(neurons, activation = SIGMOID) (oapNetwork.h:53):
   * the input layer's activation is not used. */
  void createLayer(uint neurons, const Activation& activation = Activation::SIGMOID) {
    if (h_) throw Error(OAPB_ERR_ARG, "Network::createLayer: network already built");
    const int a = static_cast<int>(activation);
    if (neurons == 0 || a < OAPB_ACT_LINEAR || a > OAPB_ACT_SIN)
      throw Error(OAPB_ERR_ARG, "Network::createLayer: no neurons or unknown activation");
    sizes_.push_back(neurons);
    acts_.push_back(activation);
  }
  uint getLayersCount() const { return h_ ? oapb_mlp_num_layers(h_, nullptr) + 1 : (uint)sizes_.size(); }
  void setLearningRate(floatt lr) { lr_ = lr; }
  floatt getLearningRate() const { return lr_; }

  /* device FP32 arrays of `samples` rows */
  void setInputs(const float* inputs, uint samples) {
    inputs_ = inputs;
    samples_ = samples;
  }
  void setExpected(const float* expected, uint samples) {
    expected_ = expected;
    samples_ = samples;
  }
  /* outputs into the device array y (samples x outputs) */
  void forwardPropagation(float* y) {
    build();
    check(oapb_mlp_forward(h_, inputs_, samples_, y, nullptr), "Network::forwardPropagation");
  }
  void backPropagation() {
    build();
    check(oapb_mlp_backward(h_, inputs_, expected_, samples_, &mse_, nullptr), "Network::backPropagation");
  }
  void updateWeights() {
    build();
    check(oapb_mlp_adam_step(h_, (float)lr_, nullptr), "Network::updateWeights");
  }
  /* one step on (inputs, expected); true while it ran */
  bool train(const float* inputs, const float* expected, uint samples) {
    setInputs(inputs, samples);
    setExpected(expected, samples);
    backPropagation();
    updateWeights();
    return true;
  }
  /* 1 / (2 samples) sum (y - expected)^2 of the last backPropagation */
  floatt calculateMSE() const { return mse_; }

  void getHostWeights(std::vector<float>& weights) {
    build();
    weights.resize(oapb_mlp_num_params(h_));
    check(oapb_mlp_copy(h_, 0, weights.data(), nullptr), "Network::getHostWeights");
  }
  void setHostWeights(const std::vector<float>& weights) {
    build();
    if (weights.size() != oapb_mlp_num_params(h_)) throw Error(OAPB_ERR_ARG, "Network::setHostWeights: size");
    check(oapb_mlp_set_params(h_, weights.data(), nullptr), "Network::setHostWeights");
  }

  void save(const std::string& path) {
    build();
    check(oapb_mlp_save(h_, path.c_str()), "Network::save");
  }
  static Network* load(const std::string& path, uint64_t seed = 1) {
    Network* net = new Network(seed);
    const int st = oapb_mlp_load(&net->h_, path.c_str(), seed);
    if (st != OAPB_OK) {
      delete net;
      throw Error(st, "Network::load");
    }
    return net;
  }

 private:
  void build() {
    if (h_) return;
    if (sizes_.size() < 2) throw Error(OAPB_ERR_ARG, "Network: fewer than two layers");
    check(oapb_mlp_create(&h_, sizes_.data(), (uint32_t)sizes_.size() - 1, seed_), "Network (create)");
    std::vector<int32_t> acts;
    for (size_t l = 1; l < acts_.size(); ++l) acts.push_back(static_cast<int32_t>(acts_[l]));
    check(oapb_mlp_set_activations(h_, acts.data(), (uint32_t)acts.size()), "Network (activations)");
  }

  uint64_t seed_;
  oapb_mlp* h_ = nullptr;
  std::vector<uint32_t> sizes_;
  std::vector<Activation> acts_;
  floatt lr_ = 1e-3;
  const float* inputs_ = nullptr;
  const float* expected_ = nullptr;
  uint samples_ = 0;
  double mse_ = 0;
};

}  // namespace oapb

#endif  // OAPB200_HPP
