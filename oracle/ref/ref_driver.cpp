// Test infrastructure: plain C entry points over the reference's own host
// implementation of the operator surface (oapMatrixCpu/HostProcedures.h:30-124,
// compiled from the reference sources by build_ref.sh), so the CPU oracle
// and the CUDA ops can be checked against the reference's code itself.
// Matrices use the reference layout (row-major split planes, element
// (c, r) at c + r * columns); im may be NULL for a real matrix.
#include <cstring>

#include "HostProcedures.h"
#include "oapHostMatrixUtils.h"

namespace {

math::Matrix* make(unsigned columns, unsigned rows, const double* re, const double* im) {
  if (im) return oap::host::NewMatrixCopyOfArray(columns, rows, re, im);
  return oap::host::NewReMatrixCopyOfArray(columns, rows, re);
}

math::Matrix* make_out(unsigned columns, unsigned rows, bool cplx) {
  return cplx ? oap::host::NewMatrix(columns, rows) : oap::host::NewReMatrix(columns, rows);
}

void fetch(const math::Matrix* m, double* re, double* im) {
  const size_t n = (size_t)m->columns * m->rows;
  if (re) std::memcpy(re, m->reValues, sizeof(double) * n);
  if (im && m->imValues) std::memcpy(im, m->imValues, sizeof(double) * n);
}

}  // namespace

extern "C" {

// output (N columns x M rows) = A (K x M) * B (N x K)   HostProcedures::dotProduct
int ref_dot_product(unsigned M, unsigned K, unsigned N, const double* a_re, const double* a_im,
                    const double* b_re, const double* b_im, double* o_re, double* o_im) {
  HostProcedures hp;
  math::Matrix* a = make(K, M, a_re, a_im);
  math::Matrix* b = make(N, K, b_re, b_im);
  math::Matrix* o = make_out(N, M, a_im || b_im);
  hp.dotProduct(o, a, b);
  fetch(o, o_re, o_im);
  oap::host::DeleteMatrix(a);
  oap::host::DeleteMatrix(b);
  oap::host::DeleteMatrix(o);
  return 0;
}

// output (rows x columns) = A^T   HostProcedures::transpose
int ref_transpose(unsigned columns, unsigned rows, const double* a_re, const double* a_im, double* o_re,
                  double* o_im) {
  HostProcedures hp;
  math::Matrix* a = make(columns, rows, a_re, a_im);
  math::Matrix* o = make_out(rows, columns, a_im != nullptr);
  hp.transpose(o, a);
  fetch(o, o_re, o_im);
  oap::host::DeleteMatrix(a);
  oap::host::DeleteMatrix(o);
  return 0;
}

// output = A - B   HostProcedures::substract
int ref_substract(unsigned columns, unsigned rows, const double* a_re, const double* a_im, const double* b_re,
                  const double* b_im, double* o_re, double* o_im) {
  HostProcedures hp;
  math::Matrix* a = make(columns, rows, a_re, a_im);
  math::Matrix* b = make(columns, rows, b_re, b_im);
  math::Matrix* o = make_out(columns, rows, a_im != nullptr);
  hp.substract(o, a, b);
  fetch(o, o_re, o_im);
  oap::host::DeleteMatrix(a);
  oap::host::DeleteMatrix(b);
  oap::host::DeleteMatrix(o);
  return 0;
}

// (sum re, sum im)   HostProcedures::sum
int ref_sum(unsigned columns, unsigned rows, const double* a_re, const double* a_im, double* s_re, double* s_im) {
  HostProcedures hp;
  math::Matrix* a = make(columns, rows, a_re, a_im);
  double re = 0, im = 0;
  hp.sum(re, im, a);
  *s_re = re;
  *s_im = im;
  oap::host::DeleteMatrix(a);
  return 0;
}

// Householder QR of a real n x n matrix, n * n <= 1024   HostProcedures::QRHT
int ref_qr_householder(unsigned n, const double* a_re, double* q_re, double* r_re) {
  if (n * n > 1024) return 1;
  HostProcedures hp;
  math::Matrix* a = make(n, n, a_re, nullptr);
  math::Matrix* q = make_out(n, n, false);
  math::Matrix* r = make_out(n, n, false);
  math::Matrix* v = make_out(1, n, false);
  math::Matrix* vt = make_out(n, 1, false);
  math::Matrix* vvt = make_out(n, n, false);
  math::Matrix* p = make_out(n, n, false);
  hp.QRHT(q, r, a, v, vt, p, vvt);
  fetch(q, q_re, nullptr);
  fetch(r, r_re, nullptr);
  for (math::Matrix* m : {a, q, r, v, vt, vvt, p}) oap::host::DeleteMatrix(m);
  return 0;
}

// V[:, column] = v (first `length` rows)   HostProcedures::setVector
int ref_set_vector(unsigned columns, unsigned rows, double* v_re, unsigned column, const double* x_re,
                   unsigned length) {
  HostProcedures hp;
  math::Matrix* V = make(columns, rows, v_re, nullptr);
  math::Matrix* x = make(1, length, x_re, nullptr);
  hp.setVector(V, column, x, length);
  fetch(V, v_re, nullptr);
  oap::host::DeleteMatrix(V);
  oap::host::DeleteMatrix(x);
  return 0;
}

// oap::host::WriteMatrix: the reference's matrix file
int ref_write_matrix(const char* path, unsigned columns, unsigned rows, const double* re, const double* im) {
  math::Matrix* m = make(columns, rows, re, im);
  const bool ok = oap::host::WriteMatrix(path, m);
  oap::host::DeleteMatrix(m);
  return ok ? 0 : 1;
}

// (oap::host::ReadMatrix is not wrapped: utils::Buffer::increaseReadIdx,
// oapUtils/Buffer.h:324-327, returns no value from a value-returning
// function, and g++ compiles the fall-through into a trap, so every read of
// a matrix file by the reference code ends the process.)

}  // extern "C"
