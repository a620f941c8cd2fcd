// eigen_seam_demo.cpp -- Eigen's own Matrix operator* running on libeigen_b200.so.
//
// Compiled against the Eigen headers with -DEIGEN_USE_BLAS, so
// Eigen/src/Core/products/GeneralMatrixMatrix_BLAS.h:53-118 re-specialises
// general_matrix_matrix_product::run to call the external dgemm_/sgemm_ symbols.
// Linked with libeigen_b200.so first, those symbols resolve to this project's B200
// path (other BLAS symbols that the headers may reference, e.g. dgemv_ for the
// runtime GEMV fallback, come from the next library on the link line).
//
// The program forms several products through the public Eigen API, checks each
// against an unblocked triple loop in long double, and prints one JSON line
// with the max relative errors and the library's call record of the last product
// (which proves the product ran in libeigen_b200.so).
#include <Eigen/Core>

#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "eigen_b200/blas.h"

template <typename Mat>
double rel_err(const Mat& got, const Mat& want) {
  return double((got - want).norm() / want.norm());
}

template <typename Mat>
Mat naive(const Mat& a, const Mat& b) {
  Mat c(a.rows(), b.cols());
  for (Eigen::Index j = 0; j < b.cols(); ++j)
    for (Eigen::Index i = 0; i < a.rows(); ++i) {
      long double s = 0;
      for (Eigen::Index l = 0; l < a.cols(); ++l) s += (long double)a(i, l) * (long double)b(l, j);
      c(i, j) = typename Mat::Scalar(s);
    }
  return c;
}

int main(int argc, char** argv) {
  const int m = argc > 1 ? std::atoi(argv[1]) : 300;
  const int n = argc > 2 ? std::atoi(argv[2]) : 200;
  const int k = argc > 3 ? std::atoi(argv[3]) : 250;
  std::srand(7);
  Eigen::MatrixXd A = Eigen::MatrixXd::Random(m, k), B = Eigen::MatrixXd::Random(k, n);
  Eigen::MatrixXd At = A.transpose();

  // 1. C = A * B                        (dgemm_ with beta = 1 after setZero)
  Eigen::MatrixXd C = A * B;
  const double e1 = rel_err(C, naive(A, B));
  eb2_call_info info1;
  eb2_last_call_info(&info1);

  // 2. C.noalias() += 2.5 * At^T * B   (transposed lhs, alpha = 2.5, beta = 1)
  Eigen::MatrixXd C2 = Eigen::MatrixXd::Random(m, n);
  Eigen::MatrixXd want2 = C2 + 2.5 * naive(Eigen::MatrixXd(At.transpose()), B);
  C2.noalias() += 2.5 * At.transpose() * B;
  const double e2 = rel_err(C2, want2);

  // 3. float product through sgemm_
  Eigen::MatrixXf Af = A.cast<float>(), Bf = B.cast<float>();
  Eigen::MatrixXf Cf = Af * Bf;
  const double e3 = rel_err(Cf, naive(Af, Bf));
  eb2_call_info info3;
  eb2_last_call_info(&info3);

  std::printf(
      "{\"m\": %d, \"n\": %d, \"k\": %d, \"err_AB\": %.3e, \"err_alpha_AtB\": %.3e, \"err_float\": %.3e, "
      "\"dgemm_method\": %d, \"dgemm_slices\": %d, \"dgemm_launches\": %d, \"sgemm_dtype\": \"%c\", "
      "\"sgemm_launches\": %d, \"last_error\": %d}\n",
      m, n, k, e1, e2, e3, info1.method, info1.slices, info1.launches, info3.dtype ? info3.dtype : '?',
      info3.launches, eb2_last_error());
  const bool ok = e1 < 1e-14 && e2 < 1e-14 && e3 < 1e-5 && info1.launches > 0 && info3.launches > 0 &&
                  eb2_last_error() == 0;
  return ok ? 0 : 1;
}
