// eigen_seam_solvers.cpp -- Eigen's own decompositions and structured products running on
// libeigen_b200.so through the external-BLAS seam.
//
// Compiled against the Eigen headers with -DEIGEN_USE_BLAS, so the *_BLAS.h headers of
// Eigen/src/Core/products re-specialise Eigen's triangular solve (dtrsm_, ztrsm_), triangular
// product (dtrmm_, ztrmm_), self-adjoint product (dsymm_, zhemm_), rank update (dsyrk_) and
// complex product (zgemm_) to call the external BLAS symbols; linked with libeigen_b200.so
// first, they resolve to this project's B200 routines.  Blocked LLT and PartialPivLU reach dtrsm_, dsyrk_ and dgemm_ from
// inside Eigen's own algorithms.
//
// Each result is checked against a plain computation (residuals for the solves, an unblocked
// long-double product for the products), and the library's per-routine call counters show
// which routines ran on the device.  One JSON line; exit status 0 when every check passes.
#include <Eigen/Cholesky>
#include <Eigen/Core>
#include <Eigen/LU>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>

#include "eigen_b200/blas.h"

using Eigen::Index;
using Eigen::MatrixXcd;
using Eigen::MatrixXd;

template <typename Mat>
Mat naive(const Mat& a, const Mat& b) {
  using S = typename Mat::Scalar;
  Mat c(a.rows(), b.cols());
  for (Index j = 0; j < b.cols(); ++j)
    for (Index i = 0; i < a.rows(); ++i) {
      std::complex<long double> s = 0;
      for (Index l = 0; l < a.cols(); ++l)
        s += std::complex<long double>(std::complex<double>(a(i, l))) *
             std::complex<long double>(std::complex<double>(b(l, j)));
      if constexpr (std::is_same_v<S, double>)
        c(i, j) = double(s.real());
      else
        c(i, j) = S(double(s.real()), double(s.imag()));
    }
  return c;
}

template <typename Mat>
double rel(const Mat& got, const Mat& want) {
  return double((got - want).norm() / want.norm());
}

int main(int argc, char** argv) {
  const int n = argc > 1 ? std::atoi(argv[1]) : 600;
  const int r = argc > 2 ? std::atoi(argv[2]) : 96;  // right-hand sides
  std::srand(11);
  MatrixXd A = MatrixXd::Random(n, n);
  MatrixXd B = MatrixXd::Random(n, r);

  // SPD matrix, factored by Eigen's blocked LLT (dtrsm_ and dsyrk_ inside), then solved
  MatrixXd S = A * A.transpose();
  S.diagonal().array() += double(n);
  Eigen::LLT<MatrixXd> llt(S);
  const MatrixXd L = llt.matrixL();
  const double e_llt = rel(MatrixXd(L * L.transpose()), S);
  const MatrixXd X1 = llt.solve(B);
  const double e_llt_solve = rel(MatrixXd(S * X1), B);

  // general matrix, Eigen's blocked PartialPivLU (dtrsm_ and dgemm_ inside)
  MatrixXd G = A;
  G.diagonal().array() += 4.0;
  Eigen::PartialPivLU<MatrixXd> lu(G);
  const MatrixXd X2 = lu.solve(B);
  const double e_lu_solve = rel(MatrixXd(G * X2), B);

  // a triangular solve with a matrix right-hand side (dtrsm_)
  MatrixXd T = A.triangularView<Eigen::Lower>();
  T.diagonal().array() += double(n) / 4;
  const MatrixXd X3 = T.triangularView<Eigen::Lower>().solve(B);
  const double e_trsm = rel(naive(T, X3), B);

  // triangular times matrix (dtrmm_)
  const MatrixXd P1 = T.triangularView<Eigen::Lower>() * B;
  const double e_trmm = rel(P1, naive(T, B));

  // self-adjoint times matrix, the lower triangle stored (dsymm_)
  MatrixXd Sl = S.triangularView<Eigen::Lower>();
  const MatrixXd P2 = Sl.selfadjointView<Eigen::Lower>() * B;
  const double e_symm = rel(P2, naive(S, B));

  // rank update of the lower triangle, C += 0.5 * A A^T (dsyrk_)
  MatrixXd C = MatrixXd::Zero(n, n);
  C.selfadjointView<Eigen::Lower>().rankUpdate(A, 0.5);
  const MatrixXd want_c = 0.5 * naive(A, MatrixXd(A.transpose()));
  const double e_syrk = double(
      (MatrixXd(C.triangularView<Eigen::Lower>()) - MatrixXd(want_c.triangularView<Eigen::Lower>())).norm() /
      MatrixXd(want_c.triangularView<Eigen::Lower>()).norm());

  // complex product (zgemm_)
  MatrixXcd Z1 = MatrixXcd::Random(n, 200), Z2 = MatrixXcd::Random(200, r);
  const MatrixXcd Z = Z1 * Z2;
  const double e_zgemm = rel(Z, naive(Z1, Z2));

  // complex: Hermitian positive definite LLT (ztrsm_ inside), a triangular solve (ztrsm_), a
  // triangular product (ztrmm_) and a self-adjoint product (zhemm_)
  MatrixXcd ZA = MatrixXcd::Random(n, n);
  MatrixXcd ZH = ZA * ZA.adjoint();
  ZH.diagonal().array() += double(n);
  const MatrixXcd ZB = MatrixXcd::Random(n, r);
  Eigen::LLT<MatrixXcd> zllt(ZH);
  const MatrixXcd ZX = zllt.solve(ZB);
  const double e_zllt_solve = rel(naive(ZH, ZX), ZB);
  MatrixXcd ZT = ZA.triangularView<Eigen::Upper>();
  ZT.diagonal().array() += double(n) / 4;
  const MatrixXcd ZX2 = ZT.triangularView<Eigen::Upper>().solve(ZB);
  const double e_ztrsm = rel(naive(ZT, ZX2), ZB);
  const MatrixXcd ZP = ZT.triangularView<Eigen::Upper>() * ZB;
  const double e_ztrmm = rel(ZP, naive(ZT, ZB));
  MatrixXcd ZHl = ZH.triangularView<Eigen::Lower>();
  const MatrixXcd ZQ = ZHl.selfadjointView<Eigen::Lower>() * ZB;
  const double e_zhemm = rel(ZQ, naive(ZH, ZB));

  const long long c_gemm = eb2_routine_calls("dgemm"), c_trsm = eb2_routine_calls("dtrsm"),
                  c_trmm = eb2_routine_calls("dtrmm"), c_symm = eb2_routine_calls("dsymm"),
                  c_syrk = eb2_routine_calls("dsyrk"), c_zgemm = eb2_routine_calls("zgemm"),
                  c_ztrsm = eb2_routine_calls("ztrsm"), c_ztrmm = eb2_routine_calls("ztrmm"),
                  c_zhemm = eb2_routine_calls("zhemm");
  std::printf(
      "{\"n\": %d, \"rhs\": %d, \"err_llt\": %.3e, \"err_llt_solve\": %.3e, \"err_lu_solve\": %.3e, "
      "\"err_trsm\": %.3e, \"err_trmm\": %.3e, \"err_symm\": %.3e, \"err_syrk\": %.3e, \"err_zgemm\": %.3e, "
      "\"err_zllt_solve\": %.3e, \"err_ztrsm\": %.3e, \"err_ztrmm\": %.3e, \"err_zhemm\": %.3e, "
      "\"calls\": {\"dgemm\": %lld, \"dtrsm\": %lld, \"dtrmm\": %lld, \"dsymm\": %lld, \"dsyrk\": %lld, "
      "\"zgemm\": %lld, \"ztrsm\": %lld, \"ztrmm\": %lld, \"zhemm\": %lld}, \"last_error\": %d}\n",
      n, r, e_llt, e_llt_solve, e_lu_solve, e_trsm, e_trmm, e_symm, e_syrk, e_zgemm, e_zllt_solve, e_ztrsm, e_ztrmm,
      e_zhemm, c_gemm, c_trsm, c_trmm, c_symm, c_syrk, c_zgemm, c_ztrsm, c_ztrmm, c_zhemm, eb2_last_error());
  const double tol = 1e-13;
  const bool ok = e_llt < tol && e_llt_solve < tol && e_lu_solve < 1e-11 && e_trsm < tol && e_trmm < tol &&
                  e_symm < tol && e_syrk < tol && e_zgemm < tol && e_zllt_solve < tol && e_ztrsm < tol &&
                  e_ztrmm < tol && e_zhemm < tol && c_gemm > 0 && c_trsm > 0 && c_trmm > 0 && c_symm > 0 &&
                  c_syrk > 0 && c_zgemm > 0 && c_ztrsm > 0 && c_ztrmm > 0 && c_zhemm > 0 && eb2_last_error() == 0;
  return ok ? 0 : 1;
}
