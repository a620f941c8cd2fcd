// eigen_seam_bench.cpp -- times Eigen's own Matrix operator* running on libeigen_b200.so, the way
// an Eigen program calls it: C.noalias() = A * B on MatrixXd (ordinary pageable host storage),
// compiled with -DEIGEN_USE_BLAS, so GeneralMatrixMatrix_BLAS.h:53-118 routes the product to
// the dgemm_ symbol with beta = 1 after Eigen's dst.setZero() (GeneralMatrixMatrix.h:450-456).
// The host -> device copies of A, B and C and the copy of C back are inside the timed region.
//
//   eigen_seam_bench <n> [reps] [warmup]   ->  one JSON line (median seconds, TFLOP/s, call record)
#include <Eigen/Core>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "eigen_b200/blas.h"

int main(int argc, char** argv) {
  const int n = argc > 1 ? std::atoi(argv[1]) : 8192;
  const int reps = argc > 2 ? std::atoi(argv[2]) : 5;
  const int warmup = argc > 3 ? std::atoi(argv[3]) : 1;
  std::srand(11);
  Eigen::MatrixXd A = Eigen::MatrixXd::Random(n, n), B = Eigen::MatrixXd::Random(n, n);
  Eigen::MatrixXd C(n, n);
  for (int i = 0; i < warmup; ++i) C.noalias() = A * B;
  std::vector<double> ts;
  for (int i = 0; i < reps; ++i) {
    const auto t0 = std::chrono::steady_clock::now();
    C.noalias() = A * B;
    ts.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  }
  std::sort(ts.begin(), ts.end());
  const double med = ts[ts.size() / 2];
  eb2_call_info info;
  eb2_last_call_info(&info);
  // a spot check of one entry against a long-double dot product
  long double s = 0;
  for (int l = 0; l < n; ++l) s += (long double)A(n / 3, l) * (long double)B(l, n / 5);
  const double spot = std::abs(double(C(n / 3, n / 5) - double(s))) / (std::abs(double(s)) + 1e-300);
  std::printf(
      "{\"n\": %d, \"reps\": %d, \"seconds_median\": %.6f, \"seconds_min\": %.6f, \"tflops\": %.4f, "
      "\"method\": %d, \"slices\": %d, \"staged\": %d, \"launches\": %d, \"kernel_ms\": %.3f, \"spot_rel_err\": %.3e, "
      "\"last_error\": %d}\n",
      n, int(ts.size()), med, ts.front(), 2.0 * double(n) * n * n / med * 1e-12, info.method, info.slices,
      info.staged, info.launches, info.kernel_ms, spot, eb2_last_error());
  return eb2_last_error() == 0 ? 0 : 1;
}
