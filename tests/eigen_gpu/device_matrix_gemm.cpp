// device_matrix_gemm.cpp -- GEMM expressions of Eigen's gpu::DeviceMatrix module running on
// libeigen_b200.so.
//
// Compiled against the reference's unsupported/Eigen/GPU with EIGEN_USE_GPU and
// eigen_b200/eigen_gpu_gemm.h, which specialises the module's single GEMM entry
// (Eigen::gpu::internal::cublaslt_gemm<double/float>) to call eb2_dgemm_device /
// eb2_sgemm_device on the module's stream.  The program evaluates the expression forms of
// DeviceDispatch.h (plain, transposed operands, scaled, accumulating, subtracting with an
// explicit gpu::Context) for double and float, checks each against Eigen's CPU product and
// prints one JSON line with the errors and the library's record of the last product.  Exit
// status 0 when every check passes.  With a fourth argument `reps` it times the FP64
// product instead.
#define EIGEN_USE_GPU
#include <unsupported/Eigen/GPU>

// Built twice: with the library's dispatch, and with EIGEN_GPU_STOCK_DISPATCH as the
// module's own cuBLASLt path (timing comparison only).
#ifndef EIGEN_GPU_STOCK_DISPATCH
#include "eigen_b200/eigen_gpu_gemm.h"
#endif

#include <algorithm>
#include <cstdio>
#include <cstdlib>

using Eigen::Index;

template <typename Mat>
double rel(const Mat& got, const Mat& want) {
  return double((got - want).norm() / want.norm());
}

#ifndef EIGEN_GPU_STOCK_DISPATCH
template <typename Scalar>
double run(Index m, Index n, Index k, eb2_call_info* info) {
  using Mat = Eigen::Matrix<Scalar, Eigen::Dynamic, Eigen::Dynamic>;
  using DM = Eigen::gpu::DeviceMatrix<Scalar>;
  const Mat A = Mat::Random(m, k), B = Mat::Random(k, n), At = A.transpose(), Bt = B.transpose();
  const Mat C0 = Mat::Random(m, n);
  const DM dA = DM::fromHost(A), dB = DM::fromHost(B), dAt = DM::fromHost(At), dBt = DM::fromHost(Bt);
  double worst = 0;
  DM dC;
  dC = dA * dB;  // C = A B
  worst = std::max(worst, rel(Mat(dC.toHost()), Mat(A * B)));
  dC = dAt.transpose() * dB;  // transposed left operand
  worst = std::max(worst, rel(Mat(dC.toHost()), Mat(A * B)));
  dC = Scalar(2.5) * dA * dBt.transpose();  // scaled, transposed right operand
  worst = std::max(worst, rel(Mat(dC.toHost()), Mat(Scalar(2.5) * A * B)));
  DM dD = DM::fromHost(C0);
  dD += dA * dB;  // beta = 1
  worst = std::max(worst, rel(Mat(dD.toHost()), Mat(C0 + A * B)));
  Eigen::gpu::Context ctx;
  DM dE = DM::fromHost(C0);
  dE.device(ctx) -= dA * dB;  // alpha = -1, beta = 1, an explicit context and stream
  worst = std::max(worst, rel(Mat(dE.toHost(ctx.stream())), Mat(C0 - A * B)));
  eb2_last_call_info(info);
  return worst;
}
#endif

// d_C = d_A * d_B (FP64, m x n x k) `reps` times on one gpu::Context after a warm-up: the
// best device time of one product (CUDA events on the context's stream).
double time_gemm(Index m, Index n, Index k, int reps) {
  using DM = Eigen::gpu::DeviceMatrix<double>;
  const DM dA = DM::fromHost(Eigen::MatrixXd::Random(m, k)), dB = DM::fromHost(Eigen::MatrixXd::Random(k, n));
  DM dC;
  Eigen::gpu::Context ctx;
  dC.device(ctx) = dA * dB;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(e0, ctx.stream());
    dC.device(ctx) = dA * dB;
    cudaEventRecord(e1, ctx.stream());
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

int main(int argc, char** argv) {
  const Index m = argc > 1 ? std::atoi(argv[1]) : 700;
  const Index n = argc > 2 ? std::atoi(argv[2]) : 500;
  const Index k = argc > 3 ? std::atoi(argv[3]) : 600;
  const int reps = argc > 4 ? std::atoi(argv[4]) : 0;
  if (reps > 0) {
    const double ms = time_gemm(m, n, k, reps);
#ifdef EIGEN_GPU_STOCK_DISPATCH
    const char* path = "cuBLASLt (the module's own dispatch)";
#else
    const char* path = "libeigen_b200";
#endif
    std::printf("{\"m\": %ld, \"n\": %ld, \"k\": %ld, \"dispatch\": \"%s\", \"ms\": %.4f, \"tflops\": %.3f}\n",
                long(m), long(n), long(k), path, ms, 2.0 * m * n * k / (ms * 1e-3) / 1e12);
    return 0;
  }
#ifdef EIGEN_GPU_STOCK_DISPATCH
  return 2;  // the stock build only times
#else
  std::srand(5);
  eb2_call_info di{}, si{};
  const double ed = run<double>(m, n, k, &di);
  const double es = run<float>(m, n, k, &si);
  std::printf(
      "{\"m\": %ld, \"n\": %ld, \"k\": %ld, \"err_double\": %.3e, \"err_float\": %.3e, \"double_method\": %d, "
      "\"double_launches\": %d, \"double_dtype\": \"%c\", \"float_launches\": %d, \"float_dtype\": \"%c\", "
      "\"last_error\": %d}\n",
      long(m), long(n), long(k), ed, es, di.method, di.launches, di.dtype ? char(di.dtype) : '?', si.launches,
      si.dtype ? char(si.dtype) : '?', eb2_last_error());
  const bool ok = ed < 1e-14 && es < 1e-5 && di.launches > 0 && si.launches > 0 && di.dtype == 'd' &&
                  si.dtype == 's' && eb2_last_error() == 0;
  return ok ? 0 : 1;
#endif
}
