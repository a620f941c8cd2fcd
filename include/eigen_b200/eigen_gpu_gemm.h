/*
 * eigen_b200/eigen_gpu_gemm.h -- routes the GEMMs of Eigen's gpu::DeviceMatrix module
 * (unsupported/Eigen/GPU) to libeigen_b200.so instead of cuBLASLt.
 *
 * Every real GEMM the module runs goes through one function template,
 * Eigen::gpu::internal::cublaslt_gemm<Scalar>
 * (unsupported/Eigen/src/GPU/CuBlasSupport.h:287-323). Its callers are the DeviceMatrix
 * expressions of DeviceDispatch.h:38-93 (d_C = d_A * d_B, adjoints, transposes, scaled and
 * accumulating forms) and the solvers' internal products. This header gives the template
 * explicit specialisations for double and float. They call eb2_dgemm_device /
 * eb2_sgemm_device on the module's stream, with the device pointers, leading dimensions
 * and α/β the module passes, so the products run on this library's B200 kernels (for FP64,
 * the CRT emulation or the FP64 kernel that the method setting chooses). Complex products
 * stay on cuBLASLt.
 *
 * Use: define EIGEN_USE_GPU, include <unsupported/Eigen/GPU>, then this header, before the
 * first DeviceMatrix product in the translation unit. Link with -leigen_b200.
 *
 * FP64 products keep the emulation's a-posteriori accuracy check, which waits for the
 * stream once per product. Define EIGEN_B200_GPU_GEMM_ASYNC before including this header
 * for fully stream-ordered products without the check.
 * A product the library refuses (an invalid argument, a device error) raises
 * std::runtime_error with the library's message.
 */
#ifndef EIGEN_B200_EIGEN_GPU_GEMM_H
#define EIGEN_B200_EIGEN_GPU_GEMM_H

#ifndef EIGEN_GPU_MODULE_H
#error "include <unsupported/Eigen/GPU> (with EIGEN_USE_GPU defined) before eigen_b200/eigen_gpu_gemm.h"
#endif

#include <stdexcept>
#include <string>

#include "eigen_b200/blas.h"

namespace Eigen {
namespace gpu {
namespace internal {

inline char eb2_op(cublasOperation_t op) { return op == CUBLAS_OP_N ? 'N' : 'T'; }  // real: C == T

inline void eb2_gemm_status(int rc) {
  if (rc != EB2_OK && rc != EB2_ERR_ACCURACY)
    throw std::runtime_error(std::string("eigen_b200 GEMM failed: ") + eb2_last_error_string());
}

template <>
inline void cublaslt_gemm<double>(cublasLtHandle_t, cublasHandle_t, cublasOperation_t transA,
                                  cublasOperation_t transB, int64_t m, int64_t n, int64_t k, const double* alpha,
                                  const double* A, int64_t lda, const double* B, int64_t ldb, const double* beta,
                                  double* C, int64_t ldc, DeviceBuffer&, CublasLtPlanCache&, std::size_t,
                                  cudaStream_t stream) {
#ifdef EIGEN_B200_GPU_GEMM_ASYNC
  const int check = 0;
#else
  const int check = 1;
#endif
  eb2_gemm_status(eb2_dgemm_device(eb2_op(transA), eb2_op(transB), m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc,
                                   stream, check));
}

template <>
inline void cublaslt_gemm<float>(cublasLtHandle_t, cublasHandle_t, cublasOperation_t transA,
                                 cublasOperation_t transB, int64_t m, int64_t n, int64_t k, const float* alpha,
                                 const float* A, int64_t lda, const float* B, int64_t ldb, const float* beta,
                                 float* C, int64_t ldc, DeviceBuffer&, CublasLtPlanCache&, std::size_t,
                                 cudaStream_t stream) {
  eb2_gemm_status(
      eb2_sgemm_device(eb2_op(transA), eb2_op(transB), m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc, stream));
}

}  // namespace internal
}  // namespace gpu
}  // namespace Eigen

#endif  // EIGEN_B200_EIGEN_GPU_GEMM_H
