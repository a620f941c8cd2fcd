/*
 * eigen_b200/eigen_tensor_gpu_contraction.h -- routes Eigen Tensor contractions evaluated on
 * the GPU device (Eigen::GpuDevice) to libeigen_b200.so when they are plain matrix products.
 *
 * Eigen's GPU contraction (unsupported/Eigen/src/Tensor/TensorContractionGpu.h) launches its
 * own SIMT kernels through LaunchKernels, a member template of the evaluator that cannot be
 * specialised from outside. eigen_tensor_gpu_contraction.patch (next to this header) adds a
 * customisation point to that file: Eigen::internal::TensorContractionGpuGemm<Scalar, Index>,
 * called from the evaluator's evalTyped when both operands are held in device memory and the
 * contraction is op(A) (m x k) * op(B) (k x n), A stored m x k or k x m and B stored k x n or
 * n x k (contracted dimensions at one end of each operand, in matching order). This header
 * specialises it for double and float: eb2_dgemm_device / eb2_sgemm_device on the device's
 * stream, with beta = 0, so the product runs on this library's B200 kernels (for FP64, the
 * CRT emulation with its accuracy check, or the FP64 kernel that the method setting
 * chooses). Contractions of any other shape, and other scalar types, keep Eigen's kernels; so
 * does a product the library refuses (it returns false and Eigen computes the result).
 *
 * Use: apply the patch to the Eigen tree, define EIGEN_USE_GPU, include
 * <unsupported/Eigen/Tensor>, then this header, before the first contraction on a GpuDevice
 * in the translation unit. Link with -leigen_b200.
 *
 * eb2_tensor_gpu_gemm_calls() counts the contractions this header ran in the library.
 */
#ifndef EIGEN_B200_EIGEN_TENSOR_GPU_CONTRACTION_H
#define EIGEN_B200_EIGEN_TENSOR_GPU_CONTRACTION_H

#if !defined(EIGEN_USE_GPU)
#error "define EIGEN_USE_GPU and include <unsupported/Eigen/Tensor> before eigen_b200/eigen_tensor_gpu_contraction.h"
#endif

#include <atomic>

#include "eigen_b200/blas.h"

inline std::atomic<long long>& eb2_tensor_gpu_gemm_counter() {
  static std::atomic<long long> calls{0};
  return calls;
}
inline long long eb2_tensor_gpu_gemm_calls() { return eb2_tensor_gpu_gemm_counter().load(); }

// Eigen's GPU contraction (and the customisation point) exists only in device-compiled
// translation units
#if defined(EIGEN_GPUCC)
namespace Eigen {
namespace internal {

template <typename Index>
struct TensorContractionGpuGemm<double, Index> {
  static bool run(bool trans_a, bool trans_b, Index m, Index n, Index k, const double* a, Index lda, const double* b,
                  Index ldb, double* c, Index ldc, const GpuDevice& device) {
    const int rc = eb2_dgemm_device(trans_a ? 'T' : 'N', trans_b ? 'T' : 'N', m, n, k, 1.0, a, lda < 1 ? 1 : lda, b,
                                    ldb < 1 ? 1 : ldb, 0.0, c, ldc < 1 ? 1 : ldc, (void*)device.stream(), 1);
    if (rc != EB2_OK) return false;
    eb2_tensor_gpu_gemm_counter().fetch_add(1);
    return true;
  }
};

template <typename Index>
struct TensorContractionGpuGemm<float, Index> {
  static bool run(bool trans_a, bool trans_b, Index m, Index n, Index k, const float* a, Index lda, const float* b,
                  Index ldb, float* c, Index ldc, const GpuDevice& device) {
    const int rc = eb2_sgemm_device(trans_a ? 'T' : 'N', trans_b ? 'T' : 'N', m, n, k, 1.0f, a, lda < 1 ? 1 : lda, b,
                                    ldb < 1 ? 1 : ldb, 0.0f, c, ldc < 1 ? 1 : ldc, (void*)device.stream());
    if (rc != EB2_OK) return false;
    eb2_tensor_gpu_gemm_counter().fetch_add(1);
    return true;
  }
};

}  // namespace internal
}  // namespace Eigen
#endif  // EIGEN_GPUCC

#endif  // EIGEN_B200_EIGEN_TENSOR_GPU_CONTRACTION_H
