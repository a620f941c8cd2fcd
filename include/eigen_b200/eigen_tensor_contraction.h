/*
 * eigen_b200/eigen_tensor_contraction.h -- runs the double-precision contractions of
 * Eigen's Tensor module on libeigen_b200.so.
 *
 * Eigen evaluates a tensor contraction as a GEMM over the contraction's row and column index
 * sets. Its evaluator (unsupported/Eigen/src/Tensor/TensorContraction.h:848-936, and the
 * thread-pool evaluator) cuts the product into blocks with
 * internal::TensorContractionBlocking and hands every block to
 * internal::TensorContractionKernel, the customisation point documented at
 * TensorContraction.h:128-157 ("by specializing contraction kernels we can use other low
 * level libraries to perform matrix multiplication"). This header specialises both for
 * double:
 *   - the blocking takes the whole product as one block (kc = k, mc = m, nc = n), so a
 *     contraction is a single product and not thousands of cache-sized ones;
 *   - the kernel packs the two operands through Eigen's contraction mappers into
 *     column-major buffers (on the host's cores for large operands), and invoke() is one
 *     dgemm_ call on the output block (alpha, and beta = 0 on the first K block:
 *     HasBeta = true). The library stages the host buffers through device memory and runs
 *     its B200 product (the CRT emulation or the FP64 kernel, with the method setting and
 *     accuracy check of dgemm_).
 * Other scalar types keep Eigen's own kernel.
 *
 * Use: include <unsupported/Eigen/Tensor>, then this header, before the first double
 * contraction in the translation unit; link with -leigen_b200. Every translation unit of a
 * program that contracts double tensors must include it, since the specialisation changes
 * what the contraction templates instantiate to.
 */
#ifndef EIGEN_B200_EIGEN_TENSOR_CONTRACTION_H
#define EIGEN_B200_EIGEN_TENSOR_CONTRACTION_H

#ifndef EIGEN_TENSOR_MODULE_H
#error "include <unsupported/Eigen/Tensor> before eigen_b200/eigen_tensor_contraction.h"
#endif

#include <thread>
#include <vector>

#include "eigen_b200/blas.h"

namespace Eigen {
namespace internal {

// Runs fn(c0, c1) over [0, cols) split into contiguous ranges on the host's cores: packing
// reads every element through Eigen's contraction mapper (index arithmetic per element), so
// for large operands it is spread over threads; small ones stay on the calling thread.
template <typename Index, typename Fn>
void eb2_parallel_columns(Index cols, Index rows, Fn&& fn) {
  const unsigned hw = std::thread::hardware_concurrency();
  const Index work = cols * rows;
  const Index nthreads = Index(hw == 0 ? 1 : hw) < cols ? Index(hw == 0 ? 1 : hw) : cols;
  if (work < (Index(1) << 20) || nthreads <= 1) {
    fn(Index(0), cols);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(size_t(nthreads));
  for (Index t = 0; t < nthreads; ++t) {
    const Index c0 = cols * t / nthreads, c1 = cols * (t + 1) / nthreads;
    pool.emplace_back([&fn, c0, c1] { fn(c0, c1); });
  }
  for (auto& th : pool) th.join();
}

// The whole product is one block.
template <typename StorageIndex, int ShardingType>
class TensorContractionBlocking<double, double, double, StorageIndex, ShardingType> {
 public:
  TensorContractionBlocking(StorageIndex k, StorageIndex m, StorageIndex n, StorageIndex /*num_threads*/ = 1)
      : kc_(k), mc_(m), nc_(n) {}
  EIGEN_ALWAYS_INLINE StorageIndex kc() const { return kc_; }
  EIGEN_ALWAYS_INLINE StorageIndex mc() const { return mc_; }
  EIGEN_ALWAYS_INLINE StorageIndex nc() const { return nc_; }

 private:
  StorageIndex kc_, mc_, nc_;
};

template <typename StorageIndex, typename OutputMapper, typename LhsMapper, typename RhsMapper>
struct TensorContractionKernel<double, double, double, StorageIndex, OutputMapper, LhsMapper, RhsMapper> {
  static constexpr bool HasBeta = true;

  TensorContractionKernel(StorageIndex m_, StorageIndex k_, StorageIndex n_, StorageIndex bm_, StorageIndex bk_,
                          StorageIndex bn_)
      : m(m_), k(k_), n(n_), bm(bm_), bk(bk_), bn(bn_) {}

  using LhsBlock = double*;
  using RhsBlock = double*;
  using BlockMemAllocator = TensorContractionBlockMemAllocator<double, double>;
  using BlockMemHandle = typename BlockMemAllocator::BlockMemHandle;

  template <typename Device>
  BlockMemHandle allocate(Device& d, LhsBlock* lhs_block, RhsBlock* rhs_block) {
    return BlockMemAllocator::allocate(d, bm, bk, bn, lhs_block, rhs_block);
  }

  template <typename Device>
  BlockMemHandle allocateSlices(Device& d, const StorageIndex num_lhs, const StorageIndex num_rhs,
                                const StorageIndex num_slices, std::vector<LhsBlock>* lhs_blocks,
                                std::vector<RhsBlock>* rhs_blocks) {
    return BlockMemAllocator::allocateSlices(d, bm, bk, bn, num_lhs, num_rhs, num_slices, lhs_blocks, rhs_blocks);
  }

  template <typename Device>
  static void deallocate(Device& d, BlockMemHandle handle) {
    BlockMemAllocator::deallocate(d, handle);
  }

  // rows x depth block of the left operand, column-major with leading dimension rows
  void packLhs(LhsBlock* block, const typename LhsMapper::SubMapper& data_mapper, const StorageIndex depth,
               const StorageIndex rows) {
    double* out = *block;
    eb2_parallel_columns(depth, rows, [&](StorageIndex l0, StorageIndex l1) {
      for (StorageIndex l = l0; l < l1; ++l)
        for (StorageIndex i = 0; i < rows; ++i) out[i + l * rows] = data_mapper(i, l);
    });
  }

  // depth x cols block of the right operand, column-major with leading dimension depth
  void packRhs(RhsBlock* block, const typename RhsMapper::SubMapper& data_mapper, const StorageIndex depth,
               const StorageIndex cols) {
    double* out = *block;
    eb2_parallel_columns(cols, depth, [&](StorageIndex j0, StorageIndex j1) {
      for (StorageIndex j = j0; j < j1; ++j)
        for (StorageIndex l = 0; l < depth; ++l) out[l + j * depth] = data_mapper(l, j);
    });
  }

  // output block := alpha * lhs * rhs + beta * output block (one dgemm_)
  void invoke(const OutputMapper& output_mapper, const LhsBlock& lhs_block, const RhsBlock& rhs_block,
              const StorageIndex rows, const StorageIndex depth, const StorageIndex cols, const double alpha,
              const double beta) {
    if (rows == 0 || cols == 0) return;
    const int64_t m64 = rows, n64 = cols, k64 = depth, lda = rows > 0 ? rows : 1, ldb = depth > 0 ? depth : 1,
                  ldc = output_mapper.stride();
    dgemm_64_("N", "N", &m64, &n64, &k64, &alpha, lhs_block, &lda, rhs_block, &ldb, &beta, &output_mapper(0, 0),
              &ldc);
  }

 private:
  const StorageIndex m, k, n, bm, bk, bn;
};

}  // namespace internal
}  // namespace Eigen

#endif  // EIGEN_B200_EIGEN_TENSOR_CONTRACTION_H
