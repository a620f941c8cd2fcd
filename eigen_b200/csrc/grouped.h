// grouped.h -- device descriptors and launcher of the grouped (batched) GEMM.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace eb2 {

struct GroupedProblem {
  int64_t m, n, k;
  int64_t lda, ldb, ldc;
  const void* a;
  const void* b;
  void* c;
  double alpha, beta;
  int trans;  // bit 0: op(A) transposed, bit 1: op(B) transposed
  int pad_;
};

struct GroupedItem {
  uint32_t problem;
  uint16_t tile_m, tile_n;  // 32 x 32 output tile coordinates
};

// Zeroes the work counter and launches the persistent grouped kernel on `stream`.
cudaError_t launch_grouped_gemm(bool f64, const GroupedProblem* problems, const GroupedItem* items,
                                int64_t num_items, unsigned long long* counter, int num_sms, cudaStream_t stream);

}  // namespace eb2
