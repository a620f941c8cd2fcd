// grouped.h -- device descriptors and launchers of the grouped (batched) GEMM.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace eb2 {

struct GroupedProblem {
  int64_t m, n, k;  // k = 0 when alpha == 0 (A and B are not read)
  int64_t lda, ldb, ldc;
  const void* a;
  const void* b;
  void* c;
  double alpha, beta;
  int trans;  // bit 0: op(A) transposed, bit 1: op(B) transposed
  int pad_;
};

constexpr uint32_t kNoProblem = 0xFFFFFFFFu;

// One warp's work: class 32 = the 32 x 32 output tile (tile_m, tile_n) of problem[0];
// class 16 = problems problem[0..1], each at most 16 x 16; class 8 = problem[0..3], each at
// most 8 x 8 (empty slots hold kNoProblem).  k = the largest k of the item's problems.
struct GroupedItem {
  uint32_t problem[4];
  int32_t k;
  uint16_t tile_m, tile_n;
  uint8_t cls;
  uint8_t pad_[7];
};
static_assert(sizeof(GroupedItem) == 32, "one 32-byte load per item");

// Grid of the persistent grouped kernel for `num_items` items (as many two-warp blocks as fit
// on the SMs, at most one warp per item); sets the kernel's shared-memory attribute.  Call it
// outside any stream capture.
cudaError_t grouped_grid(bool f64, int64_t num_items, int num_sms, unsigned* blocks);
// Launches the persistent grouped kernel for `num_items` items on `stream` with `blocks`
// blocks from grouped_grid (capturable).
cudaError_t launch_grouped_gemm(bool f64, const GroupedProblem* problems, const GroupedItem* items,
                                int64_t num_items, unsigned blocks, cudaStream_t stream);
// The same arithmetic for one product (one warp per 32 x 32 tile): the per-product launches
// that a grouped launch replaces.
cudaError_t launch_grouped_one(bool f64, const GroupedProblem& pr, cudaStream_t stream);
// Dynamic shared memory of one block of the grouped kernel.
size_t grouped_block_smem(bool f64);

// Largest max(m, n) of the products that share a warp four (class 8) or two (class 16) at a
// time; 0 disables the class.  Process-wide; read when a plan is built.
struct GroupedClasses {
  int small_max = 8;
  int mid_max = 16;
  bool automatic = true;  // not set by the caller: a forced configuration class or the picker decides
};
GroupedClasses& grouped_classes();

}  // namespace eb2
