// grouped.cu -- one persistent launch for thousands of independent small products.
//
// Eigen has no batch entry point: fixed-size products (3x3 ... 8x8) never reach GEBP
// but are unrolled coefficient-based products (Eigen/src/Core/GeneralProduct.h:76-80,
// Eigen/src/Core/ProductEvaluators.h:703-880), and dynamic ones each go through
// general_matrix_matrix_product.  Here a whole batch is one launch:
//   * every problem is cut into 32 x 32 output tiles ("work items"); an item is computed
//     by ONE warp: FP64 with mma.sync m16n8k4 (2 x 4 fragments), FP32 with FFMA
//     (4 x 8 outputs per lane), operands read straight from global memory through the
//     read-only cache (no shared memory, no block-level synchronisation, so many
//     warps per SM hide the latency of the small, scattered operands);
//   * warps pull items from a global counter; the host orders items longest-K first
//     (largest first, a greedy balance of the uneven sizes);
//   * C = alpha*op(A)op(B) + beta*C per problem with the BLAS rules (beta == 0 never reads
//     C, alpha == 0 or k == 0 leaves beta*C).
#include <cstdint>

#include "device_common.cuh"
#include "grouped.h"

namespace eb2 {

namespace {

constexpr int kTile = 32;

// op(A)(i,l) and op(B)(l,j) with zero outside the problem
template <typename T>
__device__ __forceinline__ T load_op(const T* X, int64_t ld, bool trans, int64_t r, int64_t c, int64_t rows,
                                     int64_t cols) {
  if (r >= rows || c >= cols) return T(0);
  return trans ? __ldg(X + c + r * ld) : __ldg(X + r + c * ld);
}

__device__ __forceinline__ void dmma_16x8x4_g(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// One 32 x 32 FP64 tile by one warp.
__device__ void tile_f64(const GroupedProblem& pr, int tm, int tn, int lane) {
  const int g = lane >> 2, tig = lane & 3;
  const int64_t m0 = int64_t(tm) * kTile, n0 = int64_t(tn) * kTile;
  const double* A = static_cast<const double*>(pr.a);
  const double* B = static_cast<const double*>(pr.b);
  const bool ta = pr.trans & 1, tb = (pr.trans >> 1) & 1;
  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][j][c] = 0.0;
  if (pr.alpha != 0.0) {
    // the fragments of step k0 + 4 are loaded while the MMAs of step k0 run
    auto load = [&](int64_t k0, double (&af)[2][2], double (&bf)[4]) {
      const int64_t kk = k0 + tig;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        af[i][0] = load_op(A, pr.lda, ta, m0 + i * 16 + g, kk, pr.m, pr.k);
        af[i][1] = load_op(A, pr.lda, ta, m0 + i * 16 + g + 8, kk, pr.m, pr.k);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = load_op(B, pr.ldb, tb, kk, n0 + j * 8 + g, pr.k, pr.n);
    };
    double af[2][2], bf[4];
    load(0, af, bf);
    for (int64_t k0 = 0; k0 < pr.k; k0 += 4) {
      double an[2][2], bn[4];
      const bool more = k0 + 4 < pr.k;
      if (more) load(k0 + 4, an, bn);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_16x8x4_g(acc[i][j], af[i][0], af[i][1], bf[j]);
      if (more) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          af[i][0] = an[i][0];
          af[i][1] = an[i][1];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = bn[j];
      }
    }
  }
  double* C = static_cast<double*>(pr.c);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int64_t row = m0 + i * 16 + g + h * 8;
          const int64_t col = n0 + j * 8 + tig * 2 + cc;
          if (row < pr.m && col < pr.n) {
            double* dst = C + row + col * pr.ldc;
            const double v = __dmul_rn(pr.alpha, acc[i][j][h * 2 + cc]);
            *dst = (pr.beta == 0.0) ? v : __fma_rn(pr.beta, *dst, v);
          }
        }
}

// One 32 x 32 FP32 tile by one warp: lane -> rows 4*(lane%8)..+3, cols 8*(lane/8)..+7.
__device__ void tile_f32(const GroupedProblem& pr, int tm, int tn, int lane) {
  const int64_t m0 = int64_t(tm) * kTile + 4 * (lane & 7), n0 = int64_t(tn) * kTile + 8 * (lane >> 3);
  const float* A = static_cast<const float*>(pr.a);
  const float* B = static_cast<const float*>(pr.b);
  const bool ta = pr.trans & 1, tb = (pr.trans >> 1) & 1;
  const float alpha = float(pr.alpha), beta = float(pr.beta);
  float acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  if (alpha != 0.f) {
    for (int64_t l = 0; l < pr.k; ++l) {
      float av[4], bv[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = load_op(A, pr.lda, ta, m0 + i, l, pr.m, pr.k);
#pragma unroll
      for (int j = 0; j < 8; ++j) bv[j] = load_op(B, pr.ldb, tb, l, n0 + j, pr.k, pr.n);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
  }
  float* C = static_cast<float*>(pr.c);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int64_t row = m0 + i, col = n0 + j;
      if (row < pr.m && col < pr.n) {
        float* dst = C + row + col * pr.ldc;
        const float v = __fmul_rn(alpha, acc[i][j]);
        *dst = (beta == 0.f) ? v : __fmaf_rn(beta, *dst, v);
      }
    }
}

// FP64: six two-warp blocks per SM (at most 168 registers; measured 26% faster than the
// 190 registers the compiler takes otherwise); FP32 eight (128 registers).
template <bool F64>
__global__ void __launch_bounds__(64, F64 ? 6 : 8) grouped_gemm_kernel(const GroupedProblem* __restrict__ problems,
                                                           const GroupedItem* __restrict__ items, int64_t num_items,
                                                           unsigned long long* counter) {
  const int lane = threadIdx.x & 31;
  while (true) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(counter, 1ull);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= static_cast<unsigned long long>(num_items)) break;
    const GroupedItem it = items[idx];
    const GroupedProblem pr = problems[it.problem];
    if (F64)
      tile_f64(pr, it.tile_m, it.tile_n, lane);
    else
      tile_f32(pr, it.tile_m, it.tile_n, lane);
  }
}

}  // namespace

cudaError_t launch_grouped_gemm(bool f64, const GroupedProblem* problems, const GroupedItem* items,
                                int64_t num_items, unsigned long long* counter, int num_sms, cudaStream_t stream) {
  if (num_items <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
  // two-warp blocks: an SM holds six (FP64) or eight (FP32) of them, where only one
  // eight-warp block would fit at the tile code's register count
  const int warps_per_block = 2;
  int64_t blocks = (num_items + warps_per_block - 1) / warps_per_block;
  const int64_t cap = int64_t(num_sms) * 16;
  if (blocks > cap) blocks = cap;
  if (f64)
    grouped_gemm_kernel<true><<<unsigned(blocks), 32 * warps_per_block, 0, stream>>>(problems, items, num_items,
                                                                                     counter);
  else
    grouped_gemm_kernel<false><<<unsigned(blocks), 32 * warps_per_block, 0, stream>>>(problems, items, num_items,
                                                                                      counter);
  return cudaGetLastError();
}

}  // namespace eb2
