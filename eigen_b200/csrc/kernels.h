// kernels.h -- internal host-side interface of the device kernels (launch wrappers).
// Everything here is stream-ordered and allocation-free: callers pass device
// buffers that they own.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace eb2 {

// Launch-shape knobs of the tcgen05 slice GEMM (set by the tuner; process-wide).
struct SliceTuning {
  int group_m = 0;   // row-tiles per raster group; 0 = all (column-major tile order)
  int prefetch = 0;  // L2 prefetch distance in K blocks; 0 = off
};
SliceTuning& tuning();

// A strided view of op(X) as a rows x cols matrix: element (r, l) at X[r*sr + l*sl].
template <typename T>
struct StridedView {
  const T* ptr;
  int64_t rows, cols;
  int64_t sr, sl;
};

// ------------------------------------------------------------ native FP64 / FP32
// C = alpha * op(A) op(B) + beta * C, column-major, device pointers.
// If `only_if_flag` is non-null the kernel does nothing unless *only_if_flag != 0
// (device-side fallback for inputs the emulated path cannot represent).
cudaError_t launch_dgemm_native(bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                                const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                                int64_t ldc, const int* only_if_flag, cudaStream_t stream);
cudaError_t launch_sgemm_native(bool transA, bool transB, int64_t m, int64_t n, int64_t k, float alpha,
                                const float* A, int64_t lda, const float* B, int64_t ldb, float beta, float* C,
                                int64_t ldc, const int* only_if_flag, cudaStream_t stream);
// C = beta * C (beta == 0 writes exact zeros), the BLAS pre-scale for alpha == 0 or k == 0.
cudaError_t launch_scale_matrix_d(int64_t m, int64_t n, double beta, double* C, int64_t ldc, cudaStream_t stream);
cudaError_t launch_scale_matrix_s(int64_t m, int64_t n, float beta, float* C, int64_t ldc, cudaStream_t stream);

// ------------------------------------------------------------ Ozaki (emulated FP64)
constexpr int kOzakiMaxSlices = 12;
// Tile configurations of the tcgen05 kernels: 128 / 256 = one CTA computing 128 x 128 /
// 128 x 256 tiles; kTilePair = a CTA pair (cluster of 2) computing 256 x 256 tiles.
constexpr int kTilePair = 512;
constexpr int kOzakiKBlock = 128;  // bytes of K per pipeline stage (int8 digits)
constexpr int kOzakiBM = 128;

// Per-operand workspace of the digit split.
struct OzakiOperand {
  int8_t* digits;       // [smax][rows_pad][k_pad], row r contiguous along k
  int32_t* exps;        // [rows_pad] binary exponent of each row's max |x|
  uint64_t* maxbits;    // [rows] bit pattern of max |x| (scan output)
  double* abssum;       // [k] sum over rows of |x|; optional (null skips it)
  int64_t rows, rows_pad, k, k_pad;
  int smax;
};

// Zero the scan accumulators of one operand (maxbits, abssum).
cudaError_t launch_ozaki_scan_reset(const OzakiOperand& op, cudaStream_t stream);
// Row maxima and |x| sums; sets *nonfinite when any NaN/Inf is present; accumulates the
// exponent-spread statistic into spread[0..1] (sum, count) when spread is non-null.
cudaError_t launch_ozaki_scan(const StridedView<double>& x, const OzakiOperand& op, int* nonfinite, double* spread,
                              cudaStream_t stream);
// Digits p in [p_begin, p_end) of every row (including zero padding).
cudaError_t launch_ozaki_split(const StridedView<double>& x, const OzakiOperand& op, int p_begin, int p_end,
                               cudaStream_t stream);

struct OzakiGemmArgs {
  int64_t m, n, k;
  double alpha, beta;
  double* C;
  int64_t ldc;
  int slices;          // s: digits per operand used by this call
  int diag_lo, diag_hi;  // accumulate diagonals t in [diag_lo, diag_hi] (t = p + q, digits p,q >= 1)
  bool first_writes;   // true: the first unit applies beta (C = beta*C + ...); false: C += ...
  const int* skip_if_flag;  // non-null: the kernel returns at once when *flag != 0
  double* err_sq;      // [2]: += squared contribution of diagonal diag_hi, and of diagonal 2 (may be null)
  uint32_t* status;    // device status word (EB2_DEV_*)
  int tile_n;          // 128, 256 or kTilePair
  int num_sms;
};
cudaError_t launch_ozaki_gemm(const OzakiOperand& a, const OzakiOperand& b, const OzakiGemmArgs& args,
                              cudaStream_t stream);

// ------------------------------------------------------------ split-BF16 (emulated FP32)
struct Bf16Operand {
  void* pieces;  // [3][rows_pad][k_pad] bf16: hi, mid, lo pieces, row r contiguous along k
  int64_t rows, rows_pad, k, k_pad;
};
// Split op(X) (rows x k view) into its three BF16 pieces; sets *nonfinite on NaN/Inf.
cudaError_t launch_bf16_split(const StridedView<float>& x, const Bf16Operand& op, int* nonfinite,
                              cudaStream_t stream);

struct SgemmSplitArgs {
  int64_t m, n, k;
  float alpha, beta;
  float* C;
  int64_t ldc;
  int pieces;  // s: 2 -> 3 products (hh, hm, mh), 3 -> 6 products (+ mm, hl, lh)
  const int* skip_if_flag;
  uint32_t* status;
  int tile_n;
  int num_sms;
};
cudaError_t launch_sgemm_split_bf16(const Bf16Operand& a, const Bf16Operand& b, const SgemmSplitArgs& args,
                                    cudaStream_t stream);

}  // namespace eb2
