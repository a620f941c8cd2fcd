// ozaki.cu -- FP64 GEMM emulated on the INT8 tensor cores (Ozaki scheme).
//
// Method (Ozaki, Ogita, Oishi & Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59, 2012; INT8 form after Ootomo, Ozaki &
// Yokota, IJHPCA 2024):
//   * every row i of op(A) is scaled by 2^-e_i (e_i = binary exponent of the
//     row's max |a|) and written as s balanced base-2^7 digits d_p in [-64, 64]:
//         a_ik = 2^e_i * sum_p d_p,ik * 2^(-6 - 7(p-1))  (+ remainder <= 2^(e_i-7s));
//     every column j of op(B) likewise with exponents f_j;
//   * the digit products D_t = sum_{p+q=t} Dp_A * Dq_B^T are exact in INT32
//     (tcgen05.mma kind::i8, s32 accumulate in TMEM) as long as one
//     accumulation covers fewer than 2^19 digit products per output;
//   * C = beta*C + alpha * 2^(e_i+f_j) * sum_{t=2..s+1} 2^(-12-7(t-2)) D_t, the
//     recombination done in FP64 by the GEMM's epilogue, diagonals summed from
//     the smallest weight up.
// The digit split is the GPU counterpart of Eigen's gemm_pack_lhs/gemm_pack_rhs
// (Eigen/src/Core/products/GeneralBlockPanelKernel.h:1879-2478): it reads op(A)
// and op(B) through their leading dimensions and transposes, and writes K-major,
// zero-padded panels that the TMA loads as 128-byte swizzled tiles.
#include <cuda.h>

#include <climits>

#include "device_common.cuh"
#include "kernels.h"
#include "slice_gemm.cuh"
#include "tma_host.h"

namespace eb2 {

namespace {

constexpr uint64_t kInfBits = 0x7FF0000000000000ull;

// ------------------------------------------------------------------ scan
constexpr int kScanTile = 64;

// Besides the row maxima, every 8th column tile contributes to the exponent-spread
// statistic used by the configuration picker: per row chunk, (largest exponent) minus
// (mean exponent of its nonzero entries), summed in spread[0] with the chunk count in
// spread[1].
__global__ void __launch_bounds__(256) ozaki_scan_kernel(const double* __restrict__ X, int64_t rows, int64_t cols,
                                                         int64_t sr, int64_t sl, unsigned long long* maxbits,
                                                         double* abssum, int* nonfinite, double* spread) {
  __shared__ double tile[kScanTile][kScanTile + 1];
  const int64_t r0 = int64_t(blockIdx.y) * kScanTile;
  const int64_t l0 = int64_t(blockIdx.x) * kScanTile;
  const bool rows_contig = (sr == 1);
  for (int idx = threadIdx.x; idx < kScanTile * kScanTile; idx += blockDim.x) {
    int rr, ll;
    if (rows_contig) {
      rr = idx % kScanTile;
      ll = idx / kScanTile;
    } else {
      ll = idx % kScanTile;
      rr = idx / kScanTile;
    }
    const int64_t r = r0 + rr, l = l0 + ll;
    double v = 0.0;
    if (r < rows && l < cols) v = X[r * sr + l * sl];
    tile[rr][ll] = v;
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < kScanTile) {
    const int64_t r = r0 + t;
    double chunk_spread = 0.0, chunk_count = 0.0;
    if (r < rows) {
      unsigned long long mb = 0;
      int esum = 0, ecnt = 0;
      for (int ll = 0; ll < kScanTile; ++ll) {
        unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(fabs(tile[t][ll])));
        mb = b > mb ? b : mb;
        if (b) {
          esum += int(b >> 52);
          ++ecnt;
        }
      }
      if (mb >= kInfBits) *nonfinite = 1;
      if (mb) atomicMax(&maxbits[r], mb);
      if (ecnt > 0 && mb < kInfBits) {
        chunk_spread = double(int(mb >> 52)) - double(esum) / double(ecnt);
        chunk_count = 1.0;
      }
    }
    if (spread != nullptr && (blockIdx.x & 7) == 0) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        chunk_spread += __shfl_xor_sync(0xffffffffu, chunk_spread, o);
        chunk_count += __shfl_xor_sync(0xffffffffu, chunk_count, o);
      }
      if ((t & 31) == 0 && chunk_count > 0.0) {
        atomicAdd(&spread[0], chunk_spread);
        atomicAdd(&spread[1], chunk_count);
      }
    }
  } else if (abssum != nullptr && t < 2 * kScanTile) {
    const int ll = t - kScanTile;
    const int64_t l = l0 + ll;
    if (l < cols) {
      double s = 0.0;
      for (int rr = 0; rr < kScanTile; ++rr) s += fabs(tile[rr][ll]);
      if (s != 0.0) atomicAdd(&abssum[l], s);
    }
  }
}

// ------------------------------------------------------------------ split
constexpr int kSplitRows = 32;
constexpr int kSplitCols = 128;

__device__ __forceinline__ int row_exponent(unsigned long long mb) {
  if (mb >= kInfBits) return INT_MIN;
  if (mb == 0) return 0;
  int e;
  frexp(__longlong_as_double(static_cast<long long>(mb)), &e);
  return e;
}

__global__ void __launch_bounds__(256) ozaki_split_kernel(const double* __restrict__ X, int64_t rows, int64_t cols,
                                                          int64_t sr, int64_t sl,
                                                          const unsigned long long* __restrict__ maxbits,
                                                          int8_t* __restrict__ digits, int32_t* __restrict__ exps,
                                                          int64_t rows_pad, int64_t k_pad, int p_begin, int p_end) {
  __shared__ double tile[kSplitRows][kSplitCols + 1];
  __shared__ int row_e[kSplitRows];
  const int64_t r0 = int64_t(blockIdx.y) * kSplitRows;
  const int64_t l0 = int64_t(blockIdx.x) * kSplitCols;
  const bool rows_contig = (sr == 1);
  if (threadIdx.x < kSplitRows) {
    const int64_t r = r0 + threadIdx.x;
    int e = (r < rows) ? row_exponent(maxbits[r]) : 0;
    row_e[threadIdx.x] = e;
    if (blockIdx.x == 0 && r < rows_pad) exps[r] = e;
  }
  for (int idx = threadIdx.x; idx < kSplitRows * kSplitCols; idx += blockDim.x) {
    int rr, ll;
    if (rows_contig) {
      rr = idx % kSplitRows;
      ll = idx / kSplitRows;
    } else {
      ll = idx % kSplitCols;
      rr = idx / kSplitCols;
    }
    const int64_t r = r0 + rr, l = l0 + ll;
    double v = 0.0;
    if (r < rows && l < cols) v = X[r * sr + l * sl];
    tile[rr][ll] = v;
  }
  __syncthreads();
  // thread -> (row, 16 consecutive columns)
  const int rr = threadIdx.x >> 3;
  const int cb = (threadIdx.x & 7) * 16;
  const int e = row_e[rr];
  double rem[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    double x = (e == INT_MIN) ? 0.0 : ldexp(tile[rr][cb + j], -e);
    rem[j] = __dmul_rn(x, 64.0);
  }
  const int64_t row = r0 + rr;
  for (int p = 0; p < p_end; ++p) {
    uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const double d = rint(rem[j]);
      rem[j] = __dmul_rn(__dsub_rn(rem[j], d), 128.0);
      const uint32_t byte = static_cast<uint32_t>(static_cast<int>(d)) & 0xFFu;
      w[j >> 2] |= byte << (8 * (j & 3));
    }
    if (p >= p_begin) {
      uint4* dst = reinterpret_cast<uint4*>(digits + (size_t(p) * size_t(rows_pad) + size_t(row)) * size_t(k_pad) +
                                            size_t(l0 + cb));
      *dst = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// Tile configurations of the Ozaki GEMM (the FP64 accumulator lives in registers, so a
// CTA's tile is 128 x 128 with 8 epilogue warps): one CTA per 128 x 128 tile, or a CTA
// pair per 256 x 128 tile (the default; half the B bytes per SM).
template <int BN, int STAGES, bool PAIR>
cudaError_t launch_config(const OzakiOperand& a, const OzakiOperand& b, const OzakiGemmArgs& args,
                          cudaStream_t stream) {
  constexpr int kRowsPerTile = PAIR ? 2 * kSliceBM : kSliceBM;
  if (a.rows_pad % kRowsPerTile != 0 || b.rows_pad % BN != 0) return cudaErrorInvalidValue;
  CUtensorMap tmA, tmB;
  if (!make_tensor_map_3d(&tmA, a.digits, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, uint64_t(a.k_pad), uint64_t(a.rows_pad),
                          uint64_t(a.smax), kSliceKBytes, kSliceBM))
    return cudaErrorInvalidValue;
  if (!make_tensor_map_3d(&tmB, b.digits, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, uint64_t(b.k_pad), uint64_t(b.rows_pad),
                          uint64_t(b.smax), kSliceKBytes, PAIR ? BN / 2 : BN))
    return cudaErrorInvalidValue;
  SliceGemmParams P{};
  P.m = args.m;
  P.n = args.n;
  P.num_kb = int(a.k_pad / kSliceKBytes);
  P.tiles_m = int(a.rows_pad / kRowsPerTile);
  P.tiles_n = int(b.rows_pad / BN);
  P.slices = args.slices;
  P.diag_lo = args.diag_lo;
  P.diag_hi = args.diag_hi;
  P.first_writes = args.first_writes ? 1 : 0;
  P.alpha = args.alpha;
  P.beta = args.beta;
  P.C = args.C;
  P.ldc = args.ldc;
  P.expA = a.exps;
  P.expB = b.exps;
  P.skip_if_flag = args.skip_if_flag;
  P.err_sq = args.err_sq;
  P.status = args.status;
  P.group_m = tuning().group_m > 0 ? tuning().group_m : P.tiles_m;
  P.wait_limit_ns = tuning().wait_limit_ns ? tuning().wait_limit_ns : kWaitLimitNs;
  return launch_slice_gemm<kModeOzakiI8, BN, STAGES, 8, PAIR>(tmA, tmB, P, args.num_sms, stream);
}

}  // namespace

cudaError_t launch_ozaki_scan_reset(const OzakiOperand& op, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(op.maxbits, 0, size_t(op.rows) * sizeof(uint64_t), stream);
  if (e != cudaSuccess || op.abssum == nullptr) return e;
  return cudaMemsetAsync(op.abssum, 0, size_t(op.k) * sizeof(double), stream);
}

cudaError_t launch_ozaki_scan(const StridedView<double>& x, const OzakiOperand& op, int* nonfinite, double* spread,
                              cudaStream_t stream) {
  if (x.rows == 0 || x.cols == 0) return cudaSuccess;
  dim3 grid(unsigned((x.cols + kScanTile - 1) / kScanTile), unsigned((x.rows + kScanTile - 1) / kScanTile));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  ozaki_scan_kernel<<<grid, 256, 0, stream>>>(x.ptr, x.rows, x.cols, x.sr, x.sl,
                                              reinterpret_cast<unsigned long long*>(op.maxbits), op.abssum,
                                              nonfinite, spread);
  return cudaGetLastError();
}

cudaError_t launch_ozaki_split(const StridedView<double>& x, const OzakiOperand& op, int p_begin, int p_end,
                               cudaStream_t stream) {
  if (p_end > op.smax || p_begin < 0 || p_begin >= p_end) return cudaErrorInvalidValue;
  if (op.k_pad % kSplitCols != 0 || op.rows_pad % kSplitRows != 0) return cudaErrorInvalidValue;
  dim3 grid(unsigned(op.k_pad / kSplitCols), unsigned(op.rows_pad / kSplitRows));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  ozaki_split_kernel<<<grid, 256, 0, stream>>>(x.ptr, x.rows, x.cols, x.sr, x.sl,
                                               reinterpret_cast<const unsigned long long*>(op.maxbits), op.digits,
                                               op.exps, op.rows_pad, op.k_pad, p_begin, p_end);
  return cudaGetLastError();
}

cudaError_t launch_ozaki_gemm(const OzakiOperand& a, const OzakiOperand& b, const OzakiGemmArgs& args,
                              cudaStream_t stream) {
  if (args.slices < 1 || args.slices > a.smax || args.slices > b.smax) return cudaErrorInvalidValue;
  if (a.k_pad != b.k_pad || a.k_pad % kSliceKBytes != 0) return cudaErrorInvalidValue;
  if (args.tile_n == 128) return launch_config<128, 6, false>(a, b, args, stream);
  if (args.tile_n == 256 || args.tile_n == kTilePair) return launch_config<128, 8, true>(a, b, args, stream);
  return cudaErrorInvalidValue;
}

}  // namespace eb2
