// split_bf16.cu -- SGEMM emulated on the BF16 tensor cores (split-BF16).
//
// Method (Henry, Tang & Heinecke, "Leveraging the bfloat16 Artificial Intelligence
// Datatype For Higher-Precision Computations", ARITH 2019): every FP32 input x is
// written exactly as the sum of three BF16 pieces
//     h = bf16(x),  m = bf16(x - h),  l = bf16(x - h - m),
// (each difference is exact in FP32).  The product keeps the pieces' cross products
// with p + q <= s + 1 (pieces numbered h = 1, m = 2, l = 3): s = 2 gives the three
// products hh + hm + mh ("bf16x3"), s = 3 adds mm + hl + lh ("bf16x6").  All of them
// accumulate in FP32 in one TMEM accumulator of the shared slice GEMM, smallest
// products first, and the epilogue applies C = alpha*acc + beta*C.
// The split is the GPU counterpart of Eigen's gemm_pack_lhs/gemm_pack_rhs
// (Eigen/src/Core/products/GeneralBlockPanelKernel.h:1879-2478): it reads op(A)/op(B)
// through ld and the transpose flags and writes K-major zero-padded panels.
#include <cuda.h>
#include <cuda_bf16.h>

#include "device_common.cuh"
#include "kernels.h"
#include "slice_gemm.cuh"
#include "tma_host.h"

namespace eb2 {

namespace {

constexpr int kBRows = 32;
constexpr int kBCols = 64;  // K elements per tile = 128 bytes of one BF16 piece

__global__ void __launch_bounds__(256) bf16_split_kernel(const float* __restrict__ X, int64_t rows, int64_t cols,
                                                         int64_t sr, int64_t sl, __nv_bfloat16* __restrict__ pieces,
                                                         int64_t rows_pad, int64_t k_pad, int* nonfinite) {
  __shared__ float tile[kBRows][kBCols + 1];
  const int64_t r0 = int64_t(blockIdx.y) * kBRows;
  const int64_t l0 = int64_t(blockIdx.x) * kBCols;
  const bool rows_contig = (sr == 1);
  for (int idx = threadIdx.x; idx < kBRows * kBCols; idx += blockDim.x) {
    int rr, ll;
    if (rows_contig) {
      rr = idx % kBRows;
      ll = idx / kBRows;
    } else {
      ll = idx % kBCols;
      rr = idx / kBCols;
    }
    const int64_t r = r0 + rr, l = l0 + ll;
    float v = 0.f;
    if (r < rows && l < cols) v = X[r * sr + l * sl];
    tile[rr][ll] = v;
  }
  __syncthreads();
  const int rr = threadIdx.x >> 3;       // 32 rows
  const int cb = (threadIdx.x & 7) * 8;  // 8 consecutive K elements
  __align__(16) __nv_bfloat16 hv[8], mv[8], lv[8];
  bool bad = false;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float x = tile[rr][cb + j];
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    const float r1 = __fsub_rn(x, __bfloat162float(h));
    const __nv_bfloat16 m = __float2bfloat16_rn(r1);
    const float r2 = __fsub_rn(r1, __bfloat162float(m));
    hv[j] = h;
    mv[j] = m;
    lv[j] = __float2bfloat16_rn(r2);
    bad |= !isfinite(__bfloat162float(h)) || !isfinite(x);
  }
  if (bad) *nonfinite = 1;
  const size_t plane = size_t(rows_pad) * size_t(k_pad);
  const size_t off = size_t(r0 + rr) * size_t(k_pad) + size_t(l0 + cb);
  *reinterpret_cast<uint4*>(pieces + off) = *reinterpret_cast<const uint4*>(hv);
  *reinterpret_cast<uint4*>(pieces + plane + off) = *reinterpret_cast<const uint4*>(mv);
  *reinterpret_cast<uint4*>(pieces + 2 * plane + off) = *reinterpret_cast<const uint4*>(lv);
}

template <int BN, int STAGES, bool PAIR>
cudaError_t launch_config(const Bf16Operand& a, const Bf16Operand& b, const SgemmSplitArgs& args,
                          cudaStream_t stream) {
  constexpr int kRowsPerTile = PAIR ? 2 * kSliceBM : kSliceBM;
  if (a.rows_pad % kRowsPerTile != 0 || b.rows_pad % BN != 0) return cudaErrorInvalidValue;
  CUtensorMap tmA, tmB;
  if (!make_tensor_map_3d(&tmA, a.pieces, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, uint64_t(a.k_pad),
                          uint64_t(a.rows_pad), 3, kSliceKBytes / 2, kSliceBM))
    return cudaErrorInvalidValue;
  if (!make_tensor_map_3d(&tmB, b.pieces, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, uint64_t(b.k_pad),
                          uint64_t(b.rows_pad), 3, kSliceKBytes / 2, PAIR ? BN / 2 : BN))
    return cudaErrorInvalidValue;
  SliceGemmParams P{};
  P.m = args.m;
  P.n = args.n;
  P.num_kb = int(a.k_pad / (kSliceKBytes / 2));
  P.tiles_m = int(a.rows_pad / kRowsPerTile);
  P.tiles_n = int(b.rows_pad / BN);
  P.slices = args.pieces;
  P.diag_lo = 2;
  P.diag_hi = args.pieces + 1;
  P.first_writes = 1;
  P.alpha_f = args.alpha;
  P.beta_f = args.beta;
  P.C = args.C;
  P.ldc = args.ldc;
  P.skip_if_flag = args.skip_if_flag;
  P.status = args.status;
  P.group_m = tuning().group_m > 0 ? tuning().group_m : P.tiles_m;
  P.wait_limit_ns = tuning().wait_limit_ns ? tuning().wait_limit_ns : kWaitLimitNs;
  // 128 accumulator columns per epilogue thread: 4 epilogue warps for 128-wide tiles, 8 for 256
  return launch_slice_gemm<kModeSplitBF16, BN, STAGES, BN / 32, PAIR>(tmA, tmB, P, args.num_sms, stream);
}

}  // namespace

cudaError_t launch_bf16_split(const StridedView<float>& x, const Bf16Operand& op, int* nonfinite,
                              cudaStream_t stream) {
  if (op.k_pad % kBCols != 0 || op.rows_pad % kBRows != 0) return cudaErrorInvalidValue;
  dim3 grid(unsigned(op.k_pad / kBCols), unsigned(op.rows_pad / kBRows));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  bf16_split_kernel<<<grid, 256, 0, stream>>>(x.ptr, x.rows, x.cols, x.sr, x.sl,
                                              reinterpret_cast<__nv_bfloat16*>(op.pieces), op.rows_pad, op.k_pad,
                                              nonfinite);
  return cudaGetLastError();
}

cudaError_t launch_sgemm_split_bf16(const Bf16Operand& a, const Bf16Operand& b, const SgemmSplitArgs& args,
                                    cudaStream_t stream) {
  if (args.pieces < 1 || args.pieces > 3) return cudaErrorInvalidValue;
  if (a.k_pad != b.k_pad || a.k_pad % (kSliceKBytes / 2) != 0) return cudaErrorInvalidValue;
  if (args.tile_n == kTilePair) return launch_config<256, 6, true>(a, b, args, stream);
  if (args.tile_n == 256) return launch_config<256, 4, false>(a, b, args, stream);
  if (args.tile_n == 128) return launch_config<128, 6, false>(a, b, args, stream);
  return cudaErrorInvalidValue;
}

}  // namespace eb2
