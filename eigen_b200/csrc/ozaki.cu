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
#include "tma_host.h"

namespace eb2 {

namespace {

constexpr uint64_t kInfBits = 0x7FF0000000000000ull;
// One accumulation unit covers at most this many 128-deep digit blocks per output:
// 4095 * 128 * 64 * 64 < 2^31, so the INT32 accumulator cannot overflow.
constexpr int kMaxUnitKb = 4095;

// ------------------------------------------------------------------ scan
constexpr int kScanTile = 64;

__global__ void __launch_bounds__(256) ozaki_scan_kernel(const double* __restrict__ X, int64_t rows, int64_t cols,
                                                         int64_t sr, int64_t sl, unsigned long long* maxbits,
                                                         double* abssum, int* nonfinite) {
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
    if (r < rows) {
      unsigned long long mb = 0;
      for (int ll = 0; ll < kScanTile; ++ll) {
        unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(fabs(tile[t][ll])));
        mb = b > mb ? b : mb;
      }
      if (mb >= kInfBits) *nonfinite = 1;
      if (mb) atomicMax(&maxbits[r], mb);
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

// ------------------------------------------------------------------ GEMM
template <int BN, int STAGES>
struct OzakiSmemLayout {
  static constexpr int kABytes = kOzakiBM * kOzakiKBlock;
  static constexpr int kBBytes = BN * kOzakiKBlock;
  static constexpr int kAOff = 0;
  static constexpr int kBOff = kAOff + STAGES * kABytes;
  static constexpr int kBarOff = kBOff + STAGES * kBBytes;
  // full[STAGES], empty[STAGES], tfull[2], tempty[2], drain
  static constexpr int kNumBars = 2 * STAGES + 5;
  static constexpr int kMiscOff = kBarOff + kNumBars * 8;
  static constexpr int kColExpOff = kMiscOff + 16;
  static constexpr int kTotal = kColExpOff + BN * 4;
  static constexpr int kAlloc = kTotal + 1024;  // slack for 1024-byte alignment
};

struct OzakiKernelParams {
  int64_t m, n;
  int num_kb;
  int tiles_m, tiles_n;
  int slices;
  int diag_lo, diag_hi;
  int first_writes;
  double alpha, beta;
  double* C;
  int64_t ldc;
  const int32_t* expA;
  const int32_t* expB;
  const int* skip_if_flag;
  double* err_sq;
  uint32_t* status;
};

// The schedule every role walks: tiles (persistent, strided by gridDim.x), then
// diagonals t = diag_hi .. diag_lo, each cut into units of at most kMaxUnitKb
// digit blocks; a unit's blocks run pair-major: (p, kb) for p = p_lo..p_hi.
__device__ __forceinline__ bool diag_bounds(int t, int s, int num_kb, int& p_lo, int& total) {
  p_lo = max(1, t - s);
  const int p_hi = min(s, t - 1);
  if (p_lo > p_hi) return false;
  total = (p_hi - p_lo + 1) * num_kb;
  return true;
}

template <int BN, int STAGES>
__global__ void __launch_bounds__(192, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const OzakiKernelParams P) {
  using L = OzakiSmemLayout<BN, STAGES>;
  if (P.skip_if_flag && *P.skip_if_flag) return;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::kBarOff);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* tfull = bars + 2 * STAGES;
  uint64_t* tempty = bars + 2 * STAGES + 2;
  uint64_t* drain = bars + 2 * STAGES + 4;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(smem + L::kMiscOff);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L::kMiscOff + 4);
  int* col_exp = reinterpret_cast<int*>(smem + L::kColExpOff);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < STAGES; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 128);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
  }
  if (warp == 1) {
    tmem_alloc(tmem_holder, 2 * BN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  const int num_tiles = P.tiles_m * P.tiles_n;
  const int s = P.slices;

  if (warp == 0) {
    // ------------------------------------------------ TMA producer
    if (lane == 0) {
      uint32_t issued = 0;  // stage = issued % STAGES, phase = (issued / STAGES) & 1
      bool ok = true;
      for (int tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x) {
        const int m0 = (tile % P.tiles_m) * kOzakiBM;
        const int n0 = (tile / P.tiles_m) * BN;
        for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
          int p_lo, total;
          if (!diag_bounds(t, s, P.num_kb, p_lo, total)) continue;
          for (int f = 0; f < total; ++f) {
            const int p = p_lo + f / P.num_kb;
            const int kb = f % P.num_kb;
            const int q = t - p;
            const int stage = int(issued % STAGES);
            const uint32_t phase = (issued / STAGES) & 1u;
            if (!mbar_wait(&empty[stage], phase ^ 1u, abort_flag, P.status)) {
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&full[stage], L::kABytes + L::kBBytes);
            tma_load_3d(smem + L::kAOff + stage * L::kABytes, &tmA, &full[stage], kb * kOzakiKBlock, m0, p - 1);
            tma_load_3d(smem + L::kBOff + stage * L::kBBytes, &tmB, &full[stage], kb * kOzakiKBlock, n0, q - 1);
            ++issued;
          }
        }
      }
      if (!ok) {
        // let the copies still in flight land before the CTA can exit (bounded)
        volatile int no_abort = 0;
        for (uint32_t i = issued > STAGES ? issued - STAGES : 0; i < issued; ++i)
          (void)mbar_wait(&full[i % STAGES], (i / STAGES) & 1u, &no_abort, P.status);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = make_idesc(2u /*S32*/, 1u /*S8*/, 1u /*S8*/, kOzakiBM, BN);
      int stage = 0;
      uint32_t phase = 0;
      int buf = 0;
      uint32_t tphase = 0u;  // bit b: phase of accumulator buffer b
      bool ok = true;
      for (int tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x) {
        for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
          int p_lo, total;
          if (!diag_bounds(t, s, P.num_kb, p_lo, total)) continue;
          for (int u0 = 0; u0 < total && ok; u0 += kMaxUnitKb) {
            const int u1 = min(total, u0 + kMaxUnitKb);
            if (!mbar_wait(&tempty[buf], ((tphase >> buf) & 1u) ^ 1u, abort_flag, P.status)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t d_tmem = tmem_base + uint32_t(buf * BN);
            for (int f = u0; f < u1; ++f) {
              if (!mbar_wait(&full[stage], phase, abort_flag, P.status)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint64_t adesc = make_sw128_kmajor_desc(smem_u32(smem + L::kAOff + stage * L::kABytes));
              const uint64_t bdesc = make_sw128_kmajor_desc(smem_u32(smem + L::kBOff + stage * L::kBBytes));
#pragma unroll
              for (int kk = 0; kk < kOzakiKBlock / 32; ++kk)
                mma_i8(d_tmem, adesc + uint64_t(2 * kk), bdesc + uint64_t(2 * kk), idesc,
                       (f > u0 || kk > 0) ? 1u : 0u);
              mma_commit(&empty[stage]);
              if (++stage == STAGES) {
                stage = 0;
                phase ^= 1u;
              }
            }
            if (!ok) break;
            mma_commit(&tfull[buf]);
            tphase ^= 1u << buf;
            buf ^= 1;
          }
        }
      }
      // all issued MMAs must finish before TMEM is released
      mma_commit(drain);
      volatile int no_abort = 0;
      (void)mbar_wait(drain, 0, &no_abort, P.status);
    }
  } else {
    // ------------------------------------------------ epilogue (warps 2..5)
    const int quad = warp & 3;  // TMEM lane quadrant this warp may access
    const int row = quad * 32 + lane;
    const int et = threadIdx.x - 64;  // 0..127
    int buf = 0;
    uint32_t ephase = 0u;  // bit b: phase of accumulator buffer b
    double err_hi = 0.0, err_lo = 0.0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x) {
      const int64_t m0 = int64_t(tile % P.tiles_m) * kOzakiBM;
      const int64_t n0 = int64_t(tile / P.tiles_m) * BN;
      for (int j = et; j < BN; j += 128) {
        const int64_t col = n0 + j;
        col_exp[j] = (col < P.n) ? P.expB[col] : 0;
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      const int64_t grow = m0 + row;
      const bool row_ok = grow < P.m;
      const int erow = row_ok ? P.expA[grow] : 0;
      bool first = P.first_writes != 0;
      for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
        int p_lo, total;
        if (!diag_bounds(t, s, P.num_kb, p_lo, total)) continue;
        const int wexp = -12 - 7 * (t - 2);
        // energy of the smallest diagonal (truncation estimate) and of t = 2 (|alpha*A*B| proxy)
        const int est = (P.err_sq == nullptr) ? 0 : (t == P.diag_hi ? 1 : 0) | (t == 2 ? 2 : 0);
        for (int u0 = 0; u0 < total && ok; u0 += kMaxUnitKb) {
          if (!mbar_wait(&tfull[buf], (ephase >> buf) & 1u, abort_flag, P.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t taddr = tmem_base + uint32_t(buf * BN) + (uint32_t(quad * 32) << 16);
#pragma unroll 1
          for (int c = 0; c < BN / 32; ++c) {
            uint32_t r[32];
            tmem_ld_32x32b_x32(taddr + uint32_t(c * 32), r);
            tmem_ld_wait();
            if (row_ok && erow != INT_MIN) {
              double* cp = P.C + grow + (n0 + c * 32) * P.ldc;
#pragma unroll
              for (int jj = 0; jj < 32; ++jj) {
                const int64_t col = n0 + c * 32 + jj;
                const int ce = col_exp[c * 32 + jj];
                if (col < P.n && ce != INT_MIN) {
                  const int E = erow + ce + wexp;
                  const double pw = (E > -1023 && E < 1024) ? __longlong_as_double(static_cast<long long>(E + 1023)
                                                                                   << 52)
                                                            : ldexp(1.0, E);
                  const double val = (static_cast<double>(static_cast<int32_t>(r[jj])) * pw) * P.alpha;
                  double* dst = cp + int64_t(jj) * P.ldc;
                  if (first)
                    *dst = (P.beta == 0.0) ? val : P.beta * *dst + val;
                  else
                    *dst += val;
                  if (est & 1) err_hi += val * val;
                  if (est & 2) err_lo += val * val;
                }
              }
            }
          }
          tc_fence_before();
          mbar_arrive(&tempty[buf]);
          ephase ^= 1u << buf;
          buf ^= 1;
          first = false;
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
    }
    if (P.err_sq) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        err_hi += __shfl_xor_sync(0xffffffffu, err_hi, o);
        err_lo += __shfl_xor_sync(0xffffffffu, err_lo, o);
      }
      if (lane == 0 && err_hi != 0.0) atomicAdd(&P.err_sq[0], err_hi);
      if (lane == 0 && err_lo != 0.0) atomicAdd(&P.err_sq[1], err_lo);
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, 2 * BN);
}

template <int BN, int STAGES>
cudaError_t launch_gemm_tiles(const OzakiOperand& a, const OzakiOperand& b, const OzakiGemmArgs& args,
                              cudaStream_t stream) {
  using L = OzakiSmemLayout<BN, STAGES>;
  CUtensorMap tmA, tmB;
  if (!make_tensor_map_3d(&tmA, a.digits, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, uint64_t(a.k_pad), uint64_t(a.rows_pad),
                          uint64_t(a.smax), kOzakiKBlock, kOzakiBM))
    return cudaErrorInvalidValue;
  if (!make_tensor_map_3d(&tmB, b.digits, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, uint64_t(b.k_pad), uint64_t(b.rows_pad),
                          uint64_t(b.smax), kOzakiKBlock, BN))
    return cudaErrorInvalidValue;
  OzakiKernelParams P;
  P.m = args.m;
  P.n = args.n;
  P.num_kb = int(a.k_pad / kOzakiKBlock);
  P.tiles_m = int(a.rows_pad / kOzakiBM);
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
  auto kern = ozaki_gemm_kernel<BN, STAGES>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kAlloc);
  if (e != cudaSuccess) return e;
  const int tiles = P.tiles_m * P.tiles_n;
  const int grid = tiles < args.num_sms ? tiles : args.num_sms;
  kern<<<grid, 192, L::kAlloc, stream>>>(tmA, tmB, P);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_ozaki_scan_reset(const OzakiOperand& op, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(op.maxbits, 0, size_t(op.rows) * sizeof(uint64_t), stream);
  if (e != cudaSuccess || op.abssum == nullptr) return e;
  return cudaMemsetAsync(op.abssum, 0, size_t(op.k) * sizeof(double), stream);
}

cudaError_t launch_ozaki_scan(const StridedView<double>& x, const OzakiOperand& op, int* nonfinite,
                              cudaStream_t stream) {
  if (x.rows == 0 || x.cols == 0) return cudaSuccess;
  dim3 grid(unsigned((x.cols + kScanTile - 1) / kScanTile), unsigned((x.rows + kScanTile - 1) / kScanTile));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  ozaki_scan_kernel<<<grid, 256, 0, stream>>>(x.ptr, x.rows, x.cols, x.sr, x.sl,
                                              reinterpret_cast<unsigned long long*>(op.maxbits), op.abssum,
                                              nonfinite);
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
  if (a.k_pad != b.k_pad || a.k_pad % kOzakiKBlock != 0 || a.rows_pad % kOzakiBM != 0)
    return cudaErrorInvalidValue;
  if (args.tile_n == 256) {
    if (b.rows_pad % 256 != 0) return cudaErrorInvalidValue;
    return launch_gemm_tiles<256, 4>(a, b, args, stream);
  }
  if (args.tile_n == 128) {
    if (b.rows_pad % 128 != 0) return cudaErrorInvalidValue;
    return launch_gemm_tiles<128, 6>(a, b, args, stream);
  }
  return cudaErrorInvalidValue;
}

}  // namespace eb2
