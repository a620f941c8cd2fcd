// native.cu -- plain-precision GEMM kernels: FP64 on the DMMA tensor-core path
// (mma.sync f64) and FP32 on the FFMA pipes.  They compute
//     C = alpha * op(A) * op(B) + beta * C        (column-major, any ld)
// exactly as Eigen's GEBP store does it (R = alpha*acc + R after the BLAS shim's
// beta pre-scale, Eigen/src/Core/products/GeneralBlockPanelKernel.h:1446-1455,
// blas/level3_impl.h:80-87), with beta == 0 never reading C.  The FP64 kernel is
// the on-device correctness reference for the emulated DGEMM and its fallback for
// inputs with NaN/Inf.
//
// The tile loaders play the role of gemm_pack_lhs/gemm_pack_rhs
// (GeneralBlockPanelKernel.h:1879-2478): they read op(A)/op(B) through lda/ldb and
// the transpose flags and write one fixed shared-memory layout, so the inner
// product loop is the same for NN/NT/TN/TT.
#include "device_common.cuh"
#include "kernels.h"

namespace eb2 {

namespace {

// ------------------------------------------------------------------ FP64 DMMA
// 128 x 128 tiles, K in tiles of 16 through a 4-stage shared-memory ring, warp-specialised:
// four producer warps copy the tiles with 8-byte cp.async (any alignment and leading
// dimension; edges zero-filled) and hands each stage over with cp.async.mbarrier.arrive on
// its `full` barrier; eight consumer warps (64 x 32 outputs each) wait on `full`, run DMMA
// m16n8k4 with K in steps of 4 from 0 upward for every output, and release the stage on its
// `empty` barrier.  No block-wide barrier in the main loop: measured, the copy issue and the
// per-tile __syncthreads of a cooperative ring cost a fifth of the DMMA rate.  Shared memory
// follows each operand's contiguous direction in global memory ([k][m] when op(A) is stored
// column-major, [m][k] when transposed; likewise for op(B)), padded so that the 64-bit
// fragment loads of each half-warp hit distinct banks.  Every wait is bounded (kWaitLimitNs);
// one that runs out records EB2_DEV_ERR_TIMEOUT in *status and the roles leave.
constexpr int kDBM = 128, kDBN = 128, kDBK = 16;
constexpr int kDStages = 4;
constexpr int kDPadMN = kDBM + 4;  // [k][m or n] row stride (doubles)
constexpr int kDPadK = kDBK + 4;   // [m or n][k] row stride
constexpr int kDConsumerWarps = 8;
constexpr int kDProducerWarps = 4;
constexpr int kDThreads = 32 * (kDConsumerWarps + kDProducerWarps);
constexpr int kDTileElems = (kDBK * kDPadMN > kDBM * kDPadK) ? kDBK * kDPadMN : kDBM * kDPadK;

struct DSmem {
  double a[kDStages][kDTileElems];
  double b[kDStages][kDTileElems];
  uint64_t full[kDStages], empty[kDStages];
  int abort_flag;
};

// where a native-kernel wait that ran out is recorded when the caller passes no status word
__device__ uint32_t g_native_status;

__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// The producer warps' copies of one K tile of one operand (rows x k view at X, leading
// dimension ld).  MN_CONTIG: the operand's m (or n) index is the contiguous one in global
// memory (op(A) = A column-major, op(B) = B^T of a column-major B).  V = 2: 16-byte copies of
// two neighbours along the contiguous index (X 16-byte aligned, ld even); a pair that
// straddles the edge copies its first element and zero-fills the second.
template <bool MN_CONTIG, int V>
__device__ __forceinline__ void dcopy_operand(double* st, const double* __restrict__ X, int64_t ld, int64_t rows,
                                              int64_t k, int64_t r0, int64_t k0, int pt) {
  constexpr int kPT = 32 * kDProducerWarps;
  constexpr int kRowsV = MN_CONTIG ? kDBM / V : kDBM, kColsV = MN_CONTIG ? kDBK : kDBK / V;
  constexpr int kCopies = kRowsV * kColsV / kPT;
  // thread pt copies a fixed contiguous-direction offset and steps through the other index
  // (kStep columns of K, or kStep rows) from copy to copy
  constexpr int kStep = MN_CONTIG ? kPT / kRowsV : kPT / kColsV;
  static_assert(kPT % (MN_CONTIG ? kRowsV : kColsV) == 0, "fixed contiguous offset per thread");
  const int c_off = (pt % (MN_CONTIG ? kRowsV : kColsV)) * V;  // along the contiguous index
  const int s_first = pt / (MN_CONTIG ? kRowsV : kColsV);      // first value of the stepped index
  const int64_t g_c = (MN_CONTIG ? r0 : k0) + c_off, g_s = (MN_CONTIG ? k0 : r0) + s_first;
  const int64_t lim_c = MN_CONTIG ? rows : k, lim_s = MN_CONTIG ? k : rows;
  // elements of the contiguous pair inside the matrix (0, 1 or V); the same for every copy
  const int in_c = g_c + V <= lim_c ? V : (g_c < lim_c ? int(lim_c - g_c) : 0);
  const double* src = X + g_c + g_s * ld;
  const int64_t src_step = int64_t(kStep) * ld;
  uint32_t dst = smem_u32(MN_CONTIG ? st + s_first * kDPadMN + c_off : st + s_first * kDPadK + c_off);
  constexpr uint32_t kDstStep = uint32_t(kStep * (MN_CONTIG ? kDPadMN : kDPadK) * 8);
#pragma unroll
  for (int i = 0; i < kCopies; ++i, src += src_step, dst += kDstStep) {
    const int in = (g_s + int64_t(i) * kStep < lim_s) ? in_c : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(in ? src : X), "n"(8 * V),
                 "r"(8 * in)
                 : "memory");
  }
}

// Tile t of the grid in groups of kDGroupM tile rows (column-major inside a group), so that
// the CTAs in flight share A panels in L2 as well as B panels.
constexpr int kDGroupM = 8;
__device__ __forceinline__ void dtile_coords(int64_t t, int64_t tiles_m, int64_t tiles_n, int64_t& tm, int64_t& tn) {
  const int64_t per_group = int64_t(kDGroupM) * tiles_n;
  const int64_t first_m = (t / per_group) * kDGroupM;
  const int64_t gm = tiles_m - first_m < kDGroupM ? tiles_m - first_m : kDGroupM;
  const int64_t r = t % per_group;
  tm = first_m + r % gm;
  tn = r / gm;
}

template <bool TA, bool TB, int VA, int VB>
__global__ void __launch_bounds__(kDThreads, 1)
    dgemm_dmma_kernel(int64_t m, int64_t n, int64_t k, double alpha, const double* __restrict__ A, int64_t lda,
                      const double* __restrict__ B, int64_t ldb, double beta, double* __restrict__ C, int64_t ldc,
                      const int* only_if_flag, uint32_t* status) {
  if (only_if_flag && *only_if_flag == 0) return;
  extern __shared__ __align__(16) uint8_t dsmem_raw[];
  DSmem& s = *reinterpret_cast<DSmem*>(dsmem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t tm, tn;
  dtile_coords(blockIdx.x, (m + kDBM - 1) / kDBM, (n + kDBN - 1) / kDBN, tm, tn);
  const int64_t m0 = tm * kDBM, n0 = tn * kDBN;
  // op(A) m-contiguous unless transposed; op(B)'s n index is contiguous only when transposed
  constexpr bool kAmn = !TA, kBmn = TB;
  uint32_t* const st_word = status ? status : &g_native_status;
  volatile int* const abort_flag = &s.abort_flag;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kDStages; ++i) {
      mbar_init(&s.full[i], 32 * kDProducerWarps);  // one cp.async arrival per producer thread
      mbar_init(&s.empty[i], kDConsumerWarps);  // one arrival per consumer warp
    }
    s.abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t nkt = (k + kDBK - 1) / kDBK;

  if (warp >= kDConsumerWarps) {
    // producers: tile kt into stage kt % kDStages once the consumers released its previous use
    const int pt = int(threadIdx.x) - 32 * kDConsumerWarps;
    for (int64_t kt = 0; kt < nkt; ++kt) {
      const int stg = int(kt % kDStages);
      const int64_t use = kt / kDStages;
      if (use > 0 && !mbar_wait(&s.empty[stg], uint32_t((use - 1) & 1), abort_flag, st_word)) break;
      dcopy_operand<kAmn, VA>(s.a[stg], A, lda, m, k, m0, kt * kDBK, pt);
      dcopy_operand<kBmn, VB>(s.b[stg], B, ldb, n, k, n0, kt * kDBK, pt);
      cp_async_mbar_arrive(&s.full[stg]);
    }
    cp_async_wait_all();  // no copy outlives the block
    return;
  }

  const int wm = warp & 1;   // 2 warps along M (64 rows each)
  const int wn = warp >> 1;  // 4 warps along N (32 cols each)
  const int g = lane >> 2, tig = lane & 3;
  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][j][c] = 0.0;

  bool ok = true;
  for (int64_t kt = 0; kt < nkt && ok; ++kt) {
    const int stg = int(kt % kDStages);
    if (!mbar_wait(&s.full[stg], uint32_t((kt / kDStages) & 1), abort_flag, st_word)) {
      ok = false;
      break;
    }
    const double* sa = s.a[stg];
    const double* sb = s.b[stg];
#pragma unroll
    for (int ks = 0; ks < kDBK / 4; ++ks) {
      const int kk = ks * 4 + tig;
      double af[4][2], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = wm * 64 + i * 16 + g;
        af[i][0] = kAmn ? sa[kk * kDPadMN + r] : sa[r * kDPadK + kk];
        af[i][1] = kAmn ? sa[kk * kDPadMN + r + 8] : sa[(r + 8) * kDPadK + kk];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn * 32 + j * 8 + g;
        bf[j] = kBmn ? sb[kk * kDPadMN + c] : sb[c * kDPadK + kk];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_16x8x4(acc[i][j], af[i][0], af[i][1], bf[j]);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&s.empty[stg]);
  }
  if (!ok) return;  // C is left as it was; the status word records the timeout

  // epilogue: C = alpha*acc + beta*C
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t row = m0 + wm * 64 + i * 16 + g + h * 8;
        if (row >= m) continue;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int64_t col = n0 + wn * 32 + j * 8 + tig * 2 + c;
          if (col >= n) continue;
          double* dst = C + row + col * ldc;
          const double v = __dmul_rn(alpha, acc[i][j][h * 2 + c]);
          *dst = (beta == 0.0) ? v : __fma_rn(beta, *dst, v);
        }
      }
}

// ------------------------------------------------------------------ FP32 FFMA
constexpr int kSBM = 128, kSBN = 128, kSBK = 8, kSThreads = 256;

template <bool TA, bool TB>
__global__ void __launch_bounds__(kSThreads)
    sgemm_ffma_kernel(int64_t m, int64_t n, int64_t k, float alpha, const float* __restrict__ A, int64_t lda,
                      const float* __restrict__ B, int64_t ldb, float beta, float* __restrict__ C, int64_t ldc,
                      const int* only_if_flag) {
  if (only_if_flag && *only_if_flag == 0) return;
  __shared__ float sa[2][kSBK][kSBM + 4];
  __shared__ float sb[2][kSBK][kSBN + 4];
  const int t = threadIdx.x;
  const int tx = t % 16, ty = t / 16;  // 16 x 16 threads, 8 x 8 outputs each
  const int64_t m0 = int64_t(blockIdx.x) * kSBM, n0 = int64_t(blockIdx.y) * kSBN;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  float ra[4], rb[4];
  auto load = [&](int64_t k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = t + kSThreads * i;
      int mm, kk;
      if (!TA) {
        mm = idx % kSBM;
        kk = idx / kSBM;
      } else {
        kk = idx % kSBK;
        mm = idx / kSBK;
      }
      const int64_t gm = m0 + mm, gk = k0 + kk;
      ra[i] = (gm < m && gk < k) ? (TA ? A[gk + gm * lda] : A[gm + gk * lda]) : 0.f;
      int nn;
      if (!TB) {
        kk = idx % kSBK;
        nn = idx / kSBK;
      } else {
        nn = idx % kSBN;
        kk = idx / kSBN;
      }
      const int64_t gn = n0 + nn, gk2 = k0 + kk;
      rb[i] = (gn < n && gk2 < k) ? (TB ? B[gn + gk2 * ldb] : B[gk2 + gn * ldb]) : 0.f;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = t + kSThreads * i;
      int mm, kk;
      if (!TA) {
        mm = idx % kSBM;
        kk = idx / kSBM;
      } else {
        kk = idx % kSBK;
        mm = idx / kSBK;
      }
      sa[buf][kk][mm] = ra[i];
      int nn;
      if (!TB) {
        kk = idx % kSBK;
        nn = idx / kSBK;
      } else {
        nn = idx % kSBN;
        kk = idx / kSBN;
      }
      sb[buf][kk][nn] = rb[i];
    }
  };
  const int64_t nkt = (k + kSBK - 1) / kSBK;
  load(0);
  store(0);
  __syncthreads();
  for (int64_t kt = 0; kt < nkt; ++kt) {
    const int buf = int(kt & 1);
    if (kt + 1 < nkt) load((kt + 1) * kSBK);
#pragma unroll
    for (int kk = 0; kk < kSBK; ++kk) {
      float av[8], bv[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        av[i] = sa[buf][kk][ty * 4 + i];
        av[i + 4] = sa[buf][kk][64 + ty * 4 + i];
        bv[i] = sb[buf][kk][tx * 4 + i];
        bv[i + 4] = sb[buf][kk][64 + tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (kt + 1 < nkt) store(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t row = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
    if (row >= m) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int64_t col = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
      if (col >= n) continue;
      float* dst = C + row + col * ldc;
      const float v = __fmul_rn(alpha, acc[i][j]);
      *dst = (beta == 0.f) ? v : __fmaf_rn(beta, *dst, v);
    }
  }
}

template <typename T>
__global__ void scale_matrix_kernel(int64_t m, int64_t n, T beta, T* C, int64_t ldc) {
  const int64_t total = m * n;
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx % m, j = idx / m;
    T* p = C + i + j * ldc;
    *p = (beta == T(0)) ? T(0) : T(beta * *p);
  }
}

}  // namespace

cudaError_t launch_dgemm_native(bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                                const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                                int64_t ldc, const int* only_if_flag, cudaStream_t stream) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  const int64_t tiles = ((m + kDBM - 1) / kDBM) * ((n + kDBN - 1) / kDBN);
  if (tiles > 0x7FFFFFFF) return cudaErrorInvalidConfiguration;
  const int smem = int(sizeof(DSmem));
  auto pick = [&](auto kern) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    kern<<<unsigned(tiles), kDThreads, smem, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, only_if_flag,
                                                        nullptr);
    return cudaGetLastError();
  };
  // 16-byte copies where the operand allows them
  const bool va = reinterpret_cast<uintptr_t>(A) % 16 == 0 && lda % 2 == 0;
  const bool vb = reinterpret_cast<uintptr_t>(B) % 16 == 0 && ldb % 2 == 0;
  auto by_vec = [&](auto k11, auto k12, auto k21, auto k22) -> cudaError_t {
    if (va) return vb ? pick(k22) : pick(k21);
    return vb ? pick(k12) : pick(k11);
  };
#define EB2_DMMA_VARIANTS(TA_, TB_)                                                                       \
  by_vec(dgemm_dmma_kernel<TA_, TB_, 1, 1>, dgemm_dmma_kernel<TA_, TB_, 1, 2>, dgemm_dmma_kernel<TA_, TB_, 2, 1>, \
         dgemm_dmma_kernel<TA_, TB_, 2, 2>)
  if (!transA && !transB) return EB2_DMMA_VARIANTS(false, false);
  if (transA && !transB) return EB2_DMMA_VARIANTS(true, false);
  if (!transA && transB) return EB2_DMMA_VARIANTS(false, true);
  return EB2_DMMA_VARIANTS(true, true);
#undef EB2_DMMA_VARIANTS
}

cudaError_t launch_sgemm_native(bool transA, bool transB, int64_t m, int64_t n, int64_t k, float alpha,
                                const float* A, int64_t lda, const float* B, int64_t ldb, float beta, float* C,
                                int64_t ldc, const int* only_if_flag, cudaStream_t stream) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  dim3 grid(unsigned((m + kSBM - 1) / kSBM), unsigned((n + kSBN - 1) / kSBN));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  if (!transA && !transB)
    sgemm_ffma_kernel<false, false><<<grid, kSThreads, 0, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                     only_if_flag);
  else if (transA && !transB)
    sgemm_ffma_kernel<true, false><<<grid, kSThreads, 0, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                    only_if_flag);
  else if (!transA && transB)
    sgemm_ffma_kernel<false, true><<<grid, kSThreads, 0, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                    only_if_flag);
  else
    sgemm_ffma_kernel<true, true><<<grid, kSThreads, 0, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                   only_if_flag);
  return cudaGetLastError();
}

cudaError_t launch_scale_matrix_d(int64_t m, int64_t n, double beta, double* C, int64_t ldc, cudaStream_t stream) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  const int64_t total = m * n;
  const int blocks = int(total / 256 + 1 < 148 * 16 ? total / 256 + 1 : 148 * 16);
  scale_matrix_kernel<double><<<blocks, 256, 0, stream>>>(m, n, beta, C, ldc);
  return cudaGetLastError();
}

cudaError_t launch_scale_matrix_s(int64_t m, int64_t n, float beta, float* C, int64_t ldc, cudaStream_t stream) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  const int64_t total = m * n;
  const int blocks = int(total / 256 + 1 < 148 * 16 ? total / 256 + 1 : 148 * 16);
  scale_matrix_kernel<float><<<blocks, 256, 0, stream>>>(m, n, beta, C, ldc);
  return cudaGetLastError();
}

}  // namespace eb2
