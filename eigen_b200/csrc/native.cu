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
constexpr int kDBM = 128, kDBN = 128, kDBK = 16;
constexpr int kDApad = kDBM + 4;  // sA[k][m] row stride (doubles): conflict-free fragment loads
constexpr int kDBpad = kDBK + 4;  // sB[n][k] row stride
constexpr int kDThreads = 256;

struct DSmem {
  double a[2][kDBK][kDApad];
  double b[2][kDBN][kDBpad];
};

__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

template <bool TA, bool TB>
__device__ __forceinline__ void dload_tile(const double* __restrict__ A, int64_t lda, const double* __restrict__ B,
                                           int64_t ldb, int64_t m, int64_t n, int64_t k, int64_t m0, int64_t n0,
                                           int64_t k0, double (&ra)[8], double (&rb)[8]) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int idx = t + kDThreads * i;
    int mm, kk;
    if (!TA) {
      mm = idx % kDBM;
      kk = idx / kDBM;
    } else {
      kk = idx % kDBK;
      mm = idx / kDBK;
    }
    const int64_t gm = m0 + mm, gk = k0 + kk;
    double v = 0.0;
    if (gm < m && gk < k) v = TA ? A[gk + gm * lda] : A[gm + gk * lda];
    ra[i] = v;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int idx = t + kDThreads * i;
    int nn, kk;
    if (!TB) {
      kk = idx % kDBK;
      nn = idx / kDBK;
    } else {
      nn = idx % kDBN;
      kk = idx / kDBN;
    }
    const int64_t gn = n0 + nn, gk = k0 + kk;
    double v = 0.0;
    if (gn < n && gk < k) v = TB ? B[gn + gk * ldb] : B[gk + gn * ldb];
    rb[i] = v;
  }
}

template <bool TA, bool TB>
__device__ __forceinline__ void dstore_tile(DSmem& s, int buf, const double (&ra)[8], const double (&rb)[8]) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int idx = t + kDThreads * i;
    int mm, kk;
    if (!TA) {
      mm = idx % kDBM;
      kk = idx / kDBM;
    } else {
      kk = idx % kDBK;
      mm = idx / kDBK;
    }
    s.a[buf][kk][mm] = ra[i];
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int idx = t + kDThreads * i;
    int nn, kk;
    if (!TB) {
      kk = idx % kDBK;
      nn = idx / kDBK;
    } else {
      nn = idx % kDBN;
      kk = idx / kDBN;
    }
    s.b[buf][nn][kk] = rb[i];
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(kDThreads, 1)
    dgemm_dmma_kernel(int64_t m, int64_t n, int64_t k, double alpha, const double* __restrict__ A, int64_t lda,
                      const double* __restrict__ B, int64_t ldb, double beta, double* __restrict__ C, int64_t ldc,
                      const int* only_if_flag) {
  if (only_if_flag && *only_if_flag == 0) return;
  extern __shared__ __align__(16) uint8_t dsmem_raw[];
  DSmem& s = *reinterpret_cast<DSmem*>(dsmem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp & 1;   // 2 warps along M (64 rows each)
  const int wn = warp >> 1;  // 4 warps along N (32 cols each)
  const int g = lane >> 2, tig = lane & 3;
  const int64_t m0 = int64_t(blockIdx.x) * kDBM, n0 = int64_t(blockIdx.y) * kDBN;

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][j][c] = 0.0;

  double ra[8], rb[8];
  const int64_t nkt = (k + kDBK - 1) / kDBK;
  dload_tile<TA, TB>(A, lda, B, ldb, m, n, k, m0, n0, 0, ra, rb);
  dstore_tile<TA, TB>(s, 0, ra, rb);
  __syncthreads();
  for (int64_t kt = 0; kt < nkt; ++kt) {
    const int buf = int(kt & 1);
    if (kt + 1 < nkt) dload_tile<TA, TB>(A, lda, B, ldb, m, n, k, m0, n0, (kt + 1) * kDBK, ra, rb);
#pragma unroll
    for (int ks = 0; ks < kDBK / 4; ++ks) {
      const int kk = ks * 4 + tig;
      double af[4][2], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        af[i][0] = s.a[buf][kk][wm * 64 + i * 16 + g];
        af[i][1] = s.a[buf][kk][wm * 64 + i * 16 + g + 8];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = s.b[buf][wn * 32 + j * 8 + g][kk];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_16x8x4(acc[i][j], af[i][0], af[i][1], bf[j]);
    }
    if (kt + 1 < nkt) dstore_tile<TA, TB>(s, buf ^ 1, ra, rb);
    __syncthreads();
  }

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
  dim3 grid(unsigned((m + kDBM - 1) / kDBM), unsigned((n + kDBN - 1) / kDBN));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  const int smem = int(sizeof(DSmem));
  auto pick = [&](auto kern) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kDThreads, smem, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, only_if_flag);
    return cudaGetLastError();
  };
  if (!transA && !transB) return pick(dgemm_dmma_kernel<false, false>);
  if (transA && !transB) return pick(dgemm_dmma_kernel<true, false>);
  if (!transA && transB) return pick(dgemm_dmma_kernel<false, true>);
  return pick(dgemm_dmma_kernel<true, true>);
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
