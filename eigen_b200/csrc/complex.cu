// complex.cu -- the element-wise kernels of the complex GEMM (zgemm_ / cgemm_).
//
// A complex product is two real products with the inner dimension doubled:
//   Re(op(A) op(B)) = [Ar Ai] [Br; -Bi],   Im(op(A) op(B)) = [Ar Ai] [Bi; Br]
// (Ar, Ai the real and imaginary parts of op(A), likewise for op(B)), i.e. the 4M product
// written as two GEMMs of K = 2k.  Both share the left operand, so these kernels pack
//   op(A) -> A' = [Ar Ai]                 (m x 2k, column-major, ld m)
//   op(B) -> B1 = [Br; -Bi], B2 = [Bi; Br] (2k x n each, column-major, ld 2k)
// from the interleaved (re, im) storage with the transpose or conjugate of op() applied,
// and combine the two real results into C with complex alpha and beta.  All of them are
// memory-bound: one read and one (lhs) or two (rhs) writes of every element, through a
// shared-memory tile when op() transposes so that reads and writes stay coalesced.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace eb2 {
namespace {

constexpr int kTile = 32;  // 32 x 32 element tiles, 32 x 8 threads
constexpr int kPerThread = kTile / 8;

// Element (r, c) of op(X) is X[r*sr + c*sc] (complex elements, interleaved re/im);
// `conj` negates the imaginary part.  kRhs selects the output form (see above).
template <typename T, bool kRhs>
__global__ void pack_complex_kernel(const T* __restrict__ X, int64_t sr, int64_t sc, bool conj, int64_t rows,
                                    int64_t cols, T* __restrict__ Y1, T* __restrict__ Y2, int64_t ldy) {
  __shared__ T re[kTile][kTile + 1], im[kTile][kTile + 1];  // [c][r]
  const int64_t r0 = int64_t(blockIdx.x) * kTile, c0 = int64_t(blockIdx.y) * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const bool row_fast = (sr == 1);  // consecutive rows are adjacent in memory
  for (int q = 0; q < kPerThread; ++q) {
    const int a = tx, b = ty + 8 * q;  // the fast index runs over a
    const int rl = row_fast ? a : b, cl = row_fast ? b : a;
    const int64_t r = r0 + rl, c = c0 + cl;
    if (r < rows && c < cols) {
      const T* p = X + 2 * (r * sr + c * sc);
      re[cl][rl] = p[0];
      im[cl][rl] = conj ? -p[1] : p[1];
    }
  }
  __syncthreads();
  for (int q = 0; q < kPerThread; ++q) {
    const int rl = tx, cl = ty + 8 * q;
    const int64_t r = r0 + rl, c = c0 + cl;
    if (r >= rows || c >= cols) continue;
    const T vr = re[cl][rl], vi = im[cl][rl];
    if (kRhs) {
      Y1[r + c * ldy] = vr;
      Y1[rows + r + c * ldy] = -vi;
      Y2[r + c * ldy] = vi;
      Y2[rows + r + c * ldy] = vr;
    } else {
      Y1[r + c * ldy] = vr;
      Y1[r + (cols + c) * ldy] = vi;
    }
  }
}

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// C (m x n complex, ld ldc) := alpha (Pr + i Pi) + beta C; beta == 0 does not read C;
// Pr == null stands for a zero product (C := beta C).
template <typename T>
__global__ void combine_complex_kernel(const T* __restrict__ Pr, const T* __restrict__ Pi, int64_t ldp, int64_t m,
                                       int64_t n, T ar, T ai, T br, T bi, T* __restrict__ C, int64_t ldc) {
  const int64_t i0 = int64_t(blockIdx.x) * kTile, j0 = int64_t(blockIdx.y) * kTile;
  const bool beta_zero = (br == T(0) && bi == T(0));
  for (int q = 0; q < kPerThread; ++q) {
    const int64_t i = i0 + threadIdx.x, j = j0 + threadIdx.y + 8 * q;
    if (i >= m || j >= n) continue;
    T* c = C + 2 * (i + j * ldc);
    T xr = T(0), xi = T(0);
    if (!beta_zero) {
      const T cr = c[0], ci = c[1];
      xr = fma_rn(br, cr, -bi * ci);
      xi = fma_rn(br, ci, bi * cr);
    }
    if (Pr) {
      const T pr = Pr[i + j * ldp], pi = Pi[i + j * ldp];
      xr = xr + fma_rn(ar, pr, -ai * pi);
      xi = xi + fma_rn(ar, pi, ai * pr);
    }
    c[0] = xr;
    c[1] = xi;
  }
}

dim3 grid_of(int64_t rows, int64_t cols) {
  return dim3(unsigned((rows + kTile - 1) / kTile), unsigned((cols + kTile - 1) / kTile));
}

bool fits(int64_t rows, int64_t cols) {
  return (rows + kTile - 1) / kTile <= 0x7fffffff && (cols + kTile - 1) / kTile <= 65535;
}

}  // namespace

template <typename T>
cudaError_t launch_pack_complex_lhs(const T* X, int64_t sr, int64_t sc, bool conj, int64_t rows, int64_t cols, T* Y,
                                    cudaStream_t st) {
  if (rows == 0 || cols == 0) return cudaSuccess;
  if (!fits(rows, cols)) return cudaErrorInvalidConfiguration;
  pack_complex_kernel<T, false><<<grid_of(rows, cols), dim3(kTile, 8), 0, st>>>(X, sr, sc, conj, rows, cols, Y,
                                                                                nullptr, rows);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_pack_complex_rhs(const T* X, int64_t sr, int64_t sc, bool conj, int64_t rows, int64_t cols, T* Y1,
                                    T* Y2, cudaStream_t st) {
  if (rows == 0 || cols == 0) return cudaSuccess;
  if (!fits(rows, cols)) return cudaErrorInvalidConfiguration;
  pack_complex_kernel<T, true><<<grid_of(rows, cols), dim3(kTile, 8), 0, st>>>(X, sr, sc, conj, rows, cols, Y1, Y2,
                                                                               2 * rows);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_combine_complex(const T* Pr, const T* Pi, int64_t ldp, int64_t m, int64_t n, T ar, T ai, T br,
                                   T bi, T* C, int64_t ldc, cudaStream_t st) {
  if (m == 0 || n == 0) return cudaSuccess;
  if (!fits(m, n)) return cudaErrorInvalidConfiguration;
  combine_complex_kernel<T><<<grid_of(m, n), dim3(kTile, 8), 0, st>>>(Pr, Pi, ldp, m, n, ar, ai, br, bi, C, ldc);
  return cudaGetLastError();
}

#define EB2_COMPLEX_INSTANTIATE(T)                                                                               \
  template cudaError_t launch_pack_complex_lhs<T>(const T*, int64_t, int64_t, bool, int64_t, int64_t, T*,        \
                                                  cudaStream_t);                                                \
  template cudaError_t launch_pack_complex_rhs<T>(const T*, int64_t, int64_t, bool, int64_t, int64_t, T*, T*,    \
                                                  cudaStream_t);                                                \
  template cudaError_t launch_combine_complex<T>(const T*, const T*, int64_t, int64_t, int64_t, T, T, T, T, T*, \
                                                 int64_t, cudaStream_t);
EB2_COMPLEX_INSTANTIATE(double)
EB2_COMPLEX_INSTANTIATE(float)
#undef EB2_COMPLEX_INSTANTIATE

}  // namespace eb2
