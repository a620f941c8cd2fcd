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

// out (n x n complex, ld ldo) from the triangle `upper` of the complex A (ld lda), both
// interleaved:
//   kSymmetric : out(i,j) = A(j,i) outside the triangle (zsymm);
//   kHermitian : out(i,j) = conj(A(j,i)) outside, and the diagonal's real part only (zhemm:
//                Eigen's self-adjoint packing takes real(A(k,k)),
//                Eigen/src/Core/products/SelfadjointMatrixMatrix.h:54);
//   kTriangular: 0 outside, 1 on the diagonal when `unit` (ztrmm).
// The stored triangle is the only part of A that is read; mirrored reads go through a
// shared-memory tile so that reads and writes stay coalesced.
enum ExpandMode : int { kSymmetric = 0, kHermitian = 1, kTriangular = 2 };

template <typename T>
__global__ void expand_complex_kernel(const T* __restrict__ A, int64_t lda, int64_t n, bool upper, int mode,
                                      bool unit, T* __restrict__ out, int64_t ldo) {
  __shared__ T mre[kTile][kTile + 1], mim[kTile][kTile + 1];
  const int64_t bi = int64_t(blockIdx.x) * kTile, bj = int64_t(blockIdx.y) * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  auto inside = [upper](int64_t i, int64_t j) { return upper ? i <= j : i >= j; };
  const bool any_outside = upper ? (bi + kTile - 1 > bj) : (bi < bj + kTile - 1);
  if (mode != kTriangular && any_outside) {
    for (int q = 0; q < kPerThread; ++q) {
      const int jj = ty + 8 * q;
      const int64_t r = bj + tx, c = bi + jj;  // A(r, c) mirrors out(c, r)
      if (r < n && c < n && inside(r, c)) {
        const T* a = A + 2 * (r + c * lda);
        mre[jj][tx] = a[0];
        mim[jj][tx] = a[1];
      }
    }
  }
  __syncthreads();
  for (int q = 0; q < kPerThread; ++q) {
    const int jj = ty + 8 * q;
    const int64_t i = bi + tx, j = bj + jj;
    if (i >= n || j >= n) continue;
    T re, im;
    if (i == j && mode == kTriangular && unit) {
      re = T(1);
      im = T(0);
    } else if (inside(i, j)) {
      const T* a = A + 2 * (i + j * lda);
      re = a[0];
      im = (i == j && mode == kHermitian) ? T(0) : a[1];
    } else if (mode == kTriangular) {
      re = T(0);
      im = T(0);
    } else {
      re = mre[tx][jj];
      im = mode == kHermitian ? -mim[tx][jj] : mim[tx][jj];
    }
    T* o = out + 2 * (i + j * ldo);
    o[0] = re;
    o[1] = im;
  }
}

// x := E^-1 x for `count` complex vectors against the complex triangular block E (nb x nb,
// nb <= kPanelMaxComplex, element (r, c) at complex index r*er + c*ec, conjugated when
// `conj`; the triangle `lower` or upper, unit diagonal when `unit`); element r of vector t at
// complex index r*vs + t*ts.  The complex counterpart of the real panel solve in tri.cu:
// vectors resident in shared memory, 16-row sub-blocks solved column by column by two warps
// with the reciprocal diagonal (Eigen/src/Core/products/TriangularSolverMatrix.h:61-82), the
// rows below updated by all threads (2 rows x 4 vectors each) from staged coefficients.
// An upper triangle is solved as the lower one of the index-reversed system.
constexpr int kCPanelSub = 16;
constexpr int kCPanelThreads = 256;
constexpr int kCPanelChunk = 32;            // coefficient rows staged per pass
constexpr int kCPanelXld = kPanelVecs + 1;  // row stride of the resident vectors (complex)

template <typename T>
__device__ __forceinline__ void cfma(T ar, T ai, T br, T bi, T& cr, T& ci) {  // c += a b
  cr = fma_rn(ar, br, fma_rn(-ai, bi, cr));
  ci = fma_rn(ar, bi, fma_rn(ai, br, ci));
}

template <typename T>
__global__ void __launch_bounds__(kCPanelThreads) tri_panel_solve_complex_kernel(
    const T* __restrict__ E, int64_t er, int64_t ec, int nb, bool lower, bool unit, bool conj, T* __restrict__ X,
    int64_t vs, int64_t ts, int64_t count) {
  static_assert(kPanelVecs == 64 && kCPanelThreads == 256 && kCPanelChunk == 32, "thread tiling");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Xr = reinterpret_cast<T*>(smem_raw);        // [nb][kCPanelXld] real parts
  T* Xi = Xr + nb * kCPanelXld;                  // imaginary parts
  T* Dr = Xi + nb * kCPanelXld;                  // [32][33] diagonal sub-block
  T* Di = Dr + kCPanelSub * (kCPanelSub + 1);
  T* Ir = Di + kCPanelSub * (kCPanelSub + 1);    // [32] reciprocal diagonal
  T* Ii = Ir + kCPanelSub;
  T* Cr = Ii + kCPanelSub;                       // [32][chunk] coefficients, Cr[c * chunk + row]
  T* Ci = Cr + kCPanelSub * kCPanelChunk;
  constexpr int kDld = kCPanelSub + 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tx = tid & 15, ty = tid >> 4;        // update tiling: vectors 4tx.., rows 2ty..
  const int64_t t0 = int64_t(blockIdx.x) * kPanelVecs;
  const int nv = int(count - t0 < kPanelVecs ? count - t0 : kPanelVecs);
  auto ro = [&](int r) -> int64_t { return lower ? r : nb - 1 - r; };
  auto load_e = [&](int r, int c, T& re, T& im) {
    const T* e = E + 2 * (ro(r) * er + ro(c) * ec);
    re = e[0];
    im = conj ? -e[1] : e[1];
  };
  const bool vec_fast = (ts == 1);
  for (int idx = tid; idx < nb * kPanelVecs; idx += kCPanelThreads) {
    const int t = vec_fast ? idx % kPanelVecs : idx / nb;
    const int r = vec_fast ? idx / kPanelVecs : idx % nb;
    T re = T(0), im = T(0);
    if (t < nv) {
      const T* x = X + 2 * (ro(r) * vs + (t0 + t) * ts);
      re = x[0];
      im = x[1];
    }
    Xr[r * kCPanelXld + t] = re;
    Xi[r * kCPanelXld + t] = im;
  }
  for (int jb = 0; jb < nb; jb += kCPanelSub) {
    const int bs = nb - jb < kCPanelSub ? nb - jb : kCPanelSub;
    __syncthreads();
    for (int idx = tid; idx < bs * bs; idx += kCPanelThreads) {
      const int r = idx / bs, c = idx % bs;
      T re = T(0), im = T(0);
      if (r == c && unit)
        re = T(1);
      else if (r >= c)
        load_e(jb + r, jb + c, re, im);
      Dr[r * kDld + c] = re;
      Di[r * kDld + c] = im;
      if (r == c) {  // 1 / (re + i im), scaled by the larger component (Smith's method)
        if (unit) {
          Ir[r] = T(1);
          Ii[r] = T(0);
        } else if (fabs(re) >= fabs(im)) {
          const T q = im / re, d = re + im * q;
          Ir[r] = T(1) / d;
          Ii[r] = -q / d;
        } else {
          const T q = re / im, d = re * q + im;
          Ir[r] = q / d;
          Ii[r] = T(-1) / d;
        }
      }
    }
    __syncthreads();
    if (warp < 2) {
      const int t = warp * 32 + lane;
      T sr[kCPanelSub], si[kCPanelSub];
#pragma unroll
      for (int r = 0; r < kCPanelSub; ++r) {
        sr[r] = r < bs ? Xr[(jb + r) * kCPanelXld + t] : T(0);
        si[r] = r < bs ? Xi[(jb + r) * kCPanelXld + t] : T(0);
      }
#pragma unroll
      for (int c = 0; c < kCPanelSub; ++c) {
        const int cc = c < bs ? c : 0;
        const T xr = sr[c] * Ir[cc] - si[c] * Ii[cc], xi = sr[c] * Ii[cc] + si[c] * Ir[cc];
        sr[c] = xr;
        si[c] = xi;
#pragma unroll
        for (int r = c + 1; r < kCPanelSub; ++r) cfma(-Dr[r * kDld + c], -Di[r * kDld + c], xr, xi, sr[r], si[r]);
      }
#pragma unroll
      for (int r = 0; r < kCPanelSub; ++r)
        if (r < bs) {
          Xr[(jb + r) * kCPanelXld + t] = sr[r];
          Xi[(jb + r) * kCPanelXld + t] = si[r];
        }
    }
    for (int r0 = jb + bs; r0 < nb; r0 += kCPanelChunk) {
      const int rows = nb - r0 < kCPanelChunk ? nb - r0 : kCPanelChunk;
      __syncthreads();
      for (int idx = tid; idx < kCPanelSub * kCPanelChunk; idx += kCPanelThreads) {
        const int rr = idx % kCPanelChunk, c = idx / kCPanelChunk;
        T re = T(0), im = T(0);
        if (rr < rows && c < bs) load_e(r0 + rr, jb + c, re, im);
        Cr[c * kCPanelChunk + rr] = re;
        Ci[c * kCPanelChunk + rr] = im;
      }
      __syncthreads();
      T ar[2][4], ai[2][4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) ar[i][j] = ai[i][j] = T(0);
#pragma unroll 4
      for (int c = 0; c < kCPanelSub; ++c) {
        if (c >= bs) break;
        T er_[2], ei_[2], xr[4], xi[4];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          er_[i] = Cr[c * kCPanelChunk + 2 * ty + i];
          ei_[i] = Ci[c * kCPanelChunk + 2 * ty + i];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          xr[j] = Xr[(jb + c) * kCPanelXld + 4 * tx + j];
          xi[j] = Xi[(jb + c) * kCPanelXld + 4 * tx + j];
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) cfma(er_[i], ei_[i], xr[j], xi[j], ar[i][j], ai[i][j]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int rr = 2 * ty + i;
        if (rr < rows) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            Xr[(r0 + rr) * kCPanelXld + 4 * tx + j] -= ar[i][j];
            Xi[(r0 + rr) * kCPanelXld + 4 * tx + j] -= ai[i][j];
          }
        }
      }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nb * kPanelVecs; idx += kCPanelThreads) {
    const int t = vec_fast ? idx % kPanelVecs : idx / nb;
    const int r = vec_fast ? idx / kPanelVecs : idx % nb;
    if (t < nv) {
      T* x = X + 2 * (ro(r) * vs + (t0 + t) * ts);
      x[0] = Xr[r * kCPanelXld + t];
      x[1] = Xi[r * kCPanelXld + t];
    }
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

size_t tri_panel_complex_smem(int nb, size_t elem) {
  return (2 * size_t(nb) * kCPanelXld + 2 * size_t(kCPanelSub) * (kCPanelSub + 1) + 2 * kCPanelSub +
          2 * size_t(kCPanelSub) * kCPanelChunk) *
         elem;
}

template <typename T>
cudaError_t launch_expand_complex(const T* A, int64_t lda, int64_t n, bool upper, int mode, bool unit, T* out,
                                  int64_t ldo, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  if (!fits(n, n) || mode < 0 || mode > 2) return cudaErrorInvalidConfiguration;
  expand_complex_kernel<T><<<grid_of(n, n), dim3(kTile, 8), 0, st>>>(A, lda, n, upper, mode, unit, out, ldo);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_tri_panel_solve_complex(const T* E, int64_t er, int64_t ec, int nb, bool lower, bool unit,
                                           bool conj, T* X, int64_t vs, int64_t ts, int64_t count, cudaStream_t st) {
  if (count == 0 || nb == 0) return cudaSuccess;
  if (nb < 0 || nb > kPanelMaxComplex || count < 0) return cudaErrorInvalidValue;
  const int64_t blocks = (count + kPanelVecs - 1) / kPanelVecs;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  auto kern = tri_panel_solve_complex_kernel<T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(tri_panel_complex_smem(kPanelMaxComplex, 8)));
  if (e != cudaSuccess) return e;
  kern<<<unsigned(blocks), kCPanelThreads, tri_panel_complex_smem(nb, sizeof(T)), st>>>(E, er, ec, nb, lower, unit,
                                                                                       conj, X, vs, ts, count);
  return cudaGetLastError();
}

#define EB2_COMPLEX_INSTANTIATE(T)                                                                               \
  template cudaError_t launch_pack_complex_lhs<T>(const T*, int64_t, int64_t, bool, int64_t, int64_t, T*,        \
                                                  cudaStream_t);                                                \
  template cudaError_t launch_pack_complex_rhs<T>(const T*, int64_t, int64_t, bool, int64_t, int64_t, T*, T*,    \
                                                  cudaStream_t);                                                \
  template cudaError_t launch_combine_complex<T>(const T*, const T*, int64_t, int64_t, int64_t, T, T, T, T, T*, \
                                                 int64_t, cudaStream_t);                                         \
  template cudaError_t launch_expand_complex<T>(const T*, int64_t, int64_t, bool, int, bool, T*, int64_t,       \
                                                cudaStream_t);                                                  \
  template cudaError_t launch_tri_panel_solve_complex<T>(const T*, int64_t, int64_t, int, bool, bool, bool, T*, \
                                                         int64_t, int64_t, int64_t, cudaStream_t);
EB2_COMPLEX_INSTANTIATE(double)
EB2_COMPLEX_INSTANTIATE(float)
#undef EB2_COMPLEX_INSTANTIATE

}  // namespace eb2
