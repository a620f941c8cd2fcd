// tri.cu -- the element-wise kernels the symmetric and triangular level-3 routines need
// around the GEMM: expanding a stored symmetric or triangular matrix into a full one, merging a
// product into one triangle of C, scaling a triangle or a matrix, and applying a small
// triangular diagonal block (multiply or solve) to a panel in place.
//
// Eigen's routines (blas/level3_impl.h:98-760) feed the GEBP kernel through triangular and
// self-adjoint packing (GeneralMatrixMatrixTriangular.h, SelfadjointMatrixMatrix.h,
// TriangularMatrixMatrix.h, TriangularSolverMatrix.h).  Here every product of any size goes
// through the device GEMM, and these kernels handle the triangles: they are memory-bound
// (expand, merge, scale: one read and one write per element) or, for the diagonal blocks,
// small (kTriBlock x kTriBlock) in shared memory.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"

namespace eb2 {
namespace {

constexpr int kTile = 32;  // 32 x 32 element tiles, 32 x 8 threads
constexpr int kRowsPerThread = kTile / 8;

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__device__ __forceinline__ bool in_triangle(int64_t i, int64_t j, bool upper) { return upper ? i <= j : i >= j; }

// out (n x n, ld ldo) = the symmetric matrix whose triangle `upper` is stored in A (ld lda):
// out(i,j) = A(i,j) inside the triangle and A(j,i) outside.  The mirrored reads go through
// a shared-memory tile so that both the reads and the writes are coalesced; elements of A
// outside the stored triangle are never read.
template <typename T>
__global__ void expand_symmetric_kernel(const T* __restrict__ A, int64_t lda, int64_t n, bool upper,
                                        T* __restrict__ out, int64_t ldo) {
  __shared__ T mirror[kTile][kTile + 1];
  const int64_t bi = int64_t(blockIdx.x) * kTile, bj = int64_t(blockIdx.y) * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  // tile (bj, bi) of A, needed where tile (bi, bj) is (partly) outside the triangle
  const bool any_outside = upper ? (bi + kTile - 1 > bj) : (bi < bj + kTile - 1);
  if (any_outside) {
    for (int q = 0; q < kRowsPerThread; ++q) {
      const int jj = ty + 8 * q;  // column of the mirrored tile = row of the output tile
      const int64_t r = bj + tx, c = bi + jj;  // element A(r, c) = out(c, r)
      if (r < n && c < n && in_triangle(r, c, upper)) mirror[jj][tx] = A[r + c * lda];
    }
  }
  __syncthreads();
  for (int q = 0; q < kRowsPerThread; ++q) {
    const int jj = ty + 8 * q;
    const int64_t i = bi + tx, j = bj + jj;
    if (i >= n || j >= n) continue;
    out[i + j * ldo] = in_triangle(i, j, upper) ? A[i + j * lda] : mirror[tx][jj];
  }
}

// out (n x n, ld ldo) = the triangular matrix stored in the triangle `upper` of A: A(i,j)
// inside the triangle, 0 outside, 1 on the diagonal when `unit` (then the stored diagonal is
// not read).
template <typename T>
__global__ void expand_triangular_kernel(const T* __restrict__ A, int64_t lda, int64_t n, bool upper, bool unit,
                                         T* __restrict__ out, int64_t ldo) {
  const int64_t bi = int64_t(blockIdx.x) * kTile, bj = int64_t(blockIdx.y) * kTile;
  for (int q = 0; q < kRowsPerThread; ++q) {
    const int64_t i = bi + threadIdx.x, j = bj + threadIdx.y + 8 * q;
    if (i >= n || j >= n) continue;
    T v = T(0);
    if (i == j)
      v = unit ? T(1) : A[i + j * lda];
    else if (in_triangle(i, j, upper))
      v = A[i + j * lda];
    out[i + j * ldo] = v;
  }
}

// C(i,j) = P(i,j) + beta C(i,j) on the triangle `upper` of the n x n C; beta == 0 writes P
// and never reads C; P == null stands for a zero product (C := beta C, beta == 0 writing
// exact zeros).  The other triangle is not touched.  With `only_if_flag` the kernel does
// nothing unless *only_if_flag != 0.
template <typename T>
__global__ void merge_triangle_kernel(const T* __restrict__ P, int64_t ldp, int64_t n, bool upper, T beta,
                                      T* __restrict__ C, int64_t ldc, const int* only_if_flag) {
  if (only_if_flag && *only_if_flag == 0) return;
  const int64_t bi = int64_t(blockIdx.x) * kTile, bj = int64_t(blockIdx.y) * kTile;
  for (int q = 0; q < kRowsPerThread; ++q) {
    const int64_t i = bi + threadIdx.x, j = bj + threadIdx.y + 8 * q;
    if (i >= n || j >= n || !in_triangle(i, j, upper)) continue;
    const T p = P ? P[i + j * ldp] : T(0);
    T* c = C + i + j * ldc;
    *c = beta == T(0) ? p : fma_rn(beta, *c, p);
  }
}

// X := alpha X elementwise (m x n, ld ldx): a plain multiply, so non-finite entries stay
// non-finite even for alpha == 0.
template <typename T>
__global__ void multiply_kernel(int64_t m, int64_t n, T alpha, T* __restrict__ X, int64_t ldx) {
  const int64_t bi = int64_t(blockIdx.x) * kTile, bj = int64_t(blockIdx.y) * kTile;
  for (int q = 0; q < kRowsPerThread; ++q) {
    const int64_t i = bi + threadIdx.x, j = bj + threadIdx.y + 8 * q;
    if (i < m && j < n) X[i + j * ldx] *= alpha;
  }
}

// The triangular block E (nb x nb, nb <= kTriBlock, element (r, c) at E[r*er + c*ec]; the
// triangle `lower` or upper is used, the diagonal is taken as 1 when `unit`) applied in
// place to `count` vectors x (element r of vector t at X[r*vs + t*ts]):
//   kSolve: x := E^-1 x by substitution;  otherwise x := E x.
// One thread per vector; E and a tile of kTriVecs vectors are staged in shared memory with
// coalesced loads and stores (the vector index runs fastest when ts == 1, the element index
// otherwise).
template <typename T, bool kSolve>
__global__ void __launch_bounds__(kTriVecs) tri_block_kernel(const T* __restrict__ E, int64_t er, int64_t ec, int nb,
                                                             bool lower, bool unit, T* __restrict__ X, int64_t vs,
                                                             int64_t ts, int64_t count) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Es = reinterpret_cast<T*>(smem_raw);  // [nb][nb]
  T* Xs = Es + nb * nb;                    // [nb][kTriVecs + 1], Xs[r * (kTriVecs+1) + t]
  constexpr int kXld = kTriVecs + 1;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < nb * nb; idx += kTriVecs) {
    const int r = idx / nb, c = idx % nb;
    T v = T(0);
    if (r == c)
      v = unit ? T(1) : E[r * er + c * ec];
    else if (lower ? r > c : r < c)
      v = E[r * er + c * ec];
    Es[idx] = v;
  }
  const int64_t t0 = int64_t(blockIdx.x) * kTriVecs;
  const int nv = int(count - t0 < kTriVecs ? count - t0 : kTriVecs);
  const bool vec_fast = (ts == 1);
  for (int idx = tid; idx < nb * kTriVecs; idx += kTriVecs) {
    const int t = vec_fast ? idx % kTriVecs : idx / nb;
    const int r = vec_fast ? idx / kTriVecs : idx % nb;
    if (t < nv) Xs[r * kXld + t] = X[r * vs + (t0 + t) * ts];
  }
  __syncthreads();
  if (tid < nv) {
    T* x = Xs + tid;
    if (kSolve) {
      if (lower) {
        for (int r = 0; r < nb; ++r) {
          T s = x[r * kXld];
          for (int c = 0; c < r; ++c) s = fma_rn(-Es[r * nb + c], x[c * kXld], s);
          x[r * kXld] = unit ? s : s / Es[r * nb + r];
        }
      } else {
        for (int r = nb - 1; r >= 0; --r) {
          T s = x[r * kXld];
          for (int c = r + 1; c < nb; ++c) s = fma_rn(-Es[r * nb + c], x[c * kXld], s);
          x[r * kXld] = unit ? s : s / Es[r * nb + r];
        }
      }
    } else {
      // each new x[r] uses only entries that are still old: descending rows for a lower
      // triangle, ascending for an upper one
      if (lower) {
        for (int r = nb - 1; r >= 0; --r) {
          T s = Es[r * nb + r] * x[r * kXld];
          for (int c = 0; c < r; ++c) s = fma_rn(Es[r * nb + c], x[c * kXld], s);
          x[r * kXld] = s;
        }
      } else {
        for (int r = 0; r < nb; ++r) {
          T s = Es[r * nb + r] * x[r * kXld];
          for (int c = r + 1; c < nb; ++c) s = fma_rn(Es[r * nb + c], x[c * kXld], s);
          x[r * kXld] = s;
        }
      }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nb * kTriVecs; idx += kTriVecs) {
    const int t = vec_fast ? idx % kTriVecs : idx / nb;
    const int r = vec_fast ? idx / kTriVecs : idx % nb;
    if (t < nv) X[r * vs + (t0 + t) * ts] = Xs[r * kXld + t];
  }
}

dim3 tile_grid(int64_t m, int64_t n) {
  return dim3(unsigned((m + kTile - 1) / kTile), unsigned((n + kTile - 1) / kTile));
}

bool grid_fits(int64_t m, int64_t n) {
  return (m + kTile - 1) / kTile <= 0x7fffffff && (n + kTile - 1) / kTile <= 65535;
}

}  // namespace

template <typename T>
cudaError_t launch_expand_symmetric(const T* A, int64_t lda, int64_t n, bool upper, T* out, int64_t ldo,
                                    cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  if (!grid_fits(n, n)) return cudaErrorInvalidConfiguration;
  expand_symmetric_kernel<T><<<tile_grid(n, n), dim3(kTile, 8), 0, st>>>(A, lda, n, upper, out, ldo);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_expand_triangular(const T* A, int64_t lda, int64_t n, bool upper, bool unit, T* out, int64_t ldo,
                                     cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  if (!grid_fits(n, n)) return cudaErrorInvalidConfiguration;
  expand_triangular_kernel<T><<<tile_grid(n, n), dim3(kTile, 8), 0, st>>>(A, lda, n, upper, unit, out, ldo);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_merge_triangle(const T* P, int64_t ldp, int64_t n, bool upper, T beta, T* C, int64_t ldc,
                                  cudaStream_t st, const int* only_if_flag) {
  if (n == 0) return cudaSuccess;
  if (!grid_fits(n, n)) return cudaErrorInvalidConfiguration;
  merge_triangle_kernel<T><<<tile_grid(n, n), dim3(kTile, 8), 0, st>>>(P, ldp, n, upper, beta, C, ldc, only_if_flag);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_multiply(int64_t m, int64_t n, T alpha, T* X, int64_t ldx, cudaStream_t st) {
  if (m == 0 || n == 0) return cudaSuccess;
  if (!grid_fits(m, n)) return cudaErrorInvalidConfiguration;
  multiply_kernel<T><<<tile_grid(m, n), dim3(kTile, 8), 0, st>>>(m, n, alpha, X, ldx);
  return cudaGetLastError();
}

size_t tri_block_smem(int nb, size_t elem) { return (size_t(nb) * nb + size_t(nb) * (kTriVecs + 1)) * elem; }

template <typename T>
cudaError_t launch_tri_block(bool solve, const T* E, int64_t er, int64_t ec, int nb, bool lower, bool unit, T* X,
                             int64_t vs, int64_t ts, int64_t count, cudaStream_t st) {
  if (count == 0 || nb == 0) return cudaSuccess;
  if (nb < 0 || nb > kTriBlock || count < 0) return cudaErrorInvalidValue;
  const size_t smem = tri_block_smem(nb, sizeof(T));
  const int64_t blocks = (count + kTriVecs - 1) / kTriVecs;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  auto kern = solve ? tri_block_kernel<T, true> : tri_block_kernel<T, false>;
  // one attribute call per instantiation: the largest block's footprint
  static_assert(sizeof(T) <= 8, "element size");
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tri_block_smem(kTriBlock, 8)));
  if (e != cudaSuccess) return e;
  kern<<<unsigned(blocks), kTriVecs, smem, st>>>(E, er, ec, nb, lower, unit, X, vs, ts, count);
  return cudaGetLastError();
}

#define EB2_TRI_INSTANTIATE(T)                                                                                     \
  template cudaError_t launch_expand_symmetric<T>(const T*, int64_t, int64_t, bool, T*, int64_t, cudaStream_t);     \
  template cudaError_t launch_expand_triangular<T>(const T*, int64_t, int64_t, bool, bool, T*, int64_t,             \
                                                   cudaStream_t);                                                  \
  template cudaError_t launch_merge_triangle<T>(const T*, int64_t, int64_t, bool, T, T*, int64_t, cudaStream_t,    \
                                                const int*);                                                       \
  template cudaError_t launch_multiply<T>(int64_t, int64_t, T, T*, int64_t, cudaStream_t);                          \
  template cudaError_t launch_tri_block<T>(bool, const T*, int64_t, int64_t, int, bool, bool, T*, int64_t, int64_t, \
                                           int64_t, cudaStream_t);
EB2_TRI_INSTANTIATE(double)
EB2_TRI_INSTANTIATE(float)
#undef EB2_TRI_INSTANTIATE

}  // namespace eb2
