// tri.cu -- the element-wise kernels the symmetric and triangular level-3 routines need
// around the GEMM: expanding a stored symmetric or triangular matrix into a full one, merging a
// product into one triangle of C, scaling a triangle or a matrix, and applying a triangular
// diagonal block to a panel in place (a multiply, or a solve by blocked substitution).
//
// Eigen's routines (blas/level3_impl.h:98-760) feed the GEBP kernel through triangular and
// self-adjoint packing (GeneralMatrixMatrixTriangular.h, SelfadjointMatrixMatrix.h,
// TriangularMatrixMatrix.h, TriangularSolverMatrix.h).  Here every product of any size goes
// through the device GEMM, and these kernels handle the triangles: they are memory-bound
// (expand, merge, scale: one read and one write per element) or, for the diagonal blocks,
// work on vectors staged in shared memory.
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

// x := E x in place for `count` vectors x (element r of vector t at X[r*vs + t*ts]), E the
// triangular block (nb x nb, nb <= kTriBlock, element (r, c) at E[r*er + c*ec]; the triangle
// `lower` or upper is used, the diagonal is taken as 1 when `unit`).  One thread per vector;
// E and a tile of kTriVecs vectors are staged in shared memory with coalesced loads and stores
// (the vector index runs fastest when ts == 1, the element index otherwise).
template <typename T>
__global__ void __launch_bounds__(kTriVecs) tri_block_multiply_kernel(const T* __restrict__ E, int64_t er, int64_t ec,
                                                                      int nb, bool lower, bool unit,
                                                                      T* __restrict__ X, int64_t vs, int64_t ts,
                                                                      int64_t count) {
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
  __syncthreads();
  for (int idx = tid; idx < nb * kTriVecs; idx += kTriVecs) {
    const int t = vec_fast ? idx % kTriVecs : idx / nb;
    const int r = vec_fast ? idx / kTriVecs : idx % nb;
    if (t < nv) X[r * vs + (t0 + t) * ts] = Xs[r * kXld + t];
  }
}

// Four consecutive elements of a 16-byte aligned shared-memory row as vector accesses.
__device__ __forceinline__ void load4(double (&v)[4], const double* p) {
  const double2 lo = *reinterpret_cast<const double2*>(p), hi = *reinterpret_cast<const double2*>(p + 2);
  v[0] = lo.x;
  v[1] = lo.y;
  v[2] = hi.x;
  v[3] = hi.y;
}
__device__ __forceinline__ void load4(float (&v)[4], const float* p) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x;
  v[1] = q.y;
  v[2] = q.z;
  v[3] = q.w;
}
__device__ __forceinline__ void store4(double* p, const double (&v)[4]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void store4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// x := E^-1 x for a diagonal block E of up to kPanelMax rows and `count` vectors (laid out
// as above), kPanelVecs per CTA, the CTA's vectors resident in shared memory for the whole
// block.  Blocked substitution over 32-row sub-blocks:
//   * two warps solve the sub-block (one lane per vector) against its 32 x 32 triangle,
//     column by column with the reciprocal of each diagonal entry, in the order of Eigen's
//     column-major triangular solve kernel (Eigen/src/Core/products/TriangularSolverMatrix.h:61-82);
//   * all threads subtract its contribution from the rows below, a register-tiled product
//     (4 rows x 4 vectors per thread) with the coefficient panel staged in shared memory
//     128 rows at a time.
// An upper triangle is solved as the lower one of the index-reversed system (row r <->
// nb-1-r), so both run forward.
constexpr int kPanelSub = 32;
constexpr int kPanelThreads = 512;
constexpr int kPanelChunk = 128;            // coefficient rows staged per pass
constexpr int kPanelXld = kPanelVecs + 4;   // row stride of the resident vectors (16 B aligned)
constexpr int kPanelDld = kPanelSub + 1;    // row stride of the diagonal sub-block

template <typename T>
__global__ void __launch_bounds__(kPanelThreads) tri_panel_solve_kernel(const T* __restrict__ E, int64_t er, int64_t ec,
                                                                        int nb, bool lower, bool unit,
                                                                        T* __restrict__ X, int64_t vs, int64_t ts,
                                                                        int64_t count) {
  static_assert(kPanelVecs == 64 && kPanelThreads == 512 && kPanelChunk == 128, "thread tiling");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Xs = reinterpret_cast<T*>(smem_raw);      // [nb][kPanelXld]: Xs[r * kPanelXld + t], forward row order
  T* Ds = Xs + nb * kPanelXld;                 // [kPanelSub][kPanelDld]: the diagonal sub-block
  T* Dinv = Ds + kPanelSub * kPanelDld;        // [kPanelSub]: reciprocals of the diagonal
  T* Cs = Dinv + kPanelSub;                    // [kPanelSub][kPanelChunk]: coefficients, Cs[c * chunk + row]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tx = tid & 15, ty = tid >> 4;      // product tiling: vectors 4tx.., rows 4ty..
  const int64_t t0 = int64_t(blockIdx.x) * kPanelVecs;
  const int nv = int(count - t0 < kPanelVecs ? count - t0 : kPanelVecs);
  // forward row r is row ro(r) of the stored system
  auto ro = [&](int r) -> int64_t { return lower ? r : nb - 1 - r; };
  const bool vec_fast = (ts == 1);
  for (int idx = tid; idx < nb * kPanelVecs; idx += kPanelThreads) {
    const int t = vec_fast ? idx % kPanelVecs : idx / nb;
    const int r = vec_fast ? idx / kPanelVecs : idx % nb;
    Xs[r * kPanelXld + t] = t < nv ? X[ro(r) * vs + (t0 + t) * ts] : T(0);
  }
  // the coefficient (r, c) of a panel is contiguous along r when the stored rows are
  const bool row_fast = (er == 1 || er == -1);
  for (int jb = 0; jb < nb; jb += kPanelSub) {
    const int bs = nb - jb < kPanelSub ? nb - jb : kPanelSub;
    __syncthreads();  // the rows of this sub-block are final (and, first, the load is done)
    for (int idx = tid; idx < bs * bs; idx += kPanelThreads) {
      const int r = idx / bs, c = idx % bs;
      T v = T(0);
      if (r == c)
        v = unit ? T(1) : E[ro(jb + r) * er + ro(jb + c) * ec];
      else if (r > c)
        v = E[ro(jb + r) * er + ro(jb + c) * ec];
      Ds[r * kPanelDld + c] = v;
      if (r == c) Dinv[r] = unit ? T(1) : T(1) / v;
    }
    __syncthreads();
    if (warp < 2) {
      // column by column, as Eigen's column-major kernel: x_c = s_c / d_c, then s_r -= d_rc x_c
      // for every later row r -- independent updates, so the dependent chain is two
      // operations per row instead of one per coefficient
      T* x = Xs + warp * 32 + lane;
      T sv[kPanelSub];
#pragma unroll
      for (int r = 0; r < kPanelSub; ++r) sv[r] = r < bs ? x[(jb + r) * kPanelXld] : T(0);
#pragma unroll
      for (int c = 0; c < kPanelSub; ++c) {
        const T xc = sv[c] * Dinv[c < bs ? c : 0];
        sv[c] = xc;
#pragma unroll
        for (int r = c + 1; r < kPanelSub; ++r) sv[r] = fma_rn(-Ds[r * kPanelDld + c], xc, sv[r]);
      }
#pragma unroll
      for (int r = 0; r < kPanelSub; ++r)
        if (r < bs) x[(jb + r) * kPanelXld] = sv[r];
    }
    // rows below: x[r] -= E'(r, jb..jb+bs) x[jb..jb+bs], kPanelChunk rows per pass
    for (int r0 = jb + bs; r0 < nb; r0 += kPanelChunk) {
      const int rows = nb - r0 < kPanelChunk ? nb - r0 : kPanelChunk;
      // every thread's coefficient loads are issued before its first shared store
      constexpr int kPerThread = kPanelSub * kPanelChunk / kPanelThreads;
      T cv[kPerThread];
#pragma unroll
      for (int q = 0; q < kPerThread; ++q) {
        const int idx = tid + q * kPanelThreads;
        const int rr = row_fast ? idx % kPanelChunk : idx / kPanelSub;
        const int c = row_fast ? idx / kPanelChunk : idx % kPanelSub;
        cv[q] = (rr < rows && c < bs) ? E[ro(r0 + rr) * er + ro(jb + c) * ec] : T(0);
      }
      __syncthreads();  // the sub-block solve is done / the previous chunk's Cs is consumed
#pragma unroll
      for (int q = 0; q < kPerThread; ++q) {
        const int idx = tid + q * kPanelThreads;
        const int rr = row_fast ? idx % kPanelChunk : idx / kPanelSub;
        const int c = row_fast ? idx / kPanelChunk : idx % kPanelSub;
        Cs[c * kPanelChunk + rr] = cv[q];
      }
      __syncthreads();
      T acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
#pragma unroll 8
      for (int c = 0; c < kPanelSub; ++c) {
        // four consecutive coefficients / vector entries as 16-byte loads (no bank conflicts)
        T a[4], b[4];
        load4(a, Cs + c * kPanelChunk + 4 * ty);
        load4(b, Xs + (jb + (c < bs ? c : 0)) * kPanelXld + 4 * tx);
        if (c < bs) {
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma_rn(a[i], b[j], acc[i][j]);
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rr = 4 * ty + i;
        if (rr < rows) {
          T* xp = Xs + (r0 + rr) * kPanelXld + 4 * tx;
          T x4[4];
          load4(x4, xp);
#pragma unroll
          for (int j = 0; j < 4; ++j) x4[j] -= acc[i][j];
          store4(xp, x4);
        }
      }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < nb * kPanelVecs; idx += kPanelThreads) {
    const int t = vec_fast ? idx % kPanelVecs : idx / nb;
    const int r = vec_fast ? idx / kPanelVecs : idx % nb;
    if (t < nv) X[ro(r) * vs + (t0 + t) * ts] = Xs[r * kPanelXld + t];
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
cudaError_t launch_tri_block_multiply(const T* E, int64_t er, int64_t ec, int nb, bool lower, bool unit, T* X,
                                      int64_t vs, int64_t ts, int64_t count, cudaStream_t st) {
  if (count == 0 || nb == 0) return cudaSuccess;
  if (nb < 0 || nb > kTriBlock || count < 0) return cudaErrorInvalidValue;
  const size_t smem = tri_block_smem(nb, sizeof(T));
  const int64_t blocks = (count + kTriVecs - 1) / kTriVecs;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  auto kern = tri_block_multiply_kernel<T>;
  // one attribute call per instantiation: the largest block's footprint
  static_assert(sizeof(T) <= 8, "element size");
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tri_block_smem(kTriBlock, 8)));
  if (e != cudaSuccess) return e;
  kern<<<unsigned(blocks), kTriVecs, smem, st>>>(E, er, ec, nb, lower, unit, X, vs, ts, count);
  return cudaGetLastError();
}

size_t tri_panel_smem(int nb, size_t elem) {
  return (size_t(nb) * kPanelXld + size_t(kPanelSub) * kPanelDld + kPanelSub + size_t(kPanelSub) * kPanelChunk) *
         elem;
}

template <typename T>
cudaError_t launch_tri_panel_solve(const T* E, int64_t er, int64_t ec, int nb, bool lower, bool unit, T* X, int64_t vs,
                                   int64_t ts, int64_t count, cudaStream_t st) {
  if (count == 0 || nb == 0) return cudaSuccess;
  if (nb < 0 || nb > kPanelMax || count < 0) return cudaErrorInvalidValue;
  const int64_t blocks = (count + kPanelVecs - 1) / kPanelVecs;
  if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
  auto kern = tri_panel_solve_kernel<T>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tri_panel_smem(kPanelMax, 8)));
  if (e != cudaSuccess) return e;
  kern<<<unsigned(blocks), kPanelThreads, tri_panel_smem(nb, sizeof(T)), st>>>(E, er, ec, nb, lower, unit, X, vs, ts,
                                                                              count);
  return cudaGetLastError();
}

#define EB2_TRI_INSTANTIATE(T)                                                                                     \
  template cudaError_t launch_expand_symmetric<T>(const T*, int64_t, int64_t, bool, T*, int64_t, cudaStream_t);     \
  template cudaError_t launch_expand_triangular<T>(const T*, int64_t, int64_t, bool, bool, T*, int64_t,             \
                                                   cudaStream_t);                                                  \
  template cudaError_t launch_merge_triangle<T>(const T*, int64_t, int64_t, bool, T, T*, int64_t, cudaStream_t,    \
                                                const int*);                                                       \
  template cudaError_t launch_multiply<T>(int64_t, int64_t, T, T*, int64_t, cudaStream_t);                          \
  template cudaError_t launch_tri_block_multiply<T>(const T*, int64_t, int64_t, int, bool, bool, T*, int64_t,       \
                                                    int64_t, int64_t, cudaStream_t);                               \
  template cudaError_t launch_tri_panel_solve<T>(const T*, int64_t, int64_t, int, bool, bool, T*, int64_t, int64_t, \
                                                 int64_t, cudaStream_t);
EB2_TRI_INSTANTIATE(double)
EB2_TRI_INSTANTIATE(float)
#undef EB2_TRI_INSTANTIATE

}  // namespace eb2
