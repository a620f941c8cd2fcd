// level3_api.cpp -- the other level-3 BLAS routines Eigen's BLAS library exports, built on
// the device GEMM: ?gemmtr_, ?syrk_, ?syr2k_, ?symm_, ?trmm_ and ?trsm_ (double and single
// precision) and the complex zgemm_ / cgemm_ (Fortran convention, LP64 and ILP64 _64_
// symbols).
//
// Argument checks, xerbla_ names and info codes, quick returns and the beta/alpha rules
// restate blas/level3_impl.h (gemmtr :98-228, trsm :230-364, trmm :368-503, symm :507-592,
// syrk :596-689, syr2k :693-754).  The products are Eigen's GEBP consumers
// (GeneralMatrixMatrixTriangular.h, TriangularSolverMatrix.h, TriangularMatrixMatrix.h,
// SelfadjointMatrixMatrix.h); here they are recursive block algorithms whose every product
// is one device GEMM call (so DGEMM sub-products take the emulated or native FP64 kernels
// the method setting and picker choose), with the triangles handled by the kernels of
// tri.cu:
//   gemmtr / syrk / syr2k  with the CRT emulation, one product restricted to the output
//                          tiles that meet C's triangle (its GEMM launch walks only those
//                          tiles; the reconstruction writes only the triangle; A A^T splits
//                          A once); otherwise the triangle split in two halves: the
//                          off-diagonal block is one GEMM straight into C, the two diagonal
//                          halves recurse, and a diagonal block of at most kTrLeaf is a full
//                          GEMM into a workspace merged into C's triangle;
//   symm                   the symmetric operand expanded to a full matrix, then one GEMM;
//   trmm                   with an emulated GEMM and size >= 1024, one product with the
//                          triangle expanded into a workspace (zeros, unit diagonal);
//   trmm / trsm            otherwise the triangular operand split in two halves: one GEMM
//                          for the off-diagonal block, recursion on the diagonal halves, and
//                          a shared-memory kernel for the diagonal blocks: a blocked
//                          substitution over blocks of up to kPanelMax rows (trsm), a
//                          multiply over blocks of up to kTriBlock (trmm).
// Host operands are staged through device buffers; device or managed operands are used in
// place.  The calls are synchronous.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <functional>
#include <optional>

#include "blas_common.h"
#include "context.h"
#include "eigen_b200/blas.h"
#include "gemm_driver.h"
#include "kernels.h"

namespace eb2 {
namespace {

constexpr int64_t kTrLeaf = 1024;   // largest diagonal block of gemmtr computed as a full product
constexpr int64_t kTrSplit = 256;   // gemmtr halves are rounded to this

int64_t imax1(int64_t v) { return std::max<int64_t>(1, v); }

// ---------------------------------------------------------------- argument checks
// blas/level3_impl.h:182-199
int gemmtr_info(char uplo, char ta, char tb, int64_t n, int64_t k, int64_t lda, int64_t ldb, int64_t ldc) {
  if (uplo_code(uplo) == kInvalid) return 1;
  if (op_code(ta) == kInvalid) return 2;
  if (op_code(tb) == kInvalid) return 3;
  if (n < 0) return 4;
  if (k < 0) return 5;
  if (lda < imax1(op_code(ta) == kNoTr ? n : k)) return 8;
  if (ldb < imax1(op_code(tb) == kNoTr ? k : n)) return 10;
  if (ldc < imax1(n)) return 13;
  return 0;
}

// blas/level3_impl.h:636-649
int syrk_info(char uplo, char op, int64_t n, int64_t k, int64_t lda, int64_t ldc) {
  if (uplo_code(uplo) == kInvalid) return 1;
  if (op_code(op) == kInvalid) return 2;
  if (n < 0) return 3;
  if (k < 0) return 4;
  if (lda < imax1(op_code(op) == kNoTr ? n : k)) return 7;
  if (ldc < imax1(n)) return 10;
  return 0;
}

// blas/level3_impl.h:702-717
int syr2k_info(char uplo, char op, int64_t n, int64_t k, int64_t lda, int64_t ldb, int64_t ldc) {
  if (uplo_code(uplo) == kInvalid) return 1;
  if (op_code(op) == kInvalid) return 2;
  if (n < 0) return 3;
  if (k < 0) return 4;
  if (lda < imax1(op_code(op) == kNoTr ? n : k)) return 7;
  if (ldb < imax1(op_code(op) == kNoTr ? n : k)) return 9;
  if (ldc < imax1(n)) return 12;
  return 0;
}

// blas/level3_impl.h:516-531
int symm_info(char side, char uplo, int64_t m, int64_t n, int64_t lda, int64_t ldb, int64_t ldc) {
  if (side_code(side) == kInvalid) return 1;
  if (uplo_code(uplo) == kInvalid) return 2;
  if (m < 0) return 3;
  if (n < 0) return 4;
  if (lda < imax1(side_code(side) == kLeft ? m : n)) return 7;
  if (ldb < imax1(m)) return 9;
  if (ldc < imax1(m)) return 12;
  return 0;
}

// trsm blas/level3_impl.h:330-347, trmm :467-484 (the same checks)
int trxm_info(char side, char uplo, char op, char diag, int64_t m, int64_t n, int64_t lda, int64_t ldb) {
  if (side_code(side) == kInvalid) return 1;
  if (uplo_code(uplo) == kInvalid) return 2;
  if (op_code(op) == kInvalid) return 3;
  if (diag_code(diag) == kInvalid) return 4;
  if (m < 0) return 5;
  if (n < 0) return 6;
  if (lda < imax1(side_code(side) == kLeft ? m : n)) return 9;
  if (ldb < imax1(m)) return 11;
  return 0;
}

// ---------------------------------------------------------------- products
// Summary of the GEMM calls of one routine, reported through eb2_last_call_info.
struct Summary {
  int method = 0, slices = 0, escalations = 0, nonfinite = 0, launches = 0, calls = 0;
  double err = -1.0;
  int64_t biggest = -1;  // flops of the largest call (its method is reported)
};

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  (void)cudaGetLastError();
  set_error(EB2_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return false;
}

// C = alpha op(A) op(B) + beta C on device pointers, queued on st.  DGEMM sub-products keep
// the a-posteriori accuracy check of the emulated methods (which waits for its flags);
// native products are only queued.
// uplo != 0: the CRT product of only C's upper (1) or lower (2) triangle (m == n).
int gemm(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
         int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc, cudaStream_t st,
         Summary& sum, int uplo = 0, int tri = 0) {
  if (m == 0 || n == 0) return EB2_OK;
  DgemmOptions o;
  o.sync = false;
  o.check_accuracy = true;
  o.timed = false;
  if (uplo) {
    o.method = EB2_METHOD_CRT;
    o.uplo = uplo;
  }
  o.tri_operand = tri;
  eb2_call_info ci{};
  const int rc = dgemm_on_device(cx, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st, o, ci);
  const int64_t flops = m * n * k;
  if (flops > sum.biggest) {
    sum.biggest = flops;
    sum.method = ci.method;
  }
  sum.slices = std::max(sum.slices, ci.slices);
  sum.escalations += ci.escalations;
  sum.nonfinite |= ci.nonfinite;
  sum.launches += ci.launches;
  sum.err = std::max(sum.err, ci.err_estimate);
  sum.calls += 1;
  return rc;
}

int gemm(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, float alpha, const float* A, int64_t lda,
         const float* B, int64_t ldb, float beta, float* C, int64_t ldc, cudaStream_t st, Summary& sum) {
  if (m == 0 || n == 0) return EB2_OK;
  SgemmOptions o;
  o.sync = false;
  o.timed = false;
  eb2_call_info ci{};
  const int rc = sgemm_on_device(cx, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st, o, ci);
  const int64_t flops = m * n * k;
  if (flops > sum.biggest) {
    sum.biggest = flops;
    sum.method = ci.method;
  }
  sum.slices = std::max(sum.slices, ci.slices);
  sum.nonfinite |= ci.nonfinite;
  sum.launches += ci.launches;
  sum.calls += 1;
  return rc;
}

// An accuracy miss of one sub-product is reported at the end; everything else stops.
bool keep_going(int rc, int& worst) {
  if (rc == EB2_OK) return true;
  if (rc == EB2_ERR_ACCURACY) {
    worst = EB2_ERR_ACCURACY;
    return true;
  }
  worst = rc;
  return false;
}

// ---------------------------------------------------------------- device algorithms
// Row block [r0, ..) of op(X) and column block [c0, ..) of op(X), X column-major (ld ldx).
template <typename T>
const T* op_rows(const T* X, int64_t ldx, bool trans, int64_t r0) {
  return trans ? X + r0 * ldx : X + r0;
}
template <typename T>
const T* op_cols(const T* X, int64_t ldx, bool trans, int64_t c0) {
  return trans ? X + c0 : X + c0 * ldx;
}

// The triangle `upper` of the n x n C := alpha op(A) op(B) + beta C (op(A) n x k, op(B) k x n).
template <typename T>
int gemmtr_device(Context& cx, bool upper, bool ta, bool tb, int64_t n, int64_t k, T alpha, const T* A, int64_t lda,
                  const T* B, int64_t ldb, T beta, T* C, int64_t ldc, cudaStream_t st, Summary& sum) {
  if (n == 0) return EB2_OK;
  if (k == 0 || alpha == T(0)) {
    if (beta == T(1)) return EB2_OK;
    return cuda_ok(launch_merge_triangle<T>(nullptr, 0, n, upper, beta, C, ldc, st), "scale triangle") ? EB2_OK
                                                                                                     : EB2_ERR_CUDA;
  }
  if constexpr (sizeof(T) == 8) {
    // the CRT product computes only the tiles that meet the triangle: one call, one split
    if (resolve_dgemm_method(n, n, k) == EB2_METHOD_CRT)
      return gemm(cx, ta, tb, n, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st, sum, upper ? 1 : 2);
  }
  const int64_t leaf = std::min(n, kTrLeaf);
  if (!cx.tmp.ensure(size_t(leaf) * size_t(leaf) * sizeof(T))) {
    set_error(EB2_ERR_ALLOC, "could not allocate the diagonal-block workspace");
    return EB2_ERR_ALLOC;
  }
  T* P = static_cast<T*>(cx.tmp.ptr);
  int worst = EB2_OK;
  std::function<bool(int64_t, int64_t)> rec = [&](int64_t n0, int64_t size) -> bool {
    if (size <= kTrLeaf) {
      // the diagonal block as a full product, merged into the triangle
      if (!keep_going(gemm(cx, ta, tb, size, size, k, alpha, op_rows(A, lda, ta, n0), lda, op_cols(B, ldb, tb, n0),
                           ldb, T(0), P, size, st, sum),
                      worst))
        return false;
      if (!cuda_ok(launch_merge_triangle<T>(P, size, size, upper, beta, C + n0 + n0 * ldc, ldc, st), "merge")) {
        worst = EB2_ERR_CUDA;
        return false;
      }
      return true;
    }
    const int64_t h = std::min(size - 1, (size / 2 + kTrSplit - 1) / kTrSplit * kTrSplit);
    // the off-diagonal block straight into C
    const int rc = upper ? gemm(cx, ta, tb, h, size - h, k, alpha, op_rows(A, lda, ta, n0), lda,
                                op_cols(B, ldb, tb, n0 + h), ldb, beta, C + n0 + (n0 + h) * ldc, ldc, st, sum)
                         : gemm(cx, ta, tb, size - h, h, k, alpha, op_rows(A, lda, ta, n0 + h), lda,
                                op_cols(B, ldb, tb, n0), ldb, beta, C + (n0 + h) + n0 * ldc, ldc, st, sum);
    if (!keep_going(rc, worst)) return false;
    return rec(n0, h) && rec(n0 + h, size - h);
  };
  rec(0, n);
  return worst;
}

// C := alpha A B + beta C (left, A m x m) or alpha B A + beta C (right, A n x n), A
// symmetric with the triangle `upper` stored.
template <typename T>
int symm_device(Context& cx, bool left, bool upper, int64_t m, int64_t n, T alpha, const T* A, int64_t lda,
                const T* B, int64_t ldb, T beta, T* C, int64_t ldc, cudaStream_t st, Summary& sum) {
  if (m == 0 || n == 0) return EB2_OK;
  const int64_t size = left ? m : n;
  T* S = nullptr;
  if (alpha != T(0)) {
    if (!cx.tmp.ensure(size_t(size) * size_t(size) * sizeof(T))) {
      set_error(EB2_ERR_ALLOC, "could not allocate the symmetric-operand workspace");
      return EB2_ERR_ALLOC;
    }
    S = static_cast<T*>(cx.tmp.ptr);
    if (!cuda_ok(launch_expand_symmetric<T>(A, lda, size, upper, S, size, st), "expand")) return EB2_ERR_CUDA;
  }
  // alpha == 0 reads neither operand (the GEMM then only scales C)
  return left ? gemm(cx, false, false, m, n, m, alpha, S, size, B, ldb, beta, C, ldc, st, sum)
              : gemm(cx, false, false, m, n, n, alpha, B, ldb, S, size, beta, C, ldc, st, sum);
}

// trmm as one product with the expanded triangle: where the emulated GEMM runs (its rate
// more than pays for the doubled flops and removes the recursion's many small calls).
template <typename T>
bool trmm_as_one_product(int64_t size, int64_t m, int64_t n) {
  if (size < 1024) return false;
  if constexpr (sizeof(T) == 8) return resolve_dgemm_method(m, n, size) == EB2_METHOD_CRT;
  return settings().sgemm_method.load() != EB2_METHOD_NATIVE;
}

// In place on the m x n B: B := op(A)^-1 B / B op(A)^-1 (solve) or op(A) B / B op(A)
// (multiply), A triangular (triangle `upper` stored, unit diagonal if `unit`), then
// B := alpha B.
template <typename T>
int trxm_device(Context& cx, bool solve, bool left, bool upper, bool trans, bool unit, int64_t m, int64_t n, T alpha,
                const T* A, int64_t lda, T* B, int64_t ldb, cudaStream_t st, Summary& sum) {
  if (m == 0 || n == 0) return EB2_OK;
  if (!solve && alpha != T(0) && trmm_as_one_product<T>(left ? m : n, m, n)) {
    // one GEMM with the triangle expanded (zeros, unit diagonal) into a workspace, out of
    // place, then copied back: twice the flops of the recursion, but a single large product
    const int64_t size = left ? m : n;
    if (!cx.tmp.ensure((size_t(size) * size + size_t(m) * n) * sizeof(T))) {
      set_error(EB2_ERR_ALLOC, "could not allocate the triangular-product workspace");
      return EB2_ERR_ALLOC;
    }
    T* Tf = static_cast<T*>(cx.tmp.ptr);
    T* P = Tf + size_t(size) * size;
    if (!cuda_ok(launch_expand_triangular<T>(A, lda, size, upper, unit, Tf, size, st), "expand")) return EB2_ERR_CUDA;
    sum.launches += 1;
    int rc;
    if constexpr (sizeof(T) == 8) {
      // op(triangle) is lower when the stored triangle is lower and not transposed, or upper
      // and transposed; the CRT product then skips the K blocks that are zero in it
      const bool op_lower = upper == trans;
      rc = left ? gemm(cx, trans, false, m, n, m, alpha, Tf, size, B, ldb, T(0), P, m, st, sum, 0, op_lower ? 1 : 2)
                : gemm(cx, false, trans, m, n, n, alpha, B, ldb, Tf, size, T(0), P, m, st, sum, 0, op_lower ? 3 : 4);
    } else {
      rc = left ? gemm(cx, trans, false, m, n, m, alpha, Tf, size, B, ldb, T(0), P, m, st, sum)
                : gemm(cx, false, trans, m, n, n, alpha, B, ldb, Tf, size, T(0), P, m, st, sum);
    }
    if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) return rc;
    if (!cuda_ok(cudaMemcpy2DAsync(B, size_t(ldb) * sizeof(T), P, size_t(m) * sizeof(T), size_t(m) * sizeof(T),
                                   size_t(n), cudaMemcpyDeviceToDevice, st),
                 "copy back"))
      return EB2_ERR_CUDA;
    return rc;
  }
  // M = op(A); `lower` is M's triangle
  const bool lower = trans ? upper : !upper;
  // block M[r0.., c0..] as a GEMM operand (with transpose flag `trans`)
  auto msub = [&](int64_t r0, int64_t c0) -> const T* { return trans ? A + c0 + r0 * lda : A + r0 + c0 * lda; };
  const T sign = solve ? T(-1) : T(1);
  int worst = EB2_OK;
  auto leaf = [&](int64_t i0, int64_t nb) -> bool {
    const T* D = A + i0 + i0 * lda;  // diagonal block of A (and of M)
    // M(r, c) of the block at D[r*mr + c*mc]
    const int64_t mr = trans ? lda : 1, mc = trans ? 1 : lda;
    // vectors: the columns of B's rows [i0, i0+nb) (left), or the rows of B's columns
    // [i0, i0+nb) (right: x M = b is M^T x^T = b^T)
    const int64_t er = left ? mr : mc, ec = left ? mc : mr;
    const bool elower = left ? lower : !lower;
    T* X = left ? B + i0 : B + i0 * ldb;
    const int64_t vs = left ? 1 : ldb, ts = left ? ldb : 1, count = left ? n : m;
    const cudaError_t e = solve ? launch_tri_panel_solve<T>(D, er, ec, int(nb), elower, unit, X, vs, ts, count, st)
                                : launch_tri_block_multiply<T>(D, er, ec, int(nb), elower, unit, X, vs, ts, count, st);
    if (!cuda_ok(e, "triangular block")) {
      worst = EB2_ERR_CUDA;
      return false;
    }
    return true;
  };
  // B's rows (left) or columns (right) [d0, d0+dn) += sign * (M block) * B's [s0, s0+sn)
  auto update = [&](int64_t d0, int64_t dn, int64_t s0, int64_t sn) -> bool {
    const int rc = left ? gemm(cx, trans, false, dn, n, sn, sign, msub(d0, s0), lda, B + s0, ldb, T(1), B + d0, ldb,
                               st, sum)
                        : gemm(cx, false, trans, m, dn, sn, sign, B + s0 * ldb, ldb, msub(s0, d0), lda, T(1),
                               B + d0 * ldb, ldb, st, sum);
    return keep_going(rc, worst);
  };
  // diagonal blocks: up to kPanelMax rows for the solve (one launch per block, all of its
  // vectors resident in shared memory), kTriBlock for the multiply
  const int64_t leaf_max = solve ? kPanelMax : kTriBlock;
  std::function<bool(int64_t, int64_t)> rec = [&](int64_t i0, int64_t size) -> bool {
    if (size <= leaf_max) return leaf(i0, size);
    const int64_t h = (size / 2 + leaf_max - 1) / leaf_max * leaf_max;
    const int64_t a0 = i0, an = h, b0 = i0 + h, bn = size - h;
    // The first half in the order below is the one whose new values the update does not
    // need (solve) or whose old values it still needs (multiply).
    bool first_is_a;
    if (left)
      first_is_a = solve ? lower : !lower;
    else
      first_is_a = solve ? !lower : lower;
    if (first_is_a) {
      if (solve) return rec(a0, an) && update(b0, bn, a0, an) && rec(b0, bn);
      // multiply: update a from b (old), then a, then b
      return rec(a0, an) && update(a0, an, b0, bn) && rec(b0, bn);
    }
    if (solve) return rec(b0, bn) && update(a0, an, b0, bn) && rec(a0, an);
    return rec(b0, bn) && update(b0, bn, a0, an) && rec(a0, an);
  };
  if (!rec(0, left ? m : n)) return worst;
  if (alpha != T(1) && !cuda_ok(launch_multiply<T>(m, n, alpha, B, ldb, st), "scale")) return EB2_ERR_CUDA;
  return worst;
}

// ---------------------------------------------------------------- complex products
// C := (ar + i ai) op(A) op(B) + (br + i bi) C on device pointers to interleaved complex
// matrices (leading dimensions in complex elements), op codes kNoTr / kTr / kAdj.  The
// product is two real GEMMs of inner dimension 2k on packed operands (complex.cu):
// Re = [Ar Ai][Br; -Bi], Im = [Ar Ai][Bi; Br].  Workspace: cx.cplx.
template <typename T>
int complex_gemm_device(Context& cx, int oa, int ob, int64_t m, int64_t n, int64_t k, T ar, T ai, const T* A,
                        int64_t lda, const T* B, int64_t ldb, T br, T bi, T* C, int64_t ldc, cudaStream_t st,
                        Summary& sum) {
  if (m == 0 || n == 0) return EB2_OK;
  if (k == 0 || (ar == T(0) && ai == T(0))) {
    if (br == T(1) && bi == T(0)) return EB2_OK;
    sum.launches += 1;
    return cuda_ok(launch_combine_complex<T>(nullptr, nullptr, 0, m, n, ar, ai, br, bi, C, ldc, st), "scale C")
               ? EB2_OK
               : EB2_ERR_CUDA;
  }
  // workspace: A' (m x 2k), B1 and B2 (2k x n), Pr and Pi (m x n); B1 | B2 and Pr | Pi are
  // adjacent, so the two real products are one product of width 2n, and A' is scanned and
  // split once
  const size_t e_a = size_t(m) * 2 * k, e_b = size_t(2 * k) * n, e_p = size_t(m) * n;
  if (!cx.cplx.ensure((e_a + 2 * e_b + 2 * e_p) * sizeof(T))) {
    set_error(EB2_ERR_ALLOC, "could not allocate the complex-product workspace");
    return EB2_ERR_ALLOC;
  }
  T* Ap = static_cast<T*>(cx.cplx.ptr);
  T* B1 = Ap + e_a;
  T* B2 = B1 + e_b;
  T* Pr = B2 + e_b;
  T* Pi = Pr + e_p;
  bool ok = cuda_ok(launch_pack_complex_lhs<T>(A, oa == kNoTr ? 1 : lda, oa == kNoTr ? lda : 1, oa == kAdj, m, k, Ap,
                                               st),
                    "pack op(A)");
  ok = ok && cuda_ok(launch_pack_complex_rhs<T>(B, ob == kNoTr ? 1 : ldb, ob == kNoTr ? ldb : 1, ob == kAdj, k, n, B1,
                                                B2, st),
                     "pack op(B)");
  if (!ok) return EB2_ERR_CUDA;
  sum.launches += 2;
  int worst = EB2_OK;
  if (keep_going(gemm(cx, false, false, m, 2 * n, 2 * k, T(1), Ap, m, B1, 2 * k, T(0), Pr, m, st, sum), worst)) {
    if (!cuda_ok(launch_combine_complex<T>(Pr, Pi, m, m, n, ar, ai, br, bi, C, ldc, st), "combine"))
      worst = EB2_ERR_CUDA;
    sum.launches += 1;
  }
  return worst;
}

// C := alpha S B + beta C (left, S m x m) or alpha B S + beta C (right, S n x n), S the
// symmetric (hermitian = false) or Hermitian matrix whose triangle `upper` is stored in A;
// all complex, interleaved.
template <typename T>
int complex_symm_device(Context& cx, bool hermitian, bool left, bool upper, int64_t m, int64_t n, T ar, T ai,
                        const T* A, int64_t lda, const T* B, int64_t ldb, T br, T bi, T* C, int64_t ldc,
                        cudaStream_t st, Summary& sum) {
  if (m == 0 || n == 0) return EB2_OK;
  const int64_t size = left ? m : n;
  T* S = nullptr;
  if (ar != T(0) || ai != T(0)) {
    if (!cx.tmp.ensure(size_t(size) * size * 2 * sizeof(T))) {
      set_error(EB2_ERR_ALLOC, "could not allocate the symmetric-operand workspace");
      return EB2_ERR_ALLOC;
    }
    S = static_cast<T*>(cx.tmp.ptr);
    if (!cuda_ok(launch_expand_complex<T>(A, lda, size, upper, hermitian ? 1 : 0, false, S, size, st), "expand"))
      return EB2_ERR_CUDA;
    sum.launches += 1;
  }
  return left ? complex_gemm_device<T>(cx, kNoTr, kNoTr, m, n, m, ar, ai, S, size, B, ldb, br, bi, C, ldc, st, sum)
              : complex_gemm_device<T>(cx, kNoTr, kNoTr, m, n, n, ar, ai, B, ldb, S, size, br, bi, C, ldc, st, sum);
}

// In place on the complex m x n B: B := op(A)^-1 B / B op(A)^-1 (solve) or op(A) B / B op(A)
// (multiply), A triangular (triangle `upper` stored, unit diagonal if `unit`), op code `op`
// (kNoTr, kTr, kAdj), then B := alpha B.
template <typename T>
int complex_trxm_device(Context& cx, bool solve, bool left, bool upper, int op, bool unit, int64_t m, int64_t n,
                        T ar, T ai, const T* A, int64_t lda, T* B, int64_t ldb, cudaStream_t st, Summary& sum) {
  if (m == 0 || n == 0) return EB2_OK;
  const int64_t size = left ? m : n;
  const bool trans = op != kNoTr;
  if (!solve) {
    // one product with the triangle expanded (zeros, unit diagonal), out of place, copied back
    if (!cx.tmp.ensure((size_t(size) * size + size_t(m) * n) * 2 * sizeof(T))) {
      set_error(EB2_ERR_ALLOC, "could not allocate the triangular-product workspace");
      return EB2_ERR_ALLOC;
    }
    T* Tf = static_cast<T*>(cx.tmp.ptr);
    T* P = Tf + size_t(size) * size * 2;
    if (!cuda_ok(launch_expand_complex<T>(A, lda, size, upper, 2, unit, Tf, size, st), "expand")) return EB2_ERR_CUDA;
    sum.launches += 1;
    const int rc = left ? complex_gemm_device<T>(cx, op, kNoTr, m, n, m, ar, ai, Tf, size, B, ldb, T(0), T(0), P, m,
                                                 st, sum)
                        : complex_gemm_device<T>(cx, kNoTr, op, m, n, n, ar, ai, B, ldb, Tf, size, T(0), T(0), P, m,
                                                 st, sum);
    if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) return rc;
    if (!cuda_ok(cudaMemcpy2DAsync(B, size_t(ldb) * 2 * sizeof(T), P, size_t(m) * 2 * sizeof(T),
                                   size_t(m) * 2 * sizeof(T), size_t(n), cudaMemcpyDeviceToDevice, st),
                 "copy back"))
      return EB2_ERR_CUDA;
    return rc;
  }
  // the solve: recursion on halves as in trxm_device, complex GEMM updates, complex panels
  const bool lower = trans ? upper : !upper;  // the triangle of M = op(A)
  auto msub = [&](int64_t r0, int64_t c0) -> const T* { return A + 2 * (trans ? c0 + r0 * lda : r0 + c0 * lda); };
  int worst = EB2_OK;
  auto leaf = [&](int64_t i0, int64_t nb) -> bool {
    const T* D = A + 2 * (i0 + i0 * lda);
    const int64_t mr = trans ? lda : 1, mc = trans ? 1 : lda;
    const int64_t er = left ? mr : mc, ec = left ? mc : mr;
    T* X = left ? B + 2 * i0 : B + 2 * i0 * ldb;
    const int64_t vs = left ? 1 : ldb, ts = left ? ldb : 1, count = left ? n : m;
    if (!cuda_ok(launch_tri_panel_solve_complex<T>(D, er, ec, int(nb), left ? lower : !lower, unit, op == kAdj, X, vs,
                                                   ts, count, st),
                 "triangular block")) {
      worst = EB2_ERR_CUDA;
      return false;
    }
    sum.launches += 1;
    return true;
  };
  auto update = [&](int64_t d0, int64_t dn, int64_t s0, int64_t sn) -> bool {
    const int rc = left ? complex_gemm_device<T>(cx, op, kNoTr, dn, n, sn, T(-1), T(0), msub(d0, s0), lda, B + 2 * s0,
                                                 ldb, T(1), T(0), B + 2 * d0, ldb, st, sum)
                        : complex_gemm_device<T>(cx, kNoTr, op, m, dn, sn, T(-1), T(0), B + 2 * s0 * ldb, ldb,
                                                 msub(s0, d0), lda, T(1), T(0), B + 2 * d0 * ldb, ldb, st, sum);
    return keep_going(rc, worst);
  };
  std::function<bool(int64_t, int64_t)> rec = [&](int64_t i0, int64_t sz) -> bool {
    if (sz <= kPanelMaxComplex) return leaf(i0, sz);
    const int64_t h = (sz / 2 + kPanelMaxComplex - 1) / kPanelMaxComplex * kPanelMaxComplex;
    const int64_t a0 = i0, an = h, b0 = i0 + h, bn = sz - h;
    const bool first_is_a = left ? lower : !lower;
    if (first_is_a) return rec(a0, an) && update(b0, bn, a0, an) && rec(b0, bn);
    return rec(b0, bn) && update(a0, an, b0, bn) && rec(a0, an);
  };
  if (!rec(0, size)) return worst;
  if ((ar != T(1) || ai != T(0)) &&
      !cuda_ok(launch_combine_complex<T>(nullptr, nullptr, 0, m, n, T(0), T(0), ar, ai, B, ldb, st), "scale"))
    return EB2_ERR_CUDA;
  return worst;
}

// ---------------------------------------------------------------- host entry points
// A matrix argument as the device sees it: the caller's pointer when the device can use it
// in place, else a device copy (leading dimension = rows).
template <typename T>
struct Operand {
  T* ptr = nullptr;
  int64_t ld = 0;
  bool staged = false;
};

template <typename T>
bool stage(DeviceBuffer& buf, const T* p, int64_t ld, int64_t rows, int64_t cols, bool copy_in, cudaStream_t st,
           Operand<T>& out) {
  out.ptr = const_cast<T*>(p);
  out.ld = ld;
  out.staged = false;
  if (rows == 0 || cols == 0 || device_usable(p)) return true;
  if (!buf.ensure(size_t(rows) * size_t(cols) * sizeof(T))) {
    set_error(EB2_ERR_ALLOC, "could not allocate staging memory");
    return false;
  }
  out.ptr = static_cast<T*>(buf.ptr);
  out.ld = rows;
  out.staged = true;
  return !copy_in ||
         copy_block(out.ptr, size_t(rows) * sizeof(T), p, size_t(ld) * sizeof(T), size_t(rows) * sizeof(T), cols,
                    cudaMemcpyHostToDevice, st);
}

// One routine call: the device context locked for its duration, the call record, and the
// end of the call (the output copied back when staged, the stream drained, errors printed
// like the GEMM entry points do).
struct Call {
  Context* cx = nullptr;
  std::unique_lock<std::mutex> lock;
  std::optional<StreamFence> fence;  // constructed under the lock, destroyed before it
  cudaStream_t st = nullptr;
  Summary sum;
  char dtype = 'd';

  explicit Call(char dt) : dtype(dt) {}
  ~Call() { fence.reset(); }

  bool begin() {
    cx = current_context();
    if (!cx) {
      std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
      return false;
    }
    lock = std::unique_lock<std::mutex>(cx->mu);
    st = cx->stream;
    fence.emplace(*cx, st);
    call_info() = eb2_call_info{};
    call_config() = CallConfig{};
    set_pending_timing(nullptr, false);
    return true;
  }

  // the operands are on the device: the routine's device time starts here
  void started() { cudaEventRecord(cx->ev_start, st); }

  void fail() {
    std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
    (void)cudaStreamSynchronize(st);
  }

  // rc of the device algorithm; `out` the output operand, copied back to (host, host_ld).
  template <typename T>
  void end(int rc, bool any_staged, const Operand<T>& out, T* host, int64_t host_ld, int64_t rows, int64_t cols) {
    eb2_call_info& ci = call_info();
    ci.dtype = dtype;
    ci.method = sum.method;
    ci.slices = sum.slices;
    ci.escalations = sum.escalations;
    ci.nonfinite = sum.nonfinite;
    ci.staged = any_staged ? 1 : 0;
    ci.err_estimate = sum.err;
    ci.launches = sum.launches;
    ci.kernel_ms = -1.0;
    ci.gemm_kernel_ms = -1.0;
    if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) return fail();
    if (out.staged && !copy_block(host, size_t(host_ld) * sizeof(T), out.ptr, size_t(rows) * sizeof(T),
                                  size_t(rows) * sizeof(T), cols, cudaMemcpyDeviceToHost, st))
      return fail();
    cudaEventRecord(cx->ev_stop, st);
    if (!cuda_ok(cudaStreamSynchronize(st), "level-3 routine")) return fail();
    set_pending_timing(cx, false);
  }
};

template <typename T>
constexpr char dtype_of() {
  return sizeof(T) == 8 ? 'd' : 's';
}
template <typename T>
constexpr const char* prefixed(const char* d, const char* s) {
  return sizeof(T) == 8 ? d : s;
}

// blas/level3_impl.h:98-228: C's triangle := alpha op(A) op(B) + beta C's triangle
template <typename T>
void blas_gemmtr(char uplo, char opa, char opb, int64_t n, int64_t k, T alpha, const T* a, int64_t lda, const T* b,
                 int64_t ldb, T beta, T* c, int64_t ldc) {
  int info = gemmtr_info(uplo, opa, opb, n, k, lda, ldb, ldc);
  if (info) return xerbla_(prefixed<T>("DGEMMTR", "SGEMMTR"), &info, 7);
  if (n == 0) return;
  count_call(prefixed<T>("dgemmtr", "sgemmtr"));
  Call call(dtype_of<T>());
  if (!call.begin()) return;
  const bool ta = op_code(opa) != kNoTr, tb = op_code(opb) != kNoTr;
  const bool need_ab = k > 0 && alpha != T(0);
  Operand<T> A, B, C;
  // C keeps its other triangle: the whole square goes to the device and back
  if (!stage(call.cx->stage_a, a, lda, need_ab ? (ta ? k : n) : 0, ta ? n : k, true, call.st, A) ||
      !stage(call.cx->stage_b, b, ldb, need_ab ? (tb ? n : k) : 0, tb ? k : n, true, call.st, B) ||
      !stage(call.cx->stage_c, c, ldc, n, n, true, call.st, C))
    return call.fail();
  call.started();
  const int rc = gemmtr_device<T>(*call.cx, uplo_code(uplo) == kUp, ta, tb, n, k, alpha, A.ptr, A.ld, B.ptr, B.ld,
                                  beta, C.ptr, C.ld, call.st, call.sum);
  call.end(rc, A.staged || B.staged || C.staged, C, c, ldc, n, n);
}

// blas/level3_impl.h:596-689: C's triangle := alpha op(A) op(A)^T + beta C's triangle
template <typename T>
void blas_syrk(char uplo, char op, int64_t n, int64_t k, T alpha, const T* a, int64_t lda, T beta, T* c,
               int64_t ldc) {
  int info = syrk_info(uplo, op, n, k, lda, ldc);
  if (info) return xerbla_(prefixed<T>("DSYRK ", "SSYRK "), &info, 6);
  if (n == 0) return;
  count_call(prefixed<T>("dsyrk", "ssyrk"));
  Call call(dtype_of<T>());
  if (!call.begin()) return;
  const bool ta = op_code(op) != kNoTr;
  const bool need_a = k > 0 && alpha != T(0);
  Operand<T> A, C;
  if (!stage(call.cx->stage_a, a, lda, need_a ? (ta ? k : n) : 0, ta ? n : k, true, call.st, A) ||
      !stage(call.cx->stage_c, c, ldc, n, n, true, call.st, C))
    return call.fail();
  call.started();
  // op(A) op(A)^T: the same matrix on both sides, with opposite transposes
  const int rc = gemmtr_device<T>(*call.cx, uplo_code(uplo) == kUp, ta, !ta, n, k, alpha, A.ptr, A.ld, A.ptr, A.ld,
                                  beta, C.ptr, C.ld, call.st, call.sum);
  call.end(rc, A.staged || C.staged, C, c, ldc, n, n);
}

// blas/level3_impl.h:693-754: C's triangle := alpha (op(A) op(B)^T + op(B) op(A)^T) + beta C's
template <typename T>
void blas_syr2k(char uplo, char op, int64_t n, int64_t k, T alpha, const T* a, int64_t lda, const T* b, int64_t ldb,
                T beta, T* c, int64_t ldc) {
  int info = syr2k_info(uplo, op, n, k, lda, ldb, ldc);
  if (info) return xerbla_(prefixed<T>("DSYR2K", "SSYR2K"), &info, 6);
  if (n == 0) return;
  count_call(prefixed<T>("dsyr2k", "ssyr2k"));
  Call call(dtype_of<T>());
  if (!call.begin()) return;
  const bool ta = op_code(op) != kNoTr;
  const bool need_ab = k > 0 && alpha != T(0);
  const int64_t rows = need_ab ? (ta ? k : n) : 0, cols = ta ? n : k;
  Operand<T> A, B, C;
  if (!stage(call.cx->stage_a, a, lda, rows, cols, true, call.st, A) ||
      !stage(call.cx->stage_b, b, ldb, rows, cols, true, call.st, B) ||
      !stage(call.cx->stage_c, c, ldc, n, n, true, call.st, C))
    return call.fail();
  call.started();
  const bool up = uplo_code(uplo) == kUp;
  int rc = gemmtr_device<T>(*call.cx, up, ta, !ta, n, k, alpha, A.ptr, A.ld, B.ptr, B.ld, beta, C.ptr, C.ld,
                            call.st, call.sum);
  if (rc == EB2_OK || rc == EB2_ERR_ACCURACY) {
    const int rc2 = gemmtr_device<T>(*call.cx, up, ta, !ta, n, k, alpha, B.ptr, B.ld, A.ptr, A.ld, T(1), C.ptr, C.ld,
                                     call.st, call.sum);
    if (rc2 != EB2_OK) rc = rc2;
  }
  call.end(rc, A.staged || B.staged || C.staged, C, c, ldc, n, n);
}

// blas/level3_impl.h:507-592: C := alpha A B + beta C (left) or alpha B A + beta C (right)
template <typename T>
void blas_symm(char side, char uplo, int64_t m, int64_t n, T alpha, const T* a, int64_t lda, const T* b,
               int64_t ldb, T beta, T* c, int64_t ldc) {
  int info = symm_info(side, uplo, m, n, lda, ldb, ldc);
  if (info) return xerbla_(prefixed<T>("DSYMM ", "SSYMM "), &info, 6);
  if (m == 0 || n == 0) return;
  count_call(prefixed<T>("dsymm", "ssymm"));
  Call call(dtype_of<T>());
  if (!call.begin()) return;
  const bool left = side_code(side) == kLeft;
  const int64_t size = left ? m : n;
  const bool need_ab = alpha != T(0);
  Operand<T> A, B, C;
  if (!stage(call.cx->stage_a, a, lda, need_ab ? size : 0, size, true, call.st, A) ||
      !stage(call.cx->stage_b, b, ldb, need_ab ? m : 0, n, true, call.st, B) ||
      !stage(call.cx->stage_c, c, ldc, m, n, beta != T(0), call.st, C))
    return call.fail();
  call.started();
  const int rc = symm_device<T>(*call.cx, left, uplo_code(uplo) == kUp, m, n, alpha, A.ptr, A.ld, B.ptr, B.ld, beta,
                                C.ptr, C.ld, call.st, call.sum);
  call.end(rc, A.staged || B.staged || C.staged, C, c, ldc, m, n);
}

// blas/level3_impl.h:230-364 (solve) and :368-503 (multiply), in place on B
template <typename T>
void blas_trxm(bool solve, char side, char uplo, char op, char diag, int64_t m, int64_t n, T alpha, const T* a,
               int64_t lda, T* b, int64_t ldb) {
  int info = trxm_info(side, uplo, op, diag, m, n, lda, ldb);
  if (info)
    return xerbla_(solve ? prefixed<T>("DTRSM ", "STRSM ") : prefixed<T>("DTRMM ", "STRMM "), &info, 6);
  if (m == 0 || n == 0) return;
  count_call(solve ? prefixed<T>("dtrsm", "strsm") : prefixed<T>("dtrmm", "strmm"));
  Call call(dtype_of<T>());
  if (!call.begin()) return;
  const bool left = side_code(side) == kLeft;
  const int64_t size = left ? m : n;
  Operand<T> A, B;
  if (!stage(call.cx->stage_a, a, lda, size, size, true, call.st, A) ||
      !stage(call.cx->stage_b, b, ldb, m, n, true, call.st, B))
    return call.fail();
  call.started();
  const int rc = trxm_device<T>(*call.cx, solve, left, uplo_code(uplo) == kUp, op_code(op) != kNoTr,
                                diag_code(diag) == kUnit, m, n, alpha, A.ptr, A.ld, B.ptr, B.ld, call.st, call.sum);
  call.end(rc, A.staged || B.staged, B, b, ldb, m, n);
}

// blas/level3_impl.h:12-96 with Scalar = std::complex (blas/complex_double.cpp,
// blas/complex_single.cpp): C := alpha op(A) op(B) + beta C, op in {N, T, C = conjugate
// transpose}.  beta scales C first (0: zeros); k == 0 or alpha == 0 stops there
// (Eigen/src/Core/products/GeneralMatrixMatrix.h:129-130).
template <typename T>
void blas_complex_gemm(char opa, char opb, int64_t m, int64_t n, int64_t k, const T* alpha, const T* a, int64_t lda,
                       const T* b, int64_t ldb, const T* beta, T* c, int64_t ldc) {
  int info = 0;
  {
    const int oa = op_code(opa), ob = op_code(opb);
    if (oa == kInvalid) info = 1;
    else if (ob == kInvalid) info = 2;
    else if (m < 0) info = 3;
    else if (n < 0) info = 4;
    else if (k < 0) info = 5;
    else if (lda < imax1(oa == kNoTr ? m : k)) info = 8;
    else if (ldb < imax1(ob == kNoTr ? k : n)) info = 10;
    else if (ldc < imax1(m)) info = 13;
  }
  if (info) return xerbla_(prefixed<T>("ZGEMM ", "CGEMM "), &info, 6);
  if (m == 0 || n == 0) return;
  const T ar = alpha[0], ai = alpha[1], br = beta[0], bi = beta[1];
  const bool alpha_zero = ar == T(0) && ai == T(0);
  const bool beta_one = br == T(1) && bi == T(0), beta_zero = br == T(0) && bi == T(0);
  const bool need_ab = k > 0 && !alpha_zero;
  if (!need_ab && beta_one) return;
  count_call(prefixed<T>("zgemm", "cgemm"));
  Call call(dtype_of<T>() == 'd' ? 'z' : 'c');
  if (!call.begin()) return;
  const int oa = op_code(opa), ob = op_code(opb);
  const int64_t a_rows = oa == kNoTr ? m : k, a_cols = oa == kNoTr ? k : m;
  const int64_t b_rows = ob == kNoTr ? k : n, b_cols = ob == kNoTr ? n : k;
  // complex column-major = real column-major with twice the rows and leading dimension
  Operand<T> A, B, C;
  if (!stage(call.cx->stage_a, a, 2 * lda, need_ab ? 2 * a_rows : 0, a_cols, true, call.st, A) ||
      !stage(call.cx->stage_b, b, 2 * ldb, need_ab ? 2 * b_rows : 0, b_cols, true, call.st, B) ||
      !stage(call.cx->stage_c, c, 2 * ldc, 2 * m, n, !beta_zero, call.st, C))
    return call.fail();
  call.started();
  const int rc = complex_gemm_device<T>(*call.cx, oa, ob, m, n, k, ar, ai, A.ptr, A.ld / 2, B.ptr, B.ld / 2, br, bi,
                                        C.ptr, C.ld / 2, call.st, call.sum);
  call.end(rc, A.staged || B.staged || C.staged, C, c, 2 * ldc, 2 * m, n);
}

// blas/level3_impl.h:507-592 (symm, ISCOMPLEX: the symmetric matrix, no conjugation) and
// :760-831 (hemm: the Hermitian matrix, the diagonal's real part): C := alpha S B + beta C
// (left) or alpha B S + beta C (right).  beta scales C first (0: zeros).
template <typename T>
void blas_complex_symm(bool hermitian, char side, char uplo, int64_t m, int64_t n, const T* alpha, const T* a,
                       int64_t lda, const T* b, int64_t ldb, const T* beta, T* c, int64_t ldc) {
  int info = symm_info(side, uplo, m, n, lda, ldb, ldc);
  if (info)
    return xerbla_(hermitian ? prefixed<T>("ZHEMM ", "CHEMM ") : prefixed<T>("ZSYMM ", "CSYMM "), &info, 6);
  if (m == 0 || n == 0) return;
  count_call(hermitian ? prefixed<T>("zhemm", "chemm") : prefixed<T>("zsymm", "csymm"));
  Call call(dtype_of<T>() == 'd' ? 'z' : 'c');
  if (!call.begin()) return;
  const bool left = side_code(side) == kLeft;
  const int64_t size = left ? m : n;
  const bool need_ab = alpha[0] != T(0) || alpha[1] != T(0);
  const bool beta_zero = beta[0] == T(0) && beta[1] == T(0);
  Operand<T> A, B, C;
  if (!stage(call.cx->stage_a, a, 2 * lda, need_ab ? 2 * size : 0, size, true, call.st, A) ||
      !stage(call.cx->stage_b, b, 2 * ldb, need_ab ? 2 * m : 0, n, true, call.st, B) ||
      !stage(call.cx->stage_c, c, 2 * ldc, 2 * m, n, !beta_zero, call.st, C))
    return call.fail();
  call.started();
  const int rc = complex_symm_device<T>(*call.cx, hermitian, left, uplo_code(uplo) == kUp, m, n, alpha[0], alpha[1],
                                        A.ptr, A.ld / 2, B.ptr, B.ld / 2, beta[0], beta[1], C.ptr, C.ld / 2, call.st,
                                        call.sum);
  call.end(rc, A.staged || B.staged || C.staged, C, c, 2 * ldc, 2 * m, n);
}

// blas/level3_impl.h:230-364 (trsm) and :368-503 (trmm) with Scalar = std::complex; op 'C'
// is the conjugate transpose.
template <typename T>
void blas_complex_trxm(bool solve, char side, char uplo, char op, char diag, int64_t m, int64_t n, const T* alpha,
                       const T* a, int64_t lda, T* b, int64_t ldb) {
  int info = trxm_info(side, uplo, op, diag, m, n, lda, ldb);
  if (info)
    return xerbla_(solve ? prefixed<T>("ZTRSM ", "CTRSM ") : prefixed<T>("ZTRMM ", "CTRMM "), &info, 6);
  if (m == 0 || n == 0) return;
  count_call(solve ? prefixed<T>("ztrsm", "ctrsm") : prefixed<T>("ztrmm", "ctrmm"));
  Call call(dtype_of<T>() == 'd' ? 'z' : 'c');
  if (!call.begin()) return;
  const bool left = side_code(side) == kLeft;
  const int64_t size = left ? m : n;
  Operand<T> A, B;
  if (!stage(call.cx->stage_a, a, 2 * lda, 2 * size, size, true, call.st, A) ||
      !stage(call.cx->stage_b, b, 2 * ldb, 2 * m, n, true, call.st, B))
    return call.fail();
  call.started();
  const int rc = complex_trxm_device<T>(*call.cx, solve, left, uplo_code(uplo) == kUp, op_code(op),
                                        diag_code(diag) == kUnit, m, n, alpha[0], alpha[1], A.ptr, A.ld / 2, B.ptr,
                                        B.ld / 2, call.st, call.sum);
  call.end(rc, A.staged || B.staged, B, b, 2 * ldb, 2 * m, n);
}

}  // namespace
}  // namespace eb2

using eb2::blas_complex_gemm;
using eb2::blas_complex_symm;
using eb2::blas_complex_trxm;
using eb2::blas_gemmtr;
using eb2::blas_symm;
using eb2::blas_syr2k;
using eb2::blas_syrk;
using eb2::blas_trxm;

// The exported symbols: LP64 (int) and ILP64 (int64_t, _64_ suffix), as blas/level3_impl.h
// declares them through EIGEN_BLAS_FUNC (blas/common.h).
#define EB2_LEVEL3_SYMBOLS(I, SFX)                                                                                   \
  void dgemmtr##SFX(const char* uplo, const char* ta, const char* tb, const I* n, const I* k, const double* alpha,    \
                    const double* a, const I* lda, const double* b, const I* ldb, const double* beta, double* c,     \
                    const I* ldc) {                                                                                  \
    blas_gemmtr<double>(*uplo, *ta, *tb, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                          \
  }                                                                                                                  \
  void sgemmtr##SFX(const char* uplo, const char* ta, const char* tb, const I* n, const I* k, const float* alpha,     \
                    const float* a, const I* lda, const float* b, const I* ldb, const float* beta, float* c,         \
                    const I* ldc) {                                                                                  \
    blas_gemmtr<float>(*uplo, *ta, *tb, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                           \
  }                                                                                                                  \
  void dsyrk##SFX(const char* uplo, const char* op, const I* n, const I* k, const double* alpha, const double* a,    \
                  const I* lda, const double* beta, double* c, const I* ldc) {                                       \
    blas_syrk<double>(*uplo, *op, *n, *k, *alpha, a, *lda, *beta, c, *ldc);                                          \
  }                                                                                                                  \
  void ssyrk##SFX(const char* uplo, const char* op, const I* n, const I* k, const float* alpha, const float* a,      \
                  const I* lda, const float* beta, float* c, const I* ldc) {                                         \
    blas_syrk<float>(*uplo, *op, *n, *k, *alpha, a, *lda, *beta, c, *ldc);                                           \
  }                                                                                                                  \
  void dsyr2k##SFX(const char* uplo, const char* op, const I* n, const I* k, const double* alpha, const double* a,   \
                   const I* lda, const double* b, const I* ldb, const double* beta, double* c, const I* ldc) {       \
    blas_syr2k<double>(*uplo, *op, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                                \
  }                                                                                                                  \
  void ssyr2k##SFX(const char* uplo, const char* op, const I* n, const I* k, const float* alpha, const float* a,     \
                   const I* lda, const float* b, const I* ldb, const float* beta, float* c, const I* ldc) {          \
    blas_syr2k<float>(*uplo, *op, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                                 \
  }                                                                                                                  \
  void dsymm##SFX(const char* side, const char* uplo, const I* m, const I* n, const double* alpha, const double* a,  \
                  const I* lda, const double* b, const I* ldb, const double* beta, double* c, const I* ldc) {        \
    blas_symm<double>(*side, *uplo, *m, *n, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                               \
  }                                                                                                                  \
  void ssymm##SFX(const char* side, const char* uplo, const I* m, const I* n, const float* alpha, const float* a,    \
                  const I* lda, const float* b, const I* ldb, const float* beta, float* c, const I* ldc) {           \
    blas_symm<float>(*side, *uplo, *m, *n, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);                                \
  }                                                                                                                  \
  void dtrmm##SFX(const char* side, const char* uplo, const char* op, const char* diag, const I* m, const I* n,     \
                  const double* alpha, const double* a, const I* lda, double* b, const I* ldb) {                     \
    blas_trxm<double>(false, *side, *uplo, *op, *diag, *m, *n, *alpha, a, *lda, b, *ldb);                            \
  }                                                                                                                  \
  void strmm##SFX(const char* side, const char* uplo, const char* op, const char* diag, const I* m, const I* n,     \
                  const float* alpha, const float* a, const I* lda, float* b, const I* ldb) {                        \
    blas_trxm<float>(false, *side, *uplo, *op, *diag, *m, *n, *alpha, a, *lda, b, *ldb);                             \
  }                                                                                                                  \
  void dtrsm##SFX(const char* side, const char* uplo, const char* op, const char* diag, const I* m, const I* n,     \
                  const double* alpha, const double* a, const I* lda, double* b, const I* ldb) {                     \
    blas_trxm<double>(true, *side, *uplo, *op, *diag, *m, *n, *alpha, a, *lda, b, *ldb);                             \
  }                                                                                                                  \
  void strsm##SFX(const char* side, const char* uplo, const char* op, const char* diag, const I* m, const I* n,     \
                  const float* alpha, const float* a, const I* lda, float* b, const I* ldb) {                        \
    blas_trxm<float>(true, *side, *uplo, *op, *diag, *m, *n, *alpha, a, *lda, b, *ldb);                              \
  }

// Complex GEMM: alpha, beta and the matrices as interleaved (re, im) pairs of the real type,
// the prototypes of blas/blas.h:393-398.
#define EB2_COMPLEX_GEMM_SYMBOLS(I, SFX)                                                                             \
  void zgemm##SFX(const char* ta, const char* tb, const I* m, const I* n, const I* k, const double* alpha,          \
                  const double* a, const I* lda, const double* b, const I* ldb, const double* beta, double* c,       \
                  const I* ldc) {                                                                                    \
    blas_complex_gemm<double>(*ta, *tb, *m, *n, *k, alpha, a, *lda, b, *ldb, beta, c, *ldc);                         \
  }                                                                                                                  \
  void cgemm##SFX(const char* ta, const char* tb, const I* m, const I* n, const I* k, const float* alpha,           \
                  const float* a, const I* lda, const float* b, const I* ldb, const float* beta, float* c,           \
                  const I* ldc) {                                                                                    \
    blas_complex_gemm<float>(*ta, *tb, *m, *n, *k, alpha, a, *lda, b, *ldb, beta, c, *ldc);                          \
  }

// The complex level-3 routines Eigen's external-BLAS hooks bind (?trsm_, ?trmm_, ?hemm_) and
// ?symm_: alpha, beta and the matrices as interleaved (re, im) pairs of the real type.
#define EB2_COMPLEX_LEVEL3_SYMBOLS(I, SFX, P, R)                                                                     \
  void P##symm##SFX(const char* side, const char* uplo, const I* m, const I* n, const R* alpha, const R* a,         \
                    const I* lda, const R* b, const I* ldb, const R* beta, R* c, const I* ldc) {                     \
    blas_complex_symm<R>(false, *side, *uplo, *m, *n, alpha, a, *lda, b, *ldb, beta, c, *ldc);                       \
  }                                                                                                                  \
  void P##hemm##SFX(const char* side, const char* uplo, const I* m, const I* n, const R* alpha, const R* a,         \
                    const I* lda, const R* b, const I* ldb, const R* beta, R* c, const I* ldc) {                     \
    blas_complex_symm<R>(true, *side, *uplo, *m, *n, alpha, a, *lda, b, *ldb, beta, c, *ldc);                        \
  }                                                                                                                  \
  void P##trmm##SFX(const char* side, const char* uplo, const char* op, const char* diag, const I* m, const I* n,   \
                    const R* alpha, const R* a, const I* lda, R* b, const I* ldb) {                                  \
    blas_complex_trxm<R>(false, *side, *uplo, *op, *diag, *m, *n, alpha, a, *lda, b, *ldb);                          \
  }                                                                                                                  \
  void P##trsm##SFX(const char* side, const char* uplo, const char* op, const char* diag, const I* m, const I* n,   \
                    const R* alpha, const R* a, const I* lda, R* b, const I* ldb) {                                  \
    blas_complex_trxm<R>(true, *side, *uplo, *op, *diag, *m, *n, alpha, a, *lda, b, *ldb);                           \
  }

extern "C" {
EB2_LEVEL3_SYMBOLS(int, _)
EB2_LEVEL3_SYMBOLS(int64_t, _64_)
EB2_COMPLEX_GEMM_SYMBOLS(int, _)
EB2_COMPLEX_GEMM_SYMBOLS(int64_t, _64_)
EB2_COMPLEX_LEVEL3_SYMBOLS(int, _, z, double)
EB2_COMPLEX_LEVEL3_SYMBOLS(int64_t, _64_, z, double)
EB2_COMPLEX_LEVEL3_SYMBOLS(int, _, c, float)
EB2_COMPLEX_LEVEL3_SYMBOLS(int64_t, _64_, c, float)
}
