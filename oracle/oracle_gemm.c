/*
 * oracle_gemm.c -- CPU oracle for the dense matrix-matrix product path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the tests, the smoke
 * check and the CPU-baseline leg of the benchmark call it; the product library
 * (libeigen_b200.so) never links or calls it.
 *
 * It restates, in plain C, what Eigen's BLAS shim does for ?gemm_:
 *   blas/level3_impl.h:12-96   (argument checks, quick returns, beta pre-scale,
 *                               dispatch on op(A)/op(B))
 *   blas/common.h:60-61        (N/T/C parsing, case-insensitive; C == T for reals)
 *   Eigen/src/Core/products/GeneralMatrixMatrix.h:130
 *                              (alpha == 0: C is left as the beta pre-scale made it,
 *                               A and B are not read)
 *   Eigen/src/Core/products/GeneralBlockPanelKernel.h:1446-1455
 *                              (the GEBP store is C += alpha * (A*B))
 * The arithmetic is an unblocked triple loop; rounding differs from the
 * reference's blocked GEBP, so floating-point results agree within the
 * product error bound of test/product_test_helpers.h:44-90, not bitwise.
 *
 * It also holds the accuracy checkers used by the tests:
 *   - a double-double GEMM (TwoSum / TwoProd-by-FMA, Ogita, Rump & Oishi,
 *     "Accurate sum and dot product", SISC 2005), the "exact" reference for
 *     normwise errors of native and emulated DGEMM;
 *   - the netlib Level-3 test ratio, restating the check of DMMCH in
 *     blas/testing/dblat3.f:2510-2621 (|Ct - Cc| / (eps * gauge), gauge =
 *     |alpha| |op(A)||op(B)| + |beta| |C|);
 *   - || |op(A)| |op(B)| ||_F, accumulated in double with an explicit loop as in
 *     test/product_test_helpers.h:53-71;
 *   - the row/column digit split of the Ozaki scheme (Ozaki, Ogita, Oishi &
 *     Rump, Numer. Algorithms 2012), restated from the paper's definition so
 *     the device split can be checked bit for bit.
 * Parity status: pinned.  The tests check this file against Eigen's own
 * sgemm_/dgemm_ built from the reference sources (oracle/_ref) and against the
 * committed golden fixtures.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { OR_NOTR = 0, OR_TR = 1, OR_ADJ = 2, OR_INVALID = 0xff };

/* blas/common.h:60-61: 'N'/'n' -> no transpose, 'T'/'t' -> transpose,
 * 'C'/'c' -> adjoint (a transpose for real scalars), anything else invalid. */
static int op_code(char c) {
  if (c == 'N' || c == 'n') return OR_NOTR;
  if (c == 'T' || c == 't') return OR_TR;
  if (c == 'C' || c == 'c') return OR_ADJ;
  return OR_INVALID;
}

static long lmax(long a, long b) { return a > b ? a : b; }

/* blas/level3_impl.h:61-78: the first failing check sets info; 0 means valid. */
int oracle_gemm_info(char transa, char transb, long m, long n, long k, long lda, long ldb, long ldc) {
  int oa = op_code(transa), ob = op_code(transb);
  if (oa == OR_INVALID) return 1;
  if (ob == OR_INVALID) return 2;
  if (m < 0) return 3;
  if (n < 0) return 4;
  if (k < 0) return 5;
  if (lda < lmax(1, oa == OR_NOTR ? m : k)) return 8;
  if (ldb < lmax(1, ob == OR_NOTR ? k : n)) return 10;
  if (ldc < lmax(1, m)) return 13;
  return 0;
}

/* element (i,l) of op(A) for a column-major A with leading dimension lda */
#define OPA(i, l) (ta == OR_NOTR ? A[(size_t)(i) + (size_t)(l) * (size_t)lda] : A[(size_t)(l) + (size_t)(i) * (size_t)lda])
/* element (l,j) of op(B) */
#define OPB(l, j) (tb == OR_NOTR ? B[(size_t)(l) + (size_t)(j) * (size_t)ldb] : B[(size_t)(j) + (size_t)(l) * (size_t)ldb])

/* Full ?gemm_ semantics (blas/level3_impl.h:61-96 with GeneralMatrixMatrix.h:130).
 * Returns the info code; C is untouched when info != 0. */
int oracle_dgemm(char transa, char transb, long m, long n, long k, double alpha, const double* A, long lda,
                 const double* B, long ldb, double beta, double* C, long ldc) {
  int info = oracle_gemm_info(transa, transb, m, n, k, lda, ldb, ldc);
  if (info) return info;
  if (m == 0 || n == 0) return 0;
  int ta = op_code(transa) == OR_NOTR ? OR_NOTR : OR_TR;
  int tb = op_code(transb) == OR_NOTR ? OR_NOTR : OR_TR;
  if (beta != 1.0) {
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < m; ++i) {
        double* c = &C[(size_t)i + (size_t)j * (size_t)ldc];
        *c = (beta == 0.0) ? 0.0 : beta * *c; /* beta == 0 discards NaN/Inf in C */
      }
  }
  if (k == 0) return 0;
  if (alpha == 0.0) return 0; /* A and B are not read */
#pragma omp parallel for schedule(static)
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) {
      double acc = 0.0;
      for (long l = 0; l < k; ++l) acc += OPA(i, l) * OPB(l, j);
      C[(size_t)i + (size_t)j * (size_t)ldc] += alpha * acc;
    }
  return 0;
}

/* Same semantics for float.  The dot product is accumulated in double and the
 * update C += alpha*acc is rounded to float once, so this oracle is at least as
 * accurate as the reference's float GEBP. */
int oracle_sgemm(char transa, char transb, long m, long n, long k, float alpha, const float* A, long lda,
                 const float* B, long ldb, float beta, float* C, long ldc) {
  int info = oracle_gemm_info(transa, transb, m, n, k, lda, ldb, ldc);
  if (info) return info;
  if (m == 0 || n == 0) return 0;
  int ta = op_code(transa) == OR_NOTR ? OR_NOTR : OR_TR;
  int tb = op_code(transb) == OR_NOTR ? OR_NOTR : OR_TR;
  if (beta != 1.0f) {
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < m; ++i) {
        float* c = &C[(size_t)i + (size_t)j * (size_t)ldc];
        *c = (beta == 0.0f) ? 0.0f : beta * *c;
      }
  }
  if (k == 0) return 0;
  if (alpha == 0.0f) return 0;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) {
      double acc = 0.0;
      for (long l = 0; l < k; ++l) acc += (double)OPA(i, l) * (double)OPB(l, j);
      float* c = &C[(size_t)i + (size_t)j * (size_t)ldc];
      *c = (float)((double)*c + (double)alpha * acc);
    }
  return 0;
}

/* ---- double-double arithmetic (Ogita, Rump & Oishi 2005) ---- */
static inline void two_sum(double a, double b, double* s, double* e) {
  double x = a + b;
  double z = x - a;
  *e = (a - (x - z)) + (b - z);
  *s = x;
}
static inline void two_prod(double a, double b, double* p, double* e) {
  double x = a * b;
  *e = fma(a, b, -x);
  *p = x;
}
/* (hi,lo) += a*b, keeping a normalised double-double */
static inline void dd_fma(double* hi, double* lo, double a, double b) {
  double p, pe, s, se;
  two_prod(a, b, &p, &pe);
  two_sum(*hi, p, &s, &se);
  se += *lo + pe;
  two_sum(s, se, hi, lo);
}

/* Double-double evaluation of alpha*op(A)op(B) + beta*C on the sub-block given
 * by row indices rows[0..nr) and column indices cols[0..nc) of C.  Inputs are
 * doubles; out_hi/out_lo are nr x nc column-major.  C is read (beta != 0) but
 * not written.  rows/cols may be NULL for the identity selection. */
void oracle_dgemm_dd(char transa, char transb, long m, long n, long k, double alpha, const double* A, long lda,
                     const double* B, long ldb, double beta, const double* C, long ldc, const long* rows, long nr,
                     const long* cols, long nc, double* out_hi, double* out_lo) {
  (void)m;
  (void)n;
  int ta = op_code(transa) == OR_NOTR ? OR_NOTR : OR_TR;
  int tb = op_code(transb) == OR_NOTR ? OR_NOTR : OR_TR;
#pragma omp parallel for schedule(dynamic, 1)
  for (long jj = 0; jj < nc; ++jj) {
    long j = cols ? cols[jj] : jj;
    for (long ii = 0; ii < nr; ++ii) {
      long i = rows ? rows[ii] : ii;
      double hi = 0.0, lo = 0.0;
      for (long l = 0; l < k; ++l) dd_fma(&hi, &lo, OPA(i, l), OPB(l, j));
      /* alpha * (hi + lo) in double-double */
      double p, pe, q, qe;
      two_prod(alpha, hi, &p, &pe);
      pe += alpha * lo;
      two_sum(p, pe, &p, &q);
      (void)qe;
      hi = p;
      lo = q;
      if (beta != 0.0 && C) dd_fma(&hi, &lo, beta, C[(size_t)i + (size_t)j * (size_t)ldc]);
      out_hi[(size_t)ii + (size_t)jj * (size_t)nr] = hi;
      out_lo[(size_t)ii + (size_t)jj * (size_t)nr] = lo;
    }
  }
}

/* || |op(A)| |op(B)| ||_F over the selected block, accumulated in double
 * (test/product_test_helpers.h:53-71 computes the same quantity). */
double oracle_abs_product_fro(char transa, char transb, long k, const double* A, long lda, const double* B, long ldb,
                              const long* rows, long nr, const long* cols, long nc) {
  int ta = op_code(transa) == OR_NOTR ? OR_NOTR : OR_TR;
  int tb = op_code(transb) == OR_NOTR ? OR_NOTR : OR_TR;
  double total = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
  for (long jj = 0; jj < nc; ++jj) {
    long j = cols ? cols[jj] : jj;
    for (long ii = 0; ii < nr; ++ii) {
      long i = rows ? rows[ii] : ii;
      double s = 0.0;
      for (long l = 0; l < k; ++l) s += fabs(OPA(i, l)) * fabs(OPB(l, j));
      total += s * s;
    }
  }
  return sqrt(total);
}

/* Netlib Level-3 test ratio, restating DMMCH (blas/testing/dblat3.f:2510-2621):
 * for each entry, |Ct - Cc| / eps, divided by the gauge
 * |alpha| sum|a||b| + |beta| |C_in| when that is nonzero; the maximum over all
 * entries is returned.  A ratio below the tester's threshold (16.0 in
 * blas/testing/dblat3.dat) passes.  Ct is evaluated in double-double here, so
 * the ratio measures only the tested result's error.  C_in is C before the
 * call, C_out the tested result. */
double oracle_dgemm_test_ratio(char transa, char transb, long m, long n, long k, double alpha, const double* A, long lda,
                               const double* B, long ldb, double beta, const double* C_in, long ldc,
                               const double* C_out, long ldcc, double eps) {
  int ta = op_code(transa) == OR_NOTR ? OR_NOTR : OR_TR;
  int tb = op_code(transb) == OR_NOTR ? OR_NOTR : OR_TR;
  double err = 0.0;
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) {
      double hi = 0.0, lo = 0.0, g = 0.0;
      for (long l = 0; l < k; ++l) {
        dd_fma(&hi, &lo, OPA(i, l), OPB(l, j));
        g += fabs(OPA(i, l)) * fabs(OPB(l, j));
      }
      double ct = alpha * (hi + lo) + beta * C_in[(size_t)i + (size_t)j * (size_t)ldc];
      g = fabs(alpha) * g + fabs(beta) * fabs(C_in[(size_t)i + (size_t)j * (size_t)ldc]);
      double e = fabs(ct - C_out[(size_t)i + (size_t)j * (size_t)ldcc]) / eps;
      if (g != 0.0) e /= g;
      if (e != e) return INFINITY; /* NaN in the tested result fails */
      if (e > err) err = e;
    }
  return err;
}

/* Float variant of the test ratio (sblat3.f's SMMCH has the same structure);
 * the expected value is evaluated in double-double from the float inputs. */
double oracle_sgemm_test_ratio(char transa, char transb, long m, long n, long k, float alpha, const float* A, long lda,
                               const float* B, long ldb, float beta, const float* C_in, long ldc, const float* C_out,
                               long ldcc, double eps) {
  int ta = op_code(transa) == OR_NOTR ? OR_NOTR : OR_TR;
  int tb = op_code(transb) == OR_NOTR ? OR_NOTR : OR_TR;
  double err = 0.0;
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) {
      double hi = 0.0, lo = 0.0, g = 0.0;
      for (long l = 0; l < k; ++l) {
        dd_fma(&hi, &lo, (double)OPA(i, l), (double)OPB(l, j));
        g += fabs((double)OPA(i, l)) * fabs((double)OPB(l, j));
      }
      double cin = (double)C_in[(size_t)i + (size_t)j * (size_t)ldc];
      double ct = (double)alpha * (hi + lo) + (double)beta * cin;
      g = fabs((double)alpha) * g + fabs((double)beta) * fabs(cin);
      double e = fabs(ct - (double)C_out[(size_t)i + (size_t)j * (size_t)ldcc]) / eps;
      if (g != 0.0) e /= g;
      if (e != e) return INFINITY;
      if (e > err) err = e;
    }
  return err;
}

/* ---- Ozaki digit split (Ozaki, Ogita, Oishi & Rump 2012), restated ----
 *
 * Row r of a matrix X (element (r,l) at X[r*sr + l*sl]) is scaled by 2^-e_r,
 * where e_r is the binary exponent of max_l |x_rl| (frexp convention: the
 * maximum lies in [2^(e_r-1), 2^e_r)), so every scaled element lies in (-1,1).
 * The scaled value is then written as balanced base-2^7 digits:
 *     x_rl * 2^-e_r  =  sum_{p=1..s} d_p * 2^(-6 - 7(p-1))  + remainder,
 * d_1 = rint(x' 2^6), each following digit the rint of the previous remainder
 * times 2^7, so |d_p| <= 64 and |remainder| <= 2^(-7s).  Every step is exact in
 * binary64.  digits has layout [s][rows][ld_out] (row r contiguous along l),
 * exps[r] = e_r.  A row that holds a non-finite value gets all-zero digits and
 * exps[r] = INT32_MIN (the device path treats that row with IEEE arithmetic
 * instead).  A zero row gets e_r = 0 and zero digits. */
void oracle_ozaki_split(const double* X, long rows, long cols, long sr, long sl, int s, int8_t* digits,
                        long rows_out, long ld_out, int32_t* exps) {
  for (long r = 0; r < rows; ++r) {
    double mx = 0.0;
    int finite = 1;
    for (long l = 0; l < cols; ++l) {
      double v = X[(size_t)r * (size_t)sr + (size_t)l * (size_t)sl];
      if (!isfinite(v)) finite = 0;
      double a = fabs(v);
      if (a > mx) mx = a;
    }
    int e = 0;
    if (finite && mx > 0.0) frexp(mx, &e);
    exps[r] = finite ? e : INT32_MIN;
    for (long l = 0; l < cols; ++l) {
      double x = finite ? ldexp(X[(size_t)r * (size_t)sr + (size_t)l * (size_t)sl], -e) : 0.0;
      double rem = x * 64.0;
      for (int p = 0; p < s; ++p) {
        double d = rint(rem);
        digits[((size_t)p * (size_t)rows_out + (size_t)r) * (size_t)ld_out + (size_t)l] = (int8_t)d;
        rem = (rem - d) * 128.0;
      }
    }
  }
}

/* Model of the device's emulated DGEMM, operation for operation, so the device
 * result can be checked bit for bit (integer digit products are exact; the FP64
 * recombination is replayed in the device epilogue's order):
 *   digits of op(A) rows and op(B) columns as in oracle_ozaki_split;
 *   D_t = sum_{p+q=t, 1<=p,q<=s} Dp_A Dq_B^T  (exact, int64 here);
 *   acc = 0; for t = s+1 down to 2:  acc = acc + double(D_t) * 2^(e_i + f_j - 12 - 7(t-2));
 *   v = alpha * acc;  C = (beta == 0) ? v : fma(beta, C, v).
 * Rows/columns with a non-finite entry are left to the caller (the device falls back
 * to IEEE FP64 there).  Work arrays are allocated here; sizes are small in tests. */
#include <stdlib.h>
int oracle_ozaki_dgemm(char transa, char transb, long m, long n, long k, double alpha, const double* A, long lda,
                       const double* B, long ldb, double beta, double* C, long ldc, int s) {
  int ta = op_code(transa) == OR_NOTR ? OR_NOTR : OR_TR;
  int tb = op_code(transb) == OR_NOTR ? OR_NOTR : OR_TR;
  if (m == 0 || n == 0) return 0;
  int8_t* da = (int8_t*)calloc((size_t)s * (size_t)m * (size_t)(k ? k : 1), 1);
  int8_t* db = (int8_t*)calloc((size_t)s * (size_t)n * (size_t)(k ? k : 1), 1);
  int32_t* ea = (int32_t*)calloc((size_t)m, sizeof(int32_t));
  int32_t* eb = (int32_t*)calloc((size_t)n, sizeof(int32_t));
  if (!da || !db || !ea || !eb) {
    free(da);
    free(db);
    free(ea);
    free(eb);
    return -1;
  }
  /* op(A): row i, column l at A[i + l*lda] (N) or A[l + i*lda] (T) */
  oracle_ozaki_split(A, m, k, ta == OR_NOTR ? 1 : lda, ta == OR_NOTR ? lda : 1, s, da, m, k, ea);
  /* op(B)^T: row j, column l at B[l + j*ldb] (N) or B[j + l*ldb] (T) */
  oracle_ozaki_split(B, n, k, tb == OR_NOTR ? ldb : 1, tb == OR_NOTR ? 1 : ldb, s, db, n, k, eb);
#pragma omp parallel for schedule(dynamic, 1)
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) {
      double* c = &C[(size_t)i + (size_t)j * (size_t)ldc];
      if (ea[i] == INT32_MIN || eb[j] == INT32_MIN) continue;
      double acc = 0.0;
      for (int t = s + 1; t >= 2; --t) {
        long long D = 0;
        for (int p = (t - s > 1 ? t - s : 1); p <= (s < t - 1 ? s : t - 1); ++p) {
          const int8_t* ra = da + ((size_t)(p - 1) * (size_t)m + (size_t)i) * (size_t)k;
          const int8_t* rb = db + ((size_t)(t - p - 1) * (size_t)n + (size_t)j) * (size_t)k;
          for (long l = 0; l < k; ++l) D += (long long)ra[l] * (long long)rb[l];
        }
        acc = acc + (double)D * ldexp(1.0, ea[i] + eb[j] - 12 - 7 * (t - 2));
      }
      const double v = alpha * acc;
      *c = (beta == 0.0) ? v : fma(beta, *c, v);
    }
  free(da);
  free(db);
  free(ea);
  free(eb);
  return 0;
}
