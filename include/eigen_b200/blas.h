/*
 * eigen_b200/blas.h -- C ABI of libeigen_b200.so, a B200 (sm_100a) drop-in for
 * Eigen's dense matrix-matrix product path.
 *
 * The Fortran-convention symbols below are the ones Eigen binds for its product
 * when compiled with EIGEN_USE_BLAS, and the ones Eigen's own BLAS library
 * exports, so this library serves both:
 *   - Eigen's Matrix operator* (Eigen/src/Core/products/GeneralMatrixMatrix_BLAS.h:53-118
 *     calls EIGEN_BLAS_SYM(dgemm)/EIGEN_BLAS_SYM(sgemm) with beta = 1);
 *   - any C/Fortran caller of ?gemm_ (blas/level3_impl.h:12-96, declared in
 *     blas/blas.h:384-388 and Eigen/src/misc/blas.h:61-66).
 * All matrices are column-major.  Pointers may be host memory (pageable or
 * pinned: the library stages them through device memory) or device/managed
 * memory (used in place).  The calls are synchronous like any BLAS: C is final
 * when they return.
 */
#ifndef EIGEN_B200_BLAS_H
#define EIGEN_B200_BLAS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- BLAS ABI */

/* C := alpha*op(A)*op(B) + beta*C, op(X) in {X, X^T, X^H} chosen by 'N'/'T'/'C'
 * (case-insensitive).  Replaces Eigen's dgemm_ (blas/level3_impl.h:12-96, instantiated
 * by blas/double.cpp:12-21).  Argument errors call xerbla_("DGEMM ", &info, 6) with
 * info 1,2,3,4,5,8,10,13 exactly as blas/level3_impl.h:61-78; m == 0 or n == 0
 * returns without touching C; beta == 0 sets C to exact zeros; alpha == 0 or k == 0
 * leaves beta*C and does not read A or B (Eigen/src/Core/products/GeneralMatrixMatrix.h:130). */
void dgemm_(const char* transa, const char* transb, const int* m, const int* n, const int* k, const double* alpha,
            const double* a, const int* lda, const double* b, const int* ldb, const double* beta, double* c,
            const int* ldc);

/* Single precision; replaces Eigen's sgemm_ (blas/level3_impl.h:12-96 via blas/single.cpp:11-20). */
void sgemm_(const char* transa, const char* transb, const int* m, const int* n, const int* k, const float* alpha,
            const float* a, const int* lda, const float* b, const int* ldb, const float* beta, float* c,
            const int* ldc);

/* 64-bit-integer (ILP64) variants: the symbols Eigen binds with EIGEN_64BIT_BLAS and
 * EIGEN_BLAS_SYMBOL_SUFFIX=_64 (Eigen/src/Core/util/MKL_support.h:118-147). */
void dgemm_64_(const char* transa, const char* transb, const int64_t* m, const int64_t* n, const int64_t* k,
               const double* alpha, const double* a, const int64_t* lda, const double* b, const int64_t* ldb,
               const double* beta, double* c, const int64_t* ldc);
void sgemm_64_(const char* transa, const char* transb, const int64_t* m, const int64_t* n, const int64_t* k,
               const float* alpha, const float* a, const int64_t* lda, const float* b, const int64_t* ldb,
               const float* beta, float* c, const int64_t* ldc);

/* ------------------------------------------------ the other level-3 routines
 * Eigen's BLAS library exports these beside ?gemm_ (blas/level3_impl.h, instantiated by
 * blas/double.cpp and blas/single.cpp); each replaces the routine of the same name, with
 * its argument checks (xerbla_ name and info codes), quick returns and beta/alpha rules.
 * Every product inside goes through the device GEMM above (DGEMM sub-products take the
 * method and accuracy settings of dgemm_); pointers may be host or device memory.  LP64
 * symbols take int, the _64_ symbols int64_t. */

/* Triangle `uplo` of the n x n C := alpha*op(A)*op(B) + beta*C, the other triangle untouched.
 * blas/level3_impl.h:98-228; info 1,2,3,4,5,8,10,13 to xerbla_("?GEMMTR", info, 7);
 * n == 0 returns; beta scales the triangle (beta == 0: zeros) before k == 0 returns. */
void dgemmtr_(const char* uplo, const char* transa, const char* transb, const int* n, const int* k,
              const double* alpha, const double* a, const int* lda, const double* b, const int* ldb,
              const double* beta, double* c, const int* ldc);
void sgemmtr_(const char* uplo, const char* transa, const char* transb, const int* n, const int* k,
              const float* alpha, const float* a, const int* lda, const float* b, const int* ldb, const float* beta,
              float* c, const int* ldc);
/* Triangle `uplo` of C := alpha*A*A^T + beta*C ('N') or alpha*A^T*A + beta*C ('T'/'C').
 * blas/level3_impl.h:596-689; info 1,2,3,4,7,10 to xerbla_("?SYRK ", info, 6). */
void dsyrk_(const char* uplo, const char* trans, const int* n, const int* k, const double* alpha, const double* a,
            const int* lda, const double* beta, double* c, const int* ldc);
void ssyrk_(const char* uplo, const char* trans, const int* n, const int* k, const float* alpha, const float* a,
            const int* lda, const float* beta, float* c, const int* ldc);
/* Triangle `uplo` of C := alpha*(A*B^T + B*A^T) + beta*C ('N'), transposed forms for 'T'/'C'.
 * blas/level3_impl.h:693-754; info 1,2,3,4,7,9,12 to xerbla_("?SYR2K", info, 6). */
void dsyr2k_(const char* uplo, const char* trans, const int* n, const int* k, const double* alpha, const double* a,
             const int* lda, const double* b, const int* ldb, const double* beta, double* c, const int* ldc);
void ssyr2k_(const char* uplo, const char* trans, const int* n, const int* k, const float* alpha, const float* a,
             const int* lda, const float* b, const int* ldb, const float* beta, float* c, const int* ldc);
/* C := alpha*A*B + beta*C ('L') or alpha*B*A + beta*C ('R'), A symmetric, triangle `uplo` read.
 * blas/level3_impl.h:507-592; info 1,2,3,4,7,9,12 to xerbla_("?SYMM ", info, 6). */
void dsymm_(const char* side, const char* uplo, const int* m, const int* n, const double* alpha, const double* a,
            const int* lda, const double* b, const int* ldb, const double* beta, double* c, const int* ldc);
void ssymm_(const char* side, const char* uplo, const int* m, const int* n, const float* alpha, const float* a,
            const int* lda, const float* b, const int* ldb, const float* beta, float* c, const int* ldc);
/* B := alpha*op(A)*B ('L') or alpha*B*op(A) ('R'), A triangular ('U'/'L'; diag 'N'/'U').
 * blas/level3_impl.h:368-503; info 1,2,3,4,5,6,9,11 to xerbla_("?TRMM ", info, 6). */
void dtrmm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const double* alpha, const double* a, const int* lda, double* b, const int* ldb);
void strmm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const float* alpha, const float* a, const int* lda, float* b, const int* ldb);
/* B := alpha*op(A)^-1*B ('L') or alpha*B*op(A)^-1 ('R'): the solve, then B *= alpha.
 * blas/level3_impl.h:230-364; info 1,2,3,4,5,6,9,11 to xerbla_("?TRSM ", info, 6). */
void dtrsm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const double* alpha, const double* a, const int* lda, double* b, const int* ldb);
void strsm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const float* alpha, const float* a, const int* lda, float* b, const int* ldb);

/* Complex C := alpha*op(A)*op(B) + beta*C, op 'N', 'T' or 'C' (conjugate transpose); alpha,
 * beta and the matrices hold interleaved (re, im) pairs.  Replaces Eigen's zgemm_/cgemm_
 * (blas/level3_impl.h:12-96 instantiated by blas/complex_double.cpp / complex_single.cpp;
 * prototypes blas/blas.h:393-398), which Eigen's operator* on complex matrices binds
 * (GeneralMatrixMatrix_BLAS.h:116-117).  Same info codes as ?gemm_ to xerbla_("ZGEMM ", ..)
 * / ("CGEMM ", ..); beta scales C first (0: zeros); k == 0 or alpha == 0 then returns. */
void zgemm_(const char* transa, const char* transb, const int* m, const int* n, const int* k, const double* alpha,
            const double* a, const int* lda, const double* b, const int* ldb, const double* beta, double* c,
            const int* ldc);
void cgemm_(const char* transa, const char* transb, const int* m, const int* n, const int* k, const float* alpha,
            const float* a, const int* lda, const float* b, const int* ldb, const float* beta, float* c,
            const int* ldc);
void zgemm_64_(const char* transa, const char* transb, const int64_t* m, const int64_t* n, const int64_t* k,
               const double* alpha, const double* a, const int64_t* lda, const double* b, const int64_t* ldb,
               const double* beta, double* c, const int64_t* ldc);
void cgemm_64_(const char* transa, const char* transb, const int64_t* m, const int64_t* n, const int64_t* k,
               const float* alpha, const float* a, const int64_t* lda, const float* b, const int64_t* ldb,
               const float* beta, float* c, const int64_t* ldc);

/* Complex level-3 routines (Eigen binds ?trsm_, ?trmm_ and ?hemm_ for complex operands under
 * EIGEN_USE_BLAS: TriangularSolverMatrix_BLAS.h, TriangularMatrixMatrix_BLAS.h,
 * SelfadjointMatrixMatrix_BLAS.h).  alpha, beta and the matrices hold interleaved (re, im)
 * pairs; op 'C' is the conjugate transpose.  Replace blas/level3_impl.h's trsm (:230-364),
 * trmm (:368-503), symm (:507-592) and hemm (:760-831) for std::complex, with their info codes
 * and xerbla_ names ("ZTRSM ", "CHEMM ", ...); hemm takes the real part of A's diagonal. */
void ztrsm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const double* alpha, const double* a, const int* lda, double* b, const int* ldb);
void ctrsm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const float* alpha, const float* a, const int* lda, float* b, const int* ldb);
void ztrmm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const double* alpha, const double* a, const int* lda, double* b, const int* ldb);
void ctrmm_(const char* side, const char* uplo, const char* transa, const char* diag, const int* m, const int* n,
            const float* alpha, const float* a, const int* lda, float* b, const int* ldb);
void zhemm_(const char* side, const char* uplo, const int* m, const int* n, const double* alpha, const double* a,
            const int* lda, const double* b, const int* ldb, const double* beta, double* c, const int* ldc);
void chemm_(const char* side, const char* uplo, const int* m, const int* n, const float* alpha, const float* a,
            const int* lda, const float* b, const int* ldb, const float* beta, float* c, const int* ldc);
void zsymm_(const char* side, const char* uplo, const int* m, const int* n, const double* alpha, const double* a,
            const int* lda, const double* b, const int* ldb, const double* beta, double* c, const int* ldc);
void csymm_(const char* side, const char* uplo, const int* m, const int* n, const float* alpha, const float* a,
            const int* lda, const float* b, const int* ldb, const float* beta, float* c, const int* ldc);
void ztrsm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const double* alpha, const double* a, const int64_t* lda, double* b,
               const int64_t* ldb);
void ctrsm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const float* alpha, const float* a, const int64_t* lda, float* b,
               const int64_t* ldb);
void ztrmm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const double* alpha, const double* a, const int64_t* lda, double* b,
               const int64_t* ldb);
void ctrmm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const float* alpha, const float* a, const int64_t* lda, float* b,
               const int64_t* ldb);
void zhemm_64_(const char* side, const char* uplo, const int64_t* m, const int64_t* n, const double* alpha,
               const double* a, const int64_t* lda, const double* b, const int64_t* ldb, const double* beta,
               double* c, const int64_t* ldc);
void chemm_64_(const char* side, const char* uplo, const int64_t* m, const int64_t* n, const float* alpha,
               const float* a, const int64_t* lda, const float* b, const int64_t* ldb, const float* beta, float* c,
               const int64_t* ldc);
void zsymm_64_(const char* side, const char* uplo, const int64_t* m, const int64_t* n, const double* alpha,
               const double* a, const int64_t* lda, const double* b, const int64_t* ldb, const double* beta,
               double* c, const int64_t* ldc);
void csymm_64_(const char* side, const char* uplo, const int64_t* m, const int64_t* n, const float* alpha,
               const float* a, const int64_t* lda, const float* b, const int64_t* ldb, const float* beta, float* c,
               const int64_t* ldc);

void dgemmtr_64_(const char* uplo, const char* transa, const char* transb, const int64_t* n, const int64_t* k,
                 const double* alpha, const double* a, const int64_t* lda, const double* b, const int64_t* ldb,
                 const double* beta, double* c, const int64_t* ldc);
void sgemmtr_64_(const char* uplo, const char* transa, const char* transb, const int64_t* n, const int64_t* k,
                 const float* alpha, const float* a, const int64_t* lda, const float* b, const int64_t* ldb,
                 const float* beta, float* c, const int64_t* ldc);
void dsyrk_64_(const char* uplo, const char* trans, const int64_t* n, const int64_t* k, const double* alpha,
               const double* a, const int64_t* lda, const double* beta, double* c, const int64_t* ldc);
void ssyrk_64_(const char* uplo, const char* trans, const int64_t* n, const int64_t* k, const float* alpha,
               const float* a, const int64_t* lda, const float* beta, float* c, const int64_t* ldc);
void dsyr2k_64_(const char* uplo, const char* trans, const int64_t* n, const int64_t* k, const double* alpha,
                const double* a, const int64_t* lda, const double* b, const int64_t* ldb, const double* beta,
                double* c, const int64_t* ldc);
void ssyr2k_64_(const char* uplo, const char* trans, const int64_t* n, const int64_t* k, const float* alpha,
                const float* a, const int64_t* lda, const float* b, const int64_t* ldb, const float* beta, float* c,
                const int64_t* ldc);
void dsymm_64_(const char* side, const char* uplo, const int64_t* m, const int64_t* n, const double* alpha,
               const double* a, const int64_t* lda, const double* b, const int64_t* ldb, const double* beta,
               double* c, const int64_t* ldc);
void ssymm_64_(const char* side, const char* uplo, const int64_t* m, const int64_t* n, const float* alpha,
               const float* a, const int64_t* lda, const float* b, const int64_t* ldb, const float* beta, float* c,
               const int64_t* ldc);
void dtrmm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const double* alpha, const double* a, const int64_t* lda, double* b,
               const int64_t* ldb);
void strmm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const float* alpha, const float* a, const int64_t* lda, float* b,
               const int64_t* ldb);
void dtrsm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const double* alpha, const double* a, const int64_t* lda, double* b,
               const int64_t* ldb);
void strsm_64_(const char* side, const char* uplo, const char* transa, const char* diag, const int64_t* m,
               const int64_t* n, const float* alpha, const float* a, const int64_t* lda, float* b,
               const int64_t* ldb);

/* Argument-error hook, weak like blas/xerbla.cpp:18-20: prints
 * "Eigen BLAS ERROR #<info>: <name>" unless the program defines its own. */
void xerbla_(const char* name, int* info, size_t len);

/* ---------------------------------------------------------------- extensions */

/* Status codes of the eb2_* calls and of eb2_last_error(). */
enum {
  EB2_OK = 0,
  EB2_ERR_CUDA = -1,      /* a CUDA runtime call failed (message in eb2_last_error_string) */
  EB2_ERR_ALLOC = -2,     /* device or pinned memory could not be allocated */
  EB2_ERR_TIMEOUT = -3,   /* a kernel's bounded wait ran out; results are invalid */
  EB2_ERR_ARG = -4,       /* invalid argument to an eb2_* call (BLAS calls use xerbla_) */
  EB2_ERR_NO_DEVICE = -5, /* no CUDA device, or not an sm_100 device */
  EB2_ERR_ACCURACY = -6   /* the emulated product missed its accuracy target at the maximum slice count */
};

/* Method used for DGEMM / SGEMM. */
enum {
  EB2_METHOD_AUTO = 0,     /* DGEMM: Ozaki INT8 emulation; SGEMM: split-BF16 on tcgen05 */
  EB2_METHOD_NATIVE = 1,   /* DGEMM: FP64 DMMA kernel; SGEMM: FP32 FFMA kernel */
  EB2_METHOD_EMULATED = 2, /* DGEMM: Ozaki digit slices (scheme I); SGEMM: split-BF16 */
  EB2_METHOD_CRT = 3       /* DGEMM: Ozaki scheme II, INT8 products modulo coprime moduli
                              recombined by the Chinese remainder theorem */
};

int eb2_set_dgemm_method(int method);
int eb2_set_sgemm_method(int method);
/* Digit slices per operand for the emulated DGEMM (2..12); 0 = chosen per call. */
int eb2_set_dgemm_slices(int slices);
/* Moduli of the CRT-form emulated DGEMM (8..20; 0 = default 16).  With N moduli every
 * row of op(A) and column of op(B) keeps about b bits relative to its 2-norm, b = 62 for
 * 16, 69 for 18, 77 for 20; the a-posteriori check adds two moduli at a time. */
int eb2_set_dgemm_moduli(int moduli);
/* Accuracy target of the emulated DGEMM: the a-posteriori estimate of
 * ||C - C_exact||_F / ||alpha*op(A)op(B)||_F must not exceed it (default 2^-53);
 * slices are added one at a time until it holds or 12 are used. */
int eb2_set_dgemm_tolerance(double tol);
/* BF16 pieces per FP32 operand for the emulated SGEMM: 2 keeps the three products
 * hi*hi + hi*mid + mid*hi ("bf16x3"), 3 adds mid*mid + hi*lo + lo*hi ("bf16x6", default). */
int eb2_set_sgemm_pieces(int pieces);
/* Tile configuration of the tcgen05 kernels: 128 or 256 (one CTA per 128 x 128 or
 * 128 x 256 tile), 512 (a CTA pair per 256 x 256 tile), 1024 (one CTA per 256 x 256 tile,
 * CRT DGEMM only: two M = 128 MMAs per K step share the B tile) or 0 (= chosen per call). */
int eb2_set_tile_n(int tile_n);

/* Launch-shape knobs of the tcgen05 kernels (normally set by the tuner): row-tiles per
 * raster group (0 = column-major tile order) and the L2 prefetch distance in K blocks
 * (0 = off). */
int eb2_set_slice_tuning(int group_m, int prefetch);

/* Wall-time bound, in nanoseconds, of each pipeline wait inside the tcgen05 GEMM kernels
 * (0 = the default, 2 s).  No counterpart in the reference: a kernel whose wait runs out
 * stops issuing work, lets the copies and MMAs already in flight finish, releases its tensor
 * memory and returns; the call then reports EB2_ERR_TIMEOUT and C is invalid.  The device
 * stays usable.  Values below 1 ms are meant for testing that path.  Process-wide. */
int eb2_set_wait_limit_ns(long long ns);

/* Sticky last error of this thread (EB2_OK if none) and its message. */
int eb2_last_error(void);
const char* eb2_last_error_string(void);
void eb2_clear_error(void);

/* Details of the last product computed by this thread. */
typedef struct eb2_call_info {
  int dtype;          /* 'd' or 's' */
  int method;         /* EB2_METHOD_NATIVE, EB2_METHOD_EMULATED or EB2_METHOD_CRT */
  int slices;         /* digit slices or moduli (DGEMM emulated), BF16 products (SGEMM emulated) */
  int tile_n;         /* tcgen05 tile configuration, 0 for native kernels */
  int escalations;    /* slices (or pairs of moduli) added by the a-posteriori check */
  int nonfinite;      /* 1 if NaN/Inf inputs sent the call to the native kernel */
  int staged;         /* 1 if host buffers were staged through device memory */
  double err_estimate; /* a-posteriori relative error estimate (emulated DGEMM), else -1 */
  double kernel_ms;   /* device time of all product kernels (ms), -1 if not measured */
  double gemm_kernel_ms; /* device time of the main GEMM kernel alone (ms), -1 if not measured */
  int launches;       /* kernels this library launched for the call */
  double spread;      /* emulated DGEMM: mean (largest - mean) binary exponent of 64-entry
                         row chunks of op(A) and op(B)^T, the picker's data feature; else 0 */
} eb2_call_info;
int eb2_last_call_info(eb2_call_info* out);
/* The configuration class of this thread's last product (see eb2_set_config; -1 if none) and,
 * for a CRT DGEMM, its K splits per output tile and modulus (1: no split).  A separate call,
 * so that eb2_call_info keeps its layout for programs built against it. */
int eb2_last_call_config(int* config, int* splits);

/* How many calls of the named BLAS routine ("dgemm", "zgemm", "dtrsm", "ssyrk", ...: lower
 * case, no underscore) reached the device in this process: every call past its argument
 * checks and quick returns.  -1 for a name this library does not export.  No counterpart in
 * the reference; it lets a caller see which routines an Eigen build routed here. */
long long eb2_routine_calls(const char* name);

/* Record CUDA events around every product (1) or not (0, default for the
 * eb2_*_device calls; the BLAS entry points always time).  The times appear in
 * eb2_last_call_info (which waits for the events) until the next call on the device. */
int eb2_set_timing(int on);

/* Stream-ordered product on device pointers; no host synchronisation unless the
 * a-posteriori check of the emulated DGEMM needs one (check_accuracy != 0).
 * `stream` is a cudaStream_t (NULL = the legacy default stream).  Returns EB2_*.
 * Both can be captured into a CUDA graph once a direct call of the same size has sized the
 * workspace; a captured call that would need a larger workspace returns EB2_ERR_ARG without
 * enqueueing anything (the capture stays valid), and a DGEMM with check_accuracy != 0 refuses
 * capture (EB2_ERR_ARG).  A workspace a graph captured is never freed (later growth keeps it),
 * but replays are not fenced against other calls: do not let a replay overlap another product
 * on the same GPU. */
int eb2_dgemm_device(char transa, char transb, int64_t m, int64_t n, int64_t k, double alpha, const double* a,
                     int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc, void* stream,
                     int check_accuracy);
int eb2_sgemm_device(char transa, char transb, int64_t m, int64_t n, int64_t k, float alpha, const float* a,
                     int64_t lda, const float* b, int64_t ldb, float beta, float* c, int64_t ldc, void* stream);

/* DGEMM on device pointers that allocates nothing.  No counterpart in the reference: it
 * serves callers that cannot let a library call cudaMalloc -- a process whose GPU memory
 * is already reserved by another allocator (a framework's caching allocator, a pool sized
 * at start-up), or a code path that must not allocate or free (cudaMalloc and cudaFree may
 * synchronise the device or fail).  It computes the CRT-form emulated product (16 moduli,
 * no a-posteriori check, NaN/Inf inputs on the native kernel) with all scratch in one
 * fixed 64 MiB device array that the library holds on every GPU where it is loaded, until
 * the process exits.  Square products up to 1024 x 1024 x 1024 fit; a product that
 * needs more returns EB2_ERR_ARG, with the size in eb2_last_error_string, before any launch.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress,
 * with that device current); make that first call before any stream capture.  All calls
 * share the array: calls that overlap on the GPU (other streams, other host threads)
 * race and corrupt each other's results.  Waits for `stream` before returning. */
int eb2_dgemm_device_noalloc(char transa, char transb, int64_t m, int64_t n, int64_t k, double alpha,
                             const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c,
                             int64_t ldc, void* stream);

/* ---------------------------------------------------------------- grouped products
 * Thousands of independent products C_i = alpha_i*op(A_i)op(B_i) + beta_i*C_i (device
 * pointers, column-major) in ONE persistent launch.  Eigen has no batch entry point;
 * this is the batched counterpart of its fixed-size coefficient-based products
 * (Eigen/src/Core/GeneralProduct.h:76-80) and of per-product GEMM calls.  Products of at
 * most 8 x 8 share a warp four at a time, of at most 16 x 16 two at a time; larger ones are
 * cut into 32 x 32 tiles.  The math is native FP64 (DMMA, the native DGEMM's order, so each
 * product equals a plain native dgemm bit for bit) for dtype 'd', and split-BF16 on the
 * tensor cores for 's' (x = h + m + l in bf16 pieces, six piece products per 16-deep chunk
 * with FP32 accumulation, chunk sums added in FP32 with round-to-nearest): at least the
 * accuracy of an FP32 FMA loop. */
typedef struct eb2_gemm_problem {
  char transa, transb;   /* 'N', 'T' or 'C' */
  int64_t m, n, k;
  double alpha, beta;    /* rounded to float for dtype 's' */
  const void* a;
  int64_t lda;
  const void* b;
  int64_t ldb;
  void* c;
  int64_t ldc;
} eb2_gemm_problem;

typedef struct eb2_grouped_plan* eb2_grouped_plan_t;

/* Validates the problems (BLAS argument rules; EB2_ERR_ARG names the first bad one),
 * uploads their descriptors and the tile schedule, and captures the launch in a CUDA
 * graph.  `problems` is a host array; it may be freed after the call. */
int eb2_grouped_plan_create(char dtype, int64_t count, const eb2_gemm_problem* problems, eb2_grouped_plan_t* plan);
/* Replays the captured launch on `stream` (stream-ordered, no host synchronisation). */
int eb2_grouped_plan_execute(eb2_grouped_plan_t plan, void* stream);
int eb2_grouped_plan_destroy(eb2_grouped_plan_t plan);
/* One-shot: plan, launch on `stream`, wait, release. */
int eb2_gemm_grouped(char dtype, int64_t count, const eb2_gemm_problem* problems, void* stream);

/* The same products as separate launches, one per product, of the same arithmetic (dtype
 * 'd': the native DGEMM kernel; 's': the grouped split-BF16 tile code on that product alone),
 * stream-ordered: what a caller looping over per-product calls gets, without the host
 * synchronisation.  The baseline the grouped launch is measured against; same bits. */
int eb2_gemm_each(char dtype, int64_t count, const eb2_gemm_problem* problems, void* stream);

/* Size classes of later plans (process-wide): products with max(m, n) <= small_max go four
 * to a warp, those <= mid_max two to a warp, the rest as 32 x 32 tiles.  small_max in
 * [0, 8], mid_max in [0, 16]; 0 disables a class.  (-1, -1) restores the automatic choice
 * (the default): the learned picker decides between 8 / 16 and tiles only, from the batch's
 * geometric-mean shape and count; without weights 8 / 16.  No counterpart in the reference. */
int eb2_set_grouped_classes(int small_max, int mid_max);

/* ---------------------------------------------------------------- learned picker
 * A 3-layer MLP (8 features -> 64 -> 64 -> 19, ReLU, FP32) that plays the role of Eigen's
 * computeProductBlockingSizes (Eigen/src/Core/products/GeneralBlockPanelKernel.h:202-452).
 * Features: log2 m, n, k, the dtype, the inputs' exponent spread, log2 of the batch size,
 * log2 mnk and -log2 of the accuracy target.  Outputs: 12 configuration classes and 7
 * precision classes c (eb2_picker_predict reports 6 + c; the CRT path uses 8 + 2c moduli).
 * Configuration classes (a prediction takes the best class of its kind):
 *   DGEMM   0 native FP64 kernel; CRT emulation with 1 one CTA per 128x256 tile, 2 a CTA
 *           pair per 256x256 tile, 3 / 4 the same with raster groups of 16 row tiles,
 *           5 one CTA with K split so that the work items fill the SMs;
 *   SGEMM   6 FP32 FFMA kernel; split-BF16 on 7 128x128, 8 128x256, 9 256x256 (pair) tiles;
 *   grouped 10 small products share a warp (size classes 8 and 16), 11 32x32 tiles only.
 * A DGEMM with an automatic method consults it twice: on the shape (native or emulated)
 * and, once the scan has measured the exponent spread, for the configuration and modulus
 * count; an SGEMM with an automatic method once; a grouped plan with automatic size
 * classes once, on the batch's geometric-mean shape and size.  The library loads
 * eigen_b200/data/picker_weights.bin (trained by python -m eigen_b200.tune) when its SM
 * count matches the device.  Weights are a flat float array of eb2_mlp_param_count()
 * entries:  W1[64][8] b1[64] W2[64][64] b2[64] W3[19][64] b3[19]. */
int eb2_mlp_param_count(void);
/* Installs the weights the product path consults when method/tile/moduli are automatic
 * (copied; NULL or count 0 removes the picker).  The a-posteriori accuracy check still
 * adds moduli when a prediction falls short. */
int eb2_picker_set_weights(const float* weights, int count);
int eb2_picker_features(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                        float* out8);
int eb2_picker_forward_host(const float* weights, const float* features8, float* logits19);
int eb2_picker_predict(int64_t m, int64_t n, int64_t k, char dtype, double spread, int64_t batch, double tol,
                       int* config, int* slices);
/* Forces configuration class `config` (above) for every later call of its kind with an
 * automatic method -- what the tuner times; -1 restores the picker / the size rules.
 * Explicit method, tile and size-class settings still win.  No counterpart in the reference. */
int eb2_set_config(int config);
/* Number of configuration classes (12). */
int eb2_config_count(void);
/* Training kernels (device pointers, stream-ordered): forward logits[batch][19];
 * backward writes the batch-mean gradient (and loss) of the config cross-entropy plus
 * the slice cross-entropy for samples whose slice label is >= 0; Adam step t >= 1. */
int eb2_mlp_forward(const float* w, const float* X, int batch, float* logits, void* stream);
int eb2_mlp_backward(const float* w, const float* X, const int* cfg_label, const int* slice_label, int batch,
                     float* grads, float* loss, void* stream);
int eb2_mlp_adam(float* w, const float* grads, float* m, float* v, int step, float lr, void* stream);

/* Library version string. */
const char* eb2_version(void);

#ifdef __cplusplus
}
#endif

#endif /* EIGEN_B200_BLAS_H */
