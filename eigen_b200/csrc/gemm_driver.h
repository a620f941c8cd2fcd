// gemm_driver.h -- device-level product drivers (device pointers, one stream).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "context.h"

namespace eb2 {

struct DgemmOptions {
  int method = 0;        // EB2_METHOD_*; 0 = settings
  int slices = 0;        // 0 = chosen per call
  int moduli = 0;        // CRT moduli; 0 = settings (default 16)
  int tile_n = 0;        // 0 = chosen per call
  double tol = 0.0;      // 0 = settings
  bool check_accuracy = true;  // a-posteriori estimate + added slices (needs a host sync)
  bool sync = true;      // wait for the stream before returning
  bool timed = false;    // record kernel time in call_info
  int uplo = 0;          // CRT only, m == n: 1 = compute and write only C's upper triangle
                         // (i <= j), 2 = only the lower (i >= j); the other is not touched
  int tri_operand = 0;   // CRT only: op(A) (1 lower, 2 upper) or op(B) (3 lower, 4 upper) is
                         // triangular with zeros outside; its zero K blocks are skipped (same C)
};

struct SgemmOptions {
  int method = 0;
  int pieces = 0;  // BF16 pieces per operand (2 or 3); 0 = settings
  int tile_n = 0;
  bool sync = true;
  bool timed = false;
};

int choose_tile_n(const Context& cx, int64_t m, int64_t n, bool ozaki);
int choose_slices(int64_t m, int64_t n, int64_t k);
int choose_crt_tile(const Context& cx, int64_t m, int64_t n);
// K splits of the CRT GEMM's split-K configuration (one-CTA tiles): about two waves of work
// items over the SMs, each split at least two K blocks, at most kCrtMaxSplits.
int crt_split_rule(const Context& cx, int64_t m_pad, int64_t n_pad, int64_t k_pad, int moduli);
// DGEMM method without a per-call override: the settings, else the learned picker on the
// shape, else the size rule (auto_method_rule).
int resolve_dgemm_method(int64_t m, int64_t n, int64_t k);
int auto_method_rule(int64_t m, int64_t n, int64_t k);

// The BLAS entry's DGEMM with A, B and C in host memory, as a pipeline of column blocks
// (copies overlapped with the product).  crt_pipeline_applies() tells whether it is used.
bool crt_pipeline_applies(const Context& cx, int64_t m, int64_t n, int64_t k, int method);
int dgemm_crt_pipelined(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                        const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                        int64_t ldc, eb2_call_info& info);

// C = alpha*op(A)op(B) + beta*C on device pointers.  Returns EB2_*.
int dgemm_on_device(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                    int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                    cudaStream_t st, const DgemmOptions& opt, eb2_call_info& info);
int sgemm_on_device(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, float alpha, const float* A,
                    int64_t lda, const float* B, int64_t ldb, float beta, float* C, int64_t ldc, cudaStream_t st,
                    const SgemmOptions& opt, eb2_call_info& info);

}  // namespace eb2
