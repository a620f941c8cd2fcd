// blas_api.cpp -- the exported C ABI: Fortran-convention sgemm_/dgemm_ (+ ILP64
// _64_ variants) with the exact argument semantics of Eigen's BLAS shim, and the
// eb2_* extension calls.
//
// Argument checking, quick returns and the beta/alpha rules restate
// blas/level3_impl.h:61-96 and Eigen/src/Core/products/GeneralMatrixMatrix.h:130;
// the N/T/C parsing restates blas/common.h:60-61.  Host operands are staged through
// device memory; device or managed operands are used in place.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>

#include "blas_common.h"
#include "context.h"
#include "eigen_b200/blas.h"
#include "gemm_driver.h"
#include "kernels.h"

extern "C" __attribute__((weak)) void xerbla_(const char* name, int* info, size_t len) {
  std::printf("Eigen BLAS ERROR #%i: %.*s\n", *info, static_cast<int>(len), name);
}

namespace eb2 {

namespace {
// The routines this library exports, in the order of their counters.
constexpr const char* kRoutines[] = {"sgemm", "dgemm", "cgemm", "zgemm", "sgemmtr", "dgemmtr", "ssyrk", "dsyrk",
                                     "ssyr2k", "dsyr2k", "ssymm", "dsymm", "strmm", "dtrmm", "strsm", "dtrsm",
                                     "csymm",  "zsymm",  "chemm", "zhemm", "ctrmm", "ztrmm", "ctrsm", "ztrsm"};
constexpr int kNumRoutines = int(sizeof(kRoutines) / sizeof(kRoutines[0]));
std::atomic<long long> g_calls[kNumRoutines];

int routine_index(const char* name) {
  if (!name) return -1;
  for (int i = 0; i < kNumRoutines; ++i)
    if (std::strcmp(kRoutines[i], name) == 0) return i;
  return -1;
}
}  // namespace

void count_call(const char* name) {
  const int i = routine_index(name);
  if (i >= 0) g_calls[i].fetch_add(1, std::memory_order_relaxed);
}

bool device_usable(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool copy_block(void* dst, size_t dpitch, const void* src, size_t spitch, size_t row_bytes, int64_t cols,
                cudaMemcpyKind kind, cudaStream_t st) {
  if (cols <= 0 || row_bytes == 0) return true;
  // through the context's stager (pinned bounce buffers for pageable host memory); the caller
  // holds the context's mutex.  Device -> host copies have landed when this returns.
  Context* cx = current_context();
  cudaError_t e;
  if (cx && kind == cudaMemcpyHostToDevice) {
    e = cx->stager.to_device(dst, dpitch, src, spitch, row_bytes, size_t(cols), st);
  } else if (cx && kind == cudaMemcpyDeviceToHost) {
    e = cx->stager.to_host(dst, dpitch, src, spitch, row_bytes, size_t(cols), st);
    if (e == cudaSuccess) e = cx->stager.drain();
  } else {
    e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, row_bytes, size_t(cols), kind, st);
  }
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_CUDA, "staging copy failed: %s", cudaGetErrorString(e));
    return false;
  }
  return true;
}

namespace {

// blas/level3_impl.h:61-78
int gemm_info(char ta, char tb, int64_t m, int64_t n, int64_t k, int64_t lda, int64_t ldb, int64_t ldc) {
  const int oa = op_code(ta), ob = op_code(tb);
  if (oa == kInvalid) return 1;
  if (ob == kInvalid) return 2;
  if (m < 0) return 3;
  if (n < 0) return 4;
  if (k < 0) return 5;
  if (lda < std::max<int64_t>(1, oa == kNoTr ? m : k)) return 8;
  if (ldb < std::max<int64_t>(1, ob == kNoTr ? k : n)) return 10;
  if (ldc < std::max<int64_t>(1, m)) return 13;
  return 0;
}

template <typename T>
struct Api;

template <>
struct Api<double> {
  static constexpr const char* kName = "DGEMM ";
  static int run(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                 int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc, cudaStream_t st,
                 bool sync, bool check, eb2_call_info& info) {
    DgemmOptions o;
    o.sync = sync;
    o.check_accuracy = check;
    o.timed = true;
    return dgemm_on_device(cx, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st, o, info);
  }
};
template <>
struct Api<float> {
  static constexpr const char* kName = "SGEMM ";
  static int run(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, float alpha, const float* A,
                 int64_t lda, const float* B, int64_t ldb, float beta, float* C, int64_t ldc, cudaStream_t st,
                 bool sync, bool /*check*/, eb2_call_info& info) {
    SgemmOptions o;
    o.sync = sync;
    o.timed = true;
    return sgemm_on_device(cx, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st, o, info);
  }
};

// The synchronous BLAS entry: checks, quick returns, staging, product.
template <typename T>
void blas_gemm(char transa, char transb, int64_t m, int64_t n, int64_t k, T alpha, const T* a, int64_t lda,
               const T* b, int64_t ldb, T beta, T* c, int64_t ldc) {
  int info = gemm_info(transa, transb, m, n, k, lda, ldb, ldc);
  if (info) {
    xerbla_(Api<T>::kName, &info, 6);
    return;
  }
  if (m == 0 || n == 0) return;
  count_call(sizeof(T) == 8 ? "dgemm" : "sgemm");
  Context* cx = current_context();
  if (!cx) {
    std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
    return;
  }
  std::lock_guard<std::mutex> lock(cx->mu);
  const bool ta = op_code(transa) != kNoTr, tb = op_code(transb) != kNoTr;
  const bool need_ab = (k > 0 && alpha != T(0));
  eb2_call_info& ci = call_info();
  ci = eb2_call_info{};
  call_config() = CallConfig{};
  cudaStream_t st = cx->stream;
  StreamFence fence(*cx, st);

  const bool a_dev = !need_ab || device_usable(a);
  const bool b_dev = !need_ab || device_usable(b);
  const bool c_dev = device_usable(c);
  if constexpr (sizeof(T) == 8) {
    // all three in host memory: copies overlapped with the product, block by block
    if (need_ab && !a_dev && !b_dev && !c_dev &&
        crt_pipeline_applies(*cx, m, n, k, resolve_dgemm_method(m, n, k))) {
      const int rc = dgemm_crt_pipelined(*cx, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ci);
      if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) {
        std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
        (void)cudaDeviceSynchronize();
      }
      return;
    }
  }
  const T* da = a;
  const T* db = b;
  T* dc = c;
  int64_t dlda = lda, dldb = ldb, dldc = ldc;
  ci.staged = (!a_dev || !b_dev || !c_dev) ? 1 : 0;
  if (!a_dev) {
    const int64_t rows = ta ? k : m, cols = ta ? m : k;
    if (!cx->stage_a.ensure(size_t(rows) * size_t(cols) * sizeof(T))) {
      set_error(EB2_ERR_ALLOC, "could not allocate staging memory for A");
      std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
      return;
    }
    if (!copy_block(cx->stage_a.ptr, rows * sizeof(T), a, lda * sizeof(T), rows * sizeof(T), cols,
                    cudaMemcpyHostToDevice, st))
      return;
    da = static_cast<const T*>(cx->stage_a.ptr);
    dlda = rows;
  }
  if (!b_dev) {
    const int64_t rows = tb ? n : k, cols = tb ? k : n;
    if (!cx->stage_b.ensure(size_t(rows) * size_t(cols) * sizeof(T))) {
      set_error(EB2_ERR_ALLOC, "could not allocate staging memory for B");
      std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
      return;
    }
    if (!copy_block(cx->stage_b.ptr, rows * sizeof(T), b, ldb * sizeof(T), rows * sizeof(T), cols,
                    cudaMemcpyHostToDevice, st))
      return;
    db = static_cast<const T*>(cx->stage_b.ptr);
    dldb = rows;
  }
  if (!c_dev) {
    if (!cx->stage_c.ensure(size_t(m) * size_t(n) * sizeof(T))) {
      set_error(EB2_ERR_ALLOC, "could not allocate staging memory for C");
      std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
      return;
    }
    dc = static_cast<T*>(cx->stage_c.ptr);
    dldc = m;
    // beta == 0 never reads C (blas/level3_impl.h:82-84), so it need not be copied in
    if (beta != T(0) &&
        !copy_block(dc, m * sizeof(T), c, ldc * sizeof(T), m * sizeof(T), n, cudaMemcpyHostToDevice, st))
      return;
  }
  int rc = Api<T>::run(*cx, ta, tb, m, n, k, alpha, da, dlda, db, dldb, beta, dc, dldc, st, true, true, ci);
  if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) {
    std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
    (void)cudaStreamSynchronize(st);
    return;
  }
  if (!c_dev) {
    if (!copy_block(c, ldc * sizeof(T), dc, m * sizeof(T), m * sizeof(T), n, cudaMemcpyDeviceToHost, st)) return;
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_CUDA, "GEMM failed: %s", cudaGetErrorString(e));
    std::fprintf(stderr, "eigen_b200: %s\n", eb2_last_error_string());
  }
}

}  // namespace
}  // namespace eb2

using eb2::blas_gemm;

extern "C" {

void dgemm_(const char* transa, const char* transb, const int* m, const int* n, const int* k, const double* alpha,
            const double* a, const int* lda, const double* b, const int* ldb, const double* beta, double* c,
            const int* ldc) {
  blas_gemm<double>(*transa, *transb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

void sgemm_(const char* transa, const char* transb, const int* m, const int* n, const int* k, const float* alpha,
            const float* a, const int* lda, const float* b, const int* ldb, const float* beta, float* c,
            const int* ldc) {
  blas_gemm<float>(*transa, *transb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

void dgemm_64_(const char* transa, const char* transb, const int64_t* m, const int64_t* n, const int64_t* k,
               const double* alpha, const double* a, const int64_t* lda, const double* b, const int64_t* ldb,
               const double* beta, double* c, const int64_t* ldc) {
  blas_gemm<double>(*transa, *transb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

void sgemm_64_(const char* transa, const char* transb, const int64_t* m, const int64_t* n, const int64_t* k,
               const float* alpha, const float* a, const int64_t* lda, const float* b, const int64_t* ldb,
               const float* beta, float* c, const int64_t* ldc) {
  blas_gemm<float>(*transa, *transb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

int eb2_set_dgemm_method(int method) {
  if (method < EB2_METHOD_AUTO || method > EB2_METHOD_CRT) return EB2_ERR_ARG;
  eb2::settings().dgemm_method = method;
  return EB2_OK;
}

int eb2_set_sgemm_method(int method) {
  if (method < EB2_METHOD_AUTO || method > EB2_METHOD_EMULATED) return EB2_ERR_ARG;
  eb2::settings().sgemm_method = method;
  return EB2_OK;
}

int eb2_set_dgemm_moduli(int moduli) {
  if (moduli != 0 && (moduli < 8 || moduli > eb2::kCrtMaxModuli)) return EB2_ERR_ARG;
  eb2::settings().dgemm_moduli = moduli;
  return EB2_OK;
}

int eb2_set_dgemm_slices(int slices) {
  if (slices != 0 && (slices < 2 || slices > eb2::kOzakiMaxSlices)) return EB2_ERR_ARG;
  eb2::settings().dgemm_slices = slices;
  return EB2_OK;
}

int eb2_set_sgemm_pieces(int pieces) {
  if (pieces != 2 && pieces != 3) return EB2_ERR_ARG;
  eb2::settings().sgemm_pieces = pieces;
  return EB2_OK;
}

int eb2_set_dgemm_tolerance(double tol) {
  if (!(tol > 0.0)) return EB2_ERR_ARG;
  eb2::settings().dgemm_tol = tol;
  return EB2_OK;
}

int eb2_set_tile_n(int tile_n) {
  if (tile_n != 0 && tile_n != 128 && tile_n != 256 && tile_n != eb2::kTilePair && tile_n != eb2::kTileWide)
    return EB2_ERR_ARG;
  eb2::settings().tile_n = tile_n;
  return EB2_OK;
}

int eb2_last_error(void) { return eb2::last_error(); }

void eb2_clear_error(void) { eb2::set_error(EB2_OK, ""); }

int eb2_set_slice_tuning(int group_m, int prefetch) {
  if (group_m < 0 || prefetch < 0 || prefetch > 64) return EB2_ERR_ARG;
  eb2::tuning().group_m = group_m;
  eb2::tuning().prefetch = prefetch;
  return EB2_OK;
}

int eb2_set_wait_limit_ns(long long ns) {
  if (ns < 0) return EB2_ERR_ARG;
  eb2::tuning().wait_limit_ns = static_cast<uint64_t>(ns);
  return EB2_OK;
}

int eb2_set_timing(int on) {
  eb2::settings().timing = on ? 1 : 0;
  return EB2_OK;
}

int eb2_last_call_info(eb2_call_info* out) {
  if (!out) return EB2_ERR_ARG;
  eb2::resolve_timing();
  *out = eb2::call_info();
  return EB2_OK;
}

int eb2_dgemm_device(char transa, char transb, int64_t m, int64_t n, int64_t k, double alpha, const double* a,
                     int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc, void* stream,
                     int check_accuracy) {
  if (eb2::gemm_info(transa, transb, m, n, k, lda, ldb, ldc) != 0) {
    eb2::set_error(EB2_ERR_ARG, "invalid DGEMM arguments (BLAS info %d)",
                   eb2::gemm_info(transa, transb, m, n, k, lda, ldb, ldc));
    return EB2_ERR_ARG;
  }
  eb2::Context* cx = eb2::context_for_stream(static_cast<cudaStream_t>(stream));
  if (!cx) return eb2::last_error();
  if (check_accuracy) {
    // the a-posteriori check reads the estimate on the host between kernels
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &capture) == cudaSuccess &&
        capture != cudaStreamCaptureStatusNone) {
      eb2::set_error(EB2_ERR_ARG, "a DGEMM with the accuracy check cannot be captured into a graph; "
                                  "capture it with check_accuracy = 0");
      return EB2_ERR_ARG;
    }
    (void)cudaGetLastError();
  }
  std::lock_guard<std::mutex> lock(cx->mu);
  eb2::StreamFence fence(*cx, static_cast<cudaStream_t>(stream));
  eb2::DgemmOptions o;
  o.sync = check_accuracy != 0;
  o.check_accuracy = check_accuracy != 0;
  o.timed = eb2::settings().timing.load() != 0;
  eb2_call_info& ci = eb2::call_info();
  ci = eb2_call_info{};
  eb2::call_config() = eb2::CallConfig{};
  return eb2::dgemm_on_device(*cx, eb2::op_code(transa) != eb2::kNoTr, eb2::op_code(transb) != eb2::kNoTr, m, n, k,
                              alpha, a, lda, b, ldb, beta, c, ldc, static_cast<cudaStream_t>(stream), o, ci);
}

int eb2_sgemm_device(char transa, char transb, int64_t m, int64_t n, int64_t k, float alpha, const float* a,
                     int64_t lda, const float* b, int64_t ldb, float beta, float* c, int64_t ldc, void* stream) {
  if (eb2::gemm_info(transa, transb, m, n, k, lda, ldb, ldc) != 0) {
    eb2::set_error(EB2_ERR_ARG, "invalid SGEMM arguments (BLAS info %d)",
                   eb2::gemm_info(transa, transb, m, n, k, lda, ldb, ldc));
    return EB2_ERR_ARG;
  }
  eb2::Context* cx = eb2::context_for_stream(static_cast<cudaStream_t>(stream));
  if (!cx) return eb2::last_error();
  std::lock_guard<std::mutex> lock(cx->mu);
  eb2::StreamFence fence(*cx, static_cast<cudaStream_t>(stream));
  eb2::SgemmOptions o;
  o.sync = false;
  o.timed = eb2::settings().timing.load() != 0;
  eb2_call_info& ci = eb2::call_info();
  ci = eb2_call_info{};
  eb2::call_config() = eb2::CallConfig{};
  return eb2::sgemm_on_device(*cx, eb2::op_code(transa) != eb2::kNoTr, eb2::op_code(transb) != eb2::kNoTr, m, n, k,
                              alpha, a, lda, b, ldb, beta, c, ldc, static_cast<cudaStream_t>(stream), o, ci);
}

long long eb2_routine_calls(const char* name) {
  const int i = eb2::routine_index(name);
  return i < 0 ? -1 : eb2::g_calls[i].load(std::memory_order_relaxed);
}

const char* eb2_version(void) { return "eigen_b200 0.1 (sm_100a)"; }

}  // extern "C"
