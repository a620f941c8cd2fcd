// noalloc.cu -- the CRT-form emulated DGEMM without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: a process whose device memory is
// already fully reserved by another allocator (a framework's caching allocator that owns
// the GPU, a memory pool sized at start-up), or code on a path that must never allocate or
// free (cudaMalloc and cudaFree can synchronise the device and fail at any time).  For
// them eb2_dgemm_device_noalloc runs the same kernels as the CRT path of eb2_dgemm_device
// (16 moduli, no a-posteriori check) with all of its scratch -- row maxima, norm bounds,
// scale exponents, operand residues, product residues and flags -- in one fixed
// file-scope device array.  The array costs kNoAllocScratchBytes of device memory on every
// GPU where this module is loaded, until the process exits; products whose scratch does
// not fit are rejected (EB2_ERR_ARG) before anything is launched.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "context.h"
#include "eigen_b200/blas.h"
#include "kernels.h"

namespace eb2 {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB
constexpr int kNoAllocModuli = kCrtDefaultModuli;
constexpr int64_t kNoAllocMaxDim = int64_t(1) << 20;  // larger m, n or k never fits the scratch
constexpr int kMaxDevices = 64;

// The scratch.  Host code must not use this name as an address: on the host it denotes a
// stand-in object, not device memory.  The device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

// Head of the scratch: flags the kernels report through (zeroed by every call).
struct NoAllocFlags {
  int nonfinite;
  uint32_t status;
};

struct DeviceSetup {
  uint8_t* scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int num_sms = 0;
  bool ready = false;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Once per device, with that device current: the scratch address and the SM count.
const DeviceSetup* setup_device() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_NO_DEVICE, "eb2_dgemm_device_noalloc: no usable CUDA device");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  DeviceSetup& s = g_setup[dev];
  if (s.ready) return &s;
  int major = 0, sms = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || major != 10) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_NO_DEVICE, "eb2_dgemm_device_noalloc: device %d is not an sm_100 device", dev);
    return nullptr;
  }
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || ptr == nullptr) {
    (void)cudaGetLastError();
    set_error(EB2_ERR_CUDA, "eb2_dgemm_device_noalloc: cudaGetSymbolAddress of the scratch failed: %s",
              cudaGetErrorString(e));
    return nullptr;
  }
  s.scratch = static_cast<uint8_t*>(ptr);
  s.num_sms = sms;
  s.ready = true;
  return &s;
}

bool trans_of(char t, bool& out) {
  switch (t) {
    case 'N': case 'n': out = false; return true;
    case 'T': case 't': case 'C': case 'c': out = true; return true;
    default: return false;
  }
}

bool ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  (void)cudaGetLastError();
  set_error(EB2_ERR_CUDA, "eb2_dgemm_device_noalloc: %s: %s", what, cudaGetErrorString(e));
  return false;
}

}  // namespace
}  // namespace eb2

extern "C" int eb2_dgemm_device_noalloc(char transa, char transb, int64_t m, int64_t n, int64_t k, double alpha,
                                        const double* a, int64_t lda, const double* b, int64_t ldb, double beta,
                                        double* c, int64_t ldc, void* stream) {
  using namespace eb2;
  bool ta = false, tb = false;
  if (!trans_of(transa, ta) || !trans_of(transb, tb) || m < 0 || n < 0 || k < 0 ||
      lda < std::max<int64_t>(1, ta ? k : m) || ldb < std::max<int64_t>(1, tb ? n : k) ||
      ldc < std::max<int64_t>(1, m)) {
    set_error(EB2_ERR_ARG, "eb2_dgemm_device_noalloc: invalid argument (BLAS rules for trans, sizes and leading "
                           "dimensions)");
    return EB2_ERR_ARG;
  }
  if (m == 0 || n == 0) return EB2_OK;
  // Every operand keeps 16 residue planes of at least one 128-byte K block per row, so a
  // dimension above 2^20 needs more than 2 GiB of scratch: refuse it before the layout
  // arithmetic below, whose products could otherwise wrap for absurd (BLAS-valid) sizes.
  if (m > kNoAllocMaxDim || n > kNoAllocMaxDim || k > kNoAllocMaxDim) {
    set_error(EB2_ERR_ARG,
              "eb2_dgemm_device_noalloc: a %lld x %lld x %lld product cannot fit the fixed %zu bytes of scratch; "
              "use eb2_dgemm_device for it",
              static_cast<long long>(m), static_cast<long long>(n), static_cast<long long>(k), kNoAllocScratchBytes);
    return EB2_ERR_ARG;
  }
  const DeviceSetup* ds = setup_device();
  if (!ds) return last_error();
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (k == 0 || alpha == 0.0) {
    if (beta == 1.0) return EB2_OK;
    return ok(launch_scale_matrix_d(m, n, beta, c, ldc, st), "scale C") && ok(cudaStreamSynchronize(st), "C = beta C")
               ? EB2_OK
               : EB2_ERR_CUDA;
  }

  // scratch layout (the same quantities the CRT path keeps in its workspace)
  const int64_t pair_tiles = ((m + 255) / 256) * ((n + 255) / 256);
  const int tile = 2 * pair_tiles >= ds->num_sms ? kTilePair : 256;
  const int64_t m_pad = round_up(m, crt_tile_rows(tile)), n_pad = round_up(n, crt_tile_cols(tile)),
                k_pad = round_up(k, kOzakiKBlock);
  size_t off = align256(sizeof(NoAllocFlags));
  const size_t o_mb_a = off;
  off = align256(off + size_t(m) * 8);
  const size_t o_mb_b = off;
  off = align256(off + size_t(n) * 8);
  const int64_t nchunks = k_pad / kOzakiKBlock;  // 128-column chunks of the norm bounds
  const size_t o_ss_a = off;
  off = align256(off + size_t(m) * nchunks * 8);
  const size_t o_ss_b = off;
  off = align256(off + size_t(n) * nchunks * 8);
  const size_t o_ce_a = off;
  off = align256(off + size_t(m) * nchunks * 4);
  const size_t o_ce_b = off;
  off = align256(off + size_t(n) * nchunks * 4);
  const size_t o_mu_a = off;
  off = align256(off + size_t(m_pad) * 4);
  const size_t o_mu_b = off;
  off = align256(off + size_t(n_pad) * 4);
  const size_t o_res_a = off;
  off = align256(off + size_t(kNoAllocModuli) * m_pad * k_pad);
  const size_t o_res_b = off;
  off = align256(off + size_t(kNoAllocModuli) * n_pad * k_pad);
  const size_t o_res_c = off;
  off = align256(off + size_t(kNoAllocModuli) * m_pad * n_pad);
  if (off > kNoAllocScratchBytes) {
    set_error(EB2_ERR_ARG,
              "eb2_dgemm_device_noalloc: a %lld x %lld x %lld product needs %zu bytes of scratch, more than the "
              "fixed %zu; use eb2_dgemm_device for it",
              static_cast<long long>(m), static_cast<long long>(n), static_cast<long long>(k), off,
              kNoAllocScratchBytes);
    return EB2_ERR_ARG;
  }

  uint8_t* ws = ds->scratch;
  NoAllocFlags* flags = reinterpret_cast<NoAllocFlags*>(ws);
  const StridedView<double> va =
      ta ? StridedView<double>{a, m, k, lda, 1} : StridedView<double>{a, m, k, 1, lda};  // op(A), m x k
  const StridedView<double> vb =
      tb ? StridedView<double>{b, n, k, 1, ldb} : StridedView<double>{b, n, k, ldb, 1};  // op(B)^T, n x k
  CrtOperand oa{reinterpret_cast<int8_t*>(ws + o_res_a), reinterpret_cast<int32_t*>(ws + o_mu_a),
                reinterpret_cast<uint64_t*>(ws + o_mb_a), reinterpret_cast<uint64_t*>(ws + o_ss_a),
                reinterpret_cast<int32_t*>(ws + o_ce_a), m, m_pad, k, k_pad, kNoAllocModuli};
  CrtOperand ob{reinterpret_cast<int8_t*>(ws + o_res_b), reinterpret_cast<int32_t*>(ws + o_mu_b),
                reinterpret_cast<uint64_t*>(ws + o_mb_b), reinterpret_cast<uint64_t*>(ws + o_ss_b),
                reinterpret_cast<int32_t*>(ws + o_ce_b), n, n_pad, k, k_pad, kNoAllocModuli};

  // The scratch keeps whatever the previous call left: the flags and the row maxima
  // (atomicMax, zeroed by the scan launcher) start from zero; the chunk norm bounds, scale
  // exponents and residues are overwritten.
  bool good = ok(cudaMemsetAsync(flags, 0, sizeof(NoAllocFlags), st), "reset flags");
  good = good && ok(launch_crt_scan_norms(va, oa, &flags->nonfinite, nullptr, st), "scan A");
  good = good && ok(launch_crt_scan_norms(vb, ob, &flags->nonfinite, nullptr, st), "scan B");
  good = good && ok(launch_crt_split(va, oa, kNoAllocModuli, st), "residues A");
  good = good && ok(launch_crt_split(vb, ob, kNoAllocModuli, st), "residues B");
  CrtGemmArgs g{};
  g.m = m;
  g.n = n;
  g.moduli = kNoAllocModuli;
  g.skip_if_flag = &flags->nonfinite;
  g.status = &flags->status;
  g.tile_n = tile;
  g.num_sms = ds->num_sms;
  g.cres = ws + o_res_c;
  g.ld_res = m_pad;
  good = good && ok(launch_crt_gemm(oa, ob, g, st), "CRT GEMM");
  CrtReconstructArgs r{};
  r.m = m;
  r.n = n;
  r.alpha = alpha;
  r.beta = beta;
  r.C = c;
  r.ldc = ldc;
  r.cres = ws + o_res_c;
  r.ld_res = m_pad;
  r.plane = m_pad * n_pad;
  r.moduli = kNoAllocModuli;
  r.mu_a = oa.mu;
  r.mu_b = ob.mu;
  r.err_sq = nullptr;
  r.skip_if_flag = &flags->nonfinite;
  r.write_c = true;
  good = good && ok(launch_crt_reconstruct(r, st), "CRT reconstruction");
  // IEEE semantics for NaN/Inf inputs: the FP64 kernel runs only when the scan saw one
  good = good && ok(launch_dgemm_native(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, &flags->nonfinite, st),
                    "non-finite fallback");
  if (!good) return EB2_ERR_CUDA;
  NoAllocFlags hf{};
  if (!ok(cudaMemcpyAsync(&hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st), "read flags") ||
      !ok(cudaStreamSynchronize(st), "DGEMM"))
    return EB2_ERR_CUDA;
  if (hf.status != 0) {
    set_error(EB2_ERR_TIMEOUT, "eb2_dgemm_device_noalloc: a kernel wait timed out (device status 0x%x); C is invalid",
              hf.status);
    return EB2_ERR_TIMEOUT;
  }
  return EB2_OK;
}
