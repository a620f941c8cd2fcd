// gemm_driver.cpp -- device-level product drivers: choose the method, lay out the
// workspace, launch the kernels in order and run the a-posteriori accuracy check.
//
// The role matches Eigen's general_matrix_matrix_product<...>::run
// (Eigen/src/Core/products/GeneralMatrixMatrix.h:119-246) plus the blocking choice
// of computeProductBlockingSizes (Eigen/src/Core/products/GeneralBlockPanelKernel.h:202-452):
// here "blocking" is the tcgen05 tile width and the number of digit slices.
#include "gemm_driver.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "kernels.h"
#include "mlp.h"

namespace eb2 {

namespace {

// The accuracy target of an FP32 product as a picker feature (FP32 unit roundoff).
constexpr double kSgemmTolFeature = 5.9604644775390625e-08;

// Rows / columns of C covered by one tile of a tile configuration.  The Ozaki GEMM keeps
// its FP64 accumulator in registers, so its tiles are 128 columns wide (128 and 256
// select one CTA / a CTA pair); the split-BF16 GEMM uses 128 / 256 wide single-CTA tiles
// and 256 x 256 pair tiles.
int64_t tile_m_of(int cfg, bool ozaki) { return (cfg == kTilePair || (ozaki && cfg == 256)) ? 256 : 128; }
int64_t tile_n_of(int cfg, bool ozaki) { return ozaki ? 128 : (cfg == kTilePair ? 256 : cfg); }

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

bool check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  (void)cudaGetLastError();
  set_error(EB2_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return false;
}

// Views of op(A) (m x k) and op(B)^T (n x k): row r, column l (l runs along K).
StridedView<double> view_a(bool ta, const double* A, int64_t lda, int64_t m, int64_t k) {
  // op(A)(i,l) = A[i + l*lda] (N) or A[l + i*lda] (T)
  return ta ? StridedView<double>{A, m, k, lda, 1} : StridedView<double>{A, m, k, 1, lda};
}
StridedView<double> view_bt(bool tb, const double* B, int64_t ldb, int64_t n, int64_t k) {
  // op(B)(l,j) = B[l + j*ldb] (N) or B[j + l*ldb] (T); row j of op(B)^T
  return tb ? StridedView<double>{B, n, k, 1, ldb} : StridedView<double>{B, n, k, ldb, 1};
}

}  // namespace

int choose_tile_n(const Context& cx, int64_t m, int64_t n, bool ozaki) {
  const int forced = settings().tile_n.load();
  if (forced == 128 || forced == 256 || forced == kTilePair) return forced;
  if (ozaki) {
    // CTA pairs (256 x 128) unless that leaves most SMs idle
    const int64_t pair_tiles = ((m + 255) / 256) * ((n + 127) / 128);
    return 2 * pair_tiles >= cx.num_sms ? kTilePair : 128;
  }
  if (n <= 128) return 128;
  const int64_t tiles256 = ((m + 127) / 128) * ((n + 255) / 256);
  return tiles256 < cx.num_sms ? 128 : 256;
}

int choose_slices(int64_t m, int64_t n, int64_t k) {
  (void)m;
  (void)n;
  (void)k;
  const int forced = settings().dgemm_slices.load();
  if (forced >= 2 && forced <= kOzakiMaxSlices) return forced;
  return 8;
}

int auto_method_rule(int64_t m, int64_t n, int64_t k) {
  // without picker weights: the CRT emulation where its fixed costs (scans, residues,
  // reconstruction, about 0.1 ms) and the O(mn + (m+n)k) passes are amortised
  const double mnk = double(m) * double(n) * double(k);
  return (mnk >= 4294967296.0 && k >= 1024 && std::min(m, n) >= 256) ? EB2_METHOD_CRT : EB2_METHOD_NATIVE;
}

int resolve_dgemm_method(int64_t m, int64_t n, int64_t k) {
  const int method = settings().dgemm_method.load();
  if (method != EB2_METHOD_AUTO) return method;
  const int fc = forced_config();
  if (fc >= kCfgNative && fc <= kCfgCrtSplitK) return fc == kCfgNative ? EB2_METHOD_NATIVE : EB2_METHOD_CRT;
  int cfg = -1, cls = 0;
  if (picker_weights() != nullptr && picker_predict(m, n, k, 'd', 0.0, 1, settings().dgemm_tol.load(), &cfg, &cls))
    return cfg == kCfgNative ? EB2_METHOD_NATIVE : EB2_METHOD_CRT;
  return auto_method_rule(m, n, k);
}

int crt_split_rule(const Context& cx, int64_t m_pad, int64_t n_pad, int64_t k_pad, int moduli) {
  // one-CTA tiles; about two waves of work items over the SMs, each split at least two K blocks
  const int64_t items = (m_pad / 128) * ((n_pad + 255) / 256) * moduli;
  const int64_t kb = k_pad / kOzakiKBlock;
  int64_t s = items > 0 ? (2 * int64_t(cx.num_sms)) / items : 1;
  s = std::min<int64_t>(s, std::min<int64_t>(kCrtMaxSplits, kb / 2));
  return int(std::max<int64_t>(s, 1));
}

// Padding the rows to 256 instead of 128 adds nothing (an even count of 128-row blocks) or at
// most 1/16 of the product.
static bool crt_rows256_cheap(int64_t m) { return ((m + 127) / 128) % 2 == 0 || m >= 2048; }

int choose_crt_tile(const Context& cx, int64_t m, int64_t n) {
  const int forced = settings().tile_n.load();
  if (forced == kTilePair || forced == kTileWide) return forced;
  if (forced == 128 || forced == 256) return 256;
  // 128 x 256 tiles where 256-row padding would cost; otherwise 256 x 256 tiles, on one CTA
  // while the (tile, modulus) items fill the SMs, on a CTA pair when they are few
  if (!crt_rows256_cheap(m)) return 256;
  const int64_t tiles = ((m + 255) / 256) * ((n + 255) / 256);
  return tiles * kCrtMinModuli >= cx.num_sms ? kTileWide : kTilePair;
}

namespace {

// CRT-form emulation (Ozaki scheme II): scan, norm bounds, residue split, one INT8 GEMM
// per modulus, exact reconstruction.  The a-posteriori check adds two moduli at a time;
// with beta != 0 the reconstruction keeps the old C as it writes the new one, and a product
// redone with more moduli starts again from it.
int dgemm_crt(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
              int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc, cudaStream_t st,
              const DgemmOptions& opt, eb2_call_info& info) {
  info.method = EB2_METHOD_CRT;
  const bool check = opt.check_accuracy;
  const int forced = opt.moduli ? opt.moduli : settings().dgemm_moduli.load();
  int nmod = forced ? forced : kCrtDefaultModuli;
  const bool auto_tile =
      opt.tile_n != kTilePair && opt.tile_n != kTileWide && opt.tile_n != 256 && settings().tile_n.load() == 0;
  // Stage 2 of the learned picker: tile configuration and modulus count, once the scan
  // has measured the inputs' exponent spread.  It needs the host to read the scan's result,
  // so a call captured into a graph keeps the stage-1 choice.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &capture) != cudaSuccess) {
    (void)cudaGetLastError();
    capture = cudaStreamCaptureStatusNone;
  }
  const int fc = forced_config();
  const bool forced_cfg = fc >= kCfgCrtCta && fc <= kCfgCrtSplitK;
  const bool stage2 = picker_weights() != nullptr && !forced_cfg && (auto_tile || forced == 0) &&
                      capture == cudaStreamCaptureStatusNone;
  const int nmax = (check || stage2) ? std::max(nmod, kCrtMaxModuli) : nmod;
  int tile = (opt.tile_n == kTilePair || opt.tile_n == kTileWide || opt.tile_n == 256) ? opt.tile_n
                                                                                         : choose_crt_tile(cx, m, n);
  int group_m = 0, splits = 1;
  const StridedView<double> va = view_a(ta, A, lda, m, k);
  const StridedView<double> vb = view_bt(tb, B, ldb, n, k);
  // op(B)^T == op(A) (a product A A^T, as in syrk): one scan and one split serve both
  const bool same = m == n && va.ptr == vb.ptr && va.sr == vb.sr && va.sl == vb.sl;
  // rows padded for the pair tile whenever the picker may still choose it
  // (a forced pair class switches the tile to a CTA pair below)
  const bool pair_rows =
      stage2 || same || crt_rows256_cheap(m) || (auto_tile && (fc == kCfgCrtPair || fc == kCfgCrtPairGroup));
  const int64_t m_pad = round_up(m, pair_rows ? 256 : crt_tile_rows(tile)),
                n_pad = round_up(n, crt_tile_cols(tile)), k_pad = round_up(k, kOzakiKBlock);
  const bool tri = opt.uplo == 1 || opt.uplo == 2;
  const int64_t max_tiles = (m_pad / 128) * (n_pad / 256);
  // a configuration class: tile shape, raster order, K splits (dense products only)
  const bool may_split = auto_tile && !tri && opt.tri_operand == 0;
  // the one-CTA classes take 256 x 256 tiles where the rows are padded to 256 at little cost
  const int cta_tile = (m_pad % 256 == 0 && crt_rows256_cheap(m)) ? kTileWide : 256;
  auto apply_config = [&](int c) {
    tile = (c == kCfgCrtPair || c == kCfgCrtPairGroup) ? kTilePair : (c == kCfgCrtSplitK ? 256 : cta_tile);
    group_m = (c == kCfgCrtCtaGroup || c == kCfgCrtPairGroup) ? kCfgGroupM : 0;
    splits = (c == kCfgCrtSplitK && may_split) ? crt_split_rule(cx, m_pad, n_pad, k_pad, nmod) : 1;
  };
  if (auto_tile && forced_cfg) apply_config(fc);
  // planes of the product residues per modulus: the most K splits a decision can still pick
  const int max_splits =
      splits > 1 ? splits : ((stage2 && may_split) ? crt_split_rule(cx, m_pad, n_pad, k_pad, kCrtMinModuli) : 1);
  size_t off = 0;
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
  off = align256(off + size_t(nmax) * m_pad * k_pad);
  const size_t o_res_b = off;
  off = align256(off + size_t(nmax) * n_pad * k_pad);
  const size_t o_res_c = off;
  off = align256(off + size_t(nmax) * max_splits * m_pad * n_pad);
  // triangle only: the tile list, and the non-finite fallback's full product
  const size_t o_tiles = off;
  off = align256(off + (tri ? size_t(max_tiles) * 4 : 0));
  const size_t o_full = off;
  off = align256(off + (tri ? size_t(m) * n * 8 : 0));
  // beta != 0 with the check: the old C, kept as the reconstruction overwrites it, in case the
  // product must be redone with more moduli (a triangle keeps it in the fallback buffer, which
  // only a non-finite input uses, and then no reconstruction runs)
  const bool keep_old = check && beta != 0.0;
  const size_t o_save = off;
  off = align256(off + (keep_old && !tri ? size_t(m) * n * 8 : 0));
  if (const int rc = reserve_buffer(cx.ws, off, st, "emulation workspace"); rc != EB2_OK) return rc;
  uint8_t* ws = static_cast<uint8_t*>(cx.ws.ptr);
  DeviceFlags* df = cx.dflags;
  CrtOperand oa{reinterpret_cast<int8_t*>(ws + o_res_a), reinterpret_cast<int32_t*>(ws + o_mu_a),
                reinterpret_cast<uint64_t*>(ws + o_mb_a), reinterpret_cast<uint64_t*>(ws + o_ss_a),
                reinterpret_cast<int32_t*>(ws + o_ce_a), m, m_pad, k, k_pad, nmax};
  const CrtOperand ob = same ? oa
                             : CrtOperand{reinterpret_cast<int8_t*>(ws + o_res_b), reinterpret_cast<int32_t*>(ws + o_mu_b),
                                          reinterpret_cast<uint64_t*>(ws + o_mb_b),
                                          reinterpret_cast<uint64_t*>(ws + o_ss_b),
                                          reinterpret_cast<int32_t*>(ws + o_ce_b), n, n_pad, k, k_pad, nmax};

  bool ok = check_cuda(cudaMemsetAsync(df, 0, sizeof(DeviceFlags), st), "reset flags");
  ok = ok && check_cuda(launch_crt_scan_norms(va, oa, &df->nonfinite, &df->spread[0], st), "scan A");
  if (!same) ok = ok && check_cuda(launch_crt_scan_norms(vb, ob, &df->nonfinite, &df->spread[0], st), "scan B");
  if (!ok) return EB2_ERR_CUDA;
  info.launches = same ? 1 : 2;
  // Stage 2 reads the scans' statistics on the host.  The residue split for the current
  // modulus count is launched first, so the GPU works while the host waits and decides; it is
  // redone only if the picker changes the count (both tile configurations use the same
  // residue layout).
  int split_moduli = 0;  // modulus count of the residues already launched (0: none)
  auto split = [&]() -> bool {
    bool good = check_cuda(launch_crt_split(va, oa, nmod, st), "residues A");
    if (!same) good = good && check_cuda(launch_crt_split(vb, ob, nmod, st), "residues B");
    info.launches += same ? 2 : 4;
    split_moduli = nmod;
    return good;
  };
  if (stage2) {
    if (!check_cuda(cudaMemcpyAsync(cx.hflags, df, sizeof(DeviceFlags), cudaMemcpyDeviceToHost, st), "read scan") ||
        !check_cuda(cudaEventRecord(cx.ev_scan, st), "scan event") || !split() ||
        !check_cuda(cudaEventSynchronize(cx.ev_scan), "scan"))
      return EB2_ERR_CUDA;
    const double spread = cx.hflags->spread[1] > 0 ? cx.hflags->spread[0] / cx.hflags->spread[1] : 0.0;
    int cfg = -1, cls = 0;
    if (picker_predict(m, n, k, 'd', spread, 1, opt.tol > 0 ? opt.tol : settings().dgemm_tol.load(), &cfg, &cls)) {
      // precision class c -> 8 + 2c moduli; then the configuration class (the split rule needs
      // the modulus count)
      if (forced == 0) nmod = std::min(kCrtMaxModuli, std::max(kCrtMinModuli, 8 + 2 * (cls - kMlpSliceBase)));
      if (auto_tile && cfg >= kCfgCrtCta && cfg <= kCfgCrtSplitK) {
        apply_config(cfg);
        splits = std::min(splits, max_splits);
      }
    }
  }

  CrtGemmArgs g{};
  g.m = m;
  g.n = n;
  g.skip_if_flag = &df->nonfinite;
  g.status = &df->status;
  g.tile_n = tile;
  g.num_sms = cx.num_sms;
  g.cres = ws + o_res_c;
  g.ld_res = m_pad;
  g.tri_k = opt.tri_operand;
  g.group_m = group_m;
  g.splits = splits;
  if (tri) {
    // the tiles meeting the triangle, in the kernel's raster order
    std::vector<int> tiles(static_cast<size_t>(max_tiles));
    int count = 0;
    crt_triangle_tiles(tile, m_pad, n_pad, m, opt.uplo == 1, tuning().group_m, tiles.data(), &count);
    int* dtiles = reinterpret_cast<int*>(ws + o_tiles);
    if (!check_cuda(cudaMemcpyAsync(dtiles, tiles.data(), size_t(count) * 4, cudaMemcpyHostToDevice, st),
                    "tile list"))
      return EB2_ERR_CUDA;
    g.tile_list = dtiles;
    g.num_listed = count;
  }
  CrtReconstructArgs r{};
  r.m = m;
  r.n = n;
  r.alpha = alpha;
  r.beta = beta;
  r.C = C;
  r.ldc = ldc;
  r.cres = ws + o_res_c;
  r.ld_res = m_pad;
  r.plane = int64_t(splits) * m_pad * n_pad;  // the merged residues of modulus l: plane l*splits
  r.mu_a = oa.mu;
  r.mu_b = ob.mu;
  r.err_sq = df->err_sq;
  r.skip_if_flag = &df->nonfinite;
  r.uplo = tri ? opt.uplo : 0;
  r.write_c = true;
  double* const saved = keep_old ? reinterpret_cast<double*>(ws + (tri ? o_full : o_save)) : nullptr;
  r.save = saved;
  r.ld_save = m;
  auto product = [&](bool first) -> bool {
    bool good = split_moduli == nmod || split();
    split_moduli = 0;  // a product redone with more moduli splits again
    g.moduli = r.moduli = nmod;
    if (first && opt.timed) cudaEventRecord(cx.ev_gemm0, st);
    good = good && check_cuda(launch_crt_gemm(oa, ob, g, st), "CRT GEMM");
    if (first && opt.timed) cudaEventRecord(cx.ev_gemm1, st);
    if (splits > 1) {
      good = good && check_cuda(launch_crt_merge_splits(g.cres, m_pad * n_pad, nmod, splits, st), "merge K splits");
      info.launches += 1;
    }
    good = good && check_cuda(launch_crt_reconstruct(r, st), "CRT reconstruction");
    info.launches += 2;
    return good;
  };
  ok = product(true);
  // IEEE semantics for NaN/Inf inputs: the FP64 kernel runs only when the scan saw one
  // (for a triangle into the workspace, then merged into the triangle).
  if (!tri) {
    ok = ok && check_cuda(launch_dgemm_native(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, &df->nonfinite,
                                              st),
                          "non-finite fallback");
    info.launches += 1;
  } else {
    double* full = reinterpret_cast<double*>(ws + o_full);
    ok = ok && check_cuda(launch_dgemm_native(ta, tb, m, n, k, alpha, A, lda, B, ldb, 0.0, full, m, &df->nonfinite,
                                              st),
                          "non-finite fallback");
    ok = ok && check_cuda(launch_merge_triangle<double>(full, m, n, opt.uplo == 1, beta, C, ldc, st, &df->nonfinite),
                          "non-finite merge");
    info.launches += 2;
  }
  if (!ok) return EB2_ERR_CUDA;
  info.slices = nmod;
  info.tile_n = tile;
  call_config().splits = splits;
  call_config().config = splits > 1 ? kCfgCrtSplitK
                           : (tile == kTilePair ? (group_m ? kCfgCrtPairGroup : kCfgCrtPair)
                                                : (group_m ? kCfgCrtCtaGroup : kCfgCrtCta));
  auto finish_timing = [&](bool gemm_timed) {
    if (opt.timed) {
      cudaEventRecord(cx.ev_stop, st);
      set_pending_timing(&cx, gemm_timed);
    }
  };
  if (!opt.sync && !check) {
    finish_timing(true);
    return EB2_OK;
  }

  // ---------------------------------------------------------- a-posteriori check
  const double tol = opt.tol > 0 ? opt.tol : settings().dgemm_tol.load();
  for (;;) {
    if (!check_cuda(cudaMemcpyAsync(cx.hflags, df, sizeof(DeviceFlags), cudaMemcpyDeviceToHost, st), "read flags") ||
        !check_cuda(cudaStreamSynchronize(st), "DGEMM"))
      return EB2_ERR_CUDA;
    const DeviceFlags hf = *cx.hflags;
    info.spread = hf.spread[1] > 0 ? hf.spread[0] / hf.spread[1] : 0.0;
    if (hf.status != 0) {
      set_error(EB2_ERR_TIMEOUT, "a kernel wait timed out (device status 0x%x); C is invalid", hf.status);
      return EB2_ERR_TIMEOUT;
    }
    if (hf.nonfinite) {
      info.nonfinite = 1;
      break;
    }
    // energies that overflowed (products near the FP64 range) leave the estimate unknown
    const bool known = std::isfinite(hf.err_sq[0]) && std::isfinite(hf.err_sq[1]);
    const double est = !known ? -1.0
                       : hf.err_sq[1] > 0.0 ? std::sqrt(hf.err_sq[0] / hf.err_sq[1])
                                            : (hf.err_sq[0] > 0.0 ? HUGE_VAL : 0.0);
    info.err_estimate = est;
    if (!check || !known || est <= tol || nmod + 2 > nmax) {
      if (check && est > tol)
        set_error(EB2_ERR_ACCURACY, "emulated DGEMM estimate %.3g above target %.3g with %d moduli", est, tol, nmod);
      break;
    }
    // two more moduli: b grows by 4 bits, so every residue is recomputed, from the old C
    nmod += 2;
    ++info.escalations;
    info.slices = nmod;
    if (keep_old) {
      const bool restored =
          tri ? check_cuda(launch_merge_triangle<double>(saved, m, n, opt.uplo == 1, 0.0, C, ldc, st, nullptr),
                           "restore C")
              : check_cuda(cudaMemcpy2DAsync(C, size_t(ldc) * 8, saved, size_t(m) * 8, size_t(m) * 8, size_t(n),
                                             cudaMemcpyDeviceToDevice, st),
                           "restore C");
      if (!restored) return EB2_ERR_CUDA;
      info.launches += 1;
    }
    if (!check_cuda(cudaMemsetAsync(df->err_sq, 0, sizeof(df->err_sq), st), "reset estimate") || !product(false))
      return EB2_ERR_CUDA;
  }
  finish_timing(info.escalations == 0);
  return EB2_OK;
}

}  // namespace

int dgemm_on_device(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* A,
                    int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                    cudaStream_t st, const DgemmOptions& opt, eb2_call_info& info) {
  info.dtype = 'd';
  info.slices = 0;
  info.tile_n = 0;
  info.escalations = 0;
  info.nonfinite = 0;
  info.err_estimate = -1.0;
  info.kernel_ms = -1.0;
  info.gemm_kernel_ms = -1.0;
  info.launches = 0;
  info.spread = 0.0;
  call_config().config = -1;
  call_config().splits = 1;
  set_pending_timing(nullptr, false);
  if (m == 0 || n == 0) return EB2_OK;
  if (opt.uplo != 0 && (m != n || opt.method != EB2_METHOD_CRT || k == 0 || alpha == 0.0)) {
    set_error(EB2_ERR_ARG, "a triangle-only product needs m == n, k > 0, alpha != 0 and the CRT method");
    return EB2_ERR_ARG;
  }
  if (k == 0 || alpha == 0.0) {
    info.method = EB2_METHOD_NATIVE;
    if (beta == 1.0) return EB2_OK;
    info.launches = 1;
    return check_cuda(launch_scale_matrix_d(m, n, beta, C, ldc, st), "scale C") ? EB2_OK : EB2_ERR_CUDA;
  }
  int method = opt.method ? opt.method : settings().dgemm_method.load();
  // What is left automatic is decided by a forced configuration class (the tuner), else the
  // learned picker, else the size rule.  Stage 1 here uses the shape only; the CRT path
  // consults the picker again once the scan has measured the data.
  if (method == EB2_METHOD_AUTO) {
    const int fc = forced_config();
    int pick_cfg = -1, pick_s = 0;
    if (fc >= kCfgNative && fc <= kCfgCrtSplitK)
      method = fc == kCfgNative ? EB2_METHOD_NATIVE : EB2_METHOD_CRT;
    else if (picker_weights() != nullptr &&
             picker_predict(m, n, k, 'd', 0.0, 1, opt.tol > 0 ? opt.tol : settings().dgemm_tol.load(), &pick_cfg,
                            &pick_s))
      method = pick_cfg == kCfgNative ? EB2_METHOD_NATIVE : EB2_METHOD_CRT;
    else
      method = auto_method_rule(m, n, k);
  }
  info.method = method;

  auto run_native = [&](bool from_auto) -> int {
    info.method = EB2_METHOD_NATIVE;
    call_config().config = kCfgNative;
    if (opt.timed && !from_auto) cudaEventRecord(cx.ev_start, st);
    if (opt.timed) cudaEventRecord(cx.ev_gemm0, st);
    if (!check_cuda(launch_dgemm_native(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr, st),
                    "native DGEMM"))
      return EB2_ERR_CUDA;
    info.launches += 1;
    if (opt.timed) {
      cudaEventRecord(cx.ev_gemm1, st);
      cudaEventRecord(cx.ev_stop, st);
      set_pending_timing(&cx, true);
    }
    if (opt.sync && !check_cuda(cudaStreamSynchronize(st), "DGEMM")) return EB2_ERR_CUDA;
    return EB2_OK;
  };
  if (method == EB2_METHOD_NATIVE) return run_native(false);
  if (opt.timed) cudaEventRecord(cx.ev_start, st);
  if (method == EB2_METHOD_CRT)
    return dgemm_crt(cx, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st, opt, info);

  // ---------------------------------------------------------- Ozaki emulation
  // Workspace: scan results first (they must survive the stage-2 decision), then the
  // exponents and digit panels, sized for the largest tile padding and slice count the
  // decision can pick.
  const bool check = opt.check_accuracy;
  const int s_fixed = opt.slices ? opt.slices : choose_slices(m, n, k);
  const int smax = check ? kOzakiMaxSlices : std::max(s_fixed, 8);
  const int64_t m_cap = round_up(m, 256), n_cap = round_up(n, 256), k_pad = round_up(k, kOzakiKBlock);
  size_t off = 0;
  const size_t o_mb_a = off;
  off = align256(off + size_t(m) * 8);
  const size_t o_mb_b = off;
  off = align256(off + size_t(n) * 8);
  const size_t o_exp_a = off;
  off = align256(off + size_t(m_cap) * 4);
  const size_t o_exp_b = off;
  off = align256(off + size_t(n_cap) * 4);
  const size_t o_dig_a = off;
  off = align256(off + size_t(smax) * m_cap * k_pad);
  const size_t o_dig_b = off;
  off = align256(off + size_t(smax) * n_cap * k_pad);
  if (const int rc = reserve_buffer(cx.ws, off, st, "emulation workspace"); rc != EB2_OK) return rc;
  uint8_t* ws = static_cast<uint8_t*>(cx.ws.ptr);
  const StridedView<double> va = view_a(ta, A, lda, m, k);
  const StridedView<double> vb = view_bt(tb, B, ldb, n, k);
  DeviceFlags* df = cx.dflags;
  OzakiOperand oa{reinterpret_cast<int8_t*>(ws + o_dig_a), reinterpret_cast<int32_t*>(ws + o_exp_a),
                  reinterpret_cast<uint64_t*>(ws + o_mb_a), nullptr, m, m_cap, k, k_pad, smax};
  OzakiOperand ob{reinterpret_cast<int8_t*>(ws + o_dig_b), reinterpret_cast<int32_t*>(ws + o_exp_b),
                  reinterpret_cast<uint64_t*>(ws + o_mb_b), nullptr, n, n_cap, k, k_pad, smax};

  bool ok = check_cuda(cudaMemsetAsync(df, 0, sizeof(DeviceFlags), st), "reset flags");
  ok = ok && check_cuda(launch_ozaki_scan_reset(oa, st), "scan reset A");
  ok = ok && check_cuda(launch_ozaki_scan_reset(ob, st), "scan reset B");
  ok = ok && check_cuda(launch_ozaki_scan(va, oa, &df->nonfinite, &df->spread[0], st), "scan A");
  ok = ok && check_cuda(launch_ozaki_scan(vb, ob, &df->nonfinite, &df->spread[0], st), "scan B");
  if (!ok) return EB2_ERR_CUDA;
  info.launches = 2;

  // The digit-slice form is an explicit method: tile and starting digit count from the size
  // rules (the picker's precision head counts CRT moduli); the a-posteriori check adds digits.
  const int tile_n = opt.tile_n ? opt.tile_n : choose_tile_n(cx, m, n, true);
  int s = s_fixed;
  const int64_t m_pad = round_up(m, tile_m_of(tile_n, true)), n_pad = round_up(n, tile_n_of(tile_n, true));
  oa.rows_pad = m_pad;
  ob.rows_pad = n_pad;
  ok = ok && check_cuda(launch_ozaki_split(va, oa, 0, s, st), "split A");
  ok = ok && check_cuda(launch_ozaki_split(vb, ob, 0, s, st), "split B");
  OzakiGemmArgs g{};
  g.m = m;
  g.n = n;
  g.k = k;
  g.alpha = alpha;
  g.beta = beta;
  g.C = C;
  g.ldc = ldc;
  g.slices = s;
  g.diag_lo = 2;
  g.diag_hi = s + 1;
  g.first_writes = true;
  g.skip_if_flag = &df->nonfinite;
  g.err_sq = df->err_sq;
  g.status = &df->status;
  g.tile_n = tile_n;
  g.num_sms = cx.num_sms;
  if (opt.timed) cudaEventRecord(cx.ev_gemm0, st);
  ok = ok && check_cuda(launch_ozaki_gemm(oa, ob, g, st), "Ozaki GEMM");
  if (opt.timed) cudaEventRecord(cx.ev_gemm1, st);
  // IEEE semantics for NaN/Inf inputs: the FP64 kernel runs only when the scan saw one.
  ok = ok && check_cuda(launch_dgemm_native(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, &df->nonfinite,
                                            st),
                        "non-finite fallback");
  if (!ok) return EB2_ERR_CUDA;
  info.launches += 4;  // 2 splits, GEMM, non-finite fallback (exits at once when unused)
  if (opt.timed) {
    cudaEventRecord(cx.ev_stop, st);
    set_pending_timing(&cx, true);
  }
  info.slices = s;
  info.tile_n = tile_n;
  if (!opt.sync && !check) return EB2_OK;

  // ---------------------------------------------------------- a-posteriori check
  const double tol = opt.tol > 0 ? opt.tol : settings().dgemm_tol.load();
  double lo_energy = 0.0;
  for (;;) {
    if (!check_cuda(cudaMemcpyAsync(cx.hflags, df, sizeof(DeviceFlags), cudaMemcpyDeviceToHost, st), "read flags") ||
        !check_cuda(cudaStreamSynchronize(st), "DGEMM"))
      return EB2_ERR_CUDA;
    const DeviceFlags hf = *cx.hflags;
    info.spread = hf.spread[1] > 0 ? hf.spread[0] / hf.spread[1] : 0.0;
    if (hf.status != 0) {
      set_error(EB2_ERR_TIMEOUT, "a kernel wait timed out (device status 0x%x); C is invalid", hf.status);
      return EB2_ERR_TIMEOUT;
    }
    if (hf.nonfinite) {
      info.nonfinite = 1;
      break;
    }
    if (info.escalations == 0) lo_energy = hf.err_sq[1];
    const double est = lo_energy > 0.0 ? std::sqrt(hf.err_sq[0] / lo_energy) * std::ldexp(1.0, -7) *
                                             std::sqrt(double(s + 1) / double(s))
                                       : 0.0;
    info.err_estimate = est;
    if (!check || est <= tol) break;
    if (s >= smax) {
      set_error(EB2_ERR_ACCURACY, "emulated DGEMM estimate %.3g above target %.3g at %d slices", est, tol, s);
      break;
    }
    // add digit s+1 of both operands and the diagonal t = s+2 (pairs p+q = s+2)
    ok = check_cuda(cudaMemsetAsync(df->err_sq, 0, sizeof(double), st), "reset estimate");
    ok = ok && check_cuda(launch_ozaki_split(va, oa, s, s + 1, st), "split A");
    ok = ok && check_cuda(launch_ozaki_split(vb, ob, s, s + 1, st), "split B");
    g.slices = s + 1;
    g.diag_lo = g.diag_hi = s + 2;
    g.first_writes = false;
    ok = ok && check_cuda(launch_ozaki_gemm(oa, ob, g, st), "Ozaki GEMM (added slice)");
    if (!ok) return EB2_ERR_CUDA;
    info.launches += 3;
    if (opt.timed) {
      cudaEventRecord(cx.ev_stop, st);
      set_pending_timing(&cx, false);  // the GEMM events cover only the first pass
    }
    ++s;
    ++info.escalations;
    info.slices = s;
  }
  return EB2_OK;
}

int sgemm_on_device(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, float alpha, const float* A,
                    int64_t lda, const float* B, int64_t ldb, float beta, float* C, int64_t ldc, cudaStream_t st,
                    const SgemmOptions& opt, eb2_call_info& info) {
  info.dtype = 's';
  info.slices = 0;
  info.tile_n = 0;
  info.escalations = 0;
  info.nonfinite = 0;
  info.err_estimate = -1.0;
  info.kernel_ms = -1.0;
  info.gemm_kernel_ms = -1.0;
  info.launches = 0;
  call_config().config = -1;
  call_config().splits = 1;
  set_pending_timing(nullptr, false);
  if (m == 0 || n == 0) return EB2_OK;
  if (k == 0 || alpha == 0.0f) {
    info.method = EB2_METHOD_NATIVE;
    if (beta == 1.0f) return EB2_OK;
    info.launches = 1;
    return check_cuda(launch_scale_matrix_s(m, n, beta, C, ldc, st), "scale C") ? EB2_OK : EB2_ERR_CUDA;
  }
  int method = opt.method ? opt.method : settings().sgemm_method.load();
  int cfg_tile = 0;  // tile of an automatic split-BF16 choice (0: the size rule)
  if (method == EB2_METHOD_AUTO) {
    // a forced configuration class (the tuner), else the learned picker, else split-BF16
    const int fc = forced_config();
    int cfg = -1, cls = 0;
    if (fc >= kCfgSgemmFfma && fc <= kCfgSgemmBf16Pair)
      cfg = fc;
    else if (picker_weights() == nullptr || !picker_predict(m, n, k, 's', 0.0, 1, kSgemmTolFeature, &cfg, &cls))
      cfg = -1;
    method = cfg == kCfgSgemmFfma ? EB2_METHOD_NATIVE : EB2_METHOD_EMULATED;
    if (cfg > kCfgSgemmFfma) cfg_tile = cfg == kCfgSgemmBf16_128 ? 128 : (cfg == kCfgSgemmBf16_256 ? 256 : kTilePair);
  }
  info.method = method;
  if (opt.timed) cudaEventRecord(cx.ev_start, st);
  if (method == EB2_METHOD_NATIVE) {
    call_config().config = kCfgSgemmFfma;
    if (opt.timed) cudaEventRecord(cx.ev_gemm0, st);
    if (!check_cuda(launch_sgemm_native(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, nullptr, st),
                    "native SGEMM"))
      return EB2_ERR_CUDA;
    info.launches = 1;
    if (opt.timed) {
      cudaEventRecord(cx.ev_gemm1, st);
      cudaEventRecord(cx.ev_stop, st);
      set_pending_timing(&cx, true);
    }
    if (opt.sync && !check_cuda(cudaStreamSynchronize(st), "SGEMM")) return EB2_ERR_CUDA;
    return EB2_OK;
  }

  // ---------------------------------------------------------- split-BF16 emulation
  const int tile_n = opt.tile_n ? opt.tile_n
                                : (cfg_tile && settings().tile_n.load() == 0 ? cfg_tile : choose_tile_n(cx, m, n, false));
  call_config().config = tile_n == 128 ? kCfgSgemmBf16_128 : (tile_n == 256 ? kCfgSgemmBf16_256 : kCfgSgemmBf16Pair);
  const int pieces = opt.pieces ? opt.pieces : settings().sgemm_pieces.load();
  const int64_t m_pad = round_up(m, tile_m_of(tile_n, false)), n_pad = round_up(n, tile_n_of(tile_n, false)),
                k_pad = round_up(k, 64);
  size_t off = 0;
  const size_t o_a = off;
  off = align256(off + size_t(3) * m_pad * k_pad * 2);
  const size_t o_b = off;
  off = align256(off + size_t(3) * n_pad * k_pad * 2);
  if (const int rc = reserve_buffer(cx.ws, off, st, "emulation workspace"); rc != EB2_OK) return rc;
  uint8_t* ws = static_cast<uint8_t*>(cx.ws.ptr);
  Bf16Operand oa{ws + o_a, m, m_pad, k, k_pad};
  Bf16Operand ob{ws + o_b, n, n_pad, k, k_pad};
  const StridedView<float> va = ta ? StridedView<float>{A, m, k, lda, 1} : StridedView<float>{A, m, k, 1, lda};
  const StridedView<float> vb = tb ? StridedView<float>{B, n, k, 1, ldb} : StridedView<float>{B, n, k, ldb, 1};
  DeviceFlags* df = cx.dflags;
  bool ok = check_cuda(cudaMemsetAsync(df, 0, sizeof(DeviceFlags), st), "reset flags");
  ok = ok && check_cuda(launch_bf16_split(va, oa, &df->nonfinite, st), "split A");
  ok = ok && check_cuda(launch_bf16_split(vb, ob, &df->nonfinite, st), "split B");
  SgemmSplitArgs g{};
  g.m = m;
  g.n = n;
  g.k = k;
  g.alpha = alpha;
  g.beta = beta;
  g.C = C;
  g.ldc = ldc;
  g.pieces = pieces;
  g.skip_if_flag = &df->nonfinite;
  g.status = &df->status;
  g.tile_n = tile_n;
  g.num_sms = cx.num_sms;
  if (opt.timed) cudaEventRecord(cx.ev_gemm0, st);
  ok = ok && check_cuda(launch_sgemm_split_bf16(oa, ob, g, st), "split-BF16 GEMM");
  if (opt.timed) cudaEventRecord(cx.ev_gemm1, st);
  ok = ok && check_cuda(launch_sgemm_native(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, &df->nonfinite, st),
                        "non-finite fallback");
  if (!ok) return EB2_ERR_CUDA;
  info.launches = 4;  // 2 splits, GEMM, non-finite fallback (exits at once when unused)
  info.slices = pieces * (pieces + 1) / 2;
  info.tile_n = tile_n;
  if (opt.timed) {
    cudaEventRecord(cx.ev_stop, st);
    set_pending_timing(&cx, true);
  }
  if (!opt.sync) return EB2_OK;
  if (!check_cuda(cudaMemcpyAsync(cx.hflags, df, sizeof(DeviceFlags), cudaMemcpyDeviceToHost, st), "read flags") ||
      !check_cuda(cudaStreamSynchronize(st), "SGEMM"))
    return EB2_ERR_CUDA;
  if (cx.hflags->status != 0) {
    set_error(EB2_ERR_TIMEOUT, "a kernel wait timed out (device status 0x%x); C is invalid", cx.hflags->status);
    return EB2_ERR_TIMEOUT;
  }
  info.nonfinite = cx.hflags->nonfinite ? 1 : 0;
  return EB2_OK;
}

}  // namespace eb2
