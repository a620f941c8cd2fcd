// crt_pipeline.cpp -- the BLAS entry's DGEMM on host buffers, pipelined by column blocks.
//
// When A, B and C all live in host memory (Eigen's own matrices) the copies over PCIe take
// longer than the product.  Here they overlap with it:
//   copy-in stream : A, then B (and C when beta != 0) one column block at a time;
//   compute stream : once A has arrived, its scan, norm bounds and residues (once); then per
//                    block of columns j0..j1 of C: the block's B rows, the INT8 GEMM of all
//                    moduli and the reconstruction of C[:, j0:j1];
//   copy-out stream: C[:, j0:j1] back to the host as soon as its block is done and checked.
// PCIe is full duplex, so block c goes out while block c+2 comes in.  The a-posteriori
// check is made per block: if every block meets ||E_c||_F <= tol ||alpha A B_c||_F, the
// whole product meets the same target.  A block that misses it is redone by the ordinary
// device path (which adds moduli) from the host's C, which is not touched before the
// block's result is final; the blocks after it then take the ordinary path too.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "context.h"
#include "gemm_driver.h"
#include "host_stager.h"
#include "mlp.h"
#include "kernels.h"

namespace eb2 {
namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

bool check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  (void)cudaGetLastError();
  set_error(EB2_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return false;
}

constexpr int64_t kBlockCols = 1024;  // target columns per block (rounded to the 256-column tile)

}  // namespace

bool crt_pipeline_applies(const Context& cx, int64_t m, int64_t n, int64_t k, int method) {
  (void)cx;
  return method == EB2_METHOD_CRT && n >= 2 * 512 && m >= 256 && k >= 256;
}

int dgemm_crt_pipelined(Context& cx, bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                        const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                        int64_t ldc, eb2_call_info& info) {
  const int nblocks = int(std::min<int64_t>(Context::kPipeChunks, std::max<int64_t>(2, (n + kBlockCols - 1) / kBlockCols)));
  const int64_t nc = round_up((n + nblocks - 1) / nblocks, 256);
  const int nb = int((n + nc - 1) / nc);
  const int forced = settings().dgemm_moduli.load();
  const int nmod = forced ? forced : kCrtDefaultModuli;
  const double tol = settings().dgemm_tol.load();
  const int64_t m_pad = round_up(m, 256), nc_pad = round_up(nc, 256), k_pad = round_up(k, kOzakiKBlock);

  // staging: the whole of A, B and C, so no block overwrites data still in use
  const int64_t a_rows = ta ? k : m, a_cols = ta ? m : k;
  const int64_t b_rows = tb ? n : k, b_cols = tb ? k : n;
  if (!cx.stage_a.ensure(size_t(a_rows) * a_cols * 8) || !cx.stage_b.ensure(size_t(b_rows) * b_cols * 8) ||
      !cx.stage_c.ensure(size_t(m) * n * 8)) {
    set_error(EB2_ERR_ALLOC, "could not allocate staging memory");
    return EB2_ERR_ALLOC;
  }
  // workspace: A's scan/norm/residues, one block of B, one block of C' residues, estimates
  size_t off = 0;
  auto take = [&off](size_t bytes) {
    const size_t o = off;
    off = align256(off + bytes);
    return o;
  };
  const int64_t nchunks = k_pad / kOzakiKBlock;  // 128-column chunks of the norm bounds
  const size_t o_mb_a = take(size_t(m) * 8), o_ss_a = take(size_t(m) * nchunks * 8),
               o_ce_a = take(size_t(m) * nchunks * 4), o_mu_a = take(size_t(m_pad) * 4);
  const size_t o_res_a = take(size_t(nmod) * m_pad * k_pad);
  const size_t o_mb_b = take(size_t(nc) * 8), o_ss_b = take(size_t(nc) * nchunks * 8),
               o_ce_b = take(size_t(nc) * nchunks * 4), o_mu_b = take(size_t(nc_pad) * 4);
  const size_t o_res_b = take(size_t(nmod) * nc_pad * k_pad);
  const size_t o_res_c = take(size_t(nmod) * m_pad * nc_pad);
  const size_t o_est = take(sizeof(double) * 2 * Context::kPipeChunks);
  if (!cx.ws.ensure(off)) {
    set_error(EB2_ERR_ALLOC, "could not allocate %zu bytes of emulation workspace", off);
    return EB2_ERR_ALLOC;
  }
  uint8_t* ws = static_cast<uint8_t*>(cx.ws.ptr);
  double* d_est = reinterpret_cast<double*>(ws + o_est);
  double* dA = static_cast<double*>(cx.stage_a.ptr);
  double* dB = static_cast<double*>(cx.stage_b.ptr);
  double* dC = static_cast<double*>(cx.stage_c.ptr);
  cudaStream_t st = cx.stream, cin = cx.copy_in, cout = cx.copy_out;
  DeviceFlags* df = cx.dflags;

  info.dtype = 'd';
  info.method = EB2_METHOD_CRT;
  info.slices = nmod;
  info.staged = 1;
  info.launches = 0;
  info.escalations = 0;
  info.err_estimate = 0.0;

  // ------------------------------------------------ copy-in: A, then B (and C) by blocks
  // Pinned sources are enqueued at once; pageable ones go through the stager's bounce buffers
  // (the host copies a block while the device works on the ones before it), a few blocks ahead.
  HostStager& hs = cx.stager;
  const bool all_pinned = HostStager::pinned(A) && HostStager::pinned(B) && (beta == 0.0 || HostStager::pinned(C));
  const int lookahead = all_pinned ? nb : 2;
  if (!check_cuda(hs.to_device(dA, a_rows * 8, A, lda * 8, a_rows * 8, a_cols, cin), "copy A") ||
      !check_cuda(cudaEventRecord(cx.ev_a, cin), "event"))
    return EB2_ERR_CUDA;
  int staged = 0;  // blocks whose copies are enqueued
  auto stage_block = [&](int c) -> bool {
    const int64_t j0 = c * nc, w = std::min(nc, n - j0);
    // op(B)(:, j0:j0+w) is B(:, j0:...) (N) or B(j0:..., :) (T); staged with ld = b_rows
    const bool okb = tb ? check_cuda(hs.to_device(dB + j0, b_rows * 8, B + j0, ldb * 8, w * 8, k, cin), "copy B")
                        : check_cuda(hs.to_device(dB + j0 * b_rows, b_rows * 8, B + j0 * ldb, ldb * 8, k * 8, w, cin),
                                     "copy B");
    // beta == 0 never reads C (blas/level3_impl.h:82-84)
    const bool okc =
        beta == 0.0 || check_cuda(hs.to_device(dC + j0 * m, m * 8, C + j0 * ldc, ldc * 8, m * 8, w, cin), "copy C");
    return okb && okc && check_cuda(cudaEventRecord(cx.ev_in[c], cin), "event");
  };
  while (staged < std::min(nb, lookahead))
    if (!stage_block(staged++)) return EB2_ERR_CUDA;

  // ------------------------------------------------ compute: A once
  const StridedView<double> va = ta ? StridedView<double>{dA, m, k, a_rows, 1} : StridedView<double>{dA, m, k, 1, a_rows};
  CrtOperand oa{reinterpret_cast<int8_t*>(ws + o_res_a), reinterpret_cast<int32_t*>(ws + o_mu_a),
                reinterpret_cast<uint64_t*>(ws + o_mb_a), reinterpret_cast<uint64_t*>(ws + o_ss_a),
                reinterpret_cast<int32_t*>(ws + o_ce_a), m, m_pad, k, k_pad, nmod};
  bool ok = check_cuda(cudaMemsetAsync(df, 0, sizeof(DeviceFlags), st), "reset flags");
  ok = ok && check_cuda(cudaMemsetAsync(d_est, 0, sizeof(double) * 2 * Context::kPipeChunks, st), "reset estimates");
  ok = ok && check_cuda(cudaStreamWaitEvent(st, cx.ev_a, 0), "wait A");
  cudaEventRecord(cx.ev_start, st);
  ok = ok && check_cuda(launch_crt_scan_norms(va, oa, &df->nonfinite, &df->spread[0], st), "scan A");
  ok = ok && check_cuda(launch_crt_split(va, oa, nmod, st), "residues A");
  if (!ok) return EB2_ERR_CUDA;
  info.launches += 3;

  CrtOperand ob{reinterpret_cast<int8_t*>(ws + o_res_b), reinterpret_cast<int32_t*>(ws + o_mu_b),
                reinterpret_cast<uint64_t*>(ws + o_mb_b), reinterpret_cast<uint64_t*>(ws + o_ss_b),
                reinterpret_cast<int32_t*>(ws + o_ce_b), nc, nc_pad, k, k_pad, nmod};
  bool degraded = false;  // a block missed the target: the rest takes the ordinary path

  // the ordinary device path for block c (adds moduli as needed), C block restored first
  auto ordinary_block = [&](int c) -> int {
    const int64_t j0 = c * nc, w = std::min(nc, n - j0);
    while (staged <= c)  // its B block
      if (!stage_block(staged++)) return EB2_ERR_CUDA;
    if (!check_cuda(cudaStreamWaitEvent(st, cx.ev_in[c], 0), "wait block") ||
        !check_cuda(cudaStreamSynchronize(st), "DGEMM") ||
        (beta != 0.0 &&
         !check_cuda(hs.to_device(dC + j0 * m, m * 8, C + j0 * ldc, ldc * 8, m * 8, w, st), "restore C")))
      return EB2_ERR_CUDA;
    const double* bblk = tb ? dB + j0 : dB + j0 * b_rows;
    DgemmOptions o;
    o.method = EB2_METHOD_CRT;
    o.sync = true;
    o.check_accuracy = true;
    eb2_call_info sub{};
    const int rc = dgemm_on_device(cx, ta, tb, m, w, k, alpha, dA, a_rows, bblk, b_rows, beta, dC + j0 * m, m, st,
                                   o, sub);
    info.escalations = std::max(info.escalations, sub.escalations);
    info.slices = std::max(info.slices, sub.slices);
    info.err_estimate = std::max(info.err_estimate, sub.err_estimate);
    info.launches += sub.launches;
    info.nonfinite |= sub.nonfinite;
    if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) return rc;
    if (!check_cuda(cudaEventRecord(cx.ev_done[c], st), "event")) return EB2_ERR_CUDA;
    return rc;
  };

  // block c is done on the device: check it, then send it to the host (or redo it)
  int rc_all = EB2_OK;
  auto finish_block = [&](int c) -> int {
    if (!check_cuda(cudaEventSynchronize(cx.ev_done[c]), "DGEMM")) return EB2_ERR_CUDA;
    const DeviceFlags hf = *cx.hflags;  // snapshot taken after this block (flags only accumulate)
    if (hf.status != 0) {
      set_error(EB2_ERR_TIMEOUT, "a kernel wait timed out (device status 0x%x); C is invalid", hf.status);
      return EB2_ERR_TIMEOUT;
    }
    info.nonfinite |= hf.nonfinite ? 1 : 0;
    const double e0 = cx.hchunk[2 * c], e1 = cx.hchunk[2 * c + 1];
    const bool known = std::isfinite(e0) && std::isfinite(e1);
    const double est = !known ? -1.0 : (e1 > 0.0 ? std::sqrt(e0 / e1) : (e0 > 0.0 ? HUGE_VAL : 0.0));
    if (!hf.nonfinite && known && est > tol) {
      degraded = true;
      const int rc = ordinary_block(c);
      if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) return rc;
      if (rc == EB2_ERR_ACCURACY) rc_all = rc;
    } else {
      info.err_estimate = std::max(info.err_estimate, est);
    }
    const int64_t j0 = c * nc, w = std::min(nc, n - j0);
    if (!check_cuda(cudaStreamWaitEvent(cout, cx.ev_done[c], 0), "wait block") ||
        !check_cuda(hs.to_host(C + j0 * ldc, ldc * 8, dC + j0 * m, m * 8, m * 8, w, cout), "copy C out"))
      return EB2_ERR_CUDA;
    return EB2_OK;
  };

  // ------------------------------------------------ compute: block by block
  int pending = -1;  // the block enqueued last and not yet checked
  for (int c = 0; c < nb; ++c) {
    const int64_t j0 = c * nc, w = std::min(nc, n - j0);
    if (degraded) {
      if (pending >= 0) {  // enqueued before the miss: its result is valid, check it
        const int rc = finish_block(pending);
        pending = -1;
        if (rc != EB2_OK) return rc;
      }
      const int rc = ordinary_block(c);
      if (rc != EB2_OK && rc != EB2_ERR_ACCURACY) return rc;
      if (rc == EB2_ERR_ACCURACY) rc_all = rc;
      const int64_t jj = c * nc;
      if (!check_cuda(cudaStreamWaitEvent(cout, cx.ev_done[c], 0), "wait block") ||
          !check_cuda(hs.to_host(C + jj * ldc, ldc * 8, dC + jj * m, m * 8, m * 8, w, cout), "copy C out"))
        return EB2_ERR_CUDA;
      continue;
    }
    while (staged <= c)
      if (!stage_block(staged++)) return EB2_ERR_CUDA;
    const double* bblk = tb ? dB + j0 : dB + j0 * b_rows;
    const StridedView<double> vb =
        tb ? StridedView<double>{bblk, w, k, 1, b_rows} : StridedView<double>{bblk, w, k, b_rows, 1};
    ob.rows = w;
    const int tile = choose_crt_tile(cx, m, w);
    ok = check_cuda(cudaStreamWaitEvent(st, cx.ev_in[c], 0), "wait B block");
    ok = ok && check_cuda(launch_crt_scan_norms(vb, ob, &df->nonfinite, &df->spread[0], st), "scan B");
    ok = ok && check_cuda(launch_crt_split(vb, ob, nmod, st), "residues B");
    CrtGemmArgs g{};
    g.m = m;
    g.n = w;
    g.moduli = nmod;
    g.skip_if_flag = &df->nonfinite;
    g.status = &df->status;
    g.tile_n = tile;
    g.num_sms = cx.num_sms;
    g.cres = ws + o_res_c;
    g.ld_res = m_pad;
    ok = ok && check_cuda(launch_crt_gemm(oa, ob, g, st), "CRT GEMM");
    CrtReconstructArgs r{};
    r.m = m;
    r.n = w;
    r.alpha = alpha;
    r.beta = beta;
    r.C = dC + j0 * m;
    r.ldc = m;
    r.cres = ws + o_res_c;
    r.ld_res = m_pad;
    r.plane = m_pad * nc_pad;
    r.moduli = nmod;
    r.mu_a = oa.mu;
    r.mu_b = ob.mu;
    r.err_sq = d_est + 2 * c;
    r.skip_if_flag = &df->nonfinite;
    r.write_c = true;
    ok = ok && check_cuda(launch_crt_reconstruct(r, st), "CRT reconstruction");
    // IEEE semantics for NaN/Inf inputs: the FP64 kernel runs only when a scan saw one
    ok = ok && check_cuda(launch_dgemm_native(ta, tb, m, w, k, alpha, dA, a_rows, bblk, b_rows, beta, dC + j0 * m, m,
                                              &df->nonfinite, st),
                          "non-finite fallback");
    ok = ok && check_cuda(cudaMemcpyAsync(cx.hchunk + 2 * c, d_est + 2 * c, 2 * sizeof(double),
                                          cudaMemcpyDeviceToHost, st), "read estimate");
    ok = ok && check_cuda(cudaMemcpyAsync(cx.hflags, df, sizeof(DeviceFlags), cudaMemcpyDeviceToHost, st), "read flags");
    ok = ok && check_cuda(cudaEventRecord(cx.ev_done[c], st), "event");
    if (!ok) return EB2_ERR_CUDA;
    info.launches += 8;
    // while the device computes this block: the host side of the next input block's copies
    if (staged < nb && staged < c + 1 + lookahead && !stage_block(staged++)) return EB2_ERR_CUDA;
    if (pending >= 0) {  // check the previous block while this one runs
      const int rc = finish_block(pending);
      if (rc != EB2_OK) return rc;
    }
    if (!check_cuda(hs.progress(), "copy C out")) return EB2_ERR_CUDA;
    pending = c;
  }
  if (pending >= 0) {
    const int rc = finish_block(pending);
    if (rc != EB2_OK) return rc;
  }
  cudaEventRecord(cx.ev_stop, st);
  set_pending_timing(&cx, false);
  if (!check_cuda(hs.drain(), "copy C out") || !check_cuda(cudaStreamSynchronize(cout), "copy C") ||
      !check_cuda(cudaStreamSynchronize(st), "DGEMM"))
    return EB2_ERR_CUDA;
  info.tile_n = choose_crt_tile(cx, m, nc);
  call_config().config = info.tile_n == kTilePair ? kCfgCrtPair : kCfgCrtCta;
  call_config().splits = 1;
  if (rc_all == EB2_ERR_ACCURACY)
    set_error(EB2_ERR_ACCURACY, "emulated DGEMM estimate above target %.3g in a column block", tol);
  return rc_all;
}

}  // namespace eb2
