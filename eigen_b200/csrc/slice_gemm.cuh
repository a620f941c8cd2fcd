// slice_gemm.cuh -- the persistent, warp-specialised tcgen05 GEMM over "slices".
//
// Both emulated products reduce to sums of slice products  A_p * B_q^T  over the
// triangle p + q <= s + 1 (p, q = 1..s):
//   * Ozaki DGEMM: A_p, B_q are INT8 digit panels; every diagonal t = p + q has its
//     own power-of-two weight, so each diagonal is an exact INT32 accumulation in TMEM;
//     the epilogue scales it exactly to FP64 and adds it into a per-thread FP64 register
//     accumulator, writing C once per tile: C = alpha * sum_t D_t 2^(e_i+f_j+w_t) (+ beta C);
//   * split-BF16 SGEMM: A_p, B_q are the hi/mid/lo BF16 pieces of the FP32 inputs;
//     the pieces carry their own exponents, so all of the triangle's products over a chunk
//     of K accumulate into one FP32 TMEM accumulator; the epilogue adds the chunks into
//     FP32 registers (round to nearest) and applies alpha/beta once per tile.
//
// Roles: warp 0 = TMA producer, warp 1 = MMA issuer + TMEM owner, warps 2.. = epilogue
// (NW warps; warp w may read TMEM lanes 32*(w%4)..+31, one output row per thread).
// Operand panels are K-major and zero-padded by the split kernels, loaded as 128-byte
// swizzled tiles and consumed by tcgen05.mma with K = 32 bytes per instruction.  Two TMEM
// accumulators alternate so the epilogue of one unit overlaps the MMAs of the next.
//
// PAIR = a cluster of two CTAs computes a (2*128) x BN tile with tcgen05 cta_group::2:
// each CTA loads its 128 rows of A and BN/2 of the BN rows of B per stage and holds its
// 128 x BN half of the accumulator in its own TMEM; the leader (rank 0) issues the
// M = 256 MMAs and commits separately to both CTAs' barriers.  No TMA multicast.
// Every mbarrier wait is bounded (device_common.cuh).
#pragma once
#include <cuda.h>

#include <climits>
#include <cstdint>

#include "device_common.cuh"
#include "kernels.h"

namespace eb2 {

enum SliceMode : int { kModeOzakiI8 = 0, kModeSplitBF16 = 1, kModeCrtI8 = 2, kModeCrtI8Listed = 3 };
// kModeCrtI8Listed: the CRT product over the tiles of P.tile_list only (a separate
// instantiation, so the ordinary CRT kernel carries no list lookup)
__host__ __device__ constexpr bool is_crt_mode(int mode) { return mode == kModeCrtI8 || mode == kModeCrtI8Listed; }

constexpr int kSliceBM = 128;      // rows of A per CTA (TMEM lanes)
constexpr int kSliceKBytes = 128;  // bytes of K per pipeline stage
// One Ozaki accumulation unit covers at most this many 128-deep digit blocks per
// output: 4095 * 128 * 64 * 64 < 2^31, so the INT32 accumulator cannot overflow.
constexpr int kMaxUnitKb = 4095;
// CRT residues lie in [-128, 127]: 1023 * 128 * 128 * 128 < 2^31.
constexpr int kMaxUnitKbCrt = 1023;
// Split-BF16: K blocks (64 bf16 each) per FP32 accumulation unit.  The tensor core's FP32
// accumulation is not a round-to-nearest sum: its error grows with the number of MMAs that
// add into one accumulator and with the accumulator's magnitude.  So every 256 elements of K
// the unit's sum (all pieces' products over those K) leaves TMEM and is added, rounded to
// nearest, into FP32 registers of the epilogue; the accumulator restarts from zero.
constexpr int kBf16ChunkKb = 4;

// MT: row tiles of 128 per CTA (1, or 2 for the one-CTA 256-row tile of the CRT GEMM: two
// M = 128 MMAs per K step share the B tile, and the accumulator fills the whole TMEM).
template <int BN, int STAGES, bool PAIR, int MT = 1>
struct SliceLayout {
  static constexpr int kBRows = PAIR ? BN / 2 : BN;  // rows of B loaded by one CTA
  static constexpr int kABytes = MT * kSliceBM * kSliceKBytes;
  static constexpr int kBBytes = kBRows * kSliceKBytes;
  static constexpr int kAOff = 0;
  static constexpr int kBOff = kAOff + STAGES * kABytes;
  static constexpr int kBarOff = kBOff + STAGES * kBBytes;
  // full[STAGES], empty[STAGES], tfull[2], tempty[2], drain
  static constexpr int kNumBars = 2 * STAGES + 5;
  static constexpr int kMiscOff = kBarOff + kNumBars * 8;
  static constexpr int kColExpOff = kMiscOff + 16;
  static constexpr int kTotal = kColExpOff + BN * 4;
  static constexpr int kAlloc = kTotal + 1024;  // slack for 1024-byte alignment
  static_assert(kAlloc <= 227 * 1024, "shared memory budget");
};

struct SliceGemmParams {
  int64_t m, n;
  int num_kb;            // K blocks of kSliceKBytes
  int tiles_m, tiles_n;  // tiles of (PAIR ? 256 : 128) x BN
  int slices;            // s
  int diag_lo, diag_hi;  // diagonals t = p + q processed, from diag_hi down to diag_lo
  int first_writes;      // 1: C = alpha*acc (+ beta*C); 0: C += alpha*acc
  double alpha, beta;    // Ozaki (FP64 output)
  float alpha_f, beta_f; // split-BF16 (FP32 output)
  void* C;
  int64_t ldc;
  const int32_t* expA;   // Ozaki row / column exponents
  const int32_t* expB;
  const int* skip_if_flag;
  double* err_sq;        // Ozaki: [0] += energy of diagonal diag_hi, [1] += energy of diagonal 2
  uint32_t* status;
  int group_m;           // row-tiles per raster group (>= tiles_m: column-major tile order)
  int crt;               // 1: CRT mode (unit t = modulus t, one slice pair (t, t))
  uint8_t* residues;     // CRT: [moduli][cols][ld_res] residue planes (uint8 in [0, p))
  int64_t ld_res;        // CRT: rows of one residue plane (padded m)
  const int* tile_list;  // CRT: the tiles to compute (indices of the full raster), or null for all
  int num_listed;        // CRT: entries of tile_list
  int tri_k;             // CRT: 1 = op(A) lower, 2 = op(A) upper, 3 = op(B) lower, 4 = op(B) upper
                         // triangular (zero blocks of K skipped per tile); 0 = dense
  uint64_t wait_limit_ns;  // wall-time bound of the pipeline waits (the drain waits keep kWaitLimitNs)
  int splits;            // CRT: K ranges per (tile, modulus), each with its own residue plane (1: none)
};

// Pair range of diagonal t: p = p_lo .. p_lo + total/num_kb - 1 (q = t - p).
// In CRT mode "diagonal" t is modulus t with the single pair (t, t): p_lo = t + 1 and
// the B slice is t (see b_slice()).
__device__ __forceinline__ bool diag_bounds(int t, int s, int num_kb, int& p_lo, int& total, bool crt = false) {
  if (crt) {
    p_lo = t + 1;
    total = num_kb;
    return t >= 0 && t < s;
  }
  p_lo = max(1, t - s);
  const int p_hi = min(s, t - 1);
  if (p_lo > p_hi) return false;
  total = (p_hi - p_lo + 1) * num_kb;
  return true;
}

// Tile order: groups of `group_m` row-tiles sweep all column tiles.
__device__ __forceinline__ void tile_coords(int tile, int tiles_m, int tiles_n, int group_m, int& tm, int& tn) {
  const int group_size = group_m * tiles_n;
  const int first_m = (tile / group_size) * group_m;
  const int gm = min(tiles_m - first_m, group_m);
  const int r = tile % group_size;
  tm = first_m + r % gm;
  tn = r / gm;
}

// CRT with a triangular operand (P.tri_k): the 128-byte K blocks [kb_lo, kb_hi) that can be
// nonzero for the output tile of `rows` x `cols` at raster index `tile`.  A triangle's zero
// blocks have zero residues and add exact zeros, so leaving them out changes no bit.  A tile
// wholly in the padding keeps one block (its operand rows are zero), so every role walks at
// least one block per item.
//
// CRT split-K (P.splits > 1, dense operands only): split s of an item walks the K blocks
// [s num_kb / splits, (s+1) num_kb / splits), a non-empty range since splits <= num_kb.
__device__ __forceinline__ void tile_k_range(const SliceGemmParams& P, int tile, int split, int rows, int cols,
                                             int& kb_lo, int& kb_hi) {
  kb_lo = 0;
  kb_hi = P.num_kb;
  if (P.splits > 1) {
    kb_lo = int(int64_t(split) * P.num_kb / P.splits);
    kb_hi = int(int64_t(split + 1) * P.num_kb / P.splits);
    return;
  }
  if (P.tri_k == 0) return;
  int tm, tn;
  tile_coords(tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
  const int r0 = tm * rows, c0 = tn * cols;
  if (P.tri_k == 1) kb_hi = (r0 + rows + kSliceKBytes - 1) / kSliceKBytes;  // op(A)(r, k) = 0 for k > r
  if (P.tri_k == 2) kb_lo = r0 / kSliceKBytes;                              // ... for k < r
  if (P.tri_k == 3) kb_lo = c0 / kSliceKBytes;                              // op(B)(k, c) = 0 for k < c
  if (P.tri_k == 4) kb_hi = (c0 + cols + kSliceKBytes - 1) / kSliceKBytes;  // ... for k > c
  kb_hi = min(kb_hi, P.num_kb);
  kb_lo = min(kb_lo, P.num_kb - 1);
  if (kb_hi <= kb_lo) kb_hi = kb_lo + 1;
}

// Work items: one per output tile, or in CRT mode one per (tile, K split, modulus): the
// moduli are independent products, so small outputs still spread over the SMs, and the
// items in flight at any time share one modulus (its residue planes stay in L2).
// LISTED: the tiles are P.tile_list[0 .. num_listed) (the triangle of C of a gemmtr / syrk).
template <bool LISTED>
__host__ __device__ __forceinline__ int num_work(const SliceGemmParams& P) {
  if (LISTED) return P.num_listed * P.slices;
  return P.tiles_m * P.tiles_n * (P.crt ? P.slices * P.splits : 1);
}
template <bool LISTED>
__device__ __forceinline__ void work_item(const SliceGemmParams& P, int w, int& tile, int& t_hi, int& t_lo,
                                          int& split) {
  split = 0;
  if (LISTED) {
    tile = P.tile_list[w % P.num_listed];
    t_hi = t_lo = w / P.num_listed;
  } else if (P.crt) {
    const int nt = P.tiles_m * P.tiles_n;
    tile = w % nt;
    const int r = w / nt;
    t_hi = t_lo = r / P.splits;
    split = r % P.splits;
  } else {
    tile = w;
    t_hi = P.diag_hi;
    t_lo = P.diag_lo;
  }
}

// Walks the (work item, diagonal, pair, k-block) schedule in issue order.
// CRT: each item walks the K blocks [kb_lo, kb_hi) of its tile (a compile-time branch: the
// producer's per-block path stays as short as the dense one).
template <bool LISTED, bool CRT>
struct BlockIter {
  int work, tile, t, t_lo, f, p_lo, total, stride, split;
  int rows, cols, kb_lo, kb_hi;  // tile shape; CRT: the item's K blocks
  int kbi, pi;                   // f as (K block, pair offset): f = pi * num_kb + kbi, kept by adds
  bool valid;
  __device__ __forceinline__ void load(const SliceGemmParams& P) {
    int t_hi;
    work_item<LISTED>(P, work, tile, t_hi, t_lo, split);
    t = t_hi;
    f = kbi = pi = 0;
    if constexpr (CRT) tile_k_range(P, tile, split, rows, cols, kb_lo, kb_hi);
  }
  __device__ __forceinline__ void settle(const SliceGemmParams& P, int nwork) {
    valid = false;
    while (work < nwork) {
      if (t < t_lo) {
        work += stride;
        if (work < nwork) load(P);
        continue;
      }
      if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total, CRT) || f >= (CRT ? kb_hi - kb_lo : total)) {
        --t;
        f = kbi = pi = 0;
        continue;
      }
      valid = true;
      return;
    }
  }
  __device__ __forceinline__ void start(const SliceGemmParams& P, int nwork, int first, int step, int tile_rows,
                                        int tile_cols) {
    work = first;
    stride = step;
    rows = tile_rows;
    cols = tile_cols;
    if (work < nwork) load(P);
    settle(P, nwork);
  }
  __device__ __forceinline__ void next(const SliceGemmParams& P, int nwork) {
    ++f;
    if (++kbi == P.num_kb) {
      kbi = 0;
      ++pi;
    }
    settle(P, nwork);
  }
};

// 2^E exactly for any integer E (subnormal powers included, 0 below 2^-1074, +inf above 2^1023).
__device__ __forceinline__ double exp2_int(int E) {
  if (E >= -1022)
    return E <= 1023 ? __longlong_as_double(static_cast<long long>(E + 1023) << 52)
                     : __longlong_as_double(0x7FF0000000000000LL);
  return E >= -1074 ? __longlong_as_double(1LL << (E + 1074)) : 0.0;
}

template <int MODE, int BN, bool PAIR>
struct SliceTraits {
  static constexpr bool kInt8 = MODE != kModeSplitBF16;
  static constexpr int kKElems = kInt8 ? kSliceKBytes : kSliceKBytes / 2;  // int8 / bf16
  // instruction descriptor: s8 x s8 -> s32 (Ozaki, CRT), bf16 x bf16 -> f32 (split-BF16); M = 128 or 256
  static constexpr uint32_t kIdesc = kInt8 ? make_idesc(2u, 1u, 1u, PAIR ? 256 : 128, BN)
                                           : make_idesc(1u, 1u, 1u, PAIR ? 256 : 128, BN);
  static constexpr int kUnitKb = is_crt_mode(MODE) ? kMaxUnitKbCrt : kMaxUnitKb;
};

// B slice of a block: q - 1 = t - p - 1 for Ozaki/split-BF16 diagonals, t for CRT moduli.
__device__ __forceinline__ int b_slice(int t, int p, bool crt) { return crt ? t : t - p - 1; }

// Tile loop bounds of this CTA (the two CTAs of a pair walk one tile sequence).
template <bool PAIR>
__device__ __forceinline__ int first_tile() {
  return PAIR ? int(blockIdx.x >> 1) : int(blockIdx.x);
}
template <bool PAIR>
__device__ __forceinline__ int tile_step() {
  return PAIR ? int(gridDim.x >> 1) : int(gridDim.x);
}


// ------------------------------------------------------------------ producer (warp 0, one lane)
template <int MODE, int BN, int STAGES, bool PAIR, int MT>
__device__ __forceinline__ void slice_producer(const CUtensorMap* tmA, const CUtensorMap* tmB, uint8_t* smem,
                                               uint64_t* full, uint64_t* empty, volatile int* abort_flag,
                                               const SliceGemmParams& P, uint32_t rank) {
  using L = SliceLayout<BN, STAGES, PAIR, MT>;
  constexpr int kTileRows = PAIR ? 2 * kSliceBM : MT * kSliceBM;
  constexpr int ke = SliceTraits<MODE, BN, PAIR>::kKElems;  // innermost coordinate step (elements)
  constexpr uint32_t kTx = (PAIR ? 2u : 1u) * uint32_t(L::kABytes + L::kBBytes);
  constexpr bool kListed = MODE == kModeCrtI8Listed;
  const int nwork = num_work<kListed>(P);
  const int a_row_off = PAIR ? int(rank) * kSliceBM : 0;
  const int b_row_off = PAIR ? int(rank) * L::kBRows : 0;
  uint32_t issued = 0;  // stage = issued % STAGES, phase = (issued / STAGES) & 1
  bool ok = true;
  // one stage: A piece p - 1 and B piece q_slice at K block kb of the tile (tm, tn)
  auto issue = [&](int tm, int tn, int p, int q_slice, int kb) -> bool {
    const int stage = int(issued % STAGES);
    if (!mbar_wait(&empty[stage], ((issued / STAGES) & 1u) ^ 1u, abort_flag, P.status, P.wait_limit_ns)) return false;
    const int a_row = tm * kTileRows + a_row_off;
    const int b_row = tn * BN + b_row_off;
    if (PAIR) {
      // both CTAs' bytes land on the leader's barrier; only the leader posts expect-tx
      const uint32_t leader_full = mapa_shared(smem_u32(&full[stage]), 0);
      if (rank == 0) mbar_arrive_expect_tx(&full[stage], kTx);
      tma_load_3d_pair(smem + L::kAOff + stage * L::kABytes, tmA, leader_full, kb * ke, a_row, p - 1);
      tma_load_3d_pair(smem + L::kBOff + stage * L::kBBytes, tmB, leader_full, kb * ke, b_row, q_slice);
    } else {
      mbar_arrive_expect_tx(&full[stage], kTx);
      tma_load_3d(smem + L::kAOff + stage * L::kABytes, tmA, &full[stage], kb * ke, a_row, p - 1);
      tma_load_3d(smem + L::kBOff + stage * L::kBBytes, tmB, &full[stage], kb * ke, b_row, q_slice);
    }
    ++issued;
    return true;
  };
  if constexpr (MODE == kModeSplitBF16) {
    // chunks of kBf16ChunkKb K blocks; in each, the diagonals (smallest weight first), their
    // pairs and the chunk's K blocks -- the order slice_mma consumes them in
    for (int w = first_tile<PAIR>(); w < nwork && ok; w += tile_step<PAIR>()) {
      int tm, tn;
      tile_coords(w, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
      for (int kc = 0; kc < P.num_kb && ok; kc += kBf16ChunkKb) {
        const int kend = min(P.num_kb, kc + kBf16ChunkKb);
        for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
          int p_lo, total;
          if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total)) continue;
          const int p_hi = p_lo + total / P.num_kb;
          for (int p = p_lo; p < p_hi && ok; ++p)
            for (int kb = kc; kb < kend && ok; ++kb) ok = issue(tm, tn, p, b_slice(t, p, false), kb);
        }
      }
    }
  } else {
    BlockIter<kListed, is_crt_mode(MODE)> it;
    it.start(P, nwork, first_tile<PAIR>(), tile_step<PAIR>(), kTileRows, BN);
    while (it.valid) {
      int tm, tn;
      tile_coords(it.tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
      int p, kb;
      if constexpr (is_crt_mode(MODE)) {
        p = it.p_lo;
        kb = it.kb_lo + it.f;
      } else {
        p = it.p_lo + it.pi;
        kb = it.kbi;
      }
      if (!issue(tm, tn, p, b_slice(it.t, p, P.crt != 0), kb)) {
        ok = false;
        break;
      }
      it.next(P, nwork);
  }
  }
  if (!PAIR) {
    // let the copies still in flight land before the CTA can exit (bounded).  Also when this
    // loop finished: the MMA issuer may have given up before consuming the last stages.  On
    // the normal path their phases are complete and each wait returns at once.  A pair's
    // copies complete on the leader, and the final cluster barrier keeps both CTAs alive.
    volatile int no_abort = 0;
    for (uint32_t i = issued > STAGES ? issued - STAGES : 0; i < issued; ++i)
      (void)mbar_wait(&full[i % STAGES], (i / STAGES) & 1u, &no_abort, P.status);
  }
}

// ------------------------------------------------------------------ MMA issuer (warp 1, one lane; leader only)
// Ozaki / CRT: one accumulation unit per diagonal or modulus (exact INT32, cut into chunks
// where K is too long).  Split-BF16: one unit per kBf16ChunkKb K blocks of a tile, covering
// every piece product over those K (FP32 accumulation, drained by the epilogue).
template <bool PAIR>
__device__ __forceinline__ void commit_to(uint64_t* bar) {
  if (PAIR) {
    const uint32_t a = smem_u32(bar);
    mma_commit_pair(mapa_shared(a, 0));
    mma_commit_pair(mapa_shared(a, 1));
  } else {
    mma_commit(bar);
  }
}

template <int MODE, int BN, int STAGES, bool PAIR, int MT>
__device__ __forceinline__ void slice_mma(uint8_t* smem, uint64_t* full, uint64_t* empty, uint64_t* tfull,
                                          uint64_t* tempty, uint64_t* drain, uint32_t tmem_base,
                                          volatile int* abort_flag, const SliceGemmParams& P) {
  using L = SliceLayout<BN, STAGES, PAIR, MT>;
  constexpr int kTileRows = PAIR ? 2 * kSliceBM : MT * kSliceBM;
  constexpr uint32_t idesc = SliceTraits<MODE, BN, PAIR>::kIdesc;
  constexpr bool kListed = MODE == kModeCrtI8Listed;
  const int nwork = num_work<kListed>(P);
  uint32_t consumed = 0;  // stage = consumed % STAGES, phase = (consumed / STAGES) & 1
  int buf = 0;
  uint32_t tphase = 0u;  // bit b: phase of accumulator buffer b
  bool ok = true;
  // the MMAs of one stage into accumulator d_tmem (fresh: the first overwrites it)
  auto consume = [&](uint32_t d_tmem, bool fresh) -> bool {
    const int stage = int(consumed % STAGES);
    if (!mbar_wait(&full[stage], (consumed / STAGES) & 1u, abort_flag, P.status, P.wait_limit_ns)) return false;
    tc_fence_after();
    const uint64_t adesc = make_sw128_kmajor_desc(smem_u32(smem + L::kAOff + stage * L::kABytes));
    const uint64_t bdesc = make_sw128_kmajor_desc(smem_u32(smem + L::kBOff + stage * L::kBBytes));
#pragma unroll
    for (int kk = 0; kk < kSliceKBytes / 32; ++kk) {
      const uint32_t acc = (fresh && kk == 0) ? 0u : 1u;
      const uint64_t bd = bdesc + uint64_t(2 * kk);
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        // row tile mt: 128 rows of 128 bytes further on (descriptor addresses count 16 bytes);
        // its accumulator is the TMEM region of columns mt * BN ..
        const uint64_t ad = adesc + uint64_t(mt * (kSliceBM * kSliceKBytes / 16)) + uint64_t(2 * kk);
        const uint32_t dt = d_tmem + uint32_t(mt * BN);
        if (PAIR) {
          if (MODE != kModeSplitBF16)
            mma_i8_pair(dt, ad, bd, idesc, acc);
          else
            mma_f16_pair(dt, ad, bd, idesc, acc);
        } else {
          if (MODE != kModeSplitBF16)
            mma_i8(dt, ad, bd, idesc, acc);
          else
            mma_f16(dt, ad, bd, idesc, acc);
        }
      }
    }
    commit_to<PAIR>(&empty[stage]);
    ++consumed;
    return true;
  };
  if constexpr (MODE == kModeSplitBF16) {
    // one accumulation unit per chunk of kBf16ChunkKb K blocks (order as in slice_producer)
    for (int w = first_tile<PAIR>(); w < nwork && ok; w += tile_step<PAIR>()) {
      for (int kc = 0; kc < P.num_kb && ok; kc += kBf16ChunkKb) {
        const int kend = min(P.num_kb, kc + kBf16ChunkKb);
        if (!mbar_wait(&tempty[buf], ((tphase >> buf) & 1u) ^ 1u, abort_flag, P.status, P.wait_limit_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + uint32_t(buf * BN);
        bool fresh = true;
        for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
          int p_lo, total;
          if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total)) continue;
          const int p_hi = p_lo + total / P.num_kb;
          for (int p = p_lo; p < p_hi && ok; ++p)
            for (int kb = kc; kb < kend && ok; ++kb) {
              ok = consume(d_tmem, fresh);
              fresh = false;
            }
        }
        if (!ok) break;
        commit_to<PAIR>(&tfull[buf]);
        tphase ^= 1u << buf;
        buf ^= 1;
      }
    }
  } else {
    // one accumulation unit per diagonal (Ozaki) or modulus (CRT), cut where K exceeds what
    // the INT32 accumulator holds exactly
    for (int w = first_tile<PAIR>(); w < nwork && ok; w += tile_step<PAIR>()) {
      int tile, t_hi, t_lo, split;
      work_item<kListed>(P, w, tile, t_hi, t_lo, split);
      for (int t = t_hi; t >= t_lo && ok; --t) {
        int p_lo, total;
        if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total, is_crt_mode(MODE))) continue;
        if constexpr (is_crt_mode(MODE)) {
          int kb_lo, kb_hi;
          tile_k_range(P, tile, split, kTileRows, BN, kb_lo, kb_hi);
          total = kb_hi - kb_lo;
        }
        constexpr int kUnit = SliceTraits<MODE, BN, PAIR>::kUnitKb;
        for (int u0 = 0; u0 < total && ok;) {
          const int u1 = total - u0 <= kUnit ? total : u0 + kUnit;
          if (!mbar_wait(&tempty[buf], ((tphase >> buf) & 1u) ^ 1u, abort_flag, P.status, P.wait_limit_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + uint32_t(buf * BN);
          for (int f = u0; f < u1 && ok; ++f) ok = consume(d_tmem, f == u0);
          if (!ok) break;
          commit_to<PAIR>(&tfull[buf]);
          tphase ^= 1u << buf;
          if constexpr (MT == 1) buf ^= 1;  // MT = 2: one accumulator fills the TMEM
          u0 = u1;
        }
      }
    }
  }
  // every issued MMA must finish before TMEM is released
  if (PAIR)
    mma_commit_pair(mapa_shared(smem_u32(drain), 0));
  else
    mma_commit(drain);
  volatile int no_abort = 0;
  (void)mbar_wait(drain, 0, &no_abort, P.status);
}


// ------------------------------------------------------------------ epilogues
template <bool PAIR>
__device__ __forceinline__ void acc_release(uint64_t* tempty_buf) {
  if (PAIR)
    mbar_arrive_cluster(mapa_shared(smem_u32(tempty_buf), 0));  // the leader's barrier
  else
    mbar_arrive(tempty_buf);
}

// Ozaki: each thread owns one row and kCols columns of the tile and keeps their FP64
// sums in registers across the tile's diagonals:
//   acc += double(D_t) * 2^(e_i + f_j - 12 - 7(t-2))     (exact product, one rounding per add)
// from the smallest weight up; after the last diagonal C is written once:
//   first_writes: C = alpha*acc (beta == 0) or fma(beta, C, alpha*acc);  else C = C + alpha*acc.
template <int BN, int NW, bool PAIR>
__device__ __forceinline__ void ozaki_epilogue(uint32_t tmem_base, uint64_t* tfull, uint64_t* tempty, int* col_exp,
                                               volatile int* abort_flag, const SliceGemmParams& P) {
  constexpr int kCols = BN * 4 / NW;  // columns per thread
  static_assert(kCols % 16 == 0 && kCols <= 64, "register budget of the FP64 accumulator");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3;                      // TMEM lane quadrant this warp may access
  const int col_base = ((warp - 2) >> 2) * kCols;  // column slice of this warp
  const int row = quad * 32 + lane;
  const int et = threadIdx.x - 64;  // 0 .. 32*NW-1
  const int num_tiles = P.tiles_m * P.tiles_n;
  const int row_base = PAIR ? int(cluster_ctarank()) * kSliceBM : 0;
  double* C = static_cast<double*>(P.C);
  int buf = 0;
  uint32_t ephase = 0u;
  double err_hi = 0.0, err_lo = 0.0;
  bool ok = true;
  for (int tile = first_tile<PAIR>(); tile < num_tiles && ok; tile += tile_step<PAIR>()) {
    int tm, tn;
    tile_coords(tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int64_t m0 = int64_t(tm) * (PAIR ? 2 * kSliceBM : kSliceBM) + row_base;
    const int64_t n0 = int64_t(tn) * BN;
    for (int j = et; j < BN; j += 32 * NW) {
      const int64_t col = n0 + j;
      col_exp[j] = (col < P.n) ? P.expB[col] : 0;
    }
    asm volatile("bar.sync 1, %0;" ::"r"(32 * NW) : "memory");
    const int64_t grow = m0 + row;
    const bool row_ok = grow < P.m;
    const int erow = row_ok ? P.expA[grow] : 0;
    double acc[kCols];
#pragma unroll
    for (int j = 0; j < kCols; ++j) acc[j] = 0.0;
    for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
      int p_lo, total;
      if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total)) continue;
      const int ebase = erow - 12 - 7 * (t - 2);
      const bool est_hi = P.err_sq != nullptr && t == P.diag_hi;
      const bool est_lo = P.err_sq != nullptr && t == 2;
      for (int u0 = 0; u0 < total && ok; u0 += kMaxUnitKb) {
        if (!mbar_wait(&tfull[buf], (ephase >> buf) & 1u, abort_flag, P.status, P.wait_limit_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem_base + uint32_t(buf * BN + col_base) + (uint32_t(quad * 32) << 16);
#pragma unroll
        for (int c = 0; c < kCols / 16; ++c) {
          uint32_t r[16];
          tmem_ld_32x32b_x16(taddr + uint32_t(c * 16), r);
          tmem_ld_wait();
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) {
            const double val = static_cast<double>(static_cast<int32_t>(r[jj])) *
                               exp2_int(ebase + col_exp[col_base + c * 16 + jj]);
            acc[c * 16 + jj] = __dadd_rn(acc[c * 16 + jj], val);
            if (est_hi) err_hi = fma(val, val, err_hi);
            if (est_lo) err_lo = fma(val, val, err_lo);
          }
        }
        tc_fence_before();
        acc_release<PAIR>(&tempty[buf]);
        ephase ^= 1u << buf;
        buf ^= 1;
      }
    }
    if (ok && row_ok) {
      double* cp = C + grow + (n0 + col_base) * P.ldc;
#pragma unroll
      for (int j = 0; j < kCols; ++j) {
        if (n0 + col_base + j < P.n) {
          double* dst = cp + int64_t(j) * P.ldc;
          const double v = __dmul_rn(P.alpha, acc[j]);
          if (!P.first_writes)
            *dst = __dadd_rn(*dst, v);
          else
            *dst = (P.beta == 0.0) ? v : __fma_rn(P.beta, *dst, v);
        }
      }
    }
    asm volatile("bar.sync 1, %0;" ::"r"(32 * NW) : "memory");
  }
  if (P.err_sq) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      err_hi += __shfl_xor_sync(0xffffffffu, err_hi, o);
      err_lo += __shfl_xor_sync(0xffffffffu, err_lo, o);
    }
    if (lane == 0 && err_hi != 0.0) atomicAdd(&P.err_sq[0], err_hi);
    if (lane == 0 && err_lo != 0.0) atomicAdd(&P.err_sq[1], err_lo);
  }
}

// x mod p for a 32-bit x and p <= 256, with m = floor((2^32 - 1) / p): p m >= 2^32 - p, so
// x/p - x m / 2^32 <= x / 2^32 < 1 and the estimate q = umulhi(x, m) is at most one short
// of floor(x / p): one conditional subtraction finishes it.
__device__ __forceinline__ uint32_t mod_small(uint32_t x, uint32_t p, uint32_t m) {
  const uint32_t r = x - __umulhi(x, m) * p;
  return r >= p ? r - p : r;
}

// CRT: unit t is modulus p_t; every INT32 product entry is reduced to [0, p_t) and stored
// as one byte of residue plane t (column-major, ld_res).  K beyond one unit comes in
// further chunks whose residues are added mod p_t.
// MT = 2: warp group g = (warp - 2) / 4 drains row tile g % 2 (TMEM columns (g % 2) * BN ..)
// and its columns (g / 2) * kCols ..; the accumulator has a single buffer then.
template <int BN, int NW, bool PAIR, bool LISTED, int MT>
__device__ __forceinline__ void crt_epilogue(uint32_t tmem_base, uint64_t* tfull, uint64_t* tempty,
                                             volatile int* abort_flag, const SliceGemmParams& P) {
  static_assert(NW % (4 * MT) == 0, "whole warp groups per row tile");
  constexpr int kCols = BN * 4 * MT / NW;
  static_assert(kCols % 32 == 0, "column slice");
  constexpr int kTileRows = PAIR ? 2 * kSliceBM : MT * kSliceBM;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3;
  const int group = (warp - 2) >> 2;
  const int region = group % MT;  // row tile within the CTA's tile
  const int col_base = (group / MT) * kCols;
  const int row = region * kSliceBM + quad * 32 + lane;
  const int nwork = num_work<LISTED>(P);
  const int row_base = PAIR ? int(cluster_ctarank()) * kSliceBM : 0;
  const int64_t plane = P.ld_res * int64_t(P.tiles_n) * BN;
  int buf = 0;
  uint32_t ephase = 0u;
  bool ok = true;
  for (int w = first_tile<PAIR>(); w < nwork && ok; w += tile_step<PAIR>()) {
    int tile, t_hi, t_lo, tm, tn, split;
    work_item<LISTED>(P, w, tile, t_hi, t_lo, split);
    tile_coords(tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int64_t m0 = int64_t(tm) * kTileRows + row_base;
    const int64_t n0 = int64_t(tn) * BN + col_base;
    const int64_t grow = m0 + row;
    for (int t = t_hi; t >= t_lo && ok; --t) {
      int p_lo, total;
      if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total, true)) continue;
      {
        int kb_lo, kb_hi;
        tile_k_range(P, tile, split, kTileRows, BN, kb_lo, kb_hi);
        total = kb_hi - kb_lo;
      }
      const uint32_t pm = uint32_t(crt_modulus(t));
      const uint32_t magic = 0xFFFFFFFFu / pm;
      // |v| <= 1023 * 128 * 128 * 128 = 2^31 - 2^21 for an accumulation unit, so with bias a
      // multiple of p in [2^31 - 2^21, 2^31 - 2^21 + p), v + bias lies in [0, 2^32) and
      // (v + bias) mod p = v mod p: one reduction of an unsigned word, no sign handling
      const uint32_t bias = (0x7FE00000u + pm - 1u) / pm * pm;
      uint8_t* rp = P.residues + (int64_t(t) * P.splits + split) * plane + grow;
      for (int u0 = 0; u0 < total && ok; u0 += kMaxUnitKbCrt) {
        if (!mbar_wait(&tfull[buf], (ephase >> buf) & 1u, abort_flag, P.status, P.wait_limit_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr =
            tmem_base + uint32_t((MT == 1 ? buf * BN : region * BN) + col_base) + (uint32_t(quad * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < kCols / 32; ++c) {
          uint32_t r[32];
          tmem_ld_32x32b_x32(taddr + uint32_t(c * 32), r);
          tmem_ld_wait();
          if (grow < P.ld_res) {
            uint8_t* dst = rp + (n0 + c * 32) * P.ld_res;
#pragma unroll
            for (int jj = 0; jj < 32; ++jj, dst += P.ld_res) {
              uint32_t res = mod_small(r[jj] + bias, pm, magic);
              if (u0 > 0) {
                res += *dst;
                if (res >= pm) res -= pm;
              }
              *dst = uint8_t(res);
            }
          }
        }
        tc_fence_before();
        acc_release<PAIR>(&tempty[buf]);
        ephase ^= 1u << buf;
        if constexpr (MT == 1) buf ^= 1;  // two accumulators alternate; MT = 2 fills the TMEM
      }
    }
  }
}

// Split-BF16: each thread owns one row and kCols columns of the tile.  The units of a tile
// (one per kBf16ChunkKb K blocks) are added, rounded to nearest, into FP32 registers; after
// the last one C = alpha * acc + beta * C in FP32.
template <int BN, int NW, bool PAIR>
__device__ __forceinline__ void bf16_epilogue(uint32_t tmem_base, uint64_t* tfull, uint64_t* tempty,
                                              volatile int* abort_flag, const SliceGemmParams& P) {
  constexpr int kCols = BN * 4 / NW;
  static_assert(kCols % 32 == 0 && kCols <= 128, "register budget of the FP32 accumulator");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3;
  const int col_base = ((warp - 2) >> 2) * kCols;
  const int row = quad * 32 + lane;
  const int num_tiles = P.tiles_m * P.tiles_n;
  const int row_base = PAIR ? int(cluster_ctarank()) * kSliceBM : 0;
  float* C = static_cast<float*>(P.C);
  int buf = 0;
  uint32_t ephase = 0u;
  bool ok = true;
  for (int tile = first_tile<PAIR>(); tile < num_tiles && ok; tile += tile_step<PAIR>()) {
    int tm, tn;
    tile_coords(tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int64_t m0 = int64_t(tm) * (PAIR ? 2 * kSliceBM : kSliceBM) + row_base;
    const int64_t n0 = int64_t(tn) * BN + col_base;
    float acc[kCols];
#pragma unroll
    for (int j = 0; j < kCols; ++j) acc[j] = 0.0f;
    for (int kc = 0; kc < P.num_kb; kc += kBf16ChunkKb) {
      if (!mbar_wait(&tfull[buf], (ephase >> buf) & 1u, abort_flag, P.status, P.wait_limit_ns)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + uint32_t(buf * BN + col_base) + (uint32_t(quad * 32) << 16);
#pragma unroll
      for (int c = 0; c < kCols / 16; ++c) {
        uint32_t r[16];
        tmem_ld_32x32b_x16(taddr + uint32_t(c * 16), r);
        tmem_ld_wait();
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) acc[c * 16 + jj] = __fadd_rn(acc[c * 16 + jj], __uint_as_float(r[jj]));
      }
      tc_fence_before();
      acc_release<PAIR>(&tempty[buf]);
      ephase ^= 1u << buf;
      buf ^= 1;
    }
    const int64_t grow = m0 + row;
    if (ok && grow < P.m) {
      float* cp = C + grow + n0 * P.ldc;
#pragma unroll
      for (int j = 0; j < kCols; ++j) {
        if (n0 + j < P.n) {
          float* dst = cp + int64_t(j) * P.ldc;
          const float v = __fmul_rn(P.alpha_f, acc[j]);
          *dst = (P.beta_f == 0.0f) ? v : __fmaf_rn(P.beta_f, *dst, v);
        }
      }
    }
  }
}

// ------------------------------------------------------------------ kernel
template <int MODE, int BN, int STAGES, int NW, bool PAIR, int MT = 1>
__global__ void __launch_bounds__(64 + 32 * NW, 1)
    slice_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const SliceGemmParams P) {
  static_assert(MT == 1 || (is_crt_mode(MODE) && !PAIR && MT == 2 && 2 * BN <= 512), "256-row tiles: CRT, one CTA");
  using L = SliceLayout<BN, STAGES, PAIR, MT>;
  // both CTAs of a pair read the same flag, so they leave together
  if (P.skip_if_flag && *P.skip_if_flag) return;

  extern __shared__ uint8_t slice_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(slice_smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::kBarOff);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* tfull = bars + 2 * STAGES;
  uint64_t* tempty = bars + 2 * STAGES + 2;
  uint64_t* drain = bars + 2 * STAGES + 4;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(smem + L::kMiscOff);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + L::kMiscOff + 4);
  int* col_exp = reinterpret_cast<int*>(smem + L::kColExpOff);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t rank = PAIR ? cluster_ctarank() : 0u;

  if (threadIdx.x == 0) {
    for (int i = 0; i < STAGES; ++i) {
      mbar_init(&full[i], 1);   // expect-tx arrival (+ the bytes of one or both CTAs)
      mbar_init(&empty[i], 1);  // one commit from the MMA thread
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], (PAIR ? 2 : 1) * 32 * NW);  // every epilogue thread (of both CTAs)
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
  }
  if (warp == 1) {
    if (PAIR) {
      tmem_alloc_pair(tmem_holder, 2 * BN);
      tmem_relinquish_pair();
    } else {
      tmem_alloc(tmem_holder, 2 * BN);
      tmem_relinquish();
    }
  }
  tc_fence_before();
  if (PAIR)
    cluster_sync();  // barriers of both CTAs exist before any remote arrival
  else
    __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  if (warp == 0) {
    if (lane == 0) slice_producer<MODE, BN, STAGES, PAIR, MT>(&tmA, &tmB, smem, full, empty, abort_flag, P, rank);
  } else if (warp == 1) {
    if (lane == 0 && rank == 0)
      slice_mma<MODE, BN, STAGES, PAIR, MT>(smem, full, empty, tfull, tempty, drain, tmem_base, abort_flag, P);
  } else {
    if constexpr (MODE == kModeOzakiI8)
      ozaki_epilogue<BN, NW, PAIR>(tmem_base, tfull, tempty, col_exp, abort_flag, P);
    else if constexpr (is_crt_mode(MODE))
      crt_epilogue<BN, NW, PAIR, MODE == kModeCrtI8Listed, MT>(tmem_base, tfull, tempty, abort_flag, P);
    else
      bf16_epilogue<BN, NW, PAIR>(tmem_base, tfull, tempty, abort_flag, P);
  }

  tc_fence_before();
  if (PAIR)
    cluster_sync();  // MMAs drained and both epilogues done with TMEM
  else
    __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    if (PAIR)
      tmem_dealloc_pair(tmem_base, 2 * BN);
    else
      tmem_dealloc(tmem_base, 2 * BN);
  }
}

// Host-side launch: one CTA (or one CTA pair) per SM pair, persistent over the tiles.
template <int MODE, int BN, int STAGES, int NW, bool PAIR, int MT = 1>
inline cudaError_t launch_slice_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const SliceGemmParams& P,
                                     int num_sms, cudaStream_t stream) {
  using L = SliceLayout<BN, STAGES, PAIR, MT>;
  auto kern = slice_gemm_kernel<MODE, BN, STAGES, NW, PAIR, MT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kAlloc);
  if (e != cudaSuccess) return e;
  const int tiles = num_work<MODE == kModeCrtI8Listed>(P);
  const int ctas = PAIR ? 2 * (tiles < num_sms / 2 ? tiles : num_sms / 2) : (tiles < num_sms ? tiles : num_sms);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(ctas), 1, 1);
  cfg.blockDim = dim3(unsigned(64 + 32 * NW), 1, 1);
  cfg.dynamicSmemBytes = L::kAlloc;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  if (PAIR) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, kern, tmA, tmB, P);
}

}  // namespace eb2

