// slice_gemm.cuh -- the persistent, warp-specialised tcgen05 GEMM over "slices".
//
// Both emulated products reduce to sums of slice products  A_p * B_q^T  over the
// triangle p + q <= s + 1 (p, q = 1..s):
//   * Ozaki DGEMM: A_p, B_q are INT8 digit panels; every diagonal t = p + q has its
//     own power-of-two weight, so each diagonal is an exact INT32 accumulation in
//     TMEM that the epilogue scales and adds into the FP64 output;
//   * split-BF16 SGEMM: A_p, B_q are the hi/mid/lo BF16 pieces of the FP32 inputs;
//     the pieces carry their own exponents, so the whole triangle accumulates into
//     one FP32 TMEM accumulator and the epilogue applies alpha/beta once.
//
// Roles (192 threads):  warp 0 = TMA producer, warp 1 = MMA issuer + TMEM owner,
// warps 2..5 = epilogue (one TMEM lane quadrant each, one output row per thread).
// Operand panels are K-major and zero-padded by the split kernels, loaded as
// 128-byte-swizzled tiles (128 rows x 128 bytes of A, BN rows x 128 bytes of B per
// stage), consumed by tcgen05.mma with K = 32 bytes per instruction.  Two TMEM
// accumulators alternate so the epilogue of one unit overlaps the MMAs of the next.
// Every wait is bounded (device_common.cuh).
#pragma once
#include <cuda.h>

#include <climits>
#include <cstdint>

#include "device_common.cuh"

namespace eb2 {

enum SliceMode : int { kModeOzakiI8 = 0, kModeSplitBF16 = 1 };

constexpr int kSliceBM = 128;
constexpr int kSliceKBytes = 128;  // bytes of K per pipeline stage
// One Ozaki accumulation unit covers at most this many 128-deep digit blocks per
// output: 4095 * 128 * 64 * 64 < 2^31, so the INT32 accumulator cannot overflow.
constexpr int kMaxUnitKb = 4095;

template <int BN, int STAGES>
struct SliceSmemLayout {
  static constexpr int kABytes = kSliceBM * kSliceKBytes;
  static constexpr int kBBytes = BN * kSliceKBytes;
  static constexpr int kAOff = 0;
  static constexpr int kBOff = kAOff + STAGES * kABytes;
  static constexpr int kBarOff = kBOff + STAGES * kBBytes;
  // full[STAGES], empty[STAGES], tfull[2], tempty[2], drain
  static constexpr int kNumBars = 2 * STAGES + 5;
  static constexpr int kMiscOff = kBarOff + kNumBars * 8;
  static constexpr int kColExpOff = kMiscOff + 16;
  static constexpr int kTotal = kColExpOff + BN * 4;
  static constexpr int kAlloc = kTotal + 1024;  // slack for 1024-byte alignment
};

struct SliceGemmParams {
  int64_t m, n;
  int num_kb;            // K blocks of kSliceKBytes
  int tiles_m, tiles_n;
  int slices;            // s
  int diag_lo, diag_hi;  // diagonals t = p + q processed, from diag_hi down to diag_lo
  int first_writes;      // the first unit of a tile applies beta (else it accumulates)
  double alpha, beta;    // Ozaki (FP64 output)
  float alpha_f, beta_f; // split-BF16 (FP32 output)
  void* C;
  int64_t ldc;
  const int32_t* expA;   // Ozaki row / column exponents
  const int32_t* expB;
  const int* skip_if_flag;
  double* err_sq;        // Ozaki: [0] += energy of diagonal diag_hi, [1] += energy of diagonal 2
  uint32_t* status;
  int group_m;           // row-tiles per raster group (>= tiles_m: plain column-major tile order)
  int prefetch;          // L2 prefetch distance in blocks (0: none)
};

// Pair range of diagonal t: p = p_lo .. p_lo + total/num_kb - 1 (q = t - p).
__device__ __forceinline__ bool diag_bounds(int t, int s, int num_kb, int& p_lo, int& total) {
  p_lo = max(1, t - s);
  const int p_hi = min(s, t - 1);
  if (p_lo > p_hi) return false;
  total = (p_hi - p_lo + 1) * num_kb;
  return true;
}

// Tile order: groups of `group_m` row-tiles sweep all column tiles, so the CTAs that
// run at the same time share A and B panels in L2.
__device__ __forceinline__ void tile_coords(int tile, int tiles_m, int tiles_n, int group_m, int& tm, int& tn) {
  const int group_size = group_m * tiles_n;
  const int first_m = (tile / group_size) * group_m;
  const int gm = min(tiles_m - first_m, group_m);
  const int r = tile % group_size;
  tm = first_m + r % gm;
  tn = r / gm;
}

// Walks the (tile, diagonal, pair, k-block) schedule in issue order.
struct BlockIter {
  int tile, t, f, p_lo, total, stride;
  bool valid;
  __device__ __forceinline__ void settle(const SliceGemmParams& P, int num_tiles) {
    valid = false;
    while (tile < num_tiles) {
      if (t < P.diag_lo) {
        tile += stride;
        t = P.diag_hi;
        f = 0;
        continue;
      }
      if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total) || f >= total) {
        --t;
        f = 0;
        continue;
      }
      valid = true;
      return;
    }
  }
  __device__ __forceinline__ void start(const SliceGemmParams& P, int num_tiles, int first, int step) {
    tile = first;
    stride = step;
    t = P.diag_hi;
    f = 0;
    settle(P, num_tiles);
  }
  __device__ __forceinline__ void next(const SliceGemmParams& P, int num_tiles) {
    ++f;
    settle(P, num_tiles);
  }
};

__device__ __forceinline__ double exp2_int(int E) {
  return (E > -1023 && E < 1024) ? __longlong_as_double(static_cast<long long>(E + 1023) << 52) : ldexp(1.0, E);
}


// ------------------------------------------------------------------ producer
template <int MODE>
struct SliceTraits {
  static constexpr int kKElems = MODE == kModeOzakiI8 ? kSliceKBytes : kSliceKBytes / 2;  // int8 / bf16
  static constexpr int kKPerMma = MODE == kModeOzakiI8 ? 32 : 16;
  // idesc: Ozaki s8 x s8 -> s32, split-BF16 bf16 x bf16 -> f32
  template <int BN>
  __host__ __device__ static constexpr uint32_t idesc() {
    return MODE == kModeOzakiI8 ? make_idesc(2u, 1u, 1u, kSliceBM, BN) : make_idesc(1u, 1u, 1u, kSliceBM, BN);
  }
};

template <int MODE, int BN, int STAGES>
__device__ __forceinline__ void slice_producer(const CUtensorMap* tmA, const CUtensorMap* tmB, uint8_t* smem,
                                               uint64_t* full, uint64_t* empty, volatile int* abort_flag,
                                               const SliceGemmParams& P) {
  using L = SliceSmemLayout<BN, STAGES>;
  constexpr int ke = SliceTraits<MODE>::kKElems;  // innermost coordinate step (elements)
  const int num_tiles = P.tiles_m * P.tiles_n;
  BlockIter it, pf;
  it.start(P, num_tiles, blockIdx.x, gridDim.x);
  pf.start(P, num_tiles, blockIdx.x, gridDim.x);
  for (int i = 0; i < P.prefetch && pf.valid; ++i) {
    int tm, tn;
    tile_coords(pf.tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int p = pf.p_lo + pf.f / P.num_kb, kb = pf.f % P.num_kb;
    tma_prefetch_l2_3d(tmA, kb * ke, tm * kSliceBM, p - 1);
    tma_prefetch_l2_3d(tmB, kb * ke, tn * BN, pf.t - p - 1);
    pf.next(P, num_tiles);
  }
  uint32_t issued = 0;  // stage = issued % STAGES, phase = (issued / STAGES) & 1
  bool ok = true;
  while (it.valid) {
    if (P.prefetch > 0 && pf.valid) {
      int tm, tn;
      tile_coords(pf.tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
      const int p = pf.p_lo + pf.f / P.num_kb, kb = pf.f % P.num_kb;
      tma_prefetch_l2_3d(tmA, kb * ke, tm * kSliceBM, p - 1);
      tma_prefetch_l2_3d(tmB, kb * ke, tn * BN, pf.t - p - 1);
      pf.next(P, num_tiles);
    }
    int tm, tn;
    tile_coords(it.tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int p = it.p_lo + it.f / P.num_kb, kb = it.f % P.num_kb;
    const int stage = int(issued % STAGES);
    const uint32_t phase = (issued / STAGES) & 1u;
    if (!mbar_wait(&empty[stage], phase ^ 1u, abort_flag, P.status)) {
      ok = false;
      break;
    }
    mbar_arrive_expect_tx(&full[stage], L::kABytes + L::kBBytes);
    tma_load_3d(smem + L::kAOff + stage * L::kABytes, tmA, &full[stage], kb * ke, tm * kSliceBM, p - 1);
    tma_load_3d(smem + L::kBOff + stage * L::kBBytes, tmB, &full[stage], kb * ke, tn * BN, it.t - p - 1);
    ++issued;
    it.next(P, num_tiles);
  }
  if (!ok) {
    // let the copies still in flight land before the CTA can exit (bounded)
    volatile int no_abort = 0;
    for (uint32_t i = issued > STAGES ? issued - STAGES : 0; i < issued; ++i)
      (void)mbar_wait(&full[i % STAGES], (i / STAGES) & 1u, &no_abort, P.status);
  }
}

// ------------------------------------------------------------------ MMA issuer
// Ozaki: one accumulation unit per diagonal chunk (exact INT32).  Split-BF16: the
// whole triangle of a tile is one unit (FP32 accumulation in a single accumulator).
template <int MODE, int BN, int STAGES>
__device__ __forceinline__ void slice_mma(uint8_t* smem, uint64_t* full, uint64_t* empty, uint64_t* tfull,
                                          uint64_t* tempty, uint64_t* drain, uint32_t tmem_base,
                                          volatile int* abort_flag, const SliceGemmParams& P) {
  using L = SliceSmemLayout<BN, STAGES>;
  constexpr uint32_t idesc = SliceTraits<MODE>::template idesc<BN>();
  constexpr bool kTileUnit = (MODE == kModeSplitBF16);
  const int num_tiles = P.tiles_m * P.tiles_n;
  uint32_t consumed = 0;  // stage = consumed % STAGES, phase = (consumed / STAGES) & 1
  int buf = 0;
  uint32_t tphase = 0u;  // bit b: phase of accumulator buffer b
  bool ok = true;
  for (int tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x) {
    bool fresh = true;  // next MMA overwrites the accumulator
    if (kTileUnit) {
      if (!mbar_wait(&tempty[buf], ((tphase >> buf) & 1u) ^ 1u, abort_flag, P.status)) break;
      tc_fence_after();
    }
    for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
      int p_lo, total;
      if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total)) continue;
      for (int u0 = 0; u0 < total && ok; u0 += kMaxUnitKb) {
        const int u1 = (kTileUnit || total - u0 <= kMaxUnitKb) ? total : u0 + kMaxUnitKb;
        if (!kTileUnit) {
          if (!mbar_wait(&tempty[buf], ((tphase >> buf) & 1u) ^ 1u, abort_flag, P.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          fresh = true;
        }
        const uint32_t d_tmem = tmem_base + uint32_t(buf * BN);
        for (int f = u0; f < u1; ++f) {
          const int stage = int(consumed % STAGES);
          if (!mbar_wait(&full[stage], (consumed / STAGES) & 1u, abort_flag, P.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t adesc = make_sw128_kmajor_desc(smem_u32(smem + L::kAOff + stage * L::kABytes));
          const uint64_t bdesc = make_sw128_kmajor_desc(smem_u32(smem + L::kBOff + stage * L::kBBytes));
#pragma unroll
          for (int kk = 0; kk < kSliceKBytes / 32; ++kk) {
            const uint32_t acc = (fresh && kk == 0) ? 0u : 1u;
            if (MODE == kModeOzakiI8)
              mma_i8(d_tmem, adesc + uint64_t(2 * kk), bdesc + uint64_t(2 * kk), idesc, acc);
            else
              mma_f16(d_tmem, adesc + uint64_t(2 * kk), bdesc + uint64_t(2 * kk), idesc, acc);
          }
          fresh = false;
          mma_commit(&empty[stage]);
          ++consumed;
        }
        if (!ok) break;
        if (!kTileUnit) {
          mma_commit(&tfull[buf]);
          tphase ^= 1u << buf;
          buf ^= 1;
        }
        if (kTileUnit) u0 = total;  // the tile's whole diagonal went into this unit
      }
    }
    if (kTileUnit && ok) {
      mma_commit(&tfull[buf]);
      tphase ^= 1u << buf;
      buf ^= 1;
    }
  }
  // every issued MMA must finish before TMEM is released
  mma_commit(drain);
  volatile int no_abort = 0;
  (void)mbar_wait(drain, 0, &no_abort, P.status);
}

// ------------------------------------------------------------------ epilogues
// Ozaki: C(i,j) (+)= alpha * 2^(e_i + f_j - 12 - 7(t-2)) * D_t(i,j), diagonals from the
// smallest weight up; the first unit of a tile applies beta (beta == 0 never reads C).
// PAIR: the CTA is half of a 256-row pair tile (rows rank*128 .. +127) and releases the
// accumulator on the pair leader's barrier; otherwise it owns a 128-row tile.
template <int BN, bool PAIR>
__device__ __forceinline__ void acc_release(uint64_t* tempty_buf) {
  if (PAIR)
    mbar_arrive_cluster(mapa_shared(smem_u32(tempty_buf), 0));
  else
    mbar_arrive(tempty_buf);
}

template <int BN, bool PAIR>
__device__ __forceinline__ void ozaki_epilogue(uint32_t tmem_base, uint64_t* tfull, uint64_t* tempty, int* col_exp,
                                               volatile int* abort_flag, const SliceGemmParams& P) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3;  // TMEM lane quadrant this warp may access
  const int row = quad * 32 + lane;
  const int et = threadIdx.x - 64;  // 0..127
  const int num_tiles = P.tiles_m * P.tiles_n;
  double* C = static_cast<double*>(P.C);
  int buf = 0;
  uint32_t ephase = 0u;
  double err_hi = 0.0, err_lo = 0.0;
  bool ok = true;
  const int first = PAIR ? int(blockIdx.x >> 1) : int(blockIdx.x);
  const int step = PAIR ? int(gridDim.x >> 1) : int(gridDim.x);
  const int row_base = PAIR ? int(cluster_ctarank()) * kSliceBM : 0;
  for (int tile = first; tile < num_tiles && ok; tile += step) {
    int tm, tn;
    tile_coords(tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int64_t m0 = int64_t(tm) * (PAIR ? 2 * kSliceBM : kSliceBM) + row_base;
    const int64_t n0 = int64_t(tn) * BN;
    for (int j = et; j < BN; j += 128) {
      const int64_t col = n0 + j;
      col_exp[j] = (col < P.n) ? P.expB[col] : 0;
    }
    asm volatile("bar.sync 1, 128;" ::: "memory");
    const int64_t grow = m0 + row;
    const bool row_ok = grow < P.m;
    const int erow = row_ok ? P.expA[grow] : 0;
    bool first = P.first_writes != 0;
    for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
      int p_lo, total;
      if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total)) continue;
      const int wexp = -12 - 7 * (t - 2);
      // energy of the smallest diagonal (truncation estimate) and of t = 2 (|alpha*A*B| proxy)
      const int est = (P.err_sq == nullptr) ? 0 : (t == P.diag_hi ? 1 : 0) | (t == 2 ? 2 : 0);
      for (int u0 = 0; u0 < total && ok; u0 += kMaxUnitKb) {
        if (!mbar_wait(&tfull[buf], (ephase >> buf) & 1u, abort_flag, P.status)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem_base + uint32_t(buf * BN) + (uint32_t(quad * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < BN / 32; ++c) {
          uint32_t r[32];
          tmem_ld_32x32b_x32(taddr + uint32_t(c * 32), r);
          tmem_ld_wait();
          if (row_ok && erow != INT_MIN) {
            double* cp = C + grow + (n0 + c * 32) * P.ldc;
#pragma unroll
            for (int jj = 0; jj < 32; ++jj) {
              const int64_t col = n0 + c * 32 + jj;
              const int ce = col_exp[c * 32 + jj];
              if (col < P.n && ce != INT_MIN) {
                const double val = (static_cast<double>(static_cast<int32_t>(r[jj])) * exp2_int(erow + ce + wexp)) *
                                   P.alpha;
                double* dst = cp + int64_t(jj) * P.ldc;
                if (first)
                  *dst = (P.beta == 0.0) ? val : P.beta * *dst + val;
                else
                  *dst += val;
                if (est & 1) err_hi += val * val;
                if (est & 2) err_lo += val * val;
              }
            }
          }
        }
        tc_fence_before();
        acc_release<BN, PAIR>(&tempty[buf]);
        ephase ^= 1u << buf;
        buf ^= 1;
        first = false;
      }
    }
    asm volatile("bar.sync 1, 128;" ::: "memory");
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

// Split-BF16: C = alpha * acc + beta * C in FP32, one unit per tile.
template <int BN, bool PAIR>
__device__ __forceinline__ void bf16_epilogue(uint32_t tmem_base, uint64_t* tfull, uint64_t* tempty,
                                              volatile int* abort_flag, const SliceGemmParams& P) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3;
  const int row = quad * 32 + lane;
  const int num_tiles = P.tiles_m * P.tiles_n;
  float* C = static_cast<float*>(P.C);
  int buf = 0;
  uint32_t ephase = 0u;
  const int first = PAIR ? int(blockIdx.x >> 1) : int(blockIdx.x);
  const int step = PAIR ? int(gridDim.x >> 1) : int(gridDim.x);
  const int row_base = PAIR ? int(cluster_ctarank()) * kSliceBM : 0;
  for (int tile = first; tile < num_tiles; tile += step) {
    int tm, tn;
    tile_coords(tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int64_t m0 = int64_t(tm) * (PAIR ? 2 * kSliceBM : kSliceBM) + row_base;
    const int64_t n0 = int64_t(tn) * BN;
    if (!mbar_wait(&tfull[buf], (ephase >> buf) & 1u, abort_flag, P.status)) break;
    tc_fence_after();
    const uint32_t taddr = tmem_base + uint32_t(buf * BN) + (uint32_t(quad * 32) << 16);
    const int64_t grow = m0 + row;
#pragma unroll 1
    for (int c = 0; c < BN / 32; ++c) {
      uint32_t r[32];
      tmem_ld_32x32b_x32(taddr + uint32_t(c * 32), r);
      tmem_ld_wait();
      if (grow < P.m) {
        float* cp = C + grow + (n0 + c * 32) * P.ldc;
#pragma unroll
        for (int jj = 0; jj < 32; ++jj) {
          if (n0 + c * 32 + jj < P.n) {
            float* dst = cp + int64_t(jj) * P.ldc;
            const float v = P.alpha_f * __uint_as_float(r[jj]);
            *dst = (P.beta_f == 0.0f) ? v : P.beta_f * *dst + v;
          }
        }
      }
    }
    tc_fence_before();
    acc_release<BN, PAIR>(&tempty[buf]);
    ephase ^= 1u << buf;
    buf ^= 1;
  }
}

// ------------------------------------------------------------------ kernel
template <int MODE, int BN, int STAGES>
__global__ void __launch_bounds__(192, 1)
    slice_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const SliceGemmParams P) {
  using L = SliceSmemLayout<BN, STAGES>;
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

  if (threadIdx.x == 0) {
    for (int i = 0; i < STAGES; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 128);
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
    tmem_alloc(tmem_holder, 2 * BN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  if (warp == 0) {
    if (lane == 0) slice_producer<MODE, BN, STAGES>(&tmA, &tmB, smem, full, empty, abort_flag, P);
  } else if (warp == 1) {
    if (lane == 0) slice_mma<MODE, BN, STAGES>(smem, full, empty, tfull, tempty, drain, tmem_base, abort_flag, P);
  } else {
    if (MODE == kModeOzakiI8)
      ozaki_epilogue<BN, false>(tmem_base, tfull, tempty, col_exp, abort_flag, P);
    else
      bf16_epilogue<BN, false>(tmem_base, tfull, tempty, abort_flag, P);
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, 2 * BN);
}


// ======================================================================= CTA pairs
// A cluster of two CTAs computes a 256 x 256 tile with tcgen05 cta_group::2: each CTA
// loads its 128 rows of A and its 128 of the 256 rows of B per stage (32 KB, 6 stages)
// and holds its 128 x 256 half of the accumulator in its own TMEM; the leader (rank 0)
// issues the M = 256 MMAs.  Per SM this moves 2/3 of the bytes of the single-CTA tile
// for the same MMA work.  TMA loads carry no multicast; the leader commits separately to
// both CTAs' barriers.
constexpr int kPairBN = 256;

template <int STAGES>
struct SlicePairLayout {
  static constexpr int kABytes = kSliceBM * kSliceKBytes;          // 128 rows of A
  static constexpr int kBBytes = (kPairBN / 2) * kSliceKBytes;     // 128 rows of B
  static constexpr int kAOff = 0;
  static constexpr int kBOff = kAOff + STAGES * kABytes;
  static constexpr int kBarOff = kBOff + STAGES * kBBytes;
  static constexpr int kNumBars = 2 * STAGES + 5;
  static constexpr int kMiscOff = kBarOff + kNumBars * 8;
  static constexpr int kColExpOff = kMiscOff + 16;
  static constexpr int kTotal = kColExpOff + kPairBN * 4;
  static constexpr int kAlloc = kTotal + 1024;
};

template <int MODE, int STAGES>
__device__ __forceinline__ void pair_producer(const CUtensorMap* tmA, const CUtensorMap* tmB, uint8_t* smem,
                                              uint64_t* full, uint64_t* empty, volatile int* abort_flag,
                                              const SliceGemmParams& P, uint32_t rank) {
  using L = SlicePairLayout<STAGES>;
  constexpr int ke = SliceTraits<MODE>::kKElems;
  const int num_tiles = P.tiles_m * P.tiles_n;
  BlockIter it;
  it.start(P, num_tiles, int(blockIdx.x >> 1), int(gridDim.x >> 1));
  uint32_t issued = 0;
  while (it.valid) {
    int tm, tn;
    tile_coords(it.tile, P.tiles_m, P.tiles_n, P.group_m, tm, tn);
    const int p = it.p_lo + it.f / P.num_kb, kb = it.f % P.num_kb;
    const int stage = int(issued % STAGES);
    if (!mbar_wait(&empty[stage], ((issued / STAGES) & 1u) ^ 1u, abort_flag, P.status)) break;
    const uint32_t leader_full = mapa_shared(smem_u32(&full[stage]), 0);
    if (rank == 0) mbar_arrive_expect_tx(&full[stage], 2 * (L::kABytes + L::kBBytes));
    tma_load_3d_pair(smem + L::kAOff + stage * L::kABytes, tmA, leader_full, kb * ke,
                     tm * 2 * kSliceBM + int(rank) * kSliceBM, p - 1);
    tma_load_3d_pair(smem + L::kBOff + stage * L::kBBytes, tmB, leader_full, kb * ke,
                     tn * kPairBN + int(rank) * (kPairBN / 2), it.t - p - 1);
    ++issued;
    it.next(P, num_tiles);
  }
}

template <int MODE, int STAGES>
__device__ __forceinline__ void pair_mma(uint8_t* smem, uint64_t* full, uint64_t* empty, uint64_t* tfull,
                                         uint64_t* tempty, uint64_t* drain, uint32_t tmem_base,
                                         volatile int* abort_flag, const SliceGemmParams& P) {
  using L = SlicePairLayout<STAGES>;
  constexpr uint32_t idesc = MODE == kModeOzakiI8 ? make_idesc(2u, 1u, 1u, 2 * kSliceBM, kPairBN)
                                                  : make_idesc(1u, 1u, 1u, 2 * kSliceBM, kPairBN);
  constexpr bool kTileUnit = (MODE == kModeSplitBF16);
  const int num_tiles = P.tiles_m * P.tiles_n;
  uint32_t consumed = 0;
  int buf = 0;
  uint32_t tphase = 0u;
  bool ok = true;
  auto commit_both = [&](uint64_t* bar) {
    const uint32_t a = smem_u32(bar);
    mma_commit_pair(mapa_shared(a, 0));
    mma_commit_pair(mapa_shared(a, 1));
  };
  for (int tile = int(blockIdx.x >> 1); tile < num_tiles && ok; tile += int(gridDim.x >> 1)) {
    bool fresh = true;
    if (kTileUnit) {
      if (!mbar_wait(&tempty[buf], ((tphase >> buf) & 1u) ^ 1u, abort_flag, P.status)) break;
      tc_fence_after();
    }
    for (int t = P.diag_hi; t >= P.diag_lo && ok; --t) {
      int p_lo, total;
      if (!diag_bounds(t, P.slices, P.num_kb, p_lo, total)) continue;
      for (int u0 = 0; u0 < total && ok; u0 += kMaxUnitKb) {
        const int u1 = (kTileUnit || total - u0 <= kMaxUnitKb) ? total : u0 + kMaxUnitKb;
        if (!kTileUnit) {
          if (!mbar_wait(&tempty[buf], ((tphase >> buf) & 1u) ^ 1u, abort_flag, P.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          fresh = true;
        }
        const uint32_t d_tmem = tmem_base + uint32_t(buf * kPairBN);
        for (int f = u0; f < u1; ++f) {
          const int stage = int(consumed % STAGES);
          if (!mbar_wait(&full[stage], (consumed / STAGES) & 1u, abort_flag, P.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t adesc = make_sw128_kmajor_desc(smem_u32(smem + L::kAOff + stage * L::kABytes));
          const uint64_t bdesc = make_sw128_kmajor_desc(smem_u32(smem + L::kBOff + stage * L::kBBytes));
#pragma unroll
          for (int kk = 0; kk < kSliceKBytes / 32; ++kk) {
            const uint32_t acc = (fresh && kk == 0) ? 0u : 1u;
            if (MODE == kModeOzakiI8)
              mma_i8_pair(d_tmem, adesc + uint64_t(2 * kk), bdesc + uint64_t(2 * kk), idesc, acc);
            else
              mma_f16_pair(d_tmem, adesc + uint64_t(2 * kk), bdesc + uint64_t(2 * kk), idesc, acc);
          }
          fresh = false;
          commit_both(&empty[stage]);
          ++consumed;
        }
        if (!ok) break;
        if (!kTileUnit) {
          commit_both(&tfull[buf]);
          tphase ^= 1u << buf;
          buf ^= 1;
        }
        if (kTileUnit) u0 = total;
      }
    }
    if (kTileUnit && ok) {
      commit_both(&tfull[buf]);
      tphase ^= 1u << buf;
      buf ^= 1;
    }
  }
  mma_commit_pair(mapa_shared(smem_u32(drain), 0));
  volatile int no_abort = 0;
  (void)mbar_wait(drain, 0, &no_abort, P.status);
}

template <int MODE, int STAGES>
__global__ void __launch_bounds__(192, 1)
    slice_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                           const SliceGemmParams P) {
  using L = SlicePairLayout<STAGES>;
  // both CTAs of a pair read the same flag, so they leave together
  if (P.skip_if_flag && *P.skip_if_flag) return;

  extern __shared__ uint8_t pair_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(pair_smem_raw) + 1023) & ~uintptr_t(1023));
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
  const uint32_t rank = cluster_ctarank();

  if (threadIdx.x == 0) {
    for (int i = 0; i < STAGES; ++i) {
      mbar_init(&full[i], 1);   // the leader's expect_tx arrival + both CTAs' bytes
      mbar_init(&empty[i], 1);  // one commit from the leader's MMA thread
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tfull[i], 1);
      mbar_init(&tempty[i], 2 * 128);  // used on the leader: both CTAs' epilogue threads
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
    tmem_alloc_pair(tmem_holder, 2 * kPairBN);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync();  // barriers of both CTAs are initialised before any remote arrival
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  if (warp == 0) {
    if (lane == 0) pair_producer<MODE, STAGES>(&tmA, &tmB, smem, full, empty, abort_flag, P, rank);
  } else if (warp == 1) {
    if (lane == 0 && rank == 0)
      pair_mma<MODE, STAGES>(smem, full, empty, tfull, tempty, drain, tmem_base, abort_flag, P);
  } else {
    if (MODE == kModeOzakiI8)
      ozaki_epilogue<kPairBN, true>(tmem_base, tfull, tempty, col_exp, abort_flag, P);
    else
      bf16_epilogue<kPairBN, true>(tmem_base, tfull, tempty, abort_flag, P);
  }

  tc_fence_before();
  cluster_sync();  // the pair's MMAs are drained and both epilogues are done with TMEM
  tc_fence_after();
  if (warp == 1) tmem_dealloc_pair(tmem_base, 2 * kPairBN);
}


// Host-side launch of the pair kernel (grid = 2 CTAs per pair, clusters of 2).
template <int MODE, int STAGES>
inline cudaError_t launch_slice_pair(const CUtensorMap& tmA, const CUtensorMap& tmB, const SliceGemmParams& P,
                                     int num_sms, cudaStream_t stream) {
  using L = SlicePairLayout<STAGES>;
  auto kern = slice_gemm_pair_kernel<MODE, STAGES>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kAlloc);
  if (e != cudaSuccess) return e;
  const int tiles = P.tiles_m * P.tiles_n;
  const int pairs = tiles < num_sms / 2 ? tiles : num_sms / 2;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(2 * pairs), 1, 1);
  cfg.blockDim = dim3(192, 1, 1);
  cfg.dynamicSmemBytes = L::kAlloc;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, tmA, tmB, P);
}

}  // namespace eb2

