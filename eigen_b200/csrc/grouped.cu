// grouped.cu -- one persistent launch for thousands of independent small products.
//
// Eigen has no batch entry point: fixed-size products (3x3 ... 8x8) never reach GEBP
// but are unrolled coefficient-based products (Eigen/src/Core/GeneralProduct.h:76-80,
// Eigen/src/Core/ProductEvaluators.h:703-880), and dynamic ones each go through
// general_matrix_matrix_product.  Here a whole batch is one launch:
//   * the host cuts the batch into work items of three classes: class 32 = one 32 x 32
//     output tile of a product; class 16 = two whole products of at most 16 x 16; class 8 =
//     four whole products of at most 8 x 8 (Eigen's fixed-size range), so that small
//     products share a warp instead of each filling a 32 x 32 tile;
//   * every item is computed by ONE warp.  Its operands arrive in K-chunks ("stages") of two
//     32-line panels (rows of op(A), columns of op(B)) copied by cp.async into a per-warp
//     shared-memory ring with zero fill outside the products.  The copies of the next stages
//     -- of the next item too -- are in flight while the current stage computes, which is
//     what bounds these short, scattered products: the latency of their loads;
//   * FP64: mma.sync m16n8k4 (DMMA), K in steps of 4 from 0 upward for every output, the
//     same sequence as the native DGEMM kernel, so each product equals one plain native call
//     bit for bit;  FP32: split-BF16 on the tensor cores (x = h + m + l in bf16 pieces; the
//     six products hl, lh, mm, hm, mh, hh of every 16-deep chunk, mma.sync m16n8k16 with FP32
//     accumulation, added to the FP32 result with round-to-nearest);
//   * items are ordered longest-K first by the host and strided over the persistent warps;
//   * C = alpha*op(A)op(B) + beta*C per problem with the BLAS rules (beta == 0 never reads
//     C, alpha == 0 or k == 0 leaves beta*C and reads neither A nor B).
#include <cuda_bf16.h>

#include <cstdint>

#include "device_common.cuh"
#include "grouped.h"

namespace eb2 {

namespace {

constexpr int kLineStride = 36;  // a panel's k-row: 32 lines (rows of op(A) / columns of op(B)), padded
constexpr int kKc = 8;           // K per stage: two m16n8k4 steps (FP64) or one m16n8k8 step (FP32)
constexpr int kWarpsPerBlock = 2;

template <bool F64>
struct GroupedTraits;
template <>
struct GroupedTraits<true> {
  using T = double;
  static constexpr int kStages = 3;  // 13.8 KB per warp: eight two-warp blocks per SM
};
template <>
struct GroupedTraits<false> {
  using T = float;
  static constexpr int kStages = 6;  // 13.8 KB per warp
};
constexpr int kPanelElems = kKc * kLineStride;
constexpr int kStageElems = 2 * kPanelElems;

__device__ __forceinline__ void dmma_16x8x4_g(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void mma_bf16_1688(float (&d)[4], const uint32_t (&a)[2], uint32_t b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(b));
}

// x = h + m + l with h, m exact bf16 values and the remainder l (rounded to bf16 when packed);
// each difference is exact in FP32 (Henry, Tang & Heinecke, ARITH 2019)
__device__ __forceinline__ void split3(float x, float& h, float& m, float& l) {
  h = __bfloat162float(__float2bfloat16_rn(x));
  const float r1 = __fsub_rn(x, h);
  m = __bfloat162float(__float2bfloat16_rn(r1));
  l = __fsub_rn(r1, m);
}

// two values as one bf16x2 register (first value in the low half: the smaller k)
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// The items of a launch: the plan's list (grouped launch), or the 32 x 32 tiles of one
// product passed by value (the per-product launches of the same arithmetic).
struct PlanItems {
  const GroupedProblem* problems;
  const GroupedItem* items;
  int64_t count;
  __device__ __forceinline__ GroupedItem item(int64_t i) const { return items[i]; }
  __device__ __forceinline__ GroupedProblem problem(uint32_t p) const { return problems[p]; }
  __device__ __forceinline__ const void* dummy() const { return problems; }
};
struct OneProduct {
  GroupedProblem pr;
  int tiles_m;
  int64_t count;
  __device__ __forceinline__ GroupedItem item(int64_t i) const {
    GroupedItem it{};
    it.problem[0] = 0;
    it.problem[1] = it.problem[2] = it.problem[3] = kNoProblem;
    it.k = int32_t(pr.k);
    it.tile_m = uint16_t(i % tiles_m);
    it.tile_n = uint16_t(i / tiles_m);
    it.cls = 32;
    return it;
  }
  __device__ __forceinline__ GroupedProblem problem(uint32_t) const { return pr; }
  __device__ __forceinline__ const void* dummy() const { return pr.c; }
};

__device__ __forceinline__ uint32_t slot_problem(const GroupedItem& it, int q) {
  // (a select chain: an indexed read of the item would put it in local memory)
  return q == 0 ? it.problem[0] : (q == 1 ? it.problem[1] : (q == 2 ? it.problem[2] : it.problem[3]));
}

// One panel's copies for one lane: the lanes of problem slot q are lanes q*R .. q*R+R-1 (R =
// the item's class: lines per problem).  Along the panel's contiguous direction consecutive
// lanes take consecutive elements: if the lines are contiguous (op(A) not transposed, op(B)
// transposed) lane ls takes line ls and element t is K offset t; otherwise lane ls takes K
// offset ls % 8 of lines ls / 8 + t R/8.  Either way the address, the shared-memory slot, the
// K offset and the line of element t are affine in t.  Extents fit 32 bits: a plan holds at
// most 65535 tiles of 32 per side, and its items' K are 32-bit.
template <typename T>
struct PanelCopy {
  const T* ptr;     // element t = 0 at K chunk 0
  int64_t ld;       // the operand's leading dimension
  int line0, kk0;   // line and K offset of element t = 0
  int dline;        // lines contiguous: 0 (element t is K offset kk0 + t); else R/8 (line0 + t*dline)
  int lines, k;     // the product's extent along the lines, and its K (0: empty slot)
  uint32_t dst0;    // shared-memory byte offset of element t = 0 within the panel

  __device__ __forceinline__ void set(const T* base, int64_t ldx, bool lines_contig, int first_line, int slot_off,
                                      int ls, int r, int64_t extent, int64_t kdim) {
    ld = ldx;
    lines = int(extent);
    k = int(kdim);
    if (lines_contig) {  // X(line, kk) = base[line + kk * ld]
      line0 = first_line + ls;
      dline = 0;
      kk0 = 0;
      ptr = base + line0;
      dst0 = uint32_t((slot_off + ls) * sizeof(T));
    } else {  // X(line, kk) = base[kk + line * ld]
      line0 = first_line + ls / kKc;
      dline = r / kKc;
      kk0 = ls % kKc;
      ptr = base + kk0 + int64_t(line0) * ld;
      dst0 = uint32_t((kk0 * kLineStride + slot_off + ls / kKc) * sizeof(T));
    }
  }

  __device__ __forceinline__ void issue(uint32_t panel, int k0, const void* dummy) const {
    const bool contig = dline == 0;
    const int dkk = contig ? 1 : 0;
    const int64_t step_t = contig ? ld : int64_t(dline) * ld;
    const uint32_t dst_step = uint32_t((contig ? kLineStride : dline) * sizeof(T));
    const T* p = ptr + (contig ? int64_t(k0) * ld : int64_t(k0));
    // the whole stage inside the product: no per-element checks
    const bool inside = k0 + kk0 + (kKc - 1) * dkk < k && line0 + (kKc - 1) * dline < lines;
    uint32_t d = panel + dst0;
    if (inside) {
#pragma unroll
      for (int t = 0; t < kKc; ++t, p += step_t, d += dst_step) cp_async_elem<sizeof(T)>(d, p, true);
    } else {
#pragma unroll
      for (int t = 0; t < kKc; ++t, p += step_t, d += dst_step) {
        const bool v = k0 + kk0 + t * dkk < k && line0 + t * dline < lines;
        cp_async_elem<sizeof(T)>(d, v ? static_cast<const void*>(p) : dummy, v);
      }
    }
  }
};

// The copies of one stage of an item for one lane: its slot's rows of op(A) and columns of op(B).
template <bool F64, class Src>
struct StageCopier {
  using T = typename GroupedTraits<F64>::T;
  PanelCopy<T> pa, pb;
  const void* dummy;

  __device__ __forceinline__ void load(const Src& src, const GroupedItem& it, int lane) {
    const int r = it.cls;
    const int log_r = r == 8 ? 3 : (r == 16 ? 4 : 5);
    const int q = lane >> log_r;
    const int ls = lane & (r - 1);
    dummy = src.dummy();
    const uint32_t pid = slot_problem(it, q);
    const bool ok = pid != kNoProblem;
    const GroupedProblem pr = ok ? src.problem(pid) : GroupedProblem{};
    const T* a = static_cast<const T*>(ok ? pr.a : dummy);
    const T* b = static_cast<const T*>(ok ? pr.b : dummy);
    const int first_a = r == 32 ? int(it.tile_m) * 32 : 0, first_b = r == 32 ? int(it.tile_n) * 32 : 0;
    // op(A)(i, l): contiguous along i unless transposed; op(B)(l, j): along j only if transposed
    pa.set(a, pr.lda, (pr.trans & 1) == 0, first_a, q * r, ls, r, ok ? pr.m : 0, ok ? pr.k : 0);
    pb.set(b, pr.ldb, (pr.trans & 2) != 0, first_b, q * r, ls, r, ok ? pr.n : 0, ok ? pr.k : 0);
  }

  __device__ __forceinline__ void issue(T* stage, int k0) const {
    const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(stage));
    pa.issue(sa, k0, dummy);
    pb.issue(sa + uint32_t(kPanelElems * sizeof(T)), k0, dummy);
  }
};

// ---------------------------------------------------------------- FP64 compute
// Accumulator fragments: class 32: (row block i, column block j) -> i*4 + j; class 16:
// (problem p, column block j) -> p*2 + j; class 8: problem p -> p (rows 8-15 unused).
__device__ __forceinline__ void compute_f64(double (&acc)[8][4], const double* st, int cls, int g, int tig) {
  const double* sA = st;
  const double* sB = st + kPanelElems;
#pragma unroll
  for (int ks = 0; ks < 2; ++ks) {
    const int kr = (ks * 4 + tig) * kLineStride;
    if (cls == 32) {
      double a[2][2], b[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        a[i][0] = sA[kr + i * 16 + g];
        a[i][1] = sA[kr + i * 16 + g + 8];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sB[kr + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_16x8x4_g(acc[i * 4 + j], a[i][0], a[i][1], b[j]);
    } else if (cls == 16) {
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        const double a0 = sA[kr + p * 16 + g], a1 = sA[kr + p * 16 + g + 8];
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma_16x8x4_g(acc[p * 2 + j], a0, a1, sB[kr + p * 16 + j * 8 + g]);
      }
    } else {
#pragma unroll
      for (int p = 0; p < 4; ++p) dmma_16x8x4_g(acc[p], sA[kr + p * 8 + g], 0.0, sB[kr + p * 8 + g]);
    }
  }
}

// ---------------------------------------------------------------- FP32 (split-BF16) compute
// The m16n8k8 A fragment of the 16 lines at l0 (rows 8-15 zero when `half`) and the B
// fragment of the 8 lines at l0, each as its three bf16 pieces.
__device__ __forceinline__ void frag_a(const float* sA, int l0, bool half, int g, int tig, uint32_t (&p)[3][2]) {
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int row = l0 + g + 8 * r;
    const bool zero = half && r == 1;
    const float x0 = zero ? 0.f : sA[(2 * tig) * kLineStride + row];
    const float x1 = zero ? 0.f : sA[(2 * tig + 1) * kLineStride + row];
    float h0, m0, l0v, h1, m1, l1v;
    split3(x0, h0, m0, l0v);
    split3(x1, h1, m1, l1v);
    p[0][r] = pack_bf16(h0, h1);
    p[1][r] = pack_bf16(m0, m1);
    p[2][r] = pack_bf16(l0v, l1v);
  }
}
__device__ __forceinline__ void frag_b(const float* sB, int l0, int g, int tig, uint32_t (&p)[3]) {
  float h0, m0, x0, h1, m1, x1;
  split3(sB[(2 * tig) * kLineStride + l0 + g], h0, m0, x0);
  split3(sB[(2 * tig + 1) * kLineStride + l0 + g], h1, m1, x1);
  p[0] = pack_bf16(h0, h1);
  p[1] = pack_bf16(m0, m1);
  p[2] = pack_bf16(x0, x1);
}
// the six piece products of one 8-deep chunk, smallest first, into a fresh fragment that is
// then added to the result (round to nearest)
__device__ __forceinline__ void chunk_product(float (&acc)[4], const uint32_t (&pa)[3][2], const uint32_t (&pb)[3]) {
  float d[4] = {0.f, 0.f, 0.f, 0.f};
  mma_bf16_1688(d, pa[0], pb[2]);  // h l
  mma_bf16_1688(d, pa[2], pb[0]);  // l h
  mma_bf16_1688(d, pa[1], pb[1]);  // m m
  mma_bf16_1688(d, pa[0], pb[1]);  // h m
  mma_bf16_1688(d, pa[1], pb[0]);  // m h
  mma_bf16_1688(d, pa[0], pb[0]);  // h h
#pragma unroll
  for (int e = 0; e < 4; ++e) acc[e] = __fadd_rn(acc[e], d[e]);
}

__device__ __forceinline__ void compute_f32(float (&acc)[8][4], const float* st, int cls, int g, int tig) {
  const float* sA = st;
  const float* sB = st + kPanelElems;
  if (cls == 32) {
    uint32_t pa[2][3][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) frag_a(sA, i * 16, false, g, tig, pa[i]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uint32_t pb[3];
      frag_b(sB, j * 8, g, tig, pb);
#pragma unroll
      for (int i = 0; i < 2; ++i) chunk_product(acc[i * 4 + j], pa[i], pb);
    }
  } else if (cls == 16) {
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      uint32_t pa[3][2];
      frag_a(sA, p * 16, false, g, tig, pa);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        uint32_t pb[3];
        frag_b(sB, p * 16 + j * 8, g, tig, pb);
        chunk_product(acc[p * 2 + j], pa, pb);
      }
    }
  } else {
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      uint32_t pa[3][2], pb[3];
      frag_a(sA, p * 8, true, g, tig, pa);
      frag_b(sB, p * 8, g, tig, pb);
      chunk_product(acc[p], pa, pb);
    }
  }
}

// ---------------------------------------------------------------- epilogue
// C = alpha * acc + beta * C for the fragment elements of one product: element (h, c) of the
// fragment at rows r0.., columns c0.. is row r0 + g + 8h, column c0 + 2 tig + c.  The
// descriptor's fields are copied to registers first (C stores could otherwise alias them).
template <typename T, int NF>
struct ProductStore {
  T* c;
  int64_t ldc, m, n;
  T alpha, beta;
  __device__ __forceinline__ void load(const GroupedProblem& pr) {
    c = static_cast<T*>(pr.c);
    ldc = pr.ldc;
    m = pr.m;
    n = pr.n;
    alpha = T(pr.alpha);
    beta = T(pr.beta);
  }
  __device__ __forceinline__ void put(int64_t row, int64_t col, T v) const {
    if (row < m && col < n) {
      T* dst = c + row + col * ldc;
      const T a = sizeof(T) == 8 ? T(__dmul_rn(double(alpha), double(v))) : T(__fmul_rn(float(alpha), float(v)));
      if (beta == T(0))
        *dst = a;
      else if constexpr (sizeof(T) == 8)
        *dst = __fma_rn(double(beta), double(*dst), double(a));
      else
        *dst = __fmaf_rn(float(beta), float(*dst), float(a));
    }
  }
};

template <typename T, class Src>
__device__ __forceinline__ void epilogue(const Src& src, const GroupedItem& it, T (&acc)[8][4], int g, int tig) {
  ProductStore<T, 8> ps;
  if (it.cls == 32) {
    ps.load(src.problem(it.problem[0]));
    const int64_t r0 = int64_t(it.tile_m) * 32 + g, c0 = int64_t(it.tile_n) * 32 + 2 * tig;
#pragma unroll
    for (int f = 0; f < 8; ++f)
#pragma unroll
      for (int e = 0; e < 4; ++e) ps.put(r0 + (f >> 2) * 16 + (e >> 1) * 8, c0 + (f & 3) * 8 + (e & 1), acc[f][e]);
  } else if (it.cls == 16) {
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const uint32_t pid = p == 0 ? it.problem[0] : it.problem[1];
      if (pid == kNoProblem) continue;
      ps.load(src.problem(pid));
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) ps.put(g + (e >> 1) * 8, j * 8 + tig * 2 + (e & 1), acc[p * 2 + j][e]);
    }
  } else {
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const uint32_t pid = slot_problem(it, p);
      if (pid == kNoProblem) continue;
      ps.load(src.problem(pid));
#pragma unroll
      for (int e = 0; e < 2; ++e) ps.put(g, tig * 2 + e, acc[p][e]);
    }
  }
}

// ---------------------------------------------------------------- the warp's pipeline
// Items w0, w0 + W, w0 + 2W, ... in stage order; copies run kStages - 1 stages ahead of the
// compute, across item boundaries.
template <bool F64, class Src>
__device__ __forceinline__ void run_items(const Src& src, int64_t w0, int64_t W,
                                          typename GroupedTraits<F64>::T* ring) {
  using T = typename GroupedTraits<F64>::T;
  constexpr int S = GroupedTraits<F64>::kStages;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, tig = lane & 3;
  auto stages_of = [](const GroupedItem& it) { return it.k > 0 ? (int(it.k) + kKc - 1) / kKc : 1; };

  // producer position
  int64_t p_idx = w0;
  int p_stage = 0, p_stages = 0;
  StageCopier<F64, Src> cp;
  if (p_idx < src.count) {
    const GroupedItem it = src.item(p_idx);
    cp.load(src, it, lane);
    p_stages = stages_of(it);
  }
  auto produce = [&](int slot) {
    if (p_idx < src.count) {
      cp.issue(ring + slot * kStageElems, p_stage * kKc);
      if (++p_stage == p_stages) {
        p_stage = 0;
        p_idx += W;
        if (p_idx < src.count) {
          const GroupedItem it = src.item(p_idx);
          cp.load(src, it, lane);
          p_stages = stages_of(it);
        }
      }
    }
    cp_async_commit();  // an empty group past the end keeps the group count uniform
  };
#pragma unroll
  for (int s = 0; s < S - 1; ++s) produce(s);

  // consumer position
  int64_t c_idx = w0;
  int c_stage = 0;
  GroupedItem cur{};
  int c_stages = 0;
  if (c_idx < src.count) {
    cur = src.item(c_idx);
    c_stages = stages_of(cur);
  }
  T acc[8][4];
#pragma unroll
  for (int f = 0; f < 8; ++f)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[f][e] = T(0);
  int slot = 0;
  while (c_idx < src.count) {
    cp_async_wait<S - 2>();
    __syncwarp();  // every lane's copies of this stage have landed; the slot refilled below is free
    produce(slot == 0 ? S - 1 : slot - 1);
    const T* st = ring + slot * kStageElems;
    if constexpr (F64)
      compute_f64(acc, st, cur.cls, g, tig);
    else
      compute_f32(acc, st, cur.cls, g, tig);
    slot = slot == S - 1 ? 0 : slot + 1;
    if (++c_stage == c_stages) {
      epilogue(src, cur, acc, g, tig);
#pragma unroll
      for (int f = 0; f < 8; ++f)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[f][e] = T(0);
      c_stage = 0;
      c_idx += W;
      if (c_idx < src.count) {
        cur = src.item(c_idx);
        c_stages = stages_of(cur);
      }
    }
  }
  cp_async_wait<0>();  // no copy may outlive the warp (the trailing groups are empty)
}

template <bool F64>
constexpr size_t warp_ring_bytes() {
  return size_t(GroupedTraits<F64>::kStages) * kStageElems * sizeof(typename GroupedTraits<F64>::T);
}

template <bool F64>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 8) grouped_gemm_kernel(const GroupedProblem* __restrict__ problems,
                                                                          const GroupedItem* __restrict__ items,
                                                                          int64_t num_items) {
  extern __shared__ __align__(16) unsigned char grouped_smem[];
  using T = typename GroupedTraits<F64>::T;
  const int warp = threadIdx.x >> 5;
  T* ring = reinterpret_cast<T*>(grouped_smem) + size_t(warp) * GroupedTraits<F64>::kStages * kStageElems;
  const PlanItems src{problems, items, num_items};
  run_items<F64>(src, int64_t(blockIdx.x) * kWarpsPerBlock + warp, int64_t(gridDim.x) * kWarpsPerBlock, ring);
}

// One product, one warp per 32 x 32 tile: the per-product launches of the same arithmetic.
template <bool F64>
__global__ void __launch_bounds__(32) grouped_one_kernel(const GroupedProblem pr, int tiles_m, int64_t tiles) {
  extern __shared__ __align__(16) unsigned char grouped_smem[];
  using T = typename GroupedTraits<F64>::T;
  const OneProduct src{pr, tiles_m, tiles};
  run_items<F64>(src, int64_t(blockIdx.x), int64_t(gridDim.x), reinterpret_cast<T*>(grouped_smem));
}

cudaError_t set_smem(const void* kern, size_t bytes) {
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

}  // namespace

size_t grouped_block_smem(bool f64) {
  return kWarpsPerBlock * (f64 ? warp_ring_bytes<true>() : warp_ring_bytes<false>());
}

cudaError_t grouped_grid(bool f64, int64_t num_items, int num_sms, unsigned* blocks) {
  *blocks = 0;
  const size_t smem = grouped_block_smem(f64);
  const void* kern = f64 ? reinterpret_cast<const void*>(grouped_gemm_kernel<true>)
                         : reinterpret_cast<const void*>(grouped_gemm_kernel<false>);
  cudaError_t e = set_smem(kern, smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kWarpsPerBlock, smem);
  if (e != cudaSuccess) return e;
  int64_t b = (num_items + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const int64_t cap = int64_t(num_sms) * (per_sm > 0 ? per_sm : 1);
  if (b > cap) b = cap;
  *blocks = unsigned(b > 0 ? b : 0);
  return cudaSuccess;
}

cudaError_t launch_grouped_gemm(bool f64, const GroupedProblem* problems, const GroupedItem* items,
                                int64_t num_items, unsigned blocks, cudaStream_t stream) {
  if (num_items <= 0 || blocks == 0) return cudaSuccess;
  const size_t smem = grouped_block_smem(f64);
  if (f64)
    grouped_gemm_kernel<true><<<blocks, 32 * kWarpsPerBlock, smem, stream>>>(problems, items, num_items);
  else
    grouped_gemm_kernel<false><<<blocks, 32 * kWarpsPerBlock, smem, stream>>>(problems, items, num_items);
  return cudaGetLastError();
}

cudaError_t launch_grouped_one(bool f64, const GroupedProblem& pr, cudaStream_t stream) {
  if (pr.m <= 0 || pr.n <= 0) return cudaSuccess;
  const int64_t tm = (pr.m + 31) / 32, tn = (pr.n + 31) / 32;
  if (tm > 65535 || tn > 65535) return cudaErrorInvalidValue;
  const size_t smem = f64 ? warp_ring_bytes<true>() : warp_ring_bytes<false>();
  cudaError_t e = f64 ? set_smem(reinterpret_cast<const void*>(grouped_one_kernel<true>), smem)
                      : set_smem(reinterpret_cast<const void*>(grouped_one_kernel<false>), smem);
  if (e != cudaSuccess) return e;
  const int64_t tiles = tm * tn;
  const unsigned grid = unsigned(tiles < 65535 ? tiles : 65535);
  if (f64)
    grouped_one_kernel<true><<<grid, 32, smem, stream>>>(pr, int(tm), tiles);
  else
    grouped_one_kernel<false><<<grid, 32, smem, stream>>>(pr, int(tm), tiles);
  return cudaGetLastError();
}

}  // namespace eb2
