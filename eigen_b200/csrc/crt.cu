// crt.cu -- FP64 GEMM emulated with integer residues (Ozaki scheme II, CRT form).
//
// Method (Ozaki, Uchino & Imamura, "Ozaki Scheme II: A GEMM-oriented emulation of
// floating-point matrix multiplication using an integer modular technique", 2025), here
// with exact multi-word integer reconstruction:
//   * every row i of op(A) is scaled by 2^mu_i and truncated to integers A', every row j
//     of op(B)^T by 2^nu_j to B', with mu_i, nu_j chosen from upper bounds of the rows'
//     2-norms so that ||A'_i||_2, ||B'_j||_2 <= 2^b; then |C'_ij| = |A'_i . B'_j| <= 2^(2b)
//     (Cauchy-Schwarz) and b is the largest integer with 2^(2b+1) < P = p_1 ... p_N, the
//     product of N pairwise coprime moduli <= 256;
//   * for each modulus the residues A' mod p, B' mod p (symmetric int8) are multiplied
//     exactly on the INT8 tensor cores (INT32 accumulation) and reduced mod p: N GEMMs
//     instead of the s(s+1)/2 of the digit-slice scheme (slice_gemm.cuh, CRT mode);
//   * C' is recovered from its N residues by the Chinese remainder theorem,
//     C' = sum_l r_l W_l mod P, W_l = (P/p_l) * ((P/p_l)^-1 mod p_l), in exact 192-bit
//     integer arithmetic, taken in (-P/2, P/2) (|C'| < P/2, so it is C' itself), rounded
//     once to FP64 and scaled: C = alpha * (C' 2^-(mu_i + nu_j)) (+ beta * C).
// The only approximation is the truncation A'_il = trunc(2^mu_i a_il) (error < 1 unit):
// with 16 moduli b = 62, i.e. 62 bits per row relative to the row's 2-norm.
//
// Every step is deterministic (integer norm bounds, exact products), so results are
// reproducible bit for bit and can be checked against an exact CPU model.
#include <cuda.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>

#include "device_common.cuh"
#include "kernels.h"
#include "slice_gemm.cuh"
#include "tma_host.h"

namespace eb2 {

// ------------------------------------------------------------------ host constants
namespace {

constexpr int kLimbs = kCrtLimbs;  // 192-bit integers, base 2^32

struct Big {
  uint32_t w[kLimbs] = {0, 0, 0, 0, 0, 0};
};

void big_mul_small(Big& a, uint32_t s) {
  uint64_t carry = 0;
  for (int i = 0; i < kLimbs; ++i) {
    const uint64_t v = uint64_t(a.w[i]) * s + carry;
    a.w[i] = uint32_t(v);
    carry = v >> 32;
  }
}

uint32_t big_div_small(Big& a, uint32_t s) {  // a /= s, returns a mod s
  uint64_t rem = 0;
  for (int i = kLimbs - 1; i >= 0; --i) {
    const uint64_t cur = (rem << 32) | a.w[i];
    a.w[i] = uint32_t(cur / s);
    rem = cur % s;
  }
  return uint32_t(rem);
}

int big_bits(const Big& a) {  // bit length
  for (int i = kLimbs - 1; i >= 0; --i)
    if (a.w[i]) return 32 * i + 32 - __builtin_clz(a.w[i]);
  return 0;
}

bool big_is_pow2(const Big& a) {
  int ones = 0;
  for (int i = 0; i < kLimbs; ++i) ones += __builtin_popcount(a.w[i]);
  return ones == 1;
}

double big_to_double(const Big& a) {
  double d = 0.0;
  for (int i = kLimbs - 1; i >= 0; --i) d = d * 4294967296.0 + double(a.w[i]);
  return d;
}

uint32_t inverse_mod(uint32_t a, uint32_t p) {  // a^-1 mod p (gcd(a, p) == 1)
  int64_t t = 0, nt = 1, r = p, nr = a % p;
  while (nr) {
    const int64_t q = r / nr;
    int64_t tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  return uint32_t(t < 0 ? t + p : t);
}

}  // namespace

int crt_bits(int n) {
  Big P;
  P.w[0] = 1;
  for (int l = 0; l < n; ++l) big_mul_small(P, uint32_t(crt_modulus(l)));
  // largest b with 2^(2b+1) < P: 2b+1 <= bits(P) - 1, minus one more when P = 2^(bits-1)
  const int L = big_bits(P);
  int b = (L - 2) / 2;
  if (big_is_pow2(P) && 2 * b + 1 == L - 1) --b;
  return b;
}

const CrtConstants& crt_constants(int n) {
  static CrtConstants table[kCrtMaxModuli + 1];
  static bool ready[kCrtMaxModuli + 1] = {};
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  CrtConstants& c = table[n];
  if (ready[n]) return c;
  std::memset(&c, 0, sizeof(c));
  c.n = n;
  Big P;
  P.w[0] = 1;
  for (int l = 0; l < n; ++l) big_mul_small(P, uint32_t(crt_modulus(l)));
  for (int l = 0; l < n; ++l) {
    const uint32_t p = uint32_t(crt_modulus(l));
    Big M = P;
    (void)big_div_small(M, p);  // M = P / p_l
    Big Mm = M;
    const uint32_t m_mod = big_div_small(Mm, p);
    Big W = M;
    big_mul_small(W, inverse_mod(m_mod, p));  // (P/p) * inv < P
    for (int i = 0; i < kLimbs; ++i) c.W[l][i] = W.w[i];
  }
  for (int i = 0; i < kLimbs; ++i) c.P[i] = P.w[i];
  Big half = P;
  (void)big_div_small(half, 2);
  for (int i = 0; i < kLimbs; ++i) c.half[i] = half.w[i];
  c.P_inv = 1.0 / big_to_double(P);
  c.b = crt_bits(n);
  ready[n] = true;
  return c;
}

// ------------------------------------------------------------------ kernels
namespace {

constexpr uint64_t kInfBitsCrt = 0x7FF0000000000000ull;
constexpr int kNormRows = 32;
constexpr int kNormCols = 128;
constexpr int kNormThreads = 256;

// A ROWS x COLS tile of op(X) (row r, column l at X[r*sr + l*sl], zero outside rows x cols)
// into shared memory by cp.async: all ROWS*COLS/THREADS copies of a thread are in flight at
// once without holding registers; consecutive lanes take consecutive addresses along
// whichever of the two strides is 1.  The caller synchronises the block afterwards.
template <int ROWS, int COLS, int THREADS>
__device__ __forceinline__ void load_tile(double (&tile)[ROWS][COLS + 1], const double* __restrict__ X, int64_t r0,
                                          int64_t l0, int64_t rows, int64_t cols, int64_t sr, int64_t sl) {
  static_assert(THREADS % ROWS == 0 && THREADS % COLS == 0, "a fixed row or column per thread");
  constexpr int kPer = ROWS * COLS / THREADS;
  const int t = int(threadIdx.x);
  if (sr == 1) {
    // lanes along the rows (contiguous); each thread keeps its row and steps through columns
    constexpr int kStep = THREADS / ROWS;
    const int rr = t % ROWS, l_first = t / ROWS;
    const int64_t r = r0 + rr;
    const double* src = X + r + (l0 + l_first) * sl;
    uint32_t dst = smem_u32(&tile[rr][l_first]);
#pragma unroll
    for (int q = 0; q < kPer; ++q, src += kStep * sl, dst += kStep * 8) {
      const bool valid = r < rows && l0 + l_first + q * kStep < cols;
      cp_async_elem<8>(dst, valid ? src : X, valid);
    }
  } else {
    // lanes along the columns; each thread keeps its column and steps through rows
    constexpr int kStep = THREADS / COLS;
    const int ll = t % COLS, r_first = t / COLS;
    const int64_t l = l0 + ll;
    const double* src = X + (r0 + r_first) * sr + l * sl;
    uint32_t dst = smem_u32(&tile[r_first][ll]);
#pragma unroll
    for (int q = 0; q < kPer; ++q, src += kStep * sr, dst += kStep * (COLS + 1) * 8) {
      const bool valid = l < cols && r0 + r_first + q * kStep < rows;
      cp_async_elem<8>(dst, valid ? src : X, valid);
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
}

// exponent e of a finite nonzero |x| given by its bit pattern: |x| in [2^(e-1), 2^e)
__device__ __forceinline__ int frexp_exp(unsigned long long mb) {
  int e;
  frexp(__longlong_as_double(static_cast<long long>(mb)), &e);
  return e;
}

// x * 2^e for |e| <= 2200 as two exact power-of-two products (one rounding at most, in
// the second product, when the result is subnormal)
__device__ __forceinline__ double scale2(double x, int e) {
  const int e1 = e / 2;
  return __dmul_rn(__dmul_rn(x, exp2_int(e1)), exp2_int(e - e1));
}

// One read of the operand for everything the scale exponents need.  Per row r and 128-column
// chunk c (columns 128c .. 128c+127 of op(X)^T's row, i.e. along K):
//   * the chunk maximum: row maxima (atomicMax), the NaN/Inf flag, and the exponent-spread
//     statistic of the configuration picker (the first 64 columns of every 512, as the
//     digit-slice scan computes it);
//   * e_c, the exponent of the chunk maximum, and the deterministic integer bound
//     S_c = sum over nonzero x of ceil(rn(x'^2) 2^32) + 1, x' = x 2^-e_c (|x'| < 1); the +1
//     covers the rounding of x'^2 and a product that underflows.
// Every (row, chunk) record is written by exactly one thread group.
__global__ void __launch_bounds__(kNormThreads) crt_scan_norm_kernel(const double* __restrict__ X, int64_t rows, int64_t cols,
                                                            int64_t sr, int64_t sl, unsigned long long* maxbits,
                                                            int32_t* __restrict__ chunk_e,
                                                            unsigned long long* __restrict__ chunk_s,
                                                            int64_t nchunks, int* nonfinite, double* spread) {
  __shared__ double tile[kNormRows][kNormCols + 1];
  __shared__ double spread_part[2][kNormThreads / 32];
  const int64_t r0 = int64_t(blockIdx.y) * kNormRows;
  const int64_t l0 = int64_t(blockIdx.x) * kNormCols;
  load_tile<kNormRows, kNormCols, kNormThreads>(tile, X, r0, l0, rows, cols, sr, sl);
  __syncthreads();
  // 8 threads per row, reduced with shuffles inside each 8-lane group; thread `sub` takes
  // columns sub, sub + 8, ..., so that the 8 lanes of a row read 8 consecutive words of the
  // tile (no shared-memory bank conflicts)
  const int rr = threadIdx.x >> 3;
  const int sub = threadIdx.x & 7;
  const int64_t r = r0 + rr;
  // the spread statistic: the first 64 columns of every 512 (block-uniform)
  const bool stat = spread != nullptr && (l0 & 511) == 0;
  // bit patterns of |x| order like the values, NaN above +Inf
  unsigned long long mb = 0, mb64 = 0;
  int esum = 0, ecnt = 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const unsigned long long bits =
        static_cast<unsigned long long>(__double_as_longlong(fabs(tile[rr][sub + 8 * j])));
    mb = bits > mb ? bits : mb;
    if (stat && j < 8) {
      mb64 = bits > mb64 ? bits : mb64;
      if (bits) {
        esum += int(bits >> 52);
        ++ecnt;
      }
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, mb, o);
    mb = other > mb ? other : mb;
    if (stat) {
      const unsigned long long other64 = __shfl_xor_sync(0xffffffffu, mb64, o);
      mb64 = other64 > mb64 ? other64 : mb64;
      esum += __shfl_xor_sync(0xffffffffu, esum, o);
      ecnt += __shfl_xor_sync(0xffffffffu, ecnt, o);
    }
  }
  unsigned long long s = 0;
  int e = 0;
  if (mb != 0 && mb < kInfBitsCrt) {
    e = frexp_exp(mb);
    // scale2(x, -e) with its two power-of-two factors formed once
    const double f1 = exp2_int((-e) / 2), f2 = exp2_int(-e - (-e) / 2);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const double x = tile[rr][sub + 8 * j];
      const double xs = __dmul_rn(__dmul_rn(x, f1), f2);
      // ceil(v) for v = rn(x'^2) 2^32 in [0, 2^32]: v + 2^52 rounded up is 2^52 + ceil(v)
      // exactly, read from its bits (no rounding or conversion instruction)
      const double v = __dmul_rn(__dmul_rn(xs, xs), 4294967296.0);
      const unsigned long long c = static_cast<unsigned long long>(__double_as_longlong(__dadd_ru(v, 0x1p52)) -
                                                                   __double_as_longlong(0x1p52));
      s += x != 0.0 ? c + 1ull : 0ull;
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (sub == 0 && r < rows) {
    const int64_t c = int64_t(blockIdx.x);
    chunk_e[r * nchunks + c] = e;
    chunk_s[r * nchunks + c] = mb < kInfBitsCrt ? s : 0ull;
    if (mb >= kInfBitsCrt) *nonfinite = 1;
    if (mb) atomicMax(&maxbits[r], mb);
  }
  if (stat) {
    double chunk_spread = 0.0, chunk_count = 0.0;
    if (sub == 0 && r < rows && ecnt > 0 && mb64 < kInfBitsCrt) {
      chunk_spread = double(int(mb64 >> 52)) - double(esum) / double(ecnt);
      chunk_count = 1.0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      chunk_spread += __shfl_xor_sync(0xffffffffu, chunk_spread, o);
      chunk_count += __shfl_xor_sync(0xffffffffu, chunk_count, o);
    }
    // one atomic pair per block: same-address atomics serialise in L2
    if ((threadIdx.x & 31) == 0) {
      spread_part[0][threadIdx.x >> 5] = chunk_spread;
      spread_part[1][threadIdx.x >> 5] = chunk_count;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.0, count = 0.0;
#pragma unroll
      for (int w = 0; w < kNormThreads / 32; ++w) {
        sum += spread_part[0][w];
        count += spread_part[1][w];
      }
      if (count > 0.0) {
        atomicAdd(&spread[0], sum);
        atomicAdd(&spread[1], count);
      }
    }
  }
}

// Scale exponent of each row: with e the row maximum's exponent, the chunk bounds fold into
// S = sum_c ceil(S_c 4^(e_c - e)) (exact shifts), ||x||^2 <= S 2^(2e-32), S <= 2^L (L = bit
// length of S-1), so 2^c >= ||x|| for c = e - 16 + ceil(L/2) and mu = b - c.
__global__ void __launch_bounds__(256) crt_mu_kernel(const unsigned long long* __restrict__ maxbits,
                                                     const int32_t* __restrict__ chunk_e,
                                                     const unsigned long long* __restrict__ chunk_s, int64_t nchunks,
                                                     int64_t rows, int64_t rows_pad, int b, int32_t* __restrict__ mu) {
  // one warp per row: the lanes read consecutive chunk records
  const int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = int(threadIdx.x & 31);
  if (r >= rows_pad) return;  // whole warps
  int m = kCrtZeroRow;
  const unsigned long long mb = r < rows ? maxbits[r] : 0ull;
  if (mb != 0 && mb < kInfBitsCrt) {
    const int e = frexp_exp(mb);
    unsigned long long S = 0;
    for (int64_t c = lane; c < nchunks; c += 32) {
      const unsigned long long sc = chunk_s[r * nchunks + c];
      if (sc == 0) continue;
      const int sh = 2 * (e - chunk_e[r * nchunks + c]);
      S += sh >= 64 ? 1ull : ((sc - 1) >> sh) + 1;  // ceil(sc / 2^sh), sc >= 1
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) S += __shfl_xor_sync(0xffffffffu, S, o);  // exact: integer sum
    if (S != 0) {
      const int L = S > 1 ? 64 - __clzll(static_cast<long long>(S - 1)) : 0;
      m = b - (e - 16 + (L + 1) / 2);
    }
  }
  if (lane == 0) mu[r] = m;
}

// Per-modulus constants: p, floor((2^32 - 1) / p) for mod_small, 2^21, 2^42, 2^63 and 2^32
// mod p, and RN(1/p).
struct CrtModConst {
  uint32_t p, magic, c21, c42, c63, c32;
  double inv_p;
};
__host__ __device__ constexpr uint32_t pow2_mod_const(int s, uint32_t p) {
  uint32_t v = 1u % p;
  for (int i = 0; i < s; ++i) v = (2u * v) % p;
  return v;
}
__host__ __device__ constexpr CrtModConst crt_mod_const(int l) {
  return CrtModConst{uint32_t(crt_modulus(l)),
                     0xFFFFFFFFu / uint32_t(crt_modulus(l)),
                     pow2_mod_const(21, uint32_t(crt_modulus(l))),
                     pow2_mod_const(42, uint32_t(crt_modulus(l))),
                     pow2_mod_const(63, uint32_t(crt_modulus(l))),
                     pow2_mod_const(32, uint32_t(crt_modulus(l))),
                     1.0 / double(crt_modulus(l))};
}
static_assert(kCrtMaxModuli == 20, "constant table below");
__constant__ CrtModConst kModConst[kCrtMaxModuli] = {
    crt_mod_const(0),  crt_mod_const(1),  crt_mod_const(2),  crt_mod_const(3),  crt_mod_const(4),
    crt_mod_const(5),  crt_mod_const(6),  crt_mod_const(7),  crt_mod_const(8),  crt_mod_const(9),
    crt_mod_const(10), crt_mod_const(11), crt_mod_const(12), crt_mod_const(13), crt_mod_const(14),
    crt_mod_const(15), crt_mod_const(16), crt_mod_const(17), crt_mod_const(18), crt_mod_const(19)};

// |t| < 2^84 (integer-valued) as four 21-bit chunks, |t| = a3 2^63 + a2 2^42 + a1 2^21 + a0;
// every step is exact in FP64 (power-of-two scalings, floors, and differences that are
// multiples of the ulp of |t| below the removed power).
struct Chunks21 {
  uint32_t a0, a1, a2, a3;
};
__device__ __forceinline__ Chunks21 chunks21(double at) {
  const double h3 = floor(at * 0x1p-63);
  double r = fma(-h3, 0x1p63, at);
  const double h2 = floor(r * 0x1p-42);
  r = fma(-h2, 0x1p42, r);
  const double h1 = floor(r * 0x1p-21);
  const double h0 = fma(-h1, 0x1p21, r);
  return Chunks21{__double2uint_rz(h0), __double2uint_rz(h1), __double2uint_rz(h2), __double2uint_rz(h3)};
}

// |t| mod p: the chunk sum a0 + a1 c21 + a2 c42 + a3 c63 < 2^21 (1 + 3 * 255) < 2^31
__device__ __forceinline__ uint32_t residue_of(const Chunks21& c, const CrtModConst& k) {
  return mod_small(c.a0 + c.a1 * k.c21 + c.a2 * k.c42 + c.a3 * k.c63, k.p, k.magic);
}

constexpr int kSplitRowsCrt = 32;
constexpr int kSplitColsCrt = 128;

// a warp per row (4 entries per lane), 8 rows per pass; three blocks per SM (80 registers)
// measured faster than two blocks of 512 threads (64 registers, spilled) or one (124 registers)
constexpr int kSplitThreadsCrt = 256;
constexpr int kSplitEntries = 4;      // entries (consecutive columns) per thread and row

// The 4 symmetric residues of one thread's entries for one modulus, from 21-bit chunks of
// |t| < 2^84 (more than 16 moduli), packed into 4 bytes.
__device__ __forceinline__ void store_residues_wide(const CrtModConst& k, const Chunks21 (&ch)[kSplitEntries],
                                                    uint32_t neg, int8_t* dst) {
  const int hi = int(k.p >> 1) - ((k.p & 1u) ? 0 : 1);  // largest representative kept as is
  uint32_t w = 0u;
#pragma unroll
  for (int j = 0; j < kSplitEntries; ++j) {
    const int res = int(residue_of(ch[j], k));
    int sres = res > hi ? res - int(k.p) : res;  // symmetric residue of |t|: [-(p/2), (p-1)/2]
    // of -|t|: its negation (for p = 256, 128 packs to the same byte as -128)
    if ((neg >> j) & 1u) sres = -sres;
    w |= (uint32_t(sres) & 0xFFu) << (8 * j);
  }
  *reinterpret_cast<uint32_t*>(dst) = w;
}

// An entry t = trunc(2^mu x) with |t| <= 2^62 (at most 16 moduli) as hi 2^32 + lo (hi signed,
// lo unsigned) and as the exact doubles of hi and lo.
struct SplitEntry {
  int32_t hi;
  uint32_t lo;
  double dh, dl;
};
__device__ __forceinline__ SplitEntry split_entry(long long t) {
  SplitEntry e;
  e.hi = int32_t(t >> 32);
  e.lo = uint32_t(t);
  e.dh = __int2double_rn(e.hi);  // 32-bit integers convert exactly
  e.dl = __uint2double_rn(e.lo);
  return e;
}

// The symmetric residue of t for an odd modulus p, in [-(p-1)/2, (p-1)/2], as a 32-bit two's
// complement.  s = hi c32 + lo (c32 = 2^32 mod p) is congruent to t, and |s| < 2^38 + 2^32 is
// exact in FP64.  One FMA with 1.5 2^52 rounds s/p to the nearest integer q, left in the low
// word of its result: RN(1/p) moves s/p by less than 2^-21, and for odd p the distance of s/p
// from a half-integer is at least 1/(2p), so q is the exact rounding.  s - q p, a small
// integer, is then computed modulo 2^32 from the integer parts.  The division work runs on
// the FP64 pipe and leaves two integer multiply-adds, where a 32-bit Barrett reduction of
// chunk sums takes four multiplies and a centring step.
__device__ __forceinline__ uint32_t symmetric_residue(const SplitEntry& e, const CrtModConst& k, double c32d) {
  const double s = fma(e.dh, c32d, e.dl);
  const uint32_t q = uint32_t(__double2loint(fma(s, k.inv_p, 0x1.8p52)));
  return e.lo + uint32_t(e.hi) * k.c32 - q * k.p;
}

__device__ __forceinline__ uint32_t pack_low_bytes(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// The 4 symmetric residues of one thread's entries for one modulus, packed into 4 bytes.  For
// p = 256 the residue of t is its low byte read as int8 (the representative in [-128, 127]).
__device__ __forceinline__ void store_residues(const CrtModConst& k, const SplitEntry (&e)[kSplitEntries],
                                               int8_t* dst) {
  uint32_t r[kSplitEntries];
  if ((k.p & (k.p - 1u)) == 0u) {
#pragma unroll
    for (int j = 0; j < kSplitEntries; ++j) r[j] = e[j].lo;
  } else {
    const double c32d = double(k.c32);
#pragma unroll
    for (int j = 0; j < kSplitEntries; ++j) r[j] = symmetric_residue(e[j], k, c32d);
  }
  *reinterpret_cast<uint32_t*>(dst) = pack_low_bytes(r[0], r[1], r[2], r[3]);
}

// The residues of two odd moduli pa, pb from one s = hi c + lo, c = 2^32 mod pa pb (< 2^16):
// |s| < 2^47 is exact and congruent to t modulo both, and |s / p| < 2^40 keeps RN(1/p)'s
// error below 2^-13, under the 1/(2p) distance of s/p from a half-integer, so each q is
// again the exact rounding.  Per modulus 1.5 FMAs and 1.5 multiply-adds instead of 2 and 2.
template <int LA>
__device__ __forceinline__ void store_residue_pair(const SplitEntry (&e)[kSplitEntries], int8_t* dst_a,
                                                   int8_t* dst_b) {
  constexpr CrtModConst ka = crt_mod_const(LA), kb = crt_mod_const(LA + 1);
  static_assert((ka.p & 1u) && (kb.p & 1u) && ka.p * kb.p < 65536u, "two odd moduli, product below 2^16");
  constexpr uint32_t c = pow2_mod_const(32, ka.p * kb.p);
  uint32_t ra[kSplitEntries], rb[kSplitEntries];
#pragma unroll
  for (int j = 0; j < kSplitEntries; ++j) {
    const double s = fma(e[j].dh, double(c), e[j].dl);
    const uint32_t u = e[j].lo + uint32_t(e[j].hi) * c;
    ra[j] = u - uint32_t(__double2loint(fma(s, ka.inv_p, 0x1.8p52))) * ka.p;
    rb[j] = u - uint32_t(__double2loint(fma(s, kb.inv_p, 0x1.8p52))) * kb.p;
  }
  *reinterpret_cast<uint32_t*>(dst_a) = pack_low_bytes(ra[0], ra[1], ra[2], ra[3]);
  *reinterpret_cast<uint32_t*>(dst_b) = pack_low_bytes(rb[0], rb[1], rb[2], rb[3]);
}

// Moduli L .. NT-1 with their constants as compile-time immediates; consecutive odd moduli
// in pairs.
template <int L, int NT>
__device__ __forceinline__ void store_residues_static(const SplitEntry (&e)[kSplitEntries], int8_t* dst,
                                                      size_t plane) {
  if constexpr (L < NT) {
    constexpr CrtModConst k = crt_mod_const(L);
    if constexpr ((k.p & 1u) != 0u && L + 1 < NT) {
      store_residue_pair<L>(e, dst + size_t(L) * plane, dst + size_t(L + 1) * plane);
      store_residues_static<L + 2, NT>(e, dst, plane);
    } else {
      store_residues(k, e, dst + size_t(L) * plane);
      store_residues_static<L + 1, NT>(e, dst, plane);
    }
  }
}

// Residues of A' = trunc(2^mu_r x) for moduli [0, n): plane l at residues + l*rows_pad*k_pad,
// row r contiguous along k; symmetric int8 representatives (mu from crt_mu_kernel).
// NT > 0: the modulus count is NT (constants as immediates); NT = 0: n, read at run time.
// A 32 x 128 tile per block: each warp takes a row at a time, four consecutive entries per
// lane, so that every modulus plane receives 128 contiguous bytes per warp store.
template <bool kWide, int NT>  // kWide: |t| may reach 2^63 (more than 16 moduli)
__global__ void __launch_bounds__(kSplitThreadsCrt, 3) crt_split_kernel(
    const double* __restrict__ X, int64_t rows, int64_t cols, int64_t sr, int64_t sl,
    const int32_t* __restrict__ mu, int n, int8_t* __restrict__ residues, int64_t rows_pad, int64_t k_pad) {
  static_assert(kSplitColsCrt == 32 * kSplitEntries, "a warp per tile row");
  __shared__ double tile[kSplitRowsCrt][kSplitColsCrt + 1];
  __shared__ int row_mu_s[kSplitRowsCrt];
  const int64_t r0 = int64_t(blockIdx.y) * kSplitRowsCrt;
  const int64_t l0 = int64_t(blockIdx.x) * kSplitColsCrt;
  if (threadIdx.x < kSplitRowsCrt) {
    const int64_t r = r0 + threadIdx.x;
    row_mu_s[threadIdx.x] = mu[r];
  }
  load_tile<kSplitRowsCrt, kSplitColsCrt, kSplitThreadsCrt>(tile, X, r0, l0, rows, cols, sr, sl);
  __syncthreads();
  const int cb = int(threadIdx.x & 31) * kSplitEntries;
  const size_t plane = size_t(rows_pad) * size_t(k_pad);
  constexpr int kRowsPerPass = kSplitThreadsCrt / 32;
#pragma unroll 1
  for (int rr = int(threadIdx.x >> 5); rr < kSplitRowsCrt; rr += kRowsPerPass) {
    const int m = row_mu_s[rr];
    int8_t* dst = residues + (size_t(r0 + rr)) * size_t(k_pad) + size_t(l0 + cb);
    if constexpr (kWide) {
      Chunks21 ch[kSplitEntries];
      uint32_t neg = 0;
#pragma unroll
      for (int j = 0; j < kSplitEntries; ++j) {
        // |v| <= 2^b, an exact integer (0 in zero rows: 2^kCrtZeroRow underflows to 0)
        const double v = trunc(scale2(tile[rr][cb + j], m));
        ch[j] = chunks21(fabs(v));
        neg |= (v < 0.0 ? 1u : 0u) << j;
      }
      for (int l = 0; l < n; ++l) store_residues_wide(kModConst[l], ch, neg, dst + size_t(l) * plane);
    } else {
      SplitEntry e[kSplitEntries];
      if (m >= -1022 && m <= 1023) {
        // 2^m is a normal double: one product.  It is exact where the two-step scale2 is exact,
        // and where a tiny x makes scale2's first product round, |2^m x| < 1 and the
        // truncation is 0 either way
        const double f = __hiloint2double((m + 1023) << 20, 0);
#pragma unroll
        for (int j = 0; j < kSplitEntries; ++j)
          e[j] = split_entry(__double2ll_rz(__dmul_rn(tile[rr][cb + j], f)));  // trunc
      } else {
        const double f1 = exp2_int(m / 2), f2 = exp2_int(m - m / 2);  // scale2(., m) factors
#pragma unroll
        for (int j = 0; j < kSplitEntries; ++j)
          e[j] = split_entry(__double2ll_rz(__dmul_rn(__dmul_rn(tile[rr][cb + j], f1), f2)));  // trunc
      }
      if constexpr (NT > 0) {
        store_residues_static<0, NT>(e, dst, plane);
      } else {
        for (int l = 0; l < n; ++l) store_residues(kModConst[l], e, dst + size_t(l) * plane);
      }
    }
  }
}

// CRT constants for every modulus count, computed at compile time (192-bit arithmetic in
// 32-bit limbs) and placed in constant memory: the reconstruction reads W_l, P and P/2 as
// immediate constant-bank operands, with no per-device set-up.
struct CrtTable {
  uint32_t W[kCrtMaxModuli + 1][kCrtMaxModuli][kCrtLimbs];
  uint32_t P[kCrtMaxModuli + 1][kCrtLimbs];
  uint32_t half[kCrtMaxModuli + 1][kCrtLimbs];
};

__host__ __device__ constexpr void ct_mul_small(uint32_t (&a)[kCrtLimbs], uint32_t s) {
  uint64_t carry = 0;
  for (int i = 0; i < kCrtLimbs; ++i) {
    const uint64_t v = uint64_t(a[i]) * s + carry;
    a[i] = uint32_t(v);
    carry = v >> 32;
  }
}
__host__ __device__ constexpr uint32_t ct_div_small(uint32_t (&a)[kCrtLimbs], uint32_t s) {
  uint64_t rem = 0;
  for (int i = kCrtLimbs - 1; i >= 0; --i) {
    const uint64_t cur = (rem << 32) | a[i];
    a[i] = uint32_t(cur / s);
    rem = cur % s;
  }
  return uint32_t(rem);
}
__host__ __device__ constexpr uint32_t ct_inverse_mod(uint32_t a, uint32_t p) {
  int64_t t = 0, nt = 1, r = p, nr = a % p;
  while (nr) {
    const int64_t q = r / nr;
    const int64_t t2 = t - q * nt;
    t = nt;
    nt = t2;
    const int64_t r2 = r - q * nr;
    r = nr;
    nr = r2;
  }
  return uint32_t(t < 0 ? t + p : t);
}
__host__ __device__ constexpr CrtTable make_crt_table() {
  CrtTable t{};
  for (int n = 1; n <= kCrtMaxModuli; ++n) {
    uint32_t P[kCrtLimbs] = {1, 0, 0, 0, 0, 0};
    for (int l = 0; l < n; ++l) ct_mul_small(P, uint32_t(crt_modulus(l)));
    for (int l = 0; l < n; ++l) {
      const uint32_t p = uint32_t(crt_modulus(l));
      uint32_t M[kCrtLimbs] = {P[0], P[1], P[2], P[3], P[4], P[5]};
      (void)ct_div_small(M, p);
      uint32_t Mm[kCrtLimbs] = {M[0], M[1], M[2], M[3], M[4], M[5]};
      const uint32_t m_mod = ct_div_small(Mm, p);
      ct_mul_small(M, ct_inverse_mod(m_mod, p));
      for (int i = 0; i < kCrtLimbs; ++i) t.W[n][l][i] = M[i];
    }
    uint32_t H[kCrtLimbs] = {P[0], P[1], P[2], P[3], P[4], P[5]};
    (void)ct_div_small(H, 2);
    for (int i = 0; i < kCrtLimbs; ++i) {
      t.P[n][i] = P[i];
      t.half[n][i] = H[i];
    }
  }
  return t;
}
__constant__ CrtTable kCrtTable = make_crt_table();
// the same table as a compile-time value, for constants folded into instructions
constexpr CrtTable kCrtTableC = make_crt_table();

// Moduli 2g and 2g+1 share the factor Q_g = P / (p_2g p_2g+1) of their weights:
// W_2g = Q_g X_2g and W_2g+1 = Q_g X_2g+1 with X_2g = p_2g+1 ((P/p_2g)^-1 mod p_2g) and
// X_2g+1 = p_2g ((P/p_2g+1)^-1 mod p_2g+1), both below p_2g p_2g+1 < 2^16.  A last unpaired
// modulus has Q = P/p and X = (P/p)^-1 mod p.  Then S = sum_l r_l W_l = sum_g Q_g R_g with
// R_g = r_2g X_2g + r_2g+1 X_2g+1 < 2^25: the same S, with 32-bit multiply-adds for R_g and
// half as many 64-bit ones for the 128-bit part.  Up to 16 moduli (P < 2^128).
struct CrtPairTable {
  uint32_t X[kCrtMaxModuli + 1][kCrtMaxModuli];
  uint32_t Q[kCrtMaxModuli + 1][kCrtMaxModuli / 2][4];
};
__host__ __device__ constexpr CrtPairTable make_crt_pair_table() {
  CrtPairTable t{};
  for (int n = 1; n <= 16; ++n) {
    uint32_t P[kCrtLimbs] = {1, 0, 0, 0, 0, 0};
    for (int l = 0; l < n; ++l) ct_mul_small(P, uint32_t(crt_modulus(l)));
    for (int g = 0; 2 * g < n; ++g) {
      const bool pair = 2 * g + 1 < n;
      const uint32_t pa = uint32_t(crt_modulus(2 * g)), pb = pair ? uint32_t(crt_modulus(2 * g + 1)) : 1u;
      uint32_t Q[kCrtLimbs] = {P[0], P[1], P[2], P[3], P[4], P[5]};
      (void)ct_div_small(Q, pa);
      uint32_t Ma[kCrtLimbs] = {Q[0], Q[1], Q[2], Q[3], Q[4], Q[5]};  // P / p_a
      const uint32_t ma = ct_div_small(Ma, pa);                        // (P / p_a) mod p_a
      t.X[n][2 * g] = pb * ct_inverse_mod(ma, pa);
      if (pair) {
        uint32_t Mb[kCrtLimbs] = {P[0], P[1], P[2], P[3], P[4], P[5]};
        (void)ct_div_small(Mb, pb);
        const uint32_t mb = ct_div_small(Mb, pb);  // (P / p_b) mod p_b
        t.X[n][2 * g + 1] = pa * ct_inverse_mod(mb, pb);
        (void)ct_div_small(Q, pb);
      }
      for (int q = 0; q < 4; ++q) t.Q[n][g][q] = Q[q];
    }
  }
  return t;
}
__constant__ CrtPairTable kCrtPairs = make_crt_pair_table();

struct CrtRecParams {
  uint32_t W[kCrtMaxModuli][kCrtLimbs];
  uint32_t P[kCrtLimbs];
  uint32_t half[kCrtLimbs];
  double P_inv;
  int n, b;
  int64_t m, ncols;
  double alpha, beta;
  double* C;
  int64_t ldc;
  const uint8_t* res;
  int64_t ld_res, plane;
  const int32_t* mu_a;
  const int32_t* mu_b;
  double* err_sq;  // [0] += estimated squared error, [1] += squared alpha*A*B entries
  const int* skip_if_flag;
  int write_c;
  double* save;
  int64_t ld_save;
  int cols_per_block;  // columns one block handles per pass (fewer when the grid would be small)
  int uplo;            // 0: all of C; 1: i <= j only; 2: i >= j only
};

// The columns [jb, je) of row i within [j0, j1) that the triangle `uplo` keeps.
__device__ __forceinline__ void triangle_cols(int uplo, int64_t i, int64_t j0, int64_t j1, int64_t& jb, int64_t& je) {
  jb = (uplo == 1 && j0 < i) ? i : j0;
  je = (uplo == 2 && j1 > i + 1) ? i + 1 : j1;
}

// RN(|R|) of a 192-bit magnitude as d * 2^shift, d an integer-valued double < 2^64:
// the top 64 bits below the leading one, with a sticky bit for everything under them.
__device__ __forceinline__ double limbs_to_double(const uint32_t* s, int& shift) {
  int h = kCrtLimbs - 1;
  while (h > 0 && s[h] == 0) --h;
  shift = 0;
  if (h <= 1) return __ull2double_rn((static_cast<unsigned long long>(h == 1 ? s[1] : 0u) << 32) | s[0]);
  const int lz = __clz(static_cast<int>(s[h]));
  unsigned long long u = (static_cast<unsigned long long>(s[h]) << 32) | s[h - 1];
  uint32_t sticky;
  if (lz) {
    u = (u << lz) | (s[h - 2] >> (32 - lz));
    sticky = s[h - 2] << lz;
  } else {
    sticky = s[h - 2];
  }
  for (int i = 0; i < h - 2; ++i) sticky |= s[i];
  shift = 32 * (h - 1) - lz;
  return __ull2double_rn(u | (sticky ? 1ull : 0ull));
}

// RN(d 2^e) for an integer-valued d in [1, 2^64): two exact steps, one rounding at most
__device__ __forceinline__ double scale_exp(double d, int e) {
  if (e < -1200) return d * 0.0;  // |d 2^e| < 2^-1136
  if (e > 1100) e = 1100;         // overflows to infinity either way
  return scale2(d, e);
}

// The fields the per-entry store needs, copied into registers at kernel entry: reading them
// through a reference to the __grid_constant__ parameter block would cost a load from
// parameter space per entry.
struct CrtStoreCtx {
  double alpha, beta;
  double* C;
  int64_t ldc;
  double* save;
  int64_t ld_save;
  const int32_t* mu_a;
  const int32_t* mu_b;
  int b;
  bool write_c, estimate;
};

__device__ __forceinline__ CrtStoreCtx store_ctx(const CrtRecParams& R) {
  return CrtStoreCtx{R.alpha, R.beta, R.C,       R.ldc,          R.save,
                     R.ld_save, R.mu_a, R.mu_b, R.b, R.write_c != 0, R.err_sq != nullptr};
}

// alpha C_ij from RN(C'_ij) = d 2^shift (signed d): scaled by 2^-(mu_i + nu_j); with the
// estimate, e += 2^(2(b - mu_i - nu_j)) (the squared truncation error bound, up to the factor
// 2/3 alpha^2 applied per block) and v += (alpha C')^2.
__device__ __forceinline__ double crt_value(const CrtStoreCtx& S, int mu_i, int nu_j, double d, int shift,
                                            double& e_acc, double& v_acc) {
  const double val = d != 0.0 ? scale_exp(d, shift - mu_i - nu_j) : 0.0;  // d = 0 in zero rows
  const double v = __dmul_rn(S.alpha, val);
  if (S.estimate) {
    // truncation errors need a nonzero row on both sides
    if (mu_i != kCrtZeroRow && nu_j != kCrtZeroRow) e_acc += exp2_int(2 * (S.b - mu_i - nu_j));
    v_acc += v * v;
  }
  return v;
}

// C_ij = alpha C_ij' (+ beta C_ij, the old value kept in `save` when there is one)
__device__ __forceinline__ void crt_store(const CrtStoreCtx& S, int64_t i, int64_t j, double d, int shift,
                                          double& e_acc, double& v_acc) {
  const double v = crt_value(S, S.mu_a[i], S.mu_b[j], d, shift, e_acc, v_acc);
  if (S.write_c) {
    double* c = S.C + j * S.ldc + i;
    if (S.beta == 0.0) {
      *c = v;
    } else {
      const double old = *c;
      if (S.save) S.save[j * S.ld_save + i] = old;
      *c = __fma_rn(S.beta, old, v);
    }
  }
}

// One pair of atomics per block (same-address atomics serialise in L2).
__device__ __forceinline__ void crt_reduce_energies(const CrtRecParams& R, double e_acc, double v_acc) {
  __shared__ double red[2][8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e_acc += __shfl_xor_sync(0xffffffffu, e_acc, o);
    v_acc += __shfl_xor_sync(0xffffffffu, v_acc, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = e_acc;
    red[1][w] = v_acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0, v = 0.0;
    for (int q = 0; q < 8; ++q) {
      e += red[0][q];
      v += red[1][q];
    }
    e *= (2.0 / 3.0) * R.alpha * R.alpha;  // rms of a truncation error in (-1, 1): 1/sqrt(3)
    if (e != 0.0) atomicAdd(&R.err_sq[0], e);
    if (v != 0.0) atomicAdd(&R.err_sq[1], v);
  }
}

constexpr int kRecCols = 8;  // most columns per block and pass
static_assert(kRecCols <= 32, "the estimate's column sum takes a lane per column");

// One thread per row i, cols_per_block columns per pass: C'_ij from its residues, then C_ij.
__global__ void __launch_bounds__(256) crt_reconstruct_kernel(const __grid_constant__ CrtRecParams R) {
  if (R.skip_if_flag && *R.skip_if_flag) return;
  const CrtStoreCtx sc = store_ctx(R);
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double e_acc = 0.0, v_acc = 0.0;
  // blockIdx.y walks groups of cols_per_block columns
  const int cpb = R.cols_per_block;
  const int64_t jstep = int64_t(gridDim.y) * cpb;
  for (int64_t j0 = int64_t(blockIdx.y) * cpb; i < R.m && j0 < R.ncols; j0 += jstep) {
    int64_t jb, je;
    triangle_cols(R.uplo, i, j0, j0 + cpb < R.ncols ? j0 + cpb : R.ncols, jb, je);
    for (int64_t j = jb; j < je; ++j) {
      const uint8_t* rp = R.res + j * R.ld_res + i;
      unsigned long long acc[kCrtLimbs] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
      // unrolled over the largest modulus count: the weights are immediate constant-bank operands
#pragma unroll
      for (int l = 0; l < kCrtMaxModuli; ++l) {
        if (l < R.n) {
          const uint32_t r = rp[int64_t(l) * R.plane];
#pragma unroll
          for (int q = 0; q < kCrtLimbs; ++q) acc[q] += static_cast<unsigned long long>(r) * R.W[l][q];
        }
      }
      // S = sum r_l W_l < n * 256 * P < 2^192 as six 32-bit limbs
      uint32_t s[kCrtLimbs];
      unsigned long long carry = 0;
#pragma unroll
      for (int q = 0; q < kCrtLimbs; ++q) {
        const unsigned long long v = acc[q] + carry;
        s[q] = uint32_t(v);
        carry = v >> 32;
      }
      // R = S - q P with q = rint(S / P); then R is C' or C' +- P
      double sd = 0.0;
#pragma unroll
      for (int q = kCrtLimbs - 1; q >= 0; --q) sd = fma(sd, 4294967296.0, double(s[q]));
      const uint32_t qq = uint32_t(rint(sd * R.P_inv));
      long long borrow = 0;
      unsigned long long mcarry = 0;
#pragma unroll
      for (int q = 0; q < kCrtLimbs; ++q) {
        const unsigned long long qp = static_cast<unsigned long long>(qq) * R.P[q] + mcarry;
        mcarry = qp >> 32;
        const long long d = static_cast<long long>(s[q]) - static_cast<long long>(uint32_t(qp)) + borrow;
        s[q] = uint32_t(d);
        borrow = d >> 32;  // 0 or -1
      }
      bool negative = (s[kCrtLimbs - 1] >> 31) != 0;
      if (negative) {  // two's complement negate
        unsigned long long c = 1;
#pragma unroll
        for (int q = 0; q < kCrtLimbs; ++q) {
          const unsigned long long v = static_cast<unsigned long long>(~s[q]) + c;
          s[q] = uint32_t(v);
          c = v >> 32;
        }
      }
      // |R| > P/2: the representative is P - |R| with the opposite sign
      bool above = false;
#pragma unroll
      for (int q = kCrtLimbs - 1; q >= 0; --q) {
        if (s[q] != R.half[q]) {
          above = s[q] > R.half[q];
          break;
        }
      }
      if (above) {
        long long bw = 0;
#pragma unroll
        for (int q = 0; q < kCrtLimbs; ++q) {
          const long long d = static_cast<long long>(R.P[q]) - static_cast<long long>(s[q]) + bw;
          s[q] = uint32_t(d);
          bw = d >> 32;
        }
        negative = !negative;
      }
      int shift;
      double d = limbs_to_double(s, shift);
      crt_store(sc, i, j, negative ? -d : d, shift, e_acc, v_acc);
    }
  }
  if (R.err_sq) crt_reduce_energies(R, e_acc, v_acc);
}

// C' from the residues rc[0..N) of one entry (N <= 16): RN(|C'|) = d 2^shift, returns the
// sign.  S = sum_g Q_g R_g, then R = S - q P with q = rint(S / P) and a range fix, exact in
// 128-bit two's complement.
template <int N>
__device__ __forceinline__ bool crt_combine128(const uint32_t (&rc)[N], double P_inv, double& d, int& shift) {
  using u128 = unsigned __int128;
  using s128 = __int128;
  const u128 P = (u128(kCrtTable.P[N][3]) << 96) | (u128(kCrtTable.P[N][2]) << 64) | (u128(kCrtTable.P[N][1]) << 32) |
                 u128(kCrtTable.P[N][0]);
  const s128 half = s128(P >> 1);
  // S = sum_g Q_g R_g in four 32-bit limb columns (each < 8 * 2^25 * 2^32 = 2^60); S itself
  // (< 2^28 P) may pass 2^128, and the 128-bit arithmetic below works modulo 2^128, which
  // leaves the small remainder S - q P exact
  unsigned long long acc[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll
  for (int g = 0; 2 * g < N; ++g) {
    uint32_t Rg = rc[2 * g] * kCrtPairs.X[N][2 * g];
    if (2 * g + 1 < N) Rg += rc[2 * g + 1] * kCrtPairs.X[N][2 * g + 1];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] += static_cast<unsigned long long>(Rg) * kCrtPairs.Q[N][g][q];
  }
  // q = rint(S / P) from the partial sums in FP64; it may be off by one near a
  // half-integer, which the range fix below absorbs
  const double sd =
      fma(double(acc[3]), 0x1p96, fma(double(acc[2]), 0x1p64, fma(double(acc[1]), 0x1p32, double(acc[0]))));
  const u128 q = u128(static_cast<unsigned long long>(rint(sd * P_inv)));
  const u128 S = u128(acc[0]) + (u128(acc[1]) << 32) + (u128(acc[2]) << 64) + (u128(acc[3]) << 96);
  s128 r = s128(S - q * P);
  if (r > half)
    r -= s128(P);
  else if (r < -half)
    r += s128(P);
  const bool negative = r < 0;
  const u128 mag = negative ? u128(-r) : u128(r);
  const unsigned long long hi = static_cast<unsigned long long>(mag >> 64);
  const unsigned long long lo = static_cast<unsigned long long>(mag);
  shift = 0;
  if (hi == 0) {
    d = __ull2double_rn(lo);
  } else {  // top 64 bits and a sticky bit: one correct rounding
    const int lz = __clzll(static_cast<long long>(hi));
    const unsigned long long u = lz ? (hi << lz) | (lo >> (64 - lz)) : hi;
    const unsigned long long sticky = (lo << lz) != 0ull ? 1ull : 0ull;
    d = __ull2double_rn(u | sticky);
    shift = 64 - lz;
  }
  return negative;
}

// The same for N <= 16 moduli, N a template parameter: P < 2^126, so W_l fits four limbs,
// S = sum r_l W_l is known modulo 2^128, and R = S - q P (|R| < 1.5 P < 2^127) is exact in
// 128-bit two's complement.  W_l, P and P/2 come from the compile-time table.  Bit for bit
// the result of the kernel above (both round C' once).
// Four blocks per SM (at most 64 registers): at 66 registers only three fit, 11% slower.
template <int N, bool EST>
__global__ void __launch_bounds__(256, 4) crt_reconstruct128_kernel(const __grid_constant__ CrtRecParams R) {
  static_assert(N >= 1 && N <= 16, "128-bit path");
  if (R.skip_if_flag && *R.skip_if_flag) return;
  CrtStoreCtx sc = store_ctx(R);
  sc.estimate = EST;  // compiled separately with and without the estimate
  const uint8_t* const res = R.res;
  const int64_t ld_res = R.ld_res, plane = R.plane, m = R.m, ncols = R.ncols;
  const double P_inv = R.P_inv;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double e_acc = 0.0, v_acc = 0.0;
  const int cpb = R.cols_per_block;
  const int64_t jstep = int64_t(gridDim.y) * cpb;
  for (int64_t j0 = int64_t(blockIdx.y) * cpb; i < m && j0 < ncols; j0 += jstep) {
    int64_t jb, j1;
    triangle_cols(R.uplo, i, j0, j0 + cpb < ncols ? j0 + cpb : ncols, jb, j1);
    if (jb >= j1) continue;
    // software pipeline: the residues of column j+1 are loaded while column j is reduced
    uint32_t rn[N];
#pragma unroll
    for (int l = 0; l < N; ++l) rn[l] = res[jb * ld_res + i + l * plane];
    for (int64_t j = jb; j < j1; ++j) {
      uint32_t rc[N];
#pragma unroll
      for (int l = 0; l < N; ++l) rc[l] = rn[l];
      if (j + 1 < j1) {
#pragma unroll
        for (int l = 0; l < N; ++l) rn[l] = res[(j + 1) * ld_res + i + l * plane];
      }
      double d;
      int shift;
      const bool negative = crt_combine128<N>(rc, P_inv, d, shift);
      crt_store(sc, i, j, negative ? -d : d, shift, e_acc, v_acc);
    }
  }
  if (EST) crt_reduce_energies(R, e_acc, v_acc);
}

// RN(|R| 2^escale) with its sign, for R = (r3 r2 r1 r0) in [-P/2, P/2) (128-bit two's
// complement): the magnitude's top 64 bits and a sticky bit, rounded to nearest even and
// written straight into the bits of the scaled double when that is a normal number (scaling
// by 2^escale is then exact).  Subnormal and overflowing results take the per-row kernel's
// steps (RN of the top 64 bits, then scale_exp), so every result is bit for bit that kernel's.
__device__ __forceinline__ double crt_round_magnitude(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3, int escale) {
  const bool negative = int(r3) < 0;
  // |R| = (hi64, lo64)
  unsigned long long lo64 = (static_cast<unsigned long long>(r1) << 32) | r0;
  unsigned long long hi64 = (static_cast<unsigned long long>(r3) << 32) | r2;
  if (negative) {
    lo64 = ~lo64 + 1ull;
    hi64 = ~hi64 + (lo64 == 0ull ? 1ull : 0ull);
  }
  if ((hi64 | lo64) == 0ull) return 0.0;
  // top 64 bits u (leading one at bit 63), bit length L, sticky for the bits below u
  int L;
  unsigned long long u;
  bool sticky;
  if (hi64 != 0ull) {
    const int lz = __clzll(static_cast<long long>(hi64));
    u = lz ? (hi64 << lz) | (lo64 >> (64 - lz)) : hi64;
    sticky = (lo64 << lz) != 0ull;
    L = 128 - lz;
  } else {
    const int lz = __clzll(static_cast<long long>(lo64));
    u = lo64 << lz;
    sticky = false;
    L = 64 - lz;
  }
  const int E = L - 1 + escale;  // exponent of the scaled magnitude before rounding
  if (E < -1022 || E > 1023) {
    // the per-row kernel's two steps: RN(|R|) = d 2^shift, then scale_exp
    double dd;
    int shift;
    if (hi64 == 0ull) {
      dd = __ull2double_rn(lo64);
      shift = 0;
    } else {
      const int lz = __clzll(static_cast<long long>(hi64));
      const unsigned long long uu = lz ? (hi64 << lz) | (lo64 >> (64 - lz)) : hi64;
      dd = __ull2double_rn(uu | ((lo64 << lz) != 0ull ? 1ull : 0ull));
      shift = 64 - lz;
    }
    const double v = scale_exp(dd, shift + escale);
    return negative ? -v : v;
  }
  // round the 53-bit significand to nearest even; a carry out of it moves into the exponent
  unsigned long long mant = u >> 11;
  const bool round_bit = ((u >> 10) & 1ull) != 0ull;
  const bool rest = (u & 0x3FFull) != 0ull || sticky;
  mant += (round_bit && (rest || (mant & 1ull))) ? 1ull : 0ull;
  const unsigned long long bits =
      (static_cast<unsigned long long>(E + 1022) << 52) + mant + (negative ? 0x8000000000000000ull : 0ull);
  return __longlong_as_double(static_cast<long long>(bits));
}

// RN(R 2^escale) for R = (r3 r2 r1 r0) in 128-bit two's complement, congruent to C' modulo P
// and within one P of [-P/2, P/2).  The range fix runs only when R's top 64-bit window does
// not already place it in [-P/2, P/2).  Then, with hi = the signed 64-bit window of R at limbs
// kW, kW+1 (|R| < 2^(63 + 32 kW)) and lo the limbs below it, R = hi 2^(32 kW) + lo, and two
// one-rounding forms cover all but tiny |R|:
//   * |hi| >= 2^54: RN(hi | [lo != 0]) 2^(32 kW).  The sticky bit sits below the guard bit
//     (hi has at least 55 significant bits), and hi and hi | 1 lie strictly between the same
//     two even integers, so both round like R;
//   * 8 <= |hi| < 2^54: R = h 2^(32 kW + 1) + X with h = hi >> 1 (|h| < 2^53, exact in a
//     double) and X = (hi & 1) 2^(32 kW) + lo.  For kW = 1, X < 2^33 is exact and
//     RN(R) = fma(h, 2^33, X).  For kW = 2, X >> 12 with a sticky bit in its lowest place is
//     below 2^53 and exact, and R, at least 2^67 in magnitude, has its guard bit at 2^13 or
//     above, so RN(R) = fma(h, 2^53, (X >> 12) | [X mod 2^12 != 0]) 2^12;
//   * kW = 0 (P < 2^64): R = hi exactly.
// The result is scaled by adding to the exponent field when it stays normal.  Everything else
// (|hi| < 8, subnormal or overflowing results) takes crt_round_magnitude, the per-row kernel's
// steps, so every result is bit for bit that kernel's.
template <int N>
__device__ __forceinline__ double crt_round(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3, int escale) {
  constexpr uint32_t P0 = kCrtTableC.P[N][0], P1 = kCrtTableC.P[N][1], P2 = kCrtTableC.P[N][2], P3 = kCrtTableC.P[N][3];
  // R lies in [-half, half) when the 64-bit window of R at half's two top limbs is in
  // [-Hw, Hw) and the limbs above the window extend its sign: nothing to fix then
  constexpr int kW = kCrtTableC.half[N][3] != 0 ? 2 : (kCrtTableC.half[N][2] != 0 ? 1 : 0);
  constexpr long long Hw = static_cast<long long>((static_cast<unsigned long long>(kCrtTableC.half[N][kW + 1]) << 32) |
                                                  kCrtTableC.half[N][kW]);
  const uint32_t rl[4] = {r0, r1, r2, r3};
  const long long win = static_cast<long long>((static_cast<unsigned long long>(rl[kW + 1]) << 32) | rl[kW]);
  const uint32_t ext = win < 0 ? 0xFFFFFFFFu : 0u;
  bool in_range = win >= -Hw && win < Hw;
#pragma unroll
  for (int t = kW + 2; t < 4; ++t) in_range = in_range && rl[t] == ext;
  if (!in_range) {
    using u128 = unsigned __int128;
    using s128 = __int128;
    const u128 P = (u128(P3) << 96) | (u128(P2) << 64) | (u128(P1) << 32) | u128(P0);
    const s128 half = s128(P >> 1);
    s128 r = s128((u128(r3) << 96) | (u128(r2) << 64) | (u128(r1) << 32) | u128(r0));
    if (r > half)
      r -= s128(P);
    else if (r < -half)
      r += s128(P);
    const u128 ur = u128(r);
    r0 = uint32_t(ur);
    r1 = uint32_t(ur >> 32);
    r2 = uint32_t(ur >> 64);
    r3 = uint32_t(ur >> 96);
  }
  const uint32_t rl2[4] = {r0, r1, r2, r3};
  const long long hi = static_cast<long long>((static_cast<unsigned long long>(rl2[kW + 1]) << 32) | rl2[kW]);
  double d;
  int s;
  bool fast;
  if constexpr (kW == 0) {
    d = __ll2double_rn(hi);
    s = 0;
    fast = hi != 0;
  } else if constexpr (kW == 1) {
    if (static_cast<unsigned long long>(hi + (1ll << 54)) >= (1ull << 55)) {
      d = __ll2double_rn(hi | (r0 != 0u ? 1ll : 0ll));
      s = 32;
    } else {
      const long long h = hi >> 1;
      const unsigned long long X = (static_cast<unsigned long long>(hi & 1) << 32) | r0;
      d = fma(__ll2double_rn(h), 0x1p33, __ull2double_rn(X));
      s = 0;
    }
    fast = static_cast<unsigned long long>(hi + 8) >= 16ull;
  } else {
    if (static_cast<unsigned long long>(hi + (1ll << 54)) >= (1ull << 55)) {
      d = __ll2double_rn(hi | ((r0 | r1) != 0u ? 1ll : 0ll));
      s = 64;
    } else {
      const long long h = hi >> 1;
      // x = (X >> 12) | sticky = (hi & 1) 2^52 + X', X' = (lo >> 12) | [lo mod 2^12 != 0] below
      // 2^52: the bits of 2^52 + X' assembled directly, minus 2^52 unless hi is odd (exact)
      const uint32_t xlo = (r1 << 20) | (r0 >> 12) | ((r0 & 0xFFFu) != 0u ? 1u : 0u);
      const double x = __hiloint2double(static_cast<int>(0x43300000u | (r1 >> 12)), static_cast<int>(xlo)) -
                       ((hi & 1) != 0 ? 0.0 : 0x1p52);
      d = fma(__ll2double_rn(h), 0x1p53, x);
      s = 12;
    }
    fast = static_cast<unsigned long long>(hi + 8) >= 16ull;
  }
  const int k = s + escale;
  const int hw = __double2hiint(d);
  const int be = ((hw >> 20) & 0x7FF) + k;  // biased exponent of d 2^k
  if (fast && static_cast<unsigned>(be - 1) < 2046u)
    return __hiloint2double(static_cast<int>(static_cast<unsigned>(hw) + (static_cast<unsigned>(k) << 20)),
                            __double2loint(d));
  return crt_round_magnitude(r0, r1, r2, r3, escale);
}

// RN(C' 2^escale) from S = sum_q acc[q] 2^(32q), limb columns below 2^52 (the tensor-core sum
// gives columns below 2^46): the columns are exact doubles by one integer add and one FP64
// subtraction, q = rint(S / P) comes from acc[1..3] (acc[0] / P < 2^-11 left out), or from
// acc[2..3] for 13 moduli and more (q is off by one at most either way, which the range fix
// absorbs), and R = S - q P takes its borrows column by column without carrying S first.
template <int N>
__device__ __forceinline__ double crt_finish_small(const unsigned long long (&acc)[4], double P_inv32, int escale) {
  static_assert(N >= kCrtMinModuli && N <= 16, "P at least 2^63 and below 2^128");
  auto exact = [](unsigned long long x) {  // x < 2^52
    return __longlong_as_double(static_cast<long long>(x + 0x4330000000000000ull)) - 0x1p52;
  };
  uint32_t q;
  if constexpr (N >= 13) {
    // P >= 2^102: acc[1] 2^32 + acc[0] < 2^79 moves S / P by less than 2^-23, so S / 2^64 is
    // taken from acc[3] and acc[2] alone
    const double sd = fma(exact(acc[3]), 0x1p32, exact(acc[2]));
    q = uint32_t(__double2loint(fma(sd, P_inv32 * 0x1p32, 0x1.8p52)));
  } else {
    const double sd = fma(fma(exact(acc[3]), 0x1p32, exact(acc[2])), 0x1p32, exact(acc[1]));
    q = uint32_t(__double2loint(fma(sd, P_inv32, 0x1.8p52)));
  }
  constexpr uint32_t P0 = kCrtTableC.P[N][0], P1 = kCrtTableC.P[N][1], P2 = kCrtTableC.P[N][2], P3 = kCrtTableC.P[N][3];
  const long long d0 = static_cast<long long>(acc[0]) - static_cast<long long>(static_cast<unsigned long long>(q) * P0);
  const long long d1 = static_cast<long long>(acc[1]) - static_cast<long long>(static_cast<unsigned long long>(q) * P1) +
                       (d0 >> 32);
  const long long d2 = static_cast<long long>(acc[2]) - static_cast<long long>(static_cast<unsigned long long>(q) * P2) +
                       (d1 >> 32);
  const long long d3 = static_cast<long long>(acc[3]) - static_cast<long long>(static_cast<unsigned long long>(q) * P3) +
                       (d2 >> 32);
  return crt_round<N>(uint32_t(d0), uint32_t(d1), uint32_t(d2), uint32_t(d3), escale);
}

// ---- reconstruction with the weighted residue sum on the tensor cores
// S = sum_l r_l W_l = sum_b 2^(8b) T_b with T_b = sum_l r_l w_lb, w_lb byte b of W_l (W_l < P <
// 2^128: 16 bytes) and T_b < 16 * 255 * 255 < 2^20: a [32 entries x 16 moduli] x [16 moduli x 16
// bytes] product of unsigned bytes with exact INT32 sums, four mma.sync m16n8k16 per warp, each
// from a zero accumulator.
__device__ __forceinline__ void mma_u8_16x8x16(int (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
  asm("mma.sync.aligned.m16n8k16.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%7,%7,%7,%7};"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3])
      : "r"(a0), "r"(a1), "r"(b0), "r"(0));
}

// Rows i0 .. i0+31 of one column per warp.  The warp streams the residues of its columns
// through its own ring of kRecStages shared-memory slots (a column's 16 moduli x 32 rows, 512
// bytes), kRecStages - 1 columns ahead, with 16-byte cp.async copies (lane L copies rows
// 16 (L & 1) .. +15 of modulus L / 2), so that no registers hold loads in flight.  Lane
// (g, c) = (lane / 4, lane % 4) reads moduli 4c .. 4c+3 at rows i0 + 4g .. i0 + 4g + 3 (one
// 32-bit word per modulus; the slot's words are swizzled, word w at w ^ ((w >> 2) & 0x18), so
// that these reads hit 32 distinct banks) and transposes the 4 x 4 bytes so that each word
// holds the four moduli of one row (the A fragment rows).  The MMAs leave with lane (g, c) the
// byte sums T_2c, T_2c+1, T_8+2c, T_9+2c of those four rows.  The lane packs them in pairs,
// X_c = T_2c + 2^8 T_2c+1 and Y_c = T_8+2c + 2^8 T_9+2c (each below 2^29), and the warp passes
// the pairs through its own rows of shared memory (two buffers, alternating by column, so that
// writing one never waits for the reads of the other), so that lane L reads the eight of row
// i0 + L and forms S in four 32-bit-aligned columns, X_0 + 2^16 X_1, X_2 + 2^16 X_3,
// Y_0 + 2^16 Y_1, Y_2 + 2^16 Y_3; the tail (crt_finish_small) and the store follow.  Bit for
// bit the per-row kernel: S is the same integer and it is rounded the same way.
constexpr int kRecStageStride = 10;  // words per staged row: X_0 Y_0 .. X_3 Y_3 and 2 of padding
constexpr int kRecStages = 4;        // columns of residues in each warp's ring
__device__ __forceinline__ int rec_swizzle(int w) { return w ^ ((w >> 2) & 0x18); }
template <int N, bool EST>
__global__ void __launch_bounds__(256, 4) crt_reconstruct_mma_kernel(const __grid_constant__ CrtRecParams R) {
  static_assert(N >= kCrtMinModuli && N <= 16, "16 moduli per MMA K step");
  __shared__ __align__(16) uint32_t stage[8][2][32 * kRecStageStride];
  __shared__ __align__(16) uint32_t ring[8][kRecStages][128];
  if (R.skip_if_flag && *R.skip_if_flag) return;
  uint32_t (*const wstage)[32 * kRecStageStride] = stage[threadIdx.x >> 5];
  int sbuf = 0;
  const uint32_t (*const wring)[128] = ring[threadIdx.x >> 5];
  CrtStoreCtx sc = store_ctx(R);
  const uint8_t* const res = R.res;
  const int64_t ld_res = R.ld_res, plane = R.plane, m = R.m, ncols = R.ncols;
  const int uplo = R.uplo;
  const double P_inv32 = R.P_inv * 0x1p32;
  const int lane = int(threadIdx.x & 31);
  const int g = lane >> 2, c = lane & 3;
  const int64_t i0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) - lane;  // the warp's first row
  const int64_t i = i0 + lane;                                                   // this lane's row
  // B fragments: byte (8h + g) of W_4c .. W_4c+3
  uint32_t bfrag[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int byte = 8 * h + g;
    uint32_t w = 0u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int l = 4 * c + k;
      const uint32_t wb = l < N ? (kCrtTable.W[N][l][byte >> 2] >> (8 * (byte & 3))) & 0xFFu : 0u;
      w |= wb << (8 * k);
    }
    bfrag[h] = w;
  }
  const int mu_i = i < m ? sc.mu_a[i] : kCrtZeroRow;
  double e_acc = 0.0, v_acc = 0.0;
  // copies: lane L takes rows 16 (L & 1) .. +15 of modulus L / 2 (16-byte aligned: the planes,
  // the leading dimension and i0 are multiples of 16)
  const bool copier = (lane >> 1) < N;
  const uint8_t* const cbase = res + i0 + 16 * (lane & 1) + int64_t(lane >> 1) * plane;
  const uint32_t cdst = smem_u32(&wring[0][rec_swizzle(8 * (lane >> 1) + 4 * (lane & 1))]);
  int rword[4];  // this lane's four words of a slot
#pragma unroll
  for (int k = 0; k < 4; ++k) rword[k] = rec_swizzle(8 * (4 * c + k) + g);
  const int cpb = R.cols_per_block;
  const int64_t jstep = int64_t(gridDim.y) * cpb;
  for (int64_t j0 = int64_t(blockIdx.y) * cpb; i0 < m && j0 < ncols; j0 += jstep) {
    // the columns that some row of the warp keeps
    int64_t jb = j0, j1 = j0 + cpb < ncols ? j0 + cpb : ncols;
    if (uplo == 1 && jb < i0) jb = i0;            // i <= j
    if (uplo == 2 && j1 > i0 + 32) j1 = i0 + 32;  // i >= j
    if (jb >= j1) continue;
    if (EST && uplo == 0) {
      // sum_j 2^(2(b - mu_i - nu_j)) over the pass's nonzero columns = 2^(2(b - mu_i - nu_min))
      // sum_j 2^(-2(nu_j - nu_min)): the column sum is the same for every row of the warp, so
      // lane t takes column jb + t (at most kRecCols of them) and the warp adds them up
      const int cnt = int(j1 - jb);
      const int nu = lane < cnt ? sc.mu_b[jb + lane] : kCrtZeroRow;
      const bool nz = nu != kCrtZeroRow;
      const int nu_min = __reduce_min_sync(0xffffffffu, nz ? nu : INT_MAX);
      double t = nz ? exp2_int(-2 * (nu - nu_min)) : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (mu_i != kCrtZeroRow && nu_min != INT_MAX) e_acc = fma(exp2_int(2 * (sc.b - mu_i - nu_min)), t, e_acc);
    }
    // one commit group per column (empty past j1), so that waiting for all but the newest
    // kRecStages - 1 groups leaves column j landed; every lane reads a slot before the
    // __syncwarp that precedes any copy into it
    // (32-bit column offsets jj from jb and pointers stepped by their leading dimensions)
    const int cnt = int(j1 - jb);
    const uint8_t* csrc = cbase + jb * ld_res;
#pragma unroll
    for (int t = 0; t < kRecStages - 1; ++t, csrc += ld_res) {
      if (copier && t < cnt) cp_async_16(cdst + t * 512u, csrc);
      cp_async_commit();
    }
    double* cp = sc.C + jb * sc.ldc + i;
    const int32_t* const nup = sc.mu_b + jb;
    int slot = 0;
    for (int jj = 0; jj < cnt; ++jj, csrc += ld_res, cp += sc.ldc) {
      {
        const int sn = slot == 0 ? kRecStages - 1 : slot - 1;  // (slot + kRecStages - 1) % kRecStages
        if (copier && jj + kRecStages - 1 < cnt) cp_async_16(cdst + uint32_t(sn) * 512u, csrc);
        cp_async_commit();
      }
      cp_async_wait<kRecStages - 1>();
      __syncwarp();
      uint32_t w[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) w[k] = 4 * c + k < N ? wring[slot][rword[k]] : 0u;
      slot = slot == kRecStages - 1 ? 0 : slot + 1;
      // 4 x 4 byte transpose: w[k] byte e (modulus 4c+k, row 4g+e) -> v[e] byte k
      const uint32_t t0 = __byte_perm(w[0], w[1], 0x5140), t1 = __byte_perm(w[0], w[1], 0x7362);
      const uint32_t t2 = __byte_perm(w[2], w[3], 0x5140), t3 = __byte_perm(w[2], w[3], 0x7362);
      const uint32_t v0 = __byte_perm(t0, t2, 0x5410), v1 = __byte_perm(t0, t2, 0x7632);
      const uint32_t v2 = __byte_perm(t1, t3, 0x5410), v3 = __byte_perm(t1, t3, 0x7632);
      // rows 4g+0 / 4g+1 (MMA row slots g / g+8), then rows 4g+2 / 4g+3; bytes 0..7, then 8..15
      int d0[4], d1[4], d2[4], d3[4];  // the byte sums start from zero (C operand 0)
      mma_u8_16x8x16(d0, v0, v1, bfrag[0]);
      mma_u8_16x8x16(d1, v0, v1, bfrag[1]);
      mma_u8_16x8x16(d2, v2, v3, bfrag[0]);
      mma_u8_16x8x16(d3, v2, v3, bfrag[1]);
      // (X_c, Y_c) of rows 4g+e to words 2c, 2c+1 of those rows (stride 10 words: the 64-bit
      // writes of a half-warp and the 64-bit reads below hit distinct banks)
      uint32_t* w0 = wstage[sbuf] + (4 * g) * kRecStageStride + 2 * c;
      *reinterpret_cast<uint2*>(w0) = make_uint2(uint32_t(d0[0]) + uint32_t(d0[1]) * 256u,
                                                 uint32_t(d1[0]) + uint32_t(d1[1]) * 256u);
      *reinterpret_cast<uint2*>(w0 + kRecStageStride) = make_uint2(uint32_t(d0[2]) + uint32_t(d0[3]) * 256u,
                                                                   uint32_t(d1[2]) + uint32_t(d1[3]) * 256u);
      *reinterpret_cast<uint2*>(w0 + 2 * kRecStageStride) = make_uint2(uint32_t(d2[0]) + uint32_t(d2[1]) * 256u,
                                                                       uint32_t(d3[0]) + uint32_t(d3[1]) * 256u);
      *reinterpret_cast<uint2*>(w0 + 3 * kRecStageStride) = make_uint2(uint32_t(d2[2]) + uint32_t(d2[3]) * 256u,
                                                                       uint32_t(d3[2]) + uint32_t(d3[3]) * 256u);
      __syncwarp();
      // this lane's row: S = sum_b T_b 2^(8b) as four 32-bit-aligned columns (each < 2^46)
      const uint32_t* rrow = wstage[sbuf] + lane * kRecStageStride;
      sbuf ^= 1;
      const uint2 q0 = *reinterpret_cast<const uint2*>(rrow), q1 = *reinterpret_cast<const uint2*>(rrow + 2);
      const uint2 q2 = *reinterpret_cast<const uint2*>(rrow + 4), q3 = *reinterpret_cast<const uint2*>(rrow + 6);
      const unsigned long long acc[4] = {static_cast<unsigned long long>(q1.x) * 65536ull + q0.x,
                                         static_cast<unsigned long long>(q3.x) * 65536ull + q2.x,
                                         static_cast<unsigned long long>(q1.y) * 65536ull + q0.y,
                                         static_cast<unsigned long long>(q3.y) * 65536ull + q2.y};
      const int64_t j = jb + jj;
      const bool keep = i < m && (uplo == 0 || (uplo == 1 ? i <= j : i >= j));
      if (!keep) continue;
      const int nu_j = nup[jj];
      const double v = __dmul_rn(sc.alpha, crt_finish_small<N>(acc, P_inv32, -mu_i - nu_j));
      if (EST) {
        if (uplo != 0 && mu_i != kCrtZeroRow && nu_j != kCrtZeroRow) e_acc += exp2_int(2 * (sc.b - mu_i - nu_j));
        v_acc += v * v;
      }
      if (sc.write_c) {
        if (sc.beta == 0.0) {
          *cp = v;
        } else {
          const double old = *cp;
          if (sc.save) sc.save[j * sc.ld_save + i] = old;
          *cp = __fma_rn(sc.beta, old, v);
        }
      }
    }
  }
  if (EST) crt_reduce_energies(R, e_acc, v_acc);
}

// Split-K: residue planes (l, s), s = 0 .. splits-1, of modulus l added modulo p_l into
// plane (l, 0); 16 bytes per thread, one modulus per grid row.
__global__ void __launch_bounds__(256) crt_merge_splits_kernel(uint8_t* __restrict__ cres, int64_t plane, int splits) {
  const int l = int(blockIdx.y);
  const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v * 16 >= plane) return;
  const uint32_t p = uint32_t(crt_modulus(l));
  uint8_t* base = cres + int64_t(l) * splits * plane + v * 16;
  uint32_t sum[16];
  const uint4 first = *reinterpret_cast<const uint4*>(base);
  const uint32_t w0[4] = {first.x, first.y, first.z, first.w};
#pragma unroll
  for (int b = 0; b < 16; ++b) sum[b] = (w0[b >> 2] >> (8 * (b & 3))) & 0xFFu;
  for (int s = 1; s < splits; ++s) {
    const uint4 q = *reinterpret_cast<const uint4*>(base + int64_t(s) * plane);
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int b = 0; b < 16; ++b) sum[b] += (w[b >> 2] >> (8 * (b & 3))) & 0xFFu;
  }
  uint32_t out[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int b = 0; b < 16; ++b) out[b >> 2] |= (sum[b] % p) << (8 * (b & 3));
  *reinterpret_cast<uint4*>(base) = make_uint4(out[0], out[1], out[2], out[3]);
}

template <int N>
void launch_rec128(bool est, bool mma, dim3 grid, cudaStream_t stream, const CrtRecParams& R) {
  if constexpr (N >= kCrtMinModuli) {
    if (mma) {
      if (est)
        crt_reconstruct_mma_kernel<N, true><<<grid, 256, 0, stream>>>(R);
      else
        crt_reconstruct_mma_kernel<N, false><<<grid, 256, 0, stream>>>(R);
      return;
    }
  }
  if (est)
    crt_reconstruct128_kernel<N, true><<<grid, 256, 0, stream>>>(R);
  else
    crt_reconstruct128_kernel<N, false><<<grid, 256, 0, stream>>>(R);
}

template <int BN, int STAGES, bool PAIR, int MT = 1, int NW = 4>
cudaError_t launch_gemm_config(const CrtOperand& a, const CrtOperand& b, const CrtGemmArgs& args,
                               cudaStream_t stream) {
  constexpr int kRowsPerTile = PAIR ? 2 * kSliceBM : MT * kSliceBM;
  if (a.rows_pad % kRowsPerTile != 0 || b.rows_pad % BN != 0 || args.ld_res != a.rows_pad)
    return cudaErrorInvalidValue;
  CUtensorMap tmA, tmB;
  if (!make_tensor_map_3d(&tmA, a.residues, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, uint64_t(a.k_pad), uint64_t(a.rows_pad),
                          uint64_t(a.nmax), kSliceKBytes, PAIR ? kSliceBM : MT * kSliceBM))
    return cudaErrorInvalidValue;
  if (!make_tensor_map_3d(&tmB, b.residues, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, uint64_t(b.k_pad), uint64_t(b.rows_pad),
                          uint64_t(b.nmax), kSliceKBytes, PAIR ? BN / 2 : BN))
    return cudaErrorInvalidValue;
  SliceGemmParams P{};
  P.m = args.m;
  P.n = args.n;
  P.num_kb = int(a.k_pad / kSliceKBytes);
  P.tiles_m = int(a.rows_pad / kRowsPerTile);
  P.tiles_n = int(b.rows_pad / BN);
  P.slices = args.moduli;
  P.diag_lo = 0;
  P.diag_hi = args.moduli - 1;
  P.skip_if_flag = args.skip_if_flag;
  P.status = args.status;
  const int gm = args.group_m > 0 ? args.group_m : tuning().group_m;
  P.group_m = gm > 0 ? gm : P.tiles_m;
  P.wait_limit_ns = tuning().wait_limit_ns ? tuning().wait_limit_ns : kWaitLimitNs;
  P.crt = 1;
  P.splits = args.splits > 1 ? args.splits : 1;
  if (P.splits > 1 && (args.tile_list != nullptr || args.tri_k != 0 || P.splits > P.num_kb))
    return cudaErrorInvalidValue;
  P.residues = args.cres;
  P.ld_res = args.ld_res;
  P.tile_list = args.tile_list;
  P.num_listed = args.num_listed;
  P.tri_k = args.tri_k;
  if (P.tile_list) {
    if (P.num_listed < 1 || P.num_listed > P.tiles_m * P.tiles_n) return cudaErrorInvalidValue;
    return launch_slice_gemm<kModeCrtI8Listed, BN, STAGES, NW, PAIR, MT>(tmA, tmB, P, args.num_sms, stream);
  }
  return launch_slice_gemm<kModeCrtI8, BN, STAGES, NW, PAIR, MT>(tmA, tmB, P, args.num_sms, stream);
}

}  // namespace

int64_t crt_tile_rows(int tile_n) { return (tile_n == kTilePair || tile_n == kTileWide) ? 256 : 128; }
int64_t crt_tile_cols(int tile_n) { return tile_n == 128 ? 128 : 256; }

void crt_triangle_tiles(int tile_n, int64_t rows_pad, int64_t cols_pad, int64_t n, bool upper, int group_m, int* out,
                        int* count) {
  const int64_t br = crt_tile_rows(tile_n), bc = crt_tile_cols(tile_n);
  const int tiles_m = int(rows_pad / br), tiles_n = int(cols_pad / bc);
  const int gm_all = group_m > 0 ? group_m : tiles_m;
  int c = 0;
  for (int tile = 0; tile < tiles_m * tiles_n; ++tile) {
    // the raster of tile_coords() in the GEMM kernel
    const int group_size = gm_all * tiles_n;
    const int first_m = (tile / group_size) * gm_all;
    const int gm = std::min(tiles_m - first_m, gm_all);
    const int r = tile % group_size;
    const int64_t r0 = int64_t(first_m + r % gm) * br, c0 = int64_t(r / gm) * bc;
    // tiles wholly in the padding hold no output
    const bool meets = r0 < n && c0 < n && (upper ? (r0 <= c0 + bc - 1) : (r0 + br - 1 >= c0));
    if (meets) out[c++] = tile;
  }
  *count = c;
}

cudaError_t launch_crt_scan_norms(const StridedView<double>& x, const CrtOperand& op, int* nonfinite, double* spread,
                                  cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(op.maxbits, 0, size_t(op.rows) * sizeof(uint64_t), stream);
  if (e != cudaSuccess || x.rows == 0 || x.cols == 0) return e;
  if (op.k_pad % kNormCols != 0) return cudaErrorInvalidValue;
  dim3 grid(unsigned((x.cols + kNormCols - 1) / kNormCols), unsigned((x.rows + kNormRows - 1) / kNormRows));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  crt_scan_norm_kernel<<<grid, kNormThreads, 0, stream>>>(x.ptr, x.rows, x.cols, x.sr, x.sl,
                                                 reinterpret_cast<unsigned long long*>(op.maxbits), op.chunk_e,
                                                 reinterpret_cast<unsigned long long*>(op.chunk_s),
                                                 op.k_pad / kNormCols, nonfinite, spread);
  return cudaGetLastError();
}

cudaError_t launch_crt_split(const StridedView<double>& x, const CrtOperand& op, int moduli, cudaStream_t stream) {
  if (moduli < 1 || moduli > op.nmax) return cudaErrorInvalidValue;
  if (op.k_pad % kSplitColsCrt != 0 || op.rows_pad % kSplitRowsCrt != 0) return cudaErrorInvalidValue;
  dim3 grid(unsigned(op.k_pad / kSplitColsCrt), unsigned(op.rows_pad / kSplitRowsCrt));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  const int b = crt_bits(moduli);
  crt_mu_kernel<<<unsigned((op.rows_pad + 7) / 8), 256, 0, stream>>>(
      reinterpret_cast<const unsigned long long*>(op.maxbits), op.chunk_e,
      reinterpret_cast<const unsigned long long*>(op.chunk_s), op.k_pad / kNormCols, op.rows, op.rows_pad, b, op.mu);
  if (moduli == kCrtDefaultModuli && b <= 62)
    crt_split_kernel<false, kCrtDefaultModuli><<<grid, kSplitThreadsCrt, 0, stream>>>(
        x.ptr, x.rows, x.cols, x.sr, x.sl, op.mu, moduli, op.residues, op.rows_pad, op.k_pad);
  else if (b <= 62)
    crt_split_kernel<false, 0><<<grid, kSplitThreadsCrt, 0, stream>>>(x.ptr, x.rows, x.cols, x.sr, x.sl, op.mu, moduli,
                                                                     op.residues, op.rows_pad, op.k_pad);
  else
    crt_split_kernel<true, 0><<<grid, kSplitThreadsCrt, 0, stream>>>(x.ptr, x.rows, x.cols, x.sr, x.sl, op.mu, moduli,
                                                                    op.residues, op.rows_pad, op.k_pad);
  return cudaGetLastError();
}

cudaError_t launch_crt_gemm(const CrtOperand& a, const CrtOperand& b, const CrtGemmArgs& args, cudaStream_t stream) {
  if (args.moduli < 1 || args.moduli > a.nmax || args.moduli > b.nmax) return cudaErrorInvalidValue;
  if (a.k_pad != b.k_pad || a.k_pad % kSliceKBytes != 0) return cudaErrorInvalidValue;
  if (args.tile_n == kTilePair) return launch_gemm_config<256, 6, true>(a, b, args, stream);
  if (args.tile_n == 256) return launch_gemm_config<256, 4, false>(a, b, args, stream);
  // 256 x 256 per CTA: 64 KB stages (three), sixteen epilogue warps (four per TMEM lane
  // quadrant: the single accumulator buffer is drained while the MMAs wait, so the drain is
  // spread over as many warps as the registers allow)
  if (args.tile_n == kTileWide) return launch_gemm_config<256, 3, false, 2, 16>(a, b, args, stream);
  return cudaErrorInvalidValue;
}

cudaError_t launch_crt_merge_splits(uint8_t* cres, int64_t plane, int moduli, int splits, cudaStream_t stream) {
  if (splits <= 1) return cudaSuccess;
  if (moduli < 1 || moduli > kCrtMaxModuli || splits > kCrtMaxSplits || plane % 16 != 0) return cudaErrorInvalidValue;
  const int64_t vecs = plane / 16;
  dim3 grid(unsigned((vecs + 255) / 256), unsigned(moduli));
  if (grid.x == 0) return cudaSuccess;
  crt_merge_splits_kernel<<<grid, 256, 0, stream>>>(cres, plane, splits);
  return cudaGetLastError();
}

cudaError_t launch_crt_reconstruct(const CrtReconstructArgs& args, cudaStream_t stream) {
  if (args.moduli < 1 || args.moduli > kCrtMaxModuli) return cudaErrorInvalidValue;
  if (args.m == 0 || args.n == 0) return cudaSuccess;
  const CrtConstants& k = crt_constants(args.moduli);
  CrtRecParams R;
  std::memcpy(R.W, k.W, sizeof(R.W));
  std::memcpy(R.P, k.P, sizeof(R.P));
  std::memcpy(R.half, k.half, sizeof(R.half));
  R.P_inv = k.P_inv;
  R.n = args.moduli;
  R.b = k.b;
  R.m = args.m;
  R.ncols = args.n;
  R.alpha = args.alpha;
  R.beta = args.beta;
  R.C = args.C;
  R.ldc = args.ldc;
  R.res = args.cres;
  R.ld_res = args.ld_res;
  R.plane = args.plane;
  R.mu_a = args.mu_a;
  R.mu_b = args.mu_b;
  R.err_sq = args.err_sq;
  R.skip_if_flag = args.skip_if_flag;
  R.write_c = args.write_c ? 1 : 0;
  R.save = args.save;
  R.ld_save = args.ld_save;
  R.uplo = args.uplo;
  // the tensor-core sum: whole warps of 32 rows copy the residue planes 16 bytes at a time, so
  // the planes must be 16-byte aligned and hold every row of those warps
  const bool mma = args.moduli >= kCrtMinModuli && args.moduli <= 16 && reinterpret_cast<uintptr_t>(args.cres) % 16 == 0 &&
                   args.ld_res % 32 == 0 && args.plane % 16 == 0 && args.ld_res >= (args.m + 31) / 32 * 32;
  const int64_t rows_per_block = 256;
  const unsigned gx = unsigned((args.m + rows_per_block - 1) / rows_per_block);
  // up to kRecCols columns per block, fewer while the grid is under ~4 blocks per SM
  int64_t cpb = int64_t(gx) * args.n / (4 * 148);
  cpb = cpb < 1 ? 1 : (cpb > kRecCols ? kRecCols : cpb);
  R.cols_per_block = int(cpb);
  const int64_t groups = (args.n + cpb - 1) / cpb;
  const unsigned gy = unsigned(groups < 65535 ? groups : 65535);
  const dim3 grid(gx, gy);
  const bool est = args.err_sq != nullptr;
  switch (args.moduli) {
    case 8: launch_rec128<8>(est, mma, grid, stream, R); break;
    case 9: launch_rec128<9>(est, mma, grid, stream, R); break;
    case 10: launch_rec128<10>(est, mma, grid, stream, R); break;
    case 11: launch_rec128<11>(est, mma, grid, stream, R); break;
    case 12: launch_rec128<12>(est, mma, grid, stream, R); break;
    case 13: launch_rec128<13>(est, mma, grid, stream, R); break;
    case 14: launch_rec128<14>(est, mma, grid, stream, R); break;
    case 15: launch_rec128<15>(est, mma, grid, stream, R); break;
    case 16: launch_rec128<16>(est, mma, grid, stream, R); break;
    default: crt_reconstruct_kernel<<<grid, 256, 0, stream>>>(R); break;  // other counts: 192-bit path
  }
  return cudaGetLastError();
}

}  // namespace eb2
