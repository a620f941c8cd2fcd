// kernels.h -- internal host-side interface of the device kernels (launch wrappers).
// Everything here is stream-ordered and allocation-free: callers pass device
// buffers that they own.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace eb2 {

// Launch-shape knobs of the tcgen05 slice GEMM (set by the tuner; process-wide).
struct SliceTuning {
  int group_m = 0;   // row-tiles per raster group; 0 = all (column-major tile order)
  int prefetch = 0;  // L2 prefetch distance in K blocks; 0 = off
  // wall-time limit (ns) of the GEMM's pipeline waits; 0 = the default (2 s).  The waits
  // that drain copies and MMAs already issued keep the default.
  uint64_t wait_limit_ns = 0;
};
SliceTuning& tuning();

// A strided view of op(X) as a rows x cols matrix: element (r, l) at X[r*sr + l*sl].
template <typename T>
struct StridedView {
  const T* ptr;
  int64_t rows, cols;
  int64_t sr, sl;
};

// ------------------------------------------------------------ native FP64 / FP32
// C = alpha * op(A) op(B) + beta * C, column-major, device pointers.
// If `only_if_flag` is non-null the kernel does nothing unless *only_if_flag != 0
// (device-side fallback for inputs the emulated path cannot represent).
cudaError_t launch_dgemm_native(bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                                const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                                int64_t ldc, const int* only_if_flag, cudaStream_t stream);
cudaError_t launch_sgemm_native(bool transA, bool transB, int64_t m, int64_t n, int64_t k, float alpha,
                                const float* A, int64_t lda, const float* B, int64_t ldb, float beta, float* C,
                                int64_t ldc, const int* only_if_flag, cudaStream_t stream);
// C = beta * C (beta == 0 writes exact zeros), the BLAS pre-scale for alpha == 0 or k == 0.
cudaError_t launch_scale_matrix_d(int64_t m, int64_t n, double beta, double* C, int64_t ldc, cudaStream_t stream);
cudaError_t launch_scale_matrix_s(int64_t m, int64_t n, float beta, float* C, int64_t ldc, cudaStream_t stream);

// ------------------------------------------------------------ Ozaki (emulated FP64)
constexpr int kOzakiMaxSlices = 12;
// Tile configurations of the tcgen05 kernels: 128 / 256 = one CTA computing 128 x 128 /
// 128 x 256 tiles; kTilePair = a CTA pair (cluster of 2) computing 256 x 256 tiles.
constexpr int kTilePair = 512;
// CRT GEMM only: one CTA computing 256 x 256 tiles (two M = 128 MMAs per K step share the B
// tile; the accumulator fills the TMEM, so consecutive tiles do not overlap).
constexpr int kTileWide = 1024;
constexpr int kOzakiKBlock = 128;  // bytes of K per pipeline stage (int8 digits)
constexpr int kOzakiBM = 128;

// Per-operand workspace of the digit split.
struct OzakiOperand {
  int8_t* digits;       // [smax][rows_pad][k_pad], row r contiguous along k
  int32_t* exps;        // [rows_pad] binary exponent of each row's max |x|
  uint64_t* maxbits;    // [rows] bit pattern of max |x| (scan output)
  double* abssum;       // [k] sum over rows of |x|; optional (null skips it)
  int64_t rows, rows_pad, k, k_pad;
  int smax;
};

// Zero the scan accumulators of one operand (maxbits, abssum).
cudaError_t launch_ozaki_scan_reset(const OzakiOperand& op, cudaStream_t stream);
// Row maxima and |x| sums; sets *nonfinite when any NaN/Inf is present; accumulates the
// exponent-spread statistic into spread[0..1] (sum, count) when spread is non-null.
cudaError_t launch_ozaki_scan(const StridedView<double>& x, const OzakiOperand& op, int* nonfinite, double* spread,
                              cudaStream_t stream);
// Digits p in [p_begin, p_end) of every row (including zero padding).
cudaError_t launch_ozaki_split(const StridedView<double>& x, const OzakiOperand& op, int p_begin, int p_end,
                               cudaStream_t stream);

struct OzakiGemmArgs {
  int64_t m, n, k;
  double alpha, beta;
  double* C;
  int64_t ldc;
  int slices;          // s: digits per operand used by this call
  int diag_lo, diag_hi;  // accumulate diagonals t in [diag_lo, diag_hi] (t = p + q, digits p,q >= 1)
  bool first_writes;   // true: the first unit applies beta (C = beta*C + ...); false: C += ...
  const int* skip_if_flag;  // non-null: the kernel returns at once when *flag != 0
  double* err_sq;      // [2]: += squared contribution of diagonal diag_hi, and of diagonal 2 (may be null)
  uint32_t* status;    // device status word (EB2_DEV_*)
  int tile_n;          // 128, 256 or kTilePair
  int num_sms;
};
cudaError_t launch_ozaki_gemm(const OzakiOperand& a, const OzakiOperand& b, const OzakiGemmArgs& args,
                              cudaStream_t stream);

// ------------------------------------------------------------ CRT / Ozaki-II (emulated FP64)
// Moduli of the CRT product: pairwise coprime, <= 256, largest first.
constexpr int kCrtMaxModuli = 20;
constexpr int kCrtDefaultModuli = 16;
constexpr int kCrtMinModuli = 8;  // fewest moduli the picker and the tuner use
constexpr int kCrtLimbs = 6;  // 192-bit reconstruction arithmetic (32-bit limbs)
constexpr int kCrtMaxSplits = 16;  // K splits of the CRT GEMM (split residues summed < 2^12)
constexpr int kCrtZeroRow = -(1 << 20);  // mu of a row without a nonzero finite entry
// (p - 1 packed one byte each, so device code indexes no local array)
__host__ __device__ constexpr int crt_modulus(int l) {
  return int((l < 8 ? 0xe8eef0f6fafcfeffull : l < 16 ? 0xc0c4c6d2d8dee2e4ull : 0x00000000acb2b4beull) >>
                 (8 * (l & 7)) &
             0xFFu) +
         1;
}

// P = p_0 ... p_(n-1), the CRT weights W_l = (P/p_l) ((P/p_l)^-1 mod p_l), P/2 (floor) and
// b, the largest integer with 2^(2b+1) < P (row norms of the scaled operands <= 2^b).
struct CrtConstants {
  int n, b;
  double P_inv;
  uint32_t P[kCrtLimbs], half[kCrtLimbs];
  uint32_t W[kCrtMaxModuli][kCrtLimbs];
};
const CrtConstants& crt_constants(int n);
int crt_bits(int n);
// Tile rows / columns of the CRT GEMM configurations (256: one CTA, 128 x 256 tiles;
// kTilePair: a CTA pair, 256 x 256 tiles).
int64_t crt_tile_rows(int tile_n);
int64_t crt_tile_cols(int tile_n);

// Per-operand workspace of the residue split.
struct CrtOperand {
  int8_t* residues;   // [nmax][rows_pad][k_pad] symmetric residues, row r contiguous along k
  int32_t* mu;        // [rows_pad] scale exponents: A'_r = trunc(2^mu_r x_r) (kCrtZeroRow: A'_r = 0)
  uint64_t* maxbits;  // [rows] bit pattern of max |x|
  uint64_t* chunk_s;  // [rows][k_pad/128] integer norm bound of each 128-column chunk, relative to
  int32_t* chunk_e;   // [rows][k_pad/128]   the exponent of the chunk's maximum
  int64_t rows, rows_pad, k, k_pad;
  int nmax;
};
// One read of op(X): row maxima, chunk norm bounds, the NaN/Inf flag (*nonfinite = 1) and
// the exponent-spread statistic (spread[0..1] += sum, count; may be null).
cudaError_t launch_crt_scan_norms(const StridedView<double>& x, const CrtOperand& op, int* nonfinite, double* spread,
                                  cudaStream_t stream);
// mu for `moduli` moduli, then the residues for moduli [0, moduli) (needs the scan).
cudaError_t launch_crt_split(const StridedView<double>& x, const CrtOperand& op, int moduli, cudaStream_t stream);

struct CrtGemmArgs {
  int64_t m, n;
  int moduli;
  const int* skip_if_flag;
  uint32_t* status;
  int tile_n;  // 256, kTilePair or kTileWide
  int num_sms;
  uint8_t* cres;   // [moduli][n_pad][ld_res] residues of C' (uint8 in [0, p))
  int64_t ld_res;  // = a.rows_pad
  const int* tile_list = nullptr;  // device: the output tiles to compute (null: all)
  int num_listed = 0;
  int tri_k = 0;  // triangular operand whose zero K blocks are skipped: 1/2 = op(A) lower/upper,
                  // 3/4 = op(B) lower/upper (0: dense)
  // split-K: every (tile, modulus) is computed as `splits` K ranges, each into its own residue
  // plane: cres is [moduli][splits][n_pad][ld_res], merged by launch_crt_merge_splits (dense
  // operands, no tile list, splits <= the K blocks).  1: none.
  int splits = 1;
  int group_m = 0;  // row tiles per raster group (0: the process-wide tuning)
};
cudaError_t launch_crt_gemm(const CrtOperand& a, const CrtOperand& b, const CrtGemmArgs& args, cudaStream_t stream);
// Adds the `splits` residue planes of every modulus modulo its p into the modulus's first
// plane (plane = bytes of one plane, a multiple of 16): the layout the reconstruction reads
// with a plane stride of splits * plane.
cudaError_t launch_crt_merge_splits(uint8_t* cres, int64_t plane, int moduli, int splits, cudaStream_t stream);

struct CrtReconstructArgs {
  int64_t m, n;
  double alpha, beta;
  double* C;
  int64_t ldc;
  const uint8_t* cres;
  int64_t ld_res, plane;
  int moduli;
  const int32_t* mu_a;
  const int32_t* mu_b;
  double* err_sq;  // [2]: += estimated squared error, += squared alpha*A*B entries (may be null)
  const int* skip_if_flag;
  bool write_c;    // false: only the estimate
  // beta != 0: where the old C goes as the new one is written (ld_save), so that a product
  // that must be redone with more moduli can start again from it (null: not kept)
  double* save = nullptr;
  int64_t ld_save = 0;
  int uplo = 0;    // 0: all of C; 1: only i <= j (upper triangle); 2: only i >= j (lower)
};
cudaError_t launch_crt_reconstruct(const CrtReconstructArgs& args, cudaStream_t stream);

// ------------------------------------------------------------ split-BF16 (emulated FP32)
struct Bf16Operand {
  void* pieces;  // [3][rows_pad][k_pad] bf16: hi, mid, lo pieces, row r contiguous along k
  int64_t rows, rows_pad, k, k_pad;
};
// Split op(X) (rows x k view) into its three BF16 pieces; sets *nonfinite on NaN/Inf.
cudaError_t launch_bf16_split(const StridedView<float>& x, const Bf16Operand& op, int* nonfinite,
                              cudaStream_t stream);

struct SgemmSplitArgs {
  int64_t m, n, k;
  float alpha, beta;
  float* C;
  int64_t ldc;
  int pieces;  // s: 2 -> 3 products (hh, hm, mh), 3 -> 6 products (+ mm, hl, lh)
  const int* skip_if_flag;
  uint32_t* status;
  int tile_n;
  int num_sms;
};
cudaError_t launch_sgemm_split_bf16(const Bf16Operand& a, const Bf16Operand& b, const SgemmSplitArgs& args,
                                    cudaStream_t stream);

// ------------------------------------------------------------ triangles (level-3 routines)
constexpr int kTriBlock = 64;  // largest diagonal block launch_tri_block_multiply takes
constexpr int kTriVecs = 64;   // vectors per CTA of launch_tri_block_multiply
// out (n x n) = the symmetric matrix whose triangle `upper` (else lower) is stored in A.
template <typename T>
cudaError_t launch_expand_symmetric(const T* A, int64_t lda, int64_t n, bool upper, T* out, int64_t ldo,
                                    cudaStream_t stream);
// out (n x n) = the triangular matrix in the triangle `upper` (else lower) of A, zeros
// elsewhere, ones on the diagonal if `unit` (the stored diagonal then unread).
template <typename T>
cudaError_t launch_expand_triangular(const T* A, int64_t lda, int64_t n, bool upper, bool unit, T* out, int64_t ldo,
                                     cudaStream_t stream);
// On the triangle `upper` of the n x n C only: C = P + beta C (beta == 0 does not read C;
// P == null: C = beta C, beta == 0 writing zeros).
template <typename T>
cudaError_t launch_merge_triangle(const T* P, int64_t ldp, int64_t n, bool upper, T beta, T* C, int64_t ldc,
                                  cudaStream_t stream, const int* only_if_flag = nullptr);
// The tiles of the CRT GEMM's raster (configuration `tile_n` over rows_pad x cols_pad, raster
// groups of group_m tile rows, 0 = all) that meet the triangle `upper` / lower of the n x n C,
// in raster order.
void crt_triangle_tiles(int tile_n, int64_t rows_pad, int64_t cols_pad, int64_t n, bool upper, int group_m, int* out,
                        int* count);
// X = alpha X by plain multiplication (NaN/Inf stay for alpha == 0).
template <typename T>
cudaError_t launch_multiply(int64_t m, int64_t n, T alpha, T* X, int64_t ldx, cudaStream_t stream);
// x := E x for `count` vectors (element r of vector t at X[r*vs + t*ts]), E the nb x nb
// (nb <= kTriBlock) triangle `lower`/upper at E[r*er + c*ec], unit diagonal if `unit` (then
// the stored diagonal is not read; neither is the other triangle).
template <typename T>
cudaError_t launch_tri_block_multiply(const T* E, int64_t er, int64_t ec, int nb, bool lower, bool unit, T* X,
                                      int64_t vs, int64_t ts, int64_t count, cudaStream_t stream);
constexpr int kPanelMax = 256;  // largest diagonal block launch_tri_panel_solve takes
constexpr int kPanelVecs = 64;  // vectors per CTA of launch_tri_panel_solve
// x := E^-1 x for `count` vectors laid out as for launch_tri_block_multiply, E the nb x nb
// (nb <= kPanelMax) triangle, by blocked substitution.
template <typename T>
cudaError_t launch_tri_panel_solve(const T* E, int64_t er, int64_t ec, int nb, bool lower, bool unit, T* X,
                                   int64_t vs, int64_t ts, int64_t count, cudaStream_t stream);

// ------------------------------------------------------------ complex GEMM (two real products)
// op(X) (rows x cols complex; element (r, c) at complex index r*sr + c*sc of the interleaved
// array X; imaginary parts negated if conj) -> Y = [Re | Im] (rows x 2 cols, ld rows).
template <typename T>
cudaError_t launch_pack_complex_lhs(const T* X, int64_t sr, int64_t sc, bool conj, int64_t rows, int64_t cols, T* Y,
                                    cudaStream_t stream);
// op(X) (rows x cols complex) -> Y1 = [Re; -Im], Y2 = [Im; Re] (2 rows x cols each, ld 2 rows).
template <typename T>
cudaError_t launch_pack_complex_rhs(const T* X, int64_t sr, int64_t sc, bool conj, int64_t rows, int64_t cols, T* Y1,
                                    T* Y2, cudaStream_t stream);
// C (m x n complex, interleaved, ld ldc) = (ar + i ai)(Pr + i Pi) + (br + i bi) C; beta == 0
// does not read C; Pr == null: C = beta C.
template <typename T>
cudaError_t launch_combine_complex(const T* Pr, const T* Pi, int64_t ldp, int64_t m, int64_t n, T ar, T ai, T br,
                                   T bi, T* C, int64_t ldc, cudaStream_t stream);
// out (n x n complex) from the triangle `upper` of the complex A: mode 0 symmetric (mirror),
// 1 Hermitian (conjugate mirror, real diagonal), 2 triangular (zeros outside, unit diagonal
// if `unit`).  Only the stored triangle of A is read.
template <typename T>
cudaError_t launch_expand_complex(const T* A, int64_t lda, int64_t n, bool upper, int mode, bool unit, T* out,
                                  int64_t ldo, cudaStream_t stream);
// x := E^-1 x for `count` complex vectors (element r of vector t at complex index
// r*vs + t*ts), E the nb x nb (nb <= kPanelMaxComplex) complex triangle `lower`/upper at
// complex index r*er + c*ec, conjugated when `conj`, unit diagonal if `unit`.
constexpr int kPanelMaxComplex = 128;
template <typename T>
cudaError_t launch_tri_panel_solve_complex(const T* E, int64_t er, int64_t ec, int nb, bool lower, bool unit,
                                           bool conj, T* X, int64_t vs, int64_t ts, int64_t count,
                                           cudaStream_t stream);

}  // namespace eb2
