// blas_common.h -- what every Fortran-convention entry point shares: the character-argument
// codes of blas/common.h:45-68, the test for operands the device can use in place, and the
// staging of host operands through device buffers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "context.h"

extern "C" void xerbla_(const char* name, int* info, size_t len);

namespace eb2 {

// blas/common.h:45-58 and the OP/SIDE/UPLO/DIAG parsers of :60-68 (case-insensitive)
enum { kNoTr = 0, kTr = 1, kAdj = 2, kInvalid = 0xff };
enum { kLeft = 0, kRight = 1 };
enum { kUp = 0, kLo = 1 };
enum { kNonUnit = 0, kUnit = 1 };

inline int op_code(char c) {
  if (c == 'N' || c == 'n') return kNoTr;
  if (c == 'T' || c == 't') return kTr;
  if (c == 'C' || c == 'c') return kAdj;
  return kInvalid;
}
inline int side_code(char c) {
  if (c == 'L' || c == 'l') return kLeft;
  if (c == 'R' || c == 'r') return kRight;
  return kInvalid;
}
inline int uplo_code(char c) {
  if (c == 'U' || c == 'u') return kUp;
  if (c == 'L' || c == 'l') return kLo;
  return kInvalid;
}
inline int diag_code(char c) {
  if (c == 'N' || c == 'n') return kNonUnit;
  if (c == 'U' || c == 'u') return kUnit;
  return kInvalid;
}

// Per-routine call counters behind eb2_routine_calls: a routine counts once per call that
// gets past its argument checks and quick returns (name lower-case without the trailing
// underscore, e.g. "dtrsm").
void count_call(const char* name);

// True when the device can use the pointer in place (device or managed memory).
bool device_usable(const void* p);

// Copy a column-major block of `cols` columns, `row_bytes` each, between host and device
// (pageable host memory through the context's pinned bounce buffers; a device -> host copy
// has landed when this returns); sets the thread's error and returns false when the copy
// cannot be queued.  The caller holds the context's mutex.
bool copy_block(void* dst, size_t dpitch, const void* src, size_t spitch, size_t row_bytes, int64_t cols,
                cudaMemcpyKind kind, cudaStream_t st);

}  // namespace eb2
