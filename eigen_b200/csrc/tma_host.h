// tma_host.h -- host-side creation of TMA tensor maps through the driver entry point
// (cuTensorMapEncodeTiled), without linking libcuda directly.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

namespace eb2 {

// Returns nullptr if the driver does not provide the entry point.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// 3-D tiled map over a dense [d2][d1][d0] array of `elem_bytes`-sized elements,
// box {b0, b1, 1}, 128-byte swizzle.  Returns false on failure.
bool make_tensor_map_3d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, int elem_bytes, uint64_t d0,
                        uint64_t d1, uint64_t d2, uint32_t b0, uint32_t b1);

}  // namespace eb2
