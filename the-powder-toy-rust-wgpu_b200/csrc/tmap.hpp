// tmap.hpp -- access to the driver's tensor-map encoder without linking
// libcuda (the runtime hands out the entry point).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

namespace tpt {

// cuTensorMapEncodeTiled, or null if the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// 2-D map of a grid of 4-byte elements (f32 or u32), `cols` x `rows` with a
// row stride of `pitch` elements, box `box_cols` x `box_rows`, no swizzle,
// zero fill outside the grid.
int make_grid_tmap(CUtensorMap *out, const void *base, bool is_float, uint32_t cols, uint32_t rows, uint32_t pitch,
                   uint32_t box_cols, uint32_t box_rows);

}  // namespace tpt
