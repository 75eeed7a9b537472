// air_launch.hpp -- host entry points of the air kernels.
#pragma once

#include "common.cuh"

namespace tpt {
namespace air {

// One AIR_TX x AIR_TY tile of one batched instance.
struct TileRef {
    uint32_t inst;
    uint16_t tx, ty;
};

// One tick of one grid: A (pressure+velocity), B (advection+heat), settle.
int launch_single(const AirInst &I, const uint32_t *pmap, const uint32_t *props, uint32_t nprops, uint32_t xres,
                  uint32_t yres, cudaStream_t st);

// One tick of every instance of a batch. `insts` holds two AirInst per
// instance (parity 0 and 1 of the hv / mask ping-pong).
int launch_batch_tick(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, uint32_t parity,
                      bool any_noupdate_heat, cudaStream_t st);
int launch_copy_back(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, cudaStream_t st);

}  // namespace air
}  // namespace tpt
