// air_launch.hpp -- host entry points of the air kernels.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace tpt {
namespace air {

// One AIR_TX x AIR_TY tile of one batched instance.
struct TileRef {
    uint32_t inst;
    uint16_t tx, ty;
};

// Tensor maps of one batched instance: the grids pass A and pass B stage,
// with the two halves of the heat and mask ping-pong.
enum TensorMapSlot {
    TM_PV, TM_VX, TM_VY, TM_OVX, TM_OVY, TM_OPV, TM_BA0, TM_BA1, TM_BH0, TM_BH1, TM_HV0, TM_HV1, TM_COUNT
};

// One tick of one grid: A (pressure+velocity), B (advection+heat), settle.
int launch_single(const AirInst &I, const uint32_t *pmap, const uint32_t *props, uint32_t nprops, uint32_t xres,
                  uint32_t yres, cudaStream_t st);

// One tick of every instance of a batch. `insts` holds two AirInst per
// instance (parity 0 and 1 of the hv / mask ping-pong); `tmaps` TM_COUNT
// tensor maps per instance.
int launch_batch_tick(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles,
                      uint32_t grid, uint32_t parity, bool any_noupdate_heat, cudaStream_t st);
int launch_copy_back(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, cudaStream_t st);

// Reads and clears the device error word of the batched air kernels.
int read_errors(uint32_t *out);

}  // namespace air
}  // namespace tpt
