// air_launch.hpp -- host entry points of the air kernels.
#pragma once

#include "common.cuh"

namespace tpt {
namespace air {

// One AIR_TX x AIR_TY tile of one batched instance (the pre-pass and the
// copy-back walk these).
struct TileRef {
    uint32_t inst;
    uint16_t tx, ty;
};

// ---- row sweeps (air_sweep.cu) -------------------------------------------------
// Lanes of halo on each side of a segment: the tick's stencil reaches six
// columns (block_air of the effective velocity's wall clear, five more stages
// of one column each).
constexpr int SW_H = 6;
constexpr int SW_MAXSEG = 8;          // segments packed into one work item
constexpr int SWEEP_MAX_LANES = 256;  // lanes (threads) of a sweep CTA
constexpr int SWEEP_RING_ROWS = 42;   // shared-memory rows of NL + 2 words each

// A column strip of one instance inside a work item: lanes [lane0, lane0 +
// lanes) hold columns x0 - SW_H .. x0 + nx + SW_H - 1; output columns x0 ..
// x0 + nx - 1 and rows y0 .. y0 + ny - 1.
struct SweepSeg {
    uint32_t inst;
    uint16_t lane0, lanes;
    uint16_t x0, nx;
    uint16_t y0, ny;
};
struct SweepItem {
    uint32_t nseg;
    uint32_t steps;  // max ny over the segments
    SweepSeg seg[SW_MAXSEG];
};

// Everything one tick of the sweep form needs.
struct SweepLaunch {
    const AirInst *insts;       // two per instance (parity 0 and 1 of the ping-pong pairs)
    const TileRef *tiles;       // pre-pass tiles
    uint32_t ntiles;
    const SweepItem *items;
    uint32_t nitems;
    uint32_t ninst;
    uint32_t lanes;             // threads per sweep CTA (multiple of 32, <= SWEEP_MAX_LANES)
    uint32_t grid;              // sweep CTAs
    uint32_t prepass_grid;      // pre-pass CTAs
    uint32_t *ctl;              // [0]: the sweep's work-queue counter
    uint32_t *want;             // [2][ninst]: pre-pass flags per tick parity
};

// One tick of every instance of a batch: the pre-pass of flagged instances,
// then the sweep. `parity` selects the ping-pong halves read.
int launch_sweep_tick(const SweepLaunch &s, uint32_t parity, cudaStream_t st);
int launch_prepass(const SweepLaunch &s, uint32_t parity, cudaStream_t st);
int sweep_max_ctas_per_sm(uint32_t lanes, int *out);

// One tick of one grid: A (pressure+velocity), B (advection+heat), settle.
int launch_single(const AirInst &I, const uint32_t *pmap, const uint32_t *props, uint32_t nprops, uint32_t xres,
                  uint32_t yres, cudaStream_t st);

// Copies the ping-pong halves that hold the newest state back to the
// instance's canonical buffers (after an odd number of ticks).
int launch_copy_back(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, cudaStream_t st);

// Reads and clears the device error word of the batched air kernels.
int read_errors(uint32_t *out);

}  // namespace air
}  // namespace tpt
