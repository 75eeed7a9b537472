// air_launch.hpp -- host entry points of the air kernels.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace tpt {
namespace air {

// One tile of one batched instance: AIR_TX x AIR_TY cells for the pre-pass and
// the copy-back, the tile form's shape for its passes.
struct TileRef {
    uint32_t inst;
    uint16_t tx, ty;
};

// ---- the tile form (air_tiles.cu) ---------------------------------------------
// Tensor maps of one batched instance: the grids the two passes stage, with
// the two halves of the heat and mask ping-pong.
// The velocity pass's outputs (ovx, ovy, opv) alternate between two sets by
// tick parity, so a launch that ends one tick and starts the next (the
// temporally blocked form) reads one set while it writes the other.
enum TensorMapSlot {
    TM_PV, TM_VX, TM_VY,
    TM_OV0, TM_OVX0 = TM_OV0, TM_OVY0, TM_OPV0,
    TM_OV1, TM_OVX1 = TM_OV1, TM_OVY1, TM_OPV1,
    TM_BA0, TM_BA1, TM_BH0, TM_BH1, TM_HV0, TM_HV1, TM_COUNT
};

// One tile shape of the tile form (air_tiles.cu, compiled once per shape).
// Its tiles are tx x ty cells, one thread per cell, each staged as a TMA box
// of (tx + 8) x (ty + 6) cells: the tensor maps and the tile list of a batch
// are built for the shape in use.
struct TileShape {
    uint32_t tx, ty;
    // sets the kernels' shared-memory limits and returns the resident CTAs
    // per SM of the velocity pass (A) and the advection/heat pass (B)
    int (*prepare)(int *occupancy_a, int *occupancy_b);
    // The two passes of one tick of every instance: the velocity pass (A),
    // and the advection / heat / mask pass (B, with its NoUpdate settle)
    // whose mask rebuild applies `emap_lag` pending emap decays. `insts` holds
    // two AirInst per instance (parity 0 and 1 of the hv / mask ping-pong and
    // of the velocity-pass outputs; pv/vx/vy are updated in place); `tmaps`
    // TM_COUNT tensor maps per instance. `queues`: the two passes' work-queue
    // counters (device, zero at creation), used as queues when `use_queue`
    // (else the CTAs stride the tile list statically) and cleared either way,
    // each by the launch of the other pass.
    int (*launch_a)(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles,
                    uint32_t grid, uint32_t parity, uint32_t *queues, bool use_queue, cudaStream_t st);
    int (*launch_b)(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles,
                    uint32_t grid, uint32_t parity, uint32_t emap_lag, bool any_noupdate_heat, uint32_t *queues,
                    bool use_queue, cudaStream_t st);
    // the copy-back of NoUpdate instances' convected velocity after a pass B
    int (*launch_settle)(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, uint32_t parity,
                         cudaStream_t st);
    // reads and clears the shape's device error word
    int (*read_errors)(uint32_t *out);
};
extern const TileShape tile_shape_s32x8, tile_shape_s64x8, tile_shape_s32x16, tile_shape_s64x16;
constexpr int TILE_SHAPES = 4;
// The offered shapes, 32x8 first; tile_shape(tx, ty) is null for any other.
const TileShape *const *tile_shapes();
const TileShape *tile_shape(uint32_t tx, uint32_t ty);

// ---- temporal blocking of the tile form (air_fused.cu) ----------------------------
// k ticks as A(t0), then k - 1 launches of B(t) + A(t + 1) over FUSED_TX x
// FUSED_TY tiles (each staged as one TMA box of (FUSED_TX + 16) x (FUSED_TY +
// 10) cells: its own tensor maps), then B(t0 + k - 1) with the k - 1 deferred
// emap decays.
constexpr int FUSED_TX = 32, FUSED_TY = 16;
int fused_tile_prepare(int *occupancy);
// B(t) + A(t + 1) of every instance: tick t reads parity `parity` of `insts`
// (two per instance, as the tile form's), `emap_lag` emap decays are pending.
int launch_fused_ba(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles,
                    uint32_t grid, uint32_t parity, uint32_t emap_lag, cudaStream_t st);
int read_fused_errors(uint32_t *out);

// ---- the sweep form (air_sweep.cu) ----------------------------------------------
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
