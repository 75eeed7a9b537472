// air_tiles.cu -- the batch's air tick in the tile form, for one tile shape.
//
// The Makefile compiles this file once per shape the form offers (32x8,
// 64x8, 32x16, 64x16 cells), with AIR_TILE_X / AIR_TILE_Y / AIR_SHAPE_NS
// set, so each shape has its own kernels, tile size and namespace.
//
// Persistent CTAs (one thread per tile cell) walk a tile list covering every
// instance; each tile's halo region is staged by TMA (one 2-D box per grid:
// the tile plus 4 cells on each side in x, 3 in y, zero-filled outside the
// grid), double-buffered so the next tile's loads are in flight while the
// current tile computes. The batch's grids have a 128-byte-aligned row pitch,
// which TMA needs, and every tile starts at a multiple of 32 columns, so the
// box's first column (x0 - 4) is 16-byte aligned. A tick is two launches:
// pass A (pressure, velocity) writes opv/ovx/ovy; pass B (smoothing,
// advection, vorticity, fans, heat, convection, masks) reads them and
// updates pv/vx/vy in place, with heat and the masks in ping-pong halves.
// Compiled with -fmad=false: see air.cuh.
#include <cuda.h>

#include "air.cuh"
#include "air_launch.hpp"
#include "tc.cuh"

namespace tpt {
namespace air {
inline namespace AIR_SHAPE_NS {

static_assert(TX % 32 == 0 && TX + 2 * Box::HX <= 256 && TY + 2 * Box::HY <= 256, "tile shape");
static_assert(NT <= 1024, "one thread per tile cell");

__device__ uint32_t g_tile_err;

__device__ __forceinline__ void tile_of(const TileRef *tiles, uint32_t t, uint32_t &inst, int &x0, int &y0) {
    TileRef r = tiles[t];
    inst = r.inst;
    x0 = (int)r.tx * TX;
    y0 = (int)r.ty * TY;
}

// Box load of grid `m` for the tile at (x0, y0): origin (x0 - 4, y0 - 3).
__device__ __forceinline__ void load_box(void *dst, const CUtensorMap *m, int x0, int y0, uint64_t *bar) {
    tc::tma_load_2d(dst, m, x0 - Box::HX, y0 - Box::HY, bar);
}

constexpr uint32_t BOX_BYTES = Box::N * 4;

// Dynamic shared memory of the two passes.
constexpr size_t SMEM_A = 2 * sizeof(BoxA) + Box::N * sizeof(float);
constexpr size_t SMEM_B = 2 * sizeof(BoxB) + sizeof(WorkB2);
// Resident CTAs per SM that pass B's register cap is sized for: 48 warps.
constexpr int B_MIN_CTAS = 1536 / NT > 0 ? 1536 / NT : 1;

// The dynamic shared memory, 128-byte aligned (TMA destinations). Used by
// casts of the symbol itself, so the compiler keeps shared-memory addressing
// for every access through it.
extern __shared__ __align__(128) uint8_t air_tile_smem[];

// Error exit of a CTA whose wait on full[k] timed out. Thread 0 may still have
// bulk copies in flight that write this CTA's shared memory and complete on
// its mbarriers: the one the failed wait was for, and the prefetch of the next
// tile into the other buffer (issued before the wait). A CTA must not exit
// with those outstanding, so thread 0 waits for both phases again (each wait
// bounded, recording ERR_WAIT_TIMEOUT if it gives up) before every thread
// returns. `uses` is the phase word after the failed wait was accounted for.
__device__ __forceinline__ void drain_on_timeout(uint64_t *full, int k, uint32_t uses, bool next_issued) {
    if (threadIdx.x == 0) {
        tc::mbar_wait(&full[k], ((uses >> k) & 1u) ^ 1u, &g_tile_err);
        if (next_issued) tc::mbar_wait(&full[k ^ 1], (uses >> (k ^ 1)) & 1u, &g_tile_err);
    }
    __syncthreads();
}

// ---- pass A -------------------------------------------------------------------
// Which grids pass A stages for an instance (0 = none: NoUpdate).
__device__ __forceinline__ uint32_t a_loads(const AirInst &I) { return I.air_mode == 4u ? 0u : 4u; }

__device__ __forceinline__ void issue_a(const AirInst &I, const CUtensorMap *m, uint32_t parity, int x0, int y0,
                                        BoxA *buf, uint64_t *bar) {
    tc::mbar_arrive_expect_tx(bar, 4 * BOX_BYTES);
    load_box(buf->pv, m + TM_PV, x0, y0, bar);
    load_box(buf->vx, m + TM_VX, x0, y0, bar);
    load_box(buf->vy, m + TM_VY, x0, y0, bar);
    load_box(buf->b, m + TM_BA0 + parity, x0, y0, bar);
}

// The persistent CTAs' tile order: static striding (queue == null: tiles
// blockIdx.x, + gridDim.x, ...) or an atomic work queue (each CTA takes the
// next unclaimed tile; thread 0 claims it and shares it through shared
// memory). Each pass's counter is cleared by the launch before it: pass A
// clears pass B's (`reset`) and pass B clears pass A's.
__device__ __forceinline__ uint32_t first_tile(uint32_t *queue) {
    return queue ? atomicAdd(queue, 1u) : blockIdx.x;
}
__device__ __forceinline__ uint32_t next_tile(uint32_t *queue, uint32_t t) {
    return queue ? atomicAdd(queue, 1u) : t + gridDim.x;
}

__global__ void __launch_bounds__(NT) kb_pressure_velocity(const AirInst *__restrict__ insts,
                                                           const CUtensorMap *__restrict__ tmaps,
                                                           const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                           uint32_t parity, uint32_t *queue, uint32_t *reset) {
    BoxA *buf = reinterpret_cast<BoxA *>(air_tile_smem);
    float *opv = reinterpret_cast<float *>(buf + 2);
    __shared__ uint64_t full[2];
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::fence_mbar_init();
        if (blockIdx.x == 0) *reset = 0u;
        s_tile = first_tile(queue);
    }
    __syncthreads();
    uint32_t uses = 0;  // bit k: phase parity of full[k] (a register, not an indexed array)
    auto issue = [&](uint32_t t, int k) -> bool {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst &I = insts[2 * i + parity];
        if (!a_loads(I)) return false;
        issue_a(I, tmaps + (size_t)i * TM_COUNT, parity, x0, y0, &buf[k], &full[k]);
        return true;
    };
    uint32_t t = s_tile;
    if (threadIdx.x == 0 && t < ntiles) issue(t, 0);
    int k = 0;
    while (t < ntiles) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst I = insts[2 * i + parity];
        uint32_t tn = 0;           // thread 0: the next tile
        bool next_issued = false;  // thread 0: a bulk copy into buf[k ^ 1] is in flight
        if (threadIdx.x == 0) {
            tn = next_tile(queue, t);
            if (tn < ntiles) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                next_issued = issue(tn, k ^ 1);
            }
        }
        const bool loads = a_loads(I) != 0u;
        bool ok = true;
        if (loads) {
            ok = tc::mbar_wait(&full[k], (uses >> k) & 1u, &g_tile_err);
            uses ^= 1u << k;
        }
        // every thread has read s_tile for this tile before thread 0 overwrites it
        if (!__syncthreads_and(ok)) {
            drain_on_timeout(full, k, uses, next_issued);
            return;
        }
        if (threadIdx.x == 0) s_tile = tn;
        if (loads) {
            LayoutA2 S{&buf[k], opv};
            pass_a(I, x0, y0, S);
        }
        __syncthreads();
        t = s_tile;
        k ^= 1;
    }
}

// ---- pass B -------------------------------------------------------------------
__device__ __forceinline__ uint32_t b_loads(const AirInst &I) {
    if (I.air_mode != 4u) return I.aheat ? 6u : 4u;
    return I.aheat ? 4u : 0u;
}

__device__ __forceinline__ void issue_b(const AirInst &I, const CUtensorMap *m, uint32_t parity, int x0, int y0,
                                        BoxB *buf, uint64_t *bar) {
    const uint32_t n = b_loads(I);
    tc::mbar_arrive_expect_tx(bar, n * BOX_BYTES);
    if (I.air_mode != 4u) {
        const CUtensorMap *ov = m + TM_OV0 + 3 * parity;  // this tick's velocity-pass outputs
        load_box(buf->ovx, ov + 0, x0, y0, bar);
        load_box(buf->ovy, ov + 1, x0, y0, bar);
        load_box(buf->opv, ov + 2, x0, y0, bar);
        load_box(buf->b, m + TM_BA0 + parity, x0, y0, bar);
    } else {  // NoUpdate: the heat pass reads the stored velocity
        load_box(buf->ovx, m + TM_VX, x0, y0, bar);
        load_box(buf->ovy, m + TM_VY, x0, y0, bar);
    }
    if (I.aheat) {
        load_box(buf->hv, m + TM_HV0 + parity, x0, y0, bar);
        load_box(buf->bh, m + TM_BH0 + parity, x0, y0, bar);
    }
}

// Also rebuilds the masks of its tile into the other half of the mask
// ping-pong (read by the next tick) and writes the new heat into the other
// half of the heat ping-pong, so a tick is two launches. The pass is bound
// by issue latency (barriers, shared loads, the IEEE division sequences), so
// its registers are capped for 48 resident warps per SM (40 per thread at
// 256- and 512-thread tiles); shared memory allows no more at 32x8. Measured
// on B200 at 32x8: 6 CTAs 0.47 ms, 4 CTAs 0.52 ms, 3 CTAs (69 registers)
// 0.55 ms per tick of the 6.1 M-cell batch.
__global__ void __launch_bounds__(NT, B_MIN_CTAS) kb_advect_heat(const AirInst *__restrict__ insts,
                                                              const CUtensorMap *__restrict__ tmaps,
                                                              const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                              uint32_t parity, uint32_t emap_lag, uint32_t *queue,
                                                              uint32_t *reset) {
    BoxB *buf = reinterpret_cast<BoxB *>(air_tile_smem);
    WorkB2 *work = reinterpret_cast<WorkB2 *>(buf + 2);
    __shared__ uint64_t full[2];
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::fence_mbar_init();
        if (blockIdx.x == 0) *reset = 0u;
        s_tile = first_tile(queue);
    }
    __syncthreads();
    uint32_t uses = 0;  // bit k: phase parity of full[k] (a register, not an indexed array)
    auto issue = [&](uint32_t t, int k) -> bool {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst &I = insts[2 * i + parity];
        if (!b_loads(I)) return false;
        issue_b(I, tmaps + (size_t)i * TM_COUNT, parity, x0, y0, &buf[k], &full[k]);
        return true;
    };
    uint32_t t = s_tile;
    if (threadIdx.x == 0 && t < ntiles) issue(t, 0);
    int k = 0;
    while (t < ntiles) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst I = insts[2 * i + parity];
        uint32_t tn = 0;           // thread 0: the next tile
        bool next_issued = false;  // thread 0: a bulk copy into buf[k ^ 1] is in flight
        if (threadIdx.x == 0) {
            tn = next_tile(queue, t);
            if (tn < ntiles) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                next_issued = issue(tn, k ^ 1);
            }
        }
        const bool loads = b_loads(I) != 0u;
        bool ok = true;
        if (loads) {
            ok = tc::mbar_wait(&full[k], (uses >> k) & 1u, &g_tile_err);
            uses ^= 1u << k;
        }
        // every thread has read s_tile for this tile before thread 0 overwrites it
        if (!__syncthreads_and(ok)) {
            drain_on_timeout(full, k, uses, next_issued);
            return;
        }
        if (threadIdx.x == 0) s_tile = tn;
        if (loads) {
            LayoutB2 S{&buf[k], work};
            if (I.air_mode == 4u) {  // stored velocity of the +1 ring for the heat pass
                for_ring<1>(I, x0, y0, [&](int gx, int gy) {
                    S.NVX(gx, gy, x0, y0) = S.OVX(gx, gy, x0, y0);
                    S.NVY(gx, gy, x0, y0) = S.OVY(gx, gy, x0, y0);
                });
                __syncthreads();
            }
            pass_b(I, x0, y0, S);
        }
        const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
        if (in_grid(gx, gy, I)) {
            size_t g = (size_t)gy * I.pitch + gx;
            uint32_t ba, bh;
            masks_cell(I, g, ba, bh, emap_lag);
            I.bair_out[g] = ba;
            I.bairh_out[g] = bh;
        }
        __syncthreads();
        t = s_tile;
        k ^= 1;
    }
}

// NoUpdate + ambient heat writes its convected velocity to ovx/ovy; a batch
// with such an instance copies it back after the B pass.
__global__ void kb_noupdate_settle(const AirInst *__restrict__ insts, const TileRef *__restrict__ tiles,
                                   uint32_t ntiles, uint32_t parity) {
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst I = insts[2 * i + parity];
        if (!(I.air_mode == 4u && I.aheat)) continue;
        const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
        if (in_grid(gx, gy, I)) {
            size_t g = (size_t)gy * I.pitch + gx;
            I.vx[g] = I.ovx[g];
            I.vy[g] = I.ovy[g];
        }
    }
}

}  // namespace AIR_SHAPE_NS

// ---- host side of this shape ------------------------------------------------------
namespace {
int tile_prepare(int *occupancy_a, int *occupancy_b) {
    using namespace AIR_SHAPE_NS;
    TPT_CUDA(cudaFuncSetAttribute(kb_pressure_velocity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_A));
    TPT_CUDA(cudaFuncSetAttribute(kb_advect_heat, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_B));
    // the passes keep their working set in shared memory: all of the SM's
    // unified L1 / shared storage as shared memory
    TPT_CUDA(cudaFuncSetAttribute(kb_pressure_velocity, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    TPT_CUDA(cudaFuncSetAttribute(kb_advect_heat, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    TPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy_a, kb_pressure_velocity, NT, SMEM_A));
    TPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy_b, kb_advect_heat, NT, SMEM_B));
    return TPT_OK;
}

int tile_launch_a(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles, uint32_t grid,
                  uint32_t parity, uint32_t *queues, bool use_queue, cudaStream_t st) {
    using namespace AIR_SHAPE_NS;
    kb_pressure_velocity<<<grid, NT, SMEM_A, st>>>(insts, tmaps, tiles, ntiles, parity, use_queue ? queues : nullptr,
                                                   queues + 1);
    TPT_LAUNCHED();
    return TPT_OK;
}

int tile_launch_settle(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, uint32_t parity,
                       cudaStream_t st) {
    using namespace AIR_SHAPE_NS;
    kb_noupdate_settle<<<grid, NT, 0, st>>>(insts, tiles, ntiles, parity);
    TPT_LAUNCHED();
    return TPT_OK;
}

int tile_launch_b(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles, uint32_t grid,
                  uint32_t parity, uint32_t emap_lag, bool any_noupdate_heat, uint32_t *queues, bool use_queue,
                  cudaStream_t st) {
    using namespace AIR_SHAPE_NS;
    kb_advect_heat<<<grid, NT, SMEM_B, st>>>(insts, tmaps, tiles, ntiles, parity, emap_lag,
                                             use_queue ? queues + 1 : nullptr, queues);
    TPT_LAUNCHED();
    return any_noupdate_heat ? tile_launch_settle(insts, tiles, ntiles, grid, parity, st) : TPT_OK;
}

int tile_read_errors(uint32_t *out) {
    using namespace AIR_SHAPE_NS;
    uint32_t v = 0, z = 0;
    TPT_CUDA(cudaMemcpyFromSymbol(&v, g_tile_err, sizeof(v)));
    TPT_CUDA(cudaMemcpyToSymbol(g_tile_err, &z, sizeof(z)));
    *out = v;
    return TPT_OK;
}
}  // namespace

// This shape's entry in the tile form's table (air_launch.hpp): tile_shape_<ns>.
#define AIR_CAT2(a, b) a##b
#define AIR_CAT(a, b) AIR_CAT2(a, b)
extern const TileShape AIR_CAT(tile_shape_, AIR_SHAPE_NS) = {(uint32_t)AIR_SHAPE_NS::TX, (uint32_t)AIR_SHAPE_NS::TY,
                                                            tile_prepare, tile_launch_a, tile_launch_b,
                                                            tile_launch_settle, tile_read_errors};

}  // namespace air
}  // namespace tpt
