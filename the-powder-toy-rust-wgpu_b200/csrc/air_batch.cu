// air_batch.cu -- the air tick of batched instances: the tile form, the
// sweep form's velocity pre-pass, and the copy-back.
//
// Tile form: persistent CTAs walk a tile list covering every instance; each
// tile's halo region is staged by TMA (one 2-D box per grid, zero-filled
// outside the grid), double-buffered so the next tile's loads are in flight
// while the current tile computes. The batch's grids have a 128-byte-aligned
// row pitch, which TMA needs. A tick is two launches: pass A (pressure,
// velocity) writes opv/ovx/ovy; pass B (smoothing, advection, vorticity,
// fans, heat, convection, masks) reads them and updates pv/vx/vy in place,
// with heat and the masks in ping-pong halves.
//
// Sweep form's pre-pass: the velocity pass of the instances whose previous
// tick sampled velocity outside the sweep's rings (air_sweep.cu), writing
// their ovx/ovy scratch grids so the sweep reads those samples from memory.
// Compiled with -fmad=false: see air.cuh.
#include <cuda.h>

#include "air.cuh"
#include "air_launch.hpp"
#include "tc.cuh"

namespace tpt {
namespace air {

__device__ uint32_t g_air_err;

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

// Error exit of a CTA whose wait on full[k] timed out. Thread 0 may still have
// bulk copies in flight that write this CTA's shared memory and complete on
// its mbarriers: the one the failed wait was for, and the prefetch of the next
// tile into the other buffer (issued before the wait). A CTA must not exit
// with those outstanding, so thread 0 waits for both phases again (each wait
// bounded, recording ERR_WAIT_TIMEOUT if it gives up) before every thread
// returns. `uses` is the phase word after the failed wait was accounted for.
__device__ __forceinline__ void drain_on_timeout(uint64_t *full, int k, uint32_t uses, bool next_issued) {
    if (threadIdx.x == 0) {
        tc::mbar_wait(&full[k], ((uses >> k) & 1u) ^ 1u, &g_air_err);
        if (next_issued) tc::mbar_wait(&full[k ^ 1], (uses >> (k ^ 1)) & 1u, &g_air_err);
    }
    __syncthreads();
}

// ---- the tile form: pass A ------------------------------------------------------
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

__global__ void __launch_bounds__(NT) kb_pressure_velocity(const AirInst *__restrict__ insts,
                                                           const CUtensorMap *__restrict__ tmaps,
                                                           const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                           uint32_t parity) {
    __shared__ BoxA buf[2];
    __shared__ float opv[Box::N];
    __shared__ uint64_t full[2];
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::fence_mbar_init();
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
    if (threadIdx.x == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);
    int k = 0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, k ^= 1) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst I = insts[2 * i + parity];
        const uint32_t tn = t + gridDim.x;
        bool next_issued = false;  // thread 0: a bulk copy into buf[k ^ 1] is in flight
        if (threadIdx.x == 0 && tn < ntiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            next_issued = issue(tn, k ^ 1);
        }
        if (!a_loads(I)) continue;
        bool ok = tc::mbar_wait(&full[k], (uses >> k) & 1u, &g_air_err);
        uses ^= 1u << k;
        if (!__syncthreads_and(ok)) {
            drain_on_timeout(full, k, uses, next_issued);
            return;
        }
        LayoutA2 S{&buf[k], opv};
        pass_a(I, x0, y0, S);
        __syncthreads();
    }
}

// ---- the tile form: pass B ------------------------------------------------------
__device__ __forceinline__ uint32_t b_loads(const AirInst &I) {
    if (I.air_mode != 4u) return I.aheat ? 6u : 4u;
    return I.aheat ? 4u : 0u;
}

__device__ __forceinline__ void issue_b(const AirInst &I, const CUtensorMap *m, uint32_t parity, int x0, int y0,
                                        BoxB *buf, uint64_t *bar) {
    const uint32_t n = b_loads(I);
    tc::mbar_arrive_expect_tx(bar, n * BOX_BYTES);
    if (I.air_mode != 4u) {
        load_box(buf->ovx, m + TM_OVX, x0, y0, bar);
        load_box(buf->ovy, m + TM_OVY, x0, y0, bar);
        load_box(buf->opv, m + TM_OPV, x0, y0, bar);
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
// registers are capped at 40 to keep six CTAs (48 warps) resident; shared
// memory allows no more. Measured on B200: 6 CTAs 0.47 ms, 4 CTAs 0.52 ms,
// 3 CTAs (69 registers) 0.55 ms per tick of the 6.1 M-cell batch.
__global__ void __launch_bounds__(NT, 6) kb_advect_heat(const AirInst *__restrict__ insts,
                                                     const CUtensorMap *__restrict__ tmaps,
                                                     const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                     uint32_t parity) {
    __shared__ BoxB buf[2];
    __shared__ WorkB2 work;
    __shared__ uint64_t full[2];
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::fence_mbar_init();
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
    if (threadIdx.x == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);
    int k = 0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, k ^= 1) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst I = insts[2 * i + parity];
        const uint32_t tn = t + gridDim.x;
        bool next_issued = false;  // thread 0: a bulk copy into buf[k ^ 1] is in flight
        if (threadIdx.x == 0 && tn < ntiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            next_issued = issue(tn, k ^ 1);
        }
        if (b_loads(I)) {
            bool ok = tc::mbar_wait(&full[k], (uses >> k) & 1u, &g_air_err);
            uses ^= 1u << k;
            if (!__syncthreads_and(ok)) {
                drain_on_timeout(full, k, uses, next_issued);
                return;
            }
            LayoutB2 S{&buf[k], &work};
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
            masks_cell(I, g, ba, bh);
            I.bair_out[g] = ba;
            I.bairh_out[g] = bh;
        }
        __syncthreads();
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

int launch_tile_tick(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles,
                      uint32_t grid, uint32_t parity, bool any_noupdate_heat, cudaStream_t st) {
    kb_pressure_velocity<<<grid, NT, 0, st>>>(insts, tmaps, tiles, ntiles, parity);
    TPT_LAUNCHED();
    kb_advect_heat<<<grid, NT, 0, st>>>(insts, tmaps, tiles, ntiles, parity);
    TPT_LAUNCHED();
    if (any_noupdate_heat) {
        kb_noupdate_settle<<<grid, NT, 0, st>>>(insts, tiles, ntiles, parity);
        TPT_LAUNCHED();
    }
    return TPT_OK;
}

// The pre-pass of one tick. Also clears the flags the sweep of this tick
// sets (the other parity's) and resets the sweep's work-queue counter, so a
// tick is this launch and the sweep, with no memset. `flags` are this
// parity's: tiles of instances whose flag is 0 are skipped, so a tick with no
// flagged instance costs one short launch. A flagged tile stages block_air
// with a 3-cell halo, vx/vy with 2 and pv with 1 by plain loads (zero outside
// the grid) and runs the velocity pass on them.
__global__ void __launch_bounds__(NT) kb_sweep_prepass(const AirInst *__restrict__ insts,
                                                      const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                      uint32_t parity, uint32_t ninst, uint32_t *__restrict__ ctl,
                                                      uint32_t *__restrict__ want) {
    __shared__ LayoutA1 S;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) ctl[0] = 0u;
    for (uint32_t i = tid; i < ninst; i += gridDim.x * blockDim.x) want[(size_t)(parity ^ 1u) * ninst + i] = 0u;
    const uint32_t *flags = want + (size_t)parity * ninst;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        if (flags[i] == 0u) continue;  // the same for every thread of the CTA
        const AirInst I = insts[2 * i + parity];
        stage_flag<3>(S.b, I.bair, 0xFFFFFFFFu, I, x0, y0);
        stage<float, 2>(S.vx, I.vx, I, x0, y0);
        stage<float, 2>(S.vy, I.vy, I, x0, y0);
        stage<float, 1>(S.pv, I.pv, I, x0, y0);
        __syncthreads();
        pass_a(I, x0, y0, S);
        __syncthreads();
    }
}

int launch_prepass(const SweepLaunch &s, uint32_t parity, cudaStream_t st) {
    kb_sweep_prepass<<<s.prepass_grid, NT, 0, st>>>(s.insts, s.tiles, s.ntiles, parity, s.ninst, s.ctl, s.want);
    TPT_LAUNCHED();
    return TPT_OK;
}

// Copies the ping-pong halves that hold the newest state back to the
// instance's canonical buffers (after an odd number of ticks).
__global__ void kb_copy_back(const AirInst *__restrict__ insts, const TileRef *__restrict__ tiles, uint32_t ntiles) {
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst C = insts[2 * i + 0];  // parity 0 reads canonical
        const AirInst O = insts[2 * i + 1];  // parity 1 reads the other half
        const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
        if (in_grid(gx, gy, C)) {
            size_t g = (size_t)gy * C.pitch + gx;
            C.pv[g] = O.pv[g];
            C.vx[g] = O.vx[g];
            C.vy[g] = O.vy[g];
            C.hv[g] = O.hv[g];
            C.bair[g] = O.bair[g];
            C.bairh[g] = O.bairh[g];
        }
    }
}

int launch_copy_back(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, cudaStream_t st) {
    kb_copy_back<<<grid, NT, 0, st>>>(insts, tiles, ntiles);
    TPT_LAUNCHED();
    return TPT_OK;
}

int read_errors(uint32_t *out) {
    uint32_t v = 0, z = 0;
    TPT_CUDA(cudaMemcpyFromSymbol(&v, g_air_err, sizeof(v)));
    TPT_CUDA(cudaMemcpyToSymbol(g_air_err, &z, sizeof(z)));
    *out = v;
    return TPT_OK;
}

}  // namespace air
}  // namespace tpt
