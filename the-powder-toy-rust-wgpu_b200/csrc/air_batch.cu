// air_batch.cu -- the batch's velocity pre-pass and copy-back.
//
// The pre-pass runs the velocity pass (pressure.rs:173-299) of the instances
// whose previous tick sampled velocity outside the sweep's rings
// (air_sweep.cu), writing their ovx/ovy scratch grids so the sweep reads those
// samples from memory. Persistent CTAs walk the tile list of every instance;
// each flagged tile's halo region is staged by TMA (one 2-D box per grid,
// zero-filled outside the grid), double-buffered so the next tile's loads are
// in flight while the current tile computes. The batch's grids have a
// 128-byte-aligned row pitch, which TMA needs. Compiled with -fmad=false: see
// air.cuh.
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

// Stages pv, vx, vy and block_air of the tile (the `parity` halves).
__device__ __forceinline__ void issue_a(const CUtensorMap *m, uint32_t parity, int x0, int y0, BoxA *buf,
                                        uint64_t *bar) {
    tc::mbar_arrive_expect_tx(bar, 4 * BOX_BYTES);
    load_box(buf->pv, m + TM_PV0 + parity, x0, y0, bar);
    load_box(buf->vx, m + TM_VX0 + parity, x0, y0, bar);
    load_box(buf->vy, m + TM_VY0 + parity, x0, y0, bar);
    load_box(buf->b, m + TM_BA0 + parity, x0, y0, bar);
}

// The pre-pass of one tick. Also clears the flags the sweep of this tick
// sets (the other parity's) and resets the sweep's work-queue counter, so a
// tick is this launch and the sweep, with no memset. `flags` are this
// parity's: tiles of instances whose flag is 0 are skipped, so a tick with no
// flagged instance costs one short launch.
__global__ void __launch_bounds__(NT) kb_sweep_prepass(const AirInst *__restrict__ insts,
                                                      const CUtensorMap *__restrict__ tmaps,
                                                      const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                      uint32_t parity, uint32_t ninst, uint32_t *__restrict__ ctl,
                                                      uint32_t *__restrict__ want) {
    __shared__ BoxA buf[2];
    __shared__ float opv[Box::N];
    __shared__ uint64_t full[2];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) ctl[0] = 0u;
    for (uint32_t i = tid; i < ninst; i += gridDim.x * blockDim.x) want[(size_t)(parity ^ 1u) * ninst + i] = 0u;
    const uint32_t *flags = want + (size_t)parity * ninst;
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
        if (flags[i] == 0u) return false;
        issue_a(tmaps + (size_t)i * TM_COUNT, parity, x0, y0, &buf[k], &full[k]);
        return true;
    };
    if (threadIdx.x == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);
    int k = 0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, k ^= 1) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const uint32_t tn = t + gridDim.x;
        bool next_issued = false;  // thread 0: a bulk copy into buf[k ^ 1] is in flight
        if (threadIdx.x == 0 && tn < ntiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            next_issued = issue(tn, k ^ 1);
        }
        if (flags[i] == 0u) continue;
        const AirInst I = insts[2 * i + parity];
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

int launch_prepass(const SweepLaunch &s, uint32_t parity, cudaStream_t st) {
    kb_sweep_prepass<<<s.prepass_grid, NT, 0, st>>>(s.insts, s.tmaps, s.tiles, s.ntiles, parity, s.ninst, s.ctl,
                                                    s.want);
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
