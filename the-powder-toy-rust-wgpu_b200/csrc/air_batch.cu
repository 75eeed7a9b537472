// air_batch.cu -- the batched air tick's shared pieces: the sweep form's
// velocity pre-pass, the copy-back, and the table of the tile form's shapes
// (their kernels are in air_tiles.cu).
//
// Sweep form's pre-pass: the velocity pass of the instances whose previous
// tick sampled velocity outside the sweep's rings (air_sweep.cu), writing
// their ovx/ovy scratch grids so the sweep reads those samples from memory.
// Compiled with -fmad=false: see air.cuh.
#include <cuda.h>

#include "air.cuh"
#include "air_launch.hpp"

namespace tpt {
namespace air {

__device__ __forceinline__ void tile_of(const TileRef *tiles, uint32_t t, uint32_t &inst, int &x0, int &y0) {
    TileRef r = tiles[t];
    inst = r.inst;
    x0 = (int)r.tx * TX;
    y0 = (int)r.ty * TY;
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

const TileShape *const *tile_shapes() {
    static const TileShape *const all[TILE_SHAPES] = {&tile_shape_s32x8, &tile_shape_s64x8, &tile_shape_s32x16,
                                                      &tile_shape_s64x16};
    return all;
}

const TileShape *tile_shape(uint32_t tx, uint32_t ty) {
    for (int k = 0; k < TILE_SHAPES; ++k)
        if (tile_shapes()[k]->tx == tx && tile_shapes()[k]->ty == ty) return tile_shapes()[k];
    return nullptr;
}

// The batched air kernels' error words: the tile form's, one per shape, and
// the temporally blocked launches' (the sweep form and the pre-pass have no
// waits).
int read_errors(uint32_t *out) {
    uint32_t all = 0;
    int frc = read_fused_errors(&all);
    if (frc) return frc;
    for (int k = 0; k < TILE_SHAPES; ++k) {
        uint32_t v = 0;
        int rc = tile_shapes()[k]->read_errors(&v);
        if (rc) return rc;
        all |= v;
    }
    *out = all;
    return TPT_OK;
}

}  // namespace air
}  // namespace tpt
