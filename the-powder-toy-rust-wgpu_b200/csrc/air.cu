// air.cu -- launches of the air step (single grid and batched instances).
// Compiled with -fmad=false: see air.cuh.
#include <algorithm>
#include <mutex>

#include "air.cuh"
#include "air_launch.hpp"

namespace tpt {
namespace air {

// Tile of a batched launch: instance index and tile origin in cells.
__device__ __forceinline__ void tile_of(const TileRef *tiles, uint32_t t, uint32_t &inst, int &x0, int &y0) {
    TileRef r = tiles[t];
    inst = r.inst;
    x0 = (int)r.tx * TX;
    y0 = (int)r.ty * TY;
}

// ---- single grid: one CTA per tile, the instance by value -----------------
__global__ void __launch_bounds__(NT) k_pressure_velocity(const AirInst I) {
    __shared__ SmemA S;
    tile_pressure_velocity(I, blockIdx.x * TX, blockIdx.y * TY, S);
}

__global__ void __launch_bounds__(NT) k_advect_heat(const AirInst I) {
    __shared__ SmemB S;
    tile_advect_heat(I, blockIdx.x * TX, blockIdx.y * TY, S);
}

// Settle pass: new heat -> hv, NoUpdate convection -> vx/vy, wall masks
// (settle.rs:50-93) and the optional HotAir pass (settle.rs:118-161).
__global__ void k_settle(const AirInst I, const uint32_t *__restrict__ pmap, const uint32_t *__restrict__ props,
                         uint32_t nprops, uint32_t xres, uint32_t yres) {
    const size_t n = (size_t)I.X * I.Y;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        if (I.aheat) {
            I.hv[g] = I.hv_out[g];
            if (I.air_mode == 4u) {
                I.vx[g] = I.ovx[g];
                I.vy[g] = I.ovy[g];
            }
        }
        uint32_t ba, bh;
        masks_cell(I, g, ba, bh);
        I.bair_out[g] = ba;
        I.bairh_out[g] = bh;
        if (pmap != nullptr) {
            const uint32_t cx = (uint32_t)(g % I.X), cy = (uint32_t)(g / I.X);
            float pv = I.pv[g];
            bool touched = false;
            for (uint32_t dy = 0; dy < 4; ++dy)
                for (uint32_t dx = 0; dx < 4; ++dx) {
                    uint32_t px = cx * 4 + dx, py = cy * 4 + dy;
                    if (px >= xres || py >= yres) continue;
                    uint32_t e = __ldg(pmap + (size_t)py * xres + px);
                    if (e == 0u) continue;
                    uint32_t ty = e & 0x1FFu;
                    if (ty >= nprops) continue;  // guard: no row for this id
                    float hot = __uint_as_float(__ldg(props + (size_t)ty * 32 + 11));
                    if (hot == 0.0f) continue;
                    touched = true;
                    if (ty == 10u || ty == 97u) {  // PT_GAS / PT_NBLE
                        if (pv < 3.5f) pv += 4.0f * hot * (3.5f - pv);
                    } else {
                        pv += 4.0f * hot;
                    }
                }
            if (touched) I.pv[g] = pv;
        }
    }
}

int launch_single(const AirInst &I, const uint32_t *pmap, const uint32_t *props, uint32_t nprops, uint32_t xres,
                  uint32_t yres, cudaStream_t st) {
    dim3 grid((I.X + TX - 1) / TX, (I.Y + TY - 1) / TY);
    if (I.air_mode != 4u) {
        k_pressure_velocity<<<grid, NT, 0, st>>>(I);
        TPT_LAUNCHED();
    }
    if (I.air_mode != 4u || I.aheat) {
        k_advect_heat<<<grid, NT, 0, st>>>(I);
        TPT_LAUNCHED();
    }
    size_t n = (size_t)I.X * I.Y;
    unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
    k_settle<<<blocks, 256, 0, st>>>(I, pmap, props, nprops, xres, yres);
    TPT_LAUNCHED();
    return TPT_OK;
}

// ---- batched instances: persistent CTAs over a tile list ------------------
__global__ void __launch_bounds__(NT) kb_pressure_velocity(const AirInst *__restrict__ insts,
                                                           const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                           uint32_t parity) {
    __shared__ SmemA S;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        AirInst I = insts[2 * i + parity];
        if (I.air_mode == 4u) continue;
        tile_pressure_velocity(I, x0, y0, S);
        __syncthreads();
    }
}

// The batched B pass also rebuilds the masks of its tile into the other
// half of the mask ping-pong (read by the next tick), so a tick is two
// launches. The heat result goes to the other half of the hv ping-pong.
__global__ void __launch_bounds__(NT) kb_advect_heat(const AirInst *__restrict__ insts,
                                                     const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                     uint32_t parity) {
    __shared__ SmemB S;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst I = insts[2 * i + parity];
        if (I.air_mode != 4u || I.aheat) tile_advect_heat(I, x0, y0, S);
        const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
        if (in_grid(gx, gy, I)) {
            size_t g = (size_t)gy * I.X + gx;
            uint32_t ba, bh;
            masks_cell(I, g, ba, bh);
            I.bair_out[g] = ba;
            I.bairh_out[g] = bh;
            if (!I.aheat && I.hv_out != I.hv) I.hv_out[g] = I.hv[g];
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
            size_t g = (size_t)gy * I.X + gx;
            I.vx[g] = I.ovx[g];
            I.vy[g] = I.ovy[g];
        }
    }
}

int launch_batch_tick(const AirInst *insts, const TileRef *tiles, uint32_t ntiles, uint32_t grid, uint32_t parity,
                      bool any_noupdate_heat, cudaStream_t st) {
    kb_pressure_velocity<<<grid, NT, 0, st>>>(insts, tiles, ntiles, parity);
    TPT_LAUNCHED();
    kb_advect_heat<<<grid, NT, 0, st>>>(insts, tiles, ntiles, parity);
    TPT_LAUNCHED();
    if (any_noupdate_heat) {
        kb_noupdate_settle<<<grid, NT, 0, st>>>(insts, tiles, ntiles, parity);
        TPT_LAUNCHED();
    }
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
            size_t g = (size_t)gy * C.X + gx;
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

// ---- air step with library-owned scratch (no allocation) ------------------
// The step needs four grids of scratch (new pressure, the two new velocity
// components and the new heat). tpt_air_step takes them from the caller;
// this variant takes them from one array that lives in the library's device
// image, so a call allocates nothing. Every device that loads the library
// holds the array (4 MiB) until the process exits.
static __device__ __align__(256) float g_static_scratch[4 * (size_t)TPT_STATIC_SCRATCH_MAX_CELLS];

// Device address of g_static_scratch on the current device. The name is a
// host-side stand-in in host code, so the address is looked up once per
// device with that device current, and cached.
static int static_scratch(float **out) {
    static std::mutex mu;
    static float *cache[128] = {};
    int dev = 0;
    TPT_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) TPT_FAIL(TPT_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || p == nullptr)
            TPT_FAIL(TPT_ERR_CUDA, "cudaGetSymbolAddress(static scratch) failed on device %d: %s", dev,
                     cudaGetErrorString(e));
        cache[dev] = static_cast<float *>(p);
    }
    *out = cache[dev];
    return TPT_OK;
}

}  // namespace air
}  // namespace tpt

extern "C" int tpt_air_step_static_scratch(const tpt_air_params *params, const tpt_air_bufs *b,
                                           tpt_stream_t stream) {
    using namespace tpt;
    if (!params || !b) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_air_step_static_scratch: params or bufs is NULL");
    const tpt_air_params &p = *params;
    if (p.air_mode > 4u || p.convection_mode > 2u || p.gravity_mode > 3u || p.aheat_enable > 1u)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_air_step_static_scratch: enum field out of range");
    if (p.xcells == 0 || p.ycells == 0) return TPT_OK;
    const size_t n = (size_t)p.xcells * p.ycells;
    if (p.xcells > TPT_MAX_CELLS_PER_SIDE || p.ycells > TPT_MAX_CELLS_PER_SIDE || n > TPT_STATIC_SCRATCH_MAX_CELLS)
        TPT_FAIL(TPT_ERR_INVALID_DIMS,
                 "tpt_air_step_static_scratch: grid %ux%u = %zu cells exceeds the static scratch of %u cells "
                 "(use tpt_air_step with caller-owned scratch)",
                 p.xcells, p.ycells, n, (unsigned)TPT_STATIC_SCRATCH_MAX_CELLS);
    if (!b->pv || !b->vx || !b->vy || !b->hv || !b->block_air || !b->block_airh || !b->wall_bmap || !b->wall_emap ||
        !b->fan_vx || !b->fan_vy)
        TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_air_step_static_scratch: a required grid pointer is NULL");
    if (b->pmap && (!b->elem_props || b->xres == 0 || b->yres == 0))
        TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_air_step_static_scratch: pmap given without elem_props / xres / yres");
    int rc = require_sm100();
    if (rc) return rc;
    float *s = nullptr;
    rc = air::static_scratch(&s);
    if (rc) return rc;
    // Every scratch cell the step reads is written earlier in the same step,
    // so nothing has to be cleared between calls.
    AirInst I = make_air_inst(p);
    I.pv = b->pv;
    I.vx = b->vx;
    I.vy = b->vy;
    I.hv = b->hv;
    I.opv = s;
    I.ovx = s + n;
    I.ovy = s + 2 * n;
    I.ohv = s + 3 * n;
    I.bair = b->block_air;
    I.bairh = b->block_airh;
    I.wall = b->wall_bmap;
    I.emap = b->wall_emap;
    I.eair = b->elem_block_air;
    I.eairh = b->elem_block_airh;
    I.fvx = b->fan_vx;
    I.fvy = b->fan_vy;
    I.bair_out = b->block_air;
    I.bairh_out = b->block_airh;
    I.hv_out = I.ohv;
    return air::launch_single(I, b->pmap, b->elem_props, b->n_elements, b->xres, b->yres, (cudaStream_t)stream);
}
