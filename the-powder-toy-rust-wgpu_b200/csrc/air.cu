// air.cu -- the one-grid air step (tpt_air_step and its static-scratch
// variant). Compiled with -fmad=false: see air.cuh.
#include <algorithm>

#include "air.cuh"
#include "air_launch.hpp"

namespace tpt {
namespace air {

// Pass A of one tile, staged by plain loads (the caller's grids may have any
// row length, so no TMA).
__global__ void __launch_bounds__(NT) k_pressure_velocity(const AirInst I) {
    __shared__ LayoutA1 S;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    stage_flag<3>(S.b, I.bair, 0xFFFFFFFFu, I, x0, y0);
    stage<float, 2>(S.vx, I.vx, I, x0, y0);
    stage<float, 2>(S.vy, I.vy, I, x0, y0);
    stage<float, 1>(S.pv, I.pv, I, x0, y0);
    __syncthreads();
    pass_a(I, x0, y0, S);
}

// Pass B of one tile.
__global__ void __launch_bounds__(NT) k_advect_heat(const AirInst I) {
    __shared__ LayoutB1 S;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    if (I.air_mode != 4u) {
        stage_flag<3>(S.b, I.bair, 0xFFFFFFFFu, I, x0, y0);
        stage<float, 3>(S.ovx, I.ovx, I, x0, y0);
        stage<float, 3>(S.ovy, I.ovy, I, x0, y0);
        stage<float, 2>(S.opv, I.opv, I, x0, y0);
    } else {
        stage<float, 1>(S.nvx, I.vx, I, x0, y0);
        stage<float, 1>(S.nvy, I.vy, I, x0, y0);
    }
    if (I.aheat) {
        stage_flag<1>(S.bh, I.bairh, 0x8u, I, x0, y0);
        stage<float, 1>(S.hv, I.hv, I, x0, y0);
    }
    __syncthreads();
    pass_b(I, x0, y0, S);
}

// Settle pass: new heat -> hv, NoUpdate convection -> vx/vy, wall masks
// (settle.rs:50-93) and the optional HotAir pass (settle.rs:118-161). The
// grid is dense here (pitch == X).
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

// ---- air step with library-owned scratch (no allocation) ------------------
// The step needs four grids of scratch (new pressure, the two new velocity
// components and the new heat). tpt_air_step takes them from the caller;
// this variant takes them from one array that lives in the library's device
// image, so a call allocates nothing. Every device that loads the library
// holds the array (4 MiB) until the process exits.
static __device__ __align__(256) float g_static_scratch[4 * (size_t)TPT_STATIC_SCRATCH_MAX_CELLS];

// Device address of g_static_scratch in the current device's context. The
// name is a host-side stand-in in host code, so the address is looked up
// with the device current. It is looked up on every call rather than cached:
// the lookup allocates nothing, and a cached address would go stale when the
// context is torn down and recreated (cudaDeviceReset, or a primary-context
// reset through the driver API), leaving kernels to write through a pointer
// of the old context.
static int static_scratch(float **out) {
    int dev = 0;
    TPT_CUDA(cudaGetDevice(&dev));
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr)
        TPT_FAIL(TPT_ERR_CUDA, "cudaGetSymbolAddress(static scratch) failed on device %d: %s", dev,
                 cudaGetErrorString(e));
    *out = static_cast<float *>(p);
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
