// air.cuh -- device code of the Eulerian air step (one tile of one instance).
//
// The arithmetic restates the reference kernels operation by operation
// (crates/tpt-sim/src/air_kernel/pressure.rs, advect.rs, heat.rs, settle.rs)
// and the files that include it are compiled with -fmad=false, so every f32
// operation is rounded separately exactly as in the reference's source: the
// FP32 results are bit-identical to the CPU restatement of those kernels.
//
// The seven reference launches become two tile passes and a settle pass:
//
//   A  pressure + velocity   (pressure.rs:173-299): effective velocities on
//      the tile's +2 ring, pressure on the +1 ring, velocity on the tile.
//      Needs block_air with a 3-cell halo, vx/vy with 2, pv with 1.
//   B  smooth/advect/vorticity/fans (advect.rs:174-360) on the tile's +1
//      ring (vorticity precomputed on the +2 ring), then ambient heat and
//      convection (heat.rs:31-253) on the tile. Needs ovx/ovy and block_air
//      with a 3-cell halo, opv with 2, hv and block_airh with 1. The
//      far-advection walks and bilinear samples read global memory.
//   S  settle: heat copy-back (settle.rs:21-27), wall masks (settle.rs:
//      50-93) and HotAir (settle.rs:118-161), elementwise.
//
// The one global dependency of a tick is between A and B: the far-advection
// sample can reach any cell of ovx/ovy (0.7*|v| <= 179 cells).
//
// The tile code is written once over a shared-memory layout policy `L`:
// the single-grid kernels and the sweep form's velocity pre-pass stage each
// array with its own halo (Reg<H>); the batch's tile form stages every array
// as one TMA box of the tile plus a 4-cell (x) by 3-cell (y) halo. The
// batch's sweep form (air_sweep.cu) reuses the per-cell helpers below.
//
// The tile is AIR_TX x AIR_TY (32 x 8) cells, one thread per cell, unless the
// including file defines AIR_TILE_X / AIR_TILE_Y: the batch's tile form is
// compiled once per tile shape it offers (air_tiles.cu), each copy in its own
// namespace AIR_SHAPE_NS.
#pragma once

#include "common.cuh"
#include "exact_div.cuh"

#ifndef AIR_TILE_X
#define AIR_TILE_X AIR_TX
#define AIR_TILE_Y AIR_TY
#define AIR_SHAPE_NS s32x8
#endif

namespace tpt {
namespace air {
inline namespace AIR_SHAPE_NS {

constexpr int TX = AIR_TILE_X, TY = AIR_TILE_Y, NT = TX * TY;

// Tile plus an H-cell halo on every side.
template <int H> struct Reg {
    static constexpr int W = TX + 2 * H;
    static constexpr int HGT = TY + 2 * H;
    static constexpr int N = W * HGT;
    __device__ static __forceinline__ int at(int gx, int gy, int x0, int y0) {
        return (gy - y0 + H) * W + (gx - x0 + H);
    }
};

// The TMA box of the batched kernels: x halo 4 (keeps the box start 16-byte
// aligned), y halo 3.
struct Box {
    static constexpr int HX = 4, HY = 3, W = TX + 2 * HX, HGT = TY + 2 * HY, N = W * HGT;
    static constexpr int NP = (N + 31) / 32 * 32;  // array stride: TMA destinations are 128-byte aligned
    __device__ static __forceinline__ int at(int gx, int gy, int x0, int y0) {
        return (gy - y0 + HY) * W + (gx - x0 + HX);
    }
};

__device__ __forceinline__ bool in_grid(int x, int y, const AirInst &I) {
    return x >= 0 && y >= 0 && x < (int)I.X && y < (int)I.Y;
}

// pressure.rs:9-15
__device__ __forceinline__ bool in_border(uint32_t x, uint32_t y, uint32_t X, uint32_t Y) {
    return x < 2u || y < 2u || x + 2u >= X || y + 2u >= Y;
}
// pressure.rs:20-26
__device__ __forceinline__ bool interior(uint32_t x, uint32_t y, uint32_t X, uint32_t Y) {
    return x >= 1u && y >= 1u && x + 1u < X && y + 1u < Y;
}

// mod.rs:92-102 (compare and assign; keeps NaN and -0 as the reference does).
__device__ __forceinline__ float clampf(float v, float lo, float hi) {
    float out = v;
    if (out < lo) out = lo;
    if (out > hi) out = hi;
    return out;
}

// Smoothing weight of tap (dx, dy) (advect.rs:215-225).
__device__ __forceinline__ float smooth_w(int dx, int dy) {
    float w = 0.01831564f;
    if (dx == 1) w = 0.13533528f;
    if (dy == 1) w = 0.13533528f;
    if (dx == 1 && dy == 1) w = 1.0f;
    return w;
}

// ---- shared-memory layouts ---------------------------------------------------
// Pass A working set. `vx`/`vy` hold the raw velocity, then the effective
// velocity; `pv` the raw pressure; `opv` the new pressure.
struct LayoutA1 {  // single grid: per-array halos, masks as flags
    uint8_t b[Reg<3>::N];
    float vx[Reg<2>::N], vy[Reg<2>::N];
    float pv[Reg<1>::N], opv[Reg<1>::N];
    __device__ __forceinline__ bool blk(int x, int y, int x0, int y0) const { return b[Reg<3>::at(x, y, x0, y0)] != 0; }
    __device__ __forceinline__ float &VX(int x, int y, int x0, int y0) { return vx[Reg<2>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &VY(int x, int y, int x0, int y0) { return vy[Reg<2>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float PV(int x, int y, int x0, int y0) const { return pv[Reg<1>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &OPV(int x, int y, int x0, int y0) { return opv[Reg<1>::at(x, y, x0, y0)]; }
};

struct __align__(128) BoxA {  // batched: one TMA box per array
    float pv[Box::NP];
    float vx[Box::NP];
    float vy[Box::NP];
    uint32_t b[Box::NP];
};
struct LayoutA2 {
    BoxA *in;
    float *opv;  // Box::N
    __device__ __forceinline__ bool blk(int x, int y, int x0, int y0) const { return in->b[Box::at(x, y, x0, y0)] != 0u; }
    __device__ __forceinline__ float &VX(int x, int y, int x0, int y0) { return in->vx[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &VY(int x, int y, int x0, int y0) { return in->vy[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float PV(int x, int y, int x0, int y0) const { return in->pv[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &OPV(int x, int y, int x0, int y0) { return opv[Box::at(x, y, x0, y0)]; }
};

// Pass B working set: staged ovx/ovy/opv/hv, the two masks, and the
// computed vorticity (+2 ring) and smoothed/advected velocity and pressure
// (+1 ring).
struct LayoutB1 {
    uint8_t b[Reg<3>::N];
    uint8_t bh[Reg<1>::N];
    float ovx[Reg<3>::N], ovy[Reg<3>::N];
    float opv[Reg<2>::N];
    float hv[Reg<1>::N];
    float vort[Reg<2>::N];
    float nvx[Reg<1>::N], nvy[Reg<1>::N], npv[Reg<1>::N];
    // staged regions: b/ovx/ovy cover the +3 ring, bh/hv the +1 ring
    __device__ __forceinline__ static bool has3(int x, int y, int x0, int y0) {
        return x >= x0 - 3 && x < x0 + TX + 3 && y >= y0 - 3 && y < y0 + TY + 3;
    }
    __device__ __forceinline__ static bool hasH(int x, int y, int x0, int y0) {
        return x >= x0 - 1 && x < x0 + TX + 1 && y >= y0 - 1 && y < y0 + TY + 1;
    }
    __device__ __forceinline__ bool blk(int x, int y, int x0, int y0) const { return b[Reg<3>::at(x, y, x0, y0)] != 0; }
    __device__ __forceinline__ bool hblk(int x, int y, int x0, int y0) const { return bh[Reg<1>::at(x, y, x0, y0)] != 0; }
    __device__ __forceinline__ float OVX(int x, int y, int x0, int y0) const { return ovx[Reg<3>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float OVY(int x, int y, int x0, int y0) const { return ovy[Reg<3>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float OPV(int x, int y, int x0, int y0) const { return opv[Reg<2>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float HV(int x, int y, int x0, int y0) const { return hv[Reg<1>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &VORT(int x, int y, int x0, int y0) { return vort[Reg<2>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NVX(int x, int y, int x0, int y0) { return nvx[Reg<1>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NVY(int x, int y, int x0, int y0) { return nvy[Reg<1>::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NPV(int x, int y, int x0, int y0) { return npv[Reg<1>::at(x, y, x0, y0)]; }
};

struct __align__(128) BoxB {  // batched: one TMA box per array
    float ovx[Box::NP];  // ovx (or vx when the pressure/velocity pass is off)
    float ovy[Box::NP];
    float opv[Box::NP];
    float hv[Box::NP];
    uint32_t b[Box::NP];
    uint32_t bh[Box::NP];
};
struct WorkB2 {
    float vort[Box::N], nvx[Box::N], nvy[Box::N], npv[Box::N];
};
struct LayoutB2 {
    BoxB *in;
    WorkB2 *w;
    // every staged grid covers the whole box
    __device__ __forceinline__ static bool has3(int x, int y, int x0, int y0) {
        return x >= x0 - Box::HX && x < x0 + TX + Box::HX && y >= y0 - Box::HY && y < y0 + TY + Box::HY;
    }
    __device__ __forceinline__ static bool hasH(int x, int y, int x0, int y0) { return has3(x, y, x0, y0); }
    __device__ __forceinline__ bool blk(int x, int y, int x0, int y0) const { return in->b[Box::at(x, y, x0, y0)] != 0u; }
    __device__ __forceinline__ bool hblk(int x, int y, int x0, int y0) const {
        return (in->bh[Box::at(x, y, x0, y0)] & 0x8u) != 0u;
    }
    __device__ __forceinline__ float OVX(int x, int y, int x0, int y0) const { return in->ovx[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float OVY(int x, int y, int x0, int y0) const { return in->ovy[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float OPV(int x, int y, int x0, int y0) const { return in->opv[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float HV(int x, int y, int x0, int y0) const { return in->hv[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &VORT(int x, int y, int x0, int y0) { return w->vort[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NVX(int x, int y, int x0, int y0) { return w->nvx[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NVY(int x, int y, int x0, int y0) { return w->nvy[Box::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NPV(int x, int y, int x0, int y0) { return w->npv[Box::at(x, y, x0, y0)]; }
};

// ---- staging by loads (single-grid path) -------------------------------------
template <typename T, int H>
__device__ __forceinline__ void stage(T *s, const T *g, const AirInst &I, int x0, int y0) {
    for (int i = threadIdx.x; i < Reg<H>::N; i += NT) {
        int ly = i / Reg<H>::W, lx = i - ly * Reg<H>::W;
        int gx = x0 - H + lx, gy = y0 - H + ly;
        s[i] = in_grid(gx, gy, I) ? __ldg(g + (size_t)gy * I.pitch + gx) : T(0);
    }
}
template <int H>
__device__ __forceinline__ void stage_flag(uint8_t *s, const uint32_t *g, uint32_t bitmask, const AirInst &I, int x0,
                                           int y0) {
    for (int i = threadIdx.x; i < Reg<H>::N; i += NT) {
        int ly = i / Reg<H>::W, lx = i - ly * Reg<H>::W;
        int gx = x0 - H + lx, gy = y0 - H + ly;
        s[i] = in_grid(gx, gy, I) ? ((__ldg(g + (size_t)gy * I.pitch + gx) & bitmask) != 0u) : 0;
    }
}

// Calls f(gx, gy) for every in-grid cell of the tile's +R ring (R = 0: the
// tile), spread over the block's threads.
template <int R, typename F>
__device__ __forceinline__ void for_ring(const AirInst &I, int x0, int y0, F &&f) {
    constexpr int W = TX + 2 * R, N = W * (TY + 2 * R);
    for (int i = threadIdx.x; i < N; i += NT) {
        int ly = i / W, lx = i - ly * W;
        int gx = x0 - R + lx, gy = y0 - R + ly;
        if (in_grid(gx, gy, I)) f(gx, gy);
    }
}

// ---- pass A ------------------------------------------------------------------
// pressure.rs:43-85: the three-cell wall velocity clear.
template <class L>
__device__ __forceinline__ bool wall_cleared_vx(const L &S, uint32_t x, uint32_t y, uint32_t X, uint32_t Y, int x0, int y0) {
    bool out = false;
    if (y >= 1u && y + 1u < Y) {
        if (x >= 1u && x + 1u < X && S.blk(x, y, x0, y0)) out = true;
        if (x >= 2u && S.blk((int)x - 1, y, x0, y0)) out = true;
        if (x + 2u < X && S.blk((int)x + 1, y, x0, y0)) out = true;
    }
    return out;
}
template <class L>
__device__ __forceinline__ bool wall_cleared_vy(const L &S, uint32_t x, uint32_t y, uint32_t X, uint32_t Y, int x0, int y0) {
    bool out = false;
    if (x >= 1u && x + 1u < X) {
        if (y >= 1u && y + 1u < Y && S.blk(x, y, x0, y0)) out = true;
        if (y >= 2u && S.blk(x, (int)y - 1, x0, y0)) out = true;
        if (y + 2u < Y && S.blk(x, (int)y + 1, x0, y0)) out = true;
    }
    return out;
}

// The compute of pass A once the tile is staged in S. Writes opv, ovx, ovy.
template <class L> __device__ __forceinline__ void pass_a(const AirInst &I, int x0, int y0, L &S) {
    const uint32_t X = I.X, Y = I.Y;
    // effective_vx/vy (pressure.rs:119-157) on the +2 ring, in place; this
    // is also the velocity pass's pre-gradient value (pressure.rs:265-276).
    // Every thread reads only its own cells' velocities, so no barrier is
    // needed between the reads and the in-place writes.
    for_ring<2>(I, x0, y0, [&](int gx, int gy) {
        float vx = S.VX(gx, gy, x0, y0), vy = S.VY(gx, gy, x0, y0);
        if (in_border(gx, gy, X, Y)) {
            vx = I.evx + (vx - I.evx) * 0.9f;
            vy = I.evy + (vy - I.evy) * 0.9f;
        }
        if (wall_cleared_vx(S, gx, gy, X, Y, x0, y0)) vx = 0.0f;
        if (wall_cleared_vy(S, gx, gy, X, Y, x0, y0)) vy = 0.0f;
        S.VX(gx, gy, x0, y0) = vx;
        S.VY(gx, gy, x0, y0) = vy;
    });
    __syncthreads();
    // air_pressure_kernel (pressure.rs:186-237) on the +1 ring.
    for_ring<1>(I, x0, y0, [&](int gx, int gy) {
        float cur = S.PV(gx, gy, x0, y0);
        if (in_border(gx, gy, X, Y)) cur = I.ep + (cur - I.ep) * 0.8f;
        float next = cur;
        if (interior(gx, gy, X, Y)) {
            float dp = S.VX(gx - 1, gy, x0, y0) - S.VX(gx + 1, gy, x0, y0) + S.VY(gx, gy - 1, x0, y0) -
                       S.VY(gx, gy + 1, x0, y0);
            next = I.ep + (cur - I.ep) * 0.9999f + dp * 0.15f;
        }
        S.OPV(gx, gy, x0, y0) = next;
    });
    __syncthreads();
    // air_velocity_kernel (pressure.rs:260-298) on the tile.
    const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
    if (in_grid(gx, gy, I)) {
        float nx = S.VX(gx, gy, x0, y0), ny = S.VY(gx, gy, x0, y0);
        if (interior(gx, gy, X, Y)) {
            float dx = S.OPV(gx - 1, gy, x0, y0) - S.OPV(gx + 1, gy, x0, y0);
            float dy = S.OPV(gx, gy - 1, x0, y0) - S.OPV(gx, gy + 1, x0, y0);
            nx = I.evx + (nx - I.evx) * 0.999f + dx * 0.2f;
            ny = I.evy + (ny - I.evy) * 0.999f + dy * 0.2f;
            // adjacent_blocked_x/y (pressure.rs:92-114)
            if (S.blk(gx - 1, gy, x0, y0) || S.blk(gx, gy, x0, y0) || S.blk(gx + 1, gy, x0, y0)) nx = 0.0f;
            if (S.blk(gx, gy - 1, x0, y0) || S.blk(gx, gy, x0, y0) || S.blk(gx, gy + 1, x0, y0)) ny = 0.0f;
        }
        size_t g = (size_t)gy * I.pitch + gx;
        I.ovx[g] = nx;
        I.ovy[g] = ny;
        I.opv[g] = S.OPV(gx, gy, x0, y0);
    }
}

// ---- pass B ------------------------------------------------------------------
// advect.rs:66-152. `blocked(cx, cy)` is the mask the walk tests for an
// in-grid cell: block_air != 0 (velocity walk) or block_airh & 0x8 (heat
// walk), read from shared memory when the cell is staged.
template <typename B>
__device__ __forceinline__ void far_advect_target(uint32_t x, uint32_t y, float dx, float dy, B &&blocked, uint32_t X,
                                                  uint32_t Y, float &otx, float &oty) {
    float tx = (float)x - dx * 0.7f;
    float ty = (float)y - dy * 0.7f;
    float adx = dx * 0.7f;
    if (adx < 0.0f) adx = 0.0f - adx;
    float ady = dy * 0.7f;
    if (ady < 0.0f) ady = 0.0f - ady;
    float limx = (float)X - 2.0f, limy = (float)Y - 2.0f;
    if ((adx > 1.0f || ady > 1.0f) && tx >= 2.0f && tx < limx && ty >= 2.0f && ty < limy) {
        float abs_dx = dx < 0.0f ? 0.0f - dx : dx;
        float abs_dy = dy < 0.0f ? 0.0f - dy : dy;
        float step_x, step_y;
        int step_limit;
        if (abs_dx > abs_dy) {
            step_x = dx < 0.0f ? 1.0f : -1.0f;
            step_y = 0.0f - dy / abs_dx;
            step_limit = (int)adx;
        } else {
            step_x = 0.0f - dx / abs_dy;
            step_y = dy < 0.0f ? 1.0f : -1.0f;
            step_limit = (int)ady;
        }
        tx = (float)x;
        ty = (float)y;
        bool stopped = false;
        for (int step = 0; step < step_limit; ++step) {
            tx += step_x;
            ty += step_y;
            int cx = (int)(tx + 0.5f);
            int cy = (int)(ty + 0.5f);
            bool hit = true;
            if (cx >= 0 && cy >= 0 && cx < (int)X && cy < (int)Y) hit = blocked(cx, cy);
            if (hit) {
                tx -= step_x;
                ty -= step_y;
                stopped = true;
                break;
            }
        }
        if (!stopped) {
            tx = (float)x - dx * 0.7f;
            ty = (float)y - dy * 0.7f;
        }
    }
    otx = tx;
    oty = ty;
}

// vorticity_bmap (advect.rs:10-42) of cell (x, y) from the staged ovx/ovy.
template <class L>
__device__ __forceinline__ float vorticity_bmap(const L &S, uint32_t x, uint32_t y, uint32_t X, uint32_t Y, int x0, int y0) {
    float out = 0.0f;
    if (x > 1u && x + 2u < X && y > 1u && y + 2u < Y) {
        bool here = S.blk(x, y, x0, y0);
        float dvydx = S.OVY(x + 1, y, x0, y0) - S.OVY(x - 1, y, x0, y0);
        if (here || S.blk(x + 1, y, x0, y0) || S.blk(x - 1, y, x0, y0)) dvydx = 0.0f;
        float dvxdy = S.OVX(x, y + 1, x0, y0) - S.OVX(x, y - 1, x0, y0);
        if (here || S.blk(x, y + 1, x0, y0) || S.blk(x, y - 1, x0, y0)) dvxdy = 0.0f;
        out = (dvydx - dvxdy) * 0.5f;
    }
    return out;
}

// air_smooth_advect_kernel body (advect.rs:192-358) for one cell, with the
// vorticity of the cell and its neighbours taken from S.VORT.
template <class L>
__device__ __forceinline__ void smooth_advect_cell(const AirInst &I, L &S, int x, int y, int x0, int y0, float &out_vx,
                                                   float &out_vy, float &out_pv) {
    const uint32_t X = I.X, Y = I.Y;
    const float cvx = S.OVX(x, y, x0, y0), cvy = S.OVY(x, y, x0, y0), cpv = S.OPV(x, y, x0, y0);
    float sx = 0.0f, sy = 0.0f, sp = 0.0f;
    if ((uint32_t)x >= 2u && (uint32_t)x + 3u <= X && (uint32_t)y >= 2u && (uint32_t)y + 3u <= Y) {
        // every tap is an interior cell: fixed offsets, no saturation
#pragma unroll
        for (int dyy = 0; dyy < 3; ++dyy) {
#pragma unroll
            for (int dxx = 0; dxx < 3; ++dxx) {
                const int nx = x + dxx - 1, ny = y + dyy - 1;
                const float w = smooth_w(dxx, dyy);
                const bool open = !S.blk(nx, ny, x0, y0);
                const float tx = open ? S.OVX(nx, ny, x0, y0) : cvx;
                const float ty = open ? S.OVY(nx, ny, x0, y0) : cvy;
                const float tp = open ? S.OPV(nx, ny, x0, y0) : cpv;
                sx += tx * w;
                sy += ty * w;
                sp += tp * w;
            }
        }
    } else {
#pragma unroll
        for (int dyy = 0; dyy < 3; ++dyy) {
#pragma unroll
            for (int dxx = 0; dxx < 3; ++dxx) {
                uint32_t nx = (uint32_t)x + dxx;
                nx = nx >= 1u ? nx - 1u : 0u;
                uint32_t ny = (uint32_t)y + dyy;
                ny = ny >= 1u ? ny - 1u : 0u;
                float w = smooth_w(dxx, dyy);
                bool itap = nx >= 1u && ny >= 1u && nx + 1u < X && ny + 1u < Y;
                float tx = cvx, ty = cvy, tp = cpv;
                if (itap && !S.blk(nx, ny, x0, y0)) {
                    tx = S.OVX(nx, ny, x0, y0);
                    ty = S.OVY(nx, ny, x0, y0);
                    tp = S.OPV(nx, ny, x0, y0);
                }
                sx += tx * w;
                sy += ty * w;
                sp += tp * w;
            }
        }
    }
    // / wsum: every tap adds its weight, so the sum is the constant kSmoothWsum
    float nvx = div_by_const(sx, kSmoothWsum, kSmoothWsumRcp), nvy = div_by_const(sy, kSmoothWsum, kSmoothWsumRcp),
          npv = div_by_const(sp, kSmoothWsum, kSmoothWsumRcp);

    float tx0, ty0;
    far_advect_target(
        x, y, nvx, nvy,
        [&](int cx, int cy) -> bool {
            if (S.has3(cx, cy, x0, y0)) return S.blk(cx, cy, x0, y0);
            return __ldg(I.bair + (size_t)cy * I.pitch + cx) != 0u;
        },
        X, Y, tx0, ty0);
    int i0 = (int)tx0, j0 = (int)ty0;
    float fx = tx0 - (float)i0, fy = ty0 - (float)j0;
    if (!S.blk(x, y, x0, y0) && i0 >= 2 && i0 < (int)X - 3 && j0 >= 2 && j0 < (int)Y - 3 && fx >= 0.0f && fy >= 0.0f) {
        float w00 = (1.0f - fx) * (1.0f - fy);
        float w10 = fx * (1.0f - fy);
        float w01 = (1.0f - fx) * fy;
        float w11 = fx * fy;
        float a00, a10, a01, a11, b00, b10, b01, b11;
        if (S.has3(i0, j0, x0, y0) && S.has3(i0 + 1, j0 + 1, x0, y0)) {  // sample inside the staged box
            a00 = S.OVX(i0, j0, x0, y0);
            a10 = S.OVX(i0 + 1, j0, x0, y0);
            a01 = S.OVX(i0, j0 + 1, x0, y0);
            a11 = S.OVX(i0 + 1, j0 + 1, x0, y0);
            b00 = S.OVY(i0, j0, x0, y0);
            b10 = S.OVY(i0 + 1, j0, x0, y0);
            b01 = S.OVY(i0, j0 + 1, x0, y0);
            b11 = S.OVY(i0 + 1, j0 + 1, x0, y0);
        } else {
            size_t r0 = (size_t)j0 * I.pitch + i0, r1 = r0 + I.pitch;
            a00 = __ldg(I.ovx + r0);
            a10 = __ldg(I.ovx + r0 + 1);
            a01 = __ldg(I.ovx + r1);
            a11 = __ldg(I.ovx + r1 + 1);
            b00 = __ldg(I.ovy + r0);
            b10 = __ldg(I.ovy + r0 + 1);
            b01 = __ldg(I.ovy + r1);
            b11 = __ldg(I.ovy + r1 + 1);
        }
        nvx = nvx * 0.7f + 0.3f * (a00 * w00 + a10 * w10 + a01 * w01 + a11 * w11);
        nvy = nvy * 0.7f + 0.3f * (b00 * w00 + b10 * w10 + b01 * w01 + b11 * w11);
    }
    // advect.rs:297-328
    if (I.vcoef > 0.0f && (uint32_t)x > 1u && (uint32_t)x + 2u < X && (uint32_t)y > 1u && (uint32_t)y + 2u < Y) {
        float w = S.VORT(x, y, x0, y0);
        float wxp = S.VORT(x + 1, y, x0, y0);
        float wxm = S.VORT(x - 1, y, x0, y0);
        float wyp = S.VORT(x, y + 1, x0, y0);
        float wym = S.VORT(x, y - 1, x0, y0);
        if (wxp < 0.0f) wxp = 0.0f - wxp;
        if (wxm < 0.0f) wxm = 0.0f - wxm;
        if (wyp < 0.0f) wyp = 0.0f - wyp;
        if (wym < 0.0f) wym = 0.0f - wym;
        float dwx = (wxp - wxm) * 0.5f;
        float dwy = (wyp - wym) * 0.5f;
        float norm = sqrtf(dwx * dwx + dwy * dwy);
        float k = I.vk;
        nvx += k * dwy / (norm + 0.001f) * w;
        nvy += k * (0.0f - dwx) / (norm + 0.001f) * w;
    }
    size_t g = (size_t)y * I.pitch + x;
    if (__ldg(I.wall + g) == 5u) {  // WL_FAN, advect.rs:331-334
        nvx += __ldg(I.fvx + g);
        nvy += __ldg(I.fvy + g);
    }
    nvx = clampf(nvx, -256.0f, 256.0f);
    nvy = clampf(nvy, -256.0f, 256.0f);
    npv = clampf(npv, -256.0f, 256.0f);
    if (I.air_mode == 1u) npv = 0.0f;
    if (I.air_mode == 2u) { nvx = 0.0f; nvy = 0.0f; }
    if (I.air_mode == 3u) { nvx = 0.0f; nvy = 0.0f; npv = 0.0f; }
    out_vx = nvx;
    out_vy = nvy;
    out_pv = npv;
}

// air_heat_convect_kernel (heat.rs:46-251) for one tile cell; vx/vy of the
// cell and its neighbours come from S.NVX/NVY (read-before-write
// semantics). Returns the new heat; updates v in place.
template <class L>
__device__ __forceinline__ float heat_cell(const AirInst &I, L &S, int x, int y, int x0, int y0, float &vx_io,
                                           float &vy_io) {
    const uint32_t X = I.X, Y = I.Y;
    const float ch = S.HV(x, y, x0, y0), cvx = S.NVX(x, y, x0, y0), cvy = S.NVY(x, y, x0, y0);
    float sh = 0.0f, sx = 0.0f, sy = 0.0f;
    if ((uint32_t)x >= 2u && (uint32_t)x + 3u <= X && (uint32_t)y >= 2u && (uint32_t)y + 3u <= Y) {
        // every tap is an interior cell: fixed offsets, no saturation
#pragma unroll
        for (int dyy = 0; dyy < 3; ++dyy) {
#pragma unroll
            for (int dxx = 0; dxx < 3; ++dxx) {
                const int nx = x + dxx - 1, ny = y + dyy - 1;
                const float w = smooth_w(dxx, dyy);
                const bool open = !S.hblk(nx, ny, x0, y0);
                const float th = open ? S.HV(nx, ny, x0, y0) : ch;
                const float tx = open ? S.NVX(nx, ny, x0, y0) : cvx;
                const float ty = open ? S.NVY(nx, ny, x0, y0) : cvy;
                sh += th * w;
                sx += tx * w;
                sy += ty * w;
            }
        }
    } else {
#pragma unroll
        for (int dyy = 0; dyy < 3; ++dyy) {
#pragma unroll
            for (int dxx = 0; dxx < 3; ++dxx) {
                uint32_t nx = (uint32_t)x + dxx;
                nx = nx >= 1u ? nx - 1u : 0u;
                uint32_t ny = (uint32_t)y + dyy;
                ny = ny >= 1u ? ny - 1u : 0u;
                float w = smooth_w(dxx, dyy);
                bool itap = nx >= 1u && ny >= 1u && nx + 1u < X && ny + 1u < Y;
                float th = ch, tx = cvx, ty = cvy;
                if (itap && !S.hblk(nx, ny, x0, y0)) {
                    th = S.HV(nx, ny, x0, y0);
                    tx = S.NVX(nx, ny, x0, y0);
                    ty = S.NVY(nx, ny, x0, y0);
                }
                sh += th * w;
                sx += tx * w;
                sy += ty * w;
            }
        }
    }
    float dh = div_by_const(sh, kSmoothWsum, kSmoothWsumRcp);
    float svx = div_by_const(sx, kSmoothWsum, kSmoothWsumRcp), svy = div_by_const(sy, kSmoothWsum, kSmoothWsumRcp);
    float tx, ty;
    far_advect_target(
        x, y, svx, svy,
        [&](int cx, int cy) -> bool {
            if (S.hasH(cx, cy, x0, y0)) return S.hblk(cx, cy, x0, y0);
            return (__ldg(I.bairh + (size_t)cy * I.pitch + cx) & 0x8u) != 0u;
        },
        X, Y, tx, ty);
    int i0 = (int)tx, j0 = (int)ty;
    float fx = tx - (float)i0, fy = ty - (float)j0;
    const bool here_blocked = S.hblk(x, y, x0, y0);
    if (!here_blocked && i0 >= 0 && i0 < (int)X - 1 && j0 >= 0 && j0 < (int)Y - 1 && fx >= 0.0f && fy >= 0.0f) {
        float s00, s10, s01, s11;
        if (S.hasH(i0, j0, x0, y0) && S.hasH(i0 + 1, j0 + 1, x0, y0)) {  // sample inside the staged box
            s00 = S.hblk(i0, j0, x0, y0) ? dh : S.HV(i0, j0, x0, y0);
            s10 = S.hblk(i0 + 1, j0, x0, y0) ? dh : S.HV(i0 + 1, j0, x0, y0);
            s01 = S.hblk(i0, j0 + 1, x0, y0) ? dh : S.HV(i0, j0 + 1, x0, y0);
            s11 = S.hblk(i0 + 1, j0 + 1, x0, y0) ? dh : S.HV(i0 + 1, j0 + 1, x0, y0);
        } else {
            size_t r0 = (size_t)j0 * I.pitch + i0, r1 = r0 + I.pitch;
            s00 = (__ldg(I.bairh + r0) & 0x8u) ? dh : __ldg(I.hv + r0);
            s10 = (__ldg(I.bairh + r0 + 1) & 0x8u) ? dh : __ldg(I.hv + r0 + 1);
            s01 = (__ldg(I.bairh + r1) & 0x8u) ? dh : __ldg(I.hv + r1);
            s11 = (__ldg(I.bairh + r1 + 1) & 0x8u) ? dh : __ldg(I.hv + r1 + 1);
        }
        float w00 = (1.0f - fx) * (1.0f - fy);
        float w10 = fx * (1.0f - fy);
        float w01 = (1.0f - fx) * fy;
        float w11 = fx * fy;
        dh = dh * 0.7f + 0.3f * (s00 * w00 + s10 * w10 + s01 * w01 + s11 * w11);
    }
    if (here_blocked) dh = ch;
    dh = clampf(dh, 0.0f, 9999.0f);
    if ((uint32_t)x < 2u || (uint32_t)y < 2u || (uint32_t)x + 2u >= X || (uint32_t)y + 2u >= Y) dh = I.amb;
    if (I.aheat == 0u) dh = I.amb;

    float ovx = cvx, ovy = cvy;
    if ((uint32_t)x >= 2u && (uint32_t)x + 2u < X && (uint32_t)y >= 2u && (uint32_t)y + 2u < Y) {
        float gxv = 0.0f, gyv = 0.0f;
        if (I.gmode == 0u) {
            gyv = 1.0f;
        } else if (I.gmode == 2u) {
            float rx = (float)X * 0.5f - ((float)x + 0.5f);
            float ry = (float)Y * 0.5f - ((float)y + 0.5f);
            float rd = sqrtf(rx * rx + ry * ry);
            if (rd > 0.0f) {
                gxv = rx / rd;
                gyv = ry / rd;
            }
        } else if (I.gmode == 3u) {
            gxv = I.cgx;
            gyv = I.cgy;
        }
        float convx = 0.0f - gxv, convy = 0.0f - gyv;
        float nx = cvx, ny = cvy;
        if (I.conv == 1u) {
            float weight = div_by_const((ch - S.HV(x - 1, y, x0, y0)) * convx + (ch - S.HV(x, y - 1, x0, y0)) * convy,
                                        kConvLegacy, kConvLegacyRcp);
            if (weight > 0.0f && !S.hblk(x, y - 1, x0, y0)) {
                nx += weight * convx;
                ny += weight * convy;
            }
        } else if (I.conv == 2u) {
            float gm = sqrtf(convx * convx + convy * convy);
            if (gm > 10.0f) {
                convx /= 0.1f * gm;
                convy /= 0.1f * gm;
            }
            float weight = div_by_const(ch - I.amb, kConvBouss, kConvBoussRcp);
            if (weight > 0.01f) weight = 0.01f;
            nx += weight * convx;
            ny += weight * convy;
        }
        ovx = clampf(nx, -256.0f, 256.0f);
        ovy = clampf(ny, -256.0f, 256.0f);
    }
    vx_io = ovx;
    vy_io = ovy;
    return dh;
}

// The compute of pass B once the tile is staged in S. With air_mode ==
// NoUpdate the smoothing/advection pass is skipped (mod.rs:150) and S.NVX/
// NVY already hold the stored vx/vy (staged by the caller); the convected
// velocity then goes to ovx/ovy (unused scratch in that mode) so that no CTA
// writes a vx/vy cell another CTA may still stage.
template <class L> __device__ __forceinline__ void pass_b(const AirInst &I, int x0, int y0, L &S) {
    const uint32_t X = I.X, Y = I.Y;
    const bool update = I.air_mode != 4u;
    if (update) {
        if (I.vcoef > 0.0f) {
            for_ring<2>(I, x0, y0,
                        [&](int gx, int gy) { S.VORT(gx, gy, x0, y0) = vorticity_bmap(S, gx, gy, X, Y, x0, y0); });
            __syncthreads();
        }
        // the +1 ring outside the tile is needed only as heat-smoothing taps
        if (I.aheat) {
            for_ring<1>(I, x0, y0, [&](int gx, int gy) {
                float a, b, c;
                smooth_advect_cell(I, S, gx, gy, x0, y0, a, b, c);
                S.NVX(gx, gy, x0, y0) = a;
                S.NVY(gx, gy, x0, y0) = b;
                S.NPV(gx, gy, x0, y0) = c;
            });
        } else {
            for_ring<0>(I, x0, y0, [&](int gx, int gy) {
                float a, b, c;
                smooth_advect_cell(I, S, gx, gy, x0, y0, a, b, c);
                S.NVX(gx, gy, x0, y0) = a;
                S.NVY(gx, gy, x0, y0) = b;
                S.NPV(gx, gy, x0, y0) = c;
            });
        }
        __syncthreads();
    }
    const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
    if (!in_grid(gx, gy, I)) return;
    const size_t g = (size_t)gy * I.pitch + gx;
    float vx = S.NVX(gx, gy, x0, y0), vy = S.NVY(gx, gy, x0, y0);
    if (I.aheat) {
        float h = heat_cell(I, S, gx, gy, x0, y0, vx, vy);
        I.hv_out[g] = h;
    }
    if (update) {
        I.vx[g] = vx;
        I.vy[g] = vy;
        I.pv[g] = S.NPV(gx, gy, x0, y0);
    } else if (I.aheat) {
        I.ovx[g] = vx;
        I.ovy[g] = vy;
    }
}

// ---- settle --------------------------------------------------------------------
// settle.rs:50-93 for one cell from its loaded words: wall id, emap before the
// decay, element stamps -> the two masks.
__device__ __forceinline__ void masks_of(uint32_t wall, uint32_t raw, uint32_t eair, uint32_t eairh, uint32_t &bair,
                                        uint32_t &bairh) {
    const uint32_t w = wall & 0xFFu;
    uint32_t e = raw;
    if (raw != 0u) e = raw - 1u;
    e &= 0xFFu;
    uint32_t blocked = (w == 8u || w == 1u || w == 16u || (w == 2u && e == 0u)) ? 1u : 0u;
    bair = blocked | eair;
    uint32_t heat = (blocked != 0u || w == 14u) ? 0x8u : 0u;
    bairh = heat | eairh;
}

// The emap value a tick's mask rebuild sees at cell g when the stored value
// still lacks `lag` decays: inside a temporally blocked run of ticks the
// rebuilds read emap without writing it, and the last one writes it (the
// decay saturates at 0, so `lag` decays subtract lag, down to 0).
__device__ __forceinline__ uint32_t emap_seen(uint32_t stored, uint32_t lag) {
    return stored > lag ? stored - lag : 0u;
}

// The same for cell g of an instance, decaying its emap in place (after the
// `lag` decays it still lacks).
__device__ __forceinline__ void masks_cell(const AirInst &I, size_t g, uint32_t &bair, uint32_t &bairh,
                                           uint32_t lag = 0u) {
    const uint32_t stored = I.emap[g];
    const uint32_t raw = emap_seen(stored, lag);
    const uint32_t next = raw != 0u ? raw - 1u : 0u;
    if (next != stored) I.emap[g] = next;
    masks_of(__ldg(I.wall + g), raw, I.eair ? __ldg(I.eair + g) : 0u, I.eairh ? __ldg(I.eairh + g) : 0u, bair, bairh);
}

}  // namespace AIR_SHAPE_NS
}  // namespace air
}  // namespace tpt
