// air.cuh -- device code of the Eulerian air step (one tile of one instance).
//
// The arithmetic restates the reference kernels operation by operation
// (crates/tpt-sim/src/air_kernel/pressure.rs, advect.rs, heat.rs, settle.rs)
// and this file is compiled with -fmad=false, so every f32 operation is
// rounded separately exactly as in the reference's source: the FP32 results
// are bit-identical to the CPU restatement of those kernels.
//
// The seven reference launches become two tile kernels and a settle pass:
//
//   A  pressure + velocity   (pressure.rs:173-299)
//      tile + 3-cell halo of block_air, + 2 of vx/vy, + 1 of pv staged in
//      shared memory; effective velocities on the +2 ring, pressure on the
//      +1 ring, velocity on the tile. Writes opv/ovx/ovy.
//   B  smooth/advect/vorticity/fans (advect.rs:174-360) on the tile + 1
//      ring, then ambient heat + convection (heat.rs:31-253) on the tile.
//      The far-advection walks and bilinear samples read global memory
//      (read-only in this launch). Writes vx/vy/pv and the new heat.
//   S  settle: heat copy-back (settle.rs:21-27), wall masks (settle.rs:
//      50-93) and HotAir (settle.rs:118-161), elementwise.
//
// The one global dependency of a tick is between A and B: the far-advection
// sample can reach any cell of ovx/ovy (0.7*|v| <= 179 cells).
#pragma once

#include "common.cuh"

namespace tpt {
namespace air {

constexpr int TX = AIR_TX, TY = AIR_TY, NT = TX * TY;

// Shared-memory region of the tile plus an H-cell halo.
template <int H> struct Reg {
    static constexpr int W = TX + 2 * H;
    static constexpr int HGT = TY + 2 * H;
    static constexpr int N = W * HGT;
    // (gx, gy) global -> flat index; caller guarantees it is in the region.
    __device__ static __forceinline__ int at(int gx, int gy, int x0, int y0) {
        return (gy - y0 + H) * W + (gx - x0 + H);
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

// Staged block_air (nonzero test only) with a 3-cell halo; out-of-grid = 0,
// which is what `blocked_at` returns there (pressure.rs:30-36).
struct BlockView {
    const uint8_t *s;
    int x0, y0;
    __device__ __forceinline__ bool at(int x, int y) const { return s[Reg<3>::at(x, y, x0, y0)] != 0; }
};

// pressure.rs:43-62
__device__ __forceinline__ bool wall_cleared_vx(const BlockView &b, uint32_t x, uint32_t y, uint32_t X, uint32_t Y) {
    bool out = false;
    if (y >= 1u && y + 1u < Y) {
        if (x >= 1u && x + 1u < X && b.at(x, y)) out = true;
        if (x >= 2u && b.at((int)x - 1, y)) out = true;
        if (x + 2u < X && b.at((int)x + 1, y)) out = true;
    }
    return out;
}
// pressure.rs:65-85
__device__ __forceinline__ bool wall_cleared_vy(const BlockView &b, uint32_t x, uint32_t y, uint32_t X, uint32_t Y) {
    bool out = false;
    if (x >= 1u && x + 1u < X) {
        if (y >= 1u && y + 1u < Y && b.at(x, y)) out = true;
        if (y >= 2u && b.at(x, (int)y - 1)) out = true;
        if (y + 2u < Y && b.at(x, (int)y + 1)) out = true;
    }
    return out;
}

template <typename T, int H>
__device__ __forceinline__ void stage(T *s, const T *g, const AirInst &I, int x0, int y0) {
    for (int i = threadIdx.x; i < Reg<H>::N; i += NT) {
        int ly = i / Reg<H>::W, lx = i - ly * Reg<H>::W;
        int gx = x0 - H + lx, gy = y0 - H + ly;
        s[i] = in_grid(gx, gy, I) ? __ldg(g + (size_t)gy * I.X + gx) : T(0);
    }
}
template <int H>
__device__ __forceinline__ void stage_flag(uint8_t *s, const uint32_t *g, uint32_t bitmask, const AirInst &I, int x0,
                                           int y0) {
    for (int i = threadIdx.x; i < Reg<H>::N; i += NT) {
        int ly = i / Reg<H>::W, lx = i - ly * Reg<H>::W;
        int gx = x0 - H + lx, gy = y0 - H + ly;
        s[i] = in_grid(gx, gy, I) ? ((__ldg(g + (size_t)gy * I.X + gx) & bitmask) != 0u) : 0;
    }
}

// ---------------------------------------------------------------- A ----
struct SmemA {
    uint8_t b[Reg<3>::N];
    float vx[Reg<2>::N], vy[Reg<2>::N];  // raw, then effective velocity
    float pv[Reg<1>::N];                 // raw, then opv
};

__device__ __forceinline__ void tile_pressure_velocity(const AirInst &I, int x0, int y0, SmemA &S) {
    const uint32_t X = I.X, Y = I.Y;
    stage_flag<3>(S.b, I.bair, 0xFFFFFFFFu, I, x0, y0);
    stage<float, 2>(S.vx, I.vx, I, x0, y0);
    stage<float, 2>(S.vy, I.vy, I, x0, y0);
    stage<float, 1>(S.pv, I.pv, I, x0, y0);
    __syncthreads();
    const BlockView B{S.b, x0, y0};
    // effective_vx/vy (pressure.rs:119-157) on the +2 ring; this is also the
    // velocity pass's pre-gradient value (pressure.rs:265-276).
    for (int i = threadIdx.x; i < Reg<2>::N; i += NT) {
        int ly = i / Reg<2>::W, lx = i - ly * Reg<2>::W;
        int gx = x0 - 2 + lx, gy = y0 - 2 + ly;
        if (!in_grid(gx, gy, I)) continue;
        float vx = S.vx[i], vy = S.vy[i];
        if (in_border(gx, gy, X, Y)) {
            vx = I.evx + (vx - I.evx) * 0.9f;
            vy = I.evy + (vy - I.evy) * 0.9f;
        }
        if (wall_cleared_vx(B, gx, gy, X, Y)) vx = 0.0f;
        if (wall_cleared_vy(B, gx, gy, X, Y)) vy = 0.0f;
        S.vx[i] = vx;
        S.vy[i] = vy;
    }
    __syncthreads();
    // air_pressure_kernel (pressure.rs:186-237) on the +1 ring.
    float opv_ring[2];
    int nring = 0;
    for (int i = threadIdx.x; i < Reg<1>::N; i += NT, ++nring) {
        int ly = i / Reg<1>::W, lx = i - ly * Reg<1>::W;
        int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
        float next = 0.0f;
        if (in_grid(gx, gy, I)) {
            float cur = S.pv[i];
            if (in_border(gx, gy, X, Y)) cur = I.ep + (cur - I.ep) * 0.8f;
            next = cur;
            if (interior(gx, gy, X, Y)) {
                float dp = S.vx[Reg<2>::at(gx - 1, gy, x0, y0)] - S.vx[Reg<2>::at(gx + 1, gy, x0, y0)] +
                           S.vy[Reg<2>::at(gx, gy - 1, x0, y0)] - S.vy[Reg<2>::at(gx, gy + 1, x0, y0)];
                next = I.ep + (cur - I.ep) * 0.9999f + dp * 0.15f;
            }
        }
        opv_ring[nring] = next;
    }
    __syncthreads();
    nring = 0;
    for (int i = threadIdx.x; i < Reg<1>::N; i += NT, ++nring) S.pv[i] = opv_ring[nring];
    __syncthreads();
    // air_velocity_kernel (pressure.rs:260-298) on the tile.
    const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
    if (in_grid(gx, gy, I)) {
        const int c2 = Reg<2>::at(gx, gy, x0, y0);
        float nx = S.vx[c2], ny = S.vy[c2];
        if (interior(gx, gy, X, Y)) {
            float dx = S.pv[Reg<1>::at(gx - 1, gy, x0, y0)] - S.pv[Reg<1>::at(gx + 1, gy, x0, y0)];
            float dy = S.pv[Reg<1>::at(gx, gy - 1, x0, y0)] - S.pv[Reg<1>::at(gx, gy + 1, x0, y0)];
            nx = I.evx + (nx - I.evx) * 0.999f + dx * 0.2f;
            ny = I.evy + (ny - I.evy) * 0.999f + dy * 0.2f;
            // adjacent_blocked_x/y (pressure.rs:92-114)
            if (B.at(gx - 1, gy) || B.at(gx, gy) || B.at(gx + 1, gy)) nx = 0.0f;
            if (B.at(gx, gy - 1) || B.at(gx, gy) || B.at(gx, gy + 1)) ny = 0.0f;
        }
        size_t g = (size_t)gy * X + gx;
        I.ovx[g] = nx;
        I.ovy[g] = ny;
        I.opv[g] = S.pv[Reg<1>::at(gx, gy, x0, y0)];
    }
}

// ---------------------------------------------------------------- B ----
// advect.rs:66-152. `blk` is the mask the walk tests: block_air (heat=false)
// or block_airh & 0x8 (heat=true).
__device__ __forceinline__ void far_advect_target(uint32_t x, uint32_t y, float dx, float dy, const uint32_t *blk,
                                                  uint32_t X, uint32_t Y, bool heat, float &otx, float &oty) {
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
            if (cx >= 0 && cy >= 0 && cx < (int)X && cy < (int)Y) {
                uint32_t v = __ldg(blk + (size_t)cy * X + cx);
                hit = (heat ? (v & 0x8u) : v) != 0u;
            }
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

struct SmemB {
    uint8_t b[Reg<3>::N];               // block_air != 0
    uint8_t bh[Reg<1>::N];              // block_airh & 0x8
    float ovx[Reg<3>::N], ovy[Reg<3>::N];
    float opv[Reg<2>::N];
    float hv[Reg<1>::N];
    float nvx[Reg<1>::N], nvy[Reg<1>::N], npv[Reg<1>::N];
};

// advect.rs:10-42, on staged ovx/ovy (cell and its +-1 neighbours staged).
__device__ __forceinline__ float vorticity_bmap(const SmemB &S, const BlockView &B, uint32_t x, uint32_t y,
                                                uint32_t X, uint32_t Y, int x0, int y0) {
    float out = 0.0f;
    if (x > 1u && x + 2u < X && y > 1u && y + 2u < Y) {
        bool here = B.at(x, y);
        float dvydx = S.ovy[Reg<3>::at(x + 1, y, x0, y0)] - S.ovy[Reg<3>::at(x - 1, y, x0, y0)];
        if (here || B.at(x + 1, y) || B.at(x - 1, y)) dvydx = 0.0f;
        float dvxdy = S.ovx[Reg<3>::at(x, y + 1, x0, y0)] - S.ovx[Reg<3>::at(x, y - 1, x0, y0)];
        if (here || B.at(x, y + 1) || B.at(x, y - 1)) dvxdy = 0.0f;
        out = (dvydx - dvxdy) * 0.5f;
    }
    return out;
}

// air_smooth_advect_kernel body (advect.rs:192-358) for one cell.
__device__ __forceinline__ void smooth_advect_cell(const AirInst &I, const SmemB &S, const BlockView &B, int x,
                                                   int y, int x0, int y0, float &out_vx, float &out_vy,
                                                   float &out_pv) {
    const uint32_t X = I.X, Y = I.Y;
    const int c3 = Reg<3>::at(x, y, x0, y0);
    const float cvx = S.ovx[c3], cvy = S.ovy[c3], cpv = S.opv[Reg<2>::at(x, y, x0, y0)];
    float sx = 0.0f, sy = 0.0f, sp = 0.0f, ws = 0.0f;
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
            if (itap && !B.at(nx, ny)) {
                int n3 = Reg<3>::at(nx, ny, x0, y0);
                tx = S.ovx[n3];
                ty = S.ovy[n3];
                tp = S.opv[Reg<2>::at(nx, ny, x0, y0)];
            }
            sx += tx * w;
            sy += ty * w;
            sp += tp * w;
            ws += w;
        }
    }
    float nvx = sx / ws, nvy = sy / ws, npv = sp / ws;

    float tx0, ty0;
    far_advect_target(x, y, nvx, nvy, I.bair, X, Y, false, tx0, ty0);
    int i0 = (int)tx0, j0 = (int)ty0;
    float fx = tx0 - (float)i0, fy = ty0 - (float)j0;
    if (!B.at(x, y) && i0 >= 2 && i0 < (int)X - 3 && j0 >= 2 && j0 < (int)Y - 3 && fx >= 0.0f && fy >= 0.0f) {
        size_t r0 = (size_t)j0 * X + i0, r1 = r0 + X;
        float w00 = (1.0f - fx) * (1.0f - fy);
        float w10 = fx * (1.0f - fy);
        float w01 = (1.0f - fx) * fy;
        float w11 = fx * fy;
        nvx = nvx * 0.7f + 0.3f * (__ldg(I.ovx + r0) * w00 + __ldg(I.ovx + r0 + 1) * w10 + __ldg(I.ovx + r1) * w01 +
                                   __ldg(I.ovx + r1 + 1) * w11);
        nvy = nvy * 0.7f + 0.3f * (__ldg(I.ovy + r0) * w00 + __ldg(I.ovy + r0 + 1) * w10 + __ldg(I.ovy + r1) * w01 +
                                   __ldg(I.ovy + r1 + 1) * w11);
    }
    // advect.rs:297-328
    if (I.vcoef > 0.0f && (uint32_t)x > 1u && (uint32_t)x + 2u < X && (uint32_t)y > 1u && (uint32_t)y + 2u < Y) {
        float w = vorticity_bmap(S, B, x, y, X, Y, x0, y0);
        float wxp = vorticity_bmap(S, B, x + 1, y, X, Y, x0, y0);
        float wxm = vorticity_bmap(S, B, x - 1, y, X, Y, x0, y0);
        float wyp = vorticity_bmap(S, B, x, y + 1, X, Y, x0, y0);
        float wym = vorticity_bmap(S, B, x, y - 1, X, Y, x0, y0);
        if (wxp < 0.0f) wxp = 0.0f - wxp;
        if (wxm < 0.0f) wxm = 0.0f - wxm;
        if (wyp < 0.0f) wyp = 0.0f - wyp;
        if (wym < 0.0f) wym = 0.0f - wym;
        float dwx = (wxp - wxm) * 0.5f;
        float dwy = (wyp - wym) * 0.5f;
        float norm = sqrtf(dwx * dwx + dwy * dwy);
        float k = I.vcoef / 5.0f;
        nvx += k * dwy / (norm + 0.001f) * w;
        nvy += k * (0.0f - dwx) / (norm + 0.001f) * w;
    }
    size_t g = (size_t)y * X + x;
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
// cell and its neighbours come from the staged smoothing/advection output
// (read-before-write semantics). Returns the new heat; updates v in place.
__device__ __forceinline__ float heat_cell(const AirInst &I, const SmemB &S, int x, int y, int x0, int y0,
                                           float &vx_io, float &vy_io) {
    const uint32_t X = I.X, Y = I.Y;
    const int c1 = Reg<1>::at(x, y, x0, y0);
    const float ch = S.hv[c1], cvx = S.nvx[c1], cvy = S.nvy[c1];
    float sh = 0.0f, sx = 0.0f, sy = 0.0f, ws = 0.0f;
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
            if (itap) {
                int n1 = Reg<1>::at(nx, ny, x0, y0);
                if (!S.bh[n1]) {
                    th = S.hv[n1];
                    tx = S.nvx[n1];
                    ty = S.nvy[n1];
                }
            }
            sh += th * w;
            sx += tx * w;
            sy += ty * w;
            ws += w;
        }
    }
    float dh = sh / ws;
    float svx = sx / ws, svy = sy / ws;
    float tx, ty;
    far_advect_target(x, y, svx, svy, I.bairh, X, Y, true, tx, ty);
    int i0 = (int)tx, j0 = (int)ty;
    float fx = tx - (float)i0, fy = ty - (float)j0;
    const bool here_blocked = S.bh[c1] != 0;
    if (!here_blocked && i0 >= 0 && i0 < (int)X - 1 && j0 >= 0 && j0 < (int)Y - 1 && fx >= 0.0f && fy >= 0.0f) {
        size_t r0 = (size_t)j0 * X + i0, r1 = r0 + X;
        float s00 = (__ldg(I.bairh + r0) & 0x8u) ? dh : __ldg(I.hv + r0);
        float s10 = (__ldg(I.bairh + r0 + 1) & 0x8u) ? dh : __ldg(I.hv + r0 + 1);
        float s01 = (__ldg(I.bairh + r1) & 0x8u) ? dh : __ldg(I.hv + r1);
        float s11 = (__ldg(I.bairh + r1 + 1) & 0x8u) ? dh : __ldg(I.hv + r1 + 1);
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
            float weight = ((ch - S.hv[Reg<1>::at(x - 1, y, x0, y0)]) * convx +
                            (ch - S.hv[Reg<1>::at(x, y - 1, x0, y0)]) * convy) / 5000.0f;
            if (weight > 0.0f && !S.bh[Reg<1>::at(x, y - 1, x0, y0)]) {
                nx += weight * convx;
                ny += weight * convy;
            }
        } else if (I.conv == 2u) {
            float gm = sqrtf(convx * convx + convy * convy);
            if (gm > 10.0f) {
                convx /= 0.1f * gm;
                convy /= 0.1f * gm;
            }
            float weight = (ch - I.amb) / 10000.0f;
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

// Kernel B body. With air_mode == NoUpdate the smoothing/advection pass is
// skipped (mod.rs:150) and the heat pass reads the stored vx/vy; its
// convected velocity then goes to ovx/ovy (unused scratch in that mode) so
// no CTA writes a vx/vy cell another CTA may still stage.
__device__ __forceinline__ void tile_advect_heat(const AirInst &I, int x0, int y0, SmemB &S) {
    const uint32_t X = I.X;
    const bool update = I.air_mode != 4u;
    if (update) {
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
    if (update) {
        const BlockView B{S.b, x0, y0};
        for (int i = threadIdx.x; i < Reg<1>::N; i += NT) {
            int ly = i / Reg<1>::W, lx = i - ly * Reg<1>::W;
            int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
            if (!in_grid(gx, gy, I)) continue;
            // the ring outside the tile is needed only as heat-smoothing taps
            bool need = (lx >= 1 && lx <= TX && ly >= 1 && ly <= TY) || I.aheat;
            if (!need) continue;
            float a, b, c;
            smooth_advect_cell(I, S, B, gx, gy, x0, y0, a, b, c);
            S.nvx[i] = a;
            S.nvy[i] = b;
            S.npv[i] = c;
        }
        __syncthreads();
    }
    const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
    if (!in_grid(gx, gy, I)) return;
    const int c1 = Reg<1>::at(gx, gy, x0, y0);
    const size_t g = (size_t)gy * X + gx;
    float vx = S.nvx[c1], vy = S.nvy[c1];
    if (I.aheat) {
        float h = heat_cell(I, S, gx, gy, x0, y0, vx, vy);
        I.hv_out[g] = h;
    }
    if (update) {
        I.vx[g] = vx;
        I.vy[g] = vy;
        I.pv[g] = S.npv[c1];
    } else if (I.aheat) {
        I.ovx[g] = vx;
        I.ovy[g] = vy;
    }
}

// ---------------------------------------------------------------- S ----
// settle.rs:50-93 for one cell: emap decay and the two masks.
__device__ __forceinline__ void masks_cell(const AirInst &I, size_t g, uint32_t &bair, uint32_t &bairh) {
    uint32_t w = __ldg(I.wall + g) & 0xFFu;
    uint32_t raw = I.emap[g];
    uint32_t e = raw;
    if (raw != 0u) {
        e = raw - 1u;
        I.emap[g] = e;
    }
    e &= 0xFFu;
    uint32_t blocked = (w == 8u || w == 1u || w == 16u || (w == 2u && e == 0u)) ? 1u : 0u;
    bair = blocked | (I.eair ? __ldg(I.eair + g) : 0u);
    uint32_t heat = (blocked != 0u || w == 14u) ? 0x8u : 0u;
    bairh = heat | (I.eairh ? __ldg(I.eairh + g) : 0u);
}

}  // namespace air
}  // namespace tpt
