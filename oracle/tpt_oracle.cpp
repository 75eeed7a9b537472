// tpt_oracle.cpp -- CPU ORACLE for the coarse-grid field step. TEST
// INFRASTRUCTURE ONLY: the parity tests, the smoke check and the CPU-baseline
// leg of bench.py load it as the checker. The product library never links,
// loads or calls it.
//
// A restatement of the reference's CubeCL kernels for the field step, written
// from their source (paths relative to the reference project):
//
//   air      crates/tpt-sim/src/air_kernel/{mod,pressure,advect,heat,settle}.rs
//   gravity  crates/tpt-sim/src/gravity_gpu/{mod,fft}.rs
//   masks    crates/tpt-sim/src/gravity_kernel.rs:658-712 (flood fill)
//   particles crates/tpt-sim/src/gravity_kernel.rs:217-527 (wells, force,
//            mass build, overrides, snapshot copy)
//
// Two forms, one template:
//   R = float   the FP32 mirror: the reference's operation order, every
//               operation rounded to f32 (built with -ffp-contract=off so no
//               FMA is formed), radix-2 FFT with f32 host twiddles. This is
//               "the reference's kernels" for the parity thresholds.
//   R = double  the FP64 twin: the same maths in double (the f32 literal
//               constants promoted, so only arithmetic rounding differs), and
//               for gravity a double FFT convolution with double twiddles.
//               A brute-force direct sum pins the FP64 gravity.
//
// Documented divergence from the reference: `air_heat_convect_kernel`
// (heat.rs:92-94 vs 249-250) reads neighbour vx/vy while other threads write
// vx/vy in place, so its result depends on GPU scheduling. The oracle fixes
// read-before-write (Jacobi) semantics: every read sees the vx/vy the
// smoothing/advection pass produced.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/tpt_field.h"

namespace {

// ---------------------------------------------------------------- air ----
// BORDER band width, mod.rs:75; ADVECT_DIST, mod.rs:79.
constexpr uint32_t BORDER = 2;

template <typename R> struct K {
    // The reference's f32 literals, promoted for the FP64 twin.
    static constexpr R c(float v) { return R(v); }
};

template <typename R> static inline R clampr(R v, R lo, R hi) {
    // mod.rs:92-102 (compare-and-assign, not std::clamp, same result)
    R out = v;
    if (out < lo) out = lo;
    if (out > hi) out = hi;
    return out;
}

struct Grid {
    uint32_t X, Y;
    size_t at(uint32_t x, uint32_t y) const { return (size_t)y * X + x; }
};

// pressure.rs:9-15
static inline bool in_border(uint32_t x, uint32_t y, const Grid &g) {
    return x < BORDER || y < BORDER || x + BORDER >= g.X || y + BORDER >= g.Y;
}
// pressure.rs:20-26
static inline bool interior(uint32_t x, uint32_t y, const Grid &g) {
    return x >= 1 && y >= 1 && x + 1 < g.X && y + 1 < g.Y;
}
// pressure.rs:30-36
static inline uint32_t blocked_at(const uint32_t *b, int x, int y, const Grid &g) {
    if (x >= 0 && y >= 0 && x < (int)g.X && y < (int)g.Y) return b[(size_t)y * g.X + x];
    return 0;
}
// pressure.rs:43-62
static inline bool wall_cleared_vx(const uint32_t *b, uint32_t x, uint32_t y, const Grid &g) {
    bool out = false;
    if (y >= 1 && y + 1 < g.Y) {
        if (x >= 1 && x + 1 < g.X && blocked_at(b, x, y, g) != 0) out = true;
        if (x >= 2 && blocked_at(b, (int)x - 1, y, g) != 0) out = true;
        if (x + 2 < g.X && blocked_at(b, (int)x + 1, y, g) != 0) out = true;
    }
    return out;
}
// pressure.rs:65-85
static inline bool wall_cleared_vy(const uint32_t *b, uint32_t x, uint32_t y, const Grid &g) {
    bool out = false;
    if (x >= 1 && x + 1 < g.X) {
        if (y >= 1 && y + 1 < g.Y && blocked_at(b, x, y, g) != 0) out = true;
        if (y >= 2 && blocked_at(b, x, (int)y - 1, g) != 0) out = true;
        if (y + 2 < g.Y && blocked_at(b, x, (int)y + 1, g) != 0) out = true;
    }
    return out;
}
// pressure.rs:92-114
static inline bool adjacent_blocked_x(const uint32_t *b, uint32_t x, uint32_t y, const Grid &g) {
    return blocked_at(b, (int)x - 1, y, g) != 0 || blocked_at(b, x, y, g) != 0 ||
           blocked_at(b, (int)x + 1, y, g) != 0;
}
static inline bool adjacent_blocked_y(const uint32_t *b, uint32_t x, uint32_t y, const Grid &g) {
    return blocked_at(b, x, (int)y - 1, g) != 0 || blocked_at(b, x, y, g) != 0 ||
           blocked_at(b, x, (int)y + 1, g) != 0;
}
// pressure.rs:119-157
template <typename R>
static inline R effective_vx(const R *vx, const uint32_t *b, uint32_t x, uint32_t y, const Grid &g, R evx) {
    R v = vx[g.at(x, y)];
    if (in_border(x, y, g)) v = evx + (v - evx) * K<R>::c(0.9f);
    if (wall_cleared_vx(b, x, y, g)) v = R(0);
    return v;
}
template <typename R>
static inline R effective_vy(const R *vy, const uint32_t *b, uint32_t x, uint32_t y, const Grid &g, R evy) {
    R v = vy[g.at(x, y)];
    if (in_border(x, y, g)) v = evy + (v - evy) * K<R>::c(0.9f);
    if (wall_cleared_vy(b, x, y, g)) v = R(0);
    return v;
}

// pressure.rs:173-238
template <typename R>
static void pressure_pass(const Grid &g, const tpt_air_params &p, const R *pv, const R *vx, const R *vy,
                          const uint32_t *b, R *opv) {
    const R ep = R(p.edge_pressure), evx = R(p.edge_vx), evy = R(p.edge_vy);
#pragma omp parallel for schedule(static)
    for (int yy = 0; yy < (int)g.Y; ++yy) {
        uint32_t y = (uint32_t)yy;
        for (uint32_t x = 0; x < g.X; ++x) {
            size_t idx = g.at(x, y);
            R cur = pv[idx];
            if (in_border(x, y, g)) cur = ep + (cur - ep) * K<R>::c(0.8f);
            R next = cur;
            if (interior(x, y, g)) {
                R dp = effective_vx(vx, b, x - 1, y, g, evx) - effective_vx(vx, b, x + 1, y, g, evx) +
                       effective_vy(vy, b, x, y - 1, g, evy) - effective_vy(vy, b, x, y + 1, g, evy);
                next = ep + (cur - ep) * K<R>::c(0.9999f) + dp * K<R>::c(0.15f);
            }
            opv[idx] = next;
        }
    }
}

// pressure.rs:247-299
template <typename R>
static void velocity_pass(const Grid &g, const tpt_air_params &p, const R *opv, const R *vx, const R *vy,
                          const uint32_t *b, R *ovx, R *ovy) {
    const R evx = R(p.edge_vx), evy = R(p.edge_vy);
#pragma omp parallel for schedule(static)
    for (int yy = 0; yy < (int)g.Y; ++yy) {
        uint32_t y = (uint32_t)yy;
        for (uint32_t x = 0; x < g.X; ++x) {
            size_t idx = g.at(x, y);
            R cx = vx[idx], cy = vy[idx];
            if (in_border(x, y, g)) {
                cx = evx + (cx - evx) * K<R>::c(0.9f);
                cy = evy + (cy - evy) * K<R>::c(0.9f);
            }
            if (wall_cleared_vx(b, x, y, g)) cx = R(0);
            if (wall_cleared_vy(b, x, y, g)) cy = R(0);
            R nx = cx, ny = cy;
            if (interior(x, y, g)) {
                R dx = opv[idx - 1] - opv[idx + 1];
                R dy = opv[idx - g.X] - opv[idx + g.X];
                nx = evx + (cx - evx) * K<R>::c(0.999f) + dx * K<R>::c(0.2f);
                ny = evy + (cy - evy) * K<R>::c(0.999f) + dy * K<R>::c(0.2f);
                if (adjacent_blocked_x(b, x, y, g)) nx = R(0);
                if (adjacent_blocked_y(b, x, y, g)) ny = R(0);
            }
            ovx[idx] = nx;
            ovy[idx] = ny;
        }
    }
}

// advect.rs:10-42
template <typename R>
static inline R vorticity_bmap(const R *vx, const R *vy, const uint32_t *b, const Grid &g, uint32_t x, uint32_t y) {
    R out = R(0);
    if (x > 1 && x + 2 < g.X && y > 1 && y + 2 < g.Y) {
        size_t row = (size_t)y * g.X, rm = (size_t)(y - 1) * g.X, rp = (size_t)(y + 1) * g.X;
        bool here = b[row + x] != 0;
        R dvydx = vy[row + x + 1] - vy[row + x - 1];
        if (here || b[row + x + 1] != 0 || b[row + x - 1] != 0) dvydx = R(0);
        R dvxdy = vx[rp + x] - vx[rm + x];
        if (here || b[rp + x] != 0 || b[rm + x] != 0) dvxdy = R(0);
        out = (dvydx - dvxdy) * K<R>::c(0.5f);
    }
    return out;
}

// f32 -> i32 as the kernels' `as i32` (WGSL `i32(f32)`): round toward zero
// and saturate to the i32 range; NaN gives 0, as CUDA's cvt.rzi does (WGSL
// leaves NaN to the implementation). A plain C++ cast of an out-of-range or
// NaN float is undefined behaviour, so every such conversion goes through here.
template <typename R> static inline int32_t to_i32(R v) {
    if (v != v) return 0;
    if (v >= R(2147483648.0)) return INT32_MAX;
    if (v <= R(-2147483648.0)) return INT32_MIN;
    return (int32_t)v;
}

// advect.rs:46-52
static inline uint32_t advect_blocked(const uint32_t *b, size_t idx, bool heat) {
    return heat ? (b[idx] & 0x8u) : b[idx];
}

// advect.rs:66-152 (far-advection step walk)
template <typename R>
static inline void far_advect_target(uint32_t x, uint32_t y, R dx, R dy, const uint32_t *b, const Grid &g,
                                     bool heat, R &otx, R &oty) {
    const R ad = K<R>::c(0.7f);
    R tx = R(x) - dx * ad;
    R ty = R(y) - dy * ad;
    R adx = dx * ad;
    if (adx < R(0)) adx = R(0) - adx;
    R ady = dy * ad;
    if (ady < R(0)) ady = R(0) - ady;
    R limx = R(g.X) - R(2), limy = R(g.Y) - R(2);
    if ((adx > R(1) || ady > R(1)) && tx >= R(2) && tx < limx && ty >= R(2) && ty < limy) {
        R abs_dx = dx < R(0) ? R(0) - dx : dx;
        R abs_dy = dy < R(0) ? R(0) - dy : dy;
        R step_x, step_y;
        int32_t step_limit;
        if (abs_dx > abs_dy) {
            step_x = dx < R(0) ? R(1) : R(-1);
            step_y = R(0) - dy / abs_dx;
            step_limit = to_i32(adx);
        } else {
            step_x = R(0) - dx / abs_dy;
            step_y = dy < R(0) ? R(1) : R(-1);
            step_limit = to_i32(ady);
        }
        tx = R(x);
        ty = R(y);
        bool stopped = false;
        for (int32_t step = 0; step < step_limit; ++step) {
            tx += step_x;
            ty += step_y;
            int32_t cx = to_i32(tx + R(0.5f));
            int32_t cy = to_i32(ty + R(0.5f));
            bool hit = true;
            if (cx >= 0 && cy >= 0 && cx < (int32_t)g.X && cy < (int32_t)g.Y)
                hit = advect_blocked(b, (size_t)cy * g.X + (size_t)cx, heat) != 0;
            if (hit) {
                tx -= step_x;
                ty -= step_y;
                stopped = true;
                break;
            }
        }
        if (!stopped) {
            tx = R(x) - dx * ad;
            ty = R(y) - dy * ad;
        }
    }
    otx = tx;
    oty = ty;
}

// Smoothing weights, advect.rs:215-225 (order of the 3x3 loop: dy outer).
template <typename R> static inline R smooth_w(uint32_t dx, uint32_t dy) {
    R w = K<R>::c(0.01831564f);
    if (dx == 1) w = K<R>::c(0.13533528f);
    if (dy == 1) w = K<R>::c(0.13533528f);
    if (dx == 1 && dy == 1) w = R(1);
    return w;
}

// advect.rs:174-360
template <typename R>
static void smooth_advect_pass(const Grid &g, const tpt_air_params &p, const R *ovx, const R *ovy, const R *opv,
                               const uint32_t *b, const uint32_t *wall, const R *fan_vx, const R *fan_vy, R *vx,
                               R *vy, R *pv) {
    const R vcoef = R(p.vorticity_coeff);
#pragma omp parallel for schedule(dynamic, 4)
    for (int yy = 0; yy < (int)g.Y; ++yy) {
        uint32_t y = (uint32_t)yy;
        for (uint32_t x = 0; x < g.X; ++x) {
            size_t idx = g.at(x, y);
            R cvx = ovx[idx], cvy = ovy[idx], cpv = opv[idx];
            R sx = R(0), sy = R(0), sp = R(0), ws = R(0);
            for (uint32_t dyy = 0; dyy < 3; ++dyy) {
                for (uint32_t dxx = 0; dxx < 3; ++dxx) {
                    uint32_t nx = x + dxx;
                    nx = nx >= 1 ? nx - 1 : 0;  // saturating_sub
                    uint32_t ny = y + dyy;
                    ny = ny >= 1 ? ny - 1 : 0;
                    R w = smooth_w<R>(dxx, dyy);
                    bool itap = nx >= 1 && ny >= 1 && nx + 1 < g.X && ny + 1 < g.Y;
                    size_t ni = g.at(nx, ny);
                    R tx = cvx, ty = cvy, tp = cpv;
                    if (itap && b[ni] == 0) {
                        tx = ovx[ni];
                        ty = ovy[ni];
                        tp = opv[ni];
                    }
                    sx += tx * w;
                    sy += ty * w;
                    sp += tp * w;
                    ws += w;
                }
            }
            R nvx = sx / ws, nvy = sy / ws, npv = sp / ws;

            R tx0, ty0;
            far_advect_target<R>(x, y, nvx, nvy, b, g, false, tx0, ty0);
            int32_t i0 = to_i32(tx0), j0 = to_i32(ty0);
            R fx = tx0 - R(i0), fy = ty0 - R(j0);
            if (b[idx] == 0 && i0 >= 2 && i0 < (int32_t)g.X - 3 && j0 >= 2 && j0 < (int32_t)g.Y - 3 && fx >= R(0) &&
                fy >= R(0)) {
                size_t r0 = (size_t)j0 * g.X, r1 = (size_t)(j0 + 1) * g.X, iu = (size_t)i0;
                R w00 = (R(1) - fx) * (R(1) - fy);
                R w10 = fx * (R(1) - fy);
                R w01 = (R(1) - fx) * fy;
                R w11 = fx * fy;
                nvx = nvx * K<R>::c(0.7f) +
                      K<R>::c(0.3f) * (ovx[r0 + iu] * w00 + ovx[r0 + iu + 1] * w10 + ovx[r1 + iu] * w01 +
                                       ovx[r1 + iu + 1] * w11);
                nvy = nvy * K<R>::c(0.7f) +
                      K<R>::c(0.3f) * (ovy[r0 + iu] * w00 + ovy[r0 + iu + 1] * w10 + ovy[r1 + iu] * w01 +
                                       ovy[r1 + iu + 1] * w11);
            }

            // advect.rs:297-328
            if (vcoef > R(0) && x > 1 && x + 2 < g.X && y > 1 && y + 2 < g.Y) {
                R w = vorticity_bmap(ovx, ovy, b, g, x, y);
                R wxp = vorticity_bmap(ovx, ovy, b, g, x + 1, y);
                R wxm = vorticity_bmap(ovx, ovy, b, g, x - 1, y);
                R wyp = vorticity_bmap(ovx, ovy, b, g, x, y + 1);
                R wym = vorticity_bmap(ovx, ovy, b, g, x, y - 1);
                if (wxp < R(0)) wxp = R(0) - wxp;
                if (wxm < R(0)) wxm = R(0) - wxm;
                if (wyp < R(0)) wyp = R(0) - wyp;
                if (wym < R(0)) wym = R(0) - wym;
                R dwx = (wxp - wxm) * K<R>::c(0.5f);
                R dwy = (wyp - wym) * K<R>::c(0.5f);
                R norm = std::sqrt(dwx * dwx + dwy * dwy);
                R k = vcoef / K<R>::c(5.0f);
                nvx += k * dwy / (norm + K<R>::c(0.001f)) * w;
                nvy += k * (R(0) - dwx) / (norm + K<R>::c(0.001f)) * w;
            }
            // advect.rs:331-334
            if (wall[idx] == 5u) {
                nvx += fan_vx[idx];
                nvy += fan_vy[idx];
            }
            // advect.rs:337-354
            nvx = clampr(nvx, R(-256), R(256));
            nvy = clampr(nvy, R(-256), R(256));
            npv = clampr(npv, R(-256), R(256));
            if (p.air_mode == 1u) npv = R(0);
            if (p.air_mode == 2u) { nvx = R(0); nvy = R(0); }
            if (p.air_mode == 3u) { nvx = R(0); nvy = R(0); npv = R(0); }
            vx[idx] = nvx;
            vy[idx] = nvy;
            pv[idx] = npv;
        }
    }
}

// heat.rs:31-253 with Jacobi reads of vx/vy (see the file header). Writes
// the new heat into ohv and the convected velocity into nvx/nvy (copied of
// vx/vy for cells outside 2..X-3 by the caller's copy).
template <typename R>
static void heat_convect_pass(const Grid &g, const tpt_air_params &p, const R *hv, const R *vx, const R *vy,
                              const uint32_t *bh, R *ohv, R *nvx_out, R *nvy_out) {
    const R amb = R(p.ambient_air_temp);
    const R cgx = R(p.custom_gx), cgy = R(p.custom_gy);
#pragma omp parallel for schedule(dynamic, 4)
    for (int yy = 0; yy < (int)g.Y; ++yy) {
        uint32_t y = (uint32_t)yy;
        for (uint32_t x = 0; x < g.X; ++x) {
            size_t idx = g.at(x, y);
            R ch = hv[idx], cvx = vx[idx], cvy = vy[idx];
            R sh = R(0), sx = R(0), sy = R(0), ws = R(0);
            for (uint32_t dyy = 0; dyy < 3; ++dyy) {
                for (uint32_t dxx = 0; dxx < 3; ++dxx) {
                    uint32_t nx = x + dxx;
                    nx = nx >= 1 ? nx - 1 : 0;
                    uint32_t ny = y + dyy;
                    ny = ny >= 1 ? ny - 1 : 0;
                    R w = smooth_w<R>(dxx, dyy);
                    bool itap = nx >= 1 && ny >= 1 && nx + 1 < g.X && ny + 1 < g.Y;
                    size_t ni = g.at(nx, ny);
                    R th = ch, tx = cvx, ty = cvy;
                    if (itap && (bh[ni] & 0x8u) == 0) {
                        th = hv[ni];
                        tx = vx[ni];
                        ty = vy[ni];
                    }
                    sh += th * w;
                    sx += tx * w;
                    sy += ty * w;
                    ws += w;
                }
            }
            R dh = sh / ws;
            R svx = sx / ws, svy = sy / ws;

            R tx, ty;
            far_advect_target<R>(x, y, svx, svy, bh, g, true, tx, ty);
            int32_t i0 = to_i32(tx), j0 = to_i32(ty);
            R fx = tx - R(i0), fy = ty - R(j0);
            if ((bh[idx] & 0x8u) == 0 && i0 >= 0 && i0 < (int32_t)g.X - 1 && j0 >= 0 && j0 < (int32_t)g.Y - 1 &&
                fx >= R(0) && fy >= R(0)) {
                size_t r0 = (size_t)j0 * g.X, r1 = (size_t)(j0 + 1) * g.X, iu = (size_t)i0;
                R s00 = (bh[r0 + iu] & 0x8u) ? dh : hv[r0 + iu];
                R s10 = (bh[r0 + iu + 1] & 0x8u) ? dh : hv[r0 + iu + 1];
                R s01 = (bh[r1 + iu] & 0x8u) ? dh : hv[r1 + iu];
                R s11 = (bh[r1 + iu + 1] & 0x8u) ? dh : hv[r1 + iu + 1];
                R w00 = (R(1) - fx) * (R(1) - fy);
                R w10 = fx * (R(1) - fy);
                R w01 = (R(1) - fx) * fy;
                R w11 = fx * fy;
                dh = dh * K<R>::c(0.7f) + K<R>::c(0.3f) * (s00 * w00 + s10 * w10 + s01 * w01 + s11 * w11);
            }
            if (bh[idx] & 0x8u) dh = ch;
            dh = clampr(dh, R(0), R(9999));
            if (x < BORDER || y < BORDER || x + BORDER >= g.X || y + BORDER >= g.Y) dh = amb;
            if (p.aheat_enable == 0) dh = amb;
            ohv[idx] = dh;

            R ovx = cvx, ovy = cvy;
            if (x >= 2 && x + 2 < g.X && y >= 2 && y + 2 < g.Y) {
                R gxv = R(0), gyv = R(0);
                if (p.gravity_mode == 0u) {
                    gyv = R(1);
                } else if (p.gravity_mode == 2u) {
                    R rx = R(g.X) * K<R>::c(0.5f) - (R(x) + K<R>::c(0.5f));
                    R ry = R(g.Y) * K<R>::c(0.5f) - (R(y) + K<R>::c(0.5f));
                    R rd = std::sqrt(rx * rx + ry * ry);
                    if (rd > R(0)) {
                        gxv = rx / rd;
                        gyv = ry / rd;
                    }
                } else if (p.gravity_mode == 3u) {
                    gxv = cgx;
                    gyv = cgy;
                }
                R convx = R(0) - gxv, convy = R(0) - gyv;
                R nx = cvx, ny = cvy;
                if (p.convection_mode == 1u) {
                    size_t rm = (size_t)(y - 1) * g.X;
                    R weight = ((ch - hv[idx - 1]) * convx + (ch - hv[rm + x]) * convy) / K<R>::c(5000.0f);
                    if (weight > R(0) && (bh[rm + x] & 0x8u) == 0) {
                        nx += weight * convx;
                        ny += weight * convy;
                    }
                } else if (p.convection_mode == 2u) {
                    R gm = std::sqrt(convx * convx + convy * convy);
                    if (gm > R(10)) {
                        convx /= K<R>::c(0.1f) * gm;
                        convy /= K<R>::c(0.1f) * gm;
                    }
                    R weight = (ch - amb) / K<R>::c(10000.0f);
                    if (weight > K<R>::c(0.01f)) weight = K<R>::c(0.01f);
                    nx += weight * convx;
                    ny += weight * convy;
                }
                ovx = clampr(nx, R(-256), R(256));
                ovy = clampr(ny, R(-256), R(256));
            }
            nvx_out[idx] = ovx;
            nvy_out[idx] = ovy;
        }
    }
}

// settle.rs:50-93
static void block_masks_pass(size_t cells, const uint32_t *wall, uint32_t *emap, uint32_t *bair, uint32_t *bairh,
                             const uint32_t *eair, const uint32_t *eairh) {
    for (size_t i = 0; i < cells; ++i) {
        uint32_t w = wall[i] & 0xFFu;
        uint32_t raw = emap[i];
        if (raw != 0) emap[i] = raw - 1;
        uint32_t e = emap[i] & 0xFFu;
        uint32_t blocked = (w == 8u || w == 1u || w == 16u || (w == 2u && e == 0u)) ? 1u : 0u;
        bair[i] = blocked | (eair ? eair[i] : 0u);
        uint32_t heat = (blocked != 0 || w == 14u) ? 0x8u : 0u;
        bairh[i] = heat | (eairh ? eairh[i] : 0u);
    }
}

// settle.rs:118-161 (HotAir -> pressure), one cell walks its 4x4 pixels.
template <typename R>
static void hot_air_pass(const Grid &g, R *pv, const uint32_t *pmap, const uint32_t *props, uint32_t nprops,
                         uint32_t xres, uint32_t yres) {
    for (uint32_t cy = 0; cy < g.Y; ++cy)
        for (uint32_t cx = 0; cx < g.X; ++cx) {
            size_t cell = g.at(cx, cy);
            for (uint32_t dy = 0; dy < 4; ++dy)
                for (uint32_t dx = 0; dx < 4; ++dx) {
                    uint32_t px = cx * 4 + dx, py = cy * 4 + dy;
                    if (px >= xres || py >= yres) continue;
                    uint32_t e = pmap[(size_t)py * xres + px];
                    if (e == 0) continue;
                    uint32_t ty = e & 0x1FFu;
                    if (ty >= nprops) continue;
                    float hot;
                    uint32_t bits = props[(size_t)ty * 32 + 11];
                    std::memcpy(&hot, &bits, 4);
                    if (hot == 0.0f) continue;
                    R h = R(hot);
                    if (ty == 10u || ty == 97u) {
                        if (pv[cell] < K<R>::c(3.5f)) pv[cell] += K<R>::c(4.0f) * h * (K<R>::c(3.5f) - pv[cell]);
                    } else {
                        pv[cell] += K<R>::c(4.0f) * h;
                    }
                }
        }
}

template <typename R> struct AirState {
    R *pv, *vx, *vy, *hv;
    uint32_t *wall, *emap, *bair, *bairh;
    const uint32_t *eair, *eairh;
    const R *fan_vx, *fan_vy;
    const uint32_t *pmap, *props;
    uint32_t nprops, xres, yres;
};

// mod.rs:120-299 pass order.
template <typename R> static int air_steps(const tpt_air_params &p, AirState<R> &s, int ticks) {
    Grid g{p.xcells, p.ycells};
    size_t n = (size_t)g.X * g.Y;
    if (g.X == 0 || g.Y == 0) return 0;
    std::vector<R> opv(n), ovx(n), ovy(n), ohv(n), nvx(n), nvy(n);
    for (int t = 0; t < ticks; ++t) {
        if (p.air_mode != 4u) {
            pressure_pass<R>(g, p, s.pv, s.vx, s.vy, s.bair, opv.data());
            velocity_pass<R>(g, p, opv.data(), s.vx, s.vy, s.bair, ovx.data(), ovy.data());
            smooth_advect_pass<R>(g, p, ovx.data(), ovy.data(), opv.data(), s.bair, s.wall, s.fan_vx, s.fan_vy, s.vx,
                                  s.vy, s.pv);
        }
        if (p.aheat_enable != 0u) {
            heat_convect_pass<R>(g, p, s.hv, s.vx, s.vy, s.bairh, ohv.data(), nvx.data(), nvy.data());
            std::memcpy(s.hv, ohv.data(), n * sizeof(R));
            std::memcpy(s.vx, nvx.data(), n * sizeof(R));
            std::memcpy(s.vy, nvy.data(), n * sizeof(R));
        }
        block_masks_pass(n, s.wall, s.emap, s.bair, s.bairh, s.eair, s.eairh);
        if (s.pmap != nullptr && s.xres != 0 && s.yres != 0) hot_air_pass<R>(g, s.pv, s.pmap, s.props, s.nprops, s.xres, s.yres);
    }
    return 0;
}

// ------------------------------------------------------------ gravity ----
// gravity_gpu/mod.rs:62
constexpr float M_GRAV = 6.673e-1f;

// fft.rs:255-264
static uint32_t bit_count(uint32_t n) {
    uint32_t bits = 0, v = (n > 1 ? n : 1) - 1;
    while (v > 0) { v >>= 1; ++bits; }
    return bits;
}
static uint32_t next_pow2(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// fft.rs:242-253 (f32 twiddles, f32 angle arithmetic); the double form
// evaluates the same angle in double.
template <typename R> static void build_twiddle(uint32_t max_len, std::vector<R> &re, std::vector<R> &im) {
    uint32_t half = std::max<uint32_t>(max_len / 2, 1);
    re.resize(half);
    im.resize(half);
    for (uint32_t k = 0; k < half; ++k) {
        if constexpr (sizeof(R) == 4) {
            const float PI = 3.14159265358979323846f;
            float angle = -2.0f * PI * (float)k / (float)max_len;
            re[k] = cosf(angle);
            im[k] = sinf(angle);
        } else {
            double angle = -2.0 * M_PI * (double)k / (double)max_len;
            re[k] = std::cos(angle);
            im[k] = std::sin(angle);
        }
    }
}

// fft.rs:34-69 + 78-122, the host mirror of fft_host (fft.rs:274-328): one
// 1-D radix-2 DIT transform over `rows` sequences at r*inner + i*stride.
template <typename R>
static void fft_1d(R *data, uint32_t rows, uint32_t n, uint32_t inner, uint32_t stride, const R *twr, const R *twi,
                   uint32_t tw_bits, R sign) {
    uint32_t bits = bit_count(n);
#pragma omp parallel for schedule(static) if (rows >= 64)
    for (int rr = 0; rr < (int)rows; ++rr) {
        size_t r = (size_t)rr;
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t src = i, rev = 0;
            for (uint32_t b = 0; b < bits; ++b) {
                rev = rev * 2 + src % 2;
                src /= 2;
            }
            if (i < rev) {
                size_t a = (r * inner + (size_t)i * stride) * 2, c = (r * inner + (size_t)rev * stride) * 2;
                std::swap(data[a], data[c]);
                std::swap(data[a + 1], data[c + 1]);
            }
        }
        for (uint32_t half = 1; half < n; half *= 2) {
            uint32_t len = half * 2;
            uint32_t shift = tw_bits - bit_count(len);
            for (uint32_t k = 0; k < n / 2; ++k) {
                uint32_t block = k / half, pos = k % half;
                uint32_t i0 = block * len + pos, i1 = i0 + half;
                uint32_t t = pos << shift;
                R wr = twr[t], wi = twi[t] * sign;
                size_t a = (r * inner + (size_t)i0 * stride) * 2, b = (r * inner + (size_t)i1 * stride) * 2;
                R xr = data[a], xi = data[a + 1], yr = data[b], yi = data[b + 1];
                R tr = wr * yr - wi * yi;
                R ti = wr * yi + wi * yr;
                data[a] = xr + tr;
                data[a + 1] = xi + ti;
                data[b] = xr - tr;
                data[b + 1] = xi - ti;
            }
        }
    }
}

// fft.rs:208-237 kernel field, wrapped around the transform origin.
template <typename R> static void build_kernel_field(R *out, uint32_t W, uint32_t H, R scale, int axis) {
    for (uint32_t py = 0; py < H; ++py)
        for (uint32_t px = 0; px < W; ++px) {
            R dx = R(px), dy = R(py);
            if (px * 2 >= W) dx = R(px) - R(W);
            if (py * 2 >= H) dy = R(py) - R(H);
            R v = R(0);
            if (dx != R(0) || dy != R(0)) {
                R dist = std::sqrt(dx * dx + dy * dy);
                R inv = scale / (dist * dist * dist);
                v = axis == 0 ? dx * inv : dy * inv;
            }
            size_t a = ((size_t)py * W + px) * 2;
            out[a] = v;
            out[a + 1] = R(0);
        }
}

// mod.rs:140-278: allocate, build_kernels, solve. `mass_r` (if non-null) is
// an already-scaled mass grid; otherwise `mass_i` * mass_scale_inv.
template <typename R>
static int grav_solve(uint32_t X, uint32_t Y, const int32_t *mass_i, const float *mass_f, float mass_scale_inv,
                      const uint32_t *mask, R *gx, R *gy) {
    uint32_t W = next_pow2(2 * X), H = next_pow2(2 * Y);
    uint32_t tw_bits = bit_count(std::max(W, H));
    std::vector<R> twr, twi;
    build_twiddle<R>(1u << tw_bits, twr, twi);
    size_t cells = (size_t)W * H;
    std::vector<R> kx(cells * 2), ky(cells * 2), work(cells * 2), sx(cells * 2), sy(cells * 2);
    R scale;
    if constexpr (sizeof(R) == 4) scale = -M_GRAV / (float)(W * H);
    else scale = -(double)M_GRAV / (double)((double)W * H);
    build_kernel_field<R>(kx.data(), W, H, scale, 0);
    build_kernel_field<R>(ky.data(), W, H, scale, 1);
    for (R *k : {kx.data(), ky.data()}) {
        fft_1d<R>(k, H, W, W, 1, twr.data(), twi.data(), tw_bits, R(1));
        fft_1d<R>(k, W, H, 1, W, twr.data(), twi.data(), tw_bits, R(1));
    }
    // fft.rs:152-178
    for (uint32_t py = 0; py < H; ++py)
        for (uint32_t px = 0; px < W; ++px) {
            R v = R(0);
            if (px < X && py < Y) {
                size_t c = (size_t)py * X + px;
                if (mask[c] != 0) {
                    if (mass_f) v = R(mass_f[c]);
                    else if constexpr (sizeof(R) == 4) v = (float)mass_i[c] * mass_scale_inv;
                    else v = (double)mass_i[c] * (double)mass_scale_inv;
                }
            }
            size_t a = ((size_t)py * W + px) * 2;
            work[a] = v;
            work[a + 1] = R(0);
        }
    fft_1d<R>(work.data(), H, W, W, 1, twr.data(), twi.data(), tw_bits, R(1));
    fft_1d<R>(work.data(), W, H, 1, W, twr.data(), twi.data(), tw_bits, R(1));
    // fft.rs:128-140
    for (size_t i = 0; i < cells; ++i) {
        size_t a = i * 2;
        R wr = work[a], wi = work[a + 1];
        sx[a] = wr * kx[a] - wi * kx[a + 1];
        sx[a + 1] = wr * kx[a + 1] + wi * kx[a];
        sy[a] = wr * ky[a] - wi * ky[a + 1];
        sy[a + 1] = wr * ky[a + 1] + wi * ky[a];
    }
    for (R *s : {sx.data(), sy.data()}) {
        fft_1d<R>(s, H, W, W, 1, twr.data(), twi.data(), tw_bits, R(-1));
        fft_1d<R>(s, W, H, 1, W, twr.data(), twi.data(), tw_bits, R(-1));
    }
    // fft.rs:181-200
    for (uint32_t py = 0; py < Y; ++py)
        for (uint32_t px = 0; px < X; ++px) {
            size_t c = (size_t)py * X + px;
            size_t a = ((size_t)py * W + px) * 2;
            gx[c] = mask[c] != 0 ? sx[a] : R(0);
            gy[c] = mask[c] != 0 ? sy[a] : R(0);
        }
    return 0;
}

}  // namespace

// ============================================================ C ABI ======
extern "C" {

int ora_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void ora_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ora_air_steps_f32(const tpt_air_params *p, int ticks, float *pv, float *vx, float *vy, float *hv,
                      uint32_t *wall, uint32_t *emap, uint32_t *bair, uint32_t *bairh, const uint32_t *eair,
                      const uint32_t *eairh, const float *fan_vx, const float *fan_vy, const uint32_t *pmap,
                      const uint32_t *props, uint32_t nprops, uint32_t xres, uint32_t yres) {
    AirState<float> s{pv, vx, vy, hv, wall, emap, bair, bairh, eair, eairh, fan_vx, fan_vy, pmap, props, nprops, xres, yres};
    return air_steps<float>(*p, s, ticks);
}

int ora_air_steps_f64(const tpt_air_params *p, int ticks, double *pv, double *vx, double *vy, double *hv,
                      uint32_t *wall, uint32_t *emap, uint32_t *bair, uint32_t *bairh, const uint32_t *eair,
                      const uint32_t *eairh, const double *fan_vx, const double *fan_vy, const uint32_t *pmap,
                      const uint32_t *props, uint32_t nprops, uint32_t xres, uint32_t yres) {
    AirState<double> s{pv, vx, vy, hv, wall, emap, bair, bairh, eair, eairh, fan_vx, fan_vy, pmap, props, nprops, xres, yres};
    return air_steps<double>(*p, s, ticks);
}

// Single passes, for pass-level parity tests.
void ora_block_masks(size_t cells, const uint32_t *wall, uint32_t *emap, uint32_t *bair, uint32_t *bairh,
                     const uint32_t *eair, const uint32_t *eairh) {
    block_masks_pass(cells, wall, emap, bair, bairh, eair, eairh);
}

int ora_grav_solve_f32(uint32_t X, uint32_t Y, const int32_t *mass_i, const float *mass_f, float mass_scale_inv,
                       const uint32_t *mask, float *gx, float *gy) {
    return grav_solve<float>(X, Y, mass_i, mass_f, mass_scale_inv, mask, gx, gy);
}
int ora_grav_solve_f64(uint32_t X, uint32_t Y, const int32_t *mass_i, const float *mass_f, float mass_scale_inv,
                       const uint32_t *mask, double *gx, double *gy) {
    return grav_solve<double>(X, Y, mass_i, mass_f, mass_scale_inv, mask, gx, gy);
}

// Brute-force FP64 direct sum of -M_GRAV * sum_m mass[m] (p-m)/|p-m|^3, the
// physical field the FFT solve must equal (gravity_gpu/mod.rs:17-38).
int ora_grav_direct_f64(uint32_t X, uint32_t Y, const int32_t *mass_i, const float *mass_f, float mass_scale_inv,
                        const uint32_t *mask, double *gx, double *gy) {
    size_t n = (size_t)X * Y;
    std::vector<double> m(n);
    for (size_t c = 0; c < n; ++c)
        m[c] = mask[c] == 0 ? 0.0 : (mass_f ? (double)mass_f[c] : (double)mass_i[c] * (double)mass_scale_inv);
    const double G = -(double)M_GRAV;
#pragma omp parallel for schedule(dynamic, 1)
    for (int py = 0; py < (int)Y; ++py)
        for (uint32_t px = 0; px < X; ++px) {
            double sx = 0, sy = 0;
            for (uint32_t my = 0; my < Y; ++my)
                for (uint32_t mx = 0; mx < X; ++mx) {
                    double mm = m[(size_t)my * X + mx];
                    if (mm == 0.0) continue;
                    double dx = (double)px - mx, dy = (double)py - my;
                    if (dx == 0 && dy == 0) continue;
                    double d = std::sqrt(dx * dx + dy * dy);
                    double inv = G / (d * d * d);
                    sx += mm * dx * inv;
                    sy += mm * dy * inv;
                }
            size_t c = (size_t)py * X + px;
            gx[c] = mask[c] ? sx : 0.0;
            gy[c] = mask[c] ? sy : 0.0;
        }
    return 0;
}

// Host FFT mirror for the reference's own known-answer tests (fft.rs:357-415).
void ora_fft_host_f32(float *data, uint32_t rows, uint32_t n, uint32_t inner, uint32_t stride, uint32_t tw_bits,
                      float sign) {
    std::vector<float> twr, twi;
    build_twiddle<float>(1u << tw_bits, twr, twi);
    fft_1d<float>(data, rows, n, inner, stride, twr.data(), twi.data(), tw_bits, sign);
}
uint32_t ora_bit_count(uint32_t n) { return bit_count(n); }
void ora_twiddle_f32(uint32_t max_len, float *re, float *im) {
    std::vector<float> twr, twi;
    build_twiddle<float>(max_len, twr, twi);
    std::memcpy(re, twr.data(), twr.size() * 4);
    std::memcpy(im, twi.data(), twi.size() * 4);
}

// gravity_kernel.rs:658-712 flood fill.
int ora_grav_mask(const uint32_t *wall, uint32_t *mask, uint32_t X, uint32_t Y) {
    size_t cells = (size_t)X * Y;
    if (cells == 0) return 0;
    std::fill(mask, mask + cells, 0u);
    std::vector<size_t> stack;
    auto seed = [&](size_t idx) {
        if ((wall[idx] & 0xFFu) == 14u || mask[idx] != 0u) return;
        mask[idx] = 0xFFFFFFFFu;
        stack.push_back(idx);
    };
    for (uint32_t x = 0; x < X; ++x) {
        seed(x);
        seed((size_t)(Y - 1) * X + x);
    }
    for (uint32_t y = 1; y + 1 < Y; ++y) {
        seed((size_t)y * X);
        seed((size_t)y * X + X - 1);
    }
    while (!stack.empty()) {
        size_t idx = stack.back();
        stack.pop_back();
        uint32_t x = (uint32_t)(idx % X), y = (uint32_t)(idx / X);
        if (x > 0) seed(idx - 1);
        if (x + 1 < X) seed(idx + 1);
        if (y > 0) seed(idx - X);
        if (y + 1 < Y) seed(idx + X);
    }
    return 0;
}

// crates/tpt-sim/src/engine_commands/tools.rs:272-275: PGRV/NGRV tool mass.
float ora_tool_gravity_mass(float strength, int attract) {
    float magnitude = std::fabs(strength) * 5.0f;
    return attract ? magnitude : -magnitude;
}

// crates/tpt-sim/src/engine_commands/tools.rs:281-298: pixel -> cell index,
// -1 for the reference's None.
int64_t ora_gravity_tool_cell(int32_t x, int32_t y, int32_t xres, int32_t yres, int32_t xcells, int32_t ycells) {
    if (x < 0 || y < 0 || x >= xres || y >= yres) return -1;
    int32_t cx = x / 4, cy = y / 4;
    if (cx < 0 || cy < 0 || cx >= xcells || cy >= ycells) return -1;
    return (int64_t)cy * xcells + cx;
}

// crates/tpt-core/src/particle.rs:381-383: canvas side clamped to 64 and
// rounded up to a whole cell.
uint32_t ora_align_dim(uint32_t v) {
    if (v < 64u) v = 64u;
    return (v + 3u) / 4u * 4u;
}

// gravity_kernel.rs:217-229 (seed_gravity_mass_kernel rounding).
int32_t ora_mass_to_fixed(float m) {
    float scaled = m * 65536.0f;
    if (scaled >= 0.0f) scaled += 0.5f;
    else scaled -= 0.5f;
    return to_i32(scaled);
}

// ---- gravity tick around the solve (host pointers in the ABI structs) ------
// f32 -> i32 truncation as the GPU converts: NaN -> 0, out of range saturates.
static int32_t trunc_i32(float v) {
    if (!(v == v)) return 0;
    if (v >= 2147483648.0f) return INT32_MAX;
    if (v < -2147483648.0f) return INT32_MIN;
    return (int32_t)v;
}
static int32_t to_fixed(float m) {  // gravity_kernel.rs:346-353
    float scaled = m * 65536.0f;
    if (scaled >= 0.0f) scaled += 0.5f;
    else scaled -= 0.5f;
    return trunc_i32(scaled);
}

// seed_gravity_tool_mass_kernel (gravity_kernel.rs:241-262), then
// seed_gravity_mass_kernel (:217-229) once the wells are consumed.
void ora_grav_seed(const tpt_grav_state *s, uint32_t cells) {
    for (uint32_t c = 0; c < cells; ++c) {
        if (s->tool_mass && s->tool_mass[c] != 0.0f) {
            s->mass_prev[c] = to_fixed(s->tool_mass[c]);
            s->tool_mass[c] = 0.0f;
        }
    }
    for (uint32_t c = 0; c < cells; ++c) {
        float tool = s->tool_mass ? s->tool_mass[c] : 0.0f;
        s->mass[c] = to_fixed(tool);
        if (s->tool_mass) s->tool_mass[c] = 0.0f;
    }
}

// apply_gravity_kernel (gravity_kernel.rs:434-516), all slots, then
// build_gravity_mass_kernel (:275-376), all slots; the accumulator wraps like
// the device's 32-bit atomic add.
void ora_grav_particles(const tpt_grav_state *s, const tpt_particles *q, uint32_t xcells, uint32_t ycells) {
    const int32_t xres = (int32_t)s->xres, yres = (int32_t)s->yres;
    for (uint32_t i = 0; i < q->num_slots; ++i) {
        const uint32_t ty = q->ty[i];
        if (ty == 0u || ty >= q->n_types) continue;
        const uint32_t flags = q->flags[i];
        bool eligible = (flags & 0x10u) == 0u;
        const int32_t xi = trunc_i32(q->x[i] + 0.5f), yi = trunc_i32(q->y[i] + 0.5f);
        if (xi < 0 || yi < 0 || xi >= xres || yi >= yres) eligible = false;
        if (xi < 4 || yi < 4 || xi >= xres - 4 || yi >= yres - 4) eligible = false;
        if (!eligible) continue;
        const size_t cell = (size_t)((uint32_t)yi / 4u) * xcells + (uint32_t)xi / 4u;
        if (s->wall_bmap[cell] == 18u && (s->wall_emap[cell] & 0xFFu) < 8u) continue;
        const uint32_t props = q->move_lut[(size_t)ty * 12];
        float loss;
        std::memcpy(&loss, &q->move_lut[(size_t)ty * 12 + 7], 4);
        if (!(ty == 78u && (flags & 0x08u) != 0u)) {
            q->vx[i] *= loss;
            q->vy[i] *= loss;
        }
        if ((props & 0x4u) == 0u) {
            q->vx[i] += s->newton_grav * s->gx[cell];
            q->vy[i] += s->newton_grav * s->gy[cell];
        }
    }
    for (uint32_t i = 0; i < q->num_slots; ++i) {
        const uint32_t ty = q->ty[i];
        if (ty == 0u) continue;
        float mass = 0.0f;
        bool contributes = false;
        if (ty == 39u) {  // GRVT
            int32_t tmp = q->tmp[i];
            if (tmp < -100) tmp = -100;
            if (tmp > 100) tmp = 100;
            mass = 0.2f * (float)tmp;
            contributes = true;
        } else if (ty == 40u || ty == 41u) {  // NBHL, NWHL
            float hole = 0.1f;
            if (q->tmp[i] != 0) {
                hole = 0.001f * (float)q->tmp[i];
                if (hole < 0.1f) hole = 0.1f;
                if (hole > 51.2f) hole = 51.2f;
            }
            if (ty == 41u) hole = -hole;
            mass = hole;
            contributes = true;
        } else if (ty == 42u) {  // GBMB
            if (q->life[i] > 20) {
                mass = 20.0f;
                contributes = true;
            } else if (q->life[i] >= 1) {
                mass = -80.0f;
                contributes = true;
            }
        } else if (ty == 43u) {  // GPMP
            if (q->life[i] == 10) {
                mass = 0.2f * (q->temp[i] - 273.15f);
                contributes = true;
            }
        }
        if (!contributes) continue;
        const int32_t xi = trunc_i32(q->x[i] + 0.5f), yi = trunc_i32(q->y[i] + 0.5f);
        if (xi < 0 || yi < 0 || xi >= xres || yi >= yres) continue;
        const uint32_t cx = (uint32_t)xi / 4u, cy = (uint32_t)yi / 4u;
        if (cx >= xcells || cy >= ycells) continue;
        const size_t cell = (size_t)cy * xcells + cx;
        if (s->grav_mask[cell] == 0u) continue;
        const int32_t qv = to_fixed(mass);
        if (qv != 0) s->mass[cell] = (int32_t)((uint32_t)s->mass[cell] + (uint32_t)qv);
    }
}

// apply_grav_mass_override_kernel (gravity_kernel.rs:379-391), then
// copy_gravity_mass_kernel (:518-527).
void ora_grav_finish(const tpt_grav_state *s, uint32_t cells) {
    for (uint32_t c = 0; c < cells; ++c)
        if (s->override_set && s->override_set[c] != 0u) s->mass[c] = s->override_mass[c];
    for (uint32_t c = 0; c < cells; ++c) s->mass_prev[c] = s->mass[c];
}

}  // extern "C"

// ======================================================= 3-D field step ====
// The 3-D sandbox's coarse grid (crates/tpt-sim/src/voxel3d): 64^3 cells,
// index (y << 12) | (z << 6) | x; voxels 256^3, index (y << 16) | (z << 8) | x.
// Each function is the reference kernel run over every cell in index order,
// f32 throughout (no contraction), with the reference's buffer alternation.
namespace vox {

constexpr uint32_t N = 64, SZ = 64, SY = 4096, CELLS = 262144;

static inline float clampf(float v, float lo, float hi) {  // step/mod.rs:425-435
    float out = v;
    if (out < lo) out = lo;
    if (out > hi) out = hi;
    return out;
}
static inline float seed_f32(float anchor, float v) { return anchor * 0.0f + v; }  // step/mod.rs:371-373

// air_kernel.rs:80-91
static inline float clamp_speed(float v) {
    float out = v;
    if (out > 8.0f) out = 8.0f;
    if (out < -8.0f) out = -8.0f;
    return out;
}

// air_kernel.rs:99-135
static float neighbour_average(const float *s, uint32_t i, uint32_t x, uint32_t y, uint32_t z) {
    float sum = s[i];
    float count = 1.0f;
    if (x > 0) { sum += s[i - 1]; count += 1.0f; }
    if (x + 1 < N) { sum += s[i + 1]; count += 1.0f; }
    if (z > 0) { sum += s[i - SZ]; count += 1.0f; }
    if (z + 1 < N) { sum += s[i + SZ]; count += 1.0f; }
    if (y > 0) { sum += s[i - SY]; count += 1.0f; }
    if (y + 1 < N) { sum += s[i + SY]; count += 1.0f; }
    return sum / count;
}

// air_kernel.rs:142-176
static float upwind_sample(const float *s, uint32_t i, float cur, int axis, uint32_t x, uint32_t y, uint32_t z) {
    float sample = cur;
    if (cur > 0.0f) {
        if (axis == 0 && x > 0) sample = s[i - 1];
        if (axis == 1 && y > 0) sample = s[i - SY];
        if (axis == 2 && z > 0) sample = s[i - SZ];
    } else if (cur < 0.0f) {
        if (axis == 0 && x + 1 < N) sample = s[i + 1];
        if (axis == 1 && y + 1 < N) sample = s[i + SY];
        if (axis == 2 && z + 1 < N) sample = s[i + SZ];
    }
    return sample;
}

// gravity.rs:74-109 (voxel_mass), MASS_SCALE = 1024
static int32_t voxel_mass(uint32_t ty, uint32_t life, int32_t tmp, float temp_k) {
    int32_t out = 0;  // seed_i32(tmp, 0)
    if (ty == 39u) {  // GRVT
        const int32_t t = trunc_i32(clampf((float)tmp, -100.0f, 100.0f));
        out = trunc_i32(0.2f * (float)t * 1024.0f);
    } else if (ty == 40u || ty == 41u) {  // NBHL, NWHL
        float add = seed_f32(temp_k, 0.1f);
        if (tmp != 0) add = clampf(0.001f * (float)tmp, 0.1f, 51.2f);
        out = ty == 40u ? trunc_i32(add * 1024.0f) : trunc_i32(-add * 1024.0f);
    } else if (ty == 42u) {  // GBMB
        if (life > 20u) out = trunc_i32(20.0f * 1024.0f);
        else if (life >= 1u) out = trunc_i32(-80.0f * 1024.0f);
    } else if (ty == 43u) {  // GPMP
        if (life == 10u) out = trunc_i32(0.2f * (temp_k - 273.15f) * 1024.0f);
    }
    return out;
}

static inline uint32_t brick_cell(uint32_t brick, uint32_t slot, uint32_t *bx, uint32_t *by, uint32_t *bz) {
    const uint32_t cx = (brick & 31u) * 2u + (slot & 1u);
    const uint32_t cz = ((brick >> 5) & 31u) * 2u + ((slot >> 1) & 1u);
    const uint32_t cy = ((brick >> 10) & 31u) * 2u + ((slot >> 2) & 1u);
    *bx = cx * 4u;
    *by = cy * 4u;
    *bz = cz * 4u;
    return (cy << 12) | (cz << 6) | cx;
}

}  // namespace vox

extern "C" {

// air_clear_kernel (air_kernel.rs:182-204)
void ora_vox_air_clear(const tpt_vox_world *w) {
    for (uint32_t i = 0; i < vox::CELLS; ++i) {
        w->vx[i] = 0.0f;
        w->vy[i] = 0.0f;
        w->vz[i] = 0.0f;
        w->p[i] = 0.0f;
        w->p_tmp[i] = 0.0f;
        w->temp[i] = 293.15f;
        w->solid[i] = 0.0f;
        w->pv[i] = 0;
    }
}

// air_gather_kernel (air_kernel.rs:218-278) over the first n listed bricks.
void ora_vox_air_gather(const tpt_vox_world *w, uint32_t n) {
    for (uint32_t b = 0; b < n; ++b) {
        for (uint32_t slot = 0; slot < 8u; ++slot) {
            uint32_t bx, by, bz;
            const uint32_t air = vox::brick_cell(w->sim_list[b], slot, &bx, &by, &bz);
            uint32_t occupied = 0;
            float temp_sum = 0.0f;
            for (uint32_t ly = 0; ly < 4u; ++ly)
                for (uint32_t lz = 0; lz < 4u; ++lz)
                    for (uint32_t lx = 0; lx < 4u; ++lx) {
                        const uint32_t v = w->voxel[((by + ly) << 16) | ((bz + lz) << 8) | (bx + lx)];
                        if ((v & 0xFFu) != 0u) {
                            occupied += 1u;
                            temp_sum += (float)((v >> 8) & 0xFFFFu) * 0.125f;
                        }
                    }
            w->solid[air] = (float)occupied * (1.0f / 64.0f);
            w->temp[air] = occupied > 0u ? temp_sum / (float)occupied : 293.15f;
        }
    }
}

// AirState::solve (air.rs:162-222): air_pressure_volume_kernel
// (air_kernel.rs:294-326), air_velocity_snapshot_kernel (:338-351),
// `iterations` x air_pressure_jacobi_kernel (:361-398) alternating p / p_tmp,
// then air_advect_kernel (:414-536).
void ora_vox_air_solve(const tpt_vox_world *w, uint32_t iterations) {
    using namespace vox;
    for (uint32_t i = 0; i < CELLS; ++i) {
        const uint32_t x = i & 63u, z = (i >> 6) & 63u, y = i >> 12;
        int32_t value = w->pv[i];
        if (x < 2u || x >= 62u || y < 2u || y >= 62u || z < 2u || z >= 62u) {
            value = trunc_i32((float)value * 0.2f);
        } else {
            const float dp = (w->vx[i - 1] - w->vx[i + 1]) + (w->vy[i - SY] - w->vy[i + SY]) +
                             (w->vz[i - SZ] - w->vz[i + SZ]);
            const float mixed = (float)value * 0.9999f;
            const float next = mixed + dp * 0.3f * 0.5f * 1024.0f;
            if (next > 262144.0f) value = 262144;
            else if (next < -262144.0f) value = -262144;
            else value = trunc_i32(next);
        }
        w->pv[i] = value;
    }
    std::vector<float> snap(3 * (size_t)CELLS);
    for (uint32_t i = 0; i < CELLS; ++i) {
        snap[i] = w->vx[i];
        snap[CELLS + i] = w->vy[i];
        snap[2 * CELLS + i] = w->vz[i];
    }
    float *pin = w->p, *pout = w->p_tmp;
    for (uint32_t it = 0; it < iterations; ++it) {
        for (uint32_t i = 0; i < CELLS; ++i) {
            const uint32_t x = i & 63u, z = (i >> 6) & 63u, y = i >> 12;
            const bool boundary = x == 0u || y == 0u || z == 0u || x == 63u || y == 63u || z == 63u;
            if (boundary || w->solid[i] > 0.5f) {
                pout[i] = 0.0f;
            } else {
                const float divergence = 0.5f * ((w->vx[i + 1] - w->vx[i - 1]) + (w->vy[i + SY] - w->vy[i - SY]) +
                                                 (w->vz[i + SZ] - w->vz[i - SZ]));
                const float nb = pin[i - 1] + pin[i + 1] + pin[i - SZ] + pin[i + SZ] + pin[i - SY] + pin[i + SY];
                pout[i] = (nb - divergence) / 6.0f;
            }
        }
        std::swap(pin, pout);
    }
    const float *pr = pin, *sx = snap.data(), *sy = snap.data() + CELLS, *sz = snap.data() + 2 * (size_t)CELLS;
    for (uint32_t i = 0; i < CELLS; ++i) {
        if (w->solid[i] > 0.5f) {
            w->vx[i] = 0.0f;
            w->vy[i] = 0.0f;
            w->vz[i] = 0.0f;
            continue;
        }
        const uint32_t x = i & 63u, z = (i >> 6) & 63u, y = i >> 12;
        const float local_temp = neighbour_average(w->temp, i, x, y, z);
        const uint32_t lx = x > 0 ? i - 1 : i, ux = x + 1 < N ? i + 1 : i;
        const uint32_t lz = z > 0 ? i - SZ : i, uz = z + 1 < N ? i + SZ : i;
        const uint32_t ly = y > 0 ? i - SY : i, uy = y + 1 < N ? i + SY : i;
        const float gx = (pr[ux] - pr[lx]) * 0.5f, gy = (pr[uy] - pr[ly]) * 0.5f, gz = (pr[uz] - pr[lz]) * 0.5f;
        const float ox = sx[i], oy = sy[i], oz = sz[i];
        const float buoyancy = (local_temp - 293.15f) * 0.02f;
        float nx = (ox - gx) * 0.99f, ny = (oy + buoyancy - gy) * 0.99f, nz = (oz - gz) * 0.99f;
        const float keep_n = 1.0f - 0.1f, keep_u = 1.0f - 0.25f;
        nx = nx * keep_n + neighbour_average(sx, i, x, y, z) * 0.1f;
        ny = ny * keep_n + neighbour_average(sy, i, x, y, z) * 0.1f;
        nz = nz * keep_n + neighbour_average(sz, i, x, y, z) * 0.1f;
        nx = nx * keep_u + upwind_sample(sx, i, ox, 0, x, y, z) * 0.25f;
        ny = ny * keep_u + upwind_sample(sy, i, oy, 1, x, y, z) * 0.25f;
        nz = nz * keep_u + upwind_sample(sz, i, oz, 2, x, y, z) * 0.25f;
        w->vx[i] = clamp_speed(nx);
        w->vy[i] = clamp_speed(ny);
        w->vz[i] = clamp_speed(nz);
    }
}

// gravity::solve (gravity.rs:228-260): `iterations` (24 in the reference)
// gravity_jacobi_kernel sweeps (:170-196) with the potential handles swapped
// after each, then gravity_force_kernel (:199-224). On return grav_potential
// names the last sweep, as the swapped handles do.
void ora_vox_grav_solve(const tpt_vox_world *w, uint32_t iterations) {
    using namespace vox;
    float *uin = w->grav_potential, *uout = w->grav_potential_tmp;
    for (uint32_t it = 0; it < iterations; ++it) {
        for (uint32_t i = 0; i < CELLS; ++i) {
            const uint32_t x = i & 63u, z = (i >> 6) & 63u, y = (i >> 12) & 63u;
            const bool boundary = x == 0u || x == 63u || y == 0u || y == 63u || z == 0u || z == 63u;
            float out = seed_f32(uin[i], 0.0f);
            if (!boundary) {
                const float sum = uin[i - 1] + uin[i + 1] + uin[i - SZ] + uin[i + SZ] + uin[i - SY] + uin[i + SY];
                const float rho = (float)w->grav_mass[i] * (1.0f / 1024.0f);
                out = (sum - 8.385539f * rho) * (1.0f / 6.0f);
            }
            uout[i] = out;
        }
        std::swap(uin, uout);
    }
    if (uin != w->grav_potential) {  // odd sweep count: give the names their swapped contents
        std::vector<float> t(uin, uin + CELLS);
        std::memcpy(w->grav_potential_tmp, w->grav_potential, CELLS * sizeof(float));
        std::memcpy(w->grav_potential, t.data(), CELLS * sizeof(float));
    }
    const float *u = w->grav_potential;
    for (uint32_t i = 0; i < CELLS; ++i) {
        const uint32_t x = i & 63u, z = (i >> 6) & 63u, y = (i >> 12) & 63u;
        const bool boundary = x == 0u || x == 63u || y == 0u || y == 63u || z == 0u || z == 63u;
        float fx = seed_f32(u[i], 0.0f), fy = seed_f32(u[i], 0.0f), fz = seed_f32(u[i], 0.0f);
        if (!boundary) {
            fx = (u[i - 1] - u[i + 1]) * 0.5f;
            fz = (u[i - SZ] - u[i + SZ]) * 0.5f;
            fy = (u[i - SY] - u[i + SY]) * 0.5f;
        }
        w->grav_force_x[i] = fx;
        w->grav_force_y[i] = fy;
        w->grav_force_z[i] = fz;
    }
}

// gravity_clear_kernel (gravity.rs:112-118)
void ora_vox_grav_clear_mass(const tpt_vox_world *w) {
    std::memset(w->grav_mass, 0, vox::CELLS * sizeof(int32_t));
}

// gravity_gather_kernel (gravity.rs:125-166) over the first n listed bricks;
// the i32 accumulator and the atomic add wrap.
void ora_vox_grav_gather(const tpt_vox_world *w, uint32_t n) {
    for (uint32_t b = 0; b < n; ++b) {
        for (uint32_t slot = 0; slot < 8u; ++slot) {
            uint32_t bx, by, bz;
            const uint32_t cell = vox::brick_cell(w->sim_list[b], slot, &bx, &by, &bz);
            uint32_t acc = 0;
            for (uint32_t ly = 0; ly < 4u; ++ly)
                for (uint32_t lz = 0; lz < 4u; ++lz)
                    for (uint32_t lx = 0; lx < 4u; ++lx) {
                        const uint32_t index = ((by + ly) << 16) | ((bz + lz) << 8) | (bx + lx);
                        const uint32_t word = w->voxel[index];
                        const uint32_t ty = word & 0xFFu;
                        if (ty != 0u) {
                            const uint32_t life = (word >> 24) & 0xFFu;
                            const float temp_k = (float)((word >> 8) & 0xFFFFu) * 0.125f;
                            acc += (uint32_t)vox::voxel_mass(ty, life, w->aux_tmp[index], temp_k);
                        }
                    }
            w->grav_mass[cell] = (int32_t)((uint32_t)w->grav_mass[cell] + acc);
        }
    }
}

}  // extern "C"
