// field3d_cell.cuh -- the per-cell arithmetic of the 3-D field step
// (crates/tpt-sim/src/voxel3d/{air_kernel,gravity}.rs), shared by its forms.
// Include only from sources built with -fmad=false: every f32 operation is
// then rounded separately, in the reference kernels' order.
#pragma once

#include "common.cuh"
#include "exact_div.cuh"

namespace tpt {
namespace vox {

constexpr int N = 64;
constexpr int SZ = 64, SY = 4096;
constexpr int CELLS = N * N * N;

// air_kernel.rs:55-71, 328-331
constexpr float kAmbient = 293.15f;
constexpr float kBuoyancy = 0.02f;
constexpr float kDamping = 0.99f;
constexpr float kNbrW = 0.1f, kKeepNbr = 1.0f - kNbrW;
constexpr float kUpW = 0.25f, kKeepUp = 1.0f - kUpW;
constexpr float kMaxSpeed = 8.0f;
constexpr float kPvScale = 1024.0f;
constexpr float kMaxPvQ = 256.0f * 1024.0f;
// gravity.rs:55-59, 192
constexpr float kMassScaleInv = 1.0f / 1024.0f;
constexpr float kFourPiG = 8.385539f;
constexpr float kSixth = 1.0f / 6.0f;

// ------------------------------------------------------------ per cell ----

__device__ __forceinline__ float seed_f32(float anchor, float v) { return anchor * 0.0f + v; }  // step/mod.rs:371

__device__ __forceinline__ float clampf(float v, float lo, float hi) {  // step/mod.rs:425-435
    float out = v;
    if (out < lo) out = lo;
    if (out > hi) out = hi;
    return out;
}

__device__ __forceinline__ float clamp_speed(float v) {  // air_kernel.rs:80-91
    float out = v;
    if (out > kMaxSpeed) out = kMaxSpeed;
    if (out < -kMaxSpeed) out = -kMaxSpeed;
    return out;
}

// sum / count for the neighbour counts 4..7 of a six-neighbour average.
__device__ __forceinline__ float div_count(float sum, int count) {
    if (count == 7) return div_by_const(sum, 7.0f, 1.0f / 7.0f);
    if (count == 6) return div_by_const(sum, 6.0f, 1.0f / 6.0f);
    if (count == 5) return div_by_const(sum, 5.0f, 1.0f / 5.0f);
    return div_by_const(sum, 4.0f, 0.25f);
}

// The TPT pressure update of one cell (air_kernel.rs:294-326); `dp` is the
// six-neighbour velocity difference, used only off the two-cell rim.
__device__ __forceinline__ int32_t pv_update(int32_t value, bool rim, float dp) {
    if (rim) return __float2int_rz((float)value * 0.2f);
    const float mixed = (float)value * 0.9999f;
    const float next = mixed + dp * 0.3f * 0.5f * kPvScale;
    if (next > kMaxPvQ) return (int32_t)kMaxPvQ;
    if (next < -kMaxPvQ) return -(int32_t)kMaxPvQ;
    return __float2int_rz(next);
}

// One pressure Jacobi update (air_kernel.rs:382-395).
__device__ __forceinline__ float air_sweep_cell(float xm, float xp, float zm, float zp, float ym, float yp,
                                                float divergence, bool fixed) {
    const float nb = xm + xp + zm + zp + ym + yp;
    return fixed ? 0.0f : div_by_const(nb - divergence, 6.0f, kSixth);
}

// One potential Jacobi update (gravity.rs:183-194); `src` = 4*pi*G*rho.
__device__ __forceinline__ float grav_sweep_cell(float xm, float xp, float zm, float zp, float ym, float yp,
                                                 float src, float self, bool boundary) {
    const float sum = xm + xp + zm + zp + ym + yp;
    return boundary ? seed_f32(self, 0.0f) : (sum - src) * kSixth;
}

__device__ __forceinline__ float grav_source(int32_t mass) {
    return kFourPiG * ((float)mass * kMassScaleInv);
}

// Mean of a cell and its in-world neighbours in the reference's order
// (air_kernel.rs:99-135, 438-464).
__device__ __forceinline__ float nb_average(float c, float xm, float xp, float zm, float zp, float ym, float yp,
                                            int x, int y, int z) {
    float sum = c;
    int n = 1;
    if (x > 0) { sum += xm; ++n; }
    if (x + 1 < N) { sum += xp; ++n; }
    if (z > 0) { sum += zm; ++n; }
    if (z + 1 < N) { sum += zp; ++n; }
    if (y > 0) { sum += ym; ++n; }
    if (y + 1 < N) { sum += yp; ++n; }
    return div_count(sum, n);
}

// Donor-cell sample along `axis` (air_kernel.rs:142-176): lo / hi are the
// cell's neighbours below / above along that axis, `c` its coordinate.
__device__ __forceinline__ float upwind(float cur, float lo, float hi, int c) {
    float s = cur;
    if (cur > 0.0f) {
        if (c > 0) s = lo;
    } else if (cur < 0.0f) {
        if (c + 1 < N) s = hi;
    }
    return s;
}

// The advection update of one velocity component of one non-solid cell
// (air_kernel.rs:492-533): `c` the old value, the six neighbours of the old
// component, `grad` the pressure gradient along the component's axis, `buoy`
// the buoyancy (0 except for y).
__device__ __forceinline__ float advect_cell(float c, float xm, float xp, float zm, float zp, float ym, float yp,
                                             int axis, float grad, float buoy, int x, int y, int z) {
    float next = axis == 1 ? (c + buoy - grad) * kDamping : (c - grad) * kDamping;
    const float avg = nb_average(c, xm, xp, zm, zp, ym, yp, x, y, z);
    next = next * kKeepNbr + avg * kNbrW;
    float up;
    if (axis == 0) up = upwind(c, xm, xp, x);
    else if (axis == 1) up = upwind(c, ym, yp, y);
    else up = upwind(c, zm, zp, z);
    next = next * kKeepUp + up * kUpW;
    return clamp_speed(next);
}

// One-sided at the world faces, central inside (air_kernel.rs:466-494).
__device__ __forceinline__ float pressure_grad(float lo, float hi, float self, int c) {
    const float l = c > 0 ? lo : self, h = c + 1 < N ? hi : self;
    return (h - l) * 0.5f;
}

// Fixed-point mass of one voxel (gravity.rs:74-109), branch-free so a warp
// does not diverge on the element mix. Each element's case converts one
// integer to f32 and truncates one f32 product, so the integer the voxel's
// case needs (GRVT the clamped tmp, NBHL/NWHL tmp, GPMP the 16-bit
// temperature count) is picked first and converted once, the three f32
// expressions are evaluated from it, and the voxel's one is truncated once:
// two conversions per voxel instead of one per case. GRVT: clamp((float)tmp,
// -100, 100) truncated is the integer clamp of tmp (the f32 rounding of an
// integer beyond +-100 stays beyond it). NBHL/NWHL: the reference's seed
// value of `add` is 0.1 (the temperature is always finite). GPMP: temp_k is
// the count times 0.125.
__device__ __forceinline__ int32_t voxel_mass(uint32_t ty, uint32_t life, int32_t tmp, uint32_t temp_q) {
    const bool grvt = ty == 39u, hole = ty == 40u || ty == 41u;
    const int32_t src = grvt ? min(max(tmp, -100), 100) : hole ? tmp : (int32_t)temp_q;
    const float x = (float)src;
    const float fg = 0.2f * x * 1024.0f;  // GRVT
    float add = 0.1f;
    if (tmp != 0) add = clampf(0.001f * x, 0.1f, 51.2f);
    const float fh = (ty == 41u ? -add : add) * 1024.0f;  // NBHL, NWHL
    const float fp = 0.2f * (x * 0.125f - 273.15f) * 1024.0f;  // GPMP
    const int32_t r = __float2int_rz(grvt ? fg : hole ? fh : fp);
    const int32_t gbmb = life > 20u ? 20480 : (life >= 1u ? -81920 : 0);  // GBMB
    return (grvt || hole || (ty == 43u && life == 10u)) ? r : ty == 42u ? gbmb : 0;
}

__device__ __forceinline__ float f4(const float4 &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
__device__ __forceinline__ void f4set(float4 &v, int k, float s) {
    if (k == 0) v.x = s;
    else if (k == 1) v.y = s;
    else if (k == 2) v.z = s;
    else v.w = s;
}
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float4 zero4() { return make_float4(0.0f, 0.0f, 0.0f, 0.0f); }

__device__ __forceinline__ void coords(int i, int &x, int &y, int &z) {
    x = i & 63;
    z = (i >> 6) & 63;
    y = i >> 12;
}

}  // namespace vox
}  // namespace tpt
