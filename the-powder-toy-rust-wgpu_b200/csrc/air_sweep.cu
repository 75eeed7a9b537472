// air_sweep.cu -- the batched air tick as one launch of row sweeps.
//
// One CTA lane owns one grid column; the CTA walks down a strip of rows and
// runs the whole tick (crates/tpt-sim/src/air_kernel/mod.rs:150-263) as a
// software pipeline over the rows. At the step that loads row r it computes
//
//   lag 1  effective velocity   pressure.rs:119-158 (border mix, wall clear)
//   lag 2  pressure             pressure.rs:173-238
//   lag 3  velocity             pressure.rs:247-299
//   lag 4  vorticity            advect.rs:10-42
//   lag 5  smooth/advect/fans   advect.rs:174-360, and the wall masks of the
//                               row (settle.rs:50-93)
//   lag 7  heat/convection      heat.rs:29-253
//
// so every row of every stage is computed once per column. A stage reads its
// x neighbours (columns c-1, c+1) from small per-stage row rings in shared
// memory and its y neighbours from the lane's own registers; one barrier per
// row step publishes the rings. Nothing between the passes touches DRAM: a
// tick reads the state (pv, vx, vy, hv, masks) once and writes it once, into
// the other half of a ping-pong pair, so no CTA overwrites a cell another CTA
// may still read. Each stage is predicated by the rows its consumers need, so
// a strip of `ny` output rows computes ny + 2k rows of a stage with halo k.
//
// The rings cover a window of rows and the CTA's lanes. A far-advection walk
// or bilinear sample outside that window reads global memory instead: the
// walks and the heat samples read the tick's input masks and heat, which no
// CTA writes during the launch; a velocity sample needs the velocity pass's
// output (ovx/ovy) at an arbitrary cell, which this launch does not store. For
// that, an instance whose previous tick had such a sample gets its ovx/ovy
// written by a pre-pass before this launch (kb_sweep_prepass in air_batch.cu,
// flagged per instance), and any remaining sample recomputes the four corners pointwise
// from the input state (the same arithmetic, bit for bit). Both paths give the
// reference's values; the flag only decides which one is cheaper.
//
// Narrow instances waste most lanes of a wide CTA, so one work item packs up
// to SW_MAXSEG segments side by side: each segment is a column strip of one
// instance with its own SW_H-lane halos on both sides. CTAs take items from
// an atomic work queue, largest first.
//
// Compiled with -fmad=false: see air.cuh. The f32 -> i32 conversions ((int)
// casts, cvt.rzi) round toward zero, saturate, and give 0 for NaN.
#include <cuda.h>

#include "air.cuh"
#include "air_launch.hpp"

namespace tpt {
namespace air {

// Ring depths (rows, powers of two) and their offsets (in rows of NL + 2
// words) inside the dynamic shared memory.
constexpr int RG_HIST = 2, RG_EVX = 2, RG_OPV = 8, RG_OV = 8, RG_VORT = 2, RG_NV = 4, RG_HV = 4;
constexpr int OFF_HIST = 0;
constexpr int OFF_EVX = OFF_HIST + RG_HIST;
constexpr int OFF_OPV = OFF_EVX + RG_EVX;
constexpr int OFF_OVX = OFF_OPV + RG_OPV;
constexpr int OFF_OVY = OFF_OVX + RG_OV;
constexpr int OFF_VORT = OFF_OVY + RG_OV;
constexpr int OFF_NVX = OFF_VORT + RG_VORT;
constexpr int OFF_NVY = OFF_NVX + RG_NV;
constexpr int OFF_HV = OFF_NVY + RG_NV;
constexpr int RG_ROWS = OFF_HV + RG_HV;
static_assert(RG_ROWS == SWEEP_RING_ROWS, "ring layout and its host-side size disagree");

// Row `q` (relative to the strip's first output row) of ring `off`/`depth`,
// as a pointer to lane 0 (index -1 is the left pad, NL the right pad).
__device__ __forceinline__ float *ring(float *sm, int off, int depth, int q, int P) {
    return sm + (off + (q & (depth - 1))) * P + 1;
}

// ---- pointwise velocity pass from the input state (global memory) ------------
// The same arithmetic as the sweep's stages (and pass_a), evaluated at one
// cell from the tick's input grids: used for a velocity sample that lies
// outside the rings when no pre-pass ran for the instance this tick.
__device__ __forceinline__ bool blk_g(const AirInst &I, int x, int y) {
    return x >= 0 && y >= 0 && x < (int)I.X && y < (int)I.Y && __ldg(I.bair + (size_t)y * I.pitch + x) != 0u;
}
__device__ float evx_g(const AirInst &I, int x, int y) {
    const uint32_t X = I.X, Y = I.Y;
    float v = __ldg(I.vx + (size_t)y * I.pitch + x);
    if (in_border(x, y, X, Y)) v = I.evx + (v - I.evx) * 0.9f;
    bool cl = false;
    if (y >= 1 && (uint32_t)y + 1u < Y) {
        if (x >= 1 && (uint32_t)x + 1u < X && blk_g(I, x, y)) cl = true;
        if (x >= 2 && blk_g(I, x - 1, y)) cl = true;
        if ((uint32_t)x + 2u < X && blk_g(I, x + 1, y)) cl = true;
    }
    return cl ? 0.0f : v;
}
__device__ float evy_g(const AirInst &I, int x, int y) {
    const uint32_t X = I.X, Y = I.Y;
    float v = __ldg(I.vy + (size_t)y * I.pitch + x);
    if (in_border(x, y, X, Y)) v = I.evy + (v - I.evy) * 0.9f;
    bool cl = false;
    if (x >= 1 && (uint32_t)x + 1u < X) {
        if (y >= 1 && (uint32_t)y + 1u < Y && blk_g(I, x, y)) cl = true;
        if (y >= 2 && blk_g(I, x, y - 1)) cl = true;
        if ((uint32_t)y + 2u < Y && blk_g(I, x, y + 1)) cl = true;
    }
    return cl ? 0.0f : v;
}
__device__ float opv_g(const AirInst &I, int x, int y) {
    float cur = __ldg(I.pv + (size_t)y * I.pitch + x);
    if (in_border(x, y, I.X, I.Y)) cur = I.ep + (cur - I.ep) * 0.8f;
    float next = cur;
    if (interior(x, y, I.X, I.Y)) {
        float dp = evx_g(I, x - 1, y) - evx_g(I, x + 1, y) + evy_g(I, x, y - 1) - evy_g(I, x, y + 1);
        next = I.ep + (cur - I.ep) * 0.9999f + dp * 0.15f;
    }
    return next;
}
// ovx and ovy of cell (x, y), which the callers keep in 2..X-3 x 2..Y-3.
__device__ void ov_g(const AirInst &I, int x, int y, float &ox, float &oy) {
    float nx = evx_g(I, x, y), ny = evy_g(I, x, y);
    if (interior(x, y, I.X, I.Y)) {
        float dx = opv_g(I, x - 1, y) - opv_g(I, x + 1, y);
        float dy = opv_g(I, x, y - 1) - opv_g(I, x, y + 1);
        nx = I.evx + (nx - I.evx) * 0.999f + dx * 0.2f;
        ny = I.evy + (ny - I.evy) * 0.999f + dy * 0.2f;
        if (blk_g(I, x - 1, y) || blk_g(I, x, y) || blk_g(I, x + 1, y)) nx = 0.0f;
        if (blk_g(I, x, y - 1) || blk_g(I, x, y) || blk_g(I, x, y + 1)) ny = 0.0f;
    }
    ox = nx;
    oy = ny;
}

// ---- the sweep -------------------------------------------------------------------
// Lane registers of one segment (constant over the item).
struct Lane {
    const AirInst *I;
    int c;           // grid column of the lane
    int X, Y, pitch;
    int y0, ny;      // output rows of the segment
    int lo, hi;      // the segment's lanes [lo, hi)
    int col0;        // lane of column 0 (lane of column cx is col0 + cx)
    bool act;        // the lane belongs to a segment
    bool colok;      // ... and its column lies in the grid
    bool out;        // ... and is an output column
};

__global__ void __launch_bounds__(SWEEP_MAX_LANES, 2) kb_air_sweep(const AirInst *__restrict__ insts,
                                                               const SweepItem *__restrict__ items,
                                                               uint32_t nitems, uint32_t parity, uint32_t ninst,
                                                               uint32_t *__restrict__ ctl, uint32_t *__restrict__ want) {
    extern __shared__ float sm[];
    __shared__ SweepItem s_it;
    // the item's segments' instance parameters: read from shared memory, which
    // the kernel's global stores cannot alias, so they are never reloaded from
    // global memory after a store
    __shared__ AirInst s_inst[SW_MAXSEG];
    __shared__ uint32_t s_next;
    uint32_t *smu = reinterpret_cast<uint32_t *>(sm);
    const int NL = (int)blockDim.x, P = NL + 2, l = (int)threadIdx.x;

    for (;;) {
        if (l == 0) s_next = atomicAdd(&ctl[0], 1u);
        __syncthreads();
        const uint32_t it = s_next;
        if (it >= nitems) break;
        {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(items + it);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&s_it);
            for (int k = l; k < (int)(sizeof(SweepItem) / 4); k += NL) dst[k] = __ldg(src + k);
        }
        __syncthreads();
        {
            constexpr int W = (int)(sizeof(AirInst) / 4);
            uint32_t *dst = reinterpret_cast<uint32_t *>(s_inst);
            for (int k = l; k < (int)s_it.nseg * W; k += NL) {
                const int sg = k / W, w = k - sg * W;
                dst[k] = __ldg(reinterpret_cast<const uint32_t *>(insts + 2 * (size_t)s_it.seg[sg].inst + parity) + w);
            }
        }
        __syncthreads();

        // ---- this lane's segment
        Lane L{};
        int seg = -1;
        for (int k = 0; k < (int)s_it.nseg; ++k)
            if (l >= (int)s_it.seg[k].lane0 && l < (int)s_it.seg[k].lane0 + (int)s_it.seg[k].lanes) seg = k;
        uint32_t inst = 0;
        if (seg >= 0) {
            const SweepSeg S = s_it.seg[seg];
            inst = S.inst;
            L.I = &s_inst[seg];
            L.X = (int)L.I->X;
            L.Y = (int)L.I->Y;
            L.pitch = (int)L.I->pitch;
            L.lo = S.lane0;
            L.hi = S.lane0 + S.lanes;
            L.col0 = (int)S.lane0 + SW_H - (int)S.x0;
            L.c = l - L.col0;
            L.y0 = S.y0;
            L.ny = S.ny;
            L.act = true;
            L.colok = L.c >= 0 && L.c < L.X;
            L.out = (l - (int)S.lane0) >= SW_H && (l - (int)S.lane0) < SW_H + (int)S.nx;
        } else {
            L.I = &s_inst[0];  // any valid pointer; every access below is predicated off
            L.lo = L.hi = 0;
            L.y0 = 0;
            L.ny = -100;  // no stage row range is ever entered
        }
        const AirInst &I = *L.I;
        const bool upd = L.act && I.air_mode != 4u;
        const bool aheat = L.act && I.aheat != 0u;
        const bool vort_on = upd && I.vcoef > 0.0f;
        const bool have_ov = L.act && want[(size_t)parity * ninst + inst] != 0u;
        const float ep = I.ep, e0x = I.evx, e0y = I.evy;
        const int c = L.c, X = L.X, Y = L.Y, ny = L.ny;
        bool far_seen = false;

        uint32_t hb = 0, hh = 0;  // block_air rows r, r-1, ... (bit j = row r-j); block_airh&8 rows r-5, r-6, ...
        float pv0 = 0.f, pv1 = 0.f, pv2 = 0.f, vx1 = 0.f, vy1 = 0.f;
        float evx1 = 0.f, evx2 = 0.f, evx3 = 0.f, evy1 = 0.f, evy2 = 0.f, evy3 = 0.f;
        float opv2 = 0.f, opv3 = 0.f, opv4 = 0.f;
        float ovx3 = 0.f, ovx4 = 0.f, ovx5 = 0.f;
        float vt4 = 0.f, vt5 = 0.f, vt6 = 0.f;
        float vx0 = 0.f, vy0 = 0.f;

        // The loads of a step's rows are issued one step ahead (the previous
        // step's compute hides their latency): row r of block_air and, while
        // the velocity pass runs, pv/vx/vy (NoUpdate: pv/vx/vy of row r - 5,
        // which that mode uses directly); row r - 5 of block_airh, walls and
        // heat.
        uint32_t n_b = 0u, n_bh = 0u, n_wall = 0u, n_emap = 0u, n_ea = 0u, n_eh = 0u;
        float n_pv = 0.f, n_vx = 0.f, n_vy = 0.f, n_hv = 0.f;
        auto issue_loads = [&](int rload) {
            const int rhl = rload - 5, rv = upd ? rload : rhl;
            n_b = 0u;
            n_bh = 0u;
            n_wall = 0u;
            n_emap = n_ea = n_eh = 0u;
            n_pv = n_vx = n_vy = n_hv = 0.f;
            if (L.colok && rload >= 0 && rload < Y) n_b = __ldg(I.bair + (size_t)rload * L.pitch + c) != 0u ? 1u : 0u;
            if (L.colok && rv >= 0 && rv < Y) {
                const size_t g = (size_t)rv * L.pitch + c;
                n_pv = __ldg(I.pv + g);
                n_vx = __ldg(I.vx + g);
                n_vy = __ldg(I.vy + g);
            }
            if (L.colok && rhl >= 0 && rhl < Y) {
                const size_t g = (size_t)rhl * L.pitch + c;
                n_bh = (__ldg(I.bairh + g) & 0x8u) != 0u ? 1u : 0u;
                n_wall = __ldg(I.wall + g);
                if (aheat) n_hv = __ldg(I.hv + g);
                if (L.out) {  // the mask rebuild's inputs (own cell, output columns)
                    n_emap = I.emap[g];
                    n_ea = I.eair ? __ldg(I.eair + g) : 0u;
                    n_eh = I.eairh ? __ldg(I.eairh + g) : 0u;
                }
            }
        };
        issue_loads(L.y0 - 6);

        const int steps = (int)s_it.steps;
        for (int rr = -6; rr <= steps + 6; ++rr) {
            const int r = L.y0 + rr;  // row loaded at this step
            const int rh = r - 5;     // row of the smoothing stage, the heat loads and the masks
            // ---- this step's loaded values, then the next step's loads
            const uint32_t lb = n_b, lbh = n_bh, lwall = n_wall, lemap = n_emap, lea = n_ea, leh = n_eh;
            const float lhv = n_hv, cpv = n_pv, cvx = n_vx, cvy = n_vy;
            issue_loads(r + 1);
            pv2 = pv1;
            pv1 = pv0;
            pv0 = cpv;
            vx1 = vx0;
            vy1 = vy0;
            vx0 = cvx;
            vy0 = cvy;
            const bool hok = L.colok && rh >= 0 && rh < Y;
            const size_t gh = (size_t)(hok ? rh : 0) * L.pitch + (hok ? c : 0);
            hb = (hb << 1) | lb;
            hh = (hh << 1) | lbh;
            smu[(OFF_HIST + (rr & 1)) * P + l + 1] = (hb & 0xFFFFu) | (hh << 16);
            const uint32_t *hp = smu + (OFF_HIST + ((rr - 1) & 1)) * P + 1;  // previous step's words
            if (aheat) ring(sm, OFF_HV, RG_HV, rr - 5, P)[l] = lhv;

            // ---- lag 1: effective velocity (pressure.rs:119-158) of row a = r - 1
            evx3 = evx2;
            evx2 = evx1;
            evy3 = evy2;
            evy2 = evy1;
            if (upd && rr - 1 >= -5 && rr - 1 < ny + 5) {
                const int a = r - 1;
                const bool bc = (hb >> 1) & 1u, bu = (hb >> 2) & 1u, bd = hb & 1u;
                const bool bl = hp[l - 1] & 1u, br = hp[l + 1] & 1u;
                float ex = vx1, ey = vy1;
                if (in_border(c, a, X, Y)) {
                    ex = e0x + (ex - e0x) * 0.9f;
                    ey = e0y + (ey - e0y) * 0.9f;
                }
                if (a >= 1 && a + 1 < Y && ((c >= 1 && c + 1 < X && bc) || (c >= 2 && bl) || (c + 2 < X && br)))
                    ex = 0.0f;
                if (c >= 1 && c + 1 < X && ((a >= 1 && a + 1 < Y && bc) || (a >= 2 && bu) || (a + 2 < Y && bd)))
                    ey = 0.0f;
                evx1 = ex;
                evy1 = ey;
                ring(sm, OFF_EVX, RG_EVX, rr - 1, P)[l] = ex;
            }

            // ---- lag 2: pressure (pressure.rs:173-238) of row a = r - 2
            opv4 = opv3;
            opv3 = opv2;
            if (upd && rr - 2 >= -4 && rr - 2 < ny + 4) {
                const int a = r - 2;
                float cur = pv2;
                if (in_border(c, a, X, Y)) cur = ep + (cur - ep) * 0.8f;
                float next = cur;
                if (interior(c, a, X, Y)) {
                    const float *ev = ring(sm, OFF_EVX, RG_EVX, rr - 2, P);
                    float dp = ev[l - 1] - ev[l + 1] + evy3 - evy1;
                    next = ep + (cur - ep) * 0.9999f + dp * 0.15f;
                }
                opv2 = next;
                ring(sm, OFF_OPV, RG_OPV, rr - 2, P)[l] = next;
            }

            // ---- lag 3: velocity (pressure.rs:247-299) of row a = r - 3
            ovx5 = ovx4;
            ovx4 = ovx3;
            if (upd && rr - 3 >= -3 && rr - 3 < ny + 3) {
                const int a = r - 3;
                float nx = evx3, nyv = evy3;
                if (interior(c, a, X, Y)) {
                    const float *op = ring(sm, OFF_OPV, RG_OPV, rr - 3, P);
                    float dx = op[l - 1] - op[l + 1];
                    float dy = opv4 - opv2;
                    nx = e0x + (evx3 - e0x) * 0.999f + dx * 0.2f;
                    nyv = e0y + (evy3 - e0y) * 0.999f + dy * 0.2f;
                    // adjacent_blocked_x/y (pressure.rs:92-114): rows a-1, a, a+1 = own bits 4, 3, 2
                    if (((hp[l - 1] >> 2) & 1u) || ((hb >> 3) & 1u) || ((hp[l + 1] >> 2) & 1u)) nx = 0.0f;
                    if ((hb >> 2) & 7u) nyv = 0.0f;
                }
                ovx3 = nx;
                ring(sm, OFF_OVX, RG_OV, rr - 3, P)[l] = nx;
                ring(sm, OFF_OVY, RG_OV, rr - 3, P)[l] = nyv;
            }

            // ---- lag 4: vorticity (advect.rs:10-42) of row a = r - 4
            vt6 = vt5;
            vt5 = vt4;
            if (vort_on && rr - 4 >= -2 && rr - 4 < ny + 2) {
                const int a = r - 4;
                float v = 0.0f;
                if (c > 1 && c + 2 < X && a > 1 && a + 2 < Y) {
                    const bool here = (hb >> 4) & 1u;
                    const float *oy = ring(sm, OFF_OVY, RG_OV, rr - 4, P);
                    float dvydx = oy[l + 1] - oy[l - 1];
                    if (here || ((hp[l + 1] >> 3) & 1u) || ((hp[l - 1] >> 3) & 1u)) dvydx = 0.0f;
                    float dvxdy = ovx3 - ovx5;
                    if (here || ((hb >> 3) & 1u) || ((hb >> 5) & 1u)) dvxdy = 0.0f;
                    v = (dvydx - dvxdy) * 0.5f;
                }
                vt4 = v;
                ring(sm, OFF_VORT, RG_VORT, rr - 4, P)[l] = v;
            }

            // ---- lag 5: smoothing, advection, vorticity confinement, fans (advect.rs:174-360)
            const int q5 = rr - 5;
            if (L.act && q5 >= (aheat ? -1 : 0) && q5 < ny + (aheat ? 1 : 0)) {
                const int a = rh;
                float nvx, nvy, npv;
                if (upd) {
                    const float *ox[3], *oy[3], *op[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        ox[k] = ring(sm, OFF_OVX, RG_OV, q5 - 1 + k, P);
                        oy[k] = ring(sm, OFF_OVY, RG_OV, q5 - 1 + k, P);
                        op[k] = ring(sm, OFF_OPV, RG_OPV, q5 - 1 + k, P);
                    }
                    const float cvx = ox[1][l], cvy = oy[1][l], cpv = op[1][l];
                    const bool xok[3] = {c - 1 >= 1 && c < X, c >= 1 && c + 1 < X, c + 1 >= 1 && c + 2 < X};
                    const bool yok[3] = {a - 1 >= 1 && a < Y, a >= 1 && a + 1 < Y, a + 1 >= 1 && a + 2 < Y};
                    float sx = 0.0f, sy = 0.0f, sp = 0.0f;
#pragma unroll
                    for (int dyy = 0; dyy < 3; ++dyy) {
#pragma unroll
                        for (int dxx = 0; dxx < 3; ++dxx) {
                            const int ln = l + dxx - 1;
                            // block_air of (c + dxx - 1, a + dyy - 1): previous-step word bit 5 - dyy
                            const bool open = xok[dxx] && yok[dyy] && !((hp[ln] >> (5 - dyy)) & 1u);
                            const float w = smooth_w(dxx, dyy);
                            const float tx = open ? ox[dyy][ln] : cvx;
                            const float ty = open ? oy[dyy][ln] : cvy;
                            const float tp = open ? op[dyy][ln] : cpv;
                            sx += tx * w;
                            sy += ty * w;
                            sp += tp * w;
                        }
                    }
                    nvx = div_by_const(sx, kSmoothWsum, kSmoothWsumRcp);
                    nvy = div_by_const(sy, kSmoothWsum, kSmoothWsumRcp);
                    npv = div_by_const(sp, kSmoothWsum, kSmoothWsumRcp);

                    float tx0, ty0;
                    far_advect_target(
                        c, a, nvx, nvy,
                        [&](int cx, int cy) -> bool {
                            const int ln = L.col0 + cx;
                            if (ln >= L.lo && ln < L.hi && cy <= r - 1 && cy >= r - 16 && cy >= L.y0 - 6)
                                return (hp[ln] >> (r - 1 - cy)) & 1u;
                            return __ldg(I.bair + (size_t)cy * L.pitch + cx) != 0u;
                        },
                        X, Y, tx0, ty0);
                    const int i0 = (int)tx0, j0 = (int)ty0;
                    const float fx = tx0 - (float)i0, fy = ty0 - (float)j0;
                    if (!((hb >> 5) & 1u) && i0 >= 2 && i0 < X - 3 && j0 >= 2 && j0 < Y - 3 && fx >= 0.0f &&
                        fy >= 0.0f) {
                        const float w00 = (1.0f - fx) * (1.0f - fy);
                        const float w10 = fx * (1.0f - fy);
                        const float w01 = (1.0f - fx) * fy;
                        const float w11 = fx * fy;
                        float a00, a10, a01, a11, b00, b10, b01, b11;
                        const int l0 = L.col0 + i0, qj = j0 - L.y0;
                        // ovx/ovy rows visible in the rings: written by earlier steps
                        // (rows <= r - 4), not yet overwritten (rows >= r - 10), and
                        // computed for this strip (relative rows >= -3); columns whose
                        // velocity pass had both neighbours (3 lanes in from the edges)
                        if (l0 >= L.lo + 3 && l0 + 1 < L.hi - 3 && j0 >= r - 10 && j0 + 1 <= r - 4 && qj >= -3) {
                            const float *x0r = ring(sm, OFF_OVX, RG_OV, qj, P), *x1r = ring(sm, OFF_OVX, RG_OV, qj + 1, P);
                            const float *y0r = ring(sm, OFF_OVY, RG_OV, qj, P), *y1r = ring(sm, OFF_OVY, RG_OV, qj + 1, P);
                            a00 = x0r[l0];
                            a10 = x0r[l0 + 1];
                            a01 = x1r[l0];
                            a11 = x1r[l0 + 1];
                            b00 = y0r[l0];
                            b10 = y0r[l0 + 1];
                            b01 = y1r[l0];
                            b11 = y1r[l0 + 1];
                        } else if (have_ov) {  // the pre-pass wrote this tick's ovx/ovy
                            far_seen = true;
                            const size_t r0 = (size_t)j0 * L.pitch + i0, r1 = r0 + L.pitch;
                            a00 = __ldg(I.ovx + r0);
                            a10 = __ldg(I.ovx + r0 + 1);
                            a01 = __ldg(I.ovx + r1);
                            a11 = __ldg(I.ovx + r1 + 1);
                            b00 = __ldg(I.ovy + r0);
                            b10 = __ldg(I.ovy + r0 + 1);
                            b01 = __ldg(I.ovy + r1);
                            b11 = __ldg(I.ovy + r1 + 1);
                        } else {
                            far_seen = true;
                            ov_g(I, i0, j0, a00, b00);
                            ov_g(I, i0 + 1, j0, a10, b10);
                            ov_g(I, i0, j0 + 1, a01, b01);
                            ov_g(I, i0 + 1, j0 + 1, a11, b11);
                        }
                        nvx = nvx * 0.7f + 0.3f * (a00 * w00 + a10 * w10 + a01 * w01 + a11 * w11);
                        nvy = nvy * 0.7f + 0.3f * (b00 * w00 + b10 * w10 + b01 * w01 + b11 * w11);
                    }
                    if (vort_on && c > 1 && c + 2 < X && a > 1 && a + 2 < Y) {  // advect.rs:297-328
                        const float *vr = ring(sm, OFF_VORT, RG_VORT, q5, P);
                        float w = vt5;
                        float wxp = vr[l + 1];
                        float wxm = vr[l - 1];
                        float wyp = vt4;
                        float wym = vt6;
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
                    if (lwall == 5u) {  // WL_FAN, advect.rs:331-334
                        nvx += __ldg(I.fvx + gh);
                        nvy += __ldg(I.fvy + gh);
                    }
                    nvx = clampf(nvx, -256.0f, 256.0f);
                    nvy = clampf(nvy, -256.0f, 256.0f);
                    npv = clampf(npv, -256.0f, 256.0f);
                    if (I.air_mode == 1u) npv = 0.0f;
                    if (I.air_mode == 2u) {
                        nvx = 0.0f;
                        nvy = 0.0f;
                    }
                    if (I.air_mode == 3u) {
                        nvx = 0.0f;
                        nvy = 0.0f;
                        npv = 0.0f;
                    }
                } else {  // NoUpdate (mod.rs:150): the stored velocity and pressure of row r - 5
                    nvx = cvx;
                    nvy = cvy;
                    npv = cpv;
                }
                ring(sm, OFF_NVX, RG_NV, q5, P)[l] = nvx;
                ring(sm, OFF_NVY, RG_NV, q5, P)[l] = nvy;
                if (L.out && q5 >= 0 && q5 < ny) {
                    I.pv_out[gh] = npv;
                    if (!aheat) {
                        I.vx_out[gh] = nvx;
                        I.vy_out[gh] = nvy;
                    }
                    // settle.rs:50-93: emap decay and the masks the next tick reads
                    uint32_t ba, bh;
                    masks_of(lwall, lemap, lea, leh, ba, bh);
                    if (lemap != 0u) I.emap[gh] = lemap - 1u;
                    I.bair_out[gh] = ba;
                    I.bairh_out[gh] = bh;
                }
            }

            // ---- lag 7: ambient heat and convection (heat.rs:29-253) of row a = r - 7
            const int q7 = rr - 7;
            if (aheat && q7 >= 0 && q7 < ny) {
                const int a = r - 7;
                const float *hr[3], *xr[3], *yr[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    hr[k] = ring(sm, OFF_HV, RG_HV, q7 - 1 + k, P);
                    xr[k] = ring(sm, OFF_NVX, RG_NV, q7 - 1 + k, P);
                    yr[k] = ring(sm, OFF_NVY, RG_NV, q7 - 1 + k, P);
                }
                const float ch = hr[1][l], cvx = xr[1][l], cvy = yr[1][l];
                const bool xok[3] = {c - 1 >= 1 && c < X, c >= 1 && c + 1 < X, c + 1 >= 1 && c + 2 < X};
                const bool yok[3] = {a - 1 >= 1 && a < Y, a >= 1 && a + 1 < Y, a + 1 >= 1 && a + 2 < Y};
                float sh = 0.0f, sx = 0.0f, sy = 0.0f;
#pragma unroll
                for (int dyy = 0; dyy < 3; ++dyy) {
#pragma unroll
                    for (int dxx = 0; dxx < 3; ++dxx) {
                        const int ln = l + dxx - 1;
                        // block_airh & 0x8 of (c + dxx - 1, a + dyy - 1): previous-step word bit 18 - dyy
                        const bool open = xok[dxx] && yok[dyy] && !((hp[ln] >> (18 - dyy)) & 1u);
                        const float w = smooth_w(dxx, dyy);
                        const float th = open ? hr[dyy][ln] : ch;
                        const float tx = open ? xr[dyy][ln] : cvx;
                        const float ty = open ? yr[dyy][ln] : cvy;
                        sh += th * w;
                        sx += tx * w;
                        sy += ty * w;
                    }
                }
                float dh = div_by_const(sh, kSmoothWsum, kSmoothWsumRcp);
                const float svx = div_by_const(sx, kSmoothWsum, kSmoothWsumRcp);
                const float svy = div_by_const(sy, kSmoothWsum, kSmoothWsumRcp);
                float tx, ty;
                far_advect_target(
                    c, a, svx, svy,
                    [&](int cx, int cy) -> bool {
                        const int ln = L.col0 + cx;
                        if (ln >= L.lo && ln < L.hi && cy <= r - 6 && cy >= r - 21 && cy >= L.y0 - 11)
                            return (hp[ln] >> (16 + r - 6 - cy)) & 1u;
                        return (__ldg(I.bairh + (size_t)cy * L.pitch + cx) & 0x8u) != 0u;
                    },
                    X, Y, tx, ty);
                const int i0 = (int)tx, j0 = (int)ty;
                const float fx = tx - (float)i0, fy = ty - (float)j0;
                const bool here_blocked = (hh >> 2) & 1u;
                if (!here_blocked && i0 >= 0 && i0 < X - 1 && j0 >= 0 && j0 < Y - 1 && fx >= 0.0f && fy >= 0.0f) {
                    float s00, s10, s01, s11;
                    const int l0 = L.col0 + i0, qj = j0 - L.y0;
                    // hv rows in the ring: r - 8 .. r - 6 (loaded by earlier steps)
                    if (l0 >= L.lo && l0 + 1 < L.hi && j0 >= r - 8 && j0 + 1 <= r - 6) {
                        const float *h0 = ring(sm, OFF_HV, RG_HV, qj, P), *h1 = ring(sm, OFF_HV, RG_HV, qj + 1, P);
                        const int b0 = 16 + r - 6 - j0;  // bit of row j0 in the words (row j0 + 1: b0 - 1)
                        s00 = ((hp[l0] >> b0) & 1u) ? dh : h0[l0];
                        s10 = ((hp[l0 + 1] >> b0) & 1u) ? dh : h0[l0 + 1];
                        s01 = ((hp[l0] >> (b0 - 1)) & 1u) ? dh : h1[l0];
                        s11 = ((hp[l0 + 1] >> (b0 - 1)) & 1u) ? dh : h1[l0 + 1];
                    } else {
                        const size_t r0 = (size_t)j0 * L.pitch + i0, r1 = r0 + L.pitch;
                        s00 = (__ldg(I.bairh + r0) & 0x8u) ? dh : __ldg(I.hv + r0);
                        s10 = (__ldg(I.bairh + r0 + 1) & 0x8u) ? dh : __ldg(I.hv + r0 + 1);
                        s01 = (__ldg(I.bairh + r1) & 0x8u) ? dh : __ldg(I.hv + r1);
                        s11 = (__ldg(I.bairh + r1 + 1) & 0x8u) ? dh : __ldg(I.hv + r1 + 1);
                    }
                    const float w00 = (1.0f - fx) * (1.0f - fy);
                    const float w10 = fx * (1.0f - fy);
                    const float w01 = (1.0f - fx) * fy;
                    const float w11 = fx * fy;
                    dh = dh * 0.7f + 0.3f * (s00 * w00 + s10 * w10 + s01 * w01 + s11 * w11);
                }
                if (here_blocked) dh = ch;
                dh = clampf(dh, 0.0f, 9999.0f);
                if (c < 2 || a < 2 || c + 2 >= X || a + 2 >= Y) dh = I.amb;

                float ovx = cvx, ovy = cvy;
                if (c >= 2 && c + 2 < X && a >= 2 && a + 2 < Y) {
                    float gxv = 0.0f, gyv = 0.0f;
                    if (I.gmode == 0u) {
                        gyv = 1.0f;
                    } else if (I.gmode == 2u) {
                        float rx = (float)X * 0.5f - ((float)c + 0.5f);
                        float ry = (float)Y * 0.5f - ((float)a + 0.5f);
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
                    float nx = cvx, nyv = cvy;
                    if (I.conv == 1u) {
                        float weight = div_by_const((ch - hr[1][l - 1]) * convx + (ch - hr[0][l]) * convy,
                                                    kConvLegacy, kConvLegacyRcp);
                        if (weight > 0.0f && !((hh >> 3) & 1u)) {
                            nx += weight * convx;
                            nyv += weight * convy;
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
                        nyv += weight * convy;
                    }
                    ovx = clampf(nx, -256.0f, 256.0f);
                    ovy = clampf(nyv, -256.0f, 256.0f);
                }
                if (L.out) {
                    const size_t g7 = (size_t)a * L.pitch + c;
                    I.hv_out[g7] = dh;
                    I.vx_out[g7] = ovx;
                    I.vy_out[g7] = ovy;
                }
            }
            __syncthreads();
        }
        // an instance with a velocity sample outside the rings gets the pre-pass next tick
        if (far_seen) atomicOr(&want[(size_t)(parity ^ 1u) * ninst + inst], 1u);
    }
}

int launch_sweep_tick(const SweepLaunch &s, uint32_t parity, cudaStream_t st) {
    int rc = launch_prepass(s, parity, st);  // air_batch.cu: flags, queue reset, far-sample velocity
    if (rc) return rc;
    const size_t smem = (size_t)SWEEP_RING_ROWS * (s.lanes + 2) * sizeof(float);
    kb_air_sweep<<<s.grid, s.lanes, smem, st>>>(s.insts, s.items, s.nitems, parity, s.ninst, s.ctl, s.want);
    TPT_LAUNCHED();
    return TPT_OK;
}

int sweep_max_ctas_per_sm(uint32_t lanes, int *out) {
    const size_t smem = (size_t)SWEEP_RING_ROWS * (lanes + 2) * sizeof(float);
    TPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, kb_air_sweep, (int)lanes, smem));
    return TPT_OK;
}

}  // namespace air
}  // namespace tpt
