// field3d.cu -- the 3-D sandbox's coarse field step on sm_100a: the 64^3 air
// solve and the Jacobi Poisson gravity of crates/tpt-sim/src/voxel3d
// ({air,air_kernel,gravity}.rs), and the two brick gathers that feed them.
//
// Grid: 64^3 cells, index (y << 12) | (z << 6) | x; one field is 1 MiB.
// Voxels: 256^3 u32 words, index (y << 16) | (z << 8) | x. Bricks: 8^3
// voxels = 2x2x2 cells, id (by << 10) | (bz << 5) | bx.
//
// Cluster form (the product path). One cluster of 16 CTAs x 1024 threads
// owns one field of one world for a whole solve: CTA r keeps y-planes
// 4r..4r+3 of the Jacobi pair in its shared memory (2 x 64 KiB) and reads
// the neighbouring planes of CTAs r-1 / r+1 through distributed shared
// memory. The per-cell source of the sweep (the air divergence, the gravity
// 4*pi*G*rho) lives in registers, so a sweep reads three float4 and writes
// one per thread and plane, and `cluster.sync()` (the hardware cluster
// barrier) separates the sweeps. Air and gravity clusters of any number of
// worlds run side by side in one launch. Thread t owns the x-quad
// 4*(t & 15) .. +3 of row z = t >> 4 on each of its CTA's four planes; the
// x neighbours outside the quad come from the adjacent lanes (shuffles).
//
// Per-sweep form: one launch per reference pass and per sweep, the
// reference's own launch structure, over global memory.
//
// Both forms use the same per-cell arithmetic below and are built with
// -fmad=false: every f32 operation is rounded separately, in the reference
// kernels' order, so results are bit-identical to the reference arithmetic.
#include <cooperative_groups.h>

#include "common.cuh"
#include "exact_div.cuh"
#include "field3d.hpp"

namespace cg = cooperative_groups;

namespace tpt {
namespace vox {

constexpr int N = 64;
constexpr int SZ = 64, SY = 4096;
constexpr int CELLS = N * N * N;
constexpr int CL = 16;            // CTAs per cluster
constexpr int PL = N / CL;        // y planes per CTA
constexpr int ROWS = 2;           // z rows per thread
constexpr int THREADS = (N / 4) * (N / ROWS);  // one thread per x-quad and row pair
constexpr int PLANE = N * N;      // floats per plane
constexpr int SLAB = PL * PLANE;  // floats per CTA slab
constexpr size_t CLUSTER_SMEM = 3 * SLAB * sizeof(float);
static_assert(ROWS * PL * 4 <= 32, "a thread's cells fit one 32-bit mask");

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

// Fixed-point mass of one voxel (gravity.rs:74-109).
__device__ __forceinline__ int32_t voxel_mass(uint32_t ty, uint32_t life, int32_t tmp, float temp_k) {
    int32_t out = 0;
    if (ty == 39u) {  // GRVT
        const int32_t t = __float2int_rz(clampf((float)tmp, -100.0f, 100.0f));
        out = __float2int_rz(0.2f * (float)t * 1024.0f);
    } else if (ty == 40u || ty == 41u) {  // NBHL, NWHL
        float add = seed_f32(temp_k, 0.1f);
        if (tmp != 0) add = clampf(0.001f * (float)tmp, 0.1f, 51.2f);
        out = ty == 40u ? __float2int_rz(add * 1024.0f) : __float2int_rz(-add * 1024.0f);
    } else if (ty == 42u) {  // GBMB
        if (life > 20u) out = 20480;
        else if (life >= 1u) out = -81920;
    } else if (ty == 43u) {  // GPMP
        if (life == 10u) out = __float2int_rz(0.2f * (temp_k - 273.15f) * 1024.0f);
    }
    return out;
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

// ------------------------------------------------------------- gathers ----
// One warp per listed brick. Lane l loads the 16 bytes of voxels
// x = 4*(l & 1) .. +3 of row z = (l >> 1) & 7, y = 2j + (l >> 4) of the brick
// in load j = 0..3, so every 32-byte sector a load touches is used whole.
// Lane l's words lie in cell (cx, cy, cz) = (l & 1, j >> 1, (l >> 3) & 1); the
// xor-shuffles over lane bits 1, 2 and 4 sum the eight lanes of a cell.
__device__ __forceinline__ uint32_t brick_base(uint32_t brick) {
    const uint32_t bx = brick & 31u, bz = (brick >> 5) & 31u, by = (brick >> 10) & 31u;
    return ((by * 8u) << 16) | ((bz * 8u) << 8) | (bx * 8u);
}
__device__ __forceinline__ uint32_t brick_cell(uint32_t brick, uint32_t cx, uint32_t cy, uint32_t cz) {
    const uint32_t bx = brick & 31u, bz = (brick >> 5) & 31u, by = (brick >> 10) & 31u;
    return ((by * 2u + cy) << 12) | ((bz * 2u + cz) << 6) | (bx * 2u + cx);
}
__device__ __forceinline__ uint32_t lane_offset(int lane, int j) {
    return ((uint32_t)(2 * j + (lane >> 4)) << 16) | ((uint32_t)((lane >> 1) & 7) << 8) | (uint32_t)(4 * (lane & 1));
}
__device__ __forceinline__ uint32_t cell_sum(uint32_t v) {
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 2);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 4);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 16);
    return v;
}

// air_gather_kernel (air_kernel.rs:218-278). The mean temperature's sum is
// exact in any order (at most 64 multiples of 1/8 below 8192), so it is
// summed as integers and scaled once.
__global__ void __launch_bounds__(256) k_air_gather(const uint32_t *__restrict__ voxel,
                                                    const uint32_t *__restrict__ list,
                                                    const uint32_t *__restrict__ count, float *__restrict__ solid,
                                                    float *__restrict__ temp) {
    const uint32_t n = min(__ldg(count), (uint32_t)TPT_VOX_BRICKS);
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < n; b += nwarps) {
        const uint32_t brick = __ldg(list + b) & (TPT_VOX_BRICKS - 1u);
        const uint32_t base = brick_base(brick);
        uint4 w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = __ldg(reinterpret_cast<const uint4 *>(voxel + base + lane_offset(lane, j)));
        uint32_t cnt[2] = {0u, 0u}, tq[2] = {0u, 0u};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t ws[4] = {w[j].x, w[j].y, w[j].z, w[j].w};
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if ((ws[k] & 0xFFu) != 0u) {
                    cnt[j >> 1] += 1u;
                    tq[j >> 1] += (ws[k] >> 8) & 0xFFFFu;
                }
        }
#pragma unroll
        for (int cy = 0; cy < 2; ++cy) {
            cnt[cy] = cell_sum(cnt[cy]);
            tq[cy] = cell_sum(tq[cy]);
        }
        if ((lane & 0x16) == 0) {
#pragma unroll
            for (int cy = 0; cy < 2; ++cy) {
                const uint32_t cell = brick_cell(brick, lane & 1, cy, (lane >> 3) & 1);
                solid[cell] = (float)cnt[cy] * (1.0f / 64.0f);
                temp[cell] = cnt[cy] > 0u ? __fdiv_rn((float)tq[cy] * 0.125f, (float)cnt[cy]) : kAmbient;
            }
        }
    }
}

// gravity_gather_kernel (gravity.rs:125-166): the tmp words are read only
// for loads that hold a non-empty voxel; integer sums wrap like the
// reference's i32 accumulator and atomic add.
__global__ void __launch_bounds__(256) k_grav_gather(const uint32_t *__restrict__ voxel,
                                                     const int32_t *__restrict__ aux,
                                                     const uint32_t *__restrict__ list,
                                                     const uint32_t *__restrict__ count, int32_t *__restrict__ mass) {
    const uint32_t n = min(__ldg(count), (uint32_t)TPT_VOX_BRICKS);
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < n; b += nwarps) {
        const uint32_t brick = __ldg(list + b) & (TPT_VOX_BRICKS - 1u);
        const uint32_t base = brick_base(brick);
        uint4 w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = __ldg(reinterpret_cast<const uint4 *>(voxel + base + lane_offset(lane, j)));
        uint32_t acc[2] = {0u, 0u};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t ws[4] = {w[j].x, w[j].y, w[j].z, w[j].w};
            if (((ws[0] | ws[1] | ws[2] | ws[3]) & 0xFFu) == 0u) continue;  // four empty voxels
            const int4 t = __ldg(reinterpret_cast<const int4 *>(aux + base + lane_offset(lane, j)));
            const int32_t ts[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t ty = ws[k] & 0xFFu;
                if (ty != 0u)
                    acc[j >> 1] += (uint32_t)voxel_mass(ty, (ws[k] >> 24) & 0xFFu, ts[k],
                                                        (float)((ws[k] >> 8) & 0xFFFFu) * 0.125f);
            }
        }
#pragma unroll
        for (int cy = 0; cy < 2; ++cy) acc[cy] = cell_sum(acc[cy]);
        if ((lane & 0x16) == 0) {
#pragma unroll
            for (int cy = 0; cy < 2; ++cy)
                if (acc[cy] != 0u)
                    atomicAdd(reinterpret_cast<unsigned int *>(mass) + brick_cell(brick, lane & 1, cy, (lane >> 3) & 1),
                              acc[cy]);
        }
    }
}

// air_clear_kernel (air_kernel.rs:182-204), one float4 of each field per thread.
__global__ void __launch_bounds__(256) k_air_clear(float *vx, float *vy, float *vz, float *p, float *p_tmp,
                                                   float *temp, float *solid, int32_t *pv) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (i >= CELLS) return;
    st4(vx + i, zero4());
    st4(vy + i, zero4());
    st4(vz + i, zero4());
    st4(p + i, zero4());
    st4(p_tmp + i, zero4());
    st4(temp + i, make_float4(kAmbient, kAmbient, kAmbient, kAmbient));
    st4(solid + i, zero4());
    *reinterpret_cast<int4 *>(pv + i) = make_int4(0, 0, 0, 0);
}

// ------------------------------------------------------- cluster form ----
// Shared memory of a CTA: three slabs (A, B, C) of PL planes each. Buffers
// are named by their float offset in it; a neighbouring CTA's slab is read
// through its 32-bit shared::cluster address (mapa of this CTA's base).

enum : int { SA = 0, SB = SLAB, SC = 2 * SLAB };

__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(rank));
    return out;
}
__device__ __forceinline__ float4 ld4_cluster(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(addr)
                 : "memory");
    return v;
}

// This thread's place in the cluster: rank, quad, first row, and the
// shared::cluster byte addresses of the neighbouring ranks' shared memory
// (absent where the rank is at a world y face). Cell (row j, plane pl, k) of the
// thread is bit (j * PL + pl) * 4 + k of its masks.
struct Ctx {
    float *sm;
    uint32_t below, above;  // ranks r-1 / r+1
    bool has_below, has_above;
    int r, x0, z0, o, zlo, zhi;
    size_t g0;               // cell index of the quad's first cell on plane 0, row z0
};
__device__ __forceinline__ int bit(int j, int pl, int k) { return (j * PL + pl) * 4 + k; }

// Plane PL-1 of the slab at `buf` in rank r-1 / plane 0 of rank r+1, at
// in-plane offset `off`.
__device__ __forceinline__ float4 ld_below(const Ctx &c, int buf, int off) {
    return c.has_below ? ld4_cluster(c.below + (uint32_t)(buf + (PL - 1) * PLANE + off) * 4u) : zero4();
}
__device__ __forceinline__ float4 ld_above(const Ctx &c, int buf, int off) {
    return c.has_above ? ld4_cluster(c.above + (uint32_t)(buf + off) * 4u) : zero4();
}

// A Jacobi sweep of this CTA's slab, S -> T. `fixed` marks the pinned
// cells. The per-cell source is the gravity's 4*pi*G*rho in registers (src)
// or the air's divergence in slab C of shared memory. The thread's rows are
// adjacent in z, so only the outer z neighbours are loaded.
template <bool GRAV>
__device__ __forceinline__ void sweep(const Ctx &cx, int S, int T, const float4 (&src)[ROWS][PL], uint32_t fixed) {
    const float *s = cx.sm + S;
    float4 ym[ROWS], c[ROWS];
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        ym[j] = ld_below(cx, S, cx.o + j * N);
        c[j] = ld4(s + cx.o + j * N);
    }
#pragma unroll
    for (int pl = 0; pl < PL; ++pl) {
        float4 yp[ROWS];
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            if (pl + 1 < PL) yp[j] = ld4(s + (pl + 1) * PLANE + cx.o + j * N);
            else yp[j] = ld_above(cx, S, cx.o + j * N);
        }
        const float4 zlo = ld4(s + pl * PLANE + cx.zlo), zhi = ld4(s + pl * PLANE + cx.zhi);
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            const float4 zm = j == 0 ? zlo : c[j - 1], zp = j == ROWS - 1 ? zhi : c[j + 1];
            const float l = __shfl_up_sync(0xFFFFFFFFu, c[j].w, 1, 16);
            const float r = __shfl_down_sync(0xFFFFFFFFu, c[j].x, 1, 16);
            const float4 dv = GRAV ? zero4() : ld4(cx.sm + SC + pl * PLANE + cx.o + j * N);
            float4 out;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float xm = k == 0 ? l : f4(c[j], k - 1), xp = k == 3 ? r : f4(c[j], k + 1);
                const bool fx = (fixed >> bit(j, pl, k)) & 1u;
                f4set(out, k,
                      GRAV ? grav_sweep_cell(xm, xp, f4(zm, k), f4(zp, k), f4(ym[j], k), f4(yp[j], k),
                                             f4(src[j][pl], k), f4(c[j], k), fx)
                           : air_sweep_cell(xm, xp, f4(zm, k), f4(zp, k), f4(ym[j], k), f4(yp[j], k),
                                            f4(dv, k), fx));
            }
            st4(cx.sm + T + pl * PLANE + cx.o + j * N, out);
        }
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            ym[j] = c[j];
            c[j] = yp[j];
        }
    }
}

// The six neighbours of the quad of row j on plane `pl` of a slab buffer
// (zeros beyond the world's y faces).
struct Hood {
    float4 c, zm, zp, ym, yp;
    float l, r;
};
__device__ __forceinline__ Hood hood(const Ctx &cx, int buf, int pl, int j) {
    const float *v = cx.sm + buf;
    const int z = cx.z0 + j, o = cx.o + j * N;
    Hood h;
    h.c = ld4(v + pl * PLANE + o);
    h.zm = ld4(v + pl * PLANE + max(z - 1, 0) * N + cx.x0);
    h.zp = ld4(v + pl * PLANE + min(z + 1, N - 1) * N + cx.x0);
    if (pl > 0) h.ym = ld4(v + (pl - 1) * PLANE + o);
    else h.ym = ld_below(cx, buf, o);
    if (pl + 1 < PL) h.yp = ld4(v + (pl + 1) * PLANE + o);
    else h.yp = ld_above(cx, buf, o);
    h.l = __shfl_up_sync(0xFFFFFFFFu, h.c.w, 1, 16);
    h.r = __shfl_down_sync(0xFFFFFFFFu, h.c.x, 1, 16);
    return h;
}
// The same from a field in global memory (cell index g of the quad's first cell).
__device__ __forceinline__ Hood hood_global(const float *V, size_t g, int y, int z) {
    Hood h;
    h.c = ld4(V + g);
    h.zm = z > 0 ? ld4(V + g - SZ) : zero4();
    h.zp = z + 1 < N ? ld4(V + g + SZ) : zero4();
    h.ym = y > 0 ? ld4(V + g - SY) : zero4();
    h.yp = y + 1 < N ? ld4(V + g + SY) : zero4();
    h.l = __shfl_up_sync(0xFFFFFFFFu, h.c.w, 1, 16);
    h.r = __shfl_down_sync(0xFFFFFFFFu, h.c.x, 1, 16);
    return h;
}
__device__ __forceinline__ float hx_m(const Hood &h, int k) { return k == 0 ? h.l : f4(h.c, k - 1); }
__device__ __forceinline__ float hx_p(const Hood &h, int k) { return k == 3 ? h.r : f4(h.c, k + 1); }

// New values of velocity component AXIS for the quad of row j on plane `pl`:
// V is the staged old component, P the solved pressure. The buoyancy and the
// gradient are formed first so that one neighbourhood is live at a time.
template <int AXIS>
__device__ __forceinline__ float4 advect_quad(const Ctx &cx, int V, int P, const float *temp, int pl, int j,
                                              uint32_t solid) {
    const int y = cx.r * PL + pl, z = cx.z0 + j, o = cx.o + j * N;
    float4 buoy = zero4(), grad;
    if (AXIS == 1) {
        const Hood t = hood_global(temp, cx.g0 + (size_t)pl * PLANE + (size_t)j * N, y, z);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float lt = nb_average(f4(t.c, k), hx_m(t, k), hx_p(t, k), f4(t.zm, k), f4(t.zp, k), f4(t.ym, k),
                                        f4(t.yp, k), cx.x0 + k, y, z);
            f4set(buoy, k, (lt - kAmbient) * kBuoyancy);
        }
    }
    {
        const float *p = cx.sm + P;
        const float4 pc = ld4(p + pl * PLANE + o);
        if (AXIS == 0) {
            const float l = __shfl_up_sync(0xFFFFFFFFu, pc.w, 1, 16), r = __shfl_down_sync(0xFFFFFFFFu, pc.x, 1, 16);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                f4set(grad, k,
                      pressure_grad(k == 0 ? l : f4(pc, k - 1), k == 3 ? r : f4(pc, k + 1), f4(pc, k), cx.x0 + k));
        } else if (AXIS == 1) {
            float4 lo, hi;
            if (pl > 0) lo = ld4(p + (pl - 1) * PLANE + o);
            else lo = ld_below(cx, P, o);
            if (pl + 1 < PL) hi = ld4(p + (pl + 1) * PLANE + o);
            else hi = ld_above(cx, P, o);
#pragma unroll
            for (int k = 0; k < 4; ++k) f4set(grad, k, pressure_grad(f4(lo, k), f4(hi, k), f4(pc, k), y));
        } else {
            const float4 lo = ld4(p + pl * PLANE + max(z - 1, 0) * N + cx.x0);
            const float4 hi = ld4(p + pl * PLANE + min(z + 1, N - 1) * N + cx.x0);
#pragma unroll
            for (int k = 0; k < 4; ++k) f4set(grad, k, pressure_grad(f4(lo, k), f4(hi, k), f4(pc, k), z));
        }
    }
    const Hood v = hood(cx, V, pl, j);
    float4 out;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float nv = advect_cell(f4(v.c, k), hx_m(v, k), hx_p(v, k), f4(v.zm, k), f4(v.zp, k), f4(v.ym, k),
                                     f4(v.yp, k), AXIS, f4(grad, k), f4(buoy, k), cx.x0 + k, y, z);
        f4set(out, k, ((solid >> bit(j, pl, k)) & 1u) ? 0.0f : nv);
    }
    return out;
}

// AirState::solve (air.rs:162-222) for one world.
__device__ __forceinline__ void air_job(const Job &jb, const Ctx &cx, cg::cluster_group &cl) {
    float *vx = jb.f[0], *vy = jb.f[1], *vz = jb.f[2], *p = jb.f[3], *p_tmp = jb.f[4];
    const float *temp = jb.f[5], *solid = jb.f[6];
    int32_t *pv = jb.i0;
    float *sm = cx.sm;
    const int y0 = cx.r * PL;

    // Stage p (A), vy (B) and vz (C); mark pinned and solid cells.
    uint32_t fixed = 0u, solid_bits = 0u;
#pragma unroll
    for (int j = 0; j < ROWS; ++j)
#pragma unroll
        for (int pl = 0; pl < PL; ++pl) {
            const int so = pl * PLANE + cx.o + j * N;
            const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
            st4(sm + SA + so, ld4(p + g));
            st4(sm + SB + so, ld4(vy + g));
            st4(sm + SC + so, ld4(vz + g));
            const float4 s = ld4(solid + g);
            const int y = y0 + pl, z = cx.z0 + j;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int x = cx.x0 + k;
                const bool boundary = x == 0 || y == 0 || z == 0 || x == N - 1 || y == N - 1 || z == N - 1;
                const bool sol = f4(s, k) > 0.5f;
                solid_bits |= (uint32_t)sol << bit(j, pl, k);
                fixed |= (uint32_t)(boundary || sol) << bit(j, pl, k);
            }
        }
    cl.sync();

    // pv update (air_kernel.rs:294-326) and the sweeps' divergence
    // (air_kernel.rs:385-388), both from the velocities before the solve; vx
    // comes from global memory, vy from slab B, vz from slab C. The
    // divergence then replaces vz in slab C, once every thread of the CTA
    // has read its vz rows.
#pragma unroll 1
    for (int c = 0; c < ROWS * PL; ++c) {
        const int j = c / PL, pl = c % PL;
        const int so = pl * PLANE + cx.o + j * N, z = cx.z0 + j, y = y0 + pl;
        const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
        const float4 xc = ld4(vx + g);
        const float xl = __shfl_up_sync(0xFFFFFFFFu, xc.w, 1, 16);
        const float xr = __shfl_down_sync(0xFFFFFFFFu, xc.x, 1, 16);
        const float4 ym = pl > 0 ? ld4(sm + SB + so - PLANE) : ld_below(cx, SB, cx.o + j * N);
        const float4 yp = pl + 1 < PL ? ld4(sm + SB + so + PLANE) : ld_above(cx, SB, cx.o + j * N);
        const float4 zm = ld4(sm + SC + pl * PLANE + max(z - 1, 0) * N + cx.x0);
        const float4 zp = ld4(sm + SC + pl * PLANE + min(z + 1, N - 1) * N + cx.x0);
        const int4 pv4 = *reinterpret_cast<const int4 *>(pv + g);
        int32_t pvs[4] = {pv4.x, pv4.y, pv4.z, pv4.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int x = cx.x0 + k;
            const float xm = k == 0 ? xl : f4(xc, k - 1), xp = k == 3 ? xr : f4(xc, k + 1);
            const bool rim = x < 2 || x >= N - 2 || y < 2 || y >= N - 2 || z < 2 || z >= N - 2;
            const float dp = (xm - xp) + (f4(ym, k) - f4(yp, k)) + (f4(zm, k) - f4(zp, k));
            pvs[k] = pv_update(pvs[k], rim, dp);
        }
        *reinterpret_cast<int4 *>(pv + g) = make_int4(pvs[0], pvs[1], pvs[2], pvs[3]);
    }
    {
        float4 div[ROWS][PL];
#pragma unroll
        for (int j = 0; j < ROWS; ++j)
#pragma unroll
            for (int pl = 0; pl < PL; ++pl) {
                const int so = pl * PLANE + cx.o + j * N, z = cx.z0 + j;
                const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
                const float4 xc = ld4(vx + g);
                const float xl = __shfl_up_sync(0xFFFFFFFFu, xc.w, 1, 16);
                const float xr = __shfl_down_sync(0xFFFFFFFFu, xc.x, 1, 16);
                float4 ym, yp;
                if (pl > 0) ym = ld4(sm + SB + so - PLANE);
                else ym = ld_below(cx, SB, cx.o + j * N);
                if (pl + 1 < PL) yp = ld4(sm + SB + so + PLANE);
                else yp = ld_above(cx, SB, cx.o + j * N);
                const float4 zm = ld4(sm + SC + pl * PLANE + max(z - 1, 0) * N + cx.x0);
                const float4 zp = ld4(sm + SC + pl * PLANE + min(z + 1, N - 1) * N + cx.x0);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float xm = k == 0 ? xl : f4(xc, k - 1), xp = k == 3 ? xr : f4(xc, k + 1);
                    f4set(div[j][pl], k, 0.5f * ((xp - xm) + (f4(yp, k) - f4(ym, k)) + (f4(zp, k) - f4(zm, k))));
                }
            }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < ROWS; ++j)
#pragma unroll
            for (int pl = 0; pl < PL; ++pl) st4(sm + SC + pl * PLANE + cx.o + j * N, div[j][pl]);
    }
    cl.sync();

    // Jacobi sweeps (air_kernel.rs:361-398): odd sweeps write B (the
    // reference's p_tmp), even ones A (p).
    const float4 no_src[ROWS][PL] = {};
    const uint32_t n = jb.iterations;
    for (uint32_t it = 0; it < n; ++it) {
        if ((it & 1u) == 0u) sweep<false>(cx, SA, SB, no_src, fixed);  // the divergence is in slab C
        else sweep<false>(cx, SB, SA, no_src, fixed);
        cl.sync();
    }
    const int P = (n & 1u) ? SB : SA, F = (n & 1u) ? SA : SB;

    // Publish the pair as the reference's alternation leaves it; stage vx
    // (F) and vy (C) for the advection (air_kernel.rs:414-536).
#pragma unroll
    for (int j = 0; j < ROWS; ++j)
#pragma unroll
        for (int pl = 0; pl < PL; ++pl) {
            const int so = pl * PLANE + cx.o + j * N;
            const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
            if (n >= 2u) st4(p + g, ld4(sm + SA + so));
            if (n >= 1u) st4(p_tmp + g, ld4(sm + SB + so));
            st4(sm + F + so, ld4(vx + g));
            st4(sm + SC + so, ld4(vy + g));
        }
    cl.sync();
#pragma unroll 1
    for (int c = 0; c < ROWS * PL; ++c) {
        const int j = c / PL, pl = c % PL;
        const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
        st4(vx + g, advect_quad<0>(cx, F, P, temp, pl, j, solid_bits));
        st4(vy + g, advect_quad<1>(cx, SC, P, temp, pl, j, solid_bits));
    }
    cl.sync();
#pragma unroll
    for (int j = 0; j < ROWS; ++j)
#pragma unroll
        for (int pl = 0; pl < PL; ++pl)
            st4(sm + F + pl * PLANE + cx.o + j * N, ld4(vz + cx.g0 + (size_t)pl * PLANE + (size_t)j * N));
    cl.sync();
#pragma unroll 1
    for (int c = 0; c < ROWS * PL; ++c) {
        const int j = c / PL, pl = c % PL;
        st4(vz + cx.g0 + (size_t)pl * PLANE + (size_t)j * N, advect_quad<2>(cx, F, P, temp, pl, j, solid_bits));
    }
    cl.sync();
}

// gravity::solve (gravity.rs:228-260) for one world, then optionally
// gravity::clear_mass.
__device__ __forceinline__ void grav_job(const Job &jb, const Ctx &cx, cg::cluster_group &cl) {
    float *pot = jb.f[0], *pot_tmp = jb.f[1], *fx = jb.f[2], *fy = jb.f[3], *fz = jb.f[4];
    int32_t *mass = jb.i0;
    float *sm = cx.sm;
    const int y0 = cx.r * PL;

    float4 src[ROWS][PL];
    uint32_t fixed = 0u;
#pragma unroll
    for (int j = 0; j < ROWS; ++j)
#pragma unroll
        for (int pl = 0; pl < PL; ++pl) {
            const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
            st4(sm + SA + pl * PLANE + cx.o + j * N, ld4(pot + g));
            const int4 m = *reinterpret_cast<const int4 *>(mass + g);
            src[j][pl] = make_float4(grav_source(m.x), grav_source(m.y), grav_source(m.z), grav_source(m.w));
            if (jb.clear_mass) *reinterpret_cast<int4 *>(mass + g) = make_int4(0, 0, 0, 0);
            const int y = y0 + pl, z = cx.z0 + j;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int x = cx.x0 + k;
                const bool boundary = x == 0 || x == N - 1 || y == 0 || y == N - 1 || z == 0 || z == N - 1;
                fixed |= (uint32_t)boundary << bit(j, pl, k);
            }
        }
    cl.sync();

    const uint32_t n = jb.iterations;
    for (uint32_t it = 0; it < n; ++it) {
        if ((it & 1u) == 0u) sweep<true>(cx, SA, SB, src, fixed);
        else sweep<true>(cx, SB, SA, src, fixed);
        cl.sync();
    }
    // The last sweep is grav_potential and the one before grav_potential_tmp
    // (the reference swaps the two handles after every sweep).
    const int U = (n & 1u) ? SB : SA, Uprev = (n & 1u) ? SA : SB;
#pragma unroll 1
    for (int c = 0; c < ROWS * PL; ++c) {
        const int j = c / PL, pl = c % PL;
        const int so = pl * PLANE + cx.o + j * N;
        const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
        if (n >= 1u) {
            st4(pot + g, ld4(sm + U + so));
            st4(pot_tmp + g, ld4(sm + Uprev + so));
        }
        // gravity_force_kernel (gravity.rs:199-224)
        const Hood h = hood(cx, U, pl, j);
        float4 ox, oy, oz;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const bool b = (fixed >> bit(j, pl, k)) & 1u;
            const float u = f4(h.c, k);
            f4set(ox, k, b ? seed_f32(u, 0.0f) : (hx_m(h, k) - hx_p(h, k)) * 0.5f);
            f4set(oz, k, b ? seed_f32(u, 0.0f) : (f4(h.zm, k) - f4(h.zp, k)) * 0.5f);
            f4set(oy, k, b ? seed_f32(u, 0.0f) : (f4(h.ym, k) - f4(h.yp, k)) * 0.5f);
        }
        st4(fx + g, ox);
        st4(fy + g, oy);
        st4(fz + g, oz);
    }
    cl.sync();
}

__global__ void __launch_bounds__(THREADS, 1) k_field_cluster(const __grid_constant__ Jobs J) {
    extern __shared__ __align__(16) float smem[];
    cg::cluster_group cl = cg::this_cluster();
    Ctx cx;
    cx.sm = smem;
    cx.r = (int)cl.block_rank();
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(smem);
    cx.has_below = cx.r > 0;
    cx.has_above = cx.r + 1 < CL;
    cx.below = cx.has_below ? mapa(base, (uint32_t)cx.r - 1u) : 0u;
    cx.above = cx.has_above ? mapa(base, (uint32_t)cx.r + 1u) : 0u;
    const int q = threadIdx.x & 15;
    cx.z0 = (threadIdx.x >> 4) * ROWS;
    cx.x0 = 4 * q;
    cx.o = cx.z0 * N + cx.x0;
    cx.zlo = max(cx.z0 - 1, 0) * N + cx.x0;
    cx.zhi = min(cx.z0 + ROWS, N - 1) * N + cx.x0;
    cx.g0 = (size_t)(cx.r * PL) * PLANE + cx.o;
    const Job &jb = J.job[blockIdx.x / CL];
    if (jb.kind == JOB_AIR) air_job(jb, cx, cl);
    else grav_job(jb, cx, cl);
}

// ----------------------------------------------------- per-sweep form ----
// One thread per cell, one launch per reference pass.

__device__ __forceinline__ void coords(int i, int &x, int &y, int &z) {
    x = i & 63;
    z = (i >> 6) & 63;
    y = i >> 12;
}

__global__ void __launch_bounds__(256) k_ps_pressure_volume(const float *__restrict__ vx, const float *__restrict__ vy,
                                                            const float *__restrict__ vz, int32_t *__restrict__ pv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CELLS) return;
    int x, y, z;
    coords(i, x, y, z);
    const bool rim = x < 2 || x >= N - 2 || y < 2 || y >= N - 2 || z < 2 || z >= N - 2;
    float dp = 0.0f;
    if (!rim) dp = (vx[i - 1] - vx[i + 1]) + (vy[i - SY] - vy[i + SY]) + (vz[i - SZ] - vz[i + SZ]);
    pv[i] = pv_update(pv[i], rim, dp);
}

__global__ void __launch_bounds__(256) k_ps_snapshot(const float *__restrict__ vx, const float *__restrict__ vy,
                                                     const float *__restrict__ vz, float *__restrict__ snap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CELLS) return;
    snap[i] = vx[i];
    snap[CELLS + i] = vy[i];
    snap[2 * CELLS + i] = vz[i];
}

__global__ void __launch_bounds__(256) k_ps_air_sweep(const float *__restrict__ pin, float *__restrict__ pout,
                                                      const float *__restrict__ vx, const float *__restrict__ vy,
                                                      const float *__restrict__ vz, const float *__restrict__ solid) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CELLS) return;
    int x, y, z;
    coords(i, x, y, z);
    const bool boundary = x == 0 || y == 0 || z == 0 || x == N - 1 || y == N - 1 || z == N - 1;
    if (boundary || solid[i] > 0.5f) {
        pout[i] = 0.0f;
        return;
    }
    const float divergence = 0.5f * ((vx[i + 1] - vx[i - 1]) + (vy[i + SY] - vy[i - SY]) + (vz[i + SZ] - vz[i - SZ]));
    pout[i] = air_sweep_cell(pin[i - 1], pin[i + 1], pin[i - SZ], pin[i + SZ], pin[i - SY], pin[i + SY], divergence,
                             false);
}

__global__ void __launch_bounds__(256) k_ps_air_advect(const float *__restrict__ snap, const float *__restrict__ pr,
                                                       const float *__restrict__ temp, const float *__restrict__ solid,
                                                       float *__restrict__ vx, float *__restrict__ vy,
                                                       float *__restrict__ vz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CELLS) return;
    if (solid[i] > 0.5f) {
        vx[i] = 0.0f;
        vy[i] = 0.0f;
        vz[i] = 0.0f;
        return;
    }
    int x, y, z;
    coords(i, x, y, z);
    auto at = [&](const float *f, bool ok, int j) { return ok ? f[j] : 0.0f; };
    const bool hxm = x > 0, hxp = x + 1 < N, hzm = z > 0, hzp = z + 1 < N, hym = y > 0, hyp = y + 1 < N;
    const float lt = nb_average(temp[i], at(temp, hxm, i - 1), at(temp, hxp, i + 1), at(temp, hzm, i - SZ),
                                at(temp, hzp, i + SZ), at(temp, hym, i - SY), at(temp, hyp, i + SY), x, y, z);
    const float buoy = (lt - kAmbient) * kBuoyancy;
    const float pc = pr[i];
    const float grad[3] = {pressure_grad(at(pr, hxm, i - 1), at(pr, hxp, i + 1), pc, x),
                           pressure_grad(at(pr, hym, i - SY), at(pr, hyp, i + SY), pc, y),
                           pressure_grad(at(pr, hzm, i - SZ), at(pr, hzp, i + SZ), pc, z)};
    float out[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float *s = snap + (size_t)a * CELLS;
        out[a] = advect_cell(s[i], at(s, hxm, i - 1), at(s, hxp, i + 1), at(s, hzm, i - SZ), at(s, hzp, i + SZ),
                             at(s, hym, i - SY), at(s, hyp, i + SY), a, grad[a], a == 1 ? buoy : 0.0f, x, y, z);
    }
    vx[i] = out[0];
    vy[i] = out[1];
    vz[i] = out[2];
}

__global__ void __launch_bounds__(256) k_ps_grav_sweep(const float *__restrict__ uin, float *__restrict__ uout,
                                                       const int32_t *__restrict__ mass) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CELLS) return;
    int x, y, z;
    coords(i, x, y, z);
    const bool boundary = x == 0 || x == N - 1 || y == 0 || y == N - 1 || z == 0 || z == N - 1;
    if (boundary) {
        uout[i] = seed_f32(uin[i], 0.0f);
        return;
    }
    uout[i] = grav_sweep_cell(uin[i - 1], uin[i + 1], uin[i - SZ], uin[i + SZ], uin[i - SY], uin[i + SY],
                              grav_source(mass[i]), uin[i], false);
}

__global__ void __launch_bounds__(256) k_ps_grav_force(const float *__restrict__ u, float *__restrict__ fx,
                                                       float *__restrict__ fy, float *__restrict__ fz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CELLS) return;
    int x, y, z;
    coords(i, x, y, z);
    const bool boundary = x == 0 || x == N - 1 || y == 0 || y == N - 1 || z == 0 || z == N - 1;
    if (boundary) {
        fx[i] = seed_f32(u[i], 0.0f);
        fy[i] = seed_f32(u[i], 0.0f);
        fz[i] = seed_f32(u[i], 0.0f);
        return;
    }
    fx[i] = (u[i - 1] - u[i + 1]) * 0.5f;
    fz[i] = (u[i - SZ] - u[i + SZ]) * 0.5f;
    fy[i] = (u[i - SY] - u[i + SY]) * 0.5f;
}

__global__ void __launch_bounds__(256) k_grav_clear(int32_t *mass) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (i < CELLS) *reinterpret_cast<int4 *>(mass + i) = make_int4(0, 0, 0, 0);
}

// --------------------------------------------------------------- host ----

static int g_gather_blocks = 0;

static int gather_blocks() {
    if (g_gather_blocks == 0) {
        int dev = 0, sms = 0;
        TPT_CUDA(cudaGetDevice(&dev));
        TPT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        g_gather_blocks = sms * 8;  // 8 resident blocks of 256 threads per SM
    }
    return g_gather_blocks;
}

int launch_air_clear(const World &w, cudaStream_t st) {
    k_air_clear<<<CELLS / 4 / 256, 256, 0, st>>>(w.vx, w.vy, w.vz, w.p, w.p_tmp, w.temp, w.solid, w.pv);
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_air_gather(const World &w, cudaStream_t st) {
    const int blocks = gather_blocks();
    if (blocks <= 0) return TPT_ERR_CUDA;
    k_air_gather<<<blocks, 256, 0, st>>>(w.voxel, w.sim_list, w.sim_count, w.solid, w.temp);
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_grav_gather(const World &w, cudaStream_t st) {
    const int blocks = gather_blocks();
    if (blocks <= 0) return TPT_ERR_CUDA;
    k_grav_gather<<<blocks, 256, 0, st>>>(w.voxel, w.aux_tmp, w.sim_list, w.sim_count, w.grav_mass);
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_grav_clear(const World &w, cudaStream_t st) {
    k_grav_clear<<<CELLS / 4 / 256, 256, 0, st>>>(w.grav_mass);
    TPT_LAUNCHED();
    return TPT_OK;
}

int cluster_supported(bool *ok) {
    *ok = false;
    TPT_CUDA(cudaFuncSetAttribute(k_field_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CLUSTER_SMEM));
    TPT_CUDA(cudaFuncSetAttribute(k_field_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(CL);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = CLUSTER_SMEM;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, k_field_cluster, &cfg);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return TPT_OK;
    }
    *ok = clusters > 0;
    return TPT_OK;
}

int launch_cluster(const Jobs &jobs, cudaStream_t st) {
    if (jobs.n == 0) return TPT_OK;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(CL * jobs.n);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = CLUSTER_SMEM;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TPT_CUDA(cudaLaunchKernelEx(&cfg, k_field_cluster, jobs));
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_air_per_sweep(const World &w, uint32_t iterations, float *snapshot, cudaStream_t st) {
    const int blocks = CELLS / 256;
    k_ps_pressure_volume<<<blocks, 256, 0, st>>>(w.vx, w.vy, w.vz, w.pv);
    TPT_LAUNCHED();
    k_ps_snapshot<<<blocks, 256, 0, st>>>(w.vx, w.vy, w.vz, snapshot);
    TPT_LAUNCHED();
    float *pin = w.p, *pout = w.p_tmp;
    for (uint32_t it = 0; it < iterations; ++it) {
        k_ps_air_sweep<<<blocks, 256, 0, st>>>(pin, pout, w.vx, w.vy, w.vz, w.solid);
        TPT_LAUNCHED();
        float *t = pin;
        pin = pout;
        pout = t;
    }
    k_ps_air_advect<<<blocks, 256, 0, st>>>(snapshot, pin, w.temp, w.solid, w.vx, w.vy, w.vz);
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_grav_per_sweep(const World &w, cudaStream_t st) {
    const int blocks = CELLS / 256;
    float *uin = w.grav_potential, *uout = w.grav_potential_tmp;
    for (int it = 0; it < TPT_VOX_GRAV_ITERATIONS; ++it) {
        k_ps_grav_sweep<<<blocks, 256, 0, st>>>(uin, uout, w.grav_mass);
        TPT_LAUNCHED();
        float *t = uin;
        uin = uout;
        uout = t;
    }
    static_assert(TPT_VOX_GRAV_ITERATIONS % 2 == 0, "an even sweep count leaves the last sweep in grav_potential");
    k_ps_grav_force<<<blocks, 256, 0, st>>>(uin, w.grav_force_x, w.grav_force_y, w.grav_force_z);
    TPT_LAUNCHED();
    return TPT_OK;
}

Job air_job_of(const World &w, uint32_t iterations) {
    Job j{};
    j.f[0] = w.vx;
    j.f[1] = w.vy;
    j.f[2] = w.vz;
    j.f[3] = w.p;
    j.f[4] = w.p_tmp;
    j.f[5] = w.temp;
    j.f[6] = w.solid;
    j.i0 = w.pv;
    j.kind = JOB_AIR;
    j.iterations = iterations;
    return j;
}

Job grav_job_of(const World &w, bool clear_mass) {
    Job j{};
    j.f[0] = w.grav_potential;
    j.f[1] = w.grav_potential_tmp;
    j.f[2] = w.grav_force_x;
    j.f[3] = w.grav_force_y;
    j.f[4] = w.grav_force_z;
    j.i0 = w.grav_mass;
    j.kind = JOB_GRAV;
    j.iterations = TPT_VOX_GRAV_ITERATIONS;
    j.clear_mass = clear_mass ? 1u : 0u;
    return j;
}

}  // namespace vox
}  // namespace tpt
