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

#include "field3d.hpp"
#include "field3d_cell.cuh"

namespace cg = cooperative_groups;

namespace tpt {
namespace vox {

constexpr int CL = 16;            // CTAs per cluster
constexpr int PL = N / CL;        // y planes per CTA
constexpr int ROWS = 2;           // z rows per thread
constexpr int THREADS = (N / 4) * (N / ROWS);  // one thread per x-quad and row pair
constexpr int PLANE = N * N;      // floats per plane
constexpr int SLAB = PL * PLANE;  // floats per CTA slab
constexpr size_t CLUSTER_SMEM = 3 * SLAB * sizeof(float);
static_assert(ROWS * PL * 4 <= 32, "a thread's cells fit one 32-bit mask");

// ------------------------------------------------------------- gathers ----
// One warp per listed brick, persistent warps taking the list in order. Lane
// l loads the 16 bytes of voxels x = 4*(l & 1) .. +3 of row z = (l >> 1) & 7,
// y = 2j + (l >> 4) of the brick in load j = 0..3, so every 32-byte sector a
// load touches is used whole. Lane l's words lie in cell (cx, cy, cz) =
// (l & 1, j >> 1, (l >> 3) & 1); the xor-shuffles over lane bits 1, 2 and 4
// sum the eight lanes of a cell.
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

// Per-brick multiplicity of the active list: how many times each brick id
// is listed (a compaction lists each active brick once). `mult` is cleared
// before the launch; ids are taken modulo the brick count, as the gathers do.
__global__ void k_brick_mult(const uint32_t *__restrict__ list, const uint32_t *__restrict__ count,
                             uint32_t *__restrict__ mult) {
    const uint32_t n = min(__ldg(count), (uint32_t)TPT_VOX_BRICKS);
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x)
        atomicAdd(mult + (__ldg(list + b) & (TPT_VOX_BRICKS - 1u)), 1u);
}

// gravity_gather_kernel (gravity.rs:125-166) in memory order. The reference
// adds each voxel's fixed-point mass to its cell with one atomic per voxel of
// every listed brick; in wrapping i32 arithmetic the result is each cell's
// voxel sum times the number of times its brick is listed, in any order.
// Block (zc, yc) owns the 64 cells of one cell row. Its 16 voxel rows
// (y = 4 yc + r / 4, z = 4 zc + r % 4) are read as 256-byte runs: warp w
// holds rows 2w and 2w + 1, one per half-warp, and lane l of a half the word
// quads of cells xc = 16 j + l, j = 0..3. A cell of an unlisted brick is
// neither read nor written; aux_tmp is read only for the quads holding GRVT,
// NBHL or NWHL.
__global__ void __launch_bounds__(256) k_grav_gather_rows(const uint32_t *__restrict__ voxel,
                                                          const int32_t *__restrict__ aux,
                                                          const uint32_t *__restrict__ mult,
                                                          int32_t *__restrict__ mass) {
    __shared__ uint32_t part[8][N];
    const uint32_t zc = blockIdx.x, yc = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t l = (uint32_t)lane & 15u, r = 2u * (uint32_t)warp + ((uint32_t)lane >> 4);
    const uint32_t row = ((4u * yc + (r >> 2)) << 16) | ((4u * zc + (r & 3u)) << 8);
    const uint32_t bbase = ((yc >> 1) << 10) | ((zc >> 1) << 5);
    uint32_t s[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t xc = 16u * (uint32_t)j + l;
        s[j] = 0u;
        if (__ldg(mult + (bbase | (xc >> 1))) == 0u) continue;
        const uint32_t o = row | (4u * xc);
        const uint4 w = __ldg(reinterpret_cast<const uint4 *>(voxel + o));
        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
        bool need = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) need |= ((ws[k] & 0xFFu) - 39u) < 3u;
        int4 t = make_int4(0, 0, 0, 0);
        if (need) t = __ldg(reinterpret_cast<const int4 *>(aux + o));
        const int32_t ts[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
            s[j] += (uint32_t)voxel_mass(ws[k] & 0xFFu, (ws[k] >> 24) & 0xFFu, ts[k], (ws[k] >> 8) & 0xFFFFu);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        s[j] += __shfl_xor_sync(0xFFFFFFFFu, s[j], 16);
        if (lane < 16) part[warp][16 * j + (int)l] = s[j];
    }
    __syncthreads();
    if (threadIdx.x < (unsigned)N) {
        const uint32_t xc = threadIdx.x, m = __ldg(mult + (bbase | (xc >> 1)));
        if (m != 0u) {
            uint32_t tot = 0u;
#pragma unroll
            for (int w = 0; w < 8; ++w) tot += part[w][xc];
            uint32_t *c = reinterpret_cast<uint32_t *>(mass) + ((yc << 12) | (zc << 6) | xc);
            *c += m * tot;
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
// Shared memory of a CTA: the Jacobi pair, slabs A and B of PL planes each,
// and slab H of halo planes: the plane below and the plane above this CTA's
// slab, for A and for B. A CTA writes its edge planes straight into its
// neighbours' halo planes (a store to another CTA's shared memory through
// its 32-bit shared::cluster address, mapa of the same offset), so every
// load of a sweep is local.

enum : int { SA = 0, SB = SLAB, SH = 2 * SLAB };
// Halo plane of buffer `buf` (SA or SB): below (0) or above (1) this slab.
__device__ __forceinline__ int halo(int buf, int above) { return SH + (buf == SA ? 0 : 2 * PLANE) + above * PLANE; }

__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(rank));
    return out;
}
// A store to another CTA's shared memory. Volatile: it stays between the
// cluster barriers around it (also volatile asm), whose release / acquire
// make it visible to that CTA.
__device__ __forceinline__ void st4_cluster(uint32_t addr, float4 v) {
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w));
}
// The two halves of the cluster barrier: arrive releases this thread's
// earlier shared-memory writes to the cluster, wait acquires the others'.
__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
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

// Writes an edge plane's quad into the neighbour that reads it: plane 0 of
// buffer `buf` is the plane above rank r-1's slab, plane PL-1 the plane below
// rank r+1's.
__device__ __forceinline__ void push_edge(const Ctx &c, int buf, int pl, int off, float4 v) {
    if (pl == 0 && c.has_below) st4_cluster(c.below + (uint32_t)(halo(buf, 1) + off) * 4u, v);
    if (pl == PL - 1 && c.has_above) st4_cluster(c.above + (uint32_t)(halo(buf, 0) + off) * 4u, v);
}

// One plane of a Jacobi sweep, S -> T, from the planes below / at / above it
// (ym, c, yp per row); an edge plane is also written into the neighbour that
// reads it. `fixed` marks the pinned cells; src holds the per-cell source
// (the gravity's 4*pi*G*rho or the air's divergence). The thread's rows are
// adjacent in z, so only the outer z neighbours are loaded.
template <bool GRAV>
__device__ __forceinline__ void sweep_plane(const Ctx &cx, int S, int T, int pl, const float4 (&ym)[ROWS],
                                            const float4 (&c)[ROWS], const float4 (&yp)[ROWS],
                                            const float4 (&src)[ROWS][PL], uint32_t fixed) {
    const float *s = cx.sm + S;
    float *t = cx.sm + T;
    const float4 zlo = ld4(s + pl * PLANE + cx.zlo), zhi = ld4(s + pl * PLANE + cx.zhi);
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const float4 zm = j == 0 ? zlo : c[j - 1], zp = j == ROWS - 1 ? zhi : c[j + 1];
        const float l = __shfl_up_sync(0xFFFFFFFFu, c[j].w, 1, 16);
        const float r = __shfl_down_sync(0xFFFFFFFFu, c[j].x, 1, 16);
        const uint32_t pins = (fixed >> bit(j, pl, 0)) & 0xFu;
        float4 out;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float xm = k == 0 ? l : f4(c[j], k - 1), xp = k == 3 ? r : f4(c[j], k + 1);
            const bool fx = (pins >> k) & 1u;
            f4set(out, k,
                  GRAV ? grav_sweep_cell(xm, xp, f4(zm, k), f4(zp, k), f4(ym[j], k), f4(yp[j], k),
                                         f4(src[j][pl], k), f4(c[j], k), pins != 0u && fx)
                       : air_sweep_cell(xm, xp, f4(zm, k), f4(zp, k), f4(ym[j], k), f4(yp[j], k),
                                        f4(src[j][pl], k), pins != 0u && fx));
        }
        st4(t + pl * PLANE + cx.o + j * N, out);
        push_edge(cx, T, pl, cx.o + j * N, out);
    }
}

// One Jacobi sweep of this CTA's slab, S -> T, with the cluster barrier
// split around it: the edge planes (0 and PL-1, the only ones other CTAs
// need) are computed and pushed first and released with `arrive`; the inner
// planes are computed while the barrier completes; `wait` then acquires the
// neighbours' pushes for the next sweep, and a CTA barrier publishes this
// CTA's inner planes. On entry S and its halo planes are complete.
template <bool GRAV>
__device__ __forceinline__ void sweep(const Ctx &cx, int S, int T, const float4 (&src)[ROWS][PL], uint32_t fixed) {
    static_assert(PL == 4, "edge planes 0 and 3, inner planes 1 and 2");
    const float *s = cx.sm + S;
    float4 below[ROWS], above[ROWS], p0[ROWS], p1[ROWS], p2[ROWS], p3[ROWS];
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int o = cx.o + j * N;
        below[j] = ld4(cx.sm + halo(S, 0) + o);
        above[j] = ld4(cx.sm + halo(S, 1) + o);
        p0[j] = ld4(s + o);
        p1[j] = ld4(s + PLANE + o);
        p2[j] = ld4(s + 2 * PLANE + o);
        p3[j] = ld4(s + 3 * PLANE + o);
    }
    sweep_plane<GRAV>(cx, S, T, 0, below, p0, p1, src, fixed);
    sweep_plane<GRAV>(cx, S, T, 3, p2, p3, above, src, fixed);
    cluster_arrive();
    sweep_plane<GRAV>(cx, S, T, 1, p0, p1, p2, src, fixed);
    sweep_plane<GRAV>(cx, S, T, 2, p1, p2, p3, src, fixed);
    cluster_wait();
    __syncthreads();
}

// The six neighbours of the quad of row j on plane `pl` of a slab buffer
// (its halo planes beyond the slab).
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
    h.ym = ld4(pl > 0 ? v + (pl - 1) * PLANE + o : cx.sm + halo(buf, 0) + o);
    h.yp = ld4(pl + 1 < PL ? v + (pl + 1) * PLANE + o : cx.sm + halo(buf, 1) + o);
    h.l = __shfl_up_sync(0xFFFFFFFFu, h.c.w, 1, 16);
    h.r = __shfl_down_sync(0xFFFFFFFFu, h.c.x, 1, 16);
    return h;
}
__device__ __forceinline__ float hx_m(const Hood &h, int k) { return k == 0 ? h.l : f4(h.c, k - 1); }
__device__ __forceinline__ float hx_p(const Hood &h, int k) { return k == 3 ? h.r : f4(h.c, k + 1); }

// Stages buffer A from global memory, pushes its edge planes into the
// neighbours' halo planes of A and zeroes the halo planes beyond the world's
// y faces (they feed only pinned cells).
__device__ __forceinline__ void stage_a(const Ctx &cx, const float *src) {
#pragma unroll
    for (int j = 0; j < ROWS; ++j) {
        const int o = cx.o + j * N;
#pragma unroll
        for (int pl = 0; pl < PL; ++pl) {
            const float4 v = ld4(src + cx.g0 + (size_t)pl * PLANE + (size_t)j * N);
            st4(cx.sm + SA + pl * PLANE + o, v);
            push_edge(cx, SA, pl, o, v);
        }
        if (!cx.has_below) {
            st4(cx.sm + halo(SA, 0) + o, zero4());
            st4(cx.sm + halo(SB, 0) + o, zero4());
        }
        if (!cx.has_above) {
            st4(cx.sm + halo(SA, 1) + o, zero4());
            st4(cx.sm + halo(SB, 1) + o, zero4());
        }
    }
}

// The Jacobi sweeps of AirState::solve (air_kernel.rs:361-398, air.rs:
// 195-213) for one world; the pv update, divergence and velocity snapshot
// before them and the advection after them run as grid-wide kernels.
__device__ __forceinline__ void air_job(const Job &jb, const Ctx &cx, cg::cluster_group &cl) {
    float *p = jb.f[0], *p_tmp = jb.f[1];
    const float *dsrc = jb.f[2], *solid = jb.f[3];
    float *sm = cx.sm;
    const int y0 = cx.r * PL;

    // Stage p (A) and the divergence (registers); mark the pinned cells.
    stage_a(cx, p);
    float4 div[ROWS][PL];
    uint32_t fixed = 0u;
#pragma unroll
    for (int j = 0; j < ROWS; ++j)
#pragma unroll
        for (int pl = 0; pl < PL; ++pl) {
            const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
            div[j][pl] = ld4(dsrc + g);
            const float4 sd = ld4(solid + g);
            const int y = y0 + pl, z = cx.z0 + j;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int x = cx.x0 + k;
                const bool boundary = x == 0 || y == 0 || z == 0 || x == N - 1 || y == N - 1 || z == N - 1;
                fixed |= (uint32_t)(boundary || f4(sd, k) > 0.5f) << bit(j, pl, k);
            }
        }
    cl.sync();

    // Odd sweeps write B (the reference's p_tmp), even ones A (p).
    const uint32_t n = jb.iterations;
    for (uint32_t it = 0; it < n; ++it) {
        if ((it & 1u) == 0u) sweep<false>(cx, SA, SB, div, fixed);
        else sweep<false>(cx, SB, SA, div, fixed);
    }
    // Publish the pair as the reference's alternation leaves it.
#pragma unroll
    for (int j = 0; j < ROWS; ++j)
#pragma unroll
        for (int pl = 0; pl < PL; ++pl) {
            const int so = pl * PLANE + cx.o + j * N;
            const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
            if (n >= 2u) st4(p + g, ld4(sm + SA + so));
            if (n >= 1u) st4(p_tmp + g, ld4(sm + SB + so));
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

    stage_a(cx, pot);
    float4 src[ROWS][PL];
    uint32_t fixed = 0u;
#pragma unroll
    for (int j = 0; j < ROWS; ++j)
#pragma unroll
        for (int pl = 0; pl < PL; ++pl) {
            const size_t g = cx.g0 + (size_t)pl * PLANE + (size_t)j * N;
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
    cl.sync();  // every CTA of the cluster is running before any writes into another's shared memory
    if (jb.kind == JOB_AIR) air_job(jb, cx, cl);
    else grav_job(jb, cx, cl);
}

// ----------------------------------------------------- per-sweep form ----
// One thread per cell, one launch per reference pass.


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

// The grid-wide passes of the cluster form's air solve before the sweeps:
// the pv update (air_kernel.rs:294-326), the velocity snapshot (:338-351)
// and the sweeps' divergence (:385-388), which the reference recomputes in
// every sweep from the velocities the sweeps leave unchanged.
__global__ void __launch_bounds__(256) k_air_prep(const float *__restrict__ vx, const float *__restrict__ vy,
                                                  const float *__restrict__ vz, int32_t *__restrict__ pv,
                                                  float *__restrict__ div, float *__restrict__ snap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= CELLS) return;
    int x, y, z;
    coords(i, x, y, z);
    snap[i] = vx[i];
    snap[CELLS + i] = vy[i];
    snap[2 * CELLS + i] = vz[i];
    const bool inner = x > 0 && y > 0 && z > 0 && x < N - 1 && y < N - 1 && z < N - 1;
    const bool rim = x < 2 || x >= N - 2 || y < 2 || y >= N - 2 || z < 2 || z >= N - 2;
    float dp = 0.0f, d = 0.0f;
    if (inner) {
        const float xm = vx[i - 1], xp = vx[i + 1], ym = vy[i - SY], yp = vy[i + SY], zm = vz[i - SZ],
                    zp = vz[i + SZ];
        dp = (xm - xp) + (ym - yp) + (zm - zp);
        d = 0.5f * ((xp - xm) + (yp - ym) + (zp - zm));
    }
    div[i] = d;
    pv[i] = pv_update(pv[i], rim, dp);  // the rim holds every cell outside `inner`
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

int launch_air_clear(const World &w, cudaStream_t st) {
    k_air_clear<<<CELLS / 4 / 256, 256, 0, st>>>(w.vx, w.vy, w.vz, w.p, w.p_tmp, w.temp, w.solid, w.pv);
    TPT_LAUNCHED();
    return TPT_OK;
}

// Persistent gather grid: 256-thread blocks, `per_sm` per SM of the current
// device (an attribute query, cheap next to the launch).
static int gather_blocks(int per_sm) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess || sms <= 0)
        sms = 148;
    return sms * per_sm;
}

int launch_air_gather(const World &w, cudaStream_t st) {
    k_air_gather<<<gather_blocks(8), 256, 0, st>>>(w.voxel, w.sim_list, w.sim_count, w.solid, w.temp);
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_grav_gather(const World &w, uint32_t *brick_mult, cudaStream_t st) {
    TPT_CUDA(cudaMemsetAsync(brick_mult, 0, TPT_VOX_BRICKS * sizeof(uint32_t), st));
    k_brick_mult<<<TPT_VOX_BRICKS / 256, 256, 0, st>>>(w.sim_list, w.sim_count, brick_mult);
    TPT_LAUNCHED();
    k_grav_gather_rows<<<dim3(N, N), 256, 0, st>>>(w.voxel, w.aux_tmp, brick_mult, w.grav_mass);
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

Job air_job_of(const World &w, uint32_t iterations, const AirScratch &sc) {
    Job j{};
    j.f[0] = w.p;
    j.f[1] = w.p_tmp;
    j.f[2] = sc.div;
    j.f[3] = w.solid;
    j.kind = JOB_AIR;
    j.iterations = iterations;
    return j;
}

int launch_air_prep(const World &w, const AirScratch &sc, cudaStream_t st) {
    k_air_prep<<<CELLS / 256, 256, 0, st>>>(w.vx, w.vy, w.vz, w.pv, sc.div, sc.snap);
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_air_advect(const World &w, uint32_t iterations, const AirScratch &sc, cudaStream_t st) {
    const float *pr = (iterations & 1u) ? w.p_tmp : w.p;  // the last sweep's buffer
    k_ps_air_advect<<<CELLS / 256, 256, 0, st>>>(sc.snap, pr, w.temp, w.solid, w.vx, w.vy, w.vz);
    TPT_LAUNCHED();
    return TPT_OK;
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
