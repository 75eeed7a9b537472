// field3d_batch.cu -- the batched form of the 3-D sandbox's field step
// (crates/tpt-sim/src/voxel3d/{air,gravity}.rs) on sm_100a: every world of a
// call in each launch, one launch per Jacobi sweep index.
//
//   prep    grid-wide, once: per air world the pv update, the velocity
//           snapshot, the sweeps' divergence and a 4-bit pin mask per x-quad
//           (world face or solid > 0.5); per gravity world the source
//           4*pi*G*rho. None of these changes during the sweeps, which the
//           reference recomputes in every sweep.
//   sweep s one launch per sweep index: the air sweep of every world while
//           s < air iterations and the gravity sweep of every world while
//           s < 24, side by side in the same grid. A thread updates one
//           x-quad (4 cells, a float4); the x neighbours outside the quad
//           come from the adjacent lanes.
//   finish  grid-wide, once: the air advection, the gravity force and the
//           mass clear.
//
// Every launch is a programmatic dependent launch: it lets the next launch
// start as soon as all its blocks are running (griddepcontrol.launch_dependents)
// and waits for the previous grid's completion and memory
// (griddepcontrol.wait) before touching global memory, so a sweep's launch
// latency overlaps the previous sweep's tail. The fields of a world stay in
// L2 (1 MiB each) across the sweeps.
#include "field3d.hpp"
#include "field3d_cell.cuh"

namespace tpt {
namespace vox {

namespace {

constexpr int QUADS = CELLS / 4;
constexpr int QBLOCK = 256;             // quads per block
constexpr int QBLOCKS = QUADS / QBLOCK; // blocks per field of a world
constexpr int CBLOCK = 256;             // cells per block of the per-cell passes
constexpr int CBLOCKS = CELLS / CBLOCK;
static_assert(TPT_VOX_GRAV_ITERATIONS % 2 == 0, "an even sweep count leaves the last sweep in grav_potential");

__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Which field block z of a launch works on: bit f of `fields` (f = 0 air,
// 1 gravity) marks the fields in the grid, in that order.
__device__ __forceinline__ int field_of(uint32_t fields, int z) {
    return (fields & 1u) ? z : 1;
}

__global__ void __launch_bounds__(CBLOCK) k_b_prep(const __grid_constant__ Batch B) {
    pdl_launch_dependents();
    pdl_wait();
    const BWorld &w = B.w[blockIdx.y];
    const int f = field_of(B.fields, blockIdx.z);
    const int i = blockIdx.x * CBLOCK + threadIdx.x;
    int x, y, z;
    coords(i, x, y, z);
    if (f == 1) {
        w.src[i] = grav_source(w.mass[i]);
        return;
    }
    const float *vx = w.vx, *vy = w.vy, *vz = w.vz;
    w.snap[i] = vx[i];
    w.snap[CELLS + i] = vy[i];
    w.snap[2 * CELLS + i] = vz[i];
    const bool inner = x > 0 && y > 0 && z > 0 && x < N - 1 && y < N - 1 && z < N - 1;
    const bool rim = x < 2 || x >= N - 2 || y < 2 || y >= N - 2 || z < 2 || z >= N - 2;
    float dp = 0.0f, d = 0.0f;
    if (inner) {
        const float xm = vx[i - 1], xp = vx[i + 1], ym = vy[i - SY], yp = vy[i + SY], zm = vz[i - SZ],
                    zp = vz[i + SZ];
        dp = (xm - xp) + (ym - yp) + (zm - zp);
        d = 0.5f * ((xp - xm) + (yp - ym) + (zp - zm));
    }
    w.div[i] = d;
    w.pv[i] = pv_update(w.pv[i], rim, dp);  // the rim holds every cell outside `inner`
    // pin mask of the quad: lanes 4k .. 4k+3 hold one quad's cells
    const bool pinned = !inner || w.solid[i] > 0.5f;
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, pinned);
    const int lane = threadIdx.x & 31;
    if ((lane & 3) == 0) w.pin[i >> 2] = (uint8_t)((bal >> lane) & 0xFu);
}

__global__ void __launch_bounds__(QBLOCK) k_b_sweep(const __grid_constant__ Batch B, uint32_t s) {
    pdl_launch_dependents();
    pdl_wait();
    const BWorld &w = B.w[blockIdx.y];
    const int f = field_of(B.fields, blockIdx.z);
    const int q = blockIdx.x * QBLOCK + threadIdx.x;
    const int i0 = 4 * q, x0 = i0 & 63, z = (i0 >> 6) & 63, y = i0 >> 12;
    const bool even = (s & 1u) == 0u;
    const float *S;
    float *T;
    if (f == 0) {
        S = even ? w.p : w.p_tmp;  // odd sweeps (1-based) write p_tmp, even ones p
        T = even ? w.p_tmp : w.p;
    } else {
        S = even ? w.pot : w.pot_tmp;
        T = even ? w.pot_tmp : w.pot;
    }
    const float4 c = ld4(S + i0);
    const float l = __shfl_up_sync(0xFFFFFFFFu, c.w, 1, 16);
    const float r = __shfl_down_sync(0xFFFFFFFFu, c.x, 1, 16);
    const float4 zm = z > 0 ? ld4(S + i0 - SZ) : zero4(), zp = z + 1 < N ? ld4(S + i0 + SZ) : zero4();
    const float4 ym = y > 0 ? ld4(S + i0 - SY) : zero4(), yp = y + 1 < N ? ld4(S + i0 + SY) : zero4();
    float4 out;
    if (f == 0) {
        const float4 d = ld4(w.div + i0);
        const uint32_t pins = w.pin[q];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float xm = k == 0 ? l : f4(c, k - 1), xp = k == 3 ? r : f4(c, k + 1);
            f4set(out, k, air_sweep_cell(xm, xp, f4(zm, k), f4(zp, k), f4(ym, k), f4(yp, k), f4(d, k),
                                         (pins >> k) & 1u));
        }
    } else {
        const float4 sr = ld4(w.src + i0);
        const bool face = y == 0 || z == 0 || y == N - 1 || z == N - 1;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int x = x0 + k;
            const float xm = k == 0 ? l : f4(c, k - 1), xp = k == 3 ? r : f4(c, k + 1);
            f4set(out, k, grav_sweep_cell(xm, xp, f4(zm, k), f4(zp, k), f4(ym, k), f4(yp, k), f4(sr, k), f4(c, k),
                                          face || x == 0 || x == N - 1));
        }
    }
    st4(T + i0, out);
}

__global__ void __launch_bounds__(CBLOCK) k_b_finish(const __grid_constant__ Batch B) {
    pdl_launch_dependents();
    pdl_wait();
    const BWorld &w = B.w[blockIdx.y];
    const int f = field_of(B.fields, blockIdx.z);
    const int i = blockIdx.x * CBLOCK + threadIdx.x;
    int x, y, z;
    coords(i, x, y, z);
    const bool hxm = x > 0, hxp = x + 1 < N, hzm = z > 0, hzp = z + 1 < N, hym = y > 0, hyp = y + 1 < N;
    auto at = [&](const float *a, bool ok, int j) { return ok ? a[j] : 0.0f; };
    if (f == 1) {
        // gravity_force_kernel (gravity.rs:199-224) on the last sweep, then
        // gravity_clear_kernel (gravity.rs:112-118) when asked
        const float *u = w.pot;
        const bool boundary = !(hxm && hxp && hym && hyp && hzm && hzp);
        if (boundary) {
            w.fx[i] = seed_f32(u[i], 0.0f);
            w.fy[i] = seed_f32(u[i], 0.0f);
            w.fz[i] = seed_f32(u[i], 0.0f);
        } else {
            w.fx[i] = (u[i - 1] - u[i + 1]) * 0.5f;
            w.fz[i] = (u[i - SZ] - u[i + SZ]) * 0.5f;
            w.fy[i] = (u[i - SY] - u[i + SY]) * 0.5f;
        }
        if (B.clear_mass) w.mass[i] = 0;
        return;
    }
    // air_advect_kernel (air_kernel.rs:414-536) from the snapshot
    if (w.solid[i] > 0.5f) {
        w.vx[i] = 0.0f;
        w.vy[i] = 0.0f;
        w.vz[i] = 0.0f;
        return;
    }
    const float *pr = (B.air_iters & 1u) ? w.p_tmp : w.p;  // the last sweep's buffer
    const float *temp = w.temp, *snap = w.snap;
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
        const float *sn = snap + (size_t)a * CELLS;
        out[a] = advect_cell(sn[i], at(sn, hxm, i - 1), at(sn, hxp, i + 1), at(sn, hzm, i - SZ), at(sn, hzp, i + SZ),
                             at(sn, hym, i - SY), at(sn, hyp, i + SY), a, grad[a], a == 1 ? buoy : 0.0f, x, y, z);
    }
    w.vx[i] = out[0];
    w.vy[i] = out[1];
    w.vz[i] = out[2];
}

template <typename... Args>
int launch_pdl(void (*kernel)(Args...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TPT_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
    TPT_LAUNCHED();
    return TPT_OK;
}

}  // namespace

int launch_batch(Batch &b, cudaStream_t st) {
    if (b.n == 0 || (b.fields & 3u) == 0u) return TPT_OK;
    const uint32_t nf = (b.fields & 1u) + ((b.fields >> 1) & 1u);
    int rc = launch_pdl(k_b_prep, dim3(CBLOCKS, b.n, nf), dim3(CBLOCK), st, (const Batch)b);
    if (rc) return rc;
    const uint32_t air = (b.fields & 1u) ? b.air_iters : 0u, grav = (b.fields & 2u) ? TPT_VOX_GRAV_ITERATIONS : 0u;
    const uint32_t sweeps = air > grav ? air : grav;
    Batch bs = b;
    for (uint32_t s = 0; s < sweeps; ++s) {
        bs.fields = (s < air ? 1u : 0u) | (s < grav ? 2u : 0u);
        const uint32_t n = (bs.fields & 1u) + ((bs.fields >> 1) & 1u);
        rc = launch_pdl(k_b_sweep, dim3(QBLOCKS, b.n, n), dim3(QBLOCK), st, (const Batch)bs, s);
        if (rc) return rc;
    }
    return launch_pdl(k_b_finish, dim3(CBLOCKS, b.n, nf), dim3(CBLOCK), st, (const Batch)b);
}

}  // namespace vox
}  // namespace tpt
