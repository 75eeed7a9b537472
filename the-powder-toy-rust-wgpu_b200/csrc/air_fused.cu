// air_fused.cu -- temporal blocking of the batch's tile form: one launch that
// finishes tick t and starts tick t + 1.
//
// A tick is a velocity pass (A: pressure, velocity; a stencil of radius 3
// around each cell) and an advection pass (B: smoothing, advection,
// vorticity, fans, heat, convection, masks). B's semi-Lagrangian samples
// reach up to 0.7 * 256 cells into A's output of the same tick, so A(t) and
// B(t) cannot share a launch without a grid-wide dependency; but A(t + 1)
// needs only B(t)'s output within 3 cells. So k ticks run as k + 1 launches:
//
//   A(t0) | B(t0) A(t0+1) | B(t0+1) A(t0+2) | ... | B(t0+k-1)
//
// and each middle launch (this kernel) stages tick t's inputs once for a
// 32x16 tile plus a 5-cell halo, computes B(t) on the tile's +2 ring (the
// state A(t + 1) reads), writes tick t's state of the tile, and runs A(t + 1)
// on the tile from shared memory: tick t's state is not read back from DRAM,
// and the far samples of B(t) read A(t)'s complete output from the previous
// launch, so the result is exact with no guard on the advection reach.
//
// Every staged or recomputed value is the one the two-launch tick computes:
// the same per-cell functions (air.cuh) in the same operation order,
// compiled with -fmad=false. The velocity-pass outputs alternate between two
// sets by tick parity (the launch reads one set and writes the other), like
// the heat and mask ping-pong. The emap decays are deferred: each mask
// rebuild of a block reads emap without writing it (the value it sees is
// the stored one less the decays still pending), and the block's last B
// launch applies them all.
#include <cuda.h>

#include "air.cuh"
#include "air_launch.hpp"
#include "tc.cuh"

namespace tpt {
namespace air {
inline namespace AIR_SHAPE_NS {

static_assert(TX == FUSED_TX && TY == FUSED_TY, "compiled for the fused tile");

__device__ uint32_t g_fused_err;

// The staged box: the tile plus 8 cells each side in x (keeps the box's first
// column 16-byte aligned for TMA) and 5 in y.
struct FBox {
    static constexpr int HX = 8, HY = 5, W = TX + 2 * HX, HGT = TY + 2 * HY, N = W * HGT;
    static constexpr int NP = (N + 31) / 32 * 32;  // array stride: TMA destinations are 128-byte aligned
    __device__ static __forceinline__ int at(int gx, int gy, int x0, int y0) {
        return (gy - y0 + HY) * W + (gx - x0 + HX);
    }
    __device__ static __forceinline__ bool has(int x, int y, int x0, int y0) {
        return x >= x0 - HX && x < x0 + TX + HX && y >= y0 - HY && y < y0 + TY + HY;
    }
};
constexpr uint32_t FBOX_BYTES = FBox::N * 4;

// Tick t's staged inputs.
struct __align__(128) FStage {
    float ovx[FBox::NP];  // ovx(t) (NoUpdate: the stored vx)
    float ovy[FBox::NP];
    float opv[FBox::NP];
    float hv[FBox::NP];   // hv(t)
    uint32_t b[FBox::NP];   // block_air(t)
    uint32_t bh[FBox::NP];  // block_airh(t)
};
// Computed over the box: vorticity (+4 ring; then A(t + 1)'s pressure),
// smoothed/advected velocity and pressure (+3), tick t's convected velocity
// (+2, then A(t + 1)'s effective velocity in place), block_air(t + 1) (+3).
struct FWork {
    float vort[FBox::NP];
    float nvx[FBox::NP], nvy[FBox::NP], npv[FBox::NP];
    float svx[FBox::NP], svy[FBox::NP];
    uint32_t b1[FBox::NP];
};
constexpr size_t SMEM_F = sizeof(FStage) + sizeof(FWork);

// B(t)'s view: the accessors pass_b and the per-cell functions use.
struct LayoutFB {
    FStage *in;
    FWork *w;
    __device__ __forceinline__ static bool has3(int x, int y, int x0, int y0) { return FBox::has(x, y, x0, y0); }
    __device__ __forceinline__ static bool hasH(int x, int y, int x0, int y0) { return FBox::has(x, y, x0, y0); }
    __device__ __forceinline__ bool blk(int x, int y, int x0, int y0) const { return in->b[FBox::at(x, y, x0, y0)] != 0u; }
    __device__ __forceinline__ bool hblk(int x, int y, int x0, int y0) const {
        return (in->bh[FBox::at(x, y, x0, y0)] & 0x8u) != 0u;
    }
    __device__ __forceinline__ float OVX(int x, int y, int x0, int y0) const { return in->ovx[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float OVY(int x, int y, int x0, int y0) const { return in->ovy[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float OPV(int x, int y, int x0, int y0) const { return in->opv[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float HV(int x, int y, int x0, int y0) const { return in->hv[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &VORT(int x, int y, int x0, int y0) { return w->vort[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NVX(int x, int y, int x0, int y0) { return w->nvx[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NVY(int x, int y, int x0, int y0) { return w->nvy[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &NPV(int x, int y, int x0, int y0) { return w->npv[FBox::at(x, y, x0, y0)]; }
};

// A(t + 1)'s view: tick t's state from shared memory (velocity in svx/svy,
// pressure in npv, block_air(t + 1) in b1); its pressure goes to vort.
struct LayoutFA {
    FWork *w;
    __device__ __forceinline__ bool blk(int x, int y, int x0, int y0) const { return w->b1[FBox::at(x, y, x0, y0)] != 0u; }
    __device__ __forceinline__ float &VX(int x, int y, int x0, int y0) { return w->svx[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &VY(int x, int y, int x0, int y0) { return w->svy[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float PV(int x, int y, int x0, int y0) const { return w->npv[FBox::at(x, y, x0, y0)]; }
    __device__ __forceinline__ float &OPV(int x, int y, int x0, int y0) { return w->vort[FBox::at(x, y, x0, y0)]; }
};

extern __shared__ __align__(128) uint8_t air_fused_smem[];

__device__ __forceinline__ void tile_of(const TileRef *tiles, uint32_t t, uint32_t &inst, int &x0, int &y0) {
    TileRef r = tiles[t];
    inst = r.inst;
    x0 = (int)r.tx * TX;
    y0 = (int)r.ty * TY;
}

__device__ __forceinline__ void load_fbox(void *dst, const CUtensorMap *m, int x0, int y0, uint64_t *bar) {
    tc::tma_load_2d(dst, m, x0 - FBox::HX, y0 - FBox::HY, bar);
}

__device__ __forceinline__ uint32_t f_loads(const AirInst &I) {
    if (I.air_mode != 4u) return I.aheat ? 6u : 4u;
    return I.aheat ? 4u : 0u;
}

// The loads of tick t (parity p) for one tile, as pass B stages them.
__device__ __forceinline__ void issue_f(const AirInst &I, const CUtensorMap *m, uint32_t parity, int x0, int y0,
                                        FStage *buf, uint64_t *bar) {
    tc::mbar_arrive_expect_tx(bar, f_loads(I) * FBOX_BYTES);
    if (I.air_mode != 4u) {
        const CUtensorMap *ov = m + TM_OV0 + 3 * parity;
        load_fbox(buf->ovx, ov + 0, x0, y0, bar);
        load_fbox(buf->ovy, ov + 1, x0, y0, bar);
        load_fbox(buf->opv, ov + 2, x0, y0, bar);
        load_fbox(buf->b, m + TM_BA0 + parity, x0, y0, bar);
    } else {
        load_fbox(buf->ovx, m + TM_VX, x0, y0, bar);
        load_fbox(buf->ovy, m + TM_VY, x0, y0, bar);
    }
    if (I.aheat) {
        load_fbox(buf->hv, m + TM_HV0 + parity, x0, y0, bar);
        load_fbox(buf->bh, m + TM_BH0 + parity, x0, y0, bar);
    }
}

// block_air / block_airh(t + 1) of cell g, read-only (the decays are deferred).
__device__ __forceinline__ void masks_peek(const AirInst &I, size_t g, uint32_t lag, uint32_t &ba, uint32_t &bh) {
    masks_of(__ldg(I.wall + g), emap_seen(__ldg(I.emap + g), lag), I.eair ? __ldg(I.eair + g) : 0u,
             I.eairh ? __ldg(I.eairh + g) : 0u, ba, bh);
}

// B(t) of a tile whose air is updated (air_mode != NoUpdate): the state of
// tick t on the tile's +2 ring into shared memory (svx, svy, npv), written
// to memory on the tile; block_air(t + 1) on the +3 ring (b1).
__device__ __forceinline__ void fused_b(const AirInst &I, int x0, int y0, LayoutFB &S, uint32_t lag) {
    const uint32_t X = I.X, Y = I.Y;
    FWork *w = S.w;
    // smoothing/advection on ring Rs (the heat pass reads its +1 ring)
    if (I.vcoef > 0.0f) {
        if (I.aheat)
            for_ring<4>(I, x0, y0, [&](int gx, int gy) { S.VORT(gx, gy, x0, y0) = vorticity_bmap(S, gx, gy, X, Y, x0, y0); });
        else
            for_ring<3>(I, x0, y0, [&](int gx, int gy) { S.VORT(gx, gy, x0, y0) = vorticity_bmap(S, gx, gy, X, Y, x0, y0); });
        __syncthreads();
    }
    auto smooth = [&](int gx, int gy) {
        float a, b, c;
        smooth_advect_cell(I, S, gx, gy, x0, y0, a, b, c);
        S.NVX(gx, gy, x0, y0) = a;
        S.NVY(gx, gy, x0, y0) = b;
        S.NPV(gx, gy, x0, y0) = c;
    };
    if (I.aheat)
        for_ring<3>(I, x0, y0, smooth);
    else
        for_ring<2>(I, x0, y0, smooth);
    // block_air(t + 1) on the +3 ring for A(t + 1); the tile's masks to memory
    for_ring<3>(I, x0, y0, [&](int gx, int gy) {
        const size_t g = (size_t)gy * I.pitch + gx;
        uint32_t ba, bh;
        masks_peek(I, g, lag, ba, bh);
        w->b1[FBox::at(gx, gy, x0, y0)] = ba;
        if (gx >= x0 && gx < x0 + TX && gy >= y0 && gy < y0 + TY) {
            I.bair_out[g] = ba;
            I.bairh_out[g] = bh;
        }
    });
    __syncthreads();
    // heat and convection on the +2 ring (read-before-write of the smoothed velocity)
    for_ring<2>(I, x0, y0, [&](int gx, int gy) {
        float vx = S.NVX(gx, gy, x0, y0), vy = S.NVY(gx, gy, x0, y0);
        const bool own = gx >= x0 && gx < x0 + TX && gy >= y0 && gy < y0 + TY;
        if (I.aheat) {
            const float h = heat_cell(I, S, gx, gy, x0, y0, vx, vy);
            if (own) I.hv_out[(size_t)gy * I.pitch + gx] = h;
        }
        const int k = FBox::at(gx, gy, x0, y0);
        w->svx[k] = vx;
        w->svy[k] = vy;
        if (own) {
            const size_t g = (size_t)gy * I.pitch + gx;
            I.vx[g] = vx;
            I.vy[g] = vy;
            I.pv[g] = S.NPV(gx, gy, x0, y0);
        }
    });
    __syncthreads();
}

// B(t) then A(t + 1) for every tile. insts[2 i + p]: instance i at parity p
// (heat / mask halves and velocity-pass set p); tick t reads parity `parity`,
// tick t + 1 is parity ^ 1. `lag`: emap decays pending at tick t.
__global__ void __launch_bounds__(NT, 3) kb_fused_ba(const AirInst *__restrict__ insts,
                                                     const CUtensorMap *__restrict__ tmaps,
                                                     const TileRef *__restrict__ tiles, uint32_t ntiles,
                                                     uint32_t parity, uint32_t lag) {
    FStage *in = reinterpret_cast<FStage *>(air_fused_smem);
    FWork *work = reinterpret_cast<FWork *>(in + 1);
    __shared__ uint64_t full;
    if (threadIdx.x == 0) {
        tc::mbar_init(&full, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    uint32_t ph = 0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        uint32_t i;
        int x0, y0;
        tile_of(tiles, t, i, x0, y0);
        const AirInst I = insts[2 * i + parity];
        LayoutFB S{in, work};
        if (f_loads(I)) {
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue_f(I, tmaps + (size_t)i * TM_COUNT, parity, x0, y0, in, &full);
            }
            const bool ok = tc::mbar_wait(&full, ph, &g_fused_err);
            ph ^= 1u;
            if (!__syncthreads_and(ok)) {
                // the bulk copy this wait was for may still be in flight:
                // wait for it again (bounded) before the CTA exits
                if (threadIdx.x == 0) tc::mbar_wait(&full, ph ^ 1u, &g_fused_err);
                __syncthreads();
                return;
            }
        }
        if (I.air_mode == 4u) {
            // NoUpdate: tick t is the heat pass alone, on the tile (its
            // convected velocity goes to this parity's ovx/ovy, copied back
            // by the settle launch), and tick t + 1 has no velocity pass
            if (I.aheat) {
                for_ring<1>(I, x0, y0, [&](int gx, int gy) {
                    S.NVX(gx, gy, x0, y0) = S.OVX(gx, gy, x0, y0);
                    S.NVY(gx, gy, x0, y0) = S.OVY(gx, gy, x0, y0);
                });
                __syncthreads();
                pass_b(I, x0, y0, S);
            }
            const int gx = x0 + (int)(threadIdx.x % TX), gy = y0 + (int)(threadIdx.x / TX);
            if (in_grid(gx, gy, I)) {
                const size_t g = (size_t)gy * I.pitch + gx;
                uint32_t ba, bh;
                masks_peek(I, g, lag, ba, bh);
                I.bair_out[g] = ba;
                I.bairh_out[g] = bh;
            }
        } else {
            fused_b(I, x0, y0, S, lag);
            LayoutFA SA{work};
            const AirInst In = insts[2 * i + (parity ^ 1u)];  // tick t + 1: writes the other velocity-pass set
            pass_a(In, x0, y0, SA);
        }
        __syncthreads();
    }
}

}  // namespace AIR_SHAPE_NS

namespace {
int fused_prepare(int *occupancy) {
    using namespace AIR_SHAPE_NS;
    TPT_CUDA(cudaFuncSetAttribute(kb_fused_ba, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_F));
    TPT_CUDA(cudaFuncSetAttribute(kb_fused_ba, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    int occ = 0;
    TPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kb_fused_ba, NT, SMEM_F));
    *occupancy = occ;
    return TPT_OK;
}
}  // namespace

int fused_tile_prepare(int *occupancy) { return fused_prepare(occupancy); }

int launch_fused_ba(const AirInst *insts, const CUtensorMap *tmaps, const TileRef *tiles, uint32_t ntiles,
                    uint32_t grid, uint32_t parity, uint32_t emap_lag, cudaStream_t st) {
    using namespace AIR_SHAPE_NS;
    kb_fused_ba<<<grid, NT, SMEM_F, st>>>(insts, tmaps, tiles, ntiles, parity, emap_lag);
    TPT_LAUNCHED();
    return TPT_OK;
}

int read_fused_errors(uint32_t *out) {
    using namespace AIR_SHAPE_NS;
    uint32_t v = 0, z = 0;
    TPT_CUDA(cudaMemcpyFromSymbol(&v, g_fused_err, sizeof(v)));
    TPT_CUDA(cudaMemcpyToSymbol(g_fused_err, &z, sizeof(z)));
    *out = v;
    return TPT_OK;
}

}  // namespace air
}  // namespace tpt
