// grav_particles.cu -- the particle side of a Newtonian-gravity tick: wells
// into the solved snapshot, the force applied to particles, the mass grid
// rebuilt from particles (crates/tpt-sim/src/gravity_kernel.rs:217-527).
//
// Compiled with -fmad=false: the velocity update `v = v * loss; v = v + g *
// newton` and the element masses keep the reference's separately rounded f32
// operations, so the results are bit-identical to the FP32 restatement.
//
// The reference makes five launches around the solve (seed wells, apply force,
// clear accumulator, build mass, override, copy). Here the accumulator clear
// joins the well fold (both are per-cell and precede the build), the force
// and the mass build share one pass over the particle slots (the build reads
// positions and element state, never the velocity the force writes), and the
// override joins the snapshot copy: three launches plus the solve.
#include "grav_particles.hpp"

namespace tpt {
namespace gp {

constexpr uint32_t CELL = 4;             // crates/tpt-core/src/constants.rs:9
constexpr uint32_t PT_GRVT = 39, PT_NBHL = 40, PT_NWHL = 41, PT_GBMB = 42, PT_GPMP = 43;  // constants.rs:141-149
constexpr uint32_t PT_SPNG = 78;         // constants.rs:227
constexpr uint32_t TYPE_SOLID = 0x4u;    // constants.rs:611
constexpr uint32_t WL_STASIS = 18u;      // constants.rs:700-735
constexpr uint32_t FLAG_MOVABLE = 0x08u, FLAG_RIGID = 0x10u;
constexpr uint32_t LUT_WORDS = 12, LUT_PROPS = 0, LUT_LOSS = 7;  // move_kernel record layout

// f32 -> i32 truncation as the GPU converts (NaN -> 0, saturating).
__device__ __forceinline__ int32_t trunc_i32(float v) { return __float2int_rz(v); }

// Round half away from zero of m * 65536 (gravity_kernel.rs:346-353).
__device__ __forceinline__ int32_t to_fixed(float m) {
    float scaled = m * 65536.0f;
    if (scaled >= 0.0f) scaled += 0.5f;
    else scaled -= 0.5f;
    return trunc_i32(scaled);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) {
    float out = v;
    if (out < lo) out = lo;
    if (out > hi) out = hi;
    return out;
}

// seed_gravity_tool_mass_kernel (:241-262) then seed_gravity_mass_kernel
// (:217-229, whose tool word the first step has already consumed).
__global__ void k_seed(GravGrids G, uint32_t cells) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    if (G.tool) {
        const float tool = G.tool[c];
        if (tool != 0.0f) {
            G.prev[c] = to_fixed(tool);
            G.tool[c] = 0.0f;
        }
    }
    G.mass[c] = 0;
}

// apply_gravity_kernel (:434-516) and build_gravity_mass_kernel (:275-376),
// one thread per slot.
__global__ void k_particles(GravGrids G, Parts P) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const uint32_t ty = P.ty[i];
    if (ty == 0u) return;  // PT_NONE
    const int32_t xi = trunc_i32(P.x[i] + 0.5f), yi = trunc_i32(P.y[i] + 0.5f);
    const int32_t xres = (int32_t)G.xres, yres = (int32_t)G.yres;
    const bool on_canvas = xi >= 0 && yi >= 0 && xi < xres && yi < yres;

    // ---- force: Loss, then newton_grav * g (Simulation.cpp:2361-2384 order)
    if (ty < P.n_types) {
        const uint32_t flags = P.flags[i];
        bool eligible = (flags & FLAG_RIGID) == 0u && on_canvas;
        // off-margin particles are removed by the movement pass first
        if (xi < 4 || yi < 4 || xi >= xres - 4 || yi >= yres - 4) eligible = false;
        uint32_t cell = 0;
        if (eligible) {
            cell = ((uint32_t)yi / CELL) * G.xcells + (uint32_t)xi / CELL;
            // unpowered stasis wall freezes the particle
            if (__ldg(G.wall + cell) == WL_STASIS && (__ldg(G.emap + cell) & 0xFFu) < 8u) eligible = false;
        }
        if (eligible) {
            const uint32_t *rec = P.lut + (size_t)ty * LUT_WORDS;
            const uint32_t props = __ldg(rec + LUT_PROPS);
            const float loss = __uint_as_float(__ldg(rec + LUT_LOSS));
            float vx = P.vx[i], vy = P.vy[i];
            if (!(ty == PT_SPNG && (flags & FLAG_MOVABLE) != 0u)) {
                vx *= loss;
                vy *= loss;
            }
            if ((props & TYPE_SOLID) == 0u) {
                vx += G.newton * __ldg(G.gx + cell);
                vy += G.newton * __ldg(G.gy + cell);
            }
            P.vx[i] = vx;
            P.vy[i] = vy;
        }
    }

    // ---- mass: each gravity element's contribution, fixed point
    float mass = 0.0f;
    bool contributes = false;
    if (ty == PT_GRVT) {
        int32_t tmp = P.tmp[i];  // clamped to [-100, 100] before it becomes mass
        if (tmp < -100) tmp = -100;
        if (tmp > 100) tmp = 100;
        mass = 0.2f * (float)tmp;
        contributes = true;
    } else if (ty == PT_NBHL || ty == PT_NWHL) {
        float hole = 0.1f;
        const int32_t tmp = P.tmp[i];
        if (tmp != 0) hole = clampf(0.001f * (float)tmp, 0.1f, 51.2f);
        if (ty == PT_NWHL) hole = 0.0f - hole;
        mass = hole;
        contributes = true;
    } else if (ty == PT_GBMB) {
        const int32_t life = P.life[i];
        if (life > 20) {
            mass = 20.0f;
            contributes = true;
        } else if (life >= 1) {
            mass = -80.0f;
            contributes = true;
        }
    } else if (ty == PT_GPMP) {
        if (P.life[i] == 10) {
            mass = 0.2f * (P.temp[i] - 273.15f);
            contributes = true;
        }
    }
    if (contributes && on_canvas) {
        const uint32_t cx = (uint32_t)xi / CELL, cy = (uint32_t)yi / CELL;
        if (cx < G.xcells && cy < G.ycells) {
            const uint32_t cell = cy * G.xcells + cx;
            if (__ldg(G.mask + cell) != 0u) {
                const int32_t q = to_fixed(mass);
                if (q != 0) atomicAdd(G.mass + cell, q);
            }
        }
    }
}

// apply_grav_mass_override_kernel (:379-391) then copy_gravity_mass_kernel (:518-527).
__global__ void k_finish(GravGrids G, uint32_t cells) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    int32_t m = G.mass[c];
    if (G.ovr_set && G.ovr_set[c] != 0u) {
        m = G.ovr[c];
        G.mass[c] = m;
    }
    G.prev[c] = m;
}

int launch_seed(const GravGrids &G, cudaStream_t st) {
    const uint32_t cells = G.xcells * G.ycells;
    k_seed<<<(cells + 255) / 256, 256, 0, st>>>(G, cells);
    TPT_LAUNCHED();
    return TPT_OK;
}

int launch_particles_and_finish(const GravGrids &G, const Parts &P, cudaStream_t st) {
    if (P.n) {
        k_particles<<<(P.n + 255) / 256, 256, 0, st>>>(G, P);
        TPT_LAUNCHED();
    }
    const uint32_t cells = G.xcells * G.ycells;
    k_finish<<<(cells + 255) / 256, 256, 0, st>>>(G, cells);
    TPT_LAUNCHED();
    return TPT_OK;
}

}  // namespace gp
}  // namespace tpt
