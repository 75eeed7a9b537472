// api.cu -- the C ABI (include/tpt_field.h): status codes, the one-grid air
// step, gravity plans, host helpers and diagnostics.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <vector>

#include "air_launch.hpp"
#include "grav_dft.hpp"
#include "grav_particles.hpp"
#include "grav_plan.hpp"
#include "tc.cuh"
#include "tmap.hpp"

namespace tpt {

static thread_local char g_err[512] = "";
static std::atomic<uint64_t> g_launches{0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int require_sm100() {
    int dev = 0;
    TPT_CUDA(cudaGetDevice(&dev));
    int major = 0, minor = 0;
    TPT_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    TPT_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
    if (major != 10 || minor != 0)
        TPT_FAIL(TPT_ERR_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a only", dev, major,
                 minor);
    return TPT_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

int make_grid_tmap(CUtensorMap *out, const void *base, bool is_float, uint32_t cols, uint32_t rows, uint32_t pitch,
                   uint32_t box_cols, uint32_t box_rows) {
    auto fn = tensor_map_encoder();
    if (!fn) TPT_FAIL(TPT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * 4};
    cuuint32_t box[2] = {box_cols, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(out, is_float ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT32, 2,
                    const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) TPT_FAIL(TPT_ERR_CUDA, "cuTensorMapEncodeTiled (grid %ux%u pitch %u) failed (%d)", cols, rows,
                                    pitch, (int)r);
    return TPT_OK;
}

static int check_dims(uint32_t X, uint32_t Y) {
    if (X > TPT_MAX_CELLS_PER_SIDE || Y > TPT_MAX_CELLS_PER_SIDE)
        TPT_FAIL(TPT_ERR_INVALID_DIMS, "grid %ux%u exceeds %u cells per side", X, Y, TPT_MAX_CELLS_PER_SIDE);
    return TPT_OK;
}

static int check_air_params(const tpt_air_params *p) {
    if (p->air_mode > 4u) TPT_FAIL(TPT_ERR_INVALID_ARG, "air_mode %u out of range 0..4", p->air_mode);
    if (p->convection_mode > 2u) TPT_FAIL(TPT_ERR_INVALID_ARG, "convection_mode %u out of range 0..2", p->convection_mode);
    if (p->gravity_mode > 3u) TPT_FAIL(TPT_ERR_INVALID_ARG, "gravity_mode %u out of range 0..3", p->gravity_mode);
    if (p->aheat_enable > 1u) TPT_FAIL(TPT_ERR_INVALID_ARG, "aheat_enable must be 0 or 1");
    return check_dims(p->xcells, p->ycells);
}

AirInst make_air_inst(const tpt_air_params &p) {
    AirInst I{};
    I.X = p.xcells;
    I.Y = p.ycells;
    I.pitch = p.xcells;
    I.air_mode = p.air_mode;
    I.aheat = p.aheat_enable;
    I.conv = p.convection_mode;
    I.gmode = p.gravity_mode;
    I.ep = p.edge_pressure;
    I.evx = p.edge_vx;
    I.evy = p.edge_vy;
    I.amb = p.ambient_air_temp;
    I.vcoef = p.vorticity_coeff;
    I.vk = p.vorticity_coeff / 5.0f;
    I.cgx = p.custom_gx;
    I.cgy = p.custom_gy;
    return I;
}

}  // namespace tpt

using namespace tpt;

struct tpt_grav_plan {
    uint32_t X = 0, Y = 0;
    int precision = TPT_PRECISION_FP32;
    gfft::FftSet fft;
    dft::DftSet *dft = nullptr;
};

// The failure path of the bounded device waits, run without a fault: one
// thread waits on an mbarrier that nothing arrives at, through the same
// bounded wait the tensor-core and TMA pipelines use, and gives up after
// `limit` SM clocks, recording ERR_WAIT_TIMEOUT in its own error word.
static __device__ uint32_t g_selftest_err;

__global__ void k_selftest_wait(long long limit) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
    tc::mbar_wait_limit(&bar, 0u, &g_selftest_err, limit);
}

extern "C" {

const char *tpt_last_error_string(void) { return g_err; }

int tpt_check_device_errors(void) {
    TPT_CUDA(cudaDeviceSynchronize());
    uint32_t bits = 0, abits = 0, sbits = 0, z = 0;
    int rc = dft::read_errors(&bits);
    if (rc) return rc;
    rc = air::read_errors(&abits);
    if (rc) return rc;
    TPT_CUDA(cudaMemcpyFromSymbol(&sbits, g_selftest_err, sizeof(sbits)));
    TPT_CUDA(cudaMemcpyToSymbol(g_selftest_err, &z, sizeof(z)));
    bits |= abits | sbits;
    if (bits) TPT_FAIL(TPT_ERR_DEVICE_TIMEOUT, "a device-side wait timed out (error bits 0x%x)", bits);
    return TPT_OK;
}
int tpt_selftest_wait_timeout(uint32_t limit_clocks, tpt_stream_t stream) {
    int rc = require_sm100();
    if (rc) return rc;
    k_selftest_wait<<<1, 32, 0, (cudaStream_t)stream>>>((long long)limit_clocks);
    TPT_LAUNCHED();
    return TPT_OK;
}
uint64_t tpt_kernel_launch_count(void) { return g_launches.load(); }
const char *tpt_version(void) { return "tpt-field-b200 0.1.0 (sm_100a)"; }

void tpt_air_params_default(tpt_air_params *p, uint32_t xcells, uint32_t ycells) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->xcells = xcells;
    p->ycells = ycells;
    p->air_mode = TPT_AIR_ON;
    p->aheat_enable = 0;
    p->convection_mode = TPT_AIRC_BOUSSINESQ;
    p->gravity_mode = TPT_GRAVITY_VERTICAL;
    p->edge_pressure = 0.0f;
    p->edge_vx = 0.0f;
    p->edge_vy = 0.0f;
    p->ambient_air_temp = 295.15f;
    p->vorticity_coeff = 0.1f;
    p->custom_gx = 0.0f;
    p->custom_gy = 1.0f;
}

int tpt_air_step(const tpt_air_params *params, const tpt_air_bufs *b, tpt_stream_t stream) {
    if (!params || !b) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_air_step: params or bufs is NULL");
    int rc = check_air_params(params);
    if (rc) return rc;
    if (params->xcells == 0 || params->ycells == 0) return TPT_OK;  // mod.rs:124-126
    if (!b->pv || !b->vx || !b->vy || !b->hv || !b->opv || !b->ovx || !b->ovy || !b->ohv || !b->block_air ||
        !b->block_airh || !b->wall_bmap || !b->wall_emap || !b->fan_vx || !b->fan_vy)
        TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_air_step: a required grid pointer is NULL");
    if (b->pmap && (!b->elem_props || b->xres == 0 || b->yres == 0))
        TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_air_step: pmap given without elem_props / xres / yres");
    rc = require_sm100();
    if (rc) return rc;
    AirInst I = make_air_inst(*params);
    I.pv = b->pv;
    I.vx = b->vx;
    I.vy = b->vy;
    I.hv = b->hv;
    I.opv = b->opv;
    I.ovx = b->ovx;
    I.ovy = b->ovy;
    I.ohv = b->ohv;
    I.bair = b->block_air;
    I.bairh = b->block_airh;
    I.wall = b->wall_bmap;
    I.emap = b->wall_emap;
    I.eair = b->elem_block_air;
    I.eairh = b->elem_block_airh;
    I.fvx = b->fan_vx;
    I.fvy = b->fan_vy;
    I.bair_out = b->block_air;
    I.bairh_out = b->block_airh;
    I.hv_out = b->ohv;
    return air::launch_single(I, b->pmap, b->elem_props, b->n_elements, b->xres, b->yres, (cudaStream_t)stream);
}

int tpt_wall_masks_host(const uint32_t *wall, const uint32_t *emap, uint32_t *bair, uint32_t *bairh, size_t cells) {
    if (cells == 0) return TPT_OK;
    if (!wall || !emap || !bair || !bairh) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_wall_masks_host: NULL pointer");
    for (size_t i = 0; i < cells; ++i) {
        uint32_t w = wall[i] & 0xFFu, e = emap[i] & 0xFFu;
        bool blocked = w == 8u || w == 1u || w == 16u || (w == 2u && e == 0u);
        bair[i] = blocked ? 1u : 0u;
        bairh[i] = (blocked || w == 14u) ? 0x8u : 0u;
    }
    return TPT_OK;
}

int tpt_grav_mask_rebuild(const uint32_t *wall, uint32_t *mask, uint32_t X, uint32_t Y) {
    size_t cells = (size_t)X * Y;
    if (cells == 0) return TPT_OK;
    if (!wall || !mask) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_mask_rebuild: NULL pointer");
    memset(mask, 0, cells * sizeof(uint32_t));
    std::vector<size_t> stack;
    stack.reserve(256);
    auto seed = [&](size_t idx) {
        if ((wall[idx] & 0xFFu) == (uint32_t)TPT_WL_GRAV || mask[idx] != 0u) return;
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
    return TPT_OK;
}

int32_t tpt_mass_to_fixed(float m) {
    float s = m * 65536.0f;
    if (s >= 0.0f) s += 0.5f;
    else s -= 0.5f;
    if (!(s > -2147483648.0f)) return INT32_MIN;  // saturate like a Rust `as` cast
    if (!(s < 2147483648.0f)) return s != s ? 0 : INT32_MAX;
    return (int32_t)s;
}

// ---- gravity plans ---------------------------------------------------------
int tpt_grav_plan_create(uint32_t X, uint32_t Y, int precision, tpt_grav_plan **out) {
    if (!out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_plan_create: out is NULL");
    *out = nullptr;
    if (X == 0 || Y == 0) TPT_FAIL(TPT_ERR_INVALID_DIMS, "gravity grid %ux%u is empty", X, Y);
    int rc = check_dims(X, Y);
    if (rc) return rc;
    if (precision != TPT_PRECISION_FP32 && precision != TPT_PRECISION_SPLIT_BF16)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown precision %d", precision);
    rc = require_sm100();
    if (rc) return rc;
    tpt_grav_plan *p = new (std::nothrow) tpt_grav_plan();
    if (!p) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    p->X = X;
    p->Y = Y;
    p->precision = precision;
    std::vector<JobShape> shapes{{X, Y}};
    if (precision == TPT_PRECISION_FP32) {
        rc = p->fft.create(shapes);
    } else {
        p->dft = new (std::nothrow) dft::DftSet();
        rc = p->dft ? p->dft->create(shapes) : TPT_ERR_OUT_OF_MEMORY;
    }
    if (rc) {
        tpt_grav_plan_destroy(p);
        return rc;
    }
    *out = p;
    return TPT_OK;
}

int tpt_grav_plan_destroy(tpt_grav_plan *p) {
    if (!p) return TPT_OK;
    if (p->dft) delete p->dft;
    delete p;
    return TPT_OK;
}

int tpt_grav_plan_dims(const tpt_grav_plan *p, uint32_t *n1, uint32_t *n2) {
    if (!p || !n1 || !n2) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_plan_dims: NULL pointer");
    if (p->precision == TPT_PRECISION_FP32) {
        *n1 = p->fft.jobs_host[0].n1;
        *n2 = p->fft.jobs_host[0].n2;
    } else {
        p->dft->dims(0, n1, n2);
    }
    return TPT_OK;
}

static int grav_solve_any(tpt_grav_plan *p, const int32_t *mi, const float *mf, float inv, const uint32_t *mask,
                          float *gx, float *gy, tpt_stream_t stream) {
    if (!p) TPT_FAIL(TPT_ERR_NULL_POINTER, "gravity plan is NULL");
    if ((!mi && !mf) || !mask || !gx || !gy) TPT_FAIL(TPT_ERR_NULL_POINTER, "gravity solve: NULL grid pointer");
    if (p->precision == TPT_PRECISION_FP32) {
        gfft::JobIO io{mi, mf, mask, gx, gy, inv, 1};
        return p->fft.launch((cudaStream_t)stream, &io);
    }
    dft::SolveIO io{mi, mf, mask, gx, gy, inv, p->X};
    return p->dft->launch((cudaStream_t)stream, &io);
}

int tpt_grav_solve(tpt_grav_plan *p, const int32_t *mass_fx, float inv, const uint32_t *mask, float *gx, float *gy,
                   tpt_stream_t stream) {
    if (!mass_fx) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_solve: mass is NULL");
    return grav_solve_any(p, mass_fx, nullptr, inv, mask, gx, gy, stream);
}

int tpt_grav_solve_f32(tpt_grav_plan *p, const float *mass, const uint32_t *mask, float *gx, float *gy,
                       tpt_stream_t stream) {
    if (!mass) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_solve_f32: mass is NULL");
    return grav_solve_any(p, nullptr, mass, 1.0f, mask, gx, gy, stream);
}

int tpt_grav_step(tpt_grav_plan *p, const tpt_grav_state *s, const tpt_particles *q, tpt_stream_t stream) {
    if (!p || !s || !q) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_step: NULL plan, state or particles");
    if (!s->wall_bmap || !s->wall_emap || !s->grav_mask || !s->mass || !s->mass_prev || !s->gx || !s->gy)
        TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_step: NULL grid pointer");
    if (!s->override_mass != !s->override_set)
        TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_step: override_mass and override_set must both be set or both NULL");
    if (s->xres / 4u != p->X || s->yres / 4u != p->Y)
        TPT_FAIL(TPT_ERR_INVALID_DIMS, "tpt_grav_step: canvas %ux%u px is not the plan's %ux%u cells", s->xres,
                 s->yres, p->X, p->Y);
    if (q->num_slots && (!q->ty || !q->x || !q->y || !q->vx || !q->vy || !q->life || !q->tmp || !q->temp ||
                         !q->flags || !q->move_lut))
        TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_grav_step: NULL particle array");
    gp::GravGrids G{s->xres, s->yres, p->X, p->Y, s->wall_bmap, s->wall_emap, s->grav_mask, s->mass, s->mass_prev,
                    s->tool_mass, s->override_mass, s->override_set, s->gx, s->gy, s->newton_grav};
    gp::Parts P{q->num_slots, q->n_types, q->ty, q->x, q->y, q->vx, q->vy, q->life, q->tmp, q->temp, q->flags,
                q->move_lut};
    cudaStream_t st = (cudaStream_t)stream;
    int rc = gp::launch_seed(G, st);
    if (rc) return rc;
    rc = grav_solve_any(p, s->mass_prev, nullptr, 1.0f / 65536.0f, s->grav_mask, s->gx, s->gy, stream);
    if (rc) return rc;
    return gp::launch_particles_and_finish(G, P, st);
}

}  // extern "C"
