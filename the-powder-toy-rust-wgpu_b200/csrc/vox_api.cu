// vox_api.cu -- the C ABI of the 3-D sandbox's field step
// (include/tpt_field.h, "3-D sandbox field step").
#include <new>

#include "field3d.hpp"

using namespace tpt;

struct tpt_vox_plan {
    int form = TPT_VOX_PER_SWEEP;
    // Per-sweep form: the reference's velocity snapshot (3 fields).
    // Cluster form: one AirScratch (4 fields) per world of a launch.
    // Batched form: BATCH_SCRATCH_BYTES per world of a launch.
    float *scratch = nullptr;
    uint32_t *brick_mult = nullptr;  // the gravity gather's per-brick list multiplicity
    tpt::vox::AirScratch slot(uint32_t i) const {
        float *b = scratch + (size_t)i * tpt::vox::AIR_SCRATCH_FLOATS;
        return {b, b + TPT_VOX_CELLS};
    }
    tpt::vox::BWorld bworld(uint32_t i, const tpt_vox_world &w) const {
        char *b = reinterpret_cast<char *>(scratch) + (size_t)i * tpt::vox::BATCH_SCRATCH_BYTES;
        float *f = reinterpret_cast<float *>(b);
        tpt::vox::BWorld o{};
        o.vx = w.vx;
        o.vy = w.vy;
        o.vz = w.vz;
        o.p = w.p;
        o.p_tmp = w.p_tmp;
        o.temp = w.temp;
        o.solid = w.solid;
        o.pv = w.pv;
        o.mass = w.grav_mass;
        o.pot = w.grav_potential;
        o.pot_tmp = w.grav_potential_tmp;
        o.fx = w.grav_force_x;
        o.fy = w.grav_force_y;
        o.fz = w.grav_force_z;
        o.div = f;
        o.snap = f + TPT_VOX_CELLS;
        o.src = f + 4 * TPT_VOX_CELLS;
        o.pin = reinterpret_cast<uint8_t *>(f + 5 * TPT_VOX_CELLS);
        return o;
    }
};

namespace {

constexpr uint32_t kMaxAirIterations = 65536;

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0u; }

// Checks the pointers a call reads or writes: non-NULL and 16-byte aligned
// (the kernels move float4 / uint4 words).
int check_ptrs(const char *who, std::initializer_list<const void *> ptrs) {
    for (const void *p : ptrs) {
        if (!p) TPT_FAIL(TPT_ERR_NULL_POINTER, "%s: a required buffer is NULL", who);
        if (!aligned16(p)) TPT_FAIL(TPT_ERR_INVALID_ARG, "%s: buffer %p is not 16-byte aligned", who, p);
    }
    return TPT_OK;
}

vox::World world_of(const tpt_vox_world &w) {
    vox::World v{};
    v.voxel = w.voxel;
    v.aux_tmp = w.aux_tmp;
    v.sim_list = w.sim_list;
    v.sim_count = w.sim_count;
    v.vx = w.vx;
    v.vy = w.vy;
    v.vz = w.vz;
    v.p = w.p;
    v.p_tmp = w.p_tmp;
    v.temp = w.temp;
    v.solid = w.solid;
    v.pv = w.pv;
    v.grav_mass = w.grav_mass;
    v.grav_potential = w.grav_potential;
    v.grav_potential_tmp = w.grav_potential_tmp;
    v.grav_force_x = w.grav_force_x;
    v.grav_force_y = w.grav_force_y;
    v.grav_force_z = w.grav_force_z;
    return v;
}

int check_air_solve(const tpt_vox_world *w) {
    return check_ptrs("air solve", {w->vx, w->vy, w->vz, w->p, w->p_tmp, w->temp, w->solid, w->pv});
}
int check_grav_solve(const tpt_vox_world *w) {
    return check_ptrs("gravity solve", {w->grav_mass, w->grav_potential, w->grav_potential_tmp, w->grav_force_x,
                                        w->grav_force_y, w->grav_force_z});
}
int check_gather(const tpt_vox_world *w) {
    if (!w->sim_list || !w->sim_count) TPT_FAIL(TPT_ERR_NULL_POINTER, "gather: sim_list or sim_count is NULL");
    return check_ptrs("gather", {w->voxel});
}

// One batched launch sequence of `fields` for worlds [first, first + n).
int run_batch(tpt_vox_plan *plan, const tpt_vox_world *worlds, uint32_t n, uint32_t fields, uint32_t air_iterations,
              bool clear_mass, cudaStream_t st) {
    vox::Batch b{};
    b.n = n;
    b.fields = fields;
    b.air_iters = air_iterations;
    b.clear_mass = clear_mass ? 1u : 0u;
    for (uint32_t i = 0; i < n; ++i) b.w[i] = plan->bworld(i, worlds[i]);
    return vox::launch_batch(b, st);
}

int run_air_solve(tpt_vox_plan *plan, const tpt_vox_world *w, uint32_t iterations, cudaStream_t st) {
    if (plan->form == TPT_VOX_BATCHED) return run_batch(plan, w, 1, 1u, iterations, false, st);
    const vox::World v = world_of(*w);
    if (plan->form == TPT_VOX_CLUSTER) {
        const vox::AirScratch sc = plan->slot(0);
        int rc = vox::launch_air_prep(v, sc, st);
        if (rc) return rc;
        vox::Jobs jobs{};
        jobs.n = 1;
        jobs.job[0] = vox::air_job_of(v, iterations, sc);
        rc = vox::launch_cluster(jobs, st);
        if (rc) return rc;
        return vox::launch_air_advect(v, iterations, sc, st);
    }
    return vox::launch_air_per_sweep(v, iterations, plan->scratch, st);
}

}  // namespace

extern "C" {

int tpt_vox_plan_create(int form, tpt_vox_plan **out) {
    if (!out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_plan_create: out is NULL");
    *out = nullptr;
    if (form != TPT_VOX_AUTO && form != TPT_VOX_CLUSTER && form != TPT_VOX_PER_SWEEP && form != TPT_VOX_BATCHED)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_vox_plan_create: unknown form %d", form);
    int rc = require_sm100();
    if (rc) return rc;
    if (form == TPT_VOX_CLUSTER) {
        bool cluster_ok = false;
        rc = vox::cluster_supported(&cluster_ok);
        if (rc) return rc;
        if (!cluster_ok) TPT_FAIL(TPT_ERR_UNSUPPORTED, "the device cannot schedule a 16-CTA cluster of the field kernel");
    }
    tpt_vox_plan *p = new (std::nothrow) tpt_vox_plan();
    if (!p) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    p->form = form == TPT_VOX_AUTO ? TPT_VOX_BATCHED : form;
    size_t bytes = 3ull * TPT_VOX_CELLS * sizeof(float);
    if (p->form == TPT_VOX_CLUSTER) bytes = (size_t)(vox::MAX_JOBS / 2) * vox::AIR_SCRATCH_FLOATS * sizeof(float);
    if (p->form == TPT_VOX_BATCHED) bytes = (size_t)vox::MAX_BWORLDS * vox::BATCH_SCRATCH_BYTES;
    cudaError_t e = cudaMalloc(&p->scratch, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&p->brick_mult, TPT_VOX_BRICKS * sizeof(uint32_t));
    if (e != cudaSuccess) {
        cudaFree(p->scratch);
        delete p;
        TPT_FAIL(e == cudaErrorMemoryAllocation ? TPT_ERR_OUT_OF_MEMORY : TPT_ERR_CUDA,
                 "tpt_vox_plan_create: scratch allocation failed: %s", cudaGetErrorString(e));
    }
    *out = p;
    return TPT_OK;
}

int tpt_vox_plan_destroy(tpt_vox_plan *plan) {
    if (!plan) return TPT_OK;
    if (plan->scratch) cudaFree(plan->scratch);
    if (plan->brick_mult) cudaFree(plan->brick_mult);
    delete plan;
    return TPT_OK;
}

int tpt_vox_plan_form(const tpt_vox_plan *plan) {
    if (!plan) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_plan_form: plan is NULL");
    return plan->form;
}

int tpt_vox_air_clear(const tpt_vox_world *w, tpt_stream_t stream) {
    if (!w) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_air_clear: world is NULL");
    int rc = check_air_solve(w);
    if (rc) return rc;
    return vox::launch_air_clear(world_of(*w), (cudaStream_t)stream);
}

int tpt_vox_air_gather(tpt_vox_plan *plan, const tpt_vox_world *w, tpt_stream_t stream) {
    if (!plan || !w) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_air_gather: NULL plan or world");
    int rc = check_gather(w);
    if (!rc) rc = check_ptrs("air gather", {w->solid, w->temp});
    if (rc) return rc;
    return vox::launch_air_gather(world_of(*w), (cudaStream_t)stream);
}

int tpt_vox_air_solve(tpt_vox_plan *plan, const tpt_vox_world *w, uint32_t iterations, tpt_stream_t stream) {
    if (!plan || !w) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_air_solve: NULL plan or world");
    if (iterations > kMaxAirIterations)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_vox_air_solve: %u iterations (at most %u)", iterations, kMaxAirIterations);
    int rc = check_air_solve(w);
    if (rc) return rc;
    return run_air_solve(plan, w, iterations, (cudaStream_t)stream);
}

int tpt_vox_grav_solve(tpt_vox_plan *plan, const tpt_vox_world *w, tpt_stream_t stream) {
    if (!plan || !w) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_grav_solve: NULL plan or world");
    int rc = check_grav_solve(w);
    if (rc) return rc;
    const vox::World v = world_of(*w);
    if (plan->form == TPT_VOX_BATCHED) return run_batch(plan, w, 1, 2u, 0u, false, (cudaStream_t)stream);
    if (plan->form == TPT_VOX_CLUSTER) {
        vox::Jobs jobs{};
        jobs.n = 1;
        jobs.job[0] = vox::grav_job_of(v, false);
        return vox::launch_cluster(jobs, (cudaStream_t)stream);
    }
    return vox::launch_grav_per_sweep(v, (cudaStream_t)stream);
}

int tpt_vox_grav_clear_mass(tpt_vox_plan *plan, const tpt_vox_world *w, tpt_stream_t stream) {
    if (!plan || !w) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_grav_clear_mass: NULL plan or world");
    int rc = check_ptrs("clear mass", {w->grav_mass});
    if (rc) return rc;
    return vox::launch_grav_clear(world_of(*w), (cudaStream_t)stream);
}

int tpt_vox_grav_gather(tpt_vox_plan *plan, const tpt_vox_world *w, tpt_stream_t stream) {
    if (!plan || !w) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_grav_gather: NULL plan or world");
    int rc = check_gather(w);
    if (!rc) rc = check_ptrs("gravity gather", {w->aux_tmp, w->grav_mass});
    if (rc) return rc;
    return vox::launch_grav_gather(world_of(*w), plan->brick_mult, (cudaStream_t)stream);
}

int tpt_vox_field_step(tpt_vox_plan *plan, const tpt_vox_world *worlds, uint32_t n, uint32_t air_iterations,
                       tpt_stream_t stream) {
    if (!plan) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_field_step: plan is NULL");
    if (n == 0) return TPT_OK;
    if (!worlds) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_field_step: worlds is NULL");
    if (air_iterations > kMaxAirIterations)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_vox_field_step: %u iterations (at most %u)", air_iterations,
                 kMaxAirIterations);
    for (uint32_t i = 0; i < n; ++i) {
        int rc = check_gather(&worlds[i]);
        if (!rc) rc = check_air_solve(&worlds[i]);
        if (!rc) rc = check_grav_solve(&worlds[i]);
        if (rc) return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (plan->form == TPT_VOX_BATCHED) {
        // per group of up to MAX_BWORLDS worlds: every world's gather, then
        // one batched launch sequence of air and gravity for all of them
        for (uint32_t first = 0; first < n; first += vox::MAX_BWORLDS) {
            const uint32_t m = n - first < vox::MAX_BWORLDS ? n - first : vox::MAX_BWORLDS;
            for (uint32_t i = first; i < first + m; ++i) {
                int rc = vox::launch_air_gather(world_of(worlds[i]), st);
                if (rc) return rc;
            }
            int rc = run_batch(plan, worlds + first, m, 3u, air_iterations, true, st);
            if (rc) return rc;
        }
        return TPT_OK;
    }
    if (plan->form != TPT_VOX_CLUSTER) {
        for (uint32_t i = 0; i < n; ++i) {
            const vox::World v = world_of(worlds[i]);
            int rc = vox::launch_air_gather(v, st);
            if (!rc) rc = vox::launch_air_per_sweep(v, air_iterations, plan->scratch, st);
            if (!rc) rc = vox::launch_grav_per_sweep(v, st);
            if (!rc) rc = vox::launch_grav_clear(v, st);
            if (rc) return rc;
        }
        return TPT_OK;
    }
    // Cluster form, per group of up to MAX_JOBS / 2 worlds: each world's
    // gather and pre-sweep pass, one launch of every world's air sweeps and
    // gravity solve side by side, then each world's advection.
    for (uint32_t first = 0; first < n; first += vox::MAX_JOBS / 2) {
        const uint32_t last = n - first < vox::MAX_JOBS / 2 ? n : first + vox::MAX_JOBS / 2;
        vox::Jobs jobs{};
        for (uint32_t i = first; i < last; ++i) {
            const vox::World v = world_of(worlds[i]);
            const vox::AirScratch sc = plan->slot(i - first);
            int rc = vox::launch_air_gather(v, st);
            if (!rc) rc = vox::launch_air_prep(v, sc, st);
            if (rc) return rc;
            jobs.job[jobs.n++] = vox::air_job_of(v, air_iterations, sc);
            jobs.job[jobs.n++] = vox::grav_job_of(v, true);
        }
        int rc = vox::launch_cluster(jobs, st);
        if (rc) return rc;
        for (uint32_t i = first; i < last; ++i) {
            rc = vox::launch_air_advect(world_of(worlds[i]), air_iterations, plan->slot(i - first), st);
            if (rc) return rc;
        }
    }
    return TPT_OK;
}

}  // extern "C"
