// field3d.hpp -- launchers of the 3-D sandbox's coarse field step.
#pragma once

#include "common.cuh"

namespace tpt {
namespace vox {

// One world's device buffers (the fields of tpt_vox_world).
struct World {
    const uint32_t *voxel;
    const int32_t *aux_tmp;
    const uint32_t *sim_list, *sim_count;
    float *vx, *vy, *vz, *p, *p_tmp, *temp, *solid;
    int32_t *pv;
    int32_t *grav_mass;
    float *grav_potential, *grav_potential_tmp;
    float *grav_force_x, *grav_force_y, *grav_force_z;
};

enum : uint32_t { JOB_AIR = 0, JOB_GRAV = 1 };

// One field of one world for the cluster kernel.
//   air:     f = p, p_tmp, divergence (scratch), solid
//   gravity: f = potential, potential_tmp, force x, y, z; i0 = mass
struct Job {
    float *f[7];
    int32_t *i0;
    uint32_t kind, iterations, clear_mass, pad;
};
constexpr uint32_t MAX_JOBS = 32;  // one launch; its parameters stay under 4 KiB
struct Jobs {
    uint32_t n;
    Job job[MAX_JOBS];
};
static_assert(sizeof(Jobs) <= 4096, "kernel parameters");

// Per-world scratch of the cluster form's air solve: the sweeps' divergence
// (one field) and the velocity snapshot (three fields).
struct AirScratch {
    float *div, *snap;
};
constexpr size_t AIR_SCRATCH_FLOATS = 4u * TPT_VOX_CELLS;

Job air_job_of(const World &w, uint32_t iterations, const AirScratch &sc);
// The grid-wide passes around the cluster sweeps: pv + divergence +
// snapshot before, advection after.
int launch_air_prep(const World &w, const AirScratch &sc, cudaStream_t st);
int launch_air_advect(const World &w, uint32_t iterations, const AirScratch &sc, cudaStream_t st);
Job grav_job_of(const World &w, bool clear_mass);

// ---- batched form (field3d_batch.cu) ----
// One world of a batched launch: its fields and its scratch.
struct BWorld {
    float *vx, *vy, *vz, *p, *p_tmp;
    const float *temp, *solid;
    int32_t *pv;
    int32_t *mass;
    float *pot, *pot_tmp, *fx, *fy, *fz;
    float *div, *snap, *src;  // scratch: divergence, velocity snapshot (3 fields), gravity source
    uint8_t *pin;             // scratch: pinned cells, 4 bits per x-quad
};
constexpr uint32_t MAX_BWORLDS = 16;  // per launch; the parameters stay under 4 KiB
struct Batch {
    uint32_t n;           // worlds
    uint32_t fields;      // bit 0 air solve, bit 1 gravity solve
    uint32_t air_iters;
    uint32_t clear_mass;  // clear grav_mass after the gravity solve
    BWorld w[MAX_BWORLDS];
};
static_assert(sizeof(Batch) <= 4096, "kernel parameters");
// Scratch bytes per world of a batch (divergence, snapshot, source, pins).
constexpr size_t BATCH_SCRATCH_BYTES = 5u * TPT_VOX_CELLS * sizeof(float) + TPT_VOX_CELLS / 4u;
// The pre-sweep pass, one launch per sweep index and the finishing pass of
// the batch's fields, as programmatic dependent launches on `st`.
int launch_batch(Batch &b, cudaStream_t st);

int launch_air_clear(const World &w, cudaStream_t st);
int launch_air_gather(const World &w, cudaStream_t st);
// gravity::gather; brick_mult is TPT_VOX_BRICKS words of scratch.
int launch_grav_gather(const World &w, uint32_t *brick_mult, cudaStream_t st);
int launch_grav_clear(const World &w, cudaStream_t st);
// Whether the device can hold one cluster of the cluster kernel.
int cluster_supported(bool *ok);
// One launch of the cluster kernel over jobs.n (<= MAX_JOBS) jobs.
int launch_cluster(const Jobs &jobs, cudaStream_t st);
// The reference's launch structure; `snapshot` holds 3 fields.
int launch_air_per_sweep(const World &w, uint32_t iterations, float *snapshot, cudaStream_t st);
int launch_grav_per_sweep(const World &w, cudaStream_t st);

}  // namespace vox
}  // namespace tpt
