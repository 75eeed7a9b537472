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
//   air:     f = vx, vy, vz, p, p_tmp, temp, solid; i0 = pv
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

Job air_job_of(const World &w, uint32_t iterations);
Job grav_job_of(const World &w, bool clear_mass);

int launch_air_clear(const World &w, cudaStream_t st);
int launch_air_gather(const World &w, cudaStream_t st);
int launch_grav_gather(const World &w, cudaStream_t st);
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
