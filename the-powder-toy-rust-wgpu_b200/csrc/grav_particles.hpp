// grav_particles.hpp -- launchers of the particle side of a gravity tick.
#pragma once

#include "common.cuh"

namespace tpt {
namespace gp {

// One sandbox's gravity grids (xcells * ycells cells each).
struct GravGrids {
    uint32_t xres, yres, xcells, ycells;
    const uint32_t *wall, *emap, *mask;
    int32_t *mass, *prev;
    float *tool;              // may be NULL
    const int32_t *ovr;       // may be NULL
    const uint32_t *ovr_set;  // may be NULL
    const float *gx, *gy;
    float newton;
};

// Particle slots (struct of arrays).
struct Parts {
    uint32_t n, n_types;
    const uint32_t *ty;
    const float *x, *y;
    float *vx, *vy;
    const int32_t *life, *tmp;
    const float *temp;
    const uint32_t *flags, *lut;
};

// Wells into the snapshot, accumulator cleared (before the solve).
int launch_seed(const GravGrids &G, cudaStream_t st);
// Force and mass build over the slots, then overrides and the snapshot copy
// (after the solve).
int launch_particles_and_finish(const GravGrids &G, const Parts &P, cudaStream_t st);

}  // namespace gp
}  // namespace tpt
