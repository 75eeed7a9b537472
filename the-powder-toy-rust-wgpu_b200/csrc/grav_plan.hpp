// grav_plan.hpp -- host-side objects of the gravity solve.
#pragma once

#include <vector>

#include "grav_fft.cuh"

namespace tpt {

struct JobShape {
    uint32_t X, Y;
};

namespace gfft {

uint32_t next_pow2(uint32_t v);
int build_spectra(uint32_t n1, uint32_t n2, double scale, float2 *kx, float2 *ky, double2 *out64);

// A set of independent FP32 FFT gravity solves (one plan = one job; a batch
// = one job per instance) that run as three launches.
struct FftSet {
    std::vector<Job> jobs_host;
    Job *jobs = nullptr;
    BlockRef *refs = nullptr;
    float2 *work = nullptr, *spec = nullptr, *kern = nullptr, *tw = nullptr;
    uint32_t n_rows = 0, n_cols = 0, n_inv = 0, max_n1 = 0, max_n2 = 0, max_y = 0;
    int cb_launch = 1, max_cb = 1;
    bool warp = false;  // every job's padded lengths lie in 32 .. 1024: the warp-register form

    int create(const std::vector<JobShape> &shapes);
    // Points job j at its inputs/outputs; returns 1 if anything changed
    // (the caller then re-uploads with upload_jobs()).
    int set_io(size_t j, const int32_t *mass_i, const float *mass_f, float inv, const uint32_t *mask, float *gx,
               float *gy, uint32_t pitch);
    int upload_jobs();
    // io != null: a one-job set solving on per-call pointers.
    int launch(cudaStream_t st, const JobIO *io = nullptr) const;
    void destroy();
    ~FftSet() { destroy(); }
};

}  // namespace gfft
}  // namespace tpt
