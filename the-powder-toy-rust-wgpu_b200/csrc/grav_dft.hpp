// grav_dft.hpp -- host side of the split-BF16 DFT-as-GEMM gravity solve.
#pragma once

#include <vector>

#include "common.cuh"
#include "grav_plan.hpp"

namespace tpt {
namespace dft {

// Per-call inputs/outputs of a one-job solve.
struct SolveIO {
    const int32_t *mass_i;
    const float *mass_f;
    const uint32_t *mask;
    float *gx, *gy;
    float mass_scale_inv;
    uint32_t pitch;  // row stride (elements) of mass, mask, gx, gy
};

struct DftImpl;

// A set of independent split-BF16 gravity solves (one plan = one job; a
// batch = one job per instance).
struct DftSet {
    DftImpl *impl = nullptr;
    int create(const std::vector<JobShape> &shapes);
    void dims(size_t j, uint32_t *n1, uint32_t *n2) const;
    // Binds job j to fixed inputs/outputs (a batch's arenas).
    int set_io(size_t j, const SolveIO &io);
    int launch(cudaStream_t st, const SolveIO *io = nullptr) const;
    // Concurrent y stages: true when the set holds both Toeplitz and
    // DFT-pair groups; set_side_ctas(c > 0) then runs the DFT-pair groups'
    // chain on a second stream with c CTAs per launch (0: one stream).
    bool can_split() const;
    bool split_active() const;
    uint32_t max_side_ctas() const;
    int set_side_ctas(uint32_t ctas);
    // kernel launches and executed tensor flops of one launch() of the set
    uint32_t launches() const;
    double flops() const;
    void destroy();
    ~DftSet() { destroy(); }
};

}  // namespace dft
}  // namespace tpt

namespace tpt {
namespace dft {
// Reads and clears the device error word of the tensor-core kernels.
int read_errors(uint32_t *out);
}  // namespace dft
}  // namespace tpt
