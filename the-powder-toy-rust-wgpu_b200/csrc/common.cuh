// common.cuh -- shared definitions of the B200 field-step library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <string>

#include "../../include/tpt_field.h"

namespace tpt {

// ------------------------------------------------------------ errors ----
// Thread-local message of the last failure; set by `fail()`.
void set_error(const char *fmt, ...);
inline int fail_code(int code) { return code; }

#define TPT_FAIL(code, ...)            \
    do {                               \
        ::tpt::set_error(__VA_ARGS__); \
        return (code);                 \
    } while (0)

#define TPT_CUDA(call)                                                                                         \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) {                                                                               \
            ::tpt::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);        \
            return (e_ == cudaErrorMemoryAllocation) ? TPT_ERR_OUT_OF_MEMORY : TPT_ERR_CUDA;                    \
        }                                                                                                      \
    } while (0)

// Checks the launch that was just issued.
#define TPT_LAUNCHED()                                                                                         \
    do {                                                                                                       \
        ::tpt::count_launch();                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                                                   \
        if (e_ != cudaSuccess) {                                                                               \
            ::tpt::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__);  \
            return TPT_ERR_CUDA;                                                                               \
        }                                                                                                      \
    } while (0)

void count_launch();

// Fails unless the current device is an sm_100 part.
int require_sm100();

// ------------------------------------------------------- air instance ----
// Everything one air step of one instance needs, in device-visible form.
struct AirInst {
    uint32_t X, Y;
    uint32_t pitch;  // row stride (elements) of every grid of the instance
    uint32_t air_mode, aheat, conv, gmode;
    float ep, evx, evy, amb, vcoef, cgx, cgy;
    float vk;  // vcoef / 5 (advect.rs:317), divided once on the host in f32
    float *pv, *vx, *vy, *hv;
    float *opv, *ovx, *ovy, *ohv;
    uint32_t *bair, *bairh;
    const uint32_t *wall;
    uint32_t *emap;
    const uint32_t *eair, *eairh;
    const float *fvx, *fvy;
    // where the step writes the rebuilt masks and the new heat. For the
    // one-tick entry point these are scratch and a settle pass copies them;
    // for a batch they are the other half of a ping-pong pair.
    uint32_t *bair_out, *bairh_out;
    float *hv_out;
    // the batch's sweep writes the new pv/vx/vy to the other half of their
    // ping-pong pairs (the one-grid step updates pv/vx/vy in place: null)
    float *pv_out, *vx_out, *vy_out;
};

// AirInst with the scalar fields of `p` set and every pointer null.
AirInst make_air_inst(const tpt_air_params &p);

// Air tile shape (cells). One CTA of AIR_TX*AIR_TY threads owns one tile.
constexpr int AIR_TX = 32;
constexpr int AIR_TY = 8;

}  // namespace tpt
