// grav_fft.cuh -- FP32 FFT convolution for the Newtonian gravity solve.
//
// Same maths as `FftBuffers::solve` (crates/tpt-sim/src/gravity_gpu/mod.rs:
// 204-278): the mass grid zero-padded to N1 x N2 = next_pow2(2X) x
// next_pow2(2Y), forward 2-D DFT, product with the kernel spectra, inverse
// 2-D DFT, real part of the top-left X x Y quadrant where the mask is set.
// The reference runs it as ~62 launches of global-memory radix-2 passes
// (mod.rs:285-335); here every 1-D transform runs in shared memory and the
// solve is three launches:
//
//   R  forward rows: Y mass rows -> Y spectrum rows (rows >= Y are zero and
//      never materialised)
//   C  per column block: forward column DFT, x/y kernel products, inverse
//      column DFT, keeping only the Y output rows both fields need
//   I  inverse rows: 2*Y rows -> real part of X outputs, masked
//
// Two forms of the transforms. The warp form (grav_fft_warp.cuh), for
// padded lengths 32 .. 1024 (lengths below 32 are padded up to 32): every
// 1-D transform is one warp's registers, the four-step factorisation with
// shuffles across lanes, no block barriers; the spectra stay in the warp
// FFT's permuted order between the passes, and the kernel spectra are stored
// in that order (column-major, so a warp's loads are coalesced). The shared-
// memory form, for longer lengths: forward is decimation-in-time fed in
// bit-reversed order, inverse is decimation-in-frequency read out in
// bit-reversed order, so no separate permutation pass exists. Twiddles come
// from a per-length table computed in double on the host and rounded once.
#pragma once

#include "common.cuh"

namespace tpt {
namespace gfft {

template <typename T> struct C2;
template <> struct C2<float> { using t = float2; };
template <> struct C2<double> { using t = double2; };

template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
    T2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename T2> __device__ __forceinline__ T2 cconj(T2 a) {
    a.y = -a.y;
    return a;
}

__device__ __forceinline__ uint32_t bitrev(uint32_t i, int log2n) { return __brev(i) >> (32 - log2n); }

// `ncols` independent length-n sequences at s[col*n + i], input in
// bit-reversed order, output in natural order. tw[k] = exp(-2 pi i k / n).
// `inverse` conjugates the twiddles. Block-wide; ends with __syncthreads().
template <typename T2>
__device__ void fft_dit(T2 *s, int n, int log2n, int ncols, const T2 *__restrict__ tw, bool inverse) {
    const int half_total = (n >> 1) * ncols;
    for (int lh = 0; lh < log2n; ++lh) {
        const int half = 1 << lh;
        const int tstride = n >> (lh + 1);
        for (int b = threadIdx.x; b < half_total; b += blockDim.x) {
            int col = b >> (log2n - 1);
            int k = b & ((n >> 1) - 1);
            int pos = k & (half - 1);
            int i0 = ((k >> lh) << (lh + 1)) + pos;
            T2 *base = s + (size_t)col * n;
            T2 w = __ldg(tw + pos * tstride);
            if (inverse) w = cconj(w);
            T2 x = base[i0], y = cmul(w, base[i0 + half]);
            base[i0].x = x.x + y.x;
            base[i0].y = x.y + y.y;
            base[i0 + half].x = x.x - y.x;
            base[i0 + half].y = x.y - y.y;
        }
        __syncthreads();
    }
}

// Natural-order input, bit-reversed output (decimation in frequency).
template <typename T2>
__device__ void fft_dif(T2 *s, int n, int log2n, int ncols, const T2 *__restrict__ tw, bool inverse) {
    const int half_total = (n >> 1) * ncols;
    for (int lh = log2n - 1; lh >= 0; --lh) {
        const int half = 1 << lh;
        const int tstride = n >> (lh + 1);
        for (int b = threadIdx.x; b < half_total; b += blockDim.x) {
            int col = b >> (log2n - 1);
            int k = b & ((n >> 1) - 1);
            int pos = k & (half - 1);
            int i0 = ((k >> lh) << (lh + 1)) + pos;
            T2 *base = s + (size_t)col * n;
            T2 w = __ldg(tw + pos * tstride);
            if (inverse) w = cconj(w);
            T2 x = base[i0], y = base[i0 + half];
            T2 d;
            d.x = x.x - y.x;
            d.y = x.y - y.y;
            base[i0].x = x.x + y.x;
            base[i0].y = x.y + y.y;
            base[i0 + half] = cmul(d, w);
        }
        __syncthreads();
    }
}

// One gravity solve's device state (a plan, or one instance of a batch).
struct Job {
    uint32_t X, Y, n1, n2;
    int l1, l2;                   // log2(n1), log2(n2)
    uint32_t pitch;               // row stride (elements) of mass, mask, gx, gy
    const int32_t *mass_i;        // fixed-point mass, or
    const float *mass_f;          // f32 mass (one of the two is set)
    float mass_scale_inv;
    const uint32_t *mask;
    float2 *work;                 // Y x n1 forward row spectra
    float2 *spec;                 // 2 x Y x n1 (x field, then y field)
    const float2 *kx, *ky;        // n2 x n1 kernel spectra (warp form: permuted, column-major)
    const float2 *tw1, *tw2;      // twiddles of length n1, n2 (n/2 entries; full circle in the warp form)
    float *gx, *gy;
};

// Per-call inputs/outputs of a one-job launch, passed by value so a solve
// with new pointers needs no table upload. `active` = 0: use the job's own.
struct JobIO {
    const int32_t *mass_i;
    const float *mass_f;
    const uint32_t *mask;
    float *gx, *gy;
    float mass_scale_inv;
    int active;
};

__device__ __forceinline__ Job load_job(const Job *jobs, uint32_t j, const JobIO &io) {
    Job J = jobs[j];
    if (io.active) {
        J.mass_i = io.mass_i;
        J.mass_f = io.mass_f;
        J.mask = io.mask;
        J.gx = io.gx;
        J.gy = io.gy;
        J.mass_scale_inv = io.mass_scale_inv;
    }
    return J;
}

// Block -> (job, item) maps, built on the host once per plan/batch.
struct BlockRef {
    uint32_t job;
    uint32_t item;  // row y (R), first column c0 (C), or field*Y + y (I)
};

}  // namespace gfft
}  // namespace tpt
