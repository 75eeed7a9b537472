// grav_fft_warp.cuh -- one warp, one FFT of length n = 32 * M (M = 1 .. 32),
// held in registers: the four-step factorisation n = M x 32.
//
// Lane L holds the M inputs x[32 j1 + L] (j1 = 0 .. M-1), a coalesced row of
// the sequence. With k = k1 + M k2,
//
//   X[k1 + M k2] = sum_j2 W32^(j2 k2) [ Wn^(j2 k1) sum_j1 x[32 j1 + j2] WM^(j1 k1) ]
//
// so the forward transform is (1) an M-point DFT in each lane's registers,
// (2) a multiply by the twiddle Wn^(L k1), (3) a 32-point DFT across the lanes
// for every k1, as five radix-2 decimation-in-frequency stages over
// __shfl_xor_sync. Lane L then holds X[k1 + M * bitrev5(L)] in register k1:
// the spectrum in a fixed permuted order, which the gravity solve keeps
// end to end (its kernel spectra are stored in the same order) so no
// permutation pass exists. The inverse runs the three steps backwards with
// conjugate twiddles (each radix-2 stage undone by its decimation-in-time
// mirror) and returns the unnormalised inverse x[32 j1 + L] in natural order.
//
// Twiddles come from a table tw[k] = exp(-2 pi i k / n), k < n, computed in
// double on the host and rounded once.
#pragma once

#include "common.cuh"

namespace tpt {
namespace gfft {

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulcf(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ constexpr int brev_c(int v, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
    return r;
}
__host__ __device__ constexpr int log2_c(int v) { return v <= 1 ? 0 : 1 + log2_c(v >> 1); }

template <int M> struct WarpFft {
    static constexpr int LM = log2_c(M);

    // In-register M-point DFT, natural order in and out (radix-2 DIF, then a
    // register renaming into natural order). Twiddles W_M^t = tw[32 t].
    __device__ static __forceinline__ void dft_regs(float2 (&v)[M], const float2 *__restrict__ tw) {
#pragma unroll
        for (int half = M / 2; half >= 1; half >>= 1) {
#pragma unroll
            for (int blk = 0; blk < M; blk += 2 * half) {
#pragma unroll
                for (int p = 0; p < half; ++p) {
                    const float2 a = v[blk + p], b = v[blk + p + half];
                    v[blk + p] = make_float2(a.x + b.x, a.y + b.y);
                    const float2 d = make_float2(a.x - b.x, a.y - b.y);
                    v[blk + p + half] = p == 0 ? d : cmulf(d, __ldg(tw + 32 * p * (M / (2 * half))));
                }
            }
        }
        float2 t[M];
#pragma unroll
        for (int k = 0; k < M; ++k) t[k] = v[brev_c(k, LM)];
#pragma unroll
        for (int k = 0; k < M; ++k) v[k] = t[k];
    }

    // Its mirror: natural in, unnormalised inverse natural out (x M).
    __device__ static __forceinline__ void idft_regs(float2 (&v)[M], const float2 *__restrict__ tw) {
        float2 t[M];
#pragma unroll
        for (int k = 0; k < M; ++k) t[brev_c(k, LM)] = v[k];
#pragma unroll
        for (int k = 0; k < M; ++k) v[k] = t[k];
#pragma unroll
        for (int half = 1; half <= M / 2; half <<= 1) {
#pragma unroll
            for (int blk = 0; blk < M; blk += 2 * half) {
#pragma unroll
                for (int p = 0; p < half; ++p) {
                    const float2 c = v[blk + p];
                    const float2 d = p == 0 ? v[blk + p + half]
                                            : cmulcf(v[blk + p + half], __ldg(tw + 32 * p * (M / (2 * half))));
                    v[blk + p] = make_float2(c.x + d.x, c.y + d.y);
                    v[blk + p + half] = make_float2(c.x - d.x, c.y - d.y);
                }
            }
        }
    }

    // Forward: v[j1] = x[32 j1 + lane] -> v[k1] = X[k1 + M * bitrev5(lane)].
    __device__ static __forceinline__ void forward(float2 (&v)[M], const float2 *__restrict__ tw, int lane) {
        dft_regs(v, tw);
#pragma unroll
        for (int k = 1; k < M; ++k) v[k] = cmulf(v[k], __ldg(tw + lane * k));
#pragma unroll
        for (int s = 16; s >= 1; s >>= 1) {
            const int q = lane & (s - 1);
            const float2 w = __ldg(tw + q * (16 / s) * M);  // W_(2s)^q
            const bool upper = (lane & s) != 0;
#pragma unroll
            for (int k = 0; k < M; ++k) {
                float2 p;
                p.x = __shfl_xor_sync(0xffffffffu, v[k].x, s);
                p.y = __shfl_xor_sync(0xffffffffu, v[k].y, s);
                if (!upper) {
                    v[k] = make_float2(v[k].x + p.x, v[k].y + p.y);
                } else {
                    v[k] = cmulf(make_float2(p.x - v[k].x, p.y - v[k].y), w);
                }
            }
        }
    }

    // Inverse of forward, unnormalised (x n): v[k1] = X[k1 + M * bitrev5(lane)]
    // -> v[j1] = sum_k X[k] Wn^(-(32 j1 + lane) k).
    __device__ static __forceinline__ void inverse(float2 (&v)[M], const float2 *__restrict__ tw, int lane) {
#pragma unroll
        for (int s = 1; s <= 16; s <<= 1) {
            const int q = lane & (s - 1);
            const float2 w = __ldg(tw + q * (16 / s) * M);
            const bool upper = (lane & s) != 0;
#pragma unroll
            for (int k = 0; k < M; ++k) {
                // lower lane: c = own, d = partner; upper lane: c = partner, d = own
                const float2 dd = upper ? v[k] : make_float2(0.f, 0.f);
                float2 p;
                p.x = __shfl_xor_sync(0xffffffffu, v[k].x, s);
                p.y = __shfl_xor_sync(0xffffffffu, v[k].y, s);
                if (!upper) {
                    const float2 dw = cmulcf(p, w);
                    v[k] = make_float2(v[k].x + dw.x, v[k].y + dw.y);
                } else {
                    const float2 dw = cmulcf(dd, w);
                    v[k] = make_float2(p.x - dw.x, p.y - dw.y);
                }
            }
        }
#pragma unroll
        for (int k = 1; k < M; ++k) v[k] = cmulcf(v[k], __ldg(tw + lane * k));
        idft_regs(v, tw);
    }
};

// Storage position (0 .. n-1) of frequency k in the permuted order above:
// k = k1 + M k2 is held by lane bitrev5(k2) in register k1, stored at
// k1 * 32 + lane.
__host__ __device__ inline uint32_t perm_pos(uint32_t k, uint32_t M) {
    const uint32_t k1 = k % M, k2 = k / M;
    return k1 * 32u + (uint32_t)brev_c((int)k2, 5);
}

}  // namespace gfft
}  // namespace tpt
