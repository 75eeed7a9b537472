// grav_fft.cu -- kernels and plan of the FP32 FFT gravity solve; see
// grav_fft.cuh for the algorithm.
#include <math.h>

#include <algorithm>
#include <vector>

#include "grav_fft.cuh"
#include "grav_fft_warp.cuh"
#include "grav_plan.hpp"

namespace tpt {
namespace gfft {

constexpr int NT = 256;

// ---- per-solve kernels (FP32) ---------------------------------------------
__global__ void __launch_bounds__(NT) rows_forward(const Job *__restrict__ jobs, const BlockRef *__restrict__ refs,
                                                   const JobIO io) {
    extern __shared__ float2 sm2[];
    const BlockRef r = refs[blockIdx.x];
    const Job J = load_job(jobs, r.job, io);
    const uint32_t y = r.item;
    for (uint32_t i = threadIdx.x; i < J.n1; i += NT) sm2[i] = make_float2(0.f, 0.f);
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < J.X; x += NT) {
        size_t c = (size_t)y * J.pitch + x;
        float v = 0.0f;
        if (__ldg(J.mask + c) != 0u) v = J.mass_f ? __ldg(J.mass_f + c) : (float)__ldg(J.mass_i + c) * J.mass_scale_inv;
        sm2[bitrev(x, J.l1)] = make_float2(v, 0.f);
    }
    __syncthreads();
    fft_dit(sm2, (int)J.n1, J.l1, 1, J.tw1, false);
    float2 *dst = J.work + (size_t)y * J.n1;
    for (uint32_t k = threadIdx.x; k < J.n1; k += NT) dst[k] = sm2[k];
}

// `cb` columns per block (power of two dividing n1).
__global__ void __launch_bounds__(NT) cols_convolve(const Job *__restrict__ jobs, const BlockRef *__restrict__ refs,
                                                    int cb) {
    extern __shared__ float2 sm2[];
    const BlockRef r = refs[blockIdx.x];
    const Job J = jobs[r.job];
    const uint32_t c0 = r.item, n1 = J.n1, n2 = J.n2;
    float2 *P = sm2, *Q = sm2 + (size_t)cb * n2;
    for (uint32_t i = threadIdx.x; i < (uint32_t)cb * n2; i += NT) P[i] = make_float2(0.f, 0.f);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < J.Y * (uint32_t)cb; i += NT) {
        uint32_t j = i / cb, col = i - j * cb;
        P[(size_t)col * n2 + bitrev(j, J.l2)] = J.work[(size_t)j * n1 + c0 + col];
    }
    __syncthreads();
    fft_dit(P, (int)n2, J.l2, cb, J.tw2, false);
    for (uint32_t i = threadIdx.x; i < n2 * (uint32_t)cb; i += NT) {
        uint32_t k = i / cb, col = i - k * cb;
        size_t s = (size_t)col * n2 + k, g = (size_t)k * n1 + c0 + col;
        float2 p = P[s];
        Q[s] = cmul(p, __ldg(J.ky + g));
        P[s] = cmul(p, __ldg(J.kx + g));
    }
    __syncthreads();
    fft_dif(P, (int)n2, J.l2, 2 * cb, J.tw2, true);
    float2 *sx = J.spec, *sy = J.spec + (size_t)J.Y * n1;
    for (uint32_t i = threadIdx.x; i < J.Y * (uint32_t)cb; i += NT) {
        uint32_t j = i / cb, col = i - j * cb;
        size_t s = (size_t)col * n2 + bitrev(j, J.l2), g = (size_t)j * n1 + c0 + col;
        sx[g] = P[s];
        sy[g] = Q[s];
    }
}

__global__ void __launch_bounds__(NT) rows_inverse(const Job *__restrict__ jobs, const BlockRef *__restrict__ refs,
                                                   const JobIO io) {
    extern __shared__ float2 sm2[];
    const BlockRef r = refs[blockIdx.x];
    const Job J = load_job(jobs, r.job, io);
    const uint32_t field = r.item / J.Y, y = r.item - field * J.Y;
    const float2 *src = J.spec + ((size_t)field * J.Y + y) * J.n1;
    for (uint32_t k = threadIdx.x; k < J.n1; k += NT) sm2[k] = src[k];
    __syncthreads();
    fft_dif(sm2, (int)J.n1, J.l1, 1, J.tw1, true);
    float *out = field ? J.gy : J.gx;
    for (uint32_t x = threadIdx.x; x < J.X; x += NT) {
        size_t c = (size_t)y * J.pitch + x;
        out[c] = __ldg(J.mask + c) != 0u ? sm2[bitrev(x, J.l1)].x : 0.0f;
    }
}

// ---- the warp form: one warp per 1-D transform ---------------------------------
// 128-thread CTAs: the kernels hold a whole transform per warp in registers,
// so CTAs of four warps let several share an SM where CTAs of eight warps left
// registers unused (C4 solve 1.36 -> 1.06 ms). The register caps trade a few
// spills for more resident warps: forward rows 6 CTAs per SM (80 registers),
// columns 4 (128), inverse rows 5 (96); uncapped (91, 168, 158 registers: 5,
// 3, 3 CTAs) the C4 solve took 1.074 ms per tick, capped 0.988 ms.
constexpr int NTW = 128;
constexpr int WARPS = NTW / 32;

// Forward transform of mass row y (real, zero beyond X and where the mask is
// clear), stored in the warp FFT's permuted order.
template <int M> __device__ __forceinline__ void row_fwd_warp(const Job &J, uint32_t y, int lane) {
    float2 v[M];
#pragma unroll
    for (int j1 = 0; j1 < M; ++j1) {
        const uint32_t x = 32u * j1 + lane;
        float m = 0.0f;
        if (x < J.X) {
            const size_t c = (size_t)y * J.pitch + x;
            if (__ldg(J.mask + c) != 0u) m = J.mass_f ? __ldg(J.mass_f + c) : (float)__ldg(J.mass_i + c) * J.mass_scale_inv;
        }
        v[j1] = make_float2(m, 0.0f);
    }
    WarpFft<M>::forward(v, J.tw1, lane);
    float2 *dst = J.work + (size_t)y * J.n1;
#pragma unroll
    for (int k = 0; k < M; ++k) dst[32 * k + lane] = v[k];
}

__global__ void __launch_bounds__(NTW, 6) rows_forward_w(const Job *__restrict__ jobs, const BlockRef *__restrict__ refs,
                                                     uint32_t nrefs, const JobIO io) {
    const uint32_t w = blockIdx.x * WARPS + threadIdx.x / 32;
    if (w >= nrefs) return;
    const int lane = threadIdx.x & 31;
    const BlockRef r = refs[w];
    const Job J = load_job(jobs, r.job, io);
    switch (J.n1 >> 5) {
        case 1: row_fwd_warp<1>(J, r.item, lane); break;
        case 2: row_fwd_warp<2>(J, r.item, lane); break;
        case 4: row_fwd_warp<4>(J, r.item, lane); break;
        case 8: row_fwd_warp<8>(J, r.item, lane); break;
        case 16: row_fwd_warp<16>(J, r.item, lane); break;
        case 32: row_fwd_warp<32>(J, r.item, lane); break;
        default: break;
    }
}

// The mass and the kernels are real, so the x spectrum of every row is
// Hermitian: column n1 - kx of the convolved spectra is the conjugate of
// column kx. Only the n1/2 + 1 columns with kx <= n1/2 are convolved; in the
// warp FFT's storage order they are the even lanes' positions plus position 1
// (kx = n1/2). Half-column index h maps to its storage column:
__device__ __forceinline__ uint32_t half_col(uint32_t h, uint32_t m1) {
    return h < 16u * m1 ? (h >> 4) * 32u + 2u * (h & 15u) : 1u;
}

// One column (storage column c of the row spectra): forward transform down
// the column, product with each field's kernel spectrum, inverse transform;
// the Y rows both fields need are left in tx / ty (shared memory). tx holds
// the column's input before; fs (n2 entries, the same memory as ty) holds the
// forward spectrum while the two products are taken, in the lane order the
// registers use, so each lane reads back only what it wrote and the y field's
// rows overwrite only entries their own lane has read. The two fields share
// one copy of the inverse transform's code (a loop that is not unrolled).
template <int M>
__device__ __forceinline__ void col_warp(const Job &J, uint32_t c, float2 *tx, float2 *fs, int lane) {
    float2 g[M];
#pragma unroll
    for (int j1 = 0; j1 < M; ++j1) {
        const uint32_t j = 32u * j1 + lane;
        g[j1] = j < J.Y ? tx[j] : make_float2(0.0f, 0.0f);
    }
    WarpFft<M>::forward(g, J.tw2, lane);
#pragma unroll
    for (int k = 0; k < M; ++k) fs[32 * k + lane] = g[k];
    __syncwarp();
#pragma unroll 1
    for (int f = 0; f < 2; ++f) {
        const float2 *kf = (f ? J.ky : J.kx) + (size_t)c * J.n2;
#pragma unroll
        for (int k = 0; k < M; ++k) g[k] = cmulf(fs[32 * k + lane], __ldg(kf + 32 * k + lane));
        WarpFft<M>::inverse(g, J.tw2, lane);
        float2 *dst = f ? fs : tx;
#pragma unroll
        for (int j1 = 0; j1 < M; ++j1) {
            const uint32_t j = 32u * j1 + lane;
            if (j < J.Y) dst[j] = g[j1];
        }
    }
}

// A block takes WARPS consecutive half-column indices of one job: the Y x
// WARPS tile is staged through shared memory (each row's columns lie within
// 2 * WARPS consecutive positions), each warp transforms one column, and both
// fields' Y x WARPS tiles go back the same way. Per warp: `ystride` entries of
// the x field tile, `fstride` (>= n2) of the spectrum stash / y field tile.
__global__ void __launch_bounds__(NTW, 4) cols_convolve_w(const Job *__restrict__ jobs, const BlockRef *__restrict__ refs,
                                                      uint32_t ystride, uint32_t fstride) {
    extern __shared__ float2 sm2[];
    const BlockRef r = refs[blockIdx.x];
    const Job J = jobs[r.job];
    const uint32_t h0 = r.item, n1 = J.n1, Y = J.Y, m1 = n1 >> 5, nh = n1 / 2 + 1;
    float2 *TX = sm2, *TY = sm2 + (size_t)WARPS * ystride;
    for (uint32_t i = threadIdx.x; i < Y * WARPS; i += NTW) {
        const uint32_t j = i / WARPS, col = i - j * WARPS;
        if (h0 + col < nh) TX[(size_t)col * ystride + j] = J.work[(size_t)j * n1 + half_col(h0 + col, m1)];
    }
    __syncthreads();
    const int wi = threadIdx.x / 32, lane = threadIdx.x & 31;
    float2 *tx = TX + (size_t)wi * ystride, *ty = TY + (size_t)wi * fstride;
    if (h0 + wi < nh) {
        const uint32_t c = half_col(h0 + wi, m1);
        switch (J.n2 >> 5) {
            case 1: col_warp<1>(J, c, tx, ty, lane); break;
            case 2: col_warp<2>(J, c, tx, ty, lane); break;
            case 4: col_warp<4>(J, c, tx, ty, lane); break;
            case 8: col_warp<8>(J, c, tx, ty, lane); break;
            case 16: col_warp<16>(J, c, tx, ty, lane); break;
            case 32: col_warp<32>(J, c, tx, ty, lane); break;
            default: break;
        }
    }
    __syncthreads();
    float2 *sx = J.spec, *sy = J.spec + (size_t)Y * n1;
    for (uint32_t i = threadIdx.x; i < Y * WARPS; i += NTW) {
        const uint32_t j = i / WARPS, col = i - j * WARPS;
        if (h0 + col >= nh) continue;
        const size_t g = (size_t)j * n1 + half_col(h0 + col, m1);
        sx[g] = TX[(size_t)col * ystride + j];
        sy[g] = TY[(size_t)col * fstride + j];
    }
}

// Inverse transform of spectrum row y of both fields at once: both outputs
// are real, so gx + i gy is the inverse of Sx + i Sy. The full row spectra
// are rebuilt from the convolved half: position p of the permuted order holds
// frequency kx; an odd lane's position (except kx = n1/2) holds kx > n1/2,
// whose value is the conjugate of the stored kx' = n1 - kx. Outputs: the first
// X, masked.
template <int M> __device__ __forceinline__ void row_inv_warp(const Job &J, uint32_t y, int lane) {
    const float2 *rx = J.spec + (size_t)y * J.n1, *ry = J.spec + ((size_t)J.Y + y) * J.n1;
    float2 v[M];
#pragma unroll
    for (int k1 = 0; k1 < M; ++k1) {
        const bool direct = (lane & 1) == 0 || (k1 == 0 && lane == 1);
        uint32_t p = 32u * k1 + lane;
        if (!direct) {
            const uint32_t kx = (uint32_t)k1 + (uint32_t)M * (uint32_t)brev_c(lane, 5);
            const uint32_t km = J.n1 - kx;
            p = (km % (uint32_t)M) * 32u + (__brev(km / (uint32_t)M) >> 27);
        }
        float2 sx = rx[p], sy = ry[p];
        if (!direct) {
            sx.y = -sx.y;
            sy.y = -sy.y;
        }
        v[k1] = make_float2(sx.x - sy.y, sx.y + sy.x);  // sx + i sy
    }
    WarpFft<M>::inverse(v, J.tw1, lane);
#pragma unroll
    for (int j1 = 0; j1 < M; ++j1) {
        const uint32_t x = 32u * j1 + lane;
        if (x < J.X) {
            const size_t c = (size_t)y * J.pitch + x;
            const bool on = __ldg(J.mask + c) != 0u;
            J.gx[c] = on ? v[j1].x : 0.0f;
            J.gy[c] = on ? v[j1].y : 0.0f;
        }
    }
}

__global__ void __launch_bounds__(NTW, 5) rows_inverse_w(const Job *__restrict__ jobs, const BlockRef *__restrict__ refs,
                                                     uint32_t nrefs, const JobIO io) {
    const uint32_t w = blockIdx.x * WARPS + threadIdx.x / 32;
    if (w >= nrefs) return;
    const int lane = threadIdx.x & 31;
    const BlockRef r = refs[w];
    const Job J = load_job(jobs, r.job, io);
    switch (J.n1 >> 5) {
        case 1: row_inv_warp<1>(J, r.item, lane); break;
        case 2: row_inv_warp<2>(J, r.item, lane); break;
        case 4: row_inv_warp<4>(J, r.item, lane); break;
        case 8: row_inv_warp<8>(J, r.item, lane); break;
        case 16: row_inv_warp<16>(J, r.item, lane); break;
        case 32: row_inv_warp<32>(J, r.item, lane); break;
        default: break;
    }
}

// Kernel spectra from the natural order (row ky, column kx) into the warp
// form's layout: storage column c (frequency kx of permuted position c along
// x), then permuted position p along y.
__global__ void permute_spectrum(const float2 *__restrict__ nat, float2 *__restrict__ out, uint32_t n1, uint32_t n2) {
    const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (size_t)n1 * n2) return;
    const uint32_t c = (uint32_t)(id / n2), p = (uint32_t)(id - (size_t)c * n2);
    const uint32_t m1 = n1 / 32, m2 = n2 / 32;
    const uint32_t kx = (c / 32) + m1 * (uint32_t)brev_c((int)(c % 32), 5);
    const uint32_t ky = (p / 32) + m2 * (uint32_t)brev_c((int)(p % 32), 5);
    out[id] = nat[(size_t)ky * n1 + kx];
}

// ---- kernel spectra, FP64 (once per plan) ---------------------------------
// build_kernel_field_kernel (crates/tpt-sim/src/gravity_gpu/fft.rs:208-237)
// in double: K(d) = scale * d / |d|^3 with d folded into (-N/2, N/2].
__global__ void kernel_field_f64(double2 *out, uint32_t n1, uint32_t n2, double scale) {
    size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t cells = (size_t)n1 * n2;
    if (id >= cells) return;
    uint32_t px = (uint32_t)(id % n1), py = (uint32_t)(id / n1);
    double dx = px, dy = py;
    if (px * 2u >= n1) dx = (double)px - (double)n1;
    if (py * 2u >= n2) dy = (double)py - (double)n2;
    double vx = 0.0, vy = 0.0;
    if (dx != 0.0 || dy != 0.0) {
        double d = sqrt(dx * dx + dy * dy);
        double inv = scale / (d * d * d);
        vx = dx * inv;
        vy = dy * inv;
    }
    out[id] = make_double2(vx, 0.0);
    out[cells + id] = make_double2(vy, 0.0);
}

__global__ void spectrum_rows_f64(double2 *buf, uint32_t n1, uint32_t n2, int l1, const double2 *tw1) {
    extern __shared__ double2 smd[];
    const uint32_t row = blockIdx.x;  // field * n2 + y
    double2 *src = buf + (size_t)row * n1;
    for (uint32_t i = threadIdx.x; i < n1; i += blockDim.x) smd[bitrev(i, l1)] = src[i];
    __syncthreads();
    fft_dit(smd, (int)n1, l1, 1, tw1, false);
    for (uint32_t i = threadIdx.x; i < n1; i += blockDim.x) src[i] = smd[i];
}

__global__ void spectrum_cols_f64(const double2 *buf, uint32_t n1, uint32_t n2, int l2, const double2 *tw2,
                                  double2 *out64, float2 *kx, float2 *ky) {
    extern __shared__ double2 smd[];
    const uint32_t field = blockIdx.x / n1, c = blockIdx.x - field * n1;
    const double2 *src = buf + (size_t)field * n1 * n2;
    for (uint32_t j = threadIdx.x; j < n2; j += blockDim.x) smd[bitrev(j, l2)] = src[(size_t)j * n1 + c];
    __syncthreads();
    fft_dit(smd, (int)n2, l2, 1, tw2, false);
    float2 *dst = field ? ky : kx;
    for (uint32_t j = threadIdx.x; j < n2; j += blockDim.x) {
        double2 v = smd[j];
        if (out64) out64[(size_t)field * n1 * n2 + (size_t)j * n1 + c] = v;
        if (dst) dst[(size_t)j * n1 + c] = make_float2((float)v.x, (float)v.y);
    }
}

// Twiddle table exp(-2 pi i k / n), k < n/2 (or k < n: `full`), evaluated in
// double.
template <typename T2> static std::vector<T2> twiddles(uint32_t n, bool full = false) {
    std::vector<T2> t(std::max<uint32_t>(full ? n : n / 2, 1));
    for (uint32_t k = 0; k < t.size(); ++k) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        t[k].x = cos(a);
        t[k].y = sin(a);
    }
    return t;
}

static int log2u(uint32_t n) {
    int l = 0;
    while ((1u << l) < n) ++l;
    return l;
}

uint32_t next_pow2(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

int col_block(uint32_t n2) {
    int cb = 16;
    while (cb > 1 && (size_t)cb * 2 * n2 * sizeof(float2) > 96 * 1024) cb >>= 1;
    return cb;
}

int init_kernel_attrs() {
    static bool done = false;
    if (done) return TPT_OK;
    TPT_CUDA(cudaFuncSetAttribute(rows_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    TPT_CUDA(cudaFuncSetAttribute(cols_convolve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    TPT_CUDA(cudaFuncSetAttribute(rows_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    TPT_CUDA(cudaFuncSetAttribute(spectrum_rows_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024));
    TPT_CUDA(cudaFuncSetAttribute(spectrum_cols_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024));
    TPT_CUDA(cudaFuncSetAttribute(cols_convolve_w, cudaFuncAttributeMaxDynamicSharedMemorySize, WARPS * (512 + 1024) * 8));
    done = true;
    return TPT_OK;
}

// Builds the FP64 kernel spectra of an n1 x n2 transform and stores them as
// f32 (kx, ky) and/or keeps the f64 copy (out64: 2 x n2 x n1, may be null).
// `scale` = -M_GRAV / (n1 * n2). Synchronous.
int build_spectra(uint32_t n1, uint32_t n2, double scale, float2 *kx, float2 *ky, double2 *out64) {
    int rc = init_kernel_attrs();
    if (rc) return rc;
    size_t cells = (size_t)n1 * n2;
    double2 *buf = nullptr, *t1 = nullptr, *t2 = nullptr;
    auto tw1 = twiddles<double2>(n1), tw2 = twiddles<double2>(n2);
    cudaError_t e = cudaMalloc(&buf, 2 * cells * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&t1, tw1.size() * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&t2, tw2.size() * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemcpy(t1, tw1.data(), tw1.size() * sizeof(double2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t2, tw2.data(), tw2.size() * sizeof(double2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        kernel_field_f64<<<(unsigned)((cells + 255) / 256), 256>>>(buf, n1, n2, scale);
        count_launch();
        spectrum_rows_f64<<<2 * n2, 256, n1 * sizeof(double2)>>>(buf, n1, n2, log2u(n1), t1);
        count_launch();
        spectrum_cols_f64<<<2 * n1, 256, n2 * sizeof(double2)>>>(buf, n1, n2, log2u(n2), t2, out64, kx, ky);
        count_launch();
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    cudaFree(buf);
    cudaFree(t1);
    cudaFree(t2);
    if (e != cudaSuccess) TPT_FAIL(e == cudaErrorMemoryAllocation ? TPT_ERR_OUT_OF_MEMORY : TPT_ERR_CUDA,
                                   "gravity spectrum build failed: %s", cudaGetErrorString(e));
    return TPT_OK;
}

// The same spectra in the warp form's layout (permute_spectrum).
int build_spectra_permuted(uint32_t n1, uint32_t n2, double scale, float2 *kx, float2 *ky) {
    const size_t cells = (size_t)n1 * n2;
    float2 *nat = nullptr;
    TPT_CUDA(cudaMalloc(&nat, 2 * cells * sizeof(float2)));
    int rc = build_spectra(n1, n2, scale, nat, nat + cells, nullptr);
    if (rc == TPT_OK) {
        const unsigned blocks = (unsigned)((cells + 255) / 256);
        permute_spectrum<<<blocks, 256>>>(nat, kx, n1, n2);
        count_launch();
        permute_spectrum<<<blocks, 256>>>(nat + cells, ky, n1, n2);
        count_launch();
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            set_error("gravity spectrum permutation failed: %s", cudaGetErrorString(e));
            rc = TPT_ERR_CUDA;
        }
    }
    cudaFree(nat);
    return rc;
}

// ---- FFT gravity set (one plan or a batch) --------------------------------
int FftSet::create(const std::vector<JobShape> &shapes) {
    int rc = init_kernel_attrs();
    if (rc) return rc;
    destroy();
    const size_t nj = shapes.size();
    jobs_host.resize(nj);
    warp = true;
    for (const JobShape &sh : shapes)
        if (next_pow2(2 * sh.X) > 1024u || next_pow2(2 * sh.Y) > 1024u) warp = false;
    // padded lengths: next_pow2(2X) as the reference pads (gravity_gpu/mod.rs:
    // 140-167), at least 32 in the warp form (any length >= 2X gives the same
    // linear convolution)
    auto pad = [&](uint32_t v) { return warp ? std::max<uint32_t>(32u, next_pow2(2 * v)) : next_pow2(2 * v); };
    std::vector<BlockRef> rr, cr, ir;
    size_t work_elems = 0, spec_elems = 0, kern_elems = 0;
    std::vector<size_t> woff(nj), soff(nj), koff(nj);
    std::vector<std::pair<uint32_t, uint32_t>> sizes;  // distinct (n1, n2)
    std::vector<size_t> size_off;
    for (size_t j = 0; j < nj; ++j) {
        const JobShape &s = shapes[j];
        uint32_t n1 = pad(s.X), n2 = pad(s.Y);
        woff[j] = work_elems;
        work_elems += (size_t)s.Y * n1;
        soff[j] = spec_elems;
        spec_elems += (size_t)2 * s.Y * n1;
        auto key = std::make_pair(n1, n2);
        auto it = std::find(sizes.begin(), sizes.end(), key);
        if (it == sizes.end()) {  // spectra depend on the padded size only
            sizes.push_back(key);
            size_off.push_back(kern_elems);
            koff[j] = kern_elems;
            kern_elems += (size_t)2 * n1 * n2;
        } else {
            koff[j] = size_off[it - sizes.begin()];
        }
        max_n1 = std::max(max_n1, n1);
        max_n2 = std::max(max_n2, n2);
    }
    // one twiddle table per distinct length
    std::vector<uint32_t> lens;
    for (auto &s : shapes) {
        lens.push_back(pad(s.X));
        lens.push_back(pad(s.Y));
    }
    std::sort(lens.begin(), lens.end());
    lens.erase(std::unique(lens.begin(), lens.end()), lens.end());
    size_t tw_elems = 0;
    std::vector<size_t> twoff(lens.size());
    for (size_t i = 0; i < lens.size(); ++i) {
        twoff[i] = tw_elems;
        tw_elems += std::max<uint32_t>(warp ? lens[i] : lens[i] / 2, 1);
    }
    TPT_CUDA(cudaMalloc(&work, std::max<size_t>(work_elems, 1) * sizeof(float2)));
    TPT_CUDA(cudaMalloc(&spec, std::max<size_t>(spec_elems, 1) * sizeof(float2)));
    TPT_CUDA(cudaMalloc(&kern, std::max<size_t>(kern_elems, 1) * sizeof(float2)));
    TPT_CUDA(cudaMalloc(&tw, std::max<size_t>(tw_elems, 1) * sizeof(float2)));
    std::vector<float2> twh(tw_elems);
    for (size_t i = 0; i < lens.size(); ++i) {
        auto t = twiddles<float2>(lens[i], warp);
        std::copy(t.begin(), t.end(), twh.begin() + twoff[i]);
    }
    TPT_CUDA(cudaMemcpy(tw, twh.data(), tw_elems * sizeof(float2), cudaMemcpyHostToDevice));
    auto tw_of = [&](uint32_t n) {
        size_t i = std::lower_bound(lens.begin(), lens.end(), n) - lens.begin();
        return tw + twoff[i];
    };
    // kernel spectra: one build per distinct (n1, n2), copied to each job
    std::vector<std::pair<uint32_t, uint32_t>> built;
    std::vector<size_t> built_off;
    max_cb = 1;
    for (size_t j = 0; j < nj; ++j) {
        const JobShape &s = shapes[j];
        Job &J = jobs_host[j];
        J = Job{};
        J.X = s.X;
        J.pitch = s.X;
        J.Y = s.Y;
        J.n1 = pad(s.X);
        J.n2 = pad(s.Y);
        J.l1 = log2u(J.n1);
        J.l2 = log2u(J.n2);
        J.mass_scale_inv = 1.0f / 65536.0f;
        J.work = work + woff[j];
        J.spec = spec + soff[j];
        J.tw1 = tw_of(J.n1);
        J.tw2 = tw_of(J.n2);
        size_t plane = (size_t)J.n1 * J.n2;
        auto key = std::make_pair(J.n1, J.n2);
        auto it = std::find(built.begin(), built.end(), key);
        if (it == built.end()) {
            float2 *kx = kern + koff[j], *ky = kx + plane;
            double scale = -(double)6.673e-1f / ((double)J.n1 * (double)J.n2);
            int brc = warp ? build_spectra_permuted(J.n1, J.n2, scale, kx, ky)
                           : build_spectra(J.n1, J.n2, scale, kx, ky, nullptr);
            if (brc) return brc;
            built.push_back(key);
            built_off.push_back(koff[j]);
            J.kx = kx;
            J.ky = ky;
        } else {
            size_t o = built_off[it - built.begin()];
            J.kx = kern + o;
            J.ky = kern + o + plane;
        }
        for (uint32_t y = 0; y < s.Y; ++y) rr.push_back({(uint32_t)j, y});
        int cb = std::min<int>(col_block(J.n2), (int)J.n1);
        max_cb = std::max(max_cb, cb);
        // warp form: one inverse row per y (both fields); shared-memory form:
        // one per (field, y)
        for (uint32_t i = 0; i < (warp ? 1u : 2u) * s.Y; ++i) ir.push_back({(uint32_t)j, i});
    }
    // the column kernel needs one cb for the whole launch: use the smallest
    // needed by any job (power-of-two, divides every n1); the warp form
    // takes WARPS columns per block
    cb_launch = 16;
    for (auto &J : jobs_host) cb_launch = std::min(cb_launch, std::min<int>(col_block(J.n2), (int)J.n1));
    if (warp) cb_launch = WARPS;
    max_y = 0;
    for (auto &J : jobs_host) max_y = std::max(max_y, J.Y);
    cr.clear();
    for (size_t j = 0; j < nj; ++j) {
        // warp form: WARPS half-column indices per block (n1/2 + 1 columns)
        const uint32_t ncol = warp ? jobs_host[j].n1 / 2 + 1 : jobs_host[j].n1;
        for (uint32_t c = 0; c < ncol; c += cb_launch) cr.push_back({(uint32_t)j, c});
    }
    if (warp) {
        // blocks of the same transform length run the same code: keep them
        // together so that co-resident blocks share the instruction cache
        auto by = [&](bool col) {
            return [&, col](const BlockRef &a, const BlockRef &b) {
                const uint32_t la = col ? jobs_host[a.job].n2 : jobs_host[a.job].n1;
                const uint32_t lb = col ? jobs_host[b.job].n2 : jobs_host[b.job].n1;
                return la > lb;
            };
        };
        std::stable_sort(rr.begin(), rr.end(), by(false));
        std::stable_sort(cr.begin(), cr.end(), by(true));
        std::stable_sort(ir.begin(), ir.end(), by(false));
    }
    n_rows = (uint32_t)rr.size();
    n_cols = (uint32_t)cr.size();
    n_inv = (uint32_t)ir.size();
    TPT_CUDA(cudaMalloc(&jobs, nj * sizeof(Job)));
    TPT_CUDA(cudaMalloc(&refs, (rr.size() + cr.size() + ir.size()) * sizeof(BlockRef)));
    TPT_CUDA(cudaMemcpy(refs, rr.data(), rr.size() * sizeof(BlockRef), cudaMemcpyHostToDevice));
    TPT_CUDA(cudaMemcpy(refs + rr.size(), cr.data(), cr.size() * sizeof(BlockRef), cudaMemcpyHostToDevice));
    TPT_CUDA(cudaMemcpy(refs + rr.size() + cr.size(), ir.data(), ir.size() * sizeof(BlockRef), cudaMemcpyHostToDevice));
    return upload_jobs();
}

int FftSet::upload_jobs() {
    TPT_CUDA(cudaMemcpy(jobs, jobs_host.data(), jobs_host.size() * sizeof(Job), cudaMemcpyHostToDevice));
    return TPT_OK;
}

int FftSet::set_io(size_t j, const int32_t *mass_i, const float *mass_f, float inv, const uint32_t *mask, float *gx,
                   float *gy, uint32_t pitch) {
    Job &J = jobs_host[j];
    J.pitch = pitch;
    bool changed = J.mass_i != mass_i || J.mass_f != mass_f || J.mass_scale_inv != inv || J.mask != mask ||
                   J.gx != gx || J.gy != gy;
    J.mass_i = mass_i;
    J.mass_f = mass_f;
    J.mass_scale_inv = inv;
    J.mask = mask;
    J.gx = gx;
    J.gy = gy;
    return changed ? 1 : 0;
}

int FftSet::launch(cudaStream_t st, const JobIO *io) const {
    if (n_rows == 0) return TPT_OK;
    JobIO none{};
    const JobIO &a = io ? *io : none;
    if (warp) {
        rows_forward_w<<<(n_rows + WARPS - 1) / WARPS, NTW, 0, st>>>(jobs, refs, n_rows, a);
        TPT_LAUNCHED();
        cols_convolve_w<<<n_cols, NTW, (size_t)WARPS * (max_y + max_n2) * sizeof(float2), st>>>(jobs, refs + n_rows,
                                                                                               max_y, max_n2);
        TPT_LAUNCHED();
        rows_inverse_w<<<(n_inv + WARPS - 1) / WARPS, NTW, 0, st>>>(jobs, refs + n_rows + n_cols, n_inv, a);
        TPT_LAUNCHED();
        return TPT_OK;
    }
    rows_forward<<<n_rows, NT, max_n1 * sizeof(float2), st>>>(jobs, refs, a);
    TPT_LAUNCHED();
    cols_convolve<<<n_cols, NT, (size_t)cb_launch * 2 * max_n2 * sizeof(float2), st>>>(jobs, refs + n_rows,
                                                                                        cb_launch);
    TPT_LAUNCHED();
    rows_inverse<<<n_inv, NT, max_n1 * sizeof(float2), st>>>(jobs, refs + n_rows + n_cols, a);
    TPT_LAUNCHED();
    return TPT_OK;
}

void FftSet::destroy() {
    cudaFree(work);
    cudaFree(spec);
    cudaFree(kern);
    cudaFree(tw);
    cudaFree(jobs);
    cudaFree(refs);
    work = spec = kern = tw = nullptr;
    jobs = nullptr;
    refs = nullptr;
    jobs_host.clear();
    n_rows = n_cols = n_inv = 0;
    max_n1 = max_n2 = max_y = 0;
    warp = false;
}

}  // namespace gfft
}  // namespace tpt
