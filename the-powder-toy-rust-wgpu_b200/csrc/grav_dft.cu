// grav_dft.cu -- the gravity solve as split-BF16 DFT-as-GEMM on tcgen05.
//
// Same result as the FFT solve (crates/tpt-sim/src/gravity_gpu/mod.rs:204-278):
// g = mask * (mass * K) for K(d) = -M_GRAV d / |d|^3, the linear convolution
// of the X x Y mass grid, computed through an N1 x N2 = 2X x 2Y padded DFT.
// The 1-D transforms are dense matrix products on the tensor cores:
//
//   R    A[y,kx]  = sum_x  m[y,x]   e^{-2 pi i kx x / N1}    kx < N1/2+1 (Hermitian half)
//   C    B[ky,kx] = sum_y  F2[ky,y] A[y,kx]                  F2 = e^{-2 pi i ky y / N2}
//        S_f      = B * i Ks_f[ky,kx]                         (kernel spectra are imaginary)
//   C^-1 C_f[y,kx]= sum_ky G2[y,ky] S_f[ky,kx]               G2 = e^{+2 pi i y ky / N2}
//   R^-1 g_f[y,x] = sum_kx Re(C_f[y,kx] w_kx e^{+2 pi i kx x / N1})   w = 1, 2, ..., 2, 1
//
// Every operand is stored as bf16 hi/lo planes (v = hi + lo, 16 significant
// bits) and each product is the 3-term split hi*hi + hi*lo + lo*hi,
// accumulated in FP32 in TMEM. Instances of equal shape form a group whose
// data operands are stacked along M or N, so a group is four GEMMs; all
// groups' tiles run in one persistent launch per stage. The kernel spectra
// and DFT matrices are built once in FP64 on the device.
//
// Groups with many instances replace the C / C^-1 pair by one direct
// (Toeplitz) convolution along y per x frequency, which needs no padding to
// 2Y and no y spectrum:
//
//   T    C_f[y,kx] = sum_y' Tf_kx[y - y'] A[y',kx]     Tf_kx(dy) = sum_dx K_f(dx,dy) e^{-2 pi i kx dx/N1} / N1
//
// Tx is purely imaginary (Kx is odd in dx) and Ty real (Ky is even in dx),
// so T is a real GEMM per (f, kx): M = the group's instances' real and
// imaginary parts (2G rows), K = y', N = y. Its B operand, the Y x Y
// Toeplitz matrix, is a window of a strip precomputed once per (f, kx)
// (one TMA load per tile). Its epilogue writes R^-1's A operand M-major,
// rows m' = ((y / 8) * G + inst) * 8 + y % 8 per (f, kx), which R^-1 reads
// as an MN-major tcgen05 operand. Groups of at least 8 instances with
// Y <= 256 take T; smaller groups are cheaper through the y DFT.
//
// R^-1 keeps only the real part, so it runs as one real GEMM over the
// concatenated K' = [kx of Re C | kx of Im C] against [G1r ; -G1i] (the
// second half with the A-negate bit), with 256-wide N tiles.
//
// GEMM kernel: 320 threads. Warp 0 issues TMA tile loads (64-byte swizzle,
// 32-wide K tiles, no multicast) into a shared-memory ring of 3 to 6
// stages; warp 1 issues tcgen05.mma (M=128, N<=256, K=16) into a
// double-buffered TMEM accumulator; warps 2-9 read the accumulator with
// tcgen05.ld and run the stage's epilogue, which writes the next stage's
// operand planes. Every mbarrier wait is bounded (see tc.cuh).
#include <cudaTypedefs.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <vector>

#include "grav_dft.hpp"
#include "tc.cuh"

namespace tpt {
namespace dft {

using bf16 = __nv_bfloat16;

constexpr int KT = 32;             // K elements per tile (64 bytes)
constexpr int MT = 128;            // rows per M tile
constexpr int NT = 128;            // complex columns per N tile
constexpr int TILE_BYTES = MT * KT * 2;      // one plane of one tile: 8 KB
constexpr int RING_BYTES = 24 * TILE_BYTES;  // shared-memory ring of K-tile stages: 192 KB
// R and R^-1: 3 stages of 48 KB and no transpose buffers (their epilogues
// store straight from registers). Smaller than the others' 231 KB, so an SM
// running one of them keeps room for air CTAs beside it; measured on the C5
// step 0.640 -> 0.636 ms per tick (gravity alone 0.244 -> 0.240 ms).
constexpr int RING_R_BYTES = 18 * TILE_BYTES;
constexpr int MAX_STAGES = 6;
constexpr int EPI_WARPS = 8;             // two per TMEM lane quarter, one column half each
constexpr int XPOSE_BYTES = 32 * 33 * 4; // per epilogue warp: a 32x32 f32 transpose buffer
constexpr int SMEM_BYTES = RING_BYTES + 1024 + EPI_WARPS * XPOSE_BYTES;
constexpr int SMEM_R_BYTES = RING_R_BYTES + 1024;
constexpr int THREADS = 64 + 32 * EPI_WARPS;

// Toeplitz stage T. A Toeplitz matrix shifted by 32 columns is the same
// matrix shifted by 32 rows, so the B operand of every K tile of a T tile
// is a window of one strip of (N + K - 32) rows x 32 columns, loaded once
// per tile: K tile kt reads rows from (K - 32 - 32 kt). T groups have
// Y <= T_NMAX, so one N tile covers all y.
constexpr int T_NMAX = 256;                          // y rows of a T tile (MMA N at most)
constexpr int T_STRIP_ROWS = 512;                    // strip buffer rows (>= 2 T_NMAX - 32 + box rounding)
constexpr int T_STRIP_PLANE = T_STRIP_ROWS * KT * 2; // 32 KB
constexpr int T_RING_BYTES = 6 * 2 * TILE_BYTES;     // T's A stages: 6 x 16 KB
static_assert(T_RING_BYTES + 2 * 2 * T_STRIP_PLANE + 1024 <= SMEM_BYTES, "T shared memory");
static_assert(T_STRIP_ROWS >= 2 * T_NMAX - KT + 2 * 7, "strip buffer holds two rounded boxes");

enum Stage : int { ST_R = 0, ST_C = 1, ST_CI = 2, ST_RI = 3, ST_T = 4 };

__device__ uint32_t g_dft_err;

// One group of equal-shape instances (device copy).
struct Group {
    uint32_t X, Y, N1, N2, N1h, G, inst0;
    uint32_t N1hp;                       // N1h rounded up to 32: per-instance column stride of C and C^-1
    uint32_t kpR, kpC, kpCi, kpRi;       // K pitches (elements)
    uint32_t rowsR, rowsC, rowsCi, rowsRi;  // rows per plane of the data operands
    uint32_t toe;                        // 1: y stage is the Toeplitz GEMM T
    uint32_t rowsT;                      // T: rows per plane of its A operand bT (N1h * 2G)
    uint32_t nTy;                        // T: MMA N (Y rounded up to 16)
    uint32_t Yp;                         // T: rows per instance in aRiT (Y rounded up to 8)
    uint32_t MpT;                        // T: row length of aRiT (G * Yp rounded up to 32)
    uint32_t SR, sbox, snb;              // T: strip rows per (f, kx); TMA box rows; boxes per strip
    uint32_t wR, wRI;                    // N tile widths of R (complex columns) and R^-1 (multiples of 16)
    bf16 *aR, *bC, *bCi, *aRi;           // data operands (planes stacked), DFT form
    bf16 *bT, *aRiT;                     // T's A operand [plane][kx][inst][re/im][y]; R^-1's A [plane][f][kx][m']
    const float *kxs, *kys;              // imaginary parts of the kernel spectra, [kx][ky]
};

struct InstIO {
    const int32_t *mass_i;
    const float *mass_f;
    const uint32_t *mask;
    float *gx, *gy;
    float inv;
    uint32_t pitch;  // row stride of the four grids
};

struct Problem {
    const CUtensorMap *ta, *tb;
    uint32_t group, M, N, ktiles, a_rows, b_rows;
    uint32_t a_mn;  // R^-1 of a Toeplitz group: A is MN-major (aRiT), field f = a_mn - 1
};

struct Tile {
    uint32_t problem;
    uint16_t mt, nt;
    uint32_t sub;  // Toeplitz stage: f * N1h + kx (the matrix of this tile)
};

// ---- helpers ---------------------------------------------------------------
__device__ __forceinline__ void split_store(bf16 *hi, bf16 *lo, float v) {
    bf16 h = __float2bfloat16_rn(v);
    *hi = h;
    *lo = __float2bfloat16_rn(v - __bfloat162float(h));
}

// Splits 32 floats (times sgn) into packed bf16 hi and lo words.
__device__ __forceinline__ void split_pack32(const float (&v)[32], float sgn, uint32_t (&hw)[16], uint32_t (&lw)[16]) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float v0 = sgn * v[2 * i], v1 = sgn * v[2 * i + 1];
        const bf16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
        const bf16 l0 = __float2bfloat16_rn(v0 - __bfloat162float(h0));
        const bf16 l1 = __float2bfloat16_rn(v1 - __bfloat162float(h1));
        hw[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        lw[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
}

// ---- the GEMM kernel ---------------------------------------------------------
template <int STAGE>
__global__ void __launch_bounds__(THREADS, 1)
    dft_gemm(const Problem *__restrict__ probs, const Tile *__restrict__ tiles, uint32_t ntiles,
             const Group *__restrict__ groups, const InstIO *__restrict__ ios, InstIO io0, int io0_active,
             uint32_t *err) {
    // R^-1 keeps only the real part, so it runs as one real GEMM over K' =
    // [kx of Re C | kx of Im C] against [G1r ; -G1i]: each K tile loads one
    // hi/lo plane pair of A and of B, and its N tiles are 256 wide. T's B
    // (the Toeplitz strip) lives outside the ring.
    constexpr bool A_COMPLEX = STAGE == ST_C || STAGE == ST_CI;
    constexpr bool B_COMPLEX = STAGE == ST_R || STAGE == ST_C || STAGE == ST_CI;
    constexpr bool OUT_COMPLEX = B_COMPLEX;
    constexpr bool WIDE = STAGE == ST_RI || STAGE == ST_T;         // real N tiles of 256
    constexpr uint32_t NTS = WIDE ? 2 * NT : NT;                     // N tile (complex columns if complex)
    constexpr uint32_t A_PLANES = A_COMPLEX ? 4 : 2;
    constexpr uint32_t B_PLANES = STAGE == ST_T ? 0 : (B_COMPLEX ? 4 : 2);
    constexpr uint32_t BPB = STAGE == ST_RI ? 2 * TILE_BYTES : TILE_BYTES;  // bytes of one B plane
    constexpr uint32_t SBYTES = A_PLANES * TILE_BYTES + B_PLANES * BPB;   // one stage
    constexpr uint32_t RING = STAGE == ST_T                       ? T_RING_BYTES
                              : (STAGE == ST_R || STAGE == ST_RI) ? RING_R_BYTES
                                                                  : RING_BYTES;
    constexpr uint32_t NSTG = RING / SBYTES < MAX_STAGES ? RING / SBYTES : MAX_STAGES;  // 3 (C, C^-1), 4, 6 (T)
    constexpr uint32_t B_OFF = A_PLANES * TILE_BYTES;
    constexpr uint32_t BLO = (B_COMPLEX ? 2 : 1) * BPB;  // B lo block from B hi block
    static_assert(NSTG >= 3, "stage ring");

    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *strip = smem + T_RING_BYTES;  // T: two strip buffers, [hi plane | lo plane] each
    __shared__ uint64_t full_bar[MAX_STAGES], empty_bar[MAX_STAGES], acc_full[2], acc_empty[2];
    __shared__ uint64_t strip_full[2], strip_empty[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < NSTG; ++s) {
            tc::mbar_init(&full_bar[s], 1);
            tc::mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&acc_full[a], 1);
            tc::mbar_init(&acc_empty[a], EPI_WARPS);
            tc::mbar_init(&strip_full[a], 1);
            tc::mbar_init(&strip_empty[a], 1);
        }
        abort_flag = 0;
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(&tmem_slot, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            uint32_t s = 0, ph = 0, tl = 0;
            for (uint32_t t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++tl) {
                const Tile T = tiles[t];
                const Problem P = probs[T.problem];
                int32_t m0 = T.mt * MT;
                // R and R^-1 tiles are the group's N width (little padding of N1h or X)
                const uint32_t wN = STAGE == ST_R ? groups[P.group].wR : STAGE == ST_RI ? groups[P.group].wRI : NTS;
                const int32_t n0 = T.nt * wN;
                const uint32_t tx = STAGE == ST_R    ? 2 * TILE_BYTES + 4 * wN * KT * 2
                                    : STAGE == ST_RI ? 2 * TILE_BYTES + 2 * wN * KT * 2
                                                     : SBYTES;
                if (STAGE == ST_T) {
                    // A = this tile's frequency slice of bT; B = the (f, kx) strip
                    const Group &Gq = groups[P.group];
                    m0 += (int32_t)((T.sub % Gq.N1h) * 2 * Gq.G);
                    const uint32_t sb = tl & 1u;
                    if (!tc::mbar_wait(&strip_empty[sb], ((tl >> 1) & 1u) ^ 1u, err)) {
                        abort_flag = 1;
                        break;
                    }
                    uint8_t *sdst = strip + sb * 2 * T_STRIP_PLANE;
                    tc::mbar_arrive_expect_tx(&strip_full[sb], 2 * Gq.snb * Gq.sbox * KT * 2);
                    for (uint32_t p = 0; p < 2; ++p)
                        for (uint32_t b = 0; b < Gq.snb; ++b)
                            tc::tma_load_2d(sdst + p * T_STRIP_PLANE + b * Gq.sbox * KT * 2, P.tb, 0,
                                            (int32_t)((p * 2 * Gq.N1h + T.sub) * Gq.SR + b * Gq.sbox),
                                            &strip_full[sb]);
                }
                for (uint32_t kt = 0; kt < P.ktiles; ++kt) {
                    if (!tc::mbar_wait(&empty_bar[s], ph ^ 1u, err)) {
                        abort_flag = 1;
                        break;
                    }
                    uint8_t *st = smem + s * SBYTES;
                    tc::mbar_arrive_expect_tx(&full_bar[s], tx);
                    if (STAGE == ST_RI) {
                        // K' tile kt: real parts (planes 0, 1), then imaginary parts (2, 3)
                        const uint32_t kh = P.ktiles / 2, part = kt >= kh ? 1u : 0u;
                        const int32_t k0 = (int32_t)((kt - part * kh) * KT);
                        if (P.a_mn) {
                            // MN-major A: planes 2 part (hi) and 2 part + 1 (lo), each four
                            // 32(m) x 32(k) blocks 2 KB apart, as one 4-D box
                            const uint32_t f = P.a_mn - 1;
                            tc::tma_load_4d(st, P.ta, 0, (int32_t)((4 * part + f) * P.a_rows) + k0, m0 / 32, 0,
                                            &full_bar[s]);
                        }
                        for (uint32_t p = 0; p < 2; ++p) {
                            const uint32_t pl = 2 * part + p;
                            if (!P.a_mn)
                                tc::tma_load_2d(st + p * TILE_BYTES, P.ta, k0, (int32_t)(pl * P.a_rows) + m0,
                                                &full_bar[s]);
                            tc::tma_load_2d(st + B_OFF + p * BPB, P.tb, k0, (int32_t)(pl * P.b_rows) + n0,
                                            &full_bar[s]);
                        }
                    } else {
                        const int32_t k0 = kt * KT;
                        for (uint32_t p = 0; p < A_PLANES; ++p)
                            tc::tma_load_2d(st + p * TILE_BYTES, P.ta, k0, (int32_t)(p * P.a_rows) + m0,
                                            &full_bar[s]);
                        if (B_COMPLEX) {
                            // B: hi block [r_hi | i_hi], lo block [r_lo | i_lo]
                            uint8_t *bb = st + B_OFF;
                            tc::tma_load_2d(bb, P.tb, k0, (int32_t)(0 * P.b_rows) + n0, &full_bar[s]);
                            tc::tma_load_2d(bb + BLO, P.tb, k0, (int32_t)(1 * P.b_rows) + n0, &full_bar[s]);
                            tc::tma_load_2d(bb + TILE_BYTES, P.tb, k0, (int32_t)(2 * P.b_rows) + n0, &full_bar[s]);
                            tc::tma_load_2d(bb + BLO + TILE_BYTES, P.tb, k0, (int32_t)(3 * P.b_rows) + n0,
                                            &full_bar[s]);
                        }
                    }
                    if (++s == NSTG) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            constexpr uint32_t I256 = tc::idesc_bf16(128, 256);
            uint32_t s = 0, ph = 0, acc = 0, acc_ph = 0, tl = 0;
            for (uint32_t t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x, ++tl) {
                const Problem P = probs[tiles[t].problem];
                // MN-major A only in R^-1 of Toeplitz groups; T's N is the group's y count
                const bool amn = STAGE == ST_RI && P.a_mn != 0;
                const uint32_t nmma = STAGE == ST_T ? groups[P.group].nTy : 128u;
                const uint32_t kpT = STAGE == ST_T ? groups[P.group].kpC : 0u;
                const uint32_t I128 = tc::idesc_bf16(128, nmma, false, amn);
                const uint32_t I128N = tc::idesc_bf16(128, 128, true, amn);
                const uint32_t wRI = STAGE == ST_RI ? groups[P.group].wRI : 256u;
                const uint32_t IRI = tc::idesc_bf16(128, wRI, false, amn), IRIN = tc::idesc_bf16(128, wRI, true, amn);
                const uint32_t IR = tc::idesc_bf16(128, STAGE == ST_R ? groups[P.group].wR : 128u);
                const uint32_t sb = tl & 1u;
                if (STAGE == ST_T && !tc::mbar_wait(&strip_full[sb], (tl >> 1) & 1u, err)) {
                    abort_flag = 1;
                    break;
                }
                if (!tc::mbar_wait(&acc_empty[acc], acc_ph ^ 1u, err)) {
                    abort_flag = 1;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d = tmem + acc * 256;
                for (uint32_t kt = 0; kt < P.ktiles; ++kt) {
                    if (!tc::mbar_wait(&full_bar[s], ph, err)) {
                        abort_flag = 1;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t st = tc::smem_u32(smem + s * SBYTES);
                    uint32_t bhi = st + B_OFF, blo = bhi + BLO;
                    if (STAGE == ST_T) {
                        // rows (K - 32 - 32 kt) .. of the strip
                        bhi = tc::smem_u32(strip + sb * 2 * T_STRIP_PLANE) + (kpT - KT - kt * KT) * KT * 2;
                        blo = bhi + T_STRIP_PLANE;
                    }
#pragma unroll
                    for (int j = 0; j < KT / 16; ++j) {
                        const uint32_t o = j * 32;  // 16 bf16 along K (K-major rows)
                        const uint32_t first = (kt == 0 && j == 0) ? 0u : 1u;
                        // A planes: K-major (+32 B per K step) or MN-major (+16 rows of 64 B)
                        auto ad = [&](uint32_t plane) {
                            const uint32_t a = st + plane * TILE_BYTES;
                            return amn ? tc::sdesc_mn64(a + j * 1024, 2048, 512) : tc::sdesc_k64(a + o);
                        };
                        const uint64_t arh = ad(0), arl = ad(1);
                        if (STAGE == ST_T) {
                            // D = A * B, real x real
                            tc::mma_bf16(d, arh, tc::sdesc_k64(bhi + o), I128, first);
                            tc::mma_bf16(d, arh, tc::sdesc_k64(blo + o), I128, 1);
                            tc::mma_bf16(d, arl, tc::sdesc_k64(bhi + o), I128, 1);
                        } else if (STAGE == ST_RI) {
                            // D += Ar * Br over the first half of K', D -= Ai * Bi over the second
                            const uint32_t id = kt < P.ktiles / 2 ? IRI : IRIN;
                            tc::mma_bf16(d, arh, tc::sdesc_k64(bhi + o), id, first);
                            tc::mma_bf16(d, arh, tc::sdesc_k64(blo + o), id, 1);
                            tc::mma_bf16(d, arl, tc::sdesc_k64(bhi + o), id, 1);
                        } else if (STAGE == ST_R) {
                            // Dr += Ar * Br, Di += Ar * Bi, each wR columns wide
                            tc::mma_bf16(d, arh, tc::sdesc_k64(bhi + o), IR, first);
                            tc::mma_bf16(d, arh, tc::sdesc_k64(blo + o), IR, 1);
                            tc::mma_bf16(d, arl, tc::sdesc_k64(bhi + o), IR, 1);
                            tc::mma_bf16(d + 128, arh, tc::sdesc_k64(bhi + TILE_BYTES + o), IR, first);
                            tc::mma_bf16(d + 128, arh, tc::sdesc_k64(blo + TILE_BYTES + o), IR, 1);
                            tc::mma_bf16(d + 128, arl, tc::sdesc_k64(bhi + TILE_BYTES + o), IR, 1);
                        } else {
                            // [Dr | Di] += Ar * [Br | Bi]
                            tc::mma_bf16(d, arh, tc::sdesc_k64(bhi + o), I256, first);
                            tc::mma_bf16(d, arh, tc::sdesc_k64(blo + o), I256, 1);
                            tc::mma_bf16(d, arl, tc::sdesc_k64(bhi + o), I256, 1);
                            if (A_COMPLEX) {
                                const uint64_t aih = ad(2), ail = ad(3);
                                // Dr -= Ai * Bi ; Di += Ai * Br
                                tc::mma_bf16(d, aih, tc::sdesc_k64(bhi + TILE_BYTES + o), I128N, 1);
                                tc::mma_bf16(d, aih, tc::sdesc_k64(blo + TILE_BYTES + o), I128N, 1);
                                tc::mma_bf16(d, ail, tc::sdesc_k64(bhi + TILE_BYTES + o), I128N, 1);
                                tc::mma_bf16(d + 128, aih, tc::sdesc_k64(bhi + o), I128, 1);
                                tc::mma_bf16(d + 128, aih, tc::sdesc_k64(blo + o), I128, 1);
                                tc::mma_bf16(d + 128, ail, tc::sdesc_k64(bhi + o), I128, 1);
                            }
                        }
                    }
                    tc::mma_commit(&empty_bar[s]);  // frees the stage when these MMAs finish
                    if (++s == NSTG) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (STAGE == ST_T) tc::mma_commit(&strip_empty[sb]);  // the strip is free once they finish
                tc::mma_commit(&acc_full[acc]);
                if (++acc == 2) {
                    acc = 0;
                    acc_ph ^= 1u;
                }
            }
        }
    } else {
        // ---------------- epilogue (warps 2..9) ----------------
        // Warp e reads TMEM lane quarter warp%4 (the only lanes it may
        // access) and the e/4-th half of the tile's columns, in 32-column
        // chunks; C and C^-1 columns are padded per instance to N1hp, so a
        // chunk never straddles an instance or field.
        const uint32_t ew = warp - 2, q = warp & 3, half = ew >> 2;
        float *xbuf = reinterpret_cast<float *>(smem + RING_BYTES) + ew * (32 * 33);
        uint32_t acc = 0, acc_ph = 0;
        for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const Tile T = tiles[t];
            const Problem P = probs[T.problem];
            const Group Gp = groups[P.group];
            if (!tc::mbar_wait(&acc_full[acc], acc_ph, err)) {
                abort_flag = 1;
                break;
            }
            tc::tc_fence_after();
            const uint32_t mrow0 = T.mt * MT + q * 32;  // first row of this warp
            const uint32_t m = mrow0 + lane;            // this thread's row
            const uint32_t d = tmem + acc * 256 + ((q * 32u) << 16);
            const uint32_t wN = STAGE == ST_R ? Gp.wR : STAGE == ST_RI ? Gp.wRI : NTS;
            for (uint32_t c0 = half * (NTS / 2); c0 < (half + 1) * (NTS / 2); c0 += 32) {
                if (c0 >= wN) continue;  // warp-uniform: past this tile's N width
                const uint32_t nb = T.nt * wN + c0, jmax = wN - c0;  // columns j < jmax belong to the tile
                const bool row_ok = m < P.M;
                if constexpr (STAGE == ST_C) {
                    // row m = ky ; col = (inst, kx) -> B operand of C^-1: row (inst, f, kx), k = ky.
                    // S_f = B * i Ks_f: real = -Bi Ks, imag = Br Ks. Each part is
                    // transposed through shared memory so each lane writes one
                    // destination row's 32 consecutive ky as 16-byte stores.
                    const uint32_t il = nb / Gp.N1hp, kx0 = nb - il * Gp.N1hp;
                    if (mrow0 >= P.M || il >= Gp.G) continue;  // warp-uniform
                    const size_t plane = (size_t)Gp.rowsCi * Gp.kpCi;
                    const uint32_t kx = kx0 + lane;  // after the transpose
                    // Each field's 32 spectrum values are loaded once (one round
                    // trip) and serve both parts.
#pragma unroll 1
                    for (int f = 0; f < 2; ++f) {
                        const float *ks = f ? Gp.kys : Gp.kxs;
                        float kv[32];
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            kv[j] = (row_ok && kx0 + j < Gp.N1h) ? __ldg(ks + (size_t)(kx0 + j) * Gp.N2 + m) : 0.0f;
#pragma unroll 1
                        for (int part = 0; part < 2; ++part) {
                            float v[32];
                            tc::tmem_ld32(d + (part ? 0u : 128u) + c0, v);  // part 0 needs Bi, part 1 Br
                            const float sgn = part ? 1.0f : -1.0f;
#pragma unroll
                            for (int j = 0; j < 32; ++j) xbuf[lane * 33 + j] = sgn * v[j] * kv[j];
                            __syncwarp();
                            if (kx < Gp.N1h) {
                                bf16 *o = Gp.bCi + (size_t)((il * 2 + f) * Gp.N1hp + kx) * Gp.kpCi + mrow0 +
                                          (size_t)(2 * part) * plane;
                                uint32_t hw[16], lw[16];
#pragma unroll
                                for (int i = 0; i < 16; ++i) {
                                    const float v0 = xbuf[(2 * i) * 33 + lane], v1 = xbuf[(2 * i + 1) * 33 + lane];
                                    const bf16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
                                    const bf16 l0 = __float2bfloat16_rn(v0 - __bfloat162float(h0));
                                    const bf16 l1 = __float2bfloat16_rn(v1 - __bfloat162float(h1));
                                    hw[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
                                    lw[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
                                }
                                uint4 *oh = reinterpret_cast<uint4 *>(o), *ol = reinterpret_cast<uint4 *>(o + plane);
#pragma unroll
                                for (int i = 0; i < 4; ++i) {
                                    oh[i] = make_uint4(hw[4 * i], hw[4 * i + 1], hw[4 * i + 2], hw[4 * i + 3]);
                                    ol[i] = make_uint4(lw[4 * i], lw[4 * i + 1], lw[4 * i + 2], lw[4 * i + 3]);
                                }
                            }
                            __syncwarp();
                        }
                    }
                    continue;
                }
                if constexpr (STAGE == ST_T) {
                    // row m = (inst, re/im) ; col = y -> R^-1's M-major A operand
                    // aRiT[plane][f][kx][m'], m' = ((y / 8) * G + inst) * 8 + y % 8:
                    // a lane's 8-y piece sits next to the next instance's, so the
                    // 16 lanes of one part write 256 contiguous bytes per store.
                    if (mrow0 >= 2 * Gp.G || nb >= Gp.Yp) continue;  // warp-uniform
                    float v[32];
                    tc::tmem_ld32(d + c0, v);
                    if (m >= 2 * Gp.G) continue;
                    const uint32_t f = T.sub / Gp.N1h, kx = T.sub - f * Gp.N1h;
                    const uint32_t inst = m >> 1, ri = m & 1u;
                    // Tx = -i tx: C_x = -i P (Re = P_i, Im = -P_r); Ty is real: C_y = Q
                    const uint32_t part = f ? ri : (ri ^ 1u);  // 0: Re C, 1: Im C
                    const float sgn = (f == 0 && ri == 0) ? -1.0f : 1.0f;
                    const size_t pst = (size_t)2 * Gp.kpRi * Gp.MpT;  // plane stride
                    bf16 *o = Gp.aRiT + (size_t)((4 * part + f) * Gp.kpRi + kx) * Gp.MpT;
                    uint32_t hw[16], lw[16];
                    split_pack32(v, sgn, hw, lw);
                    // Yp is a multiple of 8: an 8-element piece is wholly inside or past the instance
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint32_t yb = (nb >> 3) + k;
                        if (8 * yb < Gp.Yp) {
                            const size_t e = ((size_t)yb * Gp.G + inst) * 8;
                            *reinterpret_cast<uint4 *>(o + e) = make_uint4(hw[4 * k], hw[4 * k + 1], hw[4 * k + 2], hw[4 * k + 3]);
                            *reinterpret_cast<uint4 *>(o + pst + e) =
                                make_uint4(lw[4 * k], lw[4 * k + 1], lw[4 * k + 2], lw[4 * k + 3]);
                        }
                    }
                    continue;
                }
                float vr[32], vi[32];
                tc::tmem_ld32(d + c0, vr);
                if (OUT_COMPLEX) tc::tmem_ld32(d + 128 + c0, vi);
                if (mrow0 >= P.M) continue;  // warp-uniform
                if (STAGE == ST_R) {
                    if (!row_ok) continue;
                    const uint32_t il = m / Gp.Y, y = m - il * Gp.Y;
                    if (Gp.toe) {
                        // row m = (inst, y) ; col = kx -> A operand of T: row (kx, inst, re/im), k = y
                        const size_t plane = (size_t)Gp.rowsT * Gp.kpC, step = (size_t)2 * Gp.G * Gp.kpC;
                        bf16 *o = Gp.bT + (size_t)(nb * 2 * Gp.G + il * 2) * Gp.kpC + y;
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            if (nb + j < Gp.N1h && (uint32_t)j < jmax) {
                                split_store(o, o + plane, vr[j]);
                                split_store(o + Gp.kpC, o + Gp.kpC + plane, vi[j]);
                            }
                            o += step;
                        }
                        continue;
                    }
                    // row m = (inst, y) ; col = kx -> B operand of C: row (inst, kx), k = y
                    const size_t plane = (size_t)Gp.rowsC * Gp.kpC;
                    bf16 *o = Gp.bC + (size_t)(il * Gp.N1hp + nb) * Gp.kpC + y;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        if (nb + j < Gp.N1h && (uint32_t)j < jmax) {
                            split_store(o, o + plane, vr[j]);
                            split_store(o + 2 * plane, o + 3 * plane, vi[j]);
                        }
                        o += Gp.kpC;
                    }
                } else if (STAGE == ST_CI) {
                    // row m = y ; col = (inst, f, kx) -> A operand of R^-1: row (inst, f, y), k = kx.
                    // Each lane writes its own row's 32 consecutive kx as 16-byte stores.
                    const uint32_t il = nb / (2 * Gp.N1hp), rem = nb - il * 2 * Gp.N1hp;
                    if (il >= Gp.G || !row_ok) continue;
                    const uint32_t f = rem >= Gp.N1hp ? 1u : 0u, kx0 = rem - f * Gp.N1hp;
                    const size_t plane = (size_t)Gp.rowsRi * Gp.kpRi;
                    bf16 *o = Gp.aRi + (size_t)((il * 2 + f) * Gp.Y + m) * Gp.kpRi + kx0;
#pragma unroll
                    for (int part = 0; part < 2; ++part) {
                        uint32_t hw[16], lw[16];
                        split_pack32(part ? vi : vr, 1.0f, hw, lw);
                        uint4 *oh = reinterpret_cast<uint4 *>(o + (size_t)(2 * part) * plane);
                        uint4 *ol = reinterpret_cast<uint4 *>(o + (size_t)(2 * part + 1) * plane);
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            oh[i] = make_uint4(hw[4 * i], hw[4 * i + 1], hw[4 * i + 2], hw[4 * i + 3]);
                            ol[i] = make_uint4(lw[4 * i], lw[4 * i + 1], lw[4 * i + 2], lw[4 * i + 3]);
                        }
                    }
                } else {
                    // row m = (inst, f, y), or (inst, y) of field a_mn - 1 ; col = x
                    // -> g_f[y * pitch + x], masked
                    if (!row_ok) continue;
                    uint32_t il, f, y;
                    if (P.a_mn) {
                        // aRiT rows are m = ((y / 8) * G + inst) * 8 + y % 8
                        const uint32_t t8 = m >> 3, yb = t8 / Gp.G;
                        il = t8 - yb * Gp.G;
                        y = yb * 8 + (m & 7u);
                        f = P.a_mn - 1;
                        if (y >= Gp.Y) continue;
                    } else {
                        il = m / (2 * Gp.Y);
                        const uint32_t r2 = m - il * 2 * Gp.Y;
                        f = r2 >= Gp.Y ? 1u : 0u;
                        y = r2 - f * Gp.Y;
                    }
                    const uint32_t inst = Gp.inst0 + il;
                    const InstIO io = (io0_active && inst == 0) ? io0 : ios[inst];
                    float *out = (f ? io.gy : io.gx) + (size_t)y * io.pitch;
                    const uint32_t *mask = io.mask + (size_t)y * io.pitch;
                    if (nb + 32 <= Gp.X && jmax >= 32u &&
                        ((reinterpret_cast<uintptr_t>(out + nb) | reinterpret_cast<uintptr_t>(mask + nb)) & 15u) == 0u) {
                        // whole chunk, 16-byte aligned
                        const uint4 *mk = reinterpret_cast<const uint4 *>(mask + nb);
                        float4 *o4 = reinterpret_cast<float4 *>(out + nb);
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const uint4 mm = __ldg(mk + i);
                            o4[i] = make_float4(mm.x ? vr[4 * i] : 0.0f, mm.y ? vr[4 * i + 1] : 0.0f,
                                                mm.z ? vr[4 * i + 2] : 0.0f, mm.w ? vr[4 * i + 3] : 0.0f);
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const uint32_t x = nb + j;
                            if (x < Gp.X && (uint32_t)j < jmax) out[x] = __ldg(mask + x) != 0u ? vr[j] : 0.0f;
                        }
                    }
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&acc_empty[acc]);
            if (++acc == 2) {
                acc = 0;
                acc_ph ^= 1u;
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

// ---- per-solve input preparation: mass rows -> A operand of stage R --------
struct PrepRef {
    uint32_t group, row;  // row = inst_local * Y + y
};

__global__ void prep_mass(const Group *__restrict__ groups, const PrepRef *__restrict__ refs,
                          const InstIO *__restrict__ ios, InstIO io0, int io0_active) {
    const PrepRef r = refs[blockIdx.x];
    const Group Gp = groups[r.group];
    const uint32_t il = r.row / Gp.Y, y = r.row - il * Gp.Y, inst = Gp.inst0 + il;
    const InstIO io = (io0_active && inst == 0) ? io0 : ios[inst];
    const size_t plane = (size_t)Gp.rowsR * Gp.kpR;
    bf16 *o = Gp.aR + (size_t)r.row * Gp.kpR;
    const size_t c0 = (size_t)y * io.pitch;
    const void *src = io.mass_f ? (const void *)(io.mass_f + c0) : (const void *)(io.mass_i + c0);
    // 8 cells per thread with 16-byte accesses when the rows allow it (pitch a
    // multiple of 8, so the chunk that holds x = X-1 ends inside the row);
    // the aR row is 64-byte aligned and padded to a multiple of 32.
    const bool vec = (io.pitch & 7u) == 0u &&
                     ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(io.mask + c0)) & 15u) == 0u;
    for (uint32_t x0 = threadIdx.x * 8; x0 < Gp.X; x0 += blockDim.x * 8) {
        float v[8];
        if (vec) {
            const uint4 *mk = reinterpret_cast<const uint4 *>(io.mask + c0 + x0);
            const uint4 m0 = __ldg(mk), m1 = __ldg(mk + 1);
            const uint32_t mm[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
            float a[8];
            if (io.mass_f) {
                const float4 *p = reinterpret_cast<const float4 *>(io.mass_f + c0 + x0);
                const float4 q0 = __ldg(p), q1 = __ldg(p + 1);
                a[0] = q0.x, a[1] = q0.y, a[2] = q0.z, a[3] = q0.w, a[4] = q1.x, a[5] = q1.y, a[6] = q1.z, a[7] = q1.w;
            } else {
                const int4 *p = reinterpret_cast<const int4 *>(io.mass_i + c0 + x0);
                const int4 q0 = __ldg(p), q1 = __ldg(p + 1);
                const int32_t qi[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                for (int j = 0; j < 8; ++j) a[j] = (float)qi[j] * io.inv;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = (x0 + j < Gp.X && mm[j] != 0u) ? a[j] : 0.0f;
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const size_t c = c0 + x0 + j;
                v[j] = 0.0f;
                if (x0 + j < Gp.X && __ldg(io.mask + c) != 0u)
                    v[j] = io.mass_f ? __ldg(io.mass_f + c) : (float)__ldg(io.mass_i + c) * io.inv;
            }
        }
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const bf16 h0 = __float2bfloat16_rn(v[2 * i]), h1 = __float2bfloat16_rn(v[2 * i + 1]);
            const bf16 l0 = __float2bfloat16_rn(v[2 * i] - __bfloat162float(h0));
            const bf16 l1 = __float2bfloat16_rn(v[2 * i + 1] - __bfloat162float(h1));
            hw[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
            lw[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
        }
        *reinterpret_cast<uint4 *>(o + x0) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4 *>(o + plane + x0) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
}

// ---- FP64 precompute ---------------------------------------------------------
__device__ __forceinline__ void split_store_d(bf16 *hi, bf16 *lo, double v) {
    bf16 h = __double2bfloat16(v);
    *hi = h;
    *lo = __double2bfloat16(v - (double)__bfloat162float(h));
}

// Complex DFT matrix into 4 planes: rows r < rows, k < kvalid,
// value = w(k) * exp(sign * 2 pi i * (r * k mod n) / n). `weights` = 1 gives
// the Hermitian weights w = 1 (k == 0 or 2k == n) else 2 (on k).
__global__ void dft_matrix(bf16 *out, uint32_t rows, uint32_t kvalid, uint32_t kpitch, uint32_t n, int sign,
                           int weights) {
    size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (size_t)rows * kvalid) return;
    uint32_t r = (uint32_t)(id / kvalid), k = (uint32_t)(id - (size_t)r * kvalid);
    uint64_t t = ((uint64_t)r * k) % n;
    double s, c;
    sincospi(2.0 * (double)t / (double)n, &s, &c);
    double w = 1.0;
    if (weights) w = (k == 0 || 2 * k == n) ? 1.0 : 2.0;
    const size_t plane = (size_t)rows * kpitch, e = (size_t)r * kpitch + k;
    split_store_d(out + e, out + plane + e, w * c);
    split_store_d(out + 2 * plane + e, out + 3 * plane + e, w * (double)sign * s);
}

// Imaginary parts of the x/y kernel spectra, first over x:
// tx[j][kx] = sum_dx Kx(dx, dy_j) sin(2 pi kx dx / N1), ty = sum_dx Ky cos(..),
// with K(d) = scale * d / |d|^3, d folded into (-N/2, N/2) (the +N/2 offset
// is never used by the linear convolution and is left out, which makes Kx
// exactly odd in x and Ky exactly odd in y).
__global__ void spectra_x(double *tx, double *ty, uint32_t N1, uint32_t N2, uint32_t N1h, double scale) {
    size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (size_t)N2 * N1h) return;
    uint32_t j = (uint32_t)(id / N1h), kx = (uint32_t)(id - (size_t)j * N1h);
    if (2 * j == N2) {
        tx[id] = 0.0;
        ty[id] = 0.0;
        return;
    }
    double dy = 2 * j < N2 ? (double)j : (double)j - (double)N2;
    double sx = 0.0, sy = 0.0;
    for (uint32_t dxi = 0; dxi < N1; ++dxi) {
        if (2 * dxi == N1) continue;
        double dx = 2 * dxi < N1 ? (double)dxi : (double)dxi - (double)N1;
        if (dx == 0.0 && dy == 0.0) continue;
        double r2 = dx * dx + dy * dy, d = sqrt(r2);
        double inv = scale / (r2 * d);
        uint64_t t = ((uint64_t)kx * dxi) % N1;
        double s, c;
        sincospi(2.0 * (double)t / (double)N1, &s, &c);
        sx += dx * inv * s;
        sy += dy * inv * c;
    }
    tx[id] = sx;
    ty[id] = sy;
}

// then over y: kxs = -sum_j tx[j] cos(2 pi ky j / N2), kys = -sum_j ty[j] sin(..)
__global__ void spectra_y(const double *tx, const double *ty, float *kxs, float *kys, uint32_t N2, uint32_t N1h) {
    size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (size_t)N2 * N1h) return;
    uint32_t ky = (uint32_t)(id / N1h), kx = (uint32_t)(id - (size_t)ky * N1h);
    double ax = 0.0, ay = 0.0;
    for (uint32_t j = 0; j < N2; ++j) {
        uint64_t t = ((uint64_t)ky * j) % N2;
        double s, c;
        sincospi(2.0 * (double)t / (double)N2, &s, &c);
        ax += tx[(size_t)j * N1h + kx] * c;
        ay += ty[(size_t)j * N1h + kx] * s;
    }
    kxs[(size_t)kx * N2 + ky] = (float)(-ax);
    kys[(size_t)kx * N2 + ky] = (float)(-ay);
}

// Toeplitz strips of the y stage, into 2 planes: row (f * N1h + kx) * SR + r,
// column c < 32 holds t_f[(r - (kp - 32) - c) mod N2][kx], with t_x = tx and
// t_y = ty from spectra_x with the 1/N1 scale only. Rows r .. r + N of a
// strip are the Toeplitz matrix T[y][y'] = t_f[(y - y') mod N2] for
// y' in [kp - 32 - r, kp - r); the -i of Tx is applied in T's epilogue.
__global__ void toeplitz_strip(const double *tx, const double *ty, bf16 *out, uint32_t SR, uint32_t N2,
                               uint32_t N1h, uint32_t kp) {
    const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (size_t)2 * N1h * SR * KT) return;
    const uint32_t c = (uint32_t)(id % KT);
    const size_t row = id / KT;  // (f * N1h + kx) * SR + r
    const uint32_t r = (uint32_t)(row % SR), sub = (uint32_t)(row / SR), f = sub / N1h, kx = sub - f * N1h;
    const int64_t d = (int64_t)r - (int64_t)(kp - KT) - (int64_t)c;
    const uint32_t j = (uint32_t)(((d % (int64_t)N2) + (int64_t)N2) % (int64_t)N2);
    const double v = (f ? ty : tx)[(size_t)j * N1h + kx];
    const size_t plane = (size_t)2 * N1h * SR * KT;
    split_store_d(out + id, out + plane + id, v);
}

// ---- host ---------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

static uint32_t round_up(uint32_t v, uint32_t m) { return (v + m - 1) / m * m; }

struct HostGroup {
    Group g;
    bf16 *f1 = nullptr, *f2 = nullptr, *g2 = nullptr, *g1 = nullptr, *ts = nullptr;
    uint32_t kpF1 = 0, kpF2 = 0, kpG2 = 0, kpG1 = 0;
    float *kxs = nullptr;
    double flops = 0;  // executed tensor flops of one solve of the group
};

constexpr int NSTAGES = 5;  // R, C, C^-1, R^-1, T (indexed by Stage)

struct DftImpl {
    std::vector<JobShape> shapes;
    std::vector<HostGroup> hg;
    std::vector<void *> allocs;
    Group *groups = nullptr;
    InstIO *ios = nullptr;
    std::vector<InstIO> ios_host;
    std::vector<uint32_t> inst_group, inst_local;
    CUtensorMap *tmaps = nullptr;
    Problem *probs = nullptr;
    Tile *tiles[NSTAGES] = {};
    uint32_t ntiles[NSTAGES] = {};
    PrepRef *prep = nullptr;
    uint32_t nprep = 0;
    uint32_t grid[NSTAGES] = {};
    // The same tiles split by the form of the group's y stage: branch 0 the
    // Toeplitz groups (R, T, R^-1), branch 1 the DFT-pair groups (R, C,
    // C^-1, R^-1). With side_ctas > 0 and both branches non-empty, branch 1
    // runs on `side` with side_ctas CTAs per launch, concurrently with branch
    // 0 on the caller's stream with the remaining SMs.
    Tile *btiles[2][NSTAGES] = {};
    uint32_t bntiles[2][NSTAGES] = {};
    bool split_ok = false;
    uint32_t side_ctas = 0;
    uint32_t sms = 148;
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    double flops = 0;
    uint32_t *err = nullptr;  // device address of g_dft_err
    ~DftImpl() {
        for (void *p : allocs) cudaFree(p);
        if (side) cudaStreamDestroy(side);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
    template <typename T> int alloc(T **p, size_t n) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "split-BF16 gravity: allocation failed");
        e = cudaMemset(q, 0, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) TPT_FAIL(TPT_ERR_CUDA, "cudaMemset failed: %s", cudaGetErrorString(e));
        allocs.push_back(q);
        *p = static_cast<T *>(q);
        return TPT_OK;
    }
};

// Row-major bf16 matrix of `rows_total` rows of `kpitch` elements; boxes of
// 32 elements (64 bytes) x box_rows rows.
// R^-1's MN-major A operand of a Toeplitz group (aRiT: rows (plane, f, kx)
// of MpT m' each) as one box per K tile: both planes of one part (hi, lo:
// 2 * kpRi rows apart), four blocks of 32 m' (64 bytes apart in memory),
// 32 kx rows -- in shared memory [plane][m block][kx][32 m'], i.e. the four
// 32 x 32 boxes per plane 2 KB apart that the MN-major descriptor reads.
// Dims (m' in block, row, m block, plane); rows cover the bases (4 part + f)
// kpRi + k0 the loads use.
static int make_tmap_mn4(CUtensorMap *out, const bf16 *base, uint32_t MpT, uint32_t kpRi) {
    auto fn = encode_fn();
    if (!fn) TPT_FAIL(TPT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t dims[4] = {32, (cuuint64_t)6 * kpRi, MpT / 32, 2};
    cuuint64_t strides[3] = {(cuuint64_t)MpT * 2, 64, (cuuint64_t)2 * kpRi * MpT * 2};
    cuuint32_t box[4] = {32, KT, 4, 2};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) TPT_FAIL(TPT_ERR_CUDA, "cuTensorMapEncodeTiled (4-D MN-major operand) failed (%d)", (int)r);
    return TPT_OK;
}

static int make_tmap(CUtensorMap *out, const bf16 *base, uint32_t kpitch, uint32_t rows_total,
                     uint32_t box_rows = MT) {
    auto fn = encode_fn();
    if (!fn) TPT_FAIL(TPT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t dims[2] = {kpitch, rows_total};
    cuuint64_t strides[1] = {(cuuint64_t)kpitch * 2};
    cuuint32_t box[2] = {KT, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) TPT_FAIL(TPT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TPT_OK;
}

static int init_attrs() {
    static bool done = false;
    if (done) return TPT_OK;
    TPT_CUDA(cudaFuncSetAttribute(dft_gemm<ST_R>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_R_BYTES));
    TPT_CUDA(cudaFuncSetAttribute(dft_gemm<ST_C>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    TPT_CUDA(cudaFuncSetAttribute(dft_gemm<ST_CI>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    TPT_CUDA(cudaFuncSetAttribute(dft_gemm<ST_RI>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_R_BYTES));
    TPT_CUDA(cudaFuncSetAttribute(dft_gemm<ST_T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    done = true;
    return TPT_OK;
}

// Smallest group that takes the Toeplitz y stage by default.
constexpr uint32_t kToeMinGroup = 8;
enum YMode { YMODE_AUTO = 0, YMODE_DFT = 1, YMODE_TOEPLITZ = 2 };

// TPT_SPLIT_BF16_Y_STAGE = dft | toeplitz | toeplitz:<n> forces the y form
// (toeplitz:<n>: Toeplitz for groups of at least n instances, DFT for the
// rest), for comparisons; unset or anything else lets the cost model choose.
static YMode y_mode_from_env(uint32_t *min_group) {
    *min_group = 1;
    const char *s = getenv("TPT_SPLIT_BF16_Y_STAGE");
    if (!s) return YMODE_AUTO;
    if (!strcmp(s, "dft")) return YMODE_DFT;
    if (!strcmp(s, "toeplitz")) return YMODE_TOEPLITZ;
    if (!strncmp(s, "toeplitz:", 9)) {
        const long n = strtol(s + 9, nullptr, 10);
        *min_group = n > 1 ? (uint32_t)n : 1u;
        return YMODE_TOEPLITZ;
    }
    return YMODE_AUTO;
}

int DftSet::create(const std::vector<JobShape> &shapes) {
    destroy();
    int rc = init_attrs();
    if (rc) return rc;
    uint32_t toe_min_group = 1;
    const YMode ymode = y_mode_from_env(&toe_min_group);
    if (!encode_fn()) TPT_FAIL(TPT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available from the driver");
    DftImpl *I = new (std::nothrow) DftImpl();
    if (!I) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    impl = I;
    I->shapes = shapes;
    TPT_CUDA(cudaGetSymbolAddress((void **)&I->err, g_dft_err));
    const uint32_t n = (uint32_t)shapes.size();
    // group instances by shape, keeping first-seen order
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> gid;
    std::vector<std::vector<uint32_t>> members;
    for (uint32_t i = 0; i < n; ++i) {
        auto key = std::make_pair(shapes[i].X, shapes[i].Y);
        auto it = gid.find(key);
        if (it == gid.end()) {
            gid[key] = (uint32_t)members.size();
            members.push_back({});
            it = gid.find(key);
        }
        members[it->second].push_back(i);
    }
    // instance order = grouped order; instance IO table is indexed by the
    // position in that order (inst0 + local)
    std::vector<uint32_t> order;
    for (auto &mv : members) order.insert(order.end(), mv.begin(), mv.end());
    I->inst_group.resize(n);
    I->inst_local.resize(n);
    I->hg.resize(members.size());
    uint32_t inst0 = 0;
    for (size_t gi = 0; gi < members.size(); ++gi) {
        HostGroup &H = I->hg[gi];
        Group &g = H.g;
        g.X = shapes[members[gi][0]].X;
        g.Y = shapes[members[gi][0]].Y;
        g.N1 = 2 * g.X;
        g.N2 = 2 * g.Y;
        g.N1h = g.N1 / 2 + 1;
        g.N1hp = round_up(g.N1h, 32);
        g.G = (uint32_t)members[gi].size();
        g.inst0 = inst0;
        for (uint32_t l = 0; l < g.G; ++l) {
            I->inst_group[members[gi][l]] = (uint32_t)gi;
            I->inst_local[members[gi][l]] = inst0 + l;
        }
        inst0 += g.G;
        g.kpR = round_up(g.X, KT);
        g.kpC = round_up(g.Y, KT);
        g.kpCi = round_up(g.N2, KT);
        g.kpRi = round_up(g.N1h, KT);
        g.rowsR = g.G * g.Y;
        g.rowsC = g.G * g.N1hp;
        g.rowsCi = 2 * g.G * g.N1hp;
        g.rowsRi = 2 * g.G * g.Y;
        g.rowsT = g.N1h * 2 * g.G;
        g.nTy = std::min<uint32_t>(T_NMAX, round_up(g.Y, 16));
        g.Yp = round_up(g.Y, 8);
        g.MpT = round_up(g.G * g.Yp, 32);
        g.SR = g.nTy + g.kpC - KT;                               // strip rows
        // R / R^-1 N tiles: the fewest tiles of at most 128 complex / 256 real
        // columns, each a multiple of 16 wide (X = 400: 2 x 208 rather than 2 x 256)
        const uint32_t ntR = (g.N1h + NT - 1) / NT, ntRI = (g.X + 2 * NT - 1) / (2 * NT);
        g.wR = round_up((g.N1h + ntR - 1) / ntR, 16);
        g.wRI = round_up((g.X + ntRI - 1) / ntRI, 16);
        g.snb = (g.SR + T_NMAX - 1) / T_NMAX;                    // TMA boxes per strip (box rows <= 256)
        g.sbox = round_up((g.SR + g.snb - 1) / g.snb, 8);        // box rows, 512-byte multiples
        H.kpF1 = g.kpR;   // F1: N1h rows, K = x
        H.kpF2 = g.kpC;   // F2: N2 rows, K = y
        H.kpG2 = g.kpCi;  // G2: Y rows, K = ky
        H.kpG1 = g.kpRi;  // G1: X rows, K = kx
        // executed tensor flops (3-term split, padded tiles) of both y forms
        auto tiles_of = [](uint32_t v, uint32_t t) { return (double)((v + t - 1) / t) * t; };
        const double fR = 2.0 * tiles_of(g.rowsR, MT) * tiles_of(g.N1h, g.wR) * 2 * g.kpR * 3;
        const double fC = 2.0 * tiles_of(g.N2, MT) * tiles_of(g.rowsC, NT) * 4 * g.kpC * 3;
        const double fCi = 2.0 * tiles_of(g.Y, MT) * tiles_of(g.rowsCi, NT) * 4 * g.kpCi * 3;
        const double fRi = 2.0 * tiles_of(g.rowsRi, MT) * tiles_of(g.X, g.wRI) * 2 * g.kpRi * 3;
        const double fT = 2.0 * 2 * g.N1h * tiles_of(2 * g.G, MT) * g.nTy * g.kpC * 3;
        const double fRiT = 2.0 * 2 * tiles_of(g.G * g.Yp, MT) * tiles_of(g.X, g.wRI) * 2 * g.kpRi * 3;
        // Form of the y stage: Toeplitz when the group has at least
        // kToeMinGroup instances (below that, T's M tile of 2G instance rows
        // is mostly padding, and a lone instance's y DFT pair is cheaper:
        // measured on B200 with single-instance groups of 32..512 cells), Y
        // fits one T tile, and T executes fewer tensor flops than the y DFT pair.
        const bool toe_ok = g.Y <= (uint32_t)T_NMAX;
        const bool toe_cheaper = g.G >= kToeMinGroup && fT + fRiT < fC + fCi + fRi;
        g.toe = !toe_ok                   ? 0u
                : ymode == YMODE_TOEPLITZ ? (g.G >= toe_min_group ? 1u : 0u)
                : ymode == YMODE_DFT      ? 0u
                                          : (toe_cheaper ? 1u : 0u);
        if ((rc = I->alloc(&g.aR, (size_t)2 * g.rowsR * g.kpR))) return rc;
        if ((rc = I->alloc(&H.f1, (size_t)4 * g.N1h * H.kpF1))) return rc;
        if ((rc = I->alloc(&H.g1, (size_t)4 * g.X * H.kpG1))) return rc;
        if (g.toe) {
            if ((rc = I->alloc(&g.bT, (size_t)2 * g.rowsT * g.kpC))) return rc;
            if ((rc = I->alloc(&H.ts, (size_t)2 * 2 * g.N1h * g.SR * KT))) return rc;
            if ((rc = I->alloc(&g.aRiT, (size_t)4 * 2 * g.kpRi * g.MpT))) return rc;
        } else {
            if ((rc = I->alloc(&g.bC, (size_t)4 * g.rowsC * g.kpC))) return rc;
            if ((rc = I->alloc(&g.bCi, (size_t)4 * g.rowsCi * g.kpCi))) return rc;
            if ((rc = I->alloc(&g.aRi, (size_t)4 * g.rowsRi * g.kpRi))) return rc;
            if ((rc = I->alloc(&H.f2, (size_t)4 * g.N2 * H.kpF2))) return rc;
            if ((rc = I->alloc(&H.g2, (size_t)4 * g.Y * H.kpG2))) return rc;
            if ((rc = I->alloc(&H.kxs, (size_t)2 * g.N2 * g.N1h))) return rc;
            g.kxs = H.kxs;
            g.kys = H.kxs + (size_t)g.N2 * g.N1h;
        }
        // constants in FP64, rounded once to the hi/lo planes
        auto blocks = [](size_t cnt) { return (unsigned)((cnt + 255) / 256); };
        dft_matrix<<<blocks((size_t)g.N1h * g.X), 256>>>(H.f1, g.N1h, g.X, H.kpF1, g.N1, -1, 0);
        dft_matrix<<<blocks((size_t)g.X * g.N1h), 256>>>(H.g1, g.X, g.N1h, H.kpG1, g.N1, +1, 1);
        count_launch();
        count_launch();
        double *tx = nullptr;
        TPT_CUDA(cudaMalloc(&tx, (size_t)2 * g.N2 * g.N1h * sizeof(double)));
        double *ty = tx + (size_t)g.N2 * g.N1h;
        if (g.toe) {
            // y handled directly: only the x transform's 1/N1
            const double scale = -(double)6.673e-1f / (double)g.N1;
            spectra_x<<<blocks((size_t)g.N2 * g.N1h), 256>>>(tx, ty, g.N1, g.N2, g.N1h, scale);
            toeplitz_strip<<<blocks((size_t)2 * g.N1h * g.SR * KT), 256>>>(tx, ty, H.ts, g.SR, g.N2, g.N1h, g.kpC);
        } else {
            dft_matrix<<<blocks((size_t)g.N2 * g.Y), 256>>>(H.f2, g.N2, g.Y, H.kpF2, g.N2, -1, 0);
            dft_matrix<<<blocks((size_t)g.Y * g.N2), 256>>>(H.g2, g.Y, g.N2, H.kpG2, g.N2, +1, 0);
            count_launch();
            count_launch();
            const double scale = -(double)6.673e-1f / ((double)g.N1 * (double)g.N2);
            spectra_x<<<blocks((size_t)g.N2 * g.N1h), 256>>>(tx, ty, g.N1, g.N2, g.N1h, scale);
            spectra_y<<<blocks((size_t)g.N2 * g.N1h), 256>>>(tx, ty, H.kxs, H.kxs + (size_t)g.N2 * g.N1h, g.N2,
                                                             g.N1h);
        }
        count_launch();
        count_launch();
        cudaError_t e = cudaDeviceSynchronize();
        cudaFree(tx);
        if (e != cudaSuccess) TPT_FAIL(TPT_ERR_CUDA, "split-BF16 precompute failed: %s", cudaGetErrorString(e));
        H.flops = g.toe ? fR + fT + fRiT : fR + fC + fCi + fRi;
        I->flops += H.flops;
    }
    // device tables: groups, tensor maps, problems, tiles
    const size_t ng = I->hg.size();
    if ((rc = I->alloc(&I->groups, ng))) return rc;
    std::vector<Group> gh(ng);
    for (size_t gi = 0; gi < ng; ++gi) gh[gi] = I->hg[gi].g;
    TPT_CUDA(cudaMemcpy(I->groups, gh.data(), ng * sizeof(Group), cudaMemcpyHostToDevice));
    // Tensor map slots per group: 0 aR, 1 F1, 2 F2 | strips, 3 bC | bT, 4 G2,
    // 5 bCi, 6 aRi | aRiT, 7 G1.
    std::vector<CUtensorMap> tm(8 * ng);
    std::vector<Problem> pr;
    if ((rc = I->alloc(&I->tmaps, tm.size()))) return rc;
    std::vector<Tile> tl[NSTAGES];
    std::vector<Tile> btl[2][NSTAGES];  // per y-stage form: 0 Toeplitz, 1 DFT pair
    std::vector<PrepRef> pref;
    // Consecutive CTAs share the data operand's tile (L2 reuse): in C and
    // C^-1 the data is B (M tiles fastest), in R and R^-1 it is A (N tiles
    // fastest); the other operand is a small constant matrix.
    auto add_tiles = [&](int st, uint32_t prob, bool m_fastest) {
        const Problem &P = pr[prob];
        const Group &gq = I->hg[P.group].g;
        const uint32_t nts = st == ST_R ? gq.wR : st == ST_RI ? gq.wRI : NT;
        std::vector<Tile> &bl = btl[gq.toe ? 0 : 1][st];
        auto push = [&](uint32_t mt, uint32_t nt) {
            tl[st].push_back({prob, (uint16_t)mt, (uint16_t)nt, 0});
            bl.push_back({prob, (uint16_t)mt, (uint16_t)nt, 0});
        };
        if (m_fastest) {
            for (uint32_t nt = 0; nt * nts < P.N; ++nt)
                for (uint32_t mt = 0; mt * MT < P.M; ++mt) push(mt, nt);
        } else {
            for (uint32_t mt = 0; mt * MT < P.M; ++mt)
                for (uint32_t nt = 0; nt * nts < P.N; ++nt) push(mt, nt);
        }
    };
    for (size_t gi = 0; gi < ng; ++gi) {
        const HostGroup &H = I->hg[gi];
        const Group &g = H.g;
        CUtensorMap *tmd = I->tmaps + 8 * gi;
        CUtensorMap *tmh = tm.data() + 8 * gi;
        const uint32_t gi32 = (uint32_t)gi;
        // stage R: A = aR (2 planes), B = F1
        if ((rc = make_tmap(&tmh[0], g.aR, g.kpR, 2 * g.rowsR))) return rc;
        if ((rc = make_tmap(&tmh[1], H.f1, H.kpF1, 4 * g.N1h, g.wR))) return rc;
        if ((rc = make_tmap(&tmh[7], H.g1, H.kpG1, 4 * g.X, g.wRI))) return rc;
        pr.push_back({tmd + 0, tmd + 1, gi32, g.rowsR, g.N1h, g.kpR / KT, g.rowsR, g.N1h, 0});
        add_tiles(ST_R, (uint32_t)pr.size() - 1, false);
        if (g.toe) {
            // T: A = bT (rows (kx, inst, re/im)), B = the (f, kx) strips (sbox-row boxes)
            if ((rc = make_tmap(&tmh[2], H.ts, KT, 2 * 2 * g.N1h * g.SR, g.sbox))) return rc;
            if ((rc = make_tmap(&tmh[3], g.bT, g.kpC, 2 * g.rowsT))) return rc;
            // R^-1: A = aRiT read M-major, both planes of a K tile in one 4-D box
            if ((rc = make_tmap_mn4(&tmh[6], g.aRiT, g.MpT, g.kpRi))) return rc;
            const uint32_t pt = (uint32_t)pr.size();
            pr.push_back({tmd + 3, tmd + 2, gi32, 2 * g.G, g.Y, g.kpC / KT, g.rowsT, 0, 0});
            // kx slowest, so the tiles of one kx (both fields, all M tiles)
            // share the A slice while it is in L2
            for (uint32_t kx = 0; kx < g.N1h; ++kx)
                for (uint32_t f = 0; f < 2; ++f)
                    for (uint32_t mt = 0; mt * MT < 2 * g.G; ++mt) {
                        tl[ST_T].push_back({pt, (uint16_t)mt, 0, f * g.N1h + kx});
                        btl[0][ST_T].push_back({pt, (uint16_t)mt, 0, f * g.N1h + kx});
                    }
            for (uint32_t f = 0; f < 2; ++f) {
                pr.push_back({tmd + 6, tmd + 7, gi32, g.G * g.Yp, g.X, 2 * g.kpRi / KT, g.kpRi, g.X, f + 1});
                add_tiles(ST_RI, (uint32_t)pr.size() - 1, false);
            }
        } else {
            // stage C: A = F2, B = bC
            if ((rc = make_tmap(&tmh[2], H.f2, H.kpF2, 4 * g.N2))) return rc;
            if ((rc = make_tmap(&tmh[3], g.bC, g.kpC, 4 * g.rowsC))) return rc;
            // stage C^-1: A = G2, B = bCi
            if ((rc = make_tmap(&tmh[4], H.g2, H.kpG2, 4 * g.Y))) return rc;
            if ((rc = make_tmap(&tmh[5], g.bCi, g.kpCi, 4 * g.rowsCi))) return rc;
            // stage R^-1: A = aRi, B = G1
            if ((rc = make_tmap(&tmh[6], g.aRi, g.kpRi, 4 * g.rowsRi))) return rc;
            pr.push_back({tmd + 2, tmd + 3, gi32, g.N2, g.rowsC, g.kpC / KT, g.N2, g.rowsC, 0});
            add_tiles(ST_C, (uint32_t)pr.size() - 1, true);
            pr.push_back({tmd + 4, tmd + 5, gi32, g.Y, g.rowsCi, g.kpCi / KT, g.Y, g.rowsCi, 0});
            add_tiles(ST_CI, (uint32_t)pr.size() - 1, true);
            pr.push_back({tmd + 6, tmd + 7, gi32, g.rowsRi, g.X, 2 * g.kpRi / KT, g.rowsRi, g.X, 0});
            add_tiles(ST_RI, (uint32_t)pr.size() - 1, false);
        }
        for (uint32_t r = 0; r < g.rowsR; ++r) pref.push_back({gi32, r});
    }
    TPT_CUDA(cudaMemcpy(I->tmaps, tm.data(), tm.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    if ((rc = I->alloc(&I->probs, pr.size()))) return rc;
    TPT_CUDA(cudaMemcpy(I->probs, pr.data(), pr.size() * sizeof(Problem), cudaMemcpyHostToDevice));
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Longest K loops first: CTA b takes tiles b, b + grid, ..., so a long
    // tile placed late would start late and stretch the launch.
    auto upload = [&](std::vector<Tile> &v, Tile **dst, uint32_t *n) -> int {
        std::stable_sort(v.begin(), v.end(),
                         [&](const Tile &a, const Tile &b) { return pr[a.problem].ktiles > pr[b.problem].ktiles; });
        int r = I->alloc(dst, v.size());
        if (r) return r;
        TPT_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(Tile), cudaMemcpyHostToDevice));
        *n = (uint32_t)v.size();
        return TPT_OK;
    };
    I->sms = (uint32_t)sms;
    size_t in_branch[2] = {0, 0};
    for (int st = 0; st < NSTAGES; ++st) {
        if ((rc = upload(tl[st], &I->tiles[st], &I->ntiles[st]))) return rc;
        I->grid[st] = std::min<uint32_t>(I->ntiles[st], (uint32_t)sms);
        for (int b = 0; b < 2; ++b) {
            if ((rc = upload(btl[b][st], &I->btiles[b][st], &I->bntiles[b][st]))) return rc;
            in_branch[b] += btl[b][st].size();
        }
    }
    I->split_ok = in_branch[0] > 0 && in_branch[1] > 0 && sms > 1;
    if (I->split_ok) {
        TPT_CUDA(cudaStreamCreateWithFlags(&I->side, cudaStreamNonBlocking));
        TPT_CUDA(cudaEventCreateWithFlags(&I->fork, cudaEventDisableTiming));
        TPT_CUDA(cudaEventCreateWithFlags(&I->join, cudaEventDisableTiming));
    }
    if ((rc = I->alloc(&I->prep, pref.size()))) return rc;
    TPT_CUDA(cudaMemcpy(I->prep, pref.data(), pref.size() * sizeof(PrepRef), cudaMemcpyHostToDevice));
    I->nprep = (uint32_t)pref.size();
    I->ios_host.assign(n, InstIO{});
    if ((rc = I->alloc(&I->ios, n))) return rc;
    return TPT_OK;
}

void DftSet::dims(size_t j, uint32_t *n1, uint32_t *n2) const {
    const JobShape &s = impl->shapes[j];
    *n1 = 2 * s.X;
    *n2 = 2 * s.Y;
}

int DftSet::set_io(size_t j, const SolveIO &io) {
    DftImpl *I = impl;
    uint32_t pos = I->inst_local[j];
    I->ios_host[pos] = InstIO{io.mass_i, io.mass_f, io.mask, io.gx, io.gy, io.mass_scale_inv, io.pitch};
    TPT_CUDA(cudaMemcpy(I->ios + pos, &I->ios_host[pos], sizeof(InstIO), cudaMemcpyHostToDevice));
    return TPT_OK;
}

// One stage's GEMM launch over a tile list, `ctas` persistent CTAs at most.
// CTA b takes tiles b, b + grid, ..., so the launch lasts ceil(n / grid)
// tile rounds; the grid is the fewest CTAs that need no more rounds than
// `ctas` would (450 tiles on 148 SMs: 113 CTAs, 4 rounds each at most), which
// leaves the SMs that would only idle in the last round to the air launches
// running beside the gravity chain.
template <int S>
static int stage_launch(const DftImpl *I, const Tile *tiles, uint32_t n, uint32_t ctas, cudaStream_t st,
                        const InstIO &io0, int act) {
    if (n == 0) return TPT_OK;
    const uint32_t cap = std::max<uint32_t>(1u, std::min(n, ctas));
    const uint32_t rounds = (n + cap - 1) / cap;
    const uint32_t grid = (n + rounds - 1) / rounds;
    constexpr int smem = (S == ST_R || S == ST_RI) ? SMEM_R_BYTES : SMEM_BYTES;
    dft_gemm<S><<<grid, THREADS, smem, st>>>(I->probs, tiles, n, I->groups, I->ios, io0, act, I->err);
    TPT_LAUNCHED();
    return TPT_OK;
}

int DftSet::launch(cudaStream_t st, const SolveIO *io) const {
    const DftImpl *I = impl;
    InstIO io0{};
    int act = 0;
    if (io) {
        io0 = InstIO{io->mass_i, io->mass_f, io->mask, io->gx, io->gy, io->mass_scale_inv, io->pitch};
        act = 1;
    }
    prep_mass<<<I->nprep, 64, 0, st>>>(I->groups, I->prep, I->ios, io0, act);
    TPT_LAUNCHED();
    int rc;
    if (!split_active()) {
        // R, then the y stage of each group (DFT pair or Toeplitz), then R^-1
        if ((rc = stage_launch<ST_R>(I, I->tiles[ST_R], I->ntiles[ST_R], I->grid[ST_R], st, io0, act))) return rc;
        if ((rc = stage_launch<ST_C>(I, I->tiles[ST_C], I->ntiles[ST_C], I->grid[ST_C], st, io0, act))) return rc;
        if ((rc = stage_launch<ST_CI>(I, I->tiles[ST_CI], I->ntiles[ST_CI], I->grid[ST_CI], st, io0, act))) return rc;
        if ((rc = stage_launch<ST_T>(I, I->tiles[ST_T], I->ntiles[ST_T], I->grid[ST_T], st, io0, act))) return rc;
        return stage_launch<ST_RI>(I, I->tiles[ST_RI], I->ntiles[ST_RI], I->grid[ST_RI], st, io0, act);
    }
    // The two forms of y stage touch disjoint groups: fork the DFT-pair
    // groups' chain onto the side stream with side_ctas CTAs per launch and
    // run the Toeplitz groups' chain beside it on the remaining SMs.
    const uint32_t cs = I->side_ctas, cm = I->sms - I->side_ctas;
    TPT_CUDA(cudaEventRecord(I->fork, st));
    TPT_CUDA(cudaStreamWaitEvent(I->side, I->fork, 0));
    Tile *const *b1 = I->btiles[1];
    const uint32_t *n1 = I->bntiles[1];
    if ((rc = stage_launch<ST_R>(I, b1[ST_R], n1[ST_R], cs, I->side, io0, act))) return rc;
    if ((rc = stage_launch<ST_C>(I, b1[ST_C], n1[ST_C], cs, I->side, io0, act))) return rc;
    if ((rc = stage_launch<ST_CI>(I, b1[ST_CI], n1[ST_CI], cs, I->side, io0, act))) return rc;
    if ((rc = stage_launch<ST_RI>(I, b1[ST_RI], n1[ST_RI], cs, I->side, io0, act))) return rc;
    Tile *const *b0 = I->btiles[0];
    const uint32_t *n0 = I->bntiles[0];
    if ((rc = stage_launch<ST_R>(I, b0[ST_R], n0[ST_R], cm, st, io0, act))) return rc;
    if ((rc = stage_launch<ST_T>(I, b0[ST_T], n0[ST_T], cm, st, io0, act))) return rc;
    if ((rc = stage_launch<ST_RI>(I, b0[ST_RI], n0[ST_RI], cm, st, io0, act))) return rc;
    TPT_CUDA(cudaEventRecord(I->join, I->side));
    TPT_CUDA(cudaStreamWaitEvent(st, I->join, 0));
    return TPT_OK;
}

bool DftSet::can_split() const { return impl && impl->split_ok; }

bool DftSet::split_active() const { return impl && impl->split_ok && impl->side_ctas > 0; }

uint32_t DftSet::max_side_ctas() const { return impl && impl->split_ok ? impl->sms / 2 : 0u; }

int DftSet::set_side_ctas(uint32_t ctas) {
    if (ctas > max_side_ctas())
        TPT_FAIL(TPT_ERR_INVALID_ARG, "grav_side_ctas %u above %u", ctas, max_side_ctas());
    impl->side_ctas = ctas;
    return TPT_OK;
}

uint32_t DftSet::launches() const {
    uint32_t n = 1;  // prep_mass
    if (!impl) return n;
    if (split_active()) {
        for (int b = 0; b < 2; ++b)
            for (int s = 0; s < NSTAGES; ++s) n += impl->bntiles[b][s] ? 1u : 0u;
    } else {
        for (int s = 0; s < NSTAGES; ++s) n += impl->ntiles[s] ? 1u : 0u;
    }
    return n;
}
double DftSet::flops() const { return impl ? impl->flops : 0.0; }

void DftSet::destroy() {
    delete impl;
    impl = nullptr;
}

// Reads and clears the device error word of the tensor-core kernels.
int read_errors(uint32_t *out) {
    uint32_t v = 0, z = 0;
    TPT_CUDA(cudaMemcpyFromSymbol(&v, g_dft_err, sizeof(v)));
    TPT_CUDA(cudaMemcpyToSymbol(g_dft_err, &z, sizeof(z)));
    *out = v;
    return TPT_OK;
}

}  // namespace dft
}  // namespace tpt
