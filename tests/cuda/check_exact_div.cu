// Exhaustive check of div_by_const (the library's correctly rounded division
// by a constant) against IEEE division on the device: every one of the 2^32
// f32 inputs, for every divisor the library uses it with. Prints one line per
// divisor: "<divisor bits> <mismatches> <first mismatching input bits> <largest
// mismatching finite |input| bits>" (hex), NaN results compared as NaN.
// Built and run by tests/test_gpu_exact_div.py.
#include <cstdio>
#include <cstdint>
#include <cstring>

#include "exact_div.cuh"

__global__ void check(float c, float rc, unsigned long long *bad, uint32_t *first, uint32_t *maxmag) {
    const uint64_t n = 1ull << 32;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((uint32_t)i);
        const float a = tpt::div_by_const(x, c, rc), b = __fdiv_rn(x, c);
        const bool same = (a != a && b != b) || __float_as_uint(a) == __float_as_uint(b);
        if (!same) {
            atomicAdd(bad, 1ull);
            atomicMin(first, (uint32_t)i);
            if (((uint32_t)i & 0x7F800000u) != 0x7F800000u)  // largest finite |x| that differs (bit order)
                atomicMax(maxmag, (uint32_t)i & 0x7FFFFFFFu);
        }
    }
}

int main() {
    // The 2-D air divisors, then the 3-D field step's: the six-neighbour
    // counts 4..7 of its averages and the 6 of its pressure sweep.
    const float cs[7][2] = {{tpt::kSmoothWsum, tpt::kSmoothWsumRcp},
                            {tpt::kConvLegacy, tpt::kConvLegacyRcp},
                            {tpt::kConvBouss, tpt::kConvBoussRcp},
                            {4.0f, 1.0f / 4.0f},
                            {5.0f, 1.0f / 5.0f},
                            {6.0f, 1.0f / 6.0f},
                            {7.0f, 1.0f / 7.0f}};
    unsigned long long *bad;
    uint32_t *first, *maxmag;
    if (cudaMalloc(&bad, sizeof(*bad)) != cudaSuccess || cudaMalloc(&first, sizeof(*first)) != cudaSuccess ||
        cudaMalloc(&maxmag, sizeof(*maxmag)) != cudaSuccess)
        return 2;
    for (auto &c : cs) {
        unsigned long long h = 0;
        uint32_t f = 0xFFFFFFFFu;
        cudaMemcpy(bad, &h, sizeof(h), cudaMemcpyHostToDevice);
        uint32_t mm = 0;
        cudaMemcpy(first, &f, sizeof(f), cudaMemcpyHostToDevice);
        cudaMemcpy(maxmag, &mm, sizeof(mm), cudaMemcpyHostToDevice);
        check<<<148 * 8, 256>>>(c[0], c[1], bad, first, maxmag);
        if (cudaDeviceSynchronize() != cudaSuccess) return 3;
        cudaMemcpy(&h, bad, sizeof(h), cudaMemcpyDeviceToHost);
        cudaMemcpy(&f, first, sizeof(f), cudaMemcpyDeviceToHost);
        cudaMemcpy(&mm, maxmag, sizeof(mm), cudaMemcpyDeviceToHost);
        uint32_t cb;
        memcpy(&cb, &c[0], 4);
        printf("%08x %llu %08x %08x\n", cb, h, f, mm);
    }
    return 0;
}
