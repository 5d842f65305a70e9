// Compares div_by_rcp (hpgl_b200/csrc/device_common.cuh: quotient from the
// correctly rounded reciprocal plus one fused correction) with CUDA's IEEE
// division __ddiv_rn on the GPU over random operands: operands drawn with
// kriging-like magnitudes and over a wide exponent range.  Prints
// "mismatches <count> of <total>" and exits non-zero on any mismatch.
#include <cstdio>
#include <cstdlib>
#include "../../hpgl_b200/csrc/device_common.cuh"

__device__ unsigned long long g_bad;

__device__ __forceinline__ unsigned long long mix(unsigned long long x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

__global__ void check(unsigned long long n, unsigned long long seed, int wide) {
    unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    unsigned long long bad = 0;
    for (; i < n; i += stride) {
        unsigned long long u = mix(i * 2 + seed), v = mix(i * 2 + 1 + seed);
        double a, b;
        if (wide) {
            // random sign/mantissa, exponent in [-300, 300]
            a = __longlong_as_double((long long)((u & 0x800FFFFFFFFFFFFFULL) | ((unsigned long long)(1023 - 300 + (u >> 52) % 601) << 52)));
            b = __longlong_as_double((long long)((v & 0x800FFFFFFFFFFFFFULL) | ((unsigned long long)(1023 - 300 + (v >> 52) % 601) << 52)));
        } else {
            a = ((double)(u >> 11) / 9007199254740992.0 - 0.5) * 4.0;            // [-2, 2)
            b = 1e-3 + (double)(v >> 11) / 9007199254740992.0 * 2.0;             // (0, 2]
        }
        const double y = __drcp_rn(b);
        const double q1 = __ddiv_rn(a, b), q2 = hpgl_b200::div_by_rcp(a, b, y);
        if (__double_as_longlong(q1) != __double_as_longlong(q2)) ++bad;
    }
    if (bad) atomicAdd(&g_bad, bad);
}

int main(int argc, char **argv) {
    unsigned long long n = argc > 1 ? strtoull(argv[1], 0, 10) : 100000000ULL;
    unsigned long long total_bad = 0;
    for (int wide = 0; wide < 2; ++wide) {
        unsigned long long zero = 0;
        cudaMemcpyToSymbol(g_bad, &zero, sizeof(zero));
        check<<<1184, 256>>>(n, 12345 + wide, wide);
        if (cudaDeviceSynchronize() != cudaSuccess) { printf("cuda error\n"); return 2; }
        unsigned long long bad = 0;
        cudaMemcpyFromSymbol(&bad, g_bad, sizeof(bad));
        printf("%s operands: mismatches %llu of %llu\n", wide ? "wide" : "kriging-range", bad, n);
        total_bad += bad;
    }
    return total_bad ? 1 : 0;
}
