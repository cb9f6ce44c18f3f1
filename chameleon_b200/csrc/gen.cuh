// gen.cuh -- the reference's seeded matrix generator, on the device.
#pragma once
#include <cuda_runtime.h>

namespace chb {

// LCG skip-ahead of the reference generator (coreblas/include/coreblas/random.h
// :32-73): x_{k+1} = a x_k + c mod 2^64, a = 6364136223846793005, c = 1; the
// n-th state is reached by composing the affine map with itself over the bits
// of n (Brown, "Random number generation with arbitrary strides", 1994).
__host__ __device__ __forceinline__ unsigned long long lcg_skip(unsigned long long n, unsigned long long x) {
    unsigned long long a = 6364136223846793005ULL, c = 1ULL;
    while (n) {
        if (n & 1ULL) x = a * x + c;
        c = c * (a + 1ULL);
        a = a * a;
        n >>= 1;
    }
    return x;
}
// Uniform value of state x: 0.5 - x * 2^-64 (random.h CORE_dlaran), no
// contraction so that the rounding matches the host code.
__device__ __forceinline__ double lcg_value(unsigned long long x) {
    return __dsub_rn(0.5, __dmul_rn(__ull2double_rn(x), 5.4210108624275222e-20));
}

}  // namespace chb
