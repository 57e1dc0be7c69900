// order.cuh - spatial ordering of arbitrary k-point batches.
//
// The FP32 team Jacobi warm-starts each point from the previous point of its team's contiguous
// range, which pays when consecutive points are neighbours (mesh runs).  Arbitrary batches (the
// adaptive integrator's nodes, random sampling) are put in Morton (Z-curve) order of their
// fractional coordinates first: 10 bits per axis of k mod 1, interleaved into a 30-bit key, a
// stable radix sort of (key, index) pairs, and a gather of the k-points (and weights) in that
// order.  Per-point outputs are written back to their original rows through the sorted indices;
// weighted sums do not depend on the order except through the summation order, which the sort
// fixes deterministically.
#pragma once
#include <cstdint>

// Spreads the low 10 bits of v to every third bit (bit i -> bit 3i).
__device__ __forceinline__ uint32_t morton_spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void morton_keys_kernel(const double *__restrict__ k, int64_t n, uint32_t *__restrict__ keys,
                                   int *__restrict__ index) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t code = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double f = k[3 * i + a];
        f -= floor(f);                                   // k mod 1 in [0, 1); NaN stays NaN
        double q = f * 1024.0;
        int qi = (q >= 0.0 && q < 1024.0) ? (int)q : 0;  // NaN and rounding to 1024 map in range
        code |= morton_spread3((uint32_t)qi) << a;
    }
    keys[i] = code;
    index[i] = (int)i;
}

__global__ void gather_points_kernel(const double *__restrict__ k, const double *__restrict__ w,
                                     const int *__restrict__ perm, int64_t n, double *__restrict__ k_out,
                                     double *__restrict__ w_out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int64_t p = perm[j];
    k_out[3 * j] = k[3 * p];
    k_out[3 * j + 1] = k[3 * p + 1];
    k_out[3 * j + 2] = k[3 * p + 2];
    if (w) w_out[j] = w[p];
}
