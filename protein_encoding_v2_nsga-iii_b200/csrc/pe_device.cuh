// pe_device.cuh -- device helpers: counter-based RNG, deterministic exp, reductions.
//
// All floating-point arithmetic in this engine is written as single IEEE
// operations in a fixed order and compiled with --fmad=false, so results are
// bit-identical to a sequential host restatement of the same formulas.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pe {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).  Keyed by the instance seed; the counter carries
// (tag, generation, individual, position) so each draw is independent of the
// launch shape -- the reference's per-thread XORWOW state (src/main.cu:35)
// made results depend on the grid.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// word j of the draw stream (tag, gen, idx, pos)
__device__ __forceinline__ uint32_t draw(uint64_t seed, uint32_t tag, uint32_t gen, uint32_t idx, uint32_t pos,
                                         uint32_t j)
{
    uint4 o = philox4x32_10(make_uint4(tag, gen, idx, pos * 8u + (j >> 2)),
                            make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    switch (j & 3u) {
    case 0: return o.x;
    case 1: return o.y;
    case 2: return o.z;
    default: return o.w;
    }
}

// uniform integer in [0, k) by multiply-shift
__device__ __forceinline__ uint32_t rng_uint(uint32_t r, uint32_t k) { return __umulhi(r, k); }
// uniform float in (0, 1] on a 24-bit grid
__device__ __forceinline__ float rng_u01(uint32_t r)
{
    return __fmul_rn((float)((r >> 8) + 1u), 1.0f / 16777216.0f);
}

// exp(x) for x <= 0 from IEEE double add/mul/fma only: Cody-Waite reduction by
// ln 2, degree-13 Taylor polynomial (Horner), exact scaling by 2^k.
__device__ __forceinline__ double det_exp(double x)
{
    if (x < -700.0) return 0.0;
    const double inv_ln2 = 1.4426950408889634;
    const double ln2_hi = 0.6931471803691238;
    const double ln2_lo = 1.9082149292705877e-10;
    double kd = rint(__dmul_rn(x, inv_ln2));
    double r = fma(-kd, ln2_hi, x);
    r = fma(-kd, ln2_lo, r);
    double p = 1.6059043836821613e-10;
    p = fma(p, r, 2.08767569878681e-09);
    p = fma(p, r, 2.505210838544172e-08);
    p = fma(p, r, 2.755731922398589e-07);
    p = fma(p, r, 2.7557319223985893e-06);
    p = fma(p, r, 2.48015873015873e-05);
    p = fma(p, r, 0.0001984126984126984);
    p = fma(p, r, 0.001388888888888889);
    p = fma(p, r, 0.008333333333333333);
    p = fma(p, r, 0.041666666666666664);
    p = fma(p, r, 0.16666666666666666);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    int k = (int)kd;
    double scale = __longlong_as_double((long long)(k + 1023) << 52);
    return __dmul_rn(p, scale);
}

template <class T> __device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_max_i(int v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ __forceinline__ int warp_min_i(int v) { return __reduce_min_sync(0xffffffffu, v); }

}  // namespace pe
