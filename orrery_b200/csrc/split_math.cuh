// Packed FP32x2 arithmetic of the precision form (split hi/lo positions,
// Newton-refined SFU rsqrt, Kahan-compensated FP32 partials), shared by the
// direct and batched kernels. Each operation works on a pair of targets; its
// two lanes are exactly the scalar operations of one target.
//
// Source layout (two float4 each for hi and lo, every value stored twice so a
// 16-byte load yields packed operands):
//   hi = (x, x, y, y), (z, z, m, m)       FP32 rounded coordinates and mass
//   lo = (x', x', y', y'), (z', z', 0, 0)  x' = FP32(x - FP32(x)), the rest
#pragma once

#include "common.cuh"

namespace ob {

__device__ __forceinline__ float2 pair_low(const float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 pair_high(const float4 v) { return make_float2(v.z, v.w); }

// A pair of targets: negated hi and lo parts of their coordinates.
struct SplitTargets {
    float2 nhx, nhy, nhz, nlx, nly, nlz;
};

// Loads targets i0 and i1 from the duplicated hi / lo source arrays.
__device__ __forceinline__ SplitTargets load_split_targets(const float4 *hi, const float4 *lo,
                                                           size_t i0, size_t i1) {
    const float4 a0 = hi[2 * i0], a1 = hi[2 * i0 + 1], b0 = hi[2 * i1], b1 = hi[2 * i1 + 1];
    const float4 c0 = lo[2 * i0], c1 = lo[2 * i0 + 1], d0 = lo[2 * i1], d1 = lo[2 * i1 + 1];
    SplitTargets t;
    t.nhx = make_float2(-a0.x, -b0.x);
    t.nhy = make_float2(-a0.z, -b0.z);
    t.nhz = make_float2(-a1.x, -b1.x);
    t.nlx = make_float2(-c0.x, -d0.x);
    t.nly = make_float2(-c0.z, -d0.z);
    t.nlz = make_float2(-c1.x, -d1.x);
    return t;
}

// Kahan step (sum, c) += f d with the compensation kept negated (nc = -c):
//   y = f d - c;  t = sum + y;  c = (t - sum) - y;  sum = t.
__device__ __forceinline__ void kahan2(float2 &sum, float2 &nc, float2 f, float2 d) {
    const float2 m1 = make_float2(-1.0f, -1.0f);
    const float2 y = __ffma2_rn(f, d, nc);
    const float2 t = __fadd2_rn(sum, y);
    const float2 u = __ffma2_rn(sum, m1, t); // t - sum
    nc = __ffma2_rn(u, m1, y);                // y - (t - sum) = -c
    sum = t;
}

// SFU rsqrt estimate refined by one Newton-Raphson step,
// y <- y + (y/2)(1 - r2 y^2), to about one ulp.
__device__ __forceinline__ float2 refined_rsqrt2(float2 r2) {
    const float2 y = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    const float2 ne = __ffma2_rn(r2, __fmul2_rn(y, y), make_float2(-1.0f, -1.0f)); // -(1 - r2 y^2)
    return __ffma2_rn(__fmul2_rn(y, make_float2(-0.5f, -0.5f)), ne, y);
}

// Coordinate differences source - target from the split: the hi parts are
// close, so their difference is exact or nearly; the lo parts restore the
// bits FP32 positions would lose.
__device__ __forceinline__ void split_offsets(const SplitTargets &t, float4 h0, float4 h1,
                                              float4 l0, float4 l1, float2 &dx, float2 &dy,
                                              float2 &dz) {
    dx = __fadd2_rn(__fadd2_rn(pair_low(h0), t.nhx), __fadd2_rn(pair_low(l0), t.nlx));
    dy = __fadd2_rn(__fadd2_rn(pair_high(h0), t.nhy), __fadd2_rn(pair_high(l0), t.nly));
    dz = __fadd2_rn(__fadd2_rn(pair_low(h1), t.nhz), __fadd2_rn(pair_low(l1), t.nlz));
}

} // namespace ob
