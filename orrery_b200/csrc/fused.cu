// Whole integration steps of a small system in one cooperative launch: the
// velocity-Verlet (or Yoshida-4) kicks and drifts and the FP32 direct forces
// of every substep, for systems whose sources fit in one CTA's shared memory.
//
// At a few thousand particles a step is four short launches (kick-drift,
// source packing, forces, kick) whose launch gaps and thin force grid leave
// most of the GPU idle. Here each CTA owns 32 targets (one per lane of each
// warp) and keeps all N sources in shared memory; its W warps (32 where the
// grid fits one CTA per SM, else 16) each sum one W-th of the sources for the
// same targets (the pair loop unrolled so that independent pairs hide each
// other's latency). Per substep:
//   A. each CTA kicks and drifts its own targets (the previous substep's
//      closing kick first, as a separate rounding, then this substep's
//      kick-drift: the same explicitly rounded FP64 operations, in the same
//      order, as kick_kernel and kick_drift_kernel) and writes their FP32
//      positions and masses into buffer s % 2;
//   B. a grid barrier: every position of the substep is written;
//   C. each CTA loads all sources from buffer s % 2 into shared memory and
//      evaluates its targets' accelerations: FP32 pair arithmetic two
//      sources per packed FP32x2 instruction, each warp's slice summed in
//      FP32, the W slices added in FP64 in slice order.
// One barrier per substep suffices: a CTA can only write buffer (s + 2) % 2
// after the barrier of substep s + 1, which every CTA reaches only after it
// has finished loading buffer s % 2. After the last substep each CTA gives
// its targets the closing kick.
//
// The grid barrier is a counter and a generation word in global memory; its
// waits are bounded (kSpinLimit polls, then the timeout bit of the status
// word and no further work), and the launch is cooperative, so every CTA is
// resident. The pair arithmetic is that of the FP32 direct kernel (positions
// rounded to FP32, softened, FP32 sums per slice, FP64 across slices); with
// softening the target's own entry adds exactly zero unless m / eps^3 of the
// target overflows FP32, in which case the warp skips it explicitly.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "internal.hpp"
#include "runtime.hpp"

namespace ob {
namespace {

constexpr uint32_t kFusedTargets = 32; // per CTA: one per lane
constexpr uint32_t kFusedMaxWarps = 32;
// Source padding: a whole number of pairs per slice for 16 or 32 warps.
constexpr uint32_t kFusedGroup = 2 * kFusedMaxWarps;
constexpr size_t kFusedSmemCap = 200u * 1024u; // dynamic shared memory (sources)

struct FusedArgs {
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
    const double *m;
    float4 *buf0, *buf1; // FP32 x y z m per particle, double-buffered
    unsigned *barrier;   // [0] arrivals, [1] generation
    unsigned *status;
    uint32_t n, padded;  // padded: a multiple of kFusedGroup
    uint32_t substeps;   // total substeps of the launch
    uint32_t cycle;      // substeps per step: 1 (velocity Verlet) or 3 (Yoshida-4)
    double h[3];         // substep timesteps of the cycle
    double half[3];      // their halves, computed on the host as the unfused path does
    float eps2;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Waits until every CTA of the grid has arrived. Returns false when the wait
// ran out (the timeout bit is then set).
__device__ bool grid_barrier(unsigned *barrier, unsigned &generation, unsigned *status) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned target = generation + 1u;
        __threadfence();
        const unsigned arrived = atomicAdd(&barrier[0], 1u);
        if (arrived == gridDim.x - 1u) {
            barrier[0] = 0u;
            __threadfence();
            atomicExch(&barrier[1], target);
        } else {
            uint32_t polls = 0;
            while (*reinterpret_cast<volatile unsigned *>(&barrier[1]) != target) {
                if (++polls > kSpinLimit) {
                    atomicOr(status, kStatusTimeout);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        generation = target;
    }
    __syncthreads();
    return ok != 0;
}

// Kick: v += half a (kick_kernel's rounding).
__device__ __forceinline__ double kick(double v, double half, double a) {
    return __dadd_rn(v, __dmul_rn(half, a));
}

template <uint32_t WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    fused_steps_kernel(FusedArgs g) {
    constexpr uint32_t kThreads = WARPS * 32;
    extern __shared__ __align__(16) float4 src[]; // pairs: (x0 x1 y0 y1) (z0 z1 m0 m1)
    __shared__ double partial[WARPS][3][kFusedTargets];
    __shared__ unsigned generation_seen;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t first = blockIdx.x * kFusedTargets;
    const uint32_t i = first + lane; // this lane's target in every warp
    const bool mine = i < g.n;
    unsigned generation = 0;
    if (threadIdx.x == 0) {
        generation_seen = *reinterpret_cast<volatile unsigned *>(&g.barrier[1]);
    }
    __syncthreads();
    generation = generation_seen;

    const uint32_t pairs = g.padded / 2u;
    const uint32_t slice = pairs / WARPS; // pairs per warp
    const float2 e2 = f2(g.eps2, g.eps2);
    bool ok = true;
    for (uint32_t s = 0; s < g.substeps && ok; ++s) {
        const uint32_t c = s % g.cycle;
        float4 *buf = (s & 1u) != 0u ? g.buf1 : g.buf0;
        // A. Kick and drift this CTA's targets (warp 0), write their FP32 copy.
        if (warp == 0 && mine) {
            double vx = g.vx[i], vy = g.vy[i], vz = g.vz[i];
            const double ax = g.ax[i], ay = g.ay[i], az = g.az[i];
            if (s > 0) {
                const double hp = g.half[(s - 1u) % g.cycle];
                vx = kick(vx, hp, ax);
                vy = kick(vy, hp, ay);
                vz = kick(vz, hp, az);
            }
            vx = kick(vx, g.half[c], ax);
            vy = kick(vy, g.half[c], ay);
            vz = kick(vz, g.half[c], az);
            const double x = __dadd_rn(g.x[i], __dmul_rn(g.h[c], vx));
            const double y = __dadd_rn(g.y[i], __dmul_rn(g.h[c], vy));
            const double z = __dadd_rn(g.z[i], __dmul_rn(g.h[c], vz));
            g.vx[i] = vx;
            g.vy[i] = vy;
            g.vz[i] = vz;
            g.x[i] = x;
            g.y[i] = y;
            g.z[i] = z;
            buf[i] = make_float4(__double2float_rn(x), __double2float_rn(y),
                                 __double2float_rn(z), __double2float_rn(g.m[i]));
        }
        // B. Every position of this substep is written.
        ok = grid_barrier(g.barrier, generation, g.status);
        if (!ok) {
            break;
        }
        // C. All sources into shared memory (zero-mass padding at the origin).
        for (uint32_t p = threadIdx.x; p < pairs; p += kThreads) {
            const uint32_t j = 2u * p;
            const float4 a = j < g.n ? __ldcg(&buf[j]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const float4 b =
                j + 1u < g.n ? __ldcg(&buf[j + 1u]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            src[2u * p] = make_float4(a.x, b.x, a.y, b.y);
            src[2u * p + 1u] = make_float4(a.z, b.z, a.w, b.w);
        }
        __syncthreads();
        float tx = 0.0f, ty = 0.0f, tz = 0.0f, tm = 0.0f;
        if (mine) {
            const float4 q0 = src[2u * (i >> 1)], q1 = src[2u * (i >> 1) + 1u];
            const bool odd = (i & 1u) != 0u;
            tx = odd ? q0.y : q0.x;
            ty = odd ? q0.w : q0.z;
            tz = odd ? q1.y : q1.x;
            tm = odd ? q1.w : q1.z;
        }
        // With softening the target's own entry adds exactly zero (d = 0)
        // unless m / eps^3 overflows FP32; then the warp skips it by index.
        const float self_inv = rsqrt_approx(g.eps2);
        const float self_term = (tm * self_inv) * (self_inv * self_inv);
        const bool skip_self = __any_sync(0xffffffffu, mine && !(fabsf(self_term) < 3.0e38f));
        const float2 ntx = f2(-tx, -tx), nty = f2(-ty, -ty), ntz = f2(-tz, -tz);
        float2 sx = f2(0.0f, 0.0f), sy = sx, sz = sx;
        const uint32_t p0 = warp * slice, p1 = p0 + slice;
#pragma unroll 4
        for (uint32_t p = p0; p < p1; ++p) {
            const float4 q0 = src[2u * p], q1 = src[2u * p + 1u];
            const float2 dx = __fadd2_rn(f2(q0.x, q0.y), ntx);
            const float2 dy = __fadd2_rn(f2(q0.z, q0.w), nty);
            const float2 dz = __fadd2_rn(f2(q1.x, q1.y), ntz);
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, e2)));
            float inv0 = rsqrt_approx(r2.x), inv1 = rsqrt_approx(r2.y);
            if (skip_self) {
                inv0 = 2u * p == i ? 0.0f : inv0;
                inv1 = 2u * p + 1u == i ? 0.0f : inv1;
            }
            const float2 inv = f2(inv0, inv1);
            const float2 f = __fmul2_rn(__fmul2_rn(f2(q1.z, q1.w), inv), __fmul2_rn(inv, inv));
            sx = __ffma2_rn(f, dx, sx);
            sy = __ffma2_rn(f, dy, sy);
            sz = __ffma2_rn(f, dz, sz);
        }
        partial[warp][0][lane] = static_cast<double>(sx.x) + static_cast<double>(sx.y);
        partial[warp][1][lane] = static_cast<double>(sy.x) + static_cast<double>(sy.y);
        partial[warp][2][lane] = static_cast<double>(sz.x) + static_cast<double>(sz.y);
        __syncthreads();
        if (warp == 0 && mine) {
            double a[3] = {0.0, 0.0, 0.0};
            for (uint32_t w = 0; w < WARPS; ++w) {
                for (int k = 0; k < 3; ++k) {
                    a[k] += partial[w][k][lane];
                }
            }
            g.ax[i] = a[0];
            g.ay[i] = a[1];
            g.az[i] = a[2];
        }
        // The next substep reuses the shared arrays only after its barrier.
    }
    // The closing kick of the last substep.
    if (ok && warp == 0 && mine && g.substeps > 0) {
        const double hp = g.half[(g.substeps - 1u) % g.cycle];
        g.vx[i] = kick(g.vx[i], hp, g.ax[i]);
        g.vy[i] = kick(g.vy[i], hp, g.ay[i]);
        g.vz[i] = kick(g.vz[i], hp, g.az[i]);
    }
}

size_t fused_smem(uint32_t padded) { return static_cast<size_t>(padded) * 16u; }

uint32_t fused_padded(uint32_t n) {
    return (n + kFusedGroup - 1u) / kFusedGroup * kFusedGroup;
}

// Whether a grid of `blocks` CTAs of the WARPS-warp kernel, with `smem` bytes
// of sources, is resident at once (the cooperative launch requires it).
template <uint32_t WARPS>
bool fused_resident(uint64_t blocks, size_t smem, int sms) {
    static std::atomic<uint64_t> configured{0};
    const void *kernel = reinterpret_cast<const void *>(fused_steps_kernel<WARPS>);
    int per_sm = 0;
    if (set_smem_limit_once(kernel, static_cast<int>(kFusedSmemCap), configured) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, WARPS * 32, smem) !=
            cudaSuccess) {
        return false;
    }
    return blocks <= static_cast<uint64_t>(per_sm) * static_cast<uint64_t>(sms);
}

} // namespace

uint32_t fused_steps_warps(uint32_t n) {
    if (n < 2u) {
        return 0u;
    }
    const size_t smem = fused_smem(fused_padded(n));
    if (smem > kFusedSmemCap) {
        return 0u;
    }
    int device = 0, sms = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        return 0u;
    }
    const uint64_t blocks = (n + kFusedTargets - 1u) / kFusedTargets;
    if (fused_resident<32>(blocks, smem, sms)) {
        return 32u;
    }
    return fused_resident<16>(blocks, smem, sms) ? 16u : 0u;
}

size_t fused_scratch_floats4(uint32_t n) { return 2ull * fused_padded(n); }

cudaError_t launch_fused_steps(double *const *state, const double *m, uint32_t n,
                               uint64_t steps, int cycle, const double *h, float eps2,
                               float4 *scratch, unsigned *barrier, unsigned *status,
                               uint32_t warps, cudaStream_t stream) {
    if (n == 0 || steps == 0) {
        return cudaSuccess;
    }
    if (warps != 16u && warps != 32u) {
        return cudaErrorInvalidValue;
    }
    FusedArgs g{};
    g.x = state[0];
    g.y = state[1];
    g.z = state[2];
    g.vx = state[3];
    g.vy = state[4];
    g.vz = state[5];
    g.ax = state[6];
    g.ay = state[7];
    g.az = state[8];
    g.m = m;
    g.padded = fused_padded(n);
    g.buf0 = scratch;
    g.buf1 = scratch + g.padded;
    g.barrier = barrier;
    g.status = status;
    g.n = n;
    g.cycle = static_cast<uint32_t>(cycle);
    if (steps * static_cast<uint64_t>(cycle) > 0xffffffffull) {
        return cudaErrorInvalidValue;
    }
    g.substeps = static_cast<uint32_t>(steps * static_cast<uint64_t>(cycle));
    for (int k = 0; k < cycle && k < 3; ++k) {
        g.h[k] = h[k];
        g.half[k] = h[k] / 2.0; // as enqueue_substep computes it
    }
    g.eps2 = eps2;
    const uint32_t blocks = (n + kFusedTargets - 1u) / kFusedTargets;
    void *args[] = {&g};
    const void *kernel = warps == 32u ? reinterpret_cast<const void *>(fused_steps_kernel<32>)
                                      : reinterpret_cast<const void *>(fused_steps_kernel<16>);
    return cudaLaunchCooperativeKernel(kernel, dim3(blocks), dim3(warps * 32u), args,
                                       fused_smem(g.padded), stream);
}

} // namespace ob
