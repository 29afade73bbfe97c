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
// other's latency). The FP64 state of the CTA's targets stays in shared
// memory for the whole launch (read at the start, written back at the end).
// Per substep:
//   A. warp 0 kicks and drifts the CTA's targets (the previous substep's
//      closing kick first, as a separate rounding, then this substep's
//      kick-drift: the same explicitly rounded FP64 operations, in the same
//      order, as kick_kernel and kick_drift_kernel), writes their FP32
//      positions and masses into buffer s % 2 (already in the pair layout
//      the pair loop reads) and then raises the CTA's ready word to this
//      substep's number;
//   B. every warp copies its share of the sources from buffer s % 2 into
//      shared memory, each 32-source chunk by one bulk copy once the ready
//      word of the CTA that wrote it has reached this substep (no grid-wide
//      barrier: a warp waits only for the chunks it copies; the CTA waits on
//      an mbarrier for the bytes of all of them);
//   C. the CTA evaluates its targets' accelerations: FP32 pair arithmetic
//      two sources per packed FP32x2 instruction, each warp's slice summed
//      in FP32, the W slices added in FP64 in slice order by warp 0.
// Double buffering is safe with per-CTA words: a CTA writes buffer s % 2
// again only at substep s + 2, after its forces of substep s + 1, which need
// every CTA's chunk of substep s + 1, which each CTA publishes only after its
// copies of buffer s % 2 have landed. After the last substep warp 0 gives the
// targets the closing kick and writes their state back.
//
// Ready words count substeps across launches (the host passes the count so
// far, `epoch`, and clears the words together with it); waits are bounded
// (kSpinLimit polls, or fewer where a test asks, then the timeout bit of the
// status word, and every CTA stops after the substep it is in), and the
// launch is cooperative, so every CTA is resident. The pair arithmetic is that of the FP32 direct kernel
// (positions rounded to FP32, softened, FP32 sums per slice, FP64 across
// slices); with softening the target's own entry adds exactly zero unless
// m / eps^3 of the target overflows FP32, in which case the warp skips it
// explicitly.
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
// Every warp's chunks have their ready words polled by one lane each.
static_assert(kFusedSmemCap / 16u / 32u / 16u <= 32u, "at most 32 chunks per warp");
// Ready words one 128-byte line apart: polls of different CTAs' words then go
// to different L2 lines instead of queueing on a few.
constexpr uint32_t kReadyStride = 32;

struct FusedArgs {
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
    const double *m;
    float4 *buf0, *buf1; // FP32 sources in pairs (x0 x1 y0 y1) (z0 z1 m0 m1), double-buffered
    unsigned *ready;     // per CTA (kReadyStride apart): substeps published, across launches
    unsigned *status;
    uint32_t n, padded;  // padded: a multiple of kFusedGroup
    uint32_t substeps;   // total substeps of the launch
    uint32_t cycle;      // substeps per step: 1 (velocity Verlet) or 3 (Yoshida-4)
    uint32_t epoch;      // substeps published by earlier launches since the words were cleared
    uint32_t poll_limit; // polls of a ready word before the wait gives up (kSpinLimit)
    uint32_t silent_cta; // a CTA that never publishes (tests of the bounded wait), or ~0
    double h[3];         // substep timesteps of the cycle
    double half[3];      // their halves, computed on the host as the unfused path does
    float eps2;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Kick: v += half a (kick_kernel's rounding).
__device__ __forceinline__ double kick(double v, double half, double a) {
    return __dadd_rn(v, __dmul_rn(half, a));
}

// Whether a ready word has reached `target` (the counts wrap at 2^32).
__device__ __forceinline__ bool reached(unsigned word, unsigned target) {
    return static_cast<int>(word - target) >= 0;
}

// A ready word, read with acquire semantics at GPU scope: this thread's later
// loads see every write the publishing CTA made before raising it.
__device__ __forceinline__ unsigned load_acquire(const unsigned *word) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(word) : "memory");
    return v;
}

// Raises a ready word with release semantics at GPU scope.
__device__ __forceinline__ void store_release(unsigned *word, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" : : "l"(word), "r"(v) : "memory");
}

// Pairs [p0, p1) of the staged sources against the lane's target (offset
// -t): FP32 terms two sources per packed instruction, added to the slice
// sums. SKIP_SELF zeroes the target's own term by index.
template <bool SKIP_SELF>
__device__ __forceinline__ void pair_slice(const float4 *src, uint32_t p0, uint32_t p1,
                                           uint32_t i, float2 ntx, float2 nty, float2 ntz,
                                           float2 e2, float2 &sx, float2 &sy, float2 &sz) {
#pragma unroll 4
    for (uint32_t p = p0; p < p1; ++p) {
        const float4 q0 = src[2u * p], q1 = src[2u * p + 1u];
        const float2 dx = __fadd2_rn(f2(q0.x, q0.y), ntx);
        const float2 dy = __fadd2_rn(f2(q0.z, q0.w), nty);
        const float2 dz = __fadd2_rn(f2(q1.x, q1.y), ntz);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, e2)));
        float inv0 = rsqrt_approx(r2.x), inv1 = rsqrt_approx(r2.y);
        if (SKIP_SELF) {
            inv0 = 2u * p == i ? 0.0f : inv0;
            inv1 = 2u * p + 1u == i ? 0.0f : inv1;
        }
        const float2 inv = f2(inv0, inv1);
        const float2 f = __fmul2_rn(__fmul2_rn(f2(q1.z, q1.w), inv), __fmul2_rn(inv, inv));
        sx = __ffma2_rn(f, dx, sx);
        sy = __ffma2_rn(f, dy, sy);
        sz = __ffma2_rn(f, dz, sz);
    }
}

template <uint32_t WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    fused_steps_kernel(FusedArgs g) {
    extern __shared__ __align__(16) float4 src[]; // pairs: (x0 x1 y0 y1) (z0 z1 m0 m1)
    __shared__ double partial[WARPS][3][kFusedTargets];
    __shared__ double state[9][kFusedTargets]; // x y z vx vy vz ax ay az of the CTA's targets
    __shared__ int stop;
    __shared__ __align__(8) uint64_t loaded; // the substep's source chunks have landed
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * kFusedTargets + lane; // this lane's target in every warp
    const bool mine = i < g.n;
    double *const global_state[9] = {g.x, g.y, g.z, g.vx, g.vy, g.vz, g.ax, g.ay, g.az};
    float mass = 0.0f;
    if (warp == 0) {
        for (int k = 0; k < 9; ++k) {
            state[k][lane] = mine ? global_state[k][i] : 0.0;
        }
        mass = mine ? __double2float_rn(g.m[i]) : 0.0f;
    }
    if (threadIdx.x == 0) {
        stop = 0;
        mbar_init(&loaded, 1);
        fence_barrier_init();
    }
    __syncthreads();
    const uint32_t blocks = gridDim.x;
    const uint32_t chunks = g.padded / 32u; // 32-source chunks, padding included
    const uint32_t slice = g.padded / 2u / WARPS; // pairs per warp
    const float2 e2 = f2(g.eps2, g.eps2);
    uint32_t s = 0;
    for (; s < g.substeps; ++s) {
        const uint32_t c = s % g.cycle;
        const unsigned target = g.epoch + s + 1u;
        float4 *buf = (s & 1u) != 0u ? g.buf1 : g.buf0;
        // A. Kick and drift this CTA's targets, publish their FP32 copy.
        if (warp == 0) {
            if (mine) {
                double vx = state[3][lane], vy = state[4][lane], vz = state[5][lane];
                const double ax = state[6][lane], ay = state[7][lane], az = state[8][lane];
                if (s > 0) {
                    const double hp = g.half[(s - 1u) % g.cycle];
                    vx = kick(vx, hp, ax);
                    vy = kick(vy, hp, ay);
                    vz = kick(vz, hp, az);
                }
                vx = kick(vx, g.half[c], ax);
                vy = kick(vy, g.half[c], ay);
                vz = kick(vz, g.half[c], az);
                const double x = __dadd_rn(state[0][lane], __dmul_rn(g.h[c], vx));
                const double y = __dadd_rn(state[1][lane], __dmul_rn(g.h[c], vy));
                const double z = __dadd_rn(state[2][lane], __dmul_rn(g.h[c], vz));
                state[0][lane] = x;
                state[1][lane] = y;
                state[2][lane] = z;
                state[3][lane] = vx;
                state[4][lane] = vy;
                state[5][lane] = vz;
                // Slot i % 2 of pair i / 2: (x0 x1 y0 y1) (z0 z1 m0 m1), the
                // layout the pair loop reads, so that chunks copy as they are.
                float *lo = reinterpret_cast<float *>(&buf[2u * (i >> 1)]) + (i & 1u);
                float *hi = reinterpret_cast<float *>(&buf[2u * (i >> 1) + 1u]) + (i & 1u);
                lo[0] = __double2float_rn(x);
                lo[2] = __double2float_rn(y);
                hi[0] = __double2float_rn(z);
                hi[2] = mass;
            }
            asm volatile("fence.proxy.async.global;" ::: "memory");
            __threadfence();
            __syncwarp();
            if (lane == 0 && blockIdx.x != g.silent_cta) {
                store_release(&g.ready[blockIdx.x * kReadyStride], target);
            }
        }
        // B. Sources into shared memory, chunk q = sources 32q .. 32q + 31
        // (512 bytes; zero-mass padding at the origin past N, zeroed once on
        // the host and never written), once the CTA that wrote each chunk has
        // published it. Warp w copies chunks w, w + W, ...: lane k polls the
        // ready word of the warp's k-th chunk (at most 32) and then starts
        // its bulk copy, completing on `loaded`, whose byte count thread 0
        // posts for the substep. A chunk whose wait ran out is copied all
        // the same, so that the barrier completes and no copy is left in
        // flight; the substep is then abandoned.
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(&loaded, g.padded * 16u);
        }
        {
            const uint32_t q = warp + WARPS * lane;
            const bool copies = q < chunks;
            const bool polling = copies && q < blocks;
            for (uint32_t polls = 0;; ++polls) {
                const bool behind =
                    polling && !reached(load_acquire(&g.ready[q * kReadyStride]), target);
                if (!__any_sync(0xffffffffu, behind)) {
                    break;
                }
                if (polls >= g.poll_limit) {
                    if (lane == 0) {
                        atomicOr(g.status, kStatusTimeout);
                        stop = 1;
                    }
                    break;
                }
            }
            if (copies) {
                // The chunk's generic-proxy writes (acquired above) before
                // the async-proxy read; this CTA's reads of the previous
                // substep's sources before the async-proxy write.
                asm volatile("fence.proxy.async.global;" ::: "memory");
                fence_proxy_async_shared();
                bulk_copy_g2s(&src[32u * q], &buf[32u * q], 512u, &loaded);
            }
        }
        if (!mbar_wait_bounded(&loaded, s & 1u, g.status)) {
            stop = 1;
        }
        __syncthreads();
        if (stop != 0) {
            break; // every thread reads the same word after the barrier
        }
        // C. This CTA's targets against every source.
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
        // The warp-uniform choice is made once, outside the pair loop.
        if (skip_self) {
            pair_slice<true>(src, p0, p1, i, ntx, nty, ntz, e2, sx, sy, sz);
        } else {
            pair_slice<false>(src, p0, p1, i, ntx, nty, ntz, e2, sx, sy, sz);
        }
        partial[warp][0][lane] = static_cast<double>(sx.x) + static_cast<double>(sx.y);
        partial[warp][1][lane] = static_cast<double>(sy.x) + static_cast<double>(sy.y);
        partial[warp][2][lane] = static_cast<double>(sz.x) + static_cast<double>(sz.y);
        // The sources are read and the partials written: warp 0 adds the
        // slices while the other warps go on to the next substep's loads,
        // which wait for warp 0's next publication.
        __syncthreads();
        if (warp == 0) {
            double a[3] = {0.0, 0.0, 0.0};
            for (uint32_t w = 0; w < WARPS; ++w) {
                for (int k = 0; k < 3; ++k) {
                    a[k] += partial[w][k][lane];
                }
            }
            state[6][lane] = a[0];
            state[7][lane] = a[1];
            state[8][lane] = a[2];
        }
    }
    // The closing kick of the last substep, and the state back to HBM (as
    // far as it got when a wait ran out).
    if (warp == 0 && mine) {
        if (s == g.substeps && s > 0) {
            const double hp = g.half[(s - 1u) % g.cycle];
            state[3][lane] = kick(state[3][lane], hp, state[6][lane]);
            state[4][lane] = kick(state[4][lane], hp, state[7][lane]);
            state[5][lane] = kick(state[5][lane], hp, state[8][lane]);
        }
        for (int k = 0; k < 9; ++k) {
            global_state[k][i] = state[k][lane];
        }
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

uint32_t fused_blocks(uint32_t n) { return (n + kFusedTargets - 1u) / kFusedTargets; }

size_t fused_ready_words(uint32_t n) { return static_cast<size_t>(fused_blocks(n)) * kReadyStride; }

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
    const uint64_t blocks = fused_blocks(n);
    if (fused_resident<32>(blocks, smem, sms)) {
        return 32u;
    }
    return fused_resident<16>(blocks, smem, sms) ? 16u : 0u;
}

size_t fused_scratch_floats4(uint32_t n) { return 2ull * fused_padded(n); }

cudaError_t launch_fused_steps(double *const *state, const double *m, uint32_t n,
                               uint64_t steps, int cycle, const double *h, float eps2,
                               float4 *scratch, unsigned *ready, uint32_t epoch,
                               unsigned *status, uint32_t warps, cudaStream_t stream,
                               uint32_t poll_limit, uint32_t silent_cta) {
    if (n == 0 || steps == 0) {
        return cudaSuccess;
    }
    if (warps != 16u && warps != 32u) {
        return cudaErrorInvalidValue;
    }
    if (steps * static_cast<uint64_t>(cycle) > 0x7fffffffull) {
        return cudaErrorInvalidValue; // ready words compare within 2^31 substeps
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
    g.ready = ready;
    g.status = status;
    g.n = n;
    g.cycle = static_cast<uint32_t>(cycle);
    g.epoch = epoch;
    g.poll_limit = poll_limit == 0u ? kSpinLimit : poll_limit;
    g.silent_cta = silent_cta;
    g.substeps = static_cast<uint32_t>(steps * static_cast<uint64_t>(cycle));
    for (int k = 0; k < cycle && k < 3; ++k) {
        g.h[k] = h[k];
        g.half[k] = h[k] / 2.0; // as enqueue_substep computes it
    }
    g.eps2 = eps2;
    void *args[] = {&g};
    const void *kernel = warps == 32u ? reinterpret_cast<const void *>(fused_steps_kernel<32>)
                                      : reinterpret_cast<const void *>(fused_steps_kernel<16>);
    return cudaLaunchCooperativeKernel(kernel, dim3(fused_blocks(n)), dim3(warps * 32u), args,
                                       fused_smem(g.padded), stream);
}

} // namespace ob
