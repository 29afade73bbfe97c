// Integrator updates and energy terms, FP64 on the device.
//
// The updates restate kick/drift of src/integrators/velocity_verlet.cpp:20-55
// element for element. The reference's host code has no FMA, so every
// multiply and add here is an explicitly rounded intrinsic: a device step is
// bit-identical to the reference's host step given the same accelerations.
#include "common.cuh"
#include "internal.hpp"

namespace ob {
namespace {

constexpr uint32_t kThreads = 256;

uint32_t blocks_for(uint32_t n) {
    const uint32_t b = ceil_div(n, kThreads);
    return b < 148u * 8u ? (b == 0 ? 1 : b) : 148u * 8u;
}

__global__ void kick_drift_kernel(double *__restrict__ x, double *__restrict__ y,
                                  double *__restrict__ z, double *__restrict__ vx,
                                  double *__restrict__ vy, double *__restrict__ vz,
                                  const double *__restrict__ ax, const double *__restrict__ ay,
                                  const double *__restrict__ az, uint32_t n, double h,
                                  double dt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ux = __dadd_rn(vx[i], __dmul_rn(h, ax[i]));
        const double uy = __dadd_rn(vy[i], __dmul_rn(h, ay[i]));
        const double uz = __dadd_rn(vz[i], __dmul_rn(h, az[i]));
        vx[i] = ux;
        vy[i] = uy;
        vz[i] = uz;
        x[i] = __dadd_rn(x[i], __dmul_rn(dt, ux));
        y[i] = __dadd_rn(y[i], __dmul_rn(dt, uy));
        z[i] = __dadd_rn(z[i], __dmul_rn(dt, uz));
    }
}

__global__ void kick_kernel(double *__restrict__ vx, double *__restrict__ vy,
                            double *__restrict__ vz, const double *__restrict__ ax,
                            const double *__restrict__ ay, const double *__restrict__ az,
                            uint32_t n, double h) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        vx[i] = __dadd_rn(vx[i], __dmul_rn(h, ax[i]));
        vy[i] = __dadd_rn(vy[i], __dmul_rn(h, ay[i]));
        vz[i] = __dadd_rn(vz[i], __dmul_rn(h, az[i]));
    }
}

// Classical Runge-Kutta 4 (src/integrators/runge_kutta4.cpp:64-139) as three
// update kernels between the four force evaluations of a step. `save` holds
// 12n doubles: the step's start x0 (x y z), v0 (vx vy vz) and the weighted
// derivative sums Sx, Sv. Each moves the state to a stage as
// advance_to_stage does (runge_kutta4.cpp:31-40): x = x0 + s v, v = v0 + s a,
// with v and a those of the stage before.
struct Rk4State {
    double *p[3];
    double *v[3];
    const double *a[3];
    double *save;
    uint32_t n;
};

// The first stage: remember x0 and v0, seed the sums with v0 and a0 (the
// first stage's derivatives, :101-102), move to the first midpoint.
__global__ void rk4_begin_kernel(Rk4State s, double scale) {
    const uint32_t n = s.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double x = s.p[c][i], v = s.v[c][i], a = s.a[c][i];
            s.save[c * n + i] = x;
            s.save[(3 + c) * n + i] = v;
            s.save[(6 + c) * n + i] = v;
            s.save[(9 + c) * n + i] = a;
            s.p[c][i] = __dadd_rn(x, __dmul_rn(scale, v));
            s.v[c][i] = __dadd_rn(v, __dmul_rn(scale, a));
        }
    }
}

// Adds the stage just evaluated to the sums with `weight` (accumulate_component,
// :42-46), then moves to the next stage.
__global__ void rk4_next_kernel(Rk4State s, double weight, double scale) {
    const uint32_t n = s.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = s.v[c][i], a = s.a[c][i];
            s.save[(6 + c) * n + i] = __dadd_rn(s.save[(6 + c) * n + i], __dmul_rn(weight, v));
            s.save[(9 + c) * n + i] = __dadd_rn(s.save[(9 + c) * n + i], __dmul_rn(weight, a));
            s.p[c][i] = __dadd_rn(s.save[c * n + i], __dmul_rn(scale, v));
            s.v[c][i] = __dadd_rn(s.save[(3 + c) * n + i], __dmul_rn(scale, a));
        }
    }
}

// Adds the last stage, then sets x = x0 + scale Sx, v = v0 + scale Sv
// (combine_component, :48-53, with scale h/6).
__global__ void rk4_finish_kernel(Rk4State s, double weight, double scale) {
    const uint32_t n = s.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double sx = __dadd_rn(s.save[(6 + c) * n + i], __dmul_rn(weight, s.v[c][i]));
            const double sv = __dadd_rn(s.save[(9 + c) * n + i], __dmul_rn(weight, s.a[c][i]));
            s.p[c][i] = __dadd_rn(s.save[c * n + i], __dmul_rn(scale, sx));
            s.v[c][i] = __dadd_rn(s.save[(3 + c) * n + i], __dmul_rn(scale, sv));
        }
    }
}

// Per-particle kinetic terms m |v|^2 (src/core/diagnostics.cpp:118-127); the
// host sums them in index order with the reference's Neumaier summation.
__global__ void kinetic_terms_kernel(const double *__restrict__ vx, const double *__restrict__ vy,
                                     const double *__restrict__ vz, const double *__restrict__ m,
                                     uint32_t n, double *terms) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx[i], vx[i]), __dmul_rn(vy[i], vy[i])),
                                    __dmul_rn(vz[i], vz[i]));
        terms[i] = __dmul_rn(m[i], v2);
    }
}

// Per-particle potential rows -m_i sum_{j>i} m_j / sqrt(|d|^2 + eps^2) in the
// order of core::potential_energy (src/core/diagnostics.cpp:129-158).
constexpr uint32_t kPeThreads = 128;
constexpr uint32_t kPeTile = 256;

__global__ void __launch_bounds__(kPeThreads)
    potential_rows_kernel(const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, const double *__restrict__ m, uint32_t n,
                          double eps2, double *rows) {
    __shared__ double tx[kPeTile], ty[kPeTile], tz[kPeTile], tm[kPeTile];
    const uint32_t i = blockIdx.x * kPeThreads + threadIdx.x;
    const bool valid = i < n;
    const double px = valid ? x[i] : 0.0, py = valid ? y[i] : 0.0, pz = valid ? z[i] : 0.0;
    double interaction = 0.0;
    // Sources j > i only; the first tile starts at this block's first target.
    for (uint32_t base = blockIdx.x * kPeThreads; base < n; base += kPeTile) {
        for (uint32_t k = threadIdx.x; k < kPeTile; k += kPeThreads) {
            const uint32_t j = base + k;
            tx[k] = j < n ? x[j] : 0.0;
            ty[k] = j < n ? y[j] : 0.0;
            tz[k] = j < n ? z[j] : 0.0;
            tm[k] = j < n ? m[j] : 0.0;
        }
        __syncthreads();
        const uint32_t count = min(kPeTile, n - base);
        for (uint32_t k = 0; k < count; ++k) {
            if (base + k <= i) {
                continue;
            }
            const double dx = __dsub_rn(tx[k], px);
            const double dy = __dsub_rn(ty[k], py);
            const double dz = __dsub_rn(tz[k], pz);
            const double s2 =
                __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const double inv = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(s2, eps2)));
            interaction = __dadd_rn(interaction, __dmul_rn(tm[k], inv));
        }
        __syncthreads();
    }
    if (valid) {
        rows[i] = __dmul_rn(__dmul_rn(-1.0, m[i]), interaction);
    }
}

} // namespace

cudaError_t launch_kick_drift(double *x, double *y, double *z, double *vx, double *vy,
                              double *vz, const double *ax, const double *ay, const double *az,
                              uint32_t n, double h, double dt, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    kick_drift_kernel<<<blocks_for(n), kThreads, 0, stream>>>(x, y, z, vx, vy, vz, ax, ay, az, n,
                                                               h, dt);
    return cudaGetLastError();
}

cudaError_t launch_kick(double *vx, double *vy, double *vz, const double *ax, const double *ay,
                        const double *az, uint32_t n, double h, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    kick_kernel<<<blocks_for(n), kThreads, 0, stream>>>(vx, vy, vz, ax, ay, az, n, h);
    return cudaGetLastError();
}

cudaError_t launch_rk4_stage(int phase, double *const *state, double *save, uint32_t n,
                             double weight, double scale, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    const Rk4State s{{state[0], state[1], state[2]},
                     {state[3], state[4], state[5]},
                     {state[6], state[7], state[8]},
                     save,
                     n};
    if (phase == 0) {
        rk4_begin_kernel<<<blocks_for(n), kThreads, 0, stream>>>(s, scale);
    } else if (phase == 1) {
        rk4_next_kernel<<<blocks_for(n), kThreads, 0, stream>>>(s, weight, scale);
    } else {
        rk4_finish_kernel<<<blocks_for(n), kThreads, 0, stream>>>(s, weight, scale);
    }
    return cudaGetLastError();
}

uint32_t energy_partials_needed(uint32_t n) { return n; }

cudaError_t launch_kinetic_partials(const double *vx, const double *vy, const double *vz,
                                    const double *m, uint32_t n, double *partials,
                                    cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    kinetic_terms_kernel<<<blocks_for(n), kThreads, 0, stream>>>(vx, vy, vz, m, n, partials);
    return cudaGetLastError();
}

cudaError_t launch_potential_rows(const double *x, const double *y, const double *z,
                                  const double *m, uint32_t n, double eps2, double *rows,
                                  cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    potential_rows_kernel<<<ceil_div(n, kPeThreads), kPeThreads, 0, stream>>>(x, y, z, m, n,
                                                                            eps2, rows);
    return cudaGetLastError();
}

} // namespace ob
