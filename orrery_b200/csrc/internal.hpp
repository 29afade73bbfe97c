// Internal launch interface shared by the library's translation units. Raw
// device pointers and counts only; every launcher enqueues on `stream` and
// returns the launch status without synchronising.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ob {

// Tile shape of the direct kernels: THREADS threads per CTA, R targets per
// thread, and S CTAs (one thread-block cluster) splitting the source range of
// one target tile. Chosen by the autotuner (direct_config_for).
struct DirectConfig {
    int threads = 256;
    int targets_per_thread = 4;
    int split = 1;
    int groups = 1; // thread groups of a CTA that split each tile's sources
};

// Source particles per staged shared-memory tile.
constexpr uint32_t kDirectTile = 512;

// Length the packed source arrays must be padded to for a configuration.
uint32_t direct_padded_count(uint32_t n, const DirectConfig &config);

// Packs FP64 SoA into the direct kernels' source layout, zero-padded to
// `padded` particles. FP32 form (lo == nullptr): 2 * padded float4 in `hi`,
// (x, x, y, y) and (z, z, m, m) per particle. Split form: `hi` = (x, y, z, m)
// rounded and `lo` = (x - hi, y - hi, z - hi, 0), padded float4 each.
cudaError_t pack_sources(const double *x, const double *y, const double *z, const double *m,
                         uint32_t n, uint32_t padded, float4 *hi, float4 *lo,
                         cudaStream_t stream);

// Plain FP32 direct sum. `sources` is the packed float4 array.
cudaError_t launch_direct_f32(const float4 *sources, uint32_t n, uint32_t padded, float eps2,
                              double *ax, double *ay, double *az, const DirectConfig &config,
                              unsigned *status, cudaStream_t stream);

// Whole integration steps of a small FP32-direct system in one cooperative
// launch (fused.cu): `steps` steps of `cycle` substeps with timesteps h[0..cycle)
// (velocity Verlet: 1, Yoshida-4: 3), state = x y z vx vy vz ax ay az.
// fused_steps_warps(n) gives the warps per CTA of a grid that is resident at
// once (32 or 16), or 0 when the system does not fit; the caller passes it to
// the launch. `scratch` holds fused_scratch_floats4(n) float4, zeroed once
// (the padding past n is read, never written); `ready` holds
// fused_ready_words(n) words, zeroed together with the caller's substep count
// `epoch`, which then grows by steps * cycle per launch. poll_limit (0: the
// library's limit) and silent_cta (a CTA that never publishes; ~0 for none)
// exist for tests of the bounded wait.
uint32_t fused_steps_warps(uint32_t n);
uint32_t fused_blocks(uint32_t n);
size_t fused_ready_words(uint32_t n);
size_t fused_scratch_floats4(uint32_t n);
cudaError_t launch_fused_steps(double *const *state, const double *m, uint32_t n,
                               uint64_t steps, int cycle, const double *h, float eps2,
                               float4 *scratch, unsigned *ready, uint32_t epoch,
                               unsigned *status, uint32_t warps, cudaStream_t stream,
                               uint32_t poll_limit = 0, uint32_t silent_cta = ~0u);

// Precision form: hi/lo split positions, Kahan FP32 partials, FP64 tiles.
cudaError_t launch_direct_split(const float4 *hi, const float4 *lo, uint32_t n, uint32_t padded,
                                float eps2, double *ax, double *ay, double *az,
                                const DirectConfig &config, unsigned *status,
                                cudaStream_t stream);

// FP64 direct sum in the reference scalar kernel's order (bit-identical).
cudaError_t launch_direct_f64(const double *x, const double *y, const double *z, const double *m,
                              uint32_t n, double eps2, double *ax, double *ay, double *az,
                              cudaStream_t stream);

// Candidate configurations of each direct form and the heuristic default.
int direct_candidates(bool split, DirectConfig *out, int capacity);
DirectConfig direct_default_config(uint32_t n, bool split, int sm_count);

// Integrator updates, FP64 with no contraction (bit-identical to the
// reference's host kick/drift, src/integrators/velocity_verlet.cpp:20-55).
//   kick_drift: v += h*a; x += dt*v           (first half of a VV substep)
//   kick:       v += h*a                      (second half)
cudaError_t launch_kick_drift(double *x, double *y, double *z, double *vx, double *vy,
                              double *vz, const double *ax, const double *ay, const double *az,
                              uint32_t n, double h, double dt, cudaStream_t stream);
cudaError_t launch_kick(double *vx, double *vy, double *vz, const double *ax, const double *ay,
                        const double *az, uint32_t n, double h, cudaStream_t stream);
// One of the three RK4 update kernels between force evaluations: phase 0
// starts the step and moves to the first stage, 1 accumulates a stage and moves
// to the next, 2 accumulates the last and combines. `state` = x y z vx vy vz
// ax ay az; `save` holds 12n doubles.
cudaError_t launch_rk4_stage(int phase, double *const *state, double *save, uint32_t n,
                             double weight, double scale, cudaStream_t stream);

// Energies: per-block partial sums written to `partials` (length returned by
// energy_partials_needed); the host folds them with Neumaier summation.
uint32_t energy_partials_needed(uint32_t n);
cudaError_t launch_kinetic_partials(const double *vx, const double *vy, const double *vz,
                                    const double *m, uint32_t n, double *partials,
                                    cudaStream_t stream);
cudaError_t launch_potential_rows(const double *x, const double *y, const double *z,
                                  const double *m, uint32_t n, double eps2, double *rows,
                                  cudaStream_t stream);

} // namespace ob
