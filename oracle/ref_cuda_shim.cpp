// C entry points over the reference's own CUDA solvers (CudaDirectSolver,
// CudaTreeSolver), so that the benchmark can time the reference's GPU path on
// the same device and inputs as this backend's kernels.
//
// MEASUREMENT AND TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile with
// the reference's sources, read where they lie: target ref_cuda (double
// precision) into oracle/_ref/libref_orrery_cuda.so, target ref_cuda_single
// (ORRERY_SINGLE_PRECISION, Real = float) into
// oracle/_ref/libref_orrery_cuda_single.so. Nothing in the product links it.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <memory>

#include "orrery/backend/work_stealing_executor.hpp"
#include "orrery/core/particle_data.hpp"
#include "orrery/core/softening.hpp"
#include "orrery/solvers/cuda_direct_solver.hpp"
#include "orrery/solvers/cuda_tree_solver.hpp"

namespace {

using orrery::core::ParticleData;
using orrery::core::Real;
using orrery::core::Vec3;

// The inputs are FP64; a single-precision build (Real = float) rounds them
// as its own callers would.
ParticleData make_data(std::size_t n, const double* x, const double* y, const double* z,
                       const double* m) {
    ParticleData data;
    data.reserve(n);
    for (std::size_t i = 0; i < n; ++i) {
        data.add(Vec3{static_cast<Real>(x[i]), static_cast<Real>(y[i]), static_cast<Real>(z[i])},
                 Vec3{}, static_cast<Real>(m[i]));
    }
    return data;
}

void copy_accelerations(const ParticleData& d, double* ax, double* ay, double* az) {
    const auto a = d.accelerations();
    for (std::size_t i = 0; i < d.size(); ++i) {
        ax[i] = a.x[i];
        ay[i] = a.y[i];
        az[i] = a.z[i];
    }
}

double seconds(orrery::backend::Duration d) { return std::chrono::duration<double>(d).count(); }

} // namespace

extern "C" {

// sizeof(Real) of this build: 8 (double) or 4 (single precision).
int ref_cuda_real_bytes() { return static_cast<int>(sizeof(Real)); }

// 1 when the reference's CUDA direct solver finds a usable device.
int ref_cuda_available() {
    const orrery::core::Softening softening{static_cast<Real>(0.01)};
    return orrery::solvers::CudaDirectSolver::try_create(softening) ? 1 : 0;
}

// `repeats` evaluations after one warm-up; wall seconds per evaluation (the
// solver's host-buffer evaluate: staging, transfers, kernel) and the kernel's
// own time per evaluation from its timings. Returns 0, or -1 without a device.
int ref_cuda_direct_timed(std::size_t n, const double* x, const double* y, const double* z,
                          const double* m, double softening, int repeats, double* wall,
                          double* kernel, double* ax, double* ay, double* az) {
    auto solver = orrery::solvers::CudaDirectSolver::try_create(
        orrery::core::Softening{static_cast<Real>(softening)});
    if (!solver) {
        return -1;
    }
    ParticleData data = make_data(n, x, y, z, m);
    solver->evaluate(data.positions(), data.masses(), data.accelerations());
    double kernel_total = 0.0;
    const auto start = std::chrono::steady_clock::now();
    for (int r = 0; r < repeats; ++r) {
        solver->evaluate(data.positions(), data.masses(), data.accelerations());
        kernel_total += seconds(solver->timings().kernel);
    }
    const auto stop = std::chrono::steady_clock::now();
    const int reps = std::max(repeats, 1);
    *wall = std::chrono::duration<double>(stop - start).count() / reps;
    *kernel = kernel_total / reps;
    copy_accelerations(data, ax, ay, az);
    return 0;
}

// The same for the reference's CUDA tree solver (host sort and build on
// `threads` workers, traversal on the device); counts[0..1] = pair and cell
// terms of the last evaluation.
int ref_cuda_tree_timed(std::size_t n, const double* x, const double* y, const double* z,
                        const double* m, double softening, double opening_angle,
                        std::uint64_t leaf_capacity, int quadrupole, int threads, int repeats,
                        double* wall, double* kernel, double* ax, double* ay, double* az,
                        std::uint64_t* counts) {
    orrery::solvers::TreeParameters params;
    params.opening_angle = opening_angle;
    params.leaf_capacity = leaf_capacity;
    params.quadrupole = quadrupole != 0;
    std::unique_ptr<orrery::backend::WorkStealingExecutor> executor;
    if (threads > 1) {
        executor = std::make_unique<orrery::backend::WorkStealingExecutor>(
            static_cast<unsigned>(threads));
    }
    auto solver = orrery::solvers::CudaTreeSolver::try_create(
        params, orrery::core::Softening{static_cast<Real>(softening)}, executor.get());
    if (!solver) {
        return -1;
    }
    ParticleData data = make_data(n, x, y, z, m);
    solver->evaluate(data.positions(), data.masses(), data.accelerations());
    double kernel_total = 0.0;
    solver->reset_interaction_count();
    const auto start = std::chrono::steady_clock::now();
    for (int r = 0; r < repeats; ++r) {
        solver->evaluate(data.positions(), data.masses(), data.accelerations());
        kernel_total += seconds(solver->timings().kernel);
    }
    const auto stop = std::chrono::steady_clock::now();
    const int reps = std::max(repeats, 1);
    *wall = std::chrono::duration<double>(stop - start).count() / reps;
    *kernel = kernel_total / reps;
    const auto c = solver->interaction_count();
    counts[0] = static_cast<std::uint64_t>(c.particle_particle) / reps;
    counts[1] = static_cast<std::uint64_t>(c.particle_cell) / reps;
    copy_accelerations(data, ax, ay, az);
    return 0;
}

} // extern "C"
