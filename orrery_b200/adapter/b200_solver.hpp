#pragma once

// The B200 backend behind the reference's own C++ interfaces.
//
// B200DirectSolver and B200TreeSolver are orrery::solvers::ForceSolver
// implementations (include/orrery/solvers/force_solver.hpp:41-87) that any of
// the reference's integrators, simulations, tests or benchmarks can be handed
// in place of DirectSolver, BarnesHutSolver, CudaDirectSolver or
// CudaTreeSolver. They follow the reference's CUDA solvers' conventions:
//   - construction goes through try_create, which returns null when no usable
//     device exists (CudaDirectSolver::try_create,
//     src/solvers/cuda_direct_solver.cpp:140-164; CudaTreeSolver::try_create,
//     src/solvers/cuda_tree_solver.cpp:205-221);
//   - evaluate is synchronous on host spans and writes the accelerations;
//   - run-time failures throw B200Error, a std::runtime_error carrying the
//     library's status code, as backend::CudaError carries a cudaError_t
//     (include/orrery/backend/cuda_memory.hpp:129-143);
//   - interaction counts are the reference's: N(N-1) per direct evaluation,
//     and per-target pair and cell counts exactly as walk_tree counts them.
//
// B200Integrator is an orrery::integrators::Integrator
// (include/orrery/integrators/integrator.hpp:56-88) that advances the whole
// step -- kicks, drifts and every force evaluation -- on the device, uploading
// the ParticleData's positions, velocities, carried accelerations and masses
// and writing positions, velocities and accelerations back. Its name, order,
// symplecticity and evaluations per step are those of the reference's
// VelocityVerlet, Yoshida4 and RungeKutta4.
//
// Precision: B200Precision::fp64 makes the direct solver's forces, and the
// tree solver's, bit-identical to the reference's scalar DirectSolver /
// BarnesHutSolver in a double-precision build (Real = double, the
// reference's default, which this adapter requires). fp32 is the fast path
// (FP32 pair arithmetic on FP64 state); split is the direct precision form
// (FP32 pair arithmetic on hi/lo-split FP64 positions, <= 2e-6 per-particle
// relative error).
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <string_view>
#include <type_traits>

#include "orrery/core/particle_data.hpp"
#include "orrery/core/softening.hpp"
#include "orrery/core/types.hpp"
#include "orrery/integrators/acceleration_field.hpp"
#include "orrery/integrators/integrator.hpp"
#include "orrery/solvers/force_solver.hpp"
#include "orrery/solvers/interaction_count.hpp"
#include "orrery/solvers/octree.hpp"
#include "orrery_b200.h"

namespace orrery::integrators {
class B200Integrator;
} // namespace orrery::integrators

namespace orrery::solvers {

static_assert(std::is_same_v<core::Real, double>,
              "the B200 backend takes and returns FP64 particle data (Real = double)");

// A failure reported by the B200 library: its status code (OB_ERROR_*) and
// message (ob_last_error).
class B200Error : public std::runtime_error {
public:
    B200Error(int status, const std::string &what) : std::runtime_error(what), status_(status) {}
    [[nodiscard]] int status() const noexcept { return status_; }

private:
    int status_;
};

enum class B200Precision : std::int32_t {
    fp32 = OB_PRECISION_FP32,
    split = OB_PRECISION_SPLIT,
    fp64 = OB_PRECISION_FP64,
};

// What the direct and the tree solver share: the library handle, the
// parameters it was created with and the counts of device steps taken through
// B200Integrator (whose evaluations happen inside the device step, not in
// evaluate).
class B200Solver : public ForceSolver {
public:
    ~B200Solver() override;
    B200Solver(const B200Solver &) = delete;
    B200Solver &operator=(const B200Solver &) = delete;

    void evaluate(core::Vec3Span<const core::Real> positions, std::span<const core::Real> masses,
                  core::Vec3Span<core::Real> accelerations) override;

    [[nodiscard]] core::Softening softening() const noexcept override { return softening_; }
    [[nodiscard]] InteractionCount interaction_count() const noexcept override;
    void reset_interaction_count() noexcept override;

    [[nodiscard]] B200Precision precision() const noexcept {
        return static_cast<B200Precision>(params_.precision);
    }
    // The library handle, for callers that use the C ABI beside this class
    // (ob_solver_timings, ob_tree_copy, ...).
    [[nodiscard]] ob_solver *handle() const noexcept { return handle_; }
    [[nodiscard]] const ob_solver_params &library_parameters() const noexcept { return params_; }

protected:
    B200Solver(ob_solver *handle, const ob_solver_params &params, core::Softening softening)
        : handle_(handle), params_(params), softening_(softening) {}

    // Creates the library solver; null when no usable device exists, throws
    // B200Error on any other failure.
    static ob_solver *create_handle(const ob_solver_params &params);

private:
    friend class integrators::B200Integrator;
    void add_device_step_counts(const ob_counts &counts) noexcept;

    ob_solver *handle_;
    ob_solver_params params_;
    core::Softening softening_;
    ob_counts device_steps_{}; // evaluations made inside B200Integrator steps
};

// The direct O(N^2) sum on the device (DirectSolver's arithmetic at fp64).
class B200DirectSolver final : public B200Solver {
public:
    [[nodiscard]] static std::unique_ptr<B200DirectSolver>
    try_create(core::Softening softening = {}, B200Precision precision = B200Precision::fp32);

    [[nodiscard]] std::string_view name() const noexcept override { return "b200-direct"; }

private:
    using B200Solver::B200Solver;
};

// Barnes-Hut on the device: Morton order, octree, multipoles and the
// theta-walk, all in HBM (BarnesHutSolver's tree and decisions).
class B200TreeSolver final : public B200Solver {
public:
    [[nodiscard]] static std::unique_ptr<B200TreeSolver>
    try_create(TreeParameters parameters = {}, core::Softening softening = {},
               B200Precision precision = B200Precision::fp32);

    [[nodiscard]] std::string_view name() const noexcept override { return "b200-tree"; }
    [[nodiscard]] const TreeParameters &parameters() const noexcept { return parameters_; }

private:
    B200TreeSolver(ob_solver *handle, const ob_solver_params &params, core::Softening softening,
                   TreeParameters parameters)
        : B200Solver(handle, params, softening), parameters_(parameters) {}
    TreeParameters parameters_;
};

} // namespace orrery::solvers

namespace orrery::integrators {

// Integrator::step with the whole step on the device. The field handed to
// step must be a B200DirectSolver or B200TreeSolver: its parameters define
// the device system's evaluations (created on the first step, and again when
// the particle count or the solver changes), and the evaluations the step
// makes are added to its interaction count. Any other field is refused with
// std::invalid_argument, because this integrator evaluates no host field.
class B200Integrator final : public Integrator {
public:
    enum class Method : std::int32_t {
        velocity_verlet = OB_INTEGRATOR_VV,
        yoshida4 = OB_INTEGRATOR_YOSHIDA4,
        runge_kutta4 = OB_INTEGRATOR_RK4,
    };

    explicit B200Integrator(Method method) noexcept : method_(method) {}
    ~B200Integrator() override;
    B200Integrator(const B200Integrator &) = delete;
    B200Integrator &operator=(const B200Integrator &) = delete;

    void step(core::ParticleData &data, core::Real timestep, AccelerationField &field) override;

    // The reference integrators' own values (velocity_verlet.hpp,
    // yoshida4.hpp:48-54, runge_kutta4.hpp:52-65).
    [[nodiscard]] std::string_view name() const noexcept override;
    [[nodiscard]] int order() const noexcept override;
    [[nodiscard]] bool is_symplectic() const noexcept override;
    [[nodiscard]] core::Index force_evaluations_per_step() const noexcept override;

    [[nodiscard]] Method method() const noexcept { return method_; }

private:
    Method method_;
    ob_system *system_ = nullptr;
    std::uint64_t system_size_ = 0;
    ob_solver_params system_params_{};
};

} // namespace orrery::integrators
