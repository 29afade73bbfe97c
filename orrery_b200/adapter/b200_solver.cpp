// The B200 backend behind the reference's ForceSolver and Integrator
// interfaces; see b200_solver.hpp for the contract.
#include "b200_solver.hpp"

#include <cstring>

namespace orrery::solvers {
namespace {

[[noreturn]] void fail(int status) { throw B200Error(status, ob_last_error()); }

void check(int status) {
    if (status != OB_OK) {
        fail(status);
    }
}

ob_solver_params params_for(std::int32_t kind, B200Precision precision,
                            core::Softening softening) {
    ob_solver_params p{};
    p.kind = kind;
    p.precision = static_cast<std::int32_t>(precision);
    p.softening_squared = softening.squared(); // the stored square: FP64 parity needs it
    p.opening_angle = 0.5;
    p.leaf_capacity = 32;
    p.quadrupole = 0;
    return p;
}

} // namespace

ob_solver *B200Solver::create_handle(const ob_solver_params &params) {
    ob_solver *handle = nullptr;
    const int status = ob_solver_create(&params, &handle);
    if (status == OB_ERROR_NO_DEVICE) {
        return nullptr;
    }
    check(status);
    return handle;
}

B200Solver::~B200Solver() { ob_solver_destroy(handle_); }

void B200Solver::evaluate(core::Vec3Span<const core::Real> positions,
                          std::span<const core::Real> masses,
                          core::Vec3Span<core::Real> accelerations) {
    // The three views have the same length and order (an unchecked
    // precondition of the interface, acceleration_field.hpp:47-50); the
    // masses give the count.
    check(ob_solver_evaluate(handle_, masses.size(), positions.x.data(), positions.y.data(),
                             positions.z.data(), masses.data(), accelerations.x.data(),
                             accelerations.y.data(), accelerations.z.data()));
}

InteractionCount B200Solver::interaction_count() const noexcept {
    ob_counts c{};
    if (ob_solver_counts(handle_, &c) != OB_OK) {
        c = ob_counts{};
    }
    return InteractionCount{c.evaluations + device_steps_.evaluations,
                            c.particle_particle + device_steps_.particle_particle,
                            c.particle_cell + device_steps_.particle_cell};
}

void B200Solver::reset_interaction_count() noexcept {
    ob_solver_reset_counts(handle_);
    device_steps_ = ob_counts{};
}

void B200Solver::add_device_step_counts(const ob_counts &counts) noexcept {
    device_steps_.evaluations += counts.evaluations;
    device_steps_.particle_particle += counts.particle_particle;
    device_steps_.particle_cell += counts.particle_cell;
}

std::unique_ptr<B200DirectSolver> B200DirectSolver::try_create(core::Softening softening,
                                                               B200Precision precision) {
    const ob_solver_params p = params_for(OB_SOLVER_DIRECT, precision, softening);
    ob_solver *handle = create_handle(p);
    if (handle == nullptr) {
        return nullptr;
    }
    return std::unique_ptr<B200DirectSolver>(new B200DirectSolver(handle, p, softening));
}

std::unique_ptr<B200TreeSolver> B200TreeSolver::try_create(TreeParameters parameters,
                                                           core::Softening softening,
                                                           B200Precision precision) {
    ob_solver_params p = params_for(OB_SOLVER_TREE, precision, softening);
    p.opening_angle = parameters.opening_angle;
    p.leaf_capacity = parameters.leaf_capacity;
    p.quadrupole = parameters.quadrupole ? 1 : 0;
    ob_solver *handle = create_handle(p);
    if (handle == nullptr) {
        return nullptr;
    }
    // The library clamps the parameters as corrected_parameters does
    // (octree.cpp:189-194); report what it uses.
    ob_solver_params used{};
    check(ob_solver_get_params(handle, &used));
    parameters.opening_angle = used.opening_angle;
    parameters.leaf_capacity = used.leaf_capacity;
    parameters.quadrupole = used.quadrupole != 0;
    return std::unique_ptr<B200TreeSolver>(new B200TreeSolver(handle, used, softening, parameters));
}

} // namespace orrery::solvers

namespace orrery::integrators {

B200Integrator::~B200Integrator() {
    if (system_ != nullptr) {
        ob_system_destroy(system_);
    }
}

void B200Integrator::step(core::ParticleData &data, core::Real timestep,
                          AccelerationField &field) {
    auto *solver = dynamic_cast<solvers::B200Solver *>(&field);
    if (solver == nullptr) {
        throw std::invalid_argument(
            "B200Integrator steps on the device and needs a B200DirectSolver or B200TreeSolver "
            "as its field");
    }
    const std::uint64_t n = data.size();
    const ob_solver_params &params = solver->library_parameters();
    if (system_ == nullptr || n != system_size_ ||
        std::memcmp(&params, &system_params_, sizeof params) != 0) {
        if (system_ != nullptr) {
            ob_system_destroy(system_);
            system_ = nullptr;
        }
        solvers::check(ob_system_create(&params, n, &system_));
        system_size_ = n;
        system_params_ = params;
    }
    ob_counts before{}, after{};
    solvers::check(ob_system_counts(system_, &before));
    const auto x = data.positions();
    const auto v = data.velocities();
    const auto a = data.accelerations();
    solvers::check(ob_system_step_host(system_, static_cast<std::int32_t>(method_), timestep, 1,
                                       x.x.data(), x.y.data(), x.z.data(), v.x.data(),
                                       v.y.data(), v.z.data(), a.x.data(), a.y.data(),
                                       a.z.data(), data.masses().data()));
    solvers::check(ob_system_counts(system_, &after));
    solver->add_device_step_counts(ob_counts{after.evaluations - before.evaluations,
                                             after.particle_particle - before.particle_particle,
                                             after.particle_cell - before.particle_cell});
}

std::string_view B200Integrator::name() const noexcept {
    switch (method_) {
    case Method::velocity_verlet:
        return "velocity Verlet";
    case Method::yoshida4:
        return "Yoshida 4";
    case Method::runge_kutta4:
        return "RK4";
    }
    return "";
}

int B200Integrator::order() const noexcept { return method_ == Method::velocity_verlet ? 2 : 4; }

bool B200Integrator::is_symplectic() const noexcept { return method_ != Method::runge_kutta4; }

core::Index B200Integrator::force_evaluations_per_step() const noexcept {
    switch (method_) {
    case Method::velocity_verlet:
        return 1;
    case Method::yoshida4:
        return 3;
    case Method::runge_kutta4:
        return 4;
    }
    return 0;
}

} // namespace orrery::integrators
