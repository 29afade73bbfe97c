// C entry points that drive the reference's own integrators (VelocityVerlet,
// Yoshida4, RungeKutta4) over either the reference's CPU solvers or the B200
// ForceSolver adapters (orrery_b200/adapter/b200_solver.hpp), so that Python
// tests can hold the adapters to the reference's runs.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile (target ref_adapter)
// against the reference's headers, linked with oracle/_ref/libref_orrery.so
// (the reference's own sources) and orrery_b200/_lib/liborrery_b200.so, into
// oracle/_ref/libref_adapter.so. Nothing in the product links it.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>

#include "b200_solver.hpp"
#include "orrery/core/particle_data.hpp"
#include "orrery/integrators/runge_kutta4.hpp"
#include "orrery/integrators/velocity_verlet.hpp"
#include "orrery/integrators/yoshida4.hpp"
#include "orrery/solvers/barnes_hut_solver.hpp"
#include "orrery/solvers/direct_solver.hpp"

namespace {

using orrery::core::ParticleData;
using orrery::core::Vec3;
namespace integ = orrery::integrators;
namespace sol = orrery::solvers;

thread_local std::string g_error;

enum Field { kRefDirect = 0, kRefTree = 1, kB200Direct = 2, kB200Tree = 3 };

int fail(const std::exception &e) {
    g_error = e.what();
    if (const auto *b = dynamic_cast<const sol::B200Error *>(&e)) {
        return 100 + b->status();
    }
    return -1;
}

std::unique_ptr<integ::Integrator> reference_integrator(int method) {
    switch (method) {
    case 1:
        return std::make_unique<integ::Yoshida4>();
    case 2:
        return std::make_unique<integ::RungeKutta4>();
    default:
        return std::make_unique<integ::VelocityVerlet>();
    }
}

integ::B200Integrator::Method device_method(int method) {
    switch (method) {
    case 1:
        return integ::B200Integrator::Method::yoshida4;
    case 2:
        return integ::B200Integrator::Method::runge_kutta4;
    default:
        return integ::B200Integrator::Method::velocity_verlet;
    }
}

sol::TreeParameters tree_parameters(double theta, std::uint64_t leaf, int quadrupole) {
    sol::TreeParameters p;
    p.opening_angle = theta;
    p.leaf_capacity = leaf;
    p.quadrupole = quadrupole != 0;
    return p;
}

} // namespace

extern "C" {

const char *ra_last_error() { return g_error.c_str(); }

// 1 when the adapter's try_create gives a solver, 0 when it gives null (no
// usable device), otherwise an error code (ra_last_error has the message).
int ra_try_create(int tree, int precision) {
    try {
        const auto p = static_cast<sol::B200Precision>(precision);
        if (tree != 0) {
            return sol::B200TreeSolver::try_create({}, orrery::core::Softening{0.01}, p) ? 1 : 0;
        }
        return sol::B200DirectSolver::try_create(orrery::core::Softening{0.01}, p) ? 1 : 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// The name, order, symplecticity and evaluations per step of B200Integrator
// (adapter != 0) or of the reference's class for the same method.
int ra_integrator_traits(int adapter, int method, char *name, std::size_t capacity, int *order,
                         int *symplectic, std::uint64_t *evaluations) {
    std::unique_ptr<integ::Integrator> in =
        adapter != 0 ? std::make_unique<integ::B200Integrator>(device_method(method))
                     : reference_integrator(method);
    const std::string_view n = in->name();
    if (capacity > 0) {
        const std::size_t k = std::min(capacity - 1, n.size());
        std::memcpy(name, n.data(), k);
        name[k] = '\0';
    }
    *order = in->order();
    *symplectic = in->is_symplectic() ? 1 : 0;
    *evaluations = in->force_evaluations_per_step();
    return 0;
}

// Establishes the acceleration invariant with the chosen field
// (integrators::refresh_accelerations), then takes `steps` steps of the
// reference's integrator for `method` (0 velocity Verlet, 1 Yoshida-4, 2 RK4)
// -- or, with device_integrator != 0, of B200Integrator -- and writes the
// final state and the field's interaction count (evaluations, pairs, cells)
// and name. Fields: 0 the reference's DirectSolver, 1 its BarnesHutSolver
// (both scalar kernels, serial), 2 B200DirectSolver, 3 B200TreeSolver (at
// `precision`). Returns 0, 1 when the B200 adapter found no device, or an
// error code.
int ra_run(int field, int precision, int method, int device_integrator, double softening,
           double theta, std::uint64_t leaf, int quadrupole, std::size_t n, double *x, double *y,
           double *z, double *vx, double *vy, double *vz, double *ax, double *ay, double *az,
           const double *m, double dt, std::uint64_t steps, std::uint64_t *counts, char *name,
           std::size_t capacity) {
    try {
        ParticleData data;
        data.reserve(n);
        for (std::size_t i = 0; i < n; ++i) {
            data.add(Vec3{x[i], y[i], z[i]}, Vec3{vx[i], vy[i], vz[i]}, m[i]);
        }
        const orrery::core::Softening eps{softening};
        const auto p = static_cast<sol::B200Precision>(precision);
        std::unique_ptr<sol::ForceSolver> solver;
        switch (field) {
        case kRefDirect: {
            auto s = std::make_unique<sol::DirectSolver>(eps);
            s->select_kernel(sol::KernelKind::kScalar);
            solver = std::move(s);
            break;
        }
        case kRefTree: {
            auto s = std::make_unique<sol::BarnesHutSolver>(tree_parameters(theta, leaf,
                                                                            quadrupole),
                                                            eps);
            s->select_kernel(sol::KernelKind::kScalar);
            solver = std::move(s);
            break;
        }
        case kB200Direct:
            solver = sol::B200DirectSolver::try_create(eps, p);
            break;
        case kB200Tree:
            solver = sol::B200TreeSolver::try_create(tree_parameters(theta, leaf, quadrupole),
                                                     eps, p);
            break;
        default:
            g_error = "unknown field";
            return -1;
        }
        if (!solver) {
            return 1;
        }
        std::unique_ptr<integ::Integrator> integrator =
            device_integrator != 0
                ? std::make_unique<integ::B200Integrator>(device_method(method))
                : reference_integrator(method);
        integ::refresh_accelerations(data, *solver);
        for (std::uint64_t s = 0; s < steps; ++s) {
            integrator->step(data, dt, *solver);
        }
        const auto pos = data.positions();
        const auto vel = data.velocities();
        const auto acc = data.accelerations();
        for (std::size_t i = 0; i < n; ++i) {
            x[i] = pos.x[i];
            y[i] = pos.y[i];
            z[i] = pos.z[i];
            vx[i] = vel.x[i];
            vy[i] = vel.y[i];
            vz[i] = vel.z[i];
            ax[i] = acc.x[i];
            ay[i] = acc.y[i];
            az[i] = acc.z[i];
        }
        const sol::InteractionCount c = solver->interaction_count();
        counts[0] = c.evaluations;
        counts[1] = c.particle_particle;
        counts[2] = c.particle_cell;
        if (capacity > 0) {
            const std::string_view nm = solver->name();
            const std::size_t k = std::min(capacity - 1, nm.size());
            std::memcpy(name, nm.data(), k);
            name[k] = '\0';
        }
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

} // extern "C"
