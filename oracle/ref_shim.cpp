// C entry points over the reference's own CPU classes, so that Python tests
// can pin the oracle restatement (oracle.c) to the reference's real outputs.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile together with the
// reference's sources (read where they lie, never copied) into
// oracle/_ref/libref_orrery.so. Nothing in the product links it.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <span>
#include <vector>

#include "orrery/backend/thread_pool.hpp"
#include "orrery/backend/work_stealing_executor.hpp"
#include "orrery/core/diagnostics.hpp"
#include "orrery/core/particle_data.hpp"
#include "orrery/core/random.hpp"
#include "orrery/core/softening.hpp"
#include "orrery/initial_conditions/kepler.hpp"
#include "orrery/initial_conditions/plummer.hpp"
#include "orrery/integrators/runge_kutta4.hpp"
#include "orrery/integrators/velocity_verlet.hpp"
#include "orrery/integrators/yoshida4.hpp"
#include "orrery/solvers/barnes_hut_solver.hpp"
#include "orrery/solvers/direct_solver.hpp"
#include "orrery/solvers/morton.hpp"
#include "orrery/solvers/octree.hpp"
#include "orrery/solvers/reference_kernel.hpp"

namespace {

using orrery::core::Index;
using orrery::core::ParticleData;
using orrery::core::Real;
using orrery::core::Vec3;

ParticleData make_data(std::size_t n, const double* x, const double* y, const double* z,
                       const double* vx, const double* vy, const double* vz, const double* m) {
    ParticleData data;
    data.reserve(n);
    for (std::size_t i = 0; i < n; ++i) {
        const Vec3 v = vx == nullptr ? Vec3{} : Vec3{vx[i], vy[i], vz[i]};
        data.add(Vec3{x[i], y[i], z[i]}, v, m[i]);
    }
    return data;
}

void copy_out(const ParticleData& d, double* x, double* y, double* z, double* vx, double* vy,
              double* vz, double* ax, double* ay, double* az, double* m) {
    const auto p = d.positions();
    const auto v = d.velocities();
    const auto a = d.accelerations();
    const auto mass = d.masses();
    for (std::size_t i = 0; i < d.size(); ++i) {
        if (x != nullptr) {
            x[i] = p.x[i];
            y[i] = p.y[i];
            z[i] = p.z[i];
        }
        if (vx != nullptr) {
            vx[i] = v.x[i];
            vy[i] = v.y[i];
            vz[i] = v.z[i];
        }
        if (ax != nullptr) {
            ax[i] = a.x[i];
            ay[i] = a.y[i];
            az[i] = a.z[i];
        }
        if (m != nullptr) {
            m[i] = mass[i];
        }
    }
}

std::unique_ptr<orrery::backend::WorkStealingExecutor> executor_for(int threads) {
    if (threads <= 1) {
        return nullptr;
    }
    return std::make_unique<orrery::backend::WorkStealingExecutor>(static_cast<unsigned>(threads));
}

orrery::solvers::KernelKind kernel_for(int kernel) {
    return kernel == 1 ? orrery::solvers::KernelKind::kAvx2 : orrery::solvers::KernelKind::kScalar;
}

} // namespace

extern "C" {

unsigned ref_default_worker_count() { return orrery::backend::ThreadPool::default_worker_count(); }

int ref_plummer(std::size_t count, double total_mass, double scale_radius, std::uint64_t seed,
                double* x, double* y, double* z, double* vx, double* vy, double* vz, double* m) {
    orrery::core::RandomSource random{seed};
    orrery::initial_conditions::PlummerParameters params;
    params.count = count;
    params.total_mass = total_mass;
    params.scale_radius = scale_radius;
    const ParticleData data = orrery::initial_conditions::make_plummer_sphere(params, random);
    copy_out(data, x, y, z, vx, vy, vz, nullptr, nullptr, nullptr, m);
    return static_cast<int>(data.size() == count ? 0 : -1);
}

// make_kepler_orbit and kepler_period: the two bodies' state (2 entries per
// array) and the period. Returns -1, writing nothing, where the reference
// refuses the parameters.
int ref_kepler_orbit(double primary_mass, double secondary_mass, double semi_major_axis,
                     double eccentricity, double* x, double* y, double* z, double* vx, double* vy,
                     double* vz, double* m, double* period) {
    orrery::initial_conditions::KeplerParameters params;
    params.primary_mass = primary_mass;
    params.secondary_mass = secondary_mass;
    params.semi_major_axis = semi_major_axis;
    params.eccentricity = eccentricity;
    try {
        const ParticleData data = orrery::initial_conditions::make_kepler_orbit(params);
        copy_out(data, x, y, z, vx, vy, vz, nullptr, nullptr, nullptr, m);
        *period = orrery::initial_conditions::kepler_period(params);
    } catch (const std::exception&) {
        return -1;
    }
    return 0;
}

int ref_direct(std::size_t n, const double* x, const double* y, const double* z, const double* m,
               double softening, int kernel, int threads, double* ax, double* ay, double* az,
               std::uint64_t* pairs) {
    ParticleData data = make_data(n, x, y, z, nullptr, nullptr, nullptr, m);
    auto executor = executor_for(threads);
    orrery::solvers::DirectSolver solver =
        executor ? orrery::solvers::DirectSolver{orrery::core::Softening{softening}, *executor}
                 : orrery::solvers::DirectSolver{orrery::core::Softening{softening}};
    solver.select_kernel(kernel_for(kernel));
    solver.evaluate(data.positions(), data.masses(), data.accelerations());
    copy_out(data, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, ax, ay, az, nullptr);
    if (pairs != nullptr) {
        *pairs = solver.interaction_count().particle_particle;
    }
    return 0;
}

// Times `repeats` evaluations of one DirectSolver on one data set; returns
// seconds per evaluation through *seconds (the CPU baseline).
int ref_direct_timed(std::size_t n, const double* x, const double* y, const double* z,
                     const double* m, double softening, int kernel, int threads, int repeats,
                     double* seconds) {
    ParticleData data = make_data(n, x, y, z, nullptr, nullptr, nullptr, m);
    auto executor = executor_for(threads);
    orrery::solvers::DirectSolver solver =
        executor ? orrery::solvers::DirectSolver{orrery::core::Softening{softening}, *executor}
                 : orrery::solvers::DirectSolver{orrery::core::Softening{softening}};
    solver.select_kernel(kernel_for(kernel));
    solver.evaluate(data.positions(), data.masses(), data.accelerations());
    const auto start = orrery::backend::Clock::now();
    for (int r = 0; r < repeats; ++r) {
        solver.evaluate(data.positions(), data.masses(), data.accelerations());
    }
    const auto stop = orrery::backend::Clock::now();
    *seconds = std::chrono::duration<double>(stop - start).count() / std::max(repeats, 1);
    return 0;
}

int ref_reference_acceleration(std::size_t n, const double* x, const double* y, const double* z,
                               const double* m, std::size_t target, double softening,
                               double* out) {
    ParticleData data = make_data(n, x, y, z, nullptr, nullptr, nullptr, m);
    const auto r = orrery::solvers::reference_acceleration(data.positions(), data.masses(), target,
                                                           orrery::core::Softening{softening});
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    return 0;
}

int ref_morton(std::size_t n, const double* x, const double* y, const double* z, int threads,
               std::uint64_t* codes, std::uint64_t* indices, double* origin, double* size) {
    const std::vector<double> unit_masses(n, 1.0);
    ParticleData data = make_data(n, x, y, z, nullptr, nullptr, nullptr, unit_masses.data());
    auto executor = executor_for(threads);
    orrery::solvers::MortonOrdering ordering;
    ordering.build(data.positions(), executor.get());
    for (std::size_t i = 0; i < n; ++i) {
        codes[i] = ordering.keys()[i].code;
        indices[i] = ordering.keys()[i].index;
    }
    origin[0] = ordering.cube().origin.x;
    origin[1] = ordering.cube().origin.y;
    origin[2] = ordering.cube().origin.z;
    *size = ordering.cube().size;
    return 0;
}

std::uint64_t ref_spread_bits(std::uint32_t v) { return orrery::solvers::spread_bits(v); }

std::uint64_t ref_morton_code_grid(std::uint32_t gx, std::uint32_t gy, std::uint32_t gz) {
    return orrery::solvers::morton_code(gx, gy, gz);
}

// A tree built by a BarnesHutSolver evaluation, kept for the caller to copy.
struct RefTree {
    std::vector<orrery::solvers::TreeNode> nodes;
    std::vector<orrery::solvers::Quadrupole> quadrupoles;
    std::size_t leaves{};
    unsigned depth{};
};

// Runs BarnesHutSolver::evaluate (scalar leaves unless kernel == 1), writes the
// accelerations and counters, and returns the tree it built through *tree_out
// (free with ref_tree_free). The node layout is 5 doubles + 3 uint64 per node.
int ref_barnes_hut(std::size_t n, const double* x, const double* y, const double* z,
                   const double* m, double softening, double opening_angle,
                   std::uint64_t leaf_capacity, int quadrupole, int kernel, int threads,
                   double* ax, double* ay, double* az, std::uint64_t* counts, void** tree_out) {
    ParticleData data = make_data(n, x, y, z, nullptr, nullptr, nullptr, m);
    auto executor = executor_for(threads);
    orrery::solvers::TreeParameters params;
    params.opening_angle = opening_angle;
    params.leaf_capacity = leaf_capacity;
    params.quadrupole = quadrupole != 0;
    orrery::solvers::BarnesHutSolver solver =
        executor ? orrery::solvers::BarnesHutSolver{params, orrery::core::Softening{softening},
                                                    *executor}
                 : orrery::solvers::BarnesHutSolver{params, orrery::core::Softening{softening}};
    solver.select_kernel(kernel_for(kernel));
    solver.evaluate(data.positions(), data.masses(), data.accelerations());
    copy_out(data, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, ax, ay, az, nullptr);
    if (counts != nullptr) {
        counts[0] = solver.interaction_count().evaluations;
        counts[1] = solver.interaction_count().particle_particle;
        counts[2] = solver.interaction_count().particle_cell;
    }
    if (tree_out != nullptr) {
        auto* t = new RefTree;
        t->nodes.assign(solver.tree().nodes().begin(), solver.tree().nodes().end());
        t->quadrupoles.assign(solver.tree().quadrupoles().begin(),
                              solver.tree().quadrupoles().end());
        t->leaves = solver.tree().leaf_count();
        t->depth = solver.tree().depth();
        *tree_out = t;
    }
    return 0;
}

// Seconds per BarnesHutSolver evaluation over `repeats` evaluations.
int ref_barnes_hut_timed(std::size_t n, const double* x, const double* y, const double* z,
                         const double* m, double softening, double opening_angle,
                         std::uint64_t leaf_capacity, int quadrupole, int threads, int repeats,
                         double* seconds) {
    ParticleData data = make_data(n, x, y, z, nullptr, nullptr, nullptr, m);
    auto executor = executor_for(threads);
    orrery::solvers::TreeParameters params;
    params.opening_angle = opening_angle;
    params.leaf_capacity = leaf_capacity;
    params.quadrupole = quadrupole != 0;
    orrery::solvers::BarnesHutSolver solver =
        executor ? orrery::solvers::BarnesHutSolver{params, orrery::core::Softening{softening},
                                                    *executor}
                 : orrery::solvers::BarnesHutSolver{params, orrery::core::Softening{softening}};
    const auto start = orrery::backend::Clock::now();
    for (int r = 0; r < repeats; ++r) {
        solver.evaluate(data.positions(), data.masses(), data.accelerations());
    }
    const auto stop = orrery::backend::Clock::now();
    *seconds = std::chrono::duration<double>(stop - start).count() / std::max(repeats, 1);
    return 0;
}

std::size_t ref_tree_node_count(void* tree) { return static_cast<RefTree*>(tree)->nodes.size(); }
std::size_t ref_tree_leaf_count(void* tree) { return static_cast<RefTree*>(tree)->leaves; }
unsigned ref_tree_depth(void* tree) { return static_cast<RefTree*>(tree)->depth; }

void ref_tree_copy(void* tree, double* reals, std::uint64_t* indices, double* quads) {
    const auto* t = static_cast<RefTree*>(tree);
    for (std::size_t i = 0; i < t->nodes.size(); ++i) {
        const auto& node = t->nodes[i];
        reals[5 * i + 0] = node.mass;
        reals[5 * i + 1] = node.centre_of_mass.x;
        reals[5 * i + 2] = node.centre_of_mass.y;
        reals[5 * i + 3] = node.centre_of_mass.z;
        reals[5 * i + 4] = node.acceptance_radius_squared;
        indices[3 * i + 0] = node.next;
        indices[3 * i + 1] = node.first_particle;
        indices[3 * i + 2] = node.particle_count;
    }
    if (quads != nullptr) {
        for (std::size_t i = 0; i < t->quadrupoles.size(); ++i) {
            const auto& q = t->quadrupoles[i];
            quads[6 * i + 0] = q.xx;
            quads[6 * i + 1] = q.xy;
            quads[6 * i + 2] = q.xz;
            quads[6 * i + 3] = q.yy;
            quads[6 * i + 4] = q.yz;
            quads[6 * i + 5] = q.zz;
        }
    }
}

void ref_tree_free(void* tree) { delete static_cast<RefTree*>(tree); }

// Integrates `steps` steps of velocity Verlet (integrator 0) or Yoshida-4
// (integrator 1) with a scalar DirectSolver, starting from the given state and
// accelerations, in place.
int ref_integrate_direct(std::size_t n, double* x, double* y, double* z, double* vx, double* vy,
                         double* vz, double* ax, double* ay, double* az, const double* m,
                         double softening, double dt, std::uint64_t steps, int integrator,
                         int kernel) {
    ParticleData data = make_data(n, x, y, z, vx, vy, vz, m);
    const auto acc = data.accelerations();
    for (std::size_t i = 0; i < n; ++i) {
        acc.x[i] = ax[i];
        acc.y[i] = ay[i];
        acc.z[i] = az[i];
    }
    orrery::solvers::DirectSolver solver{orrery::core::Softening{softening}};
    solver.select_kernel(kernel_for(kernel));
    orrery::integrators::VelocityVerlet vv;
    orrery::integrators::Yoshida4 y4;
    orrery::integrators::RungeKutta4 rk4;
    orrery::integrators::Integrator& chosen =
        integrator == 1   ? static_cast<orrery::integrators::Integrator&>(y4)
        : integrator == 2 ? static_cast<orrery::integrators::Integrator&>(rk4)
                          : vv;
    for (std::uint64_t s = 0; s < steps; ++s) {
        chosen.step(data, dt, solver);
    }
    copy_out(data, x, y, z, vx, vy, vz, ax, ay, az, nullptr);
    return 0;
}

double ref_potential_energy(std::size_t n, const double* x, const double* y, const double* z,
                            const double* m, double softening) {
    ParticleData data = make_data(n, x, y, z, nullptr, nullptr, nullptr, m);
    return orrery::core::potential_energy(data.positions(), data.masses(),
                                          orrery::core::Softening{softening});
}

// core::measure_diagnostics: kinetic, potential, linear momentum (3), angular
// momentum (3) into out[8].
int ref_diagnostics(std::size_t n, const double* x, const double* y, const double* z,
                    const double* vx, const double* vy, const double* vz, const double* m,
                    double softening, double* out) {
    ParticleData data = make_data(n, x, y, z, vx, vy, vz, m);
    const orrery::core::Diagnostics d =
        orrery::core::measure_diagnostics(data, orrery::core::Softening{softening});
    out[0] = d.kinetic_energy;
    out[1] = d.potential_energy;
    out[2] = d.linear_momentum.x;
    out[3] = d.linear_momentum.y;
    out[4] = d.linear_momentum.z;
    out[5] = d.angular_momentum.x;
    out[6] = d.angular_momentum.y;
    out[7] = d.angular_momentum.z;
    return 0;
}

double ref_kinetic_energy(std::size_t n, const double* vx, const double* vy, const double* vz,
                          const double* m) {
    ParticleData data = make_data(n, vx, vy, vz, nullptr, nullptr, nullptr, m);
    return orrery::core::kinetic_energy(data.positions(), data.masses());
}

} // extern "C"
