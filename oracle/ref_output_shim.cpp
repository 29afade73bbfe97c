// C entry points over the reference's own checkpoint, trajectory and
// diagnostics-log code (src/sim/checkpoint.cpp, src/sim/trajectory.cpp,
// src/sim/diagnostics_log.cpp, src/sim/config_file.cpp),
// so that the tests can compare this backend's files with the reference's
// byte for byte and read each side's files with the other's reader.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile (target ref) into
// oracle/_ref/libref_orrery.so beside ref_shim.cpp. Nothing in the product
// links it.
#include <cstdint>
#include <cstring>
#include <exception>
#include <sstream>
#include <string>

#include "orrery/core/particle_data.hpp"
#include "orrery/core/vec3_array.hpp"
#include "orrery/sim/checkpoint.hpp"
#include "orrery/sim/config_file.hpp"
#include "orrery/sim/configuration.hpp"
#include "orrery/sim/diagnostics_log.hpp"
#include "orrery/sim/trajectory.hpp"

namespace {

thread_local std::string g_error;

using orrery::core::ParticleData;

// m x y z vx vy vz ax ay az into a ParticleData of n particles.
ParticleData state_of(std::size_t n, const double* const a[10]) {
    ParticleData d;
    d.resize(n);
    auto m = d.masses();
    auto p = d.positions();
    auto v = d.velocities();
    auto acc = d.accelerations();
    for (std::size_t i = 0; i < n; ++i) {
        m[i] = a[0][i];
        p.x[i] = a[1][i];
        p.y[i] = a[2][i];
        p.z[i] = a[3][i];
        v.x[i] = a[4][i];
        v.y[i] = a[5][i];
        v.z[i] = a[6][i];
        acc.x[i] = a[7][i];
        acc.y[i] = a[8][i];
        acc.z[i] = a[9][i];
    }
    return d;
}

template <typename F> int guarded(F&& body) {
    try {
        body();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

} // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

// The text sim::write_configuration gives for a default Configuration; returns
// its length and copies up to `capacity` bytes of it.
std::size_t ref_default_configuration(char* out, std::size_t capacity) {
    std::ostringstream text;
    orrery::sim::write_configuration(text, orrery::sim::Configuration{});
    const std::string s = text.str();
    if (out != nullptr) {
        std::memcpy(out, s.data(), s.size() < capacity ? s.size() : capacity);
    }
    return s.size();
}

// sim::write_checkpoint of {default configuration, step, state}.
int ref_write_checkpoint(const char* path, std::uint64_t step, std::size_t n, const double* m,
                         const double* x, const double* y, const double* z, const double* vx,
                         const double* vy, const double* vz, const double* ax, const double* ay,
                         const double* az) {
    return guarded([&] {
        const double* a[10] = {m, x, y, z, vx, vy, vz, ax, ay, az};
        orrery::sim::Checkpoint c;
        c.step = step;
        c.particles = state_of(n, a);
        orrery::sim::write_checkpoint(path, c);
    });
}

// sim::read_checkpoint: the step, the particle count, and (when `capacity` holds
// them) the ten arrays; the configuration is written back out with
// sim::write_configuration into `text` (up to `text_capacity` bytes).
int ref_read_checkpoint(const char* path, std::uint64_t* step, std::uint64_t* n,
                        std::size_t capacity, double* m, double* x, double* y, double* z,
                        double* vx, double* vy, double* vz, double* ax, double* ay, double* az,
                        char* text, std::size_t text_capacity, std::size_t* text_length) {
    return guarded([&] {
        const orrery::sim::Checkpoint c = orrery::sim::read_checkpoint(path);
        *step = c.step;
        *n = c.particles.size();
        if (c.particles.size() <= capacity) {
            double* out[10] = {m, x, y, z, vx, vy, vz, ax, ay, az};
            const auto mass = c.particles.masses();
            const auto p = c.particles.positions();
            const auto v = c.particles.velocities();
            const auto acc = c.particles.accelerations();
            for (std::size_t i = 0; i < c.particles.size(); ++i) {
                out[0][i] = mass[i];
                out[1][i] = p.x[i];
                out[2][i] = p.y[i];
                out[3][i] = p.z[i];
                out[4][i] = v.x[i];
                out[5][i] = v.y[i];
                out[6][i] = v.z[i];
                out[7][i] = acc.x[i];
                out[8][i] = acc.y[i];
                out[9][i] = acc.z[i];
            }
        }
        std::ostringstream t;
        orrery::sim::write_configuration(t, c.configuration);
        const std::string s = t.str();
        *text_length = s.size();
        if (text != nullptr) {
            std::memcpy(text, s.data(), s.size() < text_capacity ? s.size() : text_capacity);
        }
    });
}

// sim::TrajectoryWriter: the header, then `frames` frames; xyz holds each
// frame's x, y, z (3n doubles per frame), v its vx, vy, vz when written.
int ref_write_trajectory(const char* path, std::size_t n, const double* masses, double timestep,
                         int with_velocities, std::size_t frames, const std::uint64_t* steps,
                         const double* times, const double* xyz, const double* v) {
    return guarded([&] {
        orrery::sim::TrajectoryWriter w(path, std::span<const double>(masses, n), timestep,
                                        with_velocities != 0);
        ParticleData d;
        d.resize(n);
        for (std::size_t f = 0; f < frames; ++f) {
            auto p = d.positions();
            auto vel = d.velocities();
            const double* base = xyz + f * 3 * n;
            for (std::size_t i = 0; i < n; ++i) {
                p.x[i] = base[i];
                p.y[i] = base[n + i];
                p.z[i] = base[2 * n + i];
                if (with_velocities != 0) {
                    const double* vb = v + f * 3 * n;
                    vel.x[i] = vb[i];
                    vel.y[i] = vb[n + i];
                    vel.z[i] = vb[2 * n + i];
                }
            }
            w.write_frame(steps[f], times[f], d);
        }
        w.flush();
        if (!w.ok()) {
            throw std::runtime_error("the trajectory could not be written");
        }
    });
}

// sim::TrajectoryReader: header facts, and up to `capacity` frames (steps,
// times, positions and, when present, velocities as in ref_write_trajectory).
int ref_read_trajectory(const char* path, std::uint64_t* n, double* timestep,
                        int* with_velocities, std::size_t* frames, std::size_t capacity,
                        std::size_t n_capacity, double* masses, std::uint64_t* steps,
                        double* times, double* xyz, double* v) {
    return guarded([&] {
        orrery::sim::TrajectoryReader r(path);
        *n = r.info().particle_count;
        *timestep = r.info().timestep;
        *with_velocities = r.info().has_velocities ? 1 : 0;
        const std::size_t count = r.info().particle_count;
        const bool fits = count <= n_capacity;
        if (fits && masses != nullptr) {
            std::memcpy(masses, r.masses().data(), count * sizeof(double));
        }
        orrery::sim::TrajectoryFrame frame;
        std::size_t f = 0;
        while (r.read_frame(frame)) {
            if (fits && f < capacity) {
                steps[f] = frame.step;
                times[f] = frame.time;
                const auto p = frame.positions.view();
                for (std::size_t i = 0; i < count; ++i) {
                    xyz[f * 3 * count + i] = p.x[i];
                    xyz[f * 3 * count + count + i] = p.y[i];
                    xyz[f * 3 * count + 2 * count + i] = p.z[i];
                }
                if (r.info().has_velocities && v != nullptr) {
                    const auto q = frame.velocities.view();
                    for (std::size_t i = 0; i < count; ++i) {
                        v[f * 3 * count + i] = q.x[i];
                        v[f * 3 * count + count + i] = q.y[i];
                        v[f * 3 * count + 2 * count + i] = q.z[i];
                    }
                }
            }
            ++f;
        }
        *frames = f;
    });
}

// sim::DiagnosticsLog: the header row, then one row per measurement; row r is
// step[r], time[r] and the core::Diagnostics of kinetic[r], potential[r],
// linear[3r..3r+2], angular[3r..3r+2].
int ref_write_diagnostics_log(const char* path, std::size_t rows, const std::uint64_t* steps,
                              const double* times, const double* kinetic,
                              const double* potential, const double* linear,
                              const double* angular) {
    return guarded([&] {
        orrery::sim::DiagnosticsLog log(path);
        for (std::size_t r = 0; r < rows; ++r) {
            orrery::core::Diagnostics d;
            d.kinetic_energy = kinetic[r];
            d.potential_energy = potential[r];
            d.linear_momentum = {linear[3 * r], linear[3 * r + 1], linear[3 * r + 2]};
            d.angular_momentum = {angular[3 * r], angular[3 * r + 1], angular[3 * r + 2]};
            log.record(steps[r], times[r], d);
        }
        log.flush();
        if (!log.ok()) {
            throw std::runtime_error("the diagnostics log could not be written");
        }
    });
}

} // extern "C"
