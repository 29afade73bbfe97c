// Solver: the device side of the ForceSolver drop-in.
//
// Mirrors CudaDirectSolver / CudaTreeSolver (src/solvers/cuda_direct_solver.cpp,
// src/solvers/cuda_tree_solver.cpp) as far as the caller can see -- capacity
// kept between calls, counters, per-phase timings -- but the evaluation is a
// device-resident pipeline: the host entry point copies the FP64 SoA in, every
// phase (packing, Morton order, tree, walk or direct sum) runs on the device,
// and only the accelerations come back.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "solver.hpp"
#include "tree.hpp"

namespace ob {

ob_solver_params corrected(const ob_solver_params &in) {
    ob_solver_params p = in;
    if (p.kind != OB_SOLVER_DIRECT && p.kind != OB_SOLVER_TREE) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "unknown solver kind");
    }
    if (p.precision != OB_PRECISION_FP32 && p.precision != OB_PRECISION_SPLIT &&
        p.precision != OB_PRECISION_FP64) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "unknown precision");
    }
    if (p.kind == OB_SOLVER_TREE && p.precision == OB_PRECISION_SPLIT) {
        throw Error(OB_ERROR_UNSUPPORTED,
                    "the tree solver computes FP32 forces (precision FP32) or the reference's "
                    "FP64 forces (precision FP64)");
    }
    if (!(p.softening_squared >= 0.0) || !std::isfinite(p.softening_squared)) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "softening squared must be finite and >= 0");
    }
    // corrected_parameters: theta clamped to [0, 1], leaf capacity >= 1.
    if (!(p.opening_angle >= 0.0)) {
        p.opening_angle = 0.0;
    }
    if (p.opening_angle > 1.0) {
        p.opening_angle = 1.0;
    }
    if (p.leaf_capacity < 1) {
        p.leaf_capacity = 1;
    }
    return p;
}

unsigned read_and_clear_status(unsigned *device_word, cudaStream_t stream) {
    unsigned value = 0;
    check(cudaMemcpyAsync(&value, device_word, sizeof(unsigned), cudaMemcpyDeviceToHost, stream),
          "reading the device status word");
    check(cudaStreamSynchronize(stream), "synchronising for the status word");
    if (value != 0) {
        check(cudaMemsetAsync(device_word, 0, sizeof(unsigned), stream), "clearing status");
    }
    return value;
}

Solver::Solver(const ob_solver_params &params) : params_(corrected(params)) {
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device),
          "querying the SM count");
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "creating a stream");
    for (auto &e : events_) {
        check(cudaEventCreate(&e), "creating an event");
    }
    status_.reserve(1);
    check(cudaMemset(status_.data(), 0, sizeof(unsigned)), "clearing the status word");
    if (params_.kind == OB_SOLVER_TREE) {
        tree_ = std::make_unique<TreePipeline>(params_);
    }
}

Solver::~Solver() {
    for (auto &e : events_) {
        if (e != nullptr) {
            cudaEventDestroy(e);
        }
    }
    if (stream_ != nullptr) {
        cudaStreamDestroy(stream_);
    }
}

namespace {
// Shapes the autotuner chose, shared by every solver in the process, keyed by
// (precision, n).
std::mutex g_tuned_mutex;
std::map<std::pair<int, uint32_t>, DirectConfig> g_tuned;
} // namespace

bool tuned_shape(int precision, uint32_t n, DirectConfig &out) {
    std::lock_guard<std::mutex> lock(g_tuned_mutex);
    const auto it = g_tuned.find({precision, n});
    if (it == g_tuned.end()) {
        return false;
    }
    out = it->second;
    return true;
}

void remember_shape(int precision, uint32_t n, const DirectConfig &c) {
    std::lock_guard<std::mutex> lock(g_tuned_mutex);
    g_tuned[{precision, n}] = c;
}

DirectConfig Solver::direct_config(uint32_t n) {
    const auto it = configs_.find(n);
    if (it != configs_.end()) {
        return it->second;
    }
    DirectConfig tuned;
    if (tuned_shape(params_.precision, n, tuned)) {
        configs_[n] = tuned;
        return tuned;
    }
    const DirectConfig c =
        direct_default_config(n, params_.precision == OB_PRECISION_SPLIT, sm_count_);
    configs_[n] = c;
    return c;
}

void Solver::evaluate_direct(uint32_t n, const double *x, const double *y, const double *z,
                             const double *m, double *ax, double *ay, double *az,
                             cudaStream_t stream, cudaEvent_t ordered, cudaEvent_t built,
                             bool external) {
    const double eps2d = params_.softening_squared;
    if (params_.precision == OB_PRECISION_FP64) {
        record(ordered, stream, external);
        record(built, stream, external);
        check(launch_direct_f64(x, y, z, m, n, eps2d, ax, ay, az, stream), "FP64 direct kernel");
        return;
    }
    const bool split = params_.precision == OB_PRECISION_SPLIT;
    const DirectConfig config = direct_config(n);
    const uint32_t padded = direct_padded_count(n, config);
    if (hi_.reserve(2ull * padded)) {
        ++generation_;
    }
    if (split && lo_.reserve(2ull * padded)) {
        ++generation_;
    }
    check(pack_sources(x, y, z, m, n, padded, hi_.data(), split ? lo_.data() : nullptr, stream),
          "packing sources");
    record(ordered, stream, external);
    record(built, stream, external);
    const auto eps2 = static_cast<float>(eps2d);
    if (split) {
        check(launch_direct_split(hi_.data(), lo_.data(), n, padded, eps2, ax, ay, az, config,
                                  status_.data(), stream),
              "split-precision direct kernel");
    } else {
        check(launch_direct_f32(hi_.data(), n, padded, eps2, ax, ay, az, config, status_.data(),
                                stream),
              "FP32 direct kernel");
    }
}

double Solver::autotune(uint32_t n, DirectConfig &chosen) {
    if (params_.kind != OB_SOLVER_DIRECT || params_.precision == OB_PRECISION_FP64) {
        throw Error(OB_ERROR_UNSUPPORTED, "only the FP32 and split direct kernels have shapes");
    }
    if (n == 0) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "autotune needs at least one particle");
    }
    const bool split = params_.precision == OB_PRECISION_SPLIT;
    // Synthetic sources: a deterministic scatter in the unit cube.
    std::vector<double> host(4ull * n);
    uint64_t state = 0x9e3779b97f4a7c15ull;
    for (size_t i = 0; i < 3ull * n; ++i) {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        host[i] = static_cast<double>(state >> 11) * (1.0 / 9007199254740992.0);
    }
    for (size_t i = 3ull * n; i < 4ull * n; ++i) {
        host[i] = 1.0 / n;
    }
    DeviceArray<double> dev;
    dev.reserve(7ull * n);
    check(cudaMemcpyAsync(dev.data(), host.data(), sizeof(double) * 4ull * n,
                          cudaMemcpyHostToDevice, stream_),
          "uploading autotune sources");
    DirectConfig candidates[128];
    const int count = direct_candidates(split, candidates, 128);
    const auto eps2 = static_cast<float>(params_.softening_squared + 1e-6);
    double best = 1e300;
    const double *d = dev.data();
    double *out = dev.data() + 4ull * n;
    for (int k = 0; k < count && k < 128; ++k) {
        const DirectConfig c = candidates[k];
        if (static_cast<uint32_t>(c.split) > ceil_div(n, kDirectTile)) {
            continue;
        }
        const uint32_t padded = direct_padded_count(n, c);
        hi_.reserve(2ull * padded);
        if (split) {
            lo_.reserve(2ull * padded);
        }
        ++generation_;
        check(pack_sources(d, d + n, d + 2ull * n, d + 3ull * n, n, padded, hi_.data(),
                           split ? lo_.data() : nullptr, stream_),
              "packing autotune sources");
        auto launch = [&]() {
            return split ? launch_direct_split(hi_.data(), lo_.data(), n, padded, eps2, out,
                                               out + n, out + 2ull * n, c, status_.data(), stream_)
                         : launch_direct_f32(hi_.data(), n, padded, eps2, out, out + n,
                                             out + 2ull * n, c, status_.data(), stream_);
        };
        if (launch() != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        const int reps = 2;
        check(cudaEventRecord(events_[0], stream_), "recording an event");
        for (int r = 0; r < reps; ++r) {
            check(launch(), "autotune launch");
        }
        check(cudaEventRecord(events_[5], stream_), "recording an event");
        check(cudaEventSynchronize(events_[5]), "autotune timing");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, events_[0], events_[5]), "autotune timing");
        const double per = ms / reps;
        if (per < best) {
            best = per;
            chosen = c;
        }
    }
    check(cudaStreamSynchronize(stream_), "autotune");
    check_status(stream_);
    if (best == 1e300) {
        throw Error(OB_ERROR_CUDA, "no direct kernel shape could be launched");
    }
    configs_[n] = chosen;
    remember_shape(params_.precision, n, chosen);
    ++generation_;
    return best;
}

void Solver::account(uint64_t evaluations, uint64_t n) {
    counts_.evaluations += evaluations;
    if (params_.kind == OB_SOLVER_DIRECT) {
        counts_.particle_particle += evaluations * direct_pairs(n);
    }
}

void Solver::evaluate_device(uint32_t n, const double *x, const double *y, const double *z,
                             const double *m, double *ax, double *ay, double *az,
                             cudaStream_t stream, bool count, const cudaEvent_t *marks) {
    const bool external = marks != nullptr;
    const cudaEvent_t *e = external ? marks : &events_[1];
    record(e[0], stream, external);
    if (params_.kind == OB_SOLVER_DIRECT) {
        evaluate_direct(n, x, y, z, m, ax, ay, az, stream, e[1], e[2], external);
    } else {
        tree_->evaluate(n, x, y, z, m, ax, ay, az, status_.data(), e[1], e[2], external, stream);
    }
    record(e[3], stream, external);
    if (count) {
        account(1, n);
    }
}

void Solver::evaluate_host(uint64_t n64, const double *x, const double *y, const double *z,
                           const double *m, double *ax, double *ay, double *az) {
    if (n64 > 0xffffffffull) {
        throw Error(OB_ERROR_CAPACITY, "the B200 solvers index particles with 32 bits");
    }
    const auto n = static_cast<uint32_t>(n64);
    if (n == 0) {
        account(1, 0);
        timed_host_ = false;
        return;
    }
    staging_.reserve(7ull * n);
    double *d = staging_.data();
    const size_t bytes = sizeof(double) * n;
    for (int attempt = 0; attempt < 2; ++attempt) {
        check(cudaEventRecord(events_[0], stream_), "recording an event");
        const double *in[4] = {x, y, z, m};
        for (int k = 0; k < 4; ++k) {
            check(cudaMemcpyAsync(d + static_cast<size_t>(k) * n, in[k], bytes,
                                  cudaMemcpyHostToDevice, stream_),
                  "copying particles to the device");
        }
        evaluate_device(n, d, d + n, d + 2ull * n, d + 3ull * n, d + 4ull * n, d + 5ull * n,
                        d + 6ull * n, stream_, attempt == 0);
        double *out[3] = {ax, ay, az};
        for (int k = 0; k < 3; ++k) {
            check(cudaMemcpyAsync(out[k], d + static_cast<size_t>(4 + k) * n, bytes,
                                  cudaMemcpyDeviceToHost, stream_),
                  "copying accelerations to the host");
        }
        check(cudaEventRecord(events_[5], stream_), "recording an event");
        check(cudaStreamSynchronize(stream_), "evaluating forces");
        timed_host_ = true;
        if (!grew_after_overflow(stream_)) {
            return;
        }
    }
    throw Error(OB_ERROR_CAPACITY, "the octree outgrew its node capacity twice");
}

TreePipeline &Solver::tree() {
    if (!tree_) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "not a tree solver");
    }
    return *tree_;
}

uint64_t Solver::generation() const noexcept {
    return generation_ + (tree_ ? tree_->generation() : 0);
}

bool Solver::grew_after_overflow(cudaStream_t stream) {
    const unsigned status = read_and_clear_status(status_.data(), stream);
    if (status & kStatusTimeout) {
        throw Error(OB_ERROR_TIMEOUT, "a device-side wait ran out of its bound");
    }
    if (status & kStatusInvalid) {
        throw Error(OB_ERROR_CUDA, "a kernel met an index its data structure cannot hold");
    }
    if ((status & kStatusOverflow) && tree_) {
        const uint32_t required = tree_->meta().required;
        tree_->grow_nodes(required + required / 4 + 1024);
        return true;
    }
    if (status & kStatusOverflow) {
        throw Error(OB_ERROR_CAPACITY, "a device-side buffer bound was exceeded");
    }
    return false;
}

void Solver::check_status(cudaStream_t stream) {
    const unsigned status = read_and_clear_status(status_.data(), stream);
    if (status & kStatusTimeout) {
        throw Error(OB_ERROR_TIMEOUT, "a device-side wait ran out of its bound");
    }
    if (status & kStatusInvalid) {
        throw Error(OB_ERROR_CUDA, "a kernel met an index its data structure cannot hold");
    }
    if (status & kStatusOverflow) {
        throw Error(OB_ERROR_CAPACITY, "a device-side buffer bound was exceeded");
    }
}

ob_counts Solver::counts() {
    ob_counts c = counts_;
    if (tree_) {
        const ob_counts t = tree_->device_counts();
        c.particle_particle += t.particle_particle;
        c.particle_cell += t.particle_cell;
    }
    return c;
}

void Solver::reset_counts() {
    counts_ = ob_counts{};
    if (tree_) {
        tree_->reset_counts();
    }
}

ob_timings Solver::timings() const {
    ob_timings t{};
    auto span = [&](int a, int b) {
        float ms = 0.0f;
        if (cudaEventSynchronize(events_[b]) != cudaSuccess ||
            cudaEventElapsedTime(&ms, events_[a], events_[b]) != cudaSuccess) {
            cudaGetLastError();
            return 0.0;
        }
        return static_cast<double>(ms);
    };
    if (timed_host_) {
        t.transfer_in_ms = span(0, 1);
        t.transfer_out_ms = span(4, 5);
    }
    t.ordering_ms = span(1, 2);
    t.construction_ms = span(2, 3);
    t.traversal_ms = span(3, 4);
    return t;
}

} // namespace ob
