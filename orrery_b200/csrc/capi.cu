// The extern "C" boundary (include/orrery_b200.h) and the device-resident
// system that integrates on the GPU.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "orrery_b200.h"
#include "solver.hpp"
#include "batch.hpp"
#include "output.hpp"
#include "system.hpp"
#include "tree.hpp"
#include "tree_kernels.hpp"

namespace ob {

namespace {
thread_local std::string g_last_error;

template <typename F> int guarded(F &&body) {
    try {
        body();
        return OB_OK;
    } catch (const Error &e) {
        return set_error(e.code(), e.what());
    } catch (const std::bad_alloc &) {
        return set_error(OB_ERROR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception &e) {
        return set_error(OB_ERROR_INVALID_ARGUMENT, e.what());
    }
}

// The try_create contract: OB_ERROR_NO_DEVICE when there is no usable
// Blackwell device (src/solvers/cuda_direct_solver.cpp:140-164).
void require_device() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error(OB_ERROR_NO_DEVICE, "no CUDA device is visible");
    }
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    int major = 0;
    check(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device),
          "querying the compute capability");
    if (major != 10) {
        throw Error(OB_ERROR_NO_DEVICE, "the device is not an sm_100 (Blackwell) GPU");
    }
}

void require(bool condition, const char *message) {
    if (!condition) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, message);
    }
}
} // namespace

int set_error(int code, const std::string &message) {
    g_last_error = message;
    return code;
}

// --------------------------------------------------------------------------
// System
// --------------------------------------------------------------------------

System::System(const ob_solver_params &params, uint32_t n, cudaStream_t stream)
    : solver_(std::make_unique<Solver>(params)), n_(n) {
    state_.reserve(10ull * (n == 0 ? 1 : n));
    check(cudaMemset(state_.data(), 0, state_.bytes()), "clearing state");
    if (stream != nullptr) {
        stream_ = stream;
        owns_stream_ = false;
    } else {
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "creating a stream");
    }
}

System::~System() {
    drop_graph();
    for (auto e : marks_) {
        cudaEventDestroy(e);
    }
    if (copy_stream_ != nullptr) {
        cudaStreamDestroy(copy_stream_);
        cudaEventDestroy(drifted_);
    }
    for (auto e : ring_) {
        cudaEventDestroy(e);
    }
    for (auto &pair : fused_marks_) {
        cudaEventDestroy(pair.first);
        cudaEventDestroy(pair.second);
    }
    if (stream_ != nullptr && owns_stream_) {
        cudaStreamDestroy(stream_);
    }
}

void System::drop_graph() {
    if (graph_ != nullptr) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    if (marked_graph_ != nullptr) {
        cudaGraphExecDestroy(marked_graph_);
        marked_graph_ = nullptr;
    }
    if (marked_template_ != nullptr) {
        cudaGraphDestroy(marked_template_);
        marked_template_ = nullptr;
    }
    mark_nodes_.clear();
}

void System::upload(int first, int count, const double *const *host) {
    for (int k = 0; k < count; ++k) {
        double *dst = array(first + k);
        if (host[k] == nullptr) {
            check(cudaMemsetAsync(dst, 0, sizeof(double) * n_, stream_), "clearing an array");
        } else {
            check(cudaMemcpyAsync(dst, host[k], sizeof(double) * n_, cudaMemcpyHostToDevice,
                                  stream_),
                  "uploading state");
        }
    }
}

void System::set_state(const double *x, const double *y, const double *z, const double *vx,
                       const double *vy, const double *vz, const double *m) {
    require(n_ == 0 || (x && y && z && m), "positions and masses are required");
    const double *in[7] = {x, y, z, vx, vy, vz, nullptr};
    upload(kX, 6, in);
    upload(kM, 1, &m);
    refresh();
}

void System::set_accelerations(const double *ax, const double *ay, const double *az) {
    const double *in[3] = {ax, ay, az};
    upload(kAx, 3, in);
    check(cudaStreamSynchronize(stream_), "uploading accelerations");
}

void System::refresh() {
    for (int attempt = 0; attempt < 2; ++attempt) {
        evaluate(attempt == 0);
        check(cudaStreamSynchronize(stream_), "evaluating accelerations");
        if (!solver_->grew_after_overflow(stream_)) {
            return;
        }
    }
    throw Error(OB_ERROR_CAPACITY, "the octree outgrew its node capacity twice");
}

void System::evaluate(bool count, const cudaEvent_t *marks) {
    solver_->evaluate_device(n_, array(kX), array(kY), array(kZ), array(kM), array(kAx),
                             array(kAy), array(kAz), stream_, count, marks);
}

namespace {
// Checkpoint order (m x y z vx vy vz ax ay az) as System arrays.
constexpr int kCheckpointOrder[10] = {System::kM,  System::kX,  System::kY,  System::kZ,
                                      System::kVx, System::kVy, System::kVz, System::kAx,
                                      System::kAy, System::kAz};
} // namespace

void System::snapshot(double *const *arrays) {
    check(cudaStreamSynchronize(stream_), "finishing the steps before a snapshot");
    for (int k = 0; k < 10 && n_ > 0; ++k) {
        check(cudaMemcpyAsync(arrays[k], array(kCheckpointOrder[k]), sizeof(double) * n_,
                              cudaMemcpyDeviceToHost, stream_),
              "downloading state");
    }
    check(cudaStreamSynchronize(stream_), "downloading state");
}

void System::restore(const double *const *arrays) {
    for (int k = 0; k < 10 && n_ > 0; ++k) {
        check(cudaMemcpyAsync(array(kCheckpointOrder[k]), arrays[k], sizeof(double) * n_,
                              cudaMemcpyHostToDevice, stream_),
              "uploading state");
    }
    check(cudaStreamSynchronize(stream_), "uploading state");
}

void System::get_state(double *const *out) {
    for (int k = 0; k < 9; ++k) {
        if (out[k] != nullptr && n_ > 0) {
            check(cudaMemcpyAsync(out[k], array(k), sizeof(double) * n_, cudaMemcpyDeviceToHost,
                                  stream_),
                  "downloading state");
        }
    }
    check(cudaStreamSynchronize(stream_), "downloading state");
}

// Yoshida-4 substep weights, computed as src/integrators/yoshida4.cpp:24-30.
static void yoshida_weights(double &outer, double &inner) {
    constexpr double cube_root_of_two = 1.2599210498948731647672106;
    outer = 1.0 / (2.0 - cube_root_of_two);
    inner = -cube_root_of_two / (2.0 - cube_root_of_two);
}

int System::evaluations_per_step(int integrator) {
    return integrator == OB_INTEGRATOR_YOSHIDA4 ? 3 : integrator == OB_INTEGRATOR_RK4 ? 4 : 1;
}

void System::enqueue_rk4_step(double dt, const cudaEvent_t *marks, cudaEvent_t drifted) {
    // RungeKutta4::step (src/integrators/runge_kutta4.cpp:64-139): stages at
    // h/2, h/2 and h weighted 2, 2, 1 after the first, the h/6 combination, and
    // the evaluation that leaves the carried accelerations at the final state.
    double *state[9];
    for (int k = 0; k < 9; ++k) {
        state[k] = array(kX + k);
    }
    double *save = rk4_.data();
    const double half = dt / 2.0;
    const double sixth = dt / 6.0;
    auto mark = [&](int e) { return marks != nullptr ? marks + 4 * e : nullptr; };
    check(launch_rk4_stage(0, state, save, n_, 0.0, half, stream_), "RK4 first stage");
    evaluate(false, mark(0));
    check(launch_rk4_stage(1, state, save, n_, 2.0, half, stream_), "RK4 second stage");
    evaluate(false, mark(1));
    check(launch_rk4_stage(1, state, save, n_, 2.0, dt, stream_), "RK4 third stage");
    evaluate(false, mark(2));
    check(launch_rk4_stage(2, state, save, n_, 1.0, sixth, stream_), "RK4 combination");
    if (drifted != nullptr) {
        check(cudaEventRecord(drifted, stream_), "recording the final positions");
    }
    evaluate(false, mark(3));
}

void System::enqueue_substep(double timestep, const cudaEvent_t *marks, cudaEvent_t drifted) {
    // velocity_verlet_step (src/integrators/velocity_verlet.cpp:59-72).
    const double half = timestep / 2.0;
    check(launch_kick_drift(array(kX), array(kY), array(kZ), array(kVx), array(kVy), array(kVz),
                            array(kAx), array(kAy), array(kAz), n_, half, timestep, stream_),
          "kick and drift");
    if (drifted != nullptr) {
        check(cudaEventRecord(drifted, stream_), "recording the final positions");
    }
    evaluate(false, marks);
    check(launch_kick(array(kVx), array(kVy), array(kVz), array(kAx), array(kAy), array(kAz), n_,
                      half, stream_),
          "kick");
}

void System::enqueue_step(int integrator, double dt, bool marked, cudaEvent_t drifted) {
    // Without marks the solver records its own events, which a capture turns
    // into ordering only (no graph nodes).
    const cudaEvent_t *m = marked ? marks_.data() : nullptr;
    if (integrator == OB_INTEGRATOR_YOSHIDA4) {
        double outer = 0.0, inner = 0.0;
        yoshida_weights(outer, inner);
        enqueue_substep(outer * dt, m);
        enqueue_substep(inner * dt, marked ? m + 4 : nullptr);
        enqueue_substep(outer * dt, marked ? m + 8 : nullptr, drifted);
    } else if (integrator == OB_INTEGRATOR_RK4) {
        enqueue_rk4_step(dt, m, drifted);
    } else {
        enqueue_substep(dt, m, drifted);
    }
}

cudaGraph_t System::capture_step(int integrator, double dt, bool marked) {
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed),
          "beginning graph capture");
    try {
        enqueue_step(integrator, dt, marked);
    } catch (...) {
        cudaStreamEndCapture(stream_, &graph);
        if (graph != nullptr) {
            cudaGraphDestroy(graph);
        }
        throw;
    }
    check(cudaStreamEndCapture(stream_, &graph), "ending graph capture");
    return graph;
}

void System::ensure_graph(int integrator, double dt) {
    if (graph_ != nullptr && graph_integrator_ == integrator && graph_dt_ == dt &&
        graph_generation_ == solver_->generation()) {
        return;
    }
    drop_graph();
    if (integrator == OB_INTEGRATOR_RK4) {
        rk4_.reserve(12ull * (n_ == 0 ? 1 : n_)); // before the capture: no allocation inside it
    }
    cudaGraph_t graph = capture_step(integrator, dt, false);
    size_t count = 0;
    cudaError_t err = cudaGraphGetNodes(graph, nullptr, &count);
    std::vector<cudaGraphNode_t> nodes(count);
    if (err == cudaSuccess) {
        err = cudaGraphGetNodes(graph, nodes.data(), &count);
    }
    graph_kernels_ = 0;
    for (size_t k = 0; err == cudaSuccess && k < count; ++k) {
        cudaGraphNodeType type;
        err = cudaGraphNodeGetType(nodes[k], &type);
        graph_kernels_ += err == cudaSuccess && type == cudaGraphNodeTypeKernel ? 1u : 0u;
    }
    if (err == cudaSuccess) {
        err = cudaGraphInstantiate(&graph_, graph, 0);
    }
    cudaGraphDestroy(graph);
    check(err, "instantiating the step graph");
    graph_integrator_ = integrator;
    graph_dt_ = dt;
    graph_generation_ = solver_->generation();
}

void System::ensure_marked_graph() {
    if (marked_graph_ != nullptr) {
        return;
    }
    const size_t needed = 4u * static_cast<size_t>(evaluations_per_step(graph_integrator_));
    while (marks_.size() < needed) {
        cudaEvent_t e = nullptr;
        check(cudaEventCreate(&e), "creating an event");
        marks_.push_back(e);
    }
    cudaGraph_t graph = capture_step(graph_integrator_, graph_dt_, true);
    marked_template_ = graph;
    check(cudaGraphInstantiate(&marked_graph_, graph, 0), "instantiating the profiled step graph");
    // Find the event-record node of each placeholder.
    size_t count = 0;
    check(cudaGraphGetNodes(graph, nullptr, &count), "listing graph nodes");
    std::vector<cudaGraphNode_t> nodes(count);
    check(cudaGraphGetNodes(graph, nodes.data(), &count), "listing graph nodes");
    mark_nodes_.assign(needed, nullptr);
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        check(cudaGraphNodeGetType(node, &type), "reading a node type");
        if (type == cudaGraphNodeTypeEventRecord) {
            cudaEvent_t e = nullptr;
            check(cudaGraphEventRecordNodeGetEvent(node, &e), "reading an event node");
            for (size_t k = 0; k < needed; ++k) {
                if (marks_[k] == e) {
                    mark_nodes_[k] = node;
                }
            }
        }
    }
}

void System::set_marks(const std::vector<cudaEvent_t> &events, size_t offset) {
    for (size_t k = 0; k < mark_nodes_.size(); ++k) {
        if (mark_nodes_[k] != nullptr) {
            check(cudaGraphExecEventRecordNodeSetEvent(marked_graph_, mark_nodes_[k],
                                                       events[offset + k]),
                  "retargeting an event node");
        }
    }
}

void System::profile(uint32_t steps) {
    synchronize();
    for (auto e : ring_) {
        cudaEventDestroy(e);
    }
    ring_.clear();
    for (auto &pair : fused_marks_) {
        cudaEventDestroy(pair.first);
        cudaEventDestroy(pair.second);
    }
    fused_marks_.clear();
    fused_mark_evals_.clear();
    ring_steps_ = steps;
    ring_used_ = 0;
    const size_t per_step = kMarksPerStep;
    ring_.resize(per_step * steps, nullptr);
    for (auto &e : ring_) {
        check(cudaEventCreate(&e), "creating an event");
    }
}

ob_timings System::phase_times(uint32_t &evaluations) {
    synchronize();
    ob_timings t{};
    evaluations = 0;
    const size_t per_eval_marks = 4;
    const size_t evals = mark_nodes_.size() / per_eval_marks;
    for (uint32_t s = 0; s < ring_used_; ++s) {
        for (size_t e = 0; e < evals; ++e) {
            const cudaEvent_t *m = &ring_[s * kMarksPerStep + e * 4];
            float a = 0, b = 0, c = 0;
            check(cudaEventElapsedTime(&a, m[0], m[1]), "phase timing");
            check(cudaEventElapsedTime(&b, m[1], m[2]), "phase timing");
            check(cudaEventElapsedTime(&c, m[2], m[3]), "phase timing");
            t.ordering_ms += a;
            t.construction_ms += b;
            t.traversal_ms += c;
            ++evaluations;
        }
    }
    // Fused launches: the whole launch counts as force evaluation time (its
    // kicks and drifts are a few microseconds of it), per evaluation.
    for (size_t k = 0; k < fused_marks_.size(); ++k) {
        float ms = 0;
        check(cudaEventElapsedTime(&ms, fused_marks_[k].first, fused_marks_[k].second),
              "phase timing");
        t.traversal_ms += ms;
        evaluations += static_cast<uint32_t>(fused_mark_evals_[k]);
    }
    if (evaluations > 0) {
        t.ordering_ms /= evaluations;
        t.construction_ms /= evaluations;
        t.traversal_ms /= evaluations;
    }
    return t;
}

bool System::set_fused_steps(bool enable) {
    fused_enabled_ = enable;
    return fused_for(OB_INTEGRATOR_VV);
}

bool System::arm_fused_timeout(uint32_t poll_limit) {
    if (!fused_for(OB_INTEGRATOR_VV)) {
        return false;
    }
    fused_test_polls_ = poll_limit;
    return true;
}

bool System::fused_for(int integrator) {
    const ob_solver_params &p = solver_->params();
    if (!fused_enabled_ || (integrator != OB_INTEGRATOR_VV && integrator != OB_INTEGRATOR_YOSHIDA4) ||
        p.kind != OB_SOLVER_DIRECT || p.precision != OB_PRECISION_FP32 ||
        !(p.softening_squared > 0.0) || !(static_cast<float>(p.softening_squared) > 0.0f)) {
        return false;
    }
    if (fused_warps_ < 0) {
        fused_warps_ = static_cast<int>(fused_steps_warps(n_));
        cudaGetLastError();
    }
    return fused_warps_ > 0;
}

uint32_t System::step_kernels(int integrator, double dt) {
    require(integrator == OB_INTEGRATOR_VV || integrator == OB_INTEGRATOR_YOSHIDA4 ||
                integrator == OB_INTEGRATOR_RK4,
            "unknown integrator");
    if (fused_for(integrator)) {
        return 1; // one launch per call, whatever the number of steps
    }
    ensure_graph(integrator, dt);
    return graph_kernels_;
}

void System::step_async(int integrator, double dt, uint64_t steps) {
    require(integrator == OB_INTEGRATOR_VV || integrator == OB_INTEGRATOR_YOSHIDA4 ||
                integrator == OB_INTEGRATOR_RK4,
            "unknown integrator");
    require(std::isfinite(dt), "the timestep must be finite");
    if (steps == 0 || n_ == 0) {
        solver_->account(steps * evaluations_per_step(integrator), n_);
        return;
    }
    if (fused_for(integrator)) {
        if (fused_buf_.size() == 0) {
            fused_buf_.reserve(fused_scratch_floats4(n_));
            // The padding past N is copied as it is and never written.
            check(cudaMemsetAsync(fused_buf_.data(), 0, fused_buf_.bytes(), stream_),
                  "clearing the fused source buffers");
            fused_ready_.reserve(fused_ready_words(n_));
            fused_ready_reset_ = true;
        }
        if (fused_ready_reset_) {
            check(cudaMemsetAsync(fused_ready_.data(), 0,
                                  fused_ready_words(n_) * sizeof(unsigned), stream_),
                  "clearing the ready words");
            fused_epoch_ = 0;
            fused_ready_reset_ = false;
        }
        double h[3] = {dt, dt, dt};
        int cycle = 1;
        if (integrator == OB_INTEGRATOR_YOSHIDA4) {
            double outer = 0.0, inner = 0.0;
            yoshida_weights(outer, inner);
            h[0] = outer * dt;
            h[1] = inner * dt;
            h[2] = outer * dt;
            cycle = 3;
        }
        double *state[9];
        for (int k = 0; k < 9; ++k) {
            state[k] = array(kX + k);
        }
        const bool timed = fused_marks_.size() < ring_steps_;
        std::pair<cudaEvent_t, cudaEvent_t> marks{nullptr, nullptr};
        if (timed) {
            check(cudaEventCreate(&marks.first), "creating an event");
            check(cudaEventCreate(&marks.second), "creating an event");
            fused_marks_.push_back(marks);
            fused_mark_evals_.push_back(steps * static_cast<uint64_t>(cycle));
            check(cudaEventRecord(marks.first, stream_), "timing the fused steps");
        }
        // At most 2^30 substeps per launch (ready words compare within 2^31).
        const uint64_t per_launch = (uint64_t{1} << 30) / static_cast<uint64_t>(cycle);
        for (uint64_t left = steps; left > 0;) {
            const uint64_t chunk = std::min(left, per_launch);
            const uint32_t polls = fused_test_polls_;
            fused_test_polls_ = 0;
            check(launch_fused_steps(state, array(kM), n_, chunk, cycle, h,
                                     static_cast<float>(solver_->params().softening_squared),
                                     fused_buf_.data(), fused_ready_.data(), fused_epoch_,
                                     solver_->status_word(),
                                     static_cast<uint32_t>(fused_warps_), stream_, polls,
                                     polls != 0 ? 0u : ~0u),
                  "fused integration steps");
            fused_epoch_ += static_cast<uint32_t>(chunk * static_cast<uint64_t>(cycle));
            left -= chunk;
        }
        if (timed) {
            check(cudaEventRecord(marks.second, stream_), "timing the fused steps");
        }
        solver_->account(steps * evaluations_per_step(integrator), n_);
        return;
    }
    ensure_graph(integrator, dt);
    for (uint64_t s = 0; s < steps; ++s) {
        if (ring_used_ < ring_steps_) {
            ensure_marked_graph();
            set_marks(ring_, static_cast<size_t>(ring_used_) * kMarksPerStep);
            ++ring_used_;
            check(cudaGraphLaunch(marked_graph_, stream_), "launching the profiled step graph");
        } else {
            check(cudaGraphLaunch(graph_, stream_), "launching the step graph");
        }
    }
    solver_->account(steps * evaluations_per_step(integrator), n_);
}

void System::step_host(int integrator, double dt, uint64_t steps, double *const *io,
                       const double *m) {
    for (int k = 0; k < 9; ++k) {
        require(n_ == 0 || io[k] != nullptr, "every state array is required");
    }
    require(n_ == 0 || m != nullptr, "masses are required");
    const double *in[9] = {io[0], io[1], io[2], io[3], io[4], io[5], io[6], io[7], io[8]};
    upload(kX, 9, in);
    upload(kM, 1, &m);
    if (steps == 0 || n_ == 0 || fused_for(integrator)) {
        step_async(integrator, dt, steps);
        get_state(io);
        synchronize();
        return;
    }
    // All but the last step replay the step graph; the last is enqueued
    // directly with an event once its positions are final, so that their
    // download overlaps its force evaluation (same kernels, same order).
    step_async(integrator, dt, steps - 1);
    ensure_graph(integrator, dt); // checks the integrator, reserves RK4's area
    if (copy_stream_ == nullptr) {
        check(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking), "a copy stream");
        check(cudaEventCreateWithFlags(&drifted_, cudaEventDisableTiming), "an event");
    }
    enqueue_step(integrator, dt, false, drifted_);
    solver_->account(evaluations_per_step(integrator), n_);
    check(cudaStreamWaitEvent(copy_stream_, drifted_, 0), "ordering the position download");
    for (int k = 0; k < 3; ++k) {
        check(cudaMemcpyAsync(io[k], array(kX + k), sizeof(double) * n_, cudaMemcpyDeviceToHost,
                              copy_stream_),
              "downloading positions");
    }
    for (int k = 3; k < 9; ++k) {
        check(cudaMemcpyAsync(io[k], array(kX + k), sizeof(double) * n_, cudaMemcpyDeviceToHost,
                              stream_),
              "downloading state");
    }
    check(cudaStreamSynchronize(copy_stream_), "downloading positions");
    synchronize();
}

void System::synchronize() {
    check(cudaStreamSynchronize(stream_), "integrating");
    try {
        solver_->check_status(stream_);
    } catch (const Error &) {
        // A fused launch that gave up waiting may have left the ready words
        // short of the host's substep count: clear both before the next one.
        fused_ready_reset_ = true;
        throw;
    }
}

// Neumaier summation in index order, as core::CompensatedSum
// (src/core/diagnostics.cpp:36-59).
static double compensated_sum(const std::vector<double> &terms) {
    double total = 0.0, correction = 0.0;
    for (const double term : terms) {
        const double updated = total + term;
        if (std::fabs(total) >= std::fabs(term)) {
            correction += (total - updated) + term;
        } else {
            correction += (term - updated) + total;
        }
        total = updated;
    }
    return total + correction;
}

// core::measure_diagnostics (src/core/diagnostics.cpp:179-200): the energies
// as System::energy computes them (device terms, compensated host sums), and
// the linear and angular momentum as compensated sums of v m and (x cross v) m
// in index order, one Neumaier sum per component, over the downloaded state.
ob_diagnostics System::diagnostics() {
    ob_diagnostics d{};
    energy(&d.kinetic_energy, &d.potential_energy);
    if (n_ == 0) {
        return d;
    }
    std::vector<double> host(7ull * n_);
    const int arrays[7] = {kX, kY, kZ, kVx, kVy, kVz, kM};
    for (int k = 0; k < 7; ++k) {
        check(cudaMemcpyAsync(host.data() + k * n_, array(arrays[k]), sizeof(double) * n_,
                              cudaMemcpyDeviceToHost, stream_),
              "downloading state");
    }
    check(cudaStreamSynchronize(stream_), "downloading state");
    const double *x = host.data(), *y = x + n_, *z = y + n_;
    const double *vx = z + n_, *vy = vx + n_, *vz = vy + n_, *m = vz + n_;
    std::vector<double> terms[6];
    for (auto &t : terms) {
        t.resize(n_);
    }
    for (uint32_t i = 0; i < n_; ++i) {
        terms[0][i] = vx[i] * m[i];
        terms[1][i] = vy[i] * m[i];
        terms[2][i] = vz[i] * m[i];
        terms[3][i] = ((y[i] * vz[i]) - (z[i] * vy[i])) * m[i];
        terms[4][i] = ((z[i] * vx[i]) - (x[i] * vz[i])) * m[i];
        terms[5][i] = ((x[i] * vy[i]) - (y[i] * vx[i])) * m[i];
    }
    for (int c = 0; c < 3; ++c) {
        d.linear_momentum[c] = compensated_sum(terms[c]);
        d.angular_momentum[c] = compensated_sum(terms[3 + c]);
    }
    return d;
}

void System::energy(double *kinetic, double *potential) {
    if (n_ == 0) {
        if (kinetic) *kinetic = 0.0;
        if (potential) *potential = 0.0;
        return;
    }
    terms_.reserve(n_);
    std::vector<double> host(n_);
    if (kinetic != nullptr) {
        check(launch_kinetic_partials(array(kVx), array(kVy), array(kVz), array(kM), n_,
                                      terms_.data(), stream_),
              "kinetic energy terms");
        check(cudaMemcpyAsync(host.data(), terms_.data(), sizeof(double) * n_,
                              cudaMemcpyDeviceToHost, stream_),
              "downloading kinetic terms");
        check(cudaStreamSynchronize(stream_), "kinetic energy");
        *kinetic = compensated_sum(host) / 2.0;
    }
    if (potential != nullptr) {
        const double eps2 = solver_->params().softening_squared;
        check(launch_potential_rows(array(kX), array(kY), array(kZ), array(kM), n_, eps2,
                                    terms_.data(), stream_),
              "potential energy rows");
        check(cudaMemcpyAsync(host.data(), terms_.data(), sizeof(double) * n_,
                              cudaMemcpyDeviceToHost, stream_),
              "downloading potential rows");
        check(cudaStreamSynchronize(stream_), "potential energy");
        *potential = compensated_sum(host);
    }
}

} // namespace ob

// ---------------------------------------------------------------------------
// extern "C"
// ---------------------------------------------------------------------------

struct ob_solver {
    std::unique_ptr<ob::Solver> impl;
};

struct ob_system {
    std::unique_ptr<ob::System> impl;
};

struct ob_batch {
    std::unique_ptr<ob::Batch> impl;
};

using ob::guarded;
using ob::require;

extern "C" {

const char *ob_version(void) { return "orrery_b200 0.1.0 (sm_100a)"; }

const char *ob_last_error(void) { return ob::g_last_error.c_str(); }

int ob_device_count(int *count) {
    return guarded([&] {
        require(count != nullptr, "count is NULL");
        *count = 0;
        if (cudaGetDeviceCount(count) != cudaSuccess) {
            cudaGetLastError();
            *count = 0;
        }
    });
}

int ob_solver_create(const ob_solver_params *params, ob_solver **out) {
    return guarded([&] {
        require(out != nullptr && params != nullptr, "NULL argument");
        *out = nullptr;
        const ob_solver_params checked = ob::corrected(*params);
        ob::require_device();
        auto s = std::make_unique<ob_solver>();
        s->impl = std::make_unique<ob::Solver>(checked);
        *out = s.release();
    });
}

void ob_solver_destroy(ob_solver *solver) { delete solver; }

int ob_solver_get_params(const ob_solver *solver, ob_solver_params *params) {
    return guarded([&] {
        require(solver != nullptr && params != nullptr, "NULL argument");
        *params = solver->impl->params();
    });
}

int ob_solver_evaluate(ob_solver *solver, uint64_t n, const double *x, const double *y,
                       const double *z, const double *m, double *ax, double *ay, double *az) {
    return guarded([&] {
        require(solver != nullptr, "solver is NULL");
        require(n == 0 || (x && y && z && m && ax && ay && az), "NULL array");
        solver->impl->evaluate_host(n, x, y, z, m, ax, ay, az);
    });
}

int ob_solver_evaluate_device(ob_solver *solver, uint64_t n, const double *x, const double *y,
                              const double *z, const double *m, double *ax, double *ay,
                              double *az, void *stream) {
    return guarded([&] {
        require(solver != nullptr, "solver is NULL");
        require(n <= 0xffffffffull, "the B200 solvers index particles with 32 bits");
        require(n == 0 || (x && y && z && m && ax && ay && az), "NULL array");
        solver->impl->evaluate_device(static_cast<uint32_t>(n), x, y, z, m, ax, ay, az,
                                      static_cast<cudaStream_t>(stream));
    });
}

int ob_solver_counts(ob_solver *solver, ob_counts *counts) {
    return guarded([&] {
        require(solver != nullptr && counts != nullptr, "NULL argument");
        *counts = solver->impl->counts();
    });
}

int ob_solver_reset_counts(ob_solver *solver) {
    return guarded([&] {
        require(solver != nullptr, "solver is NULL");
        solver->impl->reset_counts();
    });
}

int ob_solver_timings(const ob_solver *solver, ob_timings *timings) {
    return guarded([&] {
        require(solver != nullptr && timings != nullptr, "NULL argument");
        *timings = solver->impl->timings();
    });
}

int ob_test_set_walk_stack_cap(ob_solver *solver, uint32_t cap) {
    return guarded([&] {
        require(solver != nullptr, "solver is NULL");
        require(cap <= ob::walk_stack_capacity(), "stack cap above the walk's capacity");
        const ob_solver_params &p = solver->impl->params();
        if (p.kind != OB_SOLVER_TREE || p.precision == OB_PRECISION_FP64) {
            throw ob::Error(OB_ERROR_UNSUPPORTED, "the stack cap applies to the FP32 tree walk");
        }
        solver->impl->tree().set_walk_stack_cap(cap);
    });
}

int ob_tree_stats(ob_solver *solver, uint64_t *nodes, uint64_t *leaves, uint32_t *depth) {
    return guarded([&] {
        require(solver != nullptr, "solver is NULL");
        const ob::TreeMeta m = solver->impl->tree().meta();
        if (nodes != nullptr) *nodes = m.node_count;
        if (leaves != nullptr) *leaves = m.leaf_count;
        if (depth != nullptr) *depth = m.depth;
    });
}

int ob_tree_copy(ob_solver *solver, double *reals, uint64_t *idx, double *quads) {
    return guarded([&] {
        require(solver != nullptr && reals != nullptr && idx != nullptr, "NULL argument");
        solver->impl->tree().copy_tree(reals, idx, quads, nullptr, nullptr);
    });
}

int ob_tree_copy_order(ob_solver *solver, uint64_t *codes, uint32_t *indices, double *origin,
                       double *size) {
    return guarded([&] {
        require(solver != nullptr, "solver is NULL");
        solver->impl->tree().copy_order(codes, indices, origin, size);
    });
}

int ob_direct_shapes(int32_t precision, ob_direct_shape *out, int32_t capacity, int32_t *count) {
    return guarded([&] {
        require(count != nullptr, "count is NULL");
        require(precision == OB_PRECISION_FP32 || precision == OB_PRECISION_SPLIT,
                "shapes exist for the FP32 and split direct kernels");
        ob::DirectConfig all[128];
        const int total = ob::direct_candidates(precision == OB_PRECISION_SPLIT, all, 128);
        for (int k = 0; k < total && k < capacity && out != nullptr; ++k) {
            out[k] = ob_direct_shape{all[k].threads, all[k].targets_per_thread, all[k].split,
                                     all[k].groups};
        }
        *count = total;
    });
}

int ob_solver_set_direct_shape(ob_solver *solver, uint64_t n, const ob_direct_shape *shape) {
    return guarded([&] {
        require(solver != nullptr && shape != nullptr, "NULL argument");
        require(n <= 0xffffffffull, "the B200 solvers index particles with 32 bits");
        const ob_solver_params &p = solver->impl->params();
        require(p.kind == OB_SOLVER_DIRECT && p.precision != OB_PRECISION_FP64,
                "only the FP32 and split direct kernels have shapes");
        const int groups = shape->groups == 0 ? 1 : shape->groups;
        ob::DirectConfig all[128];
        const int total = ob::direct_candidates(p.precision == OB_PRECISION_SPLIT, all, 128);
        bool known = false;
        for (int k = 0; k < total; ++k) {
            known = known || (all[k].threads == shape->threads &&
                              all[k].targets_per_thread == shape->targets_per_thread &&
                              all[k].split == shape->split && all[k].groups == groups);
        }
        require(known, "the library implements no such direct kernel shape");
        solver->impl->set_direct_config(
            static_cast<uint32_t>(n),
            ob::DirectConfig{shape->threads, shape->targets_per_thread, shape->split, groups});
    });
}

int ob_solver_autotune(ob_solver *solver, uint64_t n, ob_direct_shape *chosen, double *best_ms) {
    return guarded([&] {
        require(solver != nullptr, "solver is NULL");
        require(n <= 0xffffffffull, "the B200 solvers index particles with 32 bits");
        ob::DirectConfig c;
        const double ms = solver->impl->autotune(static_cast<uint32_t>(n), c);
        if (chosen != nullptr) {
            *chosen = ob_direct_shape{c.threads, c.targets_per_thread, c.split, c.groups};
        }
        if (best_ms != nullptr) {
            *best_ms = ms;
        }
    });
}

int ob_system_create(const ob_solver_params *params, uint64_t n, ob_system **out) {
    return guarded([&] {
        require(out != nullptr && params != nullptr, "NULL argument");
        *out = nullptr;
        require(n <= 0xffffffffull, "the B200 solvers index particles with 32 bits");
        const ob_solver_params checked = ob::corrected(*params);
        ob::require_device();
        auto s = std::make_unique<ob_system>();
        s->impl = std::make_unique<ob::System>(checked, static_cast<uint32_t>(n));
        *out = s.release();
    });
}

void ob_system_destroy(ob_system *system) { delete system; }

int ob_system_set_state(ob_system *system, const double *x, const double *y, const double *z,
                        const double *vx, const double *vy, const double *vz, const double *m) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        system->impl->set_state(x, y, z, vx, vy, vz, m);
    });
}

int ob_system_set_accelerations(ob_system *system, const double *ax, const double *ay,
                                const double *az) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        system->impl->set_accelerations(ax, ay, az);
    });
}

int ob_system_step_host(ob_system *system, int32_t integrator, double dt, uint64_t steps,
                        double *x, double *y, double *z, double *vx, double *vy, double *vz,
                        double *ax, double *ay, double *az, const double *m) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        double *io[9] = {x, y, z, vx, vy, vz, ax, ay, az};
        system->impl->step_host(integrator, dt, steps, io, m);
    });
}

int ob_system_get_state(ob_system *system, double *x, double *y, double *z, double *vx,
                        double *vy, double *vz, double *ax, double *ay, double *az) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        double *out[9] = {x, y, z, vx, vy, vz, ax, ay, az};
        system->impl->get_state(out);
    });
}

int ob_system_step(ob_system *system, int32_t integrator, double dt, uint64_t steps) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        system->impl->step_async(integrator, dt, steps);
        system->impl->synchronize();
    });
}

int ob_system_step_async(ob_system *system, int32_t integrator, double dt, uint64_t steps) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        system->impl->step_async(integrator, dt, steps);
    });
}

int ob_system_synchronize(ob_system *system) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        system->impl->synchronize();
    });
}

int ob_system_energy(ob_system *system, double *kinetic, double *potential) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        system->impl->energy(kinetic, potential);
    });
}

int ob_system_diagnostics(ob_system *system, ob_diagnostics *out) {
    return guarded([&] {
        require(system != nullptr && out != nullptr, "NULL argument");
        *out = system->impl->diagnostics();
    });
}

int ob_system_restore(ob_system *system, const double *m, const double *x, const double *y,
                      const double *z, const double *vx, const double *vy, const double *vz,
                      const double *ax, const double *ay, const double *az) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        const double *arrays[10] = {m, x, y, z, vx, vy, vz, ax, ay, az};
        for (const double *a : arrays) {
            require(system->impl->size() == 0 || a != nullptr, "every state array is required");
        }
        system->impl->restore(arrays);
    });
}

int ob_system_snapshot(ob_system *system, double *m, double *x, double *y, double *z,
                       double *vx, double *vy, double *vz, double *ax, double *ay, double *az) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        double *const arrays[10] = {m, x, y, z, vx, vy, vz, ax, ay, az};
        for (double *a : arrays) {
            require(system->impl->size() == 0 || a != nullptr, "every state array is required");
        }
        system->impl->snapshot(arrays);
    });
}

int ob_system_device_arrays(ob_system *system, void **arrays) {
    return guarded([&] {
        require(system != nullptr && arrays != nullptr, "NULL argument");
        for (int k = 0; k < 10; ++k) {
            arrays[k] = system->impl->size() == 0 ? nullptr : system->impl->array(k);
        }
    });
}

int ob_system_set_fused_steps(ob_system *system, int32_t enable, int32_t *active) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        const bool on = system->impl->set_fused_steps(enable != 0);
        if (active != nullptr) {
            *active = on ? 1 : 0;
        }
    });
}

int ob_test_fused_timeout(ob_system *system, uint32_t poll_limit) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        require(poll_limit > 0, "the poll limit must be positive");
        if (!system->impl->arm_fused_timeout(poll_limit)) {
            throw ob::Error(OB_ERROR_UNSUPPORTED, "the system does not take fused steps");
        }
    });
}

int ob_system_counts(ob_system *system, ob_counts *counts) {
    return guarded([&] {
        require(system != nullptr && counts != nullptr, "NULL argument");
        *counts = system->impl->solver().counts();
    });
}

int ob_system_autotune(ob_system *system, ob_direct_shape *chosen, double *best_ms) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        ob::DirectConfig c;
        const double ms = system->impl->solver().autotune(system->impl->size(), c);
        if (chosen != nullptr) {
            *chosen = ob_direct_shape{c.threads, c.targets_per_thread, c.split, c.groups};
        }
        if (best_ms != nullptr) {
            *best_ms = ms;
        }
    });
}

int ob_system_stream(ob_system *system, void **stream) {
    return guarded([&] {
        require(system != nullptr && stream != nullptr, "NULL argument");
        *stream = system->impl->stream();
    });
}

int ob_system_profile(ob_system *system, uint32_t steps) {
    return guarded([&] {
        require(system != nullptr, "system is NULL");
        system->impl->profile(steps);
    });
}

int ob_system_phase_times(ob_system *system, ob_timings *average, uint32_t *evaluations) {
    return guarded([&] {
        require(system != nullptr && average != nullptr, "NULL argument");
        uint32_t count = 0;
        *average = system->impl->phase_times(count);
        if (evaluations != nullptr) {
            *evaluations = count;
        }
    });
}

int ob_system_step_kernels(ob_system *system, int32_t integrator, double dt, uint32_t *kernels) {
    return guarded([&] {
        require(system != nullptr && kernels != nullptr, "NULL argument");
        *kernels = system->impl->step_kernels(integrator, dt);
    });
}

int ob_system_size(const ob_system *system, uint64_t *n) {
    return guarded([&] {
        require(system != nullptr && n != nullptr, "NULL argument");
        *n = system->impl->size();
    });
}

int ob_batch_create(uint32_t systems, const uint64_t *counts, const double *softening_squared,
                    ob_batch **out) {
    return guarded([&] {
        require(out != nullptr && counts != nullptr && softening_squared != nullptr,
                "NULL argument");
        *out = nullptr;
        require(systems > 0, "a batch needs at least one system");
        ob::require_device();
        auto b = std::make_unique<ob_batch>();
        b->impl = std::make_unique<ob::Batch>(systems, counts, softening_squared);
        *out = b.release();
    });
}

void ob_batch_destroy(ob_batch *batch) { delete batch; }

int ob_batch_set_state(ob_batch *batch, uint32_t system, const double *x, const double *y,
                       const double *z, const double *vx, const double *vy, const double *vz,
                       const double *m) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        batch->impl->set_state(system, x, y, z, vx, vy, vz, m);
    });
}

int ob_batch_get_state(ob_batch *batch, uint32_t system, double *x, double *y, double *z,
                       double *vx, double *vy, double *vz, double *ax, double *ay, double *az) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        double *out[9] = {x, y, z, vx, vy, vz, ax, ay, az};
        batch->impl->get_state(system, out);
    });
}

int ob_batch_refresh(ob_batch *batch) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        batch->impl->refresh();
    });
}

int ob_batch_step(ob_batch *batch, int32_t integrator, double dt, uint64_t steps) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        require(std::isfinite(dt), "the timestep must be finite");
        batch->impl->step_async(integrator, dt, steps);
        batch->impl->synchronize();
    });
}

int ob_batch_step_async(ob_batch *batch, int32_t integrator, double dt, uint64_t steps) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        require(std::isfinite(dt), "the timestep must be finite");
        batch->impl->step_async(integrator, dt, steps);
    });
}

int ob_batch_synchronize(ob_batch *batch) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        batch->impl->synchronize();
    });
}

int ob_batch_energy(ob_batch *batch, uint32_t system, double *kinetic, double *potential) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        batch->impl->energy(system, kinetic, potential);
    });
}

int ob_batch_autotune(ob_batch *batch, ob_batch_shape *chosen, double *best_ms) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        ob::BatchConfig c;
        const double ms = batch->impl->autotune(c);
        if (chosen != nullptr) {
            *chosen = ob_batch_shape{c.threads, c.targets_per_thread, c.chunk_tiles, c.groups};
        }
        if (best_ms != nullptr) {
            *best_ms = ms;
        }
    });
}

int ob_batch_set_shape(ob_batch *batch, const ob_batch_shape *shape) {
    return guarded([&] {
        require(batch != nullptr && shape != nullptr, "NULL argument");
        const int groups = shape->groups == 0 ? 1 : shape->groups;
        require(ob::batch_shape_known(shape->threads, shape->targets_per_thread, groups),
                "the library implements no such batch kernel shape");
        batch->impl->set_config(ob::BatchConfig{shape->threads, shape->targets_per_thread,
                                                shape->chunk_tiles, groups});
    });
}

int ob_batch_stats(ob_batch *batch, uint64_t *pairs_per_evaluation, uint64_t *evaluations,
                   uint32_t *items) {
    return guarded([&] {
        require(batch != nullptr, "batch is NULL");
        if (pairs_per_evaluation != nullptr) *pairs_per_evaluation = batch->impl->pair_interactions();
        if (evaluations != nullptr) *evaluations = batch->impl->evaluations();
        if (items != nullptr) *items = batch->impl->items();
    });
}

int ob_batch_stream(ob_batch *batch, void **stream) {
    return guarded([&] {
        require(batch != nullptr && stream != nullptr, "NULL argument");
        *stream = batch->impl->stream();
    });
}

// --------------------------------------------------------------------------
// Run output: ORRERYCK checkpoints and ORRERYTJ trajectories (output.hpp)
// --------------------------------------------------------------------------

int ob_checkpoint_write(const char *path, uint64_t step, const char *configuration,
                        uint64_t configuration_bytes, uint64_t n, const double *m,
                        const double *x, const double *y, const double *z, const double *vx,
                        const double *vy, const double *vz, const double *ax, const double *ay,
                        const double *az) {
    return guarded([&] {
        require(path != nullptr, "path is NULL");
        require(configuration != nullptr || configuration_bytes == 0, "configuration is NULL");
        const double *arrays[ob::kCheckpointArrays] = {m, x, y, z, vx, vy, vz, ax, ay, az};
        ob::write_checkpoint_file(path, step, std::string(configuration ? configuration : "",
                                                          configuration_bytes),
                                  n, arrays);
    });
}

int ob_checkpoint_info(const char *path, uint64_t *step, uint64_t *n,
                       uint64_t *configuration_bytes) {
    return guarded([&] {
        require(path != nullptr, "path is NULL");
        const ob::CheckpointHeader h = ob::read_checkpoint_file(path, nullptr, 0);
        if (step != nullptr) *step = h.step;
        if (n != nullptr) *n = h.n;
        if (configuration_bytes != nullptr) *configuration_bytes = h.configuration.size();
    });
}

int ob_checkpoint_read(const char *path, char *configuration, uint64_t configuration_capacity,
                       uint64_t n, double *m, double *x, double *y, double *z, double *vx,
                       double *vy, double *vz, double *ax, double *ay, double *az) {
    return guarded([&] {
        require(path != nullptr, "path is NULL");
        double *const arrays[ob::kCheckpointArrays] = {m, x, y, z, vx, vy, vz, ax, ay, az};
        for (double *a : arrays) {
            require(n == 0 || a != nullptr, "every state array is required");
        }
        const ob::CheckpointHeader h = ob::read_checkpoint_file(path, arrays, n);
        if (configuration != nullptr) {
            require(h.configuration.size() <= configuration_capacity,
                    "the configuration buffer is too small (see ob_checkpoint_info)");
            std::memcpy(configuration, h.configuration.data(), h.configuration.size());
        }
    });
}

int ob_system_write_checkpoint(ob_system *system, const char *path, uint64_t step,
                               const char *configuration, uint64_t configuration_bytes) {
    return guarded([&] {
        require(system != nullptr && path != nullptr, "NULL argument");
        require(configuration != nullptr || configuration_bytes == 0, "configuration is NULL");
        const uint64_t n = system->impl->size();
        std::vector<double> host(10 * n);
        double *arrays[ob::kCheckpointArrays];
        for (int k = 0; k < ob::kCheckpointArrays; ++k) {
            arrays[k] = host.data() + k * n;
        }
        system->impl->snapshot(arrays);
        const double *const *in = arrays;
        ob::write_checkpoint_file(path, step, std::string(configuration ? configuration : "",
                                                          configuration_bytes),
                                  n, in);
    });
}

int ob_system_read_checkpoint(ob_system *system, const char *path, uint64_t *step,
                              char *configuration, uint64_t configuration_capacity,
                              uint64_t *configuration_bytes) {
    return guarded([&] {
        require(system != nullptr && path != nullptr, "NULL argument");
        const uint64_t n = system->impl->size();
        std::vector<double> host(10 * n);
        double *arrays[ob::kCheckpointArrays];
        for (int k = 0; k < ob::kCheckpointArrays; ++k) {
            arrays[k] = host.data() + k * n;
        }
        const ob::CheckpointHeader h = ob::read_checkpoint_file(path, arrays, n);
        if (configuration != nullptr) {
            require(h.configuration.size() <= configuration_capacity,
                    "the configuration buffer is too small (see ob_checkpoint_info)");
            std::memcpy(configuration, h.configuration.data(), h.configuration.size());
        }
        const double *const *in = arrays;
        system->impl->restore(in);
        if (step != nullptr) *step = h.step;
        if (configuration_bytes != nullptr) *configuration_bytes = h.configuration.size();
    });
}

} // extern "C"

struct ob_trajectory {
    std::unique_ptr<ob::TrajectoryFile> host;     // host-array frames only
    std::unique_ptr<ob::DeviceTrajectory> device; // bound to a system
};

extern "C" {

int ob_trajectory_create(const char *path, uint64_t n, const double *masses, double timestep,
                         int32_t with_velocities, ob_trajectory **out) {
    return guarded([&] {
        require(path != nullptr && out != nullptr, "NULL argument");
        *out = nullptr;
        auto t = std::make_unique<ob_trajectory>();
        t->host = std::make_unique<ob::TrajectoryFile>(path, n, masses, timestep,
                                                       with_velocities != 0);
        *out = t.release();
    });
}

int ob_trajectory_create_for_system(const char *path, ob_system *system, double timestep,
                                    int32_t with_velocities, ob_trajectory **out) {
    return guarded([&] {
        require(path != nullptr && system != nullptr && out != nullptr, "NULL argument");
        *out = nullptr;
        auto t = std::make_unique<ob_trajectory>();
        t->device = std::make_unique<ob::DeviceTrajectory>(path, *system->impl, timestep,
                                                           with_velocities != 0);
        *out = t.release();
    });
}

int ob_trajectory_write_frame(ob_trajectory *trajectory, uint64_t step, double time,
                              const double *x, const double *y, const double *z,
                              const double *vx, const double *vy, const double *vz) {
    return guarded([&] {
        require(trajectory != nullptr, "trajectory is NULL");
        const double *xyz[3] = {x, y, z};
        const double *v[3] = {vx, vy, vz};
        if (trajectory->device) {
            trajectory->device->write_host_frame(step, time, xyz, v);
            return;
        }
        ob::TrajectoryFile &f = *trajectory->host;
        for (int c = 0; c < 3; ++c) {
            require(f.size() == 0 || (xyz[c] != nullptr &&
                                      (!f.with_velocities() || v[c] != nullptr)),
                    "a frame needs every array the file carries");
        }
        f.write_frame(step, time, xyz, v);
    });
}

int ob_trajectory_write_system_frame(ob_trajectory *trajectory, uint64_t step, double time) {
    return guarded([&] {
        require(trajectory != nullptr, "trajectory is NULL");
        require(trajectory->device != nullptr, "the trajectory is not bound to a system");
        trajectory->device->write_frame(step, time);
    });
}

int ob_trajectory_flush(ob_trajectory *trajectory) {
    return guarded([&] {
        require(trajectory != nullptr, "trajectory is NULL");
        if (trajectory->device) {
            trajectory->device->flush();
        } else {
            trajectory->host->flush();
        }
    });
}

int ob_trajectory_frames(ob_trajectory *trajectory, uint64_t *frames) {
    return guarded([&] {
        require(trajectory != nullptr && frames != nullptr, "NULL argument");
        *frames = trajectory->device ? trajectory->device->frames() : trajectory->host->frames();
    });
}

int ob_trajectory_close(ob_trajectory *trajectory) {
    if (trajectory == nullptr) {
        return OB_OK;
    }
    const int rc = ob_trajectory_flush(trajectory);
    delete trajectory;
    return rc;
}

} // extern "C"
