// The solver object behind ob_solver: owns device buffers, counters and
// timing events, and enqueues one force evaluation on device arrays.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <memory>

#include <cuda_runtime.h>

#include "internal.hpp"
#include "orrery_b200.h"
#include "runtime.hpp"

namespace ob {

class TreePipeline; // tree.cu

// Validated parameters: corrected_parameters (src/solvers/octree.cpp:189-194)
// for the tree fields, softening >= 0, known kind/precision combinations.
ob_solver_params corrected(const ob_solver_params &params);

class Solver {
public:
    explicit Solver(const ob_solver_params &params);
    ~Solver();
    Solver(const Solver &) = delete;
    Solver &operator=(const Solver &) = delete;

    [[nodiscard]] const ob_solver_params &params() const noexcept { return params_; }

    // Enqueues a = f(x, m) for n particles of device arrays on `stream`.
    // `count` = false leaves the host counters alone (graph capture, where
    // System::step accounts for the replays instead).
    // `marks`, when given, are four events recorded as graph-visible event
    // nodes (cudaEventRecordExternal) at the start, after ordering, after
    // construction and at the end of the evaluation.
    void evaluate_device(uint32_t n, const double *x, const double *y, const double *z,
                         const double *m, double *ax, double *ay, double *az, cudaStream_t stream,
                         bool count = true, const cudaEvent_t *marks = nullptr);

    // Adds `evaluations` evaluations of n particles to the host counters
    // (direct pairs in closed form, as src/solvers/cuda_direct_solver.cpp:284-292).
    void account(uint64_t evaluations, uint64_t n);

    // Host arrays in and out; synchronous.
    void evaluate_host(uint64_t n, const double *x, const double *y, const double *z,
                       const double *m, double *ax, double *ay, double *az);

    ob_counts counts();
    void reset_counts();
    ob_timings timings() const;

    // Raises OB_ERROR_TIMEOUT if a kernel gave up on a bounded wait.
    void check_status(cudaStream_t stream);
    // The device status word kernels of this solver's evaluations report to.
    [[nodiscard]] unsigned *status_word() const noexcept { return status_.data(); }

    // Pair interactions the last direct evaluation computed, N(N-1).
    static uint64_t direct_pairs(uint64_t n) { return n > 1 ? n * (n - 1) : 0; }

    // Chooses (and caches) the direct kernel shape for n particles.
    DirectConfig direct_config(uint32_t n);
    void set_direct_config(uint32_t n, const DirectConfig &config) {
        configs_[n] = config;
        ++generation_;
    }

    int sm_count() const noexcept { return sm_count_; }

    // The tree pipeline (tree solvers only; throws otherwise).
    TreePipeline &tree();

    // Changes whenever a device buffer the evaluation uses is reallocated.
    uint64_t generation() const noexcept;

    // After a synchronised evaluation: true if the tree ran out of node
    // capacity, in which case the capacity has been raised and the
    // evaluation must be repeated.
    bool grew_after_overflow(cudaStream_t stream);

    // Times every implemented shape on synthetic sources of n particles and
    // keeps the fastest for n. Returns the time per evaluation in ms.
    double autotune(uint32_t n, DirectConfig &chosen);

private:
    void evaluate_direct(uint32_t n, const double *x, const double *y, const double *z,
                         const double *m, double *ax, double *ay, double *az,
                         cudaStream_t stream, cudaEvent_t ordered, cudaEvent_t built,
                         bool external);

    ob_solver_params params_;
    int sm_count_ = 148;
    DeviceArray<float4> hi_;
    DeviceArray<float4> lo_;
    DeviceArray<double> staging_;
    DeviceArray<unsigned> status_;
    ob_counts counts_{};
    std::array<cudaEvent_t, 6> events_{};
    bool timed_host_ = false;
    cudaStream_t stream_ = nullptr;
    std::map<uint32_t, DirectConfig> configs_;
    uint64_t generation_ = 0;
    std::unique_ptr<TreePipeline> tree_;
};

} // namespace ob
