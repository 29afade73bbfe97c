// A particle system resident in HBM, integrated on the device.
//
// The device counterpart of sim::Simulation's state handling
// (src/sim/simulation.cpp:16-70): positions, velocities, accelerations and
// masses as ten FP64 SoA arrays that never leave the device between steps.
// One integrator step is captured once as a CUDA graph and replayed.
#pragma once

#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "runtime.hpp"
#include "solver.hpp"

namespace ob {

class System {
public:
    enum Array { kX = 0, kY, kZ, kVx, kVy, kVz, kAx, kAy, kAz, kM };

    // With `stream` given, the system issues all its work on that stream (and
    // does not own it); otherwise it creates its own.
    System(const ob_solver_params &params, uint32_t n, cudaStream_t stream = nullptr);
    ~System();
    System(const System &) = delete;
    System &operator=(const System &) = delete;

    void set_state(const double *x, const double *y, const double *z, const double *vx,
                   const double *vy, const double *vz, const double *m);
    void set_accelerations(const double *ax, const double *ay, const double *az);
    void get_state(double *const *out); // x y z vx vy vz ax ay az, NULL entries skipped
    // The ten state arrays in a checkpoint's order: m x y z vx vy vz ax ay az.
    void snapshot(double *const *arrays);
    // Installs a checkpoint's ten arrays as they are; the accelerations are the
    // ones the run carried, not re-evaluated (sim::Simulation::restore with
    // accelerations_are_current, include/orrery/sim/simulation.hpp:101-102).
    void restore(const double *const *arrays);
    void refresh();
    void step_async(int integrator, double dt, uint64_t steps);
    // Uploads x y z vx vy vz ax ay az (io) and m, steps, downloads io.
    void step_host(int integrator, double dt, uint64_t steps, double *const *io, const double *m);
    void synchronize();
    void energy(double *kinetic, double *potential);
    ob_diagnostics diagnostics();

    [[nodiscard]] Solver &solver() noexcept { return *solver_; }
    [[nodiscard]] uint32_t size() const noexcept { return n_; }
    [[nodiscard]] double *array(int k) const noexcept {
        return state_.data() + static_cast<size_t>(k) * n_;
    }
    [[nodiscard]] cudaStream_t stream() const noexcept { return stream_; }

    static int evaluations_per_step(int integrator);

    // Per-phase timing of graph replays (see ob_system_profile).
    void profile(uint32_t steps);

    // Whole steps of a small FP32-direct system in one launch (fused.cu), used
    // for velocity Verlet and Yoshida-4 where the system fits; on by default.
    // Returns whether the next such step will use it.
    bool set_fused_steps(bool enable);
    // Tests of the fused launch's bounded wait: the next fused launch polls at
    // most `poll_limit` times and its CTA 0 never publishes. Returns whether
    // the system takes fused steps.
    bool arm_fused_timeout(uint32_t poll_limit);
    bool fused_for(int integrator);
    ob_timings phase_times(uint32_t &evaluations);
    uint32_t step_kernels(int integrator, double dt);

private:
    void upload(int first, int count, const double *const *host);
    void evaluate(bool count, const cudaEvent_t *marks = nullptr);
    // `drifted` (optional) is recorded once the step's positions are final.
    void enqueue_substep(double timestep, const cudaEvent_t *marks, cudaEvent_t drifted = nullptr);
    void enqueue_step(int integrator, double dt, bool marked, cudaEvent_t drifted = nullptr);
    void enqueue_rk4_step(double dt, const cudaEvent_t *marks, cudaEvent_t drifted = nullptr);
    cudaGraph_t capture_step(int integrator, double dt, bool marked);
    void drop_graph();
    void ensure_graph(int integrator, double dt);
    void ensure_marked_graph();
    void set_marks(const std::vector<cudaEvent_t> &events, size_t offset);

    std::unique_ptr<Solver> solver_;
    uint32_t n_;
    DeviceArray<double> state_;
    DeviceArray<double> terms_;
    DeviceArray<double> rk4_; // RK4: x0, v0 and the derivative sums (12n), reserved on first use
    cudaStream_t stream_ = nullptr;
    // step_host: downloads the positions on this stream while the last step's
    // force evaluation runs (created on first use).
    cudaStream_t copy_stream_ = nullptr;
    cudaEvent_t drifted_ = nullptr;
    bool owns_stream_ = true;
    // The step as a CUDA graph, without event nodes: what every step replays
    // unless it is profiled.
    cudaGraphExec_t graph_ = nullptr;
    int graph_integrator_ = -1;
    double graph_dt_ = 0.0;
    uint32_t graph_kernels_ = 0;
    uint64_t graph_generation_ = 0;

    // The same step with four placeholder events per evaluation captured as
    // event nodes, built on the first profiled step; before each profiled
    // replay its nodes are pointed at a fresh slot of ring_. The template is
    // kept so that its event nodes can be retargeted.
    cudaGraph_t marked_template_ = nullptr;
    cudaGraphExec_t marked_graph_ = nullptr;
    std::vector<cudaEvent_t> marks_;
    std::vector<cudaGraphNode_t> mark_nodes_;
    static constexpr size_t kMarksPerStep = 16; // four per evaluation, RK4's four at most
    // The fused small-system path: its position buffers and ready words,
    // whether it is allowed, the warps per CTA of its launch (0: this system
    // does not fit it; -1: not yet asked), and the event pairs timing its
    // launches while profiling.
    DeviceArray<float4> fused_buf_;
    DeviceArray<unsigned> fused_ready_; // per CTA: substeps published (fused.cu)
    uint32_t fused_epoch_ = 0;          // substeps launched since the words were cleared
    bool fused_enabled_ = true;
    bool fused_ready_reset_ = false;    // clear the ready words before the next fused launch
    int fused_warps_ = -1;
    uint32_t fused_test_polls_ = 0; // nonzero: the next fused launch's test wait (above)
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> fused_marks_;
    std::vector<uint64_t> fused_mark_evals_;
    std::vector<cudaEvent_t> ring_;
    uint32_t ring_steps_ = 0;     // capacity in steps
    uint32_t ring_used_ = 0;      // steps recorded
};

} // namespace ob
