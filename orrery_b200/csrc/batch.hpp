// Many independent particle systems integrated together on one device.
//
// The reference integrates one system per Simulation
// (src/sim/simulation.cpp:16-70) with one Softening per solver
// (include/orrery/core/softening.hpp:50-60). A batch holds many systems of
// uneven size, each with its own softening, in one padded FP64 SoA, and
// evaluates all their direct-sum forces in a single persistent launch.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include <cuda_runtime.h>

#include "internal.hpp"
#include "orrery_b200.h"
#include "runtime.hpp"

namespace ob {

// One unit of the batched force kernel's work queue: BT targets of one system
// against one chunk of that system's sources.
struct BatchItem {
    uint32_t system;
    uint32_t target_begin;  // first target (padded global index)
    uint32_t target_count;  // valid targets in this tile (<= BT)
    uint32_t source_begin;  // first source (padded global index, tile aligned)
    uint32_t source_tiles;  // 512-source tiles in the chunk
    uint32_t slot;          // partial-sum slot, or kDirectWrite
};
constexpr uint32_t kDirectWrite = 0xffffffffu;

// Targets whose sums are spread over several items' partial slots.
struct BatchGroup {
    uint32_t target_begin;
    uint32_t target_count;
    uint32_t first_slot;
    uint32_t slots;
};

// Tile shape of the batched kernel.
struct BatchConfig {
    int threads = 128;
    int targets_per_thread = 2;
    uint32_t chunk_tiles = 0; // source tiles per item; 0 = a whole system
};

// Batched kernel launch (batch.cu).
cudaError_t launch_batch_forces(const float4 *hi, const float4 *lo, const float *eps2,
                                const BatchItem *items, uint32_t item_count,
                                const BatchConfig &config, double *ax, double *ay, double *az,
                                double *partial, uint32_t *queue, unsigned *status,
                                int sm_count, cudaStream_t stream);
cudaError_t launch_batch_reduce(const BatchGroup *groups, uint32_t group_count,
                                const double *partial, uint32_t bt, double *ax, double *ay,
                                double *az, cudaStream_t stream);

class Batch {
public:
    Batch(uint32_t systems, const uint64_t *counts, const double *softening_squared);
    ~Batch();
    Batch(const Batch &) = delete;
    Batch &operator=(const Batch &) = delete;

    void set_state(uint32_t system, const double *x, const double *y, const double *z,
                   const double *vx, const double *vy, const double *vz, const double *m);
    void get_state(uint32_t system, double *const *out);
    void refresh();
    void step_async(int integrator, double dt, uint64_t steps);
    void synchronize();
    void energy(uint32_t system, double *kinetic, double *potential);
    double autotune(BatchConfig &chosen);
    void set_config(const BatchConfig &config);

    [[nodiscard]] uint32_t systems() const noexcept { return static_cast<uint32_t>(count_.size()); }
    [[nodiscard]] uint64_t pair_interactions() const noexcept { return pairs_; }
    [[nodiscard]] uint64_t evaluations() const noexcept { return evaluations_; }
    [[nodiscard]] cudaStream_t stream() const noexcept { return stream_; }
    [[nodiscard]] uint32_t items() const noexcept { return item_count_; }
    [[nodiscard]] const BatchConfig &config() const noexcept { return config_; }

private:
    enum Array { kX = 0, kY, kZ, kVx, kVy, kVz, kAx, kAy, kAz, kM };
    double *array(int k) const noexcept { return state_.data() + static_cast<size_t>(k) * total_; }
    void build_items(const BatchConfig &config);
    void evaluate();
    void enqueue_step(int integrator, double dt);
    void drop_graph();

    std::vector<uint32_t> count_;    // particles per system
    std::vector<uint32_t> offset_;   // padded start of each system
    std::vector<double> eps2_host_;
    uint32_t total_ = 0;             // padded particles of all systems
    uint64_t pairs_ = 0;             // sum N(N-1) over systems
    uint64_t evaluations_ = 0;
    int sm_count_ = 148;
    BatchConfig config_;
    uint32_t item_count_ = 0;
    uint32_t group_count_ = 0;
    uint32_t slots_ = 0;
    DeviceArray<double> state_;
    DeviceArray<float4> hi_;
    DeviceArray<float4> lo_;
    DeviceArray<float> eps2_;
    DeviceArray<BatchItem> items_;
    DeviceArray<BatchGroup> groups_;
    DeviceArray<double> partial_;
    DeviceArray<uint32_t> queue_;
    DeviceArray<unsigned> status_;
    DeviceArray<double> terms_;
    cudaStream_t stream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    int graph_integrator_ = -1;
    double graph_dt_ = 0.0;
};

} // namespace ob
