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
#include <utility>
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

// Tile shape of the batched kernel. The default is the shape the autotuner
// picks on B200 for 512 systems of 256 to 16,384 particles.
struct BatchConfig {
    int threads = 256;
    int targets_per_thread = 4; // even: targets are processed in packed pairs
    uint32_t chunk_tiles = 0; // source tiles per item; 0 = a whole system
    int groups = 8;           // thread groups of a CTA that split each tile's sources
    // Targets of one work item (one CTA).
    [[nodiscard]] uint32_t targets_per_block() const {
        return static_cast<uint32_t>(threads * targets_per_thread / groups);
    }
};

// (threads, targets per thread, source groups) of the implemented batched
// kernels.
inline constexpr int kBatchShapes[][3] = {{128, 2, 1}, {128, 4, 1}, {256, 2, 1}, {256, 4, 1},
                                          {128, 2, 4}, {256, 2, 8}, {256, 4, 4}, {256, 4, 8}};
inline bool batch_shape_known(int threads, int targets_per_thread, int groups) {
    for (const auto &s : kBatchShapes) {
        if (s[0] == threads && s[1] == targets_per_thread && s[2] == groups) {
            return true;
        }
    }
    return false;
}

// Batched kernel launch (batch.cu).
cudaError_t launch_batch_forces(const float4 *hi, const float4 *lo, const float *eps2,
                                const BatchItem *items, uint32_t item_count,
                                const BatchConfig &config, double *ax, double *ay, double *az,
                                double *partial, uint32_t *queue, unsigned *status,
                                int sm_count, cudaStream_t stream);
cudaError_t launch_batch_reduce(const BatchGroup *groups, uint32_t group_count,
                                const double *partial, uint32_t bt, double *ax, double *ay,
                                double *az, cudaStream_t stream);

// A set of systems sharing one padded arena in HBM. Members can be added and
// removed between steps (the serving loop's continuous batching); the work
// items and the step graph are rebuilt when membership changes.
class Batch {
public:
    // An empty batch whose arena holds `capacity` padded particles. With
    // `stream` given, the batch issues all its work on that stream (and does
    // not own it); otherwise it creates its own.
    explicit Batch(uint64_t capacity, cudaStream_t stream = nullptr);
    // A batch of exactly these systems (ids 0 .. systems-1).
    Batch(uint32_t systems, const uint64_t *counts, const double *softening_squared);
    ~Batch();
    Batch(const Batch &) = delete;
    Batch &operator=(const Batch &) = delete;

    // Reserves room for a system of n particles; returns its id, or -1 when
    // the arena has no free region large enough. The region starts zeroed.
    int64_t add(uint32_t n, double softening_squared);
    // Frees a member's region (zeroed so it no longer contributes anything).
    void remove(uint32_t id);
    [[nodiscard]] bool active(uint32_t id) const noexcept;
    [[nodiscard]] uint32_t count(uint32_t id) const noexcept { return members_[id].count; }
    // Padded particles the arena would take for a system of n particles.
    static uint64_t footprint(uint32_t n);
    // Device bytes per padded particle of the arena.
    static constexpr uint64_t kBytesPerParticle = 10 * 8 + 64;

    void set_state(uint32_t id, const double *x, const double *y, const double *z,
                   const double *vx, const double *vy, const double *vz, const double *m);
    void get_state(uint32_t id, double *const *out);
    // Enqueues the download of a member's 9 arrays (x y z vx vy vz ax ay az;
    // NULL entries skipped) on the batch stream without waiting.
    void get_state_async(uint32_t id, double *const *out);
    // Evaluates the accelerations of every member, or of the listed members.
    void refresh();
    void refresh_members(const std::vector<uint32_t> &ids);
    void step_async(int integrator, double dt, uint64_t steps);
    void synchronize();
    void energy(uint32_t id, double *kinetic, double *potential);
    double autotune(BatchConfig &chosen);
    void set_config(const BatchConfig &config);

    [[nodiscard]] uint32_t members() const noexcept { return active_count_; }
    [[nodiscard]] uint64_t pair_interactions() const noexcept { return pairs_; }
    [[nodiscard]] uint64_t evaluations() const noexcept { return evaluations_; }
    [[nodiscard]] cudaStream_t stream() const noexcept { return stream_; }
    [[nodiscard]] uint32_t items() {
        rebuild_if_needed();
        return item_count_;
    }
    [[nodiscard]] const BatchConfig &config() const noexcept { return config_; }

private:
    struct Member {
        uint32_t count = 0;
        uint32_t offset = 0;
        uint32_t padded = 0;
        double eps2 = 0.0;
        bool active = false;
    };
    enum Array { kX = 0, kY, kZ, kVx, kVy, kVz, kAx, kAy, kAz, kM };
    double *array(int k) const noexcept { return state_.data() + static_cast<size_t>(k) * total_; }
    void init(uint64_t capacity, cudaStream_t stream);
    void check_member(uint32_t id) const;
    std::vector<BatchItem> make_items(const BatchConfig &config, const std::vector<uint32_t> &ids,
                                      std::vector<BatchGroup> &groups, uint32_t &slots) const;
    void rebuild_if_needed();
    void upload_items(const std::vector<BatchItem> &items, const std::vector<BatchGroup> &groups,
                      uint32_t slots);
    void evaluate();
    void enqueue_step(int integrator, double dt);
    void drop_graph();

    std::vector<Member> members_;
    std::vector<uint32_t> free_ids_;
    std::vector<std::pair<uint32_t, uint32_t>> free_regions_; // (offset, size), by offset
    uint32_t active_count_ = 0;
    uint32_t total_ = 0;  // arena capacity in padded particles (plus slack)
    uint32_t high_ = 0;   // end of the highest active region
    uint64_t pairs_ = 0;  // sum N(N-1) over active members
    uint64_t evaluations_ = 0;
    int sm_count_ = 148;
    BatchConfig config_{256, 2, 8};
    bool dirty_ = true;
    uint32_t item_count_ = 0;
    uint32_t group_count_ = 0;
    DeviceArray<double> state_;
    DeviceArray<float4> hi_;
    DeviceArray<float4> lo_;
    DeviceArray<float> eps2_;
    DeviceArray<BatchItem> items_;
    DeviceArray<BatchItem> side_items_;
    DeviceArray<BatchGroup> groups_;
    DeviceArray<double> partial_;
    DeviceArray<uint32_t> queue_;
    DeviceArray<unsigned> status_;
    DeviceArray<double> terms_;
    cudaStream_t stream_ = nullptr;
    bool owns_stream_ = true;
    cudaGraphExec_t graph_ = nullptr;
    int graph_integrator_ = -1;
    double graph_dt_ = 0.0;
};

} // namespace ob
