// Barnes-Hut pipeline on the device: bounding cube, Morton keys, radix sort,
// gather, octree layout, multipole upward pass and the theta-criterion walk.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "orrery_b200.h"
#include "runtime.hpp"

namespace ob {

// One octree node as the walk reads it: FP64 centre of mass, mass and squared
// acceptance radius (the FP64 accept test of src/solvers/tree_walk.cpp:46 is
// reproduced exactly), FP32 geometric centre of the cell, and the escape /
// particle-range fields of TreeNode (include/orrery/solvers/octree.hpp:104-139)
// narrowed to 32 bits as the reference's CudaTreeNode does
// (include/orrery/solvers/cuda_kernels.hpp:137-145).
struct alignas(16) DeviceNode {
    double com_x, com_y, com_z;
    double mass;
    double r2;          // acceptance radius squared (+inf when theta = 0)
    uint32_t next;      // escape index: first node after this subtree
    uint32_t first;     // first particle (sorted order)
    uint32_t count;     // particle count if a leaf, 0 for internal nodes
    uint32_t level;     // depth of the cell (root 0)
    double centre_x, centre_y, centre_z; // geometric centre of the cell
    double size;        // edge length of the cell
};

// Traceless quadrupole (include/orrery/solvers/octree.hpp:89-96).
struct DeviceQuadrupole {
    double xx, xy, xz, yy, yz, zz;
};

// Scalars the pipeline keeps on the device between its kernels.
struct TreeMeta {
    double origin[3];
    double size;
    double root_centre[3];
    uint32_t node_count;
    uint32_t leaf_count;
    uint32_t depth;
    uint32_t pad;
    unsigned long long pairs;
    unsigned long long cells;
};

class TreePipeline {
public:
    explicit TreePipeline(const ob_solver_params &params);
    ~TreePipeline();
    TreePipeline(const TreePipeline &) = delete;
    TreePipeline &operator=(const TreePipeline &) = delete;

    // Enqueues the whole evaluation; records `ordered` after the Morton order
    // and gather, `built` after the octree. Never synchronises, so it can be
    // captured in a CUDA graph.
    void evaluate(uint32_t n, const double *x, const double *y, const double *z, const double *m,
                  double *ax, double *ay, double *az, unsigned *status, cudaEvent_t ordered,
                  cudaEvent_t built, bool external, cudaStream_t stream);

    ob_counts device_counts();
    void reset_counts();

    // Inspection (tests): copies the last tree and ordering to the host.
    // nodes: 5 doubles per node (mass, com xyz, r2); idx: 3 uint64 per node
    // (next, first, count); quads: 6 doubles per node or NULL.
    uint32_t node_count();
    void copy_tree(double *reals, uint64_t *idx, double *quads, uint32_t *leaf_count,
                   uint32_t *depth);
    void copy_order(uint64_t *codes, uint32_t *indices, double *origin, double *size);
    uint32_t capacity_nodes() const noexcept { return node_capacity_; }

private:
    void reserve(uint32_t n);

    ob_solver_params params_;
    uint32_t capacity_ = 0;
    uint32_t node_capacity_ = 0;
    int sm_count_ = 148;
    DeviceArray<unsigned long long> keys_[2];    // Morton codes (double-buffered)
    DeviceArray<uint32_t> perm_[2];              // particle index payload
    DeviceArray<uint32_t> hist_;                 // radix histograms
    DeviceArray<uint32_t> lookback_;             // onesweep tile status words
    DeviceArray<uint32_t> tile_counter_;         // onesweep tile ticket counters
    DeviceArray<double> sorted_;                 // x, y, z, m in Morton order (FP64)
    DeviceArray<float4> leaf_rel_;               // FP32 position - leaf centre, mass
    DeviceArray<uint32_t> node_start_;           // nodes starting at each particle (+ scan)
    DeviceArray<uint32_t> scan_partials_;        // decoupled scan tile status
    DeviceArray<uint32_t> node_of_particle_;     // leaf index of each sorted particle
    DeviceArray<DeviceNode> nodes_;
    DeviceArray<DeviceQuadrupole> quads_;
    DeviceArray<uint32_t> level_offsets_;        // nodes per level (upward pass)
    DeviceArray<uint32_t> level_lists_;          // node indices grouped by level
    DeviceArray<double> acc_sorted_;             // accelerations in Morton order
    DeviceArray<TreeMeta> meta_;
    DeviceArray<double> reduce_;                 // cube min/max partials
};

} // namespace ob
