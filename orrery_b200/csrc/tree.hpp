// Barnes-Hut pipeline on the device: bounding cube, Morton keys, radix sort,
// gather, octree layout, multipole upward pass and the theta-criterion walk.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "orrery_b200.h"
#include "runtime.hpp"

namespace ob {

// One octree node, 64 bytes, read by the walk as four 16-byte loads: FP64
// centre of mass and squared acceptance radius (so the accept test of
// src/solvers/tree_walk.cpp:46 is reproduced exactly), FP64 mass, and the
// escape / particle-range fields of TreeNode (include/orrery/solvers/
// octree.hpp:104-139) narrowed to 32 bits as the reference's CudaTreeNode
// does (include/orrery/solvers/cuda_kernels.hpp:137-145).
struct alignas(16) DeviceNode {
    double com_x, com_y;
    double com_z, r2;    // r2: acceptance radius squared (+inf when theta = 0)
    double mass;
    uint32_t next;       // escape index: first node after this subtree
    uint32_t count;      // particle count if a leaf, 0 for internal nodes
    uint32_t first;      // first particle of the cell (sorted order)
    uint32_t level;      // depth of the cell (root 0)
    uint32_t parent;     // parent node (the root points at itself)
    uint32_t pad;
};
static_assert(sizeof(DeviceNode) == 64, "DeviceNode is four 16-byte words");

// The walk's compact copy of a node, four 16-byte words:
//   a = (com_x hi, com_y hi, com_z hi, mass)       FP32
//   b = (com_x lo, com_y lo, com_z lo, r2)         FP32 (r2 rounded to nearest)
//   c = (Qxx, Qxy, Qxz, Qyy)                       FP32 quadrupole
//   d = (Qyz, Qzz, link, count)                    link/count as uint32 bits:
//                                                   link is the escape index of
//                                                   an internal node and the
//                                                   first particle of a leaf
//                                                   (whose escape index is its
//                                                   own + 1); the top bit of
//                                                   count is set when the node
//                                                   has a next sibling (escape
//                                                   index < parent's)
// hi + lo carries each FP64 coordinate to ~2^-48 relative, so offsets to the
// target (also split) come out in FP32 to ~1e-7 relative without conversions.
struct alignas(16) WalkNode {
    float4 a, b, c, d;
};
constexpr uint32_t kWalkSiblingBit = 0x80000000u;
constexpr uint32_t kWalkCountMask = 0x7fffffffu;
static_assert(sizeof(WalkNode) == 64, "WalkNode is four 16-byte words");

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
    uint32_t required;  // nodes the layout needed (reported on overflow)
    uint32_t cube_blocks_done; // bounding-cube blocks finished (the last one folds)
    uint32_t reserved;
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

    // Raises the node capacity used from the next evaluation on.
    void grow_nodes(uint32_t at_least);

    // Bounds the walk's per-warp traversal stack (0 = its full capacity) from
    // the next evaluation on; a warp whose stack fills finishes with the
    // per-target union walk. For tests of that fallback.
    void set_walk_stack_cap(uint32_t cap) noexcept { walk_stack_cap_ = cap; }

    // The device scalars of the last evaluation (synchronous).
    TreeMeta meta();

    // Bumped whenever a device buffer is reallocated (captured graphs that
    // hold the old pointers must be captured again).
    uint64_t generation() const noexcept { return generation_; }

private:
    void reserve(uint32_t n);
    uint32_t nodes_for(uint32_t n) const;

    ob_solver_params params_;
    uint32_t capacity_ = 0;
    uint32_t node_capacity_ = 0;
    uint32_t grow_to_ = 0;
    uint64_t generation_ = 0;
    uint32_t last_n_ = 0;
    uint32_t walk_stack_cap_ = 0;
    int sm_count_ = 148;
    DeviceArray<unsigned long long> keys_[2];    // Morton codes (double-buffered)
    DeviceArray<uint32_t> perm_[2];              // particle index payload
    DeviceArray<uint32_t> hist_;                 // digit histograms, then offsets
    DeviceArray<uint32_t> lookback_;             // onesweep tile status words
    DeviceArray<uint32_t> tile_counter_;         // onesweep tile tickets
    DeviceArray<double> sorted_;                 // x, y, z, m in Morton order (FP64)
    DeviceArray<float4> leaf_rel_;               // FP32 position - leaf centre of mass, mass
    DeviceArray<uint32_t> node_start_;           // nodes starting at each particle + scan
    DeviceArray<uint32_t> scan_partials_;        // block sums of the scan
    DeviceArray<DeviceNode> nodes_;
    DeviceArray<DeviceQuadrupole> quads_;        // FP64 moments (parity, upward pass)
    DeviceArray<WalkNode> walk_nodes_;           // compact FP32 node records the walk reads
    DeviceArray<uint32_t> first_of_;             // first particle of each node (leaves)
    DeviceArray<uint32_t> level_lists_;          // child slots, child counts, arrival counts
    DeviceArray<TreeMeta> meta_;
    DeviceArray<double> reduce_;                 // cube min/max partials
    DeviceArray<unsigned long long> counters_;   // pair and cell counts (accumulating)
};

} // namespace ob
