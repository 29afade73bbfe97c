// Launch interface of the Barnes-Hut pipeline's kernels (sort.cu, tree.cu,
// walk.cu). Raw device pointers; every launcher enqueues on `stream` only.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "tree.hpp"

namespace ob {

// ---------------------------------------------------------------- ordering

// Radix sort geometry: 8-bit digits, 8 passes over the 63-bit codes.
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kRadixPasses = 8;
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr uint32_t kSortTile = kSortThreads * kSortItems;

// Bounding-cube reduction: blocks of the min/max pass (4 per SM); the
// partials buffer holds 6 doubles per block.
constexpr uint32_t kCubeThreads = 256;
constexpr uint32_t kCubeBlocks = 592;

// Largest particle count the onesweep status words can carry (30-bit counts).
constexpr uint32_t kMaxTreeParticles = (1u << 30) - 1;

uint32_t sort_tiles(uint32_t n);
size_t cube_partials_needed(uint32_t n);

// Bounding cube (src/solvers/morton.cpp:60-104) into meta->origin/size and
// meta->root_centre; `partials` holds cube_partials_needed() doubles and
// meta->cube_blocks_done starts at zero (the last block to finish folds the
// partials).
cudaError_t launch_bounding_cube(const double *x, const double *y, const double *z, uint32_t n,
                                 double *partials, TreeMeta *meta, cudaStream_t stream);

// Morton codes (morton.cpp:128-164) with index payload, and the eight digit
// histograms of the codes (hist: kRadixPasses x kRadix, zeroed beforehand).
cudaError_t launch_encode(const double *x, const double *y, const double *z, uint32_t n,
                          const TreeMeta *meta, unsigned long long *codes, uint32_t *indices,
                          uint32_t *hist, cudaStream_t stream);

// Exclusive scan of each pass's histogram, in place.
cudaError_t launch_scan_histograms(uint32_t *hist, cudaStream_t stream);

// One onesweep pass (stable) over digit `pass`. `lookback` holds
// sort_tiles(n) * kRadix status words for this pass and `ticket` one counter,
// both zeroed beforehand. A tile polls a predecessor's look-back word at most
// `poll_limit` times (the default is far above any legitimate wait); when the
// polls run out it sets the timeout bit in `status` and returns unscattered.
constexpr uint32_t kLookbackPollLimit = 1u << 24;
cudaError_t launch_onesweep(const unsigned long long *keys_in, const uint32_t *vals_in,
                            unsigned long long *keys_out, uint32_t *vals_out, uint32_t n,
                            int pass, const uint32_t *offsets, uint32_t *lookback,
                            uint32_t *ticket, unsigned *status, cudaStream_t stream,
                            uint32_t poll_limit = kLookbackPollLimit);

// sorted[k * n + i] = source_k[perm[i]] for x, y, z, m.
cudaError_t launch_gather(const double *x, const double *y, const double *z, const double *m,
                          const uint32_t *perm, uint32_t n, double *sorted, cudaStream_t stream);

// Exclusive scan of n uint32 values into out[0..n] (out[n] = total). `scratch`
// holds scan_partials_needed(n) words.
size_t scan_partials_needed(uint32_t n);
cudaError_t launch_exclusive_scan(const uint32_t *in, uint32_t *out, uint32_t n,
                                  uint32_t *scratch, cudaStream_t stream);

// ------------------------------------------------------------------ octree

// Per sorted particle b: the number of octree nodes whose first particle is b.
cudaError_t launch_layout_count(const unsigned long long *codes, uint32_t n, uint32_t leaf_cap,
                                uint32_t *counts, cudaStream_t stream);

// Writes the node records (escape, first, count, level, parent), counts each
// internal node's children and lists them (in arrival order) in its
// kMaxChildren slots of child_slots. `offsets` is the exclusive scan of counts.
constexpr uint32_t kMaxChildren = 8;
cudaError_t launch_layout_write(const unsigned long long *codes, uint32_t n, uint32_t leaf_cap,
                                const uint32_t *offsets, uint32_t node_capacity,
                                DeviceNode *nodes, uint32_t *children, uint32_t *child_slots,
                                TreeMeta *meta, unsigned *status, cudaStream_t stream);

// Moments bottom-up (mass, centre of mass, quadrupole, acceptance radius) and
// the leaf-relative FP32 source positions the walk reads.
cudaError_t launch_moments(const double *sorted, const unsigned long long *codes, uint32_t n,
                           DeviceNode *nodes, DeviceQuadrupole *quads, WalkNode *walk_nodes,
                           uint32_t *first_of, const uint32_t *children,
                           const uint32_t *child_slots, uint32_t *arrived, float4 *leaf_rel,
                           TreeMeta *meta, double opening_angle, uint32_t node_capacity,
                           cudaStream_t stream);

// ------------------------------------------------------------------- walk

// Accelerations written in the caller's (unsorted) order through perm;
// pair and cell counts added to counters[0] and counters[1]. stack_cap (0 =
// the walk's full per-warp stack) bounds the group traversal's stack; a warp
// whose stack fills finishes with the per-target union walk.
uint32_t walk_stack_capacity();
cudaError_t launch_walk(const DeviceNode *nodes, const WalkNode *walk_nodes,
                        const uint32_t *first_of, const float4 *leaf_rel, const double *sorted,
                        const uint32_t *perm, uint32_t n, double eps2, bool quadrupole,
                        double *ax, double *ay, double *az, TreeMeta *meta,
                        unsigned long long *counters, unsigned *status, cudaStream_t stream,
                        uint32_t stack_cap = 0);

// The FP64 walk of the parity mode (walk_f64.cu); `quads` NULL without
// quadrupoles; `sorted` = x, y, z, m in Morton order.
cudaError_t launch_walk_f64(const DeviceNode *nodes, const DeviceQuadrupole *quads,
                            const double *sorted, const uint32_t *perm, uint32_t n, double eps2,
                            double *ax, double *ay, double *az, const TreeMeta *meta,
                            unsigned long long *counters, unsigned *status, cudaStream_t stream);

} // namespace ob
