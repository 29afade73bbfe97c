// Octree construction on the device, node for node the reference's tree.
//
// The reference builds top-down by recursion (src/solvers/octree.cpp:273-372):
// a cell is split while it holds more than leaf_capacity particles and is
// above level 21, empty octants are skipped, and nodes are emitted in
// depth-first pre-order with octants in order 0..7. This file computes the
// same node set and layout without recursion, one thread per sorted particle:
//
//   * the cells whose first particle is b are the level-L cells starting at b
//     for L above c(b), the number of leading octal digits b's code shares with
//     b-1's; those that are nodes form one contiguous run of levels, from
//     c(b)+1 (when the enclosing level-c(b) cell is split) down to the first
//     leaf;
//   * ordering all nodes by (first particle, level) is the pre-order, so a
//     node's index is the exclusive prefix sum of per-particle node counts plus
//     its rank in its run, and its escape index (TreeNode::next) is the prefix
//     sum at the end of its particle range.
//
// Moments are then formed bottom-up in one kernel: each leaf's thread sums its
// particles, and the last child to finish computes its parent (an atomic
// arrival count; no thread ever waits). All arithmetic is FP64 with explicitly
// rounded operations in the reference's order (set_leaf_moments,
// gather_moments, add_displaced_moment, acceptance_radius_squared;
// octree.cpp:75-185, 374-387), so masses, centres of mass, quadrupoles and
// acceptance radii are bit-identical to the reference's.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "tree.hpp"
#include "tree_kernels.hpp"

namespace ob {
namespace {

constexpr uint32_t kLevels = 21;
constexpr uint32_t kThreads = 256;

// Leading octal digits (levels) that codes a and b share; kLevels when equal.
__device__ __forceinline__ int shared_levels(unsigned long long a, unsigned long long b) {
    const unsigned long long x = a ^ b;
    if (x == 0ull) {
        return static_cast<int>(kLevels);
    }
    const int high = 63 - __clzll(static_cast<long long>(x));
    return 20 - high / 3;
}

__device__ __forceinline__ int common_levels(const unsigned long long *codes, uint32_t b) {
    return b == 0 ? -1 : shared_levels(codes[b], codes[b - 1]);
}

__device__ __forceinline__ unsigned long long prefix(unsigned long long code, uint32_t level) {
    return level == 0 ? 0ull : code >> (3u * (kLevels - level));
}

// First index after i whose level-`level` prefix differs from codes[i]'s.
__device__ uint32_t cell_end(const unsigned long long *codes, uint32_t n, uint32_t i,
                             uint32_t level) {
    if (level == 0) {
        return n;
    }
    const unsigned long long p = prefix(codes[i], level);
    uint32_t lo = i; // known inside
    uint32_t step = 1;
    while (lo + step < n && prefix(codes[lo + step], level) == p) {
        lo += step;
        step <<= 1;
    }
    uint32_t hi = min(lo + step, n); // first candidate outside (or n)
    while (hi - lo > 1) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (prefix(codes[mid], level) == p) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return hi;
}

// First index of the level-`level` cell containing i.
__device__ uint32_t cell_start(const unsigned long long *codes, uint32_t i, uint32_t level) {
    if (level == 0) {
        return 0;
    }
    const unsigned long long p = prefix(codes[i], level);
    uint32_t hi = i; // known inside
    uint32_t step = 1;
    while (step <= hi && prefix(codes[hi - step], level) == p) {
        hi -= step;
        step <<= 1;
    }
    // Outside candidate below hi: hi - step (or none if step > hi).
    int64_t lo = static_cast<int64_t>(hi) - static_cast<int64_t>(step);
    if (lo < 0) {
        lo = -1;
    }
    while (static_cast<int64_t>(hi) - lo > 1) {
        const uint32_t mid = static_cast<uint32_t>(lo + (static_cast<int64_t>(hi) - lo) / 2);
        if (prefix(codes[mid], level) == p) {
            hi = mid;
        } else {
            lo = mid;
        }
    }
    return hi;
}

// max(first index of the level-`level` cell holding i, i - cap): a binary
// search over the cap + 1 codes up to i (the cell is a contiguous run of the
// sorted codes).
__device__ uint32_t clipped_start(const unsigned long long *codes, uint32_t i, uint32_t level,
                                  uint32_t cap) {
    const unsigned long long code = codes[i];
    uint32_t lo = i > cap ? i - cap : 0u, hi = i; // codes[hi] is inside
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (shared_levels(codes[mid], code) >= static_cast<int>(level)) {
            hi = mid;
        } else {
            lo = mid + 1u;
        }
    }
    return lo;
}

// min(end of the level-`level` cell whose first particle is b, b + cap + 1, n):
// the exact end when the cell holds at most cap particles.
__device__ uint32_t clipped_end(const unsigned long long *codes, uint32_t n, uint32_t b,
                                uint32_t level, uint32_t cap) {
    const unsigned long long code = codes[b];
    uint32_t lo = b + 1u, hi = min(b + cap + 1u, n); // the end lies in [lo, hi]
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (shared_levels(codes[mid], code) >= static_cast<int>(level)) {
            lo = mid + 1u;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// The run of node levels starting at particle b: [lo, hi], or lo > hi for none.
// A level-L cell whose first particle is f holds more than cap particles
// exactly when codes[f + cap] exists and shares L levels with codes[f], so
// each size test is one probe rather than a search for the cell's end.
__device__ void node_run(const unsigned long long *codes, uint32_t n, uint32_t cap, uint32_t b,
                         int &c, uint32_t &lo, uint32_t &hi) {
    c = common_levels(codes, b);
    if (b > 0) {
        if (c >= static_cast<int>(kLevels)) {
            lo = 1;
            hi = 0;
            return;
        }
        // The enclosing level-c cell holds b - 1 and b and is split when it
        // holds more than cap particles; from a start clipped to b - 1 - cap
        // the probe at start + cap = b - 1 lies inside, as it should.
        const uint32_t level = static_cast<uint32_t>(c);
        const uint32_t start = clipped_start(codes, b - 1, level, cap);
        if (!(start + cap < n && shared_levels(codes[start], codes[start + cap]) >= c)) {
            lo = 1;
            hi = 0;
            return;
        }
        lo = level + 1;
    } else {
        lo = 0;
    }
    // The cells starting at b hold more than cap particles at the levels up
    // to shared_levels(codes[b], codes[b + cap]); the run ends at the first
    // level past them (or at the deepest level).
    if (b + cap >= n) {
        hi = lo;
    } else {
        const uint32_t split = static_cast<uint32_t>(shared_levels(codes[b], codes[b + cap]));
        hi = max(lo, min(split + 1u, kLevels));
    }
}

__global__ void __launch_bounds__(kThreads)
    layout_count_kernel(const unsigned long long *__restrict__ codes, uint32_t n, uint32_t cap,
                        uint32_t *counts) {
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
        int c;
        uint32_t lo, hi;
        node_run(codes, n, cap, b, c, lo, hi);
        counts[b] = lo <= hi ? hi - lo + 1 : 0u;
    }
}

__global__ void __launch_bounds__(kThreads)
    layout_write_kernel(const unsigned long long *__restrict__ codes, uint32_t n, uint32_t cap,
                        const uint32_t *__restrict__ offsets, uint32_t capacity,
                        DeviceNode *nodes, uint32_t *children, uint32_t *child_slots,
                        TreeMeta *meta, unsigned *status) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t total = offsets[n];
        meta->node_count = total <= capacity ? total : 0u;
        meta->required = total;
        if (total > capacity) {
            atomicOr(status, kStatusOverflow);
        }
    }
    if (offsets[n] > capacity) {
        return;
    }
    uint32_t leaves = 0, depth = 0;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
        int c;
        uint32_t lo, hi;
        node_run(codes, n, cap, b, c, lo, hi);
        if (lo > hi) {
            continue;
        }
        uint32_t index = offsets[b];
        uint32_t parent;
        if (b == 0) {
            parent = index; // the root is its own parent
        } else {
            // The enclosing level-c cell starts at `start`; its node is in the
            // run of `start` at rank c - (c(start) + 1).
            const uint32_t level = static_cast<uint32_t>(c);
            const uint32_t start = cell_start(codes, b - 1, level);
            const int cs = common_levels(codes, start);
            const uint32_t first_level = start == 0 ? 0u : static_cast<uint32_t>(cs + 1);
            parent = offsets[start] + (level - first_level);
        }
        for (uint32_t level = lo; level <= hi; ++level, ++index) {
            const bool leaf = level == hi;
            // A leaf above the deepest level holds at most cap particles.
            const uint32_t end = leaf && level < kLevels ? clipped_end(codes, n, b, level, cap)
                                                         : cell_end(codes, n, b, level);
            DeviceNode node;
            node.com_x = node.com_y = node.com_z = 0.0;
            node.r2 = 0.0;
            node.mass = 0.0;
            node.next = offsets[end];
            node.count = leaf ? end - b : 0u;
            node.first = b;
            node.level = level;
            node.parent = parent;
            node.pad = 0;
            nodes[index] = node;
            if (parent != index) {
                // A cell has at most eight children; their slots are filled
                // in arrival order and sorted by the moments pass.
                const uint32_t slot = atomicAdd(&children[parent], 1u);
                if (slot < kMaxChildren) {
                    child_slots[static_cast<size_t>(parent) * kMaxChildren + slot] = index;
                } else {
                    atomicOr(status, kStatusInvalid);
                }
            }
            parent = index;
            if (leaf) {
                ++leaves;
                depth = max(depth, level);
            }
        }
    }
    // Block-reduce the leaf count and depth before touching the globals.
    for (int off = 16; off > 0; off >>= 1) {
        leaves += __shfl_down_sync(0xffffffffu, leaves, off);
        depth = max(depth, __shfl_down_sync(0xffffffffu, depth, off));
    }
    if ((threadIdx.x & 31u) == 0 && leaves > 0) {
        atomicAdd(&meta->leaf_count, leaves);
        atomicMax(&meta->depth, depth);
    }
}

// Geometric centre and edge of the cell at `level` holding `code`, by the
// reference's recursion: child centre = centre +- size/4 per axis, child size
// = size/2 (octree.cpp:41-47, 305-310). Division by 4 or 2 is multiplication
// by the exact reciprocal (both give the correctly rounded quotient), so the
// divisions are written as one multiplication each.
__device__ void cell_geometry(const TreeMeta *meta, unsigned long long code, uint32_t level,
                              double c[3], double &size) {
    c[0] = meta->root_centre[0];
    c[1] = meta->root_centre[1];
    c[2] = meta->root_centre[2];
    size = meta->size;
    for (uint32_t l = 1; l <= level; ++l) {
        const uint32_t octant = static_cast<uint32_t>((code >> (3u * (kLevels - l))) & 7u);
        const double quarter = __dmul_rn(size, 0.25);
        c[0] = __dadd_rn(c[0], (octant & 4u) ? quarter : -quarter);
        c[1] = __dadd_rn(c[1], (octant & 2u) ? quarter : -quarter);
        c[2] = __dadd_rn(c[2], (octant & 1u) ? quarter : -quarter);
        size = __dmul_rn(size, 0.5);
    }
}

// add_displaced_moment (octree.cpp:75-84).
__device__ __forceinline__ void add_displaced(DeviceQuadrupole &q, double mass, double dx,
                                              double dy, double dz) {
    const double trace =
        __dmul_rn(mass, __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                  __dmul_rn(dz, dz)));
    const double m3 = __dmul_rn(3.0, mass);
    q.xx = __dadd_rn(q.xx, __dsub_rn(__dmul_rn(__dmul_rn(m3, dx), dx), trace));
    q.xy = __dadd_rn(q.xy, __dmul_rn(__dmul_rn(m3, dx), dy));
    q.xz = __dadd_rn(q.xz, __dmul_rn(__dmul_rn(m3, dx), dz));
    q.yy = __dadd_rn(q.yy, __dsub_rn(__dmul_rn(__dmul_rn(m3, dy), dy), trace));
    q.yz = __dadd_rn(q.yz, __dmul_rn(__dmul_rn(m3, dy), dz));
    q.zz = __dadd_rn(q.zz, __dsub_rn(__dmul_rn(__dmul_rn(m3, dz), dz), trace));
}

// acceptance_radius_squared (octree.cpp:374-387) of a cell with its moments.
__device__ double acceptance(const TreeMeta *meta, unsigned long long code, uint32_t level,
                             double cx, double cy, double cz, double theta) {
    double centre[3], size;
    cell_geometry(meta, code, level, centre, size);
    const double ox = __dsub_rn(cx, centre[0]);
    const double oy = __dsub_rn(cy, centre[1]);
    const double oz = __dsub_rn(cz, centre[2]);
    const double offset =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)), __dmul_rn(oz, oz)));
    if (!(theta > 0.0)) {
        return INFINITY;
    }
    const double radius = __dadd_rn(__ddiv_rn(size, theta), offset);
    return __dmul_rn(radius, radius);
}

// Sorts eight values in registers (Batcher's odd-even merge network).
__device__ __forceinline__ void sort8(uint32_t (&v)[8]) {
    constexpr int kPairs[19][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6},
                                   {5, 7}, {1, 2}, {5, 6}, {0, 4}, {1, 5}, {2, 6}, {3, 7},
                                   {2, 4}, {3, 5}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
    for (int p = 0; p < 19; ++p) {
        const uint32_t a = v[kPairs[p][0]], b = v[kPairs[p][1]];
        v[kPairs[p][0]] = min(a, b);
        v[kPairs[p][1]] = max(a, b);
    }
}

// Writes the walk's compact record of node k (see WalkNode). `sibling`: the
// node has a next sibling, i.e. its escape index lies inside its parent's
// subtree (carried in the top bit of the count word). A leaf's escape index is
// always k + 1, so a leaf's record carries its first particle in its place.
__device__ void store_walk_node(WalkNode *walk, uint32_t *first_of, uint32_t k,
                                const DeviceNode &node, const DeviceQuadrupole *q,
                                bool sibling) {
    const uint32_t count_word = node.count | (sibling ? kWalkSiblingBit : 0u);
    const uint32_t link = node.count > 0 ? node.first : node.next;
    const float hx = __double2float_rn(node.com_x);
    const float hy = __double2float_rn(node.com_y);
    const float hz = __double2float_rn(node.com_z);
    WalkNode w;
    w.a = make_float4(hx, hy, hz, __double2float_rn(node.mass));
    w.b = make_float4(__double2float_rn(__dsub_rn(node.com_x, static_cast<double>(hx))),
                      __double2float_rn(__dsub_rn(node.com_y, static_cast<double>(hy))),
                      __double2float_rn(__dsub_rn(node.com_z, static_cast<double>(hz))),
                      __double2float_rn(node.r2));
    if (q != nullptr) {
        w.c = make_float4(__double2float_rn(q->xx), __double2float_rn(q->xy),
                          __double2float_rn(q->xz), __double2float_rn(q->yy));
        w.d = make_float4(__double2float_rn(q->yz), __double2float_rn(q->zz),
                          __uint_as_float(link), __uint_as_float(count_word));
    } else {
        w.c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.d = make_float4(0.0f, 0.0f, __uint_as_float(link), __uint_as_float(count_word));
    }
    walk[k] = w;
    first_of[k] = node.first;
}

__global__ void __launch_bounds__(kThreads)
    moments_kernel(const double *__restrict__ sorted, const unsigned long long *__restrict__ codes,
                   uint32_t n, DeviceNode *nodes, DeviceQuadrupole *quads, WalkNode *walk,
                   uint32_t *first_of, const uint32_t *__restrict__ children,
                   const uint32_t *__restrict__ child_slots, uint32_t *arrived,
                   float4 *leaf_rel, TreeMeta *meta, double theta) {
    const double *X = sorted;
    const double *Y = sorted + n;
    const double *Z = sorted + 2ull * n;
    const double *M = sorted + 3ull * n;
    const uint32_t count_nodes = meta->node_count;
    const bool with_quads = quads != nullptr;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count_nodes;
         k += gridDim.x * blockDim.x) {
        if (nodes[k].count == 0) {
            continue; // internal nodes are formed by their last child
        }
        // set_leaf_moments (octree.cpp:91-135).
        const uint32_t begin = nodes[k].first;
        const uint32_t end = begin + nodes[k].count;
        double mass = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
        for (uint32_t i = begin; i < end; ++i) {
            const double pm = M[i];
            mass = __dadd_rn(mass, pm);
            wx = __dadd_rn(wx, __dmul_rn(X[i], pm));
            wy = __dadd_rn(wy, __dmul_rn(Y[i], pm));
            wz = __dadd_rn(wz, __dmul_rn(Z[i], pm));
        }
        double cx, cy, cz;
        if (mass > 0.0) {
            cx = __ddiv_rn(wx, mass);
            cy = __ddiv_rn(wy, mass);
            cz = __ddiv_rn(wz, mass);
        } else {
            cx = X[begin];
            cy = Y[begin];
            cz = Z[begin];
        }
        DeviceQuadrupole q{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (uint32_t i = begin; i < end; ++i) {
            if (with_quads) {
                add_displaced(q, M[i], __dsub_rn(X[i], cx), __dsub_rn(Y[i], cy),
                              __dsub_rn(Z[i], cz));
            }
            // Sources relative to the leaf's centre of mass, for the FP32 walk.
            leaf_rel[i] = make_float4(__double2float_rn(__dsub_rn(X[i], cx)),
                                      __double2float_rn(__dsub_rn(Y[i], cy)),
                                      __double2float_rn(__dsub_rn(Z[i], cz)),
                                      __double2float_rn(M[i]));
        }
        const uint32_t level = nodes[k].level;
        nodes[k].mass = mass;
        nodes[k].com_x = cx;
        nodes[k].com_y = cy;
        nodes[k].com_z = cz;
        nodes[k].r2 = acceptance(meta, codes[begin], level, cx, cy, cz, theta);
        if (with_quads) {
            quads[k] = q;
        }
        {
            // Escape indices and parents were written by the layout kernel.
            const uint32_t up = nodes[k].parent;
            const bool sibling = up != k && nodes[k].next < nodes[up].next;
            store_walk_node(walk, first_of, k, nodes[k], with_quads ? &q : nullptr, sibling);
        }

        // Climb while this thread completes its parent (gather_moments,
        // octree.cpp:142-185). A cell has at most 22 ancestors.
        uint32_t current = k;
        for (int climb = 0; climb < 64; ++climb) {
            __threadfence();
            const uint32_t parent = nodes[current].parent;
            if (parent == current) {
                break;
            }
            const uint32_t before = atomicAdd(&arrived[parent], 1u);
            if (before + 1 != children[parent]) {
                break;
            }
            __threadfence();
            const uint32_t stop = __ldcg(&nodes[parent].next);
            // The parent's children in index (octant) order: its slots,
            // sorted, so that their loads need no walk along escape indices.
            const uint32_t kids = min(children[parent], kMaxChildren);
            const uint4 *slots =
                reinterpret_cast<const uint4 *>(child_slots + static_cast<size_t>(parent) *
                                                                  kMaxChildren);
            const uint4 s0 = __ldcg(slots), s1 = __ldcg(slots + 1);
            uint32_t kid[kMaxChildren] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
#pragma unroll
            for (uint32_t k = 0; k < kMaxChildren; ++k) {
                kid[k] = k < kids && kid[k] < count_nodes ? kid[k] : 0xffffffffu;
            }
            sort8(kid);
            double pm = 0.0, px = 0.0, py = 0.0, pz = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
            for (uint32_t k = 0; k < kMaxChildren; ++k) {
                if (kid[k] != 0xffffffffu) {
                    const uint32_t child = kid[k];
                    const double cm = __ldcg(&nodes[child].mass);
                    const double ccx = __ldcg(&nodes[child].com_x);
                    const double ccy = __ldcg(&nodes[child].com_y);
                    const double ccz = __ldcg(&nodes[child].com_z);
                    pm = __dadd_rn(pm, cm);
                    px = __dadd_rn(px, __dmul_rn(ccx, cm));
                    py = __dadd_rn(py, __dmul_rn(ccy, cm));
                    pz = __dadd_rn(pz, __dmul_rn(ccz, cm));
                    mx = __dadd_rn(mx, ccx);
                    my = __dadd_rn(my, ccy);
                    mz = __dadd_rn(mz, ccz);
                }
            }
            double gx, gy, gz;
            if (pm > 0.0) {
                gx = __ddiv_rn(px, pm);
                gy = __ddiv_rn(py, pm);
                gz = __ddiv_rn(pz, pm);
            } else {
                const double cnt = static_cast<double>(kids == 0 ? 1u : kids);
                gx = __ddiv_rn(mx, cnt);
                gy = __ddiv_rn(my, cnt);
                gz = __ddiv_rn(mz, cnt);
            }
            if (with_quads) {
                DeviceQuadrupole moment{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (uint32_t k = 0; k < kMaxChildren; ++k) {
                    if (kid[k] != 0xffffffffu) {
                        const uint32_t child = kid[k];
                        moment.xx = __dadd_rn(moment.xx, __ldcg(&quads[child].xx));
                        moment.xy = __dadd_rn(moment.xy, __ldcg(&quads[child].xy));
                        moment.xz = __dadd_rn(moment.xz, __ldcg(&quads[child].xz));
                        moment.yy = __dadd_rn(moment.yy, __ldcg(&quads[child].yy));
                        moment.yz = __dadd_rn(moment.yz, __ldcg(&quads[child].yz));
                        moment.zz = __dadd_rn(moment.zz, __ldcg(&quads[child].zz));
                        add_displaced(moment, __ldcg(&nodes[child].mass),
                                      __dsub_rn(__ldcg(&nodes[child].com_x), gx),
                                      __dsub_rn(__ldcg(&nodes[child].com_y), gy),
                                      __dsub_rn(__ldcg(&nodes[child].com_z), gz));
                    }
                }
                quads[parent] = moment;
            }
            const uint32_t plevel = __ldcg(&nodes[parent].level);
            const uint32_t pfirst = __ldcg(&nodes[parent].first);
            nodes[parent].mass = pm;
            nodes[parent].com_x = gx;
            nodes[parent].com_y = gy;
            nodes[parent].com_z = gz;
            nodes[parent].r2 = acceptance(meta, codes[pfirst], plevel, gx, gy, gz, theta);
            {
                DeviceNode copy;
                copy.com_x = gx;
                copy.com_y = gy;
                copy.com_z = gz;
                copy.mass = pm;
                copy.r2 = nodes[parent].r2;
                copy.next = stop;
                copy.count = 0;
                copy.first = pfirst;
                const DeviceQuadrupole *pq = with_quads ? &quads[parent] : nullptr;
                const uint32_t up = __ldcg(&nodes[parent].parent);
                const bool sibling = up != parent && stop < __ldcg(&nodes[up].next);
                store_walk_node(walk, first_of, parent, copy, pq, sibling);
            }
            current = parent;
        }
    }
}

uint32_t grid_for(uint32_t n) { return std::max(1u, std::min(ceil_div(n, kThreads), 148u * 8u)); }

} // namespace

cudaError_t launch_layout_count(const unsigned long long *codes, uint32_t n, uint32_t leaf_cap,
                                uint32_t *counts, cudaStream_t stream) {
    layout_count_kernel<<<grid_for(n), kThreads, 0, stream>>>(codes, n, leaf_cap, counts);
    return cudaGetLastError();
}

cudaError_t launch_layout_write(const unsigned long long *codes, uint32_t n, uint32_t leaf_cap,
                                const uint32_t *offsets, uint32_t node_capacity,
                                DeviceNode *nodes, uint32_t *children, uint32_t *child_slots,
                                TreeMeta *meta, unsigned *status, cudaStream_t stream) {
    layout_write_kernel<<<grid_for(n), kThreads, 0, stream>>>(codes, n, leaf_cap, offsets,
                                                             node_capacity, nodes, children,
                                                             child_slots, meta, status);
    return cudaGetLastError();
}

cudaError_t launch_moments(const double *sorted, const unsigned long long *codes, uint32_t n,
                           DeviceNode *nodes, DeviceQuadrupole *quads, WalkNode *walk_nodes,
                           uint32_t *first_of, const uint32_t *children,
                           const uint32_t *child_slots, uint32_t *arrived, float4 *leaf_rel,
                           TreeMeta *meta, double opening_angle, uint32_t node_capacity,
                           cudaStream_t stream) {
    if (reinterpret_cast<uintptr_t>(child_slots) % 16u != 0u) {
        return cudaErrorMisalignedAddress; // the climb reads a node's slots as two uint4
    }
    moments_kernel<<<grid_for(node_capacity), kThreads, 0, stream>>>(
        sorted, codes, n, nodes, quads, walk_nodes, first_of, children, child_slots, arrived,
        leaf_rel, meta, opening_angle);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// TreePipeline
// ---------------------------------------------------------------------------

TreePipeline::TreePipeline(const ob_solver_params &params) : params_(params) {
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device), "SMs");
    meta_.reserve(1);
    check(cudaMemset(meta_.data(), 0, sizeof(TreeMeta)), "clearing tree scalars");
    counters_.reserve(2);
    check(cudaMemset(counters_.data(), 0, 2 * sizeof(unsigned long long)), "clearing counters");
}

TreePipeline::~TreePipeline() = default;

uint32_t TreePipeline::nodes_for(uint32_t n) const {
    const uint64_t cap = params_.leaf_capacity < 1 ? 1 : params_.leaf_capacity;
    const uint64_t estimate = 8ull * n / cap + n / 2 + 1024;
    const uint64_t bound = 22ull * n + 1;
    return static_cast<uint32_t>(std::min<uint64_t>(std::min(estimate, bound), 0xffffffffull));
}

void TreePipeline::reserve(uint32_t n) {
    if (n > kMaxTreeParticles) {
        throw Error(OB_ERROR_CAPACITY, "the tree solver handles at most 2^30 - 1 particles");
    }
    if (n > capacity_) {
        ++generation_;
        for (int k = 0; k < 2; ++k) {
            keys_[k].reserve(n);
            perm_[k].reserve(n);
        }
        sorted_.reserve(4ull * n);
        leaf_rel_.reserve(n);
        node_start_.reserve(2ull * n + 1);
        scan_partials_.reserve(scan_partials_needed(n));
        reduce_.reserve(cube_partials_needed(n));
        hist_.reserve(kRadixPasses * kRadix);
        lookback_.reserve(static_cast<size_t>(kRadixPasses) * sort_tiles(n) * kRadix);
        tile_counter_.reserve(kRadixPasses);
        capacity_ = n;
    }
    const uint32_t want = std::max(nodes_for(n), grow_to_);
    if (want > node_capacity_) {
        ++generation_;
        nodes_.reserve(want);
        if (params_.quadrupole) {
            quads_.reserve(want);
        }
        walk_nodes_.reserve(want);
        first_of_.reserve(want);
        // kMaxChildren child slots per node (first, so that a node's slots
        // start on a 16-byte boundary for their vector loads), then child
        // counts and arrival counts.
        level_lists_.reserve((kMaxChildren + 2ull) * want);
        node_capacity_ = want;
    }
}

void TreePipeline::evaluate(uint32_t n, const double *x, const double *y, const double *z,
                            const double *m, double *ax, double *ay, double *az,
                            unsigned *status, cudaEvent_t ordered, cudaEvent_t built,
                            bool external, cudaStream_t stream) {
    if (n == 0) {
        record(ordered, stream, external);
        record(built, stream, external);
        return;
    }
    reserve(n);
    last_n_ = n;
    const uint32_t tiles = sort_tiles(n);
    // Per-evaluation scalars and scratch.
    check(cudaMemsetAsync(meta_.data(), 0, sizeof(TreeMeta), stream), "clearing tree scalars");
    check(cudaMemsetAsync(hist_.data(), 0, hist_.bytes(), stream), "clearing histograms");
    check(cudaMemsetAsync(lookback_.data(), 0,
                          sizeof(uint32_t) * kRadixPasses * static_cast<size_t>(tiles) * kRadix,
                          stream),
          "clearing look-back words");
    check(cudaMemsetAsync(tile_counter_.data(), 0, sizeof(uint32_t) * kRadixPasses, stream),
          "clearing tile tickets");
    check(cudaMemsetAsync(level_lists_.data() + kMaxChildren * static_cast<size_t>(node_capacity_),
                          0, sizeof(uint32_t) * 2ull * node_capacity_, stream),
          "clearing child counts");

    // Ordering: cube, codes + histograms, eight onesweep passes, gather.
    check(launch_bounding_cube(x, y, z, n, reduce_.data(), meta_.data(), stream), "cube");
    check(launch_encode(x, y, z, n, meta_.data(), keys_[0].data(), perm_[0].data(), hist_.data(),
                        stream),
          "Morton codes");
    check(launch_scan_histograms(hist_.data(), stream), "digit offsets");
    for (int pass = 0; pass < kRadixPasses; ++pass) {
        const int src = pass & 1;
        check(launch_onesweep(keys_[src].data(), perm_[src].data(), keys_[1 - src].data(),
                              perm_[1 - src].data(), n, pass, hist_.data(),
                              lookback_.data() + static_cast<size_t>(pass) * tiles * kRadix,
                              tile_counter_.data() + pass, status, stream),
              "radix sort pass");
    }
    // Eight passes end in buffer 0.
    const unsigned long long *codes = keys_[0].data();
    const uint32_t *perm = perm_[0].data();
    check(launch_gather(x, y, z, m, perm, n, sorted_.data(), stream), "gather");
    record(ordered, stream, external);

    // Construction: layout, node offsets, records, moments.
    const uint32_t cap = static_cast<uint32_t>(std::min<uint64_t>(params_.leaf_capacity,
                                                                 0xffffffffull));
    uint32_t *counts = node_start_.data();
    uint32_t *offsets = node_start_.data() + n;
    check(launch_layout_count(codes, n, cap, counts, stream), "node counts");
    check(launch_exclusive_scan(counts, offsets, n, scan_partials_.data(), stream), "node scan");
    uint32_t *child_slots = level_lists_.data();
    uint32_t *children = child_slots + kMaxChildren * static_cast<size_t>(node_capacity_);
    uint32_t *arrived = children + node_capacity_;
    check(launch_layout_write(codes, n, cap, offsets, node_capacity_, nodes_.data(), children,
                              child_slots, meta_.data(), status, stream),
          "node layout");
    check(launch_moments(sorted_.data(), codes, n, nodes_.data(),
                         params_.quadrupole ? quads_.data() : nullptr, walk_nodes_.data(),
                         first_of_.data(), children, child_slots, arrived, leaf_rel_.data(),
                         meta_.data(), params_.opening_angle, node_capacity_, stream),
          "moments");
    record(built, stream, external);

    // Traversal: FP32 forces, or the FP64 parity walk.
    if (params_.precision == OB_PRECISION_FP64) {
        check(launch_walk_f64(nodes_.data(), params_.quadrupole ? quads_.data() : nullptr,
                              sorted_.data(), perm, n, params_.softening_squared, ax, ay, az,
                              meta_.data(), counters_.data(), status, stream),
              "FP64 tree walk");
        return;
    }
    check(launch_walk(nodes_.data(), walk_nodes_.data(), first_of_.data(), leaf_rel_.data(),
                      sorted_.data(), perm, n, params_.softening_squared,
                      params_.quadrupole != 0, ax, ay, az, meta_.data(), counters_.data(),
                      status, stream, walk_stack_cap_),
          "tree walk");
}

ob_counts TreePipeline::device_counts() {
    unsigned long long host[2] = {0, 0};
    check(cudaMemcpy(host, counters_.data(), sizeof(host), cudaMemcpyDeviceToHost),
          "reading tree counters");
    ob_counts c{};
    c.particle_particle = host[0];
    c.particle_cell = host[1];
    return c;
}

void TreePipeline::reset_counts() {
    check(cudaMemset(counters_.data(), 0, 2 * sizeof(unsigned long long)), "clearing counters");
}

TreeMeta TreePipeline::meta() {
    TreeMeta h{};
    check(cudaMemcpy(&h, meta_.data(), sizeof(TreeMeta), cudaMemcpyDeviceToHost),
          "reading tree scalars");
    return h;
}

uint32_t TreePipeline::node_count() { return meta().node_count; }

void TreePipeline::copy_tree(double *reals, uint64_t *idx, double *quads, uint32_t *leaf_count,
                             uint32_t *depth) {
    const TreeMeta h = meta();
    std::vector<DeviceNode> nodes(h.node_count);
    if (h.node_count > 0) {
        check(cudaMemcpy(nodes.data(), nodes_.data(), sizeof(DeviceNode) * h.node_count,
                         cudaMemcpyDeviceToHost),
              "copying the tree");
    }
    for (uint32_t k = 0; k < h.node_count; ++k) {
        reals[5ull * k + 0] = nodes[k].mass;
        reals[5ull * k + 1] = nodes[k].com_x;
        reals[5ull * k + 2] = nodes[k].com_y;
        reals[5ull * k + 3] = nodes[k].com_z;
        reals[5ull * k + 4] = nodes[k].r2;
        idx[3ull * k + 0] = nodes[k].next;
        // The reference sets first_particle on leaves only (octree.cpp:335-337);
        // internal nodes keep their default of 0.
        idx[3ull * k + 1] = nodes[k].count > 0 ? nodes[k].first : 0u;
        idx[3ull * k + 2] = nodes[k].count;
    }
    if (quads != nullptr && params_.quadrupole && h.node_count > 0) {
        check(cudaMemcpy(quads, quads_.data(), sizeof(DeviceQuadrupole) * h.node_count,
                         cudaMemcpyDeviceToHost),
              "copying quadrupoles");
    }
    if (leaf_count != nullptr) {
        *leaf_count = h.leaf_count;
    }
    if (depth != nullptr) {
        *depth = h.depth;
    }
}

void TreePipeline::copy_order(uint64_t *codes, uint32_t *indices, double *origin, double *size) {
    const TreeMeta h = meta();
    if (last_n_ > 0) {
        if (codes != nullptr) {
            check(cudaMemcpy(codes, keys_[0].data(), sizeof(uint64_t) * last_n_,
                             cudaMemcpyDeviceToHost),
                  "copying codes");
        }
        if (indices != nullptr) {
            check(cudaMemcpy(indices, perm_[0].data(), sizeof(uint32_t) * last_n_,
                             cudaMemcpyDeviceToHost),
                  "copying the permutation");
        }
    }
    if (origin != nullptr) {
        origin[0] = h.origin[0];
        origin[1] = h.origin[1];
        origin[2] = h.origin[2];
    }
    if (size != nullptr) {
        *size = h.size;
    }
}

void TreePipeline::grow_nodes(uint32_t at_least) { grow_to_ = std::max(grow_to_, at_least); }

} // namespace ob
