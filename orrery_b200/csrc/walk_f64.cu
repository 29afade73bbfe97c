// Barnes-Hut theta walk in FP64 with the reference's arithmetic: the parity
// mode of the tree solver (precision FP64).
//
// One thread per target (Morton order) follows walk_tree
// (src/solvers/tree_walk.cpp:20-83) node for node: the stackless pre-order
// walk (accept -> next, leaf -> pair sums -> next, else the first child at
// node + 1), one FP64 accumulator per component, monopole then quadrupole
// term added separately (tree_walk.hpp:129-181), and a leaf added as a fresh
// partial sum over its index range (accumulate_range_scalar,
// src/solvers/direct_kernel_scalar.cpp:31-59), the target's own leaf as the
// two ranges either side of it. Every operation is an explicitly rounded
// intrinsic in the reference's order (no contraction), and the tree, the
// Morton order and the sorted positions are the reference's, so each
// acceleration is bit-identical to BarnesHutSolver's with its scalar leaf
// kernel. Counts are the reference's per-target pair and cell counts.
//
// The warp walks the union of its targets' walks in node order (each lane's
// cursor is its own next node), so lanes at the same node read it, and the
// same leaf sources, together.
//
// Index checks: an escape index that does not move forward or a leaf range
// past n (neither of which a valid tree produces) sets kStatusInvalid and ends
// that target's walk.
#include "common.cuh"
#include "tree_kernels.hpp"

namespace ob {
namespace {

constexpr int kWalk64Threads = 128;
constexpr uint32_t kFull = 0xffffffffu;

// softened_inverse_distance (include/orrery/core/softening.hpp:83-100).
__device__ __forceinline__ double inverse_distance(double r2, double eps2) {
    return __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(r2, eps2)));
}

// (x x + y y) + z z, as core::squared_norm.
__device__ __forceinline__ double norm2(double x, double y, double z) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// (a.x b.x + a.y b.y) + a.z b.z, as core::dot.
__device__ __forceinline__ double dot3(double ax, double ay, double az, double bx, double by,
                                       double bz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

// Pair sum over sources [begin, end) in index order, from zero.
__device__ __forceinline__ void range_sum(const double *__restrict__ sx,
                                          const double *__restrict__ sy,
                                          const double *__restrict__ sz,
                                          const double *__restrict__ sm, uint32_t begin,
                                          uint32_t end, double px, double py, double pz,
                                          double eps2, double &rx, double &ry, double &rz) {
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (uint32_t j = begin; j < end; ++j) {
        const double dx = __dsub_rn(sx[j], px);
        const double dy = __dsub_rn(sy[j], py);
        const double dz = __dsub_rn(sz[j], pz);
        const double inv = inverse_distance(norm2(dx, dy, dz), eps2);
        const double factor = __dmul_rn(sm[j], __dmul_rn(__dmul_rn(inv, inv), inv));
        ax = __dadd_rn(ax, __dmul_rn(factor, dx));
        ay = __dadd_rn(ay, __dmul_rn(factor, dy));
        az = __dadd_rn(az, __dmul_rn(factor, dz));
    }
    rx = ax;
    ry = ay;
    rz = az;
}

__global__ void __launch_bounds__(kWalk64Threads)
    walk_f64_kernel(const DeviceNode *__restrict__ nodes,
                    const DeviceQuadrupole *__restrict__ quads, const double *__restrict__ sorted,
                    const uint32_t *__restrict__ perm, uint32_t n, double eps2, double *ax,
                    double *ay, double *az, const TreeMeta *meta, unsigned long long *counters,
                    unsigned *status) {
    const uint32_t i = blockIdx.x * kWalk64Threads + threadIdx.x;
    const bool active = i < n;
    const uint32_t node_count = meta->node_count;
    const double *sx = sorted;
    const double *sy = sorted + n;
    const double *sz = sorted + 2ull * n;
    const double *sm = sorted + 3ull * n;
    unsigned long long pairs = 0, cells = 0;
    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
    const double px = active ? sx[i] : 0.0, py = active ? sy[i] : 0.0, pz = active ? sz[i] : 0.0;
    // Each lane's cursor is the next node of its own pre-order walk; the warp
    // visits the union of its lanes' walks in node order, taking the smallest
    // cursor each time, and the lanes standing at that node handle it
    // together (their node and source reads are broadcasts). A lane still
    // performs exactly its own operations in its own order.
    constexpr uint32_t kDone = 0xffffffffu;
    uint32_t node = active ? 0u : kDone;
    while (true) {
        const uint32_t cur = __reduce_min_sync(kFull, node < node_count ? node : kDone);
        if (cur == kDone) {
            break;
        }
        if (node == cur) {
            const DeviceNode cell = nodes[cur];
            const double ox = __dsub_rn(cell.com_x, px);
            const double oy = __dsub_rn(cell.com_y, py);
            const double oz = __dsub_rn(cell.com_z, pz);
            const double d2 = norm2(ox, oy, oz);
            uint32_t following;
            if (d2 >= cell.r2) {
                // The monopole and quadrupole terms each take the softened
                // inverse distance and its square of the same d2 (two calls
                // in the reference, equal to the last bit): taken once here.
                const double inv = inverse_distance(d2, eps2);
                const double inv2 = __dmul_rn(inv, inv);
                const double factor = __dmul_rn(cell.mass, __dmul_rn(inv2, inv));
                acc_x = __dadd_rn(acc_x, __dmul_rn(ox, factor));
                acc_y = __dadd_rn(acc_y, __dmul_rn(oy, factor));
                acc_z = __dadd_rn(acc_z, __dmul_rn(oz, factor));
                if (quads != nullptr) {
                    const DeviceQuadrupole q = quads[cur];
                    const double inv5 = __dmul_rn(__dmul_rn(inv2, inv2), inv);
                    const double inv7 = __dmul_rn(inv5, inv2);
                    // Q d with the symmetric tensor's six components.
                    const double cx = dot3(q.xx, q.xy, q.xz, ox, oy, oz);
                    const double cy = dot3(q.xy, q.yy, q.yz, ox, oy, oz);
                    const double cz = dot3(q.xz, q.yz, q.zz, ox, oy, oz);
                    const double quadratic = dot3(ox, oy, oz, cx, cy, cz);
                    const double scale = __dmul_rn(__dmul_rn(2.5, quadratic), inv7);
                    const double m5 = -inv5;
                    acc_x = __dadd_rn(acc_x, __dadd_rn(__dmul_rn(cx, m5), __dmul_rn(ox, scale)));
                    acc_y = __dadd_rn(acc_y, __dadd_rn(__dmul_rn(cy, m5), __dmul_rn(oy, scale)));
                    acc_z = __dadd_rn(acc_z, __dadd_rn(__dmul_rn(cz, m5), __dmul_rn(oz, scale)));
                }
                ++cells;
                following = cell.next;
            } else if (cell.count > 0) {
                const uint32_t begin = cell.first;
                if (begin > n || cell.count > n - begin) {
                    atomicOr(status, kStatusInvalid);
                    following = kDone;
                } else {
                    const uint32_t end = begin + cell.count;
                    double rx, ry, rz;
                    if (i >= begin && i < end) {
                        range_sum(sx, sy, sz, sm, begin, i, px, py, pz, eps2, rx, ry, rz);
                        acc_x = __dadd_rn(acc_x, rx);
                        acc_y = __dadd_rn(acc_y, ry);
                        acc_z = __dadd_rn(acc_z, rz);
                        range_sum(sx, sy, sz, sm, i + 1, end, px, py, pz, eps2, rx, ry, rz);
                        pairs += cell.count - 1;
                    } else {
                        range_sum(sx, sy, sz, sm, begin, end, px, py, pz, eps2, rx, ry, rz);
                        pairs += cell.count;
                    }
                    acc_x = __dadd_rn(acc_x, rx);
                    acc_y = __dadd_rn(acc_y, ry);
                    acc_z = __dadd_rn(acc_z, rz);
                    following = cell.next;
                }
            } else {
                following = cur + 1;
            }
            if (following <= cur) { // a pre-order walk only moves forward
                atomicOr(status, kStatusInvalid);
                following = kDone;
            }
            node = following;
        }
        __syncwarp();
    }
    if (active) {
        const uint32_t j = perm[i];
        ax[j] = acc_x;
        ay[j] = acc_y;
        az[j] = acc_z;
    }
    for (int off = 16; off > 0; off >>= 1) {
        pairs += __shfl_down_sync(kFull, pairs, off);
        cells += __shfl_down_sync(kFull, cells, off);
    }
    if ((threadIdx.x & 31u) == 0 && (pairs | cells) != 0ull) {
        atomicAdd(&counters[0], pairs);
        atomicAdd(&counters[1], cells);
    }
}

} // namespace

cudaError_t launch_walk_f64(const DeviceNode *nodes, const DeviceQuadrupole *quads,
                            const double *sorted, const uint32_t *perm, uint32_t n, double eps2,
                            double *ax, double *ay, double *az, const TreeMeta *meta,
                            unsigned long long *counters, unsigned *status, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    const uint32_t blocks = ceil_div(n, static_cast<uint32_t>(kWalk64Threads));
    walk_f64_kernel<<<blocks, kWalk64Threads, 0, stream>>>(nodes, quads, sorted, perm, n, eps2,
                                                           ax, ay, az, meta, counters, status);
    return cudaGetLastError();
}

} // namespace ob
