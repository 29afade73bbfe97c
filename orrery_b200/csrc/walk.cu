// Barnes-Hut theta-criterion walk, one warp per 32 Morton-consecutive targets.
//
// Semantics are those of walk_tree (src/solvers/tree_walk.cpp:20-83) for every
// target separately: a cell is accepted when |com - x|^2 >= r2 (FP64, the
// reference's operation order, so each accept/open decision and therefore
// every counter is exactly the reference's); an accepted cell contributes its
// monopole and, when present, quadrupole (tree_walk.hpp:129-181); an opened
// leaf contributes a pair sum that skips the target itself; an opened
// internal node is descended. Pair and cell counts are the reference's.
//
// The warp walks the union of its lanes' walks: each lane keeps its own
// cursor, the warp visits the smallest cursor any lane holds, and only lanes
// whose cursor is that node act on it (lanes that accepted an ancestor have
// already jumped past it). Every lane loads the same node, so the loads are
// broadcasts. When lanes open a leaf, the warp stages the leaf's particles in
// shared memory once and each interested lane sums them from there.
//
// Arithmetic: the accept test and the offset to each cell's centre of mass
// are FP64; force terms are FP32 on offsets that are already small (leaf
// sources are stored relative to their leaf's centre of mass, the target is
// taken relative to the same point), and each cell's or leaf's FP32
// contribution is added to FP64 per-lane accumulators.
#include "common.cuh"
#include "tree_kernels.hpp"

namespace ob {
namespace {

constexpr int kWalkThreads = 128;
constexpr int kWalkWarps = kWalkThreads / 32;

__device__ __forceinline__ uint32_t warp_min(uint32_t v) {
    return __reduce_min_sync(0xffffffffu, v);
}

__global__ void __launch_bounds__(kWalkThreads)
    walk_kernel(const DeviceNode *__restrict__ nodes, const float *__restrict__ quads32,
                const float4 *__restrict__ leaf_rel, const double *__restrict__ sorted,
                const uint32_t *__restrict__ perm, uint32_t n, double eps2d, double *ax,
                double *ay, double *az, const TreeMeta *meta, unsigned long long *counters) {
    __shared__ float4 staged[kWalkWarps][32];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t i = (blockIdx.x * kWalkWarps + warp) * 32u + lane;
    const bool active = i < n;
    const uint32_t node_count = meta->node_count;
    const float eps2 = static_cast<float>(eps2d);

    const double px = active ? sorted[i] : 0.0;
    const double py = active ? sorted[static_cast<size_t>(n) + i] : 0.0;
    const double pz = active ? sorted[2ull * n + i] : 0.0;

    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
    uint32_t pairs = 0, cells = 0;
    uint32_t cursor = active ? 0u : 0xffffffffu;

    while (true) {
        const uint32_t cur = warp_min(cursor);
        if (cur >= node_count) {
            break;
        }
        const DeviceNode nd = nodes[cur];
        const bool here = cursor == cur;
        bool open_leaf = false;
        float tx = 0.0f, ty = 0.0f, tz = 0.0f;
        if (here) {
            const double dx = __dsub_rn(nd.com_x, px);
            const double dy = __dsub_rn(nd.com_y, py);
            const double dz = __dsub_rn(nd.com_z, pz);
            const double d2 =
                __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            if (d2 >= nd.r2) {
                const float fx = __double2float_rn(dx);
                const float fy = __double2float_rn(dy);
                const float fz = __double2float_rn(dz);
                const float r2 = fmaf(fz, fz, fmaf(fy, fy, fmaf(fx, fx, eps2)));
                const float inv = rsqrt_approx(r2);
                const float inv2 = inv * inv;
                const float mass = __double2float_rn(nd.mass);
                const float f = (mass * inv) * inv2;
                float gx = fx * f, gy = fy * f, gz = fz * f;
                if (quads32 != nullptr) {
                    const float4 q0 = reinterpret_cast<const float4 *>(quads32)[2ull * cur];
                    const float4 q1 = reinterpret_cast<const float4 *>(quads32)[2ull * cur + 1];
                    // q0 = (xx, xy, xz, yy), q1 = (yz, zz, -, -)
                    const float cx = fmaf(q0.x, fx, fmaf(q0.y, fy, q0.z * fz));
                    const float cy = fmaf(q0.y, fx, fmaf(q0.w, fy, q1.x * fz));
                    const float cz = fmaf(q0.z, fx, fmaf(q1.x, fy, q1.y * fz));
                    const float quadratic = fmaf(fx, cx, fmaf(fy, cy, fz * cz));
                    const float inv5 = (inv2 * inv2) * inv;
                    const float inv7 = inv5 * inv2;
                    const float s = (2.5f * quadratic) * inv7;
                    gx = fmaf(cx, -inv5, fmaf(fx, s, gx));
                    gy = fmaf(cy, -inv5, fmaf(fy, s, gy));
                    gz = fmaf(cz, -inv5, fmaf(fz, s, gz));
                }
                acc_x += gx;
                acc_y += gy;
                acc_z += gz;
                ++cells;
                cursor = nd.next > cur ? nd.next : cur + 1;
            } else if (nd.count > 0) {
                open_leaf = true;
                // The target relative to the leaf's centre of mass.
                tx = -__double2float_rn(dx);
                ty = -__double2float_rn(dy);
                tz = -__double2float_rn(dz);
                cursor = nd.next > cur ? nd.next : cur + 1;
            } else {
                cursor = cur + 1;
            }
        }
        if (__any_sync(0xffffffffu, open_leaf)) {
            const uint32_t first = nd.first;
            const uint32_t count = nd.count;
            float sx = 0.0f, sy = 0.0f, sz = 0.0f;
            for (uint32_t base = 0; base < count; base += 32) {
                if (base + lane < count) {
                    staged[warp][lane] = leaf_rel[first + base + lane];
                }
                __syncwarp();
                if (open_leaf) {
                    const uint32_t chunk = min(32u, count - base);
                    for (uint32_t j = 0; j < chunk; ++j) {
                        const float4 s = staged[warp][j];
                        const bool self = first + base + j == i;
                        const float dx = s.x - tx;
                        const float dy = s.y - ty;
                        const float dz = s.z - tz;
                        const float r2 =
                            self ? 1.0f : fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
                        const float w = self ? 0.0f : s.w;
                        const float inv = rsqrt_approx(r2);
                        const float f = (w * inv) * (inv * inv);
                        sx = fmaf(f, dx, sx);
                        sy = fmaf(f, dy, sy);
                        sz = fmaf(f, dz, sz);
                    }
                }
                __syncwarp();
            }
            if (open_leaf) {
                acc_x += sx;
                acc_y += sy;
                acc_z += sz;
                const bool holds = i >= first && i < first + count;
                pairs += count - (holds ? 1u : 0u);
            }
        }
    }

    if (active) {
        const uint32_t j = perm[i];
        ax[j] = acc_x;
        ay[j] = acc_y;
        az[j] = acc_z;
    }
    unsigned long long p = pairs, c = cells;
    for (int off = 16; off > 0; off >>= 1) {
        p += __shfl_down_sync(0xffffffffu, p, off);
        c += __shfl_down_sync(0xffffffffu, c, off);
    }
    if (lane == 0 && (p | c) != 0ull) {
        atomicAdd(&counters[0], p);
        atomicAdd(&counters[1], c);
    }
}

} // namespace

cudaError_t launch_walk(const DeviceNode *nodes, const float *quads32, const float4 *leaf_rel,
                        const double *sorted, const uint32_t *perm, uint32_t n, double eps2,
                        double *ax, double *ay, double *az, TreeMeta *meta,
                        unsigned long long *counters, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    const uint32_t blocks = ceil_div(n, kWalkThreads);
    walk_kernel<<<blocks, kWalkThreads, 0, stream>>>(nodes, quads32, leaf_rel, sorted, perm, n,
                                                     eps2, ax, ay, az, meta, counters);
    return cudaGetLastError();
}

} // namespace ob
