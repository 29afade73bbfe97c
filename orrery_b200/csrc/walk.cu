// Barnes-Hut theta-criterion walk, one warp per 32 Morton-consecutive targets.
//
// Semantics are those of walk_tree (src/solvers/tree_walk.cpp:20-83) for every
// target separately: a cell is accepted when |com - x|^2 >= r2 in FP64 (the
// reference's test, so every accept/open decision and therefore every counter
// is exactly the reference's); an accepted cell contributes its monopole and,
// when present, quadrupole (tree_walk.hpp:129-181); an opened leaf contributes
// a pair sum that skips the target itself; an opened internal node is
// descended. Pair and cell counts are the reference's.
//
// The warp walks the union of its lanes' walks: each lane keeps its own
// cursor, the warp visits the smallest cursor any lane holds, and only lanes
// whose cursor is that node act on it. Every lane loads the same node, so the
// loads are broadcasts. When lanes open a leaf, the warp stages the leaf's
// particles in shared memory once and each interested lane sums them.
//
// Arithmetic. Positions and centres of mass are carried as FP32 hi + lo pairs
// (exact to ~2^-48 relative), so the offset to a cell comes out in FP32 to
// about 2e-7 relative with no FP64 work and no conversions. The accept test is
// decided in FP32 whenever |d^2 - r2| is clearly larger than the FP32 error
// bound (a relative margin of 4e-6 against a worst case of about 6e-7); only
// the rare cells inside the margin repeat the reference's FP64 test exactly.
// Force terms are FP32, accumulated in FP32 between leaf visits and flushed
// into FP64 per-lane sums.
#include "common.cuh"
#include "tree_kernels.hpp"

namespace ob {
namespace {

constexpr int kWalkThreads = 128;
constexpr int kWalkWarps = kWalkThreads / 32;
constexpr float kAcceptMargin = 4e-6f;

__device__ __forceinline__ uint32_t warp_min(uint32_t v) {
    return __reduce_min_sync(0xffffffffu, v);
}

// The reference's accept test in FP64 (tree_walk.cpp:44-46), for cells whose
// FP32 test fell inside the margin.
__device__ __noinline__ bool exact_accept(const DeviceNode *nodes, uint32_t cur,
                                          const double *sorted, uint32_t n, uint32_t i) {
    const double px = sorted[i];
    const double py = sorted[static_cast<size_t>(n) + i];
    const double pz = sorted[2ull * n + i];
    const double dx = __dsub_rn(nodes[cur].com_x, px);
    const double dy = __dsub_rn(nodes[cur].com_y, py);
    const double dz = __dsub_rn(nodes[cur].com_z, pz);
    const double d2 =
        __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return d2 >= nodes[cur].r2;
}

template <bool QUAD>
__global__ void __launch_bounds__(kWalkThreads)
    walk_kernel(const DeviceNode *__restrict__ nodes, const WalkNode *__restrict__ walk,
                const uint32_t *__restrict__ first_of, const float4 *__restrict__ leaf_rel,
                const double *__restrict__ sorted, const uint32_t *__restrict__ perm, uint32_t n,
                float eps2, double *ax, double *ay, double *az, const TreeMeta *meta,
                unsigned long long *counters) {
    __shared__ float4 staged[kWalkWarps][32];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t i = (blockIdx.x * kWalkWarps + warp) * 32u + lane;
    const bool active = i < n;
    const uint32_t node_count = meta->node_count;

    float pxh = 0.0f, pyh = 0.0f, pzh = 0.0f, pxl = 0.0f, pyl = 0.0f, pzl = 0.0f;
    if (active) {
        const double X = sorted[i];
        const double Y = sorted[static_cast<size_t>(n) + i];
        const double Z = sorted[2ull * n + i];
        pxh = __double2float_rn(X);
        pyh = __double2float_rn(Y);
        pzh = __double2float_rn(Z);
        pxl = __double2float_rn(X - static_cast<double>(pxh));
        pyl = __double2float_rn(Y - static_cast<double>(pyh));
        pzl = __double2float_rn(Z - static_cast<double>(pzh));
    }

    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0; // FP64 sums
    float cx32 = 0.0f, cy32 = 0.0f, cz32 = 0.0f;   // FP32 cell terms since the last flush
    uint32_t pairs = 0, cells = 0;
    uint32_t cursor = active ? 0u : 0xffffffffu;

    while (true) {
        const uint32_t cur = warp_min(cursor);
        if (cur >= node_count) {
            break;
        }
        const float4 A = walk[cur].a;
        const float4 B = walk[cur].b;
        const float4 D = walk[cur].d;
        const uint32_t next = __float_as_uint(D.z);
        const uint32_t count = __float_as_uint(D.w);
        bool open_leaf = false;
        float dx = 0.0f, dy = 0.0f, dz = 0.0f;
        if (cursor == cur) {
            dx = (A.x - pxh) + (B.x - pxl);
            dy = (A.y - pyh) + (B.y - pyl);
            dz = (A.z - pzh) + (B.z - pzl);
            const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            const float r2 = B.w;
            bool accept;
            if (d2 >= r2 * (1.0f + kAcceptMargin) && r2 > 1e-30f) {
                accept = true;
            } else if (d2 <= r2 * (1.0f - kAcceptMargin)) {
                accept = false;
            } else {
                accept = exact_accept(nodes, cur, sorted, n, i);
            }
            if (accept) {
                const float r2e = d2 + eps2;
                const float inv = rsqrt_approx(r2e);
                const float inv2 = inv * inv;
                const float f = (A.w * inv) * inv2;
                float gx = dx * f, gy = dy * f, gz = dz * f;
                if (QUAD) {
                    const float4 C = walk[cur].c; // (xx, xy, xz, yy); D.xy = (yz, zz)
                    const float qx = fmaf(C.x, dx, fmaf(C.y, dy, C.z * dz));
                    const float qy = fmaf(C.y, dx, fmaf(C.w, dy, D.x * dz));
                    const float qz = fmaf(C.z, dx, fmaf(D.x, dy, D.y * dz));
                    const float quadratic = fmaf(dx, qx, fmaf(dy, qy, dz * qz));
                    const float inv5 = (inv2 * inv2) * inv;
                    const float s = (2.5f * quadratic) * (inv5 * inv2);
                    gx = fmaf(qx, -inv5, fmaf(dx, s, gx));
                    gy = fmaf(qy, -inv5, fmaf(dy, s, gy));
                    gz = fmaf(qz, -inv5, fmaf(dz, s, gz));
                }
                cx32 += gx;
                cy32 += gy;
                cz32 += gz;
                ++cells;
                cursor = next > cur ? next : cur + 1;
            } else if (count > 0) {
                open_leaf = true;
                cursor = next > cur ? next : cur + 1;
            } else {
                cursor = cur + 1;
            }
        }
        if (__any_sync(0xffffffffu, open_leaf)) {
            const uint32_t first = first_of[cur];
            // Target relative to the leaf's centre of mass: -d.
            const float tx = -dx, ty = -dy, tz = -dz;
            const bool own = open_leaf && i >= first && i < first + count;
            const bool masked = __any_sync(0xffffffffu, own);
            float sx = 0.0f, sy = 0.0f, sz = 0.0f;
            for (uint32_t base = 0; base < count; base += 32) {
                if (base + lane < count) {
                    staged[warp][lane] = leaf_rel[first + base + lane];
                }
                __syncwarp();
                if (open_leaf) {
                    const uint32_t chunk = min(32u, count - base);
                    if (!masked) {
#pragma unroll 4
                        for (uint32_t j = 0; j < chunk; ++j) {
                            const float4 s = staged[warp][j];
                            const float ex = s.x - tx;
                            const float ey = s.y - ty;
                            const float ez = s.z - tz;
                            const float r2 = fmaf(ez, ez, fmaf(ey, ey, fmaf(ex, ex, eps2)));
                            const float inv = rsqrt_approx(r2);
                            const float f = (s.w * inv) * (inv * inv);
                            sx = fmaf(f, ex, sx);
                            sy = fmaf(f, ey, sy);
                            sz = fmaf(f, ez, sz);
                        }
                    } else {
                        for (uint32_t j = 0; j < chunk; ++j) {
                            const float4 s = staged[warp][j];
                            const bool self = first + base + j == i;
                            const float ex = s.x - tx;
                            const float ey = s.y - ty;
                            const float ez = s.z - tz;
                            const float r2 =
                                self ? 1.0f : fmaf(ez, ez, fmaf(ey, ey, fmaf(ex, ex, eps2)));
                            const float w = self ? 0.0f : s.w;
                            const float inv = rsqrt_approx(r2);
                            const float f = (w * inv) * (inv * inv);
                            sx = fmaf(f, ex, sx);
                            sy = fmaf(f, ey, sy);
                            sz = fmaf(f, ez, sz);
                        }
                    }
                }
                __syncwarp();
            }
            if (open_leaf) {
                acc_x += static_cast<double>(sx) + static_cast<double>(cx32);
                acc_y += static_cast<double>(sy) + static_cast<double>(cy32);
                acc_z += static_cast<double>(sz) + static_cast<double>(cz32);
                cx32 = cy32 = cz32 = 0.0f;
                pairs += count - (own ? 1u : 0u);
            }
        }
    }

    if (active) {
        const uint32_t j = perm[i];
        ax[j] = acc_x + static_cast<double>(cx32);
        ay[j] = acc_y + static_cast<double>(cy32);
        az[j] = acc_z + static_cast<double>(cz32);
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

cudaError_t launch_walk(const DeviceNode *nodes, const WalkNode *walk_nodes,
                        const uint32_t *first_of, const float4 *leaf_rel, const double *sorted,
                        const uint32_t *perm, uint32_t n, double eps2, bool quadrupole,
                        double *ax, double *ay, double *az, TreeMeta *meta,
                        unsigned long long *counters, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    const uint32_t blocks = ceil_div(n, kWalkThreads);
    const float eps2f = static_cast<float>(eps2);
    if (quadrupole) {
        walk_kernel<true><<<blocks, kWalkThreads, 0, stream>>>(
            nodes, walk_nodes, first_of, leaf_rel, sorted, perm, n, eps2f, ax, ay, az, meta,
            counters);
    } else {
        walk_kernel<false><<<blocks, kWalkThreads, 0, stream>>>(
            nodes, walk_nodes, first_of, leaf_rel, sorted, perm, n, eps2f, ax, ay, az, meta,
            counters);
    }
    return cudaGetLastError();
}

} // namespace ob
