// Direct O(N^2) force sum on sm_100a.
//
// Replaces the reference's direct_kernel (src/solvers/cuda_direct_kernel.cu:87-184)
// and the CPU DirectSolver it mirrors (src/solvers/direct_solver.cpp:20-80).
// The force law is the reference's Plummer-softened one,
// a_i = sum_{j != i} m_j d_ij (|d_ij|^2 + eps^2)^{-3/2}
// (include/orrery/core/softening.hpp:83-100), with G = 1.
//
// Layout and schedule (FP32 and split forms):
//   * sources are packed once per evaluation into float4 (x, y, z, m), padded
//     with zero-mass entries to a whole number of tiles;
//   * a CTA owns THREADS*R targets held in registers (R per thread) and walks a
//     contiguous range of source tiles, each 512-particle tile brought into
//     shared memory by one 1-D bulk copy (cp.async.bulk) on an mbarrier,
//     double-buffered so the next tile lands while this one is summed;
//   * every thread reads the same source at the same time, so each float4 read
//     is a shared-memory broadcast amortised over the R targets of the thread;
//   * tiles run a branch-free loop; with softening the target's own entry and
//     the zero-mass padding add exactly zero (self_term_vanishes), and
//     without it the tiles that hold them select zero mass for j == i and
//     j >= n, as the reference kernel masks (cuda_direct_kernel.cu:155-160);
//   * when the targets alone cannot fill 148 SMs, S CTAs of one thread-block
//     cluster split the source range and their partial sums are reduced through
//     distributed shared memory in a fixed rank order (deterministic).
#include <cooperative_groups.h>
#include <type_traits>

#include "common.cuh"
#include "runtime.hpp"
#include "internal.hpp"
#include "split_math.cuh"

namespace cg = cooperative_groups;

namespace ob {
namespace {

struct DirectArgs {
    const float4 *hi;
    const float4 *lo;
    uint32_t n;
    uint32_t padded;
    float eps2;
    double *ax;
    double *ay;
    double *az;
    unsigned *status;
};

// Range of source tiles [tb, te) handled by split rank `rank`.
__device__ __forceinline__ void source_tiles(uint32_t n, uint32_t split, uint32_t rank,
                                             uint32_t &tb, uint32_t &te) {
    const uint32_t tiles = ceil_div(n, kDirectTile);
    const uint32_t per = ceil_div(tiles, split);
    tb = min(rank * per, tiles);
    te = min(tb + per, tiles);
}

// Sources per unrolled step of the tile loop: a thread with a single target
// pair (the shapes for small systems, few warps per SM) gets more independent
// chains to overlap.
template <int P> constexpr int kSourceUnroll = P == 1 ? 4 : 2;

// Tiles holding the CTA's own targets or padding need no masks when those
// entries add exactly zero. A target's own entry is its packed position, so
// d = 0 exactly and r2 = eps2, and its term is f * 0 = 0 whenever
// f = (m y)(y y) at r2 = eps2 is finite; padded entries (zero mass, at the
// origin) have r2 >= eps2 and give (0 y)(y y) = 0. The masked loop adds f = 0
// for the same entries in the same order, so both loops give the same sums.
// `f_self` is that f for one target, computed as the loop computes it.
__device__ __forceinline__ bool self_term_vanishes(float eps2, float f_self) {
    return eps2 >= 1.17549435e-38f && isfinite(f_self); // eps2 normal: no flush to zero
}

// Source groups. With K > 1 the threads of a CTA form K groups of TP =
// THREADS / K: thread tid serves target lane tid % TP over the sources of
// slice tid / TP of every tile (kDirectTile / K consecutive sources), so a
// small system gets K times the warps. The K partial sums of a target are
// added in slice order, so the result does not depend on scheduling.
template <int THREADS, int K> struct SourceGroups {
    static_assert(THREADS % K == 0 && (THREADS / K) % 32 == 0, "groups are whole warps");
    static_assert(kDirectTile % K == 0, "a tile splits evenly");
    static constexpr uint32_t lanes = THREADS / K;       // target lanes per group
    static constexpr uint32_t sources = kDirectTile / K; // sources per slice of a tile
};

// Shared-memory type of the CTA's per-target sums: FP32 sums pass through
// exactly as float when a CTA has one group; group sums are FP64.
template <int K, typename T> using PartialType = std::conditional_t<K == 1, T, double>;

// Writes the CTA's per-target sums, reducing across the cluster when split.
// `partial` holds 3*BT values of type T laid out [component][slot] (K*3*BT
// doubles, one block per group, when K > 1). Target slot r*TP + lane.
template <int THREADS, int R, int K, typename T>
__device__ __forceinline__ void finish_targets(const DirectArgs &a, uint32_t t0, T *partial,
                                               const double (&sx)[R], const double (&sy)[R],
                                               const double (&sz)[R]) {
    constexpr uint32_t TP = SourceGroups<THREADS, K>::lanes;
    constexpr uint32_t BT = TP * R;
    const uint32_t split = gridDim.x;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid % TP;
    const uint32_t group = tid / TP;
    if (K == 1 && split == 1) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t i = t0 + r * THREADS + tid;
            if (i < a.n) {
                a.ax[i] = sx[r];
                a.ay[i] = sy[r];
                a.az[i] = sz[r];
            }
        }
        return;
    }
    if constexpr (K == 1) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t slot = r * THREADS + tid;
            partial[slot] = static_cast<T>(sx[r]);
            partial[BT + slot] = static_cast<T>(sy[r]);
            partial[2 * BT + slot] = static_cast<T>(sz[r]);
        }
    } else {
        static_assert(sizeof(T) == sizeof(double), "group sums are FP64");
        // Each group's sums in its own block, then added in group order into
        // block 0 (each slot by one thread, which reads every group's value of
        // a component before it overwrites block 0's).
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t slot = r * TP + lane;
            partial[(group * 3 + 0) * BT + slot] = sx[r];
            partial[(group * 3 + 1) * BT + slot] = sy[r];
            partial[(group * 3 + 2) * BT + slot] = sz[r];
        }
        __syncthreads();
        for (uint32_t slot = tid; slot < BT; slot += THREADS) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
#pragma unroll
                for (int g = 0; g < K; ++g) {
                    s += partial[(g * 3 + c) * BT + slot];
                }
                partial[c * BT + slot] = s;
            }
        }
        __syncthreads();
        if (split == 1) {
            for (uint32_t slot = tid; slot < BT; slot += THREADS) {
                const uint32_t i = t0 + slot;
                if (i < a.n) {
                    a.ax[i] = partial[slot];
                    a.ay[i] = partial[BT + slot];
                    a.az[i] = partial[2 * BT + slot];
                }
            }
            return;
        }
    }
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    const uint32_t rank = blockIdx.x;
    const uint32_t per = BT / split;
    for (uint32_t k = tid; k < per; k += THREADS) {
        const uint32_t slot = rank * per + k;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (uint32_t q = 0; q < split; ++q) {
            const T *remote = cluster.map_shared_rank(partial, q);
            s0 += static_cast<double>(remote[slot]);
            s1 += static_cast<double>(remote[BT + slot]);
            s2 += static_cast<double>(remote[2 * BT + slot]);
        }
        const uint32_t i = t0 + slot;
        if (i < a.n) {
            a.ax[i] = s0;
            a.ay[i] = s1;
            a.az[i] = s2;
        }
    }
    cluster.sync();
}

// Sources of the FP32 kernel are stored pre-duplicated, two float4 per
// particle: (x, x, y, y) and (z, z, m, m), so that each half is already a
// packed FP32x2 operand for a pair of targets and no register moves are needed.
template <int THREADS, int R, int K>
__global__ void __launch_bounds__(THREADS) direct_f32_kernel(const DirectArgs a) {
    static_assert(R % 2 == 0, "targets are processed in packed pairs");
    constexpr int P = R / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr uint32_t TP = SourceGroups<THREADS, K>::lanes;
    constexpr uint32_t JS = SourceGroups<THREADS, K>::sources;
    constexpr uint32_t BT = TP * R;
    using PT = PartialType<K, float>;
    float4 *tiles = reinterpret_cast<float4 *>(smem); // 2 buffers x 2*kDirectTile
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 4 * kDirectTile * sizeof(float4));
    PT *partial = reinterpret_cast<PT *>(bars + 2);

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid % TP;
    const uint32_t jb = (tid / TP) * JS; // this thread's slice of every tile
    const uint32_t t0 = blockIdx.y * BT;
    const float2 eps2 = make_float2(a.eps2, a.eps2);

    // Target r = 2p + h is slot (2p + h) * TP + lane; pair p packs h = 0, 1.
    float2 nx[P], ny[P], nz[P], ax[P], ay[P], az[P];
    const float y_self = rsqrt_approx(a.eps2);
    bool vanish = true;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const float4 u0 = a.hi[2ull * (t0 + (2 * p) * TP + lane)];
        const float4 u1 = a.hi[2ull * (t0 + (2 * p) * TP + lane) + 1];
        const float4 v0 = a.hi[2ull * (t0 + (2 * p + 1) * TP + lane)];
        const float4 v1 = a.hi[2ull * (t0 + (2 * p + 1) * TP + lane) + 1];
        nx[p] = make_float2(-u0.x, -v0.x);
        ny[p] = make_float2(-u0.z, -v0.z);
        nz[p] = make_float2(-u1.x, -v1.x);
        ax[p] = ay[p] = az[p] = make_float2(0.0f, 0.0f);
        const float2 ys = make_float2(y_self, y_self);
        const float2 f_self = __fmul2_rn(__fmul2_rn(make_float2(u1.z, v1.z), ys), __fmul2_rn(ys, ys));
        vanish = vanish && self_term_vanishes(a.eps2, f_self.x) &&
                 self_term_vanishes(a.eps2, f_self.y);
    }

    uint32_t tb, te;
    source_tiles(a.n, gridDim.x, blockIdx.x, tb, te);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    const bool unmasked = __syncthreads_and(vanish ? 1 : 0) != 0;
    constexpr uint32_t tile_bytes = 2 * kDirectTile * sizeof(float4);
    auto stage = [&](uint32_t k, uint32_t buf) {
        mbar_arrive_expect_tx(&bars[buf], tile_bytes);
        bulk_copy_g2s(tiles + buf * 2 * kDirectTile,
                      a.hi + 2ull * static_cast<size_t>(k) * kDirectTile, tile_bytes, &bars[buf]);
    };
    if (tid == 0) {
        for (uint32_t k = tb; k < min(tb + 2, te); ++k) {
            stage(k, k - tb);
        }
    }

    bool ok = true;
    for (uint32_t k = tb; k < te; ++k) {
        const uint32_t it = k - tb;
        const uint32_t buf = it & 1u;
        if (ok) {
            ok = mbar_wait_bounded(&bars[buf], (it >> 1) & 1u, a.status);
        }
        if (ok) {
            const float4 *tile = tiles + buf * 2 * kDirectTile;
            const uint32_t j0 = k * kDirectTile;
            const bool masked = !unmasked && ((j0 + kDirectTile > a.n) ||
                                              (j0 < t0 + BT && t0 < j0 + kDirectTile));
            if (!masked) {
#pragma unroll(kSourceUnroll<P>)
                for (uint32_t jj = jb; jj < jb + JS; ++jj) {
                    const float4 s0 = tile[2 * jj];     // (x, x, y, y)
                    const float4 s1 = tile[2 * jj + 1]; // (z, z, m, m)
                    const float2 sx = make_float2(s0.x, s0.y);
                    const float2 sy = make_float2(s0.z, s0.w);
                    const float2 sz = make_float2(s1.x, s1.y);
                    const float2 sm = make_float2(s1.z, s1.w);
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        const float2 dx = __fadd2_rn(sx, nx[p]);
                        const float2 dy = __fadd2_rn(sy, ny[p]);
                        const float2 dz = __fadd2_rn(sz, nz[p]);
                        float2 r2 = __ffma2_rn(dx, dx, eps2);
                        r2 = __ffma2_rn(dy, dy, r2);
                        r2 = __ffma2_rn(dz, dz, r2);
                        const float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                        const float2 f = __fmul2_rn(__fmul2_rn(sm, inv), __fmul2_rn(inv, inv));
                        ax[p] = __ffma2_rn(f, dx, ax[p]);
                        ay[p] = __ffma2_rn(f, dy, ay[p]);
                        az[p] = __ffma2_rn(f, dz, az[p]);
                    }
                }
            } else {
                for (uint32_t jj = jb; jj < jb + JS; ++jj) {
                    const float4 s0 = tile[2 * jj];
                    const float4 s1 = tile[2 * jj + 1];
                    const uint32_t j = j0 + jj;
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        const uint32_t i0 = t0 + (2 * p) * TP + lane;
                        const uint32_t i1 = i0 + TP;
                        const bool skip0 = (j == i0) || (j >= a.n);
                        const bool skip1 = (j == i1) || (j >= a.n);
                        const float2 dx = __fadd2_rn(make_float2(s0.x, s0.y), nx[p]);
                        const float2 dy = __fadd2_rn(make_float2(s0.z, s0.w), ny[p]);
                        const float2 dz = __fadd2_rn(make_float2(s1.x, s1.y), nz[p]);
                        float2 r2 = __ffma2_rn(dx, dx, eps2);
                        r2 = __ffma2_rn(dy, dy, r2);
                        r2 = __ffma2_rn(dz, dz, r2);
                        r2.x = skip0 ? 1.0f : r2.x;
                        r2.y = skip1 ? 1.0f : r2.y;
                        const float2 w = make_float2(skip0 ? 0.0f : s1.z, skip1 ? 0.0f : s1.w);
                        const float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                        const float2 f = __fmul2_rn(__fmul2_rn(w, inv), __fmul2_rn(inv, inv));
                        ax[p] = __ffma2_rn(f, dx, ax[p]);
                        ay[p] = __ffma2_rn(f, dy, ay[p]);
                        az[p] = __ffma2_rn(f, dz, az[p]);
                    }
                }
            }
        }
        __syncthreads();
        if (tid == 0 && ok && k + 2 < te) {
            fence_proxy_async_shared();
            stage(k + 2, buf);
        }
    }

    double sx[R], sy[R], sz[R];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        sx[2 * p] = ax[p].x;
        sx[2 * p + 1] = ax[p].y;
        sy[2 * p] = ay[p].x;
        sy[2 * p + 1] = ay[p].y;
        sz[2 * p] = az[p].x;
        sz[2 * p + 1] = az[p].y;
    }
    finish_targets<THREADS, R, K, PT>(a, t0, partial, sx, sy, sz);
}

// Split (precision) form: targets r = 2p + h are packed in pairs p and every
// operation is an FP32x2 instruction (split_math.cuh). Tiles carry 512 sources
// of hi and lo parts (64 bytes per source).
template <int THREADS, int R, int K>
__global__ void __launch_bounds__(THREADS) direct_split_kernel(const DirectArgs a) {
    static_assert(R % 2 == 0, "targets are processed in packed pairs");
    constexpr int P = R / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr uint32_t TP = SourceGroups<THREADS, K>::lanes;
    constexpr uint32_t JS = SourceGroups<THREADS, K>::sources;
    constexpr uint32_t BT = TP * R;
    float4 *tiles_hi = reinterpret_cast<float4 *>(smem);     // 2 buffers x 2*kDirectTile
    float4 *tiles_lo = tiles_hi + 4 * kDirectTile;           // 2 buffers x 2*kDirectTile
    uint64_t *bars = reinterpret_cast<uint64_t *>(tiles_lo + 4 * kDirectTile);
    double *partial = reinterpret_cast<double *>(bars + 2);

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid % TP;
    const uint32_t jb = (tid / TP) * JS; // this thread's slice of every tile
    const uint32_t t0 = blockIdx.y * BT;
    const float2 eps2 = make_float2(a.eps2, a.eps2);

    SplitTargets tg[P];
    double sx[R], sy[R], sz[R];
    const float2 y_self = refined_rsqrt2(eps2);
    bool vanish = true;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const size_t i0 = t0 + (2 * p) * TP + lane;
        tg[p] = load_split_targets(a.hi, a.lo, i0, i0 + TP);
        const float2 m = make_float2(a.hi[2 * i0 + 1].z, a.hi[2 * (i0 + TP) + 1].z);
        const float2 f_self = __fmul2_rn(__fmul2_rn(m, y_self), __fmul2_rn(y_self, y_self));
        vanish = vanish && self_term_vanishes(a.eps2, f_self.x) &&
                 self_term_vanishes(a.eps2, f_self.y);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        sx[r] = sy[r] = sz[r] = 0.0;
    }

    uint32_t tb, te;
    source_tiles(a.n, gridDim.x, blockIdx.x, tb, te);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    const bool unmasked = __syncthreads_and(vanish ? 1 : 0) != 0;
    constexpr uint32_t tile_bytes = 2 * kDirectTile * sizeof(float4);
    auto stage = [&](uint32_t k, uint32_t buf) {
        mbar_arrive_expect_tx(&bars[buf], 2 * tile_bytes);
        const size_t off = 2ull * static_cast<size_t>(k) * kDirectTile;
        bulk_copy_g2s(tiles_hi + buf * 2 * kDirectTile, a.hi + off, tile_bytes, &bars[buf]);
        bulk_copy_g2s(tiles_lo + buf * 2 * kDirectTile, a.lo + off, tile_bytes, &bars[buf]);
    };
    if (tid == 0) {
        for (uint32_t k = tb; k < min(tb + 2, te); ++k) {
            stage(k, k - tb);
        }
    }

    bool ok = true;
    for (uint32_t k = tb; k < te; ++k) {
        const uint32_t it = k - tb;
        const uint32_t buf = it & 1u;
        if (ok) {
            ok = mbar_wait_bounded(&bars[buf], (it >> 1) & 1u, a.status);
        }
        if (ok) {
            const float4 *th = tiles_hi + buf * 2 * kDirectTile;
            const float4 *tl = tiles_lo + buf * 2 * kDirectTile;
            const uint32_t j0 = k * kDirectTile;
            const bool masked = !unmasked && ((j0 + kDirectTile > a.n) ||
                                              (j0 < t0 + BT && t0 < j0 + kDirectTile));
            float2 kx[P], ky[P], kz[P], cx[P], cy[P], cz[P];
#pragma unroll
            for (int p = 0; p < P; ++p) {
                kx[p] = ky[p] = kz[p] = cx[p] = cy[p] = cz[p] = make_float2(0.0f, 0.0f);
            }
            if (!masked) {
#pragma unroll(kSourceUnroll<P>)
                for (uint32_t jj = jb; jj < jb + JS; ++jj) {
                    const float4 h0 = th[2 * jj], h1 = th[2 * jj + 1];
                    const float4 l0 = tl[2 * jj], l1 = tl[2 * jj + 1];
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        float2 dx, dy, dz;
                        split_offsets(tg[p], h0, h1, l0, l1, dx, dy, dz);
                        const float2 r2 =
                            __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, eps2)));
                        const float2 y = refined_rsqrt2(r2);
                        const float2 f = __fmul2_rn(__fmul2_rn(pair_high(h1), y), __fmul2_rn(y, y));
                        kahan2(kx[p], cx[p], f, dx);
                        kahan2(ky[p], cy[p], f, dy);
                        kahan2(kz[p], cz[p], f, dz);
                    }
                }
            } else {
                for (uint32_t jj = jb; jj < jb + JS; ++jj) {
                    const float4 h0 = th[2 * jj], h1 = th[2 * jj + 1];
                    const float4 l0 = tl[2 * jj], l1 = tl[2 * jj + 1];
                    const uint32_t j = j0 + jj;
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        const uint32_t i0 = t0 + (2 * p) * TP + lane;
                        const bool skip0 = (j == i0) || (j >= a.n);
                        const bool skip1 = (j == i0 + TP) || (j >= a.n);
                        float2 dx, dy, dz;
                        split_offsets(tg[p], h0, h1, l0, l1, dx, dy, dz);
                        float2 r2 =
                            __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, eps2)));
                        r2 = make_float2(skip0 ? 1.0f : r2.x, skip1 ? 1.0f : r2.y);
                        const float2 w = make_float2(skip0 ? 0.0f : h1.z, skip1 ? 0.0f : h1.w);
                        const float2 y = refined_rsqrt2(r2);
                        const float2 f = __fmul2_rn(__fmul2_rn(w, y), __fmul2_rn(y, y));
                        kahan2(kx[p], cx[p], f, dx);
                        kahan2(ky[p], cy[p], f, dy);
                        kahan2(kz[p], cz[p], f, dz);
                    }
                }
            }
            // Fold the tile's compensated FP32 partials into FP64.
#pragma unroll
            for (int p = 0; p < P; ++p) {
                sx[2 * p] += static_cast<double>(kx[p].x) + static_cast<double>(cx[p].x);
                sx[2 * p + 1] += static_cast<double>(kx[p].y) + static_cast<double>(cx[p].y);
                sy[2 * p] += static_cast<double>(ky[p].x) + static_cast<double>(cy[p].x);
                sy[2 * p + 1] += static_cast<double>(ky[p].y) + static_cast<double>(cy[p].y);
                sz[2 * p] += static_cast<double>(kz[p].x) + static_cast<double>(cz[p].x);
                sz[2 * p + 1] += static_cast<double>(kz[p].y) + static_cast<double>(cz[p].y);
            }
        }
        __syncthreads();
        if (tid == 0 && ok && k + 2 < te) {
            fence_proxy_async_shared();
            stage(k + 2, buf);
        }
    }
    finish_targets<THREADS, R, K, double>(a, t0, partial, sx, sy, sz);
}

// FP64 direct sum in the order of accumulate_range_scalar
// (src/solvers/direct_kernel_scalar.cpp:31-59) with the split at i of
// DirectSolver::evaluate (src/solvers/direct_solver.cpp:49-56): every operation
// is an explicitly rounded FP64 intrinsic, so nothing is contracted and the
// result is bit-identical to the reference's scalar kernel.
constexpr int kF64Threads = 128;
constexpr int kF64Tile = 256;

__global__ void __launch_bounds__(kF64Threads)
    direct_f64_kernel(const double *__restrict__ x, const double *__restrict__ y,
                      const double *__restrict__ z, const double *__restrict__ m, uint32_t n,
                      double eps2, double *ax, double *ay, double *az) {
    __shared__ double tx[kF64Tile], ty[kF64Tile], tz[kF64Tile], tm[kF64Tile];
    const uint32_t i = blockIdx.x * kF64Threads + threadIdx.x;
    const bool valid = i < n;
    const double px = valid ? x[i] : 0.0;
    const double py = valid ? y[i] : 0.0;
    const double pz = valid ? z[i] : 0.0;
    double bx = 0.0, by = 0.0, bz = 0.0; // sources before i
    double fx = 0.0, fy = 0.0, fz = 0.0; // sources after i
    for (uint32_t base = 0; base < n; base += kF64Tile) {
        for (uint32_t k = threadIdx.x; k < kF64Tile; k += kF64Threads) {
            const uint32_t j = base + k;
            tx[k] = j < n ? x[j] : 0.0;
            ty[k] = j < n ? y[j] : 0.0;
            tz[k] = j < n ? z[j] : 0.0;
            tm[k] = j < n ? m[j] : 0.0;
        }
        __syncthreads();
        const uint32_t count = min(static_cast<uint32_t>(kF64Tile), n - base);
        for (uint32_t k = 0; k < count; ++k) {
            const uint32_t j = base + k;
            if (j == i) {
                continue;
            }
            const double dx = __dsub_rn(tx[k], px);
            const double dy = __dsub_rn(ty[k], py);
            const double dz = __dsub_rn(tz[k], pz);
            const double s2 =
                __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const double inv = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(s2, eps2)));
            const double f = __dmul_rn(tm[k], __dmul_rn(__dmul_rn(inv, inv), inv));
            if (j < i) {
                bx = __dadd_rn(bx, __dmul_rn(f, dx));
                by = __dadd_rn(by, __dmul_rn(f, dy));
                bz = __dadd_rn(bz, __dmul_rn(f, dz));
            } else {
                fx = __dadd_rn(fx, __dmul_rn(f, dx));
                fy = __dadd_rn(fy, __dmul_rn(f, dy));
                fz = __dadd_rn(fz, __dmul_rn(f, dz));
            }
        }
        __syncthreads();
    }
    if (valid) {
        ax[i] = __dadd_rn(bx, fx);
        ay[i] = __dadd_rn(by, fy);
        az[i] = __dadd_rn(bz, fz);
    }
}

// Packs FP64 SoA into the kernels' source layout: two float4 per particle,
// (x, x, y, y) and (z, z, m, m) rounded to FP32, and in the split form (lo
// given) two more, (x', x', y', y') and (z', z', 0, 0) with x' = x - FP32(x).
__global__ void pack_kernel(const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, const double *__restrict__ m,
                            uint32_t n, uint32_t padded, float4 *hi, float4 *lo) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < padded;
         i += gridDim.x * blockDim.x) {
        const bool real = i < n;
        const double X = real ? x[i] : 0.0, Y = real ? y[i] : 0.0, Z = real ? z[i] : 0.0;
        const float hx = __double2float_rn(X);
        const float hy = __double2float_rn(Y);
        const float hz = __double2float_rn(Z);
        const float hm = real ? __double2float_rn(m[i]) : 0.0f;
        hi[2ull * i] = make_float4(hx, hx, hy, hy);
        hi[2ull * i + 1] = make_float4(hz, hz, hm, hm);
        if (lo != nullptr) {
            // X - hx is exact in FP64; rounding it gives the low part.
            const float lx = __double2float_rn(X - static_cast<double>(hx));
            const float ly = __double2float_rn(Y - static_cast<double>(hy));
            const float lz = __double2float_rn(Z - static_cast<double>(hz));
            lo[2ull * i] = make_float4(lx, lx, ly, ly);
            lo[2ull * i + 1] = make_float4(lz, lz, 0.0f, 0.0f);
        }
    }
}

template <int THREADS, int R, int K, bool SPLIT> size_t direct_smem_bytes() {
    const size_t tiles = (SPLIT ? 8 : 4) * kDirectTile * sizeof(float4);
    // 3 sums per target: THREADS * R / K targets, one block per group.
    const size_t partial =
        3 * THREADS * R * (SPLIT ? sizeof(double) : sizeof(PartialType<K, float>));
    return tiles + 2 * sizeof(uint64_t) + partial;
}

template <int THREADS, int R, int K, bool SPLIT> auto direct_kernel_for() {
    if constexpr (SPLIT) {
        return direct_split_kernel<THREADS, R, K>;
    } else {
        return direct_f32_kernel<THREADS, R, K>;
    }
}

template <int THREADS, int R, int K, bool SPLIT>
cudaError_t launch_direct_t(const DirectArgs &args, int split, cudaStream_t stream) {
    const uint32_t bt = SourceGroups<THREADS, K>::lanes * R;
    const dim3 grid(static_cast<unsigned>(split), ceil_div(args.n, bt), 1);
    const size_t smem = direct_smem_bytes<THREADS, R, K, SPLIT>();
    auto kernel = direct_kernel_for<THREADS, R, K, SPLIT>();
    // Set once per device, on the first launch there (before any graph
    // capture reaches it: solvers evaluate once before they capture).
    static std::atomic<uint64_t> configured{0};
    const cudaError_t err = set_smem_limit_once(reinterpret_cast<const void *>(kernel),
                                                static_cast<int>(smem), configured);
    if (err != cudaSuccess) {
        return err;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(split);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args);
}

template <bool SPLIT>
cudaError_t dispatch_direct(const DirectArgs &args, const DirectConfig &c, cudaStream_t stream) {
#define OB_DIRECT_CASE(T, RR, KK)                                                                  \
    if (c.threads == T && c.targets_per_thread == RR && c.groups == KK)                            \
        return launch_direct_t<T, RR, KK, SPLIT>(args, c.split, stream);
    OB_DIRECT_CASE(64, 2, 1)
    OB_DIRECT_CASE(64, 4, 1)
    OB_DIRECT_CASE(128, 2, 1)
    OB_DIRECT_CASE(128, 4, 1)
    OB_DIRECT_CASE(256, 2, 1)
    OB_DIRECT_CASE(256, 4, 1)
    OB_DIRECT_CASE(128, 2, 2)
    OB_DIRECT_CASE(128, 2, 4)
    OB_DIRECT_CASE(256, 2, 4)
    OB_DIRECT_CASE(256, 2, 8)
    OB_DIRECT_CASE(256, 4, 4)
    OB_DIRECT_CASE(256, 4, 8)
    if constexpr (!SPLIT) {
        OB_DIRECT_CASE(128, 8, 1)
        OB_DIRECT_CASE(256, 8, 1)
    }
#undef OB_DIRECT_CASE
    return cudaErrorInvalidValue;
}

bool valid_split(int split) { return split == 1 || split == 2 || split == 4 || split == 8; }

} // namespace

uint32_t direct_padded_count(uint32_t n, const DirectConfig &config) {
    const uint32_t bt =
        static_cast<uint32_t>(config.threads * config.targets_per_thread / config.groups);
    const uint32_t unit = bt > kDirectTile ? bt : kDirectTile;
    const uint32_t padded = ceil_div(n, unit) * unit;
    return padded == 0 ? unit : padded;
}

cudaError_t pack_sources(const double *x, const double *y, const double *z, const double *m,
                         uint32_t n, uint32_t padded, float4 *hi, float4 *lo,
                         cudaStream_t stream) {
    if (padded == 0) {
        return cudaSuccess;
    }
    const uint32_t threads = 256;
    const uint32_t blocks = min(ceil_div(padded, threads), 148u * 16u);
    pack_kernel<<<blocks, threads, 0, stream>>>(x, y, z, m, n, padded, hi, lo);
    return cudaGetLastError();
}

cudaError_t launch_direct_f32(const float4 *sources, uint32_t n, uint32_t padded, float eps2,
                              double *ax, double *ay, double *az, const DirectConfig &config,
                              unsigned *status, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    if (!valid_split(config.split) || padded < direct_padded_count(n, config)) {
        return cudaErrorInvalidValue;
    }
    const DirectArgs args{sources, nullptr, n, padded, eps2, ax, ay, az, status};
    return dispatch_direct<false>(args, config, stream);
}

cudaError_t launch_direct_split(const float4 *hi, const float4 *lo, uint32_t n, uint32_t padded,
                                float eps2, double *ax, double *ay, double *az,
                                const DirectConfig &config, unsigned *status,
                                cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    if (!valid_split(config.split) || padded < direct_padded_count(n, config)) {
        return cudaErrorInvalidValue;
    }
    const DirectArgs args{hi, lo, n, padded, eps2, ax, ay, az, status};
    return dispatch_direct<true>(args, config, stream);
}

cudaError_t launch_direct_f64(const double *x, const double *y, const double *z, const double *m,
                              uint32_t n, double eps2, double *ax, double *ay, double *az,
                              cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    direct_f64_kernel<<<ceil_div(n, kF64Threads), kF64Threads, 0, stream>>>(x, y, z, m, n, eps2,
                                                                          ax, ay, az);
    return cudaGetLastError();
}

int direct_candidates(bool split, DirectConfig *out, int capacity) {
    // (threads, targets per thread, source groups). 64-thread CTAs and source
    // groups give small systems (a few thousand particles) enough warps to
    // occupy the SMs.
    static const int split_shapes[][3] = {{64, 2, 1},  {64, 4, 1},  {128, 2, 1}, {128, 4, 1},
                                          {256, 2, 1}, {256, 4, 1}, {128, 2, 2}, {128, 2, 4},
                                          {256, 2, 4}, {256, 2, 8}, {256, 4, 4}, {256, 4, 8}};
    static const int fp32_shapes[][3] = {{64, 2, 1},  {64, 4, 1},  {128, 2, 1}, {128, 4, 1},
                                         {128, 8, 1}, {256, 2, 1}, {256, 4, 1}, {256, 8, 1},
                                         {128, 2, 2}, {128, 2, 4}, {256, 2, 4}, {256, 2, 8},
                                         {256, 4, 4}, {256, 4, 8}};
    const int(*shapes)[3] = split ? split_shapes : fp32_shapes;
    const int shape_count = split ? 12 : 14;
    static const int splits[] = {1, 2, 4, 8};
    int count = 0;
    for (int s = 0; s < shape_count; ++s) {
        for (int k = 0; k < 4; ++k) {
            if (count < capacity) {
                out[count] = DirectConfig{shapes[s][0], shapes[s][1], splits[k], shapes[s][2]};
            }
            ++count;
        }
    }
    return count;
}

DirectConfig direct_default_config(uint32_t n, bool split, int sm_count) {
    // The pattern of the shapes the autotuner picks on B200 from 1,000 to
    // 262,144 particles: 256-thread CTAs in source groups of one warp (of two
    // for the split form's four-target threads, whose registers allow fewer
    // warps), two targets per thread for small systems and four from 8192 on,
    // and the sources split across a cluster until about four CTAs per SM.
    const uint32_t sms = static_cast<uint32_t>(sm_count > 0 ? sm_count : 148);
    DirectConfig c;
    c.threads = 256;
    c.targets_per_thread = n >= 8192u ? 4 : 2;
    c.groups = split && c.targets_per_thread == 4 ? 4 : 8;
    const uint32_t bt = static_cast<uint32_t>(c.threads * c.targets_per_thread / c.groups);
    const uint32_t blocks = ceil_div(n, bt);
    const uint32_t tiles = ceil_div(n, kDirectTile);
    while (c.split < 8 && blocks * static_cast<uint32_t>(c.split) < 4u * sms &&
           static_cast<uint32_t>(c.split * 2) <= tiles) {
        c.split *= 2;
    }
    return c;
}

} // namespace ob
