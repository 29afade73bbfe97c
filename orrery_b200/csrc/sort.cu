// Morton ordering on the device: bounding cube, 63-bit codes, and a stable
// least-significant-digit radix sort of (code, index) in onesweep form.
//
// Parity with MortonOrdering::build (src/solvers/morton.cpp:180-197) is exact:
//   * the cube is the reference's (morton.cpp:60-104) with every FP64
//     operation explicitly rounded and min/max exact in any order;
//   * codes use the reference's grid mapping (morton.cpp:128-164), truncation
//     and clamps; x, y, z interleaved with x the high bit of each triple;
//   * a stable sort of codes whose payload starts as the identity orders ties
//     by ascending index, which is exactly std::sort on MortonKey's
//     (code, index) ordering (include/orrery/solvers/morton.hpp:155-175).
//
// The sort: one histogram pass (fused into encoding) computes all eight digit
// histograms; then each of the eight passes is a single kernel in which a CTA
// takes the next tile in launch order (ticket counter), ranks its keys stably
// with warp match operations, publishes its per-digit counts, resolves its
// global offsets by decoupled look-back over earlier tiles (every wait bounded)
// and scatters through shared memory so the global writes are contiguous runs.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "runtime.hpp"
#include "tree_kernels.hpp"

namespace ob {
namespace {

constexpr uint32_t kReduceThreads = kCubeThreads;
constexpr uint32_t kReduceBlocks = kCubeBlocks;

__device__ __forceinline__ void min_max(double v, double &lo, double &hi) {
    lo = v < lo ? v : lo;
    hi = hi < v ? v : hi;
}

// Block-wide min (k < 3) / max (k >= 3) of the six values each thread holds
// in v[]; thread k < 6 receives component k in `out`.
__device__ __forceinline__ void block_min_max(double (&v)[6], double &out) {
    __shared__ double s[6][kReduceThreads / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v[k], off);
            v[k] = k < 3 ? (o < v[k] ? o : v[k]) : (v[k] < o ? o : v[k]);
        }
        if (lane == 0) {
            s[k][warp] = v[k];
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        double r = s[k][0];
        for (uint32_t w = 1; w < kReduceThreads / 32; ++w) {
            r = k < 3 ? (s[k][w] < r ? s[k][w] : r) : (r < s[k][w] ? s[k][w] : r);
        }
        out = r;
    }
}

// The cube from the extremes (morton.cpp:60-104): edge = the largest extent
// (1 when it is not positive), centred on the box.
__device__ void write_cube(const double *ext, uint32_t n, TreeMeta *meta) {
    if (n == 0) {
        for (int a = 0; a < 3; ++a) {
            meta->origin[a] = 0.0;
            meta->root_centre[a] = 0.0;
        }
        meta->size = 0.0;
        return;
    }
    const double ex = __dsub_rn(ext[3], ext[0]);
    const double ey = __dsub_rn(ext[4], ext[1]);
    const double ez = __dsub_rn(ext[5], ext[2]);
    double size = ex;
    size = size < ey ? ey : size;
    size = size < ez ? ez : size;
    if (!(size > 0.0)) {
        size = 1.0;
    }
    const double half = __ddiv_rn(size, 2.0);
    for (int a = 0; a < 3; ++a) {
        const double centre = __ddiv_rn(__dadd_rn(ext[a], ext[3 + a]), 2.0);
        const double origin = __dsub_rn(centre, half);
        meta->origin[a] = origin;
        // BoundingCube::centre (morton.hpp:93-95): origin + size/2.
        meta->root_centre[a] = __dadd_rn(origin, half);
    }
    meta->size = size;
}

// One pass over the positions: each block writes its six extremes, and the
// last block to finish (an atomic count in meta) folds all blocks' partials
// with the whole block and writes the cube. Min and max are exact, so the
// order of the fold does not change the result.
__global__ void __launch_bounds__(kReduceThreads)
    cube_kernel(const double *__restrict__ x, const double *__restrict__ y,
                const double *__restrict__ z, uint32_t n, double *partials, TreeMeta *meta) {
    double v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        min_max(x[i], v[0], v[3]);
        min_max(y[i], v[1], v[4]);
        min_max(z[i], v[2], v[5]);
    }
    double mine = 0.0;
    block_min_max(v, mine);
    __shared__ bool last;
    if (threadIdx.x < 6) {
        partials[blockIdx.x * 6 + threadIdx.x] = mine;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        last = atomicAdd(&meta->cube_blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) {
        return;
    }
    __threadfence();
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        v[k] = k < 3 ? INFINITY : -INFINITY;
    }
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            // Empty blocks hold (+inf, -inf): lows only lower, highs only raise.
            const double p = __ldcg(partials + b * 6 + k);
            v[k] = k < 3 ? (p < v[k] ? p : v[k]) : (v[k] < p ? p : v[k]);
        }
    }
    __syncthreads(); // block_min_max's shared array is reused
    __shared__ double ext[6];
    double folded = 0.0;
    block_min_max(v, folded);
    if (threadIdx.x < 6) {
        ext[threadIdx.x] = folded;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        write_cube(ext, n, meta);
    }
}

// Dilation by table: each 7-bit chunk of a grid coordinate maps to 21 bits
// with its bits three apart; three chunks make the 63-bit interleave slot.
__device__ __forceinline__ unsigned long long dilate(const unsigned long long *table,
                                                     uint32_t v) {
    return table[v & 127u] | (table[(v >> 7) & 127u] << 21) | (table[(v >> 14) & 127u] << 42);
}

__device__ __forceinline__ uint32_t to_grid(double coordinate, double origin, double scale) {
    const double cell = __dmul_rn(__dsub_rn(coordinate, origin), scale);
    if (!(cell > 0.0)) {
        return 0u;
    }
    if (cell >= 2097152.0) {
        return 2097151u;
    }
    return __double2uint_rz(cell);
}

__global__ void __launch_bounds__(kReduceThreads)
    encode_kernel(const double *__restrict__ x, const double *__restrict__ y,
                  const double *__restrict__ z, uint32_t n, const TreeMeta *meta,
                  unsigned long long *codes, uint32_t *indices, uint32_t *hist) {
    __shared__ unsigned long long table[128];
    __shared__ uint32_t local[kRadixPasses * kRadix];
    for (uint32_t k = threadIdx.x; k < 128; k += blockDim.x) {
        unsigned long long d = 0;
        for (int b = 0; b < 7; ++b) {
            d |= static_cast<unsigned long long>((k >> b) & 1u) << (3 * b);
        }
        table[k] = d;
    }
    for (uint32_t k = threadIdx.x; k < kRadixPasses * kRadix; k += blockDim.x) {
        local[k] = 0;
    }
    __syncthreads();
    const double size = meta->size;
    const bool degenerate = !(size > 0.0);
    const double scale = degenerate ? 0.0 : __ddiv_rn(2097152.0, size);
    const double ox = meta->origin[0], oy = meta->origin[1], oz = meta->origin[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned long long code = 0;
        if (!degenerate) {
            code = (dilate(table, to_grid(x[i], ox, scale)) << 2) |
                   (dilate(table, to_grid(y[i], oy, scale)) << 1) |
                   dilate(table, to_grid(z[i], oz, scale));
        }
        codes[i] = code;
        indices[i] = i;
#pragma unroll
        for (int p = 0; p < kRadixPasses; ++p) {
            atomicAdd(&local[p * kRadix + ((code >> (kRadixBits * p)) & (kRadix - 1))], 1u);
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < kRadixPasses * kRadix; k += blockDim.x) {
        if (local[k] != 0) {
            atomicAdd(&hist[k], local[k]);
        }
    }
}

__global__ void scan_histograms_kernel(uint32_t *hist) {
    __shared__ uint32_t s[kRadix];
    uint32_t *h = hist + blockIdx.x * kRadix;
    const uint32_t t = threadIdx.x;
    s[t] = h[t];
    __syncthreads();
    for (uint32_t off = 1; off < kRadix; off <<= 1) {
        const uint32_t v = t >= off ? s[t - off] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    h[t] = t == 0 ? 0u : s[t - 1];
}

// Status words of the look-back: 2-bit flag over a 30-bit count.
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;

__device__ __forceinline__ uint32_t load_volatile(const uint32_t *p) {
    return *reinterpret_cast<const volatile uint32_t *>(p);
}

__device__ __forceinline__ void store_volatile(uint32_t *p, uint32_t v) {
    *reinterpret_cast<volatile uint32_t *>(p) = v;
}

constexpr uint32_t kWarps = kSortThreads / 32;

// One onesweep pass. CTAs are persistent: each takes tiles by atomic ticket
// (so every tile's predecessors were taken by CTAs that are running or done,
// which publish without waiting on later tiles) until the tiles run out.
__global__ void __launch_bounds__(kSortThreads, 5)
    onesweep_kernel(const unsigned long long *__restrict__ keys_in,
                    const uint32_t *__restrict__ vals_in, unsigned long long *keys_out,
                    uint32_t *vals_out, uint32_t n, uint32_t tiles, uint32_t shift,
                    const uint32_t *__restrict__ offsets, uint32_t *lookback, uint32_t *ticket,
                    unsigned *status, uint32_t poll_limit) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long *s_keys = reinterpret_cast<unsigned long long *>(smem);
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + kSortTile);
    uint32_t *s_warp = s_vals + kSortTile;            // [kWarps][kRadix] counts, then prefixes
    uint32_t *s_start = s_warp + kWarps * kRadix;     // tile-local digit start
    uint32_t *s_base = s_start + kRadix;              // global output base per digit
    uint32_t *s_tile = s_base + kRadix;

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t *hist = s_warp + warp * kRadix;
    while (true) {
        if (tid == 0) {
            *s_tile = atomicAdd(ticket, 1u);
        }
        for (uint32_t k = tid; k < kWarps * kRadix; k += kSortThreads) {
            s_warp[k] = 0;
        }
        __syncthreads();
        const uint32_t tile = *s_tile;
        if (tile >= tiles) {
            return; // uniform: every thread read the same ticket
        }
        const uint32_t base = tile * kSortTile;

        // Warp-striped load: the tile order of (warp, item, lane) is this order.
        unsigned long long key[kSortItems];
        uint32_t val[kSortItems], digit[kSortItems], rank[kSortItems];
#pragma unroll
        for (int it = 0; it < kSortItems; ++it) {
            const uint32_t i = base + warp * (kSortItems * 32) + it * 32 + lane;
            const bool valid = i < n;
            key[it] = valid ? keys_in[i] : 0ull;
            val[it] = valid ? vals_in[i] : 0u;
            digit[it] = valid ? static_cast<uint32_t>((key[it] >> shift) & (kRadix - 1)) : kRadix;
            // Stable warp-local rank: earlier items first, then lower lanes.
            const uint32_t peers = __match_any_sync(0xffffffffu, digit[it]);
            const uint32_t before = __popc(peers & lt_mask);
            const uint32_t running = valid ? hist[digit[it]] : 0u;
            __syncwarp();
            if (valid && before == 0) {
                hist[digit[it]] = running + __popc(peers);
            }
            __syncwarp();
            rank[it] = running + before;
        }
        __syncthreads();

        // Thread t owns digit t: tile count, warp prefixes, publish, look back.
        const uint32_t d = tid;
        uint32_t count = 0;
        for (uint32_t w = 0; w < kWarps; ++w) {
            const uint32_t c = s_warp[w * kRadix + d];
            s_warp[w * kRadix + d] = count;
            count += c;
        }
        uint32_t *mine = lookback + static_cast<size_t>(tile) * kRadix + d;
        if (tile == 0) {
            store_volatile(mine, kFlagPrefix | count);
        } else {
            store_volatile(mine, kFlagAggregate | count);
        }
        uint32_t exclusive = 0;
        bool ok = true;
        if (tile > 0) {
            int64_t j = static_cast<int64_t>(tile) - 1;
            uint32_t polls = 0;
            while (j >= 0) {
                const uint32_t s = load_volatile(lookback + static_cast<size_t>(j) * kRadix + d);
                const uint32_t flag = s & ~kCountMask;
                if (flag == 0u) {
                    if (++polls > poll_limit) {
                        atomicOr(status, kStatusTimeout);
                        ok = false;
                        break;
                    }
                    continue;
                }
                exclusive += s & kCountMask;
                if (flag == kFlagPrefix) {
                    break;
                }
                --j;
            }
            __threadfence();
            store_volatile(mine, kFlagPrefix | ((exclusive + count) & kCountMask));
        }
        s_base[d] = offsets[d] + exclusive;

        // Exclusive scan of the tile's digit counts gives each digit's run start.
        s_start[d] = count;
        __syncthreads();
        for (uint32_t off = 1; off < kRadix; off <<= 1) {
            const uint32_t v = d >= off ? s_start[d - off] : 0u;
            __syncthreads();
            s_start[d] += v;
            __syncthreads();
        }
        s_start[d] -= count;
        __syncthreads();
        if (!__syncthreads_and(ok ? 1 : 0)) {
            return; // a timed-out tile stays unscattered; the CTA takes no more tiles
        }

        // Place keys in shared memory in digit order, then write contiguous runs.
#pragma unroll
        for (int it = 0; it < kSortItems; ++it) {
            if (digit[it] < kRadix) {
                const uint32_t pos =
                    s_start[digit[it]] + s_warp[warp * kRadix + digit[it]] + rank[it];
                s_keys[pos] = key[it];
                s_vals[pos] = val[it];
            }
        }
        __syncthreads();
        const uint32_t valid_in_tile = n > base ? min(kSortTile, n - base) : 0u;
        for (uint32_t k = tid; k < valid_in_tile; k += kSortThreads) {
            const unsigned long long kk = s_keys[k];
            const uint32_t dd = static_cast<uint32_t>((kk >> shift) & (kRadix - 1));
            const uint32_t dst = s_base[dd] + (k - s_start[dd]);
            keys_out[dst] = kk;
            vals_out[dst] = s_vals[k];
        }
        __syncthreads(); // the next tile reuses the shared arrays
    }
}

__global__ void gather_kernel(const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const double *__restrict__ m,
                              const uint32_t *__restrict__ perm, uint32_t n, double *sorted) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t j = perm[i];
        sorted[i] = x[j];
        sorted[static_cast<size_t>(n) + i] = y[j];
        sorted[2ull * n + i] = z[j];
        sorted[3ull * n + i] = m[j];
    }
}

// Three-phase exclusive scan: block sums, a scan of the sums, block scans.
constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *s, uint32_t &total) {
    const uint32_t t = threadIdx.x;
    s[t] = v;
    __syncthreads();
    for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
        const uint32_t u = t >= off ? s[t - off] : 0u;
        __syncthreads();
        s[t] += u;
        __syncthreads();
    }
    total = s[blockDim.x - 1];
    const uint32_t r = s[t] - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_reduce_kernel(const uint32_t *__restrict__ in, uint32_t n, uint32_t *sums) {
    __shared__ uint32_t s[kScanThreads];
    const uint32_t base = blockIdx.x * kScanTile;
    uint32_t local = 0;
    for (uint32_t k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k * kScanThreads + threadIdx.x;
        local += i < n ? in[i] : 0u;
    }
    uint32_t total;
    block_exclusive_scan(local, s, total);
    if (threadIdx.x == 0) {
        sums[blockIdx.x] = total;
    }
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(uint32_t *sums, uint32_t blocks) {
    __shared__ uint32_t s[1024];
    uint32_t carry = 0;
    for (uint32_t start = 0; start < blocks; start += 1024) {
        const uint32_t i = start + threadIdx.x;
        const uint32_t v = i < blocks ? sums[i] : 0u;
        uint32_t total;
        const uint32_t r = block_exclusive_scan(v, s, total);
        if (i < blocks) {
            sums[i] = carry + r;
        }
        carry += total;
    }
    if (threadIdx.x == 0) {
        sums[blocks] = carry;
    }
}

__global__ void __launch_bounds__(kScanThreads)
    scan_apply_kernel(const uint32_t *__restrict__ in, uint32_t *out, uint32_t n,
                      const uint32_t *sums, uint32_t blocks) {
    __shared__ uint32_t s[kScanThreads];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (uint32_t k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        local += v[k];
    }
    uint32_t total;
    uint32_t running = sums[blockIdx.x] + block_exclusive_scan(local, s, total);
#pragma unroll
    for (uint32_t k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k;
        if (i < n) {
            out[i] = running;
        }
        running += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out[n] = sums[blocks];
    }
}

size_t onesweep_smem() {
    return kSortTile * (sizeof(unsigned long long) + sizeof(uint32_t)) +
           (kWarps * kRadix + 2 * kRadix + 4) * sizeof(uint32_t);
}

} // namespace

uint32_t sort_tiles(uint32_t n) { return ceil_div(n == 0 ? 1 : n, kSortTile); }

size_t cube_partials_needed(uint32_t) { return 6ull * kCubeBlocks; }

cudaError_t launch_bounding_cube(const double *x, const double *y, const double *z, uint32_t n,
                                 double *partials, TreeMeta *meta, cudaStream_t stream) {
    cube_kernel<<<kCubeBlocks, kCubeThreads, 0, stream>>>(x, y, z, n, partials, meta);
    return cudaGetLastError();
}

cudaError_t launch_encode(const double *x, const double *y, const double *z, uint32_t n,
                          const TreeMeta *meta, unsigned long long *codes, uint32_t *indices,
                          uint32_t *hist, cudaStream_t stream) {
    const uint32_t blocks = max(1u, min(ceil_div(n, kReduceThreads), kReduceBlocks));
    encode_kernel<<<blocks, kReduceThreads, 0, stream>>>(x, y, z, n, meta, codes, indices, hist);
    return cudaGetLastError();
}

cudaError_t launch_scan_histograms(uint32_t *hist, cudaStream_t stream) {
    scan_histograms_kernel<<<kRadixPasses, kRadix, 0, stream>>>(hist);
    return cudaGetLastError();
}

cudaError_t launch_onesweep(const unsigned long long *keys_in, const uint32_t *vals_in,
                            unsigned long long *keys_out, uint32_t *vals_out, uint32_t n,
                            int pass, const uint32_t *offsets, uint32_t *lookback,
                            uint32_t *ticket, unsigned *status, cudaStream_t stream,
                            uint32_t poll_limit) {
    static_assert(kLookbackPollLimit == kSpinLimit, "one bound for every device wait");
    static std::atomic<uint64_t> configured{0};
    const cudaError_t err = set_smem_limit_once(reinterpret_cast<const void *>(onesweep_kernel),
                                                static_cast<int>(onesweep_smem()), configured);
    if (err != cudaSuccess) {
        return err;
    }
    // Persistent CTAs: as many as fit on the device at once, at most one per tile.
    static std::atomic<int> resident{0};
    if (resident.load(std::memory_order_relaxed) == 0) {
        int per_sm = 0, sms = 0, device = 0;
        cudaError_t e = cudaGetDevice(&device);
        if (e == cudaSuccess) {
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        }
        if (e == cudaSuccess) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_kernel,
                                                              kSortThreads, onesweep_smem());
        }
        if (e != cudaSuccess) {
            return e;
        }
        resident.store(std::max(1, per_sm) * std::max(1, sms), std::memory_order_relaxed);
    }
    const uint32_t tiles = sort_tiles(n);
    const uint32_t grid = std::min(tiles, static_cast<uint32_t>(resident.load()));
    onesweep_kernel<<<grid, kSortThreads, onesweep_smem(), stream>>>(
        keys_in, vals_in, keys_out, vals_out, n, tiles, static_cast<uint32_t>(kRadixBits * pass),
        offsets + pass * kRadix, lookback, ticket, status, poll_limit);
    return cudaGetLastError();
}

cudaError_t launch_gather(const double *x, const double *y, const double *z, const double *m,
                          const uint32_t *perm, uint32_t n, double *sorted, cudaStream_t stream) {
    const uint32_t blocks = max(1u, min(ceil_div(n, 256), 148u * 16u));
    gather_kernel<<<blocks, 256, 0, stream>>>(x, y, z, m, perm, n, sorted);
    return cudaGetLastError();
}

size_t scan_partials_needed(uint32_t n) { return ceil_div(n == 0 ? 1 : n, kScanTile) + 1ull; }

cudaError_t launch_exclusive_scan(const uint32_t *in, uint32_t *out, uint32_t n,
                                  uint32_t *scratch, cudaStream_t stream) {
    const uint32_t blocks = ceil_div(n == 0 ? 1 : n, kScanTile);
    scan_reduce_kernel<<<blocks, kScanThreads, 0, stream>>>(in, n, scratch);
    scan_sums_kernel<<<1, 1024, 0, stream>>>(scratch, blocks);
    scan_apply_kernel<<<blocks, kScanThreads, 0, stream>>>(in, out, n, scratch, blocks);
    return cudaGetLastError();
}

} // namespace ob
