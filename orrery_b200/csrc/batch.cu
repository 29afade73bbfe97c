// Batched direct sums: many systems of uneven size in one persistent launch.
//
// Work is a queue of (system, target tile, source chunk) items, ordered
// largest first and pulled by CTAs with an atomic ticket, so big and small
// systems share the SMs without a per-system launch. Each item runs the
// precision form's arithmetic (hi/lo split positions, Newton-refined SFU
// rsqrt, Kahan-compensated FP32 partials per 512-source tile folded into
// FP64) with its own system's softening. Items that cover a whole system's
// sources write accelerations directly; otherwise each writes a partial slot
// and a second kernel sums a target tile's slots in chunk order, so results
// do not depend on which CTA took which item.
//
// Each system's particles are padded to a multiple of the 512-source tile
// with zero-mass entries; with every softening positive, a zero-mass source
// and the target itself contribute exactly zero, so the kernel needs no masks.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "batch.hpp"
#include "common.cuh"
#include "runtime.hpp"
#include "split_math.cuh"

namespace ob {
namespace {

struct BatchArgs {
    const float4 *hi;
    const float4 *lo;
    const float *eps2;
    const BatchItem *items;
    uint32_t item_count;
    double *ax;
    double *ay;
    double *az;
    double *partial;
    uint32_t *queue;
    unsigned *status;
};

// Targets r = 2p + h of a thread are packed in pairs p; the arithmetic is
// the split form's, in FP32x2 instructions (split_math.cuh). With K source
// groups the CTA's threads form K groups of TP = THREADS / K: thread tid
// serves target lane tid % TP over slice tid / TP of every tile
// (kDirectTile / K sources), and the K partial sums of a target are added in
// slice order before they are written.
template <int THREADS, int R, int K>
__global__ void __launch_bounds__(THREADS) batch_split_kernel(const BatchArgs a) {
    static_assert(R % 2 == 0, "targets are processed in packed pairs");
    static_assert(THREADS % K == 0 && (THREADS / K) % 32 == 0, "groups are whole warps");
    static_assert(kDirectTile % K == 0, "a tile splits evenly");
    constexpr int P = R / 2;
    constexpr uint32_t TP = THREADS / K;
    constexpr uint32_t JS = kDirectTile / K;
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr uint32_t BT = TP * R;
    float4 *tiles_hi = reinterpret_cast<float4 *>(smem);   // 2 buffers x 2*kDirectTile
    float4 *tiles_lo = tiles_hi + 4 * kDirectTile;         // 2 buffers x 2*kDirectTile
    uint64_t *bars = reinterpret_cast<uint64_t *>(tiles_lo + 4 * kDirectTile);
    double *group_sums = reinterpret_cast<double *>(bars + 2); // K x 3 x BT when K > 1
    __shared__ uint32_t s_item;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid % TP;
    const uint32_t group = tid / TP;
    const uint32_t jb = group * JS; // this thread's slice of every tile
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    constexpr uint32_t bytes = 2 * kDirectTile * sizeof(float4);
    auto stage = [&](uint32_t tile, uint32_t buf) {
        mbar_arrive_expect_tx(&bars[buf], 2 * bytes);
        const size_t off = 2ull * static_cast<size_t>(tile) * kDirectTile;
        bulk_copy_g2s(tiles_hi + buf * 2 * kDirectTile, a.hi + off, bytes, &bars[buf]);
        bulk_copy_g2s(tiles_lo + buf * 2 * kDirectTile, a.lo + off, bytes, &bars[buf]);
    };

    uint32_t sequence = 0; // tiles this CTA has consumed (pipeline phase)
    bool ok = true;
    while (true) {
        if (tid == 0) {
            s_item = atomicAdd(a.queue, 1u);
        }
        __syncthreads();
        const uint32_t w = s_item;
        __syncthreads();
        if (w >= a.item_count) {
            break;
        }
        const BatchItem item = a.items[w];
        const float2 eps2 = make_float2(a.eps2[item.system], a.eps2[item.system]);
        SplitTargets tg[P];
        double sx[R], sy[R], sz[R];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const size_t i0 = item.target_begin + (2 * p) * TP + lane;
            tg[p] = load_split_targets(a.hi, a.lo, i0, i0 + TP);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            sx[r] = sy[r] = sz[r] = 0.0;
        }
        const uint32_t first_tile = item.source_begin / kDirectTile;
        const uint32_t tiles = item.source_tiles;
        if (tid == 0) {
            for (uint32_t k = 0; k < min(2u, tiles); ++k) {
                stage(first_tile + k, (sequence + k) & 1u);
            }
        }
        for (uint32_t k = 0; k < tiles; ++k) {
            const uint32_t g = sequence + k;
            const uint32_t buf = g & 1u;
            if (ok) {
                ok = mbar_wait_bounded(&bars[buf], (g >> 1) & 1u, a.status);
            }
            if (ok) {
                const float4 *th = tiles_hi + buf * 2 * kDirectTile;
                const float4 *tl = tiles_lo + buf * 2 * kDirectTile;
                float2 kx[P], ky[P], kz[P], cx[P], cy[P], cz[P];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    kx[p] = ky[p] = kz[p] = cx[p] = cy[p] = cz[p] = make_float2(0.0f, 0.0f);
                }
#pragma unroll 2
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
            if (tid == 0 && ok && k + 2 < tiles) {
                fence_proxy_async_shared();
                stage(first_tile + k + 2, buf);
            }
        }
        sequence += tiles;
        auto write = [&](uint32_t slot, double x, double y, double z) {
            if (slot < item.target_count) {
                if (item.slot == kDirectWrite) {
                    const uint32_t i = item.target_begin + slot;
                    a.ax[i] = x;
                    a.ay[i] = y;
                    a.az[i] = z;
                } else {
                    double *p = a.partial + static_cast<size_t>(item.slot) * 3 * BT;
                    p[slot] = x;
                    p[BT + slot] = y;
                    p[2 * BT + slot] = z;
                }
            }
        };
        if constexpr (K == 1) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                write(r * THREADS + tid, sx[r], sy[r], sz[r]);
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t slot = r * TP + lane;
                group_sums[(group * 3 + 0) * BT + slot] = sx[r];
                group_sums[(group * 3 + 1) * BT + slot] = sy[r];
                group_sums[(group * 3 + 2) * BT + slot] = sz[r];
            }
            __syncthreads();
            for (uint32_t slot = tid; slot < BT; slot += THREADS) {
                double s[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int g = 0; g < K; ++g) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        s[c] += group_sums[(g * 3 + c) * BT + slot];
                    }
                }
                write(slot, s[0], s[1], s[2]);
            }
            // The next item's group sums reuse the buffer after the barrier
            // that follows.
        }
        if (!__syncthreads_and(ok ? 1 : 0)) {
            break;
        }
    }
}

__global__ void batch_reduce_kernel(const BatchGroup *__restrict__ groups, uint32_t count,
                                    const double *__restrict__ partial, uint32_t bt, double *ax,
                                    double *ay, double *az) {
    for (uint32_t g = blockIdx.x; g < count; g += gridDim.x) {
        const BatchGroup grp = groups[g];
        for (uint32_t k = threadIdx.x; k < grp.target_count; k += blockDim.x) {
            double x = 0.0, y = 0.0, z = 0.0;
            for (uint32_t s = 0; s < grp.slots; ++s) {
                const double *p = partial + static_cast<size_t>(grp.first_slot + s) * 3 * bt;
                x += p[k];
                y += p[bt + k];
                z += p[2 * bt + k];
            }
            ax[grp.target_begin + k] = x;
            ay[grp.target_begin + k] = y;
            az[grp.target_begin + k] = z;
        }
    }
}

template <int THREADS, int R, int K>
cudaError_t launch_batch_t(const BatchArgs &args, int sm_count, cudaStream_t stream) {
    const size_t smem = 8 * kDirectTile * sizeof(float4) + 2 * sizeof(uint64_t) +
                        (K > 1 ? 3 * THREADS * R * sizeof(double) : 0);
    auto kernel = batch_split_kernel<THREADS, R, K>;
    static std::atomic<uint64_t> configured{0};
    const cudaError_t err = set_smem_limit_once(reinterpret_cast<const void *>(kernel),
                                                static_cast<int>(smem), configured);
    if (err != cudaSuccess) {
        return err;
    }
    static int resident = 0;
    if (resident == 0) {
        const cudaError_t err =
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, THREADS, smem);
        if (err != cudaSuccess || resident < 1) {
            resident = 1;
        }
    }
    const uint32_t blocks = static_cast<uint32_t>(std::max(1, sm_count) * resident);
    kernel<<<blocks, THREADS, smem, stream>>>(args);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_batch_forces(const float4 *hi, const float4 *lo, const float *eps2,
                                const BatchItem *items, uint32_t item_count,
                                const BatchConfig &config, double *ax, double *ay, double *az,
                                double *partial, uint32_t *queue, unsigned *status,
                                int sm_count, cudaStream_t stream) {
    if (item_count == 0) {
        return cudaSuccess;
    }
    const BatchArgs args{hi, lo, eps2, items, item_count, ax, ay, az, partial, queue, status};
#define OB_BATCH_CASE(T, RR, KK)                                                                   \
    if (config.threads == T && config.targets_per_thread == RR && config.groups == KK)             \
        return launch_batch_t<T, RR, KK>(args, sm_count, stream);
    OB_BATCH_CASE(128, 2, 1)
    OB_BATCH_CASE(128, 4, 1)
    OB_BATCH_CASE(256, 2, 1)
    OB_BATCH_CASE(256, 4, 1)
    OB_BATCH_CASE(128, 2, 4)
    OB_BATCH_CASE(256, 2, 8)
    OB_BATCH_CASE(256, 4, 4)
    OB_BATCH_CASE(256, 4, 8)
#undef OB_BATCH_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_batch_reduce(const BatchGroup *groups, uint32_t group_count,
                                const double *partial, uint32_t bt, double *ax, double *ay,
                                double *az, cudaStream_t stream) {
    if (group_count == 0) {
        return cudaSuccess;
    }
    const uint32_t blocks = std::min(group_count, 148u * 8u);
    batch_reduce_kernel<<<blocks, 128, 0, stream>>>(groups, group_count, partial, bt, ax, ay, az);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------

uint64_t Batch::footprint(uint32_t n) {
    return static_cast<uint64_t>(ceil_div(n, kDirectTile)) * kDirectTile;
}

void Batch::init(uint64_t capacity, cudaStream_t stream) {
    // Slack past the arena for target tiles that run over (<= 1024).
    const uint64_t total = capacity + 1024;
    if (total > 0x7fffffffull) {
        throw Error(OB_ERROR_CAPACITY, "a batch holds at most 2^31 padded particles");
    }
    total_ = static_cast<uint32_t>(total);
    free_regions_.assign(1, {0u, static_cast<uint32_t>(capacity)});
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device), "SMs");
    if (stream != nullptr) {
        stream_ = stream;
        owns_stream_ = false;
    } else {
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "creating a stream");
    }
    state_.reserve(10ull * total_);
    check(cudaMemset(state_.data(), 0, state_.bytes()), "clearing state");
    hi_.reserve(2ull * total_);
    lo_.reserve(2ull * total_);
    queue_.reserve(1);
    status_.reserve(1);
    check(cudaMemset(status_.data(), 0, sizeof(unsigned)), "clearing status");
}

Batch::Batch(uint64_t capacity, cudaStream_t stream) { init(capacity, stream); }

Batch::Batch(uint32_t systems, const uint64_t *counts, const double *softening_squared) {
    if (systems == 0) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "a batch needs at least one system");
    }
    uint64_t capacity = 0;
    for (uint32_t s = 0; s < systems; ++s) {
        if (counts[s] == 0 || counts[s] > 0xffffffffull) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "every system needs 1 .. 2^32-1 particles");
        }
        capacity += footprint(static_cast<uint32_t>(counts[s]));
    }
    init(capacity, nullptr);
    for (uint32_t s = 0; s < systems; ++s) {
        if (add(static_cast<uint32_t>(counts[s]), softening_squared[s]) < 0) {
            throw Error(OB_ERROR_CAPACITY, "the batch arena could not place a system");
        }
    }
}

Batch::~Batch() {
    drop_graph();
    if (stream_ != nullptr && owns_stream_) {
        cudaStreamDestroy(stream_);
    }
}

void Batch::drop_graph() {
    if (graph_ != nullptr) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
}

bool Batch::active(uint32_t id) const noexcept {
    return id < members_.size() && members_[id].active;
}

void Batch::check_member(uint32_t id) const {
    if (!active(id)) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "no such system in the batch");
    }
}

int64_t Batch::add(uint32_t n, double softening_squared) {
    if (n == 0) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "every system needs 1 .. 2^32-1 particles");
    }
    if (!(softening_squared > 0.0) || !std::isfinite(softening_squared)) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "batched systems need a positive, finite softening");
    }
    const uint64_t need = footprint(n);
    // First fit over the free regions, lowest offset first.
    for (size_t r = 0; r < free_regions_.size(); ++r) {
        if (free_regions_[r].second >= need) {
            Member m;
            m.count = n;
            m.offset = free_regions_[r].first;
            m.padded = static_cast<uint32_t>(need);
            m.eps2 = softening_squared;
            m.active = true;
            free_regions_[r].first += m.padded;
            free_regions_[r].second -= m.padded;
            if (free_regions_[r].second == 0) {
                free_regions_.erase(free_regions_.begin() + static_cast<std::ptrdiff_t>(r));
            }
            uint32_t id;
            if (!free_ids_.empty()) {
                id = free_ids_.back();
                free_ids_.pop_back();
                members_[id] = m;
            } else {
                id = static_cast<uint32_t>(members_.size());
                members_.push_back(m);
            }
            if (eps2_.size() < members_.size()) {
                DeviceArray<float> grown;
                grown.reserve(std::max<size_t>(64, 2 * members_.size()));
                if (eps2_.size() > 0) {
                    check(cudaMemcpyAsync(grown.data(), eps2_.data(), eps2_.bytes(),
                                          cudaMemcpyDeviceToDevice, stream_),
                          "growing softenings");
                    check(cudaStreamSynchronize(stream_), "growing softenings");
                }
                eps2_ = std::move(grown);
            }
            const float e = static_cast<float>(softening_squared);
            check(cudaMemcpyAsync(eps2_.data() + id, &e, sizeof(float), cudaMemcpyHostToDevice,
                                  stream_),
                  "uploading a softening");
            check(cudaStreamSynchronize(stream_), "uploading a softening");
            high_ = std::max(high_, m.offset + m.padded);
            pairs_ += static_cast<uint64_t>(n) * (n - 1);
            ++active_count_;
            dirty_ = true;
            return id;
        }
    }
    return -1;
}

void Batch::remove(uint32_t id) {
    check_member(id);
    Member &m = members_[id];
    for (int k = 0; k < 10; ++k) {
        check(cudaMemsetAsync(array(k) + m.offset, 0, sizeof(double) * m.padded, stream_),
              "clearing a region");
    }
    // Return the region, merging with free neighbours.
    std::pair<uint32_t, uint32_t> region{m.offset, m.padded};
    auto it = std::lower_bound(free_regions_.begin(), free_regions_.end(), region);
    it = free_regions_.insert(it, region);
    if (it + 1 != free_regions_.end() && it->first + it->second == (it + 1)->first) {
        it->second += (it + 1)->second;
        free_regions_.erase(it + 1);
    }
    if (it != free_regions_.begin() && (it - 1)->first + (it - 1)->second == it->first) {
        (it - 1)->second += it->second;
        free_regions_.erase(it);
    }
    pairs_ -= static_cast<uint64_t>(m.count) * (m.count - 1);
    m.active = false;
    free_ids_.push_back(id);
    --active_count_;
    high_ = 0;
    for (const Member &other : members_) {
        if (other.active) {
            high_ = std::max(high_, other.offset + other.padded);
        }
    }
    dirty_ = true;
}

std::vector<BatchItem> Batch::make_items(const BatchConfig &config,
                                         const std::vector<uint32_t> &ids,
                                         std::vector<BatchGroup> &groups, uint32_t &slots) const {
    const uint32_t bt = config.targets_per_block();
    std::vector<BatchItem> items;
    for (const uint32_t s : ids) {
        const Member &m = members_[s];
        const uint32_t tiles = ceil_div(m.count, kDirectTile);
        const uint32_t chunk =
            config.chunk_tiles == 0 ? tiles : std::min(config.chunk_tiles, tiles);
        const uint32_t chunks = ceil_div(tiles, chunk);
        for (uint32_t t = 0; t < m.count; t += bt) {
            const uint32_t n_targets = std::min(bt, m.count - t);
            if (chunks > 1) {
                groups.push_back(BatchGroup{m.offset + t, n_targets, slots, chunks});
            }
            for (uint32_t c = 0; c < chunks; ++c) {
                const uint32_t first = c * chunk;
                items.push_back(BatchItem{s, m.offset + t, n_targets,
                                          m.offset + first * kDirectTile,
                                          std::min(chunk, tiles - first),
                                          chunks > 1 ? slots + c : kDirectWrite});
            }
            if (chunks > 1) {
                slots += chunks;
            }
        }
    }
    // Largest first, ties in creation order: the queue then balances itself.
    std::stable_sort(items.begin(), items.end(), [](const BatchItem &l, const BatchItem &r) {
        return static_cast<uint64_t>(l.target_count) * l.source_tiles >
               static_cast<uint64_t>(r.target_count) * r.source_tiles;
    });
    return items;
}

void Batch::upload_items(const std::vector<BatchItem> &items,
                         const std::vector<BatchGroup> &groups, uint32_t slots) {
    const uint32_t bt = config_.targets_per_block();
    const bool moved_items = items_.reserve(std::max<size_t>(1, items.size()));
    const bool moved_groups = groups_.reserve(std::max<size_t>(1, groups.size()));
    const bool moved_partial =
        partial_.reserve(std::max<size_t>(1, static_cast<size_t>(slots) * 3 * bt));
    if (moved_items || moved_groups || moved_partial) {
        drop_graph();
    }
    if (!items.empty()) {
        check(cudaMemcpyAsync(items_.data(), items.data(), sizeof(BatchItem) * items.size(),
                              cudaMemcpyHostToDevice, stream_),
              "uploading work items");
    }
    if (!groups.empty()) {
        check(cudaMemcpyAsync(groups_.data(), groups.data(), sizeof(BatchGroup) * groups.size(),
                              cudaMemcpyHostToDevice, stream_),
              "uploading reduction groups");
    }
    check(cudaStreamSynchronize(stream_), "uploading work items");
    item_count_ = static_cast<uint32_t>(items.size());
    group_count_ = static_cast<uint32_t>(groups.size());
}

void Batch::rebuild_if_needed() {
    if (!dirty_) {
        return;
    }
    std::vector<uint32_t> ids;
    for (uint32_t s = 0; s < members_.size(); ++s) {
        if (members_[s].active) {
            ids.push_back(s);
        }
    }
    std::vector<BatchGroup> groups;
    uint32_t slots = 0;
    const std::vector<BatchItem> items = make_items(config_, ids, groups, slots);
    upload_items(items, groups, slots);
    drop_graph();
    dirty_ = false;
}

void Batch::set_config(const BatchConfig &config) {
    config_ = config;
    dirty_ = true;
    rebuild_if_needed();
}

void Batch::set_state(uint32_t id, const double *x, const double *y, const double *z,
                      const double *vx, const double *vy, const double *vz, const double *m) {
    check_member(id);
    if (!x || !y || !z || !m) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "positions and masses are required");
    }
    const Member &mb = members_[id];
    // The kernel has no masks: a target's own entry enters its sum as f * 0
    // with f = m / eps^3 in FP32, which is zero only while f is finite (the
    // bound leaves room for the rounding of the device's 1 / eps).
    const double inverse_cube = std::pow(mb.eps2, -1.5);
    for (uint32_t i = 0; i < mb.count; ++i) {
        if (!(std::fabs(m[i]) * inverse_cube < 1e37)) {
            throw Error(OB_ERROR_INVALID_ARGUMENT,
                        "a mass / softening^3 beyond the FP32 range of the batched kernel");
        }
    }
    const double *in[7] = {x, y, z, vx, vy, vz, m};
    const int arrays[7] = {kX, kY, kZ, kVx, kVy, kVz, kM};
    const size_t bytes = sizeof(double) * mb.count;
    for (int k = 0; k < 7; ++k) {
        double *dst = array(arrays[k]) + mb.offset;
        if (in[k] == nullptr) {
            check(cudaMemsetAsync(dst, 0, bytes, stream_), "clearing");
        } else {
            check(cudaMemcpyAsync(dst, in[k], bytes, cudaMemcpyHostToDevice, stream_), "upload");
        }
    }
    check(cudaStreamSynchronize(stream_), "uploading a system");
}

void Batch::get_state_async(uint32_t id, double *const *out) {
    check_member(id);
    const Member &mb = members_[id];
    for (int k = 0; k < 9; ++k) {
        if (out[k] != nullptr) {
            check(cudaMemcpyAsync(out[k], array(k) + mb.offset, sizeof(double) * mb.count,
                                  cudaMemcpyDeviceToHost, stream_),
                  "download");
        }
    }
}

void Batch::get_state(uint32_t id, double *const *out) {
    get_state_async(id, out);
    check(cudaStreamSynchronize(stream_), "downloading a system");
}

void Batch::evaluate() {
    rebuild_if_needed();
    check(pack_sources(array(kX), array(kY), array(kZ), array(kM), high_, high_, hi_.data(),
                       lo_.data(), stream_),
          "packing sources");
    check(cudaMemsetAsync(queue_.data(), 0, sizeof(uint32_t), stream_), "resetting the queue");
    check(launch_batch_forces(hi_.data(), lo_.data(), eps2_.data(), items_.data(), item_count_,
                              config_, array(kAx), array(kAy), array(kAz), partial_.data(),
                              queue_.data(), status_.data(), sm_count_, stream_),
          "batched forces");
    check(launch_batch_reduce(groups_.data(), group_count_, partial_.data(),
                              config_.targets_per_block(),
                              array(kAx), array(kAy), array(kAz), stream_),
          "reducing partial sums");
}

void Batch::refresh() {
    evaluate();
    ++evaluations_;
    synchronize();
}

void Batch::refresh_members(const std::vector<uint32_t> &ids) {
    for (const uint32_t id : ids) {
        check_member(id);
    }
    if (ids.empty()) {
        return;
    }
    // Whole-system items (no partial slots) for just these members.
    BatchConfig whole = config_;
    whole.chunk_tiles = 0;
    std::vector<BatchGroup> groups;
    uint32_t slots = 0;
    const std::vector<BatchItem> items = make_items(whole, ids, groups, slots);
    side_items_.reserve(items.size()); // the step graph never reads side_items_
    check(cudaMemcpyAsync(side_items_.data(), items.data(), sizeof(BatchItem) * items.size(),
                          cudaMemcpyHostToDevice, stream_),
          "uploading work items");
    check(pack_sources(array(kX), array(kY), array(kZ), array(kM), high_, high_, hi_.data(),
                       lo_.data(), stream_),
          "packing sources");
    check(cudaMemsetAsync(queue_.data(), 0, sizeof(uint32_t), stream_), "resetting the queue");
    check(launch_batch_forces(hi_.data(), lo_.data(), eps2_.data(), side_items_.data(),
                              static_cast<uint32_t>(items.size()), whole, array(kAx), array(kAy),
                              array(kAz), partial_.data(), queue_.data(), status_.data(),
                              sm_count_, stream_),
          "batched forces");
    check(cudaStreamSynchronize(stream_), "evaluating new members");
}

static void yoshida(double &outer, double &inner) {
    constexpr double cube_root_of_two = 1.2599210498948731647672106;
    outer = 1.0 / (2.0 - cube_root_of_two);
    inner = -cube_root_of_two / (2.0 - cube_root_of_two);
}

void Batch::enqueue_step(int integrator, double dt) {
    auto substep = [&](double h) {
        const double half = h / 2.0;
        check(launch_kick_drift(array(kX), array(kY), array(kZ), array(kVx), array(kVy),
                                array(kVz), array(kAx), array(kAy), array(kAz), high_, half, h,
                                stream_),
              "kick and drift");
        evaluate();
        check(launch_kick(array(kVx), array(kVy), array(kVz), array(kAx), array(kAy), array(kAz),
                          high_, half, stream_),
              "kick");
    };
    if (integrator == OB_INTEGRATOR_YOSHIDA4) {
        double outer = 0.0, inner = 0.0;
        yoshida(outer, inner);
        substep(outer * dt);
        substep(inner * dt);
        substep(outer * dt);
    } else {
        substep(dt);
    }
}

void Batch::step_async(int integrator, double dt, uint64_t steps) {
    if (integrator == OB_INTEGRATOR_RK4) {
        throw Error(OB_ERROR_UNSUPPORTED, "batches step with VV or Yoshida-4 (RK4: ob_system_*)");
    }
    if (integrator != OB_INTEGRATOR_VV && integrator != OB_INTEGRATOR_YOSHIDA4) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "unknown integrator");
    }
    if (active_count_ == 0 || steps == 0) {
        return;
    }
    rebuild_if_needed();
    if (graph_ == nullptr || graph_integrator_ != integrator || graph_dt_ != dt) {
        drop_graph();
        cudaGraph_t graph = nullptr;
        check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed), "begin capture");
        try {
            enqueue_step(integrator, dt);
        } catch (...) {
            cudaStreamEndCapture(stream_, &graph);
            if (graph != nullptr) {
                cudaGraphDestroy(graph);
            }
            throw;
        }
        check(cudaStreamEndCapture(stream_, &graph), "end capture");
        const cudaError_t err = cudaGraphInstantiate(&graph_, graph, 0);
        cudaGraphDestroy(graph);
        check(err, "instantiating the batch step graph");
        graph_integrator_ = integrator;
        graph_dt_ = dt;
    }
    for (uint64_t s = 0; s < steps; ++s) {
        check(cudaGraphLaunch(graph_, stream_), "launching the batch step");
    }
    evaluations_ += steps * (integrator == OB_INTEGRATOR_YOSHIDA4 ? 3 : 1);
}

void Batch::synchronize() {
    check(cudaStreamSynchronize(stream_), "batched integration");
    const unsigned status = read_and_clear_status(status_.data(), stream_);
    if (status & kStatusTimeout) {
        throw Error(OB_ERROR_TIMEOUT, "a device-side wait ran out of its bound");
    }
}

static double neumaier(const std::vector<double> &terms) {
    double total = 0.0, correction = 0.0;
    for (const double term : terms) {
        const double updated = total + term;
        if (std::fabs(total) >= std::fabs(term)) {
            correction += (total - updated) + term;
        } else {
            correction += (term - updated) + total;
        }
        total = updated;
    }
    return total + correction;
}

void Batch::energy(uint32_t id, double *kinetic, double *potential) {
    check_member(id);
    const uint32_t n = members_[id].count;
    const uint32_t o = members_[id].offset;
    terms_.reserve(n);
    std::vector<double> host(n);
    if (kinetic != nullptr) {
        check(launch_kinetic_partials(array(kVx) + o, array(kVy) + o, array(kVz) + o,
                                      array(kM) + o, n, terms_.data(), stream_),
              "kinetic terms");
        check(cudaMemcpyAsync(host.data(), terms_.data(), sizeof(double) * n,
                              cudaMemcpyDeviceToHost, stream_),
              "download");
        check(cudaStreamSynchronize(stream_), "kinetic energy");
        *kinetic = neumaier(host) / 2.0;
    }
    if (potential != nullptr) {
        check(launch_potential_rows(array(kX) + o, array(kY) + o, array(kZ) + o, array(kM) + o, n,
                                    members_[id].eps2, terms_.data(), stream_),
              "potential rows");
        check(cudaMemcpyAsync(host.data(), terms_.data(), sizeof(double) * n,
                              cudaMemcpyDeviceToHost, stream_),
              "download");
        check(cudaStreamSynchronize(stream_), "potential energy");
        *potential = neumaier(host);
    }
}

double Batch::autotune(BatchConfig &chosen) {
    static const uint32_t chunks[] = {0, 16, 8, 4};
    cudaEvent_t start, stop;
    check(cudaEventCreate(&start), "event");
    check(cudaEventCreate(&stop), "event");
    double best = 1e300;
    BatchConfig best_config = config_;
    for (const auto &shape : kBatchShapes) {
        for (const uint32_t chunk : chunks) {
            set_config(BatchConfig{shape[0], shape[1], chunk, shape[2]});
            evaluate();
            check(cudaEventRecord(start, stream_), "event");
            evaluate();
            evaluate();
            check(cudaEventRecord(stop, stream_), "event");
            check(cudaEventSynchronize(stop), "autotune timing");
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, start, stop), "autotune timing");
            if (ms / 2.0 < best) {
                best = ms / 2.0;
                best_config = config_;
            }
        }
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    set_config(best_config);
    // The timing runs overwrote the carried accelerations: recompute them.
    evaluate();
    synchronize();
    chosen = best_config;
    return best;
}

} // namespace ob
