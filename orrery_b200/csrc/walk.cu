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
// Group traversal. The warp walks the tree once for its 32 targets, carrying
// with every node the mask of targets whose own walks reach it (those that
// opened all its ancestors). Lanes take different nodes of a depth-first
// stack of (node, reach mask) items, up to 32 per round; an item pushes its
// next sibling (a bit of the node record says whether it has one) and, when
// opened, its first child. Each lane classifies its node against the
// bounding box of the warp's targets from the node's compact record: the
// per-axis distances from the centre of mass to the nearest and farthest box
// faces are formed from FP32 hi + lo parts (so each is accurate to a few ulps
// of itself), and with a 4e-6 relative margin on the acceptance radius
//   nearest^2 >= r2 (1 + m)  ->  every target accepts the cell,
//   farthest^2 <  r2 (1 - m)  ->  every target opens it,
// exactly as the reference's FP64 test decides for each target (every target
// lies in the box; the margin covers the FP32 error of the distances and of
// r2). The remaining ("mixed") nodes are decided per target: an FP32 hi/lo
// test with the same margin, and the reference's FP64 test inside it.
//
// The lane that accepts a cell stages it at once in shared memory (centre of
// mass relative to the box centre G, mass, 2.5 Q, target mask), packed so that
// one 16-byte load gives two cells' values; an opened leaf is queued with its
// centre relative to G, its particle range and mask. Batches of cells are then
// evaluated by every lane for its own target, two cells per packed FP32x2
// instruction (a lane outside a cell's mask contributes exactly zero), and
// queued leaves likewise, their sources staged in shared memory per leaf.
//
// Arithmetic. Positions and centres of mass are carried as FP32 hi + lo pairs
// (exact to ~2^-48 relative); force terms are FP32, summed in FP32 within a
// batch and flushed into FP64 per-target sums.
//
// A round takes no more items than the stack has room to push back (each
// pushes at most two), so the stack (256 entries per warp; with this rule the
// 2M two-disc collision rarely fills it) only stops the traversal when
// completely full;
// the warp then discards its partial sums and walks its targets with the
// per-target union walk (union_walk below), which gives the same counts.
//
// Warp discipline. Between the warp's votes and barriers there is no long
// lane-divergent stretch of work: lanes outside a leaf's or cell's mask run
// the same arithmetic with zero weight, and the FP64 accept test runs on
// every lane once any lane needs it. (Votes and warp barriers of the same kind
// may be satisfied by lanes standing at different instructions, so a warp
// whose lanes spent long, different times in divergent code was seen to fall
// out of step.) Node and particle indices are checked before every gather; an
// index out of range (which a valid tree never produces) sets kStatusInvalid
// and is skipped.
#include "common.cuh"
#include "tree_kernels.hpp"

namespace ob {
namespace {

constexpr int kWalkWarps = 4;
constexpr int kWalkThreads = kWalkWarps * 32;
constexpr float kAcceptMargin = 4e-6f;
constexpr uint32_t kFull = 0xffffffffu;

// Per-warp shared-memory capacities (entries). A round takes at most 32 items;
// each adds at most two stack items (its next sibling and, opened, its first
// child) and at most one cell or one leaf, so a round of t items adds at most
// 2t stack items, t cells and t leaves. A round takes at most stack room
// (capacity - size) items, so the stack cannot overflow while it has room;
// cells and leaves are evaluated once more than capacity - 32 are queued.
// Sized so that 8 CTAs of 4 warps fit in an SM's shared memory.
constexpr uint32_t kStackCap = 256;
constexpr uint32_t kCellCap = 48;
constexpr uint32_t kLeafCap = 40;
// Staged cell fields, as quads of packed pairs: quad f of pair p holds
// (a_j, a_j+1, b_j, b_j+1) for the two fields a, b of group f and the cells
// j = 2p, 2p+1: (x, y) (z, mass) (2.5 Qxx, 2.5 Qxy) (2.5 Qxz, 2.5 Qyy)
// (2.5 Qyz, 2.5 Qzz), centres relative to the box centre G.
constexpr int kCellQuads = 5;
// Leaf sources staged per chunk of 32: (x, y) (z, mass), leaf-relative.
constexpr int kLeafQuads = 2;
// Offset given to lanes outside a leaf's mask and to the neutral partner: the
// terms it produces underflow to exactly zero in FP32.
constexpr float kFar = 1e18f;

struct __align__(16) WarpSpace {
    float4 cells[kCellQuads][kCellCap / 2 + 1]; // +1: the neutral partner of an odd count
    uint32_t cell_mask[kCellCap + 2];
    float4 leaf_pos[kLeafCap];  // leaf centre of mass - G (FP32), particle count bits
    uint2 leaf_meta[kLeafCap];  // (first particle | may-hold-a-target bit, target mask)
    uint2 stack[kStackCap];     // (node, reach mask)
    union {                     // used one at a time
        float4 leaf_quads[kLeafQuads][17];
        float4 union_staged[32]; // the union walk's leaf staging (after a fallback)
    };
    // Box of the warp's targets as FP32 hi + lo parts: lo hi, lo lo, hi hi,
    // hi lo; then the box centre G hi, G lo (x, y, z; w unused).
    float4 box[6];
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

__device__ __forceinline__ uint32_t warp_min(uint32_t v) { return __reduce_min_sync(kFull, v); }

__device__ __forceinline__ uint32_t lanes_below(uint32_t lane) { return (1u << lane) - 1u; }

// Writes fields (a, b) of staged entry j into quad array q (see kCellQuads).
__device__ __forceinline__ void put(float4 *q, uint32_t j, float a, float b) {
    float *slot = reinterpret_cast<float *>(&q[j >> 1]) + (j & 1u);
    slot[0] = a;
    slot[2] = b;
}

// Splits an FP64 value into FP32 hi + lo with hi + lo = v to ~2^-48.
__device__ __forceinline__ void split(double v, float &hi, float &lo) {
    hi = __double2float_rn(v);
    lo = __double2float_rn(v - static_cast<double>(hi));
}

// The reference's accept test in FP64 (tree_walk.cpp:44-46), for cells whose
// FP32 test fell inside the margin.
__device__ __forceinline__ bool exact_accept(const DeviceNode *nodes, uint32_t cur,
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

// One target's FP32 accept test of a walk record, with the FP64 fallback
// inside the margin. Also returns the FP32 offset d = com - target.
__device__ __forceinline__ bool lane_accepts(const float4 A, const float4 B, float pxh, float pyh,
                                             float pzh, float pxl, float pyl, float pzl,
                                             const DeviceNode *nodes, uint32_t cur,
                                             const double *sorted, uint32_t n, uint32_t i,
                                             float &dx, float &dy, float &dz) {
    dx = (A.x - pxh) + (B.x - pxl);
    dy = (A.y - pyh) + (B.y - pyl);
    dz = (A.z - pzh) + (B.z - pzl);
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float r2 = B.w;
    if (d2 >= r2 * (1.0f + kAcceptMargin) && r2 > 1e-30f) {
        return true;
    }
    if (d2 <= r2 * (1.0f - kAcceptMargin)) {
        return false;
    }
    return exact_accept(nodes, cur, sorted, n, i);
}

// The per-target union walk: the warp visits the smallest cursor any lane
// holds and only lanes whose cursor is that node act on it. Used when the
// group traversal's stack would overflow. Sums go to acc (FP64, including all
// FP32 partials), counts to pairs / cells.
template <bool QUAD>
__device__ void union_walk(const DeviceNode *__restrict__ nodes,
                           const WalkNode *__restrict__ walk, const uint32_t *__restrict__ first_of,
                           const float4 *__restrict__ leaf_rel, const double *__restrict__ sorted,
                           uint32_t n, uint32_t node_count, float eps2, uint32_t i, bool active,
                           float pxh, float pyh, float pzh, float pxl, float pyl, float pzl,
                           float4 *staged, double &acc_x, double &acc_y, double &acc_z,
                           uint32_t &pairs, uint32_t &cells) {
    const uint32_t lane = threadIdx.x & 31u;
    float cx32 = 0.0f, cy32 = 0.0f, cz32 = 0.0f;
    uint32_t cursor = active ? 0u : 0xffffffffu;
    while (true) {
        const uint32_t cur = warp_min(cursor);
        if (cur >= node_count) {
            break;
        }
        const float4 A = walk[cur].a;
        const float4 B = walk[cur].b;
        const float4 D = walk[cur].d;
        const uint32_t count = __float_as_uint(D.w) & kWalkCountMask;
        const uint32_t next = count > 0u ? cur + 1u : __float_as_uint(D.z);
        bool open_leaf = false;
        float dx = 0.0f, dy = 0.0f, dz = 0.0f;
        if (cursor == cur) {
            const bool accept = lane_accepts(A, B, pxh, pyh, pzh, pxl, pyl, pzl, nodes, cur,
                                             sorted, n, i, dx, dy, dz);
            if (accept) {
                const float r2e = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) + eps2;
                const float inv = rsqrt_approx(r2e);
                const float inv2 = inv * inv;
                const float f = (A.w * inv) * inv2;
                float gx = dx * f, gy = dy * f, gz = dz * f;
                if (QUAD) {
                    const float4 C = walk[cur].c;
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
        if (__any_sync(kFull, open_leaf)) {
            const uint32_t first = first_of[cur];
            const bool own = open_leaf && i >= first && i < first + count;
            const bool masked = __any_sync(kFull, own);
            float sx = 0.0f, sy = 0.0f, sz = 0.0f;
            for (uint32_t base = 0; base < count; base += 32) {
                if (base + lane < count) {
                    staged[lane] = leaf_rel[first + base + lane];
                }
                __syncwarp();
                if (open_leaf) {
                    const uint32_t chunk = min(32u, count - base);
                    for (uint32_t j = 0; j < chunk; ++j) {
                        const float4 s = staged[j];
                        const bool self = masked && first + base + j == i;
                        const float ex = s.x + dx;
                        const float ey = s.y + dy;
                        const float ez = s.z + dz;
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
    acc_x += static_cast<double>(cx32);
    acc_y += static_cast<double>(cy32);
    acc_z += static_cast<double>(cz32);
}


// A node's centre of mass relative to the box centre G, from hi + lo parts.
__device__ __forceinline__ float3 centre_rel(const float4 A, const float4 B, const float4 Gh,
                                             const float4 Gl) {
    return make_float3((A.x - Gh.x) + (B.x - Gl.x), (A.y - Gh.y) + (B.y - Gl.y),
                       (A.z - Gh.z) + (B.z - Gl.z));
}

// Stages accepted cell j: centre relative to G, mass, 2.5 Q and target mask.
template <bool QUAD>
__device__ __forceinline__ void stage_cell(WarpSpace &ws, uint32_t j, float3 c, float m,
                                           uint32_t mask, const float4 C, const float4 D) {
    put(ws.cells[0], j, c.x, c.y);
    put(ws.cells[1], j, c.z, m);
    if (QUAD) {
        put(ws.cells[2], j, 2.5f * C.x, 2.5f * C.y);
        put(ws.cells[3], j, 2.5f * C.z, 2.5f * C.w);
        put(ws.cells[4], j, 2.5f * D.x, 2.5f * D.y);
    }
    ws.cell_mask[j] = mask;
}

// Queues opened leaf k: centre relative to G, size, first particle (with a
// bit when its range may hold one of the warp's targets) and target mask.
__device__ __forceinline__ void queue_leaf(WarpSpace &ws, uint32_t k, float3 c, uint32_t size,
                                           uint32_t first, uint32_t mask, uint32_t warp_first,
                                           uint32_t warp_end) {
    const bool holds = first < warp_end && first + size > warp_first;
    ws.leaf_pos[k] = make_float4(c.x, c.y, c.z, __uint_as_float(size));
    ws.leaf_meta[k] = make_uint2(first | (holds ? 0x80000000u : 0u), mask);
}

// A leaf's first particle and size, checked against the particle count.
__device__ __forceinline__ void leaf_range(uint32_t link, uint32_t count, uint32_t n,
                                           unsigned *status, uint32_t &first, uint32_t &size) {
    first = link;
    size = count;
    if (first > n || size > n - first) {
        atomicOr(status, kStatusInvalid);
        first = 0u;
        size = 0u;
    }
}

// Two staged cells (pair p) for this lane's target: m d / r^3 and, with QUAD,
// the quadrupole term, added to the packed sums (zero outside a cell's mask).
template <bool QUAD>
__device__ __forceinline__ void cell_pair(const WarpSpace &ws, uint32_t p, float2 ntx, float2 nty,
                                          float2 ntz, float2 eps2, uint32_t lane_bit, float2 &sx,
                                          float2 &sy, float2 &sz) {
    const float4 q0 = ws.cells[0][p], q1 = ws.cells[1][p];
    const uint2 masks = *reinterpret_cast<const uint2 *>(&ws.cell_mask[2 * p]);
    const float2 dx = __fadd2_rn(f2(q0.x, q0.y), ntx);
    const float2 dy = __fadd2_rn(f2(q0.z, q0.w), nty);
    const float2 dz = __fadd2_rn(f2(q1.x, q1.y), ntz);
    const float2 r2e = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, eps2)));
    const float inv0 = rsqrt_approx(r2e.x);
    const float inv1 = rsqrt_approx(r2e.y);
    const float2 inv = f2((masks.x & lane_bit) != 0u ? inv0 : 0.0f,
                          (masks.y & lane_bit) != 0u ? inv1 : 0.0f);
    const float2 inv2 = __fmul2_rn(inv, inv);
    const float2 inv3 = __fmul2_rn(inv2, inv);
    // Monopole m d / r^3 (tree_walk.hpp:129-140).
    float2 coef = __fmul2_rn(f2(q1.z, q1.w), inv3);
    if (QUAD) {
        // Quadrupole -Q d / r^5 + 2.5 (d.Q d) d / r^7 (tree_walk.hpp:142-181),
        // folded with the monopole: d (m / r^3 + 2.5 (d.Q d) / r^7) - Q d / r^5.
        const float4 q2 = ws.cells[2][p], q3 = ws.cells[3][p], q4 = ws.cells[4][p];
        const float2 xx = f2(q2.x, q2.y), xy = f2(q2.z, q2.w);
        const float2 xz = f2(q3.x, q3.y), yy = f2(q3.z, q3.w);
        const float2 yz = f2(q4.x, q4.y), zz = f2(q4.z, q4.w);
        const float2 qx = __ffma2_rn(xx, dx, __ffma2_rn(xy, dy, __fmul2_rn(xz, dz)));
        const float2 qy = __ffma2_rn(xy, dx, __ffma2_rn(yy, dy, __fmul2_rn(yz, dz)));
        const float2 qz = __ffma2_rn(xz, dx, __ffma2_rn(yz, dy, __fmul2_rn(zz, dz)));
        // q = 2.5 Q d, quadratic = 2.5 d.Q d.
        const float2 quadratic = __ffma2_rn(dx, qx, __ffma2_rn(dy, qy, __fmul2_rn(dz, qz)));
        const float2 inv5 = __fmul2_rn(inv3, inv2);
        coef = __ffma2_rn(quadratic, __fmul2_rn(inv5, inv2), coef);
        const float2 ninv5 = __fmul2_rn(inv5, f2(-0.4f, -0.4f));
        sx = __ffma2_rn(qx, ninv5, sx);
        sy = __ffma2_rn(qy, ninv5, sy);
        sz = __ffma2_rn(qz, ninv5, sz);
    }
    sx = __ffma2_rn(dx, coef, sx);
    sy = __ffma2_rn(dy, coef, sy);
    sz = __ffma2_rn(dz, coef, sz);
}

// Evaluates the staged cells: every lane sums every cell for its target (zero
// outside the cell's mask), two cells per FP32x2 instruction, four per loop
// step (the batch is padded with neutral entries to a multiple of four).
// Each lane holds its target relative to G, so the offset to a cell is one
// subtraction.
template <bool QUAD>
__device__ __forceinline__ void flush_cells(WarpSpace &ws, uint32_t count, float2 ntx, float2 nty,
                                            float2 ntz, float2 eps2, uint32_t lane_bit,
                                            double &acc_x, double &acc_y, double &acc_z) {
    const uint32_t lane = threadIdx.x & 31u;
    if ((count & 1u) != 0u && lane == 0) {
        // The odd entry's partner: no target, zero mass, at G.
        for (int q = 0; q < kCellQuads; ++q) {
            put(ws.cells[q], count, 0.0f, 0.0f);
        }
        ws.cell_mask[count] = 0u;
    }
    __syncwarp();
    float2 sx = f2(0.0f, 0.0f), sy = sx, sz = sx;
    for (uint32_t j = 0; j < count; j += 2) {
        cell_pair<QUAD>(ws, j >> 1, ntx, nty, ntz, eps2, lane_bit, sx, sy, sz);
    }
    __syncwarp();
    acc_x += static_cast<double>(sx.x) + static_cast<double>(sx.y);
    acc_y += static_cast<double>(sy.x) + static_cast<double>(sy.y);
    acc_z += static_cast<double>(sz.x) + static_cast<double>(sz.y);
}

// Evaluates the queued leaves: for each, every lane sums its particles for its
// own target (staged in shared memory once per chunk of 32; lanes outside the
// leaf's mask sit far away and add exactly zero), two sources per FP32x2
// instruction, skipping the target itself where the leaf's range may hold it.
__device__ __forceinline__ void flush_leaves(WarpSpace &ws, uint32_t count,
                                             const float4 *__restrict__ leaf_rel, float tgx,
                                             float tgy, float tgz, float eps2, uint32_t i,
                                             uint32_t lane_bit, double &acc_x, double &acc_y,
                                             double &acc_z, uint32_t &pairs) {
    const uint32_t lane = threadIdx.x & 31u;
    const float2 e2 = f2(eps2, eps2);
    float2 sx = f2(0.0f, 0.0f), sy = sx, sz = sx;
    for (uint32_t k = 0; k < count; ++k) {
        const float4 pos = ws.leaf_pos[k];
        const uint2 e = ws.leaf_meta[k];
        const uint32_t size = __float_as_uint(pos.w);
        const uint32_t first = e.x & 0x7fffffffu;
        const bool masked = (e.x >> 31) != 0u; // uniform: every lane reads the same entry
        const bool in = (e.y & lane_bit) != 0u;
        const bool own = in && i >= first && i < first + size;
        // Offset leaf centre of mass - target; source - target = source + d.
        // Lanes outside the mask sit far away: their terms are exactly zero.
        const float dx = in ? pos.x - tgx : kFar;
        const float dy = in ? pos.y - tgy : kFar;
        const float dz = in ? pos.z - tgz : kFar;
        const float2 dx2 = f2(dx, dx), dy2 = f2(dy, dy), dz2 = f2(dz, dz);
        for (uint32_t base = 0; base < size; base += 32) {
            const uint32_t chunk = min(32u, size - base);
            float4(*lq)[17] = ws.leaf_quads;
            if (lane < chunk) {
                const float4 src = leaf_rel[first + base + lane];
                put(lq[0], lane, src.x, src.y);
                put(lq[1], lane, src.z, src.w);
            } else if (lane == chunk) {
                // Neutral partner: far away and massless.
                put(lq[0], lane, kFar, kFar);
                put(lq[1], lane, kFar, 0.0f);
            }
            __syncwarp();
            // Every lane runs the loop (no divergent region).
            if (!masked) {
                for (uint32_t j = 0; j < chunk; j += 2) {
                    const uint32_t p = j >> 1;
                    const float4 s0 = lq[0][p], s1 = lq[1][p];
                    const float2 ex = __fadd2_rn(f2(s0.x, s0.y), dx2);
                    const float2 ey = __fadd2_rn(f2(s0.z, s0.w), dy2);
                    const float2 ez = __fadd2_rn(f2(s1.x, s1.y), dz2);
                    const float2 r2 =
                        __ffma2_rn(ez, ez, __ffma2_rn(ey, ey, __ffma2_rn(ex, ex, e2)));
                    const float2 inv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                    const float2 f =
                        __fmul2_rn(__fmul2_rn(f2(s1.z, s1.w), inv), __fmul2_rn(inv, inv));
                    sx = __ffma2_rn(f, ex, sx);
                    sy = __ffma2_rn(f, ey, sy);
                    sz = __ffma2_rn(f, ez, sz);
                }
            } else {
                for (uint32_t j = 0; j < chunk; j += 2) {
                    const uint32_t p = j >> 1;
                    const float4 s0 = lq[0][p], s1 = lq[1][p];
                    const float2 ex = __fadd2_rn(f2(s0.x, s0.y), dx2);
                    const float2 ey = __fadd2_rn(f2(s0.z, s0.w), dy2);
                    const float2 ez = __fadd2_rn(f2(s1.x, s1.y), dz2);
                    float2 r2 = __ffma2_rn(ez, ez, __ffma2_rn(ey, ey, __ffma2_rn(ex, ex, e2)));
                    // The target itself contributes nothing.
                    const uint32_t index = first + base + j;
                    const bool skip0 = index == i;
                    const bool skip1 = index + 1 == i;
                    r2 = f2(skip0 ? 1.0f : r2.x, skip1 ? 1.0f : r2.y);
                    const float2 m = f2(skip0 ? 0.0f : s1.z, skip1 ? 0.0f : s1.w);
                    const float2 inv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                    const float2 f = __fmul2_rn(__fmul2_rn(m, inv), __fmul2_rn(inv, inv));
                    sx = __ffma2_rn(f, ex, sx);
                    sy = __ffma2_rn(f, ey, sy);
                    sz = __ffma2_rn(f, ez, sz);
                }
            }
            __syncwarp();
        }
        pairs += in ? size - (own ? 1u : 0u) : 0u;
    }
    acc_x += static_cast<double>(sx.x) + static_cast<double>(sx.y);
    acc_y += static_cast<double>(sy.x) + static_cast<double>(sy.y);
    acc_z += static_cast<double>(sz.x) + static_cast<double>(sz.y);
}

template <bool QUAD>
__global__ void __launch_bounds__(kWalkThreads, 8)
    walk_kernel(const DeviceNode *__restrict__ nodes, const WalkNode *__restrict__ walk,
                const uint32_t *__restrict__ first_of, const float4 *__restrict__ leaf_rel,
                const double *__restrict__ sorted, const uint32_t *__restrict__ perm, uint32_t n,
                float eps2, double *ax, double *ay, double *az, const TreeMeta *meta,
                unsigned long long *counters, unsigned *status, uint32_t stack_cap) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    WarpSpace &ws = reinterpret_cast<WarpSpace *>(smem)[warp];
    const uint32_t i = (blockIdx.x * kWalkWarps + warp) * 32u + lane;
    const bool active = i < n;
    const uint32_t live = __ballot_sync(kFull, active);
    if (live == 0u) {
        return; // the whole warp lies past the last target
    }
    const uint32_t node_count = meta->node_count;
    const uint32_t lane_bit = 1u << lane;
    const uint32_t warp_first = i - lane;
    const uint32_t warp_end = min(warp_first + 32u, n);

    double X = 0.0, Y = 0.0, Z = 0.0;
    float pxh = 0.0f, pyh = 0.0f, pzh = 0.0f, pxl = 0.0f, pyl = 0.0f, pzl = 0.0f;
    if (active) {
        X = sorted[i];
        Y = sorted[static_cast<size_t>(n) + i];
        Z = sorted[2ull * n + i];
        split(X, pxh, pxl);
        split(Y, pyh, pyl);
        split(Z, pzh, pzl);
    }
    const float2 eps2v = f2(eps2, eps2);

    // FP64 bounding box of the warp's targets.
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    double lox = active ? X : inf, loy = active ? Y : inf, loz = active ? Z : inf;
    double hix = active ? X : -inf, hiy = active ? Y : -inf, hiz = active ? Z : -inf;
    for (int off = 16; off > 0; off >>= 1) {
        lox = fmin(lox, __shfl_xor_sync(kFull, lox, off));
        loy = fmin(loy, __shfl_xor_sync(kFull, loy, off));
        loz = fmin(loz, __shfl_xor_sync(kFull, loz, off));
        hix = fmax(hix, __shfl_xor_sync(kFull, hix, off));
        hiy = fmax(hiy, __shfl_xor_sync(kFull, hiy, off));
        hiz = fmax(hiz, __shfl_xor_sync(kFull, hiz, off));
    }

    // The box centre G and this lane's target relative to it (FP32).
    const double gcx = 0.5 * (lox + hix), gcy = 0.5 * (loy + hiy), gcz = 0.5 * (loz + hiz);
    const float tgx = __double2float_rn(X - gcx), tgy = __double2float_rn(Y - gcy),
                tgz = __double2float_rn(Z - gcz);
    const float2 ntx = f2(-tgx, -tgx), nty = f2(-tgy, -tgy), ntz = f2(-tgz, -tgz);
    if (lane < 6) {
        // Lanes 0-5 split one box value each: lo, hi, G (x, y, z).
        const double v[3] = {lane < 2 ? lox : lane < 4 ? hix : gcx,
                             lane < 2 ? loy : lane < 4 ? hiy : gcy,
                             lane < 2 ? loz : lane < 4 ? hiz : gcz};
        float h[3], l[3];
        for (int a = 0; a < 3; ++a) {
            split(v[a], h[a], l[a]);
        }
        // Slots: 0 lo hi, 1 lo lo, 2 hi hi, 3 hi lo, 4 G hi, 5 G lo.
        ws.box[lane] = (lane & 1u) == 0u ? make_float4(h[0], h[1], h[2], 0.0f)
                                          : make_float4(l[0], l[1], l[2], 0.0f);
    }
    __syncwarp();

    double acc_x = 0.0, acc_y = 0.0, acc_z = 0.0;
    uint32_t pairs = 0, cells = 0;
    uint32_t size = 1, ncell = 0, nleaf = 0;
    bool overflow = false;
    uint32_t rounds = 0;
    if (lane == 0) {
        ws.stack[0] = make_uint2(0u, live);
    }
    __syncwarp();
    while (size > 0) {
        // Popping t items and pushing up to 2t needs size + t <= stack_cap.
        const uint32_t take = min(min(size, 32u), stack_cap - min(size, stack_cap));
        // A valid tree visits each node at most once, so more rounds than
        // nodes (or a full stack) hands the warp to the union walk, whose
        // cursors only move forward.
        if (take == 0u || ++rounds > node_count + 1u) {
            overflow = true;
            break;
        }
        size -= take;
        const bool has = lane < take;
        uint2 item = make_uint2(0u, 0u);
        if (has) {
            item = ws.stack[size + lane];
            if (item.x >= node_count) {
                atomicOr(status, kStatusInvalid);
                item.x = node_count; // skipped below
            }
        }
        __syncwarp();

        // Classify the lane's node against the box from its compact record:
        // every target accepts it (cell_mask = the item's mask), every target
        // opens it (open_mask), or each target decides for itself (mixed).
        bool sibling = false, mixed = false;
        uint32_t next = 0, count = 0, cell_mask = 0u, open_mask = 0u;
        float4 A = make_float4(0.0f, 0.0f, 0.0f, 0.0f), B = A, C = A, D = A;
        if (has && item.x < node_count) {
            A = walk[item.x].a;
            B = walk[item.x].b;
            D = walk[item.x].d;
            const uint32_t word = __float_as_uint(D.w);
            count = word & kWalkCountMask;
            next = count > 0u ? item.x + 1u : __float_as_uint(D.z);
            sibling = (word & kWalkSiblingBit) != 0u;
            const float4 loh = ws.box[0], lol = ws.box[1], hih = ws.box[2], hil = ws.box[3];
            // Signed distances lo - c and c - hi per axis, from hi + lo parts.
            const float lx = (loh.x - A.x) + (lol.x - B.x), ux = (A.x - hih.x) + (B.x - hil.x);
            const float ly = (loh.y - A.y) + (lol.y - B.y), uy = (A.y - hih.y) + (B.y - hil.y);
            const float lz = (loh.z - A.z) + (lol.z - B.z), uz = (A.z - hih.z) + (B.z - hil.z);
            const float nx = fmaxf(fmaxf(lx, ux), 0.0f);
            const float ny = fmaxf(fmaxf(ly, uy), 0.0f);
            const float nz = fmaxf(fmaxf(lz, uz), 0.0f);
            const float fx = fmaxf(fabsf(lx), fabsf(ux));
            const float fy = fmaxf(fabsf(ly), fabsf(uy));
            const float fz = fmaxf(fabsf(lz), fabsf(uz));
            const float near2 = fmaf(nz, nz, fmaf(ny, ny, nx * nx));
            const float far2 = fmaf(fz, fz, fmaf(fy, fy, fx * fx));
            const float r2 = B.w;
            if (near2 >= r2 * (1.0f + kAcceptMargin) && r2 > 1e-30f) {
                cell_mask = item.y;
            } else if (far2 < r2 * (1.0f - kAcceptMargin)) {
                open_mask = item.y;
            } else {
                mixed = true;
            }
        }
        const uint32_t below = lanes_below(lane);
        const uint32_t bs = __ballot_sync(kFull, sibling);
        if (sibling) {
            ws.stack[size + __popc(bs & below)] = make_uint2(next, item.y);
        }
        size += __popc(bs);

        // Mixed nodes: each target in the mask decides for itself; the lane
        // that classified the node keeps the accepted and opened masks.
        for (uint32_t bm = __ballot_sync(kFull, mixed); bm != 0u; bm &= bm - 1u) {
            const uint32_t owner = __ffs(bm) - 1u;
            const uint32_t v = __shfl_sync(kFull, item.x, owner);
            const uint32_t mask = __shfl_sync(kFull, item.y, owner);
            const float4 MA = walk[v].a;
            const float4 MB = walk[v].b;
            // FP32 test on every lane; the FP64 test, when any lane of the
            // mask falls inside the margin, on every lane too.
            const bool reach = (mask & lane_bit) != 0u;
            const float dx = (MA.x - pxh) + (MB.x - pxl);
            const float dy = (MA.y - pyh) + (MB.y - pyl);
            const float dz = (MA.z - pzh) + (MB.z - pzl);
            const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            const float r2 = MB.w;
            const bool sure_accept = d2 >= r2 * (1.0f + kAcceptMargin) && r2 > 1e-30f;
            const bool sure_open = d2 <= r2 * (1.0f - kAcceptMargin);
            bool accept = reach && sure_accept;
            const bool unsure = reach && !sure_accept && !sure_open;
            if (__any_sync(kFull, unsure)) {
                const bool exact = exact_accept(nodes, v, sorted, n, active ? i : 0u);
                accept = accept || (unsure && exact);
            }
            const uint32_t accepted = __ballot_sync(kFull, accept) & mask;
            if (lane == owner) {
                cell_mask = accepted;
                open_mask = mask & ~accepted;
            }
        }

        // Every lane files its node's outcome: a staged cell for the targets
        // that accept it, and for those that open it a queued leaf or a pushed
        // first child.
        const bool cell = cell_mask != 0u;
        const bool leaf = open_mask != 0u && count > 0u;
        const bool child = open_mask != 0u && count == 0u;
        const uint32_t ba = __ballot_sync(kFull, cell);
        const uint32_t bl = __ballot_sync(kFull, leaf);
        const uint32_t bc = __ballot_sync(kFull, child);
        if (child) {
            ws.stack[size + __popc(bc & below)] = make_uint2(item.x + 1u, open_mask);
        }
        if (cell || leaf) {
            const float4 Gh = ws.box[4], Gl = ws.box[5];
            const float3 c = centre_rel(A, B, Gh, Gl);
            if (cell) {
                if (QUAD) {
                    C = walk[item.x].c;
                }
                stage_cell<QUAD>(ws, ncell + __popc(ba & below), c, A.w, cell_mask, C, D);
                cells += __popc(cell_mask); // every target of the mask takes the cell
            }
            if (leaf) {
                uint32_t first, lsize;
                leaf_range(__float_as_uint(D.z), count, n, status, first, lsize);
                queue_leaf(ws, nleaf + __popc(bl & below), c, lsize, first, open_mask,
                           warp_first, warp_end);
            }
        }
        size += __popc(bc);
        ncell += __popc(ba);
        nleaf += __popc(bl);
        __syncwarp();
        if (ncell > kCellCap - 32u) {
            flush_cells<QUAD>(ws, ncell, ntx, nty, ntz, eps2v, lane_bit, acc_x, acc_y, acc_z);
            ncell = 0;
        }
        if (nleaf > kLeafCap - 32u) {
            flush_leaves(ws, nleaf, leaf_rel, tgx, tgy, tgz, eps2, i, lane_bit, acc_x, acc_y,
                         acc_z, pairs);
            nleaf = 0;
        }
    }
    if (overflow) {
        acc_x = acc_y = acc_z = 0.0;
        pairs = cells = 0;
        union_walk<QUAD>(nodes, walk, first_of, leaf_rel, sorted, n, node_count, eps2, i, active,
                         pxh, pyh, pzh, pxl, pyl, pzl, ws.union_staged, acc_x, acc_y, acc_z, pairs,
                         cells);
    } else {
        flush_cells<QUAD>(ws, ncell, ntx, nty, ntz, eps2v, lane_bit, acc_x, acc_y, acc_z);
        flush_leaves(ws, nleaf, leaf_rel, tgx, tgy, tgz, eps2, i, lane_bit, acc_x, acc_y, acc_z,
                     pairs);
    }

    if (active) {
        const uint32_t j = perm[i];
        ax[j] = acc_x;
        ay[j] = acc_y;
        az[j] = acc_z;
    }
    // pairs: per target; cells: tallied by the lanes that queued the entries.
    unsigned long long p = active ? pairs : 0u, c = cells;
    for (int off = 16; off > 0; off >>= 1) {
        p += __shfl_down_sync(kFull, p, off);
        c += __shfl_down_sync(kFull, c, off);
    }
    if (lane == 0 && (p | c) != 0ull) {
        atomicAdd(&counters[0], p);
        atomicAdd(&counters[1], c);
    }
}

} // namespace

uint32_t walk_stack_capacity() { return kStackCap; }

cudaError_t launch_walk(const DeviceNode *nodes, const WalkNode *walk_nodes,
                        const uint32_t *first_of, const float4 *leaf_rel, const double *sorted,
                        const uint32_t *perm, uint32_t n, double eps2, bool quadrupole,
                        double *ax, double *ay, double *az, TreeMeta *meta,
                        unsigned long long *counters, unsigned *status, cudaStream_t stream,
                        uint32_t stack_cap) {
    if (n == 0) {
        return cudaSuccess;
    }
    const uint32_t cap = stack_cap == 0u || stack_cap > kStackCap ? kStackCap : stack_cap;
    const uint32_t blocks = ceil_div(n, static_cast<uint32_t>(kWalkThreads));
    const float eps2f = static_cast<float>(eps2);
    const size_t smem = kWalkWarps * sizeof(WarpSpace);
    if (quadrupole) {
        walk_kernel<true><<<blocks, kWalkThreads, smem, stream>>>(
            nodes, walk_nodes, first_of, leaf_rel, sorted, perm, n, eps2f, ax, ay, az, meta,
            counters, status, cap);
    } else {
        walk_kernel<false><<<blocks, kWalkThreads, smem, stream>>>(
            nodes, walk_nodes, first_of, leaf_rel, sorted, perm, n, eps2f, ax, ay, az, meta,
            counters, status, cap);
    }
    return cudaGetLastError();
}

} // namespace ob
