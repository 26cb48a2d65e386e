// Tree evaluation: the traversal of vortex_tree.tree_velocity (src/openfawe/aero/vortex_tree.py:508-568) on the GPU.
//
// A warp walks the tree depth first (left child first) with one shared stack whose entries carry the mask of lanes
// (targets) that opened the parent.  Each lane decides acceptance for itself, with the reference's FP64 test
// (bound < theta |R|, |R| - bound >= clearance * core, no excluded segment inside), so every target visits exactly the
// nodes, in exactly the order, of the per-target CPU traversal; lanes only share the walk.  Targets are sorted by the
// Morton key of their positions so that a warp's targets are neighbours and their node sets overlap.
// Exclusions: the target's excluded segments as sorted tree positions (vortex_tree._positions, :571-580) and a cursor
// that only moves forward, because depth-first visits see non-decreasing range starts.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <thread>

#include "bs_sort.cuh"
#include <cstdlib>

#include "bs_tree.cuh"

namespace bs {

constexpr int STACK_DEPTH = 128;
constexpr int FAR_COST = 16;              // list cost units: one far evaluation ~ sixteen near pairs (measured)
constexpr int LIST_WARPS = 4;             // warps per block of the list kernel
constexpr int LIST_NEAR_BLOCKS = 4;       // near-leaf kernel blocks a SM (128 registers a thread)
constexpr int LIST_FAR_BLOCKS = 3;        // far-node kernel blocks a SM (57.9 KB of shared memory each)
constexpr int FAR_GROUPS = 4;             // open groups of disjoint far entries in the far list kernel
constexpr int FAR_STAGE = 4;              // distinct nodes a group holds: their FP32 records are staged together
constexpr int FAR_REC4 = 100;             // float4 of a staged node: FP32 far records to fifth order (12 + 16 + 28 +
                                          // 42), then its centre (three doubles and a pad)
constexpr int ENTRY_BUF = 64;             // list entries a warp of the list kernels reads ahead into shared memory
constexpr int FAR_QUEUE = 32;             // closed far groups a warp queues before it evaluates them
// dynamic shared memory a warp of the far list kernel uses: two staging buffers, the group queue, the entry buffer
constexpr size_t FAR_WARP_SMEM = 2 * FAR_STAGE * FAR_REC4 * sizeof(float4) +
                                 FAR_QUEUE * (2 * FAR_STAGE + 1) * sizeof(int) + ENTRY_BUF * sizeof(int2);

struct TreeView {
    const NodeRec *nodes;
    const Far64 *far64;
    const Far32 *far32;
    const Far64x *far64x;  // third-order records, or null
    const Far32x *far32x;
    const Far64y *far64y;  // fourth-order records, or null
    const Far32y *far32y;
    const Far64z *far64z;  // fifth-order records, or null
    const Far32z *far32z;
    const Seg64 *seg64;
    const Seg32 *seg32;
    const Seg32x2 *seg32x2;
    const Seg32c2 *seg32c2;
};

struct EvalArgs {
    int64_t n;
    const double *points;
    const int32_t *perm;
    const int64_t *ex_ptr;
    const int32_t *ex_pos;
    TreeView tv;
    double theta, theta2, clearance;
    int order, model, raise_singular, stack_limit;
    int deferred;  // the segment and far records may still be in computation while the walk runs: it must not read them
    int fill;      // a leaf opened for a lane is summed exactly for every lane of the warp that reached it (below)
    float near2;
    // interaction lists: entries live in chunks of LIST_CHUNK taken from a shared pool; warp gw of targets lists its
    // chunks in unit_chunks[gw][0 .. LIST_CHUNKS)
    int2 *list;          // (node, lane mask); far entries carry FAR_BIT in the node
    int *list_cost;      // cost before each entry
    int *unit_chunks;
    unsigned long long *pool_cursor;
    unsigned long long pool_chunks;
    int *list_len;       // entries per warp
    int *list_total;     // total cost per warp
    // what the walk evaluates itself (list overflow) and per-target results
    double *walk_u;
    int8_t *walk_flag;
    int64_t *far_counts;
    int *overflow;
    unsigned long long *counters;  // far evaluations, near pairs, fp64 pairs, visits, lane slots of leaf walks
    // list kernel: work items by warp of targets, each warp's list cut into a number of items proportional to its cost
    // (item_off [target_warps + 1], from item_plan_kernel), and the items' partial sums
    int *item_off;
    int *item_warp;      // [capacity]: the warp of targets of each item
    int *item_first;     // [capacity]: the first list entry of each item (item_bounds_kernel)
    int item_want;       // items wanted in all (about 96 a SM); the capacity is item_want + target warps
    double *partial;     // [items][32 lanes][3]: each item's near leaves (tree_list_kernel<.., 0>), then its far
                         // nodes added (tree_list_kernel<.., 1>, which runs after it)
    int8_t *pflag;       // [items][32 lanes]
    const int32_t *root_of;       // forests: root node of each (sorted) target's wake, -1 for none; null: node 0
    unsigned long long *queue;    // work counter of the persistent list kernel
    const uint8_t *exact;         // per target (input order), or null: nonzero = no far node is accepted for it (its
                                  // velocity is the exact sum over every segment, in tree order)
};

// Per-lane state of a target.
struct Target {
    double x0, x1, x2;
    float xh0, xl0, xh1, xl1, xh2, xl2;
    int64_t p;
    bool valid;
    bool packed;  // finite coordinates below 1e30: the packed pair may take this target
    __device__ void load(const EvalArgs &a, int64_t i) {
        valid = i < a.n;
        p = valid ? a.perm[i] : 0;
        x0 = x1 = x2 = 0.0;
        if (valid) { x0 = a.points[3 * p]; x1 = a.points[3 * p + 1]; x2 = a.points[3 * p + 2]; }
        split2(x0, xh0, xl0);
        split2(x1, xh1, xl1);
        split2(x2, xh2, xl2);
        packed = fabs(x0) < 1e30 && fabs(x1) < 1e30 && fabs(x2) < 1e30;
    }
};

// Sums of one target in its precision: FP64 for fp64/mixed, FP32 for fp32.
template <int PREC> struct Acc {
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;
    __device__ void add64(double a, double b, double c) {
        if (PREC == 2) { f0 += (float)a; f1 += (float)b; f2 += (float)c; }
        else { u0 += a; u1 += b; u2 += c; }
    }
    __device__ void add32(float a, float b, float c) {
        if (PREC == 2) { f0 += a; f1 += b; f2 += c; }
        else { u0 += a; u1 += b; u2 += c; }
    }
    __device__ double x() const { return PREC == 2 ? (double)f0 : u0; }
    __device__ double y() const { return PREC == 2 ? (double)f1 : u1; }
    __device__ double z() const { return PREC == 2 ? (double)f2 : u2; }
};

template <int PREC>
__device__ __forceinline__ void far_node(const EvalArgs &a, const Target &t, int node, Acc<PREC> &acc) {
    const NodeRec nr = a.tv.nodes[node];
    const double rx = t.x0 - nr.cx, ry = t.x1 - nr.cy, rz = t.x2 - nr.cz;
    if (PREC == 0) {
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        far_eval<double>(rx, ry, rz, a.tv.far64[node].v, a.order, g0, g1, g2,
                         a.order >= 3 ? a.tv.far64x[node].v : nullptr, a.order >= 4 ? a.tv.far64y[node].v : nullptr,
                         a.order >= 5 ? a.tv.far64z[node].v : nullptr);
        acc.add64(g0, g1, g2);
    } else {
        float g0 = 0.f, g1 = 0.f, g2 = 0.f;
        far_eval32v((float)rx, (float)ry, (float)rz, reinterpret_cast<const float4 *>(a.tv.far32[node].v), a.order,
                    g0, g1, g2, a.order >= 3 ? reinterpret_cast<const float4 *>(a.tv.far32x[node].v) : nullptr,
                    a.order >= 4 ? reinterpret_cast<const float4 *>(a.tv.far32y[node].v) : nullptr,
                    a.order >= 5 ? reinterpret_cast<const float4 *>(a.tv.far32z[node].v) : nullptr);
        acc.add32(g0, g1, g2);
    }
}

// float4 i of node j's FP32 far records in staging order (Far32, then Far32x, Far32y, Far32z as the order has them).
__device__ __forceinline__ const float4 *far_rec4(const TreeView &tv, int j, int i) {
    if (i < 12) return reinterpret_cast<const float4 *>(tv.far32[j].v) + i;
    if (i < 28) return reinterpret_cast<const float4 *>(tv.far32x[j].v) + (i - 12);
    if (i < 56) return reinterpret_cast<const float4 *>(tv.far32y[j].v) + (i - 28);
    return reinterpret_cast<const float4 *>(tv.far32z[j].v) + (i - 56);
}

// float4 of FP32 far records a node carries at `order`.
__device__ __forceinline__ int far_rec4_count(int order) {
    return 12 + (order >= 3 ? 16 : 0) + (order >= 4 ? 28 : 0) + (order >= 5 ? 42 : 0);
}

// far_node (single precision) from a staged copy of the node's records (far_rec4 order).
template <int PREC>
__device__ __forceinline__ void far_node_staged(const EvalArgs &a, const Target &t, int node, const float4 *st,
                                                Acc<PREC> &acc) {
    const double *c = reinterpret_cast<const double *>(st + FAR_REC4 - 2);  // the staged centre
    const double rx = t.x0 - c[0], ry = t.x1 - c[1], rz = t.x2 - c[2];
    float g0 = 0.f, g1 = 0.f, g2 = 0.f;
    far_eval32v<true>((float)rx, (float)ry, (float)rz, st, a.order, g0, g1, g2, a.order >= 3 ? st + 12 : nullptr,
                      a.order >= 4 ? st + 28 : nullptr, a.order >= 5 ? st + 56 : nullptr);
    acc.add32(g0, g1, g2);
}

// FP64 re-evaluation of the pairs of segments base + j (bits of `need`): value added or flag recorded.
template <int PREC, int MODEL>
__device__ __forceinline__ void pairs_in_fp64(const EvalArgs &a, const Target &t, int base, unsigned need,
                                              Acc<PREC> &acc, int &flag) {
    while (need) {
        const int j = __ffs(need) - 1;
        need &= need - 1;
        double v0 = 0.0, v1 = 0.0, v2 = 0.0;
        const int fl = pair64_at(t.x0, t.x1, t.x2, a.tv.seg64[base + j], MODEL, a.raise_singular, v0, v1, v2);
        if (fl != BS_FLAG_OK) {
            if (flag == BS_FLAG_OK) flag = fl;
        } else {
            acc.add64(v0, v1, v2);
        }
    }
}

// One segment for one lane in single precision, read from the tree-ordered Seg32 array (the leaf's odd ends and the
// tiles the packed path leaves out).
template <int PREC, int MODEL>
__device__ __forceinline__ void single_pair(const EvalArgs &a, const Target &t, int s, float &t0, float &t1, float &t2,
                                            Acc<PREC> &acc, int &flag, long long &fp64_pairs) {
    const Seg32 r = a.tv.seg32[s];
    const float q0 = (t.xh0 - r.hi.x) + (t.xl0 - r.lo.x);
    const float q1 = (t.xh1 - r.hi.y) + (t.xl1 - r.lo.y);
    const float q2 = (t.xh2 - r.hi.z) + (t.xl2 - r.lo.z);
    if (pair32<MODEL>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) {
        ++fp64_pairs;
        pairs_in_fp64<PREC, MODEL>(a, t, s, 1u, acc, flag);
    }
}

// One leaf of a single-precision evaluation with MODEL 0..2, two segments per operation: the leaf's whole pairs of
// consecutive segments [2 p0, 2 p1) are staged a tile at a time, and a walking lane evaluates a tile
// two segments per operation when none of its segments is excluded for it (otherwise, and for targets the packed
// pair does not take, segment by segment with pair32); the odd ends of the leaf go through pair32.  When every
// walking lane is clear of the leaf (`wide`: see pair32x2_clear) the tiles are 32 Seg32c2 records and the pairs
// pair32x2_clear, from the lane's offset `rel` to the leaf's centre; otherwise 16 Seg32x2 records and pair32x2.
// Exclusions are consumed in position order through the lane's cursor e.
template <int PREC, int MODEL>
__device__ __forceinline__ void leaf_pairs_packed(const EvalArgs &a, const Target &t, int lo, int hi, bool walk,
                                                  bool all_clear, bool wide, float3 rel, int64_t &e, int64_t e1,
                                                  float4 *tile, Acc<PREC> &acc, int &flag, long long &near_pairs,
                                                  long long &fp64_pairs) {
    const int lane = threadIdx.x & 31;
    float t0 = 0.f, t1 = 0.f, t2 = 0.f;
    float2 u0 = make_float2(0.f, 0.f), u1 = u0, u2 = u0;
    const float2 txh = make_float2(t.xh0, t.xh0), tyh = make_float2(t.xh1, t.xh1), tzh = make_float2(t.xh2, t.xh2);
    const float2 txl = make_float2(t.xl0, t.xl0), tyl = make_float2(t.xl1, t.xl1), tzl = make_float2(t.xl2, t.xl2);
    const float2 rx = make_float2(rel.x, rel.x), ry = make_float2(rel.y, rel.y), rz = make_float2(rel.z, rel.z);
    // an excluded segment at position s: consume it and report
    auto excluded = [&](int s) -> bool {
        while (e < e1 && a.ex_pos[e] < s) ++e;
        if (e < e1 && a.ex_pos[e] == s) {
            ++e;
            return true;
        }
        return false;
    };
    const int p0 = (lo + 1) >> 1, p1 = hi >> 1;
    if (walk && (lo & 1)) {  // the leaf's first segment, when it starts a pair with the previous leaf's last
        if (!excluded(lo)) {
            ++near_pairs;
            single_pair<PREC, MODEL>(a, t, lo, t0, t1, t2, acc, flag, fp64_pairs);
        }
    }
    // clear leaves: tiles of 32 Seg32c2 records (the warp's 3 KB), 64 segments
    for (int pb = p0; wide && pb < p1; pb += 32) {
        const int np = min(32, p1 - pb), base = 2 * pb, cnt = 2 * np;
        __syncwarp();
        const float4 *src = reinterpret_cast<const float4 *>(a.tv.seg32c2 + pb);
        for (int i = lane; i < 6 * np; i += 32) tile[i] = __ldg(src + i);
        __syncwarp();
        if (!walk) continue;
        unsigned long long excl = 0;
        while (e < e1 && a.ex_pos[e] < base + cnt) excl |= 1ull << (a.ex_pos[e++] - base);
        near_pairs += cnt - __popcll(excl);
        if (excl == 0 && t.packed) {
#pragma unroll 4
            for (int q = 0; q < np; ++q) pair32x2_clear<MODEL>(rx, ry, rz, tile + 6 * q, u0, u1, u2);
        } else {
            unsigned long long need = 0;
            for (int j = 0; j < cnt; ++j) {
                if ((excl >> j) & 1ull) continue;
                const Seg32 r = a.tv.seg32[base + j];
                const float q0 = (t.xh0 - r.hi.x) + (t.xl0 - r.lo.x);
                const float q1 = (t.xh1 - r.hi.y) + (t.xl1 - r.lo.y);
                const float q2 = (t.xh2 - r.hi.z) + (t.xl2 - r.lo.z);
                if (pair32<MODEL>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1ull << j;
            }
            fp64_pairs += __popcll(need);
            pairs_in_fp64<PREC, MODEL>(a, t, base, (unsigned)need, acc, flag);
            pairs_in_fp64<PREC, MODEL>(a, t, base + 32, (unsigned)(need >> 32), acc, flag);
        }
    }
    for (int pb = p0; !wide && pb < p1; pb += 16) {
        const int np = min(16, p1 - pb), base = 2 * pb, cnt = 2 * np;
        __syncwarp();
        const float4 *src = reinterpret_cast<const float4 *>(a.tv.seg32x2 + pb);
        for (int i = lane; i < 8 * np; i += 32) tile[i] = __ldg(src + i);
        __syncwarp();
        if (!walk) continue;
        unsigned excl = 0;
        while (e < e1 && a.ex_pos[e] < base + cnt) excl |= 1u << (a.ex_pos[e++] - base);
        near_pairs += cnt - __popc(excl);
        unsigned need = 0;
        if (excl == 0 && t.packed) {
            if (all_clear) {
#pragma unroll 4
                for (int q = 0; q < np; ++q)
                    need |= pair32x2<MODEL, false>(txh, tyh, tzh, txl, tyl, tzl, tile + 8 * q, a.near2, u0, u1, u2)
                            << (2 * q);
            } else {
#pragma unroll 2
                for (int q = 0; q < np; ++q)
                    need |= pair32x2<MODEL, true>(txh, tyh, tzh, txl, tyl, tzl, tile + 8 * q, a.near2, u0, u1, u2)
                            << (2 * q);
            }
        } else {
            for (int j = 0; j < cnt; ++j) {
                if ((excl >> j) & 1u) continue;
                const Seg32 r = a.tv.seg32[base + j];
                const float q0 = (t.xh0 - r.hi.x) + (t.xl0 - r.lo.x);
                const float q1 = (t.xh1 - r.hi.y) + (t.xl1 - r.lo.y);
                const float q2 = (t.xh2 - r.hi.z) + (t.xl2 - r.lo.z);
                if (pair32<MODEL>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1u << j;
            }
        }
        fp64_pairs += __popc(need);
        pairs_in_fp64<PREC, MODEL>(a, t, base, need, acc, flag);
    }
    if (walk && (hi & 1) && hi - 1 >= lo && hi - 1 >= 2 * p1) {  // the leaf's last segment, when it ends unpaired
        if (!excluded(hi - 1)) {
            ++near_pairs;
            single_pair<PREC, MODEL>(a, t, hi - 1, t0, t1, t2, acc, flag, fp64_pairs);
        }
    }
    if (walk) acc.add32(t0 + (u0.x + u0.y), t1 + (u1.x + u1.y), t2 + (u2.x + u2.y));
}

// One leaf for the lanes in `walk`: the warp stages the leaf's records in shared memory 32 at a time, then every
// walking lane evaluates its pairs (exclusions skipped through the lane's forward cursor e).
template <int PREC, int MODEL>
__device__ __forceinline__ void leaf_pairs(const EvalArgs &a, const Target &t, const NodeRec &nr, bool walk,
                                           int64_t &e, int64_t e1, Seg64 *seg64_tile, Seg32 *seg32_tile,
                                           Acc<PREC> &acc, int &flag, long long &near_pairs,
                                           long long &fp64_pairs) {
    const int lane = threadIdx.x & 31, lo = nr.lo, hi = nr.hi;
    if (walk) while (e < e1 && a.ex_pos[e] < lo) ++e;
    float t0 = 0.f, t1 = 0.f, t2 = 0.f;
    // When every walking lane is farther from the leaf's bounding sphere than sqrt(near2) of its largest core radius
    // (with a 1% margin for rounding), no pair of the leaf can need FP64 for its core: the pairs skip that test.
    // Without a core (MODEL 0) the test is "within L/4 of the segment", and a lane 1.5 bounding radii from the centre
    // is at least half a radius, so L/4 (L <= 2 radii), from every segment.  When moreover every walking lane lies at
    // least 1.5 bounding radii from the leaf's centre (within FP32's range), the packed pairs take the clear-leaf form
    // (pair32x2_clear).
    bool clear = true, wide = true;
    float3 rel = make_float3(0.f, 0.f, 0.f);
    if (PREC != 0 && walk) {
        const double rx = t.x0 - nr.cx, ry = t.x1 - nr.cy, rz = t.x2 - nr.cz;
        const double r2 = rx * rx + ry * ry + rz * rz;
        clear = MODEL != 0 ? sqrt(r2) - nr.bound > 1.01 * sqrt((double)a.near2) * nr.clear_core
                           : r2 >= 2.25 * nr.bound * nr.bound;
        wide = clear && r2 >= 2.25 * nr.bound * nr.bound && r2 > 1e-16 && r2 < 1e18 && nr.bound < 1e9;
        rel = make_float3((float)rx, (float)ry, (float)rz);
    }
    const bool all_clear = __all_sync(0xffffffffu, clear);
    if constexpr (PREC != 0 && MODEL <= 2) {
        // the warp's tile space is sized for 32 Seg64 (3 KB): 16 Seg32x2 (2 KB) or 32 Seg32c2 (3 KB) fit
        const bool all_wide = __all_sync(0xffffffffu, wide);
        leaf_pairs_packed<PREC, MODEL>(a, t, lo, hi, walk, all_clear, all_wide, rel, e, e1,
                                       reinterpret_cast<float4 *>(seg64_tile), acc, flag, near_pairs, fp64_pairs);
    } else {
        for (int base = lo; base < hi; base += 32) {
            const int cnt = min(32, hi - base);
            __syncwarp();
            if (lane < cnt) {
                if (PREC == 0) seg64_tile[lane] = a.tv.seg64[base + lane];
                else seg32_tile[lane] = a.tv.seg32[base + lane];
            }
            __syncwarp();
            if (!walk) continue;
            unsigned excl = 0;
            while (e < e1 && a.ex_pos[e] < base + cnt) excl |= 1u << (a.ex_pos[e++] - base);
            near_pairs += cnt - __popc(excl);
            if (PREC == 0) {
                double u0 = 0.0, u1 = 0.0, u2 = 0.0;
                for (int j = 0; j < cnt; ++j) {
                    if ((excl >> j) & 1u) continue;
                    int fl = pair64_at(t.x0, t.x1, t.x2, seg64_tile[j], a.model, a.raise_singular, u0, u1, u2);
                    if (fl != BS_FLAG_OK && flag == BS_FLAG_OK) flag = fl;
                }
                acc.add64(u0, u1, u2);
                continue;
            }
            unsigned need = 0;
            if (excl == 0 && all_clear && cnt == 32) {  // the common case: a full tile, every pair counts, none near a core
    #pragma unroll 8
                for (int j = 0; j < 32; ++j) {
                    const Seg32 &r = seg32_tile[j];
                    const float q0 = (t.xh0 - r.hi.x) + (t.xl0 - r.lo.x);
                    const float q1 = (t.xh1 - r.hi.y) + (t.xl1 - r.lo.y);
                    const float q2 = (t.xh2 - r.hi.z) + (t.xl2 - r.lo.z);
                    if (pair32<MODEL, false>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1u << j;
                }
            } else if (excl == 0 && all_clear) {
    #pragma unroll 4
                for (int j = 0; j < cnt; ++j) {
                    const Seg32 &r = seg32_tile[j];
                    const float q0 = (t.xh0 - r.hi.x) + (t.xl0 - r.lo.x);
                    const float q1 = (t.xh1 - r.hi.y) + (t.xl1 - r.lo.y);
                    const float q2 = (t.xh2 - r.hi.z) + (t.xl2 - r.lo.z);
                    if (pair32<MODEL, false>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1u << j;
                }
            } else if (excl == 0) {  // every pair counts
    #pragma unroll 4
                for (int j = 0; j < cnt; ++j) {
                    const Seg32 &r = seg32_tile[j];
                    const float q0 = (t.xh0 - r.hi.x) + (t.xl0 - r.lo.x);
                    const float q1 = (t.xh1 - r.hi.y) + (t.xl1 - r.lo.y);
                    const float q2 = (t.xh2 - r.hi.z) + (t.xl2 - r.lo.z);
                    if (pair32<MODEL>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1u << j;
                }
            } else {
                for (int j = 0; j < cnt; ++j) {
                    if ((excl >> j) & 1u) continue;
                    const Seg32 &r = seg32_tile[j];
                    const float q0 = (t.xh0 - r.hi.x) + (t.xl0 - r.lo.x);
                    const float q1 = (t.xh1 - r.hi.y) + (t.xl1 - r.lo.y);
                    const float q2 = (t.xh2 - r.hi.z) + (t.xl2 - r.lo.z);
                    if (pair32<MODEL>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1u << j;
                }
            }
            // pairs near a segment, its axis or out of FP32 range: FP64 from FP64 inputs
            fp64_pairs += __popc(need);
            while (need) {
                const int j = __ffs(need) - 1;
                need &= need - 1;
                double v0 = 0.0, v1 = 0.0, v2 = 0.0;
                int fl = pair64_at(t.x0, t.x1, t.x2, a.tv.seg64[base + j], MODEL, a.raise_singular, v0, v1, v2);
                if (fl != BS_FLAG_OK) {
                    if (flag == BS_FLAG_OK) flag = fl;
                } else {
                    acc.add64(v0, v1, v2);
                }
            }
        }
        if (walk && PREC != 0) acc.add32(t0, t1, t2);
    }
}

// The walk's own evaluations of what does not fit in its list (rare): out of line, with their inputs by value, so
// that the traversal loop keeps the code and registers of the walk alone.
struct LeafSum {
    double u0, u1, u2;
    long long near_pairs, fp64_pairs;
    int flag;
};

template <int PREC, int MODEL>
__device__ __noinline__ LeafSum walk_leaf(const EvalArgs a, const Target t, const NodeRec nr, bool walk, int64_t e,
                                         int64_t e1, Seg64 *seg64_tile, Seg32 *seg32_tile) {
    Acc<PREC> acc;
    LeafSum r{};
    r.flag = BS_FLAG_OK;
    leaf_pairs<PREC, MODEL>(a, t, nr, walk, e, e1, seg64_tile, seg32_tile, acc, r.flag, r.near_pairs, r.fp64_pairs);
    r.u0 = acc.x();
    r.u1 = acc.y();
    r.u2 = acc.z();
    return r;
}

template <int PREC>
__device__ __noinline__ double3 walk_far(const EvalArgs a, const Target t, int node) {
    Acc<PREC> acc;
    far_node<PREC>(a, t, node, acc);
    return make_double3(acc.x(), acc.y(), acc.z());
}

// Phase 1: the traversal.  Each warp walks the tree once for its 32 targets and writes an interaction list: far
// nodes and near leaves with the mask of lanes concerned, in depth-first order, and the cost before each entry.  What
// does not fit in the list is evaluated here.
template <int PREC, int MODEL, int POP>
__global__ void __launch_bounds__(128) tree_walk_kernel(EvalArgs a) {
    extern __shared__ __align__(16) unsigned char eval_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    int2 *stack = reinterpret_cast<int2 *>(eval_smem) + warp * STACK_DEPTH;
    unsigned char *tiles = eval_smem + (size_t)warps * STACK_DEPTH * sizeof(int2);
    Seg64 *seg64_tile = reinterpret_cast<Seg64 *>(tiles) + warp * 32;
    Seg32 *seg32_tile = reinterpret_cast<Seg32 *>(tiles) + warp * 32;
    const int64_t gw = (int64_t)blockIdx.x * warps + warp;  // warp of targets
    if (gw * 32 >= a.n) return;  // warp-uniform: warps past the last target own no list
    Target t;
    t.load(a, gw * 32 + lane);
    int64_t e = 0, e1 = 0;
    if (t.valid && a.ex_ptr) { e = a.ex_ptr[t.p]; e1 = a.ex_ptr[t.p + 1]; }
    const bool exact = a.exact && t.valid && a.exact[t.p];
    Acc<PREC> acc;
    int flag = BS_FLAG_OK;
    long long far = 0, far_total = 0, near_pairs = 0, fp64_pairs = 0, visits = 0, pair_slots = 0;
    int *my_chunks = a.unit_chunks + gw * LIST_CHUNKS;
    int len = 0, running = 0, chunk = -1;
    bool full = false;  // the unit's chunk table or the pool ran out: the rest is evaluated here
    // Room for one more entry (warp-uniform): a new chunk every LIST_CHUNK entries.
    auto room = [&]() -> bool {
        if (full) return false;
        if ((len & (LIST_CHUNK - 1)) == 0) {
            int c = -1;
            if (len / LIST_CHUNK < LIST_CHUNKS && lane == 0) {
                const unsigned long long got = atomicAdd(a.pool_cursor, 1ull);
                if (got < a.pool_chunks) {
                    c = (int)got;
                    my_chunks[len / LIST_CHUNK] = c;
                }
            }
            c = __shfl_sync(0xffffffffu, c, 0);
            if (c < 0) {
                full = true;
                return false;
            }
            chunk = c;
        }
        return true;
    };
    // Roots: node 0, or in a forest the root of each lane's wake; one stack entry per distinct root.
    const int root = a.root_of ? (t.valid ? a.root_of[gw * 32 + lane] : -1) : 0;
    const bool live = t.valid && root >= 0;
    const unsigned peers = __match_any_sync(0xffffffffu, live ? root : -1);
    const bool leader = live && (__ffs(peers) - 1) == lane;
    const unsigned leaders = __ballot_sync(0xffffffffu, leader);
    if (leader) stack[__popc(leaders & ((1u << lane) - 1u))] = make_int2(root, (int)peers);
    int top = __popc(leaders);
    __syncwarp();
    // One node for the lanes of `mask`: per-lane acceptance, then a far entry, a near-leaf entry or two pushed
    // children.  Returns false when the stack would overflow.
    // This lane's decision at a node of `mask`: accept it as far (true) or open it.  Kept apart from the visit so that
    // a step's two decisions (independent FP64 chains) overlap.
    auto decide = [&](const unsigned mask, const NodeRec &nr) -> bool {
        const bool mine = (mask >> lane) & 1u;
        bool accept = false;
        if (mine) {
            ++visits;
            const double rx = t.x0 - nr.cx, ry = t.x1 - nr.cy, rz = t.x2 - nr.cz;
            // |R|^2 as the reference forms it, without contraction
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
            // The reference's test, bound < theta |R| and |R| - bound >= clearance * core, in squared form (no square
            // root); only within 1e-12 (relative) of either boundary are the two forms allowed to round differently,
            // and there the reference's own expression decides, so the decisions equal the CPU's.
            const double cc = __dmul_rn(a.clearance, nr.clear_core);
            const double b2 = nr.bound * nr.bound, lhs1 = a.theta2 * r2;
            const double reach = nr.bound + cc, rhs2 = reach * reach;
            const double q1 = lhs1 - b2, q2 = r2 - rhs2;
            if (fabs(q1) > 1e-12 * fmax(lhs1, b2) && fabs(q2) > 1e-12 * fmax(r2, rhs2)) {
                accept = q1 > 0.0 && q2 > 0.0;
            } else {
                const double dist = sqrt(r2);
                accept = nr.bound < __dmul_rn(a.theta, dist) && __dsub_rn(dist, nr.bound) >= cc;
            }
            if (accept && e < e1) {  // an excluded segment inside the node keeps it open
                int64_t q = e;
                while (q < e1 && a.ex_pos[q] < nr.lo) ++q;
                if (q < e1 && a.ex_pos[q] < nr.hi) accept = false;
            }
            if (exact) accept = false;  // a target summed exactly opens every node
        }
        return accept;
    };
    auto visit = [&](const int node, const unsigned mask, const NodeRec &nr, bool accept) -> bool {
        const bool mine = (mask >> lane) & 1u;
        unsigned farm = __ballot_sync(0xffffffffu, mine && accept);
        unsigned openm = mask & ~farm;
        const unsigned openers = __ballot_sync(0xffffffffu, mine && !accept && !exact);
        // Fill: a leaf that some lane opens is evaluated by the warp anyway, and the lanes that accepted it as far
        // would idle beside its pairs: they sum it exactly instead of through its expansion (same time, no far
        // evaluation, more exact).  Morton trees in single precision only: median trees and FP64 keep each
        // target's own decisions, the reference's.  Exact targets (which open every leaf) do not count, so that
        // they leave the others' results as they are.
        if (a.fill && nr.left < 0 && openers && farm) {
            openm = mask;
            farm = 0u;
            accept = false;
        }
        if (farm) {
            if (mine && accept) ++far;
            far_total += __popc(farm);
            if (room()) {
                if (lane == 0) {
                    const int64_t k = (int64_t)chunk * LIST_CHUNK + (len & (LIST_CHUNK - 1));
                    a.list[k] = make_int2(node | FAR_BIT, (int)farm);
                    a.list_cost[k] = running;
                }
                ++len;
                running += FAR_COST;
            } else if (mine && accept) {
                // far records still being computed: evaluated again by the host once they are complete
                if (a.deferred) {
                    atomicOr(a.overflow + 1, 1);
                } else {
                    const double3 v = walk_far<PREC>(a, t, node);
                    acc.add64(v.x, v.y, v.z);
                }
            }
        }
        if (openm) {
            if (nr.left < 0) {
                pair_slots += (long long)(nr.hi - nr.lo);
                if (room()) {
                    if (lane == 0) {
                        const int64_t k = (int64_t)chunk * LIST_CHUNK + (len & (LIST_CHUNK - 1));
                        a.list[k] = make_int2(node, (int)openm);
                        a.list_cost[k] = running;
                    }
                    ++len;
                    running += (nr.hi - nr.lo) + 2;
                } else if (a.deferred) {  // segment records still being written: evaluated again by the host
                    if (mine && !accept) atomicOr(a.overflow + 1, 1);
                } else {
                    const LeafSum r = walk_leaf<PREC, MODEL>(a, t, nr, mine && !accept, e, e1, seg64_tile, seg32_tile);
                    acc.add64(r.u0, r.u1, r.u2);
                    near_pairs += r.near_pairs;
                    fp64_pairs += r.fp64_pairs;
                    if (flag == BS_FLAG_OK) flag = r.flag;
                }
            } else {
                if (top + 2 > a.stack_limit) {
                    if (lane == 0) atomicExch(a.overflow, 1);
                    return false;
                }
                if (lane == 0) {
                    stack[top] = make_int2(nr.right, (int)openm);
                    stack[top + 1] = make_int2(nr.left, (int)openm);
                }
                top += 2;
            }
        }
        return true;
    };
    // POP entries per step: their node records load together, so that with POP = 2 two independent loads are in
    // flight per step of the (latency-bound) walk.  The set of visited nodes does not depend on the order.
    while (top > 0) {
        if (POP == 2 && top >= 2) {
            const int2 x = stack[top - 1], y = stack[top - 2];
            top -= 2;
            const NodeRec nx = a.tv.nodes[x.x], ny = a.tv.nodes[y.x];
            __syncwarp();
            const bool ax = decide((unsigned)x.y, nx), ay = decide((unsigned)y.y, ny);
            if (!visit(x.x, (unsigned)x.y, nx, ax)) break;
            if (!visit(y.x, (unsigned)y.y, ny, ay)) break;
        } else {
            const int2 x = stack[--top];
            const NodeRec nx = a.tv.nodes[x.x];
            __syncwarp();
            if (!visit(x.x, (unsigned)x.y, nx, decide((unsigned)x.y, nx))) break;
        }
        __syncwarp();
    }
    if (lane == 0) {
        a.list_len[gw] = len;
        a.list_total[gw] = running;
    }
    if (t.valid) {
        a.walk_u[3 * t.p] = acc.x();
        a.walk_u[3 * t.p + 1] = acc.y();
        a.walk_u[3 * t.p + 2] = acc.z();
        a.walk_flag[t.p] = (int8_t)flag;
        if (a.far_counts) a.far_counts[t.p] = far;
    }
    for (int o = 16; o > 0; o >>= 1) {
        near_pairs += __shfl_xor_sync(0xffffffffu, near_pairs, o);
        fp64_pairs += __shfl_xor_sync(0xffffffffu, fp64_pairs, o);
        visits += __shfl_xor_sync(0xffffffffu, visits, o);
    }
    if (lane == 0) {
        atomicAdd(&a.counters[0], (unsigned long long)far_total);
        atomicAdd(&a.counters[1], (unsigned long long)near_pairs);
        atomicAdd(&a.counters[2], (unsigned long long)fp64_pairs);
        atomicAdd(&a.counters[3], (unsigned long long)visits);
        atomicAdd(&a.counters[4], (unsigned long long)(32 * pair_slots));
    }
}

// Phase 2: two persistent kernels over the same work items, (warp of targets, chunk) pairs, chunk c holding the c-th
// slice (by cost) of that warp's list; each warp of a kernel takes items from its own device counter until none is
// left.  PART 0 evaluates the item's near leaves, PART 1 its far nodes (apart, each kernel holds only its own code and
// registers).  Partial sums per (chunk, target) are combined in chunk order by the reduce kernel.
template <int PREC, int MODEL, int PART>
__device__ __forceinline__ void list_item(const EvalArgs &a, int64_t gw, int c, int chunks, int64_t item,
                                          Seg64 *seg64_tile, Seg32 *seg32_tile, float4 *stage, int2 *ebuf,
                                          long long &near_pairs, long long &fp64_pairs) {
    const int lane = threadIdx.x & 31;
    // chunk c is the c-th slice of this warp's list by cost: entries [item_first[item], item_first[item + 1]), the
    // last slice ending at the list's end
    const int len = a.list_len[gw];
    const int *chunks_of = a.unit_chunks + gw * LIST_CHUNKS;
    auto at = [&](int k) -> int64_t {  // pool index of the list's k-th entry
        return (int64_t)chunks_of[k / LIST_CHUNK] * LIST_CHUNK + (k & (LIST_CHUNK - 1));
    };
    const int first = a.item_first[item], last = c + 1 < chunks ? a.item_first[item + 1] : len;
    // entry k of the list (warp-uniform k): read ahead ENTRY_BUF entries at a time into the warp's buffer, so that
    // the entries cost one coalesced load a block instead of two dependent loads each
    int buf_lo = first, buf_hi = first;
    auto entry_at = [&](int k) -> int2 {
        if (k >= buf_hi) {
            __syncwarp();
            buf_lo = k;
            buf_hi = min(last, k + ENTRY_BUF);
            for (int i = lane; i < buf_hi - buf_lo; i += 32) ebuf[i] = a.list[at(buf_lo + i)];
            __syncwarp();
        }
        return ebuf[k - buf_lo];
    };
    Target t;
    t.load(a, gw * 32 + lane);
    int64_t e = 0, e1 = 0;
    if (t.valid && a.ex_ptr) { e = a.ex_ptr[t.p]; e1 = a.ex_ptr[t.p + 1]; }
    Acc<PREC> acc;
    int flag = BS_FLAG_OK;
    if constexpr (PART == 0) {
        for (int k = first; k < last; ++k) {
            const int2 entry = entry_at(k);
            if (entry.x & FAR_BIT) continue;
            const bool mine = ((unsigned)entry.y >> lane) & 1u;
            const NodeRec nr = a.tv.nodes[entry.x];
            int64_t ec = e;  // list entries are not in position order: each leaf scans the exclusions from the start
            leaf_pairs<PREC, MODEL>(a, t, nr, mine, ec, e1, seg64_tile, seg32_tile, acc, flag, near_pairs,
                                    fp64_pairs);
        }
    } else {
        // Far entries are packed first-fit into FAR_GROUPS open groups of disjoint lane masks and at most FAR_STAGE
        // entries, each lane of a group at its own node.  A group closes when an entry fits none (the fullest one
        // closes) or when the list ends; closed groups queue (up to FAR_QUEUE) and are then evaluated in order, every
        // lane at its node at once.  A far entry holds about a third of the warp's lanes, so a group fills the warp
        // from a few entries.  In single precision the records of the next group's nodes are copied into the warp's
        // other staging buffer (cp.async) while the current group is evaluated from its copy.
        int *q_node = reinterpret_cast<int *>(stage + 2 * FAR_STAGE * FAR_REC4);  // [FAR_QUEUE][FAR_STAGE]
        unsigned *q_mask = reinterpret_cast<unsigned *>(q_node + FAR_QUEUE * FAR_STAGE);
        int *q_cnt = reinterpret_cast<int *>(q_mask + FAR_QUEUE * FAR_STAGE);
        unsigned group[FAR_GROUPS], gmask[FAR_GROUPS][FAR_STAGE];
        int gnode[FAR_GROUPS][FAR_STAGE], gcount[FAR_GROUPS];
#pragma unroll
        for (int q = 0; q < FAR_GROUPS; ++q) {
            group[q] = 0u;
            gcount[q] = 0;
#pragma unroll
            for (int r = 0; r < FAR_STAGE; ++r) {
                gnode[q][r] = -1;
                gmask[q][r] = 0u;
            }
        }
        const int n4 = far_rec4_count(a.order);
        int nq = 0;  // closed groups queued
        auto close = [&](int go) {
#pragma unroll
            for (int q = 0; q < FAR_GROUPS; ++q)
                if (q == go) {
                    if (lane < FAR_STAGE) {
                        int nd = -1;
                        unsigned mk = 0u;
#pragma unroll
                        for (int r = 0; r < FAR_STAGE; ++r)
                            if (r == lane) {
                                nd = gnode[q][r];
                                mk = gmask[q][r];
                            }
                        q_node[nq * FAR_STAGE + lane] = nd;
                        q_mask[nq * FAR_STAGE + lane] = mk;
                    }
                    if (lane == 0) q_cnt[nq] = gcount[q];
                    group[q] = 0u;
                    gcount[q] = 0;
                }
            ++nq;
        };
        // the records of queued group g into staging buffer b: every lane copies its share, then commits
        auto issue = [&](int g, int b) {
            if (PREC != 0 && g < nq) {
                float4 *buf = stage + b * FAR_STAGE * FAR_REC4;
                const int cnt = q_cnt[g];
                for (int r = 0; r < cnt; ++r) {
                    const int nd = q_node[g * FAR_STAGE + r];
                    for (int i = lane; i < n4; i += 32) cp_async16(buf + r * FAR_REC4 + i, far_rec4(a.tv, nd, i));
                    if (lane < 2)  // the centre: cx, cy, cz of the node's traversal record
                        cp_async16(buf + r * FAR_REC4 + FAR_REC4 - 2 + lane,
                                   reinterpret_cast<const float4 *>(a.tv.nodes + nd) + lane);
                }
            }
            cp_async_commit();
        };
        int k = first;
        for (;;) {
            while (k < last && nq < FAR_QUEUE - FAR_GROUPS) {  // room left to close every open group at the end
                const int2 entry = entry_at(k);
                if (!(entry.x & FAR_BIT)) {
                    ++k;
                    continue;
                }
                const unsigned m = (unsigned)entry.y;
                int fit = -1;
#pragma unroll
                for (int q = 0; q < FAR_GROUPS; ++q)
                    if (fit < 0 && !(group[q] & m) && gcount[q] < FAR_STAGE) fit = q;
                if (fit < 0) {
                    int most = -1, go = 0;
#pragma unroll
                    for (int q = 0; q < FAR_GROUPS; ++q)
                        if (__popc(group[q]) > most) {
                            most = __popc(group[q]);
                            go = q;
                        }
                    close(go);
                    continue;  // the entry is placed again, into the emptied group at least
                }
                const int node = entry.x & ~FAR_BIT;
#pragma unroll
                for (int q = 0; q < FAR_GROUPS; ++q)
                    if (q == fit) {
                        group[q] |= m;
#pragma unroll
                        for (int r = 0; r < FAR_STAGE; ++r)
                            if (r == gcount[q]) {
                                gnode[q][r] = node;
                                gmask[q][r] = m;
                            }
                        ++gcount[q];
                    }
                ++k;
            }
            const bool done = k >= last;
            if (done) {
#pragma unroll
                for (int q = 0; q < FAR_GROUPS; ++q)
                    if (group[q]) close(q);
            }
            __syncwarp();  // the queue is written
            issue(0, 0);
            for (int g = 0; g < nq; ++g) {
                issue(g + 1, (g + 1) & 1);
                cp_async_wait<1>();
                __syncwarp();  // group g's records are in its buffer
                int slot = -1;
                for (int r = 0; r < q_cnt[g]; ++r)
                    if ((q_mask[g * FAR_STAGE + r] >> lane) & 1u) slot = r;
                if (slot >= 0) {
                    const int node = q_node[g * FAR_STAGE + slot];
                    if constexpr (PREC != 0)
                        far_node_staged<PREC>(a, t, node, stage + (g & 1) * FAR_STAGE * FAR_REC4 + slot * FAR_REC4,
                                              acc);
                    else
                        far_node<PREC>(a, t, node, acc);
                }
                __syncwarp();  // buffer g & 1 is free for group g + 2
            }
            cp_async_wait<0>();
            nq = 0;
            if (done) break;
        }
    }
    if (t.valid) {
        const int64_t o = item * 32 + lane;
        if (PART == 0) {
            a.partial[3 * o] = acc.x();
            a.partial[3 * o + 1] = acc.y();
            a.partial[3 * o + 2] = acc.z();
            a.pflag[o] = (int8_t)flag;
        } else {
            a.partial[3 * o] += acc.x();
            a.partial[3 * o + 1] += acc.y();
            a.partial[3 * o + 2] += acc.z();
        }
    }
}

// The near-leaf kernel at four blocks a SM (128 registers a thread: more warps to hide the packed pairs' dependent
// chains, measured faster than three blocks at 160 registers); the far-node kernel at three (57.9 KB of shared memory
// a block, up to 168 registers).
// PART 0: near leaves (counter a.queue[0]); PART 1: far nodes (counter a.queue[2]; no tiles).
template <int PREC, int MODEL, int PART>
__global__ void __launch_bounds__(LIST_WARPS * 32, PART == 0 ? LIST_NEAR_BLOCKS : LIST_FAR_BLOCKS)
    tree_list_kernel(EvalArgs a, int64_t target_warps) {
    // near kernel: static tiles and entry buffers; far kernel: FAR_WARP_SMEM of dynamic shared memory a warp
    __shared__ __align__(16) unsigned char tile_mem[PART == 0 ? LIST_WARPS * 32 * sizeof(Seg64) : 16];
    __shared__ int2 entry_mem[PART == 0 ? LIST_WARPS * ENTRY_BUF : 1];
    extern __shared__ __align__(16) unsigned char list_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Seg64 *seg64_tile = reinterpret_cast<Seg64 *>(tile_mem) + warp * 32;
    Seg32 *seg32_tile = reinterpret_cast<Seg32 *>(tile_mem) + warp * 32;
    float4 *stage = reinterpret_cast<float4 *>(list_smem + warp * FAR_WARP_SMEM);  // far kernel only
    int2 *ebuf = PART == 0 ? entry_mem + warp * ENTRY_BUF
                           : reinterpret_cast<int2 *>(list_smem + (warp + 1) * FAR_WARP_SMEM) - ENTRY_BUF;
    const unsigned long long items = (unsigned long long)a.item_off[target_warps];
    long long near_pairs = 0, fp64_pairs = 0;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(a.queue + (PART == 0 ? 0 : 2), 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= items) break;
        const int64_t lo = a.item_warp[item];  // the warp of targets whose list this item slices
        const int first = a.item_off[lo];
        list_item<PREC, MODEL, PART>(a, lo, (int)(item - first), a.item_off[lo + 1] - first, (int64_t)item,
                                     seg64_tile, seg32_tile, stage, ebuf, near_pairs, fp64_pairs);
    }
    if constexpr (PART == 0) {
        for (int o = 16; o > 0; o >>= 1) {
            near_pairs += __shfl_xor_sync(0xffffffffu, near_pairs, o);
            fp64_pairs += __shfl_xor_sync(0xffffffffu, fp64_pairs, o);
        }
        if (lane == 0) {
            atomicAdd(&a.counters[1], (unsigned long long)near_pairs);
            atomicAdd(&a.counters[2], (unsigned long long)fp64_pairs);
        }
    }
}

// Work items of the list kernel: warp gw gets max(1, ceil(cost / unit)) items (at most 64), unit = total cost / want,
// so every item costs about the same whatever its warp; item_off is their exclusive scan (one block).  The sum of the
// items stays below want + target_warps, the capacity the caller allocates.
__global__ void __launch_bounds__(1024) item_plan_kernel(int64_t target_warps, const int *list_total, int want,
                                                         int *item_off, int *item_warp) {
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const int64_t per = (target_warps + 1023) / 1024, a0 = min(target_warps, t * per),
                  a1 = min(target_warps, a0 + per);
    long long cost = 0;
    for (int64_t w = a0; w < a1; ++w) cost += list_total[w];
    part[t] = cost;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (t < o) part[t] += part[t + o];
        __syncthreads();
    }
    const long long total = part[0];
    __syncthreads();
    const long long unit = max(1ll, (total + want - 1) / want);
    long long items = 0;
    for (int64_t w = a0; w < a1; ++w) items += min(64ll, max(1ll, ((long long)list_total[w] + unit - 1) / unit));
    // exclusive scan of the threads' item counts: within each warp by shuffles, then over the 32 warp totals
    const int lane = t & 31, wid = t >> 5;
    long long inc = items;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) part[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        long long w = part[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += v;
        }
        part[lane] = w;  // inclusive over the warps
        if (lane == 31) item_off[target_warps] = (int)w;
    }
    __syncthreads();
    long long run = inc - items + (wid ? part[wid - 1] : 0);
    for (int64_t w = a0; w < a1; ++w) {
        item_off[w] = (int)run;
        const long long k = min(64ll, max(1ll, ((long long)list_total[w] + unit - 1) / unit));
        for (long long q = 0; q < k; ++q) item_warp[run + q] = (int)w;
        run += k;
    }
}

// The first list entry of every work item, one warp per warp of targets, its lanes reading the list's cost starts in
// order: item c of warp gw (of `chunks`) begins at the first entry whose cost start reaches floor(total c / chunks).
// The cost starts rise strictly (every entry costs at least 1), so entry k begins the items whose threshold lies in
// (cost[k - 1], cost[k]], and the items whose threshold lies past the last start are empty (they begin at len).
__global__ void item_bounds_kernel(EvalArgs a, int64_t target_warps) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw >= target_warps) return;
    const int base = a.item_off[gw], chunks = a.item_off[gw + 1] - base, len = a.list_len[gw];
    const long long total = a.list_total[gw];
    const int *chunks_of = a.unit_chunks + gw * LIST_CHUNKS;
    if (len == 0 || total <= 0) {
        for (int c = lane; c < chunks; c += 32) a.item_first[base + c] = 0;
        return;
    }
    // the chunk table (at most 32 chunks) one entry a lane; entry k's chunk is then a shuffle away
    const int my_chunk = lane < LIST_CHUNKS && lane * LIST_CHUNK < len ? chunks_of[lane] : 0;
    long long carry = -1;  // cost start of the entry before this round's first
    for (int k0 = 0; k0 < len; k0 += 32) {
        const int k = k0 + lane;
        const int ch = __shfl_sync(0xffffffffu, my_chunk, (k < len ? k : len - 1) / LIST_CHUNK);
        const long long ck = k < len ? a.list_cost[(int64_t)ch * LIST_CHUNK + (k & (LIST_CHUNK - 1))] : 0;
        const long long up = __shfl_up_sync(0xffffffffu, ck, 1);
        const long long cp = lane == 0 ? carry : up;
        carry = __shfl_sync(0xffffffffu, ck, 31);
        if (k >= len) continue;
        // floor(total c / chunks) > cp  <=>  c >= ceil((cp + 1) chunks / total);
        // floor(total c / chunks) <= ck <=>  c <= ceil((ck + 1) chunks / total) - 1
        const long long c0 = ((cp + 1) * chunks + total - 1) / total;
        const long long c1 = min((long long)chunks - 1, ((ck + 1) * chunks + total - 1) / total - 1);
        for (long long c = c0; c <= c1; ++c) a.item_first[base + c] = k;
        if (k == len - 1)
            for (long long c = max(c0, c1 + 1); c < chunks; ++c) a.item_first[base + c] = len;
    }
}

// A target's items in order, then what the walk evaluated itself (later in depth-first order); first flag wins.
template <int PREC>
__global__ void tree_reduce_kernel(EvalArgs a, double *out, int8_t *flags) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // sorted target
    if (i >= a.n) return;
    const int64_t p = a.perm[i], gw = i >> 5;
    const int lane = (int)(i & 31);
    Acc<PREC> acc;
    int flag = BS_FLAG_OK;
    for (int item = a.item_off[gw]; item < a.item_off[gw + 1]; ++item) {
        const int64_t o = (int64_t)item * 32 + lane;
        acc.add64(a.partial[3 * o], a.partial[3 * o + 1], a.partial[3 * o + 2]);
        if (flag == BS_FLAG_OK) flag = a.pflag[o];
    }
    acc.add64(a.walk_u[3 * p], a.walk_u[3 * p + 1], a.walk_u[3 * p + 2]);
    if (flag == BS_FLAG_OK) flag = a.walk_flag[p];
    const double u0 = acc.x(), u1 = acc.y(), u2 = acc.z();
    if (!(isfinite(u0) && isfinite(u1) && isfinite(u2)) && flag == BS_FLAG_OK) flag = BS_FLAG_NONFINITE;
    out[3 * p] = u0;
    out[3 * p + 1] = u1;
    out[3 * p + 2] = u2;
    flags[p] = (int8_t)flag;
}

// Morton keys of the targets inside their own box (for locality only; any order gives the same per-target result).
__global__ void target_box_kernel(int64_t n, const double *points, unsigned long long *box) {
    __shared__ unsigned long long sb[6];
    auto ob = [](double x) -> unsigned long long {
        unsigned long long b = (unsigned long long)__double_as_longlong(x + 0.0);
        return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
    };
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? ob(INFINITY) : ob(-INFINITY);
    __syncthreads();
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            atomicMin(&sb[a], ob(points[3 * p + a]));
            atomicMax(&sb[3 + a], ob(points[3 * p + a]));
        }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&box[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&box[threadIdx.x], sb[threadIdx.x]);
}

__global__ void target_box_init_kernel(unsigned long long *box) {
    auto ob = [](double x) -> unsigned long long {
        unsigned long long b = (unsigned long long)__double_as_longlong(x + 0.0);
        return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
    };
    if (threadIdx.x < 3) box[threadIdx.x] = ob(INFINITY);
    else if (threadIdx.x < 6) box[threadIdx.x] = ob(-INFINITY);
}

__device__ __forceinline__ double unordered(unsigned long long k) {
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__device__ __forceinline__ uint64_t spread3_t(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void target_keys_kernel(int64_t n, const double *points, const unsigned long long *box,
                                   const uint8_t *exact, uint64_t *keys, int32_t *vals) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double ext = 0.0, lo[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = unordered(box[a]);
        ext = fmax(ext, unordered(box[3 + a]) - lo[a]);
    }
    double inv = ext > 0.0 ? 2097152.0 / ext : 0.0;
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) q[a] = min(2097151u, (uint32_t)((points[3 * p + a] - lo[a]) * inv));
    keys[p] = (spread3_t(q[0]) << 2) | (spread3_t(q[1]) << 1) | spread3_t(q[2]) |
              ((exact && exact[p]) ? 1ull << 63 : 0ull);  // exact targets after the others
    vals[p] = (int32_t)p;
}

// Excluded segment ids -> tree positions, sorted per target (insertion sort; a target excludes few segments).
__global__ void exclusion_positions_kernel(int64_t n, const int64_t *ex_ptr, const int64_t *ex_seg,
                                           const int32_t *inverse, int32_t *ex_pos) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int64_t a = ex_ptr[p], b = ex_ptr[p + 1];
    for (int64_t k = a; k < b; ++k) {
        int32_t v = inverse[ex_seg[k]];
        int64_t j = k - 1;
        while (j >= a && ex_pos[j] > v) { ex_pos[j + 1] = ex_pos[j]; --j; }
        ex_pos[j + 1] = v;
    }
}

static inline unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// Events that eval_run records around the walk and list kernels (null while a graph is being captured), and the event
// the list kernel waits for when the far records were still in computation (null: nothing to wait for).
static thread_local cudaEvent_t *t_marks = nullptr;
static thread_local cudaEvent_t t_far_ready = nullptr;
static thread_local cudaEvent_t t_records_ready = nullptr;

template <int PREC, int MODEL>
static void launch_pair(unsigned walk_grid, int block, size_t smem, uint2 list_grid, int64_t target_warps,
                        unsigned reduce_grid, cudaStream_t s, const EvalArgs &args, double *out, int8_t *flags) {
    if (t_marks) cudaEventRecord(t_marks[0], s);
    tree_walk_kernel<PREC, MODEL, 2><<<walk_grid, block, smem, s>>>(args);  // two stack entries a step
    item_plan_kernel<<<1, 1024, 0, s>>>(target_warps, args.list_total, args.item_want, args.item_off,
                                        args.item_warp);
    item_bounds_kernel<<<(unsigned)((target_warps * 32 + 255) / 256), 256, 0, s>>>(args, target_warps);
    // the near-leaf kernel reads the segment and clear-leaf records, the far-node kernel the far records: each waits
    // for its own (with a side stream the leaf pass ends before the climb and the far records)
    if (t_records_ready) cudaStreamWaitEvent(s, t_records_ready, 0);
    else if (t_far_ready) cudaStreamWaitEvent(s, t_far_ready, 0);
    if (t_marks) cudaEventRecord(t_marks[1], s);
    tree_list_kernel<PREC, MODEL, 0><<<list_grid.x, LIST_WARPS * 32, 0, s>>>(args, target_warps);
    if (t_marks) cudaEventRecord(t_marks[2], s);
    if (t_records_ready && t_far_ready) cudaStreamWaitEvent(s, t_far_ready, 0);
    static const bool far_smem = cudaFuncSetAttribute(tree_list_kernel<PREC, MODEL, 1>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)(LIST_WARPS * FAR_WARP_SMEM)) == cudaSuccess;
    (void)far_smem;  // a refusal shows as the launch's error
    tree_list_kernel<PREC, MODEL, 1><<<list_grid.y, LIST_WARPS * 32, LIST_WARPS * FAR_WARP_SMEM, s>>>(args,
                                                                                                     target_warps);
    if (t_marks) cudaEventRecord(t_marks[3], s);
    tree_reduce_kernel<PREC><<<reduce_grid, 256, 0, s>>>(args, out, flags);
}

template <int PREC>
static void launch_model(int model, unsigned walk_grid, int block, size_t smem, uint2 list_grid, int64_t tw,
                         unsigned reduce_grid, cudaStream_t s, const EvalArgs &args, double *out, int8_t *flags) {
    switch (model) {
        case 0: launch_pair<PREC, 0>(walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags); break;
        case 1: launch_pair<PREC, 1>(walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags); break;
        case 2: launch_pair<PREC, 2>(walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags); break;
        case 3: launch_pair<PREC, 3>(walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags); break;
        case 4: launch_pair<PREC, 4>(walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags); break;
        default: launch_pair<PREC, 5>(walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags); break;
    }
}

// FP64 evaluates the core model at run time (one instantiation); the single precisions are specialised per model.
static void launch_eval(int precision, int model, unsigned walk_grid, int block, size_t smem, uint2 list_grid,
                        int64_t tw, unsigned reduce_grid, cudaStream_t s, const EvalArgs &args, double *out,
                        int8_t *flags) {
    if (precision == BS_FP64) launch_pair<0, 0>(walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags);
    else if (precision == BS_MIXED) launch_model<1>(model, walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags);
    else launch_model<2>(model, walk_grid, block, smem, list_grid, tw, reduce_grid, s, args, out, flags);
}

// exact (may be null): targets marked exact sort after all the others (the key's top bit), in their own warps but
// for one, so that the other targets keep the warps, and with fill the results, they have without them.
int target_order(int64_t n, const double *points, int32_t *perm, Scratch &scratch, cudaStream_t s,
                 const uint8_t *exact = nullptr) {
    unsigned long long *box = scratch.get<unsigned long long>(6);
    uint64_t *keys = scratch.get<uint64_t>(n);
    if (!box || !keys) return scratch.status;
    target_box_init_kernel<<<1, 32, 0, s>>>(box);
    target_box_kernel<<<std::min<unsigned>(nblocks(n, 256), 592), 256, 0, s>>>(n, points, box);
    target_keys_kernel<<<nblocks(n, 256), 256, 0, s>>>(n, points, box, exact, keys, perm);
    BS_CHECK_LAUNCH("target keys");
    // the order groups nearby targets into warps: the top 32 Morton bits (about 10.7 per axis) do that in four passes
    // (a fifth for the exact bit)
    return radix_sort(keys, perm, n, 31, exact ? 64 : 63, scratch, s);
}

// Forest targets: sorted by (wake, Morton key in the wake's own target box); each sorted target learns its root.
__device__ __forceinline__ int target_wake(const int64_t *ptr, int nw, int64_t i) {
    int lo = 0, hi = nw;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (ptr[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ unsigned long long ordered64(double x) {
    unsigned long long b = (unsigned long long)__double_as_longlong(x + 0.0);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// Each wake's target box: blockIdx.x is the wake, the blocks along y stride over its targets; a block folds its part
// in shared memory and adds six atomics.
__global__ void forest_target_box_kernel(const double *points, const int64_t *ptr, unsigned long long *box) {
    __shared__ unsigned long long sb[6];
    const int w = blockIdx.x;
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? ordered64(INFINITY) : ordered64(-INFINITY);
    __syncthreads();
    unsigned long long lo[3] = {ordered64(INFINITY), ordered64(INFINITY), ordered64(INFINITY)};
    unsigned long long hi[3] = {ordered64(-INFINITY), ordered64(-INFINITY), ordered64(-INFINITY)};
    for (int64_t p = ptr[w] + (int64_t)blockIdx.y * blockDim.x + threadIdx.x; p < ptr[w + 1];
         p += (int64_t)gridDim.y * blockDim.x) {
        for (int a = 0; a < 3; ++a) {
            const unsigned long long o = ordered64(points[3 * p + a]);
            lo[a] = o < lo[a] ? o : lo[a];
            hi[a] = o > hi[a] ? o : hi[a];
        }
    }
    for (int a = 0; a < 3; ++a) {
        atomicMin(&sb[a], lo[a]);
        atomicMax(&sb[3 + a], hi[a]);
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&box[6 * w + threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&box[6 * w + threadIdx.x], sb[threadIdx.x]);
}

__global__ void forest_target_box_init_kernel(int nw, unsigned long long *box) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6 * nw) box[i] = (i % 6) < 3 ? ordered64(INFINITY) : ordered64(-INFINITY);
}

__global__ void forest_target_keys_kernel(int64_t n, const double *points, const int64_t *ptr, int nw,
                                          const unsigned long long *box, int bits, const uint8_t *exact,
                                          uint64_t *keys, int32_t *vals) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int w = target_wake(ptr, nw, p);
    double ext = 0.0, lo[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = unordered(box[6 * w + a]);
        ext = fmax(ext, unordered(box[6 * w + 3 + a]) - lo[a]);
    }
    const double inv = ext > 0.0 ? (double)(1u << bits) / ext : 0.0;
    uint64_t key = 0;
    for (int a = 0; a < 3; ++a) {
        uint32_t q = min((1u << bits) - 1u, (uint32_t)((points[3 * p + a] - lo[a]) * inv));
        for (int b = 0; b < bits; ++b) key |= (uint64_t)((q >> b) & 1u) << (3 * b + 2 - a);
    }
    // wake and key use at most 63 bits: the top bit puts exact targets after all the others (see target_order)
    keys[p] = ((uint64_t)w << (3 * bits)) | key | ((exact && exact[p]) ? 1ull << 63 : 0ull);
    vals[p] = (int32_t)p;
}

__global__ void forest_roots_of_kernel(int64_t n, const int32_t *perm, const int64_t *ptr, int nw,
                                       const int32_t *wake_root, int32_t *root_of) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    root_of[i] = wake_root[target_wake(ptr, nw, perm[i])];
}

}  // namespace bs

using namespace bs;

namespace {

int check_eval_args(const bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
                    const bs_kernel_params *kp, const double *out, const int8_t *flags) {
    if (!ctx || !tree || !tp || !tgt || !kp || (tgt->n > 0 && (!tgt->points || !out || !flags))) {
        set_error("tree evaluation: null argument");
        return BS_ERR_ARG;
    }
    if (!(tp->theta > 0.0 && tp->theta < 1.0) || tp->order < 0 || tp->order > 5 || !(tp->clearance >= 0.0)) {
        set_error("tree evaluation: theta must lie in (0, 1), order in 0..5, clearance >= 0");
        return BS_ERR_ARG;
    }
    if ((tp->order == 3 && !tree->order3) || (tp->order == 4 && !tree->order4) || (tp->order == 5 && !tree->order5)) {
        set_error("tree evaluation: order %d needs a tree built with order %d (its moments)", tp->order, tp->order);
        return BS_ERR_ARG;
    }
    if (kp->model < 0 || kp->model > 5 || kp->precision < 0 || kp->precision > 2 ||
        (kp->block != 32 && kp->block != 64 && kp->block != 128 && kp->block != 256)) {
        set_error("tree evaluation: model 0..5, precision 0..2, block 32/64/128/256");
        return BS_ERR_ARG;
    }
    if (tgt->n >= (int64_t(1) << 31)) {
        set_error("tree evaluation: at most 2^31 - 1 targets");
        return BS_ERR_ARG;
    }
    return BS_OK;
}

// What a tree sum prepared beside its build: the sorted target order (perm, complete at perm_ready) and the end of
// the far records' computation (far_ready), for eval_enqueue; all may be null.
struct EvalPre {
    const int32_t *perm = nullptr;
    cudaEvent_t perm_ready = nullptr;
    cudaEvent_t far_ready = nullptr;
    const uint8_t *exact = nullptr;  // EvalArgs::exact
    cudaEvent_t records_ready = nullptr;  // the segment and clear-leaf records complete (before far_ready), or null
};

// Everything the evaluation launches, on stream s, with scratch from `scratch` (pool or arena).  No host
// synchronisation: the counters and the overflow flags stay in `state` (device, 6 words: overflow + 5 counters).
int eval_enqueue(const bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
                 const int64_t *target_wake_ptr, int nw, const bs_kernel_params *kp, double *out, int8_t *flags,
                 int64_t *far_counts, unsigned long long *state, Scratch &scratch, cudaStream_t s,
                 const EvalPre *pre = nullptr) {
    const int64_t n = tgt->n;
    const bool sorted = pre && pre->perm && !target_wake_ptr;
    int32_t *perm = sorted ? const_cast<int32_t *>(pre->perm) : scratch.get<int32_t>(n);
    // near list-kernel work counter, list-pool cursor, far list-kernel work counter
    unsigned long long *queue = scratch.get<unsigned long long>(3);
    int32_t *ex_pos = nullptr, *root_of = nullptr;
    if (!perm || !queue) return scratch.status;
    int rc;
    if (sorted) {
        if (pre->perm_ready) BS_CUDA(cudaStreamWaitEvent(s, pre->perm_ready, 0));
    } else if (target_wake_ptr) {
        int wbits = 0;
        while ((1 << wbits) < nw) ++wbits;
        const int bits = (63 - wbits) / 3;
        unsigned long long *box = scratch.get<unsigned long long>(6 * (size_t)nw);
        uint64_t *keys = scratch.get<uint64_t>(n);
        root_of = scratch.get<int32_t>(n);
        if (!box || !keys || !root_of) return scratch.status;
        forest_target_box_init_kernel<<<nblocks(6 * (int64_t)nw, 256), 256, 0, s>>>(nw, box);
        forest_target_box_kernel<<<dim3((unsigned)nw, 4), 256, 0, s>>>(tgt->points, target_wake_ptr, box);
        forest_target_keys_kernel<<<nblocks(n, 256), 256, 0, s>>>(n, tgt->points, target_wake_ptr, nw, box, bits,
                                                                  pre ? pre->exact : nullptr, keys, perm);
        BS_CHECK_LAUNCH("forest target keys");
        rc = radix_sort(keys, perm, n, 32, 64, scratch, s);  // wake, then the leading Morton bits
        if (rc != BS_OK) return rc;
        forest_roots_of_kernel<<<nblocks(n, 256), 256, 0, s>>>(n, perm, target_wake_ptr, nw, tree->wake_root,
                                                               root_of);
        BS_CHECK_LAUNCH("forest_roots_of_kernel");
    } else {
        rc = target_order(n, tgt->points, perm, scratch, s, pre ? pre->exact : nullptr);
        if (rc != BS_OK) return rc;
    }
    if (tgt->ex_ptr && tgt->e > 0) {
        ex_pos = scratch.get<int32_t>(tgt->e);
        if (!ex_pos) return scratch.status;
        exclusion_positions_kernel<<<nblocks(n, 128), 128, 0, s>>>(n, tgt->ex_ptr, tgt->ex_seg, tree->inverse,
                                                                    ex_pos);
        BS_CHECK_LAUNCH("exclusion_positions_kernel");
    }
    BS_CUDA(cudaMemsetAsync(state, 0, 6 * sizeof(unsigned long long), s));
    BS_CUDA(cudaMemsetAsync(queue, 0, 3 * sizeof(unsigned long long), s));
    const int block = std::min(kp->block, 128);
    const int64_t target_warps = (n + 31) / 32;
    // ~96 cost-balanced work items a SM in all, each warp's list cut in proportion to its cost (item_plan_kernel): the
    // persistent list kernel's last items then end close together, whatever the spread of the warps' costs (32 a SM
    // left a 3-4% tail on the bench workload)
    const int want = ctx->sm_count * 96;
    const size_t capacity = (size_t)want + (size_t)target_warps;
    const size_t slots = (size_t)target_warps, pool = (size_t)target_warps * LIST_POOL;
    int2 *list = scratch.get<int2>(pool);
    int *list_cost = scratch.get<int>(pool);
    int *unit_chunks = scratch.get<int>(slots * LIST_CHUNKS);
    int *list_len = scratch.get<int>(slots), *list_total = scratch.get<int>(slots);
    double *walk_u = scratch.get<double>((size_t)3 * n), *partial = scratch.get<double>(capacity * 32 * 3);
    int8_t *walk_flag = scratch.get<int8_t>((size_t)n), *pflag = scratch.get<int8_t>(capacity * 32);
    int *item_off = scratch.get<int>(slots + 1), *item_warp = scratch.get<int>(capacity);
    int *item_first = scratch.get<int>(capacity);
    if (!list || !list_cost || !unit_chunks || !list_len || !list_total || !walk_u || !partial || !walk_flag || !pflag ||
        !item_off || !item_warp || !item_first)
        return scratch.status;
    EvalArgs args;
    args.n = n;
    args.points = tgt->points;
    args.perm = perm;
    args.ex_ptr = ex_pos ? tgt->ex_ptr : nullptr;
    args.ex_pos = ex_pos;
    args.tv = TreeView{tree->nodes,  tree->far64,  tree->far32, tree->far64x, tree->far32x,
                       tree->far64y, tree->far32y, tree->far64z, tree->far32z, tree->seg64, tree->seg32,
                       tree->seg32x2, tree->seg32c2};
    args.theta = tp->theta;
    args.theta2 = tp->theta * tp->theta;
    args.clearance = tp->clearance;
    args.order = tp->order;
    args.model = kp->model;
    args.raise_singular = kp->raise_singular ? 1 : 0;
    args.deferred = (pre && pre->far_ready) ? 1 : 0;
    args.fill = (tree->kind == BS_TREE_MORTON && kp->precision != BS_FP64) ? 1 : 0;
    args.near2 = (float)(kp->near_cores * kp->near_cores);
    args.stack_limit = (tp->stack_limit > 0 && tp->stack_limit < STACK_DEPTH) ? tp->stack_limit : STACK_DEPTH;
    args.list = list;
    args.list_cost = list_cost;
    args.list_len = list_len;
    args.list_total = list_total;
    args.walk_u = walk_u;
    args.walk_flag = walk_flag;
    args.far_counts = far_counts;
    args.overflow = reinterpret_cast<int *>(state);
    args.counters = state + 1;
    args.partial = partial;
    args.pflag = pflag;
    args.item_off = item_off;
    args.item_warp = item_warp;
    args.item_first = item_first;
    args.item_want = want;
    args.root_of = root_of;
    args.exact = pre ? pre->exact : nullptr;
    args.unit_chunks = unit_chunks;
    args.pool_cursor = queue + 1;
    args.pool_chunks = pool / LIST_CHUNK;
    args.queue = queue;
    const size_t smem = (size_t)(block / 32) * (STACK_DEPTH * sizeof(int2) + 32 * sizeof(Seg64));
    const unsigned walk_grid = (unsigned)((target_warps + block / 32 - 1) / (block / 32));
    // persistent blocks (they take items from a counter): one wave of each list kernel, no more than the items need
    const int64_t list_cap = ((int64_t)capacity + LIST_WARPS - 1) / LIST_WARPS;
    const uint2 list_grid = make_uint2(
        (unsigned)std::max<int64_t>(1, std::min<int64_t>(list_cap, (int64_t)ctx->sm_count * LIST_NEAR_BLOCKS)),
        (unsigned)std::max<int64_t>(1, std::min<int64_t>(list_cap, (int64_t)ctx->sm_count * LIST_FAR_BLOCKS)));
    t_far_ready = args.deferred ? pre->far_ready : nullptr;
    t_records_ready = args.deferred ? pre->records_ready : nullptr;
    launch_eval(kp->precision, kp->model, walk_grid, block, smem, list_grid, target_warps, nblocks(n, 256), s, args,
                out, flags);
    t_far_ready = nullptr;
    t_records_ready = nullptr;
    BS_CHECK_LAUNCH("tree evaluation");
    return BS_OK;
}

}  // namespace

namespace bs {

int tree_lists(const bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
               const bs_kernel_params *kp, Scratch &scratch, cudaStream_t s, TreeLists *lists) {
    const int64_t n = tgt->n;
    int32_t *perm = scratch.get<int32_t>(n);
    unsigned long long *queue = scratch.get<unsigned long long>(2);
    unsigned long long *state = scratch.get<unsigned long long>(6);
    if (!perm || !queue || !state) return scratch.status;
    int rc = target_order(n, tgt->points, perm, scratch, s);
    if (rc != BS_OK) return rc;
    int32_t *ex_pos = nullptr;
    if (tgt->ex_ptr && tgt->e > 0) {
        ex_pos = scratch.get<int32_t>(tgt->e);
        if (!ex_pos) return scratch.status;
        exclusion_positions_kernel<<<nblocks(n, 128), 128, 0, s>>>(n, tgt->ex_ptr, tgt->ex_seg, tree->inverse,
                                                                    ex_pos);
        BS_CHECK_LAUNCH("exclusion_positions_kernel");
    }
    BS_CUDA(cudaMemsetAsync(state, 0, 6 * sizeof(unsigned long long), s));
    BS_CUDA(cudaMemsetAsync(queue, 0, 2 * sizeof(unsigned long long), s));
    const int block = std::min(kp->block, 128);
    const int64_t target_warps = (n + 31) / 32;
    const size_t slots = (size_t)target_warps, pool = (size_t)target_warps * LIST_POOL;
    int2 *list = scratch.get<int2>(pool);
    int *list_cost = scratch.get<int>(pool);
    int *unit_chunks = scratch.get<int>(slots * LIST_CHUNKS);
    int *list_len = scratch.get<int>(slots), *list_total = scratch.get<int>(slots);
    double *walk_u = scratch.get<double>((size_t)3 * n);
    int8_t *walk_flag = scratch.get<int8_t>((size_t)n);
    if (!list || !list_cost || !unit_chunks || !list_len || !list_total || !walk_u || !walk_flag)
        return scratch.status;
    EvalArgs args{};
    args.n = n;
    args.points = tgt->points;
    args.perm = perm;
    args.ex_ptr = ex_pos ? tgt->ex_ptr : nullptr;
    args.ex_pos = ex_pos;
    args.tv = TreeView{tree->nodes,  tree->far64,  tree->far32, tree->far64x, tree->far32x,
                       tree->far64y, tree->far32y, tree->far64z, tree->far32z, tree->seg64, tree->seg32,
                       tree->seg32x2, tree->seg32c2};
    args.theta = tp->theta;
    args.theta2 = tp->theta * tp->theta;
    args.clearance = tp->clearance;
    args.order = tp->order;
    args.model = kp->model;
    args.raise_singular = kp->raise_singular ? 1 : 0;
    args.deferred = 1;  // nothing is evaluated in the walk: what does not fit in the lists is reported
    args.fill = (tree->kind == BS_TREE_MORTON && kp->precision != BS_FP64) ? 1 : 0;  // the forward's lists
    args.near2 = (float)(kp->near_cores * kp->near_cores);
    args.stack_limit = (tp->stack_limit > 0 && tp->stack_limit < STACK_DEPTH) ? tp->stack_limit : STACK_DEPTH;
    args.list = list;
    args.list_cost = list_cost;
    args.list_len = list_len;
    args.list_total = list_total;
    args.walk_u = walk_u;
    args.walk_flag = walk_flag;
    args.overflow = reinterpret_cast<int *>(state);
    args.counters = state + 1;
    args.unit_chunks = unit_chunks;
    args.pool_cursor = queue + 1;
    args.pool_chunks = pool / LIST_CHUNK;
    args.queue = queue;
    const size_t smem = (size_t)(block / 32) * (STACK_DEPTH * sizeof(int2) + 32 * sizeof(Seg64));
    const unsigned walk_grid = (unsigned)((target_warps + block / 32 - 1) / (block / 32));
    switch (kp->model) {
        case 0: tree_walk_kernel<1, 0, 2><<<walk_grid, block, smem, s>>>(args); break;
        case 1: tree_walk_kernel<1, 1, 2><<<walk_grid, block, smem, s>>>(args); break;
        case 2: tree_walk_kernel<1, 2, 2><<<walk_grid, block, smem, s>>>(args); break;
        case 3: tree_walk_kernel<1, 3, 2><<<walk_grid, block, smem, s>>>(args); break;
        case 4: tree_walk_kernel<1, 4, 2><<<walk_grid, block, smem, s>>>(args); break;
        case 5: tree_walk_kernel<1, 5, 2><<<walk_grid, block, smem, s>>>(args); break;
        default:
            set_error("tree lists: core model must be 0..5");
            return BS_ERR_ARG;
    }
    BS_CHECK_LAUNCH("tree_walk_kernel (lists)");
    lists->n = n;
    lists->target_warps = target_warps;
    lists->perm = perm;
    lists->ex_pos = ex_pos;
    lists->ex_ptr = ex_pos ? tgt->ex_ptr : nullptr;
    lists->list = list;
    lists->unit_chunks = unit_chunks;
    lists->list_len = list_len;
    lists->state = state;
    return BS_OK;
}

}  // namespace bs

namespace {

// Runs the evaluation, waits for it and reads counters and the overflow flag into the context's statistics.
int eval_run(bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
             const int64_t *target_wake_ptr, int nw, const bs_kernel_params *kp, double *out, int8_t *flags,
             int64_t *far_counts, cudaStream_t s, const EvalPre *pre = nullptr) {
    Scratch scratch(ctx->pool, s);
    unsigned long long *state = scratch.get<unsigned long long>(7);  // flags, 5 counters, sort fault
    if (!state) return scratch.status;
    cudaEvent_t e0, e1, marks[4];
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (auto &m : marks) cudaEventCreate(&m);
    cudaEventRecord(e0, s);
    t_marks = marks;
    int rc = eval_enqueue(ctx, tree, tp, tgt, target_wake_ptr, nw, kp, out, flags, far_counts, state, scratch, s,
                          pre);
    t_marks = nullptr;
    cudaEventRecord(e1, s);
    unsigned long long host[7] = {0, 0, 0, 0, 0, 0, 0};
    cudaError_t le = cudaSuccess;
    // the sort-fault flag travels back with the counters: one round trip, into the context's pinned words when it has
    // them (an asynchronous copy), copied out at once (a retry below runs this function again)
    const int *fault = sort_fault_flag();
    unsigned long long *pinned = ctx_pinned(ctx);
    unsigned long long *landing = pinned ? pinned + 8 : host;
    if (rc == BS_OK && fault) le = cudaMemcpyAsync(state + 6, fault, sizeof(int), cudaMemcpyDeviceToDevice, s);
    if (rc == BS_OK && le == cudaSuccess) le = cudaMemcpyAsync(landing, state, sizeof host, cudaMemcpyDeviceToHost, s);
    scratch.release();  // stream-ordered frees, queued while the device still works (a retry takes its own scratch)
    if (le == cudaSuccess) le = cudaStreamSynchronize(s);
    if (rc == BS_OK && le == cudaSuccess && landing != host) memcpy(host, landing, sizeof host);
    float ms = 0.f, walk_ms = 0.f, list_ms = 0.f, far_ms = 0.f;
    if (rc == BS_OK && le == cudaSuccess) {
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventElapsedTime(&walk_ms, marks[0], marks[1]);
        cudaEventElapsedTime(&list_ms, marks[1], marks[2]);
        cudaEventElapsedTime(&far_ms, marks[2], marks[3]);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (auto &m : marks) cudaEventDestroy(m);
    if (rc != BS_OK) return rc;
    if (le != cudaSuccess) return cuda_fail(le, "tree evaluation");
    rc = fault ? sort_fault_seen((int)(host[6] & 0xffffffffull)) : check_sort_fault();
    if (rc != BS_OK) return rc;
    ctx->stats.points = tgt->n;
    ctx->stats.segments = tree->m;
    ctx->stats.nodes = tree->count;
    ctx->stats.launches = 3;
    ctx->stats.far_evaluations = (int64_t)host[1];
    ctx->stats.near_pairs = (int64_t)host[2];
    ctx->stats.fp64_pairs = (int64_t)host[3];
    ctx->stats.visits = (int64_t)host[4];
    ctx->stats.pair_slots = (int64_t)host[5];
    ctx->stats.evaluate_ms = ms;
    ctx->stats.walk_ms = walk_ms;
    ctx->stats.list_ms = list_ms;
    ctx->stats.far_ms = far_ms;
    if (host[0] & 0xffffffffull) {
        set_error("tree traversal stack overflow on the GPU (depth %d)",
                  (tp->stack_limit > 0 && tp->stack_limit < STACK_DEPTH) ? tp->stack_limit : STACK_DEPTH);
        return BS_ERR_STACK;
    }
    if (host[0] >> 32) {  // a full list met a node whose records were still being computed: again, with them complete
        EvalPre again;
        if (pre) {
            again.perm = pre->perm;
            again.exact = pre->exact;
        }
        return eval_run(ctx, tree, tp, tgt, target_wake_ptr, nw, kp, out, flags, far_counts, s, &again);
    }
    return BS_OK;
}

// A tree sum's side stream: the target sort is queued there at once (the targets are on the device when s reaches
// this point) and the far records later, so that both run beside the build and the walk on s.
int side_stream(bs_ctx *ctx, cudaStream_t *side) {
    if (!ctx->side_stream) BS_CUDA(cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking));
    *side = ctx->side_stream;
    return BS_OK;
}

int sort_targets_beside(bs_ctx *ctx, const bs_targets *tgt, int32_t *perm, cudaStream_t s, cudaStream_t side,
                        cudaEvent_t *ready) {
    cudaEvent_t fork;
    BS_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(side, fork, 0);
    cudaEventDestroy(fork);
    int rc;
    {
        Scratch scratch(ctx->pool, side);  // allocated and freed in the side stream's order
        rc = target_order(tgt->n, tgt->points, perm, scratch, side);
    }
    if (rc != BS_OK) return rc;
    BS_CUDA(cudaEventCreateWithFlags(ready, cudaEventDisableTiming));
    BS_CUDA(cudaEventRecord(*ready, side));
    return BS_OK;
}

}  // namespace

extern "C" int bs_tree_eval(bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
                            const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts,
                            bs_stream stream) {
    int rc = check_eval_args(ctx, tree, tp, tgt, kp, out, flags);
    if (rc != BS_OK || tgt->n == 0) return rc;
    BS_CUDA(cudaSetDevice(ctx->device));
    return eval_run(ctx, tree, tp, tgt, nullptr, 1, kp, out, flags, far_counts, (cudaStream_t)stream);
}

extern "C" int bs_forest_eval(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp, const bs_targets *tgt,
                              const int64_t *target_wake_ptr, const bs_kernel_params *kp, double *out, int8_t *flags,
                              int64_t *far_counts, bs_stream stream) {
    int rc = check_eval_args(ctx, forest, tp, tgt, kp, out, flags);
    if (rc != BS_OK || tgt->n == 0) return rc;
    if (!forest->wake_root || !target_wake_ptr) {
        set_error("bs_forest_eval: not a forest, or no target ranges");
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaSetDevice(ctx->device));
    return eval_run(ctx, forest, tp, tgt, target_wake_ptr, forest->nwakes, kp, out, flags, far_counts,
                    (cudaStream_t)stream);
}

extern "C" int bs_forest_eval_exact(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp,
                                    const bs_targets *tgt, const int64_t *target_wake_ptr, const uint8_t *exact,
                                    const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts,
                                    bs_stream stream) {
    int rc = check_eval_args(ctx, forest, tp, tgt, kp, out, flags);
    if (rc != BS_OK || tgt->n == 0) return rc;
    if (!forest->wake_root || !target_wake_ptr) {
        set_error("bs_forest_eval_exact: not a forest, or no target ranges");
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaSetDevice(ctx->device));
    EvalPre pre;
    pre.exact = exact;
    return eval_run(ctx, forest, tp, tgt, target_wake_ptr, forest->nwakes, kp, out, flags, far_counts,
                    (cudaStream_t)stream, &pre);
}

extern "C" int bs_tree_sum_host(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, const bs_targets *tgt,
                                const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts,
                                bs_stream stream) {
    if (!ctx || !src || !tp || !tgt || !kp) {
        set_error("bs_tree_sum_host: null argument");
        return BS_ERR_ARG;
    }
    const int64_t n = tgt->n, m = src->m, e = (tgt->ex_ptr && tgt->ex_seg) ? tgt->e : 0;
    if (n < 0 || m < 0 || e < 0 || (n > 0 && (!tgt->points || !out || !flags)) ||
        (m > 0 && (!src->starts || !src->directions || !src->lengths || !src->gamma || !src->radius))) {
        set_error("bs_tree_sum_host: invalid arrays");
        return BS_ERR_ARG;
    }
    if (n == 0) return BS_OK;
    BS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    int rc = BS_OK;
    {
        Scratch scratch(ctx->pool, s);
        double *d_points = scratch.get<double>(3 * n), *d_out = scratch.get<double>(3 * n);
        int8_t *d_flags = scratch.get<int8_t>(n);
        int64_t *d_far = far_counts ? scratch.get<int64_t>(n) : nullptr;
        int64_t *d_ex_ptr = e > 0 ? scratch.get<int64_t>(n + 1) : nullptr;
        int64_t *d_ex_seg = e > 0 ? scratch.get<int64_t>(e) : nullptr;
        double *d_seg = m > 0 ? scratch.get<double>((size_t)9 * m) : nullptr;  // starts, directions, L, gamma, rc
        if (!d_points || !d_out || !d_flags || (far_counts && !d_far) || (e > 0 && (!d_ex_ptr || !d_ex_seg)) ||
            (m > 0 && !d_seg))
            return scratch.status;
        bs_sources dsrc{m, d_seg, d_seg + 3 * m, d_seg + 6 * m, d_seg + 7 * m, d_seg + 8 * m};
        bs_targets dtgt{n, d_points, d_ex_ptr, d_ex_seg, e};
        // 1. targets, exclusions and what the keys and topology need, in one pass of the staging ring
        {
            void *dst[6] = {d_points, d_ex_ptr, d_ex_seg, (void *)dsrc.starts, (void *)dsrc.directions,
                            (void *)dsrc.lengths};
            const void *from[6] = {tgt->points, tgt->ex_ptr, tgt->ex_seg, src->starts, src->directions, src->lengths};
            size_t bytes[6] = {(size_t)3 * n * sizeof(double), e > 0 ? (size_t)(n + 1) * sizeof(int64_t) : 0,
                               (size_t)e * sizeof(int64_t), (size_t)3 * m * sizeof(double),
                               (size_t)3 * m * sizeof(double), (size_t)m * sizeof(double)};
            rc = bs_upload_many(ctx, 6, dst, from, bytes, stream);
            if (rc != BS_OK) return rc;
        }
        double upload_ms = 0.0;
        if (m == 0) {
            BS_CUDA(cudaMemsetAsync(d_out, 0, 3 * n * sizeof(double), s));
            BS_CUDA(cudaMemsetAsync(d_flags, 0, n, s));
            if (d_far) BS_CUDA(cudaMemsetAsync(d_far, 0, n * sizeof(int64_t), s));
            upload_ms = std::chrono::duration<double, std::milli>(clock::now() - t0).count();
        } else {
            // 2. circulations and core radii: staged by the context's staging thread on the copy stream right away
            // (the ring keeps running) while this thread queues the key sort and topology, which need neither
            if (!ctx->copy_stream) BS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
            cudaEvent_t landed;
            BS_CUDA(cudaEventCreateWithFlags(&landed, cudaEventDisableTiming));
            {
                void *dst[2] = {(void *)dsrc.gamma, (void *)dsrc.radius};
                const void *from[2] = {src->gamma, src->radius};
                size_t bytes[2] = {(size_t)m * sizeof(double), (size_t)m * sizeof(double)};
                rc = bs_stage_async(ctx, 2, dst, from, bytes, ctx->copy_stream);
                if (rc != BS_OK) {
                    cudaEventDestroy(landed);
                    return rc;
                }
            }
            bool joined = false;
            auto rest = [&]() -> int {  // before any kernel reads gamma or radius
                const int staged = bs_stage_wait(ctx);
                joined = true;
                upload_ms = std::chrono::duration<double, std::milli>(clock::now() - t0).count();
                if (staged != BS_OK) return staged;
                BS_CUDA(cudaEventRecord(landed, ctx->copy_stream));
                BS_CUDA(cudaStreamWaitEvent(s, landed, 0));
                return BS_OK;
            };
            // the target sort on the side stream, queued while the node count travels back (the device starts on
            // the keys at once; the sort runs beside the packing and the node geometry)
            cudaStream_t side = nullptr;
            cudaEvent_t sorted = nullptr;
            int32_t *perm = scratch.get<int32_t>(n);
            rc = perm ? side_stream(ctx, &side) : scratch.status;
            auto rest_and_sort = [&]() -> int {
                const int r = rest();
                return r != BS_OK ? r : sort_targets_beside(ctx, &dtgt, perm, s, side, &sorted);
            };
            bs_tree *tree = nullptr;
            if (rc == BS_OK) rc = tree_build(ctx, &dsrc, tp, &tree, s, false, rest_and_sort, side);
            if (rc == BS_OK) rc = check_eval_args(ctx, tree, tp, &dtgt, kp, d_out, d_flags);
            if (rc == BS_OK && !sorted) rc = sort_targets_beside(ctx, &dtgt, perm, s, side, &sorted);
            if (rc == BS_OK) {
                const EvalPre pre{perm, sorted, tree->moments_done, nullptr, tree->marks[3]};
                rc = eval_run(ctx, tree, tp, &dtgt, nullptr, 1, kp, d_out, d_flags, d_far, s, &pre);
            }
            if (tree) {
                if (rc == BS_OK) tree_stage_times(tree);
                ctx->stats.build_ms = tree->build_ms;
                ctx->stats.moments_ms = tree->moments_ms;
                tree_release(tree, s);
            }
            if (sorted) {  // the side stream's use of perm ends before perm is freed on s
                cudaStreamWaitEvent(s, sorted, 0);
                cudaEventDestroy(sorted);
            } else if (side) {
                cudaStreamSynchronize(side);
            }
            if (!joined) bs_stage_wait(ctx);
            cudaStreamSynchronize(ctx->copy_stream);  // the staging of the rest has finished on any return
            cudaEventDestroy(landed);
            if (rc != BS_OK) return rc;
        }
        // 3. results through the ring
        const auto t1 = clock::now();
        void *dst[3] = {out, flags, far_counts};
        const void *from[3] = {d_out, d_flags, d_far};
        size_t bytes[3] = {(size_t)3 * n * sizeof(double), (size_t)n, far_counts ? (size_t)n * sizeof(int64_t) : 0};
        rc = bs_download_many(ctx, 3, dst, from, bytes, stream);
        ctx->stats.upload_ms = upload_ms;
        ctx->stats.download_ms = std::chrono::duration<double, std::milli>(clock::now() - t1).count();
    }
    return rc;
}

struct bs_graph {
    int device;
    cudaGraphExec_t exec = nullptr;
    void *arena = nullptr;
    unsigned long long *state = nullptr;
};

static int forest_graph(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp, const bs_targets *tgt,
                        const int64_t *target_wake_ptr, const uint8_t *exact, const bs_kernel_params *kp,
                        double *out, int8_t *flags, int64_t *far_counts, bs_graph **graph) {
    if (!graph) {
        set_error("bs_forest_graph: null output");
        return BS_ERR_ARG;
    }
    *graph = nullptr;
    int rc = check_eval_args(ctx, forest, tp, tgt, kp, out, flags);
    if (rc != BS_OK) return rc;
    if (tgt->n == 0 || (target_wake_ptr && !forest->wake_root)) {
        set_error("bs_forest_graph: no targets, or target ranges for a tree that is not a forest");
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaSetDevice(ctx->device));
    const int nw = target_wake_ptr ? forest->nwakes : 1;
    cudaStream_t s = nullptr;
    BS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    // 1. an ordinary run sizes the arena (and checks that the evaluation succeeds)
    size_t need = 0;
    {
        Scratch probe(ctx->pool, s);
        unsigned long long *state = probe.get<unsigned long long>(6);
        EvalPre pre;
        pre.exact = exact;
        rc = state ? eval_enqueue(ctx, forest, tp, tgt, target_wake_ptr, nw, kp, out, flags, far_counts, state, probe,
                                  s, &pre)
                   : probe.status;
        need = probe.requested;
        cudaError_t e = cudaStreamSynchronize(s);
        if (rc == BS_OK && e != cudaSuccess) rc = cuda_fail(e, "bs_forest_graph sizing run");
        if (rc == BS_OK) rc = check_sort_fault();
    }
    bs_graph *g = new bs_graph();
    g->device = ctx->device;
    cudaError_t e = rc == BS_OK ? cudaMalloc(&g->arena, need + 4096) : cudaSuccess;
    if (rc == BS_OK && e == cudaSuccess) e = cudaMalloc((void **)&g->state, 6 * sizeof(unsigned long long));
    if (rc == BS_OK && e != cudaSuccess) rc = cuda_fail(e, "bs_forest_graph buffers");
    // 2. capture the same launches with scratch carved from the arena
    cudaGraph_t cg = nullptr;
    if (rc == BS_OK) {
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamBeginCapture");
    }
    if (rc == BS_OK) {
        Scratch arena(g->arena, need + 4096, s);
        EvalPre pre;
        pre.exact = exact;
        int rc2 = eval_enqueue(ctx, forest, tp, tgt, target_wake_ptr, nw, kp, out, flags, far_counts, g->state,
                               arena, s, &pre);
        e = cudaStreamEndCapture(s, &cg);
        if (rc2 != BS_OK) rc = rc2;
        else if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture");
    }
    if (rc == BS_OK) {
        e = cudaGraphInstantiate(&g->exec, cg, 0);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate");
    }
    if (cg) cudaGraphDestroy(cg);
    cudaStreamDestroy(s);
    if (rc != BS_OK) {
        bs_graph_free(g);
        return rc;
    }
    *graph = g;
    return BS_OK;
}

extern "C" int bs_forest_graph(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp, const bs_targets *tgt,
                               const int64_t *target_wake_ptr, const bs_kernel_params *kp, double *out,
                               int8_t *flags, int64_t *far_counts, bs_graph **graph) {
    return forest_graph(ctx, forest, tp, tgt, target_wake_ptr, nullptr, kp, out, flags, far_counts, graph);
}

extern "C" int bs_forest_graph_exact(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp,
                                     const bs_targets *tgt, const int64_t *target_wake_ptr, const uint8_t *exact,
                                     const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts,
                                     bs_graph **graph) {
    return forest_graph(ctx, forest, tp, tgt, target_wake_ptr, exact, kp, out, flags, far_counts, graph);
}

extern "C" int bs_graph_launch(bs_graph *g, bs_stream stream) {
    if (!g || !g->exec) {
        set_error("bs_graph_launch: null graph");
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return BS_OK;
}

extern "C" int bs_graph_status(bs_graph *g, bs_stats *stats) {
    if (!g || !stats) {
        set_error("bs_graph_status: null argument");
        return BS_ERR_ARG;
    }
    unsigned long long host[6];
    BS_CUDA(cudaMemcpy(host, g->state, sizeof host, cudaMemcpyDeviceToHost));
    const int sorted = check_sort_fault();
    if (sorted != BS_OK) return sorted;
    memset(stats, 0, sizeof *stats);
    stats->far_evaluations = (int64_t)host[1];
    stats->near_pairs = (int64_t)host[2];
    stats->fp64_pairs = (int64_t)host[3];
    stats->visits = (int64_t)host[4];
    stats->pair_slots = (int64_t)host[5];
    if (host[0] & 0xffffffffull) {
        set_error("tree traversal stack overflow on the GPU");
        return BS_ERR_STACK;
    }
    return BS_OK;
}

extern "C" void bs_graph_free(bs_graph *g) {
    if (!g) return;
    cudaSetDevice(g->device);
    cudaDeviceSynchronize();
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->arena) cudaFree(g->arena);
    if (g->state) cudaFree(g->state);
    delete g;
}

extern "C" int bs_tree_sum(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, const bs_targets *tgt,
                           const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts,
                           bs_stream stream) {
    if (!ctx || !src || !tgt) {
        set_error("bs_tree_sum: null argument");
        return BS_ERR_ARG;
    }
    if (tgt->n == 0) return BS_OK;
    if (src->m == 0) {
        cudaStream_t s = (cudaStream_t)stream;
        BS_CUDA(cudaMemsetAsync(out, 0, tgt->n * 3 * sizeof(double), s));
        BS_CUDA(cudaMemsetAsync(flags, 0, tgt->n, s));
        if (far_counts) BS_CUDA(cudaMemsetAsync(far_counts, 0, tgt->n * sizeof(int64_t), s));
        return BS_OK;
    }
    // the evaluation queues behind the build on the same stream: no wait in between; the target sort and the far
    // records run on the side stream beside the build and the walk; the tree is freed in stream order after the
    // evaluation (which synchronises before it returns)
    cudaStream_t s = (cudaStream_t)stream, side = nullptr;
    BS_CUDA(cudaSetDevice(ctx->device));
    int rc = side_stream(ctx, &side);
    if (rc != BS_OK) return rc;
    float b = 0.f, mm = 0.f;
    {
        Scratch scratch(ctx->pool, s);
        int32_t *perm = scratch.get<int32_t>(tgt->n);
        if (!perm) return scratch.status;
        cudaEvent_t sorted = nullptr;
        // the target sort is queued on the side stream while the node count travels back, so that the device
        // starts on the segments' keys at once
        auto sort_hook = [&]() -> int { return sort_targets_beside(ctx, tgt, perm, s, side, &sorted); };
        bs_tree *tree = nullptr;
        rc = tree_build(ctx, src, tp, &tree, s, false, sort_hook, side);
        if (rc == BS_OK) rc = check_eval_args(ctx, tree, tp, tgt, kp, out, flags);
        if (rc == BS_OK && !sorted) rc = sort_hook();  // (a build that returned before its hook ran)
        if (rc == BS_OK) {
            const EvalPre pre{perm, sorted, tree->moments_done, nullptr, tree->marks[3]};
            rc = eval_run(ctx, tree, tp, tgt, nullptr, 1, kp, out, flags, far_counts, s, &pre);
        }
        if (tree) {
            if (rc == BS_OK) tree_stage_times(tree);
            b = tree->build_ms;
            mm = tree->moments_ms;
            tree_release(tree, s);
        }
        // on every path the side stream's use of perm ends before perm is freed on s
        if (sorted) {
            cudaStreamWaitEvent(s, sorted, 0);
            cudaEventDestroy(sorted);
        } else {
            cudaStreamSynchronize(side);
        }
    }
    ctx->stats.build_ms = b;
    ctx->stats.moments_ms = mm;
    return rc;
}
