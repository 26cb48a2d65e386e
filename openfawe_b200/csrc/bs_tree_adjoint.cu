// Adjoint of the tree sum: for a cotangent w [n,3] of the velocities bs_tree_sum returns, the gradients of
// L = sum_p w_p . u_p with respect to the targets, both segment endpoints and the circulations, as the derivative of
// the forward the tree code actually evaluates (the same tree, the same accepted nodes, the same near pairs).  The
// reference has no adjoint; its forward is vortex_tree.tree_velocity (src/openfawe/aero/vortex_tree.py:508-568) with
// the far field of vortex_tree.far_velocity (:450-497), here to order 5.
//
// The tree is built again (the build is deterministic, so it is the forward's tree) and the walk runs again, writing
// its interaction lists; nothing of the forward is stored.  Then:
//   1. the lists are transposed: for every near leaf the targets that evaluate its pairs, for every accepted node the
//      targets that use its expansion;
//   2. near pairs, segment-major: a thread owns a segment of the leaf and keeps its gradient in registers while the
//      leaf's targets pass by; a lane owns a target's gradient for each group of 32 targets, the pair terms reaching
//      it by shuffles (pair_vjp32, with pair_vjp64 where the forward evaluates the pair in FP64);
//   3. far entries, node-major, in FP64: with b_v = (1/v!) d^v (1/r) at R = x - c (orders 0 .. order + 2, by the
//      recurrence n r^2 b_v + (2n - 1) sum_i R_i b_(v - e_i) + (n - 1) sum_i b_(v - 2 e_i) = 0), the far field of the
//      node's raw moments M_(i;u) = Gamma l_i <rho^u> is
//        u_j = -(1/4 pi) sum_u (-1)^|u| sum_k (u_k + 1) eps_jik M_(i;u) b_(u + e_k),
//      so a target's gradient is -(1/4 pi) sum_u (-1)^|u| sum_(k,m) (u_k + 1)(u_m + delta_km + 1) (w x M_u)_k
//      b_(u + e_k + e_m), and the node's moment cotangent g_(i;u) = -(1/4 pi) (-1)^|u| sum_(k,j) eps_ikj (u_k + 1)
//      H_(u + e_k, j) with H_v = sum over the node's targets of b_v w;
//   4. moment cotangents down the tree: a leaf's segments see its own cotangent plus every ancestor's, carried down by
//      the transpose of the moment translation (g_leaf(i;k) += sum over u >= k of C(u,k) D^(u-k) g_anc(i;u),
//      D = c_leaf - c_anc), and each segment's moments about its leaf centre are differentiated exactly with the
//      three-point Gauss-Legendre rule of the forward (<rho^u> and its derivatives are polynomials of degree <= 5 in
//      the segment parameter).
// Node centres and acceptance decisions are held fixed (they move only where a segment is extreme in its node, and
// the expansion's dependence on its centre is of the truncation order).  Gradients are summed with atomics: the
// result is repeatable to rounding, not bit for bit.
#include <algorithm>
#include <type_traits>

#include "bs_pair_vjp.cuh"
#include "bs_sort.cuh"
#include "bs_tree.cuh"

namespace bs {

namespace {

constexpr int ADJ_ORDER_MAX = 5;
constexpr int N_RAW = 56;   // tuples of orders 0..5 (raw moments of a node, per component)
constexpr int N_DER = 120;  // tuples of orders 0..7 (derivatives of 1/r for the fifth-order gradients)
constexpr int NEAR_TARGETS = 128;  // targets per near work item
constexpr int FAR_TARGETS = 128;   // targets per far work item (four batches of 32)
constexpr int NEAR_THREADS = 128;

// Tuples of an order n in storage order: c0 = n .. 0, then c1 = n - c0 .. 0 (the lexicographic order of the sorted
// index lists, the build's order).
__host__ __device__ constexpr int tuple_offset(int n) { return n * (n + 1) * (n + 2) / 6; }
__host__ __device__ constexpr int tuple_index(int c0, int c1, int c2) {
    return tuple_offset(c0 + c1 + c2) + (c1 + c2) * (c1 + c2 + 1) / 2 + c2;
}

struct TupleCounts {
    unsigned char c[N_DER][3];
};
constexpr TupleCounts make_counts() {
    TupleCounts t{};
    for (int n = 0; n <= 7; ++n)
        for (int c0 = n; c0 >= 0; --c0)
            for (int c1 = n - c0; c1 >= 0; --c1) {
                const int i = tuple_index(c0, c1, n - c0 - c1);
                t.c[i][0] = (unsigned char)c0;
                t.c[i][1] = (unsigned char)c1;
                t.c[i][2] = (unsigned char)(n - c0 - c1);
            }
    return t;
}
__constant__ TupleCounts c_tc = make_counts();
__constant__ double c_binom[6][6] = {{1, 0, 0, 0, 0, 0},  {1, 1, 0, 0, 0, 0},  {1, 2, 1, 0, 0, 0},
                                     {1, 3, 3, 1, 0, 0},  {1, 4, 6, 4, 1, 0},  {1, 5, 10, 10, 5, 1}};

struct AdjArgs {
    int64_t n, m, count;
    int order, model;
    float near2;
    const NodeRec *nodes;
    const Seg32 *seg32;
    const Seg32c2 *seg32c2;  // clear-leaf records: the forward's (tree order, relative to each leaf's centre)
    const Seg64 *seg64;
    const int32_t *order32;  // tree position -> segment
    const double *starts, *directions, *lengths, *gamma;
    const int32_t *perm;
    const int64_t *ex_ptr;
    const int32_t *ex_pos;
    const double *points, *cot;
    const int64_t *near_off, *near_item_off, *far_off, *far_item_off;
    const int32_t *near_items, *far_items;
    const int32_t *parent;
    const int *far_count;
    const double *raw;  // [count][3][56]
    double *G;          // [count][3][56] moment cotangents
    double *gx;         // [n][3]
    double *gseg;       // [m][7] tree order: dA, dB, dGamma
    unsigned long long *queue;  // near, far work counters
    int64_t near_total, far_total;
};

// Raw moments M_(i;u) of every node from the tree's FP64 arrays: m0, m1, m2 (the reference's layout) and the
// symmetric order-3..5 rows of the far records.
__global__ void raw_moments_kernel(AdjArgs a, const double *m0, const double *m1, const double *m2, const Far64x *fx,
                                   const Far64y *fy, const Far64z *fz, double *raw) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.count) return;
    double *out = raw + (size_t)j * 3 * N_RAW;
    for (int i = 0; i < 3; ++i)
        for (int u = 0; u < N_RAW; ++u) {
            const int c0 = c_tc.c[u][0], c1 = c_tc.c[u][1], c2 = c_tc.c[u][2], n = c0 + c1 + c2;
            const int rank = u - tuple_offset(n);
            double v = 0.0;
            if (n <= a.order) {
                if (n == 0) {
                    v = m0[3 * j + i];
                } else if (n == 1) {
                    v = m1[9 * j + 3 * i + (c0 ? 0 : (c1 ? 1 : 2))];
                } else if (n == 2) {  // (a, b) = (0,0) (0,1) (0,2) (1,1) (1,2) (2,2) at 3 a + b
                    const int p = c0 == 2 ? 0 : (c0 == 1 ? (c1 ? 1 : 2) : (c1 == 2 ? 4 : (c1 ? 5 : 8)));
                    v = m2[27 * j + 9 * i + p];
                } else if (n == 3) {
                    v = fx[j].v[G_M3 + 10 * i + rank];
                } else if (n == 4) {
                    v = fy[j].v[K_ROW * i + K_M4 + rank];
                } else {
                    v = fz[j].v[Z_ROW * i + Z_M5 + rank];
                }
            }
            out[i * N_RAW + u] = v;
        }
}

__global__ void parent_of_kernel(int64_t count, const int64_t *left, const int64_t *right, int32_t *parent) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    if (left[j] >= 0) parent[left[j]] = (int32_t)j;
    if (right[j] >= 0) parent[right[j]] = (int32_t)j;
}

// A target at x clear of leaf nr (the forward's pair32x2_clear conditions): at least 1.5 bounding radii from its
// centre, outside the core test's reach (MODEL != 0), within FP32's range.
__device__ __forceinline__ bool adj_clear(double x0, double x1, double x2, const NodeRec &nr, int model, float near2) {
    const double rx = x0 - nr.cx, ry = x1 - nr.cy, rz = x2 - nr.cz;
    const double r2 = rx * rx + ry * ry + rz * rz;
    const bool core = model == 0 || sqrt(r2) - nr.bound > 1.01 * sqrt((double)near2) * nr.clear_core;
    return core && r2 >= 2.25 * nr.bound * nr.bound && r2 > 1e-16 && r2 < 1e18 && nr.bound < 1e9 &&
           fabs(x0) < 1e30 && fabs(x1) < 1e30 && fabs(x2) < 1e30;
}

// 1. Transposition: one warp per warp of targets walks its list.  Counting pass (FILL = false) and filling pass; in
// the filling pass a near leaf's clear targets (adj_clear) fill its list from the front and the others from the back,
// so that its work items of NEAR_TARGETS are all clear but one.
template <bool FILL>
__global__ void transpose_kernel(TreeLists L, int *far_count, int *near_count, int *near_back, const int64_t *far_off,
                                 const int64_t *near_off, int32_t *far_items, int32_t *near_items,
                                 const NodeRec *nodes, const double *points, int model, float near2) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw >= L.target_warps) return;
    const int len = L.list_len[gw];
    const int *chunks = L.unit_chunks + gw * LIST_CHUNKS;
    for (int k = lane; k < len; k += 32) {
        const int2 e = L.list[(int64_t)chunks[k / LIST_CHUNK] * LIST_CHUNK + (k & (LIST_CHUNK - 1))];
        const bool far = e.x & FAR_BIT;
        const int node = e.x & ~FAR_BIT;
        unsigned mask = (unsigned)e.y;
        const int c = __popc(mask);
        if (FILL && !far) {
            const NodeRec nr = nodes[node];
            int32_t *dst = near_items + near_off[node];
            const int64_t total = near_off[node + 1] - near_off[node];
            while (mask) {
                const int l = __ffs(mask) - 1;
                mask &= mask - 1;
                const int64_t p = L.perm[gw * 32 + l];
                const bool clear = adj_clear(points[3 * p], points[3 * p + 1], points[3 * p + 2], nr, model, near2);
                const int64_t at = clear ? atomicAdd(near_count + node, 1)
                                         : total - 1 - atomicAdd(near_back + node, 1);
                dst[at] = (int32_t)(gw * 32 + l);
            }
            continue;
        }
        int *cnt = far ? far_count + node : near_count + node;
        const int base = atomicAdd(cnt, c);
        if (FILL) {
            int32_t *dst = far_items + far_off[node];
            for (int q = 0; mask; ++q) {
                const int l = __ffs(mask) - 1;
                mask &= mask - 1;
                dst[base + q] = (int32_t)(gw * 32 + l);
            }
        }
    }
}

// Offsets of the transposed lists and of their work items (one block): element offsets, then items of NEAR_TARGETS
// / FAR_TARGETS targets.  Zeroes the counts for the filling pass; totals[0..3] = far elements, near elements, far
// items, near items.
__global__ void __launch_bounds__(1024) transpose_scan_kernel(int64_t count, int *far_count, int *near_count,
                                                              int64_t *far_off, int64_t *near_off,
                                                              int64_t *far_item_off, int64_t *near_item_off,
                                                              int64_t *totals) {
    __shared__ int64_t part[4][1024];
    const int t = threadIdx.x;
    const int64_t per = (count + 1023) / 1024, a0 = std::min<int64_t>(count, t * per),
                  a1 = std::min<int64_t>(count, a0 + per);
    int64_t s[4] = {0, 0, 0, 0};
    for (int64_t j = a0; j < a1; ++j) {
        s[0] += far_count[j];
        s[1] += near_count[j];
        s[2] += (far_count[j] + FAR_TARGETS - 1) / FAR_TARGETS;
        s[3] += (near_count[j] + NEAR_TARGETS - 1) / NEAR_TARGETS;
    }
    for (int q = 0; q < 4; ++q) part[q][t] = s[q];
    __syncthreads();
    if (t < 4) {  // exclusive scan of the 1024 partials, one quantity per thread
        int64_t run = 0;
        for (int k = 0; k < 1024; ++k) {
            const int64_t v = part[t][k];
            part[t][k] = run;
            run += v;
        }
        totals[t] = run;
    }
    __syncthreads();
    int64_t r[4] = {part[0][t], part[1][t], part[2][t], part[3][t]};
    for (int64_t j = a0; j < a1; ++j) {
        far_off[j] = r[0];
        near_off[j] = r[1];
        far_item_off[j] = r[2];
        near_item_off[j] = r[3];
        r[0] += far_count[j];
        r[1] += near_count[j];
        r[2] += (far_count[j] + FAR_TARGETS - 1) / FAR_TARGETS;
        r[3] += (near_count[j] + NEAR_TARGETS - 1) / NEAR_TARGETS;
        far_count[j] = 0;
        near_count[j] = 0;
    }
    if (t == 1023) {
        far_off[count] = r[0];
        near_off[count] = r[1];
        far_item_off[count] = r[2];
        near_item_off[count] = r[3];
    }
}

// Node of work item `item`: the last node whose item offset is <= item.
__device__ __forceinline__ int64_t item_node(const int64_t *off, int64_t count, int64_t item) {
    int64_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (off[mid] <= item) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool position_excluded(const int32_t *ex_pos, int64_t e0, int64_t e1, int s) {
    while (e0 < e1) {  // sorted positions: binary search
        const int64_t mid = (e0 + e1) >> 1;
        const int v = ex_pos[mid];
        if (v == s) return true;
        if (v < s) e0 = mid + 1; else e1 = mid;
    }
    return false;
}

// 2. Near pairs, segment-major.  A block takes (leaf, up to NEAR_TARGETS of its targets) items from a counter; its
// threads own the leaf's segments 128 at a time.  In each group of 32 targets, lane l evaluates target (l + j) mod 32
// at step j and passes that target's term to its owner lane by a shuffle, so segment sums stay in registers and each
// target gets one shared-memory add per warp and group.
template <int PREC, int MODEL>
__global__ void __launch_bounds__(NEAR_THREADS) near_adjoint_kernel(AdjArgs a) {
    using T = typename std::conditional<PREC == 0, double, float>::type;  // the sums' type: FP64 in FP64 mode
    __shared__ float4 shi[NEAR_TARGETS], slo[NEAR_TARGETS];  // two-float target: (hi x, y, z, w_x), (lo x, y, z, w_y)
    __shared__ float sw2[NEAR_TARGETS];                      // w_z
    __shared__ float4 srel[NEAR_TARGETS];                    // x - O (leaf centre), FP32, and w_x
    __shared__ float2 sw12[NEAR_TARGETS];                    // w_y, w_z (zero past the item's targets)
    __shared__ T sacc[3][NEAR_TARGETS];
    __shared__ int sp[NEAR_TARGETS];
    __shared__ long long se0[NEAR_TARGETS], se1[NEAR_TARGETS];
    __shared__ long long s_item;
    const int tid = threadIdx.x, lane = tid & 31;
    for (;;) {
        if (tid == 0) s_item = (long long)atomicAdd(a.queue, 1ull);
        __syncthreads();
        const int64_t item = s_item;
        if (item >= a.near_total) break;
        const int64_t leaf = item_node(a.near_item_off, a.count, item);
        const int64_t first = a.near_off[leaf] + (item - a.near_item_off[leaf]) * NEAR_TARGETS;
        const int nt = (int)std::min<int64_t>(NEAR_TARGETS, a.near_off[leaf + 1] - first);
        const NodeRec nr = a.nodes[leaf];
        bool wide = true;  // this target is clear of the leaf: its pairs take pair_vjp32_clear (pair32x2_clear's test)
        if (tid < nt) {
            const int p = a.perm[a.near_items[first + tid]];
            sp[tid] = p;
            float hi[3], lo[3];
            for (int k = 0; k < 3; ++k) {
                split2(a.points[3 * (int64_t)p + k], hi[k], lo[k]);
                sacc[k][tid] = T(0);
            }
            shi[tid] = make_float4(hi[0], hi[1], hi[2], (float)a.cot[3 * (int64_t)p]);
            slo[tid] = make_float4(lo[0], lo[1], lo[2], (float)a.cot[3 * (int64_t)p + 1]);
            sw2[tid] = (float)a.cot[3 * (int64_t)p + 2];
            se0[tid] = a.ex_ptr ? a.ex_ptr[p] : 0;
            se1[tid] = a.ex_ptr ? a.ex_ptr[p + 1] : 0;
            const double x0 = a.points[3 * (int64_t)p], x1 = a.points[3 * (int64_t)p + 1],
                         x2 = a.points[3 * (int64_t)p + 2];
            wide = adj_clear(x0, x1, x2, nr, MODEL, a.near2);
            srel[tid] = make_float4((float)(x0 - nr.cx), (float)(x1 - nr.cy), (float)(x2 - nr.cz),
                                    (float)a.cot[3 * (int64_t)p]);
            sw12[tid] = make_float2((float)a.cot[3 * (int64_t)p + 1], (float)a.cot[3 * (int64_t)p + 2]);
        } else if (tid < NEAR_TARGETS) {  // past the item's targets: the first target's offset, zero cotangent
            const int p = a.perm[a.near_items[first]];
            srel[tid] = make_float4((float)(a.points[3 * (int64_t)p] - nr.cx),
                                    (float)(a.points[3 * (int64_t)p + 1] - nr.cy),
                                    (float)(a.points[3 * (int64_t)p + 2] - nr.cz), 0.0f);
            sw12[tid] = make_float2(0.0f, 0.0f);
        }
        // every target of the item clear: the item's pairs take the clear form (uniform over the block); the barriers
        // also publish the targets staged above
        const int all_wide = __syncthreads_and(wide);
        const int any_excl = __syncthreads_or(tid < nt && se0[tid] < se1[tid]);
        const bool clear_all = PREC != 0 && a.seg32c2 && all_wide;
        for (int base = nr.lo; base < nr.hi; base += NEAR_THREADS) {
            const int s = base + tid;
            const bool valid = s < nr.hi;
            Seg32 r{};
            ClearSeg cq{};
            if (valid && PREC != 0) {
                if (clear_all) {
                    const float *half = reinterpret_cast<const float *>(a.seg32c2 + (s >> 1)) + (s & 1);
                    cq = ClearSeg{half[0], half[2], half[4], half[6], half[8], half[10], half[12], half[14]};
                } else {
                    r = a.seg32[s];
                }
            }
            T sg[7] = {0, 0, 0, 0, 0, 0, 0};
            if (PREC != 0 && clear_all) {
                // the clear form, packed: two groups of 32 targets a pass (.x: g0 + .., .y: g0 + 32 + ..); a target
                // past the item's end or excluded for this segment takes zero cotangent at a valid target's offset
                const float L2 = cq.lx * cq.lx + cq.ly * cq.ly + cq.lz * cq.lz;
                const float iL2 = valid && L2 > 0.0f ? 1.0f / L2 : 0.0f;
                if (!valid) cq.w = INFINITY;  // no segment: zero Gamma, and outside every core range
                float sgf[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (!any_excl) {
                    // no exclusions: the padded offsets and zero cotangents past the item's end need no tests; the
                    // sums stay packed until the end of the item
                    float2 sg2[7];
                    for (int k = 0; k < 7; ++k) sg2[k] = make_float2(0.f, 0.f);
                    for (int g0 = 0; g0 < nt; g0 += 64) {
                        float2 tacc0 = make_float2(0.f, 0.f), tacc1 = tacc0, tacc2 = tacc0;
                        for (int j = 0; j < 32; ++j) {
                            const int tA = g0 + ((lane + j) & 31), tB = tA + 32;
                            const float4 rA = srel[tA], rB = srel[tB];
                            const float2 wA = sw12[tA], wB = sw12[tB];
                            float2 f1[3], f2[3], fg;
                            pair_vjp32_clear2<MODEL>(make_float2(rA.x, rB.x), make_float2(rA.y, rB.y),
                                                     make_float2(rA.z, rB.z), cq, iL2, make_float2(rA.w, rB.w),
                                                     make_float2(wA.x, wB.x), make_float2(wA.y, wB.y), f1, f2, fg);
                            sg2[0] = add2(sg2[0], f1[0]); sg2[1] = add2(sg2[1], f1[1]); sg2[2] = add2(sg2[2], f1[2]);
                            sg2[3] = add2(sg2[3], f2[0]); sg2[4] = add2(sg2[4], f2[1]); sg2[5] = add2(sg2[5], f2[2]);
                            sg2[6] = add2(sg2[6], fg);
                            // lane q owns targets g0 + q and g0 + 32 + q; it receives their terms from lane q - j
                            const int from = (lane - j) & 31;
                            const float2 d0 = add2(f1[0], f2[0]), d1 = add2(f1[1], f2[1]), d2 = add2(f1[2], f2[2]);
                            tacc0 = add2(tacc0, make_float2(__shfl_sync(0xffffffffu, d0.x, from),
                                                            __shfl_sync(0xffffffffu, d0.y, from)));
                            tacc1 = add2(tacc1, make_float2(__shfl_sync(0xffffffffu, d1.x, from),
                                                            __shfl_sync(0xffffffffu, d1.y, from)));
                            tacc2 = add2(tacc2, make_float2(__shfl_sync(0xffffffffu, d2.x, from),
                                                            __shfl_sync(0xffffffffu, d2.y, from)));
                        }
                        if (g0 + lane < nt) {
                            atomicAdd(&sacc[0][g0 + lane], (T)tacc0.x);
                            atomicAdd(&sacc[1][g0 + lane], (T)tacc1.x);
                            atomicAdd(&sacc[2][g0 + lane], (T)tacc2.x);
                        }
                        if (g0 + 32 + lane < nt) {
                            atomicAdd(&sacc[0][g0 + 32 + lane], (T)tacc0.y);
                            atomicAdd(&sacc[1][g0 + 32 + lane], (T)tacc1.y);
                            atomicAdd(&sacc[2][g0 + 32 + lane], (T)tacc2.y);
                        }
                    }
                    for (int k = 0; k < 6; ++k) sgf[k] = -(sg2[k].x + sg2[k].y);
                    sgf[6] = sg2[6].x + sg2[6].y;
                }
                for (int g0 = 0; any_excl && g0 < nt; g0 += 64) {
                    float2 tacc0 = make_float2(0.f, 0.f), tacc1 = tacc0, tacc2 = tacc0;
                    for (int j = 0; j < 32; ++j) {
                        const int tA = g0 + ((lane + j) & 31), tB = tA + 32;
                        auto live = [&](int t) {
                            return valid && t < nt &&
                                   !(a.ex_ptr && se0[t] < se1[t] && position_excluded(a.ex_pos, se0[t], se1[t], s));
                        };
                        const bool okA = live(tA), okB = live(tB);
                        const int iA = tA < nt ? tA : 0, iB = tB < nt ? tB : 0;
                        const float4 rA = srel[iA], rB = srel[iB];
                        const float2 w0 = make_float2(okA ? shi[iA].w : 0.f, okB ? shi[iB].w : 0.f);
                        const float2 w1 = make_float2(okA ? slo[iA].w : 0.f, okB ? slo[iB].w : 0.f);
                        const float2 w2 = make_float2(okA ? sw2[iA] : 0.f, okB ? sw2[iB] : 0.f);
                        float2 f1[3], f2[3], fg;
                        pair_vjp32_clear2<MODEL>(make_float2(rA.x, rB.x), make_float2(rA.y, rB.y),
                                                 make_float2(rA.z, rB.z), cq, iL2, w0, w1, w2, f1, f2, fg);
                        sgf[0] -= f1[0].x + f1[0].y; sgf[1] -= f1[1].x + f1[1].y; sgf[2] -= f1[2].x + f1[2].y;
                        sgf[3] -= f2[0].x + f2[0].y; sgf[4] -= f2[1].x + f2[1].y; sgf[5] -= f2[2].x + f2[2].y;
                        sgf[6] += fg.x + fg.y;
                        // lane q owns targets g0 + q and g0 + 32 + q and receives their terms from lane (q - j) mod 32
                        const int from = (lane - j) & 31;
                        tacc0.x += __shfl_sync(0xffffffffu, f1[0].x + f2[0].x, from);
                        tacc1.x += __shfl_sync(0xffffffffu, f1[1].x + f2[1].x, from);
                        tacc2.x += __shfl_sync(0xffffffffu, f1[2].x + f2[2].x, from);
                        tacc0.y += __shfl_sync(0xffffffffu, f1[0].y + f2[0].y, from);
                        tacc1.y += __shfl_sync(0xffffffffu, f1[1].y + f2[1].y, from);
                        tacc2.y += __shfl_sync(0xffffffffu, f1[2].y + f2[2].y, from);
                    }
                    if (g0 + lane < nt) {
                        atomicAdd(&sacc[0][g0 + lane], (T)tacc0.x);
                        atomicAdd(&sacc[1][g0 + lane], (T)tacc1.x);
                        atomicAdd(&sacc[2][g0 + lane], (T)tacc2.x);
                    }
                    if (g0 + 32 + lane < nt) {
                        atomicAdd(&sacc[0][g0 + 32 + lane], (T)tacc0.y);
                        atomicAdd(&sacc[1][g0 + 32 + lane], (T)tacc1.y);
                        atomicAdd(&sacc[2][g0 + 32 + lane], (T)tacc2.y);
                    }
                }
                if (valid)
                    for (int k = 0; k < 7; ++k) atomicAdd(&a.gseg[7 * (int64_t)s + k], (double)sgf[k]);
                continue;
            }
            for (int g0 = 0; g0 < nt; g0 += 32) {
                T tacc0 = 0, tacc1 = 0, tacc2 = 0;
                for (int j = 0; j < 32; ++j) {
                    const int t = g0 + ((lane + j) & 31);
                    T g1[3] = {0, 0, 0}, g2[3] = {0, 0, 0}, gg = 0;
                    if (valid && t < nt &&
                        !(a.ex_ptr && se0[t] < se1[t] && position_excluded(a.ex_pos, se0[t], se1[t], s))) {
                        bool need64 = true;
                        if (PREC != 0) {
                            float f1[3], f2[3], fg = 0.f;
                            const float4 th = shi[t], tl = slo[t];
                            if (clear_all) {
                                const float4 tr = srel[t];
                                pair_vjp32_clear<MODEL>(tr.x, tr.y, tr.z, cq, th.w, tl.w, sw2[t], f1, f2, fg);
                                need64 = false;
                            } else {
                                need64 = pair_vjp32<MODEL>(th.x, th.y, th.z, tl.x, tl.y, tl.z, r, th.w, tl.w, sw2[t],
                                                           a.near2, f1, f2, fg);
                            }
                            if (!need64) {
                                for (int k = 0; k < 3; ++k) { g1[k] = (T)f1[k]; g2[k] = (T)f2[k]; }
                                gg = (T)fg;
                            }
                        }
                        if (need64) {
                            const Seg64 q = a.seg64[s];
                            const double L = q.len;
                            AdjSeg as;
                            as.ax = q.sx; as.ay = q.sy; as.az = q.sz;
                            as.bx = q.sx + L * q.dx; as.by = q.sy + L * q.dy; as.bz = q.sz + L * q.dz;
                            as.gamma = a.gamma[a.order32[s]];
                            as.irc2L2 = (MODEL >= 1 && MODEL <= 3 && q.radius > 0.0)
                                            ? 1.0 / (L * L * q.radius * q.radius) : 0.0;
                            as.invL2 = q.inv_len * q.inv_len;
                            as.rc2 = (MODEL >= 4 && q.radius > 0.0) ? q.radius * q.radius : 0.0;
                            const int p = sp[t];
                            double h1[3], h2[3], hg = 0.0;
                            if (pair_vjp64(a.points[3 * (int64_t)p], a.points[3 * (int64_t)p + 1],
                                           a.points[3 * (int64_t)p + 2], as, MODEL, a.cot[3 * (int64_t)p],
                                           a.cot[3 * (int64_t)p + 1], a.cot[3 * (int64_t)p + 2], h1, h2, hg)) {
                                for (int k = 0; k < 3; ++k) { g1[k] = (T)h1[k]; g2[k] = (T)h2[k]; }
                                gg = (T)hg;
                            }
                        }
                    }
                    sg[0] -= g1[0]; sg[1] -= g1[1]; sg[2] -= g1[2];
                    sg[3] -= g2[0]; sg[4] -= g2[1]; sg[5] -= g2[2];
                    sg[6] += gg;
                    // lane q owns target g0 + q and receives its term from lane (q - j) mod 32
                    const int from = (lane - j) & 31;
                    tacc0 += __shfl_sync(0xffffffffu, g1[0] + g2[0], from);
                    tacc1 += __shfl_sync(0xffffffffu, g1[1] + g2[1], from);
                    tacc2 += __shfl_sync(0xffffffffu, g1[2] + g2[2], from);
                }
                if (g0 + lane < nt) {
                    atomicAdd(&sacc[0][g0 + lane], tacc0);
                    atomicAdd(&sacc[1][g0 + lane], tacc1);
                    atomicAdd(&sacc[2][g0 + lane], tacc2);
                }
            }
            if (valid)
                for (int k = 0; k < 7; ++k) atomicAdd(&a.gseg[7 * (int64_t)s + k], (double)sg[k]);
        }
        __syncthreads();
        if (tid < nt)
            for (int k = 0; k < 3; ++k) atomicAdd(&a.gx[3 * (int64_t)sp[tid] + k], (double)sacc[k][tid]);
        __syncthreads();
    }
}

// 3. Far entries, node-major, FP64.  One warp per (node, up to FAR_TARGETS of its targets) item.  Lane t of a batch of
// 32 computes its target's b_v (orders 0 .. order + 2) into its row of shared memory and its target gradient; then
// lane l sums H_v = sum_t b_v w_t for its share of v (orders 1 .. order + 1) over the batch.  At the end of the item
// the lanes turn H into the node's moment cotangents and add them.
constexpr int DER_ROW = N_DER + 1;  // odd row length: lanes' rows fall in different banks
constexpr int H_SLOTS = 3;          // v of orders 1..6 per lane: 83 over 32 lanes

template <int ORDER>
__global__ void __launch_bounds__(32) far_adjoint_kernel(AdjArgs a) {
    constexpr int NU = tuple_offset(ORDER + 1);      // moment tuples
    constexpr int NV = tuple_offset(ORDER + 2) - 1;  // v of orders 1 .. ORDER + 1
    __shared__ double sb[32 * DER_ROW];
    __shared__ double sm[3 * N_RAW];
    __shared__ double swv[32][3];
    __shared__ long long s_item;
    const int lane = threadIdx.x;
    double *row = sb + lane * DER_ROW;
    for (;;) {
        if (lane == 0) s_item = (long long)atomicAdd(a.queue + 1, 1ull);
        __syncwarp();
        const int64_t item = s_item;
        __syncwarp();
        if (item >= a.far_total) break;
        const int64_t node = item_node(a.far_item_off, a.count, item);
        const int64_t first = a.far_off[node] + (item - a.far_item_off[node]) * FAR_TARGETS;
        const int nt = (int)std::min<int64_t>(FAR_TARGETS, a.far_off[node + 1] - first);
        for (int q = lane; q < 3 * N_RAW; q += 32) sm[q] = a.raw[(size_t)node * 3 * N_RAW + q];
        const NodeRec nr = a.nodes[node];
        double H[H_SLOTS][3];
        for (int q = 0; q < H_SLOTS; ++q) H[q][0] = H[q][1] = H[q][2] = 0.0;
        __syncwarp();
        for (int b0 = 0; b0 < nt; b0 += 32) {
            const int nb = min(32, nt - b0);
            if (lane < nb) {
                const int p = a.perm[a.far_items[first + b0 + lane]];
                const double R0 = a.points[3 * (int64_t)p] - nr.cx, R1 = a.points[3 * (int64_t)p + 1] - nr.cy,
                             R2 = a.points[3 * (int64_t)p + 2] - nr.cz;
                const double w0 = a.cot[3 * (int64_t)p], w1 = a.cot[3 * (int64_t)p + 1],
                             w2 = a.cot[3 * (int64_t)p + 2];
                swv[lane][0] = w0;
                swv[lane][1] = w1;
                swv[lane][2] = w2;
                const double r2 = R0 * R0 + R1 * R1 + R2 * R2, ir2 = 1.0 / r2;
                row[0] = sqrt(ir2);
#pragma unroll
                for (int n = 1; n <= ORDER + 2; ++n) {
                    const double f1 = (double)(2 * n - 1), f2 = (double)(n - 1), fn = -ir2 / (double)n;
#pragma unroll
                    for (int c0 = n; c0 >= 0; --c0) {
#pragma unroll
                        for (int c1 = n - c0; c1 >= 0; --c1) {
                            const int c2 = n - c0 - c1;
                            double s1 = 0.0, s2 = 0.0;
                            if (c0 >= 1) s1 = fma(R0, row[tuple_index(c0 - 1, c1, c2)], s1);
                            if (c1 >= 1) s1 = fma(R1, row[tuple_index(c0, c1 - 1, c2)], s1);
                            if (c2 >= 1) s1 = fma(R2, row[tuple_index(c0, c1, c2 - 1)], s1);
                            if (c0 >= 2) s2 += row[tuple_index(c0 - 2, c1, c2)];
                            if (c1 >= 2) s2 += row[tuple_index(c0, c1 - 2, c2)];
                            if (c2 >= 2) s2 += row[tuple_index(c0, c1, c2 - 2)];
                            row[tuple_index(c0, c1, c2)] = fn * fma(f1, s1, f2 * s2);
                        }
                    }
                }
                // read the row back from shared memory rather than keeping all of it in registers
                asm volatile("" ::: "memory");
                // the target's gradient: -(1/4 pi) sum_u (-1)^|u| sum_(k,m) (u_k + 1)(u_m + delta_km + 1)
                //                        (w x M_u)_k b_(u + e_k + e_m)
                double gm[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int n = 0; n <= ORDER; ++n) {
#pragma unroll
                    for (int c0 = n; c0 >= 0; --c0) {
#pragma unroll
                        for (int c1 = n - c0; c1 >= 0; --c1) {
                            const int c[3] = {c0, c1, n - c0 - c1};
                            const int u = tuple_index(c[0], c[1], c[2]);
                            const double M0 = sm[u], M1 = sm[N_RAW + u], M2 = sm[2 * N_RAW + u];
                            const double sign = (n & 1) ? -1.0 : 1.0;
                            const double Q[3] = {sign * (w1 * M2 - w2 * M1), sign * (w2 * M0 - w0 * M2),
                                                 sign * (w0 * M1 - w1 * M0)};
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
#pragma unroll
                                for (int mm = 0; mm < 3; ++mm) {
                                    int e[3] = {c[0], c[1], c[2]};
                                    e[k] += 1;
                                    const double ck = (double)e[k];  // u_k + 1
                                    e[mm] += 1;
                                    const double cm = (double)e[mm];  // u_m + delta_km + 1
                                    gm[mm] = fma(ck * cm * Q[k], row[tuple_index(e[0], e[1], e[2])], gm[mm]);
                                }
                            }
                        }
                    }
                }
                atomicAdd(&a.gx[3 * (int64_t)p], -INV_FOUR_PI * gm[0]);
                atomicAdd(&a.gx[3 * (int64_t)p + 1], -INV_FOUR_PI * gm[1]);
                atomicAdd(&a.gx[3 * (int64_t)p + 2], -INV_FOUR_PI * gm[2]);
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < H_SLOTS; ++q) {
                const int v = 1 + lane + 32 * q;
                if (v - 1 < NV) {
                    for (int t = 0; t < nb; ++t) {
                        const double b = sb[t * DER_ROW + v];
                        H[q][0] = fma(b, swv[t][0], H[q][0]);
                        H[q][1] = fma(b, swv[t][1], H[q][1]);
                        H[q][2] = fma(b, swv[t][2], H[q][2]);
                    }
                }
            }
            __syncwarp();
        }
        // H into shared (the rows are free now), then g_(i;u) = -(1/4 pi)(-1)^|u| sum_(k,j) eps_ikj (u_k + 1)
        // H_(u + e_k, j)
#pragma unroll
        for (int q = 0; q < H_SLOTS; ++q) {
            const int v = 1 + lane + 32 * q;
            if (v - 1 < NV)
                for (int j = 0; j < 3; ++j) sb[3 * v + j] = H[q][j];
        }
        __syncwarp();
        for (int u = lane; u < NU; u += 32) {
            const int c0 = c_tc.c[u][0], c1 = c_tc.c[u][1], c2 = c_tc.c[u][2];
            const double sign = -INV_FOUR_PI * (((c0 + c1 + c2) & 1) ? -1.0 : 1.0);
            const double *H0 = sb + 3 * tuple_index(c0 + 1, c1, c2), *H1 = sb + 3 * tuple_index(c0, c1 + 1, c2),
                         *H2 = sb + 3 * tuple_index(c0, c1, c2 + 1);
            const double k0 = c0 + 1.0, k1 = c1 + 1.0, k2 = c2 + 1.0;
            // eps_ikj V_k H_j with V_k = (u_k + 1) H_(u + e_k), componentwise
            const double g0 = k1 * H1[2] - k2 * H2[1];
            const double g1 = k2 * H2[0] - k0 * H0[2];
            const double g2 = k0 * H0[1] - k1 * H1[0];
            double *G = a.G + (size_t)node * 3 * N_RAW;
            atomicAdd(G + u, sign * g0);
            atomicAdd(G + N_RAW + u, sign * g1);
            atomicAdd(G + 2 * N_RAW + u, sign * g2);
        }
        __syncwarp();
    }
}

// 4a. One warp per leaf: the leaf's effective moment cotangent, its own plus every ancestor's translated down, written
// over its row of G (nothing else reads a leaf's row after this); leaf_of marks the leaf's segment positions, or -1
// when no cotangent reaches the leaf.
__global__ void __launch_bounds__(128) pushdown_kernel(AdjArgs a, int32_t *leaf_of) {
    __shared__ double sd[4][3][6];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t leaf = (int64_t)blockIdx.x * 4 + wib;
    if (leaf >= a.count) return;
    const NodeRec nr = a.nodes[leaf];
    if (nr.left >= 0) return;  // warp-uniform
    const int order = a.order, nu = tuple_offset(order + 1);
    bool any = a.far_count[leaf] > 0;
    double acc[2][3] = {{0, 0, 0}, {0, 0, 0}};
    for (int anc = a.parent[leaf]; anc >= 0; anc = a.parent[anc]) {
        if (a.far_count[anc] == 0) continue;
        any = true;
        const NodeRec ar = a.nodes[anc];
        const double D[3] = {nr.cx - ar.cx, nr.cy - ar.cy, nr.cz - ar.cz};
        __syncwarp();
        if (lane < 3) {
            double pw = 1.0;
            for (int e = 0; e < 6; ++e) {
                sd[wib][lane][e] = pw;
                pw *= D[lane];
            }
        }
        __syncwarp();
        const double *Ga = a.G + (size_t)anc * 3 * N_RAW;
        for (int h = 0; h < 2; ++h) {
            const int k = lane + 32 * h;
            if (k >= nu) break;
            const int k0 = c_tc.c[k][0], k1 = c_tc.c[k][1], k2 = c_tc.c[k][2];
            for (int u0 = k0; u0 <= order; ++u0)
                for (int u1 = k1; u0 + u1 <= order; ++u1)
                    for (int u2 = k2; u0 + u1 + u2 <= order; ++u2) {
                        const double coef = c_binom[u0][k0] * c_binom[u1][k1] * c_binom[u2][k2] *
                                            sd[wib][0][u0 - k0] * sd[wib][1][u1 - k1] * sd[wib][2][u2 - k2];
                        const int u = tuple_index(u0, u1, u2);
                        acc[h][0] += coef * Ga[u];
                        acc[h][1] += coef * Ga[N_RAW + u];
                        acc[h][2] += coef * Ga[2 * N_RAW + u];
                    }
        }
    }
    double *g = a.G + (size_t)leaf * 3 * N_RAW;
    for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        if (k < nu)
            for (int i = 0; i < 3; ++i) g[i * N_RAW + k] = (a.far_count[leaf] > 0 ? g[i * N_RAW + k] : 0.0) + acc[h][i];
    }
    for (int pos = nr.lo + lane; pos < nr.hi; pos += 32) leaf_of[pos] = any ? (int32_t)leaf : -1;
}

// 4b. One thread per segment: the derivative of its moments about its leaf centre against the leaf's effective
// cotangent, by the three-point Gauss-Legendre rule on t in [0, 1] (exact for these degree <= 5 polynomials).
template <int ORDER>
__global__ void __launch_bounds__(128) segment_moments_adjoint_kernel(AdjArgs a, const int32_t *leaf_of) {
    const int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= a.m) return;
    const int leaf = leaf_of[pos];
    if (leaf < 0) return;
    const double *g = a.G + (size_t)leaf * 3 * N_RAW;
    const NodeRec nr = a.nodes[leaf];
    const int id = a.order32[pos];
    const double A0 = a.starts[3 * (int64_t)id], A1 = a.starts[3 * (int64_t)id + 1],
                 A2 = a.starts[3 * (int64_t)id + 2];
    const double L = a.lengths[id];
    const double l0 = a.directions[3 * (int64_t)id] * L, l1 = a.directions[3 * (int64_t)id + 1] * L,
                 l2 = a.directions[3 * (int64_t)id + 2] * L;
    const double Gm = a.gamma[id];
    const double al[3] = {Gm * l0, Gm * l1, Gm * l2};
    const double gt[3] = {0.5 - 0.5 * 0.7745966692414834, 0.5, 0.5 + 0.5 * 0.7745966692414834};
    const double gw[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
    double dal[3] = {0, 0, 0}, drA[3] = {0, 0, 0}, drB[3] = {0, 0, 0};
#pragma unroll 1
    for (int q = 0; q < 3; ++q) {
        const double rho[3] = {A0 + gt[q] * l0 - nr.cx, A1 + gt[q] * l1 - nr.cy, A2 + gt[q] * l2 - nr.cz};
        double pw[3][6];
        for (int ax = 0; ax < 3; ++ax) {
            pw[ax][0] = 1.0;
            for (int e = 1; e <= ORDER; ++e) pw[ax][e] = pw[ax][e - 1] * rho[ax];
        }
        double P[3] = {0, 0, 0}, dP[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // dP[i][axis]
#pragma unroll 1
        for (int u = 0; u < tuple_offset(ORDER + 1); ++u) {
            const int c0 = c_tc.c[u][0], c1 = c_tc.c[u][1], c2 = c_tc.c[u][2];
            const double p12 = pw[1][c1] * pw[2][c2];
            const double mono = pw[0][c0] * p12;
            const double d0 = c0 ? c0 * pw[0][c0 - 1] * p12 : 0.0;
            const double d1 = c1 ? c1 * pw[0][c0] * pw[1][c1 - 1] * pw[2][c2] : 0.0;
            const double d2 = c2 ? c2 * pw[0][c0] * pw[1][c1] * pw[2][c2 - 1] : 0.0;
            for (int i = 0; i < 3; ++i) {
                const double gv = g[i * N_RAW + u];
                P[i] = fma(gv, mono, P[i]);
                dP[i][0] = fma(gv, d0, dP[i][0]);
                dP[i][1] = fma(gv, d1, dP[i][1]);
                dP[i][2] = fma(gv, d2, dP[i][2]);
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) dal[i] += gw[q] * P[i];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const double dr = al[0] * dP[0][ax] + al[1] * dP[1][ax] + al[2] * dP[2][ax];
            drA[ax] += gw[q] * (1.0 - gt[q]) * dr;
            drB[ax] += gw[q] * gt[q] * dr;
        }
    }
    double *o = a.gseg + 7 * pos;
    for (int ax = 0; ax < 3; ++ax) {
        o[ax] += -Gm * dal[ax] + drA[ax];
        o[3 + ax] += Gm * dal[ax] + drB[ax];
    }
    o[6] += dal[0] * l0 + dal[1] * l1 + dal[2] * l2;
}

__global__ void adjoint_scatter_kernel(int64_t m, const int32_t *order32, const double *gseg, double *gA, double *gB,
                                       double *gG) {
    const int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= m) return;
    const int64_t id = order32[pos];
    const double *v = gseg + 7 * pos;
    if (gA) for (int k = 0; k < 3; ++k) gA[3 * id + k] = v[k];
    if (gB) for (int k = 0; k < 3; ++k) gB[3 * id + k] = v[3 + k];
    if (gG) gG[id] = v[6];
}

unsigned blocks(int64_t n, int t) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

template <int ORDER>
void launch_far_segments(unsigned far_grid, bool far, int64_t m, cudaStream_t s, const AdjArgs &a,
                         const int32_t *leaf_of, cudaEvent_t mid) {
    if (far) far_adjoint_kernel<ORDER><<<far_grid, 32, 0, s>>>(a);
    cudaEventRecord(mid, s);
    pushdown_kernel<<<blocks(a.count, 4), 128, 0, s>>>(a, const_cast<int32_t *>(leaf_of));
    segment_moments_adjoint_kernel<ORDER><<<blocks(m, 128), 128, 0, s>>>(a, leaf_of);
}

// Models 0-2 in the requested precision; the Vatistas, offset and Rosenhead-Moore cores (3-5, which the reference's
// tree code does not take) with FP64 near pairs (pair_vjp64) in either precision.
template <int PREC>
void launch_near(int model, unsigned grid, cudaStream_t s, const AdjArgs &a) {
    switch (model) {
        case 0: near_adjoint_kernel<PREC, 0><<<grid, NEAR_THREADS, 0, s>>>(a); break;
        case 1: near_adjoint_kernel<PREC, 1><<<grid, NEAR_THREADS, 0, s>>>(a); break;
        case 2: near_adjoint_kernel<PREC, 2><<<grid, NEAR_THREADS, 0, s>>>(a); break;
        case 3: near_adjoint_kernel<0, 3><<<grid, NEAR_THREADS, 0, s>>>(a); break;
        case 4: near_adjoint_kernel<0, 4><<<grid, NEAR_THREADS, 0, s>>>(a); break;
        default: near_adjoint_kernel<0, 5><<<grid, NEAR_THREADS, 0, s>>>(a); break;
    }
}

}  // namespace

}  // namespace bs

using namespace bs;

extern "C" int bs_tree_adjoint(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, const bs_targets *tgt,
                               const bs_kernel_params *kp, const double *cotangent, double *grad_points,
                               double *grad_starts, double *grad_ends, double *grad_gamma, bs_stream stream) {
    if (!ctx || !src || !tp || !tgt || !kp || (tgt->n > 0 && (!tgt->points || !cotangent))) {
        set_error("bs_tree_adjoint: null argument");
        return BS_ERR_ARG;
    }
    if (src->m < 0 || tgt->n < 0 || (src->m > 0 && (!src->starts || !src->directions || !src->lengths ||
                                                     !src->gamma || !src->radius))) {
        set_error("bs_tree_adjoint: invalid arrays");
        return BS_ERR_ARG;
    }
    if (kp->model < 0 || kp->model > 5) {
        set_error("bs_tree_adjoint: core model must be 0..5");
        return BS_ERR_ARG;
    }
    if (!(tp->theta > 0.0 && tp->theta < 1.0) || tp->order < 0 || tp->order > ADJ_ORDER_MAX ||
        !(tp->clearance >= 0.0) || kp->precision < 0 || kp->precision > 2 ||
        (kp->block != 32 && kp->block != 64 && kp->block != 128 && kp->block != 256)) {
        set_error("bs_tree_adjoint: theta in (0, 1), order 0..5, clearance >= 0, precision 0..2, block 32..256");
        return BS_ERR_ARG;
    }
    if (tgt->n >= (int64_t(1) << 31)) {
        set_error("bs_tree_adjoint: at most 2^31 - 1 targets");
        return BS_ERR_ARG;
    }
    const int64_t n = tgt->n, m = src->m;
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    if (grad_points && n) BS_CUDA(cudaMemsetAsync(grad_points, 0, 3 * n * sizeof(double), s));
    if (grad_starts && m) BS_CUDA(cudaMemsetAsync(grad_starts, 0, 3 * m * sizeof(double), s));
    if (grad_ends && m) BS_CUDA(cudaMemsetAsync(grad_ends, 0, 3 * m * sizeof(double), s));
    if (grad_gamma && m) BS_CUDA(cudaMemsetAsync(grad_gamma, 0, m * sizeof(double), s));
    if (n == 0 || m == 0) return BS_OK;
    cudaEvent_t ev[6];
    for (auto &e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], s);
    bs_tree *tree = nullptr;
    // the moment phase (and the segment records) on the side stream, beside the walk and the list transposition,
    // which read neither; the kernels that do wait for them below
    if (!ctx->side_stream) BS_CUDA(cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking));
    int rc = tree_build(ctx, src, tp, &tree, s, false, {}, ctx->side_stream);
    if (rc != BS_OK) {
        for (auto &e : ev) cudaEventDestroy(e);
        return rc;
    }
    int64_t totals[4] = {0, 0, 0, 0};
    unsigned long long state[6] = {0, 0, 0, 0, 0, 0};
    {
        Scratch scratch(ctx->pool, s);
        TreeLists lists;
        rc = tree_lists(ctx, tree, tp, tgt, kp, scratch, s, &lists);
        const int64_t K = tree->count;
        double *raw = scratch.get<double>((size_t)K * 3 * N_RAW), *G = scratch.get<double>((size_t)K * 3 * N_RAW);
        double *gseg = scratch.get<double>((size_t)7 * m);
        double *gx = grad_points ? grad_points : scratch.get<double>((size_t)3 * n);
        int32_t *parent = scratch.get<int32_t>(K), *leaf_of = scratch.get<int32_t>(m);
        int *counts = scratch.get<int>((size_t)3 * K);  // far, near (front), near (back)
        int64_t *offs = scratch.get<int64_t>((size_t)4 * (K + 1));
        int64_t *d_totals = scratch.get<int64_t>(4);
        unsigned long long *queue = scratch.get<unsigned long long>(2);
        if (rc == BS_OK && (!raw || !G || !gseg || !gx || !parent || !leaf_of || !counts || !offs || !d_totals ||
                            !queue))
            rc = scratch.status;
        int *far_count = counts, *near_count = counts + K, *near_back = counts + 2 * K;
        int64_t *far_off = offs, *near_off = offs + (K + 1), *far_item_off = offs + 2 * (K + 1),
                *near_item_off = offs + 3 * (K + 1);
        AdjArgs a{};
        if (rc == BS_OK) {
            cudaMemsetAsync(G, 0, (size_t)K * 3 * N_RAW * sizeof(double), s);
            cudaMemsetAsync(gseg, 0, (size_t)7 * m * sizeof(double), s);
            if (!grad_points) cudaMemsetAsync(gx, 0, (size_t)3 * n * sizeof(double), s);
            cudaMemsetAsync(parent, 0xff, K * sizeof(int32_t), s);
            cudaMemsetAsync(counts, 0, 2 * K * sizeof(int), s);
            cudaMemsetAsync(queue, 0, 2 * sizeof(unsigned long long), s);
            a.n = n;
            a.m = m;
            a.count = K;
            a.order = tp->order;
            a.model = kp->model;
            a.near2 = (float)(kp->near_cores * kp->near_cores);
            a.nodes = tree->nodes;
            a.seg32 = tree->seg32;
            a.seg32c2 = tree->seg32c2;
            a.seg64 = tree->seg64;
            a.order32 = tree->order32;
            a.starts = src->starts;
            a.directions = src->directions;
            a.lengths = src->lengths;
            a.gamma = src->gamma;
            a.perm = lists.perm;
            a.ex_ptr = lists.ex_ptr;
            a.ex_pos = lists.ex_pos;
            a.points = tgt->points;
            a.cot = cotangent;
            a.near_off = near_off;
            a.near_item_off = near_item_off;
            a.far_off = far_off;
            a.far_item_off = far_item_off;
            a.parent = parent;
            a.far_count = far_count;
            a.raw = raw;
            a.G = G;
            a.gx = gx;
            a.gseg = gseg;
            a.queue = queue;
            parent_of_kernel<<<blocks(K, 256), 256, 0, s>>>(K, tree->left, tree->right, parent);
            const unsigned tgrid = blocks(lists.target_warps * 32, 256);
            transpose_kernel<false><<<tgrid, 256, 0, s>>>(lists, far_count, near_count, nullptr, nullptr, nullptr,
                                                          nullptr, nullptr, tree->nodes, tgt->points, kp->model,
                                                          (float)(kp->near_cores * kp->near_cores));
            transpose_scan_kernel<<<1, 1024, 0, s>>>(K, far_count, near_count, far_off, near_off, far_item_off,
                                                     near_item_off, d_totals);
            cudaError_t le = cudaGetLastError();
            if (le == cudaSuccess) le = cudaMemcpyAsync(totals, d_totals, sizeof totals, cudaMemcpyDeviceToHost, s);
            if (le == cudaSuccess) le = cudaMemcpyAsync(state, lists.state, sizeof state, cudaMemcpyDeviceToHost, s);
            if (le == cudaSuccess) le = cudaStreamSynchronize(s);
            if (le != cudaSuccess) rc = cuda_fail(le, "bs_tree_adjoint: lists");
            if (rc == BS_OK && (state[0] & 0xffffffffull)) {
                set_error("tree traversal stack overflow on the GPU");
                rc = BS_ERR_STACK;
            }
            if (rc == BS_OK && (state[0] >> 32)) {
                set_error("bs_tree_adjoint: an interaction list exceeded the list pool (%d entries a warp of targets)",
                          LIST_POOL);
                rc = BS_ERR_OOM;
            }
        }
        cudaEventRecord(ev[1], s);
        int32_t *far_items = nullptr, *near_items = nullptr;
        if (rc == BS_OK) {
            far_items = scratch.get<int32_t>((size_t)std::max<int64_t>(1, totals[0]));
            near_items = scratch.get<int32_t>((size_t)std::max<int64_t>(1, totals[1]));
            if (!far_items || !near_items) rc = scratch.status;
        }
        if (rc == BS_OK) {
            a.far_items = far_items;
            a.near_items = near_items;
            a.far_total = totals[2];
            a.near_total = totals[3];
            const unsigned tgrid = blocks(lists.target_warps * 32, 256);
            // the counts come back to the filled lengths: the far counts then mark the nodes with cotangents
            cudaMemsetAsync(near_back, 0, (size_t)K * sizeof(int), s);
            transpose_kernel<true><<<tgrid, 256, 0, s>>>(lists, far_count, near_count, near_back, far_off, near_off,
                                                         far_items, near_items, tree->nodes, tgt->points, kp->model,
                                                         (float)(kp->near_cores * kp->near_cores));
            static const int near_resident = [] {
                int r = 0;
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, near_adjoint_kernel<1, 2>, NEAR_THREADS,
                                                                     0) == cudaSuccess ? std::max(1, r) : 1;
            }();
            static const int far_resident = [] {
                int r = 0;
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, far_adjoint_kernel<5>, 32, 0) == cudaSuccess
                           ? std::max(1, r) : 1;
            }();
            const unsigned near_grid = (unsigned)std::max<int64_t>(
                1, std::min<int64_t>(totals[3], (int64_t)ctx->sm_count * near_resident));
            const unsigned far_grid = (unsigned)std::max<int64_t>(
                1, std::min<int64_t>(totals[2], (int64_t)ctx->sm_count * far_resident));
            if (tree->moments_done) cudaStreamWaitEvent(s, tree->moments_done, 0);  // moments and segment records
            raw_moments_kernel<<<blocks(K, 128), 128, 0, s>>>(a, tree->m0, tree->m1, tree->m2, tree->far64x,
                                                              tree->far64y, tree->far64z, raw);
            cudaEventRecord(ev[2], s);
            if (totals[3] > 0) {
                if (kp->precision == BS_FP64) launch_near<0>(kp->model, near_grid, s, a);
                else launch_near<1>(kp->model, near_grid, s, a);
            }
            cudaEventRecord(ev[3], s);
            const bool far = totals[2] > 0;
            switch (tp->order) {
                case 0: launch_far_segments<0>(far_grid, far, m, s, a, leaf_of, ev[4]); break;
                case 1: launch_far_segments<1>(far_grid, far, m, s, a, leaf_of, ev[4]); break;
                case 2: launch_far_segments<2>(far_grid, far, m, s, a, leaf_of, ev[4]); break;
                case 3: launch_far_segments<3>(far_grid, far, m, s, a, leaf_of, ev[4]); break;
                case 4: launch_far_segments<4>(far_grid, far, m, s, a, leaf_of, ev[4]); break;
                default: launch_far_segments<5>(far_grid, far, m, s, a, leaf_of, ev[4]); break;
            }
            adjoint_scatter_kernel<<<blocks(m, 256), 256, 0, s>>>(m, tree->order32, gseg, grad_starts, grad_ends,
                                                                  grad_gamma);
            cudaEventRecord(ev[5], s);
            cudaError_t le = cudaGetLastError();
            if (le == cudaSuccess) le = cudaStreamSynchronize(s);
            if (le != cudaSuccess) rc = cuda_fail(le, "bs_tree_adjoint");
        }
        if (rc == BS_OK) rc = check_sort_fault();
        if (rc == BS_OK) {
            float total = 0.f, lists_ms = 0.f, near_ms = 0.f, far_ms = 0.f, seg_ms = 0.f;
            cudaEventElapsedTime(&total, ev[0], ev[5]);
            cudaEventElapsedTime(&lists_ms, ev[0], ev[1]);
            cudaEventElapsedTime(&near_ms, ev[2], ev[3]);
            cudaEventElapsedTime(&far_ms, ev[3], ev[4]);
            cudaEventElapsedTime(&seg_ms, ev[4], ev[5]);
            ctx->stats.points = n;
            ctx->stats.segments = m;
            ctx->stats.nodes = K;
            ctx->stats.launches = 12;
            ctx->stats.far_evaluations = totals[0];
            ctx->stats.near_pairs = 0;
            ctx->stats.evaluate_ms = total;
            ctx->stats.build_ms = lists_ms;  // build, walk and transposition
            ctx->stats.walk_ms = near_ms;    // near pairs
            ctx->stats.list_ms = far_ms;     // far entries
            ctx->stats.far_ms = 0.0;
            ctx->stats.moments_ms = seg_ms;  // push-down, segment moments, scatter
        }
    }
    tree_release(tree, s);
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
}
