// Tree construction on the device: segment packing, Morton-key tree, the reference's median-split tree, node moments.
//
// Median tree: the rule of vortex_tree.build_tree (src/openfawe/aero/vortex_tree.py:51-115, 208-306): split a node of
// more than leaf_size segments with a positive midpoint extent at the middle of its range after a stable sort along the
// longest axis of the midpoint box (lower axis on a tie); depth-first numbering.  The sort is a radix sort by
// (node, dense rank of the coordinate on its axis): LSD radix sorting is stable, so equal coordinates keep their current
// order exactly as numpy's mergesort does.  The host walks the levels (reading one flag per node per level back), as the
// reference's own GPU build does (src/openfawe/aero/vortex_cuda_build.py:234-275).
//
// Morton tree: 16-bit quantisation per axis in IEEE FP64 (no contraction), 48-bit interleaved keys, stable radix sort,
// Karras's binary radix tree (ties broken by position), and a traversal tree made of the internal nodes holding more
// than leaf_size segments plus their small children as leaves.  oracle/morton_oracle.c restates it on the CPU.
//
// Moments: vortex_tree.node_moments (vortex_tree.py:309-376) per node, split into chunks of CHUNK positions so that big
// nodes use many blocks; partial sums are combined in chunk order (run-to-run repeatable).
#include <algorithm>
#include <functional>
#include <vector>

#include "bs_sort.cuh"
#include "bs_tree.cuh"

namespace bs {

constexpr int CHUNK = 2048;
constexpr int MOM_THREADS = 256;
constexpr int MOM_PARTS = 31;   // r2 + m0 (3) + m1 (9) + m2 symmetric (18)
constexpr int MOM_PARTS3 = 61;  // ... + m3 symmetric (30), for third-order trees
constexpr int MOM_PARTS4 = 106; // ... + m4 symmetric (45), for fourth-order trees
constexpr int MOM_PARTS5 = 169; // ... + m5 symmetric (63), for fifth-order trees

__device__ __forceinline__ uint64_t ordered_bits(double x) {
    uint64_t b = (uint64_t)__double_as_longlong(x + 0.0);  // -0.0 -> +0.0 (equal keys compare equal)
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered(uint64_t k) {
    uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

// ---------------------------------------------------------------------------------------------------------------------
// Packing.
// ---------------------------------------------------------------------------------------------------------------------
__global__ void pack_kernel(int64_t m, const double *starts, const double *directions, const double *lengths,
                            const double *gamma, const double *radius, const int32_t *order, Seg64 *seg64,
                            Seg32 *seg32, SegGeo *geo, Seg32x2 *pairs) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    int64_t s = order ? order[k] : k;
    double sx = starts[3 * s], sy = starts[3 * s + 1], sz = starts[3 * s + 2];
    double dx = directions[3 * s], dy = directions[3 * s + 1], dz = directions[3 * s + 2];
    double L = lengths[s], g = gamma[s], r = radius[s];
    if (seg64) {
        Seg64 q;
        q.sx = sx; q.sy = sy; q.sz = sz;
        q.len = L;
        q.dx = dx; q.dy = dy; q.dz = dz;
        q.gfac = (g / L) / 12.566370614359172;  // (gamma / length) / (4 pi), vortex_numba.py:105
        q.rcl = r / L;
        q.radius = r;
        q.inv_len = 1.0 / L;
        q.pad = 0.0;
        seg64[k] = q;
    }
    if (seg32) {
        Seg32 q;
        split2(sx, q.hi.x, q.lo.x);
        split2(sy, q.hi.y, q.lo.y);
        split2(sz, q.hi.z, q.lo.z);
        // a core with rc/L below FP32's comfortable range sends all its pairs to FP64: 1/L is stored as NaN, which
        // fails the pair's "suspect" test; (L/rc)^2 then 0, as without a core
        const double rcl = r / L;
        const bool tiny = r > 0.0 && rcl < 1e-15;
        q.hi.w = tiny ? __int_as_float(0x7fc00000) : (float)(1.0 / L);
        q.lo.w = (float)((g / L) / 12.566370614359172);
        q.dir = make_float4((float)dx, (float)dy, (float)dz, (r > 0.0 && !tiny) ? (float)(1.0 / (rcl * rcl)) : 0.0f);
        seg32[k] = q;
        if (pairs) {  // the packed-pair record (Seg32x2): this segment's half of pair k / 2
            float v[16];
            const bool ok = !tiny && fabsf(q.hi.x) < 1e30f && fabsf(q.hi.y) < 1e30f && fabsf(q.hi.z) < 1e30f;
            v[0] = ok ? -q.hi.x : 0.f; v[1] = ok ? -q.hi.y : 0.f; v[2] = ok ? -q.hi.z : 0.f; v[3] = ok ? q.hi.w : 0.f;
            v[4] = ok ? -q.lo.x : 0.f; v[5] = ok ? -q.lo.y : 0.f; v[6] = ok ? -q.lo.z : 0.f; v[7] = q.lo.w;
            v[8] = q.dir.x; v[9] = q.dir.y; v[10] = q.dir.z; v[11] = q.dir.w;
            v[12] = -q.dir.x; v[13] = -q.dir.y; v[14] = -q.dir.z; v[15] = 0.f;
            float *half = reinterpret_cast<float *>(pairs + (k >> 1)) + (k & 1);
            for (int f = 0; f < 16; ++f) half[2 * f] = v[f];
            if ((m & 1) && k == m - 1)  // the padding half of an odd count's last pair
                for (int f = 0; f < 16; ++f) half[2 * f + 1] = 0.f;
        }
    }
    if (geo) {
        SegGeo q;
        double lx = __dmul_rn(dx, L), ly = __dmul_rn(dy, L), lz = __dmul_rn(dz, L);
        q.sx = sx; q.sy = sy; q.sz = sz;
        q.ex = __dadd_rn(sx, lx); q.ey = __dadd_rn(sy, ly); q.ez = __dadd_rn(sz, lz);
        q.lx = lx; q.ly = ly; q.lz = lz;
        q.gamma = g;
        q.radius = r;
        q.pad = 0.0;
        geo[k] = q;
    }
}

int pack_segments(const bs_sources *src, const int32_t *order, Seg64 *seg64, Seg32 *seg32, SegGeo *geo,
                  cudaStream_t s, Seg32x2 *pairs) {
    if (src->m == 0) return BS_OK;
    pack_kernel<<<(unsigned)((src->m + 255) / 256), 256, 0, s>>>(src->m, src->starts, src->directions, src->lengths,
                                                                 src->gamma, src->radius, order, seg64, seg32, geo,
                                                                 pairs);
    BS_CHECK_LAUNCH("pack_kernel");
    return BS_OK;
}

// mid = 0.5 * (start + end) exactly as numpy forms it.
__device__ __forceinline__ void midpoint(const SegGeo &g, double &x, double &y, double &z) {
    x = __dmul_rn(0.5, __dadd_rn(g.sx, g.ex));
    y = __dmul_rn(0.5, __dadd_rn(g.sy, g.ey));
    z = __dmul_rn(0.5, __dadd_rn(g.sz, g.ez));
}

// ---------------------------------------------------------------------------------------------------------------------
// Morton tree.
// ---------------------------------------------------------------------------------------------------------------------
__global__ void box_init_kernel(unsigned long long *box) {
    if (threadIdx.x < 3) box[threadIdx.x] = ordered_bits(INFINITY);
    else if (threadIdx.x < 6) box[threadIdx.x] = ordered_bits(-INFINITY);
}

// The midpoint midpoint() forms from a SegGeo, formed from the input arrays with the same roundings (pack_kernel's
// end s + (d L)), so that Morton keys need only starts, directions and lengths.
__device__ __forceinline__ void midpoint_raw(const bs_sources &src, int64_t s, double &x, double &y, double &z) {
    const double L = src.lengths[s];
    const double sx = src.starts[3 * s], sy = src.starts[3 * s + 1], sz = src.starts[3 * s + 2];
    const double ex = __dadd_rn(sx, __dmul_rn(src.directions[3 * s], L));
    const double ey = __dadd_rn(sy, __dmul_rn(src.directions[3 * s + 1], L));
    const double ez = __dadd_rn(sz, __dmul_rn(src.directions[3 * s + 2], L));
    x = __dmul_rn(0.5, __dadd_rn(sx, ex));
    y = __dmul_rn(0.5, __dadd_rn(sy, ey));
    z = __dmul_rn(0.5, __dadd_rn(sz, ez));
}

__global__ void mid_box_kernel(int64_t m, const bs_sources src, unsigned long long *box) {
    __shared__ unsigned long long sb[6];
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? ordered_bits(INFINITY) : ordered_bits(-INFINITY);
    __syncthreads();
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < m; s += (int64_t)gridDim.x * blockDim.x) {
        double v[3];
        midpoint_raw(src, s, v[0], v[1], v[2]);
        for (int a = 0; a < 3; ++a) {
            atomicMin(&sb[a], ordered_bits(v[a]));
            atomicMax(&sb[3 + a], ordered_bits(v[a]));
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&box[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&box[threadIdx.x], sb[threadIdx.x]);
}

__device__ __forceinline__ uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

// Keys of the spec in morton_oracle.c: q = min(2^16 - 1, trunc((mid - lo) * inv)), inv = 2^16 / max extent; 48-bit
// keys sort in six 8-bit passes.
__global__ void morton_keys_kernel(int64_t m, const bs_sources src, const unsigned long long *box, uint64_t *keys,
                                   int32_t *vals) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= m) return;
    double lo[3], ext = 0.0;
    for (int a = 0; a < 3; ++a) {
        lo[a] = from_ordered(box[a]);
        double e = __dsub_rn(from_ordered(box[3 + a]), lo[a]);
        if (e > ext) ext = e;
    }
    double inv = ext > 0.0 ? __ddiv_rn(65536.0, ext) : 0.0;
    double v[3];
    midpoint_raw(src, s, v[0], v[1], v[2]);
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        uint32_t u = __double2uint_rz(__dmul_rn(__dsub_rn(v[a], lo[a]), inv));
        q[a] = u > 65535u ? 65535u : u;
    }
    keys[s] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    vals[s] = (int32_t)s;
}

__device__ __forceinline__ int kdelta(const uint64_t *k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = k[i], b = k[j];
    if (a == b) return 64 + __clzll((long long)(i ^ j));
    return __clzll((long long)(a ^ b));
}

__global__ void karras_kernel(int64_t n, const uint64_t *k, int32_t *first, int32_t *last, int32_t *split) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = kdelta(k, n, i, i + 1) - kdelta(k, n, i, i - 1) > 0 ? 1 : -1;
    int dmin = kdelta(k, n, i, i - d);
    int64_t lmax = 2;
    while (kdelta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(k, n, i, i + (l + t) * d) > dmin) l += t;
    int64_t j = i + l * d;
    int dnode = kdelta(k, n, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (kdelta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    split[i] = (int32_t)(i + s * d + (d < 0 ? -1 : 0));
    first[i] = (int32_t)(i < j ? i : j);
    last[i] = (int32_t)(i < j ? j : i);
}

// An internal node is "big" (a traversal node with children) when it holds more than leaf segments or, in a forest,
// when its keys span more than one wake (wake_shift > 0: the bit position of the wake number in the keys).
__device__ __forceinline__ bool big_range(const uint64_t *keys, int wake_shift, int64_t leaf, int64_t f, int64_t l) {
    return (l - f + 1) > leaf || (wake_shift > 0 && (keys[f] >> wake_shift) != (keys[l] >> wake_shift));
}

__device__ __forceinline__ bool big_internal(const uint64_t *keys, int wake_shift, const int32_t *first,
                                             const int32_t *last, int64_t leaf, int64_t c, bool is_leaf_segment) {
    return !is_leaf_segment && big_range(keys, wake_shift, leaf, first[c], last[c]);
}

__global__ void slot_count_kernel(int64_t n, const uint64_t *keys, int wake_shift, const int32_t *first,
                                  const int32_t *last, const int32_t *split, int64_t leaf, int64_t *count) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int64_t c = 0;
    if (big_range(keys, wake_shift, leaf, first[i], last[i])) {
        int32_t g = split[i];
        c = 1 + !big_internal(keys, wake_shift, first, last, leaf, g, g == first[i]) +
            !big_internal(keys, wake_shift, first, last, leaf, g + 1, g + 1 == last[i]);
    }
    count[i] = c;
}

__global__ void slot_fill_kernel(int64_t n, const uint64_t *keys, int wake_shift, const int32_t *first,
                                 const int32_t *last, const int32_t *split, int64_t leaf, const int64_t *slot,
                                 int64_t *lo, int64_t *hi, int64_t *left, int64_t *right) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    if (!big_range(keys, wake_shift, leaf, first[i], last[i])) return;
    int64_t me = slot[i], next = me + 1;
    int32_t g = split[i];
    lo[me] = first[i];
    hi[me] = (int64_t)last[i] + 1;
    if (big_internal(keys, wake_shift, first, last, leaf, g, g == first[i])) {
        left[me] = slot[g];
    } else {
        left[me] = next;
        lo[next] = first[i];
        hi[next] = (int64_t)g + 1;
        left[next] = right[next] = -1;
        ++next;
    }
    if (big_internal(keys, wake_shift, first, last, leaf, g + 1, g + 1 == last[i])) {
        right[me] = slot[g + 1];
    } else {
        right[me] = next;
        lo[next] = (int64_t)g + 1;
        hi[next] = (int64_t)last[i] + 1;
        left[next] = right[next] = -1;
    }
}

__global__ void single_leaf_kernel(int64_t m, int64_t *lo, int64_t *hi, int64_t *left, int64_t *right) {
    lo[0] = 0;
    hi[0] = m;
    left[0] = -1;
    right[0] = -1;
}

__global__ void widen_order_kernel(int64_t m, const int32_t *order32, int64_t *order, int32_t *inverse) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    int32_t s = order32[k];
    order[k] = s;
    inverse[s] = (int32_t)k;
}

__global__ void iota_kernel(int64_t m, int32_t *v) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) v[k] = (int32_t)k;
}

static inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Traversal tree from stably sorted keys (t->order32 holds the sorted segment ids): Karras's binary radix tree, then
// the big internal nodes and their small children numbered by an exclusive scan.
// `while_counting` (may be empty) runs on the host while the node count is on its way back.
static int topology_from_sorted(bs_tree *t, const uint64_t *keys, int wake_shift, Scratch &scratch, cudaStream_t s,
                                const std::function<int()> &while_counting = {}) {
    const int64_t m = t->m;
    if ((m <= t->leaf_size && wake_shift == 0) || m == 1) {
        t->count = 1;
        t->lo = t->alloc<int64_t>(1, s);
        t->hi = t->alloc<int64_t>(1, s);
        t->left = t->alloc<int64_t>(1, s);
        t->right = t->alloc<int64_t>(1, s);
        if (!t->lo || !t->hi || !t->left || !t->right) return BS_ERR_OOM;
        single_leaf_kernel<<<1, 1, 0, s>>>(m, t->lo, t->hi, t->left, t->right);
        BS_CHECK_LAUNCH("single_leaf_kernel");
        return BS_OK;
    }
    int32_t *first = scratch.get<int32_t>(m - 1), *last = scratch.get<int32_t>(m - 1);
    int32_t *split = scratch.get<int32_t>(m - 1);
    int64_t *slot = scratch.get<int64_t>(m - 1), *total = scratch.get<int64_t>(1);
    if (!first || !last || !split || !slot || !total) return scratch.status;
    karras_kernel<<<blocks_for(m - 1, 256), 256, 0, s>>>(m, keys, first, last, split);
    slot_count_kernel<<<blocks_for(m - 1, 256), 256, 0, s>>>(m, keys, wake_shift, first, last, split, t->leaf_size,
                                                             slot);
    BS_CHECK_LAUNCH("karras");
    int rc = scan_exclusive(slot, slot, m - 1, total, scratch, s);
    if (rc != BS_OK) return rc;
    // the count travels back into a pinned word (asynchronously) while the hook queues work that does not need it;
    // the host then waits for the count alone, not for what the hook queued behind it
    int64_t local = 0;
    int64_t *dst = t->host_count ? t->host_count : &local;
    BS_CUDA(cudaMemcpyAsync(dst, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    cudaEvent_t counted = nullptr;
    BS_CUDA(cudaEventCreateWithFlags(&counted, cudaEventDisableTiming));
    cudaError_t ce = cudaEventRecord(counted, s);
    if (ce == cudaSuccess && while_counting) rc = while_counting();
    if (ce == cudaSuccess) ce = cudaEventSynchronize(counted);
    cudaEventDestroy(counted);
    if (ce != cudaSuccess) return cuda_fail(ce, "node count");
    if (rc != BS_OK) return rc;
    const int64_t count = *dst;
    t->count = count;
    t->lo = t->alloc<int64_t>(count, s);
    t->hi = t->alloc<int64_t>(count, s);
    t->left = t->alloc<int64_t>(count, s);
    t->right = t->alloc<int64_t>(count, s);
    if (!t->lo || !t->hi || !t->left || !t->right) return BS_ERR_OOM;
    slot_fill_kernel<<<blocks_for(m - 1, 256), 256, 0, s>>>(m, keys, wake_shift, first, last, split, t->leaf_size,
                                                            slot, t->lo, t->hi, t->left, t->right);
    BS_CHECK_LAUNCH("slot_fill_kernel");
    return BS_OK;
}

static int build_morton(bs_tree *t, const bs_sources *src, Scratch &scratch, cudaStream_t s,
                        const std::function<int()> &while_counting) {
    const int64_t m = t->m;
    unsigned long long *box = scratch.get<unsigned long long>(6);
    uint64_t *keys = scratch.get<uint64_t>(m);
    t->keys = t->alloc<uint64_t>(m, s);
    t->order32 = t->alloc<int32_t>(m, s);
    if (!box || !keys || !t->keys || !t->order32) return scratch.status != BS_OK ? scratch.status : BS_ERR_OOM;
    box_init_kernel<<<1, 32, 0, s>>>(box);
    mid_box_kernel<<<std::min<unsigned>(blocks_for(m, 256), 1184), 256, 0, s>>>(m, *src, box);
    morton_keys_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, *src, box, keys, t->order32);
    BS_CHECK_LAUNCH("morton keys");
    BS_CUDA(cudaMemcpyAsync(t->keys, keys, m * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    int rc = radix_sort(keys, t->order32, m, 0, 48, scratch, s);
    if (rc != BS_OK) return rc;
    return topology_from_sorted(t, keys, 0, scratch, s, while_counting);
}

// ---------------------------------------------------------------------------------------------------------------------
// Forest: many wakes in one Morton tree.  Keys carry the wake number above a per-wake Morton key (each wake quantised
// in its own box), so the radix tree's upper splits fall exactly on wake boundaries, nodes spanning two wakes are
// always split, and every wake's segment range is one node of the traversal tree: its root.
// ---------------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ int wake_of(const int64_t *ptr, int nw, int64_t i) {
    int lo = 0, hi = nw;  // largest w with ptr[w] <= i
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (ptr[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void forest_box_init_kernel(int nw, unsigned long long *box) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6 * nw) box[i] = (i % 6) < 3 ? ordered_bits(INFINITY) : ordered_bits(-INFINITY);
}

// Each wake's midpoint box: blockIdx.x is the wake, the blocks along y stride over its segment range; a block folds
// its part in shared memory and adds six atomics (per-segment atomics on a few hundred words serialise).
__global__ void forest_box_kernel(const SegGeo *geo, const int64_t *wake_ptr, unsigned long long *box) {
    __shared__ unsigned long long sb[6];
    const int w = blockIdx.x;
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? ordered_bits(INFINITY) : ordered_bits(-INFINITY);
    __syncthreads();
    const int64_t a = wake_ptr[w], b = wake_ptr[w + 1];
    unsigned long long lo[3] = {ordered_bits(INFINITY), ordered_bits(INFINITY), ordered_bits(INFINITY)};
    unsigned long long hi[3] = {ordered_bits(-INFINITY), ordered_bits(-INFINITY), ordered_bits(-INFINITY)};
    for (int64_t s = a + (int64_t)blockIdx.y * blockDim.x + threadIdx.x; s < b; s += (int64_t)gridDim.y * blockDim.x) {
        double v[3];
        midpoint(geo[s], v[0], v[1], v[2]);
        for (int x = 0; x < 3; ++x) {
            const unsigned long long o = ordered_bits(v[x]);
            lo[x] = o < lo[x] ? o : lo[x];
            hi[x] = o > hi[x] ? o : hi[x];
        }
    }
    for (int x = 0; x < 3; ++x) {
        atomicMin(&sb[x], lo[x]);
        atomicMax(&sb[3 + x], hi[x]);
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&box[6 * w + threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&box[6 * w + threadIdx.x], sb[threadIdx.x]);
}

__device__ __forceinline__ uint64_t spread_bits(uint32_t v, int bits) {
    uint64_t out = 0;
    for (int i = 0; i < bits; ++i) out |= (uint64_t)((v >> i) & 1u) << (3 * i);
    return out;
}

__global__ void forest_keys_kernel(int64_t m, const SegGeo *geo, const int64_t *wake_ptr, int nw,
                                   const unsigned long long *box, int bits, uint64_t *keys, int32_t *vals) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= m) return;
    const int w = wake_of(wake_ptr, nw, s);
    double lo[3], ext = 0.0;
    for (int a = 0; a < 3; ++a) {
        lo[a] = from_ordered(box[6 * w + a]);
        ext = fmax(ext, __dsub_rn(from_ordered(box[6 * w + 3 + a]), lo[a]));
    }
    const double scale = (double)(1u << bits);
    const double inv = ext > 0.0 ? __ddiv_rn(scale, ext) : 0.0;
    double v[3];
    midpoint(geo[s], v[0], v[1], v[2]);
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        uint32_t u = __double2uint_rz(__dmul_rn(__dsub_rn(v[a], lo[a]), inv));
        q[a] = min(u, (1u << bits) - 1u);
    }
    keys[s] = ((uint64_t)w << (3 * bits)) | (spread_bits(q[0], bits) << 2) | (spread_bits(q[1], bits) << 1) |
              spread_bits(q[2], bits);
    vals[s] = (int32_t)s;
}

// The traversal node whose range is exactly a wake's segment range is that wake's root.
__global__ void forest_roots_kernel(int64_t count, const int64_t *lo, const int64_t *hi, const int64_t *wake_ptr,
                                    int nw, int32_t *roots) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const int w = wake_of(wake_ptr, nw, lo[j]);
    if (lo[j] == wake_ptr[w] && hi[j] == wake_ptr[w + 1]) roots[w] = (int32_t)j;
}

static int build_forest(bs_tree *t, const SegGeo *geo, const int64_t *wake_ptr, int nw, Scratch &scratch,
                        cudaStream_t s) {
    const int64_t m = t->m;
    int wbits = 0;
    while ((1 << wbits) < nw) ++wbits;
    const int bits = (63 - wbits) / 3;
    unsigned long long *box = scratch.get<unsigned long long>(6 * (size_t)nw);
    uint64_t *keys = scratch.get<uint64_t>(m);
    t->keys = t->alloc<uint64_t>(m, s);
    t->order32 = t->alloc<int32_t>(m, s);
    t->wake_root = t->alloc<int32_t>(nw, s);
    if (!box || !keys || !t->keys || !t->order32 || !t->wake_root)
        return scratch.status != BS_OK ? scratch.status : BS_ERR_OOM;
    t->nwakes = nw;
    forest_box_init_kernel<<<blocks_for(6 * (int64_t)nw, 256), 256, 0, s>>>(nw, box);
    forest_box_kernel<<<dim3((unsigned)nw, 16), 256, 0, s>>>(geo, wake_ptr, box);
    forest_keys_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, geo, wake_ptr, nw, box, bits, keys, t->order32);
    BS_CHECK_LAUNCH("forest keys");
    BS_CUDA(cudaMemcpyAsync(t->keys, keys, m * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    int rc = radix_sort(keys, t->order32, m, 0, 64, scratch, s);
    if (rc != BS_OK) return rc;
    rc = topology_from_sorted(t, keys, nw > 1 ? 3 * bits : 0, scratch, s);
    if (rc != BS_OK) return rc;
    BS_CUDA(cudaMemsetAsync(t->wake_root, 0xff, nw * sizeof(int32_t), s));  // -1: a wake without segments
    forest_roots_kernel<<<blocks_for(t->count, 256), 256, 0, s>>>(t->count, t->lo, t->hi, wake_ptr, nw, t->wake_root);
    BS_CHECK_LAUNCH("forest_roots_kernel");
    return BS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// Median tree (the reference's rule).
// ---------------------------------------------------------------------------------------------------------------------
__global__ void axis_keys_kernel(int64_t m, const SegGeo *geo, int axis, uint64_t *keys, int32_t *vals) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= m) return;
    double v[3];
    midpoint(geo[s], v[0], v[1], v[2]);
    keys[s] = ordered_bits(v[axis]);
    vals[s] = (int32_t)s;
}

__global__ void distinct_kernel(int64_t m, const uint64_t *keys, int64_t *flag) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    flag[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1 : 0;
}

__global__ void dense_rank_kernel(int64_t m, const int64_t *flag_scan, const int64_t *flag, const int32_t *vals,
                                  uint32_t *rank) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    rank[vals[k]] = (uint32_t)(flag_scan[k] + flag[k] - 1);  // inclusive count - 1
}

struct Item {
    int32_t node, start, end, pad;
};

// Midpoint box of one chunk of a level node's range.
__global__ void level_box_kernel(const Item *items, int64_t nitems, const int32_t *order, const SegGeo *geo,
                                 double *partial) {
    __shared__ double red[6][MOM_THREADS / 32];
    for (int64_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        Item item = items[it];
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = item.start + threadIdx.x; k < item.end; k += blockDim.x) {
            double v[3];
            midpoint(geo[order[k]], v[0], v[1], v[2]);
            for (int a = 0; a < 3; ++a) {
                lo[a] = fmin(lo[a], v[a]);
                hi[a] = fmax(hi[a], v[a]);
            }
        }
        for (int o = 16; o > 0; o >>= 1)
            for (int a = 0; a < 3; ++a) {
                lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
            }
        int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0)
            for (int a = 0; a < 3; ++a) { red[a][warp] = lo[a]; red[3 + a][warp] = hi[a]; }
        __syncthreads();
        if (threadIdx.x < 6) {
            double v = red[threadIdx.x][0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
                v = threadIdx.x < 3 ? fmin(v, red[threadIdx.x][w]) : fmax(v, red[threadIdx.x][w]);
            partial[6 * it + threadIdx.x] = v;
        }
        __syncthreads();
    }
}

// Per level node: combine its chunks, longest axis (lowest on ties), split flag.
// degenerate (may be null): set when a node large enough to split has a box of zero extent and so does not split.
__global__ void level_split_kernel(int64_t nodes, const int64_t *first_item, const int64_t *item_count,
                                   const double *partial, int8_t *split, int8_t *axis_of, int *degenerate) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nodes) return;
    if (item_count[j] == 0) {
        split[j] = 0;
        axis_of[j] = 0;
        return;
    }
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t it = first_item[j]; it < first_item[j] + item_count[j]; ++it)
        for (int a = 0; a < 3; ++a) {
            lo[a] = fmin(lo[a], partial[6 * it + a]);
            hi[a] = fmax(hi[a], partial[6 * it + 3 + a]);
        }
    int axis = 0;
    double extent = hi[0] - lo[0];
    for (int c = 1; c < 3; ++c)
        if (hi[c] - lo[c] > extent) { extent = hi[c] - lo[c]; axis = c; }
    split[j] = extent > 0.0 ? 1 : 0;
    axis_of[j] = (int8_t)axis;
    if (degenerate && !(extent > 0.0)) atomicOr(degenerate, 1);
}

// The axis of every node of the sort list: axis_of[map[r]].
__global__ void sort_axis_kernel(int64_t count, const int64_t *map, const int8_t *axis_of, int8_t *sort_axis) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < count) sort_axis[r] = axis_of[map[r]];
}

// Keys (node rank in the sort list, dense coordinate rank on its axis) for the elements of splitting nodes.
__global__ void level_gather_kernel(const Item *items, int64_t nitems, const int64_t *dest_offset,
                                    const int8_t *axis_of, const int32_t *order, const uint32_t *rank_x,
                                    const uint32_t *rank_y, const uint32_t *rank_z, int rank_bits, uint64_t *keys,
                                    int32_t *vals) {
    for (int64_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        Item item = items[it];  // node = index in the sort list; start/end: positions; pad: node's range start
        const uint32_t *rank = axis_of[item.node] == 0 ? rank_x : (axis_of[item.node] == 1 ? rank_y : rank_z);
        for (int k = item.start + threadIdx.x; k < item.end; k += blockDim.x) {
            int32_t s = order[k];
            int64_t d = dest_offset[item.node] + (k - item.pad);
            keys[d] = ((uint64_t)item.node << rank_bits) | rank[s];
            vals[d] = s;
        }
    }
}

__global__ void level_scatter_kernel(const Item *items, int64_t nitems, const int64_t *dest_offset,
                                     const int32_t *vals, int32_t *order) {
    for (int64_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        Item item = items[it];
        for (int k = item.start + threadIdx.x; k < item.end; k += blockDim.x)
            order[k] = vals[dest_offset[item.node] + (k - item.pad)];
    }
}

static int bits_for(int64_t v) {
    int b = 0;
    while ((int64_t(1) << b) <= v) ++b;
    return b;
}

template <class T> static int upload(Scratch &scratch, const std::vector<T> &v, T **dev, cudaStream_t s) {
    *dev = scratch.get<T>(v.size());
    if (!*dev) return scratch.status;
    if (!v.empty()) BS_CUDA(cudaMemcpyAsync(*dev, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return BS_OK;
}

static int build_median(bs_tree *t, const SegGeo *geo, Scratch &scratch, cudaStream_t s) {
    const int64_t m = t->m, leaf = t->leaf_size;
    t->order32 = t->alloc<int32_t>(m, s);
    if (!t->order32) return BS_ERR_OOM;
    iota_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, t->order32);
    BS_CHECK_LAUNCH("iota_kernel");
    // Dense coordinate ranks per axis (equal coordinates share a rank).
    uint32_t *rank[3];
    uint64_t *keys = scratch.get<uint64_t>(m);
    int32_t *vals = scratch.get<int32_t>(m);
    int64_t *flag = scratch.get<int64_t>(m), *flag_scan = scratch.get<int64_t>(m);
    if (!keys || !vals || !flag || !flag_scan) return scratch.status;
    bool needs_sort = m > leaf;
    for (int a = 0; a < 3 && needs_sort; ++a) {
        rank[a] = scratch.get<uint32_t>(m);
        if (!rank[a]) return scratch.status;
        axis_keys_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, geo, a, keys, vals);
        BS_CHECK_LAUNCH("axis_keys_kernel");
        int rc = radix_sort(keys, vals, m, 0, 64, scratch, s);
        if (rc != BS_OK) return rc;
        distinct_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, keys, flag);
        rc = scan_exclusive(flag, flag_scan, m, nullptr, scratch, s);
        if (rc != BS_OK) return rc;
        dense_rank_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, flag_scan, flag, vals, rank[a]);
        BS_CHECK_LAUNCH("dense_rank_kernel");
    }
    const int rank_bits = bits_for(m);
    int64_t capacity = 4 * (m / std::max<int64_t>(leaf, 1) + 1) + 1;
    std::vector<int64_t> lo(capacity), hi(capacity), left(capacity, -1), right(capacity, -1);
    lo[0] = 0;
    hi[0] = m;
    int64_t count = 1;
    // Planned levels: a node larger than a leaf splits at its middle unless its box has no extent, so the topology
    // follows from m and the leaf size alone unless some node is degenerate.  Every level is queued at once on that
    // plan (the axes are chosen and used on the device, no read-back between levels); one read-back at the end says
    // whether a degenerate node occurred, and then the levels below are run again one at a time with their decisions
    // read back.
    if (needs_sort) {
        int *degenerate = scratch.get<int>(1);
        if (!degenerate) return scratch.status;
        BS_CUDA(cudaMemsetAsync(degenerate, 0, sizeof(int), s));
        std::vector<int64_t> level{0};
        while (!level.empty()) {
            Scratch ls(t->pool, s);  // this level's temporaries, freed in stream order
            std::vector<Item> items, sort_items;
            std::vector<int64_t> first_item(level.size()), item_count(level.size()), dest, map, following;
            int64_t total = 0;
            for (size_t j = 0; j < level.size(); ++j) {
                const int64_t node = level[j], a = lo[node], b = hi[node];
                first_item[j] = (int64_t)items.size();
                if (b - a > leaf) {
                    for (int64_t c = a; c < b; c += CHUNK)
                        items.push_back({(int32_t)j, (int32_t)c, (int32_t)std::min(b, c + CHUNK), 0});
                    const int64_t middle = (a + b) / 2, f = count, g = count + 1;
                    count += 2;
                    lo[f] = a; hi[f] = middle; lo[g] = middle; hi[g] = b;
                    left[node] = f; right[node] = g;
                    following.push_back(f);
                    following.push_back(g);
                    const int32_t r = (int32_t)dest.size();
                    dest.push_back(total);
                    map.push_back((int64_t)j);
                    for (int64_t c = a; c < b; c += CHUNK)
                        sort_items.push_back({r, (int32_t)c, (int32_t)std::min(b, c + CHUNK), (int32_t)a});
                    total += b - a;
                }
                item_count[j] = (int64_t)items.size() - first_item[j];
            }
            if (items.empty()) break;
            Item *d_items, *d_sort_items;
            int64_t *d_first, *d_count, *d_dest, *d_map;
            double *partial = ls.get<double>(6 * items.size());
            int8_t *d_split = ls.get<int8_t>(level.size()), *d_axis = ls.get<int8_t>(level.size());
            int8_t *d_sort_axis = ls.get<int8_t>(dest.size());
            int rc = upload(ls, items, &d_items, s);
            if (rc == BS_OK) rc = upload(ls, first_item, &d_first, s);
            if (rc == BS_OK) rc = upload(ls, item_count, &d_count, s);
            if (rc == BS_OK) rc = upload(ls, sort_items, &d_sort_items, s);
            if (rc == BS_OK) rc = upload(ls, dest, &d_dest, s);
            if (rc == BS_OK) rc = upload(ls, map, &d_map, s);
            if (rc != BS_OK || !partial || !d_split || !d_axis || !d_sort_axis) return rc != BS_OK ? rc : ls.status;
            level_box_kernel<<<(unsigned)std::min<size_t>(items.size(), 4096), MOM_THREADS, 0, s>>>(
                d_items, (int64_t)items.size(), t->order32, geo, partial);
            level_split_kernel<<<blocks_for((int64_t)level.size(), 128), 128, 0, s>>>(
                (int64_t)level.size(), d_first, d_count, partial, d_split, d_axis, degenerate);
            sort_axis_kernel<<<blocks_for((int64_t)dest.size(), 128), 128, 0, s>>>((int64_t)dest.size(), d_map, d_axis,
                                                                                   d_sort_axis);
            const unsigned grid = (unsigned)std::min<size_t>(sort_items.size(), 4096);
            level_gather_kernel<<<grid, 256, 0, s>>>(d_sort_items, (int64_t)sort_items.size(), d_dest, d_sort_axis,
                                                     t->order32, rank[0], rank[1], rank[2], rank_bits, keys, vals);
            BS_CHECK_LAUNCH("planned median level");
            rc = radix_sort(keys, vals, total, 0, rank_bits + bits_for((int64_t)dest.size() - 1), ls, s);
            if (rc != BS_OK) return rc;
            level_scatter_kernel<<<grid, 256, 0, s>>>(d_sort_items, (int64_t)sort_items.size(), d_dest, vals,
                                                      t->order32);
            BS_CHECK_LAUNCH("level_scatter_kernel");
            level.swap(following);
        }
        int found = 0;
        BS_CUDA(cudaMemcpyAsync(&found, degenerate, sizeof(int), cudaMemcpyDeviceToHost, s));
        BS_CUDA(cudaStreamSynchronize(s));
        if (!found) {
            needs_sort = false;  // the planned levels are the tree
        } else {  // start again, one level at a time
            iota_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, t->order32);
            BS_CHECK_LAUNCH("iota_kernel");
            std::fill(left.begin(), left.end(), -1);
            std::fill(right.begin(), right.end(), -1);
            count = 1;
        }
    }
    std::vector<int64_t> level{0};
    while (!level.empty() && needs_sort) {
        Scratch scratch(t->pool, s);  // this level's temporaries (shadows the call's scratch)
        // chunks of every node that may split
        std::vector<Item> items;
        std::vector<int64_t> first_item(level.size()), item_count(level.size());
        for (size_t j = 0; j < level.size(); ++j) {
            int64_t a = lo[level[j]], b = hi[level[j]];
            first_item[j] = (int64_t)items.size();
            if (b - a > leaf)
                for (int64_t c = a; c < b; c += CHUNK) items.push_back({(int32_t)j, (int32_t)c, (int32_t)std::min(b, c + CHUNK), 0});
            item_count[j] = (int64_t)items.size() - first_item[j];
        }
        std::vector<int8_t> split(level.size(), 0), axis_of(level.size(), 0);
        if (!items.empty()) {
            Item *d_items;
            int64_t *d_first, *d_count;
            double *partial = scratch.get<double>(6 * items.size());
            int8_t *d_split = scratch.get<int8_t>(level.size()), *d_axis = scratch.get<int8_t>(level.size());
            int rc = upload(scratch, items, &d_items, s);
            if (rc == BS_OK) rc = upload(scratch, first_item, &d_first, s);
            if (rc == BS_OK) rc = upload(scratch, item_count, &d_count, s);
            if (rc != BS_OK || !partial || !d_split || !d_axis) return rc != BS_OK ? rc : scratch.status;
            level_box_kernel<<<(unsigned)std::min<size_t>(items.size(), 4096), MOM_THREADS, 0, s>>>(
                d_items, (int64_t)items.size(), t->order32, geo, partial);
            level_split_kernel<<<blocks_for((int64_t)level.size(), 128), 128, 0, s>>>(
                (int64_t)level.size(), d_first, d_count, partial, d_split, d_axis, nullptr);
            BS_CHECK_LAUNCH("level box/split");
            BS_CUDA(cudaMemcpyAsync(split.data(), d_split, level.size(), cudaMemcpyDeviceToHost, s));
            BS_CUDA(cudaMemcpyAsync(axis_of.data(), d_axis, level.size(), cudaMemcpyDeviceToHost, s));
            BS_CUDA(cudaStreamSynchronize(s));
        }
        // children (vortex_tree._next_level) and the sort list
        std::vector<int64_t> following;
        std::vector<Item> sort_items;
        std::vector<int64_t> dest;
        std::vector<int8_t> sort_axis;
        int64_t total = 0;
        for (size_t j = 0; j < level.size(); ++j) {
            if (!split[j]) continue;
            int64_t node = level[j], a = lo[node], b = hi[node], middle = (a + b) / 2;
            int64_t f = count, g = count + 1;
            count += 2;
            lo[f] = a; hi[f] = middle; lo[g] = middle; hi[g] = b;
            left[node] = f; right[node] = g;
            following.push_back(f);
            following.push_back(g);
            int32_t r = (int32_t)dest.size();
            dest.push_back(total);
            sort_axis.push_back(axis_of[j]);
            for (int64_t c = a; c < b; c += CHUNK) sort_items.push_back({r, (int32_t)c, (int32_t)std::min(b, c + CHUNK), (int32_t)a});
            total += b - a;
        }
        if (total > 0) {
            Item *d_items;
            int64_t *d_dest;
            int8_t *d_axis;
            int rc = upload(scratch, sort_items, &d_items, s);
            if (rc == BS_OK) rc = upload(scratch, dest, &d_dest, s);
            if (rc == BS_OK) rc = upload(scratch, sort_axis, &d_axis, s);
            if (rc != BS_OK) return rc;
            unsigned grid = (unsigned)std::min<size_t>(sort_items.size(), 4096);
            level_gather_kernel<<<grid, 256, 0, s>>>(d_items, (int64_t)sort_items.size(), d_dest, d_axis, t->order32,
                                                     rank[0], rank[1], rank[2], rank_bits, keys, vals);
            BS_CHECK_LAUNCH("level_gather_kernel");
            rc = radix_sort(keys, vals, total, 0, rank_bits + bits_for((int64_t)dest.size() - 1), scratch, s);
            if (rc != BS_OK) return rc;
            level_scatter_kernel<<<grid, 256, 0, s>>>(d_items, (int64_t)sort_items.size(), d_dest, vals, t->order32);
            BS_CHECK_LAUNCH("level_scatter_kernel");
        }
        level.swap(following);
    }
    // depth-first numbering (vortex_tree._renumber)
    std::vector<int64_t> number(count), olo(count), ohi(count), oleft(count, -1), oright(count, -1), stack;
    number[0] = 0;
    olo[0] = lo[0];
    ohi[0] = hi[0];
    int64_t assigned = 1;
    stack.push_back(0);
    while (!stack.empty()) {
        int64_t node = stack.back();
        stack.pop_back();
        if (left[node] < 0) continue;
        int64_t f = assigned, g = assigned + 1;
        assigned += 2;
        number[left[node]] = f;
        number[right[node]] = g;
        oleft[number[node]] = f;
        oright[number[node]] = g;
        olo[f] = lo[left[node]]; ohi[f] = hi[left[node]];
        olo[g] = lo[right[node]]; ohi[g] = hi[right[node]];
        stack.push_back(right[node]);
        stack.push_back(left[node]);
    }
    t->count = count;
    t->lo = t->alloc<int64_t>(count, s);
    t->hi = t->alloc<int64_t>(count, s);
    t->left = t->alloc<int64_t>(count, s);
    t->right = t->alloc<int64_t>(count, s);
    if (!t->lo || !t->hi || !t->left || !t->right) return BS_ERR_OOM;
    BS_CUDA(cudaMemcpyAsync(t->lo, olo.data(), count * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    BS_CUDA(cudaMemcpyAsync(t->hi, ohi.data(), count * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    BS_CUDA(cudaMemcpyAsync(t->left, oleft.data(), count * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    BS_CUDA(cudaMemcpyAsync(t->right, oright.data(), count * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    BS_CUDA(cudaStreamSynchronize(s));  // the host vectors above go out of scope
    return BS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// Moments.
// ---------------------------------------------------------------------------------------------------------------------
// Index of the symmetric third-order component (j, k, l) in 000,001,002,011,012,022,111,112,122,222.
__device__ __forceinline__ int sym3(int j, int k, int l) {
    int a = j, b = k, c = l, t;
    if (a > b) { t = a; a = b; b = t; }
    if (b > c) { t = b; b = c; c = t; }
    if (a > b) { t = a; a = b; b = t; }
    return a == 0 ? (b == 0 ? c : (b == 1 ? 2 + c : 5)) : (a == 1 ? (b == 1 ? 5 + c : 8) : 9);
}

// Index of the symmetric fourth-order component (j, k, l, m) in 0000,0001,0002,0011,0012,0022,0111,0112,0122,0222,
// 1111,1112,1122,1222,2222: the base-3 code of the sorted indices through a table (-1: not sorted).
__constant__ signed char c_sym4[81] = {
    0,  1,  2,  -1, 3,  4,  -1, -1, 5,  -1, -1, -1, -1, 6,  7,  -1, -1, 8,  -1, -1, -1, -1, -1, -1, -1, -1, 9,
    -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, 10, 11, -1, -1, 12, -1, -1, -1, -1, -1, -1, -1, -1, 13,
    -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, 14};
__device__ __forceinline__ int sym4(int j, int k, int l, int m) {
    int t;
    if (j > k) { t = j; j = k; k = t; }
    if (l > m) { t = l; l = m; m = t; }
    if (j > l) { t = j; j = l; l = t; }
    if (k > m) { t = k; k = m; m = t; }
    if (k > l) { t = k; k = l; l = t; }
    return c_sym4[27 * j + 9 * k + 3 * l + m];
}

// The symmetric index pairs (m2, T4) and triples (m3, W4) in storage order.
__constant__ signed char c_kl[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
__constant__ signed char c_jkl[10][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 1, 1}, {0, 1, 2},
                                         {0, 2, 2}, {1, 1, 1}, {1, 1, 2}, {1, 2, 2}, {2, 2, 2}};

// The traversal record of node j with bounding radius b.
__device__ __forceinline__ NodeRec node_record(int64_t j, double b, const double *centre, const double *core,
                                               const int64_t *lo, const int64_t *hi, const int64_t *left,
                                               const int64_t *right) {
    NodeRec r;
    r.cx = centre[3 * j]; r.cy = centre[3 * j + 1]; r.cz = centre[3 * j + 2];
    r.bound = b;
    r.clear_core = core[j];
    r.lo = (int)lo[j]; r.hi = (int)hi[j]; r.left = (int)left[j]; r.right = (int)right[j];
    r.pad = 0.0;
    return r;
}

// The outputs of the moment pipelines for one node.
struct NodeOut {
    const int64_t *lo, *hi, *left, *right;
    const double *centre, *core;
    double *bound, *m0, *m1, *m2, *w1, *t2, *w2;
    NodeRec *nodes;
    Far64 *far64;
    Far32 *far32;
    Far64x *far64x;
    Far32x *far32x;
    Far64y *far64y;
    Far32y *far32y;
    Far64z *far64z;
    Far32z *far32z;
};

// A record's n values (n even; 16-byte aligned destinations) in FP64 and FP32: 16-byte stores, so that a thread
// writing one node's records issues a quarter to a half of the scalar stores.
__device__ __forceinline__ void store_pair(double *d64, float *d32, const double *v, int n) {
    for (int q = 0; q < n; q += 2) reinterpret_cast<double2 *>(d64)[q / 2] = make_double2(v[q], v[q + 1]);
    int q = 0;
    for (; q + 4 <= n; q += 4)
        reinterpret_cast<float4 *>(d32)[q / 4] = make_float4((float)v[q], (float)v[q + 1], (float)v[q + 2], (float)v[q + 3]);
    for (; q < n; ++q) d32[q] = (float)v[q];
}

// Node j from its sums v (bound^2, m0, m1, symmetric m2 [, symmetric m3 [, symmetric m4 [, symmetric m5]]]) about
// its centre: the export arrays, the contractions and the packed far records, and with RECORDS the bounding radius and
// the traversal record (the bottom-up pipeline writes those two earlier, in node_rec_kernel, and leaves v[0] unused).
// PART -1 does all of it; PART 0 the records of orders 0-3 (and the export arrays and traversal record), PART 1-3 the
// order-4 and order-5 rows of component PART - 1, so that four threads can share a node.
template <int PARTS, bool RECORDS = true, int PART = -1>
__device__ void finalize_node(int64_t j, const double *__restrict__ v, const NodeOut &o) {
    double *bound = o.bound, *m0 = o.m0, *m1 = o.m1, *m2 = o.m2, *w1 = o.w1, *t2 = o.t2, *w2 = o.w2;
    Far64 *far64 = o.far64;
    Far32 *far32 = o.far32;
    Far64x *far64x = o.far64x;
    Far32x *far32x = o.far32x;
    if (PART <= 0) {
    const double b = sqrt(v[0]) * (1.0 + 1e-12);
    if (RECORDS) bound[j] = b;
    const double *M0 = v + 1, *M1 = v + 4, *S = v + 13;  // S[6 i + p], p over (00,01,02,11,12,22)
    auto M2 = [&](int i, int a, int c) -> double {
        int lo_ = a < c ? a : c, hi_ = a < c ? c : a;
        int p = lo_ == 0 ? hi_ : (lo_ == 1 ? 2 + hi_ : 5);
        return S[6 * i + p];
    };
    for (int i = 0; i < 3; ++i) {
        m0[3 * j + i] = M0[i];
        for (int a = 0; a < 3; ++a) {
            m1[9 * j + 3 * i + a] = M1[3 * i + a];
            for (int c = 0; c < 3; ++c) m2[27 * j + 9 * i + 3 * a + c] = M2(i, a, c);
        }
    }
    double W1[3] = {M1[5] - M1[7], M1[6] - M1[2], M1[1] - M1[3]};
    double T2[3], W2[9];
    for (int i = 0; i < 3; ++i) T2[i] = M2(i, 0, 0) + M2(i, 1, 1) + M2(i, 2, 2);
    for (int k = 0; k < 3; ++k) {
        W2[0 + k] = M2(1, 2, k) - M2(2, 1, k);
        W2[3 + k] = M2(2, 0, k) - M2(0, 2, k);
        W2[6 + k] = M2(0, 1, k) - M2(1, 0, k);
    }
    for (int i = 0; i < 3; ++i) { w1[3 * j + i] = W1[i]; t2[3 * j + i] = T2[i]; }
    for (int q = 0; q < 9; ++q) w2[9 * j + q] = W2[q];
    double f[BS_FAR_N];
    for (int i = 0; i < 3; ++i) f[F_M0 + i] = M0[i];
    for (int q = 0; q < 9; ++q) f[F_M1 + q] = M1[q];
    for (int i = 0; i < 3; ++i) { f[F_W1 + i] = W1[i]; f[F_T2 + i] = T2[i]; }
    for (int q = 0; q < 9; ++q) f[F_W2 + q] = W2[q];
    for (int q = 0; q < 18; ++q) f[F_M2 + q] = S[q];
    {
        double fp[BS_FAR_N + 3];  // the records' padding as zeros (Far64: 46 doubles, Far32: 48 floats)
        for (int q = 0; q < BS_FAR_N + 3; ++q) fp[q] = q < BS_FAR_N ? f[q] : 0.0;
        for (int q = 0; q < BS_FAR_N + 1; q += 2)
            reinterpret_cast<double2 *>(far64[j].v)[q / 2] = make_double2(fp[q], fp[q + 1]);
        for (int q = 0; q < BS_FAR_N + 3; q += 4)
            reinterpret_cast<float4 *>(far32[j].v)[q / 4] =
                make_float4((float)fp[q], (float)fp[q + 1], (float)fp[q + 2], (float)fp[q + 3]);
    }
    if (PARTS >= MOM_PARTS3) {
        const double *M3 = v + 31;  // M3[10 b + sym3(j, k, l)]
        double g[BS_FAR3_N], T3[9];
        for (int q = 0; q < 30; ++q) g[G_M3 + q] = M3[q];
        for (int b3 = 0; b3 < 3; ++b3)
            for (int l3 = 0; l3 < 3; ++l3)
                T3[3 * b3 + l3] = M3[10 * b3 + sym3(0, 0, l3)] + M3[10 * b3 + sym3(1, 1, l3)] +
                                  M3[10 * b3 + sym3(2, 2, l3)];
        for (int q = 0; q < 9; ++q) g[G_T3 + q] = T3[q];
        const int kl[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
        for (int p = 0; p < 6; ++p) {
            const int k3 = kl[p][0], l3 = kl[p][1];
            g[G_W3 + 0 * 6 + p] = M3[10 * 1 + sym3(2, k3, l3)] - M3[10 * 2 + sym3(1, k3, l3)];
            g[G_W3 + 1 * 6 + p] = M3[10 * 2 + sym3(0, k3, l3)] - M3[10 * 0 + sym3(2, k3, l3)];
            g[G_W3 + 2 * 6 + p] = M3[10 * 0 + sym3(1, k3, l3)] - M3[10 * 1 + sym3(0, k3, l3)];
        }
        g[G_W3V + 0] = T3[3 * 1 + 2] - T3[3 * 2 + 1];
        g[G_W3V + 1] = T3[3 * 2 + 0] - T3[3 * 0 + 2];
        g[G_W3V + 2] = T3[3 * 0 + 1] - T3[3 * 1 + 0];
        for (int q = 0; q < 64; q += 2)
            reinterpret_cast<double2 *>(far64x[j].v)[q / 2] =
                make_double2(q < BS_FAR3_N ? g[q] : 0.0, q + 1 < BS_FAR3_N ? g[q + 1] : 0.0);
        float h[64];
        for (int q = 0; q < 64; ++q) h[q] = 0.f;
        for (int i = 0; i < 3; ++i) {
            for (int q = 0; q < 10; ++q) h[H_ROW * i + H_M3 + q] = (float)g[G_M3 + 10 * i + q];
            for (int q = 0; q < 3; ++q) h[H_ROW * i + H_T3 + q] = (float)g[G_T3 + 3 * i + q];
            for (int q = 0; q < 6; ++q) h[H_ROW * i + H_W3 + q] = (float)g[G_W3 + 6 * i + q];
        }
        for (int q = 0; q < 3; ++q) h[H_W3V + q] = (float)g[G_W3V + q];
        for (int q = 0; q < 64; q += 4)
            reinterpret_cast<float4 *>(far32x[j].v)[q / 4] = make_float4(h[q], h[q + 1], h[q + 2], h[q + 3]);
    }
    }
    if (PARTS >= MOM_PARTS4) {
        const double *M4 = v + 61;  // M4[15 b + sym4(j, k, l, m)]
        double T4[3][6];            // T4[b][(l, m)] = M4[b][j][j][l][m]
        for (int b4 = 0; b4 < 3; ++b4)
            for (int p = 0; p < 6; ++p) {
                const int l4 = c_kl[p][0], n4 = c_kl[p][1];
                T4[b4][p] = M4[15 * b4 + sym4(0, 0, l4, n4)] + M4[15 * b4 + sym4(1, 1, l4, n4)] +
                            M4[15 * b4 + sym4(2, 2, l4, n4)];
            }
        auto t4 = [&](int b4, int c4, int n4) {
            const int x = c4 < n4 ? c4 : n4, y = c4 < n4 ? n4 : c4;
            return T4[b4][x == 0 ? y : (x == 1 ? 2 + y : 5)];
        };
        // eps_ibc X[b][c] = X[b'][c'] - X[c'][b'] with (b', c') = (1, 2), (2, 0), (0, 1) for i = 0, 1, 2
        for (int i = 0; i < 3; ++i) {
            if (PART > 0 && i != PART - 1) continue;
            const int b4 = (i + 1) % 3, c4 = (i + 2) % 3;
            double row[K_ROW];
            for (int q = 0; q < K_ROW; ++q) row[q] = 0.0;
            for (int q = 0; q < 15; ++q) row[K_M4 + q] = M4[15 * i + q];
            for (int p = 0; p < 6; ++p) row[K_T4 + p] = T4[i][p];
            row[K_TAU4] = T4[i][0] + T4[i][3] + T4[i][5];
            for (int q = 0; q < 10; ++q) {
                const int k4 = c_jkl[q][0], l4 = c_jkl[q][1], n4 = c_jkl[q][2];
                row[K_W4 + q] = M4[15 * b4 + sym4(c4, k4, l4, n4)] - M4[15 * c4 + sym4(b4, k4, l4, n4)];
            }
            for (int n4 = 0; n4 < 3; ++n4) row[K_W4T + n4] = t4(b4, c4, n4) - t4(c4, b4, n4);
            store_pair(o.far64y[j].v + K_ROW * i, o.far32y[j].v + K_ROW * i, row, K_ROW);
        }
        if (PART <= 1)
            for (int q = 3 * K_ROW; q < 112; ++q) {
                o.far64y[j].v[q] = 0.0;
                o.far32y[j].v[q] = 0.f;
            }
    }
    if (PARTS == MOM_PARTS5) {
        // symmetric tensors by index counts (c0, c1, c2): rank among the order-n tuples in storage order
        auto rank = [](int n, int c0, int c1) { return (n - c0) * (n - c0 + 1) / 2 + (n - c0 - c1); };
        const double *M5 = v + 106;  // M5[21 b + rank(5, ...)]
        auto m5 = [&](int b5, int c0, int c1) { return M5[21 * b5 + rank(5, c0, c1)]; };
        // T5[b][3-tuple] = sum_j M5[b][j j + tuple]; TT5[b][k] = sum_j T5[b][j j k]
        double T5[3][10], TT5[3][3];
        for (int b5 = 0; b5 < 3; ++b5) {
            int q = 0;
            for (int c0 = 3; c0 >= 0; --c0)
                for (int c1 = 3 - c0; c1 >= 0; --c1, ++q)
                    T5[b5][q] = m5(b5, c0 + 2, c1) + m5(b5, c0, c1 + 2) + m5(b5, c0, c1);
            for (int k = 0; k < 3; ++k) {
                const int k0 = k == 0, k1 = k == 1;
                // T5 tuple with counts (2 + k0, k1, ...), (k0, 2 + k1, ...), (k0, k1, ...) + 2 on z
                TT5[b5][k] = T5[b5][rank(3, 2 + k0, k1)] + T5[b5][rank(3, k0, 2 + k1)] + T5[b5][rank(3, k0, k1)];
            }
        }
        auto t5 = [&](int b5, int c0, int c1) { return T5[b5][rank(3, c0, c1)]; };
        for (int i = 0; i < 3; ++i) {
            if (PART > 0 && i != PART - 1) continue;
            const int b5 = (i + 1) % 3, c5 = (i + 2) % 3;  // eps_ibc X[b][c] = X[b5][c5] - X[c5][b5]
            const int e0b = c5 == 0, e1b = c5 == 1, e0c = b5 == 0, e1c = b5 == 1;  // count shifts of index c5 / b5
            double row[Z_ROW];
            for (int q = 0; q < 21; ++q) row[Z_M5 + q] = M5[21 * i + q];
            for (int q = 0; q < 10; ++q) row[Z_T5 + q] = T5[i][q];
            for (int k = 0; k < 3; ++k) row[Z_TT5 + k] = TT5[i][k];
            int q = 0;
            for (int c0 = 4; c0 >= 0; --c0)  // W5 over the 4-tuples
                for (int c1 = 4 - c0; c1 >= 0; --c1, ++q)
                    row[Z_W5 + q] = m5(b5, c0 + e0b, c1 + e1b) - m5(c5, c0 + e0c, c1 + e1c);
            q = 0;
            for (int c0 = 2; c0 >= 0; --c0)  // W5T over the 2-tuples
                for (int c1 = 2 - c0; c1 >= 0; --c1, ++q)
                    row[Z_W5T + q] = t5(b5, c0 + e0b, c1 + e1b) - t5(c5, c0 + e0c, c1 + e1c);
            row[Z_W5TT] = TT5[b5][c5] - TT5[c5][b5];
            store_pair(o.far64z[j].v + Z_ROW * i, o.far32z[j].v + Z_ROW * i, row, Z_ROW);
        }
    }
    if (PART <= 0 && RECORDS) {
        const double b = sqrt(v[0]) * (1.0 + 1e-12);
        o.nodes[j] = node_record(j, b, o.centre, o.core, o.lo, o.hi, o.left, o.right);
    }
}

// ---------------------------------------------------------------------------------------------------------------------
// Bottom-up moments (Morton trees and forests).  Leaves sum their own segments; an internal node takes its box and
// core from its children (exact) and its moments by translating the children's to its centre
//   m1_ij += m0_i D_j,  m2_ijk += m1_ij D_k + m1_ik D_j + m0_i D_j D_k,
//   m3_ijkl += D_j m2_ikl + D_k m2_ijl + D_l m2_ijk + D_j D_k m1_il + D_j D_l m1_ik + D_k D_l m1_ij + D_j D_k D_l m0_i
// and for fourth-order trees
//   m4_ijklm += the 4 D m3, 6 D D m2, 4 D D D m1 and D D D D m0 terms of the same binomial expansion
// (D = child centre - node centre; left child first, then right), which equals the direct sums up to rounding.  Boxes
// and cores are unions over the leaves (exact); the bounding radius stays exact: every leaf's endpoints against each
// of its ancestors' centres.
// ---------------------------------------------------------------------------------------------------------------------
struct __align__(16) EndPts {
    double sx, sy, sz, ex, ey, ez;
};


// up[child] = (parent, the other child), the other child stored as -(it + 1) when `child` is the right one, so that a
// climbing warp knows both children and their order from one load; a root's up[].x = -1 (up[] starts as all -1).
// The leaves are listed in leaves[0 .. *nleaves) in no particular order (each leaf's work is independent of which
// thread takes it).  Every node's box (ordered bits, for atomicMin / atomicMax) starts empty and its core at zero.
__global__ void parent_kernel(int64_t count, const int64_t *left, const int64_t *right, int2 *up, int32_t *leaves,
                              unsigned *nleaves, unsigned long long *boxbits, unsigned long long *corebits) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    for (int x = 0; x < 3; ++x) {
        boxbits[6 * j + x] = ordered_bits(INFINITY);
        boxbits[6 * j + 3 + x] = ordered_bits(-INFINITY);
    }
    corebits[j] = 0ull;
    if (left[j] >= 0) {
        up[left[j]] = make_int2((int)j, (int)right[j]);
        up[right[j]] = make_int2((int)j, -(int)left[j] - 1);
    } else {
        leaves[atomicAdd(nleaves, 1u)] = (int32_t)j;
    }
}

// The symmetric index tuples of orders 0..5 in storage order (order, then lexicographic): (), 0, 1, 2, 00, 01, ...,
// 22222 -- 1 + 3 + 6 + 10 + 15 + 21 = 56.  Moment (i; tuple of order n, rank r among the order-n tuples) is stored at
// T_BASE[n] + T_CNT[n] i + r of a node's sums (index 0 holds bound^2).  src[u][mask]: where the tuple left after
// removing the positions in `mask` from tuple u is stored (T_BASE + rank, plus T_CNT << 8).
constexpr int N_TUPLES = 56;
constexpr int T_FIRST[6] = {0, 1, 4, 10, 20, 35}, T_BASE[6] = {1, 4, 13, 31, 61, 106},
              T_CNT[6] = {1, 3, 6, 10, 15, 21};
struct TupleTables {
    unsigned char n[N_TUPLES];
    unsigned short packed[N_TUPLES];                // indices, two bits each, first index in the low bits
    unsigned char out0[N_TUPLES], cnt[N_TUPLES];    // moment (i; u) is stored at out0[u] + cnt[u] i
    unsigned short src[N_TUPLES][32];
};
constexpr TupleTables make_tuple_tables() {
    TupleTables t{};
    int u = 0;
    for (int n = 0; n <= 5; ++n) {
        int codes = 1;
        for (int k = 0; k < n; ++k) codes *= 3;
        for (int code = 0; code < codes; ++code) {  // base-3 codes, first index most significant: lexicographic
            int dig[5] = {0, 0, 0, 0, 0}, c = code;
            for (int s = n - 1; s >= 0; --s) { dig[s] = c % 3; c /= 3; }
            bool sorted = true;
            for (int s = 1; s < n; ++s) sorted = sorted && dig[s - 1] <= dig[s];
            if (!sorted) continue;
            int pk = 0;
            for (int s = 0; s < n; ++s) pk |= dig[s] << (2 * s);
            t.n[u] = (unsigned char)n;
            t.packed[u] = (unsigned short)pk;
            t.out0[u] = (unsigned char)(T_BASE[n] + u - T_FIRST[n]);
            t.cnt[u] = (unsigned char)T_CNT[n];
            ++u;
        }
    }
    for (int v = 0; v < N_TUPLES; ++v) {
        const int n = t.n[v];
        for (int mask = 0; mask < (1 << n); ++mask) {
            int rest = 0, m = 0;
            for (int s = 0; s < n; ++s)
                if (!((mask >> s) & 1)) rest |= ((t.packed[v] >> (2 * s)) & 3) << (2 * m++);
            int w = T_FIRST[m];
            while (t.n[w] != m || t.packed[w] != rest) ++w;
            t.src[v][mask] = (unsigned short)((T_BASE[m] + w - T_FIRST[m]) | (T_CNT[m] << 8));
        }
    }
    return t;
}
// in global memory, not constant: the lanes of a warp read different entries
__device__ TupleTables g_tt = make_tuple_tables();

// Translation terms by index counts.  Tuple u with counts (c0, c1, c2) of the indices 0, 1, 2 translates as
//   m'_(i; u) = sum over k <= c (componentwise) of C(c0,k0) C(c1,k1) C(c2,k2) D0^k0 D1^k1 D2^k2 m_(i; c - k),
// the subset expansion with equal subsets merged (at order 5: 252 terms instead of 672).  term[u][t], t < n[u]:
// binomial product (bits 0-3), the monomial D^k as a tuple index (bits 4-9), storage offset T_BASE + rank of c - k
// (bits 10-16) and its T_CNT (bits 17-21).  rank(n, c0, c1) is the place of counts (c0, c1, n - c0 - c1) among the
// order-n tuples in storage order.
constexpr int TERMS_MAX = 18;
constexpr int tuple_rank(int n, int c0, int c1) { return (n - c0) * (n - c0 + 1) / 2 + (n - c0 - c1); }
struct TermTables {
    unsigned char n[N_TUPLES];
    unsigned term[N_TUPLES][TERMS_MAX];
};
constexpr TermTables make_term_tables() {
    TermTables t{};
    const TupleTables tt = make_tuple_tables();
    const int binom[6][6] = {{1, 0, 0, 0, 0, 0}, {1, 1, 0, 0, 0, 0}, {1, 2, 1, 0, 0, 0},
                             {1, 3, 3, 1, 0, 0}, {1, 4, 6, 4, 1, 0}, {1, 5, 10, 10, 5, 1}};
    for (int u = 0; u < N_TUPLES; ++u) {
        int c[3] = {0, 0, 0};
        for (int s = 0; s < tt.n[u]; ++s) ++c[(tt.packed[u] >> (2 * s)) & 3];
        int q = 0;
        for (int k0 = 0; k0 <= c[0]; ++k0)
            for (int k1 = 0; k1 <= c[1]; ++k1)
                for (int k2 = 0; k2 <= c[2]; ++k2) {
                    const int coef = binom[c[0]][k0] * binom[c[1]][k1] * binom[c[2]][k2];
                    const int nk = k0 + k1 + k2, nv = tt.n[u] - nk;
                    const int mono = T_FIRST[nk] + tuple_rank(nk, k0, k1);
                    const int off = T_BASE[nv] + tuple_rank(nv, c[0] - k0, c[1] - k1);
                    t.term[u][q++] = (unsigned)coef | ((unsigned)mono << 4) | ((unsigned)off << 10) |
                                     ((unsigned)T_CNT[nv] << 17);
                }
        t.n[u] = (unsigned char)q;
    }
    return t;
}
__device__ TermTables g_terms = make_term_tables();

template <int PARTS>
struct MomentTuples {
    static constexpr int n = PARTS == MOM_PARTS ? 10 : (PARTS == MOM_PARTS3 ? 20 : (PARTS == MOM_PARTS4 ? 35 : 56));
    static constexpr int slots = (n + 31) / 32;  // tuples per lane
    static constexpr int order = PARTS == MOM_PARTS ? 2 : (PARTS == MOM_PARTS3 ? 3 : (PARTS == MOM_PARTS4 ? 4 : 5));
};

// Storage index of moment (i; tuple u).
__device__ __forceinline__ int tuple_out(int u, int i) { return g_tt.out0[u] + g_tt.cnt[u] * i; }

// The box of the leaf's segments [a, b) and their largest core radius, reduced over the warp; with ends, also the
// tree-ordered endpoints of the segments.
__device__ __forceinline__ void leaf_extent(int lane, int64_t a, int64_t b, const int32_t *order, const SegGeo *geo,
                                            double *mn, double *mx, double &c, EndPts *ends = nullptr) {
    for (int x = 0; x < 3; ++x) {
        mn[x] = INFINITY;
        mx[x] = -INFINITY;
    }
    c = 0.0;
    for (int64_t k = a + lane; k < b; k += 32) {
        const SegGeo g = geo[order ? order[k] : k];
        if (ends) ends[k] = EndPts{g.sx, g.sy, g.sz, g.ex, g.ey, g.ez};
        mn[0] = fmin(mn[0], fmin(g.sx, g.ex)); mx[0] = fmax(mx[0], fmax(g.sx, g.ex));
        mn[1] = fmin(mn[1], fmin(g.sy, g.ey)); mx[1] = fmax(mx[1], fmax(g.sy, g.ey));
        mn[2] = fmin(mn[2], fmin(g.sz, g.ez)); mx[2] = fmax(mx[2], fmax(g.sz, g.ez));
        c = fmax(c, g.radius);
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int x = 0; x < 3; ++x) {
            mn[x] = fmin(mn[x], __shfl_xor_sync(0xffffffffu, mn[x], o));
            mx[x] = fmax(mx[x], __shfl_xor_sync(0xffffffffu, mx[x], o));
        }
        c = fmax(c, __shfl_xor_sync(0xffffffffu, c, o));
    }
}

// Ancestors a leaf lists for bound_up_kernel (the nearest first, -1 after the root when fewer).
constexpr int ANC_LIST = 16;

// One warp per leaf: box, core and centre from the leaf's segments (and their tree-ordered endpoints into ends), then
// bound^2 (the largest squared distance from the centre to an endpoint) into bound2 as its bit pattern.  Seven lanes
// then fold the box's six bounds and the core into every ancestor (atomicMin / atomicMax on ordered bits: the union
// of the leaves' boxes and the largest core, the same in any order), so that no climb is needed for the boxes.
__global__ void __launch_bounds__(128) leaf_geometry_kernel(const int32_t *leaves, const unsigned *nleaves,
                                                            const int64_t *lo, const int64_t *hi,
                                                            const int32_t *order, const SegGeo *geo, const int2 *up,
                                                            EndPts *ends, unsigned long long *boxbits,
                                                            unsigned long long *corebits, double *centre,
                                                            double *core, unsigned long long *bound2,
                                                            int32_t *anc_list) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5), n = *nleaves;
    for (int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n; w += warps) {
        const int64_t j = leaves[w];
        const int64_t a = lo[j], b = hi[j];
        double mn[3], mx[3], c;
        leaf_extent(lane, a, b, order, geo, mn, mx, c, ends);
        const double c0 = 0.5 * (mn[0] + mx[0]), c1 = 0.5 * (mn[1] + mx[1]), c2 = 0.5 * (mn[2] + mx[2]);
        double r2 = 0.0;
        for (int64_t k = a + lane; k < b; k += 32) {
            const SegGeo e = geo[order ? order[k] : k];
            const double a0 = e.sx - c0, a1 = e.sy - c1, a2 = e.sz - c2;
            const double b0 = e.ex - c0, b1 = e.ey - c1, b2 = e.ez - c2;
            // the reference's ((x^2 + y^2) + z^2) without contraction, as in every bound of this file
            const double ra = __dadd_rn(__dadd_rn(__dmul_rn(a0, a0), __dmul_rn(a1, a1)), __dmul_rn(a2, a2));
            const double rb = __dadd_rn(__dadd_rn(__dmul_rn(b0, b0), __dmul_rn(b1, b1)), __dmul_rn(b2, b2));
            r2 = fmax(r2, fmax(ra, rb));
        }
        for (int o = 16; o > 0; o >>= 1) r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
        if (lane == 0) {
            centre[3 * j] = c0;
            centre[3 * j + 1] = c1;
            centre[3 * j + 2] = c2;
            core[j] = c;
            bound2[j] = (unsigned long long)__double_as_longlong(r2);
        }
        if (lane < 7) {
            const double m0 = mn[0], m1 = mn[1], m2 = mn[2], x0 = mx[0], x1 = mx[1], x2 = mx[2];
            const double bv = lane == 0 ? m0 : lane == 1 ? m1 : lane == 2 ? m2 : lane == 3 ? x0 : lane == 4 ? x1 : x2;
            const unsigned long long v = lane < 6 ? ordered_bits(bv) : (unsigned long long)__double_as_longlong(c);
            if (lane < 6) boxbits[6 * j + lane] = v;
            else corebits[j] = v;
            int depth = 0;
            for (int node = up[j].x; node >= 0 && depth < 4096; node = up[node].x, ++depth) {
                if (lane < 3) atomicMin(boxbits + 6 * (int64_t)node + lane, v);
                else if (lane < 6) atomicMax(boxbits + 6 * (int64_t)node + lane, v);
                else atomicMax(corebits + node, v);
                if (lane == 6 && depth < ANC_LIST) anc_list[(int64_t)ANC_LIST * w + depth] = node;
            }
            if (lane == 6 && depth < ANC_LIST) anc_list[(int64_t)ANC_LIST * w + depth] = -1;
        }
    }
}

// <rho_a1 .. rho_an> over one segment for the index tuples u < NT in storage order, rho = d + t l with t uniform on
// [-1/2, 1/2] (<t^2> = 1/12, <t^4> = 1/80, odd moments 0): m2 takes d d + l l / 12, m3 d d d + (d l l + l d l +
// l l d) / 12, m4 d d d d + (the six placements of two l's) / 12 + l l l l / 80.  The order-5 means (NT = 56) come
// from the three-point Gauss-Legendre rule on [-1/2, 1/2] (nodes 0 and +-sqrt(3/5)/2, weights 8/18 and 5/18), exact
// for polynomials in t of degree 5: sum over the nodes of weight times the degree-5 monomials of rho.
template <int NT>
__device__ __forceinline__ void segment_means(const double *d, const double *l, double *g) {
    double dd[3][3], ll[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b) {
            dd[a][b] = dd[b][a] = d[a] * d[b];
            ll[a][b] = ll[b][a] = l[a] * l[b];
        }
    g[0] = 1.0;
    g[1] = d[0]; g[2] = d[1]; g[3] = d[2];
    int u = 4;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b) g[u++] = fma(ll[a][b], 1.0 / 12.0, dd[a][b]);
    if (NT > 10) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = a; b < 3; ++b)
#pragma unroll
                for (int c = b; c < 3; ++c)
                    g[u++] = d[a] * dd[b][c] + (d[a] * ll[b][c] + l[a] * (d[b] * l[c] + l[b] * d[c])) * (1.0 / 12.0);
    }
    if (NT > 20) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = a; b < 3; ++b)
#pragma unroll
                for (int c = b; c < 3; ++c)
#pragma unroll
                    for (int e = c; e < 3; ++e) {
                        const double pairs = ll[a][b] * dd[c][e] + ll[a][c] * dd[b][e] + ll[a][e] * dd[b][c] +
                                             ll[b][c] * dd[a][e] + ll[b][e] * dd[a][c] + ll[c][e] * dd[a][b];
                        g[u++] = dd[a][b] * dd[c][e] + pairs * (1.0 / 12.0) + ll[a][b] * ll[c][e] * (1.0 / 80.0);
                    }
    }
    if (NT > 35) {
        constexpr double tg = 0.3872983346207417;  // sqrt(3/5) / 2
        const double wt[3] = {8.0 / 18.0, 5.0 / 18.0, 5.0 / 18.0}, tt[3] = {0.0, tg, -tg};
        double m5[21];
#pragma unroll
        for (int q = 0; q < 21; ++q) m5[q] = 0.0;
#pragma unroll
        for (int gp = 0; gp < 3; ++gp) {
            const double r0 = fma(tt[gp], l[0], d[0]), r1 = fma(tt[gp], l[1], d[1]), r2 = fma(tt[gp], l[2], d[2]);
            const double x2 = r0 * r0, xy = r0 * r1, xz = r0 * r2, y2 = r1 * r1, yz = r1 * r2, z2 = r2 * r2;
            const double c3[10] = {x2 * r0, x2 * r1, x2 * r2, xy * r1, xy * r2, xz * r2, y2 * r1, y2 * r2, yz * r2,
                                   z2 * r2};
            // lexicographic degree-5 tuples: (c0, c1, c2) = (5,0,0), (4,1,0), ..., (0,0,5) as x^c0 y^c1 z^c2
            const double v[21] = {x2 * c3[0], x2 * c3[1], x2 * c3[2], x2 * c3[3], x2 * c3[4], x2 * c3[5], x2 * c3[6],
                                  x2 * c3[7], x2 * c3[8], x2 * c3[9], xy * c3[6], xy * c3[7], xy * c3[8], xy * c3[9],
                                  xz * c3[9], y2 * c3[6], y2 * c3[7], y2 * c3[8], y2 * c3[9], yz * c3[9], z2 * c3[9]};
#pragma unroll
            for (int q = 0; q < 21; ++q) m5[q] = fma(wt[gp], v[q], m5[q]);
        }
#pragma unroll
        for (int q = 0; q < 21; ++q) g[u++] = m5[q];
    }
}

// Segment k's half of its clear-leaf pair record (Seg32c2): start s relative to its leaf's centre o, negated;
// Gamma/(4 pi); l = L d and -l; 1/(L rc)^2 from l2 = |l|^2 (+inf without a core).
__device__ __forceinline__ void clear_half(Seg32c2 *out, int64_t k, double ox, double oy, double oz, double sx,
                                           double sy, double sz, double lx, double ly, double lz, double l2,
                                           double g4pi, double radius) {
    float v[12];
    v[0] = (float)(ox - sx);
    v[1] = (float)(oy - sy);
    v[2] = (float)(oz - sz);
    v[3] = (float)g4pi;
    v[4] = (float)lx;
    v[5] = (float)ly;
    v[6] = (float)lz;
    v[7] = radius > 0.0 ? (float)(1.0 / (l2 * radius * radius)) : __int_as_float(0x7f800000);
    v[8] = -v[4];
    v[9] = -v[5];
    v[10] = -v[6];
    v[11] = 0.0f;
    float *half = reinterpret_cast<float *>(out + (k >> 1)) + (k & 1);
#pragma unroll
    for (int f = 0; f < 12; ++f) half[2 * f] = v[f];
}

// Warps per block of leaf_moments_kernel (its staging takes (tuples + 3) x 33 doubles a warp).
template <int PARTS>
constexpr int leaf_warps() { return PARTS == MOM_PARTS5 ? 2 : 4; }

// One warp per leaf: the moments about the leaf's centre; sums[j][PARTS] (sums[j][0] unused).  The warp takes 32
// segments at a time: each lane forms its segment's means (segment_means) and alpha = gamma l into shared memory,
// then lane u sums, over the 32, alpha_i times the mean of index tuple u (and of u + 32) for i = 0..2.  With `clear`
// each lane also writes its segment's clear-leaf pair record, relative to the same centre.
template <int PARTS>
__global__ void __launch_bounds__(32 * leaf_warps<PARTS>()) leaf_moments_kernel(const int32_t *leaves,
                                                                              const unsigned *nleaves,
                                                                              const int64_t *lo, const int64_t *hi,
                                                                              const int32_t *order, const SegGeo *geo,
                                                                              const double *centre, double *sums,
                                                                              Seg32c2 *clear) {
    using MT = MomentTuples<PARTS>;
    constexpr int ROWS = MT::n + 3, STRIDE = 33;  // means, then alpha; padded rows: lanes of a column hit other banks
    constexpr int LW = leaf_warps<PARTS>();
    __shared__ double st[LW][ROWS * STRIDE];
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) % LW;
    double *sw = st[w];
    bool own[MT::slots];
#pragma unroll
    for (int r = 0; r < MT::slots; ++r) own[r] = lane + 32 * r < MT::n;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5), n = *nleaves;
    for (int64_t x = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); x < n; x += warps) {
        const int64_t j = leaves[x];
        const int64_t a = lo[j], b = hi[j];
        const double c0 = centre[3 * j], c1 = centre[3 * j + 1], c2 = centre[3 * j + 2];
        double acc[MT::slots][3];
#pragma unroll
        for (int r = 0; r < MT::slots; ++r) acc[r][0] = acc[r][1] = acc[r][2] = 0.0;
        // the next stage's record is loaded while this stage computes
        SegGeo next;
        if (a + lane < b) next = geo[order ? order[a + lane] : a + lane];
        for (int64_t base = a; base < b; base += 32) {
            const int64_t k = base + lane;
            const SegGeo e = next;
            if (k + 32 < b) next = geo[order ? order[k + 32] : k + 32];
            double g[MT::n], al[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < MT::n; ++q) g[q] = 0.0;
            if (k < b) {
                if (clear)
                    clear_half(clear, k, c0, c1, c2, e.sx, e.sy, e.sz, e.lx, e.ly, e.lz,
                               e.lx * e.lx + e.ly * e.ly + e.lz * e.lz, e.gamma * INV_FOUR_PI, e.radius);
                if (e.gamma != 0.0) {  // a segment without circulation adds nothing (and no non-finite geometry)
                    const double d[3] = {0.5 * (e.sx + e.ex) - c0, 0.5 * (e.sy + e.ey) - c1, 0.5 * (e.sz + e.ez) - c2};
                    const double l[3] = {e.lx, e.ly, e.lz};
                    segment_means<MT::n>(d, l, g);
                    al[0] = e.gamma * e.lx; al[1] = e.gamma * e.ly; al[2] = e.gamma * e.lz;
                }
            }
#pragma unroll
            for (int q = 0; q < MT::n; ++q) sw[q * STRIDE + lane] = g[q];
#pragma unroll
            for (int i = 0; i < 3; ++i) sw[(MT::n + i) * STRIDE + lane] = al[i];
            __syncwarp();
#pragma unroll 4
            for (int s2 = 0; s2 < 32; ++s2) {
                const double x0 = sw[MT::n * STRIDE + s2], x1 = sw[(MT::n + 1) * STRIDE + s2],
                             x2 = sw[(MT::n + 2) * STRIDE + s2];
#pragma unroll
                for (int r = 0; r < MT::slots; ++r) {
                    if (!own[r]) continue;
                    const double m = sw[(lane + 32 * r) * STRIDE + s2];
                    acc[r][0] = fma(x0, m, acc[r][0]);
                    acc[r][1] = fma(x1, m, acc[r][1]);
                    acc[r][2] = fma(x2, m, acc[r][2]);
                }
            }
            __syncwarp();
        }
        double *out = sums + (int64_t)PARTS * j;
#pragma unroll
        for (int r = 0; r < MT::slots; ++r)
            if (own[r])
                for (int i = 0; i < 3; ++i) out[tuple_out(lane + 32 * r, i)] = acc[r][i];
    }
}


// The moments of the internal nodes: one warp per leaf climbs towards the root; at each parent the second of the
// two arriving warps combines the children (their results were published, and fenced, before the arrival count
// moved), so every internal node is combined exactly once and no warp waits for another (centres known): both
// children's sums are staged in shared memory; lane u translates index tuple u over its distinct sub-tuples with
// binomial weights (g_terms), D = child centre - node centre; left child first, then right.
template <int PARTS>
__global__ void __launch_bounds__(128, 6) bottom_up_kernel(const int32_t *leaves, const unsigned *nleaves,
                                                        const int2 *up, unsigned *arrive, const double *centre,
                                                        double *sums) {
    using MT = MomentTuples<PARTS>;
    // lane's tuple in each slot, so that slot 1 runs few terms: fourth-order trees put the first order-1 tuple and the
    // 31 of orders 2-4 in slot 0 (at most 12 terms), the order-0 tuple and the other two of order 1 in slot 1 (2);
    // fifth-order trees the 21 tuples of order 5 and the last 11 of order 4 in slot 0 (18), the other 24 in slot 1 (9)
    constexpr int T0 = MT::n == 56 ? 18 : (MT::n == 35 ? 12 : (MT::n == 20 ? 8 : 4));  // terms a slot runs
    constexpr int T1 = MT::n == 56 ? 9 : 2;
    __shared__ double sm[4][2][PARTS];
    __shared__ double mono[4][2][MT::n];        // D^k per warp and side, by tuple index
    __shared__ unsigned term[2][T0 > T1 ? T0 : T1][32];  // by slot, term, lane: a warp reads adjacent words
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) & 3;
    int tu[MT::slots], tp[MT::slots];
    bool tok[MT::slots];
#pragma unroll
    for (int r = 0; r < MT::slots; ++r) {
        int u = lane;
        bool ok = u < MT::n;
        if (MT::n == 35) {
            u = r == 0 ? (lane == 0 ? 1 : lane + 3) : (lane == 0 ? 0 : lane + 1);
            ok = r == 0 || lane < 3;
        } else if (MT::n == 56) {
            u = r == 0 ? (lane < 21 ? 35 + lane : lane + 3) : lane;
            ok = r == 0 || lane < 24;
        }
        tu[r] = u;
        tok[r] = ok;
        tp[r] = ok ? g_tt.packed[u] : 0;
    }
    // the term table in the slot layout; unused places add zero (coefficient 0, offset 1)
    if (w == 0) {
#pragma unroll
        for (int r = 0; r < MT::slots; ++r) {
            const int tmax = r == 0 ? T0 : T1;
            for (int q = 0; q < tmax; ++q)
                term[r][q][lane] = (tok[r] && q < g_terms.n[tu[r]]) ? g_terms.term[tu[r]][q] : (1u << 10);
        }
    }
    __syncthreads();
    // lane's monomials of D: tuples lane and lane + 32, by their packed indices
    int mn_[2], mp_[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int u = lane + 32 * r;
        mn_[r] = u < MT::n ? g_tt.n[u] : -1;
        mp_[r] = u < MT::n ? g_tt.packed[u] : 0;
    }
    // a grid that stays resident, so that every leaf's climb starts at once (more leaves than resident warps: a warp
    // takes them one after another)
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5), n = *nleaves;
    for (int64_t x = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); x < n; x += warps) {
    int64_t node = leaves[x];
    for (int depth = 0; depth < 4096; ++depth) {
        const int2 pu = up[node];
        const int32_t p = pu.x;
        if (p < 0) break;
        __threadfence();
        __syncwarp();
        unsigned prior = 0;
        if (lane == 0) prior = atomicAdd(&arrive[p], 1u);
        prior = __shfl_sync(0xffffffffu, prior, 0);
        if (prior == 0) break;
        __threadfence();
        const int64_t l = pu.y >= 0 ? node : -(int64_t)pu.y - 1, r = pu.y >= 0 ? (int64_t)pu.y : node;
        // every load first (one round trip), then the stores to shared memory
        constexpr int PER = (PARTS + 31) / 32;
        double vl[PER], vr[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int q = lane + 32 * k;
            vl[k] = q < PARTS ? __ldcg(sums + (int64_t)PARTS * l + q) : 0.0;
            vr[k] = q < PARTS ? __ldcg(sums + (int64_t)PARTS * r + q) : 0.0;
        }
        double D[2][3];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            const double cx = centre[3 * (int64_t)p + x];
            D[0][x] = centre[3 * l + x] - cx;
            D[1][x] = centre[3 * r + x] - cx;
        }
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int q = lane + 32 * k;
            if (q < PARTS) {
                sm[w][0][q] = vl[k];
                sm[w][1][q] = vr[k];
            }
        }
        __syncwarp();
        // D^k for every tuple k of order <= the tree's, both sides
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            if (mn_[r] < 0) continue;
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                double f = 1.0;
#pragma unroll
                for (int s2 = 0; s2 < MT::order; ++s2) {
                    const int xi = (mp_[r] >> (2 * s2)) & 3;
                    const double dx = xi == 0 ? D[side][0] : (xi == 1 ? D[side][1] : D[side][2]);
                    f = s2 < mn_[r] ? f * dx : f;
                }
                mono[w][side][lane + 32 * r] = f;
            }
        }
        __syncwarp();
        double acc[MT::slots][3];
#pragma unroll
        for (int q = 0; q < MT::slots; ++q) {
            acc[q][0] = acc[q][1] = acc[q][2] = 0.0;
            if (!tok[q]) continue;
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const double *sv = sm[w][side], *mo = mono[w][side];
#pragma unroll 3
                for (int t = 0; t < (q == 0 ? T0 : T1); ++t) {
                    const unsigned e = term[q][t][lane];
                    const double f = (double)(e & 15u) * mo[(e >> 4) & 63u];
                    const int o0 = (int)((e >> 10) & 127u), cn = (int)(e >> 17);
                    acc[q][0] = fma(f, sv[o0], acc[q][0]);
                    acc[q][1] = fma(f, sv[o0 + cn], acc[q][1]);
                    acc[q][2] = fma(f, sv[o0 + 2 * cn], acc[q][2]);
                }
            }
        }
        __syncwarp();
        double *out = sums + (int64_t)PARTS * p;
#pragma unroll
        for (int q = 0; q < MT::slots; ++q)
            if (tok[q])
                for (int i = 0; i < 3; ++i) out[tuple_out(tu[q], i)] = acc[q][i];
        node = p;
    }
    }
}

// Bound^2 of every internal node, exactly: one warp per leaf folds the largest squared distance from each of the
// leaf's ancestors' centres (the midpoints of their boxes) to the leaf's tree-ordered endpoints into that ancestor's
// bound2 with an integer atomicMax (non-negative doubles order like their bit patterns: the same value in any order).
// The ancestors go eight at a time, their centres in registers, so that the leaf's endpoints are read once a group;
// the first ANC_LIST come from the leaf pass's list (no chain of dependent loads), deeper ones from up[].
constexpr int BOUND_GROUP = 8;
__global__ void __launch_bounds__(128) bound_up_kernel(const int32_t *leaves, const unsigned *nleaves,
                                                       const int64_t *lo, const int64_t *hi, const int2 *up,
                                                       const EndPts *ends, const double *centre,
                                                       const int32_t *anc_list, unsigned long long *bound2) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5), n = *nleaves;
    for (int64_t x = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); x < n; x += warps) {
        const int64_t j = leaves[x], a = lo[j], b = hi[j];
        if (b <= a) continue;
        const int32_t *al = anc_list + (int64_t)ANC_LIST * x;
        int next = -1;
        bool done = false;
        for (int depth0 = 0; !done && depth0 < 4096; depth0 += BOUND_GROUP) {
            int anc[BOUND_GROUP];
            double c[BOUND_GROUP][3], r2[BOUND_GROUP];
#pragma unroll
            for (int g = 0; g < BOUND_GROUP; ++g) {
                const int d = depth0 + g;
                int nd = -1;
                if (!done) {
                    nd = d < ANC_LIST ? al[d] : next;
                    if (nd < 0) done = true;
                    else if (d >= ANC_LIST - 1) next = up[nd].x;
                }
                anc[g] = nd;
                r2[g] = 0.0;
                const int64_t q = nd >= 0 ? nd : 0;
                c[g][0] = centre[3 * q];
                c[g][1] = centre[3 * q + 1];
                c[g][2] = centre[3 * q + 2];
            }
            for (int64_t k = a + lane; k < b; k += 32) {
                const EndPts e = ends[k];
#pragma unroll
                for (int g = 0; g < BOUND_GROUP; ++g) {
                    const double a0 = e.sx - c[g][0], a1 = e.sy - c[g][1], a2 = e.sz - c[g][2];
                    const double b0 = e.ex - c[g][0], b1 = e.ey - c[g][1], b2 = e.ez - c[g][2];
                    // the reference's ((x^2 + y^2) + z^2) without contraction, as in every bound of this file
                    const double ra = __dadd_rn(__dadd_rn(__dmul_rn(a0, a0), __dmul_rn(a1, a1)), __dmul_rn(a2, a2));
                    const double rb = __dadd_rn(__dadd_rn(__dmul_rn(b0, b0), __dmul_rn(b1, b1)), __dmul_rn(b2, b2));
                    r2[g] = fmax(r2[g], fmax(ra, rb));
                }
            }
#pragma unroll
            for (int g = 0; g < BOUND_GROUP; ++g) {
                for (int o = 16; o > 0; o >>= 1) r2[g] = fmax(r2[g], __shfl_xor_sync(0xffffffffu, r2[g], o));
                if (lane == 0 && anc[g] >= 0)
                    atomicMax(bound2 + anc[g], (unsigned long long)__double_as_longlong(r2[g]));
            }
        }
    }
}

// The centre (box midpoint) and core of every internal node, from the boxes and cores the leaves folded in.
__global__ void node_centre_kernel(int64_t count, const int64_t *left, const unsigned long long *boxbits,
                                   const unsigned long long *corebits, double *centre, double *core) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count || left[j] < 0) return;
    for (int x = 0; x < 3; ++x)
        centre[3 * j + x] = 0.5 * (from_ordered(boxbits[6 * j + x]) + from_ordered(boxbits[6 * j + 3 + x]));
    core[j] = __longlong_as_double((long long)corebits[j]);
}

// The bounding radius (bound^2 from leaf_geometry_kernel or bound_up_kernel) and the traversal record of every node:
// all that the walk reads.
__global__ void node_rec_kernel(int64_t count, const unsigned long long *bound2, const double *centre,
                                const double *core, const int64_t *lo, const int64_t *hi, const int64_t *left,
                                const int64_t *right, double *bound, NodeRec *nodes) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const double b = sqrt(__longlong_as_double((long long)bound2[j])) * (1.0 + 1e-12);
    bound[j] = b;
    nodes[j] = node_record(j, b, centre, core, lo, hi, left, right);
}

// Every node's export arrays and far records from its sums (read in place); for fourth- and fifth-order trees
// blockIdx.y picks the part (0: orders 0-3, 1-3: the order-4 and order-5 rows of one component).
template <int PARTS>
__global__ void node_final_kernel(int64_t count, const double *sums, NodeOut o) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const double *v = sums + (int64_t)PARTS * j;
    if (PARTS < MOM_PARTS4) {
        finalize_node<PARTS, false, -1>(j, v, o);
        return;
    }
    switch (blockIdx.y) {
        case 0: finalize_node<PARTS, false, 0>(j, v, o); break;
        case 1: finalize_node<PARTS, false, 1>(j, v, o); break;
        case 2: finalize_node<PARTS, false, 2>(j, v, o); break;
        default: finalize_node<PARTS, false, 3>(j, v, o); break;
    }
}

// Bottom-up pipeline in two phases.  Geometry, on s: leaf boxes, centres, cores and bounds, each leaf folding its box
// and core into its ancestors, the internal centres and cores, then (after the moment phase is queued) the internal
// nodes' exact bounds (every leaf's endpoints against its ancestors' centres) and the traversal records.  Moments, on
// `side` when given (once s has the centres, beside the bounds and records; t->moments_done marks their end) or else
// on s: leaf sums, the internal nodes' translated sums, the far records.  What the moment
// phase reads lives with the tree when it runs on the side stream (freed with the tree, after the evaluation that
// waited for it), else in scratch.
template <int PARTS>
static int moments_bottom_up(bs_tree *t, const SegGeo *geo, Scratch &scratch, cudaStream_t s, cudaStream_t side) {
    const int64_t count = t->count, m = t->m;
    const bool defer = side != nullptr;
    unsigned long long *boxbits = scratch.get<unsigned long long>(7 * count);  // six bounds a node, then the cores
    EndPts *ends = scratch.get<EndPts>(m);
    unsigned long long *bound2 = scratch.get<unsigned long long>(count);
    int32_t *anc_list = scratch.get<int32_t>((size_t)ANC_LIST * count);
    if (!boxbits || !ends || !bound2 || !anc_list) return scratch.status;
    unsigned long long *corebits = boxbits + 6 * count;
    double *sums = defer ? t->alloc<double>((size_t)PARTS * count, s) : scratch.get<double>((size_t)PARTS * count);
    int2 *parent = defer ? t->alloc<int2>(count, s) : scratch.get<int2>(count);
    unsigned *arrive_m = defer ? t->alloc<unsigned>(count + 1, s) : scratch.get<unsigned>(count + 1);
    int32_t *leaves = defer ? t->alloc<int32_t>(count, s) : scratch.get<int32_t>(count);
    if (!sums || !parent || !arrive_m || !leaves) return defer ? BS_ERR_OOM : scratch.status;
    unsigned *nleaves = arrive_m + count;
    BS_CUDA(cudaMemsetAsync(arrive_m, 0, (count + 1) * sizeof(unsigned), s));
    BS_CUDA(cudaMemsetAsync(bound2, 0, count * sizeof(unsigned long long), s));
    BS_CUDA(cudaMemsetAsync(parent, 0xff, count * sizeof(int2), s));
    parent_kernel<<<blocks_for(count, 256), 256, 0, s>>>(count, t->left, t->right, parent, leaves, nleaves, boxbits,
                                                         corebits);
    const int32_t *geo_order = t->geo_sorted ? nullptr : t->order32;  // geo in input order: read through the order
    int sms = 0;
    BS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, t->device));
    const unsigned leaf_blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((count + 3) / 4, (int64_t)sms * 16));
    leaf_geometry_kernel<<<leaf_blocks, 128, 0, s>>>(leaves, nleaves, t->lo, t->hi, geo_order, geo, parent, ends,
                                                      boxbits, corebits, t->centre, t->core, bound2, anc_list);
    node_centre_kernel<<<blocks_for(count, 256), 256, 0, s>>>(count, t->left, boxbits, corebits, t->centre, t->core);
    BS_CHECK_LAUNCH("node geometry");
    // the moments need the centres only: they start here, beside the exact bounds and the node records
    cudaStream_t ms = s;
    if (defer) {
        cudaEvent_t centres;
        BS_CUDA(cudaEventCreateWithFlags(&centres, cudaEventDisableTiming));
        cudaEventRecord(centres, s);
        cudaStreamWaitEvent(side, centres, 0);
        cudaEventDestroy(centres);
        ms = side;
    }
    constexpr int LW = leaf_warps<PARTS>();
    // resident blocks a SM (one wave takes as many leaves as fit), asked once: a property of the compiled kernel
    static const int leaf_resident = [] {
        int r = 0;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, leaf_moments_kernel<PARTS>, 32 * LW, 0) ==
                       cudaSuccess ? r : 1;
    }();
    const unsigned moment_blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((count + LW - 1) / LW, (int64_t)std::max(1, leaf_resident) * sms));
    leaf_moments_kernel<PARTS><<<moment_blocks, 32 * LW, 0, ms>>>(leaves, nleaves, t->lo, t->hi, geo_order, geo,
                                                                  t->centre, sums, t->seg64 ? t->seg32c2 : nullptr);
    if (defer && cudaEventCreateWithFlags(&t->marks[3], cudaEventDisableTiming) == cudaSuccess)
        cudaEventRecord(t->marks[3], ms);  // the records the near-leaf kernel reads are complete
    static const int climb_blocks = [] {  // resident blocks: one wave holds every climbing warp
        int r = 0;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, bottom_up_kernel<PARTS>, 128, 0) == cudaSuccess ? r
                                                                                                        : 1;
    }();
    const unsigned climb_grid = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(blocks_for(count, 4), (int64_t)std::max(1, climb_blocks) * sms));
    bottom_up_kernel<PARTS><<<climb_grid, 128, 0, ms>>>(leaves, nleaves, parent, arrive_m, t->centre, sums);
    const NodeOut out{t->lo, t->hi, t->left, t->right, t->centre, t->core, t->bound, t->m0, t->m1, t->m2,
                      t->w1, t->t2, t->w2, t->nodes, t->far64, t->far32, t->far64x, t->far32x,
                      t->far64y, t->far32y, t->far64z, t->far32z};
    // one warp per block: the thread per node is long, so the nodes spread over every SM
    node_final_kernel<PARTS><<<dim3(blocks_for(count, 32), PARTS >= MOM_PARTS4 ? 4 : 1), 32, 0, ms>>>(count, sums, out);
    BS_CHECK_LAUNCH("bottom-up moments");
    bound_up_kernel<<<leaf_blocks, 128, 0, s>>>(leaves, nleaves, t->lo, t->hi, parent, ends, t->centre, anc_list,
                                                 bound2);
    node_rec_kernel<<<blocks_for(count, 256), 256, 0, s>>>(count, bound2, t->centre, t->core, t->lo, t->hi, t->left,
                                                            t->right, t->bound, t->nodes);
    BS_CHECK_LAUNCH("node records");
    return BS_OK;
}

// The next n elements of T in a carved block (256-byte aligned pieces); with base null only the size is counted.
template <class T>
static T *carve(char *base, size_t &off, size_t n) {
    T *p = base ? reinterpret_cast<T *>(base + off) : nullptr;
    off += ((n ? n : 1) * sizeof(T) + 255) / 256 * 256;
    return p;
}

int compute_moments(bs_tree *t, const SegGeo *geo, Scratch &scratch, cudaStream_t s, cudaStream_t side) {
    const size_t count = (size_t)t->count;
    // every per-node array of the tree in one pool allocation (the host enqueues no allocation per array while the
    // device waits for the node count's consumers): one pass to size the block, one to hand out its pieces
    char *base = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        size_t off = 0;
        t->centre = carve<double>(base, off, 3 * count);
        t->bound = carve<double>(base, off, count);
        t->core = carve<double>(base, off, count);
        t->m0 = carve<double>(base, off, 3 * count);
        t->m1 = carve<double>(base, off, 9 * count);
        t->m2 = carve<double>(base, off, 27 * count);
        t->w1 = carve<double>(base, off, 3 * count);
        t->t2 = carve<double>(base, off, 3 * count);
        t->w2 = carve<double>(base, off, 9 * count);
        t->nodes = carve<NodeRec>(base, off, count);
        t->far64 = carve<Far64>(base, off, count);
        t->far32 = carve<Far32>(base, off, count);
        t->far64x = t->order3 ? carve<Far64x>(base, off, count) : nullptr;
        t->far32x = t->order3 ? carve<Far32x>(base, off, count) : nullptr;
        t->far64y = t->order4 ? carve<Far64y>(base, off, count) : nullptr;
        t->far32y = t->order4 ? carve<Far32y>(base, off, count) : nullptr;
        t->far64z = t->order5 ? carve<Far64z>(base, off, count) : nullptr;
        t->far32z = t->order5 ? carve<Far32z>(base, off, count) : nullptr;
        if (pass == 0) {
            base = t->alloc<char>(off, s);
            if (!base) return BS_ERR_OOM;
        }
    }
    // the bottom-up pipeline for every kind and order: its box, centre and bound equal the direct sums', its moments
    // equal them up to rounding (the translations of the children's moments), at O(m) work instead of O(m depth)
    if (t->order5) return moments_bottom_up<MOM_PARTS5>(t, geo, scratch, s, side);
    if (t->order4) return moments_bottom_up<MOM_PARTS4>(t, geo, scratch, s, side);
    return t->order3 ? moments_bottom_up<MOM_PARTS3>(t, geo, scratch, s, side)
                     : moments_bottom_up<MOM_PARTS>(t, geo, scratch, s, side);
}

}  // namespace bs

using namespace bs;

// The inverse permutation, the int64 order and the tree-ordered segment records: everything of a tree sized by its
// segments, not its nodes (queued while a Morton tree's node count travels back).  Once.
static int segment_records(bs_tree *t, const bs_sources *src, cudaStream_t s, cudaStream_t side) {
    if (t->records_done) return BS_OK;
    t->records_done = true;
    const int64_t m = t->m;
    if (!t->order) t->order = t->alloc<int64_t>(m, s);
    t->inverse = t->alloc<int32_t>(m, s);
    t->seg64 = t->alloc<Seg64>(m, s);
    t->seg32 = t->alloc<Seg32>(m, s);
    t->seg32x2 = t->alloc<Seg32x2>((m + 1) / 2, s);
    t->seg32c2 = t->alloc<Seg32c2>((m + 1) / 2, s);
    if (!t->order || !t->inverse || !t->seg64 || !t->seg32 || !t->seg32x2 || !t->seg32c2) return BS_ERR_OOM;
    widen_order_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, t->order32, t->order, t->inverse);
    BS_CHECK_LAUNCH("widen_order_kernel");
    // with a side stream (bottom-up trees of a tree sum) the segment records are packed there, beside the node
    // geometry and the walk, which do not read them
    const bool bottom_up = t->order4 || t->kind == BS_TREE_MORTON;
    cudaStream_t ps = (side && bottom_up) ? side : s;
    if (ps != s) {
        cudaEvent_t ready;
        BS_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        cudaEventRecord(ready, s);
        cudaStreamWaitEvent(ps, ready, 0);
        cudaEventDestroy(ready);
    }
    return pack_segments(src, t->order32, t->seg64, t->seg32, nullptr, ps, t->seg32x2);
}

// Shared tail of both constructors: the segment records (unless already queued), then the moments.
static int finish_tree(bs_tree *t, const bs_sources *src, const SegGeo *geo, Scratch &scratch, cudaStream_t s,
                       cudaStream_t side = nullptr) {
    int rc = segment_records(t, src, s, side);
    if (rc != BS_OK) return rc;
    const bool bottom_up = t->order4 || t->kind == BS_TREE_MORTON;
    return compute_moments(t, geo, scratch, s, bottom_up ? side : nullptr);
}

static int check_sources(const bs_sources *src) {
    if (!src || src->m < 0 || (src->m > 0 && (!src->starts || !src->directions || !src->lengths || !src->gamma ||
                                               !src->radius))) {
        set_error("invalid segment arrays");
        return BS_ERR_ARG;
    }
    if (src->m >= (int64_t(1) << 31) - 1) {
        set_error("at most 2^31 - 2 segments are supported (got %lld)", (long long)src->m);
        return BS_ERR_ARG;
    }
    return BS_OK;
}

extern "C" void bs_tree_free(bs_tree *tree) {
    if (!tree) return;
    cudaSetDevice(tree->device);
    cudaDeviceSynchronize();
    for (int i = 0; i < tree->nblocks; ++i) cudaFreeAsync(tree->blocks[i], 0);
    cudaStreamSynchronize(0);
    for (auto &e : tree->marks)
        if (e) cudaEventDestroy(e);
    delete tree;
}

extern "C" int64_t bs_tree_count(const bs_tree *tree) { return tree ? tree->count : -1; }

// The build behind bs_tree_build (wait = true: synchronises, checks and records the stage times) and bs_tree_sum
// (wait = false: the evaluation is queued behind the build on the same stream, and tree_stage_times reads the times
// once the caller has synchronised).
int tree_build(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, bs_tree **out, cudaStream_t s,
               bool wait, const std::function<int()> &before_geometry, cudaStream_t side) {
    if (!ctx || !tp || !out) {
        set_error("bs_tree_build: null argument");
        return BS_ERR_ARG;
    }
    *out = nullptr;
    int rc = check_sources(src);
    if (rc != BS_OK) return rc;
    if (src->m == 0) {
        set_error("bs_tree_build: no segments");
        return BS_ERR_ARG;
    }
    if (tp->leaf_size < 1 || (tp->kind != BS_TREE_MEDIAN && tp->kind != BS_TREE_MORTON)) {
        set_error("bs_tree_build: leaf size must be positive and kind median or morton");
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaSetDevice(ctx->device));
    bs_tree *t = new bs_tree();
    cudaEvent_t &e0 = t->marks[0], &e1 = t->marks[1], &e2 = t->marks[2];
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventRecord(e0, s);
    t->device = ctx->device;
    t->pool = ctx->pool;
    t->kind = tp->kind;
    t->m = src->m;
    t->leaf_size = tp->leaf_size;
    t->order3 = tp->order >= 3;
    t->order4 = tp->order >= 4;
    t->order5 = tp->order >= 5;
    // the moment phase of the bottom-up pipeline (Morton trees, fourth-order trees) may run on the side stream
    cudaStream_t defer = (side && (t->order4 || t->kind == BS_TREE_MORTON)) ? side : nullptr;
    {
        Scratch scratch(ctx->pool, s);
        // before_geometry (may be empty) runs once, before anything reads gamma or radius: for Morton trees while the
        // node count travels back (keys and topology need only starts, directions and lengths)
        bool ran = false;
        auto gate = [&]() -> int {
            if (ran || !before_geometry) return BS_OK;
            ran = true;
            return before_geometry();
        };
        SegGeo *geo = defer ? t->alloc<SegGeo>(src->m, s) : scratch.get<SegGeo>(src->m);
        rc = geo ? BS_OK : (defer ? BS_ERR_OOM : scratch.status);
        if (rc == BS_OK && tp->kind == BS_TREE_MORTON) {
            // while the node count travels back: the caller's hook, the moment pipeline's geometry in tree order
            // (every leaf reads a contiguous range) and the segment records, none of which needs the count
            bool early_ran = false;
            auto early = [&]() -> int {
                if (early_ran) return BS_OK;
                early_ran = true;
                int r = gate();
                if (r == BS_OK) r = pack_segments(src, t->order32, nullptr, nullptr, geo, s);
                t->geo_sorted = true;
                if (r == BS_OK) r = segment_records(t, src, s, defer);
                return r;
            };
            t->host_count = reinterpret_cast<int64_t *>(ctx_pinned(ctx));
            rc = build_morton(t, src, scratch, s, early);
            if (rc == BS_OK) rc = early();  // (a tree of one leaf has no count to wait for)
        } else if (rc == BS_OK) {
            rc = gate();
            if (rc == BS_OK) rc = pack_segments(src, nullptr, nullptr, nullptr, geo, s);
            if (rc == BS_OK) rc = build_median(t, geo, scratch, s);
        }
        if (rc == BS_OK) {
            cudaEventRecord(e1, s);
            rc = finish_tree(t, src, geo, scratch, s, defer);
        }
        cudaEventRecord(e2, defer ? defer : s);
        if (defer) t->moments_done = e2;
        if (rc == BS_OK && wait) {
            cudaError_t e = cudaEventSynchronize(e2);
            if (e != cudaSuccess) rc = cuda_fail(e, "tree build");
            if (rc == BS_OK) rc = check_sort_fault();
        }
    }
    if (rc == BS_OK) {
        if (wait) tree_stage_times(t);
        ctx->stats.build_ms = t->build_ms;
        ctx->stats.moments_ms = t->moments_ms;
        ctx->stats.nodes = t->count;
        ctx->stats.segments = t->m;
        *out = t;
    } else {
        bs_tree_free(t);
    }
    return rc;
}

void tree_stage_times(bs_tree *t) {
    cudaEventElapsedTime(&t->build_ms, t->marks[0], t->marks[1]);
    cudaEventElapsedTime(&t->moments_ms, t->marks[1], t->marks[2]);
}

void tree_release(bs_tree *tree, cudaStream_t s) {
    if (!tree) return;
    cudaSetDevice(tree->device);
    if (tree->moments_done) cudaStreamWaitEvent(s, tree->moments_done, 0);  // moments still read the tree's memory
    for (int i = 0; i < tree->nblocks; ++i) cudaFreeAsync(tree->blocks[i], s);
    for (auto &e : tree->marks)
        if (e) cudaEventDestroy(e);
    delete tree;
}

extern "C" int bs_tree_build(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, bs_tree **out,
                             bs_stream stream) {
    return tree_build(ctx, src, tp, out, (cudaStream_t)stream, true, {});
}

extern "C" int bs_forest_build(bs_ctx *ctx, const bs_sources *src, int nwakes, const int64_t *wake_ptr,
                               const bs_tree_params *tp, bs_tree **out, bs_stream stream) {
    if (!ctx || !tp || !out || nwakes < 1 || !wake_ptr) {
        set_error("bs_forest_build: null argument or no wakes");
        return BS_ERR_ARG;
    }
    *out = nullptr;
    int rc = check_sources(src);
    if (rc != BS_OK) return rc;
    if (src->m == 0 || tp->leaf_size < 1 || nwakes > (1 << 20)) {
        set_error("bs_forest_build: no segments, a non-positive leaf size or more than 2^20 wakes");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventRecord(e0, s);
    bs_tree *t = new bs_tree();
    t->device = ctx->device;
    t->pool = ctx->pool;
    t->kind = BS_TREE_MORTON;
    t->m = src->m;
    t->leaf_size = tp->leaf_size;
    t->order3 = tp->order >= 3;
    t->order4 = tp->order >= 4;
    t->order5 = tp->order >= 5;
    {
        Scratch scratch(ctx->pool, s);
        SegGeo *geo = scratch.get<SegGeo>(src->m);
        rc = geo ? pack_segments(src, nullptr, nullptr, nullptr, geo, s) : scratch.status;
        if (rc == BS_OK) rc = build_forest(t, geo, wake_ptr, nwakes, scratch, s);
        if (rc == BS_OK) {
            cudaEventRecord(e1, s);
            rc = finish_tree(t, src, geo, scratch, s);
        }
        cudaEventRecord(e2, s);
        if (rc == BS_OK) {
            cudaError_t e = cudaEventSynchronize(e2);
            if (e != cudaSuccess) rc = cuda_fail(e, "forest build");
            if (rc == BS_OK) rc = check_sort_fault();
        }
    }
    if (rc == BS_OK) {
        cudaEventElapsedTime(&t->build_ms, e0, e1);
        cudaEventElapsedTime(&t->moments_ms, e1, e2);
        ctx->stats.build_ms = t->build_ms;
        ctx->stats.moments_ms = t->moments_ms;
        ctx->stats.nodes = t->count;
        ctx->stats.segments = t->m;
        *out = t;
    } else {
        bs_tree_free(t);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    return rc;
}

extern "C" int bs_forest_roots(const bs_tree *t, int32_t *roots, bs_stream stream) {
    if (!t || !t->wake_root || !roots) {
        set_error("bs_forest_roots: not a forest");
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaMemcpyAsync(roots, t->wake_root, t->nwakes * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                            (cudaStream_t)stream));
    return BS_OK;
}

__global__ void narrow_order_kernel(int64_t m, const int64_t *order, int32_t *order32) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) order32[k] = (int32_t)order[k];
}

extern "C" int bs_tree_from_arrays(bs_ctx *ctx, const bs_sources *src, const int64_t *order, const int64_t *lo,
                                   const int64_t *hi, const int64_t *left, const int64_t *right, int64_t count,
                                   bs_tree **out, bs_stream stream) {
    if (!ctx || !out || !order || !lo || !hi || !left || !right || count < 1) {
        set_error("bs_tree_from_arrays: null argument or empty tree");
        return BS_ERR_ARG;
    }
    *out = nullptr;
    int rc = check_sources(src);
    if (rc != BS_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    bs_tree *t = new bs_tree();
    t->device = ctx->device;
    t->pool = ctx->pool;
    t->kind = -1;
    t->m = src->m;
    t->count = count;
    {
        Scratch scratch(ctx->pool, s);
        SegGeo *geo = scratch.get<SegGeo>(src->m);
        t->order = t->alloc<int64_t>(t->m, s);
        t->order32 = t->alloc<int32_t>(t->m, s);
        t->lo = t->alloc<int64_t>(count, s);
        t->hi = t->alloc<int64_t>(count, s);
        t->left = t->alloc<int64_t>(count, s);
        t->right = t->alloc<int64_t>(count, s);
        if (!geo || !t->order || !t->order32 || !t->lo || !t->hi || !t->left || !t->right) rc = BS_ERR_OOM;
        if (rc == BS_OK) {
            cudaMemcpyAsync(t->order, order, t->m * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(t->lo, lo, count * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(t->hi, hi, count * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(t->left, left, count * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(t->right, right, count * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            narrow_order_kernel<<<blocks_for(t->m, 256), 256, 0, s>>>(t->m, order, t->order32);
            rc = pack_segments(src, nullptr, nullptr, nullptr, geo, s);
        }
        if (rc == BS_OK) rc = finish_tree(t, src, geo, scratch, s);
        if (rc == BS_OK) {
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) rc = cuda_fail(e, "tree from arrays");
        }
    }
    if (rc == BS_OK) *out = t;
    else bs_tree_free(t);
    return rc;
}

__global__ void widen_keys_order_kernel(int64_t m, const int32_t *order32, int64_t *out) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) out[k] = order32[k];
}

// bad[0] = 1 if an order entry lies outside [0, m) or a node range outside 0 <= lo <= hi <= m
__global__ void topology_check_kernel(int64_t m, int64_t count, const int64_t *order, const int64_t *lo,
                                      const int64_t *hi, int *bad) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m && (order[k] < 0 || order[k] >= m)) *bad = 1;
    if (k < count && (lo[k] < 0 || lo[k] > hi[k] || hi[k] > m)) *bad = 1;
}

__global__ void geo_from_mid_kernel(int64_t m, const double *mid, SegGeo *geo) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    // start = end = mid, so that 0.5 * (start + end) is mid exactly
    SegGeo q;
    q.sx = q.ex = mid[3 * k];
    q.sy = q.ey = mid[3 * k + 1];
    q.sz = q.ez = mid[3 * k + 2];
    q.lx = q.ly = q.lz = 0.0;
    q.gamma = q.radius = q.pad = 0.0;
    geo[k] = q;
}

__global__ void geo_from_ends_kernel(int64_t m, const double *starts, const double *ends, const double *lv,
                                     const double *gamma, const double *radius, SegGeo *geo) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    SegGeo q;
    q.sx = starts[3 * k]; q.sy = starts[3 * k + 1]; q.sz = starts[3 * k + 2];
    q.ex = ends[3 * k]; q.ey = ends[3 * k + 1]; q.ez = ends[3 * k + 2];
    q.lx = lv[3 * k]; q.ly = lv[3 * k + 1]; q.lz = lv[3 * k + 2];
    q.gamma = gamma[k];
    q.radius = radius[k];
    q.pad = 0.0;
    geo[k] = q;
}

extern "C" int bs_median_topology(bs_ctx *ctx, int64_t m, const double *mid, int leaf_size, int64_t *order,
                                  int64_t *lo, int64_t *hi, int64_t *left, int64_t *right, int64_t capacity,
                                  int64_t *count, bs_stream stream) {
    if (!ctx || !count || m < 0 || (m > 0 && (!mid || !order)) || leaf_size < 1 || capacity < 0 ||
        (capacity > 0 && (!lo || !hi || !left || !right))) {
        set_error("bs_median_topology: null or negative argument");
        return BS_ERR_ARG;
    }
    if (m >= (int64_t(1) << 31) - 1) {
        set_error("bs_median_topology: at most 2^31 - 2 midpoints");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    if (m == 0) {  // one empty leaf, as build_tree returns for no segments
        *count = 1;
        if (capacity >= 1) {
            const int64_t row[4] = {0, 0, -1, -1};
            BS_CUDA(cudaMemcpyAsync(lo, row, sizeof(int64_t), cudaMemcpyHostToDevice, s));
            BS_CUDA(cudaMemcpyAsync(hi, row + 1, sizeof(int64_t), cudaMemcpyHostToDevice, s));
            BS_CUDA(cudaMemcpyAsync(left, row + 2, sizeof(int64_t), cudaMemcpyHostToDevice, s));
            BS_CUDA(cudaMemcpyAsync(right, row + 3, sizeof(int64_t), cudaMemcpyHostToDevice, s));
            BS_CUDA(cudaStreamSynchronize(s));
        }
        return BS_OK;
    }
    bs_tree *t = new bs_tree();
    t->device = ctx->device;
    t->pool = ctx->pool;
    t->kind = BS_TREE_MEDIAN;
    t->m = m;
    t->leaf_size = leaf_size;
    int rc = BS_OK;
    {
        Scratch scratch(ctx->pool, s);
        SegGeo *geo = scratch.get<SegGeo>(m);
        if (!geo) rc = scratch.status;
        if (rc == BS_OK) {
            geo_from_mid_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, mid, geo);
            BS_CHECK_LAUNCH("geo_from_mid_kernel");
            rc = build_median(t, geo, scratch, s);
        }
        if (rc == BS_OK) {
            *count = t->count;
            widen_keys_order_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, t->order32, order);
            BS_CHECK_LAUNCH("widen_keys_order_kernel");
            if (t->count <= capacity) {
                const size_t c8 = (size_t)t->count * sizeof(int64_t);
                cudaMemcpyAsync(lo, t->lo, c8, cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(hi, t->hi, c8, cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(left, t->left, c8, cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(right, t->right, c8, cudaMemcpyDeviceToDevice, s);
            }
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) rc = cuda_fail(e, "bs_median_topology");
        }
    }
    bs_tree_free(t);
    return rc;
}

extern "C" int bs_node_quantities(bs_ctx *ctx, int64_t m, const double *starts, const double *ends,
                                  const double *length_vectors, const double *gamma, const double *radius,
                                  int64_t count, const int64_t *order, const int64_t *lo, const int64_t *hi,
                                  double *centre, double *bound, double *core, double *m0, double *m1, double *m2,
                                  double *w1, double *t2, double *w2, bs_stream stream) {
    if (!ctx || m < 1 || count < 1 || !starts || !ends || !length_vectors || !gamma || !radius || !order || !lo ||
        !hi) {
        set_error("bs_node_quantities: null argument or empty tree");
        return BS_ERR_ARG;
    }
    if (m >= (int64_t(1) << 31) - 1) {
        set_error("bs_node_quantities: at most 2^31 - 2 segments");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    bs_tree *t = new bs_tree();
    t->device = ctx->device;
    t->pool = ctx->pool;
    t->kind = -1;
    t->m = m;
    t->count = count;
    int rc = BS_OK;
    {
        Scratch scratch(ctx->pool, s);
        SegGeo *geo = scratch.get<SegGeo>(m);
        t->order32 = t->alloc<int32_t>(m, s);
        t->lo = t->alloc<int64_t>(count, s);
        t->hi = t->alloc<int64_t>(count, s);
        t->left = t->alloc<int64_t>(count, s);
        t->right = t->alloc<int64_t>(count, s);
        int *bad = scratch.get<int>(1);
        if (!geo || !bad || !t->order32 || !t->lo || !t->hi || !t->left || !t->right) rc = BS_ERR_OOM;
        if (rc == BS_OK) {
            int host_bad = 0;
            cudaMemsetAsync(bad, 0, sizeof(int), s);
            topology_check_kernel<<<blocks_for(std::max(m, count), 256), 256, 0, s>>>(m, count, order, lo, hi, bad);
            cudaMemcpyAsync(&host_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
            cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) rc = cuda_fail(e, "bs_node_quantities");
            else if (host_bad) {
                set_error("bs_node_quantities: order entry outside [0, m) or node range outside 0 <= lo <= hi <= m");
                rc = BS_ERR_ARG;
            }
        }
        if (rc == BS_OK) {
            cudaMemcpyAsync(t->lo, lo, count * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(t->hi, hi, count * sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
            cudaMemsetAsync(t->left, 0xff, count * sizeof(int64_t), s);
            cudaMemsetAsync(t->right, 0xff, count * sizeof(int64_t), s);
            narrow_order_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, order, t->order32);
            geo_from_ends_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, starts, ends, length_vectors, gamma, radius,
                                                                    geo);
            BS_CHECK_LAUNCH("geo_from_ends_kernel");
            rc = compute_moments(t, geo, scratch, s, nullptr);
        }
        if (rc == BS_OK) {
            rc = bs_tree_export(t, nullptr, nullptr, nullptr, nullptr, nullptr, centre, bound, core, m0, m1, m2, w1,
                                t2, w2, stream);
            cudaError_t e = cudaStreamSynchronize(s);
            if (rc == BS_OK && e != cudaSuccess) rc = cuda_fail(e, "bs_node_quantities");
        }
    }
    bs_tree_free(t);
    return rc;
}

extern "C" int bs_tree_export(const bs_tree *t, int64_t *order, int64_t *lo, int64_t *hi, int64_t *left,
                              int64_t *right, double *centre, double *bound, double *core, double *m0, double *m1,
                              double *m2, double *w1, double *t2, double *w2, bs_stream stream) {
    if (!t) {
        set_error("bs_tree_export: null tree");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t c = t->count;
    const size_t m8 = (size_t)t->m * 8, c8 = (size_t)c * 8;
    struct { void *dst; const void *src; size_t bytes; } copies[] = {
        {order, t->order, m8}, {lo, t->lo, c8}, {hi, t->hi, c8}, {left, t->left, c8}, {right, t->right, c8},
        {centre, t->centre, 3 * c8}, {bound, t->bound, c8}, {core, t->core, c8}, {m0, t->m0, 3 * c8},
        {m1, t->m1, 9 * c8}, {m2, t->m2, 27 * c8}, {w1, t->w1, 3 * c8}, {t2, t->t2, 3 * c8}, {w2, t->w2, 9 * c8}};
    for (auto &cp : copies)
        if (cp.dst) BS_CUDA(cudaMemcpyAsync(cp.dst, cp.src, cp.bytes, cudaMemcpyDeviceToDevice, s));
    return BS_OK;
}

extern "C" int bs_tree_keys(const bs_tree *t, uint64_t *keys, int64_t *sorted_order, bs_stream stream) {
    if (!t || t->kind != BS_TREE_MORTON) {
        set_error("bs_tree_keys: not a Morton tree");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (keys) BS_CUDA(cudaMemcpyAsync(keys, t->keys, t->m * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    if (sorted_order) {
        widen_keys_order_kernel<<<blocks_for(t->m, 256), 256, 0, s>>>(t->m, t->order32, sorted_order);
        BS_CHECK_LAUNCH("widen_keys_order_kernel");
    }
    return BS_OK;
}
