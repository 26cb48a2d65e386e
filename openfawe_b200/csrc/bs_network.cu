// Exclusion bookkeeping of the wake network on the device: the (point, segment) pairs whose point coincides with an
// endpoint of the segment (network_numba.incident_pairs, src/openfawe/aero/network_numba.py:242-256, and its loop
// _incident_pairs, :121-167) and their per-point CSR (vortex_numba.exclusion_csr,
// src/openfawe/aero/vortex_numba.py:228-243).  Integer and bit-pattern work: sorts, scans and gathers, HBM bound.
//
// incident_pairs.  For every segment s in order and each of its ends e = 0, 1, the reference emits (i, s) for every
// free point i (node first + i) whose coordinates equal node edges[s, e] bit for bit (a NaN coordinate never matches),
// i increasing.  Here: the nodes are sorted by their three coordinate bit patterns (stable LSD radix sort, only the bits
// that vary among the nodes), equal patterns form runs, and since the sort is stable a run lists its nodes by
// increasing index, so the free nodes of a run are the tail of the run.  Each (segment, end) entry then owns the
// positions [first free, end) of its node's run; a scan of their lengths places the output.
//
// exclusion_csr.  np.unique of the pairs (point-major, then segment) and a per-point count: one stable radix sort of
// the composite key (point, segment - min segment) when it fits in 64 bits (two sorts otherwise), a unique pass and a
// count scan.
#include <algorithm>
#include <climits>

#include "bs_internal.cuh"
#include "bs_sort.cuh"

namespace bs {

__device__ __forceinline__ bool has_nan3(const double *p) { return isnan(p[0]) || isnan(p[1]) || isnan(p[2]); }

__device__ __forceinline__ uint64_t bits_of(double v) { return (uint64_t)__double_as_longlong(v); }

// varying[c] |= bits(node c) ^ bits(node 0): the bits that differ anywhere
__global__ void varying_bits_kernel(int64_t n, const double *nodes, unsigned long long *varying) {
    __shared__ unsigned long long acc[3];
    if (threadIdx.x < 3) acc[threadIdx.x] = 0ull;
    __syncthreads();
    unsigned long long v[3] = {0ull, 0ull, 0ull};
    const uint64_t b0 = bits_of(nodes[0]), b1 = bits_of(nodes[1]), b2 = bits_of(nodes[2]);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        v[0] |= bits_of(nodes[3 * i]) ^ b0;
        v[1] |= bits_of(nodes[3 * i + 1]) ^ b1;
        v[2] |= bits_of(nodes[3 * i + 2]) ^ b2;
    }
    for (int c = 0; c < 3; ++c) {
        for (int o = 16; o; o >>= 1) v[c] |= __shfl_xor_sync(0xffffffffu, v[c], o);
        if ((threadIdx.x & 31) == 0) atomicOr(&acc[c], v[c]);
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicOr(&varying[threadIdx.x], acc[threadIdx.x]);
}

// keys[i] = bits of coordinate c of node order[i] ^ bits of node 0 (equality-preserving)
__global__ void coord_keys_kernel(int64_t n, const double *nodes, int c, const int32_t *order, uint64_t *keys) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = bits_of(nodes[3 * (int64_t)order[i] + c]) ^ bits_of(nodes[c]);
}

__global__ void iota32_kernel(int64_t n, int32_t *v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

// flag[i] = 1 where sorted position i begins a run (first position, a NaN node, a NaN predecessor, other bits)
__global__ void run_flags_kernel(int64_t n, const double *nodes, const int32_t *order, int64_t *flag) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *a = nodes + 3 * (int64_t)order[i];
    bool fresh = i == 0 || has_nan3(a);
    if (!fresh) {
        const double *b = nodes + 3 * (int64_t)order[i - 1];
        fresh = has_nan3(b) || bits_of(a[0]) != bits_of(b[0]) || bits_of(a[1]) != bits_of(b[1]) ||
                bits_of(a[2]) != bits_of(b[2]);
    }
    flag[i] = fresh ? 1 : 0;
}

// run_of[node]; run_end[r] = one past the run's last position; run_free[r] = the run's first position holding a free
// node (index >= first), or run_end[r] when it has none.  Free nodes are a suffix of their run (a run lists its nodes
// by increasing index), so exactly one position writes run_free[r]: the first free one, or the last one if none is.
__global__ void run_bounds_kernel(int64_t n, int64_t first, const int32_t *order, const int64_t *flag,
                                  const int64_t *before, int64_t *run_of, int64_t *run_end, int64_t *run_free) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t run = before[i] + flag[i] - 1;
    const int64_t node = order[i];
    run_of[node] = run;
    const bool last = i + 1 == n || flag[i + 1] != 0;
    const bool is_free = node >= first;
    if (last) run_end[run] = i + 1;
    if (is_free && (flag[i] != 0 || order[i - 1] < first)) run_free[run] = i;
    if (last && !is_free) run_free[run] = i + 1;
}

// count[k] of entry k = 2 s + e (segment s, end e): free nodes equal to node edges[s][e]
__global__ void incident_count_kernel(int64_t entries, const int64_t *edges, const double *nodes,
                                      const int64_t *run_of, const int64_t *run_end, const int64_t *run_free,
                                      int64_t *count) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= entries) return;
    const int64_t node = edges[k];
    if (has_nan3(nodes + 3 * node)) {
        count[k] = 0;
        return;
    }
    const int64_t r = run_of[node];
    count[k] = run_end[r] - run_free[r];
}

__global__ void incident_write_kernel(int64_t entries, int64_t first, const int64_t *edges, const double *nodes,
                                      const int32_t *order, const int64_t *run_of, const int64_t *run_free,
                                      const int64_t *count, const int64_t *offset, int64_t *pairs) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= entries) return;
    const int64_t c = count[k];
    if (c == 0) return;
    const int64_t r = run_of[edges[k]], segment = k >> 1;
    int64_t o = offset[k];
    for (int64_t j = 0; j < c; ++j, ++o) {
        pairs[2 * o] = (int64_t)order[run_free[r] + j] - first;
        pairs[2 * o + 1] = segment;
    }
}

// bad[0] = 1 if any edge index is outside [0, n)
__global__ void edge_range_kernel(int64_t entries, const int64_t *edges, int64_t n, int *bad) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < entries && (edges[k] < 0 || edges[k] >= n)) *bad = 1;
}

// range[0..3] = min point, max point, min segment, max segment
__global__ void pair_range_kernel(int64_t e, const int64_t *pairs, long long *range) {
    long long v[4] = {LLONG_MAX, LLONG_MIN, LLONG_MAX, LLONG_MIN};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < e; i += (int64_t)gridDim.x * blockDim.x) {
        const long long p = pairs[2 * i], s = pairs[2 * i + 1];
        v[0] = min(v[0], p);
        v[1] = max(v[1], p);
        v[2] = min(v[2], s);
        v[3] = max(v[3], s);
    }
    for (int o = 16; o; o >>= 1) {
        v[0] = min(v[0], __shfl_xor_sync(0xffffffffu, v[0], o));
        v[1] = max(v[1], __shfl_xor_sync(0xffffffffu, v[1], o));
        v[2] = min(v[2], __shfl_xor_sync(0xffffffffu, v[2], o));
        v[3] = max(v[3], __shfl_xor_sync(0xffffffffu, v[3], o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&range[0], v[0]);
        atomicMax(&range[1], v[1]);
        atomicMin(&range[2], v[2]);
        atomicMax(&range[3], v[3]);
    }
}

// key[i] = (point << sbits) | (segment - smin), or one of the two fields alone (mode 1: segment, mode 2: point of the
// pair order[i])
__global__ void pair_keys_kernel(int64_t e, const int64_t *pairs, const int32_t *order, int mode, int sbits,
                                 long long smin, uint64_t *keys) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    const int64_t j = order[i];
    const uint64_t p = (uint64_t)pairs[2 * j], s = (uint64_t)(pairs[2 * j + 1] - smin);
    keys[i] = mode == 0 ? (sbits >= 64 ? s : ((p << sbits) | s)) : mode == 1 ? s : p;
}

__global__ void unique_flags_kernel(int64_t e, const int64_t *pairs, const int32_t *order, int64_t *flag) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    const int64_t a = order[i];
    bool fresh = i == 0;
    if (!fresh) {
        const int64_t b = order[i - 1];
        fresh = pairs[2 * a] != pairs[2 * b] || pairs[2 * a + 1] != pairs[2 * b + 1];
    }
    flag[i] = fresh ? 1 : 0;
}

__global__ void unique_write_kernel(int64_t e, const int64_t *pairs, const int32_t *order, const int64_t *flag,
                                    const int64_t *position, int64_t *seg, unsigned long long *per_point) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e || !flag[i]) return;
    const int64_t a = order[i];
    seg[position[i]] = pairs[2 * a + 1];
    atomicAdd(&per_point[pairs[2 * a]], 1ull);
}

static int bit_length(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

}  // namespace bs

using namespace bs;

static unsigned grid_for(int64_t n, int threads = 256) { return (unsigned)std::max<int64_t>(1, (n + threads - 1) / threads); }

extern "C" int bs_incident_pairs(bs_ctx *ctx, const double *nodes, int64_t n, const int64_t *edges, int64_t segments,
                                 int64_t first, int64_t *pairs, int64_t capacity, int64_t *count, bs_stream stream) {
    if (!ctx || !count || n < 0 || segments < 0 || (n > 0 && !nodes) || (segments > 0 && !edges) || capacity < 0 ||
        (capacity > 0 && !pairs)) {
        set_error("bs_incident_pairs: null or negative argument");
        return BS_ERR_ARG;
    }
    if (first < 0 || first > n) {
        set_error("bs_incident_pairs: first must lie in [0, node count]");
        return BS_ERR_ARG;
    }
    if (n >= ((int64_t)1 << 31)) {
        set_error("bs_incident_pairs: more than 2^31 - 1 nodes");
        return BS_ERR_ARG;
    }
    *count = 0;
    const int64_t entries = 2 * segments;
    if (entries == 0) return BS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    Scratch scratch(ctx->pool, s);
    int *bad = scratch.get<int>(1);
    unsigned long long *varying = scratch.get<unsigned long long>(3);
    if (!bad || !varying) return scratch.status;
    BS_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    BS_CUDA(cudaMemsetAsync(varying, 0, 3 * sizeof(unsigned long long), s));
    edge_range_kernel<<<grid_for(entries), 256, 0, s>>>(entries, edges, n, bad);
    BS_CHECK_LAUNCH("edge_range_kernel");
    if (n > 0) {
        varying_bits_kernel<<<(unsigned)std::min<int64_t>(ctx->sm_count * 4, grid_for(n)), 256, 0, s>>>(n, nodes,
                                                                                                          varying);
        BS_CHECK_LAUNCH("varying_bits_kernel");
    }
    struct {
        int bad;
        unsigned long long varying[3];
    } probe;
    BS_CUDA(cudaMemcpyAsync(&probe.bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    BS_CUDA(cudaMemcpyAsync(probe.varying, varying, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    BS_CUDA(cudaStreamSynchronize(s));
    if (probe.bad) {
        set_error("bs_incident_pairs: an edge index lies outside [0, node count)");
        return BS_ERR_ARG;
    }
    // sort node indices by (x, y, z) bit patterns, least significant component first (stable)
    int32_t *order = scratch.get<int32_t>(n);
    uint64_t *keys = scratch.get<uint64_t>(n);
    int64_t *flag = scratch.get<int64_t>(n), *before = scratch.get<int64_t>(n);
    int64_t *run_of = scratch.get<int64_t>(n), *run_end = scratch.get<int64_t>(n), *run_free = scratch.get<int64_t>(n);
    int64_t *cnt = scratch.get<int64_t>(entries), *off = scratch.get<int64_t>(entries), *total = scratch.get<int64_t>(1);
    if (!order || !keys || !flag || !before || !run_of || !run_end || !run_free || !cnt || !off || !total)
        return scratch.status;
    iota32_kernel<<<grid_for(n), 256, 0, s>>>(n, order);
    BS_CHECK_LAUNCH("iota32_kernel");
    for (int c = 2; c >= 0; --c) {
        const uint64_t v = probe.varying[c];
        if (!v) continue;
        coord_keys_kernel<<<grid_for(n), 256, 0, s>>>(n, nodes, c, order, keys);
        BS_CHECK_LAUNCH("coord_keys_kernel");
        int rc = radix_sort(keys, order, n, __builtin_ctzll(v), bit_length(v), scratch, s);
        if (rc != BS_OK) return rc;
    }
    run_flags_kernel<<<grid_for(n), 256, 0, s>>>(n, nodes, order, flag);
    BS_CHECK_LAUNCH("run_flags_kernel");
    int rc = scan_exclusive(flag, before, n, nullptr, scratch, s);
    if (rc != BS_OK) return rc;
    run_bounds_kernel<<<grid_for(n), 256, 0, s>>>(n, first, order, flag, before, run_of, run_end, run_free);
    BS_CHECK_LAUNCH("run_bounds_kernel");
    incident_count_kernel<<<grid_for(entries), 256, 0, s>>>(entries, edges, nodes, run_of, run_end, run_free, cnt);
    BS_CHECK_LAUNCH("incident_count_kernel");
    rc = scan_exclusive(cnt, off, entries, total, scratch, s);
    if (rc != BS_OK) return rc;
    int64_t found = 0;
    BS_CUDA(cudaMemcpyAsync(&found, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    BS_CUDA(cudaStreamSynchronize(s));
    rc = check_sort_fault();
    if (rc != BS_OK) return rc;
    *count = found;
    if (found == 0 || found > capacity) return BS_OK;
    incident_write_kernel<<<grid_for(entries), 256, 0, s>>>(entries, first, edges, nodes, order, run_of, run_free, cnt,
                                                            off, pairs);
    BS_CHECK_LAUNCH("incident_write_kernel");
    return BS_OK;
}

extern "C" int bs_exclusion_csr(bs_ctx *ctx, int64_t n, const int64_t *pairs, int64_t e, int64_t *ptr, int64_t *seg,
                                int64_t *unique_count, bs_stream stream) {
    if (!ctx || !unique_count || n < 0 || e < 0 || !ptr || (e > 0 && (!pairs || !seg))) {
        set_error("bs_exclusion_csr: null or negative argument");
        return BS_ERR_ARG;
    }
    if (e >= ((int64_t)1 << 31)) {
        set_error("bs_exclusion_csr: more than 2^31 - 1 pairs");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    *unique_count = 0;
    if (e == 0) {
        BS_CUDA(cudaMemsetAsync(ptr, 0, (n + 1) * sizeof(int64_t), s));
        return BS_OK;
    }
    Scratch scratch(ctx->pool, s);
    long long *range = scratch.get<long long>(4);
    if (!range) return scratch.status;
    const long long init[4] = {LLONG_MAX, LLONG_MIN, LLONG_MAX, LLONG_MIN};
    long long host[4];
    BS_CUDA(cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, s));
    pair_range_kernel<<<(unsigned)std::min<int64_t>(ctx->sm_count * 4, grid_for(e)), 256, 0, s>>>(e, pairs, range);
    BS_CHECK_LAUNCH("pair_range_kernel");
    BS_CUDA(cudaMemcpyAsync(host, range, sizeof(host), cudaMemcpyDeviceToHost, s));
    BS_CUDA(cudaStreamSynchronize(s));
    if (host[0] < 0 || host[1] >= n) {
        set_error("bs_exclusion_csr: a pair's point lies outside [0, point count)");
        return BS_ERR_ARG;
    }
    const int pbits = bit_length((uint64_t)host[1]);
    const int sbits = bit_length((uint64_t)host[3] - (uint64_t)host[2]);
    int32_t *order = scratch.get<int32_t>(e);
    uint64_t *keys = scratch.get<uint64_t>(e);
    int64_t *flag = scratch.get<int64_t>(e), *position = scratch.get<int64_t>(e), *total = scratch.get<int64_t>(1);
    unsigned long long *per_point = scratch.get<unsigned long long>(n + 1);
    if (!order || !keys || !flag || !position || !total || !per_point) return scratch.status;
    iota32_kernel<<<grid_for(e), 256, 0, s>>>(e, order);
    BS_CHECK_LAUNCH("iota32_kernel");
    if (pbits + sbits <= 64) {
        pair_keys_kernel<<<grid_for(e), 256, 0, s>>>(e, pairs, order, 0, sbits, host[2], keys);
        BS_CHECK_LAUNCH("pair_keys_kernel");
        int rc = radix_sort(keys, order, e, 0, pbits + sbits, scratch, s);
        if (rc != BS_OK) return rc;
    } else {  // segment first, then point (stable)
        for (int mode = 1; mode <= 2; ++mode) {
            pair_keys_kernel<<<grid_for(e), 256, 0, s>>>(e, pairs, order, mode, sbits, host[2], keys);
            BS_CHECK_LAUNCH("pair_keys_kernel");
            int rc = radix_sort(keys, order, e, 0, mode == 1 ? sbits : pbits, scratch, s);
            if (rc != BS_OK) return rc;
        }
    }
    unique_flags_kernel<<<grid_for(e), 256, 0, s>>>(e, pairs, order, flag);
    BS_CHECK_LAUNCH("unique_flags_kernel");
    int rc = scan_exclusive(flag, position, e, total, scratch, s);
    if (rc != BS_OK) return rc;
    BS_CUDA(cudaMemsetAsync(per_point, 0, (n + 1) * sizeof(unsigned long long), s));
    unique_write_kernel<<<grid_for(e), 256, 0, s>>>(e, pairs, order, flag, position, seg, per_point);
    BS_CHECK_LAUNCH("unique_write_kernel");
    rc = scan_exclusive((const int64_t *)per_point, ptr, n + 1, nullptr, scratch, s);
    if (rc != BS_OK) return rc;
    BS_CUDA(cudaMemcpyAsync(unique_count, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    BS_CUDA(cudaStreamSynchronize(s));
    return check_sort_fault();
}
