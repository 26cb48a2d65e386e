// Exclusive scan and stable least-significant-digit radix sort for the tree builds.
//
// Radix sort: 8-bit digits, one kernel per digit with decoupled look-back across tiles (below).
#include <mutex>

#include "bs_sort.cuh"

namespace bs {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int64_t warp_inclusive(int64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int64_t o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total in *total.
__device__ int64_t block_exclusive(int64_t v, int64_t *total) {
    __shared__ int64_t warp_sums[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t inc = warp_inclusive(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        int64_t wi = warp_inclusive(w);
        warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    int64_t r = inc - v + warp_sums[warp];
    __syncthreads();
    return r;
}

__global__ void tile_sums_kernel(const int64_t *in, int64_t n, int64_t *sums) {
    __shared__ int64_t total;
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    int64_t v = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t idx = base + (int64_t)threadIdx.x * SCAN_ITEMS + i;
        if (idx < n) v += in[idx];
    }
    block_exclusive(v, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void tile_scan_kernel(const int64_t *in, int64_t *out, int64_t n, const int64_t *offsets, int64_t *total) {
    __shared__ int64_t block_total;
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    int64_t v[SCAN_ITEMS];
    int64_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t idx = base + (int64_t)threadIdx.x * SCAN_ITEMS + i;
        v[i] = idx < n ? in[idx] : 0;
        sum += v[i];
    }
    int64_t run = block_exclusive(sum, &block_total) + (offsets ? offsets[blockIdx.x] : 0);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t idx = base + (int64_t)threadIdx.x * SCAN_ITEMS + i;
        if (idx < n) out[idx] = run;
        run += v[i];
    }
    if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *total = run;
}

int scan_exclusive(const int64_t *in, int64_t *out, int64_t n, int64_t *total, Scratch &scratch, cudaStream_t s) {
    if (n <= 0) {
        if (total) BS_CUDA(cudaMemsetAsync(total, 0, sizeof(int64_t), s));
        return BS_OK;
    }
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles == 1) {
        tile_scan_kernel<<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr, total);
        BS_CHECK_LAUNCH("tile_scan_kernel");
        return BS_OK;
    }
    int64_t *sums = scratch.get<int64_t>(tiles);
    if (!sums) return scratch.status;
    tile_sums_kernel<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, sums);
    BS_CHECK_LAUNCH("tile_sums_kernel");
    int rc = scan_exclusive(sums, sums, tiles, nullptr, scratch, s);
    if (rc != BS_OK) return rc;
    tile_scan_kernel<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, out, n, sums, total);
    BS_CHECK_LAUNCH("tile_scan_kernel");
    return BS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// Radix sort: one pass over the keys counts the digits of every pass; then one kernel per 8-bit digit.  Each block of
// that kernel takes the next tile in input order (an atomic ticket), ranks its keys stably (a warp owns a contiguous
// run of the tile; inside it __match_any_sync groups equal digits, per-warp counters carry them across rounds), learns
// the number of equal digits in all earlier tiles by decoupled look-back over the per-(tile, digit) status words, and
// writes its keys out through shared memory in digit runs, so that the stores are contiguous.  A block only waits for
// tiles that took their ticket earlier (they are running and never wait for later ones); every wait is bounded, and a
// wait that runs out records a fault for the host (check_sort_fault) and goes on.
// ---------------------------------------------------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 8;                          // 32-key rounds per warp
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;       // 2048 keys per tile
constexpr int RS_MAX_PASSES = 8;
constexpr unsigned long long RS_AGGREGATE = 1ull << 62;  // status: this tile's own count
constexpr unsigned long long RS_PREFIX = 2ull << 62;     // status: count over this tile and all earlier ones
constexpr unsigned long long RS_VALUE = (1ull << 62) - 1;
constexpr int RS_SPIN_LIMIT = 1 << 22;

__device__ int g_sort_fault = 0;

// counts[p][d]: keys whose digit of pass p (bits shift0 + 8 p ..) is d.
__global__ void __launch_bounds__(RS_THREADS) radix_count_kernel(const uint64_t *keys, int64_t n, int shift0,
                                                                 int passes, unsigned long long *counts) {
    __shared__ unsigned hist[RS_MAX_PASSES][256];
    for (int q = threadIdx.x; q < RS_MAX_PASSES * 256; q += blockDim.x) hist[q >> 8][q & 255] = 0;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&hist[p][(k >> (shift0 + 8 * p)) & 255], 1u);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < passes * 256; q += blockDim.x)
        if (hist[q >> 8][q & 255]) atomicAdd(&counts[q], (unsigned long long)hist[q >> 8][q & 255]);
}

// starts[p][d] = number of keys whose pass-p digit is below d (one block per pass).
__global__ void __launch_bounds__(256) radix_starts_kernel(const unsigned long long *counts,
                                                           unsigned long long *starts) {
    __shared__ unsigned long long warp_sums[8];
    const int d = threadIdx.x, lane = d & 31, warp = d >> 5;
    const unsigned long long v = counts[256 * blockIdx.x + d];
    unsigned long long inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    unsigned long long before = 0;
    for (int w = 0; w < warp; ++w) before += warp_sums[w];
    starts[256 * blockIdx.x + d] = before + inc - v;
}

__device__ __forceinline__ unsigned long long load_status(const unsigned long long *p) {
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

__global__ void __launch_bounds__(RS_THREADS) radix_pass_kernel(const uint64_t *keys_in, const int32_t *vals_in,
                                                                uint64_t *keys_out, int32_t *vals_out, int64_t n,
                                                                int shift, const unsigned long long *starts,
                                                                unsigned long long *status, unsigned *ticket) {
    __shared__ unsigned short wcount[RS_WARPS][256];  // per-warp running, then exclusive-over-warps, digit counts
    __shared__ int local_start[256];                  // digit runs inside the staged tile
    __shared__ unsigned long long global_base[256];  // where each digit run of this tile goes
    __shared__ uint64_t skeys[RS_TILE];
    __shared__ int32_t svals[RS_TILE];
    __shared__ int tile_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) tile_s = (int)atomicAdd(ticket, 1u);
    for (int w = 0; w < RS_WARPS; ++w) wcount[w][tid] = 0;
    __syncthreads();
    const int tile = tile_s;
    const int64_t first = (int64_t)tile * RS_TILE + (int64_t)warp * (32 * RS_ROUNDS);
    uint64_t key[RS_ROUNDS];
    int32_t val[RS_ROUNDS];
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        const int64_t i = first + 32 * r + lane;
        key[r] = i < n ? keys_in[i] : 0;
        val[r] = i < n ? vals_in[i] : 0;
    }
    // stable rank inside the warp's run: earlier rounds first, then lanes in order
    int digit[RS_ROUNDS], rank[RS_ROUNDS];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        const int64_t i = first + 32 * r + lane;
        const int d = i < n ? (int)((key[r] >> shift) & 255) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        int before = 0;
        if (d < 256 && lane == leader) before = wcount[warp][d];
        before = __shfl_sync(0xffffffffu, before, leader);
        __syncwarp();
        if (d < 256 && lane == leader) wcount[warp][d] = (unsigned short)(before + __popc(peers));
        __syncwarp();
        digit[r] = d;
        rank[r] = before + __popc(peers & lt);
    }
    __syncthreads();
    // thread d: counts over the warps become exclusive offsets; the tile's total for digit d
    const int d = tid;
    int total = 0;
    for (int w = 0; w < RS_WARPS; ++w) {
        const int c = wcount[w][d];
        wcount[w][d] = (unsigned short)total;
        total += c;
    }
    // publish this tile's count, then look back for the count over all earlier tiles
    unsigned long long *mine = status + (int64_t)tile * 256 + d;
    if (tile == 0) {
        atomicExch(mine, RS_PREFIX | (unsigned long long)total);
    } else {
        atomicExch(mine, RS_AGGREGATE | (unsigned long long)total);
    }
    unsigned long long exclusive = 0;
    for (int t = tile - 1; t >= 0; --t) {
        unsigned long long v = load_status(status + (int64_t)t * 256 + d);
        int spins = 0;
        while ((v >> 62) == 0) {
            if (++spins > RS_SPIN_LIMIT) {
                atomicExch(&g_sort_fault, 1);
                break;
            }
            __nanosleep(32);
            v = load_status(status + (int64_t)t * 256 + d);
        }
        exclusive += v & RS_VALUE;
        if ((v >> 62) != 1) break;  // a prefix (or a fault): done
    }
    if (tile > 0) atomicExch(mine, RS_PREFIX | (exclusive + (unsigned long long)total));
    global_base[d] = starts[d] + exclusive;
    // digit runs of the staged tile: exclusive scan of the totals over the digits
    {
        int inc = total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        __shared__ int warp_tot[RS_WARPS];
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        int before = 0;
        for (int w = 0; w < warp; ++w) before += warp_tot[w];
        local_start[d] = before + inc - total;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        if (digit[r] < 256) {
            const int pos = local_start[digit[r]] + wcount[warp][digit[r]] + rank[r];
            skeys[pos] = key[r];
            svals[pos] = val[r];
        }
    }
    __syncthreads();
    const int64_t valid = min((int64_t)RS_TILE, n - (int64_t)tile * RS_TILE);
    for (int q = tid; q < valid; q += RS_THREADS) {
        const uint64_t k = skeys[q];
        const int dq = (int)((k >> shift) & 255);
        const unsigned long long pos = global_base[dq] + (unsigned long long)(q - local_start[dq]);
        keys_out[pos] = k;
        vals_out[pos] = svals[q];
    }
}

int radix_sort(uint64_t *keys, int32_t *vals, int64_t n, int begin_bit, int end_bit, Scratch &scratch,
               cudaStream_t s) {
    if (n <= 1 || end_bit <= begin_bit) return BS_OK;
    const int passes = (end_bit - begin_bit + 7) / 8;
    if (passes > RS_MAX_PASSES) {
        set_error("radix sort: at most 64 key bits");
        return BS_ERR_ARG;
    }
    const int64_t tiles = (n + RS_TILE - 1) / RS_TILE;
    uint64_t *k2 = scratch.get<uint64_t>(n);
    int32_t *v2 = scratch.get<int32_t>(n);
    // one zeroed block: digit counts, then the look-back status words of every pass, then the tickets
    const size_t words = (size_t)passes * 256 + (size_t)passes * 256 * tiles + (size_t)passes;
    unsigned long long *block = scratch.get<unsigned long long>(words);
    unsigned long long *starts = scratch.get<unsigned long long>((size_t)passes * 256);
    if (!k2 || !v2 || !block || !starts) return scratch.status;
    unsigned long long *counts = block, *status = block + (size_t)passes * 256;
    unsigned *tickets = reinterpret_cast<unsigned *>(status + (size_t)passes * 256 * tiles);
    BS_CUDA(cudaMemsetAsync(block, 0, words * sizeof(unsigned long long), s));
    const unsigned count_grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 4095) / 4096, 148 * 4));
    radix_count_kernel<<<count_grid, RS_THREADS, 0, s>>>(keys, n, begin_bit, passes, counts);
    radix_starts_kernel<<<passes, 256, 0, s>>>(counts, starts);
    BS_CHECK_LAUNCH("radix_count_kernel");
    uint64_t *ka = keys, *kb = k2;
    int32_t *va = vals, *vb = v2;
    for (int p = 0; p < passes; ++p) {
        radix_pass_kernel<<<(unsigned)tiles, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, begin_bit + 8 * p, starts + 256 * p,
                                                                  status + (size_t)256 * tiles * p, tickets + p);
        BS_CHECK_LAUNCH("radix_pass_kernel");
        uint64_t *kt = ka; ka = kb; kb = kt;
        int32_t *vt = va; va = vb; vb = vt;
    }
    if (passes & 1) {
        BS_CUDA(cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        BS_CUDA(cudaMemcpyAsync(vals, va, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    }
    return BS_OK;
}

// The fault word is one per device, shared by every context, stream and host thread of the process: a look-back
// timeout in one sort is reported by (and cleared by) the next call on that device that checks it, which may be
// another thread's.  A timeout is a broken-device condition, not a per-call result, so that is acceptable here.
const int *sort_fault_flag() {
    // the flag's device address, asked once per device under a lock (host threads may sort at the same time)
    static std::mutex lock;
    static const int *addr[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> guard(lock);
    if (!addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sort_fault) != cudaSuccess) return nullptr;
        addr[dev] = static_cast<const int *>(p);
    }
    return addr[dev];
}

int sort_fault_seen(int fault) {
    if (!fault) return BS_OK;
    const int zero = 0;
    cudaMemcpyToSymbol(g_sort_fault, &zero, sizeof(int));
    set_error("radix sort: a look-back wait ran out (the sorted order is not valid)");
    return BS_ERR_TIMEOUT;
}

int check_sort_fault() {
    int fault = 0;
    BS_CUDA(cudaMemcpyFromSymbol(&fault, g_sort_fault, sizeof(int)));
    if (!fault) return BS_OK;
    const int zero = 0;
    cudaMemcpyToSymbol(g_sort_fault, &zero, sizeof(int));
    set_error("radix sort: a look-back wait ran out (the sorted order is not valid)");
    return BS_ERR_TIMEOUT;
}

}  // namespace bs
