// Exclusive scan and stable least-significant-digit radix sort for the tree builds.
//
// Radix sort: 8-bit digits, one histogram kernel and one scatter kernel per pass, the per-(digit, tile) counts scanned in
// digit-major order so that equal digits keep their input order across tiles; inside a tile the rank of an element
// among equal digits comes from __match_any_sync and per-warp counters, in input order, so every pass is stable.
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
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;

__global__ void __launch_bounds__(RS_THREADS) radix_hist_kernel(const uint64_t *keys, int64_t n, int shift,
                                                                int64_t tiles, int64_t *counts) {
    __shared__ int hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int i = 0; i < RS_ITEMS; ++i) {
        int64_t idx = base + (int64_t)i * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&hist[(keys[idx] >> shift) & 255], 1);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = hist[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS) radix_scatter_kernel(const uint64_t *keys_in, const int32_t *vals_in,
                                                                   uint64_t *keys_out, int32_t *vals_out, int64_t n,
                                                                   int shift, int64_t tiles,
                                                                   const int64_t *offsets) {
    __shared__ int64_t base[256];
    __shared__ int wcount[RS_WARPS][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    base[tid] = offsets[(int64_t)tid * tiles + blockIdx.x];
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) wcount[w][tid] = 0;
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    int64_t tile0 = (int64_t)blockIdx.x * RS_TILE;
    for (int round = 0; round < RS_ITEMS; ++round) {
        int64_t idx = tile0 + (int64_t)round * RS_THREADS + tid;
        bool valid = idx < n;
        uint64_t key = valid ? keys_in[idx] : 0;
        int32_t val = valid ? vals_in[idx] : 0;
        int digit = valid ? (int)((key >> shift) & 255) : 256;
        unsigned peers = __match_any_sync(0xffffffffu, digit);
        int rank = __popc(peers & lt);
        if (valid && rank == 0) wcount[warp][digit] = __popc(peers);
        __syncthreads();
        {
            int64_t run = base[tid];
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) {
                int c = wcount[w][tid];
                wcount[w][tid] = (int)(run - base[tid]);
                run += c;
            }
            // keep the per-round prefix relative to base[tid]; base advances after everyone has read
            __syncthreads();
            if (valid) {
                int64_t pos = base[digit] + wcount[warp][digit] + rank;
                keys_out[pos] = key;
                vals_out[pos] = val;
            }
            __syncthreads();
            base[tid] = run;
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) wcount[w][tid] = 0;
            __syncthreads();
        }
    }
}

int radix_sort(uint64_t *keys, int32_t *vals, int64_t n, int begin_bit, int end_bit, Scratch &scratch,
               cudaStream_t s) {
    if (n <= 1 || end_bit <= begin_bit) return BS_OK;
    int64_t tiles = (n + RS_TILE - 1) / RS_TILE;
    uint64_t *k2 = scratch.get<uint64_t>(n);
    int32_t *v2 = scratch.get<int32_t>(n);
    int64_t *counts = scratch.get<int64_t>(256 * tiles);
    if (!k2 || !v2 || !counts) return scratch.status;
    uint64_t *ka = keys, *kb = k2;
    int32_t *va = vals, *vb = v2;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8, ++passes) {
        radix_hist_kernel<<<(unsigned)tiles, RS_THREADS, 0, s>>>(ka, n, shift, tiles, counts);
        BS_CHECK_LAUNCH("radix_hist_kernel");
        int rc = scan_exclusive(counts, counts, 256 * tiles, nullptr, scratch, s);
        if (rc != BS_OK) return rc;
        radix_scatter_kernel<<<(unsigned)tiles, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, tiles, counts);
        BS_CHECK_LAUNCH("radix_scatter_kernel");
        uint64_t *kt = ka; ka = kb; kb = kt;
        int32_t *vt = va; va = vb; vb = vt;
    }
    if (passes & 1) {
        BS_CUDA(cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        BS_CUDA(cudaMemcpyAsync(vals, va, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    }
    return BS_OK;
}

}  // namespace bs
