// Exact direct sum on the GPU: vortex_numba._sum_point (src/openfawe/aero/vortex_numba.py:112-147) for every target,
// the reference GPU kernel's job (src/openfawe/aero/vortex_cuda.py:179-351).
//
// One thread per target; the segments are cut into contiguous chunks (grid.y) so that small target counts still fill
// the 148 SMs, and each chunk streams its segment records through shared memory in tiles moved by the TMA unit
// (cp.async.bulk, double buffered, mbarrier completion).  Inside a chunk every thread walks its segments in input order,
// skipping its excluded segments with a cursor into the sorted exclusion CSR, and keeps the first flag; chunk partials
// are combined in chunk order, so a target's flag is the first in segment order as in the reference.
// Precisions: BS_FP64 evaluates every pair in FP64; BS_MIXED/BS_FP32 evaluate pairs in FP32 on two-float coordinates,
// re-evaluate in FP64 the pairs within near_cores core radii of a segment, near its axis or out of FP32 range, and
// add each tile's FP32 partial to an FP64 (mixed) or FP32 (fp32) per-target sum.
#include <algorithm>

#include "bs_tree.cuh"

namespace bs {

template <int PREC> struct TileOf { using T = Seg32; static constexpr int N = 256; };
template <> struct TileOf<0> { using T = Seg64; static constexpr int N = 128; };

struct DirectArgs {
    int64_t n, m, chunk_len;
    const double *points;
    const int64_t *ex_ptr, *ex_seg;
    const Seg64 *seg64;
    const Seg32 *seg32;
    int model, raise_singular;
    float near2;
    double *out;        // final output (one chunk) or partials [chunks][n][3]
    int8_t *flags;      // final flags or partial flags [chunks][n]
    int *error;         // bounded-wait failures
    unsigned long long *fp64_pairs;
};

template <int PREC, int MODEL>
__global__ void __launch_bounds__(256) direct_kernel(DirectArgs a) {
    using Rec = typename TileOf<PREC>::T;
    constexpr int TILE = TileOf<PREC>::N;
    __shared__ __align__(128) Rec tile[2][TILE];
    __shared__ __align__(8) uint64_t bar[2];
    const int tid = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + tid;
    const bool valid = i < a.n;
    const int64_t c0 = (int64_t)blockIdx.y * a.chunk_len;
    const int64_t c1 = min(a.m, c0 + a.chunk_len);
    const Rec *src = PREC == 0 ? (const Rec *)a.seg64 : (const Rec *)a.seg32;

    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
    if (valid) { x0 = a.points[3 * i]; x1 = a.points[3 * i + 1]; x2 = a.points[3 * i + 2]; }
    float xh0, xl0, xh1, xl1, xh2, xl2;
    split2(x0, xh0, xl0);
    split2(x1, xh1, xl1);
    split2(x2, xh2, xl2);
    // exclusion cursor: first excluded segment >= c0
    int64_t k = 0, stop = 0;
    if (valid && a.ex_ptr) {
        int64_t lo = a.ex_ptr[i], hi = a.ex_ptr[i + 1];
        stop = hi;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (a.ex_seg[mid] < c0) lo = mid + 1; else hi = mid;
        }
        k = lo;
    }
    int64_t next_ex = k < stop ? a.ex_seg[k] : INT64_MAX;

    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;
    int flag = BS_FLAG_OK;
    long long fp64_pairs = 0;

    const int64_t count = c1 - c0;
    const int ntiles = count > 0 ? (int)((count + TILE - 1) / TILE) : 0;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int t = 0; t < 2 && t < ntiles; ++t) {
            int64_t base = c0 + (int64_t)t * TILE;
            uint32_t bytes = (uint32_t)(min((int64_t)TILE, c1 - base) * sizeof(Rec));
            mbar_arrive_tx(&bar[t], bytes);
            bulk_load(tile[t], src + base, bytes, &bar[t]);
        }
    }
    bool failed = false;
    for (int t = 0; t < ntiles; ++t) {
        const int b = t & 1;
        if (!mbar_wait(&bar[b], (t >> 1) & 1)) failed = true;
        const int64_t base = c0 + (int64_t)t * TILE;
        const int cnt = (int)min((int64_t)TILE, c1 - base);
        if (valid && !failed) {
            for (int sub = 0; sub < cnt; sub += 32) {
                const int sc = min(32, cnt - sub);
                const int64_t s0 = base + sub;
                unsigned excl = 0;  // this target's excluded segments inside the sub-tile
                while (next_ex < s0 + sc) {
                    excl |= 1u << (int)(next_ex - s0);
                    ++k;
                    next_ex = k < stop ? a.ex_seg[k] : INT64_MAX;
                }
                if (PREC == 0) {
                    for (int j = 0; j < sc; ++j) {
                        if ((excl >> j) & 1u) continue;
                        const Seg64 &r = reinterpret_cast<const Seg64 &>(tile[b][sub + j]);
                        int fl = pair64_at(x0, x1, x2, r, a.model, a.raise_singular, u0, u1, u2);
                        if (fl != BS_FLAG_OK && flag == BS_FLAG_OK) flag = fl;
                    }
                    continue;
                }
                float t0 = 0.f, t1 = 0.f, t2 = 0.f;
                unsigned need = 0;
                if (excl == 0) {  // the common case: every pair of the sub-tile counts
#pragma unroll 4
                    for (int j = 0; j < sc; ++j) {
                        const Seg32 &r = reinterpret_cast<const Seg32 &>(tile[b][sub + j]);
                        const float q0 = (xh0 - r.hi.x) + (xl0 - r.lo.x);
                        const float q1 = (xh1 - r.hi.y) + (xl1 - r.lo.y);
                        const float q2 = (xh2 - r.hi.z) + (xl2 - r.lo.z);
                        if (pair32<MODEL>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1u << j;
                    }
                } else {
                    for (int j = 0; j < sc; ++j) {
                        if ((excl >> j) & 1u) continue;
                        const Seg32 &r = reinterpret_cast<const Seg32 &>(tile[b][sub + j]);
                        const float q0 = (xh0 - r.hi.x) + (xl0 - r.lo.x);
                        const float q1 = (xh1 - r.hi.y) + (xl1 - r.lo.y);
                        const float q2 = (xh2 - r.hi.z) + (xl2 - r.lo.z);
                        if (pair32<MODEL>(q0, q1, q2, r.hi, r.lo, r.dir, a.near2, t0, t1, t2)) need |= 1u << j;
                    }
                }
                fp64_pairs += __popc(need);
                while (need) {
                    const int j = __ffs(need) - 1;
                    need &= need - 1;
                    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
                    int fl = pair64_at(x0, x1, x2, a.seg64[s0 + j], MODEL, a.raise_singular, v0, v1, v2);
                    if (fl != BS_FLAG_OK) {
                        if (flag == BS_FLAG_OK) flag = fl;
                    } else if (PREC == 1) {
                        u0 += v0; u1 += v1; u2 += v2;
                    } else {
                        f0 += (float)v0; f1 += (float)v1; f2 += (float)v2;
                    }
                }
                if (PREC == 1) { u0 += t0; u1 += t1; u2 += t2; }
                else { f0 += t0; f1 += t1; f2 += t2; }
            }
        }
        __syncthreads();  // every thread is done with tile[b]
        if (tid == 0 && t + 2 < ntiles && !failed) {
            int64_t nb = c0 + (int64_t)(t + 2) * TILE;
            uint32_t bytes = (uint32_t)(min((int64_t)TILE, c1 - nb) * sizeof(Rec));
            mbar_arrive_tx(&bar[b], bytes);
            bulk_load(tile[b], src + nb, bytes, &bar[b]);
        }
    }
    if (failed) {
        atomicExch(a.error, 1);
        // wait (bounded) for copies this block still has in flight before the block exits
        for (int t = max(0, ntiles - 2); t < ntiles; ++t) mbar_wait(&bar[t & 1], (t >> 1) & 1);
    }
    if (PREC == 2) { u0 = f0; u1 = f1; u2 = f2; }
    if (valid) {
        if (gridDim.y == 1 && !(isfinite(u0) && isfinite(u1) && isfinite(u2)) && flag == BS_FLAG_OK)
            flag = BS_FLAG_NONFINITE;
        const int64_t o = (int64_t)blockIdx.y * a.n + i;
        a.out[3 * o] = u0;
        a.out[3 * o + 1] = u1;
        a.out[3 * o + 2] = u2;
        a.flags[o] = (int8_t)flag;
    }
    if (PREC != 0) {
        for (int o = 16; o > 0; o >>= 1) fp64_pairs += __shfl_xor_sync(0xffffffffu, fp64_pairs, o);
        if ((tid & 31) == 0 && fp64_pairs) atomicAdd(a.fp64_pairs, (unsigned long long)fp64_pairs);
    }
}

// Chunk partials -> result: sums in chunk order, first flag in chunk (= segment) order, then the finite check.
__global__ void direct_reduce_kernel(int64_t n, int chunks, const double *partial, const int8_t *pflags, double *out,
                                     int8_t *flags) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    int flag = BS_FLAG_OK;
    for (int c = 0; c < chunks; ++c) {
        int64_t o = (int64_t)c * n + i;
        u0 += partial[3 * o];
        u1 += partial[3 * o + 1];
        u2 += partial[3 * o + 2];
        if (flag == BS_FLAG_OK) flag = pflags[o];
    }
    if (!(isfinite(u0) && isfinite(u1) && isfinite(u2)) && flag == BS_FLAG_OK) flag = BS_FLAG_NONFINITE;
    out[3 * i] = u0;
    out[3 * i + 1] = u1;
    out[3 * i + 2] = u2;
    flags[i] = (int8_t)flag;
}

}  // namespace bs

using namespace bs;

template <int PREC>
static void launch_model(int model, dim3 grid, int block, cudaStream_t s, const DirectArgs &args) {
    switch (model) {
        case 0: direct_kernel<PREC, 0><<<grid, block, 0, s>>>(args); break;
        case 1: direct_kernel<PREC, 1><<<grid, block, 0, s>>>(args); break;
        case 2: direct_kernel<PREC, 2><<<grid, block, 0, s>>>(args); break;
        case 3: direct_kernel<PREC, 3><<<grid, block, 0, s>>>(args); break;
        case 4: direct_kernel<PREC, 4><<<grid, block, 0, s>>>(args); break;
        default: direct_kernel<PREC, 5><<<grid, block, 0, s>>>(args); break;
    }
}

// FP64 evaluates the core model at run time; the single precisions are specialised per model.
static void launch_direct(int precision, int model, dim3 grid, int block, cudaStream_t s, const DirectArgs &args) {
    if (precision == BS_FP64) direct_kernel<0, 0><<<grid, block, 0, s>>>(args);
    else if (precision == BS_MIXED) launch_model<1>(model, grid, block, s, args);
    else launch_model<2>(model, grid, block, s, args);
}

// Chunks so that (target blocks) x (chunks) covers the SMs several times, each chunk a whole number of tiles.
static int choose_chunks(int64_t n, int64_t m, int block, int tile, int sm_count) {
    int64_t target_blocks = (n + block - 1) / block;
    int64_t want = (int64_t)sm_count * 8;
    int64_t chunks = (want + target_blocks - 1) / target_blocks;
    int64_t max_chunks = std::max<int64_t>(1, (m + tile - 1) / tile);
    chunks = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(chunks, max_chunks), 4096));
    return (int)chunks;
}

extern "C" int bs_direct(bs_ctx *ctx, const bs_sources *src, const bs_targets *tgt, const bs_kernel_params *kp,
                         double *out, int8_t *flags, bs_stream stream) {
    if (!ctx || !src || !tgt || !kp || (tgt->n > 0 && (!tgt->points || !out || !flags))) {
        set_error("bs_direct: null argument");
        return BS_ERR_ARG;
    }
    if (kp->model < 0 || kp->model > 5 || kp->precision < 0 || kp->precision > 2 ||
        (kp->block != 32 && kp->block != 64 && kp->block != 128 && kp->block != 256)) {
        set_error("bs_direct: model 0..5, precision 0..2, block 32/64/128/256");
        return BS_ERR_ARG;
    }
    if (src->m < 0 || (src->m > 0 && (!src->starts || !src->directions || !src->lengths || !src->gamma ||
                                       !src->radius))) {
        set_error("bs_direct: invalid segment arrays");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    const int64_t n = tgt->n, m = src->m;
    if (n == 0) return BS_OK;
    if (m == 0) {
        BS_CUDA(cudaMemsetAsync(out, 0, n * 3 * sizeof(double), s));
        BS_CUDA(cudaMemsetAsync(flags, 0, n, s));
        return BS_OK;
    }
    Scratch scratch(ctx->pool, s);
    const int prec = kp->precision;
    Seg64 *seg64 = scratch.get<Seg64>(m);
    Seg32 *seg32 = prec != BS_FP64 ? scratch.get<Seg32>(m) : nullptr;
    int *error = scratch.get<int>(1);
    unsigned long long *fp64_pairs = scratch.get<unsigned long long>(1);
    if (!seg64 || (prec != BS_FP64 && !seg32) || !error || !fp64_pairs) return scratch.status;
    int rc = pack_segments(src, nullptr, seg64, seg32, nullptr, s);
    if (rc != BS_OK) return rc;
    BS_CUDA(cudaMemsetAsync(error, 0, sizeof(int), s));
    BS_CUDA(cudaMemsetAsync(fp64_pairs, 0, sizeof(unsigned long long), s));
    const int block = kp->block;
    const int tile = prec == BS_FP64 ? TileOf<0>::N : TileOf<1>::N;
    int chunks = choose_chunks(n, m, block, tile, ctx->sm_count);
    int64_t chunk_len = (m + chunks - 1) / chunks;
    chunk_len = (chunk_len + tile - 1) / tile * tile;
    chunks = (int)((m + chunk_len - 1) / chunk_len);
    double *partial = out;
    int8_t *pflags = flags;
    if (chunks > 1) {
        partial = scratch.get<double>((size_t)3 * n * chunks);
        pflags = scratch.get<int8_t>((size_t)n * chunks);
        if (!partial || !pflags) return scratch.status;
    }
    DirectArgs args;
    args.n = n;
    args.m = m;
    args.chunk_len = chunk_len;
    args.points = tgt->points;
    args.ex_ptr = (tgt->ex_ptr && tgt->e > 0) ? tgt->ex_ptr : nullptr;
    args.ex_seg = tgt->ex_seg;
    args.seg64 = seg64;
    args.seg32 = seg32;
    args.model = kp->model;
    args.raise_singular = kp->raise_singular ? 1 : 0;
    args.near2 = (float)(kp->near_cores * kp->near_cores);
    args.out = partial;
    args.flags = pflags;
    args.error = error;
    args.fp64_pairs = fp64_pairs;
    dim3 grid((unsigned)((n + block - 1) / block), (unsigned)chunks);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    launch_direct(prec, kp->model, grid, block, s, args);
    cudaError_t le = cudaGetLastError();
    if (le == cudaSuccess && chunks > 1) {
        direct_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, chunks, partial, pflags, out, flags);
        le = cudaGetLastError();
    }
    cudaEventRecord(e1, s);
    int host_error = 0;
    unsigned long long host_fp64 = 0;
    if (le == cudaSuccess) le = cudaMemcpyAsync(&host_error, error, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (le == cudaSuccess) le = cudaMemcpyAsync(&host_fp64, fp64_pairs, sizeof host_fp64, cudaMemcpyDeviceToHost, s);
    if (le == cudaSuccess) le = cudaStreamSynchronize(s);
    float ms = 0.f;
    if (le == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (le != cudaSuccess) return cuda_fail(le, "direct_kernel");
    ctx->stats.points = n;
    ctx->stats.segments = m;
    ctx->stats.nodes = 0;
    ctx->stats.launches = chunks > 1 ? 2 : 1;
    ctx->stats.near_pairs = n * m;
    ctx->stats.fp64_pairs = (int64_t)host_fp64;
    ctx->stats.far_evaluations = 0;
    ctx->stats.visits = 0;
    ctx->stats.evaluate_ms = ms;
    if (host_error) {
        set_error("bs_direct: a bounded wait for a segment tile gave up");
        return BS_ERR_TIMEOUT;
    }
    return BS_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// Allocation-free variant of bs_direct.
//
// For hosts that must not allocate GPU memory while they run -- a flight or control loop with a hard per-step
// deadline (an allocation can stall on the driver or fail once a framework's caching allocator has reserved the device),
// or a plugin loaded into a host program that owns all device memory -- the segment records live in one fixed array
// inside this library instead of the context's memory pool.  The array is a file-scope __device__ variable, so every
// GPU that loads the library holds it (BS_NOALLOC_SCRATCH_BYTES) until the process exits; host code must not use its
// name as a device address and asks the runtime for the address instead (cudaGetSymbolAddress, once per device).
// ---------------------------------------------------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr size_t kNoAllocSeg64 = (size_t)BS_NOALLOC_MAX_SEGMENTS * sizeof(bs::Seg64);
constexpr size_t kNoAllocSeg32 = (size_t)BS_NOALLOC_MAX_SEGMENTS * sizeof(bs::Seg32);
static_assert(kNoAllocSeg64 + kNoAllocSeg32 + 256 == BS_NOALLOC_SCRATCH_BYTES, "scratch layout");

__device__ __align__(256) unsigned char g_noalloc_scratch[BS_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_lock;
void *g_noalloc_base[kMaxDevices];  // device address of g_noalloc_scratch on each device, set on first use

}  // namespace

extern "C" int bs_direct_noalloc(const bs_sources *src, const bs_targets *tgt, const bs_kernel_params *kp,
                                 double *out, int8_t *flags, bs_stream stream) {
    if (!src || !tgt || !kp || (tgt->n > 0 && (!tgt->points || !out || !flags))) {
        set_error("bs_direct_noalloc: null argument");
        return BS_ERR_ARG;
    }
    if (kp->model < 0 || kp->model > 5 || kp->precision < 0 || kp->precision > 2 ||
        (kp->block != 32 && kp->block != 64 && kp->block != 128 && kp->block != 256)) {
        set_error("bs_direct_noalloc: model 0..5, precision 0..2, block 32/64/128/256");
        return BS_ERR_ARG;
    }
    if (src->m < 0 || (src->m > 0 && (!src->starts || !src->directions || !src->lengths || !src->gamma ||
                                       !src->radius))) {
        set_error("bs_direct_noalloc: invalid segment arrays");
        return BS_ERR_ARG;
    }
    if (src->m > BS_NOALLOC_MAX_SEGMENTS) {
        set_error("bs_direct_noalloc: %lld segments exceed the fixed scratch of %d segments; use bs_direct",
                  (long long)src->m, BS_NOALLOC_MAX_SEGMENTS);
        return BS_ERR_ARG;
    }
    int device = 0;
    BS_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= kMaxDevices) {
        set_error("bs_direct_noalloc: device %d out of range", device);
        return BS_ERR_ARG;
    }
    // every device pointer must belong to the current device, whose copy of the array the call uses
    const void *device_pointers[] = {tgt->points, out, flags, src->starts, src->directions, src->lengths, src->gamma,
                                     src->radius};
    for (const void *ptr : device_pointers) {
        if (!ptr) continue;
        cudaPointerAttributes attr;
        if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
            cudaGetLastError();
            set_error("bs_direct_noalloc: an argument is not a CUDA pointer");
            return BS_ERR_ARG;
        }
        if (attr.type == cudaMemoryTypeDevice && attr.device != device) {
            set_error("bs_direct_noalloc: an argument lives on device %d, the current device is %d", attr.device,
                      device);
            return BS_ERR_ARG;
        }
    }
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> guard(g_noalloc_lock);
        if (!g_noalloc_base[device]) {
            // once per device, with that device current: the array's device address
            cudaError_t e = cudaGetSymbolAddress(&g_noalloc_base[device], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_base[device] = nullptr;
                return cuda_fail(e, "bs_direct_noalloc: cudaGetSymbolAddress");
            }
        }
        base = g_noalloc_base[device];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = tgt->n, m = src->m;
    if (n == 0) return BS_OK;
    if (m == 0) {
        BS_CUDA(cudaMemsetAsync(out, 0, n * 3 * sizeof(double), s));
        BS_CUDA(cudaMemsetAsync(flags, 0, n, s));
        return BS_OK;
    }
    unsigned char *bytes = static_cast<unsigned char *>(base);
    Seg64 *seg64 = reinterpret_cast<Seg64 *>(bytes);
    Seg32 *seg32 = reinterpret_cast<Seg32 *>(bytes + kNoAllocSeg64);
    int *error = reinterpret_cast<int *>(bytes + kNoAllocSeg64 + kNoAllocSeg32);
    unsigned long long *fp64_pairs = reinterpret_cast<unsigned long long *>(bytes + kNoAllocSeg64 + kNoAllocSeg32 + 64);
    // the array keeps the previous call's contents: clear the error flag and the counter
    BS_CUDA(cudaMemsetAsync(error, 0, sizeof(int), s));
    BS_CUDA(cudaMemsetAsync(fp64_pairs, 0, sizeof(unsigned long long), s));
    const int prec = kp->precision;
    int rc = pack_segments(src, nullptr, seg64, prec != BS_FP64 ? seg32 : nullptr, nullptr, s);
    if (rc != BS_OK) return rc;
    DirectArgs args;
    args.n = n;
    args.m = m;
    args.chunk_len = m;  // one chunk: no partial sums, hence no further scratch
    args.points = tgt->points;
    args.ex_ptr = (tgt->ex_ptr && tgt->e > 0) ? tgt->ex_ptr : nullptr;
    args.ex_seg = tgt->ex_seg;
    args.seg64 = seg64;
    args.seg32 = seg32;
    args.model = kp->model;
    args.raise_singular = kp->raise_singular ? 1 : 0;
    args.near2 = (float)(kp->near_cores * kp->near_cores);
    args.out = out;
    args.flags = flags;
    args.error = error;
    args.fp64_pairs = fp64_pairs;
    dim3 grid((unsigned)((n + kp->block - 1) / kp->block), 1);
    launch_direct(prec, kp->model, grid, kp->block, s, args);
    cudaError_t le = cudaGetLastError();
    int host_error = 0;
    if (le == cudaSuccess) le = cudaMemcpyAsync(&host_error, error, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (le == cudaSuccess) le = cudaStreamSynchronize(s);
    if (le != cudaSuccess) return cuda_fail(le, "bs_direct_noalloc");
    if (host_error) {
        set_error("bs_direct_noalloc: a bounded wait for a segment tile gave up");
        return BS_ERR_TIMEOUT;
    }
    return BS_OK;
}
