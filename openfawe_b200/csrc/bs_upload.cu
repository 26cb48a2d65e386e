// Host -> device upload from ordinary (pageable) host memory through a pinned staging ring.  The caller's bytes are
// copied into 4 MiB pinned chunks by OpenMP threads (non-temporal stores where the CPU has AVX2) while the chunks
// before them cross PCIe (cudaMemcpyAsync on the caller's stream), so host copying and transfer overlap and the copy
// runs on several cores.  The call returns when the sources have been read; the last transfers may still be in flight
// on the stream.  bs_upload_many keeps the ring going across several arrays; bs_download_many runs it the other way.
#include <immintrin.h>
#include <omp.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "bs_internal.cuh"

struct bs_upload_ring {
    static constexpr int SLOTS = 4;
    static constexpr size_t CHUNK = size_t(4) << 20;
    void *buf[SLOTS] = {};
    cudaEvent_t done[SLOTS] = {};
    std::mutex lock;
    // a persistent host thread for uploads that overlap the caller's own work (its OpenMP team stays alive)
    std::thread worker;
    std::mutex wm;
    std::condition_variable wcv;
    std::function<int()> job;
    bool pending = false, quit = false;
    int result = BS_OK;
};

static int ring_of(bs_ctx *ctx, bs_upload_ring **out) {
    static std::mutex create;
    std::lock_guard<std::mutex> guard(create);
    if (!ctx->upload) {
        bs_upload_ring *r = new bs_upload_ring();
        for (int i = 0; i < bs_upload_ring::SLOTS; ++i) {
            cudaError_t e = cudaHostAlloc(&r->buf[i], bs_upload_ring::CHUNK, cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->done[i], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                for (int j = 0; j <= i; ++j) {
                    if (r->buf[j]) cudaFreeHost(r->buf[j]);
                    if (r->done[j]) cudaEventDestroy(r->done[j]);
                }
                delete r;
                return bs::cuda_fail(e, "bs_upload staging");
            }
        }
        ctx->upload = r;
    }
    *out = ctx->upload;
    return BS_OK;
}

void bs_upload_release(bs_ctx *ctx) {
    if (!ctx || !ctx->upload) return;
    if (ctx->upload->worker.joinable()) {
        {
            std::lock_guard<std::mutex> g(ctx->upload->wm);
            ctx->upload->quit = true;
        }
        ctx->upload->wcv.notify_all();
        ctx->upload->worker.join();
    }
    for (int i = 0; i < bs_upload_ring::SLOTS; ++i) {
        cudaEventSynchronize(ctx->upload->done[i]);
        cudaEventDestroy(ctx->upload->done[i]);
        cudaFreeHost(ctx->upload->buf[i]);
    }
    delete ctx->upload;
    ctx->upload = nullptr;
}

// Copy of one staging piece: AVX2 non-temporal stores where the CPU has them (the staging buffer is then written
// without being read into the cache first, which leaves the host's memory bandwidth to the transfers), else memcpy.
__attribute__((target("avx2"))) static void stream_copy_avx2(char *dst, const char *src, size_t n) {
    size_t i = 0;
    if ((reinterpret_cast<uintptr_t>(dst) & 31) == 0) {
        for (; i + 128 <= n; i += 128) {
            const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i));
            const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i + 32));
            const __m256i c = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i + 64));
            const __m256i d = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + i + 96));
            _mm256_stream_si256(reinterpret_cast<__m256i *>(dst + i), a);
            _mm256_stream_si256(reinterpret_cast<__m256i *>(dst + i + 32), b);
            _mm256_stream_si256(reinterpret_cast<__m256i *>(dst + i + 64), c);
            _mm256_stream_si256(reinterpret_cast<__m256i *>(dst + i + 96), d);
        }
        _mm_sfence();
    }
    if (i < n) std::memcpy(dst + i, src + i, n - i);
}

static void stage_copy(char *dst, const char *src, size_t n, bool avx2) {
    if (avx2) stream_copy_avx2(dst, src, n);
    else std::memcpy(dst, src, n);
}

// One ring pass over several host -> device copies: the chunk counter runs on across the arrays, so the next array's
// first chunk is staged while the previous array's last chunks transfer.
static int upload_list(bs_ctx *ctx, int count, void *const *dst, const void *const *src, const size_t *bytes,
                       cudaStream_t s) {
    BS_CUDA(cudaSetDevice(ctx->device));
    bs_upload_ring *r = nullptr;
    int rc = ring_of(ctx, &r);
    if (rc != BS_OK) return rc;
    std::lock_guard<std::mutex> guard(r->lock);
    static const bool avx2 = __builtin_cpu_supports("avx2");
    const int threads = std::max(1, std::min(8, omp_get_max_threads()));
    int k = 0;
    for (int a = 0; a < count; ++a) {
        const char *from = static_cast<const char *>(src[a]);
        char *to = static_cast<char *>(dst[a]);
        for (size_t off = 0; off < bytes[a]; off += bs_upload_ring::CHUNK, ++k) {
            const int slot = k % bs_upload_ring::SLOTS;
            BS_CUDA(cudaEventSynchronize(r->done[slot]));  // the slot's previous transfer has left it
            const size_t len = std::min(bs_upload_ring::CHUNK, bytes[a] - off);
            char *stage = static_cast<char *>(r->buf[slot]);
            const size_t piece = ((len + threads - 1) / threads + 127) & ~size_t(127);  // 128-byte aligned pieces
#pragma omp parallel for num_threads(threads) schedule(static)
            for (int i = 0; i < threads; ++i) {
                const size_t lo = std::min(len, (size_t)i * piece), hi = std::min(len, lo + piece);
                if (hi > lo) stage_copy(stage + lo, from + off + lo, hi - lo, avx2);
            }
            BS_CUDA(cudaMemcpyAsync(to + off, stage, len, cudaMemcpyHostToDevice, s));
            BS_CUDA(cudaEventRecord(r->done[slot], s));
        }
    }
    return BS_OK;
}

extern "C" int bs_upload(bs_ctx *ctx, void *dst, const void *src, size_t bytes, bs_stream stream) {
    if (!ctx || (bytes > 0 && (!dst || !src))) {
        bs::set_error("bs_upload: null argument");
        return BS_ERR_ARG;
    }
    if (bytes == 0) return BS_OK;
    return upload_list(ctx, 1, &dst, &src, &bytes, (cudaStream_t)stream);
}

extern "C" int bs_upload_many(bs_ctx *ctx, int count, void *const *dst, const void *const *src, const size_t *bytes,
                              bs_stream stream) {
    if (!ctx || count < 0 || (count > 0 && (!dst || !src || !bytes))) {
        bs::set_error("bs_upload_many: null argument");
        return BS_ERR_ARG;
    }
    for (int a = 0; a < count; ++a)
        if (bytes[a] > 0 && (!dst[a] || !src[a])) {
            bs::set_error("bs_upload_many: null pointer for copy %d", a);
            return BS_ERR_ARG;
        }
    if (count == 0) return BS_OK;
    return upload_list(ctx, count, dst, src, bytes, (cudaStream_t)stream);
}

// Device -> host through the same ring: chunk k's transfer into a pinned slot is in flight while the host copies chunk
// k - 1 out of its slot (OpenMP threads for large chunks).  Returns when every byte is in the host buffers.
extern "C" int bs_download_many(bs_ctx *ctx, int count, void *const *dst, const void *const *src, const size_t *bytes,
                                bs_stream stream) {
    if (!ctx || count < 0 || (count > 0 && (!dst || !src || !bytes))) {
        bs::set_error("bs_download_many: null argument");
        return BS_ERR_ARG;
    }
    for (int a = 0; a < count; ++a)
        if (bytes[a] > 0 && (!dst[a] || !src[a])) {
            bs::set_error("bs_download_many: null pointer for copy %d", a);
            return BS_ERR_ARG;
        }
    if (count == 0) return BS_OK;
    BS_CUDA(cudaSetDevice(ctx->device));
    bs_upload_ring *r = nullptr;
    int rc = ring_of(ctx, &r);
    if (rc != BS_OK) return rc;
    std::lock_guard<std::mutex> guard(r->lock);
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = std::max(1, std::min(8, omp_get_max_threads()));
    struct Pending {
        char *to;
        int slot;
        size_t len;
    };
    Pending pending[bs_upload_ring::SLOTS] = {};
    int head = 0, queued = 0, k = 0;
    auto drain_one = [&]() -> int {
        const Pending p = pending[head];
        head = (head + 1) % bs_upload_ring::SLOTS;
        --queued;
        BS_CUDA(cudaEventSynchronize(r->done[p.slot]));
        const char *stage = static_cast<const char *>(r->buf[p.slot]);
        if (p.len >= (size_t(256) << 10) && threads > 1) {
            const size_t piece = (p.len + threads - 1) / threads;
#pragma omp parallel for num_threads(threads) schedule(static)
            for (int i = 0; i < threads; ++i) {
                const size_t lo = std::min(p.len, (size_t)i * piece), hi = std::min(p.len, lo + piece);
                if (hi > lo) std::memcpy(p.to + lo, stage + lo, hi - lo);
            }
        } else {
            std::memcpy(p.to, stage, p.len);
        }
        return BS_OK;
    };
    for (int a = 0; a < count; ++a) {
        const char *from = static_cast<const char *>(src[a]);
        char *to = static_cast<char *>(dst[a]);
        for (size_t off = 0; off < bytes[a]; off += bs_upload_ring::CHUNK, ++k) {
            if (queued == bs_upload_ring::SLOTS) {
                rc = drain_one();
                if (rc != BS_OK) return rc;
            }
            const int slot = k % bs_upload_ring::SLOTS;
            BS_CUDA(cudaEventSynchronize(r->done[slot]));  // an upload may still be reading the slot
            const size_t len = std::min(bs_upload_ring::CHUNK, bytes[a] - off);
            BS_CUDA(cudaMemcpyAsync(r->buf[slot], from + off, len, cudaMemcpyDeviceToHost, s));
            BS_CUDA(cudaEventRecord(r->done[slot], s));
            pending[(head + queued) % bs_upload_ring::SLOTS] = Pending{to + off, slot, len};
            ++queued;
        }
    }
    while (queued > 0) {
        rc = drain_one();
        if (rc != BS_OK) return rc;
    }
    return BS_OK;
}

// The staging thread: runs one submitted upload at a time.
static void stage_worker(bs_upload_ring *r) {
    for (;;) {
        std::function<int()> job;
        {
            std::unique_lock<std::mutex> g(r->wm);
            r->wcv.wait(g, [&] { return r->quit || (r->pending && r->job); });
            if (r->quit) return;
            job = std::move(r->job);
            r->job = nullptr;
        }
        const int rc = job();
        {
            std::lock_guard<std::mutex> g(r->wm);
            r->result = rc;
            r->pending = false;
        }
        r->wcv.notify_all();
    }
}

int bs_stage_async(bs_ctx *ctx, int count, void *const *dst, const void *const *src, const size_t *bytes,
                   cudaStream_t s) {
    bs_upload_ring *r = nullptr;
    int rc = ring_of(ctx, &r);
    if (rc != BS_OK) return rc;
    std::vector<void *> d(dst, dst + count);
    std::vector<const void *> f(src, src + count);
    std::vector<size_t> b(bytes, bytes + count);
    std::unique_lock<std::mutex> g(r->wm);
    r->wcv.wait(g, [&] { return !r->pending; });
    if (!r->worker.joinable()) r->worker = std::thread(stage_worker, r);
    r->job = [ctx, d, f, b, s]() { return upload_list(ctx, (int)d.size(), d.data(), f.data(), b.data(), s); };
    r->pending = true;
    g.unlock();
    r->wcv.notify_all();
    return BS_OK;
}

int bs_stage_wait(bs_ctx *ctx) {
    bs_upload_ring *r = ctx->upload;
    if (!r) return BS_OK;
    std::unique_lock<std::mutex> g(r->wm);
    r->wcv.wait(g, [&] { return !r->pending; });
    return r->result;
}

