// Host -> device upload from ordinary (pageable) host memory through a pinned staging ring.  The caller's bytes are
// copied into 4 MiB pinned chunks by OpenMP threads while the chunks before them cross PCIe (cudaMemcpyAsync on the
// caller's stream), so host copying and transfer overlap and the copy runs on several cores.  The call returns when
// the source has been read; the last transfers may still be in flight on the stream.
#include <omp.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "bs_internal.cuh"

struct bs_upload_ring {
    static constexpr int SLOTS = 4;
    static constexpr size_t CHUNK = size_t(4) << 20;
    void *buf[SLOTS] = {};
    cudaEvent_t done[SLOTS] = {};
    std::mutex lock;
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
    for (int i = 0; i < bs_upload_ring::SLOTS; ++i) {
        cudaEventSynchronize(ctx->upload->done[i]);
        cudaEventDestroy(ctx->upload->done[i]);
        cudaFreeHost(ctx->upload->buf[i]);
    }
    delete ctx->upload;
    ctx->upload = nullptr;
}

extern "C" int bs_upload(bs_ctx *ctx, void *dst, const void *src, size_t bytes, bs_stream stream) {
    if (!ctx || (bytes > 0 && (!dst || !src))) {
        bs::set_error("bs_upload: null argument");
        return BS_ERR_ARG;
    }
    if (bytes == 0) return BS_OK;
    BS_CUDA(cudaSetDevice(ctx->device));
    bs_upload_ring *r = nullptr;
    int rc = ring_of(ctx, &r);
    if (rc != BS_OK) return rc;
    std::lock_guard<std::mutex> guard(r->lock);
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = std::max(1, std::min(8, omp_get_max_threads()));
    const char *from = static_cast<const char *>(src);
    char *to = static_cast<char *>(dst);
    int k = 0;
    for (size_t off = 0; off < bytes; off += bs_upload_ring::CHUNK, ++k) {
        const int slot = k % bs_upload_ring::SLOTS;
        BS_CUDA(cudaEventSynchronize(r->done[slot]));  // the slot's previous transfer has left it
        const size_t len = std::min(bs_upload_ring::CHUNK, bytes - off);
        char *stage = static_cast<char *>(r->buf[slot]);
        const size_t piece = (len + threads - 1) / threads;
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int i = 0; i < threads; ++i) {
            const size_t a = std::min(len, (size_t)i * piece), b = std::min(len, a + piece);
            if (b > a) std::memcpy(stage + a, from + off + a, b - a);
        }
        BS_CUDA(cudaMemcpyAsync(to + off, stage, len, cudaMemcpyHostToDevice, s));
        BS_CUDA(cudaEventRecord(r->done[slot], s));
    }
    return BS_OK;
}
