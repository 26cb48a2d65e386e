// Context, error text, memory pool and device probe of libbs_b200.
// The probe mirrors the reference's available() (src/openfawe/aero/vortex_cuda.py:58-77): a one-thread kernel writes
// 1.0 and the host reads it back, so a missing or broken device is reported instead of failing later.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "bs_internal.cuh"

namespace bs {

static thread_local char g_error[512] = "no error";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof g_error, fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what) {
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return e == cudaErrorMemoryAllocation ? BS_ERR_OOM : BS_ERR_CUDA;
}

__global__ void probe_kernel(double *out) { out[0] = 1.0; }

}  // namespace bs

using namespace bs;

extern "C" const char *bs_last_error(void) { return g_error; }

extern "C" int bs_version(int *major, int *minor, int *arch) {
    if (major) *major = 1;
    if (minor) *minor = 0;
    if (arch) *arch = 100;
    return BS_OK;
}

extern "C" int bs_init(int device, bs_ctx **out) {
    if (!out) {
        set_error("bs_init: null output pointer");
        return BS_ERR_ARG;
    }
    *out = nullptr;
    int count = 0;
    BS_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) {
        set_error("bs_init: device %d out of range (%d devices)", device, count);
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    BS_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        set_error("bs_init: device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
        return BS_ERR_ARG;
    }
    double *probe = nullptr;
    BS_CUDA(cudaMalloc(&probe, sizeof(double)));
    BS_CUDA(cudaMemset(probe, 0, sizeof(double)));
    probe_kernel<<<1, 1>>>(probe);
    cudaError_t e = cudaGetLastError();
    double value = 0.0;
    if (e == cudaSuccess) e = cudaMemcpy(&value, probe, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(probe);
    if (e != cudaSuccess) return cuda_fail(e, "bs_init probe kernel");
    if (value != 1.0) {
        set_error("bs_init: the probe kernel wrote %g instead of 1", value);
        return BS_ERR_CUDA;
    }
    bs_ctx *ctx = new bs_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    memset(&ctx->stats, 0, sizeof ctx->stats);
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    e = cudaMemPoolCreate(&ctx->pool, &props);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(e, "cudaMemPoolCreate");
    }
    uint64_t keep = UINT64_MAX;  // keep freed blocks cached in the pool between calls
    cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    *out = ctx;
    return BS_OK;
}

void bs_upload_release(bs_ctx *ctx);  // bs_upload.cu

extern "C" void bs_destroy(bs_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    bs_upload_release(ctx);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

extern "C" int bs_last_stats(const bs_ctx *ctx, bs_stats *stats) {
    if (!ctx || !stats) {
        set_error("bs_last_stats: null argument");
        return BS_ERR_ARG;
    }
    *stats = ctx->stats;
    return BS_OK;
}

namespace {

constexpr int PEAK_CHAINS = 8;      // independent FMA chains per thread (covers the FMA pipe's latency)
constexpr int PEAK_STEPS = 4096;    // FMAs per chain

__global__ void __launch_bounds__(256) fp32_peak_kernel(float seed, float *sink) {
    float v[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; ++c) v[c] = seed + (float)(threadIdx.x + c);
    const float a = 0.999999f, b = 1e-7f;
#pragma unroll 4
    for (int i = 0; i < PEAK_STEPS; ++i)
#pragma unroll
        for (int c = 0; c < PEAK_CHAINS; ++c) v[c] = fmaf(v[c], a, b);
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; ++c) acc += v[c];
    if (acc == 12345.678f) sink[0] = acc;  // keeps the chains live; never true for these inputs
}

}  // namespace

extern "C" int bs_fp32_peak(bs_ctx *ctx, double *tflops) {
    if (!ctx || !tflops) {
        set_error("bs_fp32_peak: null argument");
        return BS_ERR_ARG;
    }
    BS_CUDA(cudaSetDevice(ctx->device));
    float *sink = nullptr;
    BS_CUDA(cudaMalloc(&sink, sizeof(float)));
    const unsigned blocks = (unsigned)ctx->sm_count * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 0.f;
    for (int rep = 0; rep < 4; ++rep) {  // first launch warms up; the best of the rest is kept
        cudaEventRecord(e0, 0);
        fp32_peak_kernel<<<blocks, 256>>>(1.0f, sink);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(e, "bs_fp32_peak");
    const double flops = 2.0 * PEAK_CHAINS * PEAK_STEPS * (double)blocks * 256.0;
    *tflops = best > 0.f ? flops / (best * 1e-3) / 1e12 : 0.0;
    return BS_OK;
}
