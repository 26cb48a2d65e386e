// Adjoint of the direct Biot-Savart sum: gradients of L = sum_p w_p . u_p with respect to the targets x_p, both
// segment endpoints A_s, B_s and the circulations Gamma_s, for a given cotangent w.  Pair terms are recomputed, never
// stored.  The reference has no adjoint; the pair is the reference's (vortex_numba.pair_velocity,
// src/openfawe/aero/vortex_numba.py:42-109) written in its two-endpoint form, which is algebraically the same:
//   r1 = x - A, r2 = x - B, c = r1 x r2, P = |r1||r2|, d = r1.r2,
//   D = P (P + d), or P |c|^2 / (P - d) when d < 0 (the reference's rationalised branch),
//   u = Gamma/(4 pi) f(|c|^2 / (|B - A|^2 rc^2)) (|r1| + |r2|) c / D,
// with the core factor f of models 0 (none), 1 (Rankine), 2 (Lamb-Oseen with its exponent cut-off) and 3 (Vatistas),
// the offset (4) and Rosenhead-Moore (5) cores in D and the distances (bs_pair_vjp.cuh), and reverse-mode
// differentiation of that expression by hand.  Pairs on a segment's axis (the reference's roundoff guard) contribute
// nothing, as in the forward sum.
//
// One pass evaluates each pair's adjoint once (adjoint_fused_kernel): blocks tile the (target x segment) plane, target
// gradients add up over a block's segments, segment gradients over its targets, and a reduce kernel adds the block
// partials in chunk order.  Deterministic.
#include <algorithm>

#include "bs_pair_vjp.cuh"

namespace bs {

__device__ __forceinline__ bool excluded(const int64_t *ex_ptr, const int64_t *ex_seg, int64_t p, int64_t s) {
    if (!ex_ptr) return false;
    for (int64_t k = ex_ptr[p]; k < ex_ptr[p + 1]; ++k)
        if (ex_seg[k] == s) return true;
    return false;
}

constexpr int ADJ_WARPS = 8;
constexpr int ADJ_THREADS = ADJ_WARPS * 32;
constexpr int ADJ_MAX_TCHUNK = 1024;  // targets per block: their gradients live in shared memory

struct AdjArgs {
    int64_t n, m, tchunk, schunk;
    const AdjTgt *tgt;
    const AdjSeg *seg;
    const int64_t *ex_ptr, *ex_seg;
    int model;
    double *part_x;    // [segment chunks][n][3]
    double *part_seg;  // [target chunks][m][7]: gA, gB, gGamma
};

// One pass over the (target chunk x segment chunk) block of pairs computing every gradient.  Each lane owns one target
// of its warp's current group of 32 and, for the current tile of 32 segments, the accumulators of one segment: at step
// j lane l evaluates segment (l + j) mod 32 and hands that pair's segment adjoint to the segment's owner lane with
// shuffles, so no two lanes write one accumulator and no atomics are needed.  Target gradients accumulate in shared
// memory (a warp owns its groups' slots); segment accumulators of the warps are added in warp order at the end of each
// tile.  Every sum runs in a fixed order, so the result is deterministic.
__global__ void __launch_bounds__(ADJ_THREADS) adjoint_fused_kernel(AdjArgs a) {
    __shared__ double gx_acc[ADJ_MAX_TCHUNK * 3];
    __shared__ AdjSeg tile[32];
    __shared__ double red[ADJ_WARPS][7][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * a.tchunk, t1 = min(a.n, t0 + a.tchunk);
    const int64_t s0 = (int64_t)blockIdx.y * a.schunk, s1 = min(a.m, s0 + a.schunk);
    const int tn = (int)(t1 - t0), groups = (tn + 31) >> 5;
    for (int i = threadIdx.x; i < 3 * tn; i += ADJ_THREADS) gx_acc[i] = 0.0;
    for (int64_t base = s0; base < s1; base += 32) {
        const int cnt = (int)min((int64_t)32, s1 - base);
        __syncthreads();
        if (threadIdx.x < cnt) tile[threadIdx.x] = a.seg[base + threadIdx.x];
        __syncthreads();
        double sacc[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int g = warp; g < groups; g += ADJ_WARPS) {
            const int local = g * 32 + lane;
            const bool valid = local < tn;
            const int64_t p = t0 + local;
            AdjTgt t = valid ? a.tgt[p] : AdjTgt{0, 0, 0, 0, 0, 0};
            double gx0 = 0.0, gx1 = 0.0, gx2 = 0.0;
            for (int j = 0; j < 32; ++j) {
                const int si = (lane + j) & 31;
                double g1[3] = {0, 0, 0}, g2[3] = {0, 0, 0}, gg = 0.0;
                if (valid && si < cnt && !(a.ex_ptr && excluded(a.ex_ptr, a.ex_seg, p, base + si))) {
                    if (pair_vjp64(t.x, t.y, t.z, tile[si], a.model, t.wx, t.wy, t.wz, g1, g2, gg)) {
                        gx0 += g1[0] + g2[0];
                        gx1 += g1[1] + g2[1];
                        gx2 += g1[2] + g2[2];
                    }
                }
                // lane r owns segment r of the tile and receives from lane (r - j) mod 32
                const int src = (lane - j) & 31;
                sacc[0] -= __shfl_sync(0xffffffffu, g1[0], src);
                sacc[1] -= __shfl_sync(0xffffffffu, g1[1], src);
                sacc[2] -= __shfl_sync(0xffffffffu, g1[2], src);
                sacc[3] -= __shfl_sync(0xffffffffu, g2[0], src);
                sacc[4] -= __shfl_sync(0xffffffffu, g2[1], src);
                sacc[5] -= __shfl_sync(0xffffffffu, g2[2], src);
                sacc[6] += __shfl_sync(0xffffffffu, gg, src);
            }
            if (valid) {
                gx_acc[3 * local] += gx0;
                gx_acc[3 * local + 1] += gx1;
                gx_acc[3 * local + 2] += gx2;
            }
        }
        for (int k = 0; k < 7; ++k) red[warp][k][lane] = sacc[k];
        __syncthreads();
        if (threadIdx.x < cnt) {
            double *q = a.part_seg + 7 * ((int64_t)blockIdx.x * a.m + base + threadIdx.x);
            for (int k = 0; k < 7; ++k) {
                double v = 0.0;
                for (int w = 0; w < ADJ_WARPS; ++w) v += red[w][k][threadIdx.x];
                q[k] = v;
            }
        }
    }
    __syncthreads();
    double *q = a.part_x + 3 * ((int64_t)blockIdx.y * a.n + t0);
    for (int i = threadIdx.x; i < 3 * tn; i += ADJ_THREADS) q[i] = gx_acc[i];
}

__global__ void adjoint_pack_kernel(int64_t n, int64_t m, int model, const double *points, const double *cot,
                                    const double *A, const double *B, const double *gamma, const double *radius,
                                    AdjTgt *tgt, AdjSeg *seg) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) tgt[i] = AdjTgt{points[3 * i], points[3 * i + 1], points[3 * i + 2], cot[3 * i], cot[3 * i + 1],
                               cot[3 * i + 2]};
    if (i < m) {
        const double l0 = B[3 * i] - A[3 * i], l1 = B[3 * i + 1] - A[3 * i + 1], l2 = B[3 * i + 2] - A[3 * i + 2];
        const double L2 = l0 * l0 + l1 * l1 + l2 * l2, rc = radius[i];
        const double irc2L2 = (model >= 1 && model <= 3 && rc > 0.0) ? 1.0 / (L2 * rc * rc) : 0.0;
        const double rc2 = (model >= 4 && rc > 0.0) ? rc * rc : 0.0;
        seg[i] = AdjSeg{A[3 * i], A[3 * i + 1], A[3 * i + 2], B[3 * i], B[3 * i + 1], B[3 * i + 2], gamma[i], irc2L2,
                        1.0 / L2, rc2};
    }
}

__global__ void adjoint_reduce_kernel(int64_t n, int64_t m, int cx, int cs, const double *part_x,
                                      const double *part_seg, double *gx, double *gA, double *gB, double *gG) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && gx) {
        double v[3] = {0, 0, 0};
        for (int c = 0; c < cx; ++c)
            for (int k = 0; k < 3; ++k) v[k] += part_x[3 * ((int64_t)c * n + i) + k];
        for (int k = 0; k < 3; ++k) gx[3 * i + k] = v[k];
    }
    if (i < m) {
        double v[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int c = 0; c < cs; ++c)
            for (int k = 0; k < 7; ++k) v[k] += part_seg[7 * ((int64_t)c * m + i) + k];
        if (gA) for (int k = 0; k < 3; ++k) gA[3 * i + k] = v[k];
        if (gB) for (int k = 0; k < 3; ++k) gB[3 * i + k] = v[3 + k];
        if (gG) gG[i] = v[6];
    }
}

}  // namespace bs

using namespace bs;

// Target chunk: at most ADJ_MAX_TCHUNK targets (their gradients sit in shared memory); segment chunks: enough blocks
// for about eight per SM in total, each at least a few tiles long.
static void adjoint_chunks(int64_t n, int64_t m, int sm_count, int64_t &tchunk, int64_t &schunk) {
    const int64_t tc = (n + ADJ_MAX_TCHUNK - 1) / ADJ_MAX_TCHUNK;
    tchunk = (n + tc - 1) / tc;
    const int64_t want = std::max<int64_t>(1, (int64_t)sm_count * 8 / tc);
    schunk = std::max<int64_t>(128, (m + want - 1) / want);
    schunk = (schunk + 31) / 32 * 32;
}

extern "C" int bs_adjoint_direct(bs_ctx *ctx, int64_t n, const double *points, int64_t m, const double *A,
                                 const double *B, const double *gamma, const double *radius, const int64_t *ex_ptr,
                                 const int64_t *ex_seg, int64_t e, int model, const double *cotangent,
                                 double *grad_points, double *grad_A, double *grad_B, double *grad_gamma,
                                 bs_stream stream) {
    if (!ctx || n < 0 || m < 0 || (n > 0 && (!points || !cotangent)) ||
        (m > 0 && (!A || !B || !gamma || !radius))) {
        set_error("bs_adjoint_direct: null argument");
        return BS_ERR_ARG;
    }
    if (model < 0 || model > 5) {
        set_error("bs_adjoint_direct: core model must be 0..5");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    if (grad_points && n) BS_CUDA(cudaMemsetAsync(grad_points, 0, 3 * n * sizeof(double), s));
    if (grad_A && m) BS_CUDA(cudaMemsetAsync(grad_A, 0, 3 * m * sizeof(double), s));
    if (grad_B && m) BS_CUDA(cudaMemsetAsync(grad_B, 0, 3 * m * sizeof(double), s));
    if (grad_gamma && m) BS_CUDA(cudaMemsetAsync(grad_gamma, 0, m * sizeof(double), s));
    if (n == 0 || m == 0) return BS_OK;
    Scratch scratch(ctx->pool, s);
    AdjTgt *tgt = scratch.get<AdjTgt>(n);
    AdjSeg *seg = scratch.get<AdjSeg>(m);
    int64_t tchunk, schunk;
    adjoint_chunks(n, m, ctx->sm_count, tchunk, schunk);
    const int tc = (int)((n + tchunk - 1) / tchunk), sc = (int)((m + schunk - 1) / schunk);
    double *part_x = scratch.get<double>((size_t)3 * n * sc), *part_seg = scratch.get<double>((size_t)7 * m * tc);
    if (!tgt || !seg || !part_x || !part_seg) return scratch.status;
    const int64_t big = std::max(n, m);
    adjoint_pack_kernel<<<(unsigned)((big + 255) / 256), 256, 0, s>>>(n, m, model, points, cotangent, A, B, gamma,
                                                                      radius, tgt, seg);
    AdjArgs args;
    args.n = n;
    args.m = m;
    args.tchunk = tchunk;
    args.schunk = schunk;
    args.tgt = tgt;
    args.seg = seg;
    args.ex_ptr = (ex_ptr && e > 0) ? ex_ptr : nullptr;
    args.ex_seg = ex_seg;
    args.model = model;
    args.part_x = part_x;
    args.part_seg = part_seg;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    adjoint_fused_kernel<<<dim3((unsigned)tc, (unsigned)sc), ADJ_THREADS, 0, s>>>(args);
    adjoint_reduce_kernel<<<(unsigned)((big + 255) / 256), 256, 0, s>>>(n, m, sc, tc, part_x, part_seg, grad_points,
                                                                         grad_A, grad_B, grad_gamma);
    cudaError_t le = cudaGetLastError();
    cudaEventRecord(e1, s);
    if (le == cudaSuccess) le = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (le == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (le != cudaSuccess) return cuda_fail(le, "bs_adjoint_direct");
    ctx->stats.points = n;
    ctx->stats.segments = m;
    ctx->stats.evaluate_ms = ms;
    ctx->stats.launches = 3;
    return BS_OK;
}
