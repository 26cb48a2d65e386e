// Adjoint of the direct Biot-Savart sum: gradients of L = sum_p w_p . u_p with respect to the targets x_p, both
// segment endpoints A_s, B_s and the circulations Gamma_s, for a given cotangent w.  Pair terms are recomputed, never
// stored.  The reference has no adjoint; the pair is the reference's (vortex_numba.pair_velocity,
// src/openfawe/aero/vortex_numba.py:42-109) written in its two-endpoint form, which is algebraically the same:
//   r1 = x - A, r2 = x - B, c = r1 x r2, P = |r1||r2|, d = r1.r2,
//   D = P (P + d), or P |c|^2 / (P - d) when d < 0 (the reference's rationalised branch),
//   u = Gamma/(4 pi) f(|c|^2 / (|B - A|^2 rc^2)) (|r1| + |r2|) c / D,
// with the core factor f of models 0 (none), 1 (Rankine) and 2 (Lamb-Oseen with its exponent cut-off), and reverse-mode
// differentiation of that expression by hand.  Pairs on a segment's axis (the reference's roundoff guard) contribute
// nothing, as in the forward sum.
//
// Two kernels, each deterministic: target-major (thread per target, segments streamed through shared memory) for the
// target gradients, segment-major (thread per segment, targets streamed) for the endpoint and circulation gradients.
// Both are split into chunks along their inner loop and the chunk partials are added in chunk order.
#include <algorithm>

#include "bs_internal.cuh"

namespace bs {

struct AdjSeg {
    double ax, ay, az, bx, by, bz, gamma, radius;
};
struct AdjTgt {
    double x, y, z, wx, wy, wz;
};

// Adds d(w . u)/dx, d/dA, d/dB, d/dGamma of one pair.
__device__ __forceinline__ void pair_vjp64(double x0, double x1, double x2, const AdjSeg &s, int model, double w0,
                                           double w1, double w2, double *gx, double *ga, double *gb, double &gg) {
    const double r10 = x0 - s.ax, r11 = x1 - s.ay, r12 = x2 - s.az;
    const double r20 = x0 - s.bx, r21 = x1 - s.by, r22 = x2 - s.bz;
    const double l0 = s.bx - s.ax, l1 = s.by - s.ay, l2 = s.bz - s.az;
    const double L2 = l0 * l0 + l1 * l1 + l2 * l2;
    const double L = sqrt(L2);
    const double c0 = r11 * r22 - r12 * r21, c1 = r12 * r20 - r10 * r22, c2v = r10 * r21 - r11 * r20;
    const double cc = c0 * c0 + c1 * c1 + c2v * c2v;
    const double n1 = sqrt(r10 * r10 + r11 * r11 + r12 * r12), n2 = sqrt(r20 * r20 + r21 * r21 + r22 * r22);
    // the reference's roundoff axis guard, in its scaled units (h = |c|/L^2, na = n1/L, nb = n2/L)
    if (sqrt(cc) / L2 <= AXIS_EPS64 * fmax(1.0, fmax(n1, n2) / L)) return;
    const double d = r10 * r20 + r11 * r21 + r12 * r22;
    const double P = n1 * n2;
    double D, dD_dP, dD_dd, dD_dcc;
    if (d >= 0.0) {
        D = P * (P + d);
        dD_dP = 2.0 * P + d;
        dD_dd = P;
        dD_dcc = 0.0;
    } else {
        const double q = P - d, iq = 1.0 / q;
        D = P * cc * iq;
        dD_dP = -cc * d * iq * iq;
        dD_dd = P * cc * iq * iq;
        dD_dcc = P * iq;
    }
    double f = 1.0, df = 0.0, irc2L2 = 0.0;  // f(rho2), df/drho2, 1/(L2 rc^2)
    if (s.radius > 0.0 && model != 0) {
        irc2L2 = 1.0 / (L2 * s.radius * s.radius);
        const double rho2 = cc * irc2L2;
        if (model == 1) {
            if (rho2 < 1.0) { f = rho2; df = 1.0; }
        } else if (model == 2) {
            if (rho2 <= LAMB_CUT2) {
                const double e = exp(-LAMB_A * rho2);
                f = -expm1(-LAMB_A * rho2);
                df = LAMB_A * e;
            }
        }
    }
    const double S = n1 + n2;
    const double iD = 1.0 / D;
    const double coefG = INV_FOUR_PI * f * S * iD;  // u = Gamma * coefG * c
    const double wc = w0 * c0 + w1 * c1 + w2 * c2v;
    gg += coefG * wc;
    const double G = s.gamma;
    const double gcoef = G * wc;
    const double g_f = gcoef * INV_FOUR_PI * S * iD;
    const double g_S = gcoef * INV_FOUR_PI * f * iD;
    const double g_D = -gcoef * INV_FOUR_PI * f * S * iD * iD;
    const double g_rho2 = g_f * df;
    const double g_cc = g_rho2 * irc2L2 + g_D * dD_dcc;
    const double g_L2 = -g_rho2 * cc * irc2L2 / L2;
    const double g_P = g_D * dD_dP, g_d = g_D * dD_dd;
    const double g_n1 = g_S + g_P * n2, g_n2 = g_S + g_P * n1;
    const double k = G * coefG;
    const double gc0 = k * w0 + 2.0 * c0 * g_cc, gc1 = k * w1 + 2.0 * c1 * g_cc, gc2 = k * w2 + 2.0 * c2v * g_cc;
    // c = r1 x r2: dL/dr1 += r2 x g_c, dL/dr2 += g_c x r1
    const double a1 = g_n1 / n1, a2 = g_n2 / n2, b = 2.0 * g_L2;
    const double g10 = a1 * r10 + g_d * r20 + (r21 * gc2 - r22 * gc1) + b * l0;
    const double g11 = a1 * r11 + g_d * r21 + (r22 * gc0 - r20 * gc2) + b * l1;
    const double g12 = a1 * r12 + g_d * r22 + (r20 * gc1 - r21 * gc0) + b * l2;
    const double g20 = a2 * r20 + g_d * r10 + (gc1 * r12 - gc2 * r11) - b * l0;
    const double g21 = a2 * r21 + g_d * r11 + (gc2 * r10 - gc0 * r12) - b * l1;
    const double g22 = a2 * r22 + g_d * r12 + (gc0 * r11 - gc1 * r10) - b * l2;
    // L2 = |B - A|^2 = |r1 - r2|^2 with r1 - r2 = l: dL2/dr1 = 2 l, dL2/dr2 = -2 l (folded in above)
    gx[0] += g10 + g20;
    gx[1] += g11 + g21;
    gx[2] += g12 + g22;
    ga[0] -= g10; ga[1] -= g11; ga[2] -= g12;
    gb[0] -= g20; gb[1] -= g21; gb[2] -= g22;
}

__device__ __forceinline__ bool excluded(const int64_t *ex_ptr, const int64_t *ex_seg, int64_t p, int64_t s) {
    if (!ex_ptr) return false;
    for (int64_t k = ex_ptr[p]; k < ex_ptr[p + 1]; ++k)
        if (ex_seg[k] == s) return true;
    return false;
}

constexpr int ADJ_TILE = 128;

struct AdjArgs {
    int64_t n, m, chunk;
    const AdjTgt *tgt;
    const AdjSeg *seg;
    const int64_t *ex_ptr, *ex_seg;
    int model;
    double *part_x;    // [chunks][n][3]
    double *part_seg;  // [chunks][m][7]: gA, gB, gGamma
};

__global__ void __launch_bounds__(ADJ_TILE) adjoint_target_kernel(AdjArgs a) {
    __shared__ AdjSeg tile[ADJ_TILE];
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < a.n;
    const int64_t s0 = (int64_t)blockIdx.y * a.chunk, s1 = min(a.m, s0 + a.chunk);
    AdjTgt t = valid ? a.tgt[p] : AdjTgt{0, 0, 0, 0, 0, 0};
    double gx[3] = {0, 0, 0}, ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0}, gg = 0.0;
    for (int64_t base = s0; base < s1; base += ADJ_TILE) {
        const int cnt = (int)min((int64_t)ADJ_TILE, s1 - base);
        __syncthreads();
        if (threadIdx.x < cnt) tile[threadIdx.x] = a.seg[base + threadIdx.x];
        __syncthreads();
        if (!valid) continue;
        for (int j = 0; j < cnt; ++j) {
            if (a.ex_ptr && excluded(a.ex_ptr, a.ex_seg, p, base + j)) continue;
            pair_vjp64(t.x, t.y, t.z, tile[j], a.model, t.wx, t.wy, t.wz, gx, ga, gb, gg);
        }
    }
    if (valid) {
        const int64_t o = (int64_t)blockIdx.y * a.n + p;
        a.part_x[3 * o] = gx[0];
        a.part_x[3 * o + 1] = gx[1];
        a.part_x[3 * o + 2] = gx[2];
    }
}

__global__ void __launch_bounds__(ADJ_TILE) adjoint_segment_kernel(AdjArgs a) {
    __shared__ AdjTgt tile[ADJ_TILE];
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = s < a.m;
    const int64_t p0 = (int64_t)blockIdx.y * a.chunk, p1 = min(a.n, p0 + a.chunk);
    AdjSeg g = valid ? a.seg[s] : AdjSeg{0, 0, 0, 1, 0, 0, 0, 0};
    double gx[3] = {0, 0, 0}, ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0}, gg = 0.0;
    for (int64_t base = p0; base < p1; base += ADJ_TILE) {
        const int cnt = (int)min((int64_t)ADJ_TILE, p1 - base);
        __syncthreads();
        if (threadIdx.x < cnt) tile[threadIdx.x] = a.tgt[base + threadIdx.x];
        __syncthreads();
        if (!valid) continue;
        for (int j = 0; j < cnt; ++j) {
            if (a.ex_ptr && excluded(a.ex_ptr, a.ex_seg, base + j, s)) continue;
            const AdjTgt &t = tile[j];
            pair_vjp64(t.x, t.y, t.z, g, a.model, t.wx, t.wy, t.wz, gx, ga, gb, gg);
        }
    }
    if (valid) {
        const int64_t o = (int64_t)blockIdx.y * a.m + s;
        double *q = a.part_seg + 7 * o;
        q[0] = ga[0]; q[1] = ga[1]; q[2] = ga[2];
        q[3] = gb[0]; q[4] = gb[1]; q[5] = gb[2];
        q[6] = gg;
    }
}

__global__ void adjoint_pack_kernel(int64_t n, int64_t m, const double *points, const double *cot, const double *A,
                                    const double *B, const double *gamma, const double *radius, AdjTgt *tgt,
                                    AdjSeg *seg) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) tgt[i] = AdjTgt{points[3 * i], points[3 * i + 1], points[3 * i + 2], cot[3 * i], cot[3 * i + 1],
                               cot[3 * i + 2]};
    if (i < m) seg[i] = AdjSeg{A[3 * i], A[3 * i + 1], A[3 * i + 2], B[3 * i], B[3 * i + 1], B[3 * i + 2], gamma[i],
                               radius[i]};
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

static int chunks_for(int64_t rows, int64_t inner, int sm_count) {
    int64_t blocks = (rows + ADJ_TILE - 1) / ADJ_TILE;
    int64_t want = (int64_t)sm_count * 8;
    int64_t c = (want + blocks - 1) / blocks;
    c = std::min<int64_t>(c, std::max<int64_t>(1, (inner + ADJ_TILE - 1) / ADJ_TILE));
    return (int)std::max<int64_t>(1, std::min<int64_t>(c, 1024));
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
    if (model < 0 || model > 2) {
        set_error("bs_adjoint_direct: the adjoint supports core models NONE, RANKINE and LAMB_OSEEN");
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
    const int cx = chunks_for(n, m, ctx->sm_count), cs = chunks_for(m, n, ctx->sm_count);
    double *part_x = scratch.get<double>((size_t)3 * n * cx), *part_seg = scratch.get<double>((size_t)7 * m * cs);
    if (!tgt || !seg || !part_x || !part_seg) return scratch.status;
    const int64_t big = std::max(n, m);
    adjoint_pack_kernel<<<(unsigned)((big + 255) / 256), 256, 0, s>>>(n, m, points, cotangent, A, B, gamma, radius, tgt,
                                                                      seg);
    AdjArgs args;
    args.n = n;
    args.m = m;
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
    if (grad_points) {
        args.chunk = ((m + cx - 1) / cx + ADJ_TILE - 1) / ADJ_TILE * ADJ_TILE;
        dim3 grid((unsigned)((n + ADJ_TILE - 1) / ADJ_TILE), (unsigned)((m + args.chunk - 1) / args.chunk));
        adjoint_target_kernel<<<grid, ADJ_TILE, 0, s>>>(args);
    }
    int cx_used = (int)((m + args.chunk - 1) / std::max<int64_t>(1, args.chunk));
    if (!grad_points) cx_used = 0;
    int cs_used = 0;
    if (grad_A || grad_B || grad_gamma) {
        args.chunk = ((n + cs - 1) / cs + ADJ_TILE - 1) / ADJ_TILE * ADJ_TILE;
        dim3 grid((unsigned)((m + ADJ_TILE - 1) / ADJ_TILE), (unsigned)((n + args.chunk - 1) / args.chunk));
        cs_used = (int)grid.y;
        adjoint_segment_kernel<<<grid, ADJ_TILE, 0, s>>>(args);
    }
    adjoint_reduce_kernel<<<(unsigned)((big + 255) / 256), 256, 0, s>>>(n, m, cx_used, cs_used, part_x, part_seg,
                                                                         grad_points, grad_A, grad_B, grad_gamma);
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
    ctx->stats.launches = 4;
    return BS_OK;
}
