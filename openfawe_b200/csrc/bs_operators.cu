// Unit-circulation influence operators (the VSM's dense columns): the reference's vortex_numba.pair_matrix and
// assemble_columns (src/openfawe/aero/vortex_numba.py:271-308), used by vsm_wake._batched_ring_operator and
// _batched_cross_class (src/openfawe/aero/vsm_wake.py:123-170, 224-252), and a fused form that sums each column's
// signed pair velocities without storing the pair matrix.
//
// pair_matrix: out[p][s] = the FP64 pair velocity of segment s with unit circulation at point p (zero when the pair
// flags), flags[p] = the flag of the first flagged segment in segment order.  One thread per (point, segment); the
// first flag is the minimum of (s << 2 | flag) over the point's flagged pairs (an integer atomic min, deterministic).
// assemble_columns: out[p][j] = sum over the column's entries k, in order from 0.0, of sign_k * pairs[p][segment_k]:
// one thread per (point, column), the reference's order exactly (signs are +-1, so each product is exact and the sums
// equal the reference's bit for bit for equal pairs).
#include <algorithm>
#include <climits>

#include "bs_internal.cuh"

namespace bs {

__global__ void unit_pack_kernel(int64_t m, const double *starts, const double *directions, const double *lengths,
                                 const double *radius, Seg64 *seg) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    Seg64 q;
    q.sx = starts[3 * k];
    q.sy = starts[3 * k + 1];
    q.sz = starts[3 * k + 2];
    q.len = lengths[k];
    q.dx = directions[3 * k];
    q.dy = directions[3 * k + 1];
    q.dz = directions[3 * k + 2];
    q.gfac = (1.0 / q.len) / 12.566370614359172;  // (gamma / length) / (4 pi) with gamma = 1, vortex_numba.py:105
    q.rcl = radius[k] / q.len;
    q.radius = radius[k];
    q.inv_len = 1.0 / q.len;
    q.pad = 0.0;
    seg[k] = q;
}

__device__ __forceinline__ void note_flag(unsigned long long *first, int64_t p, int64_t s, int f) {
    if (f != BS_FLAG_OK) atomicMin(first + p, ((unsigned long long)s << 2) | (unsigned long long)f);
}

__global__ void pair_matrix_kernel(int64_t n, int64_t m, const double *points, const Seg64 *seg, int model,
                                   int raise_singular, double *out, unsigned long long *first) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= m) return;
    const Seg64 q = seg[s];
    for (int64_t p = blockIdx.y; p < n; p += gridDim.y) {
        double ux = 0.0, uy = 0.0, uz = 0.0;
        const int f = pair64_at(points[3 * p], points[3 * p + 1], points[3 * p + 2], q, model, raise_singular, ux, uy,
                                uz);
        note_flag(first, p, s, f);
        double *o = out + 3 * (p * m + s);
        o[0] = ux;
        o[1] = uy;
        o[2] = uz;
    }
}

__global__ void first_flag_kernel(int64_t n, const unsigned long long *first, int8_t *flags) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) flags[p] = first[p] == ULLONG_MAX ? (int8_t)BS_FLAG_OK : (int8_t)(first[p] & 3ull);
}

__global__ void assemble_columns_kernel(int64_t n, int64_t m, const double *pairs, int64_t columns,
                                        const int64_t *column_ptr, const int64_t *column_segment,
                                        const double *column_sign, double *out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= columns) return;
    const int64_t k0 = column_ptr[j], k1 = column_ptr[j + 1];
    for (int64_t p = blockIdx.y; p < n; p += gridDim.y) {
        double ux = 0.0, uy = 0.0, uz = 0.0;
        const double *row = pairs + 3 * p * m;
        for (int64_t k = k0; k < k1; ++k) {
            const double sign = column_sign[k];
            const double *v = row + 3 * column_segment[k];
            ux = __dadd_rn(ux, __dmul_rn(sign, v[0]));
            uy = __dadd_rn(uy, __dmul_rn(sign, v[1]));
            uz = __dadd_rn(uz, __dmul_rn(sign, v[2]));
        }
        double *o = out + 3 * (p * columns + j);
        o[0] = ux;
        o[1] = uy;
        o[2] = uz;
    }
}

// The fused operator: each (point, column) evaluates its entries' pairs on the fly, in column order.
__global__ void ring_columns_kernel(int64_t n, const double *points, const Seg64 *seg, int model, int raise_singular,
                                    int64_t columns, const int64_t *column_ptr, const int64_t *column_segment,
                                    const double *column_sign, double *out, unsigned long long *first) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= columns) return;
    const int64_t k0 = column_ptr[j], k1 = column_ptr[j + 1];
    for (int64_t p = blockIdx.y; p < n; p += gridDim.y) {
        const double px = points[3 * p], py = points[3 * p + 1], pz = points[3 * p + 2];
        double ux = 0.0, uy = 0.0, uz = 0.0;
        for (int64_t k = k0; k < k1; ++k) {
            const int64_t s = column_segment[k];
            double vx = 0.0, vy = 0.0, vz = 0.0;
            note_flag(first, p, s, pair64_at(px, py, pz, seg[s], model, raise_singular, vx, vy, vz));
            const double sign = column_sign[k];
            ux = __dadd_rn(ux, __dmul_rn(sign, vx));
            uy = __dadd_rn(uy, __dmul_rn(sign, vy));
            uz = __dadd_rn(uz, __dmul_rn(sign, vz));
        }
        double *o = out + 3 * (p * columns + j);
        o[0] = ux;
        o[1] = uy;
        o[2] = uz;
    }
}

// bad[0] = 1 if a column's pointer decreases or an entry names a segment outside [0, m)
__global__ void column_check_kernel(int64_t columns, int64_t m, const int64_t *column_ptr,
                                    const int64_t *column_segment, int *bad) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= columns) return;
    const int64_t k0 = column_ptr[j], k1 = column_ptr[j + 1];
    if (k1 < k0 || k0 < 0) {
        *bad = 1;
        return;
    }
    for (int64_t k = k0; k < k1; ++k)
        if (column_segment[k] < 0 || column_segment[k] >= m) *bad = 1;
}

}  // namespace bs

using namespace bs;

static bool sources_ok(const bs_sources *src) {
    return src && src->m >= 0 &&
           (src->m == 0 || (src->starts && src->directions && src->lengths && src->radius));
}

static dim3 pair_grid(int64_t inner, int64_t n, int threads) {
    return dim3((unsigned)std::max<int64_t>(1, (inner + threads - 1) / threads),
                (unsigned)std::max<int64_t>(1, std::min<int64_t>(n, 65535)));
}

// Validates a column layout on the device (one synchronisation); returns BS_OK or BS_ERR_ARG.
static int check_columns(int64_t columns, int64_t m, const int64_t *column_ptr, const int64_t *column_segment,
                         Scratch &scratch, cudaStream_t s, const char *who) {
    if (columns == 0) return BS_OK;
    int *bad = scratch.get<int>(1);
    if (!bad) return scratch.status;
    BS_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    column_check_kernel<<<(unsigned)((columns + 255) / 256), 256, 0, s>>>(columns, m, column_ptr, column_segment, bad);
    BS_CHECK_LAUNCH("column_check_kernel");
    int host = 0;
    BS_CUDA(cudaMemcpyAsync(&host, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    BS_CUDA(cudaStreamSynchronize(s));
    if (host) {
        set_error("%s: a column pointer decreases or an entry's segment lies outside [0, m)", who);
        return BS_ERR_ARG;
    }
    return BS_OK;
}

extern "C" int bs_pair_matrix(bs_ctx *ctx, int64_t n, const double *points, const bs_sources *src, int model,
                              int raise_singular, double *out, int8_t *flags, bs_stream stream) {
    if (!ctx || n < 0 || !sources_ok(src) || (n > 0 && (!points || !flags)) || (n > 0 && src->m > 0 && !out)) {
        set_error("bs_pair_matrix: null or negative argument");
        return BS_ERR_ARG;
    }
    if (model < 0 || model > 5) {
        set_error("bs_pair_matrix: core model must be 0..5");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    const int64_t m = src->m;
    if (n == 0) return BS_OK;
    if (m == 0) {
        BS_CUDA(cudaMemsetAsync(flags, 0, n, s));
        return BS_OK;
    }
    Scratch scratch(ctx->pool, s);
    Seg64 *seg = scratch.get<Seg64>(m);
    unsigned long long *first = scratch.get<unsigned long long>(n);
    if (!seg || !first) return scratch.status;
    BS_CUDA(cudaMemsetAsync(first, 0xff, n * sizeof(unsigned long long), s));
    unit_pack_kernel<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(m, src->starts, src->directions, src->lengths,
                                                                 src->radius, seg);
    BS_CHECK_LAUNCH("unit_pack_kernel");
    pair_matrix_kernel<<<pair_grid(m, n, 128), 128, 0, s>>>(n, m, points, seg, model, raise_singular, out, first);
    BS_CHECK_LAUNCH("pair_matrix_kernel");
    first_flag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, first, flags);
    BS_CHECK_LAUNCH("first_flag_kernel");
    ctx->stats.points = n;
    ctx->stats.segments = m;
    ctx->stats.launches = 3;
    return BS_OK;
}

extern "C" int bs_assemble_columns(bs_ctx *ctx, int64_t n, int64_t m, const double *pairs, int64_t columns,
                                   const int64_t *column_ptr, const int64_t *column_segment,
                                   const double *column_sign, double *out, bs_stream stream) {
    if (!ctx || n < 0 || m < 0 || columns < 0 || (columns > 0 && (!column_ptr || !column_segment || !column_sign)) ||
        (n > 0 && columns > 0 && !out) || (n > 0 && m > 0 && !pairs)) {
        set_error("bs_assemble_columns: null or negative argument");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    if (n == 0 || columns == 0) return BS_OK;
    Scratch scratch(ctx->pool, s);
    int rc = check_columns(columns, m, column_ptr, column_segment, scratch, s, "bs_assemble_columns");
    if (rc != BS_OK) return rc;
    assemble_columns_kernel<<<pair_grid(columns, n, 64), 64, 0, s>>>(n, m, pairs, columns, column_ptr, column_segment,
                                                                     column_sign, out);
    BS_CHECK_LAUNCH("assemble_columns_kernel");
    return BS_OK;
}

extern "C" int bs_ring_columns(bs_ctx *ctx, int64_t n, const double *points, const bs_sources *src, int model,
                               int raise_singular, int64_t columns, const int64_t *column_ptr,
                               const int64_t *column_segment, const double *column_sign, double *out, int8_t *flags,
                               bs_stream stream) {
    if (!ctx || n < 0 || columns < 0 || !sources_ok(src) || (n > 0 && (!points || !flags)) ||
        (columns > 0 && (!column_ptr || !column_segment || !column_sign)) || (n > 0 && columns > 0 && !out)) {
        set_error("bs_ring_columns: null or negative argument");
        return BS_ERR_ARG;
    }
    if (model < 0 || model > 5) {
        set_error("bs_ring_columns: core model must be 0..5");
        return BS_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    const int64_t m = src->m;
    if (n == 0) return BS_OK;
    Scratch scratch(ctx->pool, s);
    int rc = check_columns(columns, m, column_ptr, column_segment, scratch, s, "bs_ring_columns");
    if (rc != BS_OK) return rc;
    unsigned long long *first = scratch.get<unsigned long long>(n);
    Seg64 *seg = m > 0 ? scratch.get<Seg64>(m) : nullptr;
    if (!first || (m > 0 && !seg)) return scratch.status;
    BS_CUDA(cudaMemsetAsync(first, 0xff, n * sizeof(unsigned long long), s));
    if (m > 0) {
        unit_pack_kernel<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(m, src->starts, src->directions, src->lengths,
                                                                     src->radius, seg);
        BS_CHECK_LAUNCH("unit_pack_kernel");
    }
    if (columns > 0) {
        ring_columns_kernel<<<pair_grid(columns, n, 64), 64, 0, s>>>(n, points, seg, model, raise_singular, columns,
                                                                     column_ptr, column_segment, column_sign, out,
                                                                     first);
        BS_CHECK_LAUNCH("ring_columns_kernel");
    }
    first_flag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, first, flags);
    BS_CHECK_LAUNCH("first_flag_kernel");
    return BS_OK;
}
