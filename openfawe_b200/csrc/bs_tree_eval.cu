// Tree evaluation: the traversal of vortex_tree.tree_velocity (src/openfawe/aero/vortex_tree.py:508-568) on the GPU.
//
// A warp walks the tree depth first (left child first) with one shared stack whose entries carry the mask of lanes
// (targets) that opened the parent.  Each lane decides acceptance for itself, with the reference's FP64 test
// (bound < theta |R|, |R| - bound >= clearance * core, no excluded segment inside), so every target visits exactly the
// nodes, in exactly the order, of the per-target CPU traversal; lanes only share the walk.  Targets are sorted by the
// Morton key of their positions so that a warp's targets are neighbours and their node sets overlap.
// Exclusions: the target's excluded segments as sorted tree positions (vortex_tree._positions, :571-580) and a cursor
// that only moves forward, because depth-first visits see non-decreasing range starts.
#include "bs_sort.cuh"
#include "bs_tree.cuh"

namespace bs {

constexpr int STACK_DEPTH = 128;

struct EvalArgs {
    int64_t n;
    const double *points;
    const int32_t *perm;
    const int64_t *ex_ptr;
    const int32_t *ex_pos;
    const NodeRec *nodes;
    const Far64 *far64;
    const Far32 *far32;
    const Seg64 *seg64;
    const Seg32 *seg32;
    double theta, clearance;
    int order, model, raise_singular, stack_limit;
    float near2;
    double *out;
    int8_t *flags;
    int64_t *far_counts;
    int *overflow;
    unsigned long long *counters;  // far evaluations, near pairs, fp64 pairs, visits
};

template <int PREC>
__global__ void __launch_bounds__(256) tree_eval_kernel(EvalArgs a) {
    extern __shared__ int2 stack_mem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int2 *stack = stack_mem + warp * STACK_DEPTH;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < a.n;
    const int64_t p = valid ? a.perm[i] : 0;
    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
    if (valid) { x0 = a.points[3 * p]; x1 = a.points[3 * p + 1]; x2 = a.points[3 * p + 2]; }
    float xh0, xl0, xh1, xl1, xh2, xl2;
    split2(x0, xh0, xl0);
    split2(x1, xh1, xl1);
    split2(x2, xh2, xl2);
    int64_t e = 0, e1 = 0;
    if (valid && a.ex_ptr) { e = a.ex_ptr[p]; e1 = a.ex_ptr[p + 1]; }
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;      // FP64 accumulator (fp64, mixed)
    float f0 = 0.0f, f1 = 0.0f, f2 = 0.0f;    // FP32 accumulator (fp32)
    int flag = BS_FLAG_OK;
    long long far = 0, near_pairs = 0, fp64_pairs = 0, visits = 0;
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    if (active == 0) return;
    if (lane == 0) stack[0] = make_int2(0, (int)active);
    int top = 1;
    __syncwarp();
    while (top > 0) {
        --top;
        const int2 entry = stack[top];
        const int node = entry.x;
        const unsigned mask = (unsigned)entry.y;
        const bool mine = (mask >> lane) & 1u;
        const NodeRec nr = a.nodes[node];
        bool accept = false;
        double rx = 0.0, ry = 0.0, rz = 0.0;
        if (mine) {
            ++visits;
            rx = x0 - nr.cx;
            ry = x1 - nr.cy;
            rz = x2 - nr.cz;
            // the reference's expression, without contraction, so that decisions equal the CPU's
            double dist = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)));
            accept = nr.bound < __dmul_rn(a.theta, dist) &&
                     __dsub_rn(dist, nr.bound) >= __dmul_rn(a.clearance, nr.clear_core);
            if (accept && e < e1) {
                while (e < e1 && a.ex_pos[e] < nr.lo) ++e;
                if (e < e1 && a.ex_pos[e] < nr.hi) accept = false;
            }
        }
        const unsigned farm = __ballot_sync(0xffffffffu, mine && accept);
        const unsigned openm = mask & ~farm;
        if (mine && accept) {
            ++far;
            if (PREC == 0) {
                far_eval<double>(rx, ry, rz, a.far64[node].v, a.order, u0, u1, u2);
            } else {
                float g0 = 0.f, g1 = 0.f, g2 = 0.f;
                far_eval<float>((float)rx, (float)ry, (float)rz, a.far32[node].v, a.order, g0, g1, g2);
                if (PREC == 1) { u0 += g0; u1 += g1; u2 += g2; }
                else { f0 += g0; f1 += g1; f2 += g2; }
            }
        }
        if (openm) {
            if (nr.left < 0) {
                if (mine && !accept) {
                    while (e < e1 && a.ex_pos[e] < nr.lo) ++e;
                    float t0 = 0.f, t1 = 0.f, t2 = 0.f;
                    for (int k = nr.lo; k < nr.hi; ++k) {
                        if (e < e1 && a.ex_pos[e] == k) { ++e; continue; }
                        ++near_pairs;
                        if (PREC == 0) {
                            int fl = pair64_at(x0, x1, x2, a.seg64[k], a.model, a.raise_singular, u0, u1, u2);
                            if (fl != BS_FLAG_OK && flag == BS_FLAG_OK) flag = fl;
                        } else {
                            const Seg32 r = a.seg32[k];
                            float q0 = (xh0 - r.hi.x) + (xl0 - r.lo.x);
                            float q1 = (xh1 - r.hi.y) + (xl1 - r.lo.y);
                            float q2 = (xh2 - r.hi.z) + (xl2 - r.lo.z);
                            if (pair32(q0, q1, q2, r.hi, r.lo, r.dir, a.model, a.near2, t0, t1, t2)) {
                                ++fp64_pairs;
                                double v0 = 0.0, v1 = 0.0, v2 = 0.0;
                                int fl = pair64_at(x0, x1, x2, a.seg64[k], a.model, a.raise_singular, v0, v1, v2);
                                if (fl != BS_FLAG_OK) {
                                    if (flag == BS_FLAG_OK) flag = fl;
                                } else if (PREC == 1) {
                                    u0 += v0; u1 += v1; u2 += v2;
                                } else {
                                    f0 += (float)v0; f1 += (float)v1; f2 += (float)v2;
                                }
                            }
                        }
                    }
                    if (PREC == 1) { u0 += t0; u1 += t1; u2 += t2; }
                    else if (PREC == 2) { f0 += t0; f1 += t1; f2 += t2; }
                }
            } else {
                if (top + 2 > a.stack_limit) {
                    if (lane == 0) atomicExch(a.overflow, 1);
                    break;
                }
                if (lane == 0) {
                    stack[top] = make_int2(nr.right, (int)openm);
                    stack[top + 1] = make_int2(nr.left, (int)openm);
                }
                top += 2;
            }
        }
        __syncwarp();
    }
    if (PREC == 2) { u0 = f0; u1 = f1; u2 = f2; }
    if (valid) {
        if (!(isfinite(u0) && isfinite(u1) && isfinite(u2)) && flag == BS_FLAG_OK) flag = BS_FLAG_NONFINITE;
        a.out[3 * p] = u0;
        a.out[3 * p + 1] = u1;
        a.out[3 * p + 2] = u2;
        a.flags[p] = (int8_t)flag;
        if (a.far_counts) a.far_counts[p] = far;
    }
    for (int o = 16; o > 0; o >>= 1) {
        far += __shfl_xor_sync(0xffffffffu, far, o);
        near_pairs += __shfl_xor_sync(0xffffffffu, near_pairs, o);
        fp64_pairs += __shfl_xor_sync(0xffffffffu, fp64_pairs, o);
        visits += __shfl_xor_sync(0xffffffffu, visits, o);
    }
    if (lane == 0) {
        atomicAdd(&a.counters[0], (unsigned long long)far);
        atomicAdd(&a.counters[1], (unsigned long long)near_pairs);
        atomicAdd(&a.counters[2], (unsigned long long)fp64_pairs);
        atomicAdd(&a.counters[3], (unsigned long long)visits);
    }
}

// Morton keys of the targets inside their own box (for locality only; any order gives the same per-target result).
__global__ void target_box_kernel(int64_t n, const double *points, unsigned long long *box) {
    __shared__ unsigned long long sb[6];
    auto ob = [](double x) -> unsigned long long {
        unsigned long long b = (unsigned long long)__double_as_longlong(x + 0.0);
        return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
    };
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? ob(INFINITY) : ob(-INFINITY);
    __syncthreads();
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            atomicMin(&sb[a], ob(points[3 * p + a]));
            atomicMax(&sb[3 + a], ob(points[3 * p + a]));
        }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&box[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&box[threadIdx.x], sb[threadIdx.x]);
}

__global__ void target_box_init_kernel(unsigned long long *box) {
    auto ob = [](double x) -> unsigned long long {
        unsigned long long b = (unsigned long long)__double_as_longlong(x + 0.0);
        return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
    };
    if (threadIdx.x < 3) box[threadIdx.x] = ob(INFINITY);
    else if (threadIdx.x < 6) box[threadIdx.x] = ob(-INFINITY);
}

__device__ __forceinline__ double unordered(unsigned long long k) {
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__device__ __forceinline__ uint64_t spread3_t(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void target_keys_kernel(int64_t n, const double *points, const unsigned long long *box, uint64_t *keys,
                                   int32_t *vals) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double ext = 0.0, lo[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = unordered(box[a]);
        ext = fmax(ext, unordered(box[3 + a]) - lo[a]);
    }
    double inv = ext > 0.0 ? 2097152.0 / ext : 0.0;
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) q[a] = min(2097151u, (uint32_t)((points[3 * p + a] - lo[a]) * inv));
    keys[p] = (spread3_t(q[0]) << 2) | (spread3_t(q[1]) << 1) | spread3_t(q[2]);
    vals[p] = (int32_t)p;
}

// Excluded segment ids -> tree positions, sorted per target (insertion sort; a target excludes few segments).
__global__ void exclusion_positions_kernel(int64_t n, const int64_t *ex_ptr, const int64_t *ex_seg,
                                           const int32_t *inverse, int32_t *ex_pos) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int64_t a = ex_ptr[p], b = ex_ptr[p + 1];
    for (int64_t k = a; k < b; ++k) {
        int32_t v = inverse[ex_seg[k]];
        int64_t j = k - 1;
        while (j >= a && ex_pos[j] > v) { ex_pos[j + 1] = ex_pos[j]; --j; }
        ex_pos[j + 1] = v;
    }
}

static inline unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int target_order(int64_t n, const double *points, int32_t *perm, Scratch &scratch, cudaStream_t s) {
    unsigned long long *box = scratch.get<unsigned long long>(6);
    uint64_t *keys = scratch.get<uint64_t>(n);
    if (!box || !keys) return scratch.status;
    target_box_init_kernel<<<1, 32, 0, s>>>(box);
    target_box_kernel<<<std::min<unsigned>(nblocks(n, 256), 592), 256, 0, s>>>(n, points, box);
    target_keys_kernel<<<nblocks(n, 256), 256, 0, s>>>(n, points, box, keys, perm);
    BS_CHECK_LAUNCH("target keys");
    return radix_sort(keys, perm, n, 0, 63, scratch, s);
}

}  // namespace bs

using namespace bs;

extern "C" int bs_tree_eval(bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
                            const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts,
                            bs_stream stream) {
    if (!ctx || !tree || !tp || !tgt || !kp || (tgt->n > 0 && (!tgt->points || !out || !flags))) {
        set_error("bs_tree_eval: null argument");
        return BS_ERR_ARG;
    }
    if (!(tp->theta > 0.0 && tp->theta < 1.0) || tp->order < 0 || tp->order > 2 || !(tp->clearance >= 0.0)) {
        set_error("bs_tree_eval: theta must lie in (0, 1), order in 0..2, clearance >= 0");
        return BS_ERR_ARG;
    }
    if (kp->model < 0 || kp->model > 5 || kp->precision < 0 || kp->precision > 2 ||
        (kp->block != 32 && kp->block != 64 && kp->block != 128 && kp->block != 256)) {
        set_error("bs_tree_eval: model 0..5, precision 0..2, block 32/64/128/256");
        return BS_ERR_ARG;
    }
    if (tgt->n >= (int64_t(1) << 31)) {
        set_error("bs_tree_eval: at most 2^31 - 1 targets");
        return BS_ERR_ARG;
    }
    if (tgt->n == 0) return BS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    BS_CUDA(cudaSetDevice(ctx->device));
    Scratch scratch(ctx->pool, s);
    const int64_t n = tgt->n;
    int32_t *perm = scratch.get<int32_t>(n);
    int *overflow = scratch.get<int>(1);
    unsigned long long *counters = scratch.get<unsigned long long>(4);
    int32_t *ex_pos = nullptr;
    if (!perm || !overflow || !counters) return scratch.status;
    int rc = target_order(n, tgt->points, perm, scratch, s);
    if (rc != BS_OK) return rc;
    if (tgt->ex_ptr && tgt->e > 0) {
        ex_pos = scratch.get<int32_t>(tgt->e);
        if (!ex_pos) return scratch.status;
        exclusion_positions_kernel<<<nblocks(n, 128), 128, 0, s>>>(n, tgt->ex_ptr, tgt->ex_seg, tree->inverse,
                                                                    ex_pos);
        BS_CHECK_LAUNCH("exclusion_positions_kernel");
    }
    BS_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int), s));
    BS_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), s));
    EvalArgs args;
    args.n = n;
    args.points = tgt->points;
    args.perm = perm;
    args.ex_ptr = ex_pos ? tgt->ex_ptr : nullptr;
    args.ex_pos = ex_pos;
    args.nodes = tree->nodes;
    args.far64 = tree->far64;
    args.far32 = tree->far32;
    args.seg64 = tree->seg64;
    args.seg32 = tree->seg32;
    args.theta = tp->theta;
    args.clearance = tp->clearance;
    args.order = tp->order;
    args.model = kp->model;
    args.raise_singular = kp->raise_singular ? 1 : 0;
    args.near2 = (float)(kp->near_cores * kp->near_cores);
    args.stack_limit = (tp->stack_limit > 0 && tp->stack_limit < STACK_DEPTH) ? tp->stack_limit : STACK_DEPTH;
    args.out = out;
    args.flags = flags;
    args.far_counts = far_counts;
    args.overflow = overflow;
    args.counters = counters;
    const int block = kp->block;
    const size_t smem = (size_t)(block / 32) * STACK_DEPTH * sizeof(int2);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    if (kp->precision == BS_FP64) tree_eval_kernel<0><<<nblocks(n, block), block, smem, s>>>(args);
    else if (kp->precision == BS_MIXED) tree_eval_kernel<1><<<nblocks(n, block), block, smem, s>>>(args);
    else tree_eval_kernel<2><<<nblocks(n, block), block, smem, s>>>(args);
    cudaError_t le = cudaGetLastError();
    cudaEventRecord(e1, s);
    int host_overflow = 0;
    unsigned long long host_counters[4] = {0, 0, 0, 0};
    if (le == cudaSuccess) le = cudaMemcpyAsync(&host_overflow, overflow, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (le == cudaSuccess)
        le = cudaMemcpyAsync(host_counters, counters, sizeof host_counters, cudaMemcpyDeviceToHost, s);
    if (le == cudaSuccess) le = cudaStreamSynchronize(s);
    float ms = 0.f;
    if (le == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (le != cudaSuccess) return cuda_fail(le, "tree_eval_kernel");
    ctx->stats.points = n;
    ctx->stats.segments = tree->m;
    ctx->stats.nodes = tree->count;
    ctx->stats.launches = 1;
    ctx->stats.far_evaluations = (int64_t)host_counters[0];
    ctx->stats.near_pairs = (int64_t)host_counters[1];
    ctx->stats.fp64_pairs = (int64_t)host_counters[2];
    ctx->stats.visits = (int64_t)host_counters[3];
    ctx->stats.evaluate_ms = ms;
    if (host_overflow) {
        set_error("tree traversal stack overflow on the GPU (depth %d)", args.stack_limit);
        return BS_ERR_STACK;
    }
    return BS_OK;
}

extern "C" int bs_tree_sum(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, const bs_targets *tgt,
                           const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts,
                           bs_stream stream) {
    if (!ctx || !src || !tgt) {
        set_error("bs_tree_sum: null argument");
        return BS_ERR_ARG;
    }
    if (tgt->n == 0) return BS_OK;
    if (src->m == 0) {
        cudaStream_t s = (cudaStream_t)stream;
        BS_CUDA(cudaMemsetAsync(out, 0, tgt->n * 3 * sizeof(double), s));
        BS_CUDA(cudaMemsetAsync(flags, 0, tgt->n, s));
        if (far_counts) BS_CUDA(cudaMemsetAsync(far_counts, 0, tgt->n * sizeof(int64_t), s));
        return BS_OK;
    }
    bs_tree *tree = nullptr;
    int rc = bs_tree_build(ctx, src, tp, &tree, stream);
    if (rc != BS_OK) return rc;
    rc = bs_tree_eval(ctx, tree, tp, tgt, kp, out, flags, far_counts, stream);
    float b = tree->build_ms, mm = tree->moments_ms;
    bs_tree_free(tree);
    ctx->stats.build_ms = b;
    ctx->stats.moments_ms = mm;
    return rc;
}
