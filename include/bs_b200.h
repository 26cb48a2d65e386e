/*
 * bs_b200.h -- C ABI of the B200-native Biot-Savart hot path (libbs_b200.so, sm_100a).
 *
 * Replaces the numba.cuda backends of the reference's vortex-batch API (paths inside the reference project):
 *   cuda_sum        src/openfawe/aero/vortex_cuda.py:381-467        -> bs_direct
 *   cuda_tree_sum   src/openfawe/aero/vortex_cuda_tree.py:439-595   -> bs_tree_build + bs_tree_eval (bs_tree_sum)
 *   device_build_tree  src/openfawe/aero/vortex_cuda_build.py:234-275  -> bs_tree_build (kind BS_TREE_MEDIAN)
 *   device_node_quantities  src/openfawe/aero/vortex_cuda_moments.py:206-230 -> moments inside bs_tree_build /
 *                   bs_tree_from_arrays, read back with bs_tree_export
 *   available / probe_error  src/openfawe/aero/vortex_cuda.py:58-82 -> bs_init / bs_last_error
 *   Statistics.last  src/openfawe/aero/vortex_cuda_tree.py:429-436 -> bs_last_stats
 *
 * Conventions.  Every array argument is a DEVICE pointer owned by the caller, float64 unless stated, C-contiguous:
 * points [n,3], starts [m,3], directions [m,3] (unit), lengths [m] (> 0), gamma [m], radius [m] (>= 0);
 * exclusions as the reference's CSR (vortex_numba.exclusion_csr, vortex_numba.py:228-243): ex_ptr int64 [n+1],
 * ex_seg int64 [e], sorted and unique per target (ex_ptr may be NULL for no exclusions).  Outputs: out [n,3] float64,
 * flags int8 [n] with the reference's codes (0 ok, 1 singular, 2 non-finite; vortex_numba.py:32-34).  Flags are not
 * errors: the caller re-runs its own reference to raise, as vortex.py:488-492 does.
 * Scratch memory is taken from a per-context stream-ordered pool (cudaMallocAsync) on the call's stream.
 * Every entry point returns a bs_status and never aborts or traps; work is enqueued on `stream` and the host blocks only
 * where stated (tree builds read node counts back).
 */
#ifndef BS_B200_H
#define BS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bs_ctx bs_ctx;
typedef struct bs_tree bs_tree;
typedef void *bs_stream; /* cudaStream_t */

typedef enum {
    BS_OK = 0,
    BS_ERR_ARG = 1,      /* invalid argument (the reference raises ValueError) */
    BS_ERR_CUDA = 2,     /* a CUDA runtime call failed; bs_last_error has the text */
    BS_ERR_STACK = 3,    /* tree traversal stack overflow (the reference raises RuntimeError, vortex_cuda_tree.py:548) */
    BS_ERR_TIMEOUT = 4,  /* a bounded device-side wait gave up */
    BS_ERR_OOM = 5       /* the memory pool could not satisfy an allocation */
} bs_status;

typedef enum { BS_FP64 = 0, BS_MIXED = 1, BS_FP32 = 2 } bs_precision;
typedef enum { BS_TREE_MEDIAN = 0, BS_TREE_MORTON = 1 } bs_tree_kind;

typedef struct {
    int64_t m;
    const double *starts, *directions, *lengths, *gamma, *radius;
} bs_sources;

typedef struct {
    int64_t n;
    const double *points;
    const int64_t *ex_ptr; /* NULL: no exclusions */
    const int64_t *ex_seg;
    int64_t e;
} bs_targets;

typedef struct {
    int model;          /* CoreModel 0..5 (vortex.py:21-27) */
    int raise_singular; /* 1 for singularity='raise' */
    int precision;      /* bs_precision */
    int block;          /* threads per block: 32, 64, 128 or 256 (CudaSettings.block) */
    double near_cores;  /* single precisions: pairs within near_cores core radii of a segment are done in FP64
                           (model 0, which has no core: pairs within a quarter of the segment's length of it) */
} bs_kernel_params;

typedef struct {
    double theta;      /* opening ratio, 0 < theta < 1 (TreeSettings.theta) */
    int order;         /* expansion order 0, 1 or 2 (the reference's); 3, 4 and 5 add the third- to fifth-order
                          terms (a tree evaluated at order 3, 4 or 5 must be built with at least that order, which
                          computes the higher moments) */
    int64_t leaf_size; /* maximum segments per leaf */
    double clearance;  /* core clearance in largest core radii */
    int kind;          /* bs_tree_kind */
    int stack_limit;   /* traversal stack entries per warp, 0 = the maximum (128); overflow returns BS_ERR_STACK */
} bs_tree_params;

typedef struct {
    int64_t points, segments, nodes, launches;
    int64_t far_evaluations, near_pairs, fp64_pairs, visits; /* counters of the last tree evaluation */
    double build_ms, moments_ms, evaluate_ms;                /* device time of the last build / evaluation */
    int64_t pair_slots;  /* lane slots spent in leaf walks (32 per warp-pair); near_pairs / pair_slots = SIMT use */
    double walk_ms, list_ms; /* device time of the traversal and of the near-leaf list kernel of the last tree evaluation */
    double upload_ms, download_ms; /* host time of the last bs_tree_sum_host's uploads and of its result read-back */
    double far_ms;       /* device time of the far-node list kernel of the last tree evaluation */
} bs_stats;

/* Context: one per device.  bs_init makes `device` current, probes it with a one-thread kernel (the reference's
 * available(), vortex_cuda.py:58-77) and creates the memory pool.  A context serves one call at a time: its
 * statistics, side stream, upload ring and pinned read-back words belong to the call in progress (host threads that
 * call concurrently use a context each). */
int bs_init(int device, bs_ctx **ctx);
void bs_destroy(bs_ctx *ctx);
/* Text of the last error on this thread (never NULL). */
const char *bs_last_error(void);
int bs_last_stats(const bs_ctx *ctx, bs_stats *stats);
/* Library version and the compute capability it was built for (100 for sm_100a). */
int bs_version(int *major, int *minor, int *arch);
/* Copies `bytes` from ordinary (pageable) host memory to device memory on `stream` through a pinned staging ring:
 * several host threads fill 4 MiB pinned chunks while earlier chunks transfer.  Returns once the source has been read
 * (the last transfers may still be in flight on the stream). */
int bs_upload(bs_ctx *ctx, void *dst, const void *src, size_t bytes, bs_stream stream);
/* bs_upload for `count` arrays in one pass of the staging ring (dst[i] <- src[i], bytes[i] each): the next array's
 * first chunk is staged while the previous array's last chunks transfer.  Used by the drop-in backends, whose inputs
 * arrive as several host arrays per call.  Same return rule as bs_upload. */
int bs_upload_many(bs_ctx *ctx, int count, void *const *dst, const void *const *src, const size_t *bytes,
                   bs_stream stream);
/* Device -> ordinary host memory for `count` arrays (dst[i] host <- src[i] device, bytes[i] each) through the same
 * pinned ring: the transfer of one chunk overlaps the host copy of the previous one.  Ordered after the work queued
 * on `stream`; returns when every byte has arrived. */
int bs_download_many(bs_ctx *ctx, int count, void *const *dst, const void *const *src, const size_t *bytes,
                     bs_stream stream);
/* Measures the device's FP32 FMA throughput (TFLOP/s, an FMA counted as 2) with a kernel of independent FMA chains
 * on every SM: the denominator of the pair kernels' roofline, which run on the FP32 pipe. */
int bs_fp32_peak(bs_ctx *ctx, double *tflops);

/* Exact direct sum (vortex_numba._sum_point semantics, vortex_numba.py:112-147): every non-excluded (target, segment)
 * pair, segment order preserved inside each thread's range; BS_FP64 sums in FP64, BS_MIXED/BS_FP32 use FP32 pair
 * arithmetic on two-float coordinates with FP64 re-evaluation near segments (reference: vortex_cuda.py:179-351). */
int bs_direct(bs_ctx *ctx, const bs_sources *src, const bs_targets *tgt, const bs_kernel_params *kp, double *out,
              int8_t *flags, bs_stream stream);

/* Allocation-free direct sum.  No counterpart in the reference: for callers that must not allocate GPU memory while
 * they run (a control or flight loop with a hard per-step deadline, where an allocation can stall or fail once another
 * framework's allocator has reserved the device, or a plugin inside a host that owns all device memory).  Same
 * semantics and arguments as bs_direct without the context (it runs on the current device, in one segment chunk), but
 * its scratch is one fixed array compiled into the library, so it calls no cudaMalloc/cudaFree and no allocating
 * library routine.  Limits and caveats:
 *   - at most BS_NOALLOC_MAX_SEGMENTS segments (BS_ERR_ARG beyond); targets are not limited;
 *   - every GPU that loads the library holds the BS_NOALLOC_SCRATCH_BYTES array until the process exits;
 *   - it runs on the current device; every pointer argument must be device memory of that device (or memory the
 *     device can address), BS_ERR_ARG otherwise;
 *   - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with that device current
 *     and keeps it for the life of the process; make that first call before any stream capture, and make no call on a
 *     device after cudaDeviceReset (or any reset of its primary context) in the same process, since the kept address
 *     then no longer maps the array;
 *   - all calls share the one array: calls that overlap on the GPU (other streams, other host threads) race and must
 *     be serialised by the caller;
 *   - blocks the host until the result is ready, like bs_direct. */
#define BS_NOALLOC_MAX_SEGMENTS 65536
#define BS_NOALLOC_SCRATCH_BYTES (65536 * 144 + 256) /* 9 MiB of FP64 + FP32 segment records, 256 B of flags */
int bs_direct_noalloc(const bs_sources *src, const bs_targets *tgt, const bs_kernel_params *kp, double *out,
                      int8_t *flags, bs_stream stream);

/* bs_tree_sum from and to ordinary host memory: `src` and `tgt` hold HOST pointers (the reference backend's NumPy
 * inputs, vortex_cuda_tree.py:439-595; tgt->ex_ptr/ex_seg a host CSR or NULL), `out`, `flags` and `far_counts` (may be
 * NULL) are host buffers.  The uploads go through the pinned staging ring; for a Morton tree the circulations and core
 * radii are uploaded on a second stream while the device sorts the keys and builds the topology from starts,
 * directions and lengths.  Results equal bs_tree_sum's on the same inputs.  Blocks until the results are in `out`. */
int bs_tree_sum_host(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, const bs_targets *tgt,
                     const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts, bs_stream stream);

/* Tree build on the device (Morton keys + radix sort + binary radix tree, or the reference's median split element for
 * element).  Node moments and contractions about cell centres in FP64 (vortex_tree.node_moments semantics).  Blocks
 * the host while reading node counts back. */
int bs_tree_build(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, bs_tree **tree, bs_stream stream);
/* A tree from caller arrays (device int64 order [m], lo/hi/left/right [count]); moments computed on the device.
 * Evaluates the reference's own tree (vortex_tree.build_tree output) with these kernels. */
int bs_tree_from_arrays(bs_ctx *ctx, const bs_sources *src, const int64_t *order, const int64_t *lo,
                        const int64_t *hi, const int64_t *left, const int64_t *right, int64_t count,
                        bs_tree **tree, bs_stream stream);
void bs_tree_free(bs_tree *tree);
int64_t bs_tree_count(const bs_tree *tree);
/* Copy the tree arrays to caller DEVICE buffers (any pointer may be NULL): order [m], lo/hi/left/right [count] int64,
 * centre [count,3], bound, core [count], m0 [count,3], m1 [count,3,3], m2 [count,3,3,3], w1 [count,3], t2 [count,3],
 * w2 [count,3,3] float64. */
int bs_tree_export(const bs_tree *tree, int64_t *order, int64_t *lo, int64_t *hi, int64_t *left, int64_t *right,
                   double *centre, double *bound, double *core, double *m0, double *m1, double *m2, double *w1,
                   double *t2, double *w2, bs_stream stream);
/* Morton keys of the segment midpoints (uint64 [m]) and their stable sort permutation (int64 [m]); either may be NULL.
 * The bit-exact CPU recomputation is oracle/morton_oracle.c. */
int bs_tree_keys(const bs_tree *tree, uint64_t *keys, int64_t *sorted_order, bs_stream stream);

/* Tree evaluation (vortex_tree.tree_velocity semantics, vortex_tree.py:508-568): per-target acceptance, DFS order,
 * exclusions force nodes open, leaves use the exact pair kernel.  far_counts (int64 [n]) may be NULL.  On Morton trees
 * in BS_MIXED or BS_FP32 a leaf opened for one target of a warp (32 sorted targets) is also summed exactly for the
 * targets of that warp that accepted it as far (their far counts exclude it); median trees and BS_FP64 keep each
 * target's own decisions. */
int bs_tree_eval(bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
                 const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts, bs_stream stream);

/* Forests: many wakes in one tree, for batched evaluation (no counterpart in the reference, which evaluates one wake
 * per call).  The segments of all wakes are concatenated; wake w holds segments [wake_ptr[w], wake_ptr[w+1]) (device
 * int64 [nwakes+1]).  Keys carry the wake number above a Morton key in the wake's own box, so every wake's segment
 * range is one node of the traversal tree, its root; wakes never see each other. */
typedef struct bs_graph bs_graph;
int bs_forest_build(bs_ctx *ctx, const bs_sources *src, int nwakes, const int64_t *wake_ptr, const bs_tree_params *tp,
                    bs_tree **forest, bs_stream stream);
/* Root node of each wake (device int32 [nwakes]; -1 for a wake without segments). */
int bs_forest_roots(const bs_tree *forest, int32_t *roots, bs_stream stream);
/* Evaluate every wake at its own targets: targets of wake w are [target_wake_ptr[w], target_wake_ptr[w+1]) of the
 * concatenated target array (device int64 [nwakes+1]).  One traversal launch and one persistent list kernel for all
 * wakes; exclusion CSR segment ids are global (offset by the wake's first segment). */
int bs_forest_eval(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp, const bs_targets *tgt,
                   const int64_t *target_wake_ptr, const bs_kernel_params *kp, double *out, int8_t *flags,
                   int64_t *far_counts, bs_stream stream);
/* Capture the evaluation of bs_forest_eval (target_wake_ptr may be NULL for a plain tree) into a CUDA graph with its
 * scratch pre-allocated; bs_graph_launch replays it on any stream (same tree, same buffers; new target positions may
 * be written into the same target buffer between launches).  bs_graph_status reads the counters of the last launch
 * (blocking) and returns BS_ERR_STACK after a traversal stack overflow. */
int bs_forest_graph(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp, const bs_targets *tgt,
                    const int64_t *target_wake_ptr, const bs_kernel_params *kp, double *out, int8_t *flags,
                    int64_t *far_counts, bs_graph **graph);
/* bs_forest_eval / bs_forest_graph with targets summed exactly (the batched form of the reference's control-point
 * induction, vsm_wake.history_vsm_induction, src/openfawe/aero/vsm_wake.py:255-300, which sums the wake exactly at a
 * wing's control and load points): exact (device uint8 [n], input order; NULL = none) marks targets for which no far
 * node is accepted, so their velocity is the full sum over their wake's segments (in tree order, FP64 near-field rule
 * of the precision), evaluated in the same traversal and persistent list launch as the other targets; their far
 * counts are zero. */
int bs_forest_eval_exact(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp, const bs_targets *tgt,
                         const int64_t *target_wake_ptr, const uint8_t *exact, const bs_kernel_params *kp,
                         double *out, int8_t *flags, int64_t *far_counts, bs_stream stream);
int bs_forest_graph_exact(bs_ctx *ctx, const bs_tree *forest, const bs_tree_params *tp, const bs_targets *tgt,
                          const int64_t *target_wake_ptr, const uint8_t *exact, const bs_kernel_params *kp,
                          double *out, int8_t *flags, int64_t *far_counts, bs_graph **graph);
int bs_graph_launch(bs_graph *graph, bs_stream stream);
int bs_graph_status(bs_graph *graph, bs_stats *stats);
void bs_graph_free(bs_graph *graph);

/* Adjoint of the exact direct sum (no counterpart in the reference, which has no adjoint): given the cotangent w
 * [n,3] of the induced velocity, writes d(sum_p w_p . u_p) with respect to the targets [n,3], the segment starts A and
 * ends B [m,3] and the circulations [m]; any output may be NULL.  Segments are given by their endpoints; every core
 * model (0..5); excluded and on-axis pairs contribute nothing.  FP64, pair terms recomputed. */
int bs_adjoint_direct(bs_ctx *ctx, int64_t n, const double *points, int64_t m, const double *A, const double *B,
                      const double *gamma, const double *radius, const int64_t *ex_ptr, const int64_t *ex_seg,
                      int64_t e, int model, const double *cotangent, double *grad_points, double *grad_A,
                      double *grad_B, double *grad_gamma, bs_stream stream);

/* Adjoint of the tree sum (no counterpart in the reference, which has no adjoint): for the cotangent w [n,3] of the
 * velocities bs_tree_sum returns with the same arguments, d(sum_p w_p . u_p) with respect to the targets [n,3], the
 * segment starts A and ends B = A + L d [m,3] and the circulations [m] (any output may be NULL), as the derivative of
 * the forward the tree code evaluates: the same tree (built again), the same accepted nodes and near pairs (the walk
 * runs again), pair terms and expansions recomputed; node centres and acceptance decisions are held fixed.  Near pairs
 * in FP32 (kp->precision BS_MIXED or BS_FP32) with FP64 where the forward takes FP64, or all in FP64 (BS_FP64); the
 * far field's derivatives in FP64.  Every core model (0..5; the Vatistas, offset and Rosenhead-Moore cores with FP64
 * near pairs in either precision); orders 0..5.  Gradients are summed with
 * atomics (repeatable to rounding).  BS_ERR_OOM if a warp's interaction list exceeds the list pool.  Blocks until
 * the gradients are written.  Afterwards bs_last_stats holds its stage times: build_ms the build, walk and list
 * transposition, walk_ms the near pairs, list_ms the far entries, moments_ms the push-down and segment moments. */
int bs_tree_adjoint(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, const bs_targets *tgt,
                    const bs_kernel_params *kp, const double *cotangent, double *grad_points, double *grad_starts,
                    double *grad_ends, double *grad_gamma, bs_stream stream);

/* The reference's median-split tree from midpoints alone (replaces vortex_cuda_build.device_build_tree,
 * src/openfawe/aero/vortex_cuda_build.py:234-275, and vortex_tree.build_tree, vortex_tree.py:208-241): order [m] and,
 * when *count <= capacity, lo/hi/left/right [count] in depth-first numbering, element for element equal to
 * build_tree's.  mid [m][3] float64; all device.  Synchronises the stream. */
int bs_median_topology(bs_ctx *ctx, int64_t m, const double *mid, int leaf_size, int64_t *order, int64_t *lo,
                       int64_t *hi, int64_t *left, int64_t *right, int64_t capacity, int64_t *count, bs_stream stream);

/* Node quantities of a given tree (replaces vortex_cuda_moments.device_node_quantities,
 * src/openfawe/aero/vortex_cuda_moments.py:206-230, i.e. vortex_tree.node_moments + node_contractions): for the
 * tree (order [m], lo, hi [count]) over segments with starts, ends, length vectors [m][3], gamma, radius [m], writes
 * centre [count][3], bound, core [count], m0 [count][3], m1 [count][3][3], m2 [count][3][3][3], w1, t2 [count][3],
 * w2 [count][3][3] (any may be NULL).  The vortex vectors are gamma * length_vectors.  Synchronises. */
int bs_node_quantities(bs_ctx *ctx, int64_t m, const double *starts, const double *ends, const double *length_vectors,
                       const double *gamma, const double *radius, int64_t count, const int64_t *order,
                       const int64_t *lo, const int64_t *hi, double *centre, double *bound, double *core, double *m0,
                       double *m1, double *m2, double *w1, double *t2, double *w2, bs_stream stream);

/* Incident-endpoint exclusion pairs of a wake network (replaces network_numba.incident_pairs,
 * src/openfawe/aero/network_numba.py:242-256): for every segment s of edges [segments][2] in order and each of its two
 * ends, the pairs (i, s) of every free point i (node first + i, first in [0, n]) whose three coordinates equal that
 * end node's bit for bit (NaN never matches), i increasing.  nodes [n][3] float64, edges, pairs [capacity][2] int64,
 * all device.  *count (host) receives the number of pairs; they are written only if it is <= capacity (call again
 * with a larger buffer otherwise).  An edge index outside [0, n) is BS_ERR_ARG.  Synchronises the stream. */
int bs_incident_pairs(bs_ctx *ctx, const double *nodes, int64_t n, const int64_t *edges, int64_t segments,
                      int64_t first, int64_t *pairs, int64_t capacity, int64_t *count, bs_stream stream);

/* Per-point sorted unique excluded segments from (point, segment) pairs [e][2] (replaces vortex_numba.exclusion_csr,
 * src/openfawe/aero/vortex_numba.py:228-243, and its np.unique reference :179-190): ptr [n+1] and seg [>= e] device
 * int64; *unique_count (host) receives the length of seg.  A point outside [0, n) is BS_ERR_ARG.  Synchronises. */
int bs_exclusion_csr(bs_ctx *ctx, int64_t n, const int64_t *pairs, int64_t e, int64_t *ptr, int64_t *seg,
                     int64_t *unique_count, bs_stream stream);

/* Unit-circulation pair matrix (replaces vortex_numba.pair_matrix, src/openfawe/aero/vortex_numba.py:271-287):
 * out [n][m][3] = the FP64 velocity of segment s with circulation 1 at point p (zero for a flagged pair), flags [n] =
 * the flag of the point's first flagged segment.  src->gamma is not read. */
int bs_pair_matrix(bs_ctx *ctx, int64_t n, const double *points, const bs_sources *src, int model, int raise_singular,
                   double *out, int8_t *flags, bs_stream stream);

/* Panel columns from a pair matrix (replaces vortex_numba.assemble_columns, vortex_numba.py:290-308): out [n][columns]
 * [3][j] = sum over k in [column_ptr[j], column_ptr[j+1]), in order from 0.0, of column_sign[k] * pairs[p]
 * [column_segment[k]].  column_ptr must not decrease and every column_segment must lie in [0, m) (BS_ERR_ARG). */
int bs_assemble_columns(bs_ctx *ctx, int64_t n, int64_t m, const double *pairs, int64_t columns,
                        const int64_t *column_ptr, const int64_t *column_segment, const double *column_sign,
                        double *out, bs_stream stream);

/* bs_pair_matrix followed by bs_assemble_columns without storing the pair matrix (the VSM ring operators of
 * vsm_wake._batched_ring_operator, src/openfawe/aero/vsm_wake.py:224-252); flags as bs_pair_matrix's over the
 * segments the columns use. */
int bs_ring_columns(bs_ctx *ctx, int64_t n, const double *points, const bs_sources *src, int model, int raise_singular,
                    int64_t columns, const int64_t *column_ptr, const int64_t *column_segment,
                    const double *column_sign, double *out, int8_t *flags, bs_stream stream);

/* Build + evaluate + free (cuda_tree_sum in one call). */
int bs_tree_sum(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, const bs_targets *tgt,
                const bs_kernel_params *kp, double *out, int8_t *flags, int64_t *far_counts, bs_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* BS_B200_H */
