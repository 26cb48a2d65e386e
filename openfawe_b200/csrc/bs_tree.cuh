// Internal tree object shared by the build, moments and evaluation translation units.
#pragma once
#include <functional>

#include "bs_internal.cuh"

namespace bs {

// Per-segment geometry in input order, formed as vortex_tree.tree_sum forms it (vortex_tree.py:608-611):
// lv = d * L, end = start + lv, alpha = gamma * lv (IEEE multiply then add, no contraction).
struct __align__(16) SegGeo {
    double sx, sy, sz, ex, ey, ez;
    double lx, ly, lz, gamma, radius, pad;
};

// pairs (may be null): also the packed-pair records (Seg32x2) of the same order.
int pack_segments(const bs_sources *src, const int32_t *order, Seg64 *seg64, Seg32 *seg32, SegGeo *geo,
                  cudaStream_t s, Seg32x2 *pairs = nullptr);
// side (may be null): the stream for the moment phase of the bottom-up pipeline (bs_tree::moments_done marks its end).
int compute_moments(bs_tree *tree, const SegGeo *geo, Scratch &scratch, cudaStream_t s, cudaStream_t side);

}  // namespace bs

struct bs_tree {
    int device = 0;
    int kind = 0;
    cudaMemPool_t pool = nullptr;
    int64_t m = 0, count = 0, leaf_size = 0;
    int64_t *order = nullptr, *lo = nullptr, *hi = nullptr, *left = nullptr, *right = nullptr;  // export layout
    int32_t *order32 = nullptr, *inverse = nullptr;                                              // position <-> id
    double *centre = nullptr, *bound = nullptr, *core = nullptr, *m0 = nullptr, *m1 = nullptr, *m2 = nullptr;
    double *w1 = nullptr, *t2 = nullptr, *w2 = nullptr;
    bs::NodeRec *nodes = nullptr;
    bs::Far64 *far64 = nullptr;
    bs::Far32 *far32 = nullptr;
    bs::Far64x *far64x = nullptr;  // third-order records (trees built for order 3 or more)
    bs::Far32x *far32x = nullptr;
    bs::Far64y *far64y = nullptr;  // fourth-order records (trees built for order 4 or 5)
    bs::Far32y *far32y = nullptr;
    bs::Far64z *far64z = nullptr;  // fifth-order records (trees built for order 5 only)
    bs::Far32z *far32z = nullptr;
    int order3 = 0, order4 = 0, order5 = 0;
    bool geo_sorted = false;  // the build's segment geometry (SegGeo) is in tree order (Morton trees)
    bool records_done = false;  // the tree-ordered segment records are queued (segment_records)
    int64_t *host_count = nullptr;  // pinned word the node count is read back into (null: a pageable word)
    bs::Seg64 *seg64 = nullptr;  // tree order
    bs::Seg32 *seg32 = nullptr;  // tree order
    bs::Seg32x2 *seg32x2 = nullptr;  // tree order, consecutive pairs
    bs::Seg32c2 *seg32c2 = nullptr;  // tree order, consecutive pairs relative to their leaf's centre
    uint64_t *keys = nullptr;    // Morton keys (input order), Morton trees only
    int32_t *wake_root = nullptr;  // forests: root node of each wake (-1 for a wake without segments)
    int nwakes = 0;
    float build_ms = 0.f, moments_ms = 0.f;
    // build start, moments start, moments end; with the moments on a side stream also the end of the leaf pass (the
    // segment and clear-leaf records complete: what the near-leaf list kernel reads)
    cudaEvent_t marks[4] = {nullptr, nullptr, nullptr, nullptr}; 
    // marks[2] when the far records are still being computed on a side stream after the build returned (the node
    // records are complete): work that reads them waits for it; else null
    cudaEvent_t moments_done = nullptr;
    void *blocks[48];
    int nblocks = 0;
    template <class T> T *alloc(size_t elems, cudaStream_t s) {
        if (nblocks >= 48) return nullptr;
        void *p = nullptr;
        if (cudaMallocFromPoolAsync(&p, (elems ? elems : 1) * sizeof(T), pool, s) != cudaSuccess) return nullptr;
        blocks[nblocks++] = p;
        return static_cast<T *>(p);
    }
};

// Build without waiting (bs_tree_sum): the stage times are read by tree_stage_times after the stream synchronised;
// before_geometry (may be empty) runs on the host once, before any kernel reads gamma or radius (for Morton trees
// while the node count is read back), so that a caller can still be uploading those two arrays;
// tree_release frees the tree's memory stream-ordered on s, after the work queued there.  With a side stream (not
// waiting), the moments and far records of a bottom-up tree are computed there, concurrently with what s runs after
// the node records (the walk): bs_tree::moments_done marks their end.
int tree_build(bs_ctx *ctx, const bs_sources *src, const bs_tree_params *tp, bs_tree **out, cudaStream_t s,
               bool wait, const std::function<int()> &before_geometry, cudaStream_t side = nullptr);
void tree_stage_times(bs_tree *t);
void tree_release(bs_tree *tree, cudaStream_t s);

namespace bs {

// Interaction lists of the traversal (the walk of bs_tree_eval), shared with the adjoint.  Warp gw of the sorted
// targets owns list_len[gw] entries, entry k at list[unit_chunks[gw * LIST_CHUNKS + k / LIST_CHUNK] * LIST_CHUNK +
// k % LIST_CHUNK]: (node, lane mask) for a near leaf, (node | FAR_BIT, lane mask) for an accepted far node; lane l of
// warp gw is sorted target gw * 32 + l, target perm[gw * 32 + l].
constexpr int LIST_CHUNK = 128;  // list entries per chunk of the shared list pool
constexpr int LIST_CHUNKS = 32;  // chunks a warp's list may hold (4096 entries)
constexpr int LIST_POOL = 4096;  // pool entries per warp of targets
constexpr int FAR_BIT = int(0x80000000u);

struct TreeLists {
    int64_t n = 0, target_warps = 0;
    const int32_t *perm = nullptr;    // sorted target -> target
    const int32_t *ex_pos = nullptr;  // excluded tree positions per target (ranges ex_ptr[p] .. ex_ptr[p + 1]), or null
    const int64_t *ex_ptr = nullptr;
    const int2 *list = nullptr;
    const int *unit_chunks = nullptr;
    const int *list_len = nullptr;
    unsigned long long *state = nullptr;  // device: overflow word (low: stack, high: list full), 5 counters
};

// The walk alone, on s, every interaction going into the lists (none is evaluated): sorts the targets, maps their
// exclusions to tree positions and fills `lists`.  A warp whose list does not fit sets the overflow word's high half;
// a stack overflow sets its low half (the caller reads `state` back).  MODEL 0..2.
int tree_lists(const bs_ctx *ctx, const bs_tree *tree, const bs_tree_params *tp, const bs_targets *tgt,
               const bs_kernel_params *kp, Scratch &scratch, cudaStream_t s, TreeLists *lists);

}  // namespace bs
