/*
 * CPU recomputation of the B200 build's Morton-key tree -- TEST INFRASTRUCTURE ONLY.
 *
 * The Morton tree is this project's own design (the reference splits at the median, vortex_tree.py:51-115).  The CUDA
 * library builds it on the device; this file states the same specification on the CPU so that the device's keys,
 * sort permutation and tree arrays can be checked element for element (bit-exact), and so that the oracle's
 * tree_velocity (bs_oracle.c, the reference's traversal) can evaluate the very same tree.
 *
 * Specification (shared with openfawe_b200/csrc/bs_tree_build.cu):
 *   mid    = 0.5 * (s + (s + d*L))                       per axis, IEEE round-to-nearest, no fused multiply-add
 *   box    = [min mid, max mid] per axis;  extent = max over axes of (max - min)
 *   inv    = 65536 / extent   (0 when extent == 0)
 *   q      = min(2^16 - 1, (uint32)((mid - min) * inv))  truncation toward zero
 *   key    = bit-interleave(qx, qy, qz): bit i of x -> 3i+2, of y -> 3i+1, of z -> 3i    (48 bits)
 *   sort   = stable by key (ties keep segment index order)
 *   topology: the binary radix tree of Karras (HPG 2012) over the sorted keys, ties broken by position;
 *   traversal tree: internal nodes holding more than leaf_size segments ("big") plus their non-big children as leaves,
 *   numbered by an exclusive scan over the internal-node index (big node i at slot[i], its non-big children at
 *   slot[i]+1, slot[i]+2, left child first).  lo/hi/left/right use the reference's conventions (vortex_tree.py:53).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MORTON_BITS 16
#define MORTON_SCALE 65536.0

static uint64_t spread3(uint32_t v)
{
    uint64_t x = v & 0xffff;
    uint64_t out = 0;
    for (int i = 0; i < MORTON_BITS; ++i) out |= ((x >> i) & 1ull) << (3 * i);
    return out;
}

/* box[6] = (min x, min y, min z, max x, max y, max z) of mid; returns inv. */
double orc_morton_box(int64_t m, const double *mid, double *box)
{
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t s = 0; s < m; ++s)
        for (int a = 0; a < 3; ++a) {
            double v = mid[3 * s + a];
            if (v < lo[a]) lo[a] = v;
            if (v > hi[a]) hi[a] = v;
        }
    double extent = 0.0;
    for (int a = 0; a < 3; ++a) {
        box[a] = lo[a];
        box[3 + a] = hi[a];
        double e = hi[a] - lo[a];
        if (e > extent) extent = e;
    }
    return extent > 0.0 ? MORTON_SCALE / extent : 0.0;
}

void orc_morton_keys(int64_t m, const double *mid, const double *box, double inv, uint64_t *keys)
{
    for (int64_t s = 0; s < m; ++s) {
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            double v = (mid[3 * s + a] - box[a]) * inv;
            uint32_t u = (uint32_t)v;
            q[a] = u > 65535u ? 65535u : u;
        }
        keys[s] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    }
}

/* Stable LSD sort of (key, index): order[k] = segment at sorted position k, sorted[k] its key. */
void orc_morton_sort(int64_t m, const uint64_t *keys, int64_t *order, uint64_t *sorted)
{
    int64_t *tmp_o = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    uint64_t *tmp_k = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(m > 0 ? m : 1));
    for (int64_t i = 0; i < m; ++i) { order[i] = i; sorted[i] = keys[i]; }
    for (int pass = 0; pass < 8; ++pass) {
        int shift = 8 * pass;
        int64_t count[257];
        memset(count, 0, sizeof count);
        for (int64_t i = 0; i < m; ++i) count[((sorted[i] >> shift) & 255) + 1]++;
        for (int b = 0; b < 256; ++b) count[b + 1] += count[b];
        for (int64_t i = 0; i < m; ++i) {
            int64_t o = count[(sorted[i] >> shift) & 255]++;
            tmp_o[o] = order[i];
            tmp_k[o] = sorted[i];
        }
        memcpy(order, tmp_o, sizeof(int64_t) * (size_t)m);
        memcpy(sorted, tmp_k, sizeof(uint64_t) * (size_t)m);
    }
    free(tmp_o);
    free(tmp_k);
}

static int delta(const uint64_t *k, int64_t n, int64_t i, int64_t j)
{
    if (j < 0 || j >= n) return -1;
    if (k[i] == k[j]) return 64 + __builtin_clzll((uint64_t)(i ^ j));
    return __builtin_clzll(k[i] ^ k[j]);
}

/* Karras internal node i of n sorted keys: inclusive range [*first, *last] and split gamma. */
static void karras_node(const uint64_t *k, int64_t n, int64_t i, int64_t *first, int64_t *last, int64_t *split)
{
    int d = delta(k, n, i, i + 1) - delta(k, n, i, i - 1) > 0 ? 1 : -1;
    int dmin = delta(k, n, i, i - d);
    int64_t lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    int64_t j = i + l * d;
    int dnode = delta(k, n, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    *split = i + s * d + (d < 0 ? -1 : 0);
    *first = i < j ? i : j;
    *last = i < j ? j : i;
}

/* The traversal tree of the spec above.  Arrays of capacity 2*n (n >= 1); returns the node count. */
int64_t orc_morton_tree(int64_t n, const uint64_t *sorted, int64_t leaf_size, int64_t *lo, int64_t *hi, int64_t *left,
                        int64_t *right)
{
    if (n <= 0) return 0;
    if (n <= leaf_size || n == 1) {
        lo[0] = 0; hi[0] = n; left[0] = -1; right[0] = -1;
        return 1;
    }
    int64_t ni = n - 1;
    int64_t *first = (int64_t *)malloc(sizeof(int64_t) * (size_t)ni);
    int64_t *last = (int64_t *)malloc(sizeof(int64_t) * (size_t)ni);
    int64_t *split = (int64_t *)malloc(sizeof(int64_t) * (size_t)ni);
    int64_t *slot = (int64_t *)malloc(sizeof(int64_t) * (size_t)ni);
    for (int64_t i = 0; i < ni; ++i) karras_node(sorted, n, i, first + i, last + i, split + i);
    int64_t count = 0;
    for (int64_t i = 0; i < ni; ++i) {
        slot[i] = count;
        if (last[i] - first[i] + 1 <= leaf_size) continue;
        int64_t c = 1;
        int64_t g = split[i];
        int left_big = !(g == first[i]) && (last[g] - first[g] + 1 > leaf_size);
        int right_big = !(g + 1 == last[i]) && (last[g + 1] - first[g + 1] + 1 > leaf_size);
        c += !left_big;
        c += !right_big;
        count += c;
    }
    for (int64_t i = 0; i < ni; ++i) {
        if (last[i] - first[i] + 1 <= leaf_size) continue;
        int64_t me = slot[i], next = me + 1;
        int64_t g = split[i];
        lo[me] = first[i];
        hi[me] = last[i] + 1;
        int left_leafseg = g == first[i], right_leafseg = g + 1 == last[i];
        int left_big = !left_leafseg && (last[g] - first[g] + 1 > leaf_size);
        int right_big = !right_leafseg && (last[g + 1] - first[g + 1] + 1 > leaf_size);
        if (left_big) {
            left[me] = slot[g];
        } else {
            left[me] = next;
            lo[next] = first[i];
            hi[next] = g + 1;
            left[next] = right[next] = -1;
            ++next;
        }
        if (right_big) {
            right[me] = slot[g + 1];
        } else {
            right[me] = next;
            lo[next] = g + 1;
            hi[next] = last[i] + 1;
            left[next] = right[next] = -1;
            ++next;
        }
    }
    free(first); free(last); free(split); free(slot);
    return count;
}
