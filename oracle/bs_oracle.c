/*
 * CPU oracle for the Biot-Savart hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's FP64 algorithms, operation for operation, so that its results can be
 * compared bit for bit with the reference's own numba code (golden fixtures under tests/golden/) and used as the
 * checker of the CUDA library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the
 * product (openfawe_b200) never does.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off; no fast-math, no FMA contraction, libm's hypot and
 * expm1, exactly the calls numba makes).
 *
 * Reference files followed (paths inside the reference project):
 *   pair_velocity        src/openfawe/aero/vortex_numba.py:42-109
 *   _sum_point           src/openfawe/aero/vortex_numba.py:112-147   (direct sum, ordered per target)
 *   exclusion_csr        src/openfawe/aero/vortex_numba.py:193-243
 *   incident_pairs       src/openfawe/aero/network_numba.py:176-256
 *   pair_matrix          src/openfawe/aero/vortex_numba.py:271-287
 *   build_tree_serial    src/openfawe/aero/vortex_tree.py:51-115     (== build_tree element for element, :208-241)
 *   node_moments         src/openfawe/aero/vortex_tree.py:118-167, 320-376
 *   node_contractions    src/openfawe/aero/vortex_tree.py:425-447
 *   far_velocity         src/openfawe/aero/vortex_tree.py:450-497
 *   tree_velocity        src/openfawe/aero/vortex_tree.py:508-568
 *   _positions           src/openfawe/aero/vortex_tree.py:571-580
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FLAG_OK 0
#define FLAG_SINGULAR 1
#define FLAG_NONFINITE 2
#define TREE_STACK 512

static const double AXIS_EPS = 8.0 * 2.220446049250313e-16;   /* 8 * finfo(float64).eps */
static double lamb_cut(void) { return sqrt(10.0 / 1.25643); }
static const double FOUR_PI = 4.0 * 3.141592653589793;          /* 4 * np.pi */
static const double INV_FOUR_PI = 1.0 / (4.0 * 3.141592653589793);

static inline double norm3(double x, double y, double z) { return hypot(hypot(x, y), z); }
static inline int finite(double v) { return isfinite(v); }

/* vortex_numba.pair_velocity, vortex_numba.py:42-109. */
int orc_pair(double px, double py, double pz, double sx, double sy, double sz, double dx, double dy, double dz,
             double length, double gamma, int model, double radius, int raise_singular, double *u)
{
    u[0] = u[1] = u[2] = 0.0;
    double ax = (px - sx) / length;
    double ay = (py - sy) / length;
    double az = (pz - sz) / length;
    double t = (ax * dx + ay * dy) + az * dz;
    double cx = dy * az - dz * ay;
    double cy = dz * ax - dx * az;
    double cz = dx * ay - dy * ax;
    double h = norm3(cx, cy, cz);
    double na = norm3(ax, ay, az);
    double nb = norm3(ax - dx, ay - dy, az - dz);
    if (!(finite(h) && finite(na) && finite(nb) && finite(t))) return FLAG_NONFINITE;
    double big = na > nb ? na : nb;                 /* max(na, nb) */
    double scale = 1.0 > big ? 1.0 : big;           /* max(1.0, ...) */
    if (h <= AXIS_EPS * scale) {
        if (raise_singular && t >= 0.0 && t <= 1.0) return FLAG_SINGULAR;
        return FLAG_OK;
    }
    if (gamma == 0.0) return FLAG_OK;
    double product = na * nb;
    double dot = h * h + t * (t - 1.0);
    double plus = product + dot;
    if (dot < 0.0) plus = (h * h) / (product - dot);
    double denominator = product * plus;
    double rc = radius / length;
    double factor = 1.0;
    if (radius > 0.0 && model != 0) {
        if (model == 5) {
            na = hypot(na, rc);
            nb = hypot(nb, rc);
            product = na * nb;
            double transverse2 = h * h + rc * rc;
            dot = transverse2 + t * (t - 1.0);
            plus = product + dot;
            if (dot < 0.0) plus = transverse2 / (product - dot);
            denominator = product * plus;
        } else if (model == 4) {
            denominator = denominator + rc * rc;
        } else {
            double ratio = h / rc;
            if (!finite(ratio)) return FLAG_NONFINITE;
            if (model == 1) {
                double limited = ratio < 1.0 ? ratio : 1.0;   /* min(ratio, 1.0) */
                factor = limited * limited;
            } else if (model == 2) {
                if (ratio <= lamb_cut()) factor = -expm1(-1.25643 * (ratio * ratio));
            } else if (model == 3) {
                if (ratio < 1.0) {
                    double q = ratio * ratio;
                    factor = q / hypot(1.0, q);
                } else {
                    double inverse = 1.0 / ratio;
                    factor = 1.0 / hypot(1.0, inverse * inverse);
                }
            }
        }
    }
    double coefficient = (gamma / length) / FOUR_PI * factor * (na + nb) / denominator;
    if (!(finite(denominator) && finite(coefficient) && finite(product) && finite(dot))) return FLAG_NONFINITE;
    u[0] = coefficient * cx;
    u[1] = coefficient * cy;
    u[2] = coefficient * cz;
    return FLAG_OK;
}

/* One pair per row (the per-pair check of the CUDA pair functions). */
void orc_pairs(int64_t k, const double *points, const double *starts, const double *directions, const double *lengths,
               const double *gamma, const double *radius, int model, int raise_singular, double *out, int8_t *flags)
{
    for (int64_t i = 0; i < k; ++i) {
        flags[i] = (int8_t)orc_pair(points[3 * i], points[3 * i + 1], points[3 * i + 2], starts[3 * i],
                                    starts[3 * i + 1], starts[3 * i + 2], directions[3 * i], directions[3 * i + 1],
                                    directions[3 * i + 2], lengths[i], gamma[i], model, radius[i], raise_singular,
                                    out + 3 * i);
    }
}

/* vortex_numba._sum_point, vortex_numba.py:112-147: ordered sum over non-excluded segments, first flag wins. */
static void sum_point(int64_t p, const double *points, int64_t m, const double *starts, const double *directions,
                      const double *lengths, const double *gamma, const double *radius, int model, int raise_singular,
                      const int64_t *ex_ptr, const int64_t *ex_seg, double *out, int8_t *flags)
{
    double px = points[3 * p], py = points[3 * p + 1], pz = points[3 * p + 2];
    double ux = 0.0, uy = 0.0, uz = 0.0;
    int flag = FLAG_OK;
    int64_t k = ex_ptr[p], stop = ex_ptr[p + 1];
    for (int64_t s = 0; s < m; ++s) {
        if (k < stop && ex_seg[k] == s) { ++k; continue; }
        double v[3];
        int f = orc_pair(px, py, pz, starts[3 * s], starts[3 * s + 1], starts[3 * s + 2], directions[3 * s],
                         directions[3 * s + 1], directions[3 * s + 2], lengths[s], gamma[s], model, radius[s],
                         raise_singular, v);
        if (f != FLAG_OK) { if (flag == FLAG_OK) flag = f; continue; }
        ux += v[0]; uy += v[1]; uz += v[2];
    }
    if (!(finite(ux) && finite(uy) && finite(uz)) && flag == FLAG_OK) flag = FLAG_NONFINITE;
    out[3 * p] = ux; out[3 * p + 1] = uy; out[3 * p + 2] = uz;
    flags[p] = (int8_t)flag;
}

/* vortex_numba.direct_sum / sum_segments, vortex_numba.py:159-174, 246-260.  threads <= 0: all available. */
void orc_direct_sum(int64_t n, const double *points, int64_t m, const double *starts, const double *directions,
                    const double *lengths, const double *gamma, const double *radius, int model, int raise_singular,
                    const int64_t *ex_ptr, const int64_t *ex_seg, double *out, int8_t *flags, int threads)
{
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
#endif
    for (int64_t p = 0; p < n; ++p)
        sum_point(p, points, m, starts, directions, lengths, gamma, radius, model, raise_singular, ex_ptr, ex_seg,
                  out, flags);
}

/* vortex_numba.pair_matrix, vortex_numba.py:271-287: unit-circulation velocity of every (point, segment) pair. */
void orc_pair_matrix(int64_t n, const double *points, int64_t m, const double *starts, const double *directions,
                     const double *lengths, const double *radius, int model, int raise_singular, double *out,
                     int8_t *flags)
{
    for (int64_t p = 0; p < n; ++p) {
        int flag = FLAG_OK;
        for (int64_t s = 0; s < m; ++s) {
            double v[3];
            int f = orc_pair(points[3 * p], points[3 * p + 1], points[3 * p + 2], starts[3 * s], starts[3 * s + 1],
                             starts[3 * s + 2], directions[3 * s], directions[3 * s + 1], directions[3 * s + 2],
                             lengths[s], 1.0, model, radius[s], raise_singular, v);
            if (f != FLAG_OK && flag == FLAG_OK) flag = f;
            double *o = out + 3 * (p * m + s);
            o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
        }
        flags[p] = (int8_t)flag;
    }
}

/* vortex_numba._exclusion_csr_compiled, vortex_numba.py:193-225 (points already checked to lie in range).
 * Writes ptr[point_count+1] and seg (capacity e); returns the number of unique pairs. */
int64_t orc_exclusion_csr(int64_t point_count, int64_t e, const int64_t *pairs, int64_t *ptr, int64_t *seg)
{
    int64_t *start = (int64_t *)calloc((size_t)point_count + 1, sizeof(int64_t));
    int64_t *cursor = (int64_t *)malloc(sizeof(int64_t) * (size_t)(point_count + 1));
    for (int64_t k = 0; k < e; ++k) start[pairs[2 * k] + 1] += 1;
    for (int64_t p = 0; p < point_count; ++p) start[p + 1] += start[p];
    for (int64_t p = 0; p < point_count; ++p) cursor[p] = start[p];
    for (int64_t k = 0; k < e; ++k) { int64_t p = pairs[2 * k]; seg[cursor[p]++] = pairs[2 * k + 1]; }
    int64_t mcount = 0;
    ptr[0] = 0;
    for (int64_t p = 0; p < point_count; ++p) {
        int64_t a = start[p], b = start[p + 1];
        for (int64_t i = a + 1; i < b; ++i) {
            int64_t value = seg[i], j = i - 1;
            while (j >= a && seg[j] > value) { seg[j + 1] = seg[j]; --j; }
            seg[j + 1] = value;
        }
        for (int64_t i = a; i < b; ++i)
            if (i == a || seg[i] != seg[i - 1]) seg[mcount++] = seg[i];
        ptr[p + 1] = mcount;
    }
    free(start);
    free(cursor);
    return mcount;
}

/* network_numba.incident_pairs / _incident_pairs_sorted (src/openfawe/aero/network_numba.py:176-256): the exclusion
 * pairs (free point i, segment s) of every free node first + i whose coordinates equal an end node of segment s bit
 * for bit (NaN never matches), in segment order, end order, then member order (increasing i).  Nodes are ordered as
 * np.lexsort((bits z, bits y, bits x)) orders them (signed 64-bit patterns, stable), equal patterns form runs, groups
 * are numbered by first appearance among the free points.  Returns the number of pairs; writes them if it fits. */
static const int64_t *orc_bits_base;

static int orc_bits_cmp(const void *pa, const void *pb)
{
    int64_t a = *(const int64_t *)pa, b = *(const int64_t *)pb;
    for (int c = 0; c < 3; ++c) {
        int64_t x = orc_bits_base[3 * a + c], y = orc_bits_base[3 * b + c];
        if (x != y) return x < y ? -1 : 1;
    }
    return a < b ? -1 : (a > b);
}

int64_t orc_incident_pairs(int64_t n, const double *nodes, int64_t segments, const int64_t *edges, int64_t first,
                           int64_t *pairs, int64_t capacity)
{
    int64_t *bits = (int64_t *)malloc(sizeof(int64_t) * (size_t)(3 * n + 1));
    int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t *run_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    unsigned char *no_nan = (unsigned char *)malloc((size_t)n + 1);
    memcpy(bits, nodes, sizeof(double) * (size_t)(3 * n));
    for (int64_t i = 0; i < n; ++i) {
        order[i] = i;
        no_nan[i] = !(isnan(nodes[3 * i]) || isnan(nodes[3 * i + 1]) || isnan(nodes[3 * i + 2]));
    }
    orc_bits_base = bits;
    qsort(order, (size_t)n, sizeof(int64_t), orc_bits_cmp);
    int64_t runs = 0, previous = -1;
    for (int64_t position = 0; position < n; ++position) {
        int64_t node = order[position];
        int same = previous >= 0 && no_nan[node] && no_nan[previous] && bits[3 * node] == bits[3 * previous] &&
                   bits[3 * node + 1] == bits[3 * previous + 1] && bits[3 * node + 2] == bits[3 * previous + 2];
        if (!same) runs += 1;
        run_of[node] = runs - 1;
        previous = node;
    }
    int64_t count = n - first;
    int64_t *group_of_run = (int64_t *)malloc(sizeof(int64_t) * (size_t)(runs + 1));
    int64_t *point_group = (int64_t *)malloc(sizeof(int64_t) * (size_t)(count + 1));
    for (int64_t r = 0; r < runs; ++r) group_of_run[r] = -1;
    int64_t groups = 0;
    for (int64_t index = 0; index < count; ++index) {
        int64_t run = run_of[first + index];
        if (group_of_run[run] < 0) group_of_run[run] = groups++;
        point_group[index] = group_of_run[run];
    }
    int64_t *sizes = (int64_t *)calloc((size_t)groups + 1, sizeof(int64_t));
    int64_t *cursor = (int64_t *)malloc(sizeof(int64_t) * (size_t)(groups + 1));
    int64_t *members = (int64_t *)malloc(sizeof(int64_t) * (size_t)(count + 1));
    for (int64_t index = 0; index < count; ++index) sizes[point_group[index] + 1] += 1;
    for (int64_t g = 0; g < groups; ++g) sizes[g + 1] += sizes[g];
    for (int64_t g = 0; g < groups; ++g) cursor[g] = sizes[g];
    for (int64_t index = 0; index < count; ++index) members[cursor[point_group[index]]++] = index;
    int64_t total = 0;
    for (int64_t segment = 0; segment < segments; ++segment)
        for (int end = 0; end < 2; ++end) {
            int64_t node = edges[2 * segment + end];
            if (!no_nan[node]) continue;
            int64_t g = group_of_run[run_of[node]];
            if (g >= 0) total += sizes[g + 1] - sizes[g];
        }
    if (pairs && total <= capacity) {
        int64_t m = 0;
        for (int64_t segment = 0; segment < segments; ++segment)
            for (int end = 0; end < 2; ++end) {
                int64_t node = edges[2 * segment + end];
                if (!no_nan[node]) continue;
                int64_t g = group_of_run[run_of[node]];
                if (g < 0) continue;
                for (int64_t k = sizes[g]; k < sizes[g + 1]; ++k, ++m) {
                    pairs[2 * m] = members[k];
                    pairs[2 * m + 1] = segment;
                }
            }
    }
    free(bits); free(order); free(run_of); free(no_nan); free(group_of_run); free(point_group); free(sizes);
    free(cursor); free(members);
    return total;
}

/* ---------------------------------------------------------------------------------------------------------------- */
/* Tree code.                                                                                                         */
/* ---------------------------------------------------------------------------------------------------------------- */

/* Stable merge sort of idx[0..n) by keys[idx] (numpy's argsort(kind="mergesort") order). */
static void stable_sort(int64_t *idx, const double *keys, int64_t n, int64_t *tmp)
{
    for (int64_t width = 1; width < n; width *= 2) {
        for (int64_t lo = 0; lo < n; lo += 2 * width) {
            int64_t mid = lo + width < n ? lo + width : n;
            int64_t hi = lo + 2 * width < n ? lo + 2 * width : n;
            int64_t i = lo, j = mid, o = lo;
            while (i < mid && j < hi) {
                if (keys[idx[j]] < keys[idx[i]]) tmp[o++] = idx[j++];
                else tmp[o++] = idx[i++];
            }
            while (i < mid) tmp[o++] = idx[i++];
            while (j < hi) tmp[o++] = idx[j++];
        }
        memcpy(idx, tmp, sizeof(int64_t) * (size_t)n);
    }
}

int64_t orc_tree_capacity(int64_t n, int64_t leaf_size)
{
    return 4 * (n / (leaf_size > 1 ? leaf_size : 1) + 1) + 1;
}

/* vortex_tree.build_tree_serial, vortex_tree.py:51-115 (build_tree returns the same arrays, :208-241).
 * order[n]; lo/hi/left/right of capacity orc_tree_capacity(n, leaf); returns the node count. */
int64_t orc_build_tree(int64_t n, const double *mid, int64_t leaf_size, int64_t *order, int64_t *lo, int64_t *hi,
                       int64_t *left, int64_t *right)
{
    int64_t capacity = orc_tree_capacity(n, leaf_size);
    for (int64_t i = 0; i < n; ++i) order[i] = i;
    for (int64_t i = 0; i < capacity; ++i) { left[i] = -1; right[i] = -1; }
    lo[0] = 0;
    hi[0] = n;
    int64_t count = 1;
    int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)capacity);
    int64_t *indices = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t *perm = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    double *keys = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    stack[0] = 0;
    int64_t top = 1;
    while (top > 0) {
        int64_t node = stack[--top];
        int64_t a = lo[node], b = hi[node];
        if (b - a <= leaf_size) continue;
        double low[3] = {INFINITY, INFINITY, INFINITY}, high[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t k = a; k < b; ++k) {
            int64_t s = order[k];
            for (int axis = 0; axis < 3; ++axis) {
                double v = mid[3 * s + axis];
                if (v < low[axis]) low[axis] = v;
                if (v > high[axis]) high[axis] = v;
            }
        }
        int axis = 0;
        double extent = high[0] - low[0];
        for (int c = 1; c < 3; ++c)
            if (high[c] - low[c] > extent) { extent = high[c] - low[c]; axis = c; }
        if (!(extent > 0.0)) continue;
        int64_t len = b - a;
        for (int64_t k = 0; k < len; ++k) { indices[k] = order[a + k]; keys[k] = mid[3 * indices[k] + axis]; perm[k] = k; }
        stable_sort(perm, keys, len, tmp);
        for (int64_t k = 0; k < len; ++k) order[a + k] = indices[perm[k]];
        int64_t middle = (a + b) / 2;
        int64_t first = count, second = count + 1;
        count += 2;
        lo[first] = a; hi[first] = middle;
        lo[second] = middle; hi[second] = b;
        left[node] = first; right[node] = second;
        stack[top] = second;
        stack[top + 1] = first;
        top += 2;
    }
    free(stack); free(indices); free(perm); free(tmp); free(keys);
    return count;
}

/* vortex_tree.node_moments, vortex_tree.py:320-376.  Arrays (count): centre[3], bound, core, m0[3], m1[9], m2[27]. */
void orc_node_moments(int64_t count, const int64_t *order, const int64_t *lo, const int64_t *hi, const double *starts,
                      const double *ends, const double *alpha, const double *length_vectors, const double *radius,
                      const double *gamma, double *centre, double *bound, double *core, double *m0, double *m1,
                      double *m2, int threads)
{
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int64_t node = 0; node < count; ++node) {
        double low[3] = {INFINITY, INFINITY, INFINITY}, high[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t k = lo[node]; k < hi[node]; ++k) {
            int64_t s = order[k];
            for (int axis = 0; axis < 3; ++axis) {
                double v0 = starts[3 * s + axis], v1 = ends[3 * s + axis];
                if (v0 < low[axis]) low[axis] = v0;
                if (v0 > high[axis]) high[axis] = v0;
                if (v1 < low[axis]) low[axis] = v1;
                if (v1 > high[axis]) high[axis] = v1;
            }
        }
        double c[3];
        for (int axis = 0; axis < 3; ++axis) c[axis] = centre[3 * node + axis] = 0.5 * (low[axis] + high[axis]);
        double r2 = 0.0, largest = 0.0;
        double M0[3] = {0, 0, 0}, M1[9], M2[27];
        memset(M1, 0, sizeof M1);
        memset(M2, 0, sizeof M2);
        for (int64_t k = lo[node]; k < hi[node]; ++k) {
            int64_t s = order[k];
            for (int e = 0; e < 2; ++e) {
                const double *pt = e == 0 ? starts + 3 * s : ends + 3 * s;
                double d0 = pt[0] - c[0], d1 = pt[1] - c[1], d2 = pt[2] - c[2];
                /* (a)**2 + (b)**2 + (c)**2 in numba: left to right, each square a plain multiply */
                double q = (d0 * d0 + d1 * d1) + d2 * d2;
                if (q > r2) r2 = q;
            }
            if (radius[s] > largest) largest = radius[s];
            if (gamma[s] == 0.0) continue;
            double d[3];
            for (int axis = 0; axis < 3; ++axis) d[axis] = 0.5 * (starts[3 * s + axis] + ends[3 * s + axis]) - c[axis];
            for (int i = 0; i < 3; ++i) {
                double ai = alpha[3 * s + i];
                M0[i] += ai;
                for (int j = 0; j < 3; ++j) {
                    M1[3 * i + j] += ai * d[j];
                    for (int l = 0; l < 3; ++l)
                        M2[9 * i + 3 * j + l] += ai * (d[j] * d[l] + length_vectors[3 * s + j] * length_vectors[3 * s + l] / 12.0);
                }
            }
        }
        bound[node] = sqrt(r2) * (1.0 + 1e-12);
        core[node] = largest;
        memcpy(m0 + 3 * node, M0, sizeof M0);
        memcpy(m1 + 9 * node, M1, sizeof M1);
        memcpy(m2 + 27 * node, M2, sizeof M2);
    }
}

/* vortex_tree.node_contractions, vortex_tree.py:425-447. */
void orc_node_contractions(int64_t count, const double *m1, const double *m2, double *w1, double *t2, double *w2)
{
    for (int64_t n = 0; n < count; ++n) {
        const double *a = m1 + 9 * n, *b = m2 + 27 * n;
#define M1(i, j) a[3 * (i) + (j)]
#define M2(i, j, k) b[9 * (i) + 3 * (j) + (k)]
        w1[3 * n + 0] = M1(1, 2) - M1(2, 1);
        w1[3 * n + 1] = M1(2, 0) - M1(0, 2);
        w1[3 * n + 2] = M1(0, 1) - M1(1, 0);
        for (int i = 0; i < 3; ++i) t2[3 * n + i] = M2(i, 0, 0) + M2(i, 1, 1) + M2(i, 2, 2);
        for (int k = 0; k < 3; ++k) {
            w2[9 * n + 0 + k] = M2(1, 2, k) - M2(2, 1, k);
            w2[9 * n + 3 + k] = M2(2, 0, k) - M2(0, 2, k);
            w2[9 * n + 6 + k] = M2(0, 1, k) - M2(1, 0, k);
        }
#undef M1
#undef M2
    }
}

/* vortex_tree.far_velocity, vortex_tree.py:450-497 (contracted form, same operation order). */
void orc_far_velocity(double rx, double ry, double rz, const double *m0, const double *m1, const double *m2,
                      const double *w1, const double *t2, const double *w2, int order, double *u)
{
    double r2 = rx * rx + ry * ry + rz * rz;
    double inv3 = 1.0 / (r2 * sqrt(r2));
    double inv5 = inv3 / r2;
    double a0 = m0[0], a1 = m0[1], a2 = m0[2];
    double u0 = inv3 * (a1 * rz - a2 * ry);
    double u1 = inv3 * (a2 * rx - a0 * rz);
    double u2 = inv3 * (a0 * ry - a1 * rx);
    if (order >= 1) {
        double v0 = m1[0] * rx + m1[1] * ry + m1[2] * rz;
        double v1 = m1[3] * rx + m1[4] * ry + m1[5] * rz;
        double v2 = m1[6] * rx + m1[7] * ry + m1[8] * rz;
        u0 += 3.0 * inv5 * (v1 * rz - v2 * ry) - inv3 * w1[0];
        u1 += 3.0 * inv5 * (v2 * rx - v0 * rz) - inv3 * w1[1];
        u2 += 3.0 * inv5 * (v0 * ry - v1 * rx) - inv3 * w1[2];
    }
    if (order >= 2) {
        double inv7 = inv5 / r2;
        double q0 = 0.0, q1 = 0.0, q2 = 0.0;
        double r[3] = {rx, ry, rz};
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                double rr = r[j] * r[k];
                q0 += m2[0 * 9 + 3 * j + k] * rr;
                q1 += m2[1 * 9 + 3 * j + k] * rr;
                q2 += m2[2 * 9 + 3 * j + k] * rr;
            }
        double b0 = 7.5 * inv7 * q0 - 1.5 * inv5 * t2[0];
        double b1 = 7.5 * inv7 * q1 - 1.5 * inv5 * t2[1];
        double b2 = 7.5 * inv7 * q2 - 1.5 * inv5 * t2[2];
        double s0 = w2[0] * rx + w2[1] * ry + w2[2] * rz;
        double s1 = w2[3] * rx + w2[4] * ry + w2[5] * rz;
        double s2 = w2[6] * rx + w2[7] * ry + w2[8] * rz;
        u0 += (b1 * rz - b2 * ry) - 3.0 * inv5 * s0;
        u1 += (b2 * rx - b0 * rz) - 3.0 * inv5 * s1;
        u2 += (b0 * ry - b1 * rx) - 3.0 * inv5 * s2;
    }
    u[0] = INV_FOUR_PI * u0;
    u[1] = INV_FOUR_PI * u1;
    u[2] = INV_FOUR_PI * u2;
}

/* vortex_tree.tree_velocity, vortex_tree.py:508-568.  Works on any tree given as (order, lo, hi, left, right) plus
 * node quantities, so it also evaluates trees built by the CUDA library.  ex_pos: per-target sorted tree positions of
 * the excluded segments.  Returns 1 when a traversal stack overflowed (the reference does not check; it never does for
 * trees of depth < 255), else 0. */
int orc_tree_velocity(int64_t n, const double *points, const double *starts, const double *directions,
                      const double *lengths, const double *gamma, const double *radius, int model, int raise_singular,
                      const int64_t *order, const int64_t *lo, const int64_t *hi, const int64_t *left,
                      const int64_t *right, const double *centre, const double *bound, const double *core,
                      const double *m0, const double *m1, const double *m2, const double *w1, const double *t2,
                      const double *w2, double theta, int expansion_order, double clearance, const int64_t *ex_ptr,
                      const int64_t *ex_pos, double *out, int8_t *flags, int64_t *far_counts, int threads)
{
    int overflow = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads) reduction(| : overflow)
#endif
    for (int64_t p = 0; p < n; ++p) {
        double x0 = points[3 * p], x1 = points[3 * p + 1], x2 = points[3 * p + 2];
        double acc[3] = {0.0, 0.0, 0.0};
        int flag = FLAG_OK;
        int64_t far = 0;
        int64_t e0 = ex_ptr[p], e1 = ex_ptr[p + 1];
        int64_t stack[TREE_STACK];
        stack[0] = 0;
        int top = 1;
        while (top > 0) {
            int64_t node = stack[--top];
            double rx = x0 - centre[3 * node], ry = x1 - centre[3 * node + 1], rz = x2 - centre[3 * node + 2];
            double distance = sqrt(rx * rx + ry * ry + rz * rz);
            int accept = bound[node] < theta * distance && distance - bound[node] >= clearance * core[node];
            if (accept)
                for (int64_t k = e0; k < e1; ++k)
                    if (ex_pos[k] >= lo[node] && ex_pos[k] < hi[node]) { accept = 0; break; }
            if (accept) {
                double f[3];
                orc_far_velocity(rx, ry, rz, m0 + 3 * node, m1 + 9 * node, m2 + 27 * node, w1 + 3 * node,
                                 t2 + 3 * node, w2 + 9 * node, expansion_order, f);
                acc[0] += f[0]; acc[1] += f[1]; acc[2] += f[2];
                far += 1;
            } else if (left[node] < 0) {
                for (int64_t k = lo[node]; k < hi[node]; ++k) {
                    int skip = 0;
                    for (int64_t e = e0; e < e1; ++e)
                        if (ex_pos[e] == k) { skip = 1; break; }
                    if (skip) continue;
                    int64_t s = order[k];
                    double v[3];
                    int fl = orc_pair(x0, x1, x2, starts[3 * s], starts[3 * s + 1], starts[3 * s + 2],
                                      directions[3 * s], directions[3 * s + 1], directions[3 * s + 2], lengths[s],
                                      gamma[s], model, radius[s], raise_singular, v);
                    if (fl != FLAG_OK) { if (flag == FLAG_OK) flag = fl; continue; }
                    acc[0] += v[0]; acc[1] += v[1]; acc[2] += v[2];
                }
            } else {
                if (top + 2 > TREE_STACK) { overflow = 1; break; }
                stack[top] = right[node];
                stack[top + 1] = left[node];
                top += 2;
            }
        }
        if (!(finite(acc[0]) && finite(acc[1]) && finite(acc[2])) && flag == FLAG_OK) flag = FLAG_NONFINITE;
        out[3 * p] = acc[0]; out[3 * p + 1] = acc[1]; out[3 * p + 2] = acc[2];
        flags[p] = (int8_t)flag;
        far_counts[p] = far;
    }
    return overflow;
}

/* vortex_tree._positions, vortex_tree.py:571-580: excluded segment ids -> sorted tree positions per target. */
void orc_positions(int64_t n, const int64_t *ex_ptr, const int64_t *ex_seg, const int64_t *inverse, int64_t *positions)
{
    for (int64_t p = 0; p < n; ++p) {
        int64_t a = ex_ptr[p], b = ex_ptr[p + 1];
        for (int64_t k = a; k < b; ++k) positions[k] = inverse[ex_seg[k]];
        for (int64_t i = a + 1; i < b; ++i) {
            int64_t v = positions[i], j = i - 1;
            while (j >= a && positions[j] > v) { positions[j + 1] = positions[j]; --j; }
            positions[j + 1] = v;
        }
    }
}

/* Derived segment arrays of vortex_tree.tree_sum, vortex_tree.py:608-611 (numpy's elementwise order). */
void orc_segment_geometry(int64_t m, const double *starts, const double *directions, const double *lengths,
                          const double *gamma, double *length_vectors, double *ends, double *alpha, double *mid)
{
    for (int64_t s = 0; s < m; ++s)
        for (int a = 0; a < 3; ++a) {
            double lv = directions[3 * s + a] * lengths[s];
            length_vectors[3 * s + a] = lv;
            ends[3 * s + a] = starts[3 * s + a] + lv;
            alpha[3 * s + a] = gamma[s] * lv;
            mid[3 * s + a] = 0.5 * (starts[3 * s + a] + ends[3 * s + a]);
        }
}
