// Internal definitions of libbs_b200: device records, the pair and far-field arithmetic, status plumbing.
//
// Pair arithmetic follows the reference's vortex_numba.pair_velocity (src/openfawe/aero/vortex_numba.py:42-109)
// branch for branch: scaled offsets a = (p - s)/L, t = a.d, c = d x a, h = |c|, na = |a|, nb = |a - d|, the roundoff
// axis guard h <= 8 eps max(1, na, nb), the rationalised denominator when h^2 + t(t - 1) < 0, and the six core models.
// Per-segment constants (1/L, Gamma/(4 pi L), rc/L) are formed once when the segment records are packed.
// The far field follows vortex_tree.far_velocity (src/openfawe/aero/vortex_tree.py:450-497).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/bs_b200.h"

#define BS_FLAG_OK 0
#define BS_FLAG_SINGULAR 1
#define BS_FLAG_NONFINITE 2

namespace bs {

// ---------------------------------------------------------------------------------------------------------------------
// Error plumbing (host).
// ---------------------------------------------------------------------------------------------------------------------
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
#define BS_CUDA(call)                                                  \
    do {                                                               \
        cudaError_t _e = (call);                                       \
        if (_e != cudaSuccess) return ::bs::cuda_fail(_e, #call);      \
    } while (0)
#define BS_CHECK_LAUNCH(what)                                          \
    do {                                                               \
        cudaError_t _e = cudaGetLastError();                           \
        if (_e != cudaSuccess) return ::bs::cuda_fail(_e, what);       \
    } while (0)

// Stream-ordered scratch from the context's pool, released (stream-ordered) when the object goes out of scope.  In
// arena mode (a pre-allocated buffer, used while a CUDA graph is captured) requests are carved from the arena and
// nothing is allocated or freed.  `requested` counts the bytes asked for (256-byte granules), so a first, ordinary
// run can size the arena of a later capture.
struct Scratch {
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<void *> ptrs;
    int status = BS_OK;
    char *arena = nullptr;
    size_t arena_size = 0, arena_used = 0, requested = 0;
    Scratch(cudaMemPool_t p, cudaStream_t s) : stream(s), pool(p) {}
    Scratch(void *a, size_t bytes, cudaStream_t s) : stream(s), arena(static_cast<char *>(a)), arena_size(bytes) {}
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
    template <class T> T *get(size_t elems) {
        if (status != BS_OK) return nullptr;
        if (elems == 0) elems = 1;
        const size_t bytes = (elems * sizeof(T) + 255) / 256 * 256;
        requested += bytes;
        if (arena) {
            if (arena_used + bytes > arena_size) {
                status = BS_ERR_OOM;
                set_error("scratch arena of %zu bytes exhausted", arena_size);
                return nullptr;
            }
            void *p = arena + arena_used;
            arena_used += bytes;
            return static_cast<T *>(p);
        }
        void *p = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, stream);
        if (e != cudaSuccess) {
            status = e == cudaErrorMemoryAllocation ? BS_ERR_OOM : BS_ERR_CUDA;
            cuda_fail(e, "scratch allocation");
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    void release() {
        for (void *p : ptrs) cudaFreeAsync(p, stream);
        ptrs.clear();
    }
    ~Scratch() { release(); }
};

}  // namespace bs

struct bs_upload_ring;  // pinned staging of bs_upload (bs_upload.cu)
// bs_upload_many on the context's staging thread: returns at once; bs_stage_wait returns the upload's status once the
// sources have been read (the transfers are queued on s).  One staging at a time per context.
int bs_stage_async(bs_ctx *ctx, int count, void *const *dst, const void *const *src, const size_t *bytes,
                   cudaStream_t s);
int bs_stage_wait(bs_ctx *ctx);

struct bs_ctx {
    int device;
    int sm_count;
    cudaMemPool_t pool;
    bs_stats stats;
    bs_upload_ring *upload = nullptr;
    cudaStream_t copy_stream = nullptr;  // host-array uploads that overlap work on the caller's stream
    cudaStream_t side_stream = nullptr;  // tree sums: the target sort and the far records, beside the caller's stream
    // 64 words of pinned host memory for small read-backs (words 0-7: a build's node count, 8-15: an evaluation's
    // counters), so that those copies are asynchronous: one call at a time per context
    unsigned long long *pinned = nullptr;
};

// The context's pinned words (allocated on first use; null if the allocation failed: callers then copy through
// pageable memory, synchronously).
inline unsigned long long *ctx_pinned(bs_ctx *ctx) {
    if (!ctx->pinned) {
        void *p = nullptr;
        if (cudaHostAlloc(&p, 64 * sizeof(unsigned long long), cudaHostAllocDefault) == cudaSuccess)
            ctx->pinned = static_cast<unsigned long long *>(p);
    }
    return ctx->pinned;
}

// ---------------------------------------------------------------------------------------------------------------------
// Device records.
// ---------------------------------------------------------------------------------------------------------------------
namespace bs {

// One segment, FP64 (96 bytes; 16-byte multiple for bulk copies).
struct __align__(16) Seg64 {
    double sx, sy, sz, len;       // start, L
    double dx, dy, dz, gfac;      // unit direction, (Gamma/L)/(4 pi)
    double rcl, radius, inv_len;  // rc/L, rc (rc > 0 && model != 0 enables the core), 1/L
    double pad;
};

// One segment for the single-precision paths (48 bytes): start as a two-float (hi + lo) pair.
struct __align__(16) Seg32 {
    float4 hi;   // sx_hi, sy_hi, sz_hi, 1/L
    float4 lo;   // sx_lo, sy_lo, sz_lo, (Gamma/L)/(4 pi)
    float4 dir;  // dx, dy, dz, (L/rc)^2
};

// Two consecutive segments (tree order) for the packed-FP32 pair (128 bytes): sixteen fields, each a float2 holding the
// two segments' values, at float offset 2f: 0-2 -s_hi, 3 1/L, 4-6 -s_lo, 7 (Gamma/L)/(4 pi), 8-10 d, 11 (L/rc)^2,
// 12-14 -d, 15 zero.  A segment whose pairs all go to FP64 (a NaN 1/L in its Seg32, or coordinates beyond 1e30) has
// 1/L = 0 and a zero start here, which sends its pairs to FP64 with finite intermediates.
struct __align__(16) Seg32x2 {
    float4 g[8];
};

// Two consecutive segments (tree order) of one leaf for the clear-leaf packed pair (96 bytes), in physical units
// relative to the leaf's centre O, each field a float2 of the two segments' values, at float offset 2f: 0-2 O - s
// (the start, relative and negated), 3 Gamma/(4 pi), 4-6 l = L d, 7 1/(L rc)^2 (+inf without a core), 8-10 -l,
// 11 zero.  Only pairs that lie inside one leaf are read (a pair across two leaves holds halves of different
// centres).
struct __align__(16) Seg32c2 {
    float4 g[6];
};

// Traversal record of one node (64 bytes).
struct __align__(16) NodeRec {
    double cx, cy, cz, bound;
    double clear_core;  // clearance * largest core radius
    int lo, hi, left, right;
    double pad;
};

// Far-field coefficients: m0[3], m1[9] (row i, column j), w1[3], t2[3], w2[9], m2 symmetric [3][6] (00,01,02,11,12,22).
#define BS_FAR_N 45
struct __align__(16) Far64 { double v[BS_FAR_N + 1]; };
struct __align__(16) Far32 { float v[BS_FAR_N + 3]; };

enum { F_M0 = 0, F_M1 = 3, F_W1 = 12, F_T2 = 15, F_W2 = 18, F_M2 = 27 };

// Third-order far-field coefficients (an extension of the reference's orders 0-2): m3 symmetric in its last three
// indices [3][10] (000,001,002,011,012,022,111,112,122,222), its trace T3[b][l] = m3[b][j][j][l] [3][3],
// W3[a][k][l] = eps_abc m3[b][c][k][l] symmetric [3][6], w3[a] = eps_abc T3[b][c] [3].
#define BS_FAR3_N 60
struct __align__(16) Far64x { double v[64]; };
struct __align__(16) Far32x { float v[64]; };
enum { G_M3 = 0, G_T3 = 30, G_W3 = 39, G_W3V = 57 };
// Far32x keeps each component i's coefficients together in five float4: [20 i, 20 i + 10) m3 row, [+10, +13) T3 row,
// [+13, +19) W3 row, then w3 at [60, 63).
enum { H_ROW = 20, H_M3 = 0, H_T3 = 10, H_W3 = 13, H_W3V = 60 };

// Fourth-order far-field coefficients (trees built for order 4), one row of 36 per component i (nine float4), in both
// precisions: [0, 15) m4[i] symmetric (0000,0001,0002,0011,0012,0022,0111,0112,0122,0222,1111,1112,1122,1222,2222),
// [15, 21) T4[i][l][m] = m4[i][j][j][l][m] symmetric, [21] tau4[i] = T4[i][l][l], [22, 32) W4[i][k][l][m] =
// eps_ibc m4[b][c][k][l][m] symmetric, [32, 35) W4T[i][m] = eps_ibc T4[b][c][m], [35] zero.
enum { K_ROW = 36, K_M4 = 0, K_T4 = 15, K_TAU4 = 21, K_W4 = 22, K_W4T = 32 };
struct __align__(16) Far64y { double v[112]; };
struct __align__(16) Far32y { float v[112]; };

// Fifth-order far-field coefficients (trees built for order 5), one row of 56 per component i (fourteen float4), in
// both precisions: [0, 21) m5[i] symmetric in its five indices (lexicographic a <= b <= c <= d <= e), [21, 31)
// T5[i][k][l][m] = m5[i][j][j][k][l][m] symmetric, [31, 34) TT5[i][m] = T5[i][j][j][m], [34, 49) W5[i][k][l][m][n] =
// eps_ibc m5[b][c][k][l][m][n] symmetric, [49, 55) W5T[i][l][m] = eps_ibc T5[b][c][l][m] symmetric, [55] W5TT[i] =
// eps_ibc TT5[b][c].
enum { Z_ROW = 56, Z_M5 = 0, Z_T5 = 21, Z_TT5 = 31, Z_W5 = 34, Z_W5T = 49, Z_W5TT = 55 };
struct __align__(16) Far64z { double v[3 * Z_ROW]; };
struct __align__(16) Far32z { float v[3 * Z_ROW]; };

// ---------------------------------------------------------------------------------------------------------------------
// Arithmetic helpers.
// ---------------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double norm3d(double x, double y, double z) {
    double q = fma(x, x, fma(y, y, z * z));
    // Outside [1e-290, 1e290] squares lose range: fall back to the scaled form the reference uses.
    if (q > 1e-290 && q < 1e290) return sqrt(q);
    return hypot(hypot(x, y), z);
}

static constexpr double AXIS_EPS64 = 8.0 * 2.220446049250313e-16;
static constexpr float AXIS_EPS32 = 8.0f * 1.1920929e-07f;
static constexpr double LAMB_A = 1.25643;
static constexpr double LAMB_CUT = 2.821180356260211;   // sqrt(10 / 1.25643), OLAF's exponent cut-off
static constexpr double LAMB_CUT2 = 7.959058602548491;  // 10 / 1.25643
static constexpr double INV_FOUR_PI = 0.07957747154594767;  // 1 / (4 pi)
// Without a core (MODEL 0) the single-precision pairs take FP64 within a quarter of the segment's length of the finite
// segment: their offsets a = (x - s)/L carry ~1 ulp of |a|, and b = a - d inherits that absolute error, so near an
// end point (or near the axis) the pair's relative error grows as eps / distance; beyond L/4 it stays below ~5 eps.
static constexpr float NOCORE_NEAR2 = 0.0625f;  // (1/4)^2, units of L^2

// The reference pair (vortex_numba.pair_velocity) on an FP64 record from the scaled offset a = (p - s)/L, t = a.d and
// c = d x a.  Returns the flag; adds the velocity to (ux, uy, uz) only when the flag is ok.
__device__ __forceinline__ int pair64_core(double ax, double ay, double az, double t, double cx, double cy, double cz,
                                           const Seg64 &s, int model, int raise_singular, double &ux, double &uy,
                                           double &uz) {
    const double dx = s.dx, dy = s.dy, dz = s.dz;
    double h = norm3d(cx, cy, cz);
    double na = norm3d(ax, ay, az);
    double nb = norm3d(ax - dx, ay - dy, az - dz);
    if (!(isfinite(h) && isfinite(na) && isfinite(nb) && isfinite(t))) return BS_FLAG_NONFINITE;
    double scale = fmax(1.0, fmax(na, nb));
    if (h <= AXIS_EPS64 * scale) {
        if (raise_singular && t >= 0.0 && t <= 1.0) return BS_FLAG_SINGULAR;
        return BS_FLAG_OK;
    }
    if (s.gfac == 0.0) return BS_FLAG_OK;
    double h2 = h * h;
    double product = na * nb;
    double dot = fma(t, t - 1.0, h2);
    double plus = dot < 0.0 ? h2 / (product - dot) : product + dot;
    double denominator = product * plus;
    double factor = 1.0;
    if (s.radius > 0.0 && model != 0) {
        const double rc = s.rcl;
        if (model == 5) {  // Rosenhead-Moore
            na = hypot(na, rc);
            nb = hypot(nb, rc);
            product = na * nb;
            double tr2 = fma(rc, rc, h2);
            dot = fma(t, t - 1.0, tr2);
            plus = dot < 0.0 ? tr2 / (product - dot) : product + dot;
            denominator = product * plus;
        } else if (model == 4) {  // offset
            denominator = fma(rc, rc, denominator);
        } else {
            double ratio = h / rc;
            if (!isfinite(ratio)) return BS_FLAG_NONFINITE;
            if (model == 1) {
                double l = fmin(ratio, 1.0);
                factor = l * l;
            } else if (model == 2) {
                double r2 = ratio * ratio;
                if (ratio <= LAMB_CUT) factor = -expm1(-LAMB_A * r2);
            } else if (model == 3) {
                if (ratio < 1.0) {
                    double q = ratio * ratio;
                    factor = q / hypot(1.0, q);
                } else {
                    double inv = 1.0 / ratio;
                    factor = 1.0 / hypot(1.0, inv * inv);
                }
            }
        }
    }
    double coefficient = s.gfac * factor * (na + nb) / denominator;
    if (!(isfinite(denominator) && isfinite(coefficient) && isfinite(product) && isfinite(dot)))
        return BS_FLAG_NONFINITE;
    ux = fma(coefficient, cx, ux);
    uy = fma(coefficient, cy, uy);
    uz = fma(coefficient, cz, uz);
    return BS_FLAG_OK;
}

// The FP64 pair from an FP64 target position.  Fast form: a = (p - s) * (1/L) and fused t, c.  Where the target lies
// within 1% (in angle) of the segment's line, c = d x a cancels and its rounding decides the result, so a, t and c are
// formed again exactly as the reference forms them (IEEE division, separately rounded products and sums); the two
// forms then agree to a few units in the last place of c.
__device__ __forceinline__ int pair64_at(double px, double py, double pz, const Seg64 &s, int model,
                                         int raise_singular, double &ux, double &uy, double &uz) {
    const double dx = s.dx, dy = s.dy, dz = s.dz;
    const double rx = px - s.sx, ry = py - s.sy, rz = pz - s.sz;
    double ax = rx * s.inv_len, ay = ry * s.inv_len, az = rz * s.inv_len;
    double t = fma(az, dz, fma(ay, dy, ax * dx));
    double cx = fma(dy, az, -dz * ay);
    double cy = fma(dz, ax, -dx * az);
    double cz = fma(dx, ay, -dy * ax);
    const double h2 = fma(cx, cx, fma(cy, cy, cz * cz));
    const double a2 = fma(ax, ax, fma(ay, ay, az * az));
    if (!(h2 >= 1e-4 * a2)) {
        const double L = s.len;
        ax = __ddiv_rn(rx, L);
        ay = __ddiv_rn(ry, L);
        az = __ddiv_rn(rz, L);
        t = __dadd_rn(__dadd_rn(__dmul_rn(ax, dx), __dmul_rn(ay, dy)), __dmul_rn(az, dz));
        cx = __dsub_rn(__dmul_rn(dy, az), __dmul_rn(dz, ay));
        cy = __dsub_rn(__dmul_rn(dz, ax), __dmul_rn(dx, az));
        cz = __dsub_rn(__dmul_rn(dx, ay), __dmul_rn(dy, ax));
    }
    return pair64_core(ax, ay, az, t, cx, cy, cz, s, model, raise_singular, ux, uy, uz);
}

// The single-precision pair, in units of the segment's length: a = (p - s)/L (from two-float coordinates), b = a - d,
// c = d x a, h^2 = |c|^2, and the reference's (vortex_numba.pair_velocity)
//   u = (Gamma/L)/(4 pi) factor (|a| + |b|) / (|a| |b| (|a| |b| + a.b)) c.
// hi.w holds 1/L (NaN for a core too small for FP32), lo.w (Gamma/L)/(4 pi), dir.w (L/rc)^2, 0 for no core.  Adds
// the velocity to (ux, uy, uz) unless the pair needs FP64, which is returned as true: within sqrt(near2) core radii of
// the finite segment (MODEL 0: within L/4 of it, NOCORE_NEAR2), within 1e-4 L of its axis (the reference's "suspect"
// rule, vortex_cuda.py:123-124; a NaN 1/L fails it too), or out of FP32's comfortable range -- the FP64 pair then
// decides value and flags exactly.  Where a.b < 0, |a||b| + a.b = h^2 / (|a||b| - a.b) (|a x b| = |c|): no
// cancellation.  The common path has no data-dependent branch; the core factor is computed only where it differs
// from 1 (Lamb-Oseen inside its cut-off, Rankine and Vatistas inside one core radius).  MODEL: 0..5.  NEAR = false
// leaves out the "within sqrt(near2) core radii" (MODEL 0: "within L/4") test, for callers that know every pair of the
// batch lies farther than that from its segment.
template <int MODEL, bool NEAR = true>
__device__ __forceinline__ bool pair32(float rx, float ry, float rz, const float4 &hi, const float4 &lo,
                                       const float4 &dir, float near2, float &ux, float &uy, float &uz) {
    const float il = hi.w;
    const float ax = rx * il, ay = ry * il, az = rz * il;
    const float dx = dir.x, dy = dir.y, dz = dir.z, irc2 = dir.w;
    const float bx = ax - dx, by = ay - dy, bz = az - dz;
    const float cx = fmaf(dy, az, -dz * ay);
    const float cy = fmaf(dz, ax, -dx * az);
    const float cz = fmaf(dx, ay, -dy * ax);
    const float h2 = fmaf(cx, cx, fmaf(cy, cy, cz * cz));
    const float na2 = fmaf(ax, ax, fmaf(ay, ay, az * az));
    const float nb2 = fmaf(bx, bx, fmaf(by, by, bz * bz));
    const float dot = fmaf(ax, bx, fmaf(ay, by, az * bz));
    const float big2 = fmaxf(1.0f, fmaxf(na2, nb2));
    bool need64 = !(h2 > 1e-8f * big2) || !(big2 < 1e18f);
    if (NEAR) {
        const float t = fmaf(az, dz, fmaf(ay, dy, ax * dx));
        const float seg2 = t < 0.0f ? na2 : (t > 1.0f ? nb2 : h2);  // distance^2 to the finite segment, units of L^2
        need64 = need64 || (MODEL == 0 ? seg2 < NOCORE_NEAR2 : (irc2 > 0.0f && seg2 * irc2 < near2));
    }
    const float na = na2 * rsqrtf(na2), nb = nb2 * rsqrtf(nb2);
    const float product = na * nb;
    // coefficient = lo.w * factor * num / den: num = |a| + |b| and den = product * (product + dot), or where dot < 0
    // num = (|a| + |b|)(product - dot) and den = product * h^2; one reciprocal either way
    float num = na + nb;
    num = dot < 0.0f ? num * (product - dot) : num;
    float den = product * (dot < 0.0f ? h2 : product + dot);
    float factor = 1.0f;
    if (MODEL == 5 || MODEL == 4) {
        if (irc2 > 0.0f) {
            const float rc2 = __fdividef(1.0f, irc2);
            if (MODEL == 5) {  // Rosenhead-Moore: augmented distances
                const float pa = sqrtf(na2 + rc2), pb = sqrtf(nb2 + rc2);
                const float pr = pa * pb, tr2 = h2 + rc2, dt = dot + rc2;
                num = dt < 0.0f ? (pa + pb) * (pr - dt) : pa + pb;
                den = pr * (dt < 0.0f ? tr2 : pr + dt);
            } else {  // offset core: denominator + rc^2
                const float plus = dot < 0.0f ? __fdividef(h2, product - dot) : product + dot;
                num = na + nb;
                den = fmaf(product, plus, rc2);
            }
        }
    } else if (MODEL != 0) {
        const float r2 = h2 * irc2;  // (h / rc)^2, 0 when there is no core
        if (irc2 > 0.0f && r2 < (MODEL == 2 ? (float)LAMB_CUT2 : 1e30f)) {
            if (MODEL == 1) {
                factor = fminf(r2, 1.0f);
            } else if (MODEL == 2) {
                // 1 - exp(-x), x = 1.25643 r^2; where x is small the difference loses relative digits, but the pair
                // is then as small as x, so its absolute error stays at FP32 rounding of the pair without the core
                factor = 1.0f - __expf(-(float)LAMB_A * r2);
            } else {  // Vatistas n = 2
                factor = r2 < 1.0f ? r2 * rsqrtf(fmaf(r2, r2, 1.0f))
                                   : rsqrtf(fmaf(__fdividef(1.0f, r2), __fdividef(1.0f, r2), 1.0f));
            }
        }
    }
    const float coefficient = lo.w * factor * num * __fdividef(1.0f, den);
    if (!need64) {
        ux = fmaf(coefficient, cx, ux);
        uy = fmaf(coefficient, cy, uy);
        uz = fmaf(coefficient, cz, uz);
    }
    return need64;
}

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// pair32 for two segments at once in packed FP32 (one f32x2 add, multiply or FMA per operation for both segments;
// tests, selects and the special-function unit per component): the same arithmetic as pair32 for MODEL 0 (no core),
// 1 (Rankine) and 2 (Lamb-Oseen).  The target is (t_hi + t_lo) per axis, broadcast in both halves; `rec` is the pair's
// Seg32x2.  Accumulates into the float2 sums (one half per segment) the pairs that do not need FP64 and returns those
// that do: bit 0 for the first segment, bit 1 for the second.  The caller's target must have finite coordinates
// below 1e30 (an out-of-range pair's finite intermediates are multiplied by a zero coefficient).
template <int MODEL, bool NEAR>
__device__ __forceinline__ unsigned pair32x2(float2 txh, float2 tyh, float2 tzh, float2 txl, float2 tyl, float2 tzl,
                                             const float4 *rec, float near2, float2 &u0, float2 &u1, float2 &u2) {
    static_assert(MODEL >= 0 && MODEL <= 2, "packed pairs for the models without a per-pair special form");
    const float4 g0 = rec[0], g1 = rec[1], g2 = rec[2], g3 = rec[3], g4 = rec[4], g5 = rec[5], g6 = rec[6],
                 g7 = rec[7];
    const float2 il = make_float2(g1.z, g1.w), gf = make_float2(g3.z, g3.w);
    const float2 dx = make_float2(g4.x, g4.y), dy = make_float2(g4.z, g4.w), dz = make_float2(g5.x, g5.y);
    const float2 w = make_float2(g5.z, g5.w);
    const float2 ndx = make_float2(g6.x, g6.y), ndy = make_float2(g6.z, g6.w), ndz = make_float2(g7.x, g7.y);
    // q = (t_hi - s_hi) + (t_lo - s_lo), a = q / L, b = a - d, c = d x a
    const float2 ax = mul2(add2(add2(txh, make_float2(g0.x, g0.y)), add2(txl, make_float2(g2.x, g2.y))), il);
    const float2 ay = mul2(add2(add2(tyh, make_float2(g0.z, g0.w)), add2(tyl, make_float2(g2.z, g2.w))), il);
    const float2 az = mul2(add2(add2(tzh, make_float2(g1.x, g1.y)), add2(tzl, make_float2(g3.x, g3.y))), il);
    const float2 bx = add2(ax, ndx), by = add2(ay, ndy), bz = add2(az, ndz);
    const float2 cx = fma2(dy, az, mul2(ndz, ay));
    const float2 cy = fma2(dz, ax, mul2(ndx, az));
    const float2 cz = fma2(dx, ay, mul2(ndy, ax));
    const float2 h2 = fma2(cx, cx, fma2(cy, cy, mul2(cz, cz)));
    const float2 na2 = fma2(ax, ax, fma2(ay, ay, mul2(az, az)));
    const float2 nb2 = fma2(bx, bx, fma2(by, by, mul2(bz, bz)));
    const float2 dot = fma2(ax, bx, fma2(ay, by, mul2(az, bz)));
    const float big0 = fmaxf(1.0f, fmaxf(na2.x, nb2.x)), big1 = fmaxf(1.0f, fmaxf(na2.y, nb2.y));
    const float2 lim = mul2(make_float2(big0, big1), make_float2(1e-8f, 1e-8f));
    bool n0 = !(h2.x > lim.x) || !(big0 < 1e18f);
    bool n1 = !(h2.y > lim.y) || !(big1 < 1e18f);
    if (NEAR) {
        const float2 t = fma2(az, dz, fma2(ay, dy, mul2(ax, dx)));
        const float2 seg2 = make_float2(t.x < 0.0f ? na2.x : (t.x > 1.0f ? nb2.x : h2.x),
                                        t.y < 0.0f ? na2.y : (t.y > 1.0f ? nb2.y : h2.y));
        if (MODEL == 0) {
            n0 = n0 || seg2.x < NOCORE_NEAR2;
            n1 = n1 || seg2.y < NOCORE_NEAR2;
        } else {
            const float2 rr = mul2(seg2, w);
            n0 = n0 || (w.x > 0.0f && rr.x < near2);
            n1 = n1 || (w.y > 0.0f && rr.y < near2);
        }
    }
    const float2 na = mul2(na2, make_float2(rsqrtf(na2.x), rsqrtf(na2.y)));
    const float2 nb = mul2(nb2, make_float2(rsqrtf(nb2.x), rsqrtf(nb2.y)));
    const float2 product = mul2(na, nb);
    const float2 sum = add2(na, nb);
    // as in pair32: where a.b < 0, |a||b| + a.b = h^2 / (|a||b| - a.b)
    const float2 numr = mul2(sum, fma2(dot, make_float2(-1.0f, -1.0f), product));
    const float2 plus = add2(product, dot);
    const float2 num = make_float2(dot.x < 0.0f ? numr.x : sum.x, dot.y < 0.0f ? numr.y : sum.y);
    const float2 den = mul2(product, make_float2(dot.x < 0.0f ? h2.x : plus.x, dot.y < 0.0f ? h2.y : plus.y));
    float2 factor = make_float2(1.0f, 1.0f);
    if (MODEL == 1) {
        const float2 r2 = mul2(h2, w);
        factor = make_float2(w.x > 0.0f ? fminf(r2.x, 1.0f) : 1.0f, w.y > 0.0f ? fminf(r2.y, 1.0f) : 1.0f);
    } else if (MODEL == 2) {
        const float2 r2 = mul2(h2, w);
        const float2 x = mul2(r2, make_float2(-(float)LAMB_A, -(float)LAMB_A));
        const float2 f = fma2(make_float2(__expf(x.x), __expf(x.y)), make_float2(-1.0f, -1.0f), make_float2(1.0f, 1.0f));
        factor = make_float2(w.x > 0.0f && r2.x < (float)LAMB_CUT2 ? f.x : 1.0f,
                             w.y > 0.0f && r2.y < (float)LAMB_CUT2 ? f.y : 1.0f);
    }
    float2 coefficient = mul2(mul2(gf, factor),
                              mul2(num, make_float2(__fdividef(1.0f, den.x), __fdividef(1.0f, den.y))));
    coefficient.x = n0 ? 0.0f : coefficient.x;
    coefficient.y = n1 ? 0.0f : coefficient.y;
    u0 = fma2(coefficient, cx, u0);
    u1 = fma2(coefficient, cy, u1);
    u2 = fma2(coefficient, cz, u2);
    return (n0 ? 1u : 0u) | (n1 ? 2u : 0u);
}

// 2^x from the special-function unit (ex2.approx, flushing subnormal results to zero); e^-y = 2^(-y log2 e).
__device__ __forceinline__ float exp2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// -LAMB_A log2(e): the Lamb-Oseen exponent for exp2_approx.
static constexpr float LAMB_A_LOG2E_NEG = (float)(-LAMB_A * 1.4426950408889634);

// The pair of two segments of a leaf (a Seg32c2 record) for a target `clear` of the leaf: at least 1.5 times its
// bounding radius from its centre (every segment is then seen under less than 84 degrees, so r1.r2 >= 0.1 |r1||r2|
// and |r1||r2| + r1.r2 has no cancellation), outside the reach of the core test (no pair needs FP64 for its core) and
// within the FP32 range the caller checks (1e-8 < |x - O| < 1e9, bound < 1e9, so that |r1|^4 stays a normal float).
// (tx, ty, tz) is x - O in FP32, broadcast in both halves.  In physical units, r1 = x - s, r2 = r1 - l and
// c = l x r1 (= r1 x r2):
//   u = Gamma/(4 pi) factor (|r1| + |r2|) / (|r1| |r2| (|r1| |r2| + r1.r2)) c,
// the reference's pair (vortex_numba.pair_velocity) with numerator and denominator multiplied by L^3, the core
// factor from (h / rc)^2 = |c|^2 / (L rc)^2.  No pair of a clear target needs FP64: none lies on its segment, and
// the leaf-relative FP32 offsets carry at most about 3 ulp of |r1|, as the two-float path's rounded difference does.
// MODEL 0..2.  Adds the two segments' velocities to the float2 sums (one half each).
template <int MODEL>
__device__ __forceinline__ void pair32x2_clear(float2 tx, float2 ty, float2 tz, const float4 *rec, float2 &u0,
                                               float2 &u1, float2 &u2) {
    static_assert(MODEL >= 0 && MODEL <= 2, "clear packed pairs for the models without a per-pair special form");
    const float4 g0 = rec[0], g1 = rec[1], g2 = rec[2], g3 = rec[3], g4 = rec[4], g5 = rec[5];
    const float2 r1x = add2(tx, make_float2(g0.x, g0.y)), r1y = add2(ty, make_float2(g0.z, g0.w));
    const float2 r1z = add2(tz, make_float2(g1.x, g1.y)), gf = make_float2(g1.z, g1.w);
    const float2 lx = make_float2(g2.x, g2.y), ly = make_float2(g2.z, g2.w), lz = make_float2(g3.x, g3.y);
    const float2 w = make_float2(g3.z, g3.w);
    const float2 nlx = make_float2(g4.x, g4.y), nly = make_float2(g4.z, g4.w), nlz = make_float2(g5.x, g5.y);
    const float2 r2x = add2(r1x, nlx), r2y = add2(r1y, nly), r2z = add2(r1z, nlz);
    const float2 cx = fma2(ly, r1z, mul2(nlz, r1y));
    const float2 cy = fma2(lz, r1x, mul2(nlx, r1z));
    const float2 cz = fma2(lx, r1y, mul2(nly, r1x));
    const float2 h2 = fma2(cx, cx, fma2(cy, cy, mul2(cz, cz)));
    const float2 n12 = fma2(r1x, r1x, fma2(r1y, r1y, mul2(r1z, r1z)));
    const float2 n22 = fma2(r2x, r2x, fma2(r2y, r2y, mul2(r2z, r2z)));
    const float2 dot = fma2(r1x, r2x, fma2(r1y, r2y, mul2(r1z, r2z)));
    const float2 n1 = mul2(n12, make_float2(rsqrtf(n12.x), rsqrtf(n12.y)));
    const float2 n2 = mul2(n22, make_float2(rsqrtf(n22.x), rsqrtf(n22.y)));
    const float2 product = mul2(n1, n2);
    const float2 den = mul2(product, add2(product, dot));
    float2 k = mul2(gf, add2(n1, n2));
    if (MODEL == 1) {  // Rankine: min((h / rc)^2, 1); +inf (no core) and NaN (h = 0 without a core) give 1
        const float2 r2 = mul2(h2, w);
        k = mul2(k, make_float2(fminf(r2.x, 1.0f), fminf(r2.y, 1.0f)));
    } else if (MODEL == 2) {  // Lamb-Oseen inside its cut-off: 1 - exp(-1.25643 (h / rc)^2)
        // a clear target is seldom within the cut-off of a segment's line: the exponent is formed only when some
        // lane of those evaluating the pair needs it (a vote over the active lanes; each lane's own test is in it)
        const float2 r2 = mul2(h2, w);
        if (__any_sync(__activemask(), r2.x < (float)LAMB_CUT2 || r2.y < (float)LAMB_CUT2)) {
            const float2 x = mul2(r2, make_float2(LAMB_A_LOG2E_NEG, LAMB_A_LOG2E_NEG));
            const float2 f = fma2(make_float2(exp2_approx(x.x), exp2_approx(x.y)), make_float2(-1.0f, -1.0f),
                                  make_float2(1.0f, 1.0f));
            k = mul2(k, make_float2(r2.x < (float)LAMB_CUT2 ? f.x : 1.0f, r2.y < (float)LAMB_CUT2 ? f.y : 1.0f));
        }
    }
    const float2 coefficient = mul2(k, make_float2(__fdividef(1.0f, den.x), __fdividef(1.0f, den.y)));
    u0 = fma2(coefficient, cx, u0);
    u1 = fma2(coefficient, cy, u1);
    u2 = fma2(coefficient, cz, u2);
}

// The fourth-order term of the expansion, R = x - c:
//   (39.375 S4 / r^11 - 26.25 T4:RR / r^9 + 1.875 tau4 / r^7) x R - 17.5 W4:RRR / r^9 + 7.5 W4T R / r^7,
// S4_i = m4[i] : RRRR.  It is linear in the component rows, so row i (K_ROW values) adds its own share:
// x4_i (e_i x R) + w_i e_i.
template <class T>
__device__ __forceinline__ void far_term4_row(T rx, T ry, T rz, T inv7, T inv9, T inv11, const T *r, int i, T &u0,
                                              T &u1, T &u2) {
    const T xx = rx * rx, xy = rx * ry, xz = rx * rz, yy = ry * ry, yz = ry * rz, zz = rz * rz;
    // monomials of the symmetric components times their multiplicities
    const T q4[15] = {xx * xx, T(4) * xx * xy, T(4) * xx * xz, T(6) * xx * yy, T(12) * xx * yz, T(6) * xx * zz,
                      T(4) * xy * yy, T(12) * xy * yz, T(12) * xy * zz, T(4) * xz * zz, yy * yy, T(4) * yy * yz,
                      T(6) * yy * zz, T(4) * yz * zz, zz * zz};
    const T q3[10] = {xx * rx, T(3) * xx * ry, T(3) * xx * rz, T(3) * xy * ry, T(6) * xy * rz, T(3) * xz * rz,
                      yy * ry, T(3) * yy * rz, T(3) * yz * rz, zz * rz};
    const T q2[6] = {xx, T(2) * xy, T(2) * xz, yy, T(2) * yz, zz};
    T s4 = 0, t4 = 0, w4 = 0;
#pragma unroll
    for (int q = 0; q < 15; ++q) s4 += r[K_M4 + q] * q4[q];
#pragma unroll
    for (int q = 0; q < 6; ++q) t4 += r[K_T4 + q] * q2[q];
#pragma unroll
    for (int q = 0; q < 10; ++q) w4 += r[K_W4 + q] * q3[q];
    const T x4 = T(39.375) * inv11 * s4 - T(26.25) * inv9 * t4 + T(1.875) * inv7 * r[K_TAU4];
    const T w = T(7.5) * inv7 * (r[K_W4T] * rx + r[K_W4T + 1] * ry + r[K_W4T + 2] * rz) - T(17.5) * inv9 * w4;
    if (i == 0) { u0 += w; u1 -= x4 * rz; u2 += x4 * ry; }
    else if (i == 1) { u0 += x4 * rz; u1 += w; u2 -= x4 * rx; }
    else { u0 -= x4 * ry; u1 += x4 * rx; u2 += w; }
}

template <class T>
__device__ __forceinline__ void far_term4(T rx, T ry, T rz, T inv7, T inv9, T inv11, const T *h, T &u0, T &u1,
                                          T &u2) {
#pragma unroll
    for (int i = 0; i < 3; ++i) far_term4_row<T>(rx, ry, rz, inv7, inv9, inv11, h + K_ROW * i, i, u0, u1, u2);
}

// The fifth-order term, R = x - c (the general order-p term of the same series at p = 5):
//   (86.625 S5 / r^13 - 78.75 T5:RRR / r^11 + 13.125 TT5.R / r^9) x R
//     - 39.375 W5:RRRR / r^11 + 26.25 W5T:RR / r^9 - 1.875 W5TT / r^7,
// S5_i = m5[i] : RRRRR; row i (Z_ROW values) adds x5_i (e_i x R) + w_i e_i.
template <class T>
__device__ __forceinline__ void far_term5_row(T rx, T ry, T rz, T inv7, T inv9, T inv11, T inv13, const T *r, int i,
                                              T &u0, T &u1, T &u2) {
    const T xx = rx * rx, xy = rx * ry, xz = rx * rz, yy = ry * ry, yz = ry * rz, zz = rz * rz;
    // monomials of the symmetric components (lexicographic index tuples) times their multiplicities
    const T q2[6] = {xx, T(2) * xy, T(2) * xz, yy, T(2) * yz, zz};
    const T c3[10] = {xx * rx, xx * ry, xx * rz, xy * ry, xy * rz, xz * rz, yy * ry, yy * rz, yz * rz, zz * rz};
    const T q3[10] = {c3[0], T(3) * c3[1], T(3) * c3[2], T(3) * c3[3], T(6) * c3[4], T(3) * c3[5], c3[6],
                      T(3) * c3[7], T(3) * c3[8], c3[9]};
    const T q4[15] = {xx * xx, T(4) * xx * xy, T(4) * xx * xz, T(6) * xx * yy, T(12) * xx * yz, T(6) * xx * zz,
                      T(4) * xy * yy, T(12) * xy * yz, T(12) * xy * zz, T(4) * xz * zz, yy * yy, T(4) * yy * yz,
                      T(6) * yy * zz, T(4) * yz * zz, zz * zz};
    // degree 5: (c0, c1, c2) = (5,0,0), (4,1,0), (4,0,1), (3,2,0), (3,1,1), (3,0,2), (2,3,0), (2,2,1), (2,1,2),
    // (2,0,3), (1,4,0), (1,3,1), (1,2,2), (1,1,3), (1,0,4), (0,5,0), (0,4,1), (0,3,2), (0,2,3), (0,1,4), (0,0,5)
    const T q5[21] = {xx * c3[0],          T(5) * xx * c3[1],   T(5) * xx * c3[2],   T(10) * xx * c3[3],
                      T(20) * xx * c3[4],  T(10) * xx * c3[5],  T(10) * xx * c3[6],  T(30) * xx * c3[7],
                      T(30) * xx * c3[8],  T(10) * xx * c3[9],  T(5) * xy * c3[6],   T(20) * xy * c3[7],
                      T(30) * xy * c3[8],  T(20) * xy * c3[9],  T(5) * xz * c3[9],   yy * c3[6],
                      T(5) * yy * c3[7],   T(10) * yy * c3[8],  T(10) * yy * c3[9],  T(5) * yz * c3[9],
                      zz * c3[9]};
    T s5 = 0, t5 = 0, w5 = 0, w5t = 0;
#pragma unroll
    for (int q = 0; q < 21; ++q) s5 += r[Z_M5 + q] * q5[q];
#pragma unroll
    for (int q = 0; q < 10; ++q) t5 += r[Z_T5 + q] * q3[q];
#pragma unroll
    for (int q = 0; q < 15; ++q) w5 += r[Z_W5 + q] * q4[q];
#pragma unroll
    for (int q = 0; q < 6; ++q) w5t += r[Z_W5T + q] * q2[q];
    const T tt5 = r[Z_TT5] * rx + r[Z_TT5 + 1] * ry + r[Z_TT5 + 2] * rz;
    const T x5 = T(86.625) * inv13 * s5 - T(78.75) * inv11 * t5 + T(13.125) * inv9 * tt5;
    const T w = T(26.25) * inv9 * w5t - T(39.375) * inv11 * w5 - T(1.875) * inv7 * r[Z_W5TT];
    if (i == 0) { u0 += w; u1 -= x5 * rz; u2 += x5 * ry; }
    else if (i == 1) { u0 += x5 * rz; u1 += w; u2 -= x5 * rx; }
    else { u0 -= x5 * ry; u1 += x5 * rx; u2 += w; }
}

// vortex_tree.far_velocity with the symmetric second moment; R = x - c.  Order 3 (g: the third-order record) adds
//   (17.5 S3 / r^9 - 7.5 T3 R / r^7) x R - 7.5 (W3 : R R) / r^7 + 1.5 w3 / r^5,  S3_b = m3[b] : R R R,
// the next term of the same Taylor series of the segments' line integrals about the node centre; order 4 (k4: the
// fourth-order record) adds far_term4.
template <class T>
__device__ __forceinline__ void far_eval(T rx, T ry, T rz, const T *f, int order, T &ux, T &uy, T &uz,
                                         const T *g = nullptr, const T *k4 = nullptr, const T *z5 = nullptr) {
    T r2 = rx * rx + ry * ry + rz * rz;
    T inv3 = T(1) / (r2 * sqrt(r2));
    T inv5 = inv3 / r2;
    T u0 = inv3 * (f[F_M0 + 1] * rz - f[F_M0 + 2] * ry);
    T u1 = inv3 * (f[F_M0 + 2] * rx - f[F_M0 + 0] * rz);
    T u2 = inv3 * (f[F_M0 + 0] * ry - f[F_M0 + 1] * rx);
    if (order >= 1) {
        T v0 = f[F_M1 + 0] * rx + f[F_M1 + 1] * ry + f[F_M1 + 2] * rz;
        T v1 = f[F_M1 + 3] * rx + f[F_M1 + 4] * ry + f[F_M1 + 5] * rz;
        T v2 = f[F_M1 + 6] * rx + f[F_M1 + 7] * ry + f[F_M1 + 8] * rz;
        T k = T(3) * inv5;
        u0 += k * (v1 * rz - v2 * ry) - inv3 * f[F_W1 + 0];
        u1 += k * (v2 * rx - v0 * rz) - inv3 * f[F_W1 + 1];
        u2 += k * (v0 * ry - v1 * rx) - inv3 * f[F_W1 + 2];
    }
    if (order >= 2) {
        T inv7 = inv5 / r2;
        T xx = rx * rx, xy = rx * ry, xz = rx * rz, yy = ry * ry, yz = ry * rz, zz = rz * rz;
        T q[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const T *s = f + F_M2 + 6 * i;
            q[i] = s[0] * xx + s[3] * yy + s[5] * zz + T(2) * (s[1] * xy + s[2] * xz + s[4] * yz);
        }
        T a = T(7.5) * inv7, b = T(1.5) * inv5, k = T(3) * inv5;
        T b0 = a * q[0] - b * f[F_T2 + 0];
        T b1 = a * q[1] - b * f[F_T2 + 1];
        T b2 = a * q[2] - b * f[F_T2 + 2];
        T s0 = f[F_W2 + 0] * rx + f[F_W2 + 1] * ry + f[F_W2 + 2] * rz;
        T s1 = f[F_W2 + 3] * rx + f[F_W2 + 4] * ry + f[F_W2 + 5] * rz;
        T s2 = f[F_W2 + 6] * rx + f[F_W2 + 7] * ry + f[F_W2 + 8] * rz;
        u0 += (b1 * rz - b2 * ry) - k * s0;
        u1 += (b2 * rx - b0 * rz) - k * s1;
        u2 += (b0 * ry - b1 * rx) - k * s2;
        if (order >= 3) {
            const T inv9 = inv7 / r2;
            // cubic monomials with their multiplicities in the symmetric contraction
            const T c000 = xx * rx, c001 = T(3) * xx * ry, c002 = T(3) * xx * rz, c011 = T(3) * xy * ry;
            const T c012 = T(6) * xy * rz, c022 = T(3) * xz * rz, c111 = yy * ry, c112 = T(3) * yy * rz;
            const T c122 = T(3) * yz * rz, c222 = zz * rz;
            T x3[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T *m = g + G_M3 + 10 * i;
                const T s3 = m[0] * c000 + m[1] * c001 + m[2] * c002 + m[3] * c011 + m[4] * c012 + m[5] * c022 +
                             m[6] * c111 + m[7] * c112 + m[8] * c122 + m[9] * c222;
                const T *t3 = g + G_T3 + 3 * i;
                const T tr = t3[0] * rx + t3[1] * ry + t3[2] * rz;
                x3[i] = T(17.5) * inv9 * s3 - T(7.5) * inv7 * tr;
            }
            T w[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T *s = g + G_W3 + 6 * i;
                w[i] = s[0] * xx + s[3] * yy + s[5] * zz + T(2) * (s[1] * xy + s[2] * xz + s[4] * yz);
            }
            const T c7 = T(7.5) * inv7, c5 = T(1.5) * inv5;
            u0 += (x3[1] * rz - x3[2] * ry) - c7 * w[0] + c5 * g[G_W3V + 0];
            u1 += (x3[2] * rx - x3[0] * rz) - c7 * w[1] + c5 * g[G_W3V + 1];
            u2 += (x3[0] * ry - x3[1] * rx) - c7 * w[2] + c5 * g[G_W3V + 2];
            if (order >= 4) far_term4<T>(rx, ry, rz, inv7, inv9, inv9 / r2, k4, u0, u1, u2);
            if (order >= 5) {
                const T inv11 = inv9 / r2;
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    far_term5_row<T>(rx, ry, rz, inv7, inv9, inv11, inv11 / r2, z5 + Z_ROW * i, i, u0, u1, u2);
            }
        }
    }
    ux += T(INV_FOUR_PI) * u0;
    uy += T(INV_FOUR_PI) * u1;
    uz += T(INV_FOUR_PI) * u2;
}

// A far-record float4: through the read-only path from global memory, or (STAGED) a plain load from a copy the
// caller staged (in shared memory).
template <bool STAGED>
__device__ __forceinline__ float4 rec_ld(const float4 *p) {
    if constexpr (STAGED) return *p;
    else return __ldg(p);
}

// The fifth-order part on the unit vector n (FP32, record z5 of 42 float4), added to p5: a call of its own, so that its
// 56-float rows do not raise the register count of the kernels that inline far_eval32v.
template <bool STAGED>
static __device__ __noinline__ void far_order5_unit(float nx, float ny, float nz, const float4 *z5, float *p5) {
    float u0 = 0.f, u1 = 0.f, u2 = 0.f;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        float h[Z_ROW];
#pragma unroll
        for (int q = 0; q < Z_ROW / 4; ++q) {
            const float4 x = rec_ld<STAGED>(z5 + (Z_ROW / 4) * i + q);
            h[4 * q] = x.x; h[4 * q + 1] = x.y; h[4 * q + 2] = x.z; h[4 * q + 3] = x.w;
        }
        far_term5_row<float>(nx, ny, nz, 1.0f, 1.0f, 1.0f, 1.0f, h, i, u0, u1, u2);
    }
    p5[0] += u0;
    p5[1] += u1;
    p5[2] += u2;
}

// far_order5_unit inlined: for records staged in shared memory, whose loads then stay shared-memory loads.
template <bool STAGED>
__device__ __forceinline__ void far_order5_unit_inline(float nx, float ny, float nz, const float4 *z5, float *p5) {
    float u0 = 0.f, u1 = 0.f, u2 = 0.f;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        float h[Z_ROW];
#pragma unroll
        for (int q = 0; q < Z_ROW / 4; ++q) {
            const float4 x = rec_ld<STAGED>(z5 + (Z_ROW / 4) * i + q);
            h[4 * q] = x.x; h[4 * q + 1] = x.y; h[4 * q + 2] = x.z; h[4 * q + 3] = x.w;
        }
        far_term5_row<float>(nx, ny, nz, 1.0f, 1.0f, 1.0f, 1.0f, h, i, u0, u1, u2);
    }
    p5[0] += u0;
    p5[1] += u1;
    p5[2] += u2;
}

// far_eval<float> reading the packed records (Far32: 12 float4, Far32x: 16 float4, Far32y: 28 float4, Far32z: 42
// float4) in vector
// loads, one group at a time where it is used, so that only one order's coefficients are live at once.  The terms are
// those of far_eval written on the unit vector n = R / r: the order-p term is r^-(p+2) times a combination of the
// order-p coefficients and powers of n (R^k = r^k n^k), summed by Horner's rule in 1/r, so no intermediate carries a
// power of r beyond the order's own (r^-11 at order 4 would leave FP32's range for distances below ~1e-3.5 or above
// ~3e3 in the caller's units; here from ~1e-6 to ~1e6 every intermediate stays normal).
template <bool STAGED = false>
__device__ __forceinline__ void far_eval32v(float rx, float ry, float rz, const float4 *f, int order, float &ux,
                                            float &uy, float &uz, const float4 *g = nullptr,
                                            const float4 *k4 = nullptr, const float4 *z5 = nullptr) {
    const float r2 = rx * rx + ry * ry + rz * rz;
    // 1/r from the hardware estimate and one Newton-Raphson step for x^(-1/2) (y <- y (3 - x y^2) / 2): no IEEE
    // division or square root on this path
    float ir = rsqrtf(r2);
    ir = ir * fmaf(-0.5f * r2, ir * ir, 1.5f);
    const float nx = rx * ir, ny = ry * ir, nz = rz * ir;
    // order-p parts v_p (dimensionless in r); u = r^-2 (v0 + r^-1 (v1 + r^-1 (v2 + ...)))
    float p0[3] = {0.f, 0.f, 0.f}, p1[3] = {0.f, 0.f, 0.f}, p2[3] = {0.f, 0.f, 0.f}, p3[3] = {0.f, 0.f, 0.f},
          p4[3] = {0.f, 0.f, 0.f}, p5[3] = {0.f, 0.f, 0.f};
    const float4 q0 = rec_ld<STAGED>(f);  // m0 x y z, m1[0]
    p0[0] = q0.y * nz - q0.z * ny;
    p0[1] = q0.z * nx - q0.x * nz;
    p0[2] = q0.x * ny - q0.y * nx;
    if (order >= 1) {
        const float4 q1 = rec_ld<STAGED>(f + 1), q2 = rec_ld<STAGED>(f + 2), q3 = rec_ld<STAGED>(f + 3);  // m1[1..8], w1, t2[0]
        const float v0 = q0.w * nx + q1.x * ny + q1.y * nz;
        const float v1 = q1.z * nx + q1.w * ny + q2.x * nz;
        const float v2 = q2.y * nx + q2.z * ny + q2.w * nz;
        p1[0] = 3.0f * (v1 * nz - v2 * ny) - q3.x;
        p1[1] = 3.0f * (v2 * nx - v0 * nz) - q3.y;
        p1[2] = 3.0f * (v0 * ny - v1 * nx) - q3.z;
        if (order >= 2) {
            const float xx = nx * nx, xy = nx * ny, xz = nx * nz, yy = ny * ny, yz = ny * nz, zz = nz * nz;
            const float4 q4 = rec_ld<STAGED>(f + 4), q5 = rec_ld<STAGED>(f + 5), q6 = rec_ld<STAGED>(f + 6);  // t2[1..2], w2[0..8], m2 s[0]
            const float4 q7 = rec_ld<STAGED>(f + 7), q8 = rec_ld<STAGED>(f + 8), q9 = rec_ld<STAGED>(f + 9), q10 = rec_ld<STAGED>(f + 10),
                         q11 = rec_ld<STAGED>(f + 11);  // m2 symmetric s[1..17]
            // m2 symmetric rows (00,01,02,11,12,22) of i = 0, 1, 2 at floats 27..44
            const float s0[6] = {q6.w, q7.x, q7.y, q7.z, q7.w, q8.x};
            const float s1[6] = {q8.y, q8.z, q8.w, q9.x, q9.y, q9.z};
            const float s2[6] = {q9.w, q10.x, q10.y, q10.z, q10.w, q11.x};
            auto quad = [&](const float *sv) {
                return sv[0] * xx + sv[3] * yy + sv[5] * zz + 2.0f * (sv[1] * xy + sv[2] * xz + sv[4] * yz);
            };
            const float b0 = 7.5f * quad(s0) - 1.5f * q3.w;
            const float b1 = 7.5f * quad(s1) - 1.5f * q4.x;
            const float b2 = 7.5f * quad(s2) - 1.5f * q4.y;
            const float w0 = q4.z * nx + q4.w * ny + q5.x * nz;
            const float w1 = q5.y * nx + q5.z * ny + q5.w * nz;
            const float w2 = q6.x * nx + q6.y * ny + q6.z * nz;
            p2[0] = (b1 * nz - b2 * ny) - 3.0f * w0;
            p2[1] = (b2 * nx - b0 * nz) - 3.0f * w1;
            p2[2] = (b0 * ny - b1 * nx) - 3.0f * w2;
            if (order >= 3) {
                const float c000 = xx * nx, c001 = 3.0f * xx * ny, c002 = 3.0f * xx * nz, c011 = 3.0f * xy * ny;
                const float c012 = 6.0f * xy * nz, c022 = 3.0f * xz * nz, c111 = yy * ny, c112 = 3.0f * yy * nz;
                const float c122 = 3.0f * yz * nz, c222 = zz * nz;
                float x3[3], w[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    float h[H_ROW];  // component i's row: m3 (10), T3 (3), W3 (6), pad
#pragma unroll
                    for (int q = 0; q < H_ROW / 4; ++q) {
                        const float4 x = rec_ld<STAGED>(g + (H_ROW / 4) * i + q);
                        h[4 * q] = x.x; h[4 * q + 1] = x.y; h[4 * q + 2] = x.z; h[4 * q + 3] = x.w;
                    }
                    const float *m = h + H_M3;
                    const float s3 = m[0] * c000 + m[1] * c001 + m[2] * c002 + m[3] * c011 + m[4] * c012 +
                                     m[5] * c022 + m[6] * c111 + m[7] * c112 + m[8] * c122 + m[9] * c222;
                    const float tr = h[H_T3] * nx + h[H_T3 + 1] * ny + h[H_T3 + 2] * nz;
                    x3[i] = 17.5f * s3 - 7.5f * tr;
                    w[i] = quad(h + H_W3);
                }
                const float4 wv = rec_ld<STAGED>(g + H_W3V / 4);
                p3[0] = (x3[1] * nz - x3[2] * ny) - 7.5f * w[0] + 1.5f * wv.x;
                p3[1] = (x3[2] * nx - x3[0] * nz) - 7.5f * w[1] + 1.5f * wv.y;
                p3[2] = (x3[0] * ny - x3[1] * nx) - 7.5f * w[2] + 1.5f * wv.z;
                if (order >= 4) {
                    // one component row at a time (nine float4), through the shared fourth-order term at r = 1
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        float h[K_ROW];
#pragma unroll
                        for (int q = 0; q < K_ROW / 4; ++q) {
                            const float4 x = rec_ld<STAGED>(k4 + (K_ROW / 4) * i + q);
                            h[4 * q] = x.x; h[4 * q + 1] = x.y; h[4 * q + 2] = x.z; h[4 * q + 3] = x.w;
                        }
                        far_term4_row<float>(nx, ny, nz, 1.0f, 1.0f, 1.0f, h, i, p4[0], p4[1], p4[2]);
                    }
                    if (order >= 5) {
                        if constexpr (STAGED) far_order5_unit_inline<true>(nx, ny, nz, z5, p5);
                        else far_order5_unit<false>(nx, ny, nz, z5, p5);
                    }
                }
            }
        }
    }
    const float scale = (float)INV_FOUR_PI * ir * ir;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float v = p0[c] + ir * (p1[c] + ir * (p2[c] + ir * (p3[c] + ir * (p4[c] + ir * p5[c]))));
        if (c == 0) ux += scale * v;
        else if (c == 1) uy += scale * v;
        else uz += scale * v;
    }
}

// Two-float split of an FP64 value: hi = round(x), lo = round(x - hi).
__device__ __forceinline__ void split2(double x, float &hi, float &lo) {
    hi = __double2float_rn(x);
    lo = __double2float_rn(x - (double)hi);
}

// ---------------------------------------------------------------------------------------------------------------------
// Bulk copies (TMA) with bounded mbarrier waits.
// ---------------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Asynchronous 16-byte copies global -> shared (both addresses 16-byte aligned), committed in groups; a thread waits
// for its own copies (all but the newest N groups) and then __syncwarp()s before other lanes read them.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Global -> shared bulk copy completing on `bar`; dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Waits for `phase` of `bar`; gives up after `limit` polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase, uint32_t limit = (1u << 26)) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace bs
