// Reverse-mode pair terms shared by the adjoints of the direct sum (bs_adjoint.cu) and of the tree sum
// (bs_tree_adjoint.cu).  The pair is the reference's (vortex_numba.pair_velocity, src/openfawe/aero/vortex_numba.py:42-109)
// in its two-endpoint form, r1 = x - A, r2 = x - B, c = r1 x r2, P = |r1||r2|, d = r1.r2,
//   D = P (P + d), or P |c|^2 / (P - d) when d < 0 (the reference's rationalised branch),
//   u = Gamma/(4 pi) f(|c|^2 / (|B - A|^2 rc^2)) (|r1| + |r2|) c / D,
// with the core factor f of models 0 (none), 1 (Rankine), 2 (Lamb-Oseen with its exponent cut-off) and 3 (Vatistas
// n = 2: f = rho^2 / sqrt(1 + rho^4)); model 4 (offset core) adds rc^2 |B - A|^2 to D, model 5 (Rosenhead-Moore) takes
// |r1|, |r2| as sqrt(|r1|^2 + rc^2), sqrt(|r2|^2 + rc^2) and d as r1.r2 + rc^2 (P^2 - d^2 = |c|^2 + rc^2 |B - A|^2),
// which is the FP64 pair's form (pair64_core) in physical units.
#pragma once
#include "bs_internal.cuh"

namespace bs {

// A segment as the adjoint reads it: endpoints, circulation and the per-segment invariants of the pair.
struct AdjSeg {
    double ax, ay, az, bx, by, bz, gamma;
    double irc2L2;  // 1 / (L^2 rc^2) for a core-factor model (1, 2, 3) with rc > 0, else 0 (no core factor)
    double invL2;   // 1 / L^2
    double rc2;     // rc^2 for the offset and Rosenhead-Moore models (4, 5), else 0
};
struct AdjTgt {
    double x, y, z, wx, wy, wz;
};

static constexpr double AXIS_EPS64_SQ = AXIS_EPS64 * AXIS_EPS64;

// d(w . u)/dr1 and d(w . u)/dr2 of one pair (r1 = x - A, r2 = x - B) and d(w . u)/dGamma; false for a pair that
// contributes nothing (the roundoff axis guard).  Then d/dx = g1 + g2, d/dA = -g1, d/dB = -g2.
__device__ __forceinline__ bool pair_vjp64(double x0, double x1, double x2, const AdjSeg &s, int model, double w0,
                                           double w1, double w2, double *g1, double *g2, double &gg) {
    const double r10 = x0 - s.ax, r11 = x1 - s.ay, r12 = x2 - s.az;
    const double r20 = x0 - s.bx, r21 = x1 - s.by, r22 = x2 - s.bz;
    const double c0 = r11 * r22 - r12 * r21, c1 = r12 * r20 - r10 * r22, c2v = r10 * r21 - r11 * r20;
    const double cc = c0 * c0 + c1 * c1 + c2v * c2v;
    const double q1 = r10 * r10 + r11 * r11 + r12 * r12, q2 = r20 * r20 + r21 * r21 + r22 * r22;
    // the reference's roundoff axis guard h <= eps max(1, na, nb) in its scaled units (h = |c|/L^2,
    // na = |r1|/L, nb = |r2|/L), squared
    if (cc * s.invL2 * s.invL2 <= AXIS_EPS64_SQ * fmax(1.0, fmax(q1, q2) * s.invL2)) return false;
    // |r1|, |r2| (Rosenhead-Moore: augmented by the core) and their reciprocals
    const bool rm = model == 5 && s.rc2 > 0.0;
    const double in1 = rm ? 1.0 / sqrt(q1 + s.rc2) : rsqrt(q1), in2 = rm ? 1.0 / sqrt(q2 + s.rc2) : rsqrt(q2);
    const double n1 = rm ? sqrt(q1 + s.rc2) : q1 * in1, n2 = rm ? sqrt(q2 + s.rc2) : q2 * in2;
    const double d = r10 * r20 + r11 * r21 + r12 * r22 + (rm ? s.rc2 : 0.0);
    const double P = n1 * n2;
    const double L2 = 1.0 / s.invL2;
    const double Q = rm ? cc + s.rc2 * L2 : cc;  // P^2 - d^2
    double D, dD_dP, dD_dd, dD_dcc, dD_dL2 = 0.0;
    if (d >= 0.0) {
        D = P * (P + d);
        dD_dP = 2.0 * P + d;
        dD_dd = P;
        dD_dcc = 0.0;
    } else {  // the rationalised denominator P (P + d) = P Q / (P - d)
        const double iq = 1.0 / (P - d);
        D = P * Q * iq;
        dD_dP = -Q * d * iq * iq;
        dD_dd = P * Q * iq * iq;
        dD_dcc = P * iq;
        if (rm) dD_dL2 = s.rc2 * P * iq;
    }
    if (model == 4 && s.rc2 > 0.0) {  // offset core
        D += s.rc2 * L2;
        dD_dL2 = s.rc2;
    }
    double f = 1.0, df = 0.0, rho2 = 0.0;  // core factor f(rho2), df/drho2 with rho2 = |c|^2 / (L^2 rc^2)
    if (s.irc2L2 > 0.0) {
        rho2 = cc * s.irc2L2;
        if (model == 1) {
            if (rho2 < 1.0) { f = rho2; df = 1.0; }
        } else if (model == 3) {  // Vatistas n = 2: f = x / sqrt(1 + x^2), f' = (1 + x^2)^(-3/2)
            f = rho2 < 1.0 ? rho2 / hypot(1.0, rho2) : 1.0 / hypot(1.0, 1.0 / rho2);
            const double g = rho2 < 1.0 ? 1.0 / hypot(1.0, rho2) : (1.0 / rho2) / hypot(1.0, 1.0 / rho2);
            df = g * g * g;  // (1 + x^2)^(-3/2), as (1/x)^3 / (1 + 1/x^2)^(3/2) for large x
        } else if (rho2 <= LAMB_CUT2) {
            const double em1 = expm1(-LAMB_A * rho2);
            f = -em1;
            df = LAMB_A * (1.0 + em1);
        }
    }
    const double S = n1 + n2;
    const double iD = 1.0 / D;
    const double coefG = INV_FOUR_PI * f * S * iD;  // u = Gamma * coefG * c
    const double wc = w0 * c0 + w1 * c1 + w2 * c2v;
    gg = coefG * wc;
    const double G = s.gamma;
    const double h = G * wc * INV_FOUR_PI * iD;  // common factor of the scalar adjoints
    const double g_f = h * S;
    const double g_S = h * f;
    const double g_D = -h * f * S * iD;
    const double g_rho2 = g_f * df;
    const double g_cc = g_rho2 * s.irc2L2 + g_D * dD_dcc;
    const double g_L2 = -g_rho2 * rho2 * s.invL2 + g_D * dD_dL2;
    const double g_P = g_D * dD_dP, g_d = g_D * dD_dd;
    const double k = G * coefG;
    const double gc0 = k * w0 + 2.0 * c0 * g_cc, gc1 = k * w1 + 2.0 * c1 * g_cc, gc2 = k * w2 + 2.0 * c2v * g_cc;
    // c = r1 x r2: dL/dr1 += r2 x g_c, dL/dr2 += g_c x r1; |B - A|^2 = |r1 - r2|^2: dL2/dr1 = 2 l = -dL2/dr2
    const double a1 = (g_S + g_P * n2) * in1, a2 = (g_S + g_P * n1) * in2, b = 2.0 * g_L2;
    const double l0 = s.bx - s.ax, l1 = s.by - s.ay, l2 = s.bz - s.az;
    g1[0] = a1 * r10 + g_d * r20 + (r21 * gc2 - r22 * gc1) + b * l0;
    g1[1] = a1 * r11 + g_d * r21 + (r22 * gc0 - r20 * gc2) + b * l1;
    g1[2] = a1 * r12 + g_d * r22 + (r20 * gc1 - r21 * gc0) + b * l2;
    g2[0] = a2 * r20 + g_d * r10 + (gc1 * r12 - gc2 * r11) - b * l0;
    g2[1] = a2 * r21 + g_d * r11 + (gc2 * r10 - gc0 * r12) - b * l1;
    g2[2] = a2 * r22 + g_d * r12 + (gc0 * r11 - gc1 * r10) - b * l2;
    return true;
}

// pair_vjp64 in single precision, for the tree adjoint's near pairs: the same expression in units of the segment's
// length (a1 = r1 / L, a2 = r2 / L = a1 - d, as the forward's single-precision pair forms it, so that any length scale
// stays in range), from the forward's Seg32 record (two-float start, 1/L, (Gamma/L)/(4 pi), direction, (L/rc)^2) and a
// two-float target.  Returns true, and computes nothing, where the forward evaluates the pair in FP64: within
// sqrt(near2) core radii of the finite segment (MODEL 0: within L/4 of it), within 1e-4 L of its axis, or out of
// FP32's comfortable range (the caller then takes pair_vjp64).  Otherwise g1 = d(w . u)/dr1, g2 = d(w . u)/dr2 and
// gg = d(w . u)/dGamma.  In units of L the pair is u = (Gamma/L)/(4 pi) f S c / D with rho^2 = |c|^2 (L/rc)^2, and
// the one explicit dependence on L through rho^2 gives the bb d terms (d(|B - A|^2)/dr1 = 2 (B - A)).
template <int MODEL>
__device__ __forceinline__ bool pair_vjp32(float xh0, float xh1, float xh2, float xl0, float xl1, float xl2,
                                           const Seg32 &r, float w0, float w1, float w2, float near2, float *g1,
                                           float *g2, float &gg) {
    const float il = r.hi.w, gfac = r.lo.w, lrc2 = r.dir.w;
    const float dx = r.dir.x, dy = r.dir.y, dz = r.dir.z;
    const float a0 = ((xh0 - r.hi.x) + (xl0 - r.lo.x)) * il;
    const float a1 = ((xh1 - r.hi.y) + (xl1 - r.lo.y)) * il;
    const float a2 = ((xh2 - r.hi.z) + (xl2 - r.lo.z)) * il;
    const float b0 = a0 - dx, b1 = a1 - dy, b2 = a2 - dz;
    // c = d x a1 = a1 x a2
    const float c0 = fmaf(dy, a2, -dz * a1), c1 = fmaf(dz, a0, -dx * a2), c2 = fmaf(dx, a1, -dy * a0);
    const float cc = fmaf(c0, c0, fmaf(c1, c1, c2 * c2));
    const float q1 = fmaf(a0, a0, fmaf(a1, a1, a2 * a2)), q2 = fmaf(b0, b0, fmaf(b1, b1, b2 * b2));
    const float big2 = fmaxf(1.0f, fmaxf(q1, q2));
    bool need64 = !(cc > 1e-8f * big2) || !(big2 < 1e18f);
    {
        const float t = fmaf(a2, dz, fmaf(a1, dy, a0 * dx));
        const float seg2 = t < 0.0f ? q1 : (t > 1.0f ? q2 : cc);
        need64 = need64 || (MODEL == 0 ? seg2 < NOCORE_NEAR2 : (lrc2 > 0.0f && seg2 * lrc2 < near2));
    }
    if (need64) return true;
    const float in1 = rsqrtf(q1), in2 = rsqrtf(q2);
    const float n1 = q1 * in1, n2 = q2 * in2;
    const float dt = fmaf(a0, b0, fmaf(a1, b1, a2 * b2));
    const float P = n1 * n2;
    float D, dD_dP, dD_dd, dD_dcc;
    if (dt >= 0.0f) {
        D = P * (P + dt);
        dD_dP = 2.0f * P + dt;
        dD_dd = P;
        dD_dcc = 0.0f;
    } else {
        const float iq = __fdividef(1.0f, P - dt);
        D = P * cc * iq;
        dD_dP = -cc * dt * iq * iq;
        dD_dd = P * cc * iq * iq;
        dD_dcc = P * iq;
    }
    float f = 1.0f, df = 0.0f, rho2 = 0.0f;
    if (MODEL != 0 && lrc2 > 0.0f) {
        rho2 = cc * lrc2;
        if (MODEL == 1) {
            if (rho2 < 1.0f) { f = rho2; df = 1.0f; }
        } else if (rho2 <= (float)LAMB_CUT2) {
            const float e = __expf(-(float)LAMB_A * rho2);
            f = 1.0f - e;
            df = (float)LAMB_A * e;
        }
    }
    const float S = n1 + n2;
    const float iD = __fdividef(1.0f, D);
    const float wc = fmaf(w0, c0, fmaf(w1, c1, w2 * c2));
    const float h = gfac * wc * iD;
    gg = (float)INV_FOUR_PI * il * f * S * wc * iD;
    const float g_f = h * S, g_S = h * f, g_D = -h * f * S * iD;
    const float g_rho2 = g_f * df;
    const float g_cc = g_rho2 * lrc2 + g_D * dD_dcc;
    const float g_P = g_D * dD_dP, g_d = g_D * dD_dd;
    const float k = gfac * f * S * iD;
    const float gc0 = fmaf(2.0f * c0, g_cc, k * w0), gc1 = fmaf(2.0f * c1, g_cc, k * w1),
                gc2 = fmaf(2.0f * c2, g_cc, k * w2);
    const float s1 = (g_S + g_P * n2) * in1, s2 = (g_S + g_P * n1) * in2, bb = -2.0f * g_rho2 * rho2;
    // derivatives in a1, a2 (units of L), then d/dr = (1/L) d/da
    g1[0] = il * (s1 * a0 + g_d * b0 + (b1 * gc2 - b2 * gc1) + bb * dx);
    g1[1] = il * (s1 * a1 + g_d * b1 + (b2 * gc0 - b0 * gc2) + bb * dy);
    g1[2] = il * (s1 * a2 + g_d * b2 + (b0 * gc1 - b1 * gc0) + bb * dz);
    g2[0] = il * (s2 * b0 + g_d * a0 + (gc1 * a2 - gc2 * a1) - bb * dx);
    g2[1] = il * (s2 * b1 + g_d * a1 + (gc2 * a0 - gc0 * a2) - bb * dy);
    g2[2] = il * (s2 * b2 + g_d * a2 + (gc0 * a1 - gc1 * a0) - bb * dz);
    return false;
}

// One segment of a leaf for the tree adjoint, from its half of the clear-leaf pair record (Seg32c2): start relative
// to the leaf's centre O, negated; Gamma/(4 pi); l = L d; 1/(L rc)^2 (+inf without a core).
struct ClearSeg {
    float nsx, nsy, nsz, gf, lx, ly, lz, w;
};

// pair_vjp32 for a target clear of the segment's leaf (the conditions of pair32x2_clear: at least 1.5 bounding radii
// from the leaf's centre, outside the core test's reach, within FP32's range), in physical units from the target's
// offset (rx, ry, rz) = x - O: r1 = x - A, r2 = x - B, l = B - A = r1 - r2, c = r1 x r2, and the forward's
//   u = Gamma/(4 pi) f S c / D,  S = |r1| + |r2|,  P = |r1||r2|,  D = P (P + r1.r2),  rho^2 = |c|^2 / (L rc)^2.
// No FP64 fallback: no pair of a clear target needs one.  g1 = d(w.u)/dr1, g2 = d(w.u)/dr2, gg = d(w.u)/dGamma; the
// dependence of rho^2 on L = |l| gives the -/+ 2 g_rho2 rho2 l / L^2 terms.  MODEL 0..2.
template <int MODEL>
__device__ __forceinline__ void pair_vjp32_clear(float rx, float ry, float rz, const ClearSeg &q, float w0, float w1,
                                                 float w2, float *g1, float *g2, float &gg) {
    const float a0 = rx + q.nsx, a1 = ry + q.nsy, a2 = rz + q.nsz;  // r1
    const float b0 = a0 - q.lx, b1 = a1 - q.ly, b2 = a2 - q.lz;     // r2
    // c = l x r1 = r1 x r2
    const float c0 = fmaf(q.ly, a2, -q.lz * a1), c1 = fmaf(q.lz, a0, -q.lx * a2), c2 = fmaf(q.lx, a1, -q.ly * a0);
    const float cc = fmaf(c0, c0, fmaf(c1, c1, c2 * c2));
    const float q1 = fmaf(a0, a0, fmaf(a1, a1, a2 * a2)), q2 = fmaf(b0, b0, fmaf(b1, b1, b2 * b2));
    const float in1 = rsqrtf(q1), in2 = rsqrtf(q2);
    const float n1 = q1 * in1, n2 = q2 * in2;
    const float dt = fmaf(a0, b0, fmaf(a1, b1, a2 * b2));
    const float P = n1 * n2, D = P * (P + dt), iD = __fdividef(1.0f, D);
    float f = 1.0f, df = 0.0f, rho2 = 0.0f;
    if (MODEL != 0) {
        rho2 = cc * q.w;  // +inf or NaN without a core: f stays 1, df 0
        if (MODEL == 1) {
            if (rho2 < 1.0f) { f = rho2; df = 1.0f; }
        } else if (rho2 <= (float)LAMB_CUT2) {
            const float e = exp2_approx(rho2 * LAMB_A_LOG2E_NEG);
            f = 1.0f - e;
            df = (float)LAMB_A * e;
        }
    }
    const float S = n1 + n2;
    const float wc = fmaf(w0, c0, fmaf(w1, c1, w2 * c2));
    const float h = q.gf * wc * iD;
    gg = (float)INV_FOUR_PI * f * S * wc * iD;
    const float g_S = h * f, g_D = -h * f * S * iD;
    const float g_rho2 = h * S * df;
    const float g_cc = df != 0.0f ? g_rho2 * q.w : 0.0f;
    const float g_P = g_D * (2.0f * P + dt), g_dt = g_D * P;
    const float k = q.gf * f * S * iD;
    const float gc0 = fmaf(2.0f * c0, g_cc, k * w0), gc1 = fmaf(2.0f * c1, g_cc, k * w1),
                gc2 = fmaf(2.0f * c2, g_cc, k * w2);
    const float s1 = (g_S + g_P * n2) * in1, s2 = (g_S + g_P * n1) * in2;
    const float L2 = fmaf(q.lx, q.lx, fmaf(q.ly, q.ly, q.lz * q.lz));
    const float bb = df != 0.0f ? 2.0f * g_rho2 * rho2 * __fdividef(1.0f, L2) : 0.0f;
    g1[0] = s1 * a0 + g_dt * b0 + (b1 * gc2 - b2 * gc1) - bb * q.lx;
    g1[1] = s1 * a1 + g_dt * b1 + (b2 * gc0 - b0 * gc2) - bb * q.ly;
    g1[2] = s1 * a2 + g_dt * b2 + (b0 * gc1 - b1 * gc0) - bb * q.lz;
    g2[0] = s2 * b0 + g_dt * a0 + (gc1 * a2 - gc2 * a1) + bb * q.lx;
    g2[1] = s2 * b1 + g_dt * a1 + (gc2 * a0 - gc0 * a2) + bb * q.ly;
    g2[2] = s2 * b2 + g_dt * a2 + (gc0 * a1 - gc1 * a0) + bb * q.lz;
}

// pair_vjp32_clear for two targets of the same segment at once (f32x2: .x and .y), one packed operation for both in
// every add, multiply and FMA; special functions and the core factor's branches per half.  iL2 = 1/|l|^2 from the
// caller (0 for a thread without a segment, whose targets carry zero cotangents).  A half with zero cotangent gives
// zero gradients as long as its offset is a clear target's.  The lanes evaluating the call vote on whether any of
// their pairs lies inside the core factor's range ((h/rc)^2 below 1 for Rankine, below the cut-off for Lamb-Oseen);
// a clear target seldom does, and then f = 1, df = 0 leave out the core terms (the same values, to the sign of a zero).
template <int MODEL>
__device__ __forceinline__ void pair_vjp32_clear2(float2 rx, float2 ry, float2 rz, const ClearSeg &q, float iL2,
                                                  float2 w0, float2 w1, float2 w2, float2 *g1, float2 *g2,
                                                  float2 &gg) {
    auto bc = [](float v) { return make_float2(v, v); };
    auto neg = [](float2 v) { return make_float2(-v.x, -v.y); };
    const float2 lx = bc(q.lx), ly = bc(q.ly), lz = bc(q.lz), nlx = bc(-q.lx), nly = bc(-q.ly), nlz = bc(-q.lz);
    const float2 a0 = add2(rx, bc(q.nsx)), a1 = add2(ry, bc(q.nsy)), a2 = add2(rz, bc(q.nsz));  // r1
    const float2 b0 = add2(a0, nlx), b1 = add2(a1, nly), b2 = add2(a2, nlz);                     // r2
    const float2 c0 = fma2(ly, a2, mul2(nlz, a1)), c1 = fma2(lz, a0, mul2(nlx, a2)), c2 = fma2(lx, a1, mul2(nly, a0));
    const float2 cc = fma2(c0, c0, fma2(c1, c1, mul2(c2, c2)));
    const float2 q1 = fma2(a0, a0, fma2(a1, a1, mul2(a2, a2))), q2 = fma2(b0, b0, fma2(b1, b1, mul2(b2, b2)));
    const float2 in1 = make_float2(rsqrtf(q1.x), rsqrtf(q1.y)), in2 = make_float2(rsqrtf(q2.x), rsqrtf(q2.y));
    const float2 n1 = mul2(q1, in1), n2 = mul2(q2, in2);
    const float2 dt = fma2(a0, b0, fma2(a1, b1, mul2(a2, b2)));
    const float2 P = mul2(n1, n2), D = mul2(P, add2(P, dt));
    const float2 iD = make_float2(__fdividef(1.0f, D.x), __fdividef(1.0f, D.y));
    const float2 S = add2(n1, n2);
    const float2 wc = fma2(w0, c0, fma2(w1, c1, mul2(w2, c2)));
    const float2 wciD = mul2(wc, iD);
    const float2 h = mul2(bc(q.gf), wciD);
    float2 rho2 = bc(0.0f);  // +inf or NaN without a core: outside every range
    bool inside = false;
    if (MODEL != 0) {
        rho2 = mul2(cc, bc(q.w));
        const float lim = MODEL == 1 ? 1.0f : (float)LAMB_CUT2;
        inside = __any_sync(__activemask(), MODEL == 1 ? (rho2.x < lim || rho2.y < lim)
                                                       : (rho2.x <= lim || rho2.y <= lim));
    }
    if (!inside) {  // f = 1, df = 0
        gg = mul2(bc((float)INV_FOUR_PI), mul2(S, wciD));
        const float2 g_D = mul2(mul2(h, S), neg(iD));
        const float2 g_P = mul2(g_D, fma2(bc(2.0f), P, dt)), g_dt = mul2(g_D, P);
        const float2 k = mul2(bc(q.gf), mul2(S, iD));
        const float2 gc0 = mul2(k, w0), gc1 = mul2(k, w1), gc2 = mul2(k, w2);
        const float2 s1 = mul2(fma2(g_P, n2, h), in1), s2 = mul2(fma2(g_P, n1, h), in2);
        g1[0] = fma2(s1, a0, fma2(g_dt, b0, fma2(b1, gc2, mul2(neg(b2), gc1))));
        g1[1] = fma2(s1, a1, fma2(g_dt, b1, fma2(b2, gc0, mul2(neg(b0), gc2))));
        g1[2] = fma2(s1, a2, fma2(g_dt, b2, fma2(b0, gc1, mul2(neg(b1), gc0))));
        g2[0] = fma2(s2, b0, fma2(g_dt, a0, fma2(gc1, a2, mul2(neg(gc2), a1))));
        g2[1] = fma2(s2, b1, fma2(g_dt, a1, fma2(gc2, a0, mul2(neg(gc0), a2))));
        g2[2] = fma2(s2, b2, fma2(g_dt, a2, fma2(gc0, a1, mul2(neg(gc1), a0))));
        return;
    }
    float2 f = bc(1.0f), df = bc(0.0f);
    auto core = [&](float r2, float &fo, float &dfo) {
        if (MODEL == 1) {
            if (r2 < 1.0f) { fo = r2; dfo = 1.0f; }
        } else if (r2 <= (float)LAMB_CUT2) {
            const float e = exp2_approx(r2 * LAMB_A_LOG2E_NEG);
            fo = 1.0f - e;
            dfo = (float)LAMB_A * e;
        }
    };
    core(rho2.x, f.x, df.x);
    core(rho2.y, f.y, df.y);
    gg = mul2(mul2(bc((float)INV_FOUR_PI), f), mul2(S, wciD));
    const float2 hf = mul2(h, f);
    const float2 g_S = hf, g_D = mul2(mul2(hf, S), neg(iD));
    const float2 g_rho2 = mul2(mul2(h, S), df);
    const float2 g_cc = make_float2(df.x != 0.0f ? g_rho2.x * q.w : 0.0f, df.y != 0.0f ? g_rho2.y * q.w : 0.0f);
    const float2 g_P = mul2(g_D, fma2(bc(2.0f), P, dt)), g_dt = mul2(g_D, P);
    const float2 k = mul2(mul2(bc(q.gf), f), mul2(S, iD));
    const float2 gc0 = fma2(add2(c0, c0), g_cc, mul2(k, w0)), gc1 = fma2(add2(c1, c1), g_cc, mul2(k, w1)),
                 gc2 = fma2(add2(c2, c2), g_cc, mul2(k, w2));
    const float2 s1 = mul2(fma2(g_P, n2, g_S), in1), s2 = mul2(fma2(g_P, n1, g_S), in2);
    const float2 bb = make_float2(df.x != 0.0f ? 2.0f * g_rho2.x * rho2.x * iL2 : 0.0f,
                                  df.y != 0.0f ? 2.0f * g_rho2.y * rho2.y * iL2 : 0.0f);
    const float2 nbb = neg(bb);
    // g1 = s1 r1 + g_dt r2 + r2 x gc - bb l;  g2 = s2 r2 + g_dt r1 + gc x r1 + bb l
    g1[0] = fma2(s1, a0, fma2(g_dt, b0, fma2(b1, gc2, fma2(neg(b2), gc1, mul2(nbb, lx)))));
    g1[1] = fma2(s1, a1, fma2(g_dt, b1, fma2(b2, gc0, fma2(neg(b0), gc2, mul2(nbb, ly)))));
    g1[2] = fma2(s1, a2, fma2(g_dt, b2, fma2(b0, gc1, fma2(neg(b1), gc0, mul2(nbb, lz)))));
    g2[0] = fma2(s2, b0, fma2(g_dt, a0, fma2(gc1, a2, fma2(neg(gc2), a1, mul2(bb, lx)))));
    g2[1] = fma2(s2, b1, fma2(g_dt, a1, fma2(gc2, a0, fma2(neg(gc0), a2, mul2(bb, ly)))));
    g2[2] = fma2(s2, b2, fma2(g_dt, a2, fma2(gc0, a1, fma2(neg(gc1), a0, mul2(bb, lz)))));
}

}  // namespace bs
