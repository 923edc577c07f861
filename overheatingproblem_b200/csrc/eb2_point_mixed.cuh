// eb2_point_mixed.cuh -- per-interface arithmetic of the mixed-precision form.
//
// The conserved state, the RK stage sums and the CFL reduction stay FP64; the
// characteristic projection, WENO5 reconstruction and Riemann flux run in
// FP32 with three reformulations that keep FP32 rounding relative to the
// quantities that matter rather than to |U|:
//
//  * delta form -- the stencil is projected as differences from the cell
//    next to the interface (the "base" cell), so rounding is relative to the
//    jumps; WENO is translation invariant, the base is added back after the
//    back-projection;
//  * cancellation-free thermodynamics -- the Roe sound speed is formed from
//    h = gamma/(gamma-1) p/rho of each cell plus 1/2 wa wb |du|^2 instead of
//    H - q^2/2, b2 = b1 q^2 / 2, and interface pressures are p_base +
//    (gamma-1)(dE - dK) with dK the kinetic-energy change written in
//    differences; cell pressures themselves come from FP64;
//  * weights in range -- the JS and WENO-Z weights come from SFU reciprocals
//    of beta + eps (eps keeps them below 1e15).  eps is the reference's
//    absolute 1e-15 (Reconstruction.h:1414).  Where FP32 rounding noise in beta
//    exceeds eps the candidate values agree to that noise, so the weights it
//    picks do not show in the result.
// Interfaces next to near-vacuum cells (p < 1e-3 of the mean pressure) get
// their Roe eigenvectors from FP64 arithmetic.
#pragma once

#include "eb2_common.cuh"

namespace eb2 {
namespace f32 {

// Approximate reciprocal / reciprocal square root: the SFU instructions on the
// GPU, plain IEEE arithmetic on the host (CPU checks of this file).
EB2_HD float rcp(float x) {
#ifdef __CUDA_ARCH__
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return 1.0f / x;
#endif
}
EB2_HD float rsq(float x) {
#ifdef __CUDA_ARCH__
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return 1.0f / sqrtf(x);
#endif
}
EB2_HD float sqr(float x) { return x * rsq(x); }  // sqrt for x > 0

// --- two-lane arithmetic -----------------------------------------------------
// The two sides of an interface run the same reconstruction on mirrored
// stencils, so they ride the two lanes of one float2: .x the minus side
// (around cell i), .y the plus side (around cell i+1).  On the GPU each
// operation is one packed FP32 instruction of sm_100 (FFMA2 / FMUL2 / FADD2,
// round to nearest), which halves the issue slots of the per-side arithmetic;
// on the host (CPU checks of this file) it is two scalar operations with the
// same rounding.
using f2 = float2;
EB2_HD f2 f2s(float a) { return make_float2(a, a); }
EB2_HD f2 f2n(f2 a) { return make_float2(-a.x, -a.y); }
EB2_HD f2 fma2(f2 a, f2 b, f2 c) {
#ifdef __CUDA_ARCH__
    return __ffma2_rn(a, b, c);
#else
    return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}
EB2_HD f2 mul2(f2 a, f2 b) {
#ifdef __CUDA_ARCH__
    return __fmul2_rn(a, b);
#else
    return make_float2(a.x * b.x, a.y * b.y);
#endif
}
EB2_HD f2 add2(f2 a, f2 b) {
#ifdef __CUDA_ARCH__
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}
EB2_HD f2 sub2(f2 a, f2 b) { return add2(a, f2n(b)); }
EB2_HD f2 rcp2(f2 a) { return make_float2(rcp(a.x), rcp(a.y)); }
// the bits of a float (zero tests without floating-point compares)
EB2_HD unsigned bits(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    unsigned u;
    memcpy(&u, &x, sizeof u);
    return u;
#endif
}

// 1/x for a positive normal double to ~1e-17 relative: the SFU seed refined by
// one third-order Newton-Raphson step, y (1 + e + e^2) with e = 1 - x y.
EB2_HD double rcp64(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
#else
    return 1.0 / x;
#endif
}

// Per-cell primitive data kept in shared memory (FP32 values of FP64 results):
// a float4 (rho, u, v, p) and a float2 (h = gamma/(gamma-1) p/rho, sqrt(rho)),
// so that an interface reads each cell's record with two vector loads.

// Primitive record of one cell from its conserved state (q in FP64, qf the
// same values rounded to FP32): the pressure is formed in FP64, where E minus
// the kinetic energy cancels in low-pressure flows, then stored FP32; the
// velocities, enthalpy and sqrt(rho) need only FP32.
EB2_HD void cell_prims(const double* q, const float* qf, const Gas& g, float4* P, float2* H) {
    const double ir = rcp64(q[0]);
    const double p = fma(-0.5 * ir, fma(q[1], q[1], q[2] * q[2]), q[3]) * g.gm1;
    const float pf = (float)p, irf = rcp(qf[0]);
    *P = make_float4(qf[0], qf[1] * irf, qf[2] * irf, pf);
    *H = make_float2((float)g.gr * pf * irf, sqr(qf[0]));
}

// Eigen-system parameters at an interface (the Roe average), in the form the
// factored projections below use.
struct Eig {
    float u, v, c, hb1, hic, hq2, cg, b1, H;
};

EB2_HD Eig eig_from(float u, float v, float c2, float gm1) {
    Eig e;
    float ic = rsq(c2);
    e.u = u;
    e.v = v;
    e.c = c2 * ic;
    float b1 = gm1 * ic * ic;
    float q2 = u * u + v * v;
    e.b1 = b1;
    e.hb1 = 0.5f * b1;
    e.hic = 0.5f * ic;
    e.hq2 = 0.5f * q2;
    e.cg = c2 * (1.0f / gm1);
    e.H = e.cg + e.hq2;
    return e;
}

// Roe average from FP32 cell data: weights sqrt(rho), sound speed from the
// cell enthalpies h (no H - q^2/2 cancellation).
EB2_HD Eig roe_f32(const float4& a, const float2& ha, const float4& b, const float2& hb,
                   float gm1) {
    const float rs = rcp(ha.y + hb.y);
    const float wa = ha.y * rs, wb = hb.y * rs;
    const float u = wa * a.y + wb * b.y;
    const float v = wa * a.z + wb * b.z;
    const float du = a.y - b.y, dv = a.z - b.z;
    const float h = wa * ha.x + wb * hb.x;
    const float c2 = gm1 * (h + 0.5f * wa * wb * (du * du + dv * dv));
    return eig_from(u, v, c2, gm1);
}

// The same average in FP64 from the cells' FP64 conserved states (near-vacuum
// interfaces): the reference's own formulas (Characteriz.h:333-342).
EB2_HD Eig roe_f64(const double* qa, const double* qb, double gm1,
                                       double gr) {
    double ua = qa[1] / qa[0], va = qa[2] / qa[0];
    double ub = qb[1] / qb[0], vb = qb[2] / qb[0];
    double pa = (qa[3] - 0.5 * qa[0] * (ua * ua + va * va)) * gm1;
    double pb = (qb[3] - 0.5 * qb[0] * (ub * ub + vb * vb)) * gm1;
    double Ha = 0.5 * (ua * ua + va * va) + gr * (pa / qa[0]);
    double Hb = 0.5 * (ub * ub + vb * vb) + gr * (pb / qb[0]);
    double D = sqrt(qb[0] / qa[0]);
    double D1 = D + 1.0;
    double u = (ua + D * ub) / D1, v = (va + D * vb) / D1, H = (Ha + D * Hb) / D1;
    double c2 = gm1 * (H - 0.5 * (u * u + v * v));
    Eig e;
    double c = sqrt(c2);
    e.u = (float)u;
    e.v = (float)v;
    e.c = (float)c;
    e.b1 = (float)(gm1 / c2);
    e.hb1 = 0.5f * e.b1;
    e.hic = (float)(0.5 / c);
    e.hq2 = (float)(0.5 * (u * u + v * v));
    e.cg = (float)(c2 / gm1);
    e.H = (float)H;
    return e;
}

// Characteristic variables of a conserved difference d (left-eigenvector rows
// of Characteriz.h:346-367 / :448-469 in factored form).
template <int DIR>
EB2_HD void project(const Eig& e, float d0, float d1, float d2, float d3,
                                        float* w) {
    float K = fmaf(e.hq2, d0, d3);
    K = fmaf(-e.u, d1, K);
    K = fmaf(-e.v, d2, K);
    float A = DIR == 1 ? fmaf(e.u, d0, -d1) : fmaf(e.v, d0, -d2);
    float bK = e.hb1 * K, cA = e.hic * A;
    w[0] = bK + cA;
    w[3] = bK - cA;
    w[1] = fmaf(e.cg, d0, -K);
    w[2] = DIR == 1 ? fmaf(e.v, d0, -d2) : fmaf(-e.u, d0, d1);
}

// Conserved difference from characteristic values (right eigenvectors,
// Characteriz.h:371-392 / :473-494, factored).
template <int DIR>
EB2_HD void unproject(const Eig& e, const float* w, float* q) {
    float S = fmaf(e.b1, w[1], w[0] + w[3]);
    float D = w[0] - w[3];
    float cD = e.c * D;
    q[0] = S;
    if (DIR == 1) {
        q[1] = fmaf(e.u, S, -cD);
        q[2] = fmaf(e.v, S, -w[2]);
        q[3] = fmaf(e.H, S, fmaf(-e.u, cD, fmaf(-e.v, w[2], -w[1])));
    } else {
        q[1] = fmaf(e.u, S, w[2]);
        q[2] = fmaf(e.v, S, -cD);
        q[3] = fmaf(e.H, S, fmaf(-e.v, cD, fmaf(e.u, w[2], -w[1])));
    }
}

// WENO5 at both sides of an interface from the six characteristic values
// w[0..5] (cells i-2..i+3) with w[2] == 0 (delta form around cell i).
// Returns the minus-side value (WENO5_L on i-2..i+2) relative to cell i and
// the plus-side value (WENO5_R on i+3..i-1) relative to cell i+1 (minus w3),
// so that a flat upwind side returns its own cell's state exactly, as the
// FP64 form does.  WZ selects WENO-Z weights.
template <bool WZ>
EB2_HD void weno5_pair(float w0, float w1, float w3, float w4, float w5,
                                           float& qm, float& qp) {
    // a flat stencil reconstructs its base value on both sides (uniform
    // regions, where whole warps take this branch)
    if (fmaxf(fmaxf(fmaxf(fabsf(w0), fabsf(w1)), fmaxf(fabsf(w3), fabsf(w4))), fabsf(w5)) ==
        0.0f) {
        qm = qp = 0.0f;
        return;
    }
    const float k13 = 13.0f / 12.0f;
    // The reference's absolute epsilon of the smoothness indicators
    // (Reconstruction.h WENO5-JS/Z).  The weights below depend only on ratios
    // of (beta + eps), which side() brings into range itself, so the stencil
    // needs no scaling: FP32 rounding is relative, and a beta that underflows
    // is far below eps either way.
    const float eps = 1.0e-15f;
    // second differences shared by both sides
    float a1 = fmaf(-2.0f, w1, w0);          // w0 - 2 w1 + w2
    float a2 = w1 + w3;                      // w1 - 2 w2 + w3
    float a3 = fmaf(-2.0f, w3, w4);          // w2 - 2 w3 + w4
    float a4 = fmaf(-2.0f, w4, w5 + w3);     // w3 - 2 w4 + w5
    float A1 = k13 * a1 * a1, A2 = k13 * a2 * a2, A3 = k13 * a3 * a3, A4 = k13 * a4 * a4;
    float bl1 = fmaf(-4.0f, w1, w0);         // w0 - 4 w1 + 3 w2
    float bl2 = w1 - w3;                     // w1 - w3
    float bl3 = fmaf(-4.0f, w3, w4);         // 3 w2 - 4 w3 + w4
    float br1 = fmaf(-4.0f, w4, fmaf(3.0f, w3, w5));  // w5 - 4 w4 + 3 w3
    float br2 = w4;                          // w4 - w2
    float br3 = fmaf(3.0f, w3, w1);          // 3 w3 - 4 w2 + w1
    float bL1 = fmaf(0.25f * bl1, bl1, A1), bL2 = fmaf(0.25f * bl2, bl2, A2);
    float bL3 = fmaf(0.25f * bl3, bl3, A3);
    float bR1 = fmaf(0.25f * br1, br1, A4), bR2 = fmaf(0.25f * br2, br2, A3);
    float bR3 = fmaf(0.25f * br3, br3, A2);
    // candidate stencil values times 6 (Reconstruction.h:1452-1454), minus
    // 6 w2 = 0 on the left and minus 6 w3 on the right
    float cl1 = fmaf(2.0f, w0, -7.0f * w1);  // stencil i-2..i
    float c2 = fmaf(2.0f, w3, -w1);          // stencil i-1..i+1
    float c3 = fmaf(5.0f, w3, -w4);          // stencil i..i+2
    const float r1 = w1 - w3, r2 = -w3, r4 = w4 - w3, r5 = w5 - w3;
    float cr1 = fmaf(2.0f, r5, -7.0f * r4);  // stencil i+1..i+3
    float cr2 = fmaf(2.0f, r2, -r4);         // stencil i..i+2
    float cr3 = fmaf(5.0f, r2, -r1);         // stencil i-1..i+1
    auto side = [&](float b1, float b2, float b3, float k1, float k2, float k3) {
        float t1 = b1 + eps, t2 = b2 + eps, t3 = b3 + eps;
        // Weights from SFU reciprocals of t = beta + eps >= eps (so 1/t < 1e15):
        // JS d_k / t_k^2 (Reconstruction.h WENO5-JS), WENO-Z d_k (1 + tau5 / t_k)
        // (Reconstruction.h:1546-1551).  A t so large that its weight flushes to
        // zero has a negligible weight anyway; the floor on the sum only keeps a
        // stencil whose three weights all flush (|values| beyond 1e9) finite.
        const float r1 = rcp(t1), r2 = rcp(t2), r3 = rcp(t3);
        float g1, g2, g3;
        if (WZ) {
            const float tau = fabsf(b1 - b3);
            g1 = 0.1f * fmaf(tau, r1, 1.0f);
            g2 = 0.6f * fmaf(tau, r2, 1.0f);
            g3 = 0.3f * fmaf(tau, r3, 1.0f);
        } else {
            g1 = (0.1f * r1) * r1;
            g2 = (0.6f * r2) * r2;
            g3 = (0.3f * r3) * r3;
        }
        const float r = rcp(fmaxf(g1 + g2 + g3, 0x1p-126f)) * (1.0f / 6.0f);
        return fmaf(g1, k1, fmaf(g2, k2, g3 * k3)) * r;
    };
    qm = side(bL1, bL2, bL3, cl1, c2, c3);
    qp = side(bR1, bR2, bR3, cr1, cr2, cr3);
}

// WENO5 of both sides of an interface in the two lanes, from the characteristic
// differences y_n = w_n - w_i of cells n = i-2..i+3 (y2 = 0).  The plus side is
// WENO5_R on i-1..i+3, which is WENO5_L on the mirrored stencil i+3..i-1; taken
// relative to its own base cell i+1 it reads (y5-y3, y4-y3, 0, -y3, y1-y3).  So
// one evaluation of the left-biased formulas on the lane pairs
//   X0 = (y0, y5-y3), X1 = (y1, y4-y3), X3 = (y3, -y3), X4 = (y4, y1-y3)
// gives the minus-side value relative to cell i in .x and the plus-side value
// relative to cell i+1 in .y (Reconstruction.h:1408-1508 for the JS weights,
// :1519-1624 for WENO-Z).  A flat upwind side returns its own cell's state
// exactly, as the FP64 form does.
//
// The smoothness indicators are carried as t_k = 12/13 (beta_k + eps) =
// a_k^2 + 3/13 b_k^2 + 12/13 eps: the weights depend only on ratios of the
// t_k (and, for WENO-Z, of tau5 = |t1 - t3| to t_k), so the common factor
// drops out and saves one multiply per indicator.  eps is the reference's
// absolute 1e-15.  The weights are SFU reciprocals of t (t >= 1e-15, so 1/t
// stays below 1e15); the floor on their sum only keeps a stencil whose three
// weights all flush to zero (values beyond ~1e9) finite.
template <bool WZ>
EB2_HD f2 weno5_lanes(f2 X0, f2 X1, f2 X3, f2 X4) {
    const f2 m2 = f2s(-2.0f), m4 = f2s(-4.0f);
    const f2 a1 = fma2(X1, m2, X0), b1 = fma2(X1, m4, X0);   // w0-2w1+w2, w0-4w1+3w2
    const f2 a2 = add2(X1, X3), b2 = sub2(X1, X3);           // w1-2w2+w3, w1-w3
    const f2 a3 = fma2(X3, m2, X4), b3 = fma2(X3, m4, X4);   // w2-2w3+w4, 3w2-4w3+w4
    const f2 k = f2s(3.0f / 13.0f), e = f2s(12.0f / 13.0f * 1.0e-15f);
    const f2 t1 = fma2(a1, a1, fma2(mul2(k, b1), b1, e));
    const f2 t2 = fma2(a2, a2, fma2(mul2(k, b2), b2, e));
    const f2 t3 = fma2(a3, a3, fma2(mul2(k, b3), b3, e));
    // candidate values times 6 relative to the base (Reconstruction.h:1452-1454)
    const f2 c1 = fma2(X1, f2s(-7.0f), add2(X0, X0));        // 2w0 - 7w1 + 11w2
    const f2 c2 = fma2(X3, f2s(2.0f), f2n(X1));              // -w1 + 5w2 + 2w3
    const f2 c3 = fma2(X3, f2s(5.0f), f2n(X4));              // 2w2 + 5w3 - w4
    const f2 r1 = rcp2(t1), r2 = rcp2(t2), r3 = rcp2(t3);
    f2 g1, g2, g3;
    if (WZ) {
        const f2 d = sub2(t1, t3);
        const f2 tau = make_float2(fabsf(d.x), fabsf(d.y));
        g1 = fma2(mul2(tau, r1), f2s(0.1f), f2s(0.1f));
        g2 = fma2(mul2(tau, r2), f2s(0.6f), f2s(0.6f));
        g3 = fma2(mul2(tau, r3), f2s(0.3f), f2s(0.3f));
    } else {
        g1 = mul2(mul2(r1, f2s(0.1f)), r1);
        g2 = mul2(mul2(r2, f2s(0.6f)), r2);
        g3 = mul2(mul2(r3, f2s(0.3f)), r3);
    }
    const f2 s = add2(add2(g1, g2), g3);
    const f2 rs = mul2(rcp2(make_float2(fmaxf(s.x, 0x1p-126f), fmaxf(s.y, 0x1p-126f))),
                       f2s(1.0f / 6.0f));
    return mul2(fma2(g1, c1, fma2(g2, c2, mul2(g3, c3))), rs);
}

// Conserved differences of both sides from their characteristic values (the
// right eigenvectors of unproject, Characteriz.h:371-392 / :473-494), lane by
// lane.
template <int DIR>
EB2_HD void unproject2(const Eig& e, const f2* w, f2* q) {
    const f2 S = fma2(f2s(e.b1), w[1], add2(w[0], w[3]));
    const f2 cD = mul2(f2s(e.c), sub2(w[0], w[3]));
    q[0] = S;
    if (DIR == 1) {
        q[1] = fma2(f2s(e.u), S, f2n(cD));
        q[2] = fma2(f2s(e.v), S, f2n(w[2]));
        q[3] = fma2(f2s(e.H), S, fma2(f2s(-e.u), cD, fma2(f2s(-e.v), w[2], f2n(w[1]))));
    } else {
        q[1] = fma2(f2s(e.u), S, w[2]);
        q[2] = fma2(f2s(e.v), S, f2n(cD));
        q[3] = fma2(f2s(e.H), S, fma2(f2s(-e.v), cD, fma2(f2s(e.u), w[2], f2n(w[1]))));
    }
}

// Interface state in primitive form from the base cell and a conserved
// difference (no cancellation: see the file comment).
struct Prim {
    float r, un, ut, p, E, ir;
};

template <int DIR>
EB2_HD Prim prim_from_delta(float rb, float ub, float vb, float pb, float Eb,
                                                const float* dq, float gm1) {
    Prim s;
    float r = rb + dq[0];
    float ir = rcp(r);
    float u = fmaf(fmaf(-ub, dq[0], dq[1]), ir, ub);
    float v = fmaf(fmaf(-vb, dq[0], dq[2]), ir, vb);
    // dK = [rb (2 ub.dm - drho |ub|^2) + |dm|^2] / (2 r)
    float udm = fmaf(ub, dq[1], vb * dq[2]);
    float t = fmaf(rb, fmaf(2.0f, udm, -dq[0] * fmaf(ub, ub, vb * vb)),
                   fmaf(dq[1], dq[1], dq[2] * dq[2]));
    float dK = 0.5f * t * ir;
    s.r = r;
    s.ir = ir;
    s.p = fmaf(gm1, dq[3] - dK, pb);
    s.E = Eb + dq[3];
    s.un = DIR == 1 ? u : v;
    s.ut = DIR == 1 ? v : u;
    return s;
}

// prim_from_delta for both sides at once: lane .x from cell i and the
// minus-side difference, lane .y from cell i+1 and the plus-side difference.
template <int DIR>
EB2_HD void prim_from_delta2(f2 rb, f2 ub, f2 vb, f2 pb, f2 Eb, const f2* dq, float gm1,
                             Prim& L, Prim& R) {
    const f2 r = add2(rb, dq[0]);
    const f2 ir = rcp2(r);
    const f2 u = fma2(fma2(f2n(ub), dq[0], dq[1]), ir, ub);
    const f2 v = fma2(fma2(f2n(vb), dq[0], dq[2]), ir, vb);
    // dK = [rb (2 ub.dm - drho |ub|^2) + |dm|^2] / (2 r)
    const f2 udm = fma2(ub, dq[1], mul2(vb, dq[2]));
    const f2 q2 = fma2(ub, ub, mul2(vb, vb));
    const f2 t = fma2(rb, fma2(f2s(2.0f), udm, f2n(mul2(dq[0], q2))),
                      fma2(dq[1], dq[1], mul2(dq[2], dq[2])));
    const f2 dK = mul2(mul2(f2s(0.5f), t), ir);
    const f2 p = fma2(f2s(gm1), sub2(dq[3], dK), pb);
    const f2 E = add2(Eb, dq[3]);
    L.r = r.x;
    L.ir = ir.x;
    L.p = p.x;
    L.E = E.x;
    L.un = DIR == 1 ? u.x : v.x;
    L.ut = DIR == 1 ? v.x : u.x;
    R.r = r.y;
    R.ir = ir.y;
    R.p = p.y;
    R.E = E.y;
    R.un = DIR == 1 ? u.y : v.y;
    R.ut = DIR == 1 ? v.y : u.y;
}

// Physical flux in (mass, normal momentum, tangential momentum, energy) order.
EB2_HD void pflux(const Prim& s, float* F) {
    float m = s.r * s.un;
    F[0] = m;
    F[1] = fmaf(m, s.un, s.p);
    F[2] = m * s.ut;
    F[3] = (s.E + s.p) * s.un;
}

// HLLC with Einfeldt speeds (include/scheme.h:690-1001, sound speed
// sqrt(gamma p / rho) on both sweeps).
EB2_HD void hllc(const Prim& L, const Prim& R, float gamma, float* F) {
    float aL2 = gamma * L.p * L.ir, aR2 = gamma * R.p * R.ir;
    float sqL = sqr(L.r), sqR = sqr(R.r);
    float is = rcp(sqL + sqR);
    float nbar = (sqL * L.un + sqR * R.un) * is;
    float eta = 0.5f * sqL * sqR * is * is;
    float du = R.un - L.un;
    float dd2 = fmaf((sqL * aL2 + sqR * aR2), is, eta * du * du);
    float dd = sqr(dd2);
    float sl = nbar - dd, sr = nbar + dd;
    if (sl >= 0.0f) {
        pflux(L, F);
        return;
    }
    if (sr <= 0.0f) {
        pflux(R, F);
        return;
    }
    float mL = L.r * (sl - L.un), mR = R.r * (sr - R.un);
    float ss = (R.p - L.p + L.un * mL - R.un * mR) * rcp(mL - mR);
    const Prim& S = ss >= 0.0f ? L : R;
    float sk = ss >= 0.0f ? sl : sr;
    float mk = ss >= 0.0f ? mL : mR;
    float Fk[4];
    pflux(S, Fk);
    float f = mk * rcp(sk - ss);                      // star density
    float e = S.E * S.ir + (ss - S.un) * (ss + S.p * rcp(mk));
    F[0] = fmaf(sk, f - S.r, Fk[0]);
    F[1] = fmaf(sk, fmaf(f, ss, -S.r * S.un), Fk[1]);
    F[2] = fmaf(sk, fmaf(f, S.ut, -S.r * S.ut), Fk[2]);
    F[3] = fmaf(sk, fmaf(f, e, -S.E), Fk[3]);
}

// HLL with Einfeldt speeds (include/scheme.h:400-674).
EB2_HD void hll(const Prim& L, const Prim& R, float gamma, float* F) {
    float aL2 = gamma * L.p * L.ir, aR2 = gamma * R.p * R.ir;
    float sqL = sqr(L.r), sqR = sqr(R.r);
    float is = rcp(sqL + sqR);
    float nbar = (sqL * L.un + sqR * R.un) * is;
    float eta = 0.5f * sqL * sqR * is * is;
    float du = R.un - L.un;
    float dd = sqr(fmaf((sqL * aL2 + sqR * aR2), is, eta * du * du));
    float sl = nbar - dd, sr = nbar + dd;
    if (sl >= 0.0f) { pflux(L, F); return; }
    if (sr <= 0.0f) { pflux(R, F); return; }
    float FL[4], FR[4];
    pflux(L, FL);
    pflux(R, FR);
    float UL[4] = {L.r, L.r * L.un, L.r * L.ut, L.E}, UR[4] = {R.r, R.r * R.un, R.r * R.ut, R.E};
    float id = rcp(sr - sl), slsr = sl * sr;
#pragma unroll
    for (int k = 0; k < 4; k++) F[k] = (sr * FL[k] - sl * FR[k] + slsr * (UR[k] - UL[k])) * id;
}

// Roe flux with |lambda| (include/scheme.h:1018-1322), normal-aligned.
EB2_HD void roe(const Prim& L, const Prim& R, float gamma, float* F) {
    float gm1 = gamma - 1.0f;
    float sqL = sqr(L.r), sqR = sqr(R.r);
    float is = rcp(sqL + sqR);
    float wa = sqL * is, wb = sqR * is;
    float un = wa * L.un + wb * R.un, ut = wa * L.ut + wb * R.ut;
    float dun = R.un - L.un, dut = R.ut - L.ut;
    float hL = gamma / gm1 * L.p * L.ir, hR = gamma / gm1 * R.p * R.ir;
    float c2 = gm1 * (wa * hL + wb * hR + 0.5f * wa * wb * (dun * dun + dut * dut));
    float ic = rsq(c2), c = c2 * ic;
    float q2 = un * un + ut * ut;
    float H = c2 / gm1 + 0.5f * q2;
    float rbar = sqL * sqR;
    float dp = R.p - L.p, drho = R.r - L.r;
    float ic2 = ic * ic;
    float a0 = (dp - rbar * c * dun) * 0.5f * ic2;
    float a1 = drho - dp * ic2;
    float a2 = rbar * dut;
    float a3 = (dp + rbar * c * dun) * 0.5f * ic2;
    float l0 = 0.5f * fabsf(un - c) * a0, l1 = 0.5f * fabsf(un) * a1;
    float l2 = 0.5f * fabsf(un) * a2, l3 = 0.5f * fabsf(un + c) * a3;
    float FL[4], FR[4];
    pflux(L, FL);
    pflux(R, FR);
    F[0] = 0.5f * (FL[0] + FR[0]) - (l0 + l1 + l3);
    F[1] = 0.5f * (FL[1] + FR[1]) - (l0 * (un - c) + l1 * un + l3 * (un + c));
    F[2] = 0.5f * (FL[2] + FR[2]) - (l0 * ut + l1 * ut + l2 + l3 * ut);
    F[3] = 0.5f * (FL[3] + FR[3]) -
           (l0 * (H - un * c) + l1 * 0.5f * q2 + l2 * ut + l3 * (H + un * c));
}

// Local Lax-Friedrichs (include/scheme.h:229-381).
EB2_HD void llf(const Prim& L, const Prim& R, float gamma, float* F) {
    float aL = sqr(gamma * L.p * L.ir), aR = sqr(gamma * R.p * R.ir);
    float sp = fmaxf(fabsf(L.un) + aL, fabsf(R.un) + aR);
    float FL[4], FR[4];
    pflux(L, FL);
    pflux(R, FR);
    float UL[4] = {L.r, L.r * L.un, L.r * L.ut, L.E}, UR[4] = {R.r, R.r * R.un, R.r * R.ut, R.E};
#pragma unroll
    for (int k = 0; k < 4; k++) F[k] = 0.5f * (FL[k] + FR[k]) - 0.5f * sp * (UR[k] - UL[k]);
}

// --- the heat-conduction ("anti-overheating") fluxes, AR_scheme 11/22/33 ---
// The classical solvers above plus the reference's energy-flux term in the
// jump of the specific internal energy e = p / (rho (gamma - 1)); the
// algebra follows the FP64 forms (eb2_point_fp64.cuh, include/scheme.h
// :1860-2136, :2153-2471, :2793-3109) in this file's FP32 style.
EB2_HD float spec_e(const Prim& s, float igm1) { return s.p * s.ir * igm1; }

// HLLHC: HLL plus (s_L s_R / (s_R - s_L)) (e_R - e_L) rho_HLL on the energy
// flux in the subsonic branch.
EB2_HD void hllhc(const Prim& L, const Prim& R, float gamma, float* F) {
    float aL2 = gamma * L.p * L.ir, aR2 = gamma * R.p * R.ir;
    float sqL = sqr(L.r), sqR = sqr(R.r);
    float is = rcp(sqL + sqR);
    float nbar = (sqL * L.un + sqR * R.un) * is;
    float eta = 0.5f * sqL * sqR * is * is;
    float du = R.un - L.un;
    float dd = sqr(fmaf((sqL * aL2 + sqR * aR2), is, eta * du * du));
    float sl = nbar - dd, sr = nbar + dd;
    if (sl >= 0.0f) { pflux(L, F); return; }
    if (sr <= 0.0f) { pflux(R, F); return; }
    float FL[4], FR[4];
    pflux(L, FL);
    pflux(R, FR);
    float UL[4] = {L.r, L.r * L.un, L.r * L.ut, L.E}, UR[4] = {R.r, R.r * R.un, R.r * R.ut, R.E};
    float id = rcp(sr - sl), slsr = sl * sr;
#pragma unroll
    for (int k = 0; k < 4; k++) F[k] = (sr * FL[k] - sl * FR[k] + slsr * (UR[k] - UL[k])) * id;
    const float igm1 = rcp(gamma - 1.0f);
    const float rho_hll = (sr * R.r - sl * L.r + FL[0] - FR[0]) * id;
    F[3] = fmaf(slsr * id * (spec_e(R, igm1) - spec_e(L, igm1)), rho_hll, F[3]);
}

// HLLCHC: HLLC plus (s_L s_R / (s_R - s_L)) (e_R - e_L) times the star
// density on the energy flux of the star states.
EB2_HD void hllchc(const Prim& L, const Prim& R, float gamma, float* F) {
    float aL2 = gamma * L.p * L.ir, aR2 = gamma * R.p * R.ir;
    float sqL = sqr(L.r), sqR = sqr(R.r);
    float is = rcp(sqL + sqR);
    float nbar = (sqL * L.un + sqR * R.un) * is;
    float eta = 0.5f * sqL * sqR * is * is;
    float du = R.un - L.un;
    float dd = sqr(fmaf((sqL * aL2 + sqR * aR2), is, eta * du * du));
    float sl = nbar - dd, sr = nbar + dd;
    if (sl >= 0.0f) { pflux(L, F); return; }
    if (sr <= 0.0f) { pflux(R, F); return; }
    float mL = L.r * (sl - L.un), mR = R.r * (sr - R.un);
    float ss = (R.p - L.p + L.un * mL - R.un * mR) * rcp(mL - mR);
    const Prim& S = ss >= 0.0f ? L : R;
    float sk = ss >= 0.0f ? sl : sr;
    float mk = ss >= 0.0f ? mL : mR;
    float Fk[4];
    pflux(S, Fk);
    float f = mk * rcp(sk - ss);                      // star density
    float e = S.E * S.ir + (ss - S.un) * (ss + S.p * rcp(mk));
    const float igm1 = rcp(gamma - 1.0f);
    const float corr = sl * sr * rcp(sr - sl) * (spec_e(R, igm1) - spec_e(L, igm1));
    F[0] = fmaf(sk, f - S.r, Fk[0]);
    F[1] = fmaf(sk, fmaf(f, ss, -S.r * S.un), Fk[1]);
    F[2] = fmaf(sk, fmaf(f, S.ut, -S.r * S.ut), Fk[2]);
    F[3] = fmaf(corr, f, fmaf(sk, fmaf(f, e, -S.E), Fk[3]));
}

// RoeHC: Roe with 1e-12 in the 1/(2 c^2) and 1/c^2 wave-strength factors,
// minus 1/2 |u_n + c| (e_R - e_L) rho_bar on the energy flux.
EB2_HD void roehc(const Prim& L, const Prim& R, float gamma, float* F) {
    float gm1 = gamma - 1.0f;
    float sqL = sqr(L.r), sqR = sqr(R.r);
    float is = rcp(sqL + sqR);
    float wa = sqL * is, wb = sqR * is;
    float un = wa * L.un + wb * R.un, ut = wa * L.ut + wb * R.ut;
    float dun = R.un - L.un, dut = R.ut - L.ut;
    float hL = gamma / gm1 * L.p * L.ir, hR = gamma / gm1 * R.p * R.ir;
    float c2 = gm1 * (wa * hL + wb * hR + 0.5f * wa * wb * (dun * dun + dut * dut));
    float c = sqr(c2);
    float q2 = un * un + ut * ut;
    float H = c2 / gm1 + 0.5f * q2;
    float rbar = sqL * sqR;
    float dp = R.p - L.p, drho = R.r - L.r;
    float i2c2 = rcp(fmaf(2.0f, c2, 1.0e-12f)), ic2 = rcp(c2 + 1.0e-12f);
    float a0 = (dp - rbar * c * dun) * i2c2;
    float a1 = drho - dp * ic2;
    float a2 = rbar * dut;
    float a3 = (dp + rbar * c * dun) * i2c2;
    float l0 = 0.5f * fabsf(un - c) * a0, l1 = 0.5f * fabsf(un) * a1;
    float l2 = 0.5f * fabsf(un) * a2, l3 = 0.5f * fabsf(un + c) * a3;
    float FL[4], FR[4];
    pflux(L, FL);
    pflux(R, FR);
    const float igm1 = rcp(gm1);
    F[0] = 0.5f * (FL[0] + FR[0]) - (l0 + l1 + l3);
    F[1] = 0.5f * (FL[1] + FR[1]) - (l0 * (un - c) + l1 * un + l3 * (un + c));
    F[2] = 0.5f * (FL[2] + FR[2]) - (l0 * ut + l1 * ut + l2 + l3 * ut);
    F[3] = 0.5f * (FL[3] + FR[3]) -
           (l0 * (H - un * c) + l1 * 0.5f * q2 + l2 * ut + l3 * (H + un * c)) -
           0.5f * fabsf(un + c) * (spec_e(R, igm1) - spec_e(L, igm1)) * rbar;
}

}  // namespace f32
}  // namespace eb2
