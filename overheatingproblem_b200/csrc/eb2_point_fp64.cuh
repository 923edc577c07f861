// eb2_point_fp64.cuh -- per-interface FP64 arithmetic of the plain drop-in.
//
// Every expression keeps the reference's evaluation order and the translation
// units that include this header are compiled with -fmad=false, so each
// function returns the same bits as the reference's C code built with gcc -O3
// (which contracts nothing into FMAs on x86-64 without -march).  Reference
// locations are cited per function.
#pragma once

#include <cstring>

#include "eb2_common.cuh"
#include "eb2_fdiv.cuh"

namespace eb2 {
namespace x64 {

// Roe-averaged quantities at an interface between cells a and b
// (include/Characteriz.h:333-342 and :435-444).
struct Roe {
    double u, v, H, c, q2, b1, b2, ic, uc, vc;  // ic = 1/c, uc = u/c, vc = v/c
};

// a = (rho, u, v, p, H) of the left cell, b of the right cell.
EB2_HD Roe roe_average(const double* a, const double* b, double gm1) {
    Roe r;
    double D = sqrt(b[0] / a[0]);
    double D1 = D + 1.0;
    r.u = (a[1] + D * b[1]) / D1;
    r.v = (a[2] + D * b[2]) / D1;
    r.H = (a[4] + D * b[4]) / D1;
    r.q2 = r.u * r.u + r.v * r.v;
    double c2 = gm1 * (r.H - 0.5 * r.q2);
    r.c = sqrt(c2);
    r.b1 = gm1 / c2;
    r.b2 = 1.0 + r.b1 * r.q2 - r.b1 * r.H;
    r.ic = 1.0 / r.c;
    r.uc = r.u / r.c;
    r.vc = r.v / r.c;
    return r;
}

// roe_average through the branch-free divisions and square roots
// (eb2_fdiv.cuh): the same bits, with the operands recorded in gd.  Densities and
// c^2 are divisors ([2^-60, 2^400)), D + 1 and c small divisors (below 2^60);
// D + 1 is near 2 - 2^-52 whenever the densities nearly agree, so its
// reciprocal is taken with the all-ones case included.  The velocities are
// often tiny or subnormal ahead of fronts and take div_rn_tiny.  b[0] / a[0]
// and c^2 are in the range of sqrt_rn.
EB2_HD Roe roe_average_rn(const double* a, const double* b, double gm1, DivGuard& gd) {
#if defined(__CUDA_ARCH__)
    Roe r;
    gd.divisor(a[0]);
    gd.divisor(b[0]);
    gd.reciprocal(a[0]);
    double D = sqrt_rn(div_rn(b[0], a[0], rcp_rn(a[0])));
    double D1 = D + 1.0;
    gd.small_divisor(D1);
    const double yD = rcp_rn_any(D1);
    const double nu = a[1] + D * b[1], nv = a[2] + D * b[2], nH = a[4] + D * b[4];
    gd.finite(nu);
    gd.finite(nv);
    gd.dividend(nH);
    r.u = div_rn_tiny(nu, D1, yD);
    r.v = div_rn_tiny(nv, D1, yD);
    r.H = copysign(div_rn(nH, D1, yD), nH);
    r.q2 = r.u * r.u + r.v * r.v;
    double c2 = gm1 * (r.H - 0.5 * r.q2);
    gd.divisor(c2);
    gd.reciprocal(c2);
    r.c = sqrt_rn(c2);
    r.b1 = div_rn(gm1, c2, rcp_rn(c2));
    r.b2 = 1.0 + r.b1 * r.q2 - r.b1 * r.H;
    gd.small_divisor(r.c);
    gd.reciprocal(r.c);
    r.ic = rcp_rn(r.c);
    r.uc = div_rn_tiny(r.u, r.c, r.ic);
    r.vc = div_rn_tiny(r.v, r.c, r.ic);
    return r;
#else
    (void)gd;
    return roe_average(a, b, gm1);
#endif
}

// Row k of the left-eigenvector matrix (eigen_l[k][*], Characteriz.h:346-367
// for x, :448-469 for y).
template <int DIR>
EB2_HD void left_row(const Roe& e, int k, double* l) {
    if (DIR == 1) {
        switch (k) {
            case 0: l[0] = 0.5 * (e.b2 + e.uc); l[1] = -0.5 * (e.b1 * e.u + e.ic);
                    l[2] = -0.5 * e.b1 * e.v; l[3] = 0.5 * e.b1; break;
            case 1: l[0] = -e.q2 + e.H; l[1] = e.u; l[2] = e.v; l[3] = -1.0; break;
            case 2: l[0] = e.v; l[1] = 0.0; l[2] = -1.0; l[3] = 0.0; break;
            default: l[0] = 0.5 * (e.b2 - e.uc); l[1] = 0.5 * (-e.b1 * e.u + e.ic);
                     l[2] = 0.5 * -e.b1 * e.v; l[3] = 0.5 * e.b1; break;
        }
    } else {
        switch (k) {
            case 0: l[0] = 0.5 * (e.b2 + e.vc); l[1] = -0.5 * (e.b1 * e.u + 0.0 / e.c);
                    l[2] = -0.5 * (e.b1 * e.v + e.ic); l[3] = 0.5 * e.b1; break;
            case 1: l[0] = -e.q2 + e.H; l[1] = e.u; l[2] = e.v; l[3] = -1.0; break;
            case 2: l[0] = -e.u; l[1] = 1.0; l[2] = -0.0; l[3] = 0.0; break;
            default: l[0] = 0.5 * (e.b2 - e.vc); l[1] = 0.5 * (-e.b1 * e.u + 0.0 / e.c);
                     l[2] = 0.5 * (-e.b1 * e.v + e.ic); l[3] = 0.5 * e.b1; break;
        }
    }
}

// Row m of the right-eigenvector matrix, R[m][k] = eigen_r[m][k]
// (Characteriz.h:371-392 for x, :473-494 for y).
template <int DIR>
EB2_HD void right_row(const Roe& e, int m, double* r) {
    if (DIR == 1) {
        switch (m) {
            case 0: r[0] = 1.0; r[1] = e.b1; r[2] = 0.0; r[3] = 1.0; break;
            case 1: r[0] = e.u - 1.0 * e.c; r[1] = e.u * e.b1; r[2] = 0.0; r[3] = e.u + 1.0 * e.c; break;
            case 2: r[0] = e.v - 0.0 * e.c; r[1] = e.v * e.b1; r[2] = -1.0; r[3] = e.v + 0.0 * e.c; break;
            default: r[0] = e.H - e.u * e.c; r[1] = e.H * e.b1 - 1.0; r[2] = -e.v; r[3] = e.H + e.u * e.c; break;
        }
    } else {
        switch (m) {
            case 0: r[0] = 1.0; r[1] = e.b1; r[2] = 0.0; r[3] = 1.0; break;
            case 1: r[0] = e.u - 0.0 * e.c; r[1] = e.u * e.b1; r[2] = 1.0; r[3] = e.u + 0.0 * e.c; break;
            case 2: r[0] = e.v - 1.0 * e.c; r[1] = e.v * e.b1; r[2] = -0.0; r[3] = e.v + 1.0 * e.c; break;
            default: r[0] = e.H - e.v * e.c; r[1] = e.H * e.b1 - 1.0; r[2] = e.u; r[3] = e.H + e.v * e.c; break;
        }
    }
}

// Jiang-Shu smoothness indicators (include/Reconstruction.h:1425-1432).
EB2_HD void smooth3(double v1, double v2, double v3, double v4, double v5,
                                        double& s1, double& s2, double& s3) {
    s1 = 13.0 / 12.0 * (v1 - 2.0 * v2 + v3) * (v1 - 2.0 * v2 + v3)
       + 0.25 * (v1 - 4.0 * v2 + 3.0 * v3) * (v1 - 4.0 * v2 + 3.0 * v3);
    s2 = 13.0 / 12.0 * (v2 - 2.0 * v3 + v4) * (v2 - 2.0 * v3 + v4)
       + 0.25 * (v2 - v4) * (v2 - v4);
    s3 = 13.0 / 12.0 * (v3 - 2.0 * v4 + v5) * (v3 - 2.0 * v4 + v5)
       + 0.25 * (3.0 * v3 - 4.0 * v4 + v5) * (3.0 * v3 - 4.0 * v4 + v5);
}

// Nonlinear blend of the three candidate stencils (Reconstruction.h:1440-1454).
EB2_HD double blend3(double a1, double a2, double a3, double v1, double v2,
                                         double v3, double v4, double v5) {
    double w1 = a1 / (a1 + a2 + a3);
    double w2 = a2 / (a1 + a2 + a3);
    double w3 = a3 / (a1 + a2 + a3);
    return w1 * (2.0 * v1 - 7.0 * v2 + 11.0 * v3) / 6.0
         + w2 * (-v2 + 5.0 * v3 + 2.0 * v4) / 6.0
         + w3 * (2.0 * v3 + 5.0 * v4 - v5) / 6.0;
}

// WENO5_L with Jiang-Shu weights (Reconstruction.h:1408-1455); WENO5_R is the
// same function on the mirrored stencil.
EB2_HD double weno5_js(double v1, double v2, double v3, double v4, double v5) {
    const double eps = 1.0e-15;
    double s1, s2, s3;
    smooth3(v1, v2, v3, v4, v5, s1, s2, s3);
    double a1 = 0.1 / (eps + s1) / (eps + s1);
    double a2 = 0.6 / (eps + s2) / (eps + s2);
    double a3 = 0.3 / (eps + s3) / (eps + s3);
    return blend3(a1, a2, a3, v1, v2, v3, v4, v5);
}

// WENO5Z_L / WENO5Z_R (Reconstruction.h:1519-1624).
EB2_HD double weno5_z(double v1, double v2, double v3, double v4, double v5) {
    const double eps = 1.0e-15;
    double s1, s2, s3;
    smooth3(v1, v2, v3, v4, v5, s1, s2, s3);
    double tau = fabs(s1 - s3);
    double a1 = 0.1 * (1.0 + tau / (s1 + eps));
    double a2 = 0.6 * (1.0 + tau / (s2 + eps));
    double a3 = 0.3 * (1.0 + tau / (s3 + eps));
    return blend3(a1, a2, a3, v1, v2, v3, v4, v5);
}

EB2_HD int sgn(double x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

// TVD_minmod_* / TVD_vanleer_* (Reconstruction.h:1088-1201) with the limiters
// min_mod and van_leer of include/function.h:66-74.  side +1 returns the value
// at the right face of cell c, side -1 at its left face.
template <bool VANLEER>
EB2_HD double muscl(double lo, double c, double hi, double delta, int side) {
    double s1 = (c - lo) / delta;
    double s2 = (hi - c) / delta;
    double s;
    if (VANLEER) {
        double tiny = 1.0e-6;
        s = ((sgn(s1) + sgn(s2)) * s1 * s2) / (fabs(s1) + fabs(s2) + tiny);
    } else {
        double a = fabs(s1), b = fabs(s2);
        s = 0.5 * (sgn(s1) + sgn(s2)) * (a > b ? b : a);
    }
    return side > 0 ? c + 0.5 * s * delta : c - 0.5 * s * delta;
}

// WENO3_L / WENO3_R (include/Reconstruction.h:1326-1400): two-point
// smoothness, weights 1/3 and 2/3 over (1e-6 + beta)^2 (pow(x,2) is x*x in the
// reference's build).  WENO3_L takes v1..v3 = cells i-1, i, i+1; WENO3_R the
// mirror i+2, i+1, i.
EB2_HD double weno3(double v1, double v2, double v3) {
    const double eps = 1e-6;
    double s1 = (v2 - v1) * (v2 - v1);
    double s2 = (v3 - v2) * (v3 - v2);
    double a1 = (1.0 / 3.0) / ((eps + s1) * (eps + s1));
    double a2 = (2.0 / 3.0) / ((eps + s2) * (eps + s2));
    double w1 = a1 / (a1 + a2);
    double w2 = a2 / (a1 + a2);
    return w1 * (-0.5 * v1 + 1.5 * v2) + w2 * (0.5 * v2 + 0.5 * v3);
}

// Interface pair (minus side, plus side) from six values q[0..5] = cells
// i-2..i+3 of one field; RECON 5 = WENO5, 3 = WENO3, 2 = TVD, 1 = first order.
template <int RECON, bool WZ, bool VANLEER>
EB2_HD void recon_pair(const double* q, double delta, double& qm, double& qp) {
    if (RECON == 5) {
        if (WZ) {
            qm = weno5_z(q[0], q[1], q[2], q[3], q[4]);
            qp = weno5_z(q[5], q[4], q[3], q[2], q[1]);
        } else {
            qm = weno5_js(q[0], q[1], q[2], q[3], q[4]);
            qp = weno5_js(q[5], q[4], q[3], q[2], q[1]);
        }
    } else if (RECON == 3) {
        qm = weno3(q[1], q[2], q[3]);
        qp = weno3(q[4], q[3], q[2]);
    } else if (RECON == 2) {
        qm = muscl<VANLEER>(q[1], q[2], q[3], delta, +1);
        qp = muscl<VANLEER>(q[2], q[3], q[4], delta, -1);
    } else {
        qm = q[2];
        qp = q[3];
    }
}

// --- WENO weights with branch-free correctly rounded divisions ---
// Same expressions, same order and the same bits as weno5_js, weno5_z and
// weno3 above; each `/` becomes rcp_rn + div_rn (eb2_fdiv.cuh), sharing the
// reciprocal where the reference divides twice by one value.  The operands
// are recorded in a DivGuard; when it reports one outside the range in which
// those divisions are exact, the caller recomputes with `/`.  On the host
// these are the plain functions.
#if defined(__CUDA_ARCH__)
// (w1 c1) / 6 + (w2 c2) / 6 + (w3 c3) / 6 with w_k = a_k / (a1 + a2 + a3).
// The callers' ranges give a_k > 2^-810 and a1 + a2 + a3 < 2^562, so the
// weights are normal; the products w_k c_k only need to be finite.
__device__ __forceinline__ double blend3_rn(double a1, double a2, double a3, double v1,
                                            double v2, double v3, double v4, double v5,
                                            DivGuard& gd) {
    const double S = a1 + a2 + a3, yS = rcp_rn(S);
    gd.reciprocal(S);
    const double w1 = div_rn(a1, S, yS), w2 = div_rn(a2, S, yS), w3 = div_rn(a3, S, yS);
    const double x1 = w1 * (2.0 * v1 - 7.0 * v2 + 11.0 * v3);
    const double x2 = w2 * (-v2 + 5.0 * v3 + 2.0 * v4);
    const double x3 = w3 * (2.0 * v3 + 5.0 * v4 - v5);
    gd.finite(x1);
    gd.finite(x2);
    gd.finite(x3);
    return div6_rn(x1) + div6_rn(x2) + div6_rn(x3);
}
#endif

// With eps + s_k in [1e-15, 2^400) (recorded divisors) the quotients
// 0.1 / t / t stay in [2^-810, 2^117].
EB2_HD double weno5_js_rn(double v1, double v2, double v3, double v4, double v5,
                          DivGuard& gd) {
#if defined(__CUDA_ARCH__)
    const double eps = 1.0e-15;
    double s1, s2, s3;
    smooth3(v1, v2, v3, v4, v5, s1, s2, s3);
    const double t1 = eps + s1, t2 = eps + s2, t3 = eps + s3;
    gd.divisor(t1);
    gd.divisor(t2);
    gd.divisor(t3);
    gd.reciprocal(t1);
    gd.reciprocal(t2);
    gd.reciprocal(t3);
    const double y1 = rcp_rn(t1), y2 = rcp_rn(t2), y3 = rcp_rn(t3);
    const double a1 = div_rn(div_rn(0.1, t1, y1), t1, y1);
    const double a2 = div_rn(div_rn(0.6, t2, y2), t2, y2);
    const double a3 = div_rn(div_rn(0.3, t3, y3), t3, y3);
    return blend3_rn(a1, a2, a3, v1, v2, v3, v4, v5, gd);
#else
    return weno5_js(v1, v2, v3, v4, v5);
#endif
}

// s_k + eps in [1e-15, 2^400) and tau = |s1 - s3| zero or in [2^-500, 2^500):
// tau / t in [2^-900, 2^560), a_k in [0.1, 2^560).
EB2_HD double weno5_z_rn(double v1, double v2, double v3, double v4, double v5, DivGuard& gd) {
#if defined(__CUDA_ARCH__)
    const double eps = 1.0e-15;
    double s1, s2, s3;
    smooth3(v1, v2, v3, v4, v5, s1, s2, s3);
    const double tau = fabs(s1 - s3);
    const double t1 = s1 + eps, t2 = s2 + eps, t3 = s3 + eps;
    gd.divisor(t1);
    gd.divisor(t2);
    gd.divisor(t3);
    gd.reciprocal(t1);
    gd.reciprocal(t2);
    gd.reciprocal(t3);
    const unsigned ht = __double2hiint(tau);
    gd.fine &= tau == 0.0 || ht - (523u << 20) < (1000u << 20);
    const double a1 = 0.1 * (1.0 + div_rn(tau, t1, rcp_rn(t1)));
    const double a2 = 0.6 * (1.0 + div_rn(tau, t2, rcp_rn(t2)));
    const double a3 = 0.3 * (1.0 + div_rn(tau, t3, rcp_rn(t3)));
    return blend3_rn(a1, a2, a3, v1, v2, v3, v4, v5, gd);
#else
    return weno5_z(v1, v2, v3, v4, v5);
#endif
}

// (eps + s_k)^2 in [1e-12, 2^400): a_k in [2^-402, 2^40], weights normal.
EB2_HD double weno3_rn(double v1, double v2, double v3, DivGuard& gd) {
#if defined(__CUDA_ARCH__)
    const double eps = 1e-6;
    const double s1 = (v2 - v1) * (v2 - v1);
    const double s2 = (v3 - v2) * (v3 - v2);
    const double d1 = (eps + s1) * (eps + s1), d2 = (eps + s2) * (eps + s2);
    gd.divisor(d1);
    gd.divisor(d2);
    gd.reciprocal(d1);
    gd.reciprocal(d2);
    const double a1 = div_rn(1.0 / 3.0, d1, rcp_rn(d1));
    const double a2 = div_rn(2.0 / 3.0, d2, rcp_rn(d2));
    const double S = a1 + a2, yS = rcp_rn(S);
    gd.reciprocal(S);
    const double w1 = div_rn(a1, S, yS), w2 = div_rn(a2, S, yS);
    return w1 * (-0.5 * v1 + 1.5 * v2) + w2 * (0.5 * v2 + 0.5 * v3);
#else
    return weno3(v1, v2, v3);
#endif
}

// q[n0..n1) all have the bits of q[2] (integer compares, off the FP64 pipe).
EB2_HD bool same_bits(const double* q, int n0, int n1) {
#if defined(__CUDA_ARCH__)
    const unsigned h = __double2hiint(q[2]), l = __double2loint(q[2]);
    unsigned d = 0u;
    for (int n = n0; n < n1; n++)
        d |= (__double2hiint(q[n]) ^ h) | (__double2loint(q[n]) ^ l);
    return d == 0u;
#else
    for (int n = n0; n < n1; n++)
        if (memcmp(&q[n], &q[2], sizeof(double)) != 0) return false;
    return true;
#endif
}

// recon_pair for RECON 5 and 3 through the routines above; the caller checks
// gd.ok() and recomputes with recon_pair when it fails.  Where the stencil
// values all have the same bits (uniform regions), both sides are the same
// function of the same operands, weno(v, v, v, v, v) or weno3(v, v, v), so the
// plus side takes the minus side's bits instead of a second evaluation.
template <int RECON, bool WZ>
EB2_HD void recon_pair_rn(const double* q, double& qm, double& qp, DivGuard& gd) {
    static_assert(RECON == 5 || RECON == 3, "WENO only");
    if (RECON == 5) {
        if (WZ) {
            qm = weno5_z_rn(q[0], q[1], q[2], q[3], q[4], gd);
            if (same_bits(q, 0, 6)) qp = qm;
            else qp = weno5_z_rn(q[5], q[4], q[3], q[2], q[1], gd);
        } else {
            qm = weno5_js_rn(q[0], q[1], q[2], q[3], q[4], gd);
            if (same_bits(q, 0, 6)) qp = qm;
            else qp = weno5_js_rn(q[5], q[4], q[3], q[2], q[1], gd);
        }
    } else {
        qm = weno3_rn(q[1], q[2], q[3], gd);
        if (same_bits(q, 1, 5)) qp = qm;
        else qp = weno3_rn(q[4], q[3], q[2], gd);
    }
}

// Left/right states unpacked as the flux routines of include/scheme.h do.
struct Side {
    double r, ru, rv, re, ir, u, v, uu, vv, p;
};

EB2_HD Side unpack(const double* q, double gm1) {
    Side s;
    s.r = q[0]; s.ru = q[1]; s.rv = q[2]; s.re = q[3];
    s.ir = 1.0 / s.r;
    s.u = s.ru * s.ir;
    s.v = s.rv * s.ir;
    s.uu = s.u * s.u;
    s.vv = s.v * s.v;
    s.p = (s.re - 0.5 * s.r * (s.uu + s.vv)) * gm1;
    return s;
}

// Physical flux along DIR with total enthalpy H.
template <int DIR>
EB2_HD void phys_flux(const Side& s, double H, double* F) {
    if (DIR == 1) {
        F[0] = s.r * s.u;
        F[1] = s.r * s.uu + s.p;
        F[2] = s.r * s.v * s.u;
        F[3] = s.r * H * s.u;
    } else {
        F[0] = s.r * s.v;
        F[1] = s.r * s.u * s.v;
        F[2] = s.r * s.vv + s.p;
        F[3] = s.r * H * s.v;
    }
}

// HLLC_Flux (include/scheme.h:690-1001).  The x sweep takes the sound speed
// from the enthalpy (:745-746), the y sweep from gamma*p/rho (:895-896).
template <int DIR>
EB2_HD void flux_hllc(const double* ql, const double* qr, const Gas& g,
                                          double* F) {
    Side L = unpack(ql, g.gm1), R = unpack(qr, g.gm1);
    double HL, HR, aL, aR;
    if (DIR == 1) {
        HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
        HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
        aL = sqrt((g.gamma - 1.0) * (HL - 0.5 * (L.uu + L.vv)));
        aR = sqrt((g.gamma - 1.0) * (HR - 0.5 * (R.uu + R.vv)));
    } else {
        aL = sqrt(g.gamma * L.p * L.ir);
        aR = sqrt(g.gamma * R.p * R.ir);
        HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
        HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    }
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double unL = DIR == 1 ? L.u : L.v, unR = DIR == 1 ? R.u : R.v;
    double sqL = sqrt(L.r), sqR = sqrt(R.r);
    double ssum = sqL + sqR;
    double isum = 1.0 / ssum;
    double ubar = (sqL * L.u + sqR * R.u) * isum;
    double vbar = (sqL * L.v + sqR * R.v) * isum;
    double eta = DIR == 1 ? 0.5 * sqL * sqR * isum * isum : 0.5 * sqL * sqR / (ssum * ssum);
    double dun = unR - unL;
    double dd = sqrt((sqL * aL * aL + sqR * aR * aR) * isum + eta * dun * dun);
    double nbar = DIR == 1 ? ubar : vbar;
    double sl = nbar - dd, sr = nbar + dd;
    if (sl >= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FL[k];
        return;
    }
    if (sr <= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FR[k];
        return;
    }
    double denom = L.r * (sl - unL) - R.r * (sr - unR);
    double ss = (R.p - L.p + L.r * unL * (sl - unL) - R.r * unR * (sr - unR)) / denom;
    if (ss >= 0.0) {
        double m = L.r * (sl - unL) / (sl - ss);
        double e = L.re * L.ir + (ss - unL) * (ss + L.p / (L.r * (sl - unL)));
        F[0] = FL[0] + sl * (m - L.r);
        if (DIR == 1) {
            F[1] = FL[1] + sl * (m * ss - L.ru);
            F[2] = FL[2] + sl * (m * L.v - L.rv);
        } else {
            F[1] = FL[1] + sl * (m * L.u - L.ru);
            F[2] = FL[2] + sl * (m * ss - L.rv);
        }
        F[3] = FL[3] + sl * (m * e - L.re);
    } else {
        double m = R.r * (sr - unR) / (sr - ss);
        double e = R.re * R.ir + (ss - unR) * (ss + R.p / (R.r * (sr - unR)));
        F[0] = FR[0] + sr * (m - R.r);
        if (DIR == 1) {
            F[1] = FR[1] + sr * (m * ss - R.ru);
            F[2] = FR[2] + sr * (m * R.v - R.rv);
        } else {
            F[1] = FR[1] + sr * (m * R.u - R.ru);
            F[2] = FR[2] + sr * (m * ss - R.rv);
        }
        F[3] = FR[3] + sr * (m * e - R.re);
    }
}

// unpack and flux_hllc through the branch-free divisions and square roots
// (eb2_fdiv.cuh): the same expressions and bits, the operands recorded in gd.
// Densities and the squared sound speeds are divisors ([2^-60, 2^400)); the
// three HLLC denominators (star-speed denominator, s_L - s_*, rho_L (s_L -
// u_L)) are O(rho c) and recorded as small divisors; their dividends can be
// tiny ahead of fronts and take div_rn_tiny.
EB2_HD Side unpack_rn(const double* q, double gm1, DivGuard& gd) {
#if defined(__CUDA_ARCH__)
    Side s;
    s.r = q[0]; s.ru = q[1]; s.rv = q[2]; s.re = q[3];
    gd.divisor(s.r);
    s.ir = rcp_rn_any(s.r);
    s.u = s.ru * s.ir;
    s.v = s.rv * s.ir;
    s.uu = s.u * s.u;
    s.vv = s.v * s.v;
    s.p = (s.re - 0.5 * s.r * (s.uu + s.vv)) * gm1;
    return s;
#else
    (void)gd;
    return unpack(q, gm1);
#endif
}

template <int DIR>
EB2_HD void flux_hllc_rn(const double* ql, const double* qr, const Gas& g, double* F,
                         DivGuard& gd) {
#if defined(__CUDA_ARCH__)
    Side L = unpack_rn(ql, g.gm1, gd), R = unpack_rn(qr, g.gm1, gd);
    double HL, HR, aL, aR;
    if (DIR == 1) {
        HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
        HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
        const double cL = (g.gamma - 1.0) * (HL - 0.5 * (L.uu + L.vv));
        const double cR = (g.gamma - 1.0) * (HR - 0.5 * (R.uu + R.vv));
        gd.divisor(cL);
        gd.divisor(cR);
        aL = sqrt_rn(cL);
        aR = sqrt_rn(cR);
    } else {
        const double cL = g.gamma * L.p * L.ir, cR = g.gamma * R.p * R.ir;
        gd.divisor(cL);
        gd.divisor(cR);
        aL = sqrt_rn(cL);
        aR = sqrt_rn(cR);
        HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
        HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    }
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double unL = DIR == 1 ? L.u : L.v, unR = DIR == 1 ? R.u : R.v;
    double sqL = sqrt_rn(L.r), sqR = sqrt_rn(R.r);
    double ssum = sqL + sqR;
    double isum = rcp_rn_any(ssum);
    double ubar = (sqL * L.u + sqR * R.u) * isum;
    double vbar = (sqL * L.v + sqR * R.v) * isum;
    double eta;
    if (DIR == 1) {
        eta = 0.5 * sqL * sqR * isum * isum;
    } else {
        const double s2 = ssum * ssum;
        eta = div_rn(0.5 * sqL * sqR, s2, rcp_rn_any(s2));
    }
    double dun = unR - unL;
    const double dd2 = (sqL * aL * aL + sqR * aR * aR) * isum + eta * dun * dun;
    gd.divisor(dd2);
    double dd = sqrt_rn(dd2);
    double nbar = DIR == 1 ? ubar : vbar;
    double sl = nbar - dd, sr = nbar + dd;
    if (sl >= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FL[k];
        return;
    }
    if (sr <= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FR[k];
        return;
    }
    double denom = L.r * (sl - unL) - R.r * (sr - unR);
    const double snum = R.p - L.p + L.r * unL * (sl - unL) - R.r * unR * (sr - unR);
    gd.small_divisor(denom);
    gd.finite(snum);
    double ss = div_rn_tiny(snum, denom, rcp_rn_any(denom));
    if (ss >= 0.0) {
        const double mn = L.r * (sl - unL), md = sl - ss, pd = L.r * (sl - unL);
        gd.small_divisor(md);
        gd.small_divisor(pd);
        gd.finite(mn);
        gd.finite(L.p);
        double m = div_rn_tiny(mn, md, rcp_rn_any(md));
        double e = L.re * L.ir + (ss - unL) * (ss + div_rn_tiny(L.p, pd, rcp_rn_any(pd)));
        F[0] = FL[0] + sl * (m - L.r);
        if (DIR == 1) {
            F[1] = FL[1] + sl * (m * ss - L.ru);
            F[2] = FL[2] + sl * (m * L.v - L.rv);
        } else {
            F[1] = FL[1] + sl * (m * L.u - L.ru);
            F[2] = FL[2] + sl * (m * ss - L.rv);
        }
        F[3] = FL[3] + sl * (m * e - L.re);
    } else {
        const double mn = R.r * (sr - unR), md = sr - ss, pd = R.r * (sr - unR);
        gd.small_divisor(md);
        gd.small_divisor(pd);
        gd.finite(mn);
        gd.finite(R.p);
        double m = div_rn_tiny(mn, md, rcp_rn_any(md));
        double e = R.re * R.ir + (ss - unR) * (ss + div_rn_tiny(R.p, pd, rcp_rn_any(pd)));
        F[0] = FR[0] + sr * (m - R.r);
        if (DIR == 1) {
            F[1] = FR[1] + sr * (m * ss - R.ru);
            F[2] = FR[2] + sr * (m * R.v - R.rv);
        } else {
            F[1] = FR[1] + sr * (m * R.u - R.ru);
            F[2] = FR[2] + sr * (m * ss - R.rv);
        }
        F[3] = FR[3] + sr * (m * e - R.re);
    }
#else
    (void)gd;
    flux_hllc<DIR>(ql, qr, g, F);
#endif
}

// HLL_Flux (include/scheme.h:400-674).  Returns false where the reference
// skips the interface (`continue` on rho<=0, NaN rho, or NaN wave speed,
// :427-436 and :500-503) and leaves its flux entry untouched.
template <int DIR>
EB2_HD bool flux_hll(const double* ql, const double* qr, const Gas& g,
                                         double* F) {
    if (ql[0] <= 0.0 || qr[0] <= 0.0) return false;
    if (isnan(ql[0]) || isnan(qr[0])) return false;
    Side L = unpack(ql, g.gamma - 1.0), R = unpack(qr, g.gamma - 1.0);
    double HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
    double HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    double aL = sqrt((g.gamma - 1.0) * (HL - 0.5 * (L.uu + L.vv)));
    double aR = sqrt((g.gamma - 1.0) * (HR - 0.5 * (R.uu + R.vv)));
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double sqL = sqrt(L.r), sqR = sqrt(R.r);
    double ssum = sqL + sqR;
    double isum = 1.0 / ssum;
    double ubar = (sqL * L.u + sqR * R.u) * isum;
    double vbar = (sqL * L.v + sqR * R.v) * isum;
    double eta = 0.5 * sqL * sqR / (ssum * ssum);
    double dun = DIR == 1 ? R.u - L.u : R.v - L.v;
    double dd = sqrt((sqL * aL * aL + sqR * aR * aR) * isum + eta * dun * dun);
    if (isnan(dd)) return false;
    double nbar = DIR == 1 ? ubar : vbar;
    double sl = nbar - dd, sr = nbar + dd;
    if (sl >= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FL[k];
    } else if (sr <= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FR[k];
    } else {
        double idiff = 1.0 / (sr - sl);
        double slsr = sl * sr;
        const double UL[4] = {L.r, L.ru, L.rv, L.re}, UR[4] = {R.r, R.ru, R.rv, R.re};
        for (int k = 0; k < 4; k++)
            F[k] = (sr * FL[k] - sl * FR[k] + slsr * (UR[k] - UL[k])) * idiff;
    }
    return true;
}

// Roe_Flux (include/scheme.h:1018-1322); its entropy fix is a no-op
// (:1117-1126), so |lambda| is used directly.
template <int DIR>
EB2_HD void flux_roe(const double* ql, const double* qr, const Gas& g,
                                         double* F) {
    Side L = unpack(ql, g.gm1), R = unpack(qr, g.gm1);
    double HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
    double HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double sqL = sqrt(L.r), sqR = sqrt(R.r);
    double isum = 1.0 / (sqL + sqR);
    double rbar = sqL * sqR;
    double ubar = (sqL * L.u + sqR * R.u) * isum;
    double vbar = (sqL * L.v + sqR * R.v) * isum;
    double Hbar = (sqL * HL + sqR * HR) * isum;
    double q2 = ubar * ubar + vbar * vbar;
    double cbar = sqrt(g.gm1 * (Hbar - 0.5 * q2));
    double nbar = DIR == 1 ? ubar : vbar;
    double lam[4] = {fabs(nbar - cbar), fabs(nbar), fabs(nbar), fabs(nbar + cbar)};
    double drho = R.r - L.r, du = R.u - L.u, dv = R.v - L.v, dp = R.p - L.p;
    double c2 = cbar * cbar;
    double i2c2 = 1.0 / (2.0 * c2);
    double ic2 = 1.0 / c2;
    double dn = DIR == 1 ? du : dv, dtn = DIR == 1 ? dv : du;
    double al[4];
    al[0] = (dp - rbar * cbar * dn) * i2c2;
    al[1] = drho - dp * ic2;
    al[2] = rbar * dtn;
    al[3] = (dp + rbar * cbar * dn) * i2c2;
    double K[4][4];
    if (DIR == 1) {
        K[0][0] = 1.0; K[0][1] = ubar - cbar; K[0][2] = vbar; K[0][3] = Hbar - ubar * cbar;
        K[1][0] = 1.0; K[1][1] = ubar;        K[1][2] = vbar; K[1][3] = 0.5 * q2;
        K[2][0] = 0.0; K[2][1] = 0.0;         K[2][2] = 1.0;  K[2][3] = vbar;
        K[3][0] = 1.0; K[3][1] = ubar + cbar; K[3][2] = vbar; K[3][3] = Hbar + ubar * cbar;
    } else {
        K[0][0] = 1.0; K[0][1] = ubar; K[0][2] = vbar - cbar; K[0][3] = Hbar - vbar * cbar;
        K[1][0] = 1.0; K[1][1] = ubar; K[1][2] = vbar;        K[1][3] = 0.5 * q2;
        K[2][0] = 0.0; K[2][1] = 1.0;  K[2][2] = 0.0;         K[2][3] = ubar;
        K[3][0] = 1.0; K[3][1] = ubar; K[3][2] = vbar + cbar; K[3][3] = Hbar + vbar * cbar;
    }
    for (int c = 0; c < 4; c++) F[c] = 0.5 * (FL[c] + FR[c]);
#pragma unroll
    for (int w = 0; w < 4; w++) {
        double term = 0.5 * lam[w] * al[w];
#pragma unroll
        for (int c = 0; c < 4; c++) F[c] -= term * K[w][c];
    }
}

// LLF_Flux (include/scheme.h:229-381), the dispatch default.
template <int DIR>
EB2_HD void flux_llf(const double* ql, const double* qr, const Gas& g,
                                         double* F) {
    Side L = unpack(ql, g.gm1), R = unpack(qr, g.gm1);
    double aL = sqrt(g.gamma * L.p * L.ir), aR = sqrt(g.gamma * R.p * R.ir);
    double HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
    double HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double unL = DIR == 1 ? L.u : L.v, unR = DIR == 1 ? R.u : R.v;
    double a = fabs(unL) + aL, b = fabs(unR) + aR;
    double sp = a > b ? a : b;
    const double UL[4] = {L.r, L.ru, L.rv, L.re}, UR[4] = {R.r, R.ru, R.rv, R.re};
#pragma unroll
    for (int k = 0; k < 4; k++) F[k] = 0.5 * (FL[k] + FR[k]) - 0.5 * sp * (UR[k] - UL[k]);
}

// --- the heat-conduction ("anti-overheating") fluxes, AR_scheme 11/22/33 ---
// Each adds to the energy flux a term proportional to the jump of the
// specific internal energy e = p / (rho (gamma-1)) across the interface,
// which damps the spurious wall heating of the plain solvers.

// Specific internal energy e = inv_rho * p * (1/(gamma-1)), as the three
// solvers form it (scheme.h:1966-1967, 2270-2271, 2852-2853).
EB2_HD double specific_energy(const Side& s, double igm1) { return s.ir * s.p * igm1; }

// HLLHC_Flux (include/scheme.h:1860-2136): HLL with Einfeldt speeds (sound
// speed from gamma p / rho, eta^2 = 1/2 sqrt(rho_L rho_R) / (sum)^2 written
// with the reciprocal sum), plus (s_L s_R / (s_R - s_L)) (e_R - e_L) rho_HLL
// on the energy flux.  Only the y sweep falls back to the Roe sound speed when
// the Einfeldt speed is NaN (:2085-2089; commented out in the x sweep).
template <int DIR>
EB2_HD void flux_hllhc(const double* ql, const double* qr, const Gas& g,
                                           double* F) {
    const double igm1 = 1.0 / g.gm1;
    Side L = unpack(ql, g.gm1), R = unpack(qr, g.gm1);
    double aL = sqrt(g.gamma * L.p * L.ir), aR = sqrt(g.gamma * R.p * R.ir);
    double HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
    double HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double sqL = sqrt(L.r), sqR = sqrt(R.r);
    double ssum = sqL + sqR;
    double isum = 1.0 / ssum;
    double ubar = (sqL * L.u + sqR * R.u) * isum;
    double vbar = (sqL * L.v + sqR * R.v) * isum;
    double Hbar = (sqL * HL + sqR * HR) * isum;
    double eta = 0.5 * sqL * sqR * isum * isum;
    double dun = DIR == 1 ? R.u - L.u : R.v - L.v;
    double dd = sqrt((sqL * aL * aL + sqR * aR * aR) * isum + eta * dun * dun);
    if (DIR == 2 && isnan(dd)) dd = sqrt(g.gm1 * (Hbar - 0.5 * (ubar * ubar + vbar * vbar)));
    double nbar = DIR == 1 ? ubar : vbar;
    double sl = nbar - dd, sr = nbar + dd;
    double rho_hll = (sr * R.r - sl * L.r + FL[0] - FR[0]) / (sr - sl);
    double eL = specific_energy(L, igm1), eR = specific_energy(R, igm1);
    if (sl >= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FL[k];
    } else if (sr <= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FR[k];
    } else {
        double idiff = 1.0 / (sr - sl);
        double slsr = sl * sr;
        const double UL[4] = {L.r, L.ru, L.rv, L.re}, UR[4] = {R.r, R.ru, R.rv, R.re};
        for (int k = 0; k < 4; k++)
            F[k] = (sr * FL[k] - sl * FR[k] + slsr * (UR[k] - UL[k])) * idiff;
        F[3] = F[3] + (slsr * idiff) * (eR - eL) * rho_hll;
    }
}

// HLLCHC_Flux (include/scheme.h:2153-2471): HLLC with the enthalpy sound
// speed in both sweeps and eta^2 written with a division, plus
// (s_L s_R / (s_R - s_L)) (e_R - e_L) times the star-region density factor
// on the energy flux of the two star states.
template <int DIR>
EB2_HD void flux_hllchc(const double* ql, const double* qr, const Gas& g,
                                            double* F) {
    const double igm1 = 1.0 / g.gm1;
    Side L = unpack(ql, g.gm1), R = unpack(qr, g.gm1);
    double HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
    double HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    double aL = sqrt((g.gamma - 1.0) * (HL - 0.5 * (L.uu + L.vv)));
    double aR = sqrt((g.gamma - 1.0) * (HR - 0.5 * (R.uu + R.vv)));
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double sqL = sqrt(L.r), sqR = sqrt(R.r);
    double ssum = sqL + sqR;
    double isum = 1.0 / ssum;
    double ubar = (sqL * L.u + sqR * R.u) * isum;
    double vbar = (sqL * L.v + sqR * R.v) * isum;
    double eta = 0.5 * sqL * sqR / (ssum * ssum);
    double unL = DIR == 1 ? L.u : L.v, unR = DIR == 1 ? R.u : R.v;
    double utL = DIR == 1 ? L.v : L.u, utR = DIR == 1 ? R.v : R.u;
    double dun = unR - unL;
    double dd = sqrt((sqL * aL * aL + sqR * aR * aR) * isum + eta * dun * dun);
    double nbar = DIR == 1 ? ubar : vbar;
    double sl = nbar - dd, sr = nbar + dd;
    double denom = L.r * (sl - unL) - R.r * (sr - unR);
    double ss = (R.p - L.p + L.r * unL * (sl - unL) - R.r * unR * (sr - unR)) / denom;
    double mL = L.r * (sl - unL) / (sl - ss);
    double mR = R.r * (sr - unR) / (sr - ss);
    double feL = L.re * L.ir + (ss - unL) * (ss + L.p / (L.r * (sl - unL)));
    double feR = R.re * R.ir + (ss - unR) * (ss + R.p / (R.r * (sr - unR)));
    double eL = specific_energy(L, igm1), eR = specific_energy(R, igm1);
    double idiff = 1.0 / (sr - sl);
    double slsr = sl * sr;
    double corr = slsr * idiff * (eR - eL);
    // normal and tangential momentum slots of the conserved order
    const int kn = DIR == 1 ? 1 : 2, kt = DIR == 1 ? 2 : 1;
    if (sl >= 0.0) {
        for (int k = 0; k < 4; k++) F[k] = FL[k];
    } else if (sl < 0.0 && ss >= 0.0) {
        const double UL[4] = {L.r, L.ru, L.rv, L.re};
        F[0] = FL[0] + sl * (mL - L.r);
        F[kn] = FL[kn] + sl * (mL * ss - UL[kn]);
        F[kt] = FL[kt] + sl * (mL * utL - UL[kt]);
        F[3] = FL[3] + sl * (mL * feL - L.re) + corr * mL;
    } else if (ss < 0.0 && sr > 0.0) {
        const double UR[4] = {R.r, R.ru, R.rv, R.re};
        F[0] = FR[0] + sr * (mR - R.r);
        F[kn] = FR[kn] + sr * (mR * ss - UR[kn]);
        F[kt] = FR[kt] + sr * (mR * utR - UR[kt]);
        F[3] = FR[3] + sr * (mR * feR - R.re) + corr * mR;
    } else {
        for (int k = 0; k < 4; k++) F[k] = FR[k];
    }
}

// RoeHC_Flux (include/scheme.h:2793-3109): Roe with eps = 1e-12 in the
// 1/(2c^2) and 1/c^2 wave-strength factors, minus 1/2 |u_n + c| (e_R - e_L)
// rho_bar on the energy flux.  Returns false where the reference skips the
// interface (NaN Roe density, :2944-2947).
template <int DIR>
EB2_HD bool flux_roehc(const double* ql, const double* qr, const Gas& g,
                                           double* F) {
    const double igm1 = 1.0 / g.gm1;
    const double eps = 1e-12;
    Side L = unpack(ql, g.gm1), R = unpack(qr, g.gm1);
    double eL = specific_energy(L, igm1), eR = specific_energy(R, igm1);
    double HL = 0.5 * (L.uu + L.vv) + g.gr * (L.p * L.ir);
    double HR = 0.5 * (R.uu + R.vv) + g.gr * (R.p * R.ir);
    double FL[4], FR[4];
    phys_flux<DIR>(L, HL, FL);
    phys_flux<DIR>(R, HR, FR);
    double sqL = sqrt(L.r), sqR = sqrt(R.r);
    double isum = 1.0 / (sqL + sqR);
    double rbar = sqL * sqR;
    double ubar = (sqL * L.u + sqR * R.u) * isum;
    double vbar = (sqL * L.v + sqR * R.v) * isum;
    double Hbar = (sqL * HL + sqR * HR) * isum;
    double q2 = ubar * ubar + vbar * vbar;
    double cbar = sqrt(g.gm1 * (Hbar - 0.5 * q2));
    double nbar = DIR == 1 ? ubar : vbar;
    double lam[4] = {fabs(nbar - cbar), fabs(nbar), fabs(nbar), fabs(nbar + cbar)};
    double drho = R.r - L.r, du = R.u - L.u, dv = R.v - L.v, dp = R.p - L.p;
    double c2 = cbar * cbar;
    double i2c2 = 1.0 / (2.0 * c2 + eps);
    double ic2 = 1.0 / (c2 + eps);
    double dn = DIR == 1 ? du : dv, dtn = DIR == 1 ? dv : du;
    double al[4];
    al[0] = (dp - rbar * cbar * dn) * i2c2;
    al[1] = drho - dp * ic2;
    al[2] = rbar * dtn;
    al[3] = (dp + rbar * cbar * dn) * i2c2;
    double K[4][4];
    if (DIR == 1) {
        K[0][0] = 1.0; K[0][1] = ubar - cbar; K[0][2] = vbar; K[0][3] = Hbar - ubar * cbar;
        K[1][0] = 1.0; K[1][1] = ubar;        K[1][2] = vbar; K[1][3] = 0.5 * q2;
        K[2][0] = 0.0; K[2][1] = 0.0;         K[2][2] = 1.0;  K[2][3] = vbar;
        K[3][0] = 1.0; K[3][1] = ubar + cbar; K[3][2] = vbar; K[3][3] = Hbar + ubar * cbar;
    } else {
        K[0][0] = 1.0; K[0][1] = ubar; K[0][2] = vbar - cbar; K[0][3] = Hbar - vbar * cbar;
        K[1][0] = 1.0; K[1][1] = ubar; K[1][2] = vbar;        K[1][3] = 0.5 * q2;
        K[2][0] = 0.0; K[2][1] = 1.0;  K[2][2] = 0.0;         K[2][3] = ubar;
        K[3][0] = 1.0; K[3][1] = ubar; K[3][2] = vbar + cbar; K[3][3] = Hbar + vbar * cbar;
    }
    for (int c = 0; c < 4; c++) F[c] = 0.5 * (FL[c] + FR[c]);
#pragma unroll
    for (int w = 0; w < 4; w++) {
        double term = 0.5 * lam[w] * al[w];
#pragma unroll
        for (int c = 0; c < 4; c++) F[c] -= term * K[w][c];
    }
    if (isnan(rbar)) return false;
    F[3] = F[3] - 0.5 * lam[3] * (eR - eL) * rbar;
    return true;
}

// Riemann dispatch.  Returns false when HLL or RoeHC skipped the interface.
template <int FLUX, int DIR>
EB2_HD bool riemann(const double* ql, const double* qr, const Gas& g,
                                        double* F) {
    if (FLUX == FLUX_HLL) return flux_hll<DIR>(ql, qr, g, F);
    if (FLUX == FLUX_ROEHC) return flux_roehc<DIR>(ql, qr, g, F);
    if (FLUX == FLUX_HLLHC) flux_hllhc<DIR>(ql, qr, g, F);
    else if (FLUX == FLUX_HLLCHC) flux_hllchc<DIR>(ql, qr, g, F);
    else if (FLUX == FLUX_HLLC) flux_hllc<DIR>(ql, qr, g, F);
    else if (FLUX == FLUX_ROE) flux_roe<DIR>(ql, qr, g, F);
    else flux_llf<DIR>(ql, qr, g, F);
    return true;
}

// riemann with the HLLC flux through the branch-free operations; the other
// solvers as above.
template <int FLUX, int DIR>
EB2_HD bool riemann_rn(const double* ql, const double* qr, const Gas& g, double* F,
                       DivGuard& gd) {
    if (FLUX == FLUX_HLLC) {
        flux_hllc_rn<DIR>(ql, qr, g, F, gd);
        return true;
    }
    return riemann<FLUX, DIR>(ql, qr, g, F);
}

// Primitive state of one cell plus its enthalpy: Con_to_Pri_2D
// (include/initialize.h:1443-1446) and the H of Compute_Eigen_2DX
// (include/Characteriz.h:319).
EB2_HD void primitive5(double r, double ru, double rv, double re,
                                           const Gas& g, double* w) {
    double u = ru / r;
    double v = rv / r;
    double p = (re - 0.5 * r * (u * u + v * v)) * g.gm1;
    w[0] = r;
    w[1] = u;
    w[2] = v;
    w[3] = p;
    w[4] = 0.5 * (u * u + v * v) + g.gr * (p / r);
}

// Is a reconstructed conserved state admissible (rho > 0, p > 0, finite)?
EB2_HD bool admissible(const double* q, double gm1) {
    double r = q[0];
    if (!(r > 0.0)) return false;
    double u = q[1] / r, v = q[2] / r;
    double p = (q[3] - 0.5 * r * (u * u + v * v)) * gm1;
    return p > 0.0;
}

}  // namespace x64
}  // namespace eb2
