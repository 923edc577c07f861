// eb2_stage_mixed.cuh -- fused x+y sweep and SSP-RK stage, mixed precision.
//
// Same structure and contract as the FP64 form (eb2_stage_fp64.cuh): a CTA
// stages a TX x TY tile plus 3-cell halo, computes every interface flux the
// tile needs and applies flux difference + RK combination to its cells.
// Differences: the staged tile is FP32, per-cell primitives come from FP64
// arithmetic, interface work is FP32 in delta form (eb2_point_mixed.cuh), the
// fluxes are widened to FP64 where they are read, and the flux difference and
// RK combination are FP64 with the stage input re-read in FP64.
// Reconstruction: WENO5 in characteristic variables (Jiang-Shu or WENO-Z
// weights).
//
// Shared memory holds every per-cell and per-face record as one vector
// (float4 conserved state, float4 + float2 primitives, float4 face flux), so
// that a stencil point, a primitive record or a flux is one 16-byte load: the
// warp's 32 consecutive cells then cover four 128-byte wavefronts without
// bank conflicts, and the interfaces issue a quarter of the shared-memory
// instructions of a field-per-array layout.
#pragma once

#include <type_traits>

#include "eb2_kernels.h"
#include "eb2_point_fp64.cuh"
#include "eb2_point_mixed.cuh"

namespace eb2 {
namespace mixstage {

// A tile shape of the stage kernel: TX x TY cells per CTA of NT threads, CTAS
// CTAs resident per SM (the register budget is 65536 / (NT CTAS) per thread).
// The solve server's autotuner picks one of the shapes of MixedShapes per
// batch-shape class; single solves use Shape16.
template <int TX_, int TY_, int NT_, int CTAS_>
struct Shape {
    static constexpr int TX = TX_, TY = TY_, NT = NT_, CTAS = CTAS_;
    static constexpr int HX = TX + 6, HY = TY + 6;    // conserved tile with halos
    static constexpr int PX = TX + 2, PY = TY + 2;    // primitives: tile + first ring
    static constexpr int FS = HX * HY, PS = PX * PY;
    static constexpr int XS = (TX + 1) * TY, YS = TX * (TY + 1);  // x and y faces
    static constexpr int NJX = XS, NJY = YS;
    // FP32 face fluxes (widened exactly where read, so that both cells of a face
    // see the same value, the flux differences telescope and the step conserves
    // to FP64 round-off), FP32 tile, FP32 primitives
    static constexpr size_t SMEM =
        (size_t)(XS + YS + FS + PS) * sizeof(float4) + (size_t)PS * sizeof(float2);
    static_assert(TX * TY % NT == 0, "whole cells per thread");
    static_assert((NJX + NJY + NT - 1) / NT <= 32, "one vacuum bit per job of a thread");
};
#ifndef EB2_MIXED_CTAS
#define EB2_MIXED_CTAS 4
#endif
using Shape16 = Shape<MIXED_TILE_X, STAGE_TILE_Y, 256, EB2_MIXED_CTAS>;
using Shape8 = Shape<8, STAGE_TILE_Y, 128, 8>;
using Shape32 = Shape<32, STAGE_TILE_Y, 512, 2>;

// Conserved differences of both sides of an interface next to a near-vacuum
// cell: the stencil's six cells are read in FP64 from the stage input (cell i at
// g2, cell i+1 at g2 + step), the Roe average and the left and right
// eigenvector matrices are the reference's, in FP64 (Characteriz.h:333-392 for
// x, :435-494 for y), and so are the projections of the differences onto them
// and the back-projection; only the WENO weights and candidate values between
// the two run in FP32 lanes, as on every other interface.  Rare: the stage
// kernel runs these interfaces in a pass of their own after the others, so
// that their FP64 arithmetic does not weigh on the registers of the common
// path.
template <int DIR, bool WZ>
EB2_HD void vacuum_delta(const double* __restrict__ u, size_t g2,
                                          long long step, size_t plane, const Gas g,
                                          f32::f2* dq) {
    // the two cells next to the interface stay in registers; the other four
    // are re-read per field (cache hits)
    double qa[4], qb[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        qa[m] = u[g2 + m * plane];
        qb[m] = u[g2 + step + m * plane];
    }
    // a stencil of six equal cells (the undisturbed gas ahead of a front) has
    // zero differences on both sides: nothing to project
    bool flat = true;
#pragma unroll
    for (int m = 0; m < 4; m++) flat = flat && qa[m] == qb[m];
#pragma unroll
    for (int n = 0; n < 6; n++) {
        if (n == 2 || n == 3) continue;
#pragma unroll
        for (int m = 0; m < 4; m++) flat = flat && u[g2 + (n - 2) * step + m * plane] == qa[m];
    }
    if (flat) {
#pragma unroll
        for (int m = 0; m < 4; m++) dq[m] = f32::f2s(0.0f);
        return;
    }
    double A[5], B[5];
    x64::primitive5(qa[0], qa[1], qa[2], qa[3], g, A);
    x64::primitive5(qb[0], qb[1], qb[2], qb[3], g, B);
    const x64::Roe e = x64::roe_average(A, B, g.gm1);
    // lane stencils of weno5_lanes: minus side relative to cell i (n = 0, 1, 3,
    // 4), plus side mirrored and relative to cell i+1 (n = 5, 4, 2, 1)
    const int nm[4] = {0, 1, 3, 4}, np[4] = {5, 4, 2, 1};
    f32::f2 W[4];
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
        double l[4];
        x64::left_row<DIR>(e, k, l);
        f32::f2 X[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const size_t om = g2 + (nm[t] - 2) * step, op = g2 + (np[t] - 2) * step;
            double xm = 0.0, xp = 0.0;
#pragma unroll
            for (int m = 0; m < 4; m++) {
                xm += l[m] * (u[om + m * plane] - qa[m]);
                xp += l[m] * (u[op + m * plane] - qb[m]);
            }
            X[t] = make_float2((float)xm, (float)xp);
        }
        W[k] = f32::weno5_lanes<WZ>(X[0], X[1], X[2], X[3]);
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        double r[4];
        x64::right_row<DIR>(e, m, r);
        double sm = 0.0, sp = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            sm += r[k] * (double)W[k].x;
            sp += r[k] * (double)W[k].y;
        }
        dq[m] = make_float2((float)sm, (float)sp);
    }
}

// Is either cell next to an interface near vacuum (p below pthr, 1e-3 of the
// mean pressure)?
EB2_HD bool near_vacuum(float pa, float pb, float pthr) { return pa < pthr || pb < pthr; }

// One interface.  s: stencil cell n = 0 (i-2), `stride` records along the
// sweep; pa/ha and pb/hb: primitive records of cells i and i+1; ga/gb: the
// two cells in global memory.  VAC: an interface next to a near-vacuum cell,
// whose characteristic projections take FP64 matrices (vacuum_delta).
template <bool VAC, int DIR, bool WZ, int FLUX>
EB2_HD unsigned face_flux(const float4* __restrict__ s, int stride,
                          const float4* __restrict__ pa, const float2* __restrict__ ha,
                          const float4* __restrict__ pb, const float2* __restrict__ hb,
                          const double* __restrict__ u, size_t ga, size_t gb, size_t plane,
                          const Gas& g, int positivity, float4* __restrict__ out) {
    const float gm1 = (float)g.gm1, gamma = (float)g.gamma;
    f32::f2 dq[4];
    if constexpr (VAC) {
        vacuum_delta<DIR, WZ>(u, ga, (long long)gb - (long long)ga, plane, g, dq);
    } else {
        // (the primitive records are read where they are used, so that they
        // hold no registers across the reconstruction)
        const float4 base = s[2 * stride];
        const f32::Eig e = f32::roe_f32(*pa, *ha, *pb, *hb, gm1);
        // characteristic differences y_n = L (U_n - U_i), n = i-2..i+3 (y_2 = 0)
        float y[4][6];
#pragma unroll
        for (int n = 0; n < 6; n++) {
            if (n == 2) continue;
            const float4 q = s[n * stride];
            float c[4];
            f32::project<DIR>(e, q.x - base.x, q.y - base.y, q.z - base.z, q.w - base.w, c);
#pragma unroll
            for (int k = 0; k < 4; k++) y[k][n] = c[k];
        }
        // both sides of each field in the two lanes (weno5_lanes); a field whose
        // stencil is flat on both sides reconstructs its base values exactly, and
        // uniform regions, where whole warps agree, skip the weights
        f32::f2 W[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const unsigned any = (f32::bits(y[k][0]) | f32::bits(y[k][1]) |
                                  f32::bits(y[k][3]) | f32::bits(y[k][4]) |
                                  f32::bits(y[k][5])) << 1;
            if (any == 0u) {
                W[k] = f32::f2s(0.0f);
            } else {
                const float y3 = y[k][3];
                W[k] = f32::weno5_lanes<WZ>(make_float2(y[k][0], y[k][5] - y3),
                                            make_float2(y[k][1], y[k][4] - y3),
                                            make_float2(y3, -y3),
                                            make_float2(y[k][4], y[k][1] - y3));
            }
        }
        f32::unproject2<DIR>(e, W, dq);
    }
    // minus side around cell i, plus side around cell i+1
    const float4 A = *pa, B = *pb;
    const float ea = s[2 * stride].w, eb = s[3 * stride].w;
    f32::Prim L, R;
    f32::prim_from_delta2<DIR>(make_float2(A.x, B.x), make_float2(A.y, B.y),
                               make_float2(A.z, B.z), make_float2(A.w, B.w),
                               make_float2(ea, eb), dq, gm1, L, R);
    unsigned st = 0;
    if (!(L.r > 0.0f && L.p > 0.0f && R.r > 0.0f && R.p > 0.0f)) {
        if (positivity) {
            float z[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            L = f32::prim_from_delta<DIR>(A.x, A.y, A.z, A.w, ea, z, gm1);
            R = f32::prim_from_delta<DIR>(B.x, B.y, B.z, B.w, eb, z, gm1);
        } else {
            st |= ST_NONPHYSICAL;
        }
    }
    float F[4];
    if (FLUX == FLUX_HLLC) f32::hllc(L, R, gamma, F);
    else if (FLUX == FLUX_ROE) f32::roe(L, R, gamma, F);
    else if (FLUX == FLUX_HLL) f32::hll(L, R, gamma, F);
    else if (FLUX == FLUX_HLLHC) f32::hllhc(L, R, gamma, F);
    else if (FLUX == FLUX_HLLCHC) f32::hllchc(L, R, gamma, F);
    else if (FLUX == FLUX_ROEHC) f32::roehc(L, R, gamma, F);
    else f32::llf(L, R, gamma, F);
    // (mass, normal, tangential, energy) -> (rho, rho u, rho v, rho E)
    *out = make_float4(F[0], DIR == 1 ? F[1] : F[2], DIR == 1 ? F[2] : F[1], F[3]);
    return st;
}

// Both paths, chosen per interface (the CPU checks of the face arithmetic).
template <int DIR, bool WZ, int FLUX>
EB2_HD unsigned interface_flux(const float4* __restrict__ s, int stride,
                               const float4* __restrict__ pa, const float2* __restrict__ ha,
                               const float4* __restrict__ pb, const float2* __restrict__ hb,
                               const double* __restrict__ u, size_t ga, size_t gb, size_t plane,
                               float pthr, const Gas& g, int positivity,
                               float4* __restrict__ out) {
    if (near_vacuum(pa->w, pb->w, pthr))
        return face_flux<true, DIR, WZ, FLUX>(s, stride, pa, ha, pb, hb, u, ga, gb, plane, g,
                                              positivity, out);
    return face_flux<false, DIR, WZ, FLUX>(s, stride, pa, ha, pb, hb, u, ga, gb, plane, g,
                                           positivity, out);
}

// One tile (ti, tj) of one stage; shared by the single-solve and batched kernels.
template <class S, bool WZ, int FLUX>
__device__ __forceinline__ void stage_tile(const StageArgs& a, int ti, int tj, int tiles_x) {
    constexpr int TX = S::TX, TY = S::TY, NT = S::NT, HY = S::HY, PX = S::PX, PY = S::PY;
    constexpr int FS = S::FS, PS = S::PS, XS = S::XS, YS = S::YS, NJX = S::NJX, NJY = S::NJY;
    Ctrl* ctrl = a.ctrl;
    if (!ctrl->active) return;
    extern __shared__ float4 smv[];
    float4* sFx = smv;
    float4* sFy = sFx + XS;
    float4* sU = sFy + YS;
    float4* sP = sU + FS;
    float2* sH = reinterpret_cast<float2*>(sP + PS);
    // per tile row: max |u|+a, max |v|+a and the sum of p (the CFL partials)
    __shared__ double rowred[3][TX];

    const int rows = a.grid.rows, cols = a.grid.cols;
    const size_t plane = (size_t)rows * cols;
    const int i0 = GC + ti * TX, j0 = GC + tj * TY;
    const double* __restrict__ uin = a.uin;
    const Gas g = a.gas;
    const float pthr = (float)(1.0e-3 * ctrl->pmean);

    // 1. tile + halo as FP32; primitives of the tile and its first ring from FP64.
    // Thread t takes elements t, t + NT, ... of the HX x HY tile; all of its
    // loads are issued before any is used, so their latencies overlap.
    {
        constexpr int NE = (FS + NT - 1) / NT;
        double q[NE][4];
        int r = threadIdx.x / HY, c = threadIdx.x - r * HY;
        int er[NE], ec[NE];
#pragma unroll
        for (int t = 0; t < NE; t++) {
            er[t] = r;
            ec[t] = c;
            const int i = i0 - 3 + r, j = j0 - 3 + c;
            const bool in = threadIdx.x + t * NT < FS && i < rows && j < cols;
            const double* src = uin + (in ? (size_t)i * cols + j : 0);
#pragma unroll
            for (int k = 0; k < 4; k++) q[t][k] = in ? src[k * plane] : 0.0;
            c += NT % HY;
            r += NT / HY;
            if (c >= HY) {
                c -= HY;
                r++;
            }
        }
#pragma unroll
        for (int t = 0; t < NE; t++) {
            const int e = threadIdx.x + t * NT;
            if (e >= FS) break;
            float qf[4];
#pragma unroll
            for (int k = 0; k < 4; k++) qf[k] = (float)q[t][k];
            sU[e] = make_float4(qf[0], qf[1], qf[2], qf[3]);
            const int pr = er[t] - 2, pc = ec[t] - 2;
            if ((unsigned)pr < (unsigned)PX && (unsigned)pc < (unsigned)PY)
                f32::cell_prims(q[t], qf, g, sP + pr * PY + pc, sH + pr * PY + pc);
        }
    }
    __syncthreads();

    // 2. interface fluxes.  Interfaces next to a near-vacuum cell are marked
    // in `vac` (bit = this thread's job number) and computed in a pass of
    // their own with the FP64 eigenvector matrices.
    unsigned st = 0, vac = 0;
    const int pos = a.num.positivity;
    auto face = [&](auto vacuum, int job) -> unsigned {
        constexpr bool VAC = decltype(vacuum)::value;
        if (job < NJX) {
            int rr = job / TY, cc = job - rr * TY;
            int i = i0 - 1 + rr, j = j0 + cc;
            if (i >= rows - GC || j >= cols - GC) return 0u;  // past the domain edge
            const int pa = rr * PY + (cc + 1);
            if (!VAC && near_vacuum(sP[pa].w, sP[pa + PY].w, pthr)) return ~0u;
            size_t ga = (size_t)i * cols + j;
            return face_flux<VAC, 1, WZ, FLUX>(sU + rr * HY + (cc + 3), HY, sP + pa, sH + pa,
                                               sP + pa + PY, sH + pa + PY, uin, ga, ga + cols,
                                               plane, g, pos, sFx + rr * TY + cc);
        }
        int q = job - NJX;
        int rr = q / (TY + 1), cc = q - rr * (TY + 1);
        int i = i0 + rr, j = j0 - 1 + cc;
        if (i >= rows - GC || j >= cols - GC) return 0u;
        const int pa = (rr + 1) * PY + cc;
        if (!VAC && near_vacuum(sP[pa].w, sP[pa + 1].w, pthr)) return ~0u;
        size_t ga = (size_t)i * cols + j;
        return face_flux<VAC, 2, WZ, FLUX>(sU + (rr + 3) * HY + cc, 1, sP + pa, sH + pa,
                                           sP + pa + 1, sH + pa + 1, uin, ga, ga + 1, plane, g,
                                           pos, sFy + rr * (TY + 1) + cc);
    };
    for (int job = threadIdx.x, n = 0; job < NJX + NJY; job += NT, n++) {
        const unsigned r = face(std::false_type{}, job);
        if (r == ~0u) vac |= 1u << n;
        else st |= r;
    }
    if (__syncthreads_or(vac != 0u)) {
        for (int job = threadIdx.x, n = 0; job < NJX + NJY; job += NT, n++)
            if (vac >> n & 1u) st |= face(std::true_type{}, job);
        __syncthreads();
    }

    // 3. flux difference (widened to FP64), RK combination in FP64.  The
    // thread's cells (TX TY / NT of them) load their stage input and step
    // start state first, then combine.
    const double dt = ctrl->dt;
    const double idx = a.grid.inv_dx, idy = a.grid.inv_dy;
    const double grav = a.num.gravity;
    constexpr int NC = TX * TY / NT;
    // the CFL partials of this thread's cells (zero outside the domain)
    double cmx[NC], cmy[NC], cps[NC];
    double xs[NC][4], ys[NC][4];
#pragma unroll
    for (int t = 0; t < NC; t++) {
        const int e = threadIdx.x + t * NT;
        const int rr = e / TY, cc = e - rr * TY;
        const int i = i0 + rr, j = j0 + cc;
        const bool in = i < rows - GC && j < cols - GC;
        const size_t o = in ? (size_t)i * cols + j : 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            xs[t][k] = in ? uin[o + k * plane] : 0.0;
            ys[t][k] = in && a.combine != COMB_EULER ? a.un[o + k * plane] : xs[t][k];
        }
    }
#pragma unroll
    for (int t = 0; t < NC; t++) {
        const int e = threadIdx.x + t * NT;
        const int rr = e / TY, cc = e - rr * TY;
        const int i = i0 + rr, j = j0 + cc;
        cmx[t] = cmy[t] = cps[t] = 0.0;
        if (i >= rows - GC || j >= cols - GC) continue;
        const size_t o = (size_t)i * cols + j;
        const double* x = xs[t];
        double src[4] = {0.0, 0.0, 0.0, 0.0}, out[4];
        if (a.num.source) {
            double rho = x[0];
            src[2] = rho * grav;
            src[3] = rho * grav * (x[2] / rho);
        }
        // widened exactly; both cells of a face read the same FP32 value
        const float4 fxp = sFx[(rr + 1) * TY + cc], fxm = sFx[rr * TY + cc];
        const float4 fyp = sFy[rr * (TY + 1) + cc + 1], fym = sFy[rr * (TY + 1) + cc];
        const float fp[4] = {fxp.x, fxp.y, fxp.z, fxp.w}, fm[4] = {fxm.x, fxm.y, fxm.z, fxm.w};
        const float gp[4] = {fyp.x, fyp.y, fyp.z, fyp.w}, gm[4] = {fym.x, fym.y, fym.z, fym.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double L = -((double)fp[k] - (double)fm[k]) * idx - ((double)gp[k] - (double)gm[k]) * idy +
                       src[k];
            const double y = ys[t][k];
            double r;
            switch (a.combine) {
                case COMB_EULER: r = y + dt * L; break;
                case COMB_RK2: r = 0.5 * y + 0.5 * (x[k] + dt * L); break;
                case COMB_RK3_2: r = 0.75 * y + 0.25 * (x[k] + dt * L); break;
                default: r = (1.0 / 3.0) * y + (2.0 / 3.0) * (x[k] + dt * L); break;
            }
            out[k] = r;
            a.uout[o + k * plane] = r;
        }
        if (isnan(out[0]) || isnan(out[3])) st |= ST_NAN_STATE;
        if (a.partials) {
            double rho = out[0];
            double ir = 1.0 / rho;
            double uu = out[1] * ir, vv = out[2] * ir;
            double p = (out[3] - 0.5 * rho * (uu * uu + vv * vv)) * g.gm1;
            double c = sqrt(g.gamma * p * ir);
            cmx[t] = fabs(uu) + c;
            cmy[t] = fabs(vv) + c;
            cps[t] = p;
        }
    }

    unsigned wst = __reduce_or_sync(0xffffffffu, st);
    if (wst && (threadIdx.x & 31) == 0) atomicOr(&ctrl->status, wst);
    if (a.partials) {
        // A warp holds one tile row per t (lane = column), reduced over a fixed
        // lane tree; then one partial triple per 8-row block, its rows summed
        // in order.  So the partials, and the mean pressure summed from them,
        // are the same bits in every tile shape.
        const int w = threadIdx.x >> 5;
#pragma unroll
        for (int t = 0; t < NC; t++) {
            double x = cmx[t], y = cmy[t], p = cps[t];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ox = __shfl_down_sync(0xffffffffu, x, off);
                const double oy = __shfl_down_sync(0xffffffffu, y, off);
                const double op = __shfl_down_sync(0xffffffffu, p, off);
                if (ox > x) x = ox;
                if (oy > y) y = oy;
                p += op;
            }
            if ((threadIdx.x & 31) == 0) {
                const int row = w + t * (NT / 32);
                rowred[0][row] = x;
                rowred[1][row] = y;
                rowred[2][row] = p;
            }
        }
        __syncthreads();
        constexpr int NB = TX / MIXED_PARTIAL_ROWS;
        const int k = threadIdx.x;
        if (k < NB && ti * TX + k * MIXED_PARTIAL_ROWS < a.grid.nx) {
            double bx = 0.0, by = 0.0, bp = 0.0;
#pragma unroll
            for (int r = 0; r < MIXED_PARTIAL_ROWS; r++) {
                const int row = k * MIXED_PARTIAL_ROWS + r;
                if (rowred[0][row] > bx) bx = rowred[0][row];
                if (rowred[1][row] > by) by = rowred[1][row];
                bp += rowred[2][row];
            }
            const size_t b = (size_t)(ti * (TX / MIXED_PARTIAL_ROWS) + k) * tiles_x + tj;
            a.partials[3 * b + 0] = bx;
            a.partials[3 * b + 1] = by;
            a.partials[3 * b + 2] = bp;
        }
    }
}

// Single solve: one CTA per tile.
template <class S, bool WZ, int FLUX>
__global__ void __launch_bounds__(S::NT, S::CTAS) k_stage(StageArgs a) {
    stage_tile<S, WZ, FLUX>(a, blockIdx.y, blockIdx.x, gridDim.x);
}

// Tile shape of single solves (0: Shape16, 1: Shape8, 2: Shape32).
#ifndef EB2_MIXED_SOLVE_SHAPE
#define EB2_MIXED_SOLVE_SHAPE 0
#endif
using SolveShape = std::conditional_t<EB2_MIXED_SOLVE_SHAPE == 1, Shape8,
                                      std::conditional_t<EB2_MIXED_SOLVE_SHAPE == 2, Shape32,
                                                         Shape16>>;

template <bool WZ, int FLUX>
cudaError_t launch_one(const StageArgs& a, cudaStream_t s) {
    using S = SolveShape;
    auto kern = k_stage<S, WZ, FLUX>;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)S::SMEM);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (!a.uout) return cudaSuccess;
    dim3 grid((a.grid.ny + S::TY - 1) / S::TY, (a.grid.nx + S::TX - 1) / S::TX);
    kern<<<grid, S::NT, S::SMEM, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mixstage
}  // namespace eb2
