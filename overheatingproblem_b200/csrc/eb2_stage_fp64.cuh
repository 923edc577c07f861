// eb2_stage_fp64.cuh -- fused x+y sweep and SSP-RK stage, FP64 bit-parity form.
//
// One CTA owns a TX x TY tile of cells (x rows i, y columns j).  It stages the
// stage input of the tile plus a 3-cell halo in shared memory, converts the
// tile and its first ring to primitives (Con_to_Pri_2D), computes every x and
// y interface flux the tile needs (Roe eigenvectors, projection, WENO5/TVD
// per field, back-projection, Riemann flux: WENO5_Reconstruction /
// TVD_Reconstruction + HLLC_Flux etc. of Flux_Reconstruction_RP,
// include/CFD_convection.h:38-200), and then forms the flux difference
// (Space_Discrete_Item, include/scheme.h:3758-3777) and the SSP-RK combination
// (include/time_advance.h:831-872) for its cells.  The stage output leaves
// through one coalesced store per field; the state at the start of the step
// is read once for stages 2 and 3.  The reference makes about twelve
// full-grid passes with temporaries for the same stage.
//
// Wave-speed maxima of the new state (Get_Delta_T_2D's reduction,
// include/function.h:144-175) are reduced per block in the epilogue.
#pragma once

#include <type_traits>

#include "eb2_kernels.h"
#include "eb2_point_fp64.cuh"

namespace eb2 {
namespace fp64stage {

constexpr int TX = FP64_TILE_X, TY = STAGE_TILE_Y, NT = 256;
constexpr int HX = TX + 6, HY = TY + 6;       // U tile with halos
constexpr int PX = TX + 2, PY = TY + 2;       // primitive region (tile + first ring)
constexpr int FS = HX * HY;                   // field stride in sU
constexpr int PS = PX * PY;                   // field stride in sP
constexpr int XS = (TX + 1) * TY;             // field stride in sFx
constexpr int YS = TX * (TY + 1);             // field stride in sFy
constexpr int NJX = (TX + 1) * TY, NJY = TX * (TY + 1);

template <bool CHAR>
constexpr size_t smem_bytes() {
    return (size_t)(4 * FS + (CHAR ? 5 * PS : 0) + 4 * XS + 4 * YS) * sizeof(double);
}

// rho > 0 and p > 0 without a division: 2*rho*E > (rho u)^2 + (rho v)^2.
EB2_HD bool admissible(const double* q) {
    return q[0] > 0.0 && 2.0 * q[3] * q[0] > q[1] * q[1] + q[2] * q[2];
}

// Reconstructed states of one interface: characteristic (project on the Roe
// left eigenvectors, reconstruct each field, project back) or per conserved
// field.  RN selects the branch-free WENO divisions, whose operands are
// recorded in gd.
template <bool RN, int DIR, int RECON, bool CHAR, bool WZ>
EB2_HD void reconstruct_states(const double* __restrict__ s, int stride, const x64::Roe& e,
                               double delta, double* ql, double* qr, x64::DivGuard& gd) {
    constexpr int N0 = RECON == 5 ? 0 : (RECON == 2 || RECON == 3 ? 1 : 2);
    constexpr int N1 = RECON == 5 ? 6 : (RECON == 2 || RECON == 3 ? 5 : 4);
    if (CHAR) {
        double wm[4], wp[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double l[4];
            x64::left_row<DIR>(e, k, l);
            double q6[6];
#pragma unroll
            for (int n = N0; n < N1; n++) {
                double acc = 0.0;
#pragma unroll
                for (int m = 0; m < 4; m++) acc += s[m * FS + n * stride] * l[m];
                q6[n] = acc;
            }
            if constexpr (RN) x64::recon_pair_rn<RECON, WZ>(q6, wm[k], wp[k], gd);
            else x64::recon_pair<RECON, WZ, true>(q6, delta, wm[k], wp[k]);
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            double r[4];
            x64::right_row<DIR>(e, m, r);
            double sl = 0.0, sr = 0.0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                sl += wm[k] * r[k];
                sr += wp[k] * r[k];
            }
            ql[m] = sl;
            qr[m] = sr;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double q6[6];
#pragma unroll
            for (int n = N0; n < N1; n++) q6[n] = s[k * FS + n * stride];
            if constexpr (RN) x64::recon_pair_rn<RECON, false>(q6, ql[k], qr[k], gd);
            else x64::recon_pair<RECON, false, false>(q6, delta, ql[k], qr[k]);
        }
    }
}

// Returned by interface_flux<RN = true> when an operand left the range of the
// branch-free divisions: nothing was stored, the caller redoes the interface
// with RN = false.  Never reaches the control block.
constexpr unsigned ST_REDO = 1u << 31;

// Flux at one interface.  s points at stencil cell n=0 (i-2) of field 0,
// `stride` steps along the sweep, fields are FS apart.  pa/pb point at the
// primitive 5-tuples of the two cells next to the interface (fields PS apart).
// RN: Roe average and WENO weights (RECON 5 and 3) through the branch-free
// divisions.
template <bool RN, int DIR, int RECON, bool CHAR, bool WZ, int FLUX>
EB2_HD unsigned interface_flux(const double* __restrict__ s, int stride,
                                                   const double* __restrict__ pa,
                                                   const double* __restrict__ pb, double delta,
                                                   const Gas& g, int positivity,
                                                   double* __restrict__ out, int ostride) {
    double ql[4], qr[4];
    x64::Roe e{};
    x64::DivGuard gd;
    if (CHAR) {
        double A[5], B[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
            A[q] = pa[q * PS];
            B[q] = pb[q * PS];
        }
        e = RN ? x64::roe_average_rn(A, B, g.gm1, gd) : x64::roe_average(A, B, g.gm1);
    }
    constexpr bool kRNW = RN && (RECON == 5 || RECON == 3);
    reconstruct_states<kRNW, DIR, RECON, CHAR, WZ>(s, stride, e, delta, ql, qr, gd);
    unsigned st = 0;
    if (!(admissible(ql) && admissible(qr))) {
        if (positivity) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                ql[k] = s[k * FS + 2 * stride];
                qr[k] = s[k * FS + 3 * stride];
            }
        } else {
            st |= ST_NONPHYSICAL;
        }
    }
    double F[4];
    const bool fine = RN ? x64::riemann_rn<FLUX, DIR>(ql, qr, g, F, gd)
                         : x64::riemann<FLUX, DIR>(ql, qr, g, F);
    if (RN && !gd.ok()) return ST_REDO;
    if (!fine) {
        // the reference leaves a stale entry here; a NaN makes it visible
#pragma unroll
        for (int k = 0; k < 4; k++) F[k] = nan("");
        st |= ST_NONPHYSICAL;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) out[k * ostride] = F[k];
    return st;
}

// One tile (ti, tj) of one stage; tiles_x = tiles along y (for the partials
// index).  Shared by the single-solve kernel and the batched kernel.
template <int RECON, bool CHAR, bool WZ, int FLUX>
__device__ __forceinline__ void stage_tile(const StageArgs& a, int ti, int tj, int tiles_x) {
    Ctrl* ctrl = a.ctrl;
    if (!ctrl->active) return;
    extern __shared__ double sm[];
    double* sU = sm;
    double* sP = sU + 4 * FS;
    double* sFx = sP + (CHAR ? 5 * PS : 0);
    double* sFy = sFx + 4 * XS;
    __shared__ double red[3][NT / 32];

    const int rows = a.grid.rows, cols = a.grid.cols;
    const int i0 = GC + ti * TX, j0 = GC + tj * TY;
    const double* __restrict__ uin = a.uin;
    const Gas g = a.gas;

    // 1. stage input tile + halo (rows i0-3..i0+TX+2, columns j0-3..j0+TY+2)
    for (int e = threadIdx.x; e < 4 * FS; e += NT) {
        int k = e / FS, rem = e - k * FS;
        int r = rem / HY, c = rem - r * HY;
        int i = i0 - 3 + r, j = j0 - 3 + c;
        sU[e] = (i < rows && j < cols) ? uin[at(k, i, j, rows, cols)] : 0.0;
    }
    __syncthreads();

    // 2. primitives of the tile and its first ring
    if (CHAR) {
        for (int e = threadIdx.x; e < PS; e += NT) {
            int r = e / PY, c = e - r * PY;
            int u = (r + 2) * HY + (c + 2);
            double w[5];
            x64::primitive5(sU[u], sU[FS + u], sU[2 * FS + u], sU[3 * FS + u], g, w);
#pragma unroll
            for (int q = 0; q < 5; q++) sP[q * PS + e] = w[q];
        }
        __syncthreads();
    }

    // 3. interface fluxes: x faces (TX+1) x TY in one loop, then y faces
    // TX x (TY+1) in another, so that each loop carries one direction's code and
    // live state (with 15 x 32 tiles each takes two passes of the 256 threads).
    // A face whose WENO operands leave the range of the branch-free divisions
    // is marked in `redo` (bit = this thread's job number) and recomputed with
    // `/` after the pass, so the common pass carries no fallback code.
    unsigned st = 0;
    const int pos = a.num.positivity;
    unsigned redo = 0;
    constexpr int PXF = (NJX + NT - 1) / NT, PYF = (NJY + NT - 1) / NT;
    static_assert(PXF + PYF <= 32, "one redo bit per job of a thread");
    // (faces that no interior cell of this tile uses -- past the domain edge in
    // a partial tile -- are skipped)
    auto xface = [&](auto rn, int job) -> unsigned {
        constexpr bool RN = decltype(rn)::value;
        int rr = job / TY, cc = job - rr * TY;
        if (i0 - 1 + rr >= rows - GC || j0 + cc >= cols - GC) return 0u;
        const double* s = sU + rr * HY + (cc + 3);
        const double* pa = sP + rr * PY + (cc + 1);
        return interface_flux<RN, 1, RECON, CHAR, WZ, FLUX>(s, HY, pa, pa + PY, a.grid.dx, g,
                                                            pos, sFx + rr * TY + cc, XS);
    };
    auto yface = [&](auto rn, int q) -> unsigned {
        constexpr bool RN = decltype(rn)::value;
        int rr = q / (TY + 1), cc = q - rr * (TY + 1);
        if (i0 + rr >= rows - GC || j0 - 1 + cc >= cols - GC) return 0u;
        const double* s = sU + (rr + 3) * HY + cc;
        const double* pa = sP + (rr + 1) * PY + cc;
        return interface_flux<RN, 2, RECON, CHAR, WZ, FLUX>(s, 1, pa, pa + 1, a.grid.dy, g, pos,
                                                            sFy + rr * (TY + 1) + cc, YS);
    };
    for (int job = threadIdx.x, n = 0; job < NJX; job += NT, n++) {
        const unsigned r = xface(std::true_type{}, job);
        if (r & ST_REDO) redo |= 1u << n;
        else st |= r;
    }
    for (int q = threadIdx.x, n = PXF; q < NJY; q += NT, n++) {
        const unsigned r = yface(std::true_type{}, q);
        if (r & ST_REDO) redo |= 1u << n;
        else st |= r;
    }
    if (__syncthreads_or(redo != 0u)) {
        for (int job = threadIdx.x, n = 0; job < NJX; job += NT, n++)
            if (redo >> n & 1u) st |= xface(std::false_type{}, job);
        for (int q = threadIdx.x, n = PXF; q < NJY; q += NT, n++)
            if (redo >> n & 1u) st |= yface(std::false_type{}, q);
        __syncthreads();
    }

    // 4. flux difference, source, RK combination, wave-speed partials
    const double dt = ctrl->dt;
    const double idx = a.grid.inv_dx, idy = a.grid.inv_dy;
    const double grav = a.num.gravity;
    double mx = 0.0, my = 0.0, ps = 0.0;
    for (int e = threadIdx.x; e < TX * TY; e += NT) {
        int rr = e / TY, cc = e - rr * TY;
        int i = i0 + rr, j = j0 + cc;
        if (i >= rows - GC || j >= cols - GC) continue;
        int u = (rr + 3) * HY + (cc + 3);
        double x[4], src[4] = {0.0, 0.0, 0.0, 0.0}, o[4];
#pragma unroll
        for (int k = 0; k < 4; k++) x[k] = sU[k * FS + u];
        if (a.num.source) {
            // Source_Gravity, include/scheme.h:3738-3749
            double rho = x[0];
            double v = x[2] / rho;
            src[2] = rho * grav;
            src[3] = rho * grav * v;
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double fxp = sFx[k * XS + (rr + 1) * TY + cc], fxm = sFx[k * XS + rr * TY + cc];
            double fyp = sFy[k * YS + rr * (TY + 1) + cc + 1], fym = sFy[k * YS + rr * (TY + 1) + cc];
            double L = -(fxp - fxm) * idx - (fyp - fym) * idy + src[k];
            double y = a.combine == COMB_EULER ? x[k] : a.un[at(k, i, j, rows, cols)];
            double r;
            switch (a.combine) {
                case COMB_EULER: r = y + dt * L; break;
                case COMB_RK2: r = 0.5 * y + 0.5 * (x[k] + dt * L); break;
                case COMB_RK3_2: r = (3.0 / 4.0) * y + (1.0 / 4.0) * (x[k] + dt * L); break;
                default: r = (1.0 / 3.0) * y + (2.0 / 3.0) * (x[k] + dt * L); break;
            }
            o[k] = r;
            a.uout[at(k, i, j, rows, cols)] = r;
        }
        if (isnan(o[0]) || isnan(o[1]) || isnan(o[2]) || isnan(o[3])) st |= ST_NAN_STATE;
        if (a.partials) {
            double rho = o[0];
            double uu = o[1] / rho, vv = o[2] / rho;
            double p = (o[3] - 0.5 * rho * (uu * uu + vv * vv)) * g.gm1;
            double c = sqrt(g.gamma * p / rho);
            double lx = fabs(uu) + c, ly = fabs(vv) + c;
            if (lx > mx) mx = lx;
            if (ly > my) my = ly;
            ps += p;
        }
    }

    unsigned wst = __reduce_or_sync(0xffffffffu, st);
    if (wst && (threadIdx.x & 31) == 0) atomicOr(&ctrl->status, wst);

    if (a.partials) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            double ox = __shfl_down_sync(0xffffffffu, mx, off);
            double oy = __shfl_down_sync(0xffffffffu, my, off);
            double op = __shfl_down_sync(0xffffffffu, ps, off);
            if (ox > mx) mx = ox;
            if (oy > my) my = oy;
            ps += op;
        }
        int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) {
            red[0][w] = mx;
            red[1][w] = my;
            red[2][w] = ps;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double bx = 0.0, by = 0.0, bp = 0.0;
            for (int q = 0; q < NT / 32; q++) {
                if (red[0][q] > bx) bx = red[0][q];
                if (red[1][q] > by) by = red[1][q];
                bp += red[2][q];
            }
            size_t b = (size_t)ti * tiles_x + tj;
            a.partials[3 * b + 0] = bx;
            a.partials[3 * b + 1] = by;
            a.partials[3 * b + 2] = bp;
        }
    }
}

// Single solve: one CTA per tile.
template <int RECON, bool CHAR, bool WZ, int FLUX>
__global__ void __launch_bounds__(NT, 2) k_stage(StageArgs a) {
    stage_tile<RECON, CHAR, WZ, FLUX>(a, blockIdx.y, blockIdx.x, gridDim.x);
}

template <int RECON, bool CHAR, bool WZ, int FLUX>
cudaError_t launch_one(const StageArgs& a, cudaStream_t s) {
    constexpr size_t bytes = smem_bytes<CHAR>();
    auto kern = k_stage<RECON, CHAR, WZ, FLUX>;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)bytes);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (!a.uout) return cudaSuccess;  // configuration only (before graph capture)
    dim3 grid((a.grid.ny + TY - 1) / TY, (a.grid.nx + TX - 1) / TX);
    kern<<<grid, NT, bytes, s>>>(a);
    return cudaGetLastError();
}

template <int RECON, bool CHAR, bool WZ>
cudaError_t launch_flux(const StageArgs& a, cudaStream_t s) {
    switch (a.num.flux) {
        case FLUX_HLL: return launch_one<RECON, CHAR, WZ, FLUX_HLL>(a, s);
        case FLUX_HLLC: return launch_one<RECON, CHAR, WZ, FLUX_HLLC>(a, s);
        case FLUX_ROE: return launch_one<RECON, CHAR, WZ, FLUX_ROE>(a, s);
        case FLUX_LLF: return launch_one<RECON, CHAR, WZ, FLUX_LLF>(a, s);
        default: return cudaErrorInvalidValue;  // the heat-conduction fluxes: eb2_stage_fp64_hc.cu
    }
}

}  // namespace fp64stage

cudaError_t launch_stage_fp64_w5(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_fp64_tvd(const StageArgs& a, cudaStream_t s);
cudaError_t launch_stage_fp64_g1(const StageArgs& a, cudaStream_t s);

}  // namespace eb2
