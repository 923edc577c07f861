// eb2_loop.cuh -- device bodies shared by the single-solve and batched
// kernels: the ghost-cell fill and the end-of-step reduction/time bookkeeping.
// Included by translation units built with -fmad=false (their values must
// match the reference's bits).
#pragma once

#include "eb2_common.cuh"

namespace eb2 {

// Boundary_Conditions (include/Boundary_Condition.h:963-980) and
// BC_DoubleMach_2D (:480-692) for the ghost values e = e0, e0 + stride, ...
// of the four side strips (4 layers x 4 fields x tangential extent).  Only
// non-corner ghosts are written: no stencil, eigenvector or flux ever reads a
// corner ghost, and with at least 4 interior cells behind a mirrored or
// periodic side every source is an interior cell, so the four sides are
// independent (the reference's L, R, B, T order only matters for corners).
__device__ __forceinline__ void bc_fill(double* __restrict__ u, const Grid& g, const Boundary& b,
                                        double t, long long e0, long long stride) {
    const int rows = g.rows, cols = g.cols, nx = g.nx, ny = g.ny;
    const long long nlr = 16LL * ny, nbt = 16LL * nx;
    const long long total = 2 * nlr + 2 * nbt;
    for (long long e = e0; e < total; e += stride) {
        int side;
        long long q;
        if (e < 2 * nlr) { side = (int)(e / nlr); q = e - side * nlr; }
        else { long long f = e - 2 * nlr; side = 2 + (int)(f / nbt); q = f - (side - 2) * nbt; }
        const int km = (int)(q & 15);
        const int tpos = GC + (int)(q >> 4);    // tangential index (j for L/R, i for B/T)
        const int k = km & 3, m = km >> 2;      // field, ghost layer (0 = next to the wall)
        const bool lr = side < 2;
        const int nlen = lr ? rows : cols;
        const int ghost = (side == 0 || side == 2) ? GC - 1 - m : nlen - GC + m;
        const int normal = lr ? 1 : 2;
        int src = -1;
        double cval = 0.0, sgn = 1.0;
        if (b.dmr) {
            // BC_DoubleMach_2D constants (Boundary_Condition.h:483-513)
            const double gm = 1.4, x0 = 1.0 / 6.0;
            const double post[4] = {8.0, 8.0 * 7.1447, 8.0 * -4.125,
                                    116.5 / (gm - 1.0) + 0.5 * 8.0 * (7.1447 * 7.1447 + -4.125 * -4.125)};
            const double pre[4] = {1.4, 1.4 * 0.0, 1.4 * 0.0,
                                   1.0 / (gm - 1.0) + 0.5 * 1.4 * (0.0 * 0.0 + 0.0 * 0.0)};
            const double xnx = rows - 2 * GC;
            if (side == 0) {
                cval = post[k];
            } else if (side == 1) {
                src = rows - GC - 1;
            } else {
                double xp = (double)(tpos + 0.5 - GC) / xnx * 4.0;
                if (side == 2) {
                    if (xp > x0) { src = GC + m; if (k == 2) sgn = -1.0; }
                    else cval = post[k];
                } else {
                    double xs = x0 + (1.0 / sqrt(3.0)) + (20.0 * t / sqrt(3.0));
                    cval = xp < xs ? post[k] : pre[k];
                }
            }
        } else {
            switch (b.kind[side]) {
                case BC_OUTFLOW:
                    src = (side == 0 || side == 2) ? GC : nlen - GC - 1;
                    break;
                case BC_PERIODIC:
                    src = (side == 0 || side == 2) ? nlen - GC - 1 - m : GC + m;
                    break;
                case BC_REFLECT:
                    // left and top mirror four layers (:356-374, :443-461); right
                    // and bottom copy the wall cell (:393-407, :427-441)
                    if (side == 0) src = GC + m;
                    else if (side == 3) src = nlen - GC - 1 - m;
                    else if (side == 1) src = nlen - GC - 1;
                    else src = GC;
                    if (k == normal) sgn = -1.0;
                    break;
                case BC_INFLOW:
                    cval = b.inflow[k];
                    break;
                default:
                    cval = b.fixed[side][k];
                    break;
            }
        }
        double val;
        if (src >= 0) {
            double sv = lr ? u[at(k, src, tpos, rows, cols)] : u[at(k, tpos, src, rows, cols)];
            val = sgn < 0.0 ? -sv : sv;
        } else {
            val = cval;
        }
        if (lr) u[at(k, ghost, tpos, rows, cols)] = val;
        else u[at(k, tpos, ghost, rows, cols)] = val;
    }
}

// Block reduction of (max, max, sum) in a fixed order; the result is in
// thread 0.  red: 96 doubles of shared memory.
__device__ __forceinline__ void block_reduce3(double& mx, double& my, double& ps, double* red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        double ox = __shfl_down_sync(0xffffffffu, mx, off);
        double oy = __shfl_down_sync(0xffffffffu, my, off);
        double op = __shfl_down_sync(0xffffffffu, ps, off);
        if (ox > mx) mx = ox;
        if (oy > my) my = oy;
        ps += op;
    }
    int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w] = mx;
        red[32 + w] = my;
        red[64 + w] = ps;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bx = 0.0, by = 0.0, bp = 0.0;
        for (int q = 0; q < nw; q++) {
            if (red[q] > bx) bx = red[q];
            if (red[32 + q] > by) by = red[32 + q];
            bp += red[64 + q];
        }
        mx = bx;
        my = by;
        ps = bp;
    }
}

// Reduce the wave-speed partials and advance the device copy of the host
// time loop of src/RP_FVM.c:179-267.  mode 0: CFL time step only; mode 1:
// start of a loop; mode 2: end of a step.  Call with the whole block.
__device__ __forceinline__ void finalize_body(Ctrl* c, const double* __restrict__ partials,
                                              int nblocks, int ncells, int mode, double* red) {
    if (mode == 2 && !c->active) return;
    double mx = 0.0, my = 0.0, ps = 0.0;
    // each thread combines partials b, b + blockDim.x, ... in that order; the
    // loads of eight of them are issued before they are combined
    const int step = blockDim.x;
    int b = threadIdx.x;
    for (; b + 7 * step < nblocks; b += 8 * step) {
        double a[8][3];
#pragma unroll
        for (int u = 0; u < 8; u++)
#pragma unroll
            for (int k = 0; k < 3; k++) a[u][k] = partials[3 * (b + u * step) + k];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            if (a[u][0] > mx) mx = a[u][0];
            if (a[u][1] > my) my = a[u][1];
            ps += a[u][2];
        }
    }
    for (; b < nblocks; b += step) {
        double a0 = partials[3 * b], a1 = partials[3 * b + 1];
        if (a0 > mx) mx = a0;
        if (a1 > my) my = a1;
        ps += partials[3 * b + 2];
    }
    block_reduce3(mx, my, ps, red);
    if (threadIdx.x != 0) return;
    c->sx = mx;
    c->sy = my;
    c->pmean = ps / ncells;
    // dt = CFL * min(dx, dy) / (max|u|+a + max|v|+a)
    double dt = c->cfl * c->dmin / (mx + my);
    if (mode == 0) {
        c->dt = dt;
        return;
    }
    if (mode == 2) {
        double now = c->t + c->dt;
        if (fabs(now - c->next_out) < 1e-10 * c->out_dt) {
            c->out_pending = 1;
            c->next_out += c->out_dt;
        }
        c->t = now;
        c->step += 1;
    }
    if (c->t + dt > c->next_out) dt = c->next_out - c->t;
    if (c->t + dt >= c->tmax) dt = c->tmax - c->t;
    c->dt = dt;
    if (!(dt > 0.0) || isinf(dt)) {
        if (c->t < c->tmax) c->status |= ST_BAD_DT;
    }
    c->active = (c->t < c->tmax) && !c->out_pending && !(c->status & ST_BAD_DT) &&
                c->step < c->max_step;
}

}  // namespace eb2
