// eb2_aux.cu -- boundary fill, initial states, CFL reduction, device time-loop
// bookkeeping and the granular reference entry points (one thread per cell or
// interface).  Built with -fmad=false: every value here must match the
// reference's bits (see eb2_point_fp64.cuh).
#include "eb2_kernels.h"
#include "eb2_loop.cuh"
#include "eb2_point_fp64.cuh"

namespace eb2 {

namespace {
constexpr int NT = 256;

inline int blocks_for(long long n, int nt = NT) {
    long long b = (n + nt - 1) / nt;
    return (int)(b < 1 ? 1 : (b > 65535LL * 32 ? 65535LL * 32 : b));
}
}  // namespace

// Ghost-cell fill (body in eb2_loop.cuh).
__global__ void k_bc(double* __restrict__ u, Grid g, Boundary b, const Ctrl* ctrl,
                     double time) {
    if (ctrl && !ctrl->active) return;
    bc_fill(u, g, b, ctrl ? ctrl->t : time, blockIdx.x * (long long)blockDim.x + threadIdx.x,
            (long long)gridDim.x * blockDim.x);
}

cudaError_t launch_bc(double* u, const Grid& g, const Boundary& b, const Ctrl* ctrl,
                      double time, cudaStream_t s) {
    long long total = 32LL * g.ny + 32LL * g.nx;
    k_bc<<<blocks_for(total), NT, 0, s>>>(u, g, b, ctrl, time);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Initial states: the case initialisers of include/initialize.h write
// primitives, then initEulerconser2D (:1389-1405) converts the whole array.
// ---------------------------------------------------------------------------
__global__ void k_init(double* __restrict__ u, Grid g, Gas gas, InitDesc d,
                       const double* __restrict__ column, double* __restrict__ pri,
                       double* __restrict__ fx, double* __restrict__ gy) {
    const int rows = g.rows, cols = g.cols;
    const long long n = (long long)rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e / cols), j = (int)(e - (long long)i * cols);
        bool inside = i >= GC && i < rows - GC && j >= GC && j < cols - GC;
        bool fill = d.full || inside;
        double w[4] = {0.0, 0.0, 0.0, 0.0};
        const double* st = nullptr;
        switch (d.kind) {
            case INIT_UNIFORM: if (fill) st = d.st[0]; break;
            case INIT_HALF_X: if (fill) st = i < rows / 2 ? d.st[0] : d.st[1]; break;
            case INIT_QUADRANT:
                // the if-chain order of initEulerpri2D_Shocktube1..5 (:366-391)
                if (fill) st = d.st[(i >= rows / 2 ? 2 : 0) + (j >= cols / 2 ? 1 : 0)];
                break;
            case INIT_DMR:
                // initEulerpri2D_DoubleMachReflection (:925-952): st[0] post, st[1] pre
                if (inside) {
                    double nxd = rows - 2 * GC, nyd = cols - 2 * GC;
                    double xp = (double)(i + 0.5 - GC) / nxd * d.lx;
                    double yp = (double)(j + 0.5 - GC) / nyd * d.ly;
                    st = yp < sqrt(3.0) * (xp - 1.0 / 6.0) ? d.st[1] : d.st[0];
                }
                break;
            case INIT_FIELD:
                // a field evaluated on the host (eb2_cases.cu), every cell
                for (int k = 0; k < 4; k++) w[k] = column[at(k, i, j, rows, cols)];
                break;
            case INIT_SINE:
                // initEulerpri1D_PrecisionTest (:52-57): column GC only; the
                // densities 1 + 0.2 sin(x) come in from the host's libm
                if (inside && j == GC) {
                    w[0] = column[i - GC];
                    w[1] = 1.0;
                    w[2] = 0.0;
                    w[3] = 1.0;
                }
                break;
            default: break;
        }
        if (st) {
            w[0] = st[0]; w[1] = st[1]; w[2] = st[2]; w[3] = st[3];
        }
        double r = w[0], uu = w[1], vv = w[2], p = w[3];
        double q[4] = {r, uu * r, vv * r, p / gas.gm1 + 0.5 * r * (uu * uu + vv * vv)};
        for (int k = 0; k < 4; k++) u[at(k, i, j, rows, cols)] = q[k];
        if (pri)
            for (int k = 0; k < 4; k++) pri[at(k, i, j, rows, cols)] = w[k];
        if (fx) {
            // initEulerflux2D (:1409-1434), from the conserved values (0/0 in
            // cells the case leaves empty, as there)
            double cu = q[1] / q[0], cv = q[2] / q[0];
            double cp = (q[3] - 0.5 * r * (cu * cu + cv * cv)) * gas.gm1;
            fx[at(0, i, j, rows, cols)] = r * cu;
            fx[at(1, i, j, rows, cols)] = r * cu * cu + cp;
            fx[at(2, i, j, rows, cols)] = r * cu * cv;
            fx[at(3, i, j, rows, cols)] = (q[3] + cp) * cu;
            gy[at(0, i, j, rows, cols)] = r * cv;
            gy[at(1, i, j, rows, cols)] = r * cu * cv;
            gy[at(2, i, j, rows, cols)] = r * cv * cv + cp;
            gy[at(3, i, j, rows, cols)] = (q[3] + cp) * cv;
        }
    }
}

cudaError_t launch_init(double* u, const Grid& g, const Gas& gas, const InitDesc& d,
                        cudaStream_t s, double* pri, double* fx, double* gy) {
    const double* column = nullptr;
    double* dcol = nullptr;
    if (d.kind == INIT_FIELD) {
        // libm (or rand) initialisers: the host evaluates the reference's
        // expressions with the reference's C library, the GPU converts
        size_t bytes = (size_t)4 * g.rows * g.cols * sizeof(double);
        double* h = (double*)calloc((size_t)4 * g.rows * g.cols, sizeof(double));
        if (!h) return cudaErrorMemoryAllocation;
        if (!host_case_field(d.field_case, g.rows, g.cols, gas.gamma, d.lx, d.ly, h)) {
            free(h);
            return cudaErrorInvalidValue;
        }
        cudaError_t e = cudaMallocAsync(&dcol, bytes, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dcol, h, bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        free(h);
        if (e != cudaSuccess) return e;
        column = dcol;
    } else if (d.kind == INIT_SINE) {
        // the sine column is evaluated with the host libm, as the reference
        // does, so the initial state matches it bit for bit
        size_t bytes = (size_t)g.nx * sizeof(double);
        double* h = (double*)malloc(bytes);
        if (!h) return cudaErrorMemoryAllocation;
        double dx = d.lx / g.nx;
        for (int i = GC; i < g.rows - GC; i++) h[i - GC] = 1.0 + 0.2 * sin((i - GC + 0.5) * dx);
        cudaError_t e = cudaMallocAsync(&dcol, bytes, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dcol, h, bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        free(h);
        if (e != cudaSuccess) return e;
        column = dcol;
    }
    long long n = (long long)g.rows * g.cols;
    k_init<<<blocks_for(n), NT, 0, s>>>(u, g, gas, d, column, pri, fx, gy);
    cudaError_t e = cudaGetLastError();
    if (dcol) cudaFreeAsync(dcol, s);
    return e;
}

// ---------------------------------------------------------------------------
// CFL reduction (Get_Delta_T_2D, include/function.h:144-175).  Max is order
// independent; the pressure sum (used by the mixed form's near-vacuum test)
// is reduced in a fixed order, so both are deterministic.
// ---------------------------------------------------------------------------
__global__ void k_wave_partials(const double* __restrict__ u, Grid g, Gas gas,
                                double* __restrict__ partials) {
    __shared__ double red[96];
    const int rows = g.rows, cols = g.cols;
    const long long n = (long long)g.nx * g.ny;
    double mx = 0.0, my = 0.0, ps = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        int i = GC + (int)(e / g.ny), j = GC + (int)(e - (e / g.ny) * g.ny);
        double r = u[at(0, i, j, rows, cols)];
        double uu = u[at(1, i, j, rows, cols)] / r;
        double vv = u[at(2, i, j, rows, cols)] / r;
        double p = (u[at(3, i, j, rows, cols)] - 0.5 * r * (uu * uu + vv * vv)) * gas.gm1;
        double c = sqrt(gas.gamma * p / r);
        double lx = fabs(uu) + c, ly = fabs(vv) + c;
        if (lx > mx) mx = lx;
        if (ly > my) my = ly;
        ps += p;
    }
    block_reduce3(mx, my, ps, red);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x + 0] = mx;
        partials[3 * blockIdx.x + 1] = my;
        partials[3 * blockIdx.x + 2] = ps;
    }
}

cudaError_t launch_wave_partials(const double* u, const Grid& g, const Gas& gas,
                                 double* partials, int* nblocks, cudaStream_t s) {
    int nb = 296;  // 2 blocks per SM on a 148-SM B200; fixed, so the sum is deterministic
    long long n = (long long)g.nx * g.ny;
    if (n < (long long)nb * NT) nb = blocks_for(n);
    *nblocks = nb;
    k_wave_partials<<<nb, NT, 0, s>>>(u, g, gas, partials);
    return cudaGetLastError();
}

// End-of-step reduction and time bookkeeping (body in eb2_loop.cuh).
__global__ void __launch_bounds__(FINALIZE_THREADS) k_finalize(Ctrl* c, const double* __restrict__ partials, int nblocks,
                           int ncells, int mode) {
    __shared__ double red[96];
    finalize_body(c, partials, nblocks, ncells, mode, red);
}

cudaError_t launch_finalize(Ctrl* ctrl, const double* partials, int nblocks, int ncells,
                            int mode, cudaStream_t s) {
    k_finalize<<<1, FINALIZE_THREADS, 0, s>>>(ctrl, partials, nblocks, ncells, mode);
    return cudaGetLastError();
}

__global__ void k_copy_interior(double* __restrict__ dst, const double* __restrict__ src,
                                Grid g) {
    const long long n = 4LL * g.nx * g.ny;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        long long plane = (long long)g.nx * g.ny;
        int k = (int)(e / plane);
        long long r = e - k * plane;
        int i = GC + (int)(r / g.ny), j = GC + (int)(r % g.ny);
        size_t o = at(k, i, j, g.rows, g.cols);
        dst[o] = src[o];
    }
}

cudaError_t launch_copy_interior(double* dst, const double* src, const Grid& g, cudaStream_t s) {
    k_copy_interior<<<blocks_for(4LL * g.nx * g.ny), NT, 0, s>>>(dst, src, g);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Granular reference entry points.
// ---------------------------------------------------------------------------
// Con_to_Pri_2D on the box [GC-1, rows-GC]^2 (include/initialize.h:1437-1454)
__global__ void k_con_to_pri(const double* __restrict__ u, double* __restrict__ pri, Grid g,
                             Gas gas) {
    const int rows = g.rows, cols = g.cols;
    const int w = cols - 2 * GC + 2, h = rows - 2 * GC + 2;
    const long long n = (long long)w * h;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        int i = GC - 1 + (int)(e / w), j = GC - 1 + (int)(e % w);
        double q[5];
        x64::primitive5(u[at(0, i, j, rows, cols)], u[at(1, i, j, rows, cols)],
                        u[at(2, i, j, rows, cols)], u[at(3, i, j, rows, cols)], gas, q);
        for (int k = 0; k < 4; k++) pri[at(k, i, j, rows, cols)] = q[k];
    }
}

cudaError_t launch_con_to_pri(const double* u, double* pri, const Grid& g, const Gas& gas,
                              cudaStream_t s) {
    long long n = (long long)(g.nx + 2) * (g.ny + 2);
    k_con_to_pri<<<blocks_for(n), NT, 0, s>>>(u, pri, g, gas);
    return cudaGetLastError();
}

// interface ranges of the reference's x and y loops
__device__ __forceinline__ void face_range(int dir, const Grid& g, int& i0, int& ni, int& j0,
                                           int& nj, bool eigen) {
    if (dir == 1) { i0 = GC - 1; ni = g.nx + 1; j0 = GC; nj = g.ny; }
    else { i0 = GC; ni = g.nx; j0 = GC - 1; nj = g.ny + (eigen ? 2 : 1); }
}

// Compute_Eigen_2DX / _2DY (include/Characteriz.h:300-500): eig_l[k][m][i][j],
// eig_r[m][k][i][j] from a primitive array.
template <int DIR>
__global__ void k_eigen(const double* __restrict__ pri, double* __restrict__ el,
                        double* __restrict__ er, Grid g, Gas gas) {
    int i0, ni, j0, nj;
    face_range(DIR, g, i0, ni, j0, nj, true);
    const int rows = g.rows, cols = g.cols;
    const size_t plane = (size_t)rows * cols;
    const long long n = (long long)ni * nj;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        int i = i0 + (int)(e / nj), j = j0 + (int)(e % nj);
        int ib = DIR == 1 ? i + 1 : i, jb = DIR == 1 ? j : j + 1;
        double A[5], B[5];
        for (int k = 0; k < 4; k++) {
            A[k] = pri[at(k, i, j, rows, cols)];
            B[k] = pri[at(k, ib, jb, rows, cols)];
        }
        A[4] = 0.5 * (A[1] * A[1] + A[2] * A[2]) + gas.gr * (A[3] / A[0]);
        B[4] = 0.5 * (B[1] * B[1] + B[2] * B[2]) + gas.gr * (B[3] / B[0]);
        x64::Roe r = x64::roe_average(A, B, gas.gm1);
        for (int k = 0; k < 4; k++) {
            double l[4], rr[4];
            x64::left_row<DIR>(r, k, l);
            x64::right_row<DIR>(r, k, rr);
            for (int m = 0; m < 4; m++) {
                el[(size_t)(k * 4 + m) * plane + (size_t)i * cols + j] = l[m];
                er[(size_t)(k * 4 + m) * plane + (size_t)i * cols + j] = rr[m];
            }
        }
    }
}

cudaError_t launch_eigen(int dir, const double* pri, double* el, double* er, const Grid& g,
                         const Gas& gas, cudaStream_t s) {
    long long n = (long long)(g.nx + 2) * (g.ny + 2);
    if (dir == 1) k_eigen<1><<<blocks_for(n), NT, 0, s>>>(pri, el, er, g, gas);
    else k_eigen<2><<<blocks_for(n), NT, 0, s>>>(pri, el, er, g, gas);
    return cudaGetLastError();
}

// One interface of WENO5_Reconstruction / TVD_Reconstruction /
// Reconstruction_Godunov (include/Reconstruction.h) read straight from the
// state in global memory.
template <int DIR, int RECON, bool CHAR, bool WZ>
__device__ void recon_face(const double* __restrict__ u, int i, int j, const Grid& g,
                           const Gas& gas, double* ql, double* qr) {
    const int rows = g.rows, cols = g.cols;
    const double delta = DIR == 1 ? g.dx : g.dy;
    auto cell = [&](int k, int n) {
        return DIR == 1 ? u[at(k, i - 2 + n, j, rows, cols)] : u[at(k, i, j - 2 + n, rows, cols)];
    };
    constexpr int N0 = RECON == 5 ? 0 : (RECON == 2 || RECON == 3 ? 1 : 2);
    constexpr int N1 = RECON == 5 ? 6 : (RECON == 2 || RECON == 3 ? 5 : 4);
    if (!CHAR) {
        for (int k = 0; k < 4; k++) {
            double q6[6];
            for (int n = N0; n < N1; n++) q6[n] = cell(k, n);
            x64::recon_pair<RECON, false, false>(q6, delta, ql[k], qr[k]);
        }
        return;
    }
    double A[5], B[5];
    x64::primitive5(cell(0, 2), cell(1, 2), cell(2, 2), cell(3, 2), gas, A);
    x64::primitive5(cell(0, 3), cell(1, 3), cell(2, 3), cell(3, 3), gas, B);
    x64::Roe e = x64::roe_average(A, B, gas.gm1);
    double wm[4], wp[4];
    for (int k = 0; k < 4; k++) {
        double l[4];
        x64::left_row<DIR>(e, k, l);
        double q6[6];
        for (int n = N0; n < N1; n++) {
            double acc = 0.0;
            for (int m = 0; m < 4; m++) acc += cell(m, n) * l[m];
            q6[n] = acc;
        }
        x64::recon_pair<RECON, WZ, true>(q6, delta, wm[k], wp[k]);
    }
    for (int m = 0; m < 4; m++) {
        double r[4];
        x64::right_row<DIR>(e, m, r);
        double sl = 0.0, sr = 0.0;
        for (int k = 0; k < 4; k++) {
            sl += wm[k] * r[k];
            sr += wp[k] * r[k];
        }
        ql[m] = sl;
        qr[m] = sr;
    }
}

template <int DIR, int RECON, bool CHAR, bool WZ>
__global__ void k_recon(const double* __restrict__ u, double* __restrict__ ql,
                        double* __restrict__ qr, Grid g, Gas gas) {
    int i0, ni, j0, nj;
    face_range(DIR, g, i0, ni, j0, nj, false);
    const long long n = (long long)ni * nj;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        int i = i0 + (int)(e / nj), j = j0 + (int)(e % nj);
        double a[4], b[4];
        recon_face<DIR, RECON, CHAR, WZ>(u, i, j, g, gas, a, b);
        for (int k = 0; k < 4; k++) {
            ql[at(k, i, j, g.rows, g.cols)] = a[k];
            qr[at(k, i, j, g.rows, g.cols)] = b[k];
        }
    }
}

template <int DIR>
static cudaError_t recon_dispatch(const double* u, double* ql, double* qr, const Grid& g,
                                  const Gas& gas, const Numerics& nm, cudaStream_t s) {
    long long n = (long long)(g.nx + 1) * (g.ny + 1);
    int nb = blocks_for(n);
    bool ch = nm.characteristic != 0, wz = nm.weno_z != 0;
    switch (nm.recon) {
        case 5:
            if (!ch) k_recon<DIR, 5, false, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            else if (wz) k_recon<DIR, 5, true, true><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            else k_recon<DIR, 5, true, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            break;
        case 3:
            if (ch) k_recon<DIR, 3, true, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            else k_recon<DIR, 3, false, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            break;
        case 2:
            if (ch) k_recon<DIR, 2, true, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            else k_recon<DIR, 2, false, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            break;
        case 1:
            if (ch) k_recon<DIR, 1, true, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            else k_recon<DIR, 1, false, false><<<nb, NT, 0, s>>>(u, ql, qr, g, gas);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_recon(int dir, const double* u, double* ql, double* qr, const Grid& g,
                         const Gas& gas, const Numerics& n, unsigned* status, cudaStream_t s) {
    (void)status;
    return dir == 1 ? recon_dispatch<1>(u, ql, qr, g, gas, n, s)
                    : recon_dispatch<2>(u, ql, qr, g, gas, n, s);
}

// HLL_Flux / HLLC_Flux / Roe_Flux / LLF_Flux over the reference's interface
// range; HLL leaves skipped interfaces untouched, as the reference does.
template <int DIR, int FLUX>
__global__ void k_riemann(const double* __restrict__ ql, const double* __restrict__ qr,
                          double* __restrict__ f, Grid g, Gas gas, unsigned* status) {
    int i0, ni, j0, nj;
    face_range(DIR, g, i0, ni, j0, nj, false);
    const long long n = (long long)ni * nj;
    unsigned st = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        int i = i0 + (int)(e / nj), j = j0 + (int)(e % nj);
        double a[4], b[4], F[4];
        for (int k = 0; k < 4; k++) {
            a[k] = ql[at(k, i, j, g.rows, g.cols)];
            b[k] = qr[at(k, i, j, g.rows, g.cols)];
        }
        if (x64::riemann<FLUX, DIR>(a, b, gas, F)) {
            for (int k = 0; k < 4; k++) f[at(k, i, j, g.rows, g.cols)] = F[k];
        } else {
            st |= ST_NONPHYSICAL;
        }
    }
    if (st && status) atomicOr(status, st);
}

template <int DIR>
static cudaError_t riemann_dispatch(const double* ql, const double* qr, double* f,
                                    const Grid& g, const Gas& gas, int flux, unsigned* status,
                                    cudaStream_t s) {
    int nb = blocks_for((long long)(g.nx + 1) * (g.ny + 1));
    switch (flux) {
        case FLUX_HLL: k_riemann<DIR, FLUX_HLL><<<nb, NT, 0, s>>>(ql, qr, f, g, gas, status); break;
        case FLUX_HLLC: k_riemann<DIR, FLUX_HLLC><<<nb, NT, 0, s>>>(ql, qr, f, g, gas, status); break;
        case FLUX_ROE: k_riemann<DIR, FLUX_ROE><<<nb, NT, 0, s>>>(ql, qr, f, g, gas, status); break;
        case FLUX_HLLHC: k_riemann<DIR, FLUX_HLLHC><<<nb, NT, 0, s>>>(ql, qr, f, g, gas, status); break;
        case FLUX_HLLCHC: k_riemann<DIR, FLUX_HLLCHC><<<nb, NT, 0, s>>>(ql, qr, f, g, gas, status); break;
        case FLUX_ROEHC: k_riemann<DIR, FLUX_ROEHC><<<nb, NT, 0, s>>>(ql, qr, f, g, gas, status); break;
        default: k_riemann<DIR, FLUX_LLF><<<nb, NT, 0, s>>>(ql, qr, f, g, gas, status); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_riemann(int dir, const double* ql, const double* qr, double* f,
                           const Grid& g, const Gas& gas, int flux, unsigned* status,
                           cudaStream_t s) {
    return dir == 1 ? riemann_dispatch<1>(ql, qr, f, g, gas, flux, status, s)
                    : riemann_dispatch<2>(ql, qr, f, g, gas, flux, status, s);
}

// Space_Discrete_Item (include/scheme.h:3758-3777) with the gravity source of
// Source_Gravity (:3723-3751) taken from u when n.source is set.
__global__ void k_space_item(const double* __restrict__ f, const double* __restrict__ gf,
                             const double* __restrict__ s, const double* __restrict__ u,
                             double* __restrict__ lout, Grid g, Numerics nm) {
    const int rows = g.rows, cols = g.cols;
    const long long n = (long long)g.nx * g.ny;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        int i = GC + (int)(e / g.ny), j = GC + (int)(e % g.ny);
        double src[4] = {0.0, 0.0, 0.0, 0.0};
        if (s) {
            for (int k = 0; k < 4; k++) src[k] = s[at(k, i, j, rows, cols)];
        } else if (nm.source) {
            double rho = u[at(0, i, j, rows, cols)];
            double v = u[at(2, i, j, rows, cols)] / rho;
            src[2] = rho * nm.gravity;
            src[3] = rho * nm.gravity * v;
        }
        for (int k = 0; k < 4; k++)
            lout[at(k, i, j, rows, cols)] =
                -(f[at(k, i, j, rows, cols)] - f[at(k, i - 1, j, rows, cols)]) * g.inv_dx
                - (gf[at(k, i, j, rows, cols)] - gf[at(k, i, j - 1, rows, cols)]) * g.inv_dy
                + src[k];
    }
}

cudaError_t launch_space_item(const double* f, const double* gflux, const double* src,
                              const double* u, double* lout, const Grid& g, const Numerics& n,
                              cudaStream_t s) {
    k_space_item<<<blocks_for((long long)g.nx * g.ny), NT, 0, s>>>(f, gflux, src, u, lout, g, n);
    return cudaGetLastError();
}

}  // namespace eb2

// ---------------------------------------------------------------------------
// The backward-step flow's two-block step (RK1_TimeAd_BS,
// include/time_advance.h:886-1025): block 1 is the channel above the step,
// block 2 the inlet section beside it; each is a [4][rows][cols] array of its
// own with 4 ghost layers.
// ---------------------------------------------------------------------------
namespace eb2 {
namespace {

// Interiors of both blocks from U (block 1 starts `off` columns in), the
// rest of each block zero, as the reference starts its block arrays.
__global__ void k_bs_gather(const double* __restrict__ u, Grid g, double* __restrict__ b1,
                            Grid g1, double* __restrict__ b2, Grid g2, int off) {
    const long long n1 = 4LL * g1.rows * g1.cols, n = n1 + 4LL * g2.rows * g2.cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const bool first = e < n1;
        const Grid& b = first ? g1 : g2;
        const long long r = first ? e : e - n1;
        const long long plane = (long long)b.rows * b.cols;
        const int k = (int)(r / plane);
        const int i = (int)((r - k * plane) / b.cols), j = (int)(r - k * plane - (long long)i * b.cols);
        double v = 0.0;
        if (i >= GC && i < b.rows - GC && j >= GC && j < b.cols - GC)
            v = u[at(k, i, j + (first ? off : 0), g.rows, g.cols)];
        (first ? b1 : b2)[r] = v;
    }
}

// Ghost layers of both blocks by the rules of BC_BackwardStep_2D
// (include/Boundary_Condition.h:696-850): inflow on both blocks' left sides,
// zero-gradient outflow on block 1's right, reflecting walls (the normal
// momentum mirrored with its sign flipped) below and above block 1, below
// block 2 and on block 2's right (the step face), and where the blocks meet
// block 2's top ghosts from block 1's first interior columns and block 1's
// bottom ghosts from block 2's last ones (that exchange is the last write of
// the reference, so it wins over the wall rule on block 1's bottom).  Every
// ghost value is a copy of an interior value or the inflow state, so one
// thread per ghost element gives the reference's values in any order.
// Corners stay as they are: no stencil reads them.
__global__ void k_bs_boundary(double* __restrict__ b1, Grid g1, double* __restrict__ b2,
                              Grid g2, Boundary inflow) {
    // per block and field: 4 sides x GC layers x (rows or cols) candidates
    const int per1 = 2 * GC * (g1.rows + g1.cols), per2 = 2 * GC * (g2.rows + g2.cols);
    const long long n = 4LL * (per1 + per2);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const bool first = e < 4LL * per1;
        const long long r = first ? e : e - 4LL * per1;
        const Grid& b = first ? g1 : g2;
        double* x = first ? b1 : b2;
        const int per = first ? per1 : per2;
        const int k = (int)(r / per);
        int q = (int)(r - (long long)k * per);
        const int R = b.rows, C = b.cols;
        // sides: 0 left (i < GC), 1 right (i >= R-GC) over interior j;
        //        2 bottom (j < GC), 3 top (j >= C-GC) over interior i
        int side, m, t;
        if (q < 2 * GC * C) {
            side = q / (GC * C);
            q -= side * GC * C;
            m = q / C;
            t = q - m * C;
            if (t < GC || t >= C - GC) continue;
        } else {
            q -= 2 * GC * C;
            side = 2 + q / (GC * R);
            q -= (side - 2) * GC * R;
            m = q / R;
            t = q - m * R;
            if (t < GC || t >= R - GC) continue;
        }
        double v;
        int i, j;
        if (side == 0) {            // inflow
            i = m;
            j = t;
            v = inflow.inflow[k];
        } else if (side == 1) {     // block 1: outflow; block 2: the step face, a wall
            i = R - GC + m;
            j = t;
            if (first) {
                v = x[at(k, R - GC - 1, j, R, C)];
            } else {
                v = x[at(k, R - GC - 1 - m, j, R, C)];
                if (k == 1) v = -v;
            }
        } else if (side == 2) {     // bottom: wall, or block 2's last columns
            i = t;
            j = m;
            if (first && i < g2.rows - GC) {
                v = b2[at(k, i, g2.cols - 2 * GC + m, g2.rows, g2.cols)];
            } else {
                v = x[at(k, i, 2 * GC - 1 - m, R, C)];
                if (k == 2) v = -v;
            }
        } else {                    // top: block 1 wall; block 2 from block 1
            i = t;
            j = C - GC + m;
            if (first) {
                v = x[at(k, i, C - GC - 1 - m, R, C)];
                if (k == 2) v = -v;
            } else {
                v = b1[at(k, i, GC + m, g1.rows, g1.cols)];
            }
        }
        x[at(k, i, j, R, C)] = v;
    }
}

// Interiors of both blocks back into U.
__global__ void k_bs_scatter(double* __restrict__ u, Grid g, const double* __restrict__ b1,
                             Grid g1, const double* __restrict__ b2, Grid g2, int off) {
    const long long n1 = 4LL * g1.nx * g1.ny, n = n1 + 4LL * g2.nx * g2.ny;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const bool first = e < n1;
        const Grid& b = first ? g1 : g2;
        const long long r = first ? e : e - n1;
        const long long plane = (long long)b.nx * b.ny;
        const int k = (int)(r / plane);
        const int i = GC + (int)((r - k * plane) / b.ny);
        const int j = GC + (int)(r - k * plane - (long long)(i - GC) * b.ny);
        u[at(k, i, j + (first ? off : 0), g.rows, g.cols)] =
            (first ? b1 : b2)[at(k, i, j, b.rows, b.cols)];
    }
}

}  // namespace

cudaError_t launch_bs_gather(const double* u, const Grid& g, double* b1, const Grid& g1,
                             double* b2, const Grid& g2, int off, cudaStream_t s) {
    const long long n = 4LL * g1.rows * g1.cols + 4LL * g2.rows * g2.cols;
    k_bs_gather<<<blocks_for(n), NT, 0, s>>>(u, g, b1, g1, b2, g2, off);
    return cudaGetLastError();
}

cudaError_t launch_bs_boundary(double* b1, const Grid& g1, double* b2, const Grid& g2,
                               const Boundary& inflow, cudaStream_t s) {
    const long long n = 4LL * 2 * GC * (g1.rows + g1.cols + g2.rows + g2.cols);
    k_bs_boundary<<<blocks_for(n), NT, 0, s>>>(b1, g1, b2, g2, inflow);
    return cudaGetLastError();
}

cudaError_t launch_bs_scatter(double* u, const Grid& g, const double* b1, const Grid& g1,
                              const double* b2, const Grid& g2, int off, cudaStream_t s) {
    const long long n = 4LL * g1.nx * g1.ny + 4LL * g2.nx * g2.ny;
    k_bs_scatter<<<blocks_for(n), NT, 0, s>>>(u, g, b1, g1, b2, g2, off);
    return cudaGetLastError();
}

}  // namespace eb2
