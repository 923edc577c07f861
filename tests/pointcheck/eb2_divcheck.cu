// eb2_divcheck.cu -- GPU check of the branch-free divisions (eb2_fdiv.cuh)
// and of the WENO weight routines built on them, bit for bit against the IEEE
// division `/` and against the routines written with `/`.
//
// dc_run(seed, launches, counts) runs `launches` grids of 2^22 random cases and
// accumulates into counts[0..9]:
//   0 rcp_rn(b) != __drcp_rn(b)              b in [2^-1000, 2^1000], all signs,
//                                            significand not all ones
//   1 div_rn(a, b, rcp_rn(b)) != a / b       quotients in [2^-902, 2^902]
//   2 div6_rn(x) != x / 6                    x zero, subnormal or normal, all signs
//   3 weno5_js_rn != weno5_js where the guard holds
//   4 weno5_z_rn  != weno5_z  where the guard holds
//   5 weno3_rn    != weno3    where the guard holds
//   6, 7, 8  WENO cases (JS, Z, 3) whose guard failed (recomputed with `/`)
//   9 divisors with an all-ones significand, which DivGuard::reciprocal
//     must report (they are left out of 0 and 1)
//  10 roe_average_rn != roe_average (any of its ten outputs) where the
//     guard holds, on random left/right primitive states (velocities zero of
//     either sign, subnormal, tiny or O(1))
//  11 Roe averages whose guard failed
//  12 div_rn_tiny(a, b, rcp_rn_any(b)) != a / b   a zero, subnormal or below
//     2^900, |b| in [2^-30, 2^60) (few-bit divisors such as 2 included;
//     quotients at the subnormal/normal boundary included)
//  13 sqrt_rn(x) != sqrt(x)                 x in [2^-900, 2^1000], random and
//     squares of near-midpoints (x = RN(s nextafter(s)) and its neighbours)
// Operands mix random significands with all-ones, near-zero and few-bit
// significands; WENO stencils mix smooth data, jumps, zeros of both signs,
// tiny and huge values, infinities and NaN.
#include <cstdint>
#include <cuda_runtime.h>

#include "eb2_point_fp64.cuh"

using namespace eb2;

namespace {

__device__ __forceinline__ uint64_t mix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Random double with exponent in [emin, emax]; mode 1 gives significands near
// all ones or near zero, mode 2 few significant bits.
__device__ double make(uint64_t r, int mode, int emin, int emax) {
    uint64_t mant = r & ((1ull << 52) - 1);
    const uint64_t sel = (r >> 52) & 0xfff;
    if (mode == 1) {
        const uint64_t small = mant & 0xffff;
        mant = (sel & 1) ? ((1ull << 52) - 1 - small) : small;
    } else if (mode == 2) {
        mant &= ~((1ull << (52 - (sel % 20))) - 1);
    }
    const int e = emin + (int)(mix(r) % (uint64_t)(emax - emin + 1));
    return __longlong_as_double((long long)(((uint64_t)(e + 1023) << 52) | mant));
}

__device__ bool same(double a, double b) {
    return __double_as_longlong(a) == __double_as_longlong(b);
}

// One stencil value: mostly smooth O(1) data, sometimes a jump, a zero, a
// tiny or huge value, an infinity or a NaN.
__device__ double stencil_value(uint64_t r, int n, double base, double slope) {
    const unsigned kind = (unsigned)(r >> 56);
    const double v = base + slope * n;
    if (kind < 150) return v;
    if (kind < 190) return v + make(r, 0, -8, 8);
    if (kind < 205) return (r & 1) ? 0.0 : -0.0;
    if (kind < 225) return make(r, (int)(r % 3), -1074 + 52, -900) * ((r & 2) ? 1 : -1);
    if (kind < 245) return make(r, 0, 100, 700) * ((r & 2) ? 1 : -1);
    if (kind < 250) return (r & 1) ? __longlong_as_double(0x7ff0000000000000ll)
                                   : __longlong_as_double(0xfff0000000000000ll);
    if (kind < 253) return __longlong_as_double(0x7ff8000000000000ll);
    return __longlong_as_double((long long)(r & 0x000fffffffffffffull));   // subnormal
}

__global__ void k_divcheck(uint64_t seed, unsigned long long* counts) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t r1 = mix(seed * 0x100000001b3ull + i), r2 = mix(r1 ^ 0xabcdefull);
    const uint64_t r3 = mix(r2), r4 = mix(r3);
    const int mode_a = (int)(r3 % 3), mode_b = (int)((r3 >> 8) % 3);

    // reciprocal and quotient
    double b = make(r2, mode_b, -450, 450);
    if ((r3 >> 18) & 1) b = -b;
    double a = make(r1, mode_a, -450, 450);
    if ((r3 >> 16) & 1) a = -a;
    if (((r3 >> 20) & 7) == 0) a = b * make(r3, 0, -2, 2);
    const double y = x64::rcp_rn(b);
    x64::DivGuard gb;
    gb.reciprocal(b);
    if (gb.ok()) {
        if (!same(y, __drcp_rn(b))) atomicAdd(&counts[0], 1ull);
        if (!same(x64::div_rn(a, b, y), a / b)) atomicAdd(&counts[1], 1ull);
    } else {
        atomicAdd(&counts[9], 1ull);
    }
    double bw = make(r4, mode_b, -1000, 1000);
    if ((r4 >> 60) & 1) bw = -bw;
    x64::DivGuard gw;
    gw.reciprocal(bw);
    if (gw.ok()) {
        if (!same(x64::rcp_rn(bw), __drcp_rn(bw))) atomicAdd(&counts[0], 1ull);
    } else {
        atomicAdd(&counts[9], 1ull);
    }

    // division by six, and division of tiny dividends
    double x;
    const unsigned xk = (unsigned)((r4 >> 40) & 15);
    if (xk == 0) x = 0.0;
    else if (xk < 6) x = __longlong_as_double((long long)(r3 & 0x000fffffffffffffull) >> (r2 % 50));
    else if (xk < 10) x = make(r3 ^ r1, mode_a, -1022, -900);
    else x = make(r3 ^ r1, mode_a, -900, 1000);
    if ((r1 >> 60) & 1) x = -x;
    if (!same(x64::div6_rn(x), x / 6.0)) atomicAdd(&counts[2], 1ull);
    {
        double bt = ((r4 >> 44) & 7) == 0 ? 2.0 : make(r4 ^ r2, mode_b, -30, 59);
        if ((r4 >> 50) & 1) bt = -bt;
        double xt = ((r4 >> 47) & 1) ? x : x * 0x1p-100;
        // quotients at the subnormal/normal boundary: a = (2^-1022 (1 + e)) b
        if (((r4 >> 53) & 7) == 0)
            xt = 0x1p-1022 * (1.0 + (double)((int)(r1 & 0xff) - 128) * 0x1p-52) * bt;
        if (xt < 0x1p900 && xt > -0x1p900) {
            const double q = x64::div_rn_tiny(xt, bt, x64::rcp_rn_any(bt));
            if (!same(q, xt / bt)) atomicAdd(&counts[12], 1ull);
        }
    }

    // square roots
    {
        double xs;
        const unsigned sk = (unsigned)((r4 >> 52) & 3);
        if (sk == 0) {
            xs = make(r1 ^ r4, mode_a, -900, 999);
        } else {
            const double s0 = make(r2 ^ r4, mode_b, -440, 490);
            const double s1 = __longlong_as_double(__double_as_longlong(s0) + 1);
            xs = __longlong_as_double(__double_as_longlong(s0 * s1) + (long long)sk - 2);
        }
        if (!same(x64::sqrt_rn(xs), sqrt(xs))) atomicAdd(&counts[13], 1ull);
    }

    // WENO stencils
    double v[6];
    const double base = make(r1, 0, -3, 3) * ((r1 & 1) ? 1 : -1);
    const double slope = ((r2 >> 4) & 3) == 0 ? 0.0 : make(r2, 0, -30, 0);
    uint64_t rr = r4;
    for (int n = 0; n < 6; n++) {
        rr = mix(rr);
        v[n] = stencil_value(rr, n, base, slope);
    }
    {
        x64::DivGuard gd;
        const double f = x64::weno5_js_rn(v[0], v[1], v[2], v[3], v[4], gd);
        if (gd.ok()) {
            if (!same(f, x64::weno5_js(v[0], v[1], v[2], v[3], v[4]))) atomicAdd(&counts[3], 1ull);
        } else {
            atomicAdd(&counts[6], 1ull);
        }
    }
    {
        x64::DivGuard gd;
        const double f = x64::weno5_z_rn(v[5], v[4], v[3], v[2], v[1], gd);
        if (gd.ok()) {
            if (!same(f, x64::weno5_z(v[5], v[4], v[3], v[2], v[1]))) atomicAdd(&counts[4], 1ull);
        } else {
            atomicAdd(&counts[7], 1ull);
        }
    }
    {
        // primitive states (rho, u, v, p, H) of two cells, gamma 1.4
        const double gm1 = 0.4;
        double A[5], B[5];
        uint64_t q = r3 ^ r4;
        for (int c = 0; c < 2; c++) {
            double* w = c ? B : A;
            q = mix(q);
            const int wide = (int)(q & 7) == 0;
            const double rho = make(q, 0, wide ? -80 : -6, wide ? 80 : 6);
            q = mix(q);
            const unsigned ku = (unsigned)((q >> 3) & 7);
            const double u = ku == 0 ? ((q & 1) ? 0.0 : -0.0)
                           : ku == 1 ? __longlong_as_double((long long)((q >> 8) & 0xfffffffffull))
                                         * ((q & 2) ? 1 : -1)
                                     : make(q, 0, ku == 2 ? -1020 : -20, ku == 2 ? -900 : 4)
                                         * ((q & 2) ? 1 : -1);
            q = mix(q);
            const unsigned kv = (unsigned)((q >> 3) & 7);
            const double vv = kv == 0 ? ((q & 1) ? 0.0 : -0.0)
                            : kv == 1 ? __longlong_as_double((long long)((q >> 8) & 0xfffffffffull))
                                          * ((q & 2) ? 1 : -1)
                                      : make(q, 0, kv == 2 ? -1020 : -20, kv == 2 ? -900 : 4)
                                          * ((q & 2) ? 1 : -1);
            q = mix(q);
            const double p = make(q, 0, wide ? -80 : -6, wide ? 80 : 6);
            w[0] = rho; w[1] = u; w[2] = vv; w[3] = p;
            w[4] = (p / gm1 + 0.5 * rho * (u * u + vv * vv) + p) / rho;
        }
        x64::DivGuard gd;
        const x64::Roe f = x64::roe_average_rn(A, B, gm1, gd);
        if (gd.ok()) {
            const x64::Roe g = x64::roe_average(A, B, gm1);
            const bool eq = same(f.u, g.u) && same(f.v, g.v) && same(f.H, g.H) && same(f.c, g.c) &&
                            same(f.q2, g.q2) && same(f.b1, g.b1) && same(f.b2, g.b2) &&
                            same(f.ic, g.ic) && same(f.uc, g.uc) && same(f.vc, g.vc);
            if (!eq) atomicAdd(&counts[10], 1ull);
        } else {
            atomicAdd(&counts[11], 1ull);
        }
    }
    {
        x64::DivGuard gd;
        const double f = x64::weno3_rn(v[1], v[2], v[3], gd);
        if (gd.ok()) {
            if (!same(f, x64::weno3(v[1], v[2], v[3]))) atomicAdd(&counts[5], 1ull);
        } else {
            atomicAdd(&counts[8], 1ull);
        }
    }
}

}  // namespace

extern "C" int dc_run(unsigned long long seed, int launches, unsigned long long* counts_host) {
    unsigned long long* counts = nullptr;
    if (cudaMalloc(&counts, 14 * sizeof(unsigned long long)) != cudaSuccess) return 1;
    cudaMemset(counts, 0, 14 * sizeof(unsigned long long));
    const int threads = 256, blocks = (1 << 22) / threads;
    for (int l = 0; l < launches; l++) k_divcheck<<<blocks, threads>>>(seed + 7919ull * l, counts);
    cudaError_t err = cudaDeviceSynchronize();
    if (err == cudaSuccess)
        err = cudaMemcpy(counts_host, counts, 14 * sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost);
    cudaFree(counts);
    return err == cudaSuccess ? 0 : 2;
}
