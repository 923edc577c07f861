// eb2_divcheck.cu -- GPU check of the branch-free divisions (eb2_fdiv.cuh)
// and of the WENO weight routines built on them, bit for bit against the IEEE
// division `/` and against the routines written with `/`.
//
// dc_run(seed, launches, counts) runs `launches` grids of 2^22 random cases and
// accumulates into counts[0..8]:
//   0 rcp_rn(b) != __drcp_rn(b)              b in [2^-1000, 2^1000], all signs
//   1 div_rn(a, b, rcp_rn(b)) != a / b       quotients in [2^-900, 2^900]
//   2 copysign(div_rn(x, 6, RN(1/6)), x) != x / 6   x zero or in [2^-960, 2^1000]
//   3 weno5_js_rn != weno5_js where the guard holds
//   4 weno5_z_rn  != weno5_z  where the guard holds
//   5 weno3_rn    != weno3    where the guard holds
//   6, 7, 8  WENO cases (JS, Z, 3) whose guard failed (recomputed with `/`)
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
    if (!same(y, __drcp_rn(b))) atomicAdd(&counts[0], 1ull);
    if (!same(x64::div_rn(a, b, y), a / b)) atomicAdd(&counts[1], 1ull);
    double bw = make(r4, mode_b, -1000, 1000);
    if ((r4 >> 60) & 1) bw = -bw;
    if (!same(x64::rcp_rn(bw), __drcp_rn(bw))) atomicAdd(&counts[0], 1ull);

    // division by six
    double x = ((r4 >> 40) & 15) == 0 ? 0.0 : make(r3 ^ r1, mode_a, -960, 1000);
    if ((r1 >> 60) & 1) x = -x;
    if (!same(copysign(x64::div_rn(x, 6.0, 1.0 / 6.0), x), x / 6.0)) atomicAdd(&counts[2], 1ull);

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
        if (gd.ok<1423>()) {
            if (!same(f, x64::weno5_js(v[0], v[1], v[2], v[3], v[4]))) atomicAdd(&counts[3], 1ull);
        } else {
            atomicAdd(&counts[6], 1ull);
        }
    }
    {
        x64::DivGuard gd;
        const double f = x64::weno5_z_rn(v[5], v[4], v[3], v[2], v[1], gd);
        if (gd.ok<1423>()) {
            if (!same(f, x64::weno5_z(v[5], v[4], v[3], v[2], v[1]))) atomicAdd(&counts[4], 1ull);
        } else {
            atomicAdd(&counts[7], 1ull);
        }
    }
    {
        x64::DivGuard gd;
        const double f = x64::weno3_rn(v[1], v[2], v[3], gd);
        if (gd.ok<1423>()) {
            if (!same(f, x64::weno3(v[1], v[2], v[3]))) atomicAdd(&counts[5], 1ull);
        } else {
            atomicAdd(&counts[8], 1ull);
        }
    }
}

}  // namespace

extern "C" int dc_run(unsigned long long seed, int launches, unsigned long long* counts_host) {
    unsigned long long* counts = nullptr;
    if (cudaMalloc(&counts, 9 * sizeof(unsigned long long)) != cudaSuccess) return 1;
    cudaMemset(counts, 0, 9 * sizeof(unsigned long long));
    const int threads = 256, blocks = (1 << 22) / threads;
    for (int l = 0; l < launches; l++) k_divcheck<<<blocks, threads>>>(seed + 7919ull * l, counts);
    cudaError_t err = cudaDeviceSynchronize();
    if (err == cudaSuccess)
        err = cudaMemcpy(counts_host, counts, 9 * sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost);
    cudaFree(counts);
    return err == cudaSuccess ? 0 : 2;
}
