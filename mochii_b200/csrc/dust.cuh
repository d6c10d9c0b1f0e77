// Device side of the grain optics and of the scattered flights' random
// stream (see dust.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dust.h"
#include "physics.cuh"

namespace mochii {

// Bracket i with lam[i] <= x0 < lam[i+1] (lam[0] < x0 < lam[n-1]): the
// first index whose successor exceeds x0, as the reference's scan finds it.
__device__ __forceinline__ int dust_bracket(const DustDev& d, double x0) {
    int lo = 0, hi = d.n - 1;   // upper_bound over lam[1..n-1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(d.lam + mid) <= x0) lo = mid; else hi = mid;
    }
    return lo;
}

// interp_log / interp_lin (gas_opacity_mod.f90:277-315) at lambda x0.
__device__ __forceinline__ double dust_interp_log(const DustDev& d, const double* y, double x0) {
    if (x0 <= __ldg(d.lam)) return __ldg(y);
    if (x0 >= __ldg(d.lam + d.n - 1)) return __ldg(y + d.n - 1);
    const int i = dust_bracket(d, x0);
    const double xa = __ldg(d.lam + i), xb = __ldg(d.lam + i + 1);
    const double w = log(x0 / xa) / log(xb / xa);
    return exp(log(fmax(__ldg(y + i), kTinest)) * (1.0 - w) + log(fmax(__ldg(y + i + 1), kTinest)) * w);
}
__device__ __forceinline__ double dust_interp_lin(const DustDev& d, const double* y, double x0) {
    if (x0 <= __ldg(d.lam)) return __ldg(y);
    if (x0 >= __ldg(d.lam + d.n - 1)) return __ldg(y + d.n - 1);
    const int i = dust_bracket(d, x0);
    const double xa = __ldg(d.lam + i), xb = __ldg(d.lam + i + 1);
    const double w = (x0 - xa) / (xb - xa);
    return __ldg(y + i) * (1.0 - w) + __ldg(y + i + 1) * w;
}

// ion_dust_sabs_at / ssca_at / g_at (gas_opacity_mod.f90:231-256).
struct DustOptics {
    double sabs, ssca, g;
};
__device__ __forceinline__ DustOptics dust_optics(const DustDev& d, double E) {
    const double lb = 1.23984 / E;
    const double a = dust_interp_lin(d, d.alb, lb);
    const double c = dust_interp_log(d, d.cext, lb);
    DustOptics o;
    o.sabs = (1.0 - a) * c / d.cref;
    o.ssca = a * c / d.cref;
    o.g = dust_interp_lin(d, d.gcos, lb);
    return o;
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC11): ten rounds of two
// 32x32->64 multiplies with the Weyl key schedule.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// One packet's stream of uniforms in (0, 1): draw n is 53 bits of Philox
// block n/2 (counter (n/2, 0, packet lo, packet hi), key (seed lo,
// seed hi ^ stream)); a block serves two draws.
struct PacketStream {
    uint2 key;
    uint32_t plo, phi;
    uint32_t n;
    uint4 blk;
    __device__ __forceinline__ void init(uint64_t seed, uint32_t stream, uint64_t packet) {
        key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32) ^ stream);
        plo = (uint32_t)packet;
        phi = (uint32_t)(packet >> 32);
        n = 0;
    }
    __device__ __forceinline__ double next() {
        if ((n & 1) == 0) blk = philox4x32_10(make_uint4(n >> 1, 0u, plo, phi), key);
        const uint32_t a = (n & 1) ? blk.z : blk.x, b = (n & 1) ? blk.w : blk.y;
        ++n;
        const uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
        return ((double)m + 0.5) * (1.0 / 9007199254740992.0);
    }
};

}  // namespace mochii
