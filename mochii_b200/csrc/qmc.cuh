// Random-access Owen-scrambled Sobol points (qmc_mod.f90).
//
// x_d(i) = XOR over set bits k of i (mod 2^32) of V_d(k); the code is Owen
// scrambled by reverse -> Laine-Karras keyed permutation -> reverse
// (Burley 2020) and mapped to u = (code + 0.5) 2^-32.  Integer-exact on host
// and device, so the points match the reference bit for bit.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define QHD __host__ __device__ __forceinline__
#else
#define QHD inline
#endif

namespace mochii {

constexpr int kQmcMaxDim = 12;     // qmc_mod.f90:44
constexpr int kQmcBits = 32;

// Direction numbers and the per-(stream, dimension) Owen keys.
struct QmcTables {
    uint32_t V[kQmcMaxDim][kQmcBits];
    uint32_t key[2][kQmcMaxDim];
};

// lowbias32 avalanche hash (qmc_mod.f90:250-260), arithmetic mod 2^32.
QHD uint32_t qmc_hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}

QHD uint32_t qmc_reverse32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __brev(x);
#else
    x = (x << 16) | (x >> 16);
    x = ((x & 0x00FF00FFu) << 8) | ((x & 0xFF00FF00u) >> 8);
    x = ((x & 0x0F0F0F0Fu) << 4) | ((x & 0xF0F0F0F0u) >> 4);
    x = ((x & 0x33333333u) << 2) | ((x & 0xCCCCCCCCu) >> 2);
    x = ((x & 0x55555555u) << 1) | ((x & 0xAAAAAAAAu) >> 1);
    return x;
#endif
}

// Keyed nested permutation of Laine & Karras as the reference applies it
// (qmc_mod.f90:221-230): add the key, then four xor-multiply rounds.
QHD uint32_t qmc_owen(uint32_t code, uint32_t key) {
    uint32_t x = qmc_reverse32(code) + key;
    x ^= x * 0x6C50B47Cu;
    x ^= x * 0xB82F1E52u;
    x ^= x * 0xC7AFE638u;
    x ^= x * 0x8D22F6E6u;
    return qmc_reverse32(x);
}

// Unscrambled code of 0-based index idx in dimension d (0-based).
QHD uint32_t qmc_code(const QmcTables& t, uint64_t idx, int d) {
    uint32_t code = 0;
    uint32_t ii = (uint32_t)idx;   // bits above 32 carry no direction number
#ifdef __CUDA_ARCH__
    while (ii) {
        const int k = __ffs(ii) - 1;
        code ^= t.V[d][k];
        ii &= ii - 1;
    }
#else
    for (int k = 0; ii; ++k, ii >>= 1)
        if (ii & 1u) code ^= t.V[d][k];
#endif
    return code;
}

QHD double qmc_uniform(const QmcTables& t, uint64_t idx, int d, int stream) {
    const uint32_t c = qmc_owen(qmc_code(t, idx, d), t.key[stream][d]);
    return ((double)c + 0.5) * (1.0 / 4294967296.0);
}

// Direction numbers (Joe & Kuo new-joe-kuo-6 for dimensions 2..12, van der
// Corput for dimension 1) and keys hash32(seed + d*0x9E3779B9 [+0x85EBCA6B]),
// qmc_mod.f90:73-139.
inline void qmc_build_tables(int seed, QmcTables& t) {
    static const int deg[kQmcMaxDim] = {0, 1, 2, 3, 3, 4, 4, 5, 5, 5, 5, 5};
    static const int poly[kQmcMaxDim] = {0, 0, 1, 1, 2, 1, 4, 2, 4, 7, 11, 13};
    static const int m0[kQmcMaxDim][5] = {{0},          {1},           {1, 3},         {1, 3, 1},
                                          {1, 1, 1},    {1, 1, 3, 3},  {1, 3, 5, 13},  {1, 1, 5, 5, 17},
                                          {1, 1, 5, 5, 5}, {1, 1, 7, 11, 19}, {1, 1, 5, 1, 1}, {1, 1, 1, 3, 11}};
    for (int k = 0; k < kQmcBits; ++k) t.V[0][k] = 1u << (31 - k);
    for (int d = 1; d < kQmcMaxDim; ++d) {
        const int s = deg[d];
        for (int k = 0; k < s; ++k) t.V[d][k] = (uint32_t)m0[d][k] << (31 - k);
        for (int k = s; k < kQmcBits; ++k) {
            uint32_t v = t.V[d][k - s] ^ (t.V[d][k - s] >> s);
            for (int j = 1; j < s; ++j)
                if ((poly[d] >> (s - 1 - j)) & 1) v ^= t.V[d][k - j];
            t.V[d][k] = v;
        }
    }
    for (int d = 0; d < kQmcMaxDim; ++d) {
        const uint32_t base = (uint32_t)seed + (uint32_t)(d + 1) * 0x9E3779B9u;
        t.key[0][d] = qmc_hash32(base);
        t.key[1][d] = qmc_hash32(base + 0x85EBCA6Bu);
    }
}

}  // namespace mochii
