// Diffuse-field tables and device buffers.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace mochii {

constexpr int kMilneNT = 192, kMilneNX = 512;   // milne_recomb_spectrum_mod.f90:39-42

struct MilneHost {
    std::vector<double> lgT, xg, cdf, xbar, frac;   // cdf: (3, NT, NX); xbar/frac: (3, NT)
};

struct MilneDev {
    const double* xg;
    const double* cdf;
    const double* xbar;
    const double* frac;
    double lgT0, dlgT;   // lgT(1) and lgT(2) - lgT(1)
};

struct DiffuseBuffers {
    double* ch = nullptr;    // 4 x nleaf channel luminosities
    double* tot = nullptr;   // nleaf totals -> inclusive prefix sum
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
    double* tables = nullptr;   // xg | cdf | xbar | frac
    MilneDev m{};
    double lum = 0.0;
    long long nphot = 0;
};

void milne_tables_build(double eion_max, MilneHost& m);

}  // namespace mochii
