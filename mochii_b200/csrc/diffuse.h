// Diffuse-field tables and device buffers.
#pragma once
#include <cuda_runtime.h>

#include <string>
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

// He I 2^1S two-photon continuum above the H I edge (hei_twophoton_mod.f90):
// the energy-weighted sampling CDF on a uniform grid in y = E / 20.62 eV and
// the in-band energy per decay.
constexpr int kHe2phN = 1024;
constexpr double kHe2phEtot = 20.62;

struct HeI2phHost {
    std::vector<double> cdf_e, grid_y;   // kHe2phN each
    double n_per_decay = 0.0, e_per_decay = 0.0;
};

struct HeI2phDev {
    const double* cdf_e = nullptr;
    const double* grid_y = nullptr;
    double e_per_decay = 0.0;
};

struct DiffuseBuffers {
    double* ch = nullptr;    // 4 x nleaf channel luminosities
    double* tot = nullptr;   // nleaf totals -> inclusive prefix sum
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
    double* tables = nullptr;   // xg | cdf | xbar | frac
    MilneDev m{};
    HeI2phDev he{};          // par%hei_diffuse: the He I excited channel's two-photon table
    double* he_tab = nullptr;   // cdf_e | grid_y
    double lum = 0.0;
    long long nphot = 0;
};

void milne_tables_build(double eion_max, MilneHost& m);
// Reads the two-photon shape A(y) (two columns: y, A) and builds the table;
// false when the file cannot be read or is too short.
bool hei_2ph_build(const std::string& path, double eion_max, HeI2phHost& h);

}  // namespace mochii
