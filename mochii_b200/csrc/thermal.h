// Thermal-balance tables (host build, device layout) and the per-cell
// cooling evaluation shared by the thermal kernel.
#pragma once
#include <string>
#include <vector>

#include "mochii_gpu.h"

namespace mochii {

constexpr int kGffNT = 41, kGffNZ = 4;      // cooling_mod.f90:61 (log T = 2..6, Z = 1..4)
constexpr int kNlNT = 401, kNlNNE = 161;    // nlevel_cooling_mod.f90:58 (log T 2..6 by 0.01, log n_e -6..10 by 0.1)
constexpr int kMaxFitTerms = 8;
constexpr int kMaxLev = 40;

struct NlevelAtomData {
    struct Rad { int l, u; double A; };
    struct Ups { int l, u, type, logf; double C, dE, st_lo, st_hi; std::vector<double> c; };
    std::vector<double> g, e_cm1;
    std::vector<Rad> rad;
    std::vector<Ups> ups;
    bool load(const std::string& path);
    static double upsilon(const Ups& u, double T);
    void cooling_column(double T, const double* ne, int nne, double* out) const;
};

struct ThermalHost {
    double gff_logT[kGffNT];
    double gff[kGffNT * kGffNZ];
    int hi_nterm = 0;
    double hi_A[kMaxFitTerms], hi_T[kMaxFitTerms];
    bool use_hi_table = false;
    std::vector<double> hi_lamref, hi_Ssup;
};

// Device copy of the tables (one allocation per array).
struct ThermalDev {
    double* gff = nullptr;      // kGffNT x kGffNZ
    double* lamref = nullptr;   // kNlNT
    double* Ssup = nullptr;     // kNlNT x kNlNNE
    double* tinv = nullptr;     // kNlNT: 1 / 10^logT_i
    double* lnL = nullptr;      // kNlNT x kNlNNE: log(lamref * Ssup), 0 where not positive
    double hi_A[kMaxFitTerms], hi_T[kMaxFitTerms];
    int hi_nterm = 0, use_hi_table = 0;
};

std::string data_root();
std::string atomic_dir(const mochii_params& p);
bool thermal_tables_build(const mochii_params& p, ThermalHost& t, std::string* err);
// Collisional line-cooling fit file (cooling_mod.f90:98-122): Lambda = sum A_i exp(-T_i/T) / sqrt(T).
bool cooling_fit_read(const std::string& path, std::vector<double>& A, std::vector<double>& Ti);

}  // namespace mochii
