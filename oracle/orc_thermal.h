// Oracle (test infrastructure only): thermal-balance restatement -- free-free
// Gaunt table (gaunt.f90 getGauntFF + cooling_mod.f90 gaunt_ff_mean),
// cooling fits (cooling_mod.f90), the n-level line-cooling suppression
// tables (nlevel_mod.f90 + nlevel_cooling_mod.f90), cooling_total and the
// per-cell bisection of thermal_mod.f90.
#pragma once
#include <string>
#include <vector>

#include "orc_core.h"

namespace orc {

// getGauntFF, gaunt.f90:18-156 (single-precision Hummer 1988 expansion).
void get_gaunt_ff(float z, float log10Te, const float* xlf, int n, float* g);
double gaunt_ff_mean(double T, double Zc);           // cooling_mod.f90:182-220

struct GffTable {                                    // cooling_mod.f90:61-62,80-86
    double logT[41];
    double z[41][4];
    void build();
    double gbar(double T, int Z) const;              // cooling_mod.f90:223-234
};

struct CoolingFit {                                  // cooling_mod.f90:47-50
    std::vector<double> A, Ti;
    bool load(const std::string& path);              // cooling_mod.f90:98-122
    double eval(double T) const;                     // cooling_mod.f90:125-134
};

constexpr int NL_MAXLEV = 40, NL_MAXTR = 600;
struct NlevelAtom {                                  // nlevel_mod.f90:41-53
    int nlev = 0, nrad = 0, nups = 0;
    double g[NL_MAXLEV], e_cm1[NL_MAXLEV];
    std::vector<int> rl, ru, ul_l, ul_u, ttype, logf, nc;
    std::vector<double> A, cups, dery, st_lo, st_hi;
    std::vector<std::vector<double>> coef;
    bool load(const std::string& path);              // nlevel_mod.f90:61-105
    double ups(int k, double T) const;               // :119-152
};

struct NlevelTable {                                 // nlevel_cooling_mod.f90:58-72
    static constexpr int NT = 401, NNE = 161;
    std::vector<double> Ssup;                        // NT x NNE, Ssup[i*NNE + j]
    std::vector<double> lamref;                      // NT
    bool build(const NlevelAtom& atom);              // :106-158
    double apply(double lam_fit, double T, double ne) const;   // :163-176
    double coeff(double T, double ne) const;         // :209-234
    double col(int it, int j, double w1, double wt) const;     // :243-254
    double low_density(double T) const;              // :260-271
};

double nlevel_cooling_at(const NlevelAtom& atom, double T, double ne);

struct Thermal {
    GffTable gff;
    CoolingFit hi_fit;
    NlevelTable hi_table;
    bool use_hi_table = false;
    bool setup(const Par& p, std::string* err);
};

// cooling_total, cooling_mod.f90:240-276.
double cooling_total(const Thermal& th, const RateModel& rm, bool caseA, double yHe, double T, double nH,
                     double ne, double xHI, double xHeI, double xHeII);

}  // namespace orc
