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

// The 1D radial-marching thermal reference of the reference's G2a gate
// (tests/g2a_thermal/check_g2a.py:94-207): a uniform H/He sphere around a
// central blackbody, nr shells marched outward with the attenuated bin
// fluxes, each shell's T_e bisected in ln T on heating = cooling (every
// evaluation re-solving the ionization from the shell's state), two
// self-shielding passes per shell, Gauss-Seidel sweeps until T_e moves by
// less than 1e-6.
struct Sphere1D {
    int nnu = 32;
    double emin = 13.598, emax = 100.0, tstar = 4.0e4, lband = 3.177837e38;
    double nH = 100.0, yHe = 0.1, rsph_pc = 4.0, te_min = 3.0e3, te_max = 5.0e4;
};
int thermal_1d(const Thermal& th, const RateModel& rm, const Sphere1D& s, int nr, int nsweep, double* r_pc,
               double* xHI, double* xHeI, double* xHeII, double* Te);

}  // namespace orc
