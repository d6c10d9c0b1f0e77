// Oracle (test infrastructure only): FP64 CPU restatement of the MoCHII
// transport + balance path.  See orc_core.h for the contract.
#include "orc_core.h"
#include "orc_thermal.h"
#include "orc_species.h"
#include "orc_amr.h"

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// =========================================================================
// qmc_mod.f90
// =========================================================================
// lowbias32 avalanche hash, qmc_mod.f90:250-260 (all arithmetic mod 2^32).
uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}

// 32-bit reversal by swaps, qmc_mod.f90:233-247.
uint32_t reverse32(uint32_t n) {
    n = (n << 16) | (n >> 16);
    n = ((n & 0x00FF00FFu) << 8) | ((n & 0xFF00FF00u) >> 8);
    n = ((n & 0x0F0F0F0Fu) << 4) | ((n & 0xF0F0F0F0u) >> 4);
    n = ((n & 0x33333333u) << 2) | ((n & 0xCCCCCCCCu) >> 2);
    n = ((n & 0x55555555u) << 1) | ((n & 0xAAAAAAAAu) >> 1);
    return n;
}

// Laine-Karras nested permutation, qmc_mod.f90:221-230.  The Fortran
// multiplies two values below 2^32 in int64 and masks the low 32 bits,
// which equals the uint32 product.
uint32_t laine_karras(uint32_t x, uint32_t seed) {
    x = x + seed;
    x ^= x * 0x6C50B47Cu;
    x ^= x * 0xB82F1E52u;
    x ^= x * 0xC7AFE638u;
    x ^= x * 0x8D22F6E6u;
    return x;
}

uint32_t owen_scramble(uint32_t x, uint32_t seed) {  // qmc_mod.f90:212-219
    return reverse32(laine_karras(reverse32(x), seed));
}

// qmc_mod.f90:73-139.  Dimension 1 is van der Corput; dimensions 2..12 use
// the Joe-Kuo new-joe-kuo-6 degree / polynomial / initial integers of
// qmc_mod.f90:80-97 with the direction-number recurrence of :104-123.
void Qmc::setup(int seed) {
    static const int sdeg[13] = {0, 0, 1, 2, 3, 3, 4, 4, 5, 5, 5, 5, 5};
    static const int apoly[13] = {0, 0, 0, 1, 1, 2, 1, 4, 2, 4, 7, 11, 13};
    static const int minit[13][5] = {
        {0}, {0}, {1}, {1, 3}, {1, 3, 1}, {1, 1, 1}, {1, 1, 3, 3}, {1, 3, 5, 13},
        {1, 1, 5, 5, 17}, {1, 1, 5, 5, 5}, {1, 1, 7, 11, 19}, {1, 1, 5, 1, 1},
        {1, 1, 1, 3, 11}};
    for (int k = 1; k <= 32; ++k) V[0][k - 1] = 1u << (32 - k);
    for (int d = 2; d <= 12; ++d) {
        const int s = sdeg[d], a = apoly[d];
        for (int k = 1; k <= s; ++k)
            V[d - 1][k - 1] = (uint32_t)((uint64_t)minit[d][k - 1] << (32 - k));
        for (int k = s + 1; k <= 32; ++k) {
            uint32_t v = V[d - 1][k - s - 1] ^ (V[d - 1][k - s - 1] >> s);
            for (int j = 1; j <= s - 1; ++j)
                if ((a >> (s - 1 - j)) & 1) v ^= V[d - 1][k - j - 1];
            V[d - 1][k - 1] = v;
        }
    }
    // Owen keys, qmc_mod.f90:130-136: hash32((seed + d*0x9E3779B9 [+0x85EBCA6B]) mod 2^32)
    for (int d = 1; d <= 12; ++d) {
        const uint32_t base = (uint32_t)(int64_t)seed + (uint32_t)d * 0x9E3779B9u;
        key[0][d - 1] = hash32(base);
        key[1][d - 1] = hash32(base + 0x85EBCA6Bu);
    }
}

// sobol_code, qmc_mod.f90:192-206: XOR of V_d(k) over the set bits k of
// idx; bits above 32 carry no direction number.
uint32_t Qmc::sobol_code(int64_t idx, int d) const {
    uint32_t code = 0;
    uint64_t ii = (uint64_t)idx;
    int k = 1;
    while (ii != 0 && k <= 32) {
        if (ii & 1u) code ^= V[d - 1][k - 1];
        ii >>= 1;
        ++k;
    }
    return code;
}

uint32_t Qmc::scrambled(int64_t idx, int d, int stream) const {
    return owen_scramble(sobol_code(idx, d), key[stream - 1][d - 1]);
}

// u = (code + 0.5) 2^-32, qmc_mod.f90:166.
double Qmc::uniform(int64_t idx, int d, int stream) const {
    return ((double)scrambled(idx, d, stream) + 0.5) * (1.0 / 4294967296.0);
}

// =========================================================================
// energy_sampler_mod.f90
// =========================================================================
static void set_err(std::string* err, const char* msg) {
    if (err) *err = msg;
}

// build_tabulated_sampler, energy_sampler_mod.f90:34-64.
bool build_tabulated_sampler(Sampler& s, const std::vector<double>& e,
                             const std::vector<double>& f, std::string* err) {
    const size_t n = e.size();
    if (n < 2 || f.size() != n) {
        set_err(err, "energy sampler: table needs at least two matching columns");
        return false;
    }
    for (double v : f)
        if (v < 0.0) {
            set_err(err, "energy sampler: negative spectral density");
            return false;
        }
    for (size_t i = 0; i + 1 < n; ++i)
        if (e[i + 1] <= e[i]) {
            set_err(err, "energy sampler: energies must be strictly ascending");
            return false;
        }
    s.energy = e;
    s.density = f;
    s.cdf.assign(n, 0.0);
    for (size_t i = 0; i + 1 < n; ++i) {
        const double area = 0.5 * (f[i] + f[i + 1]) * (e[i + 1] - e[i]);
        s.cdf[i + 1] = s.cdf[i] + area;
    }
    const double total = s.cdf[n - 1];
    if (total <= 0.0) {
        set_err(err, "energy sampler: zero integrated luminosity");
        return false;
    }
    s.total_integral = total;
    for (size_t i = 0; i < n; ++i) s.cdf[i] = s.cdf[i] / total;
    s.cdf[n - 1] = 1.0;
    return true;
}

// linear_table_value, energy_sampler_mod.f90:336-359.
static double linear_table_value(const std::vector<double>& e,
                                 const std::vector<double>& f, double v) {
    const int n = (int)e.size();
    if (v <= e[0]) return f[0];
    if (v >= e[n - 1]) return f[n - 1];
    int lo = 1, hi = n;  // 1-based
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (e[mid - 1] <= v) lo = mid; else hi = mid;
    }
    const double fr = (v - e[lo - 1]) / (e[hi - 1] - e[lo - 1]);
    return f[lo - 1] + fr * (f[hi - 1] - f[lo - 1]);
}

// build_tabulated_band_sampler, energy_sampler_mod.f90:66-104.
bool build_tabulated_band_sampler(Sampler& s, const std::vector<double>& e,
                                  const std::vector<double>& f, double emin,
                                  double emax, std::string* err) {
    const size_t n = e.size();
    if (n < 2 || f.size() != n) {
        set_err(err, "energy sampler: table needs at least two matching columns");
        return false;
    }
    if (emax <= emin) {
        set_err(err, "energy sampler: invalid requested band");
        return false;
    }
    const double lo = std::max(emin, e[0]);
    const double hi = std::min(emax, e[n - 1]);
    if (hi <= lo) {
        set_err(err, "energy sampler: table does not overlap requested band");
        return false;
    }
    std::vector<double> ce, cf;
    ce.push_back(lo);
    cf.push_back(linear_table_value(e, f, lo));
    for (size_t i = 0; i < n; ++i)
        if (e[i] > lo && e[i] < hi) {
            ce.push_back(e[i]);
            cf.push_back(f[i]);
        }
    ce.push_back(hi);
    cf.push_back(linear_table_value(e, f, hi));
    return build_tabulated_sampler(s, ce, cf, err);
}

// planck_energy_shape, energy_sampler_mod.f90:277-290 (energy**3 as e*e*e).
double planck_energy_shape(double energy, double T) {
    const double x = energy / (KB_EV * T);
    const double e3 = energy * energy * energy;
    if (x <= 0.0) return 0.0;
    if (x < 1.0e-3) return e3 / (x * (1.0 + 0.5 * x + x * x / 6.0));
    if (x < 700.0) return e3 / (std::exp(x) - 1.0);
    return e3 * std::exp(-x);
}

// rough_planck_integral, energy_sampler_mod.f90:321-334.
static double rough_planck_integral(double T, double emin, double emax) {
    const int n = 256;
    double total = 0.0;
    for (int i = 1; i <= n; ++i) {
        const double e0 = emin + (emax - emin) * (double)(i - 1) / (double)n;
        const double e1 = emin + (emax - emin) * (double)i / (double)n;
        total = total + 0.5 * (planck_energy_shape(e0, T) + planck_energy_shape(e1, T)) * (e1 - e0);
    }
    return total;
}

// refine_planck_interval, energy_sampler_mod.f90:159-185 (depth-first, left
// half first, so the knots come out in ascending order).
static bool refine_planck_interval(double T, double e0, double e1, double f0,
                                   double f1, double tol, double scale,
                                   double span, int depth,
                                   std::vector<double>& we,
                                   std::vector<double>& wf) {
    const double em = 0.5 * (e0 + e1);
    const double fm = planck_energy_shape(em, T);
    const double coarse = 0.5 * (f0 + f1) * (e1 - e0);
    const double fine = 0.25 * (f0 + 2.0 * fm + f1) * (e1 - e0);
    const double err = std::fabs(fine - coarse) / 3.0;
    const double allowance = tol * (std::fabs(fine) + scale * (e1 - e0) / span);
    if (err <= allowance || depth >= 50) {
        if ((int)we.size() + 1 > MAX_PLANCK_KNOTS) return false;
        we.push_back(e1);
        wf.push_back(f1);
        return true;
    }
    if (!refine_planck_interval(T, e0, em, f0, fm, tol, scale, span, depth + 1, we, wf)) return false;
    return refine_planck_interval(T, em, e1, fm, f1, tol, scale, span, depth + 1, we, wf);
}

// build_planck_sampler, energy_sampler_mod.f90:106-157 (+ sort_unique :361-391).
bool build_planck_sampler(Sampler& s, double T, double emin, double emax,
                          double rtol, const std::vector<double>& thr,
                          std::string* err) {
    if (T <= 0.0 || emin < 0.0 || emax <= emin) {
        set_err(err, "energy sampler: invalid Planck temperature or energy band");
        return false;
    }
    const double tol = rtol;
    if (tol <= 0.0) {
        set_err(err, "energy sampler: Planck rtol must be positive");
        return false;
    }
    std::vector<double> mand;
    mand.push_back(emin);
    for (double t : thr)
        if (t > emin && t < emax) mand.push_back(t);
    mand.push_back(emax);
    // sort_unique: insertion sort then drop repeats.
    for (size_t i = 1; i < mand.size(); ++i) {
        const double hold = mand[i];
        size_t j = i;
        while (j >= 1 && mand[j - 1] > hold) {
            mand[j] = mand[j - 1];
            --j;
        }
        mand[j] = hold;
    }
    std::vector<double> uniq;
    uniq.push_back(mand[0]);
    for (size_t i = 1; i < mand.size(); ++i)
        if (mand[i] > uniq.back()) uniq.push_back(mand[i]);

    const double scale = rough_planck_integral(T, emin, emax);
    if (scale <= 0.0) {
        set_err(err, "energy sampler: zero Planck band luminosity");
        return false;
    }
    const double span = emax - emin;
    std::vector<double> we, wf;
    we.push_back(uniq[0]);
    wf.push_back(planck_energy_shape(uniq[0], T));
    for (size_t i = 0; i + 1 < uniq.size(); ++i) {
        if (!refine_planck_interval(T, uniq[i], uniq[i + 1],
                                    planck_energy_shape(uniq[i], T),
                                    planck_energy_shape(uniq[i + 1], T), tol,
                                    scale, span, 0, we, wf)) {
            set_err(err, "energy sampler: Planck knot limit");
            return false;
        }
    }
    return build_tabulated_sampler(s, we, wf, err);
}

// sample_energy_cdf, energy_sampler_mod.f90:187-238.
double sample_energy_cdf(const Sampler& s, double u) {
    const int n = (int)s.cdf.size();
    const double target = std::min(std::max(u, 0.0), 1.0);
    if (target <= 0.0) return s.energy[0];
    if (target >= 1.0) return s.energy[n - 1];
    int lo = 1, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (s.cdf[mid - 1] <= target) lo = mid; else hi = mid;
    }
    const double interval_area = s.cdf[hi - 1] - s.cdf[lo - 1];
    if (interval_area <= 0.0) return s.energy[hi - 1];
    const double dx = s.energy[hi - 1] - s.energy[lo - 1];
    const double y0 = s.density[lo - 1];
    const double y1 = s.density[hi - 1];
    const double local_area = (target - s.cdf[lo - 1]) / interval_area * (0.5 * (y0 + y1) * dx);
    const double slope = (y1 - y0) / dx;
    const double slope_scale = std::max(std::max(std::fabs(y0), std::fabs(y1)), TINEST);
    double offset;
    if (std::fabs(slope * dx) <= 64.0 * 2.220446049250313e-16 * slope_scale) {
        offset = (y0 > 0.0) ? local_area / y0 : 0.0;
    } else {
        const double disc = std::sqrt(std::max(0.0, y0 * y0 + 2.0 * slope * local_area));
        offset = 2.0 * local_area / (y0 + disc);
    }
    return s.energy[lo - 1] + std::min(std::max(offset, 0.0), dx);
}

// energy_cdf_value, energy_sampler_mod.f90:240-275.
double energy_cdf_value(const Sampler& s, double energy) {
    const int n = (int)s.energy.size();
    if (energy <= s.energy[0]) return 0.0;
    if (energy >= s.energy[n - 1]) return 1.0;
    int lo = 1, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (s.energy[mid - 1] <= energy) lo = mid; else hi = mid;
    }
    const double dx = s.energy[hi - 1] - s.energy[lo - 1];
    const double offset = energy - s.energy[lo - 1];
    const double y0 = s.density[lo - 1];
    const double slope = (s.density[hi - 1] - y0) / dx;
    const double interval_total = 0.5 * (y0 + s.density[hi - 1]) * dx;
    const double partial = y0 * offset + 0.5 * slope * offset * offset;
    if (interval_total > 0.0)
        return s.cdf[lo - 1] + (s.cdf[hi - 1] - s.cdf[lo - 1]) * partial / interval_total;
    return s.cdf[lo - 1];
}

// =========================================================================
// photo_xsec.f90
// =========================================================================
// sigma_vfky96, photo_xsec.f90:46-59 (VFKY96 Eq. 1; sigma_0 in Mb).
double sigma_vfky96(double E, double Eth, double E0, double s0, double ya,
                    double P, double yw, double y0, double y1) {
    if (E < Eth) return 0.0;
    const double x = E / E0 - y0;
    const double z = std::sqrt(x * x + y1 * y1);
    const double Q = 5.5 - 0.5 * P;
    const double xm1 = x - 1.0;
    const double Fy = (xm1 * xm1 + yw * yw) * std::pow(z, -Q) * std::pow(1.0 + std::sqrt(z / ya), -P);
    return s0 * Fy * 1.0e-18;
}

// sigma_vy95, photo_xsec.f90:69-82.
double sigma_vy95(double E, double Eth, double E0, double s0, double ya,
                  double P, double yw, double l) {
    if (E < Eth) return 0.0;
    const double y = E / E0;
    const double Q = 5.5 + l - 0.5 * P;
    const double ym1 = y - 1.0;
    const double Fy = (ym1 * ym1 + yw * yw) * std::pow(y, -Q) * std::pow(1.0 + std::sqrt(y / ya), -P);
    return s0 * Fy * 1.0e-18;
}

// sigma_hydrogenic, photo_xsec.f90:92-107 ((E_th/E)**4 by squaring).
double sigma_hydrogenic(double E, double Eth, double Z) {
    const double s0 = 6.30e-18 / (Z * Z);
    if (E < Eth) return 0.0;
    if (E > Eth) {
        const double eps = std::sqrt(E / Eth - 1.0);
        const double r = Eth / E;
        const double r2 = r * r;
        return s0 * (r2 * r2) * std::exp(4.0 - 4.0 * std::atan(eps) / eps) /
               (1.0 - std::exp(-2.0 * PI / eps));
    }
    return s0;
}

double sigma_HI(double E) { return sigma_hydrogenic(E, ETH_HI, 1.0); }       // :110-113
double sigma_HeI(double E) {                                                 // :116-120
    return sigma_vfky96(E, ETH_HEI, 1.361e1, 9.492e2, 1.469, 3.188, 2.039, 4.434e-1, 2.136);
}
double sigma_HeII(double E) { return sigma_hydrogenic(E, ETH_HEII, 2.0); }   // :123-126

// =========================================================================
// recomb_mod.f90
// =========================================================================
static double rr_badnell(double T, double A, double B, double T0, double T1,
                         double Cc, double T2) {  // recomb_mod.f90:124-130
    const double bp = B + Cc * std::exp(-T2 / T);
    const double tt = std::sqrt(T / T0);
    return A / (tt * std::pow(1.0 + tt, 1.0 - bp) * std::pow(1.0 + std::sqrt(T / T1), 1.0 + bp));
}
static double dr_HeII_badnell(double T) {  // recomb_mod.f90:132-137
    return std::pow(T, -1.5) * (1.417e-3 * std::exp(-4.633e5 / T) +
                                2.235e-4 * std::exp(-5.532e5 / T) -
                                2.185e-5 * std::exp(-8.887e5 / T));
}
static double rr_mao(double T, double a0, double b0, double c0, double a1,
                     double b1, double a2, double b2) {  // recomb_mod.f90:145-151
    const double te = T * (KBOLTZ_CGS / EV2ERG);
    return a0 * 1.0e-10 * std::pow(te, -b0 - c0 * std::log(te)) *
           (1.0 + a2 * std::pow(te, -b2)) / (1.0 + a1 * std::pow(te, -b1));
}
double alpha1_HII(double T) {  // recomb_mod.f90:188-192
    return rr_mao(T, 1.87007e-2, 1.29077, -2.17465e-3, 1.29189e1, 8.05060e-1, 8.44399e-2, 5.93940e-4);
}
double alpha1_HeIII(double T) {  // :194-198
    return rr_mao(T, 2.61525e-1, 1.39527, -3.22079e-4, 6.40708e1, 8.97582e-1, 5.01551e-1, 1.21533e-3);
}
double alpha1_HeII(double T) {  // :200-204
    return rr_mao(T, 3.26862e-3, 6.97361e-1, 3.14907e-4, 5.76341e1, 1.18534, 2.58417e1, 9.90134e-1);
}
// Hui & Gnedin fits, recomb_mod.f90:209-251.
static double hg_aA_HII(double T) {
    const double lam = 2.0 * 157807.0 / T;
    return 1.269e-13 * std::pow(lam, 1.503) / std::pow(1.0 + std::pow(lam / 0.522, 0.470), 1.923);
}
static double hg_aB_HII(double T) {
    const double lam = 2.0 * 157807.0 / T;
    return 2.753e-14 * std::pow(lam, 1.500) / std::pow(1.0 + std::pow(lam / 2.740, 0.407), 2.242);
}
static double hg_aA_HeII(double T) { return 3.000e-14 * std::pow(2.0 * 285335.0 / T, 0.654); }
static double hg_aB_HeII(double T) { return 1.260e-14 * std::pow(2.0 * 285335.0 / T, 0.750); }
static double hg_aA_HeIII(double T) {
    const double lam = 2.0 * 631515.0 / T;
    return 2.0 * 1.269e-13 * std::pow(lam, 1.503) / std::pow(1.0 + std::pow(lam / 0.522, 0.470), 1.923);
}
static double hg_aB_HeIII(double T) {
    const double lam = 2.0 * 631515.0 / T;
    return 2.0 * 2.753e-14 * std::pow(lam, 1.500) / std::pow(1.0 + std::pow(lam / 2.740, 0.407), 2.242);
}
// Public dispatch, recomb_mod.f90:47-118.
double alphaA_HII(const RateModel& m, double T) {
    return m.recomb == RECOMB_HUI_GNEDIN ? hg_aA_HII(T)
                                         : rr_badnell(T, 8.318e-11, 0.7472, 2.965, 7.001e5, 0.0, 0.0);
}
double alphaB_HII(const RateModel& m, double T) {
    return m.recomb == RECOMB_HUI_GNEDIN ? hg_aB_HII(T) : alphaA_HII(m, T) - alpha1_HII(T);
}
double alphaA_HeII(const RateModel& m, double T) {
    return m.recomb == RECOMB_HUI_GNEDIN
               ? hg_aA_HeII(T)
               : rr_badnell(T, 5.235e-11, 0.6988, 7.301, 4.475e6, 0.0829, 1.682e5) + dr_HeII_badnell(T);
}
double alphaB_HeII(const RateModel& m, double T) {
    return m.recomb == RECOMB_HUI_GNEDIN ? hg_aB_HeII(T) : alphaA_HeII(m, T) - alpha1_HeII(T);
}
double alphaA_HeIII(const RateModel& m, double T) {
    return m.recomb == RECOMB_HUI_GNEDIN ? hg_aA_HeIII(T)
                                         : rr_badnell(T, 1.818e-10, 0.7492, 1.017e1, 2.786e6, 0.0, 0.0);
}
double alphaB_HeIII(const RateModel& m, double T) {
    return m.recomb == RECOMB_HUI_GNEDIN ? hg_aB_HeIII(T) : alphaA_HeIII(m, T) - alpha1_HeIII(T);
}
// Voronov (1997), recomb_mod.f90:256-261.
double voronov(double T, double dE, double P, double A, double X, double K) {
    const double U = dE * EV2ERG / (KBOLTZ_CGS * T);
    return A * (1.0 + P * std::sqrt(U)) * std::pow(U, K) * std::exp(-U) / (X + U);
}
// Dere hybrid ratio table, recomb_mod.f90:288-311.
double ci_dere_ratio(const RateModel& m, int Z, int stage) {
    if (m.ci != CI_DERE_HYBRID) return 1.0;
    double tab[4] = {1, 1, 1, 1};
    int n = 0;
    switch (Z) {
        case 1: tab[0] = 0.9063; n = 1; break;
        case 2: tab[0] = 1.0389; tab[1] = 1.0686; n = 2; break;
        case 6: tab[0] = 1.0499; tab[1] = 0.913; tab[2] = 1.0377; n = 3; break;
        case 7: tab[0] = 1.0421; tab[1] = 1.1966; n = 2; break;
        case 8: tab[0] = 1.041; tab[1] = 1.1181; n = 2; break;
        case 10: tab[0] = 0.8089; tab[1] = 1.1395; n = 2; break;
        case 12: tab[0] = 0.3793; tab[1] = 0.9857; n = 2; break;
        case 14: tab[0] = 0.7328; tab[1] = 0.8798; tab[2] = 0.4492; tab[3] = 0.8221; n = 4; break;
        case 16: tab[0] = 1.3572; tab[1] = 0.8925; tab[2] = 0.8119; n = 3; break;
        case 17: tab[0] = 0.5412; tab[1] = 0.8428; tab[2] = 0.9237; tab[3] = 0.819; n = 4; break;
        case 18: tab[0] = 0.9242; tab[1] = 0.8644; tab[2] = 0.9752; n = 3; break;
        case 20: tab[0] = 0.7652; tab[1] = 1.1668; tab[2] = 1.0422; tab[3] = 0.8705; n = 4; break;
        case 26: tab[0] = 0.9904; tab[1] = 1.0568; tab[2] = 1.824; n = 3; break;
    }
    if (stage >= 1 && stage <= n) return tab[stage - 1];
    return 1.0;
}
double ci_HI(const RateModel& m, double T) {  // recomb_mod.f90:263-267
    return voronov(T, 13.6, 0.0, 2.91e-8, 0.232, 0.39) * ci_dere_ratio(m, 1, 1);
}
double ci_HeI(const RateModel& m, double T) {  // :269-273
    return voronov(T, 24.6, 0.0, 1.75e-8, 0.180, 0.35) * ci_dere_ratio(m, 2, 1);
}
double ci_HeII(const RateModel& m, double T) {  // :275-279
    return voronov(T, 54.4, 1.0, 2.05e-9, 0.265, 0.25) * ci_dere_ratio(m, 2, 2);
}

// =========================================================================
// namelist (setup.f90:23-35) and parameter defaults (define.f90:189-861)
// =========================================================================
Par::Par() {
    for (int i = 0; i < MAX_SRC; ++i) {
        src_tstar[i] = -999.0;
        src_lum[i] = -999.0;
        src_x[i] = src_y[i] = src_z[i] = 0.0;
    }
    for (int i = 0; i < MAX_OBS; ++i) {
        alpha[i] = beta[i] = gamma_[i] = obsx[i] = obsy[i] = obsz[i] = NAN;
        phase_angle[i] = inclination_angle[i] = position_angle[i] = NAN;
    }
}

static std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}
static std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}
static bool to_bool(const std::string& v) {
    std::string s = lower(trim(v));
    return s == ".true." || s == "t" || s == "true" || s == ".t.";
}
static double to_dbl(const std::string& v) {
    std::string s = trim(v);
    for (auto& c : s)
        if (c == 'd' || c == 'D') c = 'e';
    return std::strtod(s.c_str(), nullptr);
}
static std::string to_str(const std::string& v) {
    std::string s = trim(v);
    if (s.size() >= 2 && (s[0] == '\'' || s[0] == '"')) s = s.substr(1, s.size() - 2);
    return trim(s);
}

bool parse_namelist(const std::string& text, Par& p, std::string* err) {
    // Strip '!' comments outside quotes, then split on commas/newlines into
    // "par%key[(i)] = value[, value...]" assignments.
    std::string clean;
    bool inq = false;
    char q = 0;
    for (size_t i = 0; i < text.size(); ++i) {
        char c = text[i];
        if (inq) {
            if (c == q) inq = false;
            clean += c;
            continue;
        }
        if (c == '\'' || c == '"') {
            inq = true;
            q = c;
            clean += c;
            continue;
        }
        if (c == '!') {
            while (i < text.size() && text[i] != '\n') ++i;
            clean += '\n';
            continue;
        }
        clean += c;
    }
    // tokenise assignments: find "par%"
    std::map<std::string, std::vector<std::string>> kv;
    size_t pos = 0;
    std::string lc = lower(clean);
    while ((pos = lc.find("par%", pos)) != std::string::npos) {
        size_t eq = lc.find('=', pos);
        if (eq == std::string::npos) break;
        std::string key = trim(lc.substr(pos + 4, eq - pos - 4));
        size_t next = lc.find("par%", eq);
        size_t endslash = std::string::npos;
        // value ends at next par% or a terminating '/' outside quotes
        std::string raw = clean.substr(eq + 1, (next == std::string::npos ? clean.size() : next) - eq - 1);
        {
            bool iq = false;
            char qq = 0;
            for (size_t k = 0; k < raw.size(); ++k) {
                char c = raw[k];
                if (iq) {
                    if (c == qq) iq = false;
                    continue;
                }
                if (c == '\'' || c == '"') {
                    iq = true;
                    qq = c;
                    continue;
                }
                if (c == '/') {
                    endslash = k;
                    break;
                }
            }
        }
        if (endslash != std::string::npos) raw = raw.substr(0, endslash);
        std::vector<std::string> vals;
        {
            std::string cur;
            bool iq = false;
            char qq = 0;
            for (char c : raw) {
                if (iq) {
                    cur += c;
                    if (c == qq) iq = false;
                    continue;
                }
                if (c == '\'' || c == '"') {
                    iq = true;
                    qq = c;
                    cur += c;
                    continue;
                }
                if (c == ',' || c == '\n') {
                    if (!trim(cur).empty()) vals.push_back(trim(cur));
                    cur.clear();
                    continue;
                }
                cur += c;
            }
            if (!trim(cur).empty()) vals.push_back(trim(cur));
        }
        int index = 1;
        size_t lp = key.find('(');
        if (lp != std::string::npos) {
            index = std::atoi(key.substr(lp + 1).c_str());
            key = trim(key.substr(0, lp));
        }
        auto& slot = kv[key];
        if ((int)slot.size() < index - 1 + (int)vals.size()) slot.resize(index - 1 + vals.size());
        for (size_t k = 0; k < vals.size(); ++k) slot[index - 1 + k] = vals[k];
        pos = eq;
    }
    for (auto& it : kv) {
        const std::string& k = it.first;
        const auto& v = it.second;
        if (v.empty()) continue;
        const std::string& s = v[0];
#define D(name) else if (k == #name) p.name = to_dbl(s)
#define I(name) else if (k == #name) p.name = (int)std::llround(to_dbl(s))
#define B(name) else if (k == #name) p.name = to_bool(s)
#define S(name) else if (k == #name) p.name = to_str(s)
        if (k == "no_photons") p.nphotons = (int64_t)to_dbl(s);
        else if (k == "nphotons") p.nphotons = (int64_t)to_dbl(s);
        S(launch_sequence); I(qmc_seed); D(source_cdf_tol); D(luminosity); D(tstar);
        I(nnu_ion); D(eion_min); D(eion_max); B(add_fuv); D(efuv_min); I(nnu_fuv);
        B(ion_align_edges); S(grid_type); S(car_walk); S(amr_file);
        I(nx); I(ny); I(nz); D(xmax); D(ymax); D(zmax); D(rmax); D(rmin); D(nH_const);
        S(distance_unit); S(source_geometry); D(xs_point); D(ys_point); D(zs_point);
        I(nsource); D(xHI_init); D(xHeI_init); D(xHeII_init); D(He_abund);
        I(gas_niter); D(gas_tol); D(te_fixed); D(ion_relax); S(case_ab); S(ci_model);
        S(recomb_model); S(cooling_model); S(charge_exchange); S(conv_crit);
        B(solve_te); D(te_min); D(te_max); D(gas_tol_te); B(use_metals);
        B(diffuse_field); B(use_sec_ion); B(ion_add_dust); B(ion_dust_scatter); B(hei_diffuse);
        D(ext_intensity); D(ext_tstar); S(ext_geometry);
        S(ion_spectrum); S(src_spectrum_file); S(ext_spectrum); S(spectrum_type); D(ext_scale);
        B(xy_periodic); S(slab_faces); S(slab_top_mode); S(slab_bot_mode); D(slab_top_theta); D(slab_bot_theta);
        D(slab_top_phi); D(slab_bot_phi); D(slab_top_source); D(slab_bot_source); I(slab_nmu);
        S(dust_density_law); D(cext_dust); S(data_dir); S(atomic_dir); S(ion_dust_kext);
        S(diffuse_energy_model); D(lambda_ref); D(taumax); D(tauhomo);
        else if (k == "iseed") p.iseed = (int64_t)std::llround(to_dbl(s));
        B(ion_metal_abs); B(metal_ne); B(metal_heat); B(metal_freefree); B(fe_levels_full);
        else if (k == "abund_c") p.abund_C = to_dbl(s);
        else if (k == "abund_n") p.abund_N = to_dbl(s);
        else if (k == "abund_o") p.abund_O = to_dbl(s);
        else if (k == "abund_ne") p.abund_Ne = to_dbl(s);
        else if (k == "abund_s") p.abund_S = to_dbl(s);
        else if (k == "abund_ar") p.abund_Ar = to_dbl(s);
        else if (k == "abund_mg") p.abund_Mg = to_dbl(s);
        else if (k == "abund_fe") p.abund_Fe = to_dbl(s);
        else if (k == "abund_si") p.abund_Si = to_dbl(s);
        else if (k == "abund_cl") p.abund_Cl = to_dbl(s);
        else if (k == "abund_ca") p.abund_Ca = to_dbl(s);
        else if (k == "dgr") p.DGR = to_dbl(s);
        else if (k == "he_abund") p.He_abund = to_dbl(s);
        else if (k == "nh_const") p.nH_const = to_dbl(s);
        else if (k == "xhi_init") p.xHI_init = to_dbl(s);
        else if (k == "xhei_init") p.xHeI_init = to_dbl(s);
        else if (k == "xheii_init") p.xHeII_init = to_dbl(s);
        B(ion_peel); B(peel_bins); B(save_direc0); I(nxim); I(nyim); D(distance); D(dxim); D(dyim);
        else if (k == "alpha" || k == "beta" || k == "gamma" || k == "obsx" || k == "obsy" || k == "obsz" ||
                 k == "phase_angle" || k == "inclination_angle" || k == "position_angle") {
            double* arr = k == "alpha" ? p.alpha : k == "beta" ? p.beta : k == "gamma" ? p.gamma_
                        : k == "obsx" ? p.obsx : k == "obsy" ? p.obsy : k == "obsz" ? p.obsz
                        : k == "phase_angle" ? p.phase_angle : k == "inclination_angle" ? p.inclination_angle
                                                                                       : p.position_angle;
            for (size_t j = 0; j < v.size() && j < (size_t)MAX_OBS; ++j)
                if (!v[j].empty()) arr[j] = to_dbl(v[j]);
        }
        else if (k == "src_tstar" || k == "src_lum" || k == "src_x" || k == "src_y" || k == "src_z") {
            double* arr = k == "src_tstar" ? p.src_tstar : k == "src_lum" ? p.src_lum
                        : k == "src_x" ? p.src_x : k == "src_y" ? p.src_y : p.src_z;
            for (size_t j = 0; j < v.size() && j < (size_t)MAX_SRC; ++j)
                if (!v[j].empty()) arr[j] = to_dbl(v[j]);
        } else {
            // keys outside the hot path are accepted and ignored by the oracle
        }
#undef D
#undef I
#undef B
#undef S
    }
    // Derived values, setup.f90:72 (nphotons) and :586-595 (distance unit).
    std::string du = lower(p.distance_unit);
    if (du == "kpc") p.distance2cm = KPC2CM;
    else if (du == "pc") p.distance2cm = PC2CM;
    else if (du == "au") p.distance2cm = AU2CM;
    else if (du == "cm") p.distance2cm = 1.0;
    if (p.diffuse_field && p.case_ab != "A") p.case_ab = "A";  // setup.f90:580-583
    if (p.source_geometry == "external" || p.source_geometry == "external_rec" ||
        p.source_geometry == "external_sph") {   // the external-only shorthand, setup.f90:240-258
        p.ext_geometry = p.source_geometry == "external_sph" ? "sph" : "rec";
        p.nsource = 0;
        p.source_geometry = "external";
    }
    if (p.grid_type == "uniform") p.grid_type = "car";
    if (p.source_geometry == "slab") p.nsource = 0;   // setup.f90:327
    (void)err;
    return true;
}

// =========================================================================
// ion_band_mod.f90
// =========================================================================
// build_aligned_edges, ion_band_mod.f90:1053-1214.
bool build_aligned_edges(std::vector<double>& eedge, int nfuv, int nnu,
                         double lo, double hi, const std::vector<double>& meth,
                         std::string* err) {
    const int nion = nnu - nfuv;
    const double MERGE_TOL = 0.01;
    std::vector<double> cand;
    std::vector<int> cpri;
    auto add = [&](double E, int pri) {
        if (E > lo && E < hi) {
            cand.push_back(E);
            cpri.push_back(pri);
        }
    };
    add(ETH_HI, 1);
    add(ETH_HEI, 1);
    add(ETH_HEII, 1);
    for (double m : meth)
        if (m > 0.0) add(m, 0);
    const int ncand = (int)cand.size();
    for (int i = 1; i < ncand; ++i) {
        double tmp = cand[i];
        int itmp = cpri[i];
        int j = i - 1;
        while (j >= 0 && cand[j] > tmp) {
            cand[j + 1] = cand[j];
            cpri[j + 1] = cpri[j];
            --j;
        }
        cand[j + 1] = tmp;
        cpri[j + 1] = itmp;
    }
    std::vector<double> thr;
    std::vector<int> tpri;
    for (int i = 0; i < ncand; ++i) {
        bool dup = false;
        if (!thr.empty() && std::fabs(std::log(cand[i] / thr.back())) < MERGE_TOL) dup = true;
        if (dup) {
            if (cpri[i] > tpri.back()) {
                thr.back() = cand[i];
                tpri.back() = cpri[i];
            }
        } else {
            thr.push_back(cand[i]);
            tpri.push_back(cpri[i]);
        }
    }
    while ((int)thr.size() + 1 > nion) {
        int best = -1;
        double frac = 1.0e30;
        const int nthr = (int)thr.size();
        for (int i = 0; i < nthr; ++i) {
            if (tpri[i] != 0) continue;
            double tmp = (i == 0) ? std::log(thr[i] / lo) : std::log(thr[i] / thr[i - 1]);
            if (i == nthr - 1) tmp = std::min(tmp, std::log(hi / thr[i]));
            else tmp = std::min(tmp, std::log(thr[i + 1] / thr[i]));
            if (tmp < frac) {
                frac = tmp;
                best = i;
            }
        }
        if (best < 0) break;
        thr.erase(thr.begin() + best);
        tpri.erase(tpri.begin() + best);
    }
    const int nthr = (int)thr.size();
    std::vector<double> points;
    points.push_back(lo);
    for (double t : thr) points.push_back(t);
    points.push_back(hi);
    const int nseg = nthr + 1;
    if (nion < nseg) {
        set_err(err, "ion_align_edges: nnu_ion cannot fit the H/He thresholds");
        return false;
    }
    std::vector<double> w(nseg);
    double wsum = 0.0;
    for (int j = 0; j < nseg; ++j) {
        w[j] = std::log(points[j + 1]) - std::log(points[j]);
        wsum = wsum + w[j];
    }
    std::vector<int> nb(nseg);
    int ntot = 0;
    for (int j = 0; j < nseg; ++j) {
        nb[j] = std::max(1, (int)((double)nion * w[j] / wsum));
        ntot += nb[j];
    }
    int r = nion - ntot;
    while (r > 0) {
        int best = 0;
        double frac = -1.0;
        for (int j = 0; j < nseg; ++j) {
            double tmp = (double)nion * w[j] / wsum - (double)nb[j];
            if (tmp > frac) {
                frac = tmp;
                best = j;
            }
        }
        nb[best] += 1;
        r -= 1;
    }
    while (r < 0) {
        int best = -1;
        double frac = -1.0e30;
        for (int j = 0; j < nseg; ++j) {
            if (nb[j] <= 1) continue;
            double tmp = (double)nb[j] - (double)nion * w[j] / wsum;
            if (tmp > frac) {
                frac = tmp;
                best = j;
            }
        }
        if (best < 0) break;
        nb[best] -= 1;
        r += 1;
    }
    int off = nfuv;  // 0-based index of points(1)
    eedge[off] = points[0];
    int ipt = off;
    for (int j = 0; j < nseg; ++j)
        for (int ib = 1; ib <= nb[j]; ++ib) {
            ++ipt;
            eedge[ipt] = std::exp(std::log(points[j]) +
                                  (std::log(points[j + 1]) - std::log(points[j])) * (double)ib / (double)nb[j]);
        }
    return true;
}

// ion_bin_of, ion_band_mod.f90:624-646 (returns a 0-based bin).
int ion_bin_of(const Band& b, double eph, bool include_fuv) {
    int lo = 1, hi = b.nnu_band;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (b.eedge[mid - 1] <= eph) lo = mid; else hi = mid - 1;
    }
    int r = include_fuv ? std::min(std::max(lo, 1), b.nnu_band)
                        : std::min(std::max(lo, b.nfuv_band + 1), b.nnu_band);
    return r - 1;
}

// ---- tabulated spectra and ISRF presets (ion_band_mod.f90:870-911, 1438-1720)
static const double HC_EVANG = 12398.42;   // define.f90:62
static const double H_CGS = 6.62607015e-27;   // define.f90:59

// spec_is_physical, ion_band_mod.f90:870-877.
static bool spec_is_physical(const Par& p) {
    const std::string t = lower(p.spectrum_type);
    return t == "per_ev" || t == "per_hz" || t == "per_ang" || t == "per_um";
}

// ion_ext_preset_id, ion_band_mod.f90:895-911.
static int ext_preset_id(const std::string& name) {
    const std::string t = lower(trim(name));
    if (t == "draine") return 1;
    if (t == "habing") return 2;
    if (t == "mathis") return 3;
    return 0;
}

// draine_je, ion_band_mod.f90:1648-1658.
static double draine_je(double E) {
    if (E < 5.0 || E > 13.6) return 0.0;
    const double E2 = E * E, E3 = E2 * E, E4 = E2 * E2;
    return EV2ERG * (1.658e6 * E2 - 2.152e5 * E3 + 6.919e3 * E4);
}

// bbody_si, ion_band_mod.f90:1700-1720.
static double bbody_si(double T, double lam_um) {
    const double c_si = 2.99792458e8, h_si = 6.62606957e-34, kB_si = 1.3806488e-23;
    const double hc2 = (2.0 * h_si) * (c_si * c_si), hckB = h_si * c_si / kB_si;
    if (T <= 0.0 || lam_um <= 0.0) return 0.0;
    const double lam_m = lam_um * 1.0e-6;
    const double x = hckB / (T * lam_m);
    if (x >= 700.0) return 0.0;
    const double l2 = lam_m * lam_m, l4 = l2 * l2;
    return hc2 / (l4 * lam_m) / (std::exp(x) - 1.0);
}

// mathis_jl_si and mathis_je, ion_band_mod.f90:1660-1698.
static double mathis_je(double E) {
    const double lam = HC_EVANG * 1.0e-4 / E;
    double Jl;
    if (lam < 0.0912) Jl = 0.0;
    else if (lam < 0.110) Jl = 3069.0 * std::pow(lam, 3.4172);
    else if (lam < 0.134) Jl = 1.627;
    else if (lam < 0.250) Jl = 0.0566 * std::pow(lam, -1.6678);
    else Jl = 1.0e-14 * bbody_si(7500.0, lam) + 1.65e-13 * bbody_si(4000.0, lam) + 4.0e-13 * bbody_si(3000.0, lam);
    return Jl * (HC_EVANG * 1.0e-7) / (E * E);
}

// preset_je, ion_band_mod.f90:1627-1637.
static double preset_je(double E, int id) {
    switch (id) {
        case 1: return draine_je(E);
        case 2: return draine_je(E) / 1.71;
        case 3: return mathis_je(E);
        default: return 0.0;
    }
}

// read_shape_table / read_phys_table, ion_band_mod.f90:1438-1597: column
// icol of ncol value columns, converted to (E [eV], per eV), sorted
// ascending by insertion.
static bool read_spec_table(const Par& p, const std::string& fname, int icol, int ncol, std::vector<double>& et,
                            std::vector<double>& ft, std::string* err) {
    std::ifstream in(fname);
    if (!in) {
        set_err(err, ("cannot open " + fname).c_str());
        return false;
    }
    const std::string type = lower(p.spectrum_type);
    et.clear();
    ft.clear();
    std::string line;
    while (std::getline(in, line)) {
        std::string t = trim(line);
        if (t.empty() || t[0] == '#') continue;
        for (auto& ch : t) {
            if (ch == ',') ch = ' ';
            if (ch == 'd' || ch == 'D') ch = 'e';
        }
        std::istringstream ss(t);
        std::vector<double> row;
        double v;
        while ((int)row.size() < ncol + 1 && ss >> v) row.push_back(v);
        if ((int)row.size() < ncol + 1) {
            set_err(err, (fname + ": too few columns").c_str());
            return false;
        }
        const double c1 = row[0], cv = row[icol];
        double ee = c1, xe = cv;
        if (type == "per_hz") {
            ee = H_CGS * c1 / EV2ERG;
            xe = cv * EV2ERG / H_CGS;
        } else if (type == "per_ang") {
            ee = HC_EVANG / c1;
            xe = cv * HC_EVANG / (ee * ee);
        } else if (type == "per_um") {
            const double hc = HC_EVANG * 1.0e-4;
            ee = hc / c1;
            xe = cv * hc / (ee * ee);
        }
        et.push_back(ee);
        ft.push_back(xe);
    }
    const int n = (int)et.size();
    for (int i = 2; i <= n; ++i)
        for (int j = i; j >= 2; --j) {
            if (et[j - 2] <= et[j - 1]) break;
            std::swap(et[j - 2], et[j - 1]);
            std::swap(ft[j - 2], ft[j - 1]);
        }
    return true;
}

// source_band_luminosity, ion_band_mod.f90:379-399.
static bool source_band_L(const Sampler& s, bool is_abs, double scale, double eion_min, double* L, std::string* err) {
    if (is_abs && scale <= 0.0) {
        *L = s.total_integral;
        return true;
    }
    const double f_ion = 1.0 - energy_cdf_value(s, eion_min);
    if (f_ion <= 0.0) {
        set_err(err, "cannot rescale a source with no ionizing-band luminosity");
        return false;
    }
    *L = scale / f_ion;
    return true;
}

// build_point_source_sampler, ion_band_mod.f90:437-495 (is 1-based).
static bool point_source_sampler(const Par& p, int is, bool multi, double elo, const std::vector<double>& knots,
                                 Sampler& s, double* L, std::string* err) {
    const double scale = multi ? p.src_lum[is - 1] : p.luminosity;
    const bool phys = spec_is_physical(p);
    std::vector<double> et, ft;
    if (!p.src_spectrum_file.empty()) {
        if (!read_spec_table(p, p.src_spectrum_file, is, std::max(p.nsource, 1), et, ft, err)) return false;
        if (!build_tabulated_band_sampler(s, et, ft, elo, p.eion_max, err)) return false;
        return source_band_L(s, phys, scale, p.eion_min, L, err);
    }
    const double tst = multi ? p.src_tstar[is - 1] : -1.0;
    if (tst > 0.0) {
        if (!build_planck_sampler(s, tst, elo, p.eion_max, p.source_cdf_tol, knots, err)) return false;
        return source_band_L(s, false, scale, p.eion_min, L, err);
    }
    if (!p.ion_spectrum.empty()) {
        if (!read_spec_table(p, p.ion_spectrum, 1, 1, et, ft, err)) return false;
        if (!build_tabulated_band_sampler(s, et, ft, elo, p.eion_max, err)) return false;
        return source_band_L(s, phys, scale, p.eion_min, L, err);
    }
    if (p.tstar <= 0.0) {
        set_err(err, "oracle: point source needs a spectrum");
        return false;
    }
    if (!build_planck_sampler(s, p.tstar, elo, p.eion_max, p.source_cdf_tol, knots, err)) return false;
    return source_band_L(s, false, scale, p.eion_min, L, err);
}

// build_external_field_sampler, ion_band_mod.f90:516-615.
static bool external_field_sampler(const Par& p, double elo, const std::vector<double>& knots, const double* box,
                                   Sampler& s, double* L, std::string* err) {
    const int presid = ext_preset_id(p.ext_spectrum);
    const bool is_abs = presid > 0 || (spec_is_physical(p) && !p.ext_spectrum.empty());
    std::vector<double> et, ft;
    if (presid > 0) {
        const double ehi = std::min(p.eion_max, 13.6);
        if (ehi <= elo) {
            set_err(err, "the ISRF preset does not overlap the band");
            return false;
        }
        const int N = 4096;
        et.resize(N);
        ft.resize(N);
        for (int k = 1; k <= N; ++k) {
            et[k - 1] = elo + (ehi - elo) * (double)(k - 1) / (double)(N - 1);
            ft[k - 1] = preset_je(et[k - 1], presid) * p.ext_scale;
        }
        if (!build_tabulated_sampler(s, et, ft, err)) return false;
    } else if (!p.ext_spectrum.empty()) {
        if (!read_spec_table(p, p.ext_spectrum, 1, 1, et, ft, err)) return false;
        if (!build_tabulated_band_sampler(s, et, ft, elo, p.eion_max, err)) return false;
    } else if (p.ext_tstar > 0.0) {
        if (!build_planck_sampler(s, p.ext_tstar, elo, p.eion_max, p.source_cdf_tol, knots, err)) return false;
    } else if (!p.ion_spectrum.empty()) {
        if (!read_spec_table(p, p.ion_spectrum, 1, 1, et, ft, err)) return false;
        if (!build_tabulated_band_sampler(s, et, ft, elo, p.eion_max, err)) return false;
    } else {
        if (!build_planck_sampler(s, p.tstar, elo, p.eion_max, p.source_cdf_tol, knots, err)) return false;
    }
    double asurf;
    if (p.ext_geometry == "sph") {
        asurf = 4.0 * PI * ((p.rmax * p.distance2cm) * (p.rmax * p.distance2cm));
    } else {
        const double xr = box[0] * p.distance2cm, yr = box[1] * p.distance2cm, zr = box[2] * p.distance2cm;
        asurf = 2.0 * (xr * yr + yr * zr + zr * xr);
    }
    if (is_abs) {
        *L = p.ext_intensity > 0.0 ? PI * asurf * p.ext_intensity : PI * asurf * s.total_integral;
        return true;
    }
    const double f_ion = 1.0 - energy_cdf_value(s, p.eion_min);
    if (f_ion <= 0.0) {
        set_err(err, "the external spectrum has no luminosity inside the ionizing band");
        return false;
    }
    *L = PI * p.ext_intensity * asurf / f_ion;
    return true;
}

// ion_setup (ion_band_mod.f90:122-258) for point sources, the external
// field and the slab, with each component's spectrum chain, plus
// setup_continuous_source_sampler / build_point_source_sampler
// (:275-353, :437-495) and ion_qmc_ndim (:654-663).
bool band_setup(const Par& p0, Band& b, std::string* err, const std::vector<double>& metal_eth, const double* box) {
    // setup.f90:374-442: the luminosity sentinel and the point sources' scales
    Par p = p0;
    {
        const int npt = p.source_geometry == "external" ? 0 : p.nsource;
        const bool src_abs = spec_is_physical(p) && (!p.src_spectrum_file.empty() || !p.ion_spectrum.empty());
        if (p.luminosity < -900.0 && !(npt >= 1 && src_abs)) p.luminosity = 1.0;
        if (npt == 1 && p.src_lum[0] <= 0.0) {
            p.src_x[0] = p.xs_point; p.src_y[0] = p.ys_point; p.src_z[0] = p.zs_point;
            p.src_lum[0] = p.luminosity;
        } else if (npt > 1) {
            int nset = 0;
            for (int i = 0; i < npt; ++i) if (p.src_lum[i] > 0.0) ++nset;
            if (nset == 0 && !src_abs) {
                for (int i = 0; i < npt; ++i) p.src_lum[i] = p.luminosity / (double)npt;
            } else if (nset != 0 && nset != npt) {
                set_err(err, "set par%src_lum for ALL sources or for NONE");
                return false;
            }
        }
    }
    int nfuv = 0;
    if (p.add_fuv) {
        if (p.efuv_min >= p.eion_min) {
            set_err(err, "add_fuv requires efuv_min < eion_min");
            return false;
        }
        nfuv = p.nnu_fuv;
    }
    const int nnu = p.nnu_ion + nfuv;
    b.nnu_band = nnu;
    b.nfuv_band = nfuv;
    b.eedge.assign(nnu + 1, 0.0);
    const double lo = std::log(p.eion_min), hi = std::log(p.eion_max);
    for (int i = 1; i <= nfuv; ++i)
        b.eedge[i - 1] = std::exp(std::log(p.efuv_min) + (lo - std::log(p.efuv_min)) * (double)(i - 1) / (double)nfuv);
    const std::vector<double>& meth = metal_eth;   // ion_band_mod.f90:166-175
    if (p.ion_align_edges) {
        if (!build_aligned_edges(b.eedge, nfuv, nnu, p.eion_min, p.eion_max, meth, err)) return false;
    } else {
        for (int i = nfuv + 1; i <= nnu + 1; ++i)
            b.eedge[i - 1] = std::exp(lo + (hi - lo) * (double)(i - 1 - nfuv) / (double)(nnu - nfuv));
    }
    if (p.source_geometry == "slab") {   // slab_setup, :2083-2130, and ion_setup :312-328
        if (!p.xy_periodic || !box) {
            set_err(err, "source_geometry='slab' needs par%xy_periodic and the box extent");
            return false;
        }
        b.slab = true;
        b.ncomp = 1;
        b.multi_src = false;
        b.ext_ic = -1;
        b.qmc_ndim = 6;
        const std::string faces = lower(p.slab_faces);
        b.slab_lit[0] = faces == "top" || faces == "both";
        b.slab_lit[1] = faces == "bottom" || faces == "both";
        const double src[2] = {p.slab_top_source, p.slab_bot_source};
        const double theta[2] = {p.slab_top_theta, p.slab_bot_theta};
        const double deg2rad = PI / 180.0;
        b.slab_phi[0] = p.slab_top_phi * deg2rad;
        b.slab_phi[1] = p.slab_bot_phi * deg2rad;
        b.slab_mode[0] = lower(p.slab_top_mode) == "isotropic" ? 1 : 0;
        b.slab_mode[1] = lower(p.slab_bot_mode) == "isotropic" ? 1 : 0;
        b.slab_azface = (box[0] * p.distance2cm) * (box[1] * p.distance2cm);
        for (int f = 0; f < 2; ++f) {
            b.slab_Fz[f] = 0.0;
            b.slab_mu[f] = 1.0;
            if (!b.slab_lit[f]) continue;
            if (b.slab_mode[f] == 1) {
                b.slab_Fz[f] = PI * src[f];
            } else {
                b.slab_mu[f] = std::cos(theta[f] * deg2rad);
                b.slab_Fz[f] = b.slab_mu[f] * src[f];
            }
        }
        const double fz = b.slab_Fz[0] + b.slab_Fz[1];
        if (!(fz * b.slab_azface > 0.0)) {
            set_err(err, "source_geometry='slab' has zero entering flux");
            return false;
        }
        b.slab_ptop = b.slab_Fz[0] / fz;
        std::vector<double> knots = {ETH_HI, ETH_HEI, ETH_HEII};
        for (double e : meth) knots.push_back(e);
        if (p.add_fuv) knots.push_back(p.eion_min);
        b.samplers.resize(1);
        const double elo = p.add_fuv ? p.efuv_min : p.eion_min;
        double unused;
        if (!point_source_sampler(p, 1, false, elo, knots, b.samplers[0], &unused, err)) return false;
        const double f_ion = 1.0 - energy_cdf_value(b.samplers[0], p.eion_min);
        if (f_ion <= 0.0) {
            set_err(err, "the slab spectrum has no luminosity inside the ionizing band");
            return false;
        }
        b.ion_Ltot = fz * b.slab_azface / f_ion;
        return true;
    }
    if (p.source_geometry != "point" && p.source_geometry != "external") {
        set_err(err, "oracle: only point sources, external fields and the slab are restated");
        return false;
    }
    // components, ion_band_mod.f90:188-199 and 683-711: the point sources,
    // then the external field
    const bool ext_on = p.ext_intensity > 0.0 || ext_preset_id(p.ext_spectrum) > 0 ||
                        (spec_is_physical(p) && !p.ext_spectrum.empty());   // external_on, :884-889
    if (ext_on && !box && p.ext_geometry != "sph") {
        set_err(err, "oracle: the external field needs the box extent");
        return false;
    }
    b.ncomp = p.nsource + (ext_on ? 1 : 0);
    b.multi_src = b.ncomp >= 2;
    b.ext_ic = ext_on ? b.ncomp - 1 : -1;
    b.qmc_ndim = (!b.multi_src && p.source_geometry == "point") ? 3 : 7;   // ion_qmc_ndim, :654-663
    const double elo = p.add_fuv ? p.efuv_min : p.eion_min;
    // photoionization_threshold_knots, ion_band_mod.f90:408-419
    std::vector<double> knots = {ETH_HI, ETH_HEI, ETH_HEII};
    for (double e : meth) knots.push_back(e);
    if (p.add_fuv) knots.push_back(p.eion_min);
    b.samplers.resize(b.ncomp);
    std::vector<double> band_L(b.ncomp);
    for (int ic = 0; ic < b.ncomp; ++ic) {
        if (ic == b.ext_ic) {
            if (!external_field_sampler(p, elo, knots, box, b.samplers[ic], &band_L[ic], err)) return false;
            continue;
        }
        if (!point_source_sampler(p, ic + 1, b.multi_src, elo, knots, b.samplers[ic], &band_L[ic], err)) return false;
    }
    b.ion_Ltot = 0.0;
    for (double L : band_L) b.ion_Ltot += L;
    if (b.multi_src) {
        b.comp_kind.resize(b.ncomp);
        b.src_cdf.resize(b.ncomp);
        for (int ic = 0; ic < b.ncomp; ++ic) b.comp_kind[ic] = ic == b.ext_ic ? 0 : ic + 1;
        b.src_x.assign(p.src_x, p.src_x + MAX_SRC);
        b.src_y.assign(p.src_y, p.src_y + MAX_SRC);
        b.src_z.assign(p.src_z, p.src_z + MAX_SRC);
        b.src_cdf[0] = band_L[0];
        for (int ic = 1; ic < b.ncomp; ++ic) b.src_cdf[ic] = b.src_cdf[ic - 1] + band_L[ic];
        const double last = b.src_cdf[b.ncomp - 1];
        for (auto& c : b.src_cdf) c = c / last;
    }
    return true;
}

// =========================================================================
// Tallies
// =========================================================================
void Tally::reset(int nleaf, int nnu, int ntr, bool dust, bool fuvt) {
    hhe.assign((size_t)6 * nleaf, 0.0);
    jt.assign((size_t)nnu * nleaf, 0.0);
    metal.assign((size_t)2 * ntr * nleaf, 0.0);
    dust_abs.assign(dust ? (size_t)nleaf : 0, 0.0);
    fuv.assign(fuvt ? (size_t)nleaf : 0, 0.0);
    emitted = absorbed = escaped = 0;
    direct_segments = scattered_segments = 0;
    img_dir.clear(); img_sca.clear(); img_dir0.clear();
}
void Tally::add(const Tally& o) {
    for (size_t i = 0; i < img_dir.size() && i < o.img_dir.size(); ++i) img_dir[i] += o.img_dir[i];
    for (size_t i = 0; i < img_sca.size() && i < o.img_sca.size(); ++i) img_sca[i] += o.img_sca[i];
    for (size_t i = 0; i < img_dir0.size() && i < o.img_dir0.size(); ++i) img_dir0[i] += o.img_dir0[i];
    for (size_t i = 0; i < hhe.size(); ++i) hhe[i] += o.hhe[i];
    for (size_t i = 0; i < jt.size(); ++i) jt[i] += o.jt[i];
    for (size_t i = 0; i < metal.size(); ++i) metal[i] += o.metal[i];
    for (size_t i = 0; i < dust_abs.size(); ++i) dust_abs[i] += o.dust_abs[i];
    for (size_t i = 0; i < fuv.size(); ++i) fuv[i] += o.fuv[i];
    for (size_t i = 0; i < slab.size() && i < o.slab.size(); ++i) slab[i] += o.slab[i];
    emitted += o.emitted;
    absorbed += o.absorbed;
    escaped += o.escaped;
    direct_segments += o.direct_segments;
    scattered_segments += o.scattered_segments;
}

// =========================================================================
// Simulation: setup (setup.f90, grid_mod_amr.f90:64-147,163-200,
// gas_state_mod.f90:41-90, ion_band_mod.f90:122-258)
// =========================================================================
bool Sim::setup(const std::string& nl, std::string* err) {
    if (!parse_namelist(nl, par, err)) return false;
    rm.recomb = par.recomb_model == "hui_gnedin" ? RECOMB_HUI_GNEDIN : RECOMB_BADNELL_MILNE;
    rm.ci = par.ci_model == "dere_hybrid" ? CI_DERE_HYBRID : CI_VORONOV;
    qmc.setup(par.qmc_seed);
    if (par.grid_type != "car" && par.grid_type != "amr") {
        set_err(err, "oracle: grid_type must be 'car' or 'amr'");
        return false;
    }
    if (par.grid_type == "car" && !par.amr_file.empty()) {
        set_err(err, "oracle: a 'car' grid from a leaf file is not restated");
        return false;
    }
    if (par.use_sec_ion) {
        set_err(err, "oracle: use_sec_ion is not restated");
        return false;
    }
    if (par.ion_add_dust) {
        if (par.dust_density_law != "global_dgr" && par.dust_density_law != "none") {
            set_err(err, "oracle: dust_density_law must be 'global_dgr' or 'none'");
            return false;
        }
        if (par.taumax > 0.0 || par.tauhomo > 0.0) {
            set_err(err, "oracle: taumax / tauhomo normalisation is not restated");
            return false;
        }
        if (!dust.read(par.ion_dust_kext, par.lambda_ref, err)) return false;   // ion_dust_read
    }
    if (par.solve_te) {
        th = new Thermal();
        if (!th->setup(par, err)) return false;
    }
    std::vector<double> xl, yl, zl;
    if (par.grid_type == "amr") {
        // leaf-list octree, grid_mod_amr.f90:50-62 and octree_mod.f90:342-479
        std::vector<int> lev;
        double boxlen = 0.0;
        if (!read_leaf_list(par.amr_file, xl, yl, zl, lev, st.nH, &boxlen, err)) return false;
        const double half = 0.5 * boxlen;
        par.xmax = par.ymax = par.zmax = half;
        grid.car = false;
        grid.oct = new Octree();
        grid.oct->build(xl, yl, zl, lev, half);
        grid.nleaf = (int)xl.size();
        grid.xmin = grid.ymin = grid.zmin = -half;
        grid.xmax = grid.ymax = grid.zmax = half;
        grid.dcell = 0.0;
        grid.lhalf.resize(grid.nleaf);
        grid.lcx.resize(grid.nleaf); grid.lcy.resize(grid.nleaf); grid.lcz.resize(grid.nleaf);
        for (int l = 0; l < grid.nleaf; ++l) {
            const int c = grid.oct->icell_of_leaf[l];
            grid.lhalf[l] = grid.oct->ch[c];
            grid.lcx[l] = grid.oct->cx[c]; grid.lcy[l] = grid.oct->cy[c]; grid.lcz[l] = grid.oct->cz[c];
        }
    } else {
        // namelist car grid, grid_mod_amr.f90:64-133,193-198 and octree_mod.f90:648-674
        grid.car = true;
        grid.nx = par.nx;
        grid.ny = par.ny;
        grid.nz = par.nz;
        grid.nleaf = par.nx * par.ny * par.nz;
        grid.xmin = -par.xmax; grid.xmax = par.xmax;
        grid.ymin = -par.ymax; grid.ymax = par.ymax;
        grid.zmin = -par.zmax; grid.zmax = par.zmax;
        grid.dcell = (grid.xmax - grid.xmin) / (double)grid.nx;
        const double dcx = 2.0 * par.xmax / (double)par.nx;
        const double dcy = 2.0 * par.ymax / (double)par.ny;
        const double dcz = 2.0 * par.zmax / (double)par.nz;
        st.nH.assign(grid.nleaf, 1.0);
        xl.resize(grid.nleaf); yl.resize(grid.nleaf); zl.resize(grid.nleaf);
        int il = 0;
        for (int iz = 0; iz < par.nz; ++iz)
            for (int iy = 0; iy < par.ny; ++iy)
                for (int ix = 0; ix < par.nx; ++ix, ++il) {
                    xl[il] = -par.xmax + ((double)ix + 0.5) * dcx;
                    yl[il] = -par.ymax + ((double)iy + 0.5) * dcy;
                    zl[il] = -par.zmax + ((double)iz + 0.5) * dcz;
                }
        grid.lhalf.assign(grid.nleaf, 0.5 * grid.dcell);
        grid.lcx.resize(grid.nleaf); grid.lcy.resize(grid.nleaf); grid.lcz.resize(grid.nleaf);
        for (int l = 0; l < grid.nleaf; ++l) {   // cell_cx, octree_mod.f90:113-121
            const int ix = l % grid.nx, iy = (l / grid.nx) % grid.ny, iz = l / (grid.nx * grid.ny);
            grid.lcx[l] = grid.xmin + ((double)ix + 0.5) * grid.dcell;
            grid.lcy[l] = grid.ymin + ((double)iy + 0.5) * grid.dcell;
            grid.lcz[l] = grid.zmin + ((double)iz + 0.5) * grid.dcell;
        }
    }
    const int nleaf = grid.nleaf;
    // gas-density model on the leaf centres, grid_mod_amr.f90:137-147
    for (int il = 0; il < nleaf; ++il) {
        if (par.nH_const >= 0.0) st.nH[il] = par.nH_const;
        if (par.rmax > 0.0 || par.rmin > 0.0) {
            const double rho = std::sqrt(xl[il] * xl[il] + yl[il] * yl[il] + zl[il] * zl[il]);
            if (par.rmax > 0.0 && rho > par.rmax) st.nH[il] = 0.0;
            if (par.rmin > 0.0 && rho < par.rmin) st.nH[il] = 0.0;
        }
    }
    // gas_state_setup, gas_state_mod.f90:58-77
    st.xHI.assign(nleaf, par.xHI_init);
    st.xHeI.assign(nleaf, par.xHeI_init);
    st.xHeII.assign(nleaf, par.xHeII_init);
    st.ne.resize(nleaf);
    st.Te.assign(nleaf, par.te_fixed);
    for (int i = 0; i < nleaf; ++i)
        st.ne[i] = st.nH[i] * ((1.0 - st.xHI[i]) +
                               par.He_abund * (st.xHeII[i] + 2.0 * std::max(0.0, 1.0 - st.xHeI[i] - st.xHeII[i])));
    // species before the band: the metal thresholds pin band edges and
    // sampler knots (main.f90:64-83)
    std::vector<double> meth;
    if (par.use_metals) {
        sp = new Species();
        if (!sp->setup(par, nleaf, err)) return false;
        meth = sp->thresholds();
    }
    {
        const double box[3] = {grid.xmax - grid.xmin, grid.ymax - grid.ymin, grid.zmax - grid.zmin};
        if (!band_setup(par, band, err, meth, box)) return false;
    }
    if (par.diffuse_field) milne.setup(par.eion_max);   // main.f90:102
    if (par.diffuse_field && par.hei_diffuse) {          // main.f90:107-112
        std::string dir = par.data_dir;
        if (dir.empty()) {   // the directory above atomic_dir (<data_dir>/atomic)
            const size_t k = par.atomic_dir.find_last_of('/');
            dir = par.atomic_dir.empty() ? std::string("data")
                                         : (k == std::string::npos ? std::string(".") : par.atomic_dir.substr(0, k));
        }
        if (!hei2ph.setup(dir + "/HeI2phot.dat", par.eion_max)) {
            set_err(err, ("cannot read " + dir + "/HeI2phot.dat").c_str());
            return false;
        }
    }
    if (par.launch_sequence != "sobol") {
        set_err(err, "oracle: only the sobol launch sequence is restated");
        return false;
    }
    // grey dust opacity per code length of each leaf, grid_mod_amr.f90:233-278
    st.rhokap.assign(nleaf, 0.0);
    if (par.ion_add_dust && par.dust_density_law == "global_dgr")
        for (int il = 0; il < nleaf; ++il) st.rhokap[il] = st.nH[il] * par.cext_dust * par.DGR * par.distance2cm;
    tally.reset(nleaf, band.nnu_band, metals() ? sp->ntr : 0, par.ion_add_dust, par.add_fuv);
    gamma_HI.assign(nleaf, 0.0); gamma_HeI.assign(nleaf, 0.0); gamma_HeII.assign(nleaf, 0.0);
    heat_HI.assign(nleaf, 0.0); heat_HeI.assign(nleaf, 0.0); heat_HeII.assign(nleaf, 0.0);
    heat_dust.assign(nleaf, 0.0); g0_fuv.assign(nleaf, 0.0);
    opacity_fill();   // gas_opacity_setup -> gas_opacity_fill (gas_opacity_mod.f90:240-290)
    peel_setup();     // ion_peel_setup: observers and image plane
    return true;
}

bool Sim::metals() const { return par.use_metals && sp != nullptr && !sp->el.empty(); }

void Sim::opacity_fill() {
    if (metals()) sp->stage_cache_refresh(st, rm);
}

void Sim::metal_sigma(Photon& ph) const {
    ph.nm = 0;
    if (metals()) ph.nm = sp->packet_sigma(ph.E, ph.sm);
    // the dust part of build_ion_packet_physics (ion_packet_mod.f90:42-50)
    ph.dust_abs = ph.dust_sca = ph.dust_g = 0.0;
    if (par.ion_add_dust) {
        ph.dust_abs = dust.sabs_at(ph.E);
        ph.dust_sca = dust.ssca_at(ph.E);
        ph.dust_g = dust.g_at(ph.E);
    }
    ph.nscatt = 0;
    ph.inside = true;
}

// emit_slab_qmc, ion_band_mod.f90:2183-2208.
void Sim::emit_slab(double u_face, double u_c1, double u_c2, double u_mu, double u_phi, Photon& ph) const {
    const double xr = grid.xmax - grid.xmin, yr = grid.ymax - grid.ymin, zr = grid.zmax - grid.zmin;
    const double span = std::min(xr, std::min(yr, zr));
    const double nudge = 1.0e-6 * span;
    int f = 1;
    if (u_face > band.slab_ptop) f = 2;
    const double sgn = f == 1 ? -1.0 : 1.0;
    ph.x = grid.xmin + xr * u_c1;
    ph.y = grid.ymin + yr * u_c2;
    ph.z = f == 1 ? grid.zmax - nudge : grid.zmin + nudge;
    double mu, phv;
    if (band.slab_mode[f - 1] == 1) {
        mu = std::max(std::sqrt(u_mu), 1.0e-6);
        phv = TWOPI * u_phi;
    } else {
        mu = band.slab_mu[f - 1];
        phv = band.slab_phi[f - 1];
    }
    const double sinm = std::sqrt(std::max(1.0 - mu * mu, 0.0));
    ph.kx = sinm * std::cos(phv);
    ph.ky = sinm * std::sin(phv);
    ph.kz = sgn * mu;
}

// slab_bnd_add, jtally_mod.f90:76-86.
void Sim::slab_add(Tally& t, double kz, double lum) const {
    if (t.slab.empty()) return;
    const int nmu = par.slab_nmu;
    const double mu = std::fabs(kz);
    const int ib = std::min(std::max((int)(mu * nmu) + 1, 1), nmu);
    const int face = kz > 0.0 ? 1 : 2;
    t.slab[(size_t)(face - 1) * nmu + (ib - 1)] += lum;
}

// slab_wrap_xy, raytrace_amr.f90:330-345 (faces 0-based: 0 +x, 1 -x, 2 +y, 3 -y).
void Sim::slab_wrap_xy(int iface, double& x, double& y) const {
    switch (iface) {
        case 0: x = grid.xmin; break;
        case 1: x = grid.xmax; break;
        case 2: y = grid.ymin; break;
        case 3: y = grid.ymax; break;
        default: break;
    }
}

// emit_external_rec_qmc, ion_band_mod.f90:2253-2323.
void Sim::emit_external_rec(double u_mu, double u_phi, double u_face, double u_c1, double u_c2, Photon& ph) const {
    const double xr = grid.xmax - grid.xmin, yr = grid.ymax - grid.ymin, zr = grid.zmax - grid.zmin;
    const double nudge = 1.0e-6 * std::min(xr, std::min(yr, zr));
    double farea[6], fcum[6];
    farea[0] = yr * zr; farea[1] = farea[0];
    farea[2] = zr * xr; farea[3] = farea[2];
    farea[4] = xr * yr; farea[5] = farea[4];
    fcum[0] = farea[0];
    for (int i = 1; i < 6; ++i) fcum[i] = fcum[i - 1] + farea[i];
    const double fpick = u_face * fcum[5];
    int iface = 6;
    for (int i = 0; i < 6; ++i)
        if (fpick <= fcum[i]) { iface = i + 1; break; }
    const double mu = std::sqrt(u_mu), sinm = std::sqrt(1.0 - mu * mu), phi = TWOPI * u_phi;
    const double cphi = std::cos(phi), sphi = std::sin(phi);
    ph.from_external = true;
    ph.snx = iface == 1 ? -1.0 : iface == 2 ? 1.0 : 0.0;
    ph.sny = iface == 3 ? -1.0 : iface == 4 ? 1.0 : 0.0;
    ph.snz = iface == 5 ? -1.0 : iface == 6 ? 1.0 : 0.0;
    switch (iface) {
        case 1: ph.x = grid.xmax - nudge; ph.y = grid.ymin + yr * u_c1; ph.z = grid.zmin + zr * u_c2;
                ph.kx = -mu; ph.ky = sinm * cphi; ph.kz = sinm * sphi; break;
        case 2: ph.x = grid.xmin + nudge; ph.y = grid.ymin + yr * u_c1; ph.z = grid.zmin + zr * u_c2;
                ph.kx = mu; ph.ky = sinm * cphi; ph.kz = sinm * sphi; break;
        case 3: ph.x = grid.xmin + xr * u_c1; ph.y = grid.ymax - nudge; ph.z = grid.zmin + zr * u_c2;
                ph.kx = sinm * cphi; ph.ky = -mu; ph.kz = sinm * sphi; break;
        case 4: ph.x = grid.xmin + xr * u_c1; ph.y = grid.ymin + nudge; ph.z = grid.zmin + zr * u_c2;
                ph.kx = sinm * cphi; ph.ky = mu; ph.kz = sinm * sphi; break;
        case 5: ph.x = grid.xmin + xr * u_c1; ph.y = grid.ymin + yr * u_c2; ph.z = grid.zmax - nudge;
                ph.kx = sinm * cphi; ph.ky = sinm * sphi; ph.kz = -mu; break;
        default: ph.x = grid.xmin + xr * u_c1; ph.y = grid.ymin + yr * u_c2; ph.z = grid.zmin + nudge;
                 ph.kx = sinm * cphi; ph.ky = sinm * sphi; ph.kz = mu; break;
    }
}

// emit_external_sph_qmc and ortho_frame, ion_band_mod.f90:2328-2385.
void Sim::emit_external_sph(double u_mu, double u_phi, double u_cost, double u_saz, Photon& ph) const {
    const double xc = 0.5 * (grid.xmin + grid.xmax), yc = 0.5 * (grid.ymin + grid.ymax), zc = 0.5 * (grid.zmin + grid.zmax);
    const double cost = 2.0 * u_cost - 1.0, sint = std::sqrt(1.0 - cost * cost), phi = TWOPI * u_saz;
    const double rhx = sint * std::cos(phi), rhy = sint * std::sin(phi), rhz = cost;
    ph.x = xc + par.rmax * rhx;
    ph.y = yc + par.rmax * rhy;
    ph.z = zc + par.rmax * rhz;
    ph.from_external = true;
    ph.snx = -rhx; ph.sny = -rhy; ph.snz = -rhz;
    const double nx = -rhx, ny = -rhy, nz = -rhz;
    double tx, ty, tz;
    if (std::fabs(nx) <= std::fabs(ny) && std::fabs(nx) <= std::fabs(nz)) { tx = 0.0; ty = nz; tz = -ny; }
    else if (std::fabs(ny) <= std::fabs(nz)) { tx = -nz; ty = 0.0; tz = nx; }
    else { tx = ny; ty = -nx; tz = 0.0; }
    const double inv = 1.0 / std::sqrt(tx * tx + ty * ty + tz * tz);
    tx = tx * inv; ty = ty * inv; tz = tz * inv;
    const double bx = ny * tz - nz * ty, by = nz * tx - nx * tz, bz = nx * ty - ny * tx;
    const double mu = std::sqrt(u_mu), sinm = std::sqrt(1.0 - mu * mu), ph2 = TWOPI * u_phi;
    const double cphi = std::cos(ph2), sphi = std::sin(ph2);
    ph.kx = -mu * rhx + sinm * (cphi * tx + sphi * bx);
    ph.ky = -mu * rhy + sinm * (cphi * ty + sphi * by);
    ph.kz = -mu * rhz + sinm * (cphi * tz + sphi * bz);
    const double nudge = 1.0e-6 * std::min(grid.xmax - grid.xmin, std::min(grid.ymax - grid.ymin, grid.zmax - grid.zmin));
    ph.x = ph.x - nudge * rhx;
    ph.y = ph.y - nudge * rhy;
    ph.z = ph.z - nudge * rhz;
}

// gen_ion_photon_qmc, ion_band_mod.f90:1880-1935, with emit_point_qmc
// (:2232-2247) and build_ion_packet_physics (ion_packet_mod.f90:21-53).
void Sim::gen_photon_qmc(int64_t ip, Photon& ph) const {
    ph.from_external = false;
    ph.snx = ph.sny = ph.snz = 0.0;
    double u[12];
    for (int d = 1; d <= band.qmc_ndim; ++d) u[d - 1] = qmc.uniform(ip, d, 1);
    double e;
    double umu = 0.0, uphi = 0.0, xs = 0.0, ys = 0.0, zs = 0.0;
    int ic = 0;
    if (band.slab) {   // slab layout (:1895-1898): u1 energy, u2 face, u3/u4 xy, u5 mu, u6 phi
        emit_slab(u[1], u[2], u[3], u[4], u[5], ph);
        e = sample_energy_cdf(band.samplers[0], u[0]);
    } else if (!band.multi_src && band.qmc_ndim == 3) {
        xs = par.xs_point; ys = par.ys_point; zs = par.zs_point;
        umu = u[1]; uphi = u[2];
        e = sample_energy_cdf(band.samplers[0], u[0]);
    } else {
        if (band.multi_src) {
            ic = band.ncomp - 1;
            for (int i = 0; i < band.ncomp; ++i)
                if (u[0] <= band.src_cdf[i]) { ic = i; break; }
            const int ik = band.comp_kind[ic];
            if (ik >= 1) { xs = band.src_x[ik - 1]; ys = band.src_y[ik - 1]; zs = band.src_z[ik - 1]; }
        }
        umu = u[2]; uphi = u[3];
        e = sample_energy_cdf(band.samplers[ic], u[1]);
    }
    if (band.slab) {
    } else if (ic == band.ext_ic) {
        if (par.ext_geometry == "sph") emit_external_sph(u[2], u[3], u[4], u[5], ph);
        else emit_external_rec(u[2], u[3], u[4], u[5], u[6], ph);
    } else {
        ph.x = xs; ph.y = ys; ph.z = zs;
        const double cost = 2.0 * umu - 1.0;
        const double sint = std::sqrt(1.0 - cost * cost);
        const double phi = TWOPI * uphi;
        ph.kx = sint * std::cos(phi);
        ph.ky = sint * std::sin(phi);
        ph.kz = cost;
    }
    ph.inu = ion_bin_of(band, e, true);
    ph.wgt = 1.0;
    ph.Lpacket = band.ion_Ltot / (double)par.nphotons;
    ph.E = e;
    ph.il = amr_walk() ? leaf_find(ph.x, ph.y, ph.z) : -1;   // emit_point_qmc, ion_band_mod.f90:2245
    ph.sHI = sigma_HI(e);
    ph.sHeI = sigma_HeI(e);
    ph.sHeII = sigma_HeII(e);
    metal_sigma(ph);
}

// score_ion_path, ion_score_mod.f90:137-231 (H/He part).
static inline void score(const Sim& s, const Photon& ph, int il, double path_lum, Tally& t) {
    if (path_lum == 0.0) return;
    t.jt[(size_t)s.band.nnu_band * il + ph.inu] += path_lum;
    if (!t.dust_abs.empty()) t.dust_abs[il] += path_lum * ph.dust_abs;
    if (!t.fuv.empty() && ph.E < s.par.eion_min) t.fuv[il] += path_lum;
    if (ph.nscatt > 0) t.scattered_segments += 1;
    else t.direct_segments += 1;
    const double energy = ph.E;
    double c[6];
    c[0] = ph.sHI / (energy * EV2ERG);
    c[1] = ph.sHeI / (energy * EV2ERG);
    c[2] = ph.sHeII / (energy * EV2ERG);
    c[3] = ph.sHI * std::max(1.0 - ETH_HI / energy, 0.0);
    c[4] = ph.sHeI * std::max(1.0 - ETH_HEI / energy, 0.0);
    c[5] = ph.sHeII * std::max(1.0 - ETH_HEII / energy, 0.0);
    double* h = &t.hhe[(size_t)6 * il];
    for (int k = 0; k < 6; ++k) h[k] = h[k] + path_lum * c[k];
    if (ph.nm > 0) s.sp->score(energy, ph.sm, ph.nm, il, path_lum, t.metal.data());
}

// ion_packet_opacity, ion_packet_mod.f90:55-87 (gas, metals and grains).
static inline double opacity(const Sim& s, const Photon& ph, int il) {
    double metal = 0.0;
    if (ph.nm > 0 && s.par.ion_metal_abs) metal = s.sp->cached_opacity(ph.sm, ph.nm, il);
    double kap = s.st.nH[il] *
                 (s.st.xHI[il] * ph.sHI + s.par.He_abund * (s.st.xHeI[il] * ph.sHeI + s.st.xHeII[il] * ph.sHeII) +
                  metal) *
                 s.par.distance2cm;
    if (s.par.ion_add_dust) {
        kap = kap + s.st.rhokap[il] * ph.dust_abs;
        if (s.par.ion_dust_scatter) kap = kap + s.st.rhokap[il] * ph.dust_sca;
    }
    return kap;
}

// dda_init (raytrace_amr.f90:495-532) + raytrace_ion_to_edge_car (:534-592).
void Sim::walk_edge_car(const Photon& ph, Tally& t, double* tau_edge) const {
    const double d = grid.dcell;
    const double pos[3] = {ph.x, ph.y, ph.z};
    const double kk[3] = {ph.kx, ph.ky, ph.kz};
    const double org[3] = {grid.xmin, grid.ymin, grid.zmin};
    const int n[3] = {grid.nx, grid.ny, grid.nz};
    int idx[3];
    for (int a = 0; a < 3; ++a) idx[a] = std::min(std::max((int)((pos[a] - org[a]) / d), 0), n[a] - 1);
    int stp[3];
    double tmax[3], tdel[3];
    for (int a = 0; a < 3; ++a) {
        if (kk[a] > 0.0) {
            stp[a] = 1;
            tmax[a] = (org[a] + (double)(idx[a] + 1) * d - pos[a]) / kk[a];
            tdel[a] = d / kk[a];
        } else if (kk[a] < 0.0) {
            stp[a] = -1;
            tmax[a] = (org[a] + (double)idx[a] * d - pos[a]) / kk[a];
            tdel[a] = -d / kk[a];
        } else {
            stp[a] = 0;
            tmax[a] = HUGEST;
            tdel[a] = HUGEST;
        }
    }
    const double wl = ph.wgt * ph.Lpacket;
    double expo = 1.0, tau = 0.0, t_cur = 0.0;
    int nstep = 0;
    for (;;) {
        if (++nstep > MAX_WALK_STEPS) break;
        const int il = idx[0] + n[0] * (idx[1] + n[1] * idx[2]);
        int a = 0;
        if (tmax[1] < tmax[a]) a = 1;
        if (tmax[2] < tmax[a]) a = 2;
        const double seg = tmax[a] - t_cur;
        const double kap = opacity(*this, ph, il);
        if (kap * seg > 0.0) {
            const double expo_out = expo * std::exp(-kap * seg);
            score(*this, ph, il, wl * (expo - expo_out) / kap, t);
            expo = expo_out;
        } else {
            score(*this, ph, il, wl * expo * seg, t);
        }
        tau = tau + kap * seg;
        if (tau >= TAU_HUGE) break;
        t_cur = tmax[a];
        tmax[a] = tmax[a] + tdel[a];
        idx[a] += stp[a];
        if (idx[a] < 0 || idx[a] >= n[a]) {
            if (par.xy_periodic && a < 2) {   // :575-582, modulo
                idx[a] = ((idx[a] % n[a]) + n[a]) % n[a];
            } else {
                if (a == 2) slab_add(t, ph.kz, expo * wl);   // :583-588
                break;
            }
        }
    }
    *tau_edge = tau;
}

void Sim::walk_edge(const Photon& ph, Tally& t, double* tau_edge) const {
    if (amr_walk()) walk_edge_amr(ph, t, tau_edge);
    else walk_edge_car(ph, t, tau_edge);
}

int Sim::leaf_find(double x, double y, double z) const {
    if (!grid.car) return grid.oct->find_leaf(x, y, z);
    if (x < grid.xmin || x > grid.xmax || y < grid.ymin || y > grid.ymax || z < grid.zmin || z > grid.zmax) return -1;
    int ix = (int)((x - grid.xmin) / grid.dcell);
    int iy = (int)((y - grid.ymin) / grid.dcell);
    int iz = (int)((z - grid.zmin) / grid.dcell);
    ix = std::min(std::max(ix, 0), grid.nx - 1);
    iy = std::min(std::max(iy, 0), grid.ny - 1);
    iz = std::min(std::max(iz, 0), grid.nz - 1);
    return ix + grid.nx * (iy + grid.ny * iz);
}

void Sim::leaf_exit(int il, double x, double y, double z, double kx, double ky, double kz, double* tout,
                    int* iface) const {
    if (!grid.car) {
        grid.oct->cell_exit(grid.oct->icell_of_leaf[il], x, y, z, kx, ky, kz, tout, iface);
        return;
    }
    // cell_cx/cy/cz/ch of the car grid (octree_mod.f90:113-153), then the same exit
    const int ix = il % grid.nx, iy = (il / grid.nx) % grid.ny, iz = il / (grid.nx * grid.ny);
    const double cx = grid.xmin + ((double)ix + 0.5) * grid.dcell;
    const double cy = grid.ymin + ((double)iy + 0.5) * grid.dcell;
    const double cz = grid.zmin + ((double)iz + 0.5) * grid.dcell;
    const double h = 0.5 * grid.dcell;
    double t[6];
    if (kx > 0.0) { t[0] = (cx + h - x) / kx; t[1] = HUGEST; }
    else if (kx < 0.0) { t[0] = HUGEST; t[1] = (cx - h - x) / kx; }
    else { t[0] = HUGEST; t[1] = HUGEST; }
    if (ky > 0.0) { t[2] = (cy + h - y) / ky; t[3] = HUGEST; }
    else if (ky < 0.0) { t[2] = HUGEST; t[3] = (cy - h - y) / ky; }
    else { t[2] = HUGEST; t[3] = HUGEST; }
    if (kz > 0.0) { t[4] = (cz + h - z) / kz; t[5] = HUGEST; }
    else if (kz < 0.0) { t[4] = HUGEST; t[5] = (cz - h - z) / kz; }
    else { t[4] = HUGEST; t[5] = HUGEST; }
    int f = 0;
    for (int k = 1; k < 6; ++k)
        if (t[k] < t[f]) f = k;
    *iface = f;
    *tout = t[f];
}

int Sim::leaf_next(int il, int iface, double x, double y, double z) const {
    if (!grid.car) return grid.oct->next_leaf(grid.oct->icell_of_leaf[il], iface, x, y, z);
    int ix = il % grid.nx, iy = (il / grid.nx) % grid.ny, iz = il / (grid.nx * grid.ny);
    switch (iface) {
        case 0: ++ix; break;
        case 1: --ix; break;
        case 2: ++iy; break;
        case 3: --iy; break;
        case 4: ++iz; break;
        default: --iz; break;
    }
    if (ix < 0 || ix >= grid.nx || iy < 0 || iy >= grid.ny || iz < 0 || iz >= grid.nz) return -1;
    return ix + grid.nx * (iy + grid.ny * iz);
}

// raytrace_ion_to_edge_amr, raytrace_amr.f90:422-486 (no xy-periodic wrap):
// the octree walk, also on the car grid with par%car_walk = 'amr'.
void Sim::walk_edge_amr(const Photon& ph, Tally& t, double* tau_edge) const {
    double x = ph.x, y = ph.y, z = ph.z;
    const double kx = ph.kx, ky = ph.ky, kz = ph.kz;
    int il = ph.il;
    const double wl = ph.wgt * ph.Lpacket;
    double expo = 1.0, tau = 0.0;
    *tau_edge = 0.0;
    if (il < 0) il = leaf_find(x, y, z);
    if (il < 0) return;
    int nstep = 0;
    for (;;) {
        if (++nstep > MAX_WALK_STEPS) break;
        double texit;
        int iface;
        leaf_exit(il, x, y, z, kx, ky, kz, &texit, &iface);
        const double kap = opacity(*this, ph, il);
        if (kap * texit > 0.0) {
            const double expo_out = expo * std::exp(-kap * texit);
            score(*this, ph, il, wl * (expo - expo_out) / kap, t);
            expo = expo_out;
        } else {
            score(*this, ph, il, wl * expo * texit, t);
        }
        tau = tau + kap * texit;
        if (tau >= TAU_HUGE) break;
        x = x + texit * kx;
        y = y + texit * ky;
        z = z + texit * kz;
        int nl = leaf_next(il, iface, x, y, z);
        if (nl < 0 && par.xy_periodic) {   // :473-476
            slab_wrap_xy(iface, x, y);
            if (iface <= 3) nl = leaf_find(x, y, z);
        }
        if (nl < 0) {
            if (iface >= 4) slab_add(t, kz, expo * wl);   // :477-481
            break;
        }
        il = nl;
    }
    *tau_edge = tau;
}

void Sim::walk_to_tau(Photon& ph, double tau_in, Tally& t) const {
    const bool do_tally = ph.nscatt > 0;
    const double wl = ph.wgt * ph.Lpacket;
    if (amr_walk()) {   // raytrace_ion_to_tau_amr, raytrace_amr.f90:348-420
        double x = ph.x, y = ph.y, z = ph.z;
        int il = ph.il;
        if (il < 0) {
            il = leaf_find(x, y, z);
            if (il < 0) {
                ph.inside = false;
                return;
            }
        }
        double tau = 0.0;
        int nstep = 0;
        while (ph.inside) {
            if (++nstep > MAX_WALK_STEPS) {
                ph.inside = false;
                break;
            }
            double texit;
            int iface;
            leaf_exit(il, x, y, z, ph.kx, ph.ky, ph.kz, &texit, &iface);
            const double kap = opacity(*this, ph, il);
            if (tau + texit * kap >= tau_in) {
                const double d = kap > 0.0 ? (tau_in - tau) / kap : texit;
                if (do_tally) score(*this, ph, il, wl * d, t);
                x = x + d * ph.kx; y = y + d * ph.ky; z = z + d * ph.kz;
                break;
            }
            if (do_tally) score(*this, ph, il, wl * texit, t);
            tau = tau + texit * kap;
            x = x + texit * ph.kx; y = y + texit * ph.ky; z = z + texit * ph.kz;
            int nl = leaf_next(il, iface, x, y, z);
            if (nl < 0 && par.xy_periodic) {   // :403-406
                slab_wrap_xy(iface, x, y);
                if (iface <= 3) nl = leaf_find(x, y, z);
            }
            if (nl < 0) {
                ph.inside = false;
                if (iface >= 4) slab_add(t, ph.kz, wl);   // :407-413
                break;
            }
            il = nl;
        }
        ph.x = x; ph.y = y; ph.z = z;
        ph.il = il;
        return;
    }
    // raytrace_ion_to_tau_car, raytrace_amr.f90:594-676: dda_init from the
    // packet's point, the DDA to tau_in, the end point from the total path
    const double d = grid.dcell;
    const double pos[3] = {ph.x, ph.y, ph.z};
    const double kk[3] = {ph.kx, ph.ky, ph.kz};
    const double org[3] = {grid.xmin, grid.ymin, grid.zmin};
    const int n[3] = {grid.nx, grid.ny, grid.nz};
    int idx[3], stp[3];
    double tmax[3], tdel[3];
    for (int a = 0; a < 3; ++a) {
        idx[a] = std::min(std::max((int)((pos[a] - org[a]) / d), 0), n[a] - 1);
        if (kk[a] > 0.0) {
            stp[a] = 1; tmax[a] = (org[a] + (double)(idx[a] + 1) * d - pos[a]) / kk[a]; tdel[a] = d / kk[a];
        } else if (kk[a] < 0.0) {
            stp[a] = -1; tmax[a] = (org[a] + (double)idx[a] * d - pos[a]) / kk[a]; tdel[a] = -d / kk[a];
        } else {
            stp[a] = 0; tmax[a] = HUGEST; tdel[a] = HUGEST;
        }
    }
    double tau = 0.0, t_cur = 0.0;
    int nstep = 0;
    for (;;) {
        if (++nstep > MAX_WALK_STEPS) {
            ph.inside = false;
            break;
        }
        const int il = idx[0] + n[0] * (idx[1] + n[1] * idx[2]);
        int a = 0;
        if (tmax[1] < tmax[a]) a = 1;
        if (tmax[2] < tmax[a]) a = 2;
        const double seg = tmax[a] - t_cur;
        const double kap = opacity(*this, ph, il);
        if (tau + seg * kap >= tau_in) {
            const double ds = kap > 0.0 ? (tau_in - tau) / kap : seg;
            if (do_tally) score(*this, ph, il, wl * ds, t);
            t_cur = t_cur + ds;
            break;
        }
        if (do_tally) score(*this, ph, il, wl * seg, t);
        tau = tau + seg * kap;
        t_cur = tmax[a];
        tmax[a] = tmax[a] + tdel[a];
        idx[a] += stp[a];
        if (idx[a] < 0 || idx[a] >= n[a]) {
            if (par.xy_periodic && a < 2) {   // :639-654
                idx[a] = ((idx[a] % n[a]) + n[a]) % n[a];
            } else {
                ph.inside = false;
                if (a == 2) slab_add(t, ph.kz, wl);   // :655-660
                break;
            }
        }
    }
    ph.x = ph.x + t_cur * ph.kx;
    ph.y = ph.y + t_cur * ph.ky;
    ph.z = ph.z + t_cur * ph.kz;
    if (par.xy_periodic) {   // :666-672
        const double xr = grid.xmax - grid.xmin, yr = grid.ymax - grid.ymin;
        ph.x = ph.x - std::floor((ph.x - grid.xmin) / xr) * xr;
        ph.y = ph.y - std::floor((ph.y - grid.ymin) / yr) * yr;
    }
    if (ph.inside) ph.il = idx[0] + n[0] * (idx[1] + n[1] * idx[2]);
}

void Sim::transport_packet(Photon& ph, Tally& t) const {
    double tau_edge = 0.0;
    walk_edge(ph, t, &tau_edge);
    // ion_score_energy_packet, ion_score_mod.f90:233-252 (x87 extended)
    const double lum = ph.Lpacket * ph.wgt;
    const double tr = std::exp(-std::max(tau_edge, 0.0));
    t.emitted += (long double)lum;
    t.absorbed += (long double)(lum * (1.0 - tr));
    t.escaped += (long double)(lum * tr);
    if (!(par.ion_add_dust && par.ion_dust_scatter)) return;
    if (tau_edge <= 1.0e-12) return;
    const double WMIN = 1.0e-4, PSURV = 0.1;
    // forced first interaction (the direct field is already tallied)
    const double w1 = 1.0 - std::exp(-tau_edge);
    ph.wgt = ph.wgt * w1;
    double tau = -std::log(1.0 - ph.rng.next() * w1);
    walk_to_tau(ph, tau, t);
    int nev = 0;
    while (ph.inside) {
        const int il = ph.il;
        if (il < 0) break;
        if (++nev > MAX_SCATTERINGS) break;
        const double a_eff = st.rhokap[il] * ph.dust_sca / std::max(opacity(*this, ph, il), TINEST);
        ph.wgt = ph.wgt * a_eff;
        if (peel_on && peel_pass) peel_scatter(ph, t);   // raytrace_amr.f90:280-281
        if (ph.wgt < WMIN) {
            if (ph.rng.next() > PSURV) break;
            ph.wgt = ph.wgt / PSURV;
        }
        const double gg = ph.dust_g;
        double cost;
        if (std::fabs(gg) > 1.0e-3) {
            const double q = (1.0 - gg * gg) / (1.0 + gg * (2.0 * ph.rng.next() - 1.0));
            cost = (1.0 + gg * gg - q * q) / (2.0 * gg);
        } else {
            cost = 2.0 * ph.rng.next() - 1.0;
        }
        cost = std::min(std::max(cost, -1.0), 1.0);
        const double sint = std::sqrt(1.0 - cost * cost);
        const double phi = TWOPI * ph.rng.next();
        double kx = ph.kx, ky = ph.ky, kz = ph.kz;
        double norm = std::sqrt(kx * kx + ky * ky + kz * kz);
        if (norm <= 0.0) break;
        kx = kx / norm; ky = ky / norm; kz = kz / norm;
        double ux, uy, uz;
        if (std::fabs(kz) < 0.99) { ux = -ky; uy = kx; uz = 0.0; }
        else { ux = 0.0; uy = -kz; uz = ky; }
        norm = std::sqrt(ux * ux + uy * uy + uz * uz);
        ux = ux / norm; uy = uy / norm; uz = uz / norm;
        const double vx = ky * uz - kz * uy, vy = kz * ux - kx * uz, vz = kx * uy - ky * ux;
        const double cp = std::cos(phi), sp_ = std::sin(phi);
        double nkx = sint * (cp * ux + sp_ * vx) + cost * kx;
        double nky = sint * (cp * uy + sp_ * vy) + cost * ky;
        double nkz = sint * (cp * uz + sp_ * vz) + cost * kz;
        norm = std::sqrt(nkx * nkx + nky * nky + nkz * nkz);
        ph.kx = nkx / norm; ph.ky = nky / norm; ph.kz = nkz / norm;
        ph.nscatt += 1;
        tau = -std::log(std::max(ph.rng.next(), TINEST));
        walk_to_tau(ph, tau, t);
    }
}

// Geometry-only octree walk: the leaf sequence of one ray, 0-based.
int Sim::walk_leaves_amr(double x, double y, double z, double kx, double ky, double kz, int max_steps,
                         int32_t* out) const {
    int il = leaf_find(x, y, z), ns = 0;
    while (il >= 0 && ns < max_steps) {
        out[ns++] = il;
        double texit;
        int iface;
        leaf_exit(il, x, y, z, kx, ky, kz, &texit, &iface);
        x = x + texit * kx;
        y = y + texit * ky;
        z = z + texit * kz;
        il = leaf_next(il, iface, x, y, z);
    }
    return ns;
}

// Geometry-only DDA (no tau cut): the leaf sequence of one ray, 0-based.
int Sim::walk_leaves_car(double x, double y, double z, double kx, double ky,
                         double kz, int max_steps, int32_t* out) const {
    const double d = grid.dcell;
    const double pos[3] = {x, y, z};
    const double kk[3] = {kx, ky, kz};
    const double org[3] = {grid.xmin, grid.ymin, grid.zmin};
    const int n[3] = {grid.nx, grid.ny, grid.nz};
    int idx[3], stp[3];
    double tmax[3], tdel[3];
    for (int a = 0; a < 3; ++a) idx[a] = std::min(std::max((int)((pos[a] - org[a]) / d), 0), n[a] - 1);
    for (int a = 0; a < 3; ++a) {
        if (kk[a] > 0.0) {
            stp[a] = 1; tmax[a] = (org[a] + (double)(idx[a] + 1) * d - pos[a]) / kk[a]; tdel[a] = d / kk[a];
        } else if (kk[a] < 0.0) {
            stp[a] = -1; tmax[a] = (org[a] + (double)idx[a] * d - pos[a]) / kk[a]; tdel[a] = -d / kk[a];
        } else {
            stp[a] = 0; tmax[a] = HUGEST; tdel[a] = HUGEST;
        }
    }
    int ns = 0;
    while (ns < max_steps) {
        out[ns++] = idx[0] + n[0] * (idx[1] + n[1] * idx[2]);
        int a = 0;
        if (tmax[1] < tmax[a]) a = 1;
        if (tmax[2] < tmax[a]) a = 2;
        tmax[a] = tmax[a] + tdel[a];
        idx[a] += stp[a];
        if (idx[a] < 0 || idx[a] >= n[a]) break;
    }
    return ns;
}

// ionizing_field_and_rates, ionizing_field_mod.f90:72-170 (stellar loop,
// static cyclic packet split over threads as photon_schedule_mod's static
// schedule splits packet indices over ranks; ion_score_reduce sums them).
void Sim::transport_pass() {
    const int nleaf = grid.nleaf;
    const int nnu = band.nnu_band;
    const int nt = std::max(1, nthreads);
    std::vector<Tally> loc(nt);
    const int ntr = metals() ? sp->ntr : 0;
    const bool peel = peel_on && peel_pass;
    const size_t npix = peel ? obs.size() * (size_t)nchan * par.nxim * par.nyim : 0;
    for (auto& t : loc) {
        t.reset(nleaf, nnu, ntr, par.ion_add_dust, par.add_fuv);
        t.img_dir.assign(npix, 0.0);
        t.img_sca.assign(npix, 0.0);
        t.img_dir0.assign(peel && par.save_direc0 ? npix : 0, 0.0);
        t.slab.assign(band.slab ? 2 * (size_t)par.slab_nmu : 0, 0.0);
    }
    const int64_t np = par.nphotons;
#pragma omp parallel num_threads(nt)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        Tally& t = loc[tid];
        Photon ph;
        for (int64_t ip = 1 + tid; ip <= np; ip += nt) {
            gen_photon_qmc(ip - 1, ph);
            ph.rng = PacketRng{(uint64_t)par.iseed, (uint64_t)(ip - 1), 0u, 0u};
            if (peel) peel_direct(ph, t);   // ionizing_field_mod.f90:126
            transport_packet(ph, t);
        }
    }
    // diffuse ground-recombination packets from the current state,
    // ionizing_field_mod.f90:139-161 (stream 2, 9 launch dimensions)
    if (par.diffuse_field) {
        diffuse_build(band.ion_Ltot / (double)par.nphotons);
        const int64_t nd = diffuse_nphot;
#pragma omp parallel num_threads(nt)
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            Tally& t = loc[tid];
            Photon ph;
            for (int64_t ip = 1 + tid; ip <= nd; ip += nt) {
                gen_diffuse_qmc(ip - 1, ph);
                ph.rng = PacketRng{(uint64_t)par.iseed, (uint64_t)(ip - 1), 1u, 0u};
                if (peel) peel_direct(ph, t);   // ionizing_field_mod.f90:157
                transport_packet(ph, t);
            }
        }
    }
    tally.reset(nleaf, nnu, ntr, par.ion_add_dust, par.add_fuv);
    tally.img_dir.assign(npix, 0.0);
    tally.img_sca.assign(npix, 0.0);
    tally.img_dir0.assign(peel && par.save_direc0 ? npix : 0, 0.0);
    tally.slab.assign(band.slab ? 2 * (size_t)par.slab_nmu : 0, 0.0);
    for (auto& t : loc) tally.add(t);
    gas_rates_compute();
    if (metals()) {   // species_gamma_compute, species_mod.f90:493-512
        std::vector<double> fac(nleaf);
        for (int il = 0; il < nleaf; ++il) {
            const double w = 2.0 * grid.lhalf[il];
            fac[il] = 1.0 / ((w * w * w) * (par.distance2cm * par.distance2cm));
        }
        sp->gamma_compute(tally.metal, fac);
    }
}

// ---- milne_recomb_spectrum_mod.f90 -------------------------------------------
static double milne_sigma(int ich, double E) {
    return ich == 0 ? sigma_HI(E) : ich == 1 ? sigma_HeI(E) : sigma_HeII(E);
}

void Milne::setup(double eion_max) {   // :99-228 (the table part)
    eth[0] = ETH_HI; eth[1] = ETH_HEI; eth[2] = ETH_HEII;
    const double XMAX = 60.0, TLO = 1.0e2, THI = 1.0e6;
    for (int ix = 1; ix <= NX; ++ix) {
        const double t = (double)(ix - 1) / (double)(NX - 1);
        xg[ix - 1] = XMAX * t * t;
    }
    for (int it = 1; it <= NT; ++it)
        lgT[it - 1] = std::log10(TLO) + (std::log10(THI) - std::log10(TLO)) * (double)(it - 1) / (double)(NT - 1);
    cdf.assign((size_t)NX * NT * NCH, 0.0);
    xbar.assign((size_t)NT * NCH, 0.0);
    frac.assign((size_t)NT * NCH, 0.0);
    for (int ich = 0; ich < NCH; ++ich) {
        for (int it = 0; it < NT; ++it) {
            double* c = &cdf[((size_t)ich * NT + it) * NX];
            const double T_K = std::pow(10.0, lgT[it]);
            const double kT = KBOLTZ_CGS * T_K / EV2ERG;
            auto shape = [&](double x) {
                const double E = eth[ich] + x * kT;
                return E * E * milne_sigma(ich, E) * std::exp(-x);
            };
            const double x_hi = std::min(XMAX, (eion_max - eth[ich]) / kT);
            if (x_hi <= 0.0) {
                for (int ix = 0; ix < NX; ++ix) c[ix] = 1.0;
                xbar[(size_t)ich * NT + it] = 0.0;
                frac[(size_t)ich * NT + it] = 0.0;
                continue;
            }
            double sum_n = 0.0, sum_e = 0.0, sum_xn = 0.0;
            c[0] = 0.0;
            for (int ix = 1; ix <= NX - 1; ++ix) {
                const double xa = xg[ix - 1];
                const double xb = std::min(xg[ix], x_hi);
                if (xb > xa) {
                    const double xm = 0.5 * (xa + xb);
                    const double fa = shape(xa), fm = shape(xm), fb = shape(xb);
                    const double seg_n = (xb - xa) / 6.0 * (fa + 4.0 * fm + fb);
                    const double seg_e = (xb - xa) / 6.0 *
                                         (fa * (eth[ich] + xa * kT) + 4.0 * fm * (eth[ich] + xm * kT) + fb * (eth[ich] + xb * kT));
                    sum_n = sum_n + seg_n;
                    sum_e = sum_e + seg_e;
                    sum_xn = sum_xn + (xb - xa) / 6.0 * (fa * xa + 4.0 * fm * xm + fb * xb);
                }
                c[ix] = sum_e;
            }
            double tail_n = sum_n;
            if (x_hi < XMAX) {
                double xa = x_hi;
                while (xa < XMAX) {
                    const double xb = std::min(xa + 0.25, XMAX);
                    const double xm = 0.5 * (xa + xb);
                    tail_n = tail_n + (xb - xa) / 6.0 * (shape(xa) + 4.0 * shape(xm) + shape(xb));
                    xa = xb;
                }
            }
            if (sum_e > 0.0) {
                for (int ix = 0; ix < NX; ++ix) c[ix] = c[ix] / sum_e;
            } else {
                for (int ix = 0; ix < NX; ++ix) c[ix] = 1.0;
            }
            c[NX - 1] = 1.0;
            xbar[(size_t)ich * NT + it] = sum_xn / std::max(sum_n, TINEST);
            frac[(size_t)ich * NT + it] = sum_n / std::max(tail_n, TINEST);
        }
    }
}

void Milne::tbracket(double T, int& it, double& w) const {   // it 1-based
    double s = (std::log10(std::max(T, TINEST)) - lgT[0]) / (lgT[1] - lgT[0]);
    s = std::min(std::max(s, 0.0), (double)(NT - 1));
    it = std::min((int)s + 1, NT - 1);
    w = s - (double)(it - 1);
}

double Milne::energy_per_recomb(int ich, double T) const {
    int it;
    double w;
    tbracket(T, it, w);
    const double xb = (1.0 - w) * xbar[(size_t)ich * NT + it - 1] + w * xbar[(size_t)ich * NT + it];
    const double fk = (1.0 - w) * frac[(size_t)ich * NT + it - 1] + w * frac[(size_t)ich * NT + it];
    const double kT = KBOLTZ_CGS * T / EV2ERG;
    return fk * (eth[ich] + xb * kT);
}

double Milne::sample(int ich, double T, double u, double eion_max) const {
    int it;
    double w;
    tbracket(T, it, w);
    const double kT = KBOLTZ_CGS * T / EV2ERG;
    const double uu = std::min(std::max(u, 0.0), 1.0);
    const double* c0 = &cdf[((size_t)ich * NT + it - 1) * NX];
    const double* c1 = &cdf[((size_t)ich * NT + it) * NX];
    int lo = 1, hi = NX;
    double ca = (1.0 - w) * c0[lo - 1] + w * c1[lo - 1];
    double cb = (1.0 - w) * c0[hi - 1] + w * c1[hi - 1];
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        const double cm = (1.0 - w) * c0[mid - 1] + w * c1[mid - 1];
        if (uu > cm) { lo = mid; ca = cm; } else { hi = mid; cb = cm; }
    }
    double x;
    if (cb > ca) x = xg[lo - 1] + (xg[hi - 1] - xg[lo - 1]) * (uu - ca) / (cb - ca);
    else x = xg[lo - 1];
    double E = eth[ich] + x * kT;
    return std::min(E, eion_max * (1.0 - 1.0e-12));
}

// ---- hei_twophoton_mod.f90, hei_cascade_mod.f90 ------------------------------
double HeI2ph::shape(double y) const {
    const int n = (int)ty.size();
    if (y <= ty[0] || y >= ty[n - 1]) return 0.0;
    int i = 0;
    while (i < n - 2 && ty[i + 1] < y) ++i;
    return tA[i] + (tA[i + 1] - tA[i]) * (y - ty[i]) / (ty[i + 1] - ty[i]);
}

bool HeI2ph::setup(const std::string& path, double eion_max) {
    std::ifstream f(path);
    if (!f) return false;
    ty.clear(); tA.clear();
    double a, b;
    while (f >> a >> b) { ty.push_back(a); tA.push_back(b); }
    const int n = (int)ty.size();
    if (n < 4) return false;
    double tot = 0.0;   // Simpson over each table interval
    for (int i = 0; i < n - 1; ++i) {
        const double ya = ty[i], yb = ty[i + 1], ym = 0.5 * (ya + yb);
        tot = tot + (yb - ya) / 6.0 * (tA[i] + 4.0 * shape(ym) + tA[i + 1]);
    }
    if (tot <= 0.0) return false;
    const double y_lo = ETH_HI / E_TOT, y_hi = std::min(E_TOT, eion_max) / E_TOT;
    if (y_hi <= y_lo) {
        n_per_decay = 0.0; e_per_decay = 0.0;
        for (int i = 0; i < NCDF; ++i) { cdf_e[i] = 1.0; grid_y[i] = y_lo; }
        return true;
    }
    double an = 0.0, ae = 0.0, seg = 0.0;
    grid_y[0] = y_lo;
    cdf_e[0] = 0.0;
    for (int i = 1; i <= NCDF - 1; ++i) {
        const double ya = y_lo + (y_hi - y_lo) * (double)(i - 1) / (double)(NCDF - 1);
        const double yb = y_lo + (y_hi - y_lo) * (double)i / (double)(NCDF - 1);
        const double ym = 0.5 * (ya + yb);
        const double fa = shape(ya), fm = shape(ym), fb = shape(yb);
        an = an + (yb - ya) / 6.0 * (fa + 4.0 * fm + fb);
        ae = ae + (yb - ya) / 6.0 * (fa * ya + 4.0 * fm * ym + fb * yb) * E_TOT;
        seg = seg + (yb - ya) / 6.0 * (fa * ya + 4.0 * fm * ym + fb * yb);
        grid_y[i] = yb;
        cdf_e[i] = seg;
    }
    n_per_decay = 2.0 * an / tot;
    e_per_decay = 2.0 * ae / tot;
    for (int i = 0; i < NCDF; ++i) cdf_e[i] = seg > 0.0 ? cdf_e[i] / seg : 1.0;
    cdf_e[NCDF - 1] = 1.0;
    return true;
}

double HeI2ph::sample(double u) const {
    const double uu = std::min(std::max(u, 0.0), 1.0);
    int lo = 0, hi = NCDF - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi + 2) / 2 - 1;   // the 1-based (lo + hi) / 2 of the reference
        if (uu > cdf_e[mid]) lo = mid; else hi = mid;
    }
    const double y = cdf_e[hi] > cdf_e[lo]
                         ? grid_y[lo] + (grid_y[hi] - grid_y[lo]) * (uu - cdf_e[lo]) / (cdf_e[hi] - cdf_e[lo])
                         : grid_y[lo];
    return y * E_TOT;
}

void hei_branch_energies(const HeI2ph& h, double T, double xHI, double xHeI, double& e3s, double& e1p, double& e1s) {
    const double Tc = std::min(std::max(T, 3.0e3), 2.0e4) / 1.0e4;   // the fits are clamped, not extrapolated
    const double a3 = 2.10e-13 * std::pow(Tc, -0.381);
    const double a1s = 2.06e-14 * std::pow(Tc, -0.451);
    const double a1p = 4.17e-14 * std::pow(Tc, -0.695);
    const double sum = a3 + a1s + a1p;
    const double f3s = a3 / sum, f1s = a1s / sum, f1p = a1p / sum;
    const double p584 = 1.0 / (1.0 + 77.0 / std::sqrt(std::max(T, TINEST)) * std::max(xHeI, 0.0) / std::max(xHI, TINEST));
    e3s = f3s * 19.82;
    e1p = f1p * p584 * 21.22;
    e1s = (f1s + f1p * (1.0 - p584)) * h.e_per_decay;
}

// ---- diffuse_mod.f90 ---------------------------------------------------------
// diffuse_build, diffuse_mod.f90:60-121, with the He I excited channel
// (par%hei_diffuse, :96-106).
void Sim::diffuse_build(double lpacket) {
    const int nleaf = grid.nleaf;
    dif_ch.assign((size_t)4 * nleaf, 0.0);
    dif_cdf.assign(nleaf, 0.0);
    for (int il = 0; il < nleaf; ++il) {
        const double nH = st.nH[il];
        if (nH <= 0.0) continue;
        const double w = 2.0 * grid.lhalf[il] * par.distance2cm;
        const double vol = w * w * w;
        const double T = st.Te[il], ne = st.ne[il];
        const double kT = KBOLTZ_CGS * T / EV2ERG;
        const double xHeIII = std::max(0.0, 1.0 - st.xHeI[il] - st.xHeII[il]);
        const double nHII = nH * (1.0 - st.xHI[il]);
        const double nHeII = nH * par.He_abund * st.xHeII[il];
        const double nHeIII = nH * par.He_abund * xHeIII;
        auto mean_e = [&](int ich, double eth) {
            if (par.diffuse_energy_model == "milne") return milne.energy_per_recomb(ich, T);
            if (par.diffuse_energy_model == "exponential") return eth + kT;
            return eth;
        };
        double a1 = alphaA_HII(rm, T) - alphaB_HII(rm, T);
        dif_ch[4 * (size_t)il + 0] = ne * nHII * a1 * mean_e(0, ETH_HI) * EV2ERG * vol;
        a1 = alphaA_HeII(rm, T) - alphaB_HeII(rm, T);
        dif_ch[4 * (size_t)il + 1] = ne * nHeII * a1 * mean_e(1, ETH_HEI) * EV2ERG * vol;
        a1 = alphaA_HeIII(rm, T) - alphaB_HeIII(rm, T);
        dif_ch[4 * (size_t)il + 2] = ne * nHeIII * a1 * mean_e(2, ETH_HEII) * EV2ERG * vol;
        if (par.hei_diffuse) {
            double e3s, e1p, e1s;
            hei_branch_energies(hei2ph, T, st.xHI[il], st.xHeI[il], e3s, e1p, e1s);
            dif_ch[4 * (size_t)il + 3] = ne * nHeII * alphaB_HeII(rm, T) * vol * EV2ERG * (e3s + e1p + e1s);
        }
    }
    diffuse_lum = 0.0;
    for (int il = 0; il < nleaf; ++il) {
        const double* c = &dif_ch[4 * (size_t)il];
        diffuse_lum = diffuse_lum + (((c[0] + c[1]) + c[2]) + c[3]);
        dif_cdf[il] = diffuse_lum;
    }
    if (diffuse_lum > 0.0) {
        for (auto& v : dif_cdf) v = v / diffuse_lum;
        diffuse_nphot = (int64_t)std::llround(diffuse_lum / lpacket);
    } else {
        diffuse_nphot = 0;
    }
}

// gen_diffuse_photon_qmc, diffuse_mod.f90:221-296.
void Sim::gen_diffuse_qmc(int64_t ip, Photon& ph) const {
    ph.from_external = false;
    ph.snx = ph.sny = ph.snz = 0.0;
    double u[9];
    for (int d = 1; d <= 9; ++d) u[d - 1] = qmc.uniform(ip, d, 2);
    const int nleaf = grid.nleaf;
    int lo = 1, hi = nleaf;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (dif_cdf[mid - 1] < u[0]) lo = mid + 1; else hi = mid;
    }
    const int il = lo - 1;
    const double half = grid.lhalf[il];
    ph.x = grid.lcx[il] + (2.0 * u[1] - 1.0) * half;
    ph.y = grid.lcy[il] + (2.0 * u[2] - 1.0) * half;
    ph.z = grid.lcz[il] + (2.0 * u[3] - 1.0) * half;
    ph.il = il;
    const double cost = 2.0 * u[4] - 1.0;
    const double sint = std::sqrt(1.0 - cost * cost);
    const double phi = TWOPI * u[5];
    ph.kx = sint * std::cos(phi);
    ph.ky = sint * std::sin(phi);
    ph.kz = cost;
    const double* w = &dif_ch[4 * (size_t)il];
    const double uu = u[6] * (((w[0] + w[1]) + w[2]) + w[3]);
    int ch;
    double eph;
    if (uu <= w[0]) { ch = 0; eph = ETH_HI; }
    else if (uu <= w[0] + w[1]) { ch = 1; eph = ETH_HEI; }
    else if (uu <= w[0] + w[1] + w[2]) { ch = 2; eph = ETH_HEII; }
    else { ch = 3; eph = ETH_HI; }
    if (ch <= 2) {
        const double T = st.Te[il];
        const double kT = KBOLTZ_CGS * T / EV2ERG;
        if (par.diffuse_energy_model == "milne") eph = milne.sample(ch, T, u[7], par.eion_max);
        else if (par.diffuse_energy_model == "exponential") eph = eph + kT * (-std::log(std::max(u[7], TINEST)));
        eph = std::min(eph, par.eion_max * 0.999);
    } else {   // the He I excited channel: 2^3S line, 584 A line or two-photon continuum
        double e3s, e1p, e1s;
        hei_branch_energies(hei2ph, st.Te[il], st.xHI[il], st.xHeI[il], e3s, e1p, e1s);
        const double ub = u[7] * ((e3s + e1p) + e1s);
        if (ub <= e3s) eph = 19.82;
        else if (ub <= e3s + e1p) eph = 21.22;
        else eph = hei2ph.sample(u[8]);
    }
    ph.inu = ion_bin_of(band, eph, false);
    ph.wgt = 1.0;
    ph.Lpacket = band.ion_Ltot / (double)par.nphotons;
    ph.E = eph;
    ph.sHI = sigma_HI(eph);
    ph.sHeI = sigma_HeI(eph);
    ph.sHeII = sigma_HeII(eph);
    metal_sigma(ph);
}

// gas_rates_compute + ion_score_apply_hhe, gas_rates_mod.f90:82-153 and
// ion_score_mod.f90:298-317.
void Sim::gas_rates_compute() {
    const int nleaf = grid.nleaf;
    for (int il = 0; il < nleaf; ++il) {
        const double w = 2.0 * grid.lhalf[il];
        const double fac = 1.0 / ((w * w * w) * (par.distance2cm * par.distance2cm));
        const double* t = &tally.hhe[(size_t)6 * il];
        gamma_HI[il] = t[0] * fac;
        gamma_HeI[il] = t[1] * fac;
        gamma_HeII[il] = t[2] * fac;
        heat_HI[il] = t[3] * fac;
        heat_HeI[il] = t[4] * fac;
        heat_HeII[il] = t[5] * fac;
        // ion_score_apply_dust_heat and ion_score_apply_g0 (ion_score_mod.f90:319-355)
        if (!tally.dust_abs.empty()) heat_dust[il] = tally.dust_abs[il] * fac * st.rhokap[il] / par.distance2cm;
        if (!tally.fuv.empty()) g0_fuv[il] = tally.fuv[il] * fac / 1.6e-3;
    }
}

// solve_ion_cell, ion_balance_mod.f90:53-150.  Without metals r_cx_in =
// r_cx_out = 0 and the closed-form substitution branch is used; with the
// two-way charge exchange x_HI comes from hydrogen_neutral_fraction.
void solve_ion_cell(const RateModel& rm, double yHe, double gH, double gHe1,
                    double gHe2, double nH, double T, bool caseA, double& xHI,
                    double& xHeI, double& xHeII, double& ne, const Species* sp, int il,
                    bool metal_ne, bool two_way) {
    const bool with_ne = sp != nullptr && metal_ne;
    const bool with_cx = sp != nullptr && two_way;
    MetalCache mc;
    if (with_ne || with_cx) sp->prepare(il, T, rm, mc);
    double aH, aHe2, aHe3;
    if (caseA) {
        aH = alphaA_HII(rm, T); aHe2 = alphaA_HeII(rm, T); aHe3 = alphaA_HeIII(rm, T);
    } else {
        aH = alphaB_HII(rm, T); aHe2 = alphaB_HeII(rm, T); aHe3 = alphaB_HeIII(rm, T);
    }
    const double cH = ci_HI(rm, T), cHe1 = ci_HeI(rm, T), cHe2 = ci_HeII(rm, T);
    double xHeIII = std::max(0.0, 1.0 - xHeI - xHeII);
    ne = nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII));
    ne = std::max(ne, 1.0e-12 * nH);
    double nem = 0.0, r_cx_in = 0.0, r_cx_out = 0.0;
    for (int it = 1; it <= 200; ++it) {
        const double ne_old = ne;
        if (with_ne || with_cx) {
            sp->metal_sums(mc, nH, ne_old, nH * xHI, nH * (1.0 - xHI), nem, r_cx_in, r_cx_out);
            if (!with_cx) {
                r_cx_in = 0.0;
                r_cx_out = 0.0;
            }
        }
        if (with_cx) {
            xHI = hydrogen_neutral_fraction(*sp, mc, nH, ne, aH * ne, gH + (cH + aH) * ne);
        } else {
            const double denH = gH + (cH + aH) * ne + r_cx_in + r_cx_out;
            xHI = (denH > 0.0) ? (aH * ne + r_cx_in) / denH : 1.0;
        }
        const double r1 = std::min((gHe1 + cHe1 * ne) / (aHe2 * ne), 1.0e150);
        const double r2 = std::min((gHe2 + cHe2 * ne) / (aHe3 * ne), 1.0e150);
        xHeI = 1.0 / (1.0 + r1 + r1 * r2);
        xHeII = xHeI * r1;
        xHeIII = xHeII * r2;
        ne = nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII));
        if (with_ne) ne = ne + nem;
        ne = std::max(0.5 * (ne + ne_old), 1.0e-12 * nH);
        if (std::fabs(ne - ne_old) <= 1.0e-10 * ne) break;
    }
}

Sim::~Sim() {
    delete th;
    delete sp;
    delete grid.oct;
}

// net_rate, thermal_mod.f90:38-115 (H/He; no metals, no grain PE, no
// secondary ionisation so sec_dgamma = 0 and sec_heat = heat).
double Sim::net_rate(int il, double T, bool caseA, double& xHI, double& xHeI, double& xHeII, double& ne) const {
    const double nH = st.nH[il];
    const bool m = metals();
    solve_ion_cell(rm, par.He_abund, gamma_HI[il], gamma_HeI[il], gamma_HeII[il], nH, T, caseA, xHI, xHeI, xHeII, ne,
                   m ? sp : nullptr, il, par.metal_ne, par.charge_exchange == "two_way");
    const double heat = nH * (xHI * heat_HI[il] + par.He_abund * (xHeI * heat_HeI[il] + xHeII * heat_HeII[il]));
    double net = heat - cooling_total(*th, rm, caseA, par.He_abund, T, nH, ne, xHI, xHeI, xHeII);
    if (par.use_metals && m) {   // thermal_mod.f90:53-71
        const MetalThermal mt = sp->thermal(il, T, nH, ne, nH * xHI, nH * (1.0 - xHI), rm, th->gff);
        net = net - mt.cool;
        net = net - mt.cool_H;
        if (par.metal_freefree) net = net - mt.freefree;
        if (par.metal_heat) net = net + mt.heat;
    }
    return net;
}

// The per-leaf bisection of gas_thermal_update (thermal_mod.f90:160-188):
// T_e and the ionisation state solved at it, from the leaf's current state.
double Sim::thermal_cell(int il, double& xHI, double& xHeI, double& xHeII, double& ne) const {
    const bool caseA = par.case_ab == "A";
    xHI = st.xHI[il]; xHeI = st.xHeI[il]; xHeII = st.xHeII[il]; ne = 0.0;
    double tlo = par.te_min, thi = par.te_max, te;
    const double net_lo = net_rate(il, tlo, caseA, xHI, xHeI, xHeII, ne);
    const double net_hi = net_rate(il, thi, caseA, xHI, xHeI, xHeII, ne);
    if (net_lo <= 0.0) {
        te = tlo;
    } else if (net_hi >= 0.0) {
        te = thi;
    } else {
        for (int it = 1; it <= 60; ++it) {
            const double tmid = std::sqrt(tlo * thi);
            const double net_mid = net_rate(il, tmid, caseA, xHI, xHeI, xHeII, ne);
            if (net_mid > 0.0) tlo = tmid; else thi = tmid;
            if (thi / tlo - 1.0 < 1.0e-5) break;
        }
        te = std::sqrt(tlo * thi);
    }
    net_rate(il, te, caseA, xHI, xHeI, xHeII, ne);
    return te;
}

// gas_thermal_update, thermal_mod.f90:124-249.
void Sim::gas_thermal_update(double m[4]) {
    const double w = par.ion_relax;
    const int nleaf = grid.nleaf;
    std::vector<double> xHI_new(nleaf), xHeI_new(nleaf), xHeII_new(nleaf), ne_new(nleaf), te_new(nleaf);
#pragma omp parallel for num_threads(std::max(1, nthreads)) schedule(dynamic, 64)
    for (int il = 0; il < nleaf; ++il) {
        const double nH = st.nH[il];
        if (nH <= 0.0) {
            xHI_new[il] = st.xHI[il]; xHeI_new[il] = st.xHeI[il]; xHeII_new[il] = st.xHeII[il];
            ne_new[il] = 0.0; te_new[il] = st.Te[il];
            continue;
        }
        double xHI, xHeI, xHeII, ne;
        const double te = thermal_cell(il, xHI, xHeI, xHeII, ne);
        xHI_new[il] = (1.0 - w) * st.xHI[il] + w * xHI;
        xHeI_new[il] = (1.0 - w) * st.xHeI[il] + w * xHeI;
        xHeII_new[il] = (1.0 - w) * st.xHeII[il] + w * xHeII;
        const double xHeIII = std::max(0.0, 1.0 - xHeI_new[il] - xHeII_new[il]);
        ne_new[il] = nH * ((1.0 - xHI_new[il]) + par.He_abund * (xHeII_new[il] + 2.0 * xHeIII));
        if (par.metal_ne && metals())   // thermal_mod.f90:198-203
            ne_new[il] = charge_neutrality_ne(*sp, rm, il, te, nH, ne_new[il], xHI_new[il], ne);
        te_new[il] = te;
    }
    double mx = 0.0, mt = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    for (int il = 0; il < nleaf; ++il) {
        if (st.nH[il] <= 0.0) continue;
        const double hw = 2.0 * grid.lhalf[il];
        const double vol = hw * hw * hw;
        mx = std::max(mx, std::fabs(xHI_new[il] - st.xHI[il]));
        mt = std::max(mt, std::fabs(te_new[il] - st.Te[il]) / st.Te[il]);
        s1 = s1 + vol * std::fabs(xHI_new[il] - st.xHI[il]);
        s2 = s2 + vol * (1.0 - xHI_new[il]);
        s3 = s3 + vol * ne_new[il] * std::fabs(te_new[il] - st.Te[il]);
        s4 = s4 + vol * ne_new[il] * te_new[il];
    }
    m[0] = mx; m[1] = mt;
    m[2] = s1 / std::max(s2, TINEST);
    m[3] = s3 / std::max(s4, TINEST);
    st.xHI = xHI_new; st.xHeI = xHeI_new; st.xHeII = xHeII_new; st.ne = ne_new; st.Te = te_new;
}

// gas_equilibrium_update, ion_balance_mod.f90:352-434.
void Sim::gas_equilibrium_update(double* max_dx, double* dx_vol) {
    const double T = par.te_fixed, yHe = par.He_abund, w = par.ion_relax;
    const bool caseA = par.case_ab == "A";
    const int nleaf = grid.nleaf;
    std::vector<double> xHI_new(nleaf), xHeI_new(nleaf), xHeII_new(nleaf), ne_new(nleaf);
#pragma omp parallel for num_threads(std::max(1, nthreads)) schedule(static)
    for (int il = 0; il < nleaf; ++il) {
        const double nH = st.nH[il];
        if (nH <= 0.0) {
            xHI_new[il] = st.xHI[il]; xHeI_new[il] = st.xHeI[il];
            xHeII_new[il] = st.xHeII[il]; ne_new[il] = 0.0;
            continue;
        }
        double xHI = st.xHI[il], xHeI = st.xHeI[il], xHeII = st.xHeII[il], ne;
        solve_ion_cell(rm, yHe, gamma_HI[il], gamma_HeI[il], gamma_HeII[il], nH, T, caseA, xHI, xHeI, xHeII, ne,
                       metals() ? sp : nullptr, il, par.metal_ne, par.charge_exchange == "two_way");
        xHI_new[il] = (1.0 - w) * st.xHI[il] + w * xHI;
        xHeI_new[il] = (1.0 - w) * st.xHeI[il] + w * xHeI;
        xHeII_new[il] = (1.0 - w) * st.xHeII[il] + w * xHeII;
        const double xHeIII = std::max(0.0, 1.0 - xHeI_new[il] - xHeII_new[il]);
        ne_new[il] = nH * ((1.0 - xHI_new[il]) + yHe * (xHeII_new[il] + 2.0 * xHeIII));
        if (par.metal_ne && metals())   // ion_balance_mod.f90:401-410
            ne_new[il] = charge_neutrality_ne(*sp, rm, il, T, nH, ne_new[il], xHI_new[il], ne);
    }
    double mdx = 0.0, sdx = 0.0, sx = 0.0;
    for (int il = 0; il < nleaf; ++il) {
        if (st.nH[il] <= 0.0) continue;
        const double hw = 2.0 * grid.lhalf[il];
        const double vol = hw * hw * hw;
        const double d = std::fabs(xHI_new[il] - st.xHI[il]);
        mdx = std::max(mdx, d);
        sdx = sdx + vol * d;
        sx = sx + vol * (1.0 - xHI_new[il]);
    }
    *max_dx = mdx;
    *dx_vol = sdx / std::max(sx, TINEST);
    st.xHI = xHI_new; st.xHeI = xHeI_new; st.xHeII = xHeII_new; st.ne = ne_new;
}

// ---- peel-off imaging: ion_peel_mod.f90 and the optical-depth-only walks
// raytrace_ion_tau_only_car / _amr (raytrace_amr.f90:678-775) -------------
namespace {
constexpr double DEG2RAD = PI / 180.0, RAD2DEG = 180.0 / PI;
constexpr double FOURPI = 4.0 * PI;
bool finite(double x) { return std::isfinite(x); }
}  // namespace

// ion_peel_setup (ion_peel_mod.f90:49-206): observers from the angle lists or
// the positions, the grid -> observer rotation, the auto pixel scale.
void Sim::peel_setup() {
    Par& p = par;
    peel_on = p.ion_peel;
    obs.clear();
    if (!peel_on) return;
    for (int i = 0; i < MAX_OBS; ++i) {
        if (finite(p.phase_angle[i])) p.alpha[i] = -p.phase_angle[i];
        if (finite(p.inclination_angle[i])) p.beta[i] = -p.inclination_angle[i];
        if (finite(p.position_angle[i])) p.gamma_[i] = -p.position_angle[i];
        if (finite(p.beta[i]) && !finite(p.alpha[i])) p.alpha[i] = 0.0;
        if (finite(p.alpha[i]) && !finite(p.beta[i])) p.beta[i] = 0.0;
    }
    const double xm = std::max({grid.xmax, grid.ymax, grid.zmax});
    if (!(finite(p.alpha[0]) && finite(p.beta[0])) && !(finite(p.obsx[0]) && finite(p.obsy[0]) && finite(p.obsz[0]))) {
        if (!finite(p.distance)) p.distance = xm * 1.0e3;
        p.obsx[0] = 0.0; p.obsy[0] = 0.0; p.obsz[0] = p.distance;
        p.alpha[0] = 0.0; p.beta[0] = 0.0;
    }
    std::vector<double> ca, sa, cb, sb, cg, sg;
    if (finite(p.alpha[0]) && finite(p.beta[0])) {
        if (!finite(p.distance)) p.distance = xm * 1.0e3;
        for (int i = 0; i < MAX_OBS; ++i) {
            if (!(finite(p.alpha[i]) && finite(p.beta[i]))) continue;
            if (!finite(p.gamma_[i])) {
                if (p.beta[i] > 0.0 && p.beta[i] <= 90.0) p.gamma_[i] = 90.0;
                else if (p.beta[i] > 90.0) p.gamma_[i] = -90.0;
                else p.gamma_[i] = 0.0;
            }
            PeelObserver o;
            ca.push_back(std::cos(p.alpha[i] * DEG2RAD)); sa.push_back(std::sin(p.alpha[i] * DEG2RAD));
            cb.push_back(std::cos(p.beta[i] * DEG2RAD)); sb.push_back(std::sin(p.beta[i] * DEG2RAD));
            cg.push_back(std::cos(p.gamma_[i] * DEG2RAD)); sg.push_back(std::sin(p.gamma_[i] * DEG2RAD));
            o.x = p.distance * ca.back() * sb.back();
            o.y = p.distance * sa.back() * sb.back();
            o.z = p.distance * cb.back();
            o.alpha = p.alpha[i]; o.beta = p.beta[i]; o.gamma = p.gamma_[i]; o.distance = p.distance;
            obs.push_back(o);
        }
    } else {
        if (!finite(p.distance)) {
            p.distance = std::sqrt(p.obsx[0] * p.obsx[0] + p.obsy[0] * p.obsy[0] + p.obsz[0] * p.obsz[0]);
            if (p.distance < 10.0 * xm) p.distance = xm * 1.0e3;
        }
        for (int i = 0; i < MAX_OBS; ++i) {
            if (!(finite(p.obsx[i]) && finite(p.obsy[i]) && finite(p.obsz[i]))) continue;
            if (!finite(p.gamma_[i])) p.gamma_[i] = 0.0;
            const double robs = std::sqrt(p.obsx[i] * p.obsx[i] + p.obsy[i] * p.obsy[i] + p.obsz[i] * p.obsz[i]);
            const double ds = p.distance / robs;
            PeelObserver o;
            if (ds > 1.001) { o.x = p.obsx[i] * ds; o.y = p.obsy[i] * ds; o.z = p.obsz[i] * ds; }
            else { o.x = p.obsx[i]; o.y = p.obsy[i]; o.z = p.obsz[i]; }
            double c_b = robs > 0.0 ? p.obsz[i] / robs : 1.0;
            c_b = std::min(std::max(c_b, -1.0), 1.0);
            const double s_b = std::sqrt(1.0 - c_b * c_b);
            p.beta[i] = std::atan2(s_b, c_b) * RAD2DEG;
            double c_a, s_a;
            if (s_b == 0.0) {
                c_a = 1.0; s_a = 0.0; p.alpha[i] = 0.0;
            } else {
                const double al = std::atan2(o.y, o.x);
                c_a = std::cos(al); s_a = std::sin(al);
                p.alpha[i] = al * RAD2DEG;
            }
            ca.push_back(c_a); sa.push_back(s_a); cb.push_back(c_b); sb.push_back(s_b);
            cg.push_back(std::cos(p.gamma_[i] * DEG2RAD)); sg.push_back(std::sin(p.gamma_[i] * DEG2RAD));
            o.alpha = p.alpha[i]; o.beta = p.beta[i]; o.gamma = p.gamma_[i]; o.distance = p.distance;
            obs.push_back(o);
        }
    }
    for (size_t i = 0; i < obs.size(); ++i) {
        PeelObserver& o = obs[i];
        o.R[0][0] = ca[i] * cb[i] * cg[i] - sa[i] * sg[i];
        o.R[0][1] = sa[i] * cb[i] * cg[i] + ca[i] * sg[i];
        o.R[0][2] = -sb[i] * cg[i];
        o.R[1][0] = -ca[i] * cb[i] * sg[i] - sa[i] * cg[i];
        o.R[1][1] = -sa[i] * cb[i] * sg[i] + ca[i] * cg[i];
        o.R[1][2] = sb[i] * sg[i];
        o.R[2][0] = ca[i] * sb[i];
        o.R[2][1] = sa[i] * sb[i];
        o.R[2][2] = cb[i];
    }
    if (!(finite(p.dxim) && finite(p.dyim))) {
        p.dxim = std::atan2(xm * std::sqrt(3.0), p.distance) / (p.nxim / 2.0) * RAD2DEG;
        p.dyim = std::atan2(xm * std::sqrt(3.0), p.distance) / (p.nyim / 2.0) * RAD2DEG;
    }
    dxim = p.dxim;
    dyim = p.dyim;
    nchan = p.peel_bins ? band.nnu_band : (p.add_fuv ? 2 : 1);
}

int Sim::peel_channel(int inu) const {   // ion_peel_mod.f90:212-220 (0-based)
    if (par.peel_bins) return inu;
    if (nchan == 2 && std::sqrt(band.eedge[inu] * band.eedge[inu + 1]) < par.eion_min) return 1;
    return 0;
}

bool Sim::peel_pixel(const PeelObserver& o, double kx, double ky, double kz, int* ix, int* iy) const {
    double v[3];
    for (int i = 0; i < 3; ++i) v[i] = o.R[i][0] * kx + o.R[i][1] * ky + o.R[i][2] * kz;
    *ix = (int)std::floor(std::atan2(-v[0], v[2]) * RAD2DEG / dxim + par.nxim / 2.0);
    *iy = (int)std::floor(std::atan2(-v[1], v[2]) * RAD2DEG / dyim + par.nyim / 2.0);
    return *ix >= 0 && *ix < par.nxim && *iy >= 0 && *iy < par.nyim;
}

// Optical depth from the packet's point along (kx, ky, kz) to the box edge at
// the packet's energy, no tally; stops at tau_huge.
double Sim::tau_only(const Photon& ph, double kx, double ky, double kz) const {
    double tau = 0.0;
    if (amr_walk()) {
        double x = ph.x, y = ph.y, z = ph.z;
        int il = ph.il >= 0 ? ph.il : leaf_find(x, y, z);
        if (il < 0) return 0.0;
        for (int nstep = 1; nstep <= MAX_WALK_STEPS; ++nstep) {
            double texit;
            int iface;
            leaf_exit(il, x, y, z, kx, ky, kz, &texit, &iface);
            tau = tau + opacity(*this, ph, il) * texit;
            if (tau >= TAU_HUGE) break;
            x = x + texit * kx; y = y + texit * ky; z = z + texit * kz;
            const int nl = leaf_next(il, iface, x, y, z);
            if (nl < 0) break;
            il = nl;
        }
        return tau;
    }
    const double d = grid.dcell;
    const double pos[3] = {ph.x, ph.y, ph.z}, kk[3] = {kx, ky, kz};
    const double org[3] = {grid.xmin, grid.ymin, grid.zmin};
    const int n[3] = {grid.nx, grid.ny, grid.nz};
    int idx[3], stp[3];
    double tmax[3], tdel[3];
    for (int a = 0; a < 3; ++a) {
        idx[a] = std::min(std::max((int)((pos[a] - org[a]) / d), 0), n[a] - 1);
        if (kk[a] > 0.0) {
            stp[a] = 1; tmax[a] = (org[a] + (double)(idx[a] + 1) * d - pos[a]) / kk[a]; tdel[a] = d / kk[a];
        } else if (kk[a] < 0.0) {
            stp[a] = -1; tmax[a] = (org[a] + (double)idx[a] * d - pos[a]) / kk[a]; tdel[a] = -d / kk[a];
        } else {
            stp[a] = 0; tmax[a] = HUGEST; tdel[a] = HUGEST;
        }
    }
    double t_cur = 0.0;
    for (int nstep = 1; nstep <= MAX_WALK_STEPS; ++nstep) {
        const int il = idx[0] + n[0] * (idx[1] + n[1] * idx[2]);
        int a = 0;
        if (tmax[1] < tmax[a]) a = 1;
        if (tmax[2] < tmax[a]) a = 2;
        tau = tau + opacity(*this, ph, il) * (tmax[a] - t_cur);
        if (tau >= TAU_HUGE) break;
        t_cur = tmax[a];
        tmax[a] = tmax[a] + tdel[a];
        idx[a] += stp[a];
        if (idx[a] < 0 || idx[a] >= n[a]) break;
    }
    return tau;
}

// ion_peel_direct (ion_peel_mod.f90:225-277): the isotropic source's
// Lpacket wgt / (4 pi r^2) e^-tau to its pixel of every observer.
void Sim::peel_direct(const Photon& ph, Tally& t) const {
    const int ch = peel_channel(ph.inu);
    const int nx = par.nxim, ny = par.nyim;
    for (size_t k = 0; k < obs.size(); ++k) {
        const PeelObserver& o = obs[k];
        double kx = o.x - ph.x, ky = o.y - ph.y, kz = o.z - ph.z;
        const double r2 = kx * kx + ky * ky + kz * kz, r = std::sqrt(r2);
        kx = kx / r; ky = ky / r; kz = kz / r;
        int ix, iy;
        if (!peel_pixel(o, kx, ky, kz, &ix, &iy)) continue;
        const size_t pix = ((k * nchan + ch) * (size_t)ny + iy) * nx + ix;
        double contrib;
        if (ph.from_external) {   // ion_peel_mod.f90:254-263
            const double cos_obs = kx * ph.snx + ky * ph.sny + kz * ph.snz;
            if (cos_obs <= 0.0) continue;
            contrib = ph.Lpacket * ph.wgt * cos_obs / (PI * r2);
        } else {
            contrib = ph.Lpacket * ph.wgt / (FOURPI * r2);
        }
        if (par.save_direc0) t.img_dir0[pix] += contrib;
        const double tau = tau_only(ph, kx, ky, kz);
        if (tau > 500.0) continue;
        t.img_dir[pix] += contrib * std::exp(-tau);
    }
}

// ion_peel_scatter (ion_peel_mod.f90:284-344): at a dust interaction, after
// the albedo weight and before the new direction, the Henyey-Greenstein
// phase function toward each observer.
void Sim::peel_scatter(const Photon& ph, Tally& t) const {
    const int ch = peel_channel(ph.inu);
    const int nx = par.nxim, ny = par.nyim;
    const double gg = std::min(std::max(ph.dust_g, -0.9999), 0.9999);
    for (size_t k = 0; k < obs.size(); ++k) {
        const PeelObserver& o = obs[k];
        double kx = o.x - ph.x, ky = o.y - ph.y, kz = o.z - ph.z;
        const double r2 = kx * kx + ky * ky + kz * kz, r = std::sqrt(r2);
        kx = kx / r; ky = ky / r; kz = kz / r;
        int ix, iy;
        if (!peel_pixel(o, kx, ky, kz, &ix, &iy)) continue;
        const double tau = tau_only(ph, kx, ky, kz);
        if (tau > 500.0) continue;
        const double kn2 = ph.kx * ph.kx + ph.ky * ph.ky + ph.kz * ph.kz;
        if (kn2 <= 0.0) continue;
        double cosa = (ph.kx * kx + ph.ky * ky + ph.kz * kz) / std::sqrt(kn2);
        cosa = std::min(std::max(cosa, -1.0), 1.0);
        const double dmin = (1.0 - std::fabs(gg)) * (1.0 - std::fabs(gg));
        const double den = std::max((1.0 + gg * gg) - 2.0 * gg * cosa, dmin);
        const double peel = (1.0 - gg * gg) / (den * std::sqrt(den) * FOURPI);
        const double contrib = ph.Lpacket * ph.wgt * peel / r2 * std::exp(-tau);
        if (!std::isfinite(contrib)) continue;
        t.img_sca[((k * nchan + ch) * (size_t)ny + iy) * nx + ix] += contrib;
    }
}


}  // namespace orc
