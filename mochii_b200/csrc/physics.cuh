// Per-packet and per-cell microphysics shared by host setup and device
// kernels: physical constants, photoionisation cross sections, radiative
// recombination and collisional-ionisation rate coefficients.
//
// Constants follow define.f90:29-67; the fits follow photo_xsec.f90 and
// recomb_mod.f90 (line numbers at each function).  All FP64.
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define MHD __host__ __device__ __forceinline__
#else
#define MHD inline
#endif

namespace mochii {

constexpr double kPi = 3.141592653589793238462643383279502884197;
constexpr double kTwoPi = 6.283185307179586476925286766559005768394;
constexpr double kPc2cm = 3.0856776e18;
constexpr double kKpc2cm = kPc2cm * 1e3;
constexpr double kAu2cm = 1.4960e13;
constexpr double kHPlanck = 6.62607015e-27;  // erg s
constexpr double kEv2erg = 1.602176634e-12;
constexpr double kKboltz = 1.380649e-16;     // erg/K
constexpr double kEthHI = 13.598;            // eV
constexpr double kEthHeI = 24.587;
constexpr double kEthHeII = 54.416;
constexpr double kKbEv = 8.617333262145e-5;  // energy_sampler_mod.f90:17
constexpr double kTauHuge = 745.2;           // raytrace_amr.f90:33
constexpr int kMaxWalkSteps = 20000000;      // raytrace_amr.f90:43
constexpr double kHugest = 1.7976931348623157e308;
constexpr double kTinest = 2.2250738585072014e-308;

// Exact ground-state hydrogenic cross section (Osterbrock & Ferland 2006
// eq. 2.4), photo_xsec.f90:92-107: sigma_0 (E_th/E)^4 exp(4 - 4 atan(eps)/eps)
// / (1 - exp(-2 pi/eps)), eps = sqrt(E/E_th - 1), sigma_0 = 6.3e-18/Z^2 cm^2.
MHD double sigma_hydrogenic(double E, double Eth, double Z) {
    const double s0 = 6.30e-18 / (Z * Z);
    if (E < Eth) return 0.0;
    if (E == Eth) return s0;
    const double eps = sqrt(E / Eth - 1.0);
    const double r = Eth / E;
    const double r2 = r * r;
    return s0 * (r2 * r2) * exp(4.0 - 4.0 * atan(eps) / eps) / (1.0 - exp(-2.0 * kPi / eps));
}

// Verner, Ferland, Korista & Yakovlev (1996) eq. 1, photo_xsec.f90:46-59
// (sigma_0 in Mb, result in cm^2).
MHD double sigma_vfky96(double E, double Eth, double E0, double s0, double ya,
                        double P, double yw, double y0, double y1) {
    if (E < Eth) return 0.0;
    const double x = E / E0 - y0;
    const double z = sqrt(x * x + y1 * y1);
    const double Q = 5.5 - 0.5 * P;
    const double xm1 = x - 1.0;
    return s0 * ((xm1 * xm1 + yw * yw) * pow(z, -Q) * pow(1.0 + sqrt(z / ya), -P)) * 1.0e-18;
}

MHD double sigma_HI(double E) { return sigma_hydrogenic(E, kEthHI, 1.0); }      // photo_xsec.f90:110
MHD double sigma_HeI(double E) {                                                // photo_xsec.f90:116
    return sigma_vfky96(E, kEthHeI, 1.361e1, 9.492e2, 1.469, 3.188, 2.039, 4.434e-1, 2.136);
}
MHD double sigma_HeII(double E) { return sigma_hydrogenic(E, kEthHeII, 2.0); }  // photo_xsec.f90:123

// Rate-model selection (par%recomb_model, par%ci_model).
struct RateSel {
    int hui_gnedin;    // 0 = badnell_milne (default), 1 = hui_gnedin
    int dere_hybrid;   // 0 = voronov (default), 1 = dere_hybrid
};

// Badnell (2023) radiative recombination fit, recomb_mod.f90:124-130.
MHD double rr_badnell(double T, double A, double B, double T0, double T1, double Cc, double T2) {
    const double bp = B + Cc * exp(-T2 / T);
    const double tt = sqrt(T / T0);
    return A / (tt * pow(1.0 + tt, 1.0 - bp) * pow(1.0 + sqrt(T / T1), 1.0 + bp));
}
// He II -> He I dielectronic sum, recomb_mod.f90:132-137.
MHD double dr_HeII_badnell(double T) {
    return pow(T, -1.5) * (1.417e-3 * exp(-4.633e5 / T) + 2.235e-4 * exp(-5.532e5 / T) -
                           2.185e-5 * exp(-8.887e5 / T));
}
// Mao & Kaastra (2016) fit form for the Milne ground-level rate,
// recomb_mod.f90:145-151.
MHD double rr_mao(double T, double a0, double b0, double c0, double a1, double b1, double a2, double b2) {
    const double te = T * (kKboltz / kEv2erg);
    return a0 * 1.0e-10 * pow(te, -b0 - c0 * log(te)) * (1.0 + a2 * pow(te, -b2)) / (1.0 + a1 * pow(te, -b1));
}
MHD double alpha1_HII(double T) {   // recomb_mod.f90:188-192
    return rr_mao(T, 1.87007e-2, 1.29077, -2.17465e-3, 1.29189e1, 8.05060e-1, 8.44399e-2, 5.93940e-4);
}
MHD double alpha1_HeIII(double T) { // recomb_mod.f90:194-198
    return rr_mao(T, 2.61525e-1, 1.39527, -3.22079e-4, 6.40708e1, 8.97582e-1, 5.01551e-1, 1.21533e-3);
}
MHD double alpha1_HeII(double T) {  // recomb_mod.f90:200-204
    return rr_mao(T, 3.26862e-3, 6.97361e-1, 3.14907e-4, 5.76341e1, 1.18534, 2.58417e1, 9.90134e-1);
}
// Hui & Gnedin (1997) fits, recomb_mod.f90:209-251 (lambda = 2 T_TR / T).
MHD double hg_fit(double T, double Ttr, double pref, double p1, double l0, double p2, double p3) {
    const double lam = 2.0 * Ttr / T;
    return pref * pow(lam, p1) / pow(1.0 + pow(lam / l0, p2), p3);
}

MHD double alphaA_HII(const RateSel& s, double T) {   // recomb_mod.f90:47-57
    return s.hui_gnedin ? hg_fit(T, 157807.0, 1.269e-13, 1.503, 0.522, 0.470, 1.923)
                        : rr_badnell(T, 8.318e-11, 0.7472, 2.965, 7.001e5, 0.0, 0.0);
}
MHD double alphaB_HII(const RateSel& s, double T) {   // :59-69
    return s.hui_gnedin ? hg_fit(T, 157807.0, 2.753e-14, 1.500, 2.740, 0.407, 2.242)
                        : alphaA_HII(s, T) - alpha1_HII(T);
}
MHD double alphaA_HeII(const RateSel& s, double T) {  // :71-82
    return s.hui_gnedin ? 3.000e-14 * pow(2.0 * 285335.0 / T, 0.654)
                        : rr_badnell(T, 5.235e-11, 0.6988, 7.301, 4.475e6, 0.0829, 1.682e5) + dr_HeII_badnell(T);
}
MHD double alphaB_HeII(const RateSel& s, double T) {  // :84-94
    return s.hui_gnedin ? 1.260e-14 * pow(2.0 * 285335.0 / T, 0.750) : alphaA_HeII(s, T) - alpha1_HeII(T);
}
MHD double alphaA_HeIII(const RateSel& s, double T) { // :96-106
    return s.hui_gnedin ? 2.0 * hg_fit(T, 631515.0, 1.269e-13, 1.503, 0.522, 0.470, 1.923)
                        : rr_badnell(T, 1.818e-10, 0.7492, 1.017e1, 2.786e6, 0.0, 0.0);
}
MHD double alphaB_HeIII(const RateSel& s, double T) { // :108-118
    return s.hui_gnedin ? 2.0 * hg_fit(T, 631515.0, 2.753e-14, 1.500, 2.740, 0.407, 2.242)
                        : alphaA_HeIII(s, T) - alpha1_HeIII(T);
}

// Voronov (1997) collisional ionisation, recomb_mod.f90:256-279, with the
// Dere/Voronov hybrid ratios for H and He (recomb_mod.f90:296-297).
MHD double voronov(double T, double dE, double P, double A, double X, double K) {
    const double U = dE * kEv2erg / (kKboltz * T);
    return A * (1.0 + P * sqrt(U)) * pow(U, K) * exp(-U) / (X + U);
}
MHD double ci_HI(const RateSel& s, double T) {
    return voronov(T, 13.6, 0.0, 2.91e-8, 0.232, 0.39) * (s.dere_hybrid ? 0.9063 : 1.0);
}
MHD double ci_HeI(const RateSel& s, double T) {
    return voronov(T, 24.6, 0.0, 1.75e-8, 0.180, 0.35) * (s.dere_hybrid ? 1.0389 : 1.0);
}
MHD double ci_HeII(const RateSel& s, double T) {
    return voronov(T, 54.4, 1.0, 2.05e-9, 0.265, 0.25) * (s.dere_hybrid ? 1.0686 : 1.0);
}

}  // namespace mochii
