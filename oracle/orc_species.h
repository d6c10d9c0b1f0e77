// Oracle (test infrastructure only): the trace-metal registry of
// species_mod.f90 -- element data, packet cross sections, cached stage
// fractions, path scoring, the metal electron / charge-exchange sums, the
// charge-exchange hydrogen balance of ion_balance_mod.f90, and the metal
// cooling and heating terms of the thermal balance.
#pragma once
#include <string>
#include <vector>

#include "orc_core.h"
#include "orc_thermal.h"

namespace orc {

constexpr int MAX_EL = 11, MAX_ST = 6, MAX_TR = 64;   // species_mod.f90:53, define.f90:80

struct Element {                                     // species_mod.f90:55-91
    std::string name;
    int Z = 0, nstage = 0;
    double abund = 0.0;
    double eth[MAX_ST] = {};
    int photo_form[MAX_ST] = {1, 1, 1, 1, 1, 1};
    double photo[MAX_ST][8] = {};
    double ci[MAX_ST][5] = {};
    double rr[MAX_ST][6] = {};
    int ndr[MAX_ST] = {};
    double dr_c[MAX_ST][9] = {}, dr_e[MAX_ST][9] = {};
    bool has_dr2[MAX_ST] = {}, has_rr2[MAX_ST] = {};
    double dr2[MAX_ST][4] = {}, rr2[MAX_ST][2] = {};
    int cxi_form[MAX_ST] = {}, cxr_form[MAX_ST] = {};
    double cxi[MAX_ST][6] = {}, cxr[MAX_ST][6] = {};
    bool has_cool[MAX_ST] = {};
    CoolingFit cool[MAX_ST];
    bool has_table[MAX_ST] = {};
    NlevelTable table[MAX_ST];
};

// Per-(leaf, T) rate cache of species_ne_prepare (species_mod.f90:120-127, 517-536).
struct MetalCache {
    double gam[MAX_ST][MAX_EL], ci[MAX_ST][MAX_EL], rec[MAX_ST][MAX_EL], cxi[MAX_ST][MAX_EL], cxr[MAX_ST][MAX_EL];
};

// The four metal terms of net_rate (thermal_mod.f90:53-71).
struct MetalThermal {
    double cool = 0.0, cool_H = 0.0, freefree = 0.0, heat = 0.0;
};

struct Species {
    std::vector<Element> el;
    int ntr = 0;                                     // flat transitions sorted by threshold
    int flat_ie[MAX_TR] = {}, flat_it[MAX_TR] = {};  // 0-based element, 1-based stage
    double flat_eth[MAX_TR] = {};
    int flat_of[MAX_EL][MAX_ST] = {};                // (ie, it-1) -> flat index
    int nleaf = 0;
    std::vector<std::vector<double>> egam, eheat;    // [ie][(it-1)*nleaf + il]
    std::vector<std::vector<double>> stage_frac;     // [ie][(i-1)*nleaf + il]

    bool setup(const Par& p, int nleaf, std::string* err);                      // :143-226
    std::vector<double> thresholds() const;                                     // main.f90:65-82
    double sigma(int ie, int it, double E) const;                               // :763-778
    int packet_sigma(double E, double* sig) const;                              // :263-275
    double cached_opacity(const double* sig, int n, int il) const;              // :291-303
    // species_rate_path_score (:329-343); raw is [(il*ntr + k)*2 + m]
    void score(double E, const double* sig, int n, int il, double path_lum, double* raw) const;
    void gamma_compute(const std::vector<double>& raw, const std::vector<double>& fac);   // :493-512
    double alpha_rec(const Element& e, int it, double T) const;                 // :428-447
    void prepare(int il, double T, const RateModel& rm, MetalCache& c) const;   // :517-536
    void metal_sums(const MetalCache& c, double nH, double ne, double nHI, double nHII, double& nem,
                    double& rin, double& rout) const;                           // :566-614
    void fractions(int ie, int il, double T, double ne, double nHI, double nHII, const RateModel& rm,
                   double* frac) const;                                         // :782-813
    void stage_cache_refresh(const State& st, const RateModel& rm);             // :247-261
    // metal_cooling + metal_cooling_H + metal_freefree + metal_heating
    // (:825-846, 704-731, 852-871, 739-752) at one (leaf, T, n_e, x_HI)
    MetalThermal thermal(int il, double T, double nH, double ne, double nHI, double nHII, const RateModel& rm,
                         const GffTable& gff) const;
};

double cx_rate(int form, const double* c, double T);                // species_mod.f90:452-487
double voronov_ci(const double* c, double T);                       // :815-820

// hydrogen_neutral_fraction (ion_balance_mod.f90:177-208).
double hydrogen_neutral_fraction(const Species& sp, const MetalCache& c, double nH, double ne, double A, double B);
// charge_neutrality_ne (ion_balance_mod.f90:235-253).
double charge_neutrality_ne(const Species& sp, const RateModel& rm, int il, double T, double nH, double ne_HHe,
                            double xHI, double ne_seed);

}  // namespace orc
