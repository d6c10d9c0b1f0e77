// Host-side set-up of the ionising band: diagnostic bin edges and the
// continuous source-energy samplers (ion_band_mod.f90:122-495 and
// energy_sampler_mod.f90).  Set-up time only; the tables are uploaded to
// device memory and inverted there per packet.
#pragma once
#include <string>
#include <vector>

#include "mochii_gpu.h"

namespace mochii {

// Piecewise-linear spectral density with its analytic CDF
// (energy_sampler_type, energy_sampler_mod.f90:20-25).
struct EnergyTable {
    std::vector<double> energy, density, cdf;
    double total = 0.0;
};

bool table_from_points(EnergyTable& t, const std::vector<double>& e, const std::vector<double>& f,
                       std::string* err);
bool planck_table(EnergyTable& t, double T, double emin, double emax, double rtol,
                  const std::vector<double>& knots, std::string* err);
double table_sample(const EnergyTable& t, double u);   // sample_energy_cdf
double table_cdf(const EnergyTable& t, double e);      // energy_cdf_value

struct BandSetup {
    int nnu_band = 0, nfuv_band = 0;
    std::vector<double> eedge;          // nnu_band + 1 ascending edges [eV]
    int ncomp = 1, multi = 0, qmc_ndim = 3;
    std::vector<double> comp_cdf;       // component-selection CDF (multi only)
    std::vector<double> comp_x, comp_y, comp_z;
    std::vector<EnergyTable> tables;    // one per component
    double ion_Ltot = 0.0;
    int ext_ic = -1;                    // component of the external field, -1 none
    int ext_sph = 0;                    // its entry surface: 0 the box faces, 1 the sphere of radius rmax
    // plane-parallel slab (slab_setup, ion_band_mod.f90:2083-2130): the one
    // component; per face [0] top (+z), [1] bottom (-z): lit, mode (0 beam,
    // 1 Lambert), beam mu = cos(theta) and azimuth [rad], horizontal flux F_z
    int slab = 0;
    int slab_lit[2] = {0, 0}, slab_mode[2] = {0, 0};
    double slab_mu[2] = {1.0, 1.0}, slab_phi[2] = {0.0, 0.0}, slab_Fz[2] = {0.0, 0.0};
    double slab_ptop = 1.0;             // probability of the top face
    double slab_azface = 0.0;           // z-face area of one periodic tile [cm^2]
};

// Tabulated spectra (spectrum.cpp).  spectrum_preset_id: 'draine' 1,
// 'habing' 2, 'mathis' 3, else 0 (ion_ext_preset_id).  spectrum_read: the
// icol-th of ncol value columns of a spectrum file as ascending (E [eV],
// density per eV), converted from spectrum_type (0 shape_ev, 1 per_ev,
// 2 per_hz, 3 per_ang, 4 per_um).  table_band: the tabulated sampler
// clipped to [emin, emax].  preset_table: a preset's J_E x scale on 4096
// uniform nodes from elo to min(emax, 13.6 eV).
int spectrum_preset_id(const char* name);
double preset_je(double E, int id);
bool spectrum_read(const std::string& path, int icol, int ncol, int type, std::vector<double>& e,
                   std::vector<double>& f, std::string* err);
bool table_band(EnergyTable& t, const std::vector<double>& e, const std::vector<double>& f, double emin, double emax,
                std::string* err);
bool preset_table(EnergyTable& t, int id, double elo, double emax, double scale, std::string* err);

// metal_eth: the active metal thresholds in registry order (main.f90:65-82),
// which pin band edges and sampler knots as the H/He thresholds do.
// box: the grid's x, y, z extents in code units (the external field's entry
// surface), null when unknown.
bool band_build(const mochii_params& p, BandSetup& b, std::string* err, const std::vector<double>& metal_eth = {},
                const double* box = nullptr);

}  // namespace mochii
