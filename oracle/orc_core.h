// Oracle for the MoCHII photon-packet transport + ionisation/thermal balance
// path.  TEST INFRASTRUCTURE ONLY: a plain FP64 CPU restatement of the
// reference Fortran, used by tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py as the checker.  Nothing in the product
// (mochii_b200/) includes, links or calls this code.
//
// Every routine names the reference file:line it restates (paths relative
// to the seoncafe/MoCHII source tree).  Built with -O2 -fno-fast-math
// -ffp-contract=off so that the FP64 rounding sequence follows the
// source expressions term by term.
#pragma once
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>
#include <map>

#include "orc_dust.h"

namespace orc {

// ---- constants: define.f90:29-67, energy_sampler_mod.f90:16-18 ----------
constexpr double PI = 3.141592653589793238462643383279502884197;
// a bound on scattering events per packet (not in the reference, whose loop
// ends by the roulette alone); a packet that reaches it stops scattering
constexpr int MAX_SCATTERINGS = 100000;
constexpr double TWOPI = 6.283185307179586476925286766559005768394;
constexpr double PC2CM = 3.0856776e18;
constexpr double KPC2CM = PC2CM * 1e3;
constexpr double AU2CM = 1.4960e13;
constexpr double H_PLANCK_CGS = 6.62607015e-27;
constexpr double CLIGHT_CGS = 2.99792458e10;
constexpr double EV2ERG = 1.602176634e-12;
constexpr double KBOLTZ_CGS = 1.380649e-16;
constexpr double ETH_HI = 13.598;
constexpr double ETH_HEI = 24.587;
constexpr double ETH_HEII = 54.416;
constexpr double KB_EV = 8.617333262145e-5;
constexpr double TAU_HUGE = 745.2;             // raytrace_amr.f90:33
constexpr int MAX_WALK_STEPS = 20000000;       // raytrace_amr.f90:43
constexpr int MAX_PLANCK_KNOTS = 200000;       // energy_sampler_mod.f90:16
constexpr int MAX_SRC = 16;                    // define.f90:74
constexpr int MAX_OBS = 16;                    // peel-off observers (define.f90:76 allows 181)
constexpr double HUGEST = 1.7976931348623157e308;
constexpr double TINEST = 2.2250738585072014e-308;

// ---- qmc_mod.f90 ---------------------------------------------------------
struct Qmc {
    uint32_t V[12][32];     // Vdir(k,d), qmc_mod.f90:60
    uint32_t key[2][12];    // dkey(d,stream), qmc_mod.f90:61
    void setup(int seed);   // qmc_mod.f90:73-139
    uint32_t sobol_code(int64_t idx, int d) const;            // :192-206
    uint32_t scrambled(int64_t idx, int d, int stream) const;  // :164-166
    double uniform(int64_t idx, int d, int stream) const;      // :157-168
};
uint32_t hash32(uint32_t x);                     // qmc_mod.f90:250-260
uint32_t reverse32(uint32_t x);                  // :233-247
uint32_t laine_karras(uint32_t x, uint32_t s);   // :221-230
uint32_t owen_scramble(uint32_t x, uint32_t s);  // :212-219

// ---- energy_sampler_mod.f90 ---------------------------------------------
struct Sampler {
    std::vector<double> energy, density, cdf;
    double total_integral = 0.0;
};
bool build_tabulated_sampler(Sampler& s, const std::vector<double>& e,
                             const std::vector<double>& f, std::string* err);
bool build_tabulated_band_sampler(Sampler& s, const std::vector<double>& e,
                                  const std::vector<double>& f, double emin,
                                  double emax, std::string* err);
bool build_planck_sampler(Sampler& s, double T, double emin, double emax,
                          double rtol, const std::vector<double>& thr,
                          std::string* err);
double sample_energy_cdf(const Sampler& s, double u);
double energy_cdf_value(const Sampler& s, double e);
double planck_energy_shape(double e, double T);

// ---- photo_xsec.f90 -------------------------------------------------------
double sigma_hydrogenic(double E, double Eth, double Z);
double sigma_vfky96(double E, double Eth, double E0, double s0, double ya,
                    double P, double yw, double y0, double y1);
double sigma_vy95(double E, double Eth, double E0, double s0, double ya,
                  double P, double yw, double l);
double sigma_HI(double E);
double sigma_HeI(double E);
double sigma_HeII(double E);

// ---- recomb_mod.f90 -------------------------------------------------------
enum { RECOMB_BADNELL_MILNE = 0, RECOMB_HUI_GNEDIN = 1 };
enum { CI_VORONOV = 0, CI_DERE_HYBRID = 1 };
struct RateModel { int recomb = RECOMB_BADNELL_MILNE; int ci = CI_VORONOV; };
double alphaA_HII(const RateModel&, double T);
double alphaB_HII(const RateModel&, double T);
double alphaA_HeII(const RateModel&, double T);
double alphaB_HeII(const RateModel&, double T);
double alphaA_HeIII(const RateModel&, double T);
double alphaB_HeIII(const RateModel&, double T);
double alpha1_HII(double T);
double alpha1_HeII(double T);
double alpha1_HeIII(double T);
double ci_HI(const RateModel&, double T);
double ci_HeI(const RateModel&, double T);
double ci_HeII(const RateModel&, double T);
double ci_dere_ratio(const RateModel&, int Z, int stage);
double voronov(double T, double dE, double P, double A, double X, double K);

// ---- namelist + parameters (define.f90:189-861, setup.f90:11-626) -------
struct Par {
    // launch
    int64_t nphotons = 100000;
    std::string launch_sequence = "random";
    int qmc_seed = 12345;
    double source_cdf_tol = 1.0e-8;
    double luminosity = -999.0;
    double tstar = -999.0;
    // band
    int nnu_ion = 16;
    double eion_min = 13.598, eion_max = 100.0;
    bool add_fuv = false;
    double efuv_min = 6.0;
    int nnu_fuv = 8;
    bool ion_align_edges = true;
    // geometry
    std::string grid_type = "car";
    std::string car_walk = "dda";
    std::string amr_file;
    int nx = 1, ny = 1, nz = 11;
    double xmax = 1.0, ymax = 1.0, zmax = 1.0;
    double rmax = -999.0, rmin = 0.0, nH_const = -1.0;
    std::string distance_unit = "kpc";
    double distance2cm = KPC2CM;
    std::string source_geometry = "point";
    double ext_intensity = -1.0, ext_tstar = -999.0;   // define.f90:270-277
    std::string ext_geometry = "rec";
    // plane-parallel slab illumination on an xy-periodic grid (define.f90:217, 304-321)
    bool xy_periodic = false;
    std::string slab_faces = "top", slab_top_mode = "beam", slab_bot_mode = "beam";
    double slab_top_theta = 0.0, slab_bot_theta = 0.0, slab_top_phi = 0.0, slab_bot_phi = 0.0;
    double slab_top_source = 0.0, slab_bot_source = 0.0;
    int slab_nmu = 20;
    // tabulated spectra and ISRF presets (define.f90:276-303)
    std::string ion_spectrum, src_spectrum_file, ext_spectrum, spectrum_type = "shape_ev";
    double ext_scale = 1.0;
    double xs_point = 0.0, ys_point = 0.0, zs_point = 0.0;
    int nsource = 1;
    double src_tstar[MAX_SRC], src_lum[MAX_SRC];
    double src_x[MAX_SRC], src_y[MAX_SRC], src_z[MAX_SRC];
    // gas
    double xHI_init = 1.0, xHeI_init = 1.0, xHeII_init = 0.0;
    double He_abund = 0.1;
    int gas_niter = 0;
    double gas_tol = 1.0e-3, te_fixed = 1.0e4, ion_relax = 1.0;
    std::string case_ab = "B";
    std::string ci_model = "voronov";
    std::string recomb_model = "badnell_milne";
    std::string cooling_model = "local_ne";
    std::string charge_exchange = "two_way";
    std::string conv_crit = "cell";
    bool solve_te = false;
    double te_min = 1.0e3, te_max = 5.0e4, gas_tol_te = 1.0e-3;
    bool use_metals = false, diffuse_field = false, use_sec_ion = false, hei_diffuse = false;
    std::string diffuse_energy_model = "milne";
    bool ion_add_dust = false, ion_dust_scatter = false;
    std::string dust_density_law = "global_dgr";
    double DGR = 1.0e-2, cext_dust = 1.6059e-21;
    double lambda_ref = 0.55, taumax = -999.0, tauhomo = -999.0;   // define.f90:211-212,361
    int64_t iseed = 0;                                             // define.f90:194
    std::string data_dir, atomic_dir, ion_dust_kext;
    // metals (define.f90:578-580, 593, 622-623, 652, 843-857)
    double abund_C = 2.2e-4, abund_N = 4.0e-5, abund_O = 3.3e-4, abund_Ne = 5.0e-5, abund_S = 9.0e-6;
    double abund_Ar = 0.0, abund_Mg = 0.0, abund_Fe = 0.0, abund_Si = 0.0, abund_Cl = 0.0, abund_Ca = 0.0;
    bool ion_metal_abs = true, metal_ne = true, metal_heat = true, metal_freefree = true;
    // peel-off imaging (define.f90:518-544, 658-664); NaN = unset
    bool ion_peel = false, peel_bins = false, save_direc0 = false;
    int nxim = 129, nyim = 129;
    double distance = NAN, dxim = NAN, dyim = NAN;
    double alpha[MAX_OBS], beta[MAX_OBS], gamma_[MAX_OBS], obsx[MAX_OBS], obsy[MAX_OBS], obsz[MAX_OBS];
    double phase_angle[MAX_OBS], inclination_angle[MAX_OBS], position_angle[MAX_OBS];
    bool fe_levels_full = false;
    Par();
};
// Parse a Fortran "&parameters par%key = value /" namelist text.
bool parse_namelist(const std::string& text, Par& p, std::string* err);

// ---- band (ion_band_mod.f90) ----------------------------------------------
struct Band {
    int nnu_band = 0, nfuv_band = 0;
    std::vector<double> eedge;       // ion_eedge, size nnu_band+1
    int ncomp = 1;
    bool multi_src = false;
    std::vector<int> comp_kind;      // multi only
    std::vector<double> src_cdf;     // multi only
    std::vector<double> src_x, src_y, src_z;   // point positions after setup.f90:398-407
    int ext_ic = -1;                 // the external field's component, -1 none
    std::vector<Sampler> samplers;   // source_energy_sampler
    double ion_Ltot = 0.0;
    int qmc_ndim = 3;
    // slab_setup (ion_band_mod.f90:2083-2130), per face [top, bottom]
    bool slab = false;
    bool slab_lit[2] = {false, false};
    int slab_mode[2] = {0, 0};
    double slab_mu[2] = {1.0, 1.0}, slab_phi[2] = {0.0, 0.0}, slab_Fz[2] = {0.0, 0.0};
    double slab_ptop = 1.0, slab_azface = 0.0;
};
bool build_aligned_edges(std::vector<double>& eedge, int nfuv, int nnu,
                         double lo, double hi, const std::vector<double>& meth,
                         std::string* err);
int ion_bin_of(const Band& b, double e, bool include_fuv);
bool band_setup(const Par& p, Band& b, std::string* err, const std::vector<double>& meth = {},
                const double* box = nullptr);

// ---- car grid + state ----------------------------------------------------
struct Octree;
struct Grid {
    bool car = true;
    int nx = 0, ny = 0, nz = 0, nleaf = 0;
    double xmin, xmax, ymin, ymax, zmin, zmax, dcell;
    std::vector<double> lhalf, lcx, lcy, lcz;   // per-leaf half width and centre (leaf_half, leaf_cx..)
    Octree* oct = nullptr;                      // grid_type = 'amr'
};
struct State {
    std::vector<double> nH, xHI, xHeI, xHeII, ne, Te, rhokap;
};

// ---- tallies ----------------------------------------------------------------
struct Tally {
    std::vector<double> hhe;         // (6, nleaf), leaf-major: hhe[6*il + k]
    std::vector<double> jt;          // (nnu_band, nleaf): jt[nnu*il + inu]
    std::vector<double> metal;       // metal path estimators [(il*ntr + k)*2 + m]
    std::vector<double> dust_abs;    // dust_abs_path (nleaf), with ion_add_dust
    std::vector<double> fuv;         // fuv_field_path (nleaf), with add_fuv
    std::vector<double> img_dir, img_sca, img_dir0;   // peel-off images (nobs, nchan, nyim, nxim)
    std::vector<double> slab;        // slab_Iesc (nmu, 2) as [face * nmu + bin], face 0 top
    long double emitted = 0, absorbed = 0, escaped = 0;
    int64_t direct_segments = 0, scattered_segments = 0;
    void reset(int nleaf, int nnu, int ntr = 0, bool dust = false, bool fuv = false);
    void add(const Tally& o);
};

struct Photon {
    double x, y, z, kx, ky, kz;
    double E, wgt, Lpacket;
    int inu;
    double sHI, sHeI, sHeII;
    int nm = 0;                      // active metal transitions (E >= E_th)
    double sm[64];                   // their cross sections, threshold order
    int il = -1;                     // leaf of the start point (photon%icell_amr)
    double dust_abs = 0.0, dust_sca = 0.0, dust_g = 0.0;   // ionphys dust cache
    int nscatt = 0;
    bool inside = true;
    bool from_external = false;      // photon%from_external and the entry surface's inward normal
    double snx = 0.0, sny = 0.0, snz = 0.0;
    PacketRng rng;                   // the packet's scattering stream
};

struct Thermal;
struct Species;

// One peel-off observer (ion_peel_mod.f90 ion_peel_setup).
struct PeelObserver {
    double x, y, z, alpha, beta, gamma, distance;
    double R[3][3];            // grid -> observer frame
};

// milne_recomb_spectrum_mod.f90: ground-continuum recombination spectra.
struct Milne {
    static constexpr int NT = 192, NX = 512, NCH = 3;
    double lgT[NT], xg[NX], eth[NCH];
    std::vector<double> cdf;           // (NX, NT, NCH): cdf[(ich*NT + it)*NX + ix]
    std::vector<double> xbar, frac;    // (NT, NCH): [ich*NT + it]
    void setup(double eion_max);       // :99-228
    void tbracket(double T, int& it, double& w) const;              // :286-297
    double energy_per_recomb(int ich, double T) const;              // :302-312
    double sample(int ich, double T, double u, double eion_max) const;  // :320-350
};

// hei_twophoton_mod.f90: He I 2^1S -> 1^1S two-photon continuum above the
// H I edge (moments and energy-weighted sampling CDF of the tabulated A(y)).
struct HeI2ph {
    static constexpr int NCDF = 1024;
    static constexpr double E_TOT = 20.62;
    std::vector<double> ty, tA;
    double cdf_e[NCDF], grid_y[NCDF];
    double n_per_decay = 0.0, e_per_decay = 0.0;
    bool setup(const std::string& path, double eion_max);   // :97-192
    double shape(double y) const;                           // :82-93
    double sample(double u) const;                          // :199-219
};

// hei_cascade_mod.f90 and diffuse_mod.f90:308-325: the in-band energy per
// case-B He II recombination of the 2^3S line, the 584 A line that ionizes
// hydrogen and the two-photon continuum.
void hei_branch_energies(const HeI2ph& h, double T, double xHI, double xHeI, double& e3s, double& e1p, double& e1s);

struct Sim {
    Par par;
    Thermal* th = nullptr;           // thermal tables (solve_te)
    Species* sp = nullptr;           // metal registry (use_metals)
    RateModel rm;
    Qmc qmc;
    Band band;
    Grid grid;
    State st;
    Tally tally;
    std::vector<double> gamma_HI, gamma_HeI, gamma_HeII, heat_HI, heat_HeI, heat_HeII;
    std::vector<double> heat_dust, g0_fuv;   // ion_score_apply_dust_heat / _g0 (ion_score_mod.f90:319-355)
    DustTable dust;                          // ion_add_dust optics
    int nthreads = 1;
    // diffuse field (diffuse_mod.f90)
    Milne milne;
    HeI2ph hei2ph;                         // par%hei_diffuse
    std::vector<double> dif_ch, dif_cdf;   // (4, nleaf), (nleaf)
    double diffuse_lum = 0.0;
    int64_t diffuse_nphot = 0;
    bool defer_fill = false;   // orc_sim_set leaves the opacity refresh to the caller
    // peel-off imaging (ion_peel_mod.f90), set up by peel_setup()
    bool peel_on = false;            // par%ion_peel
    bool peel_pass = false;          // this pass peels (the imaging pass, main.f90:234-235)
    std::vector<PeelObserver> obs;
    int nchan = 1;
    double dxim = 0.0, dyim = 0.0;
    void peel_setup();                                            // ion_peel_setup, :49-206
    double tau_only(const Photon& ph, double kx, double ky, double kz) const;   // raytrace_amr.f90:678-775
    bool peel_pixel(const PeelObserver& o, double kx, double ky, double kz, int* ix, int* iy) const;
    void peel_direct(const Photon& ph, Tally& t) const;           // ion_peel_direct, :225-277
    void peel_scatter(const Photon& ph, Tally& t) const;          // ion_peel_scatter, :284-344
    int peel_channel(int inu) const;                              // :212-220
    void diffuse_build(double lpacket);                          // diffuse_mod.f90:60-121
    void gen_diffuse_qmc(int64_t ip, Photon& ph) const;          // diffuse_mod.f90:221-296
    void emit_external_rec(double u_mu, double u_phi, double u_face, double u_c1, double u_c2, Photon& ph) const;
    void emit_external_sph(double u_mu, double u_phi, double u_cost, double u_saz, Photon& ph) const;
    void emit_slab(double u_face, double u_c1, double u_c2, double u_mu, double u_phi, Photon& ph) const;
    void slab_add(Tally& t, double kz, double lum) const;            // slab_bnd_add, jtally_mod.f90:76-86
    void slab_wrap_xy(int iface, double& x, double& y) const;      // raytrace_amr.f90:330-345
    bool setup(const std::string& namelist, std::string* err);
    void transport_pass();           // ionizing_field_mod.f90:72-170
    void gas_rates_compute();        // gas_rates_mod.f90:82-153
    void gas_equilibrium_update(double* max_dx, double* dx_vol);  // ion_balance_mod.f90:352
    void gas_thermal_update(double m[4]);                         // thermal_mod.f90:124-249
    double net_rate(int il, double T, bool caseA, double& xHI, double& xHeI, double& xHeII,
                    double& ne) const;                             // thermal_mod.f90:38-115
    double thermal_cell(int il, double& xHI, double& xHeI, double& xHeII, double& ne) const;
    void opacity_fill();             // gas_opacity_fill, gas_opacity_mod.f90:299-306
    bool metals() const;             // use_metals with at least one element
    void metal_sigma(Photon& ph) const;   // species_packet_cross_sections
    ~Sim();
    void gen_photon_qmc(int64_t ip, Photon& ph) const;          // ion_band_mod.f90:1880
    void walk_edge_car(const Photon& ph, Tally& t, double* tau_edge) const;  // raytrace_amr.f90:534
    void walk_edge_amr(const Photon& ph, Tally& t, double* tau_edge) const;  // raytrace_amr.f90:422-486
    void walk_edge(const Photon& ph, Tally& t, double* tau_edge) const;
    // transport_ion_packet (raytrace_amr.f90:249-323): the edge walk, the
    // ledger, then with ion_dust_scatter the forced first interaction and the
    // scattered flights
    void transport_packet(Photon& ph, Tally& t) const;
    // raytrace_ion_to_tau_amr (:348-420) / raytrace_ion_to_tau_car (:594-676)
    void walk_to_tau(Photon& ph, double tau_in, Tally& t) const;
    // the leaf accessors of the edge walk on either grid: amr_find_leaf
    // (octree_mod.f90:69-93, car_index :185-195 on the car grid),
    // amr_cell_exit (:309-340) of the leaf's cell, amr_next_leaf (:518-559,
    // car_next :620-641 on the car grid); leaves 0-based, -1 none
    int leaf_find(double x, double y, double z) const;
    void leaf_exit(int il, double x, double y, double z, double kx, double ky, double kz, double* t,
                   int* iface) const;
    int leaf_next(int il, int iface, double x, double y, double z) const;
    bool amr_walk() const { return !grid.car || par.car_walk == "amr"; }
    int walk_leaves_amr(double x, double y, double z, double kx, double ky, double kz, int max_steps,
                        int32_t* out) const;
    int walk_leaves_car(double x, double y, double z, double kx, double ky,
                        double kz, int max_steps, int32_t* out) const;
};

// With sp != nullptr the metal electrons (metal_ne) and the two-way charge
// exchange (two_way) of leaf il join the closure.
void solve_ion_cell(const RateModel& rm, double He_abund, double gH,
                    double gHe1, double gHe2, double nH, double T, bool caseA,
                    double& xHI, double& xHeI, double& xHeII, double& ne,
                    const Species* sp = nullptr, int il = -1, bool metal_ne = false,
                    bool two_way = false);

}  // namespace orc
