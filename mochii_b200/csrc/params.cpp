// Parameter defaults and the "&parameters par%key = value /" namelist reader
// (read_input, setup.f90:11-626; defaults from type(params_type),
// define.f90:189-861).
//
// Keys that steer this path are parsed into mochii_params.  Every other
// key of the reference's params_type is accepted and has no effect here, so
// a reference input file reads unchanged; a key the reference does not know
// is an error (the Fortran namelist read fails the same way).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "mochii_gpu.h"
#include "physics.cuh"

using namespace mochii;

namespace {

// params_type components outside this path (define.f90:189-861).
const char* const kOtherKeys[] = {
    "albedo", "allsky", "allsky_nside", "allsky_x", "allsky_y", "allsky_z", "amr_type",
    "base_name", "centering", "cone_opening", "density_file", "density_powerlaw_index",
    "density_rscale", "density_zprofile", "density_zscale",
    "dust_emis_bands", "dust_emis_transport", "dust_emission_method", "dust_fast_table", "dust_model",
    "dust_niter", "dust_no_photons", "dust_nu", "dust_sed", "dust_single_teq", "dust_tol",
    "emis_output", "exetime", 
    "f_ion_dust", "f_ion_pah", "f_pah", "file_format", "geometry", "h_coll_effects",
    "hei_metastable", "hgg", "kext_file",
    "lambda0", "lambda_max", "lambda_min", "line_case", "mrw_gamma", "nlambda", "no_print",
    "nobs", "nprint", "nr", "nscatt_tot", "num_send_at_once",
    "out_bitpix", "out_bitpix_force", "out_file", "output_normalization", "pe_scale",
    "radiation_angular_pdf_file", "reduce_factor",
    "save_jlam",
    "scatt_mat_file", "sed_data_dir", "sed_dl07_sdindex", "sed_dl07_uisrf", "sed_kext", "sed_nt",
    "sed_pah_live", "sed_thi", "sed_tlo", "sightline_tau", "source_rscale", "source_spectrum", "source_zscale",
    "spiral_amp", "spiral_m", "spiral_pitch", "src_axial_ratio", "src_boxiness",
    "src_geometry", "src_reff", "src_rscale", "src_sersic_index", "src_spectrum",
    "src_zscale", "use_amr_grid", "use_dustemis", "use_master_slave", "use_mrw",
    "use_reduced_wgt", "use_sed", "use_stokes", "xyz_symmetry", "z_global", "z_ref",
    "z_symmetry", "dust_density_law_file"};

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}
std::string strip(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    return s.substr(a, s.find_last_not_of(" \t\r\n") - a + 1);
}
bool parse_real(const std::string& v, double* out) {
    std::string s = strip(v);
    for (auto& c : s)
        if (c == 'd' || c == 'D') c = 'e';
    char* end = nullptr;
    const double x = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || strip(end).size()) return false;
    *out = x;
    return true;
}
bool parse_int(const std::string& v, int64_t* out) {
    double x;
    if (!parse_real(v, &x)) return false;   // "1.0e6" into an integer field
    *out = (int64_t)std::llround(x);
    return true;
}
bool parse_bool(const std::string& v, int* out) {
    const std::string s = lower(strip(v));
    if (s == ".true." || s == "t" || s == ".t." || s == "true") { *out = 1; return true; }
    if (s == ".false." || s == "f" || s == ".f." || s == "false") { *out = 0; return true; }
    return false;
}
std::string unquote(const std::string& v) {
    std::string s = strip(v);
    if (s.size() >= 2 && (s[0] == '\'' || s[0] == '"') && s.back() == s[0]) s = s.substr(1, s.size() - 2);
    return strip(s);
}
void copy_str(char* dst, size_t cap, const std::string& s) {
    std::strncpy(dst, s.c_str(), cap - 1);
    dst[cap - 1] = 0;
}

}  // namespace

extern "C" size_t mochii_params_size(void) { return sizeof(mochii_params); }

extern "C" int mochii_params_default(mochii_params* p) {
    if (!p) return MOCHII_ERR_BAD_PARAM;
    std::memset(p, 0, sizeof(*p));
    p->nphotons = 100000;              // no_photons = 1e5
    p->launch_sobol = 0;               // launch_sequence = 'random'
    p->qmc_seed = 12345;
    p->source_cdf_tol = 1.0e-8;
    p->luminosity = -999.0;
    p->tstar = -999.0;
    p->random_seed = 0;
    p->nnu_ion = 16;
    p->eion_min = 13.598;
    p->eion_max = 100.0;
    p->efuv_min = 6.0;
    p->nnu_fuv = 8;
    p->ion_align_edges = 1;
    p->grid_car = 1;
    p->car_walk_dda = 1;
    p->nx = 1; p->ny = 1; p->nz = 11;
    p->xmax = p->ymax = p->zmax = 1.0;
    p->rmax = -999.0; p->rmin = 0.0; p->nH_const = -1.0;
    p->distance2cm = kKpc2cm;
    copy_str(p->distance_unit, sizeof(p->distance_unit), "kpc");
    p->source_point = 1;
    p->nsource = 1;
    for (int i = 0; i < MOCHII_MAX_SRC; ++i) { p->src_tstar[i] = -999.0; p->src_lum[i] = -999.0; }
    p->xHI_init = 1.0; p->xHeI_init = 1.0; p->xHeII_init = 0.0;
    p->He_abund = 0.1;
    p->gas_niter = 0;
    p->gas_tol = 1.0e-3; p->te_fixed = 1.0e4; p->ion_relax = 1.0;
    p->caseA = 0;
    p->te_min = 1.0e3; p->te_max = 5.0e4; p->gas_tol_te = 1.0e-3;
    p->abund_C = 2.2e-4; p->abund_N = 4.0e-5; p->abund_O = 3.3e-4; p->abund_Ne = 5.0e-5; p->abund_S = 9.0e-6;
    p->ion_metal_abs = 1; p->metal_ne = 1; p->metal_heat = 1; p->metal_freefree = 1;
    p->charge_exchange_two_way = 1;
    p->cooling_local_ne = 1;
    p->diffuse_model = 0;
    p->dust_law = 0;
    p->DGR = 1.0e-2; p->cext_dust = 1.6059e-21;
    p->precision = MOCHII_PREC_FP64;
    p->metal_moments = 1;
    p->lambda_ref = 0.55;
    p->taumax = -999.0;
    p->tauhomo = -999.0;
    p->solver_warp = 3;
    p->tally64 = 1;
    p->metal_rate_table = 1;
    p->packet_chunk = 1 << 22;
    p->packet_order = 2;   // 'coherent' (the launch order where it does not apply)
    p->ion_peel = 0; p->peel_bins = 0; p->save_direc0 = 0;
    p->nxim = 129; p->nyim = 129;   // define.f90:531-532
    p->refine_front = 0; p->refine_iter = 20; p->refine_lbase = 5; p->refine_lmax = 7;   // define.f90:826-831
    p->refine_eps = 1.0e-2; p->refine_dx = 0.2;
    p->ext_intensity = -1.0; p->ext_tstar = -999.0; p->ext_geometry = 0;   // define.f90:270-277
    p->slab_faces = 1; p->slab_nmu = 20;                                    // define.f90:312-321
    p->ext_scale = 1.0;                                                     // define.f90:303
    const double nan = std::numeric_limits<double>::quiet_NaN();
    p->distance = nan; p->dxim = nan; p->dyim = nan;
    for (int i = 0; i < MOCHII_MAX_OBS; ++i) {
        p->alpha[i] = p->beta[i] = p->gamma[i] = nan;
        p->obsx[i] = p->obsy[i] = p->obsz[i] = nan;
        p->phase_angle[i] = p->inclination_angle[i] = p->position_angle[i] = nan;
    }
    return MOCHII_OK;
}

namespace {
int set_key(mochii_params* p, std::string key, const std::vector<std::string>& vals, int index,
            std::string* err) {
    key = lower(strip(key));
    const std::string v = vals.empty() ? std::string() : vals[0];
    auto bad = [&](const char* what) {
        if (err) *err = "par%" + key + ": " + what + " '" + v + "'";
        return MOCHII_ERR_BAD_PARAM;
    };
    double d;
    int64_t i;
    int b;
#define REAL(name, field) if (key == name) { if (!parse_real(v, &d)) return bad("not a real"); p->field = d; return 0; }
#define INT(name, field) if (key == name) { if (!parse_int(v, &i)) return bad("not an integer"); p->field = (int)i; return 0; }
#define BOOL(name, field) if (key == name) { if (!parse_bool(v, &b)) return bad("not a logical"); p->field = b; return 0; }
    if (key == "no_photons" || key == "nphotons") {
        if (!parse_int(v, &i) || i < 1) return bad("not a positive count");
        p->nphotons = i;
        return 0;
    }
    if (key == "launch_sequence") {
        const std::string s = lower(unquote(v));
        if (s != "sobol" && s != "random") return bad("must be 'sobol' or 'random'");
        p->launch_sobol = s == "sobol";
        return 0;
    }
    INT("qmc_seed", qmc_seed) INT("iseed", random_seed)
    REAL("source_cdf_tol", source_cdf_tol) REAL("luminosity", luminosity) REAL("tstar", tstar)
    INT("nnu_ion", nnu_ion) REAL("eion_min", eion_min) REAL("eion_max", eion_max)
    BOOL("add_fuv", add_fuv) REAL("efuv_min", efuv_min) INT("nnu_fuv", nnu_fuv)
    BOOL("ion_align_edges", ion_align_edges)
    if (key == "grid_type") {
        const std::string s = lower(unquote(v));
        if (s != "car" && s != "amr" && s != "uniform") return bad("must be 'car' or 'amr'");
        p->grid_car = s != "amr";
        return 0;
    }
    if (key == "car_walk") {
        const std::string s = lower(unquote(v));
        if (s != "dda" && s != "amr") return bad("must be 'dda' or 'amr'");
        p->car_walk_dda = s == "dda";
        return 0;
    }
    INT("nx", nx) INT("ny", ny) INT("nz", nz)
    REAL("xmax", xmax) REAL("ymax", ymax) REAL("zmax", zmax)
    REAL("rmax", rmax) REAL("rmin", rmin) REAL("nh_const", nH_const)
    if (key == "distance_unit") {
        const std::string s = lower(unquote(v));
        if (s == "kpc") p->distance2cm = kKpc2cm;
        else if (s == "pc") p->distance2cm = kPc2cm;
        else if (s == "au") p->distance2cm = kAu2cm;
        else if (s == "cm") p->distance2cm = 1.0;
        else return bad("unknown unit");
        copy_str(p->distance_unit, sizeof(p->distance_unit), s);
        return 0;
    }
    if (key == "distance2cm") { if (!parse_real(v, &d)) return bad("not a real"); p->distance2cm = d; return 0; }
    if (key == "amr_file") { copy_str(p->amr_file, sizeof(p->amr_file), unquote(v)); return 0; }
    if (key == "source_geometry") {
        const std::string s = lower(unquote(v));
        p->source_point = s == "point";
        p->source_external = (s == "external" || s == "external_rec") ? 1 : s == "external_sph" ? 2 : 0;
        if (p->source_external) p->source_point = 1;   // the external-only shorthand of setup.f90:240-258
        p->source_slab = s == "slab";
        if (!p->source_point && !p->source_slab) return bad("must be 'point', 'slab', 'external_rec' or 'external_sph'");
        return 0;
    }
    BOOL("xy_periodic", xy_periodic) INT("slab_nmu", slab_nmu)
    if (key == "slab_faces") {   // setup.f90:267-271
        const std::string s = lower(unquote(v));
        if (s != "top" && s != "bottom" && s != "both") return bad("must be 'top', 'bottom' or 'both'");
        p->slab_faces = s == "top" ? 1 : s == "bottom" ? 2 : 3;
        return 0;
    }
    if (key == "slab_top_mode" || key == "slab_bot_mode") {   // setup.f90:273-277
        const std::string s = lower(unquote(v));
        if (s != "beam" && s != "isotropic") return bad("must be 'beam' or 'isotropic'");
        p->slab_mode[key == "slab_bot_mode"] = s == "isotropic";
        return 0;
    }
    REAL("slab_top_theta", slab_theta[0]) REAL("slab_bot_theta", slab_theta[1])
    REAL("slab_top_phi", slab_phi[0]) REAL("slab_bot_phi", slab_phi[1])
    REAL("slab_top_source", slab_source[0]) REAL("slab_bot_source", slab_source[1])
    if (key == "ext_geometry") {
        const std::string s = lower(unquote(v));
        if (s != "rec" && s != "sph") return bad("must be 'rec' or 'sph'");
        p->ext_geometry = s == "sph" ? 1 : 0;
        return 0;
    }
    if (key == "ext_spectrum" || key == "ion_spectrum" || key == "src_spectrum_file") {
        const std::string s = strip(unquote(v));
        char* dst = key == "ext_spectrum" ? p->ext_spectrum : key == "ion_spectrum" ? p->ion_spectrum
                                                                                : p->src_spectrum_file;
        if (s.size() >= MOCHII_STRLEN) return bad("path too long");
        copy_str(dst, MOCHII_STRLEN, s);
        if (key == "ext_spectrum") p->ext_spectrum_set = !s.empty();
        return 0;
    }
    if (key == "spectrum_type") {   // setup.f90:213-221
        const std::string s = lower(strip(unquote(v)));
        static const char* const names[] = {"shape_ev", "per_ev", "per_hz", "per_ang", "per_um"};
        for (int k = 0; k < 5; ++k)
            if (s == names[k]) { p->spectrum_type = k; return 0; }
        return bad("must be 'shape_ev', 'per_ev', 'per_hz', 'per_ang' or 'per_um'");
    }
    REAL("ext_scale", ext_scale)
    REAL("ext_intensity", ext_intensity) REAL("ext_tstar", ext_tstar)
    REAL("xs_point", xs_point) REAL("ys_point", ys_point) REAL("zs_point", zs_point)
    INT("nsource", nsource)
    if (key == "alpha" || key == "beta" || key == "gamma" || key == "obsx" || key == "obsy" || key == "obsz" ||
        key == "phase_angle" || key == "inclination_angle" || key == "position_angle") {
        double* arr = key == "alpha" ? p->alpha : key == "beta" ? p->beta : key == "gamma" ? p->gamma
                    : key == "obsx" ? p->obsx : key == "obsy" ? p->obsy : key == "obsz" ? p->obsz
                    : key == "phase_angle" ? p->phase_angle : key == "inclination_angle" ? p->inclination_angle
                                                                                       : p->position_angle;
        for (size_t k = 0; k < vals.size(); ++k) {
            const int slot = index - 1 + (int)k;
            if (slot < 0 || slot >= MOCHII_MAX_OBS) return bad("observer index outside 1..16");
            if (vals[k].empty()) continue;
            if (!parse_real(vals[k], &d)) return bad("not a real");
            arr[slot] = d;
        }
        return 0;
    }
    BOOL("ion_peel", ion_peel) BOOL("peel_bins", peel_bins) BOOL("save_direc0", save_direc0)
    INT("nxim", nxim) INT("nyim", nyim) REAL("distance", distance) REAL("dxim", dxim) REAL("dyim", dyim)
    if (key == "nobs") return 0;   // derived from the observer lists (ion_peel_setup)
    if (key == "src_tstar" || key == "src_lum" || key == "src_x" || key == "src_y" || key == "src_z") {
        double* arr = key == "src_tstar" ? p->src_tstar : key == "src_lum" ? p->src_lum
                    : key == "src_x" ? p->src_x : key == "src_y" ? p->src_y : p->src_z;
        for (size_t k = 0; k < vals.size(); ++k) {
            const int slot = index - 1 + (int)k;
            if (slot < 0 || slot >= MOCHII_MAX_SRC) return bad("index outside 1..MAX_SRC");
            if (vals[k].empty()) continue;
            if (!parse_real(vals[k], &d)) return bad("not a real");
            arr[slot] = d;
        }
        return 0;
    }
    REAL("xhi_init", xHI_init) REAL("xhei_init", xHeI_init) REAL("xheii_init", xHeII_init)
    REAL("he_abund", He_abund) INT("gas_niter", gas_niter) REAL("gas_tol", gas_tol)
    REAL("te_fixed", te_fixed) REAL("ion_relax", ion_relax)
    if (key == "case_ab") {
        const std::string s = unquote(v);
        if (s != "A" && s != "B" && s != "a" && s != "b") return bad("must be 'A' or 'B'");   // setup.f90:503-506
        p->caseA = (s == "A" || s == "a");
        return 0;
    }
    if (key == "recomb_model") {
        const std::string s = lower(unquote(v));
        if (s != "badnell_milne" && s != "hui_gnedin") return bad("must be 'badnell_milne' or 'hui_gnedin'");
        p->recomb_hui_gnedin = s == "hui_gnedin";
        return 0;
    }
    if (key == "ci_model") {
        const std::string s = lower(unquote(v));
        if (s != "voronov" && s != "dere_hybrid") return bad("must be 'voronov' or 'dere_hybrid'");
        p->ci_dere_hybrid = s == "dere_hybrid";
        return 0;
    }
    if (key == "conv_crit") {
        const std::string s = lower(unquote(v));
        if (s != "cell" && s != "vol") return bad("must be 'cell' or 'vol'");
        p->conv_vol = s == "vol";
        return 0;
    }
    if (key == "cooling_model") { p->cooling_local_ne = lower(unquote(v)) == "local_ne"; return 0; }
    if (key == "charge_exchange") { p->charge_exchange_two_way = lower(unquote(v)) == "two_way"; return 0; }
    BOOL("solve_te", solve_te) REAL("te_min", te_min) REAL("te_max", te_max) REAL("gas_tol_te", gas_tol_te)
    BOOL("require_convergence", require_convergence) BOOL("use_metals", use_metals)
    REAL("abund_c", abund_C) REAL("abund_n", abund_N) REAL("abund_o", abund_O) REAL("abund_ne", abund_Ne)
    REAL("abund_s", abund_S) REAL("abund_ar", abund_Ar) REAL("abund_mg", abund_Mg) REAL("abund_fe", abund_Fe)
    REAL("abund_si", abund_Si) REAL("abund_cl", abund_Cl) REAL("abund_ca", abund_Ca)
    BOOL("ion_metal_abs", ion_metal_abs) BOOL("metal_ne", metal_ne) BOOL("metal_heat", metal_heat)
    BOOL("metal_freefree", metal_freefree) BOOL("gaunt_vh14", gaunt_vh14)
    BOOL("fe_levels_full", fe_levels_full)
    BOOL("diffuse_field", diffuse_field) BOOL("use_sec_ion", use_sec_ion) BOOL("hei_diffuse", hei_diffuse)
    BOOL("refine_front", refine_front) INT("refine_iter", refine_iter) INT("refine_lbase", refine_lbase)
    INT("refine_lmax", refine_lmax) REAL("refine_eps", refine_eps) REAL("refine_dx", refine_dx)
    BOOL("ion_add_dust", ion_add_dust) BOOL("ion_dust_scatter", ion_dust_scatter) BOOL("grain_pe", grain_pe)
    REAL("dgr", DGR) REAL("cext_dust", cext_dust) REAL("lambda_ref", lambda_ref)
    REAL("taumax", taumax) REAL("tauhomo", tauhomo)
    if (key == "dust_density_law") {
        const std::string s = lower(unquote(v));
        p->dust_law = s == "global_dgr" ? 0 : s == "none" ? 1 : 2;
        return 0;
    }
    if (key == "diffuse_energy_model") {   // setup.f90:186-193
        const std::string s = lower(unquote(v));
        if (s == "milne") p->diffuse_model = 0;
        else if (s == "exponential") p->diffuse_model = 1;
        else if (s == "threshold") p->diffuse_model = 2;
        else return bad("must be 'milne', 'exponential' or 'threshold'");
        return 0;
    }
    if (key == "ion_dust_kext") { copy_str(p->ion_dust_kext, sizeof(p->ion_dust_kext), unquote(v)); return 0; }
    if (key == "data_dir") { copy_str(p->data_dir, sizeof(p->data_dir), unquote(v)); return 0; }
    if (key == "atomic_dir") { copy_str(p->atomic_dir, sizeof(p->atomic_dir), unquote(v)); return 0; }
    if (key == "packet_order") {
        const std::string s = lower(unquote(v));
        if (s != "direction" && s != "launch" && s != "coherent")
            return bad("must be 'coherent', 'direction' or 'launch'");
        p->packet_order = s == "coherent" ? 2 : s == "direction" ? 1 : 0;
        return 0;
    }
    if (key == "packet_chunk") {
        if (!parse_int(v, &i) || i < 1024) return bad("must be an integer >= 1024");
        p->packet_chunk = i;
        return 0;
    }
    if (key == "metal_rates") {
        const std::string s = lower(unquote(v));
        if (s != "table" && s != "exact") return bad("must be 'table' or 'exact'");
        p->metal_rate_table = s == "table";
        return 0;
    }
    if (key == "tally_precision") {
        const std::string s = lower(unquote(v));
        if (s != "compensated" && s != "fp64") return bad("must be 'compensated' or 'fp64'");
        p->tally64 = s == "fp64";
        return 0;
    }
    if (key == "cell_layout") {
        const std::string s = lower(unquote(v));
        if (s != "warp" && s != "thread" && s != "lockstep" && s != "flow" && s != "lane")
            return bad("must be 'lockstep', 'lane', 'flow' or 'warp'");
        p->solver_warp = s == "warp" ? 1 : s == "flow" ? 2 : s == "lane" ? 3 : 0;
        return 0;
    }
    if (key == "thermal_solver") {
        const std::string s = lower(unquote(v));
        if (s != "bisection" && s != "bracketed") return bad("must be 'bisection' or 'bracketed'");
        p->solver_bracketed = s == "bracketed";
        return 0;
    }
    if (key == "metal_tally") {
        const std::string s = lower(unquote(v));
        if (s != "moments" && s != "exact") return bad("must be 'moments' or 'exact'");
        p->metal_moments = s == "moments";
        return 0;
    }
    if (key == "precision") {
        const std::string s = lower(unquote(v));
        if (s != "fp64" && s != "fp32") return bad("must be 'fp64' or 'fp32'");
        p->precision = s == "fp64" ? MOCHII_PREC_FP64 : MOCHII_PREC_FP32;
        return 0;
    }
#undef REAL
#undef INT
#undef BOOL
    for (const char* k : kOtherKeys)
        if (key == k) return 0;
    if (err) *err = "par%" + key + ": not a component of the reference parameter type";
    return MOCHII_ERR_BAD_PARAM;
}

// Split "key[(i)] = v1, v2, ..." assignments out of a namelist body.
int parse_text(mochii_params* p, const std::string& text, std::string* err) {
    std::string clean;
    char q = 0;
    bool body = false;
    for (size_t i = 0; i < text.size(); ++i) {
        const char c = text[i];
        if (q) { clean += c; if (c == q) q = 0; continue; }
        if (c == '\'' || c == '"') { q = c; clean += c; continue; }
        if (c == '!') { while (i < text.size() && text[i] != '\n') ++i; clean += '\n'; continue; }
        if (c == '&') {   // group name "&parameters"
            size_t j = i + 1;
            while (j < text.size() && (std::isalnum((unsigned char)text[j]) || text[j] == '_')) ++j;
            if (lower(text.substr(i + 1, j - i - 1)) != "parameters") {
                if (err) *err = "namelist group must be &parameters";
                return MOCHII_ERR_BAD_PARAM;
            }
            body = true;
            i = j - 1;
            continue;
        }
        if (c == '/' && body) break;   // end of the group
        clean += c;
    }
    const std::string lc = lower(clean);
    size_t pos = 0;
    while ((pos = lc.find("par%", pos)) != std::string::npos) {
        const size_t eq = lc.find('=', pos);
        if (eq == std::string::npos) { if (err) *err = "assignment without '='"; return MOCHII_ERR_BAD_PARAM; }
        std::string key = strip(lc.substr(pos + 4, eq - pos - 4));
        const size_t next = lc.find("par%", eq);
        const std::string raw = clean.substr(eq + 1, (next == std::string::npos ? clean.size() : next) - eq - 1);
        std::vector<std::string> vals;
        std::string cur;
        char qq = 0;
        for (char c : raw) {
            if (qq) { cur += c; if (c == qq) qq = 0; continue; }
            if (c == '\'' || c == '"') { qq = c; cur += c; continue; }
            if (c == ',' || c == '\n') { vals.push_back(strip(cur)); cur.clear(); continue; }
            cur += c;
        }
        vals.push_back(strip(cur));
        while (!vals.empty() && vals.back().empty()) vals.pop_back();
        int index = 1;
        const size_t lp = key.find('(');
        if (lp != std::string::npos) {
            index = std::atoi(key.substr(lp + 1).c_str());
            key = strip(key.substr(0, lp));
        }
        const int rc = set_key(p, key, vals, index, err);
        if (rc) return rc;
        pos = eq;
    }
    return MOCHII_OK;
}
}  // namespace

extern "C" int mochii_params_set(mochii_params* p, const char* key, const char* value) {
    if (!p || !key || !value) return MOCHII_ERR_BAD_PARAM;
    std::string k(key);
    int index = 1;
    const size_t lp = k.find('(');
    if (lp != std::string::npos) {
        index = std::atoi(k.substr(lp + 1).c_str());
        k = k.substr(0, lp);
    }
    std::string err;
    std::vector<std::string> vals;
    std::string cur;
    for (const char* c = value; *c; ++c) {
        if (*c == ',') { vals.push_back(strip(cur)); cur.clear(); } else cur += *c;
    }
    vals.push_back(strip(cur));
    return set_key(p, k, vals, index, &err);
}

extern "C" int mochii_params_parse_namelist(mochii_params* p, const char* text, char* errbuf, size_t errlen) {
    if (!p || !text) return MOCHII_ERR_BAD_PARAM;
    std::string err;
    const int rc = parse_text(p, text, &err);
    if (errbuf && errlen) { std::strncpy(errbuf, err.c_str(), errlen - 1); errbuf[errlen - 1] = 0; }
    return rc;
}

extern "C" int mochii_params_read_namelist(mochii_params* p, const char* path, char* errbuf, size_t errlen) {
    std::ifstream f(path);
    if (!f) {
        if (errbuf && errlen) std::snprintf(errbuf, errlen, "cannot open %s", path);
        return MOCHII_ERR_BAD_PARAM;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    return mochii_params_parse_namelist(p, ss.str().c_str(), errbuf, errlen);
}
