/*
 * mochii_gpu.h -- C ABI of the B200 photon-packet transport and
 * ionisation/thermal-balance library (libmochii_gpu.so).
 *
 * The library replaces the four module entry points MoCHII's driver loop
 * calls once per iteration (main.f90:128-185, :225):
 *
 *   ionizing_field_and_rates(label, with_peel)   ionizing_field_mod.f90:72
 *   gas_equilibrium_update(max_dx, dx_vol)       ion_balance_mod.f90:352
 *   gas_thermal_update(max_dx, max_dte, dx_vol, dte_vol)   thermal_mod.f90:124
 *   gas_opacity_fill()                           gas_opacity_mod.f90:299
 *
 * and the parameter-file interface read_input (setup.f90:11-35, namelist
 * "&parameters par%key = value /").  All signatures use plain C types,
 * pointers and sizes; no CUDA or torch types cross the boundary.  Every
 * call returns an int status (MOCHII_OK = 0).  Nothing aborts, traps or
 * waits without a bound: device guards raise flags that are read after the
 * stream synchronises and come back as status codes.
 *
 * Threading: one host thread per context; calls on one context are not
 * reentrant.  Each context owns one CUDA stream on the device that was
 * current when mochii_init ran.
 */
#ifndef MOCHII_GPU_H
#define MOCHII_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (reference: MPI_ABORT / error stop sites) ---------- */
enum {
    MOCHII_OK = 0,
    MOCHII_ERR_BAD_PARAM = 1,     /* read_input validation, setup.f90:76-626      */
    MOCHII_ERR_TABLE = 2,         /* unreadable / inconsistent data table          */
    MOCHII_ERR_CUDA = 3,          /* CUDA runtime error                            */
    MOCHII_ERR_TIMEOUT = 4,       /* a bounded device loop hit its cap             */
    MOCHII_ERR_NONFINITE = 5,     /* NaN/Inf in a tally or state field             */
    MOCHII_ERR_CLOSURE = 6,       /* energy closure > 5e-13, ion_score_mod.f90:386 */
    MOCHII_ERR_NOT_CONVERGED = 7, /* require_convergence, main.f90:197-207         */
    MOCHII_ERR_UNSUPPORTED = 8,   /* configuration outside the built path          */
    MOCHII_ERR_NO_DEVICE = 9      /* no CUDA device visible                        */
};

#define MOCHII_MAX_SRC 16   /* define.f90:74 MAX_SRC */
#define MOCHII_MAX_OBS 16   /* observers of the peel-off images (define.f90:76 allows 181) */
#define MOCHII_STRLEN 256

/* Device arithmetic for the transport pass. */
enum { MOCHII_PREC_FP64 = 0, MOCHII_PREC_FP32 = 1 };

/*
 * Parameters: the subset of type(params_type) (define.f90:189-861) that the
 * transport + balance path reads, with the reference's names and defaults
 * (mochii_params_default).  Strings are NUL-terminated.
 */
typedef struct mochii_params {
    /* launch (define.f90:196-215) */
    int64_t nphotons;                /* par%no_photons                        */
    int launch_sobol;                /* par%launch_sequence == 'sobol'        */
    int qmc_seed;                    /* par%qmc_seed                          */
    double source_cdf_tol;           /* par%source_cdf_tol                    */
    double luminosity;               /* par%luminosity [erg/s]                */
    double tstar;                    /* par%tstar [K]                         */
    int random_seed;                 /* par%iseed (counter RNG key)           */
    /* band (define.f90 ion block) */
    int nnu_ion;
    double eion_min, eion_max;
    int add_fuv;
    double efuv_min;
    int nnu_fuv;
    int ion_align_edges;
    /* geometry */
    int grid_car;                    /* par%grid_type == 'car'                */
    int car_walk_dda;                /* par%car_walk == 'dda'                 */
    int nx, ny, nz;
    double xmax, ymax, zmax;
    double rmax, rmin, nH_const;
    double distance2cm;              /* from par%distance_unit                */
    char distance_unit[16];
    char amr_file[MOCHII_STRLEN];
    /* sources */
    int source_point;                /* par%source_geometry == 'point'        */
    double xs_point, ys_point, zs_point;
    int nsource;
    double src_tstar[MOCHII_MAX_SRC], src_lum[MOCHII_MAX_SRC];
    double src_x[MOCHII_MAX_SRC], src_y[MOCHII_MAX_SRC], src_z[MOCHII_MAX_SRC];
    /* gas state and iteration */
    double xHI_init, xHeI_init, xHeII_init;
    double He_abund;
    int gas_niter;
    double gas_tol, te_fixed, ion_relax;
    int caseA;                       /* par%case_ab == 'A'                    */
    int recomb_hui_gnedin;           /* par%recomb_model == 'hui_gnedin'      */
    int ci_dere_hybrid;              /* par%ci_model == 'dere_hybrid'         */
    int conv_vol;                    /* par%conv_crit == 'vol'                */
    int solve_te;
    double te_min, te_max, gas_tol_te;
    int require_convergence;
    /* metals (define.f90 abund_* and metal switches) */
    int use_metals;
    double abund_C, abund_N, abund_O, abund_Ne, abund_S, abund_Ar,
           abund_Mg, abund_Fe, abund_Si, abund_Cl, abund_Ca;
    int ion_metal_abs, metal_ne, metal_heat, metal_freefree;
    int charge_exchange_two_way;     /* par%charge_exchange == 'two_way'      */
    int cooling_local_ne;            /* par%cooling_model == 'local_ne'       */
    int gaunt_vh14;
    /* diffuse field, secondary ionisation, dust, FUV */
    int diffuse_field, use_sec_ion;
    int diffuse_model;               /* par%diffuse_energy_model: 0 milne, 1 exponential, 2 threshold */
    int ion_add_dust, ion_dust_scatter;
    int dust_law;                    /* 0 global_dgr, 1 none, 2 other         */
    double DGR, cext_dust;
    int grain_pe;
    char ion_dust_kext[MOCHII_STRLEN];
    char data_dir[MOCHII_STRLEN];
    char atomic_dir[MOCHII_STRLEN];
    /* device arithmetic (not a reference key: 'fp64' or 'fp32') */
    int precision;
    /* par%fe_levels_full: Fe n-level atoms from the '_full' files */
    int fe_levels_full;
    /* metal path tallies (not a reference key, 'moments' or 'exact'):
     * 1 = per-leaf Chebyshev energy moments in threshold-aligned bins,
     * contracted with the cross sections after the pass; 0 = one pair of
     * tallies per active transition per segment (species_rate_path_score) */
    int metal_moments;
    /* cell solver (not a reference key, 'bisection' or 'bracketed'):
     * 0 = the reference's damped n_e fixed point and bisection on log T over
     * [te_min, te_max]; 1 = the same roots found by bracketed Illinois
     * iterations, n_e from the cell's current state and T_e from a warm start
     * (the cell's current T_e, or a supplied prediction) */
    int solver_bracketed;
    /* grain optics reference wavelength [um] and the dust normalisations
     * (define.f90:211-212,361); taumax / tauhomo > 0 are not built */
    double lambda_ref, taumax, tauhomo;
    /* thermal solve with metals (not a reference key, par%cell_layout):
     * 3 'lane' = one thread per leaf, the metal rate cache in shared memory,
     * the n_e and H roots one per-lane machine, each lane claiming the next
     * leaf of the work order as it finishes (default); 0 'lockstep' (or
     * 'thread') = one thread per leaf, warp-uniform nested root loops over
     * 32-leaf chunks sorted by work, the cache in local memory; 1 'warp' = one
     * warp per leaf, the metal cascade spread over the lanes; 2 'flow' = one
     * thread per leaf, each lane's whole solve a state machine served by
     * warp-wide evaluations */
    int solver_warp;
    /* path tallies with FP32 segments (not a reference key,
     * par%tally_precision): 1 'fp64' = FP64 atomic tallies (default: on B200
     * the FP64 reduction is a native L2 atomic, faster than the two-word
     * compensated update); 0 'compensated' = (hi, lo) FP32 pairs summed in
     * FP64 after the pass */
    int tally64;
    /* metal rate coefficients in the thermal solve (not a reference key,
     * par%metal_rates): 1 'table' = interpolated from a 4096-node ln T table
     * over [te_min, te_max] (default); 0 'exact' = every evaluation direct */
    int metal_rate_table;
    /* packets per launch-walk chunk (not a reference key, par%packet_chunk):
     * the size of the packet-record buffer, default 4194304 */
    int64_t packet_chunk;
    /* walk order of a chunk's packets (not a reference key,
     * par%packet_order): 2 'coherent' (default) = the chunk sorted by source,
     * direction cell and energy quantile (diffuse packets: direction cell and
     * start neighbourhood) before its launch, each warp walking 32 nearly
     * parallel packets and summing the tallies of lanes in the same leaf and
     * bins before one reduction (the Cartesian grid without grains or FUV;
     * elsewhere the launch order);
     * 0 'launch' = the launch (Sobol) order; 1 'direction' = sorted by source
     * and direction cell after the launch, per-lane reductions */
    int packet_order;
    /* peel-off imaging (par%ion_peel; ion_peel_mod.f90, define.f90:518-544,
     * 658-664): observers by angle lists (alpha, beta, gamma [deg]; or the
     * phase, inclination and position angles) or by position (obsx/y/z,
     * code units), all NaN when unset as in the reference; at most
     * MOCHII_MAX_OBS observers here.  distance, dxim, dyim NaN: derived. */
    int ion_peel, peel_bins, save_direc0;
    int nxim, nyim;
    double distance, dxim, dyim;
    double alpha[MOCHII_MAX_OBS], beta[MOCHII_MAX_OBS], gamma[MOCHII_MAX_OBS];
    double obsx[MOCHII_MAX_OBS], obsy[MOCHII_MAX_OBS], obsz[MOCHII_MAX_OBS];
    double phase_angle[MOCHII_MAX_OBS], inclination_angle[MOCHII_MAX_OBS], position_angle[MOCHII_MAX_OBS];
    /* par%hei_diffuse (define.f90:634): with the diffuse field, a fourth
     * channel of He I excited-level recombination radiation -- the 2^3S and
     * 584 A lines and the 2^1S two-photon continuum above the H I edge
     * (diffuse_mod.f90:96-106, 274-284; hei_cascade_mod, hei_twophoton_mod),
     * the two-photon shape read from <data_dir>/HeI2phot.dat */
    int hei_diffuse;
    /* solution-driven I-front re-refinement of the octree (define.f90:821-831,
     * amr_refine_mod.f90): at iteration refine_iter the tree is rebuilt to
     * level refine_lmax where refine_eps < x_HI < 1 - refine_eps or a face
     * neighbour's x_HI differs by more than refine_dx, refine_lbase
     * elsewhere (mochii_refine_front) */
    int refine_front, refine_iter, refine_lbase, refine_lmax;
    double refine_eps, refine_dx;
    /* isotropic external radiation field (define.f90:266-278): on when
     * ext_intensity (band J [erg/s/cm^2/sr]) > 0, a source component after
     * the nsource point sources entering through the box faces
     * (ext_geometry 0 'rec') or a bounding sphere of radius rmax (1 'sph');
     * Planck spectrum at ext_tstar (> 0) else tstar.  source_geometry
     * 'external' / 'external_rec' / 'external_sph' is the external-only
     * shorthand (source_external 1 / 1 / 2: nsource taken as 0).
     * ext_spectrum_set: a par%ext_spectrum file or preset was named */
    double ext_intensity, ext_tstar;
    int ext_geometry, source_external, ext_spectrum_set;
    /* plane-parallel slab illumination (define.f90:217, 304-321):
     * source_geometry 'slab' (source_slab 1) on an xy-periodic grid
     * (xy_periodic: the walks wrap the x and y faces, z faces are open).
     * slab_faces bit 1 top (+z), bit 2 bottom (-z); per face [0] top, [1]
     * bottom: mode 0 beam / 1 isotropic, incidence theta and beam azimuth phi
     * [deg], source = F_n [erg/s/cm^2] (beam) or I [erg/s/cm^2/sr]
     * (isotropic).  slab_nmu: mu bins of the emergent-intensity tally at the
     * z faces (mochii_slab_imu) */
    int xy_periodic, source_slab, slab_faces, slab_nmu;
    int slab_mode[2];
    double slab_theta[2], slab_phi[2], slab_source[2];
    /* tabulated spectra (define.f90:276-303): ion_spectrum (the primary
     * source), src_spectrum_file (column i for point source i),
     * ext_spectrum (the external field's J: a file, or the ISRF preset
     * 'draine', 'habing' or 'mathis' scaled by ext_scale); spectrum_type
     * the column units of every file: 0 'shape_ev' (E [eV], any scale),
     * 1 'per_ev', 2 'per_hz', 3 'per_ang', 4 'per_um' (absolute densities
     * per eV, Hz, Angstrom, micron) */
    char ion_spectrum[MOCHII_STRLEN], src_spectrum_file[MOCHII_STRLEN], ext_spectrum[MOCHII_STRLEN];
    int spectrum_type;
    double ext_scale;
} mochii_params;

/* Per-pass statistics (ion_score_report_energy_closure, ion_score_mod.f90:364-387). */
typedef struct mochii_pass_stats {
    double energy_emitted, energy_absorbed, energy_escaped, closure;
    int64_t direct_segments, scattered_segments;
    int64_t packets;
    double kernel_ms;                /* device time of the transport kernel   */
    double pass_ms;                  /* device time of the whole pass         */
    int64_t walk_kills;              /* MAX_WALK_STEPS guard hits             */
    int64_t diffuse_packets;         /* diffuse_nphot of this pass            */
    double diffuse_lum;              /* diffuse_lum [erg/s]                   */
    int64_t metal_active;            /* sum over scored segments of the packet's active metal transitions */
} mochii_pass_stats;

/* Convergence measures (gas_thermal_update / gas_equilibrium_update outputs). */
typedef struct mochii_metrics {
    double max_dx, max_dte, dx_vol, dte_vol;
    int64_t cells_solved;
    int64_t fixed_point_cap_hits;    /* cells whose n_e loop used all 200 passes */
    double kernel_ms;
    int64_t fixed_point_passes;      /* n_e fixed-point passes over all cells and trial T */
    int64_t metal_sum_calls;         /* metal cascade sums (species_metal_sums) evaluated */
    int64_t rate_evaluations;        /* net_rate evaluations (thermal) or cell solves      */
    int64_t warm_accepted;           /* leaves whose learned warm start passed the residual
                                        gate at its one evaluation (mochii_mlp_warm_start)  */
} mochii_metrics;

/* Launch shapes of the transport walk (the autotuner's choice). */
typedef struct mochii_tuning {
    int lookahead;           /* cells the DDA stepper runs ahead of the scoring, 0..2 */
    int walk_blocks_per_sm;  /* persistent walk grid: SMs x this, 128-thread blocks  */
    double best_ms;          /* device time of the winning trial pass (autotune)     */
    int lane_threads;        /* per-lane thermal solve: leaves (lanes) per block, a
                                multiple of 32; 0 = as many as the rate cache fits   */
    double thermal_ms;       /* device time of the winning trial thermal update      */
} mochii_tuning;

typedef struct mochii_ctx mochii_ctx;

/* ---- parameters: read_input, setup.f90:11-35 ----------------------------- */
/* Fill *p with the define.f90 defaults. */
int mochii_params_default(mochii_params* p);
/* sizeof(mochii_params), for FFI bindings that mirror the struct. */
size_t mochii_params_size(void);
/* Set one key (the name after "par%", case-insensitive, optional "(i)"
 * index) from its namelist text value.  Unknown keys are an error. */
int mochii_params_set(mochii_params* p, const char* key, const char* value);
/* Parse a namelist text "&parameters par%key = value ... /" into *p,
 * starting from its current contents.  errbuf receives a message. */
int mochii_params_parse_namelist(mochii_params* p, const char* text, char* errbuf, size_t errlen);
/* Read a namelist file (read_input, setup.f90:33-35). */
int mochii_params_read_namelist(mochii_params* p, const char* path, char* errbuf, size_t errlen);

/* ---- context: grid_create_amr + ion_setup + gas_state_setup ---------------- */
/* Builds the grid (grid_mod_amr.f90:27-350), the band and source samplers
 * (ion_band_mod.f90:122-258), the leaf state (gas_state_mod.f90:41-90) and
 * uploads everything to device memory on the current device. */
int mochii_init(const mochii_params* p, mochii_ctx** out);
void mochii_destroy(mochii_ctx* ctx);
const char* mochii_strerror(int status);
/* Message of the last failed call on ctx (or of the last failed
 * mochii_init on this thread when ctx is NULL). */
const char* mochii_last_error(const mochii_ctx* ctx);

/* ---- the replaced entry points ------------------------------------------------- */
/* ionizing_field_and_rates (ionizing_field_mod.f90:72-170): one transport
 * pass of every stellar packet through the current opacity, the energy
 * ledger, and the rate normalisation (gas_rates_compute).  with_peel = 1 is
 * the imaging pass (below; needs par%ion_peel). */
int mochii_transport_pass(mochii_ctx* ctx, int with_peel, mochii_pass_stats* stats);
/* gas_equilibrium_update (solve_te = 0) or gas_thermal_update (solve_te = 1). */
int mochii_balance_update(mochii_ctx* ctx, int solve_te, mochii_metrics* m);
/* The imaging pass (main.f90:234-235, ionizing_field_and_rates with
 * with_peel): mochii_transport_pass(ctx, 1, st) needs par%ion_peel at
 * mochii_init; it is a full pass that also peels every stellar and diffuse
 * packet toward each observer at emission (ion_peel_direct,
 * ion_peel_mod.f90:225-277) and, with dust scattering, at every interaction
 * (ion_peel_scatter, :284-344), the optical depth to the box edge by the
 * tau-only walks (raytrace_amr.f90:678-775).  The images (nobs, nchan,
 * nyim, nxim; channels ionizing/FUV, or one per band bin with peel_bins)
 * hold erg/s per code length^2 per pixel: which = 0 direct, 1 scattered,
 * 2 unattenuated direct (save_direc0). */
int mochii_image_shape(const mochii_ctx* ctx, int* shape4);
int mochii_get_image(mochii_ctx* ctx, int which, double* out, int64_t n);
/* Observer k as ion_peel_setup derived it: x, y, z (code units), alpha,
 * beta, gamma [deg], distance, dxim, dyim [deg], then the grid -> observer
 * rotation matrix row by row (18 doubles). */
int mochii_image_observer(const mochii_ctx* ctx, int k, double* out18);
/* ion_peel_write (ion_peel_mod.f90:359-523): surface brightness images
 * [erg/s/cm^2/sr] as <base>_image/ with one .npy per block (direct_ion,
 * scatt_ion, direct_fuv ..., direc0_*, suffix _obs<k> with several
 * observers; with peel_bins the cubes and E_bin, dE_bin, wl_bin) and
 * header.json (DXIM, DIST, ALPHA, BETA, GAMMA per block). */
int mochii_write_image(mochii_ctx* ctx, const char* base);

/* The equilibrium dust temperature (dust_temp_mod.f90, par%ion_add_dust):
 * mochii_get_field(ctx, "T_dust", ...) solves Heat_dust = (rhokap / d_cm)
 * femit(T) per leaf from the last pass's grain heating (femit = 4 pi Int
 * s_abs B_nu dnu over the extinction table the transport uses), and the
 * rates file carries it as T_dust.  mochii_dust_ir: the grains' infrared
 * spectrum of it, lam[240] [um] from 1 to 1000 um, lnu[240] [erg/s/Hz] and
 * labs_lir[2] = the absorbed power sum Heat_dust V and the integral of L_nu
 * over frequency [erg/s] (dust_ir_write); mochii_write_dust_ir writes them
 * as <base>_dustir.txt. */
int mochii_dust_ir(mochii_ctx* ctx, double* lam, double* lnu, double* labs_lir);
int mochii_write_dust_ir(mochii_ctx* ctx, const char* base);

/* The plane-parallel slab's boundary tally of the last transport pass
 * (slab_Iesc, jtally_mod.f90:39-86; filled by the edge walks and the
 * scattered flights, raytrace_amr.f90:407-481, 586-660): iesc[0, nmu) the
 * luminosity [erg/s] leaving the top face (+z) per bin of mu = |k_z|,
 * iesc[nmu, 2 nmu) the bottom face, n = 2 par%slab_nmu; meta[0] L_in (the
 * entering ionizing luminosity of one tile), meta[1] A_zface [cm^2].
 * MOCHII_ERR_BAD_PARAM without source_geometry 'slab'.
 * mochii_write_slab_imu: slab_write_Imu (jtally_mod.f90:103-150), the
 * budget (escaping, absorbed, reflected / transmitted with one lit face)
 * and I(mu) = Iesc / (A_zface 2 pi mu dmu) of both faces as the text file
 * <base>_slab_Imu.txt. */
int mochii_slab_tally(mochii_ctx* ctx, double* iesc, int n, double* meta);
int mochii_write_slab_imu(mochii_ctx* ctx, const char* base);

/* amr_refine_front (amr_refine_mod.f90:46-186): the octree rebuilt on the
 * current solution.  Front leaves: gas leaves with refine_eps < x_HI <
 * 1 - refine_eps, or whose face-neighbour gas leaf differs in x_HI by more
 * than refine_dx; the new tree is level refine_lmax where a cell overlaps a
 * front leaf and refine_lbase elsewhere; nH, n_e and rhokap are remapped by
 * overlap volume, the ion fractions by nH V, T_e by (nH (1 + He/H) + n_e) V,
 * and the seven conserved box integrals (H nuclei, H I, He I, He II,
 * electrons, extinction, thermal content) must agree to 1e-8.  Every
 * leaf-indexed buffer changes size, so the result is a NEW context:
 * mochii_refine_front plans on the device (front flags, the new tree level
 * by level in depth-first order, the remap), writes the new leaf list to
 * out_list when it is a non-empty path (the generic text format, with the
 * remapped x_HI, x_HeI, x_HeII, n_e, T_e and rhokap as extra columns),
 * initialises *out from the new leaves in memory with ctx's parameters and
 * sets the remapped state; ctx is left as it was (destroy it when done).
 * The grains' rhokap of the new context follows from the remapped nH as
 * at any set-up (the same volume remap for the supported dust laws).
 * mochii_refine_plan is the host part alone (no device): the old leaf
 * list, its state (rhokap may be NULL), and the new leaf list out;
 * counts2 = new leaf count and front leaves, *worst = the largest relative
 * change of a conserved integral; mochii_refine_last_error explains a
 * failure of either. */
int mochii_refine_plan(const char* in_list, const double* nH, const double* xHI, const double* xHeI,
                       const double* xHeII, const double* ne, const double* Te, const double* rhokap,
                       double He_abund, double te_min, int lbase, int lmax, double eps, double dx,
                       const char* out_list, int64_t* counts2, double* worst);
int mochii_refine_front(mochii_ctx* ctx, const char* out_list, mochii_ctx** out);
const char* mochii_refine_last_error(void);

/* gas_opacity_fill: refresh the per-leaf absorber columns the transport reads. */
int mochii_opacity_fill(mochii_ctx* ctx);

/* ---- the rates file: gas_rates_write (gas_rates_mod.f90:216-366) -------------- */
/* The run's convergence record, written as the file's header keywords
 * (CONVERGD, NITERDON, FINALDX, FINALDTE, FLDCONS; main.f90:188-225). */
typedef struct mochii_run_info {
    int converged;          /* the gas iteration met its convergence test        */
    int iterations;         /* gas iterations run                                 */
    double final_dx;        /* final max|delta x_HII|                             */
    double final_dte;       /* final max|delta T_e|/T_e                           */
    int field_consistent;   /* the rates come from a pass through the written state */
} mochii_run_info;
/* Write the rates and state of the current iterate as the reference's rates
 * file does (gas_rates_write, with species_write for the metals): the same
 * dataset names (Gamma_HI ... Heat_HeII, Heat_dust with grains, J_nu, x_HI,
 * x_HeI, x_HeII, n_e, T_e, E_bin, dE_bin, LeafXYZ, LeafSize,
 * x_<el>_stages, Gamma_<el>_stages, Heat_<el>_stages) and header keywords,
 * in a format that needs no I/O library: directory <base>_rates/ with one
 * .npy file per dataset (FP64, C order; the reference's Fortran array
 * a(n1, n2) is shape (n2, n1), the same bytes) and header.json (keywords,
 * and per dataset its file, shape and comment).  The energy ledger keywords
 * are those of the last transport pass; run may be NULL (not converged,
 * zero iterations). */
int mochii_write_rates(mochii_ctx* ctx, const char* base, const mochii_run_info* run);

/* ---- batched nebulae (no reference counterpart: one job is one nebula) ------ */
/* Several contexts on the current device advanced together.  One iteration of
 * every nebula -- its transport pass (as mochii_transport_pass), then its
 * balance (as mochii_balance_update with solve_te; with metals and the
 * bracketed solver all nebulae's thermal solves run in ONE persistent launch
 * that claims 32-leaf chunks of every nebula from one counter) -- is recorded
 * as one CUDA graph at the first mochii_batch_iterate and replayed after.
 * The contexts must not use the diffuse field (its packet count is read back
 * mid-pass), the slab (its boundary tally is read back after each standalone
 * pass) or the MLP warm start; their own calls stay usable between
 * iterations, but changing a context's parameters or tuning (mochii_set_nphotons,
 * mochii_set_tuning, mochii_autotune, a first T_warm or MLP warm start) needs
 * a new batch: mochii_batch_iterate refuses with MOCHII_ERR_BAD_PARAM before
 * any launch when a context changed after mochii_batch_create. */
typedef struct mochii_batch mochii_batch;
int mochii_batch_create(mochii_ctx* const* ctxs, int n, mochii_batch** out);
/* stats[n], m[n] receive each nebula's pass statistics and balance metrics;
 * *device_ms the device time of the whole iteration (may be NULL). */
int mochii_batch_iterate(mochii_batch* b, int solve_te, mochii_pass_stats* stats, mochii_metrics* m,
                         double* device_ms);
void mochii_batch_destroy(mochii_batch* b);

/* ---- autotuner: packet-block, look-ahead and cell-tile shapes ----------- */
/* Time trial transport passes of sample_packets packets on the current
 * state for every walk variant and keep the fastest; with the per-lane
 * thermal solve also trial thermal updates from a saved copy of the state
 * for several lanes per block (the cell tile), the state restored after.
 * The choice is cached per (grid shape, precision, absorber set, device)
 * for the process.  The trial passes overwrite the tallies and rates, so
 * call it before a pass. */
int mochii_autotune(mochii_ctx* ctx, int64_t sample_packets, mochii_tuning* out);
int mochii_set_tuning(mochii_ctx* ctx, const mochii_tuning* t);
int mochii_get_tuning(const mochii_ctx* ctx, mochii_tuning* out);

/* ---- state exchange (host buffers; sizes in elements) ---------------------- */
int64_t mochii_nleaf(const mochii_ctx* ctx);
/* Metal registry shape: transitions and stages over all active elements
 * (species_mod.f90 n_elements / elem_nstage); both 0 without metals. */
int mochii_metal_shape(const mochii_ctx* ctx, int* ntransitions, int* nstages);
int mochii_nnu_band(const mochii_ctx* ctx);
/* mochii_set_field also takes "T_warm" (nleaf): a warm-start T_e per leaf
 * for the next bracketed thermal solve (par thermal_solver = 'bracketed'),
 * used once; without it the solve starts from the current T_e.
 * Field names: "nH" "x_HI" "x_HeI" "x_HeII" "n_e" "T_e" "gamma_HI"
 * "gamma_HeI" "gamma_HeII" "heat_HI" "heat_HeI" "heat_HeII" (nleaf each),
 * "jt_ion" (nleaf*nnu_band, leaf-major), "eedge" (nnu_band+1),
 * "leaf_half" (nleaf); with par%use_metals also "gamma_metal" and
 * "heat_metal" (nleaf*ntransitions: Gamma_<el>_stages / Heat_<el>_stages
 * of species_write) and "x_metal" (nleaf*nstages: x_<el>_stages), each
 * leaf-major with elements in registry order (c n o ne s ar mg fe si cl ca,
 * those with a positive abundance) and stages ascending. */
int mochii_get_field(mochii_ctx* ctx, const char* name, double* out, int64_t n);
/* Upload a state field ("x_HI" "x_HeI" "x_HeII" "n_e" "T_e" "nH"). */
int mochii_set_field(mochii_ctx* ctx, const char* name, const double* in, int64_t n);
/* Launch-set size of later passes (par%nphotons). */
int mochii_set_nphotons(mochii_ctx* ctx, int64_t nphotons);
double mochii_ion_Ltot(const mochii_ctx* ctx);

/* ---- test hooks (bit-exact fixtures) -------------------------------------------- */
/* Owen-scrambled Sobol uniforms computed on the device
 * (qmc_uniforms_stream, qmc_mod.f90:157-168): out[i*nd + d] for the 0-based
 * indices idx0 .. idx0+n-1, stream 1 (stellar) or 2 (diffuse), nd <= 12. */
int mochii_sobol_uniforms(int seed, int stream, int64_t idx0, int64_t n, int nd, double* out);
/* The scattered flights' random numbers computed on the device: draws
 * n0 .. n0+n-1 of the Philox4x32-10 stream of one packet (key par%iseed and
 * stream 0 stellar / 1 diffuse, counter = the packet index).  No reference
 * counterpart: the reference draws these from a per-rank MT19937
 * (random.f90 rand_number, used at raytrace_amr.f90:268-320). */
int mochii_philox_uniforms(int64_t seed, int stream, int64_t packet, int n0, int n, double* out);
/* Geometry-only cell walk of nray rays (x,y,z,kx,ky,kz each, code units)
 * on ctx's grid (raytrace_ion_to_edge_car, raytrace_amr.f90:534-592, with
 * no optical-depth cut): leaves[r*max_steps + s] (0-based leaf index, -1
 * past the last step) and nsteps[r]. */
int mochii_walk_leaves(mochii_ctx* ctx, int64_t nray, const double* rays, int max_steps,
                       int32_t* leaves, int32_t* nsteps);
/* Launch records of packets ip0..ip0+n-1: x,y,z,kx,ky,kz,E,inu (8 doubles
 * each), as gen_ion_photon_qmc (ion_band_mod.f90:1880-1935) makes them. */
int mochii_launch_records(mochii_ctx* ctx, int64_t ip0, int64_t n, double* out8);

/* Diffuse field of the current state (diffuse_build, diffuse_mod.f90:60-121)
 * and the launch of diffuse packets ip0..ip0+n-1 (gen_diffuse_photon_qmc,
 * diffuse_mod.f90:221-296): out8 per packet = start cell (ix, iy, iz), the
 * DDA tMax (x, y, z), sigma_HI [1e-18 cm^2] and the diagnostic bin; *lum =
 * diffuse_lum [erg/s], *nphot = diffuse_nphot. */
int mochii_diffuse_records(mochii_ctx* ctx, int64_t ip0, int64_t n, double* out8, double* lum, int64_t* nphot);

/* Same records as mochii_launch_records, for callers that cannot allocate
 * device memory at call time (their device memory belongs to another
 * allocator such as a PyTorch caching allocator or a host pool, or an MPS
 * limit makes cudaMalloc fail).  No counterpart in the reference: it is a
 * staging variant of this library's own hook.  Allocates nothing: the
 * records are staged in a static device array of the library (4 MiB, held
 * by every GPU that loads the library until exit).  n <= 65536 records per
 * call, larger n is refused with MOCHII_ERR_BAD_PARAM.  The first call on a
 * device looks up that array's device address (make it before any stream
 * capture).  The context's device must be the current device (else
 * MOCHII_ERR_BAD_PARAM).  Calls share the array: calls that overlap on the
 * GPU race. */
int mochii_launch_records_noalloc(mochii_ctx* ctx, int64_t ip0, int64_t n, double* out8);

/* ---- learned warm start of the thermal balance (no reference counterpart:
 * the warm start is this library's addition) -------------------------------
 * A 4-layer MLP, 16 -> 128 -> 128 -> 128 -> 4 with GELU, BF16 tensor-core
 * GEMMs with FP32 accumulation and FP32 master weights, trained with Adam on
 * (features, solved state) pairs of the cell solver.  Features per leaf
 * (16 floats, 12 used): log Gamma_HI/HeI/HeII, log heating HI/HeI/HeII,
 * log n_H, dust-absorbed power, previous x_HII, x_HeII, x_HeIII, log T_e,
 * each scaled to order one (mochii_mlp_features).  Targets per leaf (4
 * floats): x_HII, x_HeII, x_HeIII and the change of T_e over the iteration,
 * 4 (log10 T_e - log10 T_e,prev), with T_e,prev = 10^(4 + feature_11/4). */
typedef struct mochii_mlp mochii_mlp;
int mochii_mlp_create(uint64_t seed, mochii_mlp** out);
void mochii_mlp_destroy(mochii_mlp* m);
const char* mochii_mlp_last_error(const mochii_mlp* m);
int64_t mochii_mlp_num_params(void);
/* parameters in layer order: W (out x in, row-major) then b of each layer */
int mochii_mlp_get_params(mochii_mlp* m, float* out);
int mochii_mlp_set_params(mochii_mlp* m, const float* in);
/* loss gradient over one batch of n rows, parameter layout; no update */
int mochii_mlp_gradients(mochii_mlp* m, const float* X, const float* Y, int64_t n, float* grads, float* loss);
/* epochs of shuffled mini-batches with Adam; losses[epochs] = mean batch loss */
int mochii_mlp_train(mochii_mlp* m, const float* X, const float* Y, int64_t n, int epochs, int batch, float lr,
                     uint64_t seed, float* losses);
/* out4 per row: x_HII, x_HeII, x_HeIII, T_e [K] */
int mochii_mlp_predict(mochii_mlp* m, const float* X, int64_t n, double* out4);
/* features of every leaf from the nebula's current rates and state (nleaf x 16) */
int mochii_mlp_features(mochii_ctx* ctx, float* out);
/* predicted T_e of every leaf as the warm start of the next bracketed
 * thermal solve (par thermal_solver = 'bracketed'), computed on the device;
 * the solve accepts a prediction whose net heating is below 1e-6 of heating
 * plus cooling after that one evaluation (counted in
 * mochii_metrics.warm_accepted), else brackets the root from it with a first
 * step of 2.5 RMS errors of the prediction: the RMS of ln(T_e / T_warm) that
 * the nebula's last learned warm start left (measured after that update), or
 * the network's training fit before the first.  "T_warm" reads the
 * predictions through mochii_get_field until the update consumes them. */
int mochii_mlp_warm_start(mochii_ctx* ctx, mochii_mlp* m);
/* The same warm start inside a batch's recorded iteration: each nebula's
 * inference runs after its pass and the batched thermal launch starts from
 * the predictions.  Needs the batched thermal solve (metals, the bracketed
 * solver, cell_layout 'lane' or 'lockstep'); m must outlive the batch, and
 * retraining m takes effect at the next iteration (the graph reads its
 * weights where they lie). */
int mochii_batch_set_warm_start(mochii_batch* b, mochii_mlp* m);

#ifdef __cplusplus
}
#endif
#endif /* MOCHII_GPU_H */
