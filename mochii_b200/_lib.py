"""ctypes binding of libmochii_gpu.so (the C ABI in include/mochii_gpu.h).

The library is built in-tree (mochii_b200/libmochii_gpu.so).  There is no
fallback implementation: if the shared library is missing the import fails
with an error that says how to build it.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmochii_gpu.so")

MAX_SRC = 16
MAX_OBS = 16
STRLEN = 256

OK = 0
STATUS = {0: "OK", 1: "BAD_PARAM", 2: "TABLE", 3: "CUDA", 4: "TIMEOUT", 5: "NONFINITE",
          6: "CLOSURE", 7: "NOT_CONVERGED", 8: "UNSUPPORTED", 9: "NO_DEVICE"}
PREC_FP64, PREC_FP32 = 0, 1


class Params(C.Structure):
    """Mirror of struct mochii_params (define.f90 params_type subset)."""
    _fields_ = [
        ("nphotons", C.c_int64), ("launch_sobol", C.c_int), ("qmc_seed", C.c_int),
        ("source_cdf_tol", C.c_double), ("luminosity", C.c_double), ("tstar", C.c_double),
        ("random_seed", C.c_int),
        ("nnu_ion", C.c_int), ("eion_min", C.c_double), ("eion_max", C.c_double),
        ("add_fuv", C.c_int), ("efuv_min", C.c_double), ("nnu_fuv", C.c_int), ("ion_align_edges", C.c_int),
        ("grid_car", C.c_int), ("car_walk_dda", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("rmax", C.c_double), ("rmin", C.c_double), ("nH_const", C.c_double),
        ("distance2cm", C.c_double), ("distance_unit", C.c_char * 16), ("amr_file", C.c_char * STRLEN),
        ("source_point", C.c_int), ("xs_point", C.c_double), ("ys_point", C.c_double), ("zs_point", C.c_double),
        ("nsource", C.c_int),
        ("src_tstar", C.c_double * MAX_SRC), ("src_lum", C.c_double * MAX_SRC),
        ("src_x", C.c_double * MAX_SRC), ("src_y", C.c_double * MAX_SRC), ("src_z", C.c_double * MAX_SRC),
        ("xHI_init", C.c_double), ("xHeI_init", C.c_double), ("xHeII_init", C.c_double),
        ("He_abund", C.c_double), ("gas_niter", C.c_int),
        ("gas_tol", C.c_double), ("te_fixed", C.c_double), ("ion_relax", C.c_double),
        ("caseA", C.c_int), ("recomb_hui_gnedin", C.c_int), ("ci_dere_hybrid", C.c_int), ("conv_vol", C.c_int),
        ("solve_te", C.c_int), ("te_min", C.c_double), ("te_max", C.c_double), ("gas_tol_te", C.c_double),
        ("require_convergence", C.c_int),
        ("use_metals", C.c_int),
        ("abund_C", C.c_double), ("abund_N", C.c_double), ("abund_O", C.c_double), ("abund_Ne", C.c_double),
        ("abund_S", C.c_double), ("abund_Ar", C.c_double), ("abund_Mg", C.c_double), ("abund_Fe", C.c_double),
        ("abund_Si", C.c_double), ("abund_Cl", C.c_double), ("abund_Ca", C.c_double),
        ("ion_metal_abs", C.c_int), ("metal_ne", C.c_int), ("metal_heat", C.c_int), ("metal_freefree", C.c_int),
        ("charge_exchange_two_way", C.c_int), ("cooling_local_ne", C.c_int), ("gaunt_vh14", C.c_int),
        ("diffuse_field", C.c_int), ("use_sec_ion", C.c_int), ("diffuse_model", C.c_int),
        ("ion_add_dust", C.c_int), ("ion_dust_scatter", C.c_int), ("dust_law", C.c_int),
        ("DGR", C.c_double), ("cext_dust", C.c_double), ("grain_pe", C.c_int),
        ("ion_dust_kext", C.c_char * STRLEN), ("data_dir", C.c_char * STRLEN), ("atomic_dir", C.c_char * STRLEN),
        ("precision", C.c_int),
        ("fe_levels_full", C.c_int), ("metal_moments", C.c_int), ("solver_bracketed", C.c_int),
        ("lambda_ref", C.c_double), ("taumax", C.c_double), ("tauhomo", C.c_double),
        ("solver_warp", C.c_int), ("tally64", C.c_int), ("metal_rate_table", C.c_int),
        ("packet_chunk", C.c_int64), ("packet_order", C.c_int),
        ("ion_peel", C.c_int), ("peel_bins", C.c_int), ("save_direc0", C.c_int), ("nxim", C.c_int),
        ("nyim", C.c_int), ("distance", C.c_double), ("dxim", C.c_double), ("dyim", C.c_double),
        ("alpha", C.c_double * MAX_OBS), ("beta", C.c_double * MAX_OBS), ("gamma", C.c_double * MAX_OBS),
        ("obsx", C.c_double * MAX_OBS), ("obsy", C.c_double * MAX_OBS), ("obsz", C.c_double * MAX_OBS),
        ("phase_angle", C.c_double * MAX_OBS), ("inclination_angle", C.c_double * MAX_OBS),
        ("position_angle", C.c_double * MAX_OBS),
        ("hei_diffuse", C.c_int),
        ("refine_front", C.c_int), ("refine_iter", C.c_int), ("refine_lbase", C.c_int), ("refine_lmax", C.c_int),
        ("refine_eps", C.c_double), ("refine_dx", C.c_double),
        ("ext_intensity", C.c_double), ("ext_tstar", C.c_double), ("ext_geometry", C.c_int),
        ("source_external", C.c_int), ("ext_spectrum_set", C.c_int),
        ("xy_periodic", C.c_int), ("source_slab", C.c_int), ("slab_faces", C.c_int), ("slab_nmu", C.c_int),
        ("slab_mode", C.c_int * 2), ("slab_theta", C.c_double * 2), ("slab_phi", C.c_double * 2),
        ("slab_source", C.c_double * 2),
        ("ion_spectrum", C.c_char * STRLEN), ("src_spectrum_file", C.c_char * STRLEN),
        ("ext_spectrum", C.c_char * STRLEN), ("spectrum_type", C.c_int), ("ext_scale", C.c_double),
    ]


class PassStats(C.Structure):
    _fields_ = [("energy_emitted", C.c_double), ("energy_absorbed", C.c_double), ("energy_escaped", C.c_double),
                ("closure", C.c_double), ("direct_segments", C.c_int64), ("scattered_segments", C.c_int64),
                ("packets", C.c_int64), ("kernel_ms", C.c_double), ("pass_ms", C.c_double),
                ("walk_kills", C.c_int64), ("diffuse_packets", C.c_int64), ("diffuse_lum", C.c_double),
                ("metal_active", C.c_int64)]


class Metrics(C.Structure):
    _fields_ = [("max_dx", C.c_double), ("max_dte", C.c_double), ("dx_vol", C.c_double), ("dte_vol", C.c_double),
                ("cells_solved", C.c_int64), ("fixed_point_cap_hits", C.c_int64), ("kernel_ms", C.c_double),
                ("fixed_point_passes", C.c_int64), ("metal_sum_calls", C.c_int64), ("rate_evaluations", C.c_int64),
                ("warm_accepted", C.c_int64)]


class RunInfo(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("final_dx", C.c_double), ("final_dte", C.c_double),
                ("field_consistent", C.c_int)]


class Tuning(C.Structure):
    _fields_ = [("lookahead", C.c_int), ("walk_blocks_per_sm", C.c_int), ("best_ms", C.c_double),
                ("lane_threads", C.c_int), ("thermal_ms", C.c_double)]


# Every symbol the header declares, with its ctypes signature.
_P = C.POINTER
SIGNATURES = {
    "mochii_params_default": (C.c_int, [_P(Params)]),
    "mochii_params_size": (C.c_size_t, []),
    "mochii_params_set": (C.c_int, [_P(Params), C.c_char_p, C.c_char_p]),
    "mochii_params_parse_namelist": (C.c_int, [_P(Params), C.c_char_p, C.c_char_p, C.c_size_t]),
    "mochii_params_read_namelist": (C.c_int, [_P(Params), C.c_char_p, C.c_char_p, C.c_size_t]),
    "mochii_init": (C.c_int, [_P(Params), _P(C.c_void_p)]),
    "mochii_destroy": (None, [C.c_void_p]),
    "mochii_strerror": (C.c_char_p, [C.c_int]),
    "mochii_last_error": (C.c_char_p, [C.c_void_p]),
    "mochii_transport_pass": (C.c_int, [C.c_void_p, C.c_int, _P(PassStats)]),
    "mochii_balance_update": (C.c_int, [C.c_void_p, C.c_int, _P(Metrics)]),
    "mochii_opacity_fill": (C.c_int, [C.c_void_p]),
    "mochii_mlp_create": (C.c_int, [C.c_uint64, _P(C.c_void_p)]),
    "mochii_mlp_destroy": (None, [C.c_void_p]),
    "mochii_mlp_last_error": (C.c_char_p, [C.c_void_p]),
    "mochii_mlp_num_params": (C.c_int64, []),
    "mochii_mlp_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mochii_mlp_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mochii_mlp_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, _P(C.c_float)]),
    "mochii_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_float,
                                   C.c_uint64, C.c_void_p]),
    "mochii_mlp_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "mochii_mlp_features": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mochii_mlp_warm_start": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mochii_nleaf": (C.c_int64, [C.c_void_p]),
    "mochii_metal_shape": (C.c_int, [C.c_void_p, _P(C.c_int), _P(C.c_int)]),
    "mochii_nnu_band": (C.c_int, [C.c_void_p]),
    "mochii_get_field": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int64]),
    "mochii_write_rates": (C.c_int, [C.c_void_p, C.c_char_p, _P(RunInfo)]),
    "mochii_image_shape": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mochii_get_image": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]),
    "mochii_image_observer": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mochii_write_image": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mochii_dust_ir": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mochii_write_dust_ir": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mochii_slab_tally": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "mochii_write_slab_imu": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mochii_refine_plan": (C.c_int, [C.c_char_p] + [C.c_void_p] * 7 + [C.c_double, C.c_double, C.c_int, C.c_int,
                                                                       C.c_double, C.c_double, C.c_char_p,
                                                                       C.c_void_p, C.c_void_p]),
    "mochii_refine_front": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p]),
    "mochii_refine_last_error": (C.c_char_p, []),
    "mochii_set_field": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int64]),
    "mochii_set_nphotons": (C.c_int, [C.c_void_p, C.c_int64]),
    "mochii_ion_Ltot": (C.c_double, [C.c_void_p]),
    "mochii_sobol_uniforms": (C.c_int, [C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int, C.c_void_p]),
    "mochii_philox_uniforms": (C.c_int, [C.c_int64, C.c_int, C.c_int64, C.c_int, C.c_int, C.c_void_p]),
    "mochii_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mochii_batch_set_warm_start": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mochii_batch_iterate": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mochii_batch_destroy": (None, [C.c_void_p]),
    "mochii_walk_leaves": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mochii_launch_records": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p]),
    "mochii_autotune": (C.c_int, [C.c_void_p, C.c_int64, _P(Tuning)]),
    "mochii_launch_records_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p]),
    "mochii_diffuse_records": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, _P(C.c_double), _P(C.c_int64)]),
    "mochii_set_tuning": (C.c_int, [C.c_void_p, _P(Tuning)]),
    "mochii_get_tuning": (C.c_int, [C.c_void_p, _P(Tuning)]),
}

_lib = None


def load():
    """Load libmochii_gpu.so (no fallback: raise if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mochii_b200.build` "
                          "(this package has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.mochii_params_size() != C.sizeof(Params):
        raise ImportError("mochii_params layout mismatch between include/mochii_gpu.h and the ctypes mirror")
    _lib = lib
    return lib


class MochiiError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status
