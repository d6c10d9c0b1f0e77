"""ctypes wrapper of the oracle library (TEST INFRASTRUCTURE ONLY).

Imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
as the checker; the product package never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")
_lib = None


def build(force=False):
    srcs = [os.path.join(HERE, f) for f in ("orc_core.cpp", "orc_thermal.cpp", "orc_capi.cpp", "orc_core.h",
                                          "orc_thermal.h", "Makefile")]
    if force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = C.CDLL(LIB)
    V, D, I, LL = C.c_void_p, C.c_double, C.c_int, C.c_longlong
    sig = {
        "orc_qmc_uniforms": (I, [I, I, LL, LL, I, V]),
        "orc_qmc_raw_codes": (I, [LL, LL, I, V]),
        "orc_qmc_keys": (None, [I, V]),
        "orc_sampler_planck": (V, [D, D, D, D, V, I]),
        "orc_sampler_tab": (V, [V, V, I]),
        "orc_sampler_tab_band": (V, [V, V, I, D, D]),
        "orc_sampler_size": (I, [V]),
        "orc_sampler_total": (D, [V]),
        "orc_sampler_get": (None, [V, V, V, V]),
        "orc_sampler_sample": (None, [V, V, LL, V]),
        "orc_sampler_cdf": (None, [V, V, LL, V]),
        "orc_sampler_free": (None, [V]),
        "orc_eval": (I, [C.c_char_p, I, V, LL, V]),
        "orc_band_edges": (I, [C.c_char_p, V, I]),
        "orc_sim_new": (V, [C.c_char_p, I, C.c_char_p, I]),
        "orc_sim_free": (None, [V]),
        "orc_sim_nleaf": (I, [V]),
        "orc_sim_nnu": (I, [V]),
        "orc_sim_ion_Ltot": (D, [V]),
        "orc_sim_set_nphotons": (None, [V, LL]),
        "orc_sim_transport_pass": (I, [V]),
        "orc_sim_equilibrium_update": (I, [V, V]),
        "orc_sim_energy": (None, [V, V, V]),
        "orc_sim_slab": (I, [V, V, I]),
        "orc_philox": (None, [C.c_ulonglong, C.c_uint, C.c_ulonglong, C.c_uint, I, V]),
        "orc_sim_dust_optics": (I, [V, LL, V, V]),
        "orc_philox_block": (None, [V, V, V]),
        "orc_sim_get": (LL, [V, C.c_char_p, V, LL]),
        "orc_sim_set": (LL, [V, C.c_char_p, V, LL]),
        "orc_sim_photon": (None, [V, LL, V]),
        "orc_sim_walk_leaves": (I, [V, LL, V, I, V, V]),
        "orc_solve_ion_cell": (None, [I, D, D, D, D, D, D, I, V, V]),
        "orc_last_error": (C.c_char_p, []),
        "orc_sim_thermal_update": (I, [V, V]),
        "orc_sim_metal_ntr": (I, [V]),
        "orc_sim_metal_nel": (I, [V]),
        "orc_sim_metal_el": (I, [V, I, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "orc_sim_metal_eth": (D, [V, I, I]),
        "orc_sim_metal_cx": (None, [V, I, I, D, V]),
        "orc_sim_metal_sums": (None, [V, D, D, D, D, D, V]),
        "orc_sim_metal_fractions": (None, [V, I, D, D, D, D, V]),
        "orc_sim_solve_cell": (None, [V, D, D, D, D, D, I, V]),
        "orc_sim_metal_thermal": (I, [V, I, D, D, D, D, V]),
        "orc_sim_net_rate": (I, [V, I, D, V]),
        "orc_sim_thermal_sample": (LL, [V, LL]),
        "orc_sim_metal_nstage": (I, [V]),
        "orc_gff_table": (None, [V, V]),
        "orc_cooling_total": (D, [V, D, D, D, D, D, D]),
        "orc_nlevel_cooling_at": (D, [C.c_char_p, D, D]),
        "orc_sim_diffuse_build": (D, [V, V]),
        "orc_sim_diffuse_photon": (None, [V, LL, V]),
        "orc_milne_sample": (D, [V, I, D, D]),
        "orc_sim_thermal_cells": (LL, [V, V, LL, V]),
        "orc_sim_diffuse_count": (LL, [V]),
        "orc_sim_defer_fill": (None, [V, I]),
        "orc_sim_transport_pass_peel": (I, [V]),
        "orc_sim_peel_image": (LL, [V, I, V, LL, V]),
        "orc_sim_peel_observer": (I, [V, I, V]),
        "orc_thermal_1d": (I, [C.c_char_p, V, I, I, V]),
        "orc_hei_2ph": (I, [C.c_char_p, D, V, LL, V, V]),
        "orc_sim_dust_temp": (I, [V, V, V, V]),
        "orc_refine_plan": (I, [C.c_char_p, V, V, D, D, I, I, D, D, C.c_char_p, V, V]),
        "orc_hei_branch_energies": (I, [C.c_char_p, D, D, D, V]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def qmc_uniforms(seed, stream, idx0, n, nd):
    lib = load()
    out = np.zeros((n, nd))
    assert lib.orc_qmc_uniforms(seed, stream, idx0, n, nd, out.ctypes.data) == 0
    return out


def qmc_raw_codes(idx0, n, nd):
    lib = load()
    out = np.zeros((n, nd), dtype=np.uint32)
    assert lib.orc_qmc_raw_codes(idx0, n, nd, out.ctypes.data) == 0
    return out


class Sampler:
    def __init__(self, handle):
        if not handle:
            raise RuntimeError(load().orc_last_error().decode())
        self.h = handle

    @classmethod
    def planck(cls, T, emin, emax, rtol, thresholds):
        thr = np.ascontiguousarray(thresholds, dtype=float)
        return cls(load().orc_sampler_planck(T, emin, emax, rtol, thr.ctypes.data, thr.size))

    @classmethod
    def tabulated(cls, e, f):
        e = np.ascontiguousarray(e, dtype=float)
        f = np.ascontiguousarray(f, dtype=float)
        return cls(load().orc_sampler_tab(e.ctypes.data, f.ctypes.data, e.size))

    @classmethod
    def tabulated_band(cls, e, f, emin, emax):
        e = np.ascontiguousarray(e, dtype=float)
        f = np.ascontiguousarray(f, dtype=float)
        return cls(load().orc_sampler_tab_band(e.ctypes.data, f.ctypes.data, e.size, emin, emax))

    @property
    def total(self):
        return load().orc_sampler_total(self.h)

    def tables(self):
        n = load().orc_sampler_size(self.h)
        e, f, c = np.zeros(n), np.zeros(n), np.zeros(n)
        load().orc_sampler_get(self.h, e.ctypes.data, f.ctypes.data, c.ctypes.data)
        return e, f, c

    def sample(self, u):
        u = np.ascontiguousarray(u, dtype=float)
        out = np.zeros_like(u)
        load().orc_sampler_sample(self.h, u.ctypes.data, u.size, out.ctypes.data)
        return out

    def cdf(self, e):
        e = np.ascontiguousarray(e, dtype=float)
        out = np.zeros_like(e)
        load().orc_sampler_cdf(self.h, e.ctypes.data, e.size, out.ctypes.data)
        return out

    def __del__(self):
        try:
            load().orc_sampler_free(self.h)
        except Exception:
            pass


def evaluate(name, x, model=0):
    x = np.ascontiguousarray(x, dtype=float)
    out = np.zeros_like(x)
    assert load().orc_eval(name.encode(), model, x.ctypes.data, x.size, out.ctypes.data) == 0, name
    return out


def gff_table():
    logT = np.zeros(41)
    z = np.zeros((41, 4))
    load().orc_gff_table(logT.ctypes.data, z.ctypes.data)
    return logT, z


def band_edges(namelist):
    out = np.zeros(512)
    n = load().orc_band_edges(namelist.encode(), out.ctypes.data, 512)
    assert n > 0, load().orc_last_error()
    return out[:n]


def solve_ion_cell(gH, gHe1, gHe2, nH, T, caseA, x3, yHe=0.1, model=0):
    x = np.array(x3, dtype=float)
    ne = C.c_double()
    load().orc_solve_ion_cell(model, yHe, gH, gHe1, gHe2, nH, T, int(caseA), x.ctypes.data, C.byref(ne))
    return x, ne.value



def hei_2ph(path, u, eion_max=100.0):
    """The He I two-photon table (hei_twophoton_mod.f90): (photons per decay,
    in-band energy per decay [eV], sampled energies of the uniforms u)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    E = np.zeros_like(u)
    out = np.zeros(2)
    if load().orc_hei_2ph(str(path).encode(), float(eion_max), u.ctypes.data, u.size, E.ctypes.data, out.ctypes.data):
        raise RuntimeError(load().orc_last_error().decode())
    return out[0], out[1], E


def hei_branch_energies(path, T, xHI, xHeI):
    """diffuse_mod.f90 hei_branch_energies: (e3s, e1p, e1s) in eV per case-B
    He II recombination."""
    out = np.zeros(3)
    if load().orc_hei_branch_energies(str(path).encode(), float(T), float(xHI), float(xHeI), out.ctypes.data):
        raise RuntimeError(load().orc_last_error().decode())
    return tuple(out)


def refine_plan(in_list, state, rhokap=None, yHe=0.1, te_min=1.0e3, lbase=5, lmax=7, eps=1.0e-2, dx=0.2,
                out_list="refined_oracle.txt"):
    """amr_refine_front restated: (new leaves, front leaves, worst relative
    change of a conserved integral); the new list goes to out_list."""
    st = np.ascontiguousarray(np.stack([state[k] for k in ("nH", "x_HI", "x_HeI", "x_HeII", "n_e", "T_e")]),
                              dtype=np.float64)
    rk = None if rhokap is None else np.ascontiguousarray(rhokap, dtype=np.float64)
    counts = np.zeros(2, dtype=np.int64)
    worst = np.zeros(1)
    rc = load().orc_refine_plan(str(in_list).encode(), st.ctypes.data, None if rk is None else rk.ctypes.data,
                                float(yHe), float(te_min), int(lbase), int(lmax), float(eps), float(dx),
                                str(out_list).encode(), counts.ctypes.data, worst.ctypes.data)
    if rc:
        raise RuntimeError(f"orc_refine_plan: {rc} {load().orc_last_error().decode()}")
    return int(counts[0]), int(counts[1]), float(worst[0])


def thermal_1d(atomic_dir, nr=8000, nsweep=4, nnu=32, emin=13.598, emax=100.0, tstar=4.0e4,
               lband=3.177837e38, nH=100.0, yHe=0.1, rsph_pc=4.0, te_min=3.0e3, te_max=5.0e4):
    """The G2a gate's 1D thermal reference (check_g2a.py:150-207): radii [pc]
    and x_HI, x_HeI, x_HeII, T_e of nr shells of a uniform H/He sphere
    around a central blackbody."""
    cfg = np.array([nnu, emin, emax, tstar, lband, nH, yHe, rsph_pc, te_min, te_max], dtype=np.float64)
    out = np.zeros((5, nr))
    if load().orc_thermal_1d(str(atomic_dir).encode(), cfg.ctypes.data, int(nr), int(nsweep), out.ctypes.data):
        raise RuntimeError(load().orc_last_error().decode())
    return out


def philox(seed, stream, packet, n0, n):
    """Draws n0 .. n0+n-1 of one packet's scattering stream."""
    out = np.zeros(n)
    load().orc_philox(seed, stream, packet, n0, n, out.ctypes.data)
    return out

class Sim:
    """The oracle's nebula: the same namelist text the product reads."""

    def __init__(self, namelist, nthreads=None):
        lib = load()
        if nthreads is None:
            nthreads = os.cpu_count() or 1
        err = C.create_string_buffer(512)
        self.h = lib.orc_sim_new(namelist.encode(), int(nthreads), err, 512)
        if not self.h:
            raise RuntimeError("oracle setup failed: " + err.value.decode())
        self.nleaf = lib.orc_sim_nleaf(self.h)
        self.nnu = lib.orc_sim_nnu(self.h)
        self.nthreads = nthreads

    def transport_pass(self):
        load().orc_sim_transport_pass(self.h)

    def equilibrium_update(self):
        m = np.zeros(2)
        load().orc_sim_equilibrium_update(self.h, m.ctypes.data)
        return m[0], m[1]

    def set_nphotons(self, n):
        load().orc_sim_set_nphotons(self.h, int(n))

    def thermal_update(self):
        m = np.zeros(4)
        assert load().orc_sim_thermal_update(self.h, m.ctypes.data) == 0
        return tuple(m)

    def cooling_total(self, T, nH, ne, xHI, xHeI, xHeII):
        return load().orc_cooling_total(self.h, T, nH, ne, xHI, xHeI, xHeII)

    @property
    def ion_Ltot(self):
        return load().orc_sim_ion_Ltot(self.h)

    def dust_optics(self, E):
        E = np.ascontiguousarray(E, dtype=float)
        out = np.zeros((E.size, 3))
        assert load().orc_sim_dust_optics(self.h, E.size, E.ctypes.data, out.ctypes.data) == 0
        return out

    def slab_tally(self, nmu):
        """slab_Iesc of the last pass: (top face per mu bin, bottom face)."""
        out = np.zeros(2 * nmu)
        assert load().orc_sim_slab(self.h, out.ctypes.data, 2 * nmu) == 2 * nmu
        return out[:nmu], out[nmu:]

    def energy(self):
        e = np.zeros(3)
        s = np.zeros(2, dtype=np.int64)
        load().orc_sim_energy(self.h, e.ctypes.data, s.ctypes.data)
        return e, s

    # ---- metal registry probes (leaf 0) -----------------------------------
    def metal_elements(self):
        """[(name, Z, nstage)] in registry order."""
        lib = load()
        out = []
        for ie in range(lib.orc_sim_metal_nel(self.h)):
            nm = C.create_string_buffer(3)
            z, ns = C.c_int(), C.c_int()
            lib.orc_sim_metal_el(self.h, ie, nm, C.byref(z), C.byref(ns))
            out.append((nm.value.decode(), z.value, ns.value))
        return out

    def metal_eth(self, ie, it):
        return load().orc_sim_metal_eth(self.h, ie, it)

    def metal_cx(self, ie, it, T):
        o = np.zeros(2)
        load().orc_sim_metal_cx(self.h, ie, it, float(T), o.ctypes.data)
        return o[0], o[1]

    def metal_sums(self, T, nH, ne, nHI, nHII):
        o = np.zeros(3)
        load().orc_sim_metal_sums(self.h, float(T), float(nH), float(ne), float(nHI), float(nHII), o.ctypes.data)
        return tuple(o)

    def metal_fractions(self, ie, T, ne, nHI, nHII):
        o = np.zeros(8)
        load().orc_sim_metal_fractions(self.h, ie, float(T), float(ne), float(nHI), float(nHII), o.ctypes.data)
        return o[: self.metal_elements()[ie][2]]

    def solve_cell(self, gH, gHe1, gHe2, nH, T, caseA, xHI, xHeI, xHeII):
        st = np.array([xHI, xHeI, xHeII, 0.0])
        load().orc_sim_solve_cell(self.h, float(gH), float(gHe1), float(gHe2), float(nH), float(T), int(caseA),
                                  st.ctypes.data)
        return tuple(st)

    def thermal_sample(self, stride):
        """The thermal bisection on every stride-th gas leaf, state unchanged."""
        return load().orc_sim_thermal_sample(self.h, int(stride))

    def thermal_cells(self, idx):
        """The reference's thermal bisection of the leaves idx from the current
        state and rates, state unchanged: (n, 5) = T_e, x_HI, x_HeI, x_HeII, n_e."""
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        out = np.zeros((idx.size, 5))
        assert load().orc_sim_thermal_cells(self.h, idx.ctypes.data, idx.size, out.ctypes.data) == idx.size
        return out

    @property
    def diffuse_count(self):
        """Diffuse packets of the last transport pass."""
        return int(load().orc_sim_diffuse_count(self.h))

    def net_rate(self, il, T):
        """thermal_mod.f90 net_rate on leaf il at T: (net, x_HI, x_HeI, x_HeII, n_e)."""
        o = np.zeros(5)
        assert load().orc_sim_net_rate(self.h, int(il), float(T), o.ctypes.data) == 0
        return tuple(o)

    def metal_thermal(self, il, T, nH, ne, xHI):
        o = np.zeros(4)
        assert load().orc_sim_metal_thermal(self.h, int(il), float(T), float(nH), float(ne), float(xHI),
                                            o.ctypes.data) == 0
        return tuple(o)

    @property
    def metal_ntr(self):
        return load().orc_sim_metal_ntr(self.h)

    @property
    def metal_nstage(self):
        return load().orc_sim_metal_nstage(self.h)

    def get(self, name):
        lib = load()
        cap = self.nleaf * max(self.nnu, 6) + 1024
        out = np.zeros(cap)
        n = lib.orc_sim_get(self.h, name.encode(), out.ctypes.data, cap)
        if n < -1:   # larger field: the negative return is its size
            cap = -n
            out = np.zeros(cap)
            n = lib.orc_sim_get(self.h, name.encode(), out.ctypes.data, cap)
        assert n >= 0, name
        out = out[:n]
        if name == "jt_ion":
            out = out.reshape(self.nleaf, self.nnu)
        elif name in ("gamma_metal", "heat_metal"):
            out = out.reshape(self.nleaf, self.metal_ntr)
        elif name == "x_metal":
            out = out.reshape(self.nleaf, self.metal_nstage)
        elif name == "metal_raw":
            out = out.reshape(self.nleaf, self.metal_ntr, 2)
        return out

    def set(self, name, values):
        """State fields (x_HI, x_HeI, x_HeII, n_e, T_e, nH) or rates (gamma_*,
        heat_*, and with metals gamma_metal / heat_metal, leaf-major)."""
        a = np.ascontiguousarray(values, dtype=float)
        assert load().orc_sim_set(self.h, name.encode(), a.ctypes.data, a.size) == a.size, name

    def imaging_pass(self):
        """The transport pass with peel-off (par%ion_peel)."""
        assert load().orc_sim_transport_pass_peel(self.h) == 0

    def peel_image(self, which):
        """'direct', 'scattered' or 'direct0' images of the last imaging pass,
        (nobs, nchan, nyim, nxim), erg/s per code length^2 per pixel."""
        k = {"direct": 0, "scattered": 1, "direct0": 2}[which]
        shape = np.zeros(4, dtype=np.int32)
        n = load().orc_sim_peel_image(self.h, k, None, 0, shape.ctypes.data)
        out = np.zeros(max(-n, n, 0))
        load().orc_sim_peel_image(self.h, k, out.ctypes.data, out.size, shape.ctypes.data)
        return out.reshape(tuple(shape)) if out.size else out

    def peel_observer(self, k):
        out = np.zeros(18)
        assert load().orc_sim_peel_observer(self.h, int(k), out.ctypes.data) == 0
        return out

    def set_state(self, fields):
        """Several fields (dict name -> values) with one opacity refresh."""
        load().orc_sim_defer_fill(self.h, 1)
        try:
            for k, v in fields.items():
                self.set(k, v)
        finally:
            load().orc_sim_defer_fill(self.h, 0)

    def diffuse_build(self):
        n = C.c_longlong()
        lum = load().orc_sim_diffuse_build(self.h, C.byref(n))
        return lum, n.value

    def dust_temp(self):
        """dust_temp_compute and dust_ir_write's sums on the current Heat_dust:
        (T_dust per leaf, IR wavelengths [um], L_nu [erg/s/Hz], absorbed
        power [erg/s])."""
        td, lam, ir = np.zeros(self.nleaf), np.zeros(240), np.zeros(241)
        assert load().orc_sim_dust_temp(self.h, td.ctypes.data, lam.ctypes.data, ir.ctypes.data) == 0
        return td, lam, ir[:240], ir[240]

    def diffuse_photon(self, ip):
        out = np.zeros(8)
        load().orc_sim_diffuse_photon(self.h, int(ip), out.ctypes.data)
        return out

    def photon(self, ip):
        out = np.zeros(8)
        load().orc_sim_photon(self.h, int(ip), out.ctypes.data)
        return out

    def walk_leaves(self, rays, max_steps):
        rays = np.ascontiguousarray(rays, dtype=float).reshape(-1, 6)
        nray = rays.shape[0]
        leaves = np.full((nray, max_steps), -1, dtype=np.int32)
        nsteps = np.zeros(nray, dtype=np.int32)
        load().orc_sim_walk_leaves(self.h, nray, rays.ctypes.data, max_steps, leaves.ctypes.data, nsteps.ctypes.data)
        return leaves, nsteps

    def __del__(self):
        try:
            load().orc_sim_free(self.h)
        except Exception:
            pass
