"""Host side of the transport + balance path, mirroring MoCHII's interface.

    par = read_input("hii.in")                     # setup.f90:11-35
    neb = Nebula(par)                              # grid_create_amr + ion_setup + gas_state_setup
    neb.ionizing_field_and_rates()                 # ionizing_field_mod.f90:72
    max_dx, dx_vol = neb.gas_equilibrium_update()  # ion_balance_mod.f90:352
    neb.gas_opacity_fill()                         # gas_opacity_mod.f90:299
    result = run(par)                              # the driver loop, main.f90:128-225

Every call goes through libmochii_gpu.so; errors come back as MochiiError
carrying the library's status code (the reference aborts instead).
"""
import ctypes as C
import os
import tempfile

import numpy as np

from . import _lib
from ._lib import Metrics, MochiiError, Params, PassStats, Tuning

STATE_FIELDS = ("nH", "x_HI", "x_HeI", "x_HeII", "n_e", "T_e")
RATE_FIELDS = ("gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI", "heat_HeI", "heat_HeII")


def _check(lib, status, ctx=None):
    if status != _lib.OK:
        msg = lib.mochii_last_error(ctx)
        raise MochiiError(status, (msg or b"").decode() or lib.mochii_strerror(status).decode())


def default_params():
    lib = _lib.load()
    p = Params()
    _check(lib, lib.mochii_params_default(C.byref(p)))
    return p


def parse_namelist(text, base=None):
    """Parse '&parameters par%key = value ... /' text over base (or defaults)."""
    lib = _lib.load()
    p = base if base is not None else default_params()
    err = C.create_string_buffer(512)
    rc = lib.mochii_params_parse_namelist(C.byref(p), text.encode(), err, 512)
    if rc != _lib.OK:
        raise MochiiError(rc, err.value.decode())
    return p


def read_input(path):
    """read_input (setup.f90:11-35): the namelist file named on the command line."""
    lib = _lib.load()
    p = default_params()
    err = C.create_string_buffer(512)
    rc = lib.mochii_params_read_namelist(C.byref(p), str(path).encode(), err, 512)
    if rc != _lib.OK:
        raise MochiiError(rc, err.value.decode())
    return p


def set_param(p, key, value):
    lib = _lib.load()
    if isinstance(value, bool):
        value = ".true." if value else ".false."
    rc = lib.mochii_params_set(C.byref(p), key.encode(), str(value).encode())
    if rc != _lib.OK:
        raise MochiiError(rc, f"par%{key} = {value!r}")
    return p


def sobol_uniforms(seed, stream, idx0, n, nd):
    """Device Owen-scrambled Sobol uniforms (qmc_uniforms_stream), shape (n, nd)."""
    lib = _lib.load()
    out = np.zeros((n, nd), dtype=np.float64)
    rc = lib.mochii_sobol_uniforms(int(seed), int(stream), int(idx0), int(n), int(nd), out.ctypes.data)
    _check(lib, rc)
    return out


def philox_uniforms(seed, stream, packet, n0, n):
    """Draws n0 .. n0+n-1 of one packet's scattering stream, computed on the
    device (the Philox4x32-10 stream keyed by par%iseed and the packet)."""
    lib = _lib.load()
    out = np.zeros(n)
    rc = lib.mochii_philox_uniforms(int(seed), int(stream), int(packet), int(n0), int(n), out.ctypes.data)
    _check(lib, rc)
    return out


class Nebula:
    """One nebula on the current CUDA device (a mochii_ctx)."""

    def __init__(self, par, _ctx=None):
        self.lib = _lib.load()
        self.par = par
        h = _ctx
        if h is None:
            h = C.c_void_p()
            _check(self.lib, self.lib.mochii_init(C.byref(par), C.byref(h)))
        self.ctx = h
        self.nleaf = int(self.lib.mochii_nleaf(h))
        self.nnu_band = int(self.lib.mochii_nnu_band(h))
        self.last_pass = None
        self.last_metrics = None

    def close(self):
        if self.ctx:
            self.lib.mochii_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc):
        _check(self.lib, rc, self.ctx)

    # ---- the replaced module entry points ------------------------------
    def ionizing_field_and_rates(self, with_peel=False):
        st = PassStats()
        self._ok(self.lib.mochii_transport_pass(self.ctx, int(bool(with_peel)), C.byref(st)))
        self.last_pass = st
        return st

    def gas_equilibrium_update(self):
        m = Metrics()
        self._ok(self.lib.mochii_balance_update(self.ctx, 0, C.byref(m)))
        self.last_metrics = m
        return m.max_dx, m.dx_vol

    def gas_thermal_update(self):
        m = Metrics()
        self._ok(self.lib.mochii_balance_update(self.ctx, 1, C.byref(m)))
        self.last_metrics = m
        return m.max_dx, m.max_dte, m.dx_vol, m.dte_vol

    def gas_opacity_fill(self):
        self._ok(self.lib.mochii_opacity_fill(self.ctx))

    # ---- state exchange ---------------------------------------------------
    def metal_shape(self):
        """(transitions, stages) of the active metal registry; (0, 0) without metals."""
        a, b = C.c_int(), C.c_int()
        self._ok(self.lib.mochii_metal_shape(self.ctx, C.byref(a), C.byref(b)))
        return a.value, b.value

    def get(self, name):
        ntr, nst = self.metal_shape() if name in ("gamma_metal", "heat_metal", "x_metal") else (0, 0)
        n = {"jt_ion": self.nleaf * self.nnu_band, "eedge": self.nnu_band + 1,
             "gamma_metal": self.nleaf * ntr, "heat_metal": self.nleaf * ntr,
             "x_metal": self.nleaf * nst}.get(name, self.nleaf)
        out = np.zeros(n, dtype=np.float64)
        self._ok(self.lib.mochii_get_field(self.ctx, name.encode(), out.ctypes.data, n))
        if name == "jt_ion":
            out = out.reshape(self.nleaf, self.nnu_band)
        elif name in ("gamma_metal", "heat_metal"):
            out = out.reshape(self.nleaf, ntr)
        elif name == "x_metal":
            out = out.reshape(self.nleaf, nst)
        return out

    def write_rates(self, base, converged=False, iterations=0, final_dx=0.0, final_dte=0.0, field_consistent=False):
        """gas_rates_write: the rates and state of the current iterate as
        <base>_rates/ (one .npy per dataset of the reference's rates file,
        header.json with its keywords); returns the directory."""
        from ._lib import RunInfo
        ri = RunInfo(int(bool(converged)), int(iterations), float(final_dx), float(final_dte),
                     int(bool(field_consistent)))
        self._ok(self.lib.mochii_write_rates(self.ctx, str(base).encode(), C.byref(ri)))
        return str(base) + "_rates"

    def refine_front(self, out_list):
        """amr_refine_front: the octree rebuilt on the current solution
        (par%refine_lbase, refine_lmax, refine_eps, refine_dx) as a NEW
        nebula whose leaf list is written to out_list, its state remapped by
        overlap volume; this nebula stays as it was."""
        h = C.c_void_p()
        self._ok(self.lib.mochii_refine_front(self.ctx, str(out_list).encode(), C.byref(h)))
        par = _lib.Params()
        C.memmove(C.byref(par), C.byref(self.par), C.sizeof(par))
        par.amr_file = str(out_list).encode()
        return Nebula(par, _ctx=h)

    def dust_ir(self):
        """The grains' infrared spectrum of the equilibrium dust temperature
        (dust_ir_write): (lambda [um], L_nu [erg/s/Hz], absorbed power
        [erg/s], integral of L_nu over frequency [erg/s])."""
        lam, lnu, ab = np.zeros(240), np.zeros(240), np.zeros(2)
        self._ok(self.lib.mochii_dust_ir(self.ctx, lam.ctypes.data, lnu.ctypes.data, ab.ctypes.data))
        return lam, lnu, float(ab[0]), float(ab[1])

    def write_dust_ir(self, base):
        """dust_ir_write: <base>_dustir.txt; returns its path."""
        self._ok(self.lib.mochii_write_dust_ir(self.ctx, str(base).encode()))
        return str(base) + "_dustir.txt"

    def slab_tally(self):
        """The plane-parallel slab's boundary tally of the last pass
        (slab_Iesc): (escaping luminosity [erg/s] per mu bin at the top face,
        the same at the bottom face, L_in [erg/s], A_zface [cm^2])."""
        n = 2 * int(self.par.slab_nmu)
        v, meta = np.zeros(n), np.zeros(2)
        self._ok(self.lib.mochii_slab_tally(self.ctx, v.ctypes.data, n, meta.ctypes.data))
        return v[: n // 2], v[n // 2:], float(meta[0]), float(meta[1])

    def write_slab_imu(self, base):
        """slab_write_Imu: <base>_slab_Imu.txt; returns its path."""
        self._ok(self.lib.mochii_write_slab_imu(self.ctx, str(base).encode()))
        return str(base) + "_slab_Imu.txt"

    def imaging_pass(self):
        """The peel-off imaging pass (main.f90:234-235): a transport pass with
        with_peel; needs par%ion_peel."""
        return self.ionizing_field_and_rates(with_peel=True)

    def image(self, which="direct"):
        """Peel-off image of the last imaging pass: 'direct', 'scattered' or
        'direct0', shape (nobs, nchan, nyim, nxim), erg/s per code length^2
        per pixel."""
        shape = np.zeros(4, dtype=np.int32)
        self._ok(self.lib.mochii_image_shape(self.ctx, shape.ctypes.data))
        out = np.zeros(int(np.prod(shape)), dtype=np.float64)
        k = {"direct": 0, "scattered": 1, "direct0": 2}[which]
        self._ok(self.lib.mochii_get_image(self.ctx, k, out.ctypes.data, out.size))
        return out.reshape(tuple(int(v) for v in shape))

    def image_observer(self, k):
        """Observer k: x, y, z, alpha, beta, gamma, distance, dxim, dyim, R (9)."""
        out = np.zeros(18)
        self._ok(self.lib.mochii_image_observer(self.ctx, int(k), out.ctypes.data))
        return out

    def write_image(self, base):
        """ion_peel_write: <base>_image/ with the surface-brightness images."""
        self._ok(self.lib.mochii_write_image(self.ctx, str(base).encode()))
        return str(base) + "_image"

    def set(self, name, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        self._ok(self.lib.mochii_set_field(self.ctx, name.encode(), a.ctypes.data, a.size))

    def set_nphotons(self, n):
        self._ok(self.lib.mochii_set_nphotons(self.ctx, int(n)))

    def autotune(self, sample_packets=1 << 18):
        """Pick the fastest walk launch shape on the current state (tallies are
        overwritten by the trial passes)."""
        t = Tuning()
        self._ok(self.lib.mochii_autotune(self.ctx, int(sample_packets), C.byref(t)))
        return self._tuning_dict(t)

    @staticmethod
    def _tuning_dict(t):
        return {"lookahead": t.lookahead, "walk_blocks_per_sm": t.walk_blocks_per_sm, "best_ms": t.best_ms,
                "lane_threads": t.lane_threads, "thermal_ms": t.thermal_ms}

    def set_tuning(self, lookahead, walk_blocks_per_sm, lane_threads=None):
        cur = self.tuning()
        t = Tuning(int(lookahead), int(walk_blocks_per_sm), 0.0,
                   int(cur["lane_threads"] if lane_threads is None else lane_threads), 0.0)
        self._ok(self.lib.mochii_set_tuning(self.ctx, C.byref(t)))

    def tuning(self):
        t = Tuning()
        self._ok(self.lib.mochii_get_tuning(self.ctx, C.byref(t)))
        return self._tuning_dict(t)

    @property
    def ion_Ltot(self):
        return float(self.lib.mochii_ion_Ltot(self.ctx))

    def walk_leaves(self, rays, max_steps):
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 6)
        nray = rays.shape[0]
        leaves = np.full((nray, max_steps), -1, dtype=np.int32)
        nsteps = np.zeros(nray, dtype=np.int32)
        self._ok(self.lib.mochii_walk_leaves(self.ctx, nray, rays.ctypes.data, int(max_steps),
                                             leaves.ctypes.data, nsteps.ctypes.data))
        return leaves, nsteps

    def diffuse_records(self, ip0, n):
        """Diffuse field of the current state and the launch records of
        diffuse packets ip0..ip0+n-1: (ix, iy, iz, tMax_x, tMax_y, tMax_z,
        sigma_HI*1e18, inu) each; returns (records, diffuse_lum, diffuse_nphot)."""
        out = np.zeros((n, 8), dtype=np.float64)
        lum, nph = C.c_double(), C.c_int64()
        self._ok(self.lib.mochii_diffuse_records(self.ctx, int(ip0), int(n), out.ctypes.data, C.byref(lum),
                                                  C.byref(nph)))
        return out, lum.value, nph.value

    def launch_records(self, ip0, n):
        out = np.zeros((n, 8), dtype=np.float64)
        self._ok(self.lib.mochii_launch_records(self.ctx, int(ip0), int(n), out.ctypes.data))
        return out


def run(par, log=None, final_pass=True):
    """The iteration of main.f90:120-225: transport -> rates -> balance ->
    opacity feedback until converged or par%gas_niter, then one final
    consistency pass.  Returns (nebula, history)."""
    neb = Nebula(par)
    niter = max(par.gas_niter, 1)
    history = []
    converged = False
    for it in range(1, niter + 1):
        st = neb.ionizing_field_and_rates()
        rec = {"iter": it, "closure": st.closure, "segments": st.direct_segments, "transport_ms": st.kernel_ms}
        if par.gas_niter < 1:
            history.append(rec)
            break
        if par.solve_te:
            max_dx, max_dte, dx_vol, dte_vol = neb.gas_thermal_update()
            converged = (dx_vol < par.gas_tol and dte_vol < par.gas_tol_te) if par.conv_vol else \
                (max_dx < par.gas_tol and max_dte < par.gas_tol_te)
            rec.update(max_dx=max_dx, max_dte=max_dte, dx_vol=dx_vol, dte_vol=dte_vol)
        else:
            max_dx, dx_vol = neb.gas_equilibrium_update()
            converged = dx_vol < par.gas_tol if par.conv_vol else max_dx < par.gas_tol
            rec.update(max_dx=max_dx, dx_vol=dx_vol)
        rec["balance_ms"] = neb.last_metrics.kernel_ms
        neb.gas_opacity_fill()
        if par.refine_front and it == par.refine_iter:   # one re-refinement event (main.f90:172-178)
            work = tempfile.mkdtemp(prefix="mochii_refine_")
            new = neb.refine_front(os.path.join(work, f"leaves_refined_{it}.txt"))
            rec["refined"] = {"leaves_before": neb.nleaf, "leaves_after": new.nleaf}
            neb.close()
            neb, par = new, new.par
            converged = False   # keep iterating on the new grid
        history.append(rec)
        if log:
            log(rec)
        if converged:
            break
    if par.gas_niter >= 1 and not converged and par.require_convergence:
        raise MochiiError(7, f"gas iteration did not converge in {niter} iterations")
    if final_pass and par.gas_niter >= 1:
        neb.ionizing_field_and_rates()   # final consistency pass, main.f90:225
    return neb, history


def refine_plan(in_list, state, rhokap=None, He_abund=0.1, te_min=1.0e3, lbase=5, lmax=7, eps=1.0e-2, dx=0.2,
                out_list="refined.txt"):
    """The host part of amr_refine_front without a device: the leaf list
    in_list with its state (dict of nH, x_HI, x_HeI, x_HeII, n_e, T_e) to a
    new leaf list out_list (remapped state as extra columns).  Returns
    (new leaf count, front leaves, largest relative change of a conserved
    box integral)."""
    lib = _lib.load()
    f = [np.ascontiguousarray(state[k], dtype=np.float64) for k in ("nH", "x_HI", "x_HeI", "x_HeII", "n_e", "T_e")]
    rk = None if rhokap is None else np.ascontiguousarray(rhokap, dtype=np.float64)
    counts = np.zeros(2, dtype=np.int64)
    worst = C.c_double()
    rc = lib.mochii_refine_plan(str(in_list).encode(), *[a.ctypes.data for a in f],
                                None if rk is None else rk.ctypes.data, float(He_abund), float(te_min), int(lbase),
                                int(lmax), float(eps), float(dx), str(out_list).encode(), counts.ctypes.data,
                                C.byref(worst))
    if rc != _lib.OK:
        raise MochiiError(rc, lib.mochii_refine_last_error().decode())
    return int(counts[0]), int(counts[1]), worst.value


class Batch:
    """Several nebulae on one device advanced together (mochii_batch_*): one
    iteration of every nebula -- transport pass, then balance -- recorded as
    one CUDA graph at the first call and replayed; with metals and the
    bracketed solver the thermal solves of all nebulae run in one persistent
    launch.  The nebulae stay usable on their own between iterations."""

    def __init__(self, nebulae):
        self.lib = _lib.load()
        self.nebulae = list(nebulae)
        n = len(self.nebulae)
        arr = (C.c_void_p * n)(*[neb.ctx for neb in self.nebulae])
        h = C.c_void_p()
        rc = self.lib.mochii_batch_create(arr, n, C.byref(h))
        _check(self.lib, rc)
        self.h = h

    def set_warm_start(self, mlp):
        """Record the learned warm start (a trained WarmStartMLP) into the
        batch's iteration: each nebula's inference after its pass."""
        _check(self.lib, self.lib.mochii_batch_set_warm_start(self.h, mlp.h))
        self.mlp = mlp

    def iterate(self, solve_te=True):
        """One iteration of every nebula: (pass statistics, balance metrics,
        device milliseconds of the whole batch)."""
        n = len(self.nebulae)
        st = (PassStats * n)()
        m = (Metrics * n)()
        ms = C.c_double()
        rc = self.lib.mochii_batch_iterate(self.h, int(bool(solve_te)), st, m, C.byref(ms))
        _check(self.lib, rc)
        for neb, mm in zip(self.nebulae, m):
            neb.last_metrics = mm
        return list(st), list(m), ms.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.mochii_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
