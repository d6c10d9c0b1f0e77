"""Synthetic benchmark nebulae as namelist texts (the reference's own input
format), with fixed seeds.  No public dataset exists for this path; these
configurations are the workloads.

  stromgren64   pure-H Stromgren sphere: uniform 64^3 Cartesian grid whose
                box side is twice the analytic Stromgren radius, n_H = 100,
                40 kK blackbody with Q(H) = 1e49 s^-1 over 13.598-100 eV (the
                luminosity is Q(H) times the mean photon energy of that Planck
                band, 18.633 eV), case
                B, T_e fixed at 1e4 K, Owen-scrambled Sobol launch (seed
                12345), 1e6 packets, 10 iterations, FP64 arithmetic.
  hhe128        the H+He part of the 128^3 H II region (n_H = 100, He/H 0.1,
                45 kK, Q(H) = 5e49 s^-1, case A), 1e7 packets per pass, FP32
                segments with compensated FP32 tallies.
"""
import math
import os

ATOMIC_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "atomic")

PC2CM = 3.0856776e18
KB_CGS = 1.380649e-16
EV2ERG = 1.602176634e-12


def _alphaB_HII_1e4():
    """Case-B H recombination at 1e4 K as recomb_mod evaluates it by default
    (Badnell total minus the Milne ground-level fit), recomb_mod.f90:51,63,188."""
    T = 1.0e4
    tt = math.sqrt(T / 2.965)
    aA = 8.318e-11 / (tt * (1.0 + tt) ** (1.0 - 0.7472) * (1.0 + math.sqrt(T / 7.001e5)) ** (1.0 + 0.7472))
    te = T * (KB_CGS / EV2ERG)
    a1 = (1.87007e-2 * 1.0e-10 * te ** (-1.29077 + 2.17465e-3 * math.log(te))
          * (1.0 + 8.44399e-2 * te ** (-5.93940e-4)) / (1.0 + 1.29189e1 * te ** (-8.05060e-1)))
    return aA - a1


def mean_photon_energy_ev(T, emin=13.598, emax=100.0, n=200001):
    """<E> = int B_E dE / int B_E/E dE of a blackbody over [emin, emax] eV, so
    that luminosity = Q(H) <E> ev2erg gives the band photon rate Q(H)."""
    h = (emax - emin) / (n - 1)
    num = den = 0.0
    for i in range(n):
        e = emin + i * h
        w = 0.5 if i in (0, n - 1) else 1.0
        b = e ** 3 / math.expm1(e / (8.617333262145e-5 * T))
        num += w * b
        den += w * b / e
    return num / den


def stromgren_radius_pc(Q=1.0e49, nH=100.0):
    """Sharp-edge R_S = (3 Q / (4 pi n_H^2 alpha_B))^(1/3) [pc]."""
    return (3.0 * Q / (4.0 * math.pi * nH * nH * _alphaB_HII_1e4())) ** (1.0 / 3.0) / PC2CM


def stromgren64(nphotons=1_000_000, niter=10, n=64, precision="fp64", seed=12345):
    rs = stromgren_radius_pc()
    return f"""&parameters
 par%no_photons = {float(nphotons):.6e}
 par%launch_sequence = 'sobol'
 par%qmc_seed = {seed}
 par%grid_type = 'car'
 par%car_walk = 'dda'
 par%nx = {n}
 par%ny = {n}
 par%nz = {n}
 par%xmax = {rs:.10f}
 par%ymax = {rs:.10f}
 par%zmax = {rs:.10f}
 par%distance_unit = 'pc'
 par%nH_const = 100.0
 par%He_abund = 0.0
 par%xHI_init = 1.0
 par%tstar = 4.0e4
 par%luminosity = {1.0e49 * mean_photon_energy_ev(4.0e4) * EV2ERG:.6e}
 par%eion_min = 13.598
 par%eion_max = 100.0
 par%case_ab = 'B'
 par%te_fixed = 1.0e4
 par%ion_relax = 1.0
 par%gas_niter = {niter}
 par%gas_tol = 1.0e-3
 par%precision = '{precision}'
/
"""


def hii_thermal(nphotons=10_000_000, niter=20, n=128, precision="fp32", seed=12345, rs_factor=1.0):
    """H+He H II region with the thermal balance (the 128^3, n_H = 100,
    He/H 0.1, 45 kK, Q(H) = 5e49 s^-1, case A workload with T_e solved in
    [3e3, 3e4] K; the metals and the diffuse packets are separate rows)."""
    rs = stromgren_radius_pc(Q=5.0e49) * rs_factor
    return f"""&parameters
 par%no_photons = {float(nphotons):.6e}
 par%launch_sequence = 'sobol'
 par%qmc_seed = {seed}
 par%grid_type = 'car'
 par%nx = {n}
 par%ny = {n}
 par%nz = {n}
 par%xmax = {rs:.10f}
 par%ymax = {rs:.10f}
 par%zmax = {rs:.10f}
 par%distance_unit = 'pc'
 par%nH_const = 100.0
 par%He_abund = 0.1
 par%tstar = 4.5e4
 par%luminosity = {5.0e49 * mean_photon_energy_ev(4.5e4) * EV2ERG:.6e}
 par%case_ab = 'A'
 par%solve_te = .true.
 par%te_min = 3.0e3
 par%te_max = 3.0e4
 par%te_fixed = 1.0e4
 par%gas_niter = {niter}
 par%atomic_dir = '{ATOMIC_DIR}'
 par%precision = '{precision}'
/
"""


# Trace metals by number of the 128^3 H II-region workload.
METALS = dict(C=2.7e-4, N=6.8e-5, O=4.9e-4, Ne=8.5e-5, S=1.3e-5, Ar=2.5e-6, Mg=4.0e-5, Si=3.2e-5, Fe=3.2e-5,
              Cl=3.0e-7, Ca=2.0e-6)


def hii_metals(nphotons=10_000_000, niter=20, n=128, precision="fp32", seed=12345, rs_factor=1.0,
               diffuse=True, solve_te=True):
    """H+He+metals H II region with the thermal balance: 128^3 uniform grid,
    n_H = 100, He/H 0.1, eleven trace metals, a 45 kK blackbody with Q(H) =
    5e49 s^-1, case A with explicit diffuse Milne recombination packets, no
    dust; T_e solved in [3e3, 3e4] K, from an ionized start (x_HI = 1e-3,
    He half singly ionized) as the reference's H II-region inputs use."""
    rs = stromgren_radius_pc(Q=5.0e49) * rs_factor
    ab = "\n".join(f" par%abund_{k} = {v:.6e}" for k, v in METALS.items())
    return f"""&parameters
 par%no_photons = {float(nphotons):.6e}
 par%launch_sequence = 'sobol'
 par%qmc_seed = {seed}
 par%grid_type = 'car'
 par%nx = {n}
 par%ny = {n}
 par%nz = {n}
 par%xmax = {rs:.10f}
 par%ymax = {rs:.10f}
 par%zmax = {rs:.10f}
 par%distance_unit = 'pc'
 par%nH_const = 100.0
 par%He_abund = 0.1
 par%tstar = 4.5e4
 par%luminosity = {5.0e49 * mean_photon_energy_ev(4.5e4) * EV2ERG:.6e}
 par%case_ab = 'A'
 par%xHI_init = 1.0e-3
 par%xHeI_init = 0.5
 par%xHeII_init = 0.5
 par%diffuse_field = {'.true.' if diffuse else '.false.'}
 par%solve_te = {'.true.' if solve_te else '.false.'}
 par%te_min = 3.0e3
 par%te_max = 3.0e4
 par%te_fixed = 1.0e4
 par%gas_niter = {niter}
 par%use_metals = .true.
{ab}
 par%atomic_dir = '{ATOMIC_DIR}'
 par%precision = '{precision}'
/
"""


def hhe128(nphotons=10_000_000, niter=20, n=128, precision="fp32", seed=12345, rs_factor=1.0):
    """H+He H II region on a uniform grid, case A, fixed T_e (the He/H and
    source of the 128^3 H II-region workload; metals, diffuse packets and the
    thermal solve are separate rows)."""
    rs = stromgren_radius_pc(Q=5.0e49) * rs_factor
    return f"""&parameters
 par%no_photons = {float(nphotons):.6e}
 par%launch_sequence = 'sobol'
 par%qmc_seed = {seed}
 par%grid_type = 'car'
 par%nx = {n}
 par%ny = {n}
 par%nz = {n}
 par%xmax = {rs:.10f}
 par%ymax = {rs:.10f}
 par%zmax = {rs:.10f}
 par%distance_unit = 'pc'
 par%nH_const = 100.0
 par%He_abund = 0.1
 par%tstar = 4.5e4
 par%luminosity = {5.0e49 * mean_photon_energy_ev(4.5e4) * EV2ERG:.6e}
 par%case_ab = 'A'
 par%te_fixed = 1.0e4
 par%gas_niter = {niter}
 par%precision = '{precision}'
/
"""


def on_octree(namelist, amr_file, density_from_file=True):
    """The same nebula on an octree read from a generic text leaf list
    (grid_type = 'amr'): the box side comes from the file, and with
    density_from_file the leaves keep the file's n_H (the namelist's
    par%nH_const line is dropped)."""
    out = []
    for line in namelist.splitlines():
        key = line.strip().split("=")[0].strip()
        if key in ("par%grid_type", "par%car_walk", "par%nx", "par%ny", "par%nz", "par%xmax", "par%ymax", "par%zmax"):
            continue
        if density_from_file and key == "par%nH_const":
            continue
        if line.strip() == "/":
            out.append(" par%grid_type = 'amr'")
            out.append(f" par%amr_file = '{amr_file}'")
        out.append(line)
    return "\n".join(out) + "\n"


def kext_with_g(src, dst, g=0.6):
    """A copy of an extinction table whose <cos> column is g in every data
    row (the row test of the table reader: four leading reals, lambda > 0),
    so the Henyey-Greenstein asymmetry of the run is g at every energy while
    the code path stays the table read."""
    out = []
    for line in open(src):
        tok = line.split()
        try:
            v = [float(t) for t in tok[:4]]
            ok = len(v) == 4 and v[0] > 0
        except ValueError:
            ok = False
        if ok:
            tok[2] = f"{g:.4f}"
            line = " ".join(tok) + "\n"
        out.append(line)
    with open(dst, "w") as f:
        f.writelines(out)
    return dst


KEXT_MW31 = os.path.join(os.path.dirname(ATOMIC_DIR), "kext_albedo_WD_MW_3.1_60_D03.all_2003")


def clumpy_dusty(workdir, nphotons=30_000_000, niter=20, precision="fp32", seed=2024, box_pc=40.0,
                 base_level=6, max_level=10, field_n=256, growth=1.47, scatter=True, qmc_seed=12345):
    """The dusty clumpy nebula on an octree: a log-normal n_H (mean 30,
    sigma_ln n = 1) from a seeded Gaussian random field with P(k) ~ k^-11/3
    on field_n^3, an octree with base level base_level refined towards
    max_level where n_H exceeds 4 <n_H> growth^(L - base_level) (about 3e6
    leaves at the defaults), written as a text leaf list; three point
    sources at seeded positions (35, 40, 50 kK, Q(H) = 2e49 s^-1 each); MW
    R_V = 3.1 grains with the Henyey-Greenstein <cos> set to 0.6, dust-to-gas
    0.01, scattering on; the band extended down to 6 eV (FUV); T_e solved
    (H + He, case B), 3e7 packets per iteration.  Writes the leaf list and
    the extinction table into workdir (reused when present) and returns the
    namelist."""
    import numpy as np
    from . import amr
    os.makedirs(workdir, exist_ok=True)
    tag = f"s{seed}_b{base_level}_m{max_level}_n{field_n}_g{growth}_L{box_pc}"
    leaves = os.path.join(workdir, f"clumpy_{tag}.txt")
    if not os.path.exists(leaves):
        field = amr.lognormal_field(n=field_n, mean=30.0, sigma_ln=1.0, seed=seed)
        x, y, z, lev, nH = amr.clumpy_nebula(box_pc, field, base_level=base_level, max_level=max_level,
                                             threshold=120.0, growth=growth)
        tmp = leaves + ".part"
        amr.write_leaf_list(tmp, box_pc, x, y, z, lev, nH)
        os.replace(tmp, leaves)
    kext = os.path.join(workdir, "kext_MW31_g0.6.txt")
    if not os.path.exists(kext):
        kext_with_g(KEXT_MW31, kext + ".part", 0.6)
        os.replace(kext + ".part", kext)
    rng = np.random.default_rng(seed + 1)
    pos = rng.uniform(-0.3 * box_pc, 0.3 * box_pc, (3, 3))
    temps = (3.5e4, 4.0e4, 5.0e4)
    lums = [2.0e49 * mean_photon_energy_ev(t) * EV2ERG for t in temps]
    arr = lambda v: ", ".join(f"{a:.10e}" for a in v)   # noqa: E731
    return f"""&parameters
 par%no_photons = {float(nphotons):.6e}
 par%launch_sequence = 'sobol'
 par%qmc_seed = {qmc_seed}
 par%iseed = {seed}
 par%grid_type = 'amr'
 par%amr_file = '{leaves}'
 par%distance_unit = 'pc'
 par%He_abund = 0.1
 par%nsource = 3
 par%src_tstar(1) = {arr(temps)}
 par%src_lum(1) = {arr(lums)}
 par%src_x(1) = {arr(pos[:, 0])}
 par%src_y(1) = {arr(pos[:, 1])}
 par%src_z(1) = {arr(pos[:, 2])}
 par%case_ab = 'B'
 par%add_fuv = .true.
 par%efuv_min = 6.0
 par%ion_add_dust = .true.
 par%ion_dust_scatter = {'.true.' if scatter else '.false.'}
 par%ion_dust_kext = '{kext}'
 par%dust_density_law = 'global_dgr'
 par%DGR = 0.01
 par%solve_te = .true.
 par%te_min = 3.0e3
 par%te_max = 3.0e4
 par%te_fixed = 1.0e4
 par%gas_niter = {niter}
 par%atomic_dir = '{ATOMIC_DIR}'
 par%precision = '{precision}'
/
"""


def hii_instance(n, nH, tstar, Q, nphotons=2_000_000, niter=20, precision="fp32", seed=12345, rs_factor=1.2,
                 metal_tally="exact"):
    """One H II region of the batched workload: an n^3 uniform grid whose box
    half-width is rs_factor times the Stromgren radius of (Q, n_H), He/H 0.1
    and the eleven trace metals of hii_metals, a tstar blackbody with photon
    rate Q(H) over 13.598-100 eV, case A, T_e solved in [3e3, 3e4] K from an
    ionized start, no diffuse packets."""
    rs = stromgren_radius_pc(Q=Q, nH=nH) * rs_factor
    ab = "\n".join(f" par%abund_{k} = {v:.6e}" for k, v in METALS.items())
    return f"""&parameters
 par%no_photons = {float(nphotons):.6e}
 par%launch_sequence = 'sobol'
 par%qmc_seed = {seed}
 par%grid_type = 'car'
 par%nx = {n}
 par%ny = {n}
 par%nz = {n}
 par%xmax = {rs:.10f}
 par%ymax = {rs:.10f}
 par%zmax = {rs:.10f}
 par%distance_unit = 'pc'
 par%nH_const = {nH:.8e}
 par%He_abund = 0.1
 par%tstar = {tstar:.6e}
 par%luminosity = {Q * mean_photon_energy_ev(tstar, n=20001) * EV2ERG:.6e}
 par%case_ab = 'A'
 par%xHI_init = 1.0e-3
 par%xHeI_init = 0.5
 par%xHeII_init = 0.5
 par%solve_te = .true.
 par%te_min = 3.0e3
 par%te_max = 3.0e4
 par%te_fixed = 1.0e4
 par%gas_niter = {niter}
 par%use_metals = .true.
{ab}
 par%metal_tally = '{metal_tally}'
 par%atomic_dir = '{ATOMIC_DIR}'
 par%precision = '{precision}'
/
"""


def batch_instances(count=64, seed=5, nmin=32, nmax=128, nphotons=2_000_000, precision="fp32",
                    metal_tally="exact"):
    """The batched-nebulae workload: count H II regions with seeded uneven
    cubic grid sizes uniform in {nmin..nmax}, n_H log-uniform in 10-1000
    cm^-3, T_eff uniform in 30-50 kK and Q(H) log-uniform in 1e48-1e50 s^-1.
    Returns (namelists, parameters)."""
    import random
    rng = random.Random(seed)
    out, par = [], []
    for k in range(count):
        n = rng.randint(nmin, nmax)
        nH = 10.0 ** rng.uniform(1.0, 3.0)
        tstar = rng.uniform(3.0e4, 5.0e4)
        Q = 10.0 ** rng.uniform(48.0, 50.0)
        out.append(hii_instance(n, nH, tstar, Q, nphotons=nphotons, precision=precision, seed=12345 + k,
                                metal_tally=metal_tally))
        par.append(dict(n=n, nH=nH, tstar=tstar, Q=Q))
    return out, par


def prepared_state(n, front=0.7, width=1.0, he=True, T_in=8.0e3, T_out=3.0e3, nH=100.0, yHe=0.1):
    """A deterministic developed-H II-region state on an n^3 Cartesian grid
    (raster leaf order, il = ix + n (iy + n iz)): an ionized sphere of radius
    front x the box half-width around the centre, x_HI = 1e-3 inside rising
    to 1 over a logistic edge `width` cells wide; with He, He singly ionized
    where H is (x_HeI = x_HI, x_HeII = 1 - x_HI, no He III); T_e = T_in inside
    and T_out outside, blended by the same edge; n_e from charge balance.
    The benchmark's device steps and its CPU reference steps both start from
    this state, so both measure the same iteration."""
    import numpy as np
    c = (np.arange(n) + 0.5) - 0.5 * n
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z).ravel()
    s = 1.0 / (1.0 + np.exp(-(r - front * 0.5 * n) / width))   # 0 inside, 1 outside
    xHI = 1.0e-3 + (1.0 - 1.0e-3) * s
    out = {"x_HI": xHI, "T_e": T_in + (T_out - T_in) * s}
    ne = nH * (1.0 - xHI)
    if he:
        out["x_HeI"] = xHI.copy()
        out["x_HeII"] = 1.0 - xHI
        ne = ne + nH * yHe * out["x_HeII"]
    out["n_e"] = ne
    return out


def hii40(workdir, nphotons=40_000_000, niter=100, precision="fp32", level=6, rin_pc=0.97223, rout_pc=4.73154,
          production=False):
    """The Lexington HII40 H II region: a hollow uniform sphere of n_H = 100
    between rin_pc and rout_pc on a uniform octree of the given level
    spanning +-rout_pc around a 40 kK blackbody (13.598-100 eV, 32 bins),
    thermal balance in [3e3, 3e4] K with the Lexington metals (C, N, O, Ne,
    S: the reference defaults), from an ionized start, at most niter
    iterations.  Writes the leaf list into workdir and returns the namelist.

    production=False: the reference's G2 gate input (tests/g2_hii/hii40.in):
    Q(H) = 4.26e49 s^-1 (luminosity 1.353758e39 erg/s), case B on the spot,
    metal n_e and heating off, gas_tol = gas_tol_te = 5e-3.

    production=True: the reference's production input
    (tests/continuous_energy/hii40_continuous.in), for which it publishes
    <T[NpNe]> = 8169 K: luminosity 1.2734e39 erg/s, its Sobol scramble seed
    (qmc_seed 20260728), case A with the Milne
    diffuse field and its He I excited channel (hei_diffuse), metal
    absorption, metal n_e and heating on, the volume convergence criterion
    with gas_tol 5e-3 and gas_tol_te 1e-2, 2^25 packets by default."""
    import numpy as np
    from . import amr
    os.makedirs(workdir, exist_ok=True)
    leaves = os.path.join(workdir, f"hii40_L{level}.txt")
    if not os.path.exists(leaves):
        box = 2.0 * rout_pc

        def dens(x, y, z, lev):
            r = np.sqrt(x * x + y * y + z * z)
            return np.where((r >= rin_pc) & (r < rout_pc), 100.0, 0.0)

        x, y, z, lev, nH = amr.build_leaves(box, level, level, lambda *a: None, dens)
        amr.write_leaf_list(leaves + ".part", box, x, y, z, lev, nH)
        os.replace(leaves + ".part", leaves)
    if production:
        if nphotons == 40_000_000:
            nphotons = 33_554_432
        run = """ par%luminosity = 1.273400e39
 par%qmc_seed = 20260728
 par%conv_crit = 'vol'
 par%gas_tol = 5.0e-3
 par%gas_tol_te = 1.0e-2
 par%case_ab = 'A'
 par%diffuse_field = .true.
 par%diffuse_energy_model = 'milne'
 par%hei_diffuse = .true.
 par%ion_metal_abs = .true.
 par%metal_ne = .true.
 par%metal_heat = .true.
"""
    else:
        run = """ par%luminosity = 1.353758e39
 par%gas_tol = 5.0e-3
 par%gas_tol_te = 5.0e-3
 par%case_ab = 'B'
 par%metal_ne = .false.
 par%metal_heat = .false.
"""
    return f"""&parameters
 par%no_photons = {float(nphotons)!r}
 par%iseed = 1234
 par%launch_sequence = 'sobol'
 par%grid_type = 'amr'
 par%amr_file = '{leaves}'
 par%dust_density_law = 'none'
 par%distance_unit = 'pc'
 par%nnu_ion = 32
 par%eion_min = 13.598
 par%eion_max = 100.0
 par%tstar = 4.0e4
 par%xHI_init = 1.0e-3
 par%xHeI_init = 0.5
 par%xHeII_init = 0.5
 par%He_abund = 0.1
 par%ion_add_dust = .false.
 par%gas_niter = {niter}
 par%ion_relax = 1.0
 par%solve_te = .true.
 par%te_min = 3.0e3
 par%te_max = 3.0e4
 par%use_metals = .true.
{run} par%atomic_dir = '{ATOMIC_DIR}'
 par%precision = '{precision}'
/
"""


def g2a(workdir, nphotons=40_000_000, niter=100, precision="fp32", level=6):
    """The reference's G2a thermal gate input (tests/g2a_thermal/
    g2a_thermal.in): a uniform n_H = 100 sphere of radius 4 pc (He/H 0.1) on
    a uniform octree of the given level over an 8 pc box, a central 40 kK
    blackbody with Q(H) = 1e49 s^-1 (luminosity 3.177837e38 erg/s over
    13.598-100 eV, 32 bins), case B, H/He thermal balance in [3e3, 5e4] K
    with no metals, from x_HI = 1e-3, He all He II and T_e = 1e4 K; iterated
    to gas_tol = gas_tol_te = 2e-3 (at most niter).  Writes the leaf list
    into workdir and returns the namelist."""
    import numpy as np
    from . import amr
    os.makedirs(workdir, exist_ok=True)
    leaves = os.path.join(workdir, f"sphere_L{level}_nH100.txt")
    if not os.path.exists(leaves):
        def dens(x, y, z, lev):
            return np.where(np.sqrt(x * x + y * y + z * z) < 4.0, 100.0, 0.0)

        x, y, z, lev, nH = amr.build_leaves(8.0, level, level, lambda *a: None, dens)
        amr.write_leaf_list(leaves + ".part", 8.0, x, y, z, lev, nH)
        os.replace(leaves + ".part", leaves)
    return f"""&parameters
 par%no_photons = {float(nphotons)!r}
 par%iseed = 1234
 par%launch_sequence = 'sobol'
 par%grid_type = 'amr'
 par%amr_file = '{leaves}'
 par%dust_density_law = 'none'
 par%distance_unit = 'pc'
 par%nnu_ion = 32
 par%eion_min = 13.598
 par%eion_max = 100.0
 par%tstar = 4.0e4
 par%luminosity = 3.177837e38
 par%xHI_init = 1.0e-3
 par%xHeI_init = 0.0
 par%xHeII_init = 1.0
 par%He_abund = 0.1
 par%ion_add_dust = .false.
 par%gas_niter = {niter}
 par%gas_tol = 2.0e-3
 par%te_fixed = 1.0e4
 par%ion_relax = 1.0
 par%case_ab = 'B'
 par%solve_te = .true.
 par%te_min = 3.0e3
 par%te_max = 5.0e4
 par%gas_tol_te = 2.0e-3
 par%atomic_dir = '{ATOMIC_DIR}'
 par%precision = '{precision}'
/
"""


def slab(nphotons=400_000, faces="top", mode="beam", theta=0.0, phi=0.0, source=1.0e-5, nx=1, nz=64,
         car_walk="dda", precision="fp64", nH=0.1, zmax=0.5, nnu=1, niter=0, bot=None, rmax=100.0):
    """The plane-parallel slab inputs of the reference's slab gates
    (tests/slab/ga_*.in): a frozen neutral pure-hydrogen column of n_H = 0.1
    and thickness 2 zmax = 1 pc on nz = 64 cubic cells, periodic in x and y
    (nx = ny columns of side 2 zmax / nz), lit from the top face by a 40 kK
    blackbody of band flux F_n = 1e-5 erg/s/cm^2 (beam at incidence theta)
    or intensity I (isotropic), one band bin, fixed T_e = 1e4 K, no
    iteration (rates only).  bot = (mode, theta, source) lights the bottom
    face as well (faces 'both')."""
    half = zmax / nz * nx
    lines = [
        f" par%no_photons = {float(nphotons)!r}",
        " par%iseed = 1234",
        " par%launch_sequence = 'sobol'",
        " par%grid_type = 'car'",
        f" par%car_walk = '{car_walk}'",
        f" par%nx = {nx}", f" par%ny = {nx}", f" par%nz = {nz}",
        f" par%xmax = {half!r}", f" par%ymax = {half!r}", f" par%zmax = {zmax!r}",
        f" par%nH_const = {nH!r}",
        f" par%rmax = {rmax!r}",
        " par%dust_density_law = 'none'",
        " par%distance_unit = 'pc'",
        " par%xy_periodic = .true.",
        " par%ion_align_edges = .false.",
        f" par%nnu_ion = {nnu}",
        " par%eion_min = 13.598",
        " par%eion_max = 100.0",
        " par%tstar = 4.0e4",
        " par%He_abund = 0.0",
        " par%xHI_init = 1.0",
        " par%ion_add_dust = .false.",
        f" par%gas_niter = {niter}",
        " par%te_fixed = 1.0e4",
        " par%source_geometry = 'slab'",
        f" par%slab_faces = '{faces}'",
        f" par%slab_top_mode = '{mode}'",
        f" par%slab_top_theta = {theta!r}",
        f" par%slab_top_phi = {phi!r}",
        f" par%slab_top_source = {source!r}",
        f" par%atomic_dir = '{ATOMIC_DIR}'",
        f" par%precision = '{precision}'",
    ]
    if bot is not None:
        lines += [f" par%slab_bot_mode = '{bot[0]}'", f" par%slab_bot_theta = {bot[1]!r}",
                  f" par%slab_bot_source = {bot[2]!r}"]
    return "&parameters\n" + "\n".join(lines) + "\n/\n"
