"""The oracle's trace-metal registry pinned against the reference's own gates
(CPU only).

The charge-exchange gates of tests/charge_exchange restated on the oracle:
check_charge_exchange.f90 (reaction census :73 and :125-143, pairwise
conservation of every reaction :160-210, hydrogen's closed form and the
truncated-denominator assertion :212-272, on the five cell states :79-85),
check_cell_convergence.f90 (one solve_ion_cell call against 400, :20-23 and
:44-66) and check_detailed_balance.f90 (the transition-1 pairs against
detailed balance, :44-60 and :82-125).  Plus the registry order and the
threshold sort of species_setup (species_mod.f90:143-226).
"""
import math
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ATOMIC = os.path.join(ROOT, "mochii_b200", "data", "atomic")
EV2ERG = 1.602176634e-12
KB = 1.380649e-16
EPS = np.finfo(float).eps

ALL11 = dict(C=2.2e-4, N=4.0e-5, O=3.3e-4, Ne=5.0e-5, S=9.0e-6, Ar=3.0e-6, Mg=3.0e-6, Fe=3.0e-6,
             Si=3.0e-6, Cl=3.0e-7, Ca=2.0e-8)
FIVE = dict(C=2.2e-4, N=4.0e-5, O=3.3e-4, Ne=5.0e-5, S=9.0e-6, Ar=0.0, Mg=0.0, Fe=0.0, Si=0.0, Cl=0.0, Ca=0.0)


def one_cell(abund, case="B"):
    ab = "\n".join(f" par%abund_{k} = {v!r}" for k, v in abund.items())
    return f"""&parameters
 par%nphotons = 1000
 par%launch_sequence = 'sobol'
 par%tstar = 4.0e4
 par%luminosity = 1.0e38
 par%nx = 1, par%ny = 1, par%nz = 1
 par%xmax = 1.0, par%ymax = 1.0, par%zmax = 1.0
 par%distance_unit = 'pc'
 par%nH_const = 100.0
 par%He_abund = 0.1
 par%case_ab = '{case}'
 par%ci_model = 'voronov'
 par%recomb_model = 'badnell_milne'
 par%cooling_model = 'low_density'
 par%use_metals = .true.
 par%metal_ne = .true.
 par%charge_exchange = 'two_way'
 par%atomic_dir = '{ATOMIC}'
{ab}
/
"""


@pytest.fixture(scope="module")
def sim11(orc):
    return orc.Sim(one_cell(ALL11), nthreads=1)


def alphaB_HII(orc, T):
    return float(orc.evaluate("alphaB_HII", np.array([T]))[0])


def ci_HI(orc, T):
    return float(orc.evaluate("ci_HI", np.array([T]))[0])


def test_registry_order_and_threshold_sort(sim11):
    els = sim11.metal_elements()
    assert [e[0] for e in els] == ["c", "n", "o", "ne", "s", "ar", "mg", "fe", "si", "cl", "ca"]
    assert [e[1] for e in els] == [6, 7, 8, 10, 16, 18, 12, 26, 14, 17, 20]
    ntr = sum(ns - 1 for _, _, ns in els)
    assert sim11.metal_ntr == ntr == 32
    eth = [sim11.metal_eth(ie, it) for ie, (_, _, ns) in enumerate(els) for it in range(1, ns)]
    assert all(e > 0 for e in eth)


def test_reaction_census(sim11):
    """check_charge_exchange.f90:73,125-143: 7 CXI and 22 CXR reactions at 1e4 K."""
    ncxi = ncxr = 0
    for ie, (_, _, ns) in enumerate(sim11.metal_elements()):
        for it in range(1, ns):
            ki, kr = sim11.metal_cx(ie, it, 1.0e4)
            ncxi += ki > 0
            ncxr += kr > 0
    assert (ncxi, ncxr) == (7, 22)


STATES = [(8.0e3, 1.0e2, 1.0e-9), (8.0e3, 1.0e2, 1.0e-11), (1.0e4, 1.0e3, 1.0e-8), (6.0e3, 1.0e2, 1.0e-13),
          (3.0e2, 5.0e3, 1.0e-16)]


@pytest.mark.parametrize("T,nH,gH", STATES)
def test_pairwise_conservation_and_closed_form(orc, sim11, T, nH, gH):
    """check_charge_exchange.f90:145-272 on the five cell states."""
    x, h1, h2 = 0.5, 0.5, 0.5
    for _ in range(100):
        x, h1, h2, ne = sim11.solve_cell(gH, 0.0, 0.0, nH, T, False, x, h1, h2)
    nHI, nHII = nH * x, nH * (1.0 - x)
    nem, r_in, r_out = sim11.metal_sums(T, nH, ne, nHI, nHII)
    # the cascade's side from species_fractions and the registry coefficients
    cas_in = cas_out = 0.0
    abund = list(ALL11.values())
    for ie, (_, _, ns) in enumerate(sim11.metal_elements()):
        fr = sim11.metal_fractions(ie, T, ne, nHI, nHII)
        nX = abund[ie] * nH
        for it in range(1, ns):
            ki, kr = sim11.metal_cx(ie, it, T)
            cas_in += ki * nX * fr[it - 1]
            cas_out += kr * nX * fr[it]
    assert r_in == pytest.approx(cas_in, rel=1e-13, abs=1e-300)
    assert r_out == pytest.approx(cas_out, rel=1e-13, abs=1e-300)
    aH, cH = alphaB_HII(orc, T), ci_HI(orc, T)

    def resid(xx):
        loss = nH * xx * (gH + cH * ne + r_out)
        gain = (aH * ne + r_in) * nH * (1.0 - xx)
        return abs(loss - gain) / max(loss, 1e-300)

    assert resid(x) <= 1.0e-5                                    # TOL_STATE
    xf = (aH * ne + r_in) / (gH + (cH + aH) * ne + r_in + r_out)
    tol = max(1.0e-14, 4.0 * EPS / max(1.0 - xf, 1e-300))
    assert resid(xf) <= tol
    xb = (aH * ne + r_in) / (gH + (cH + aH) * ne + r_out)       # R_cx_in dropped
    assert resid(xb) > tol


@pytest.mark.parametrize("gH", [3.0e-12, 8.0e-13, 1.5e-13, 3.0e-14, 1.0e-14])
def test_cell_converges_inside_one_solve(orc, gH):
    """check_cell_convergence.f90: one call within 1e-9 of 400 repeated calls."""
    s = orc.Sim(one_cell(FIVE), nthreads=1)
    x, h1, h2, _ = s.solve_cell(gH, 0.0, 0.0, 100.0, 1.0e4, False, 0.5, 0.5, 0.5)
    xr, r1, r2 = 0.5, 0.5, 0.5
    for _ in range(400):
        xr, r1, r2, _ = s.solve_cell(gH, 0.0, 0.0, 100.0, 1.0e4, False, xr, r1, r2)
    assert 0.0 <= x <= 1.0
    assert abs(x - xr) / max(xr, 1e-300) <= 1.0e-9


def test_charge_exchange_detailed_balance(sim11):
    """check_detailed_balance.f90: k_i/k_r against g(X+)g(H0)/(g(X0)g(H+)) e^{-dE/kT}."""
    gw0 = dict(c=9, n=4, o=9, ne=1, mg=1, si=9, s=9, ar=1, fe=25, cl=6, ca=1)
    gw1 = dict(c=6, n=9, o=4, ne=6, mg=2, si=6, s=4, ar=6, fe=30, cl=9, ca=2)
    tested = 0
    for ie, (nm, _, ns) in enumerate(sim11.metal_elements()):
        if ns < 2:
            continue
        dE = (sim11.metal_eth(ie, 1) - 13.5984) * EV2ERG / KB
        ki, kr = sim11.metal_cx(ie, 1, 1.0e4)
        if ki <= 0 or kr <= 0 or min(ki, kr) < 1.0e-15:
            continue
        for T in (5.0e3, 8.0e3, 1.0e4, 2.0e4):
            ki, kr = sim11.metal_cx(ie, 1, T)
            if ki <= 0 or kr <= 0:
                continue
            req = gw1[nm] * 2.0 / gw0[nm] * math.exp(-dE / T)
            assert abs(ki / kr / req - 1.0) <= 0.35, (nm, T, ki / kr / req)
            tested += 1
    assert tested >= 4
