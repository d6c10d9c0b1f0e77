"""The oracle's He I excited diffuse channel (CPU only) against the
reference's own gates for it, tests/hei_cascade/check_hei_2ph.f90,
check_hei_branches.f90 and check_hei_584.f90, with their bars:

  two-photon continuum: the tabulated shape is symmetric about y = 1/2 and
  integrates to two photons per decay (2 %); photons and in-band energy per
  decay equal an independent midpoint quadrature of the same table (1e-4);
  every sampled energy lies in [13.598, 20.62] eV; the stratified sample mean
  is the energy-weighted mean (2e-4) and <1/E> <E>_n = 1 (5e-4);
  branch fractions: the BSS99 ratios (1e-12), summing to one, clamped below
  3e3 K and above 2e4 K, near the low-density weights 3/4, 1/12, 1/6;
  584 A closure: the three published forms agree, x(He0) = 0 gives 1.
"""
import os

import numpy as np
import pytest

from mochii_b200 import configs

TABLE = os.path.join(os.path.dirname(configs.ATOMIC_DIR), "HeI2phot.dat")
E_TOT, A2G, ETH = 20.62, 51.3, 13.598


def table():
    t = np.loadtxt(TABLE, comments="!")
    return t[:, 0], t[:, 1]


def test_two_photon_table_and_sampler(orc):
    ty, ta = table()
    tot = float(np.sum(0.5 * (ta[1:] + ta[:-1]) * np.diff(ty)))
    assert abs(tot / A2G - 2.0) < 0.02
    assert np.max(np.abs(ta - ta[::-1])) / ta.max() < 5e-3
    nq = 400000
    ylo = ETH / E_TOT
    dy = (1.0 - ylo) / nq
    y = ylo + (np.arange(nq) + 0.5) * dy
    a = np.interp(y, ty, ta)
    qn, qe, q2 = np.sum(a) * dy, np.sum(a * y * E_TOT) * dy, np.sum(a * (y * E_TOT) ** 2) * dy
    ns = 200000
    u = (np.arange(ns) + 0.5) / ns
    n_dec, e_dec, E = orc.hei_2ph(TABLE, u)
    assert abs(n_dec / (2 * qn / tot) - 1) < 1e-4
    assert abs(e_dec / (2 * qe / tot) - 1) < 1e-4
    assert E.min() >= ETH - 1e-9 and E.max() <= E_TOT + 1e-9
    assert abs(E.mean() / (q2 / qe) - 1) < 2e-4
    assert abs(np.mean(1.0 / E) * (qe / qn) - 1) < 5e-4
    # the in-band window ends at the band edge when that is lower
    n_lo, e_lo, E_lo = orc.hei_2ph(TABLE, u[::1000], eion_max=18.0)
    assert n_lo < n_dec and E_lo.max() <= 18.0 + 1e-9


@pytest.mark.parametrize("T", [3.0e3, 5.0e3, 8.0e3, 1.0e4, 1.5e4, 2.0e4])
def test_branch_fractions(orc, T):
    n_dec, e_dec, _ = orc.hei_2ph(TABLE, [0.5])
    e3s, e1p, e1s = orc.hei_branch_energies(TABLE, T, 0.5, 0.0)   # x(He0) = 0: the 584 A photon always ionizes H
    f3s, f1p, f1s = e3s / 19.82, e1p / 21.22, e1s / e_dec
    r3 = 2.10e-13 * (T / 1e4) ** -0.381
    r1s = 2.06e-14 * (T / 1e4) ** -0.451
    r1p = 4.17e-14 * (T / 1e4) ** -0.695
    s = r3 + r1s + r1p
    assert min(f3s, f1s, f1p) > 0 and abs(f3s + f1s + f1p - 1) < 1e-12
    assert max(abs(f3s - r3 / s), abs(f1s - r1s / s), abs(f1p - r1p / s)) < 1e-12
    assert abs(f3s - 0.75) < 0.05 and abs(f1s - 1 / 12) < 0.02 and abs(f1p - 1 / 6) < 0.05


def test_branch_fractions_clamped(orc):
    for T, Tc in ((1.0e2, 3.0e3), (1.0e6, 2.0e4)):
        a = orc.hei_branch_energies(TABLE, T, 0.5, 0.0)
        b = orc.hei_branch_energies(TABLE, Tc, 0.5, 0.0)
        assert np.allclose(a, b, rtol=1e-12, atol=0)


def test_584_closure_forms_agree(orc):
    f1p = orc.hei_branch_energies(TABLE, 8.0e3, 0.5, 0.0)[1] / 21.22
    assert abs(orc.hei_branch_energies(TABLE, 8.0e3, 1e-4, 0.0)[1] / 21.22 / f1p - 1) < 1e-15
    for T in (5.0e3, 8.0e3, 1.2e4):
        f1p = orc.hei_branch_energies(TABLE, T, 0.5, 0.0)[1] / 21.22
        for xh0 in (1e-4, 1e-2, 0.3):
            for xhe0 in (1e-3, 0.1, 0.9):
                p = orc.hei_branch_energies(TABLE, T, xh0, xhe0)[1] / (21.22 * f1p)
                wood = 1.0 / (1.0 + 0.77 / (np.sqrt(T) / 1e2) * xhe0 / xh0)
                cmac = np.sqrt(T) * xh0 / (np.sqrt(T) * xh0 + 77.0 * xhe0)
                assert abs(p - wood) < 1e-13 and abs(p - cmac) < 1e-13
                # converted 584 A decays leave as the two-photon pair
                n_dec, e_dec, _ = orc.hei_2ph(TABLE, [0.5])
                e1s = orc.hei_branch_energies(TABLE, T, xh0, xhe0)[2]
                e1s0 = orc.hei_branch_energies(TABLE, T, xh0, 0.0)[2]
                assert abs((e1s - e1s0) - f1p * (1 - p) * e_dec) < 1e-12
