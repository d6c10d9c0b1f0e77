"""The CPU oracle pinned against the reference's own golden vectors and
known answers (CPU only).

Sobol codes: tests/qmc/q0_raw.txt, q0_scr_*.txt, q2_*.txt of the reference,
written by its q0_dump.f90 / q2_dump.f90 drivers (committed here as integer
codes in tests/golden/qmc_golden.npz).  Samplers: the known answers of
tests/energy_sampler/energy_sampler_dump.f90:22-37 and the tolerances of
check_energy_sampler.py:59-168.  Rates: tools/python/mochii_rates.py, pinned
to the Fortran at 1e-10 by tests/rates/check_python_rates.py:38-40.
G2a 1D thermal reference: tests/g2a_thermal/check_g2a.py reference_1d,
run from the reference's own file on 400 shells (g2a_1d_golden.npz).
"""
import numpy as np
import pytest


def codes(u):
    return np.rint(u * 4294967296.0 - 0.5).astype(np.uint64).astype(np.uint32)


def test_unscrambled_codes_match_reference_dump(orc, golden_qmc):
    raw = orc.qmc_raw_codes(0, 1024, 12)
    assert np.array_equal(raw[:, :3], golden_qmc["q0_raw"])
    assert np.array_equal(raw[:256], golden_qmc["q2_raw"])


@pytest.mark.parametrize("seed", [12345, 777, 2024])
def test_stellar_stream_three_dims(orc, golden_qmc, seed):
    ref = golden_qmc[f"q0_scr_{seed}"]
    got = codes(orc.qmc_uniforms(seed, 1, 0, ref.shape[0], 3))
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("seed", [12345, 777, 2024, 55555, 999983])
def test_both_streams_twelve_dims(orc, golden_qmc, seed):
    for stream, key in ((1, f"q2_scr_{seed}"), (2, f"q2_dif_{seed}")):
        ref = golden_qmc[key]
        got = codes(orc.qmc_uniforms(seed, stream, 0, ref.shape[0], 12))
        assert np.array_equal(got, ref), key


def test_uniforms_strictly_inside_unit_interval(orc):
    u = orc.qmc_uniforms(12345, 1, 0, 4096, 12)
    assert (u > 0).all() and (u < 1).all()
    # (code + 0.5) 2^-32 is exact in FP64
    assert np.array_equal((codes(u).astype(np.float64) + 0.5) / 4294967296.0, u)


def test_unscrambled_net_equals_scipy_sobol_as_a_set(orc):
    # check_q0.py:31-41: the first 2^10 points of scipy's unscrambled Sobol
    # (same Joe-Kuo table) are the same set of integer codes.
    from scipy.stats import qmc
    n, d = 1024, 12
    s = qmc.Sobol(d=d, scramble=False, bits=32).random(n)
    ref = set(map(tuple, np.rint(s * 4294967296.0).astype(np.uint64).tolist()))
    got = set(map(tuple, orc.qmc_raw_codes(0, n, d).astype(np.uint64).tolist()))
    assert got == ref


def test_index_beyond_2_32_wraps(orc):
    # sobol_code uses the index modulo 2^32 (qmc_mod.f90:188-191)
    a = orc.qmc_uniforms(12345, 1, 5, 3, 4)
    b = orc.qmc_uniforms(12345, 1, 5 + 2**32, 3, 4)
    assert np.array_equal(a, b)


THR = [13.598, 24.383, 24.587, 54.418]


def test_band_clipped_tabulated_integral(orc):
    s = orc.Sampler.tabulated_band([10.0, 20.0, 110.0], [10.0, 20.0, 110.0], 13.598, 100.0)
    exact = 0.5 * (100.0**2 - 13.598**2)
    assert abs(s.total - exact) <= 2.0e-12 * s.total
    u = (np.arange(4096) + 0.5) / 4096
    assert np.max(np.abs(s.cdf(s.sample(u)) - u)) <= 2.0e-14


def test_tabulated_inverse_known_answers(orc):
    etab = np.array([13.598, 24.383, 24.587, 100.0])
    u = (np.arange(4096) + 0.5) / 4096
    const = orc.Sampler.tabulated(etab, np.ones(4))
    assert np.max(np.abs(const.sample(u) - (13.598 + u * (100.0 - 13.598)))) < 2e-13
    lin = orc.Sampler.tabulated(etab, 0.25 + 0.03 * (etab - etab[0]))
    # linear density f = a + b (E-E0): CDF inverse in closed form
    a, b = 0.25, 0.03
    tot = a * (100 - 13.598) + 0.5 * b * (100 - 13.598) ** 2
    x = (-a + np.sqrt(a * a + 2 * b * u * tot)) / b
    assert np.max(np.abs(lin.sample(u) - (13.598 + x))) < 2e-13 * 100
    broken = orc.Sampler.tabulated(etab, [0.2, 3.0, 0.4, 0.05])
    assert np.max(np.abs(broken.cdf(broken.sample(u)) - u)) <= 2e-14


@pytest.mark.parametrize("T", [2.0e4, 4.0e4])
def test_planck_sampler_quantiles_and_mean(orc, T):
    from scipy.integrate import quad
    from scipy.optimize import brentq
    kb = 8.617333262145e-5
    shape = lambda e: e**3 / np.expm1(e / (kb * T))
    norm = quad(shape, 13.598, 100.0, epsabs=0, epsrel=2e-12, points=THR[1:])[0]
    cdf = lambda e: quad(shape, 13.598, e, epsabs=0, epsrel=2e-12)[0] / norm
    s = orc.Sampler.planck(T, 13.598, 100.0, 1.0e-8, THR)
    e, f, c = s.tables()
    for t in THR:  # mandatory knots
        assert np.any(e == t)
    for q in (0.25, 0.5, 0.75):
        ref = brentq(lambda x: cdf(x) - q, 13.598, 100.0, xtol=1e-13)
        assert abs(s.sample(np.array([q]))[0] - ref) < 5e-8 * ref   # check_energy_sampler.py quantile tol
    mean = quad(lambda x: x * shape(x), 13.598, 100.0, epsabs=0, epsrel=2e-12)[0] / norm
    u = (np.arange(1 << 16) + 0.5) / (1 << 16)
    assert abs(s.sample(u).mean() - mean) < 3e-5 * mean


def test_rates_match_reference_python_mirror(orc, golden_rates):
    T = golden_rates["T"]
    for name in ("alphaA_HII", "alphaB_HII", "alpha1_HII", "alphaA_HeII", "alphaB_HeII", "alpha1_HeII",
                 "alphaA_HeIII", "alphaB_HeIII", "alpha1_HeIII", "ci_HI", "ci_HeI", "ci_HeII"):
        got = orc.evaluate(name, T)
        ref = golden_rates[name]
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0, err_msg=name)
    E = golden_rates["E"]
    for name in ("sigma_HI", "sigma_HeI", "sigma_HeII"):
        np.testing.assert_allclose(orc.evaluate(name, E), golden_rates[name], rtol=1e-10, atol=0, err_msg=name)


def test_cross_sections_at_thresholds(orc):
    # threshold values: hydrogenic sigma_0 = 6.3e-18/Z^2 exactly at E_th; zero below
    assert orc.evaluate("sigma_HI", [13.598])[0] == 6.30e-18
    assert orc.evaluate("sigma_HeII", [54.416])[0] == 6.30e-18 / 4
    assert orc.evaluate("sigma_HI", [13.5979])[0] == 0.0
    assert orc.evaluate("sigma_HeI", [24.586])[0] == 0.0


def test_aligned_band_edges(orc):
    nl = "&parameters par%nnu_ion = 16 par%eion_min=13.598 par%eion_max=100.0 par%tstar=4e4 par%luminosity=1e38 /"
    e = orc.band_edges(nl)
    # edges are exp(log(lo) + ...) as build_aligned_edges forms them, so a
    # threshold edge equals the threshold to rounding
    assert e.size == 17 and e[0] == 13.598 and abs(e[-1] - 100.0) < 1e-12
    for t in (24.587, 54.416):
        assert np.min(np.abs(e - t)) < 1e-12
    assert np.all(np.diff(e) > 0)
    # log-uniform inside each threshold segment
    for lo, hi in ((13.598, 24.587), (24.587, 54.416), (54.416, 100.0)):
        seg = e[(e >= lo) & (e <= hi)]
        d = np.diff(np.log(seg))
        assert np.allclose(d, d[0], rtol=1e-12)


def test_gaunt_table_matches_reference_nodes(orc, golden_rates):
    # cooling_mod's gbar_ff nodes (gaunt_ff_mean over the Hummer 1988
    # expansion, evaluated in single precision), dumped from the reference
    # build into tools/python/mochii_rates.py.  The expansion runs in REAL*4,
    # so two builds agree to single-precision rounding of the Chebyshev
    # recurrence, ~1e-5 relative.
    logT, z = orc.gff_table()
    assert np.array_equal(logT, golden_rates["gff_logT"])
    np.testing.assert_allclose(z, golden_rates["gff_z"], rtol=3e-5, atol=0)


def test_hi_nlevel_cooling_low_density_limit_equals_fit(orc):
    # the n-level H I cooling at n_e -> 0 is the ground-level excitation power
    # the cooling_h_1 fit represents (fit error 0.52%, cooling_h_1.txt header)
    import os
    from conftest import ROOT
    d = os.path.join(ROOT, "mochii_b200", "data", "atomic")
    rows = [l.split() for l in open(os.path.join(d, "cooling_h_1.txt")) if l.strip() and not l.startswith("#")]
    A = np.array([[float(x) for x in r] for r in rows[1:]])
    lib = orc.load()
    for T in (5e3, 1e4, 2e4, 5e4):
        lam = lib.orc_nlevel_cooling_at(os.path.join(d, "nlevel_h_1.txt").encode(), T, 1e-6)
        fit = np.sum(A[:, 0] * np.exp(-A[:, 1] / T)) / np.sqrt(T)
        assert abs(lam / fit - 1) < 6e-3, T


def test_g2a_1d_thermal_reference_matches_reference_script(orc):
    """The oracle's restatement of the G2a gate's 1D radial-marching thermal
    reference against reference_1d(nr=400) of check_g2a.py: T_e equal, the
    ion fractions within 1e-13."""
    import os
    from mochii_b200 import configs
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "g2a_1d_golden.npz"))
    o = orc.thermal_1d(configs.ATOMIC_DIR, nr=400)
    np.testing.assert_array_equal(o[0], g["r"])
    np.testing.assert_allclose(o[4], g["Te"], rtol=1e-12, atol=0)
    for i, k in ((1, "xHI"), (2, "xHeI"), (3, "xHeII")):
        np.testing.assert_allclose(o[i], g[k], rtol=0, atol=1e-13)
    inside = o[0] < 2.5
    assert 17e3 < o[4][inside].min() and o[4][inside].max() < 28e3   # the pure H/He overshoot
