"""GPU parity of the trace-metal path (species_mod.f90 and its callers)
against the CPU oracle, through the C ABI.

Bars: the band edges with the metal thresholds equal the oracle's; in FP64
with the per-transition tallies the metal Gamma and photoheating per (leaf,
transition) equal the oracle's to 1e-9 relative (atomic ordering and
last-ulp differences of pow/exp); the energy-moment tallies (degree-5
Chebyshev interpolation per threshold-aligned bin, 2e-7 of the bin's peak)
within 2e-6 of the per-transition ones on the same packets;
the H/He rates with the metal opacity in the packet absorption to 1e-9;
after the balance (fixed T_e, metal electrons, two-way charge exchange) the
x_HII within 1e-3 and the metal stage fractions within 1e-6 absolute of the
oracle's on the same tallies; after the thermal balance T_e within 20 K;
FP32 segments with compensated tallies within 5e-5 relative on the leaves
holding 99.9% of each rate.
"""
import numpy as np
import pytest

from mochii_b200 import Nebula, configs, parse_namelist

pytestmark = pytest.mark.gpu


def metal_nl(n=16, nphot=40000, precision="fp64", solve_te=False, diffuse=False, rs_factor=1.3, tally="exact"):
    nl = configs.hii_metals(nphotons=nphot, niter=3, n=n, precision=precision, rs_factor=rs_factor,
                            diffuse=diffuse, solve_te=solve_te)
    return nl.replace("/\n", f" par%metal_tally = '{tally}'\n/\n")


def partial_state(n, L):
    d = 2 * L / n
    c = (np.arange(n) + 0.5) * d - L
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z).ravel()
    xHI = np.clip(1e-4 + (r / (0.7 * L)) ** 6, 1e-4, 1.0)
    xHeI = np.clip(1.5 * xHI, 0.0, 1.0)
    return {"x_HI": xHI, "x_HeI": xHeI, "x_HeII": 1.0 - xHeI}


def pair(orc, nl, state):
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    for k, v in state.items():
        neb.set(k, v)
        sim.set(k, v)
    ne = neb.get("nH") * ((1 - state["x_HI"]) + 0.1 * state["x_HeII"])
    neb.set("n_e", ne)
    sim.set("n_e", ne)
    neb.gas_opacity_fill()
    return neb, sim


def close_rel(g, o, rtol, frac=1.0):
    """Every leaf (frac=1) or the leaves carrying the top `frac` of the total."""
    g, o = np.ravel(g), np.ravel(o)
    if frac < 1.0:
        idx = np.argsort(o)[::-1]
        cum = np.cumsum(o[idx])
        keep = idx[: np.searchsorted(cum, frac * cum[-1]) + 1]
        g, o = g[keep], o[keep]
    scale = np.abs(o).max()
    bad = np.abs(g - o) > rtol * np.abs(o) + 1e-30 * scale
    return not bad.any(), (np.abs(g - o) / np.maximum(np.abs(o), 1e-300)).max()


def test_band_edges_include_metal_thresholds(orc):
    nl = metal_nl()
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    np.testing.assert_array_equal(neb.get("eedge"), sim.get("eedge"))
    ntr, nst = neb.metal_shape()
    assert (ntr, nst) == (sim.metal_ntr, sim.metal_nstage) == (32, 43)
    neb.close()


def test_fp64_metal_pass_matches_oracle(orc):
    n = 16
    nl = metal_nl(n=n)
    L = parse_namelist(nl).xmax
    neb, sim = pair(orc, nl, partial_state(n, L))
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    assert st.closure <= 5e-13
    e, _ = sim.energy()
    assert abs(st.energy_absorbed / e[1] - 1) < 1e-9
    for f in ("gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI"):
        ok, worst = close_rel(neb.get(f), sim.get(f), 1e-9)
        assert ok, (f, worst)
    for f in ("gamma_metal", "heat_metal"):
        g, o = neb.get(f), sim.get(f)
        assert g.shape == o.shape == (n ** 3, 32)
        assert np.count_nonzero(o) > 0.5 * o.size
        ok, worst = close_rel(g, o, 1e-9)
        assert ok, (f, worst)
    neb.close()


def test_metal_balance_matches_oracle(orc):
    """gas_equilibrium_update with metal_ne and the two-way charge exchange,
    then gas_opacity_fill, on identical tallies (FP64 pass)."""
    n = 16
    nl = metal_nl(n=n, nphot=60000)
    L = parse_namelist(nl).xmax
    neb, sim = pair(orc, nl, partial_state(n, L))
    for _ in range(3):
        neb.ionizing_field_and_rates()
        sim.transport_pass()
        mg = neb.gas_equilibrium_update()
        mo = sim.equilibrium_update()
        assert abs(mg[0] - mo[0]) < 1e-6
        assert np.max(np.abs(neb.get("x_HI") - sim.get("x_HI"))) < 1e-3
    np.testing.assert_allclose(neb.get("n_e"), sim.get("n_e"), rtol=1e-6)
    xg, xo = neb.get("x_metal"), sim.get("x_metal")
    assert np.max(np.abs(xg - xo)) < 1e-6
    neb.close()


def test_metal_thermal_matches_oracle(orc):
    """gas_thermal_update with the metal cooling (fits under the n-level
    suppression), H-impact [C II]/[O I], metal free-free and photoheating."""
    n = 12
    nl = metal_nl(n=n, nphot=40000, solve_te=True)
    L = parse_namelist(nl).xmax
    neb, sim = pair(orc, nl, partial_state(n, L))
    for _ in range(2):
        neb.ionizing_field_and_rates()
        sim.transport_pass()
        mg = neb.gas_thermal_update()
        mo = sim.thermal_update()
        tg, to = neb.get("T_e"), sim.get("T_e")
        assert np.max(np.abs(tg - to)) < 20.0, np.max(np.abs(tg - to))
        assert np.max(np.abs(neb.get("x_HI") - sim.get("x_HI"))) < 1e-3
        assert abs(mg[1] - mo[1]) < 1e-3
    t = neb.get("T_e")
    assert 3.0e3 <= t.min() and t.max() <= 3.0e4
    neb.close()


def test_moment_tallies_match_exact_tallies():
    n = 16
    L = parse_namelist(metal_nl(n=n)).xmax
    out = {}
    for tally in ("exact", "moments"):
        neb = Nebula(parse_namelist(metal_nl(n=n, tally=tally)))
        for k, v in partial_state(n, L).items():
            neb.set(k, v)
        neb.gas_opacity_fill()
        neb.ionizing_field_and_rates()
        out[tally] = (neb.get("gamma_metal"), neb.get("heat_metal"), neb.get("gamma_HI"))
        neb.close()
    for i in range(3):
        ok, worst = close_rel(out["moments"][i], out["exact"][i], 2e-6)
        assert ok, (i, worst)


@pytest.mark.parametrize("tally,order", [("exact", "launch"), ("moments", "launch"), ("exact", "coherent"),
                                         ("moments", "coherent")])
def test_fp32_metal_pass_within_tolerance(orc, tally, order):
    n = 16
    nl = metal_nl(n=n, precision="fp32", tally=tally).replace("/\n", f" par%packet_order = '{order}'\n/\n")
    L = parse_namelist(nl).xmax
    neb, sim = pair(orc, nl, partial_state(n, L))
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    assert st.closure <= 5e-13
    for f in ("gamma_HI", "gamma_metal", "heat_metal"):
        g, o = neb.get(f), sim.get(f)
        ok, worst = close_rel(g, o, 5e-5, frac=0.999)
        assert ok, (f, worst)
        assert abs(g.sum() / o.sum() - 1) < 1e-5, f
    neb.close()


def test_metal_pass_with_diffuse_and_thermal_runs_clean():
    """The full metals workload shape (diffuse Milne packets, thermal balance,
    FP32 transport) on a small grid: closure, finite state, bounded T_e."""
    nl = configs.hii_metals(nphotons=100000, niter=3, n=24, precision="fp32", rs_factor=1.2)
    neb = Nebula(parse_namelist(nl))
    for it in range(3):
        st = neb.ionizing_field_and_rates()
        assert st.closure <= 5e-13
        assert it == 0 or st.diffuse_packets > 0   # the neutral start has no recombinations
        neb.gas_thermal_update()
    t, x = neb.get("T_e"), neb.get("x_HI")
    assert np.isfinite(t).all() and np.isfinite(x).all()
    # the cells inside half the Stromgren radius are photo-heated by the star
    # (outer cells of the ionized start are held ionized by the diffuse field,
    # whose photons sit just above 13.6 eV and heat little, and settle at te_min)
    n, L = 24, parse_namelist(nl).xmax
    c = (np.arange(n) + 0.5) * (2 * L / n) - L
    z, y, xx = np.meshgrid(c, c, c, indexing="ij")
    inner = (np.sqrt(xx * xx + y * y + z * z) < 0.5 * L / 1.2).ravel()
    assert inner.sum() > 100 and np.median(t[inner]) > 5.0e3
    xm = neb.get("x_metal")
    assert np.allclose(xm.sum(axis=1), 11.0, atol=1e-9)   # each element's stages sum to 1
    neb.close()
