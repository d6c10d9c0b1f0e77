"""Grains, the FUV band and dust scattering on the device against the oracle,
through the C ABI:

* the scattered flights' Philox stream: device draws bit-exact with the
  oracle's (so the device and the oracle make the same draws per packet);
* FP64 passes with grain absorption and the FUV band, on the Cartesian grid
  and the octree: Gamma, heating, heat_dust and G0 within 1e-9 of the oracle,
  the energy ledger within 1e-12;
* FP64 passes with scattering (forced first interaction, albedo weights,
  roulette, Henyey-Greenstein flights): the same streams, so the device
  follows the oracle's packets except where last-bit differences of exp/log/
  sin/cos move an interaction across a face -- leaf rates agree to 1e-6 at
  the median and 1e-4 in total, scattered segment counts to 0.5 %;
* FP32 segments with scattering within Monte Carlo noise of the FP64 oracle.
"""
import numpy as np
import pytest

from conftest import octree_leaf_list
from mochii_b200 import Nebula, configs, parse_namelist
from mochii_b200.host import philox_uniforms
from test_oracle_dust import KEXT, dusty

pytestmark = pytest.mark.gpu


def ionized(neb, sim, xhi=1e-3):
    for obj in (neb, sim):
        obj.set("x_HI", np.full(neb.nleaf, xhi))
    neb.gas_opacity_fill()


def test_philox_stream_matches_oracle(orc):
    for seed, stream, packet, n0 in [(0, 0, 0, 0), (77, 0, 12345, 3), (-5, 1, 2 ** 33 + 7, 0), (2024, 1, 999, 101)]:
        d = philox_uniforms(seed, stream, packet, n0, 64)
        o = orc.philox(seed & (2 ** 64 - 1), stream, packet, n0, 64)
        np.testing.assert_array_equal(d, o)


@pytest.fixture(scope="module")
def leaf_file(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("dust") / "leaves.txt")
    box = 2.0 * configs.stromgren_radius_pc(Q=5.0e49)
    octree_leaf_list(path, box, base_level=3, max_level=5, p_split=0.3, seed=13)
    return path


def pair(orc, nl):
    return Nebula(parse_namelist(nl)), orc.Sim(nl)


@pytest.mark.parametrize("grid", ["car", "amr"])
def test_grain_absorption_and_fuv_fp64_match_oracle(orc, leaf_file, grid):
    base = configs.hhe128(nphotons=150000, niter=1, n=12, precision="fp64")
    if grid == "amr":
        base = configs.on_octree(base, leaf_file)
    nl = dusty(base, fuv=True, dgr=0.05)
    neb, sim = pair(orc, nl)
    ionized(neb, sim)
    np.testing.assert_allclose(neb.get("rhokap"), sim.get("rhokap"), rtol=1e-15)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    e, _ = sim.energy()
    assert abs(st.energy_emitted / e[0] - 1) < 1e-12 and abs(st.energy_absorbed / e[1] - 1) < 1e-12
    for f in ("gamma_HI", "heat_HI", "gamma_HeI", "heat_dust", "g0_fuv"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-12 * o.max()
        assert big.sum() >= 5, f
        assert np.max(np.abs(g[big] / o[big] - 1)) < 1e-9, f
    neb.close()


@pytest.mark.parametrize("grid", ["car", "amr"])
def test_scattering_fp64_follows_oracle(orc, leaf_file, grid):
    base = configs.hhe128(nphotons=100000, niter=1, n=12, precision="fp64")
    if grid == "amr":
        base = configs.on_octree(base, leaf_file)
    nl = dusty(base, scatter=True, fuv=True, dgr=0.05)
    neb, sim = pair(orc, nl)
    ionized(neb, sim)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    e, seg = sim.energy()
    assert abs(st.energy_absorbed / e[1] - 1) < 1e-12   # the first flights
    assert seg[1] > 0.2 * seg[0]
    assert abs(st.scattered_segments / seg[1] - 1) < 5e-3
    for f in ("gamma_HI", "heat_HI", "heat_dust", "g0_fuv"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-3 * o.max()
        assert np.median(np.abs(g[big] / o[big] - 1)) < 1e-6, f
        assert abs(g.sum() / o.sum() - 1) < 1e-4, f
    neb.close()


def test_scattering_fp32_within_mc_noise(orc):
    base = configs.hhe128(nphotons=200000, niter=1, n=12, precision="fp64")
    nl = dusty(base, scatter=True, dgr=0.05)
    sim = orc.Sim(nl)
    sim.set("x_HI", np.full(sim.nleaf, 1e-3))
    sim.transport_pass()
    neb = Nebula(parse_namelist(nl.replace("'fp64'", "'fp32'")))
    neb.set("x_HI", np.full(neb.nleaf, 1e-3))
    neb.gas_opacity_fill()
    neb.ionizing_field_and_rates()
    for f in ("gamma_HI", "heat_dust"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-2 * o.max()
        assert np.median(np.abs(g[big] / o[big] - 1)) < 1e-3, f
        assert abs(g.sum() / o.sum() - 1) < 1e-3, f
    neb.close()


def test_grain_settings_errors(tmp_path):
    from mochii_b200 import MochiiError
    base = configs.stromgren64(nphotons=1000, niter=1, n=8)
    with pytest.raises(MochiiError, match="cannot open"):
        Nebula(parse_namelist(dusty(base).replace(KEXT, str(tmp_path / "none.txt"))))
    with pytest.raises(MochiiError) as ei:
        Nebula(parse_namelist(dusty(base).replace("/\n", " par%taumax = 2.0\n/\n")))
    assert ei.value.status == 8


def test_clumpy_dusty_case_matches_oracle(orc, tmp_path):
    """The dusty clumpy nebula at a reduced size (64^3 field, octree levels
    4-6): three sources on the octree, FUV band, grain absorption and
    scattering, then the thermal update, FP64 on both sides."""
    nl = configs.clumpy_dusty(str(tmp_path), nphotons=200000, base_level=4, max_level=6, field_n=64,
                              precision="fp64")
    neb, sim = pair(orc, nl)
    assert neb.nleaf == sim.nleaf > 3000
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    e, seg = sim.energy()
    assert abs(st.energy_emitted / e[0] - 1) < 1e-12 and abs(st.energy_absorbed / e[1] - 1) < 1e-12
    assert abs(st.scattered_segments / seg[1] - 1) < 5e-3
    for f in ("gamma_HI", "gamma_HeI", "heat_dust", "g0_fuv"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-3 * o.max()
        assert np.median(np.abs(g[big] / o[big] - 1)) < 1e-6, f
        assert abs(g.sum() / o.sum() - 1) < 1e-4, f
    # the thermal update on every leaf: the device state and rates before it
    # go to the oracle, whose bisection must agree with the device solve
    sim.set_state({f: neb.get(f) for f in ("x_HI", "x_HeI", "x_HeII", "n_e", "T_e")})
    for f in ("gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI", "heat_HeI", "heat_HeII"):
        sim.set(f, neb.get(f))
    ref = sim.thermal_cells(np.arange(neb.nleaf))
    neb.gas_thermal_update()
    gas = neb.get("nH") > 0
    dT = np.abs(neb.get("T_e") - ref[:, 0])[gas]
    dx = np.abs(neb.get("x_HI") - ref[:, 1])[gas]
    assert dT.max() < 20.0, dT.max()
    assert dx.max() < 1e-3, dx.max()
    neb.close()


@pytest.mark.parametrize("grid", ["car", "amr"])
def test_dust_temperature_and_ir_spectrum_match_oracle(orc, leaf_file, grid, tmp_path):
    """The equilibrium dust temperature (dust_temp_mod.f90) from the same
    pass's grain heating: every leaf within one bisection interval (1e-5 in
    T) of the oracle's, the IR spectrum and absorbed power within 1e-6, the
    integrated IR within a few percent of the absorbed power (the 1-1000 um
    window cuts the tails), T_dust in the rates file and the _dustir.txt
    file as the reference writes them."""
    base = configs.hhe128(nphotons=150000, niter=1, n=12, precision="fp64")
    if grid == "amr":
        base = configs.on_octree(base, leaf_file)
    nl = dusty(base, fuv=True, dgr=0.05)
    neb, sim = pair(orc, nl)
    ionized(neb, sim)
    neb.ionizing_field_and_rates()
    sim.transport_pass()
    np.testing.assert_allclose(neb.get("heat_dust"), sim.get("heat_dust"), rtol=1e-9, atol=0)
    sim.set("heat_dust", np.ascontiguousarray(neb.get("heat_dust")))   # the same input on both sides
    td_o, lam_o, lnu_o, labs_o = sim.dust_temp()
    td = neb.get("T_dust")
    lit = td_o > 0
    assert lit.sum() > 100 and np.array_equal(td > 0, lit)
    assert np.max(np.abs(td[lit] / td_o[lit] - 1)) < 1.1e-5
    assert np.median(np.abs(td[lit] / td_o[lit] - 1)) < 1e-12
    assert 3.0 < td[lit].min() and td[lit].max() < 3200.0
    lam, lnu, labs, lir = neb.dust_ir()
    np.testing.assert_allclose(lam, lam_o, rtol=1e-15)
    np.testing.assert_allclose(lnu, lnu_o, rtol=1e-6, atol=1e-12 * lnu_o.max())
    assert abs(labs / labs_o - 1) < 1e-10
    assert 0.9 < lir / labs < 1.01
    d = neb.write_rates(str(tmp_path / "dusty"))
    np.testing.assert_array_equal(np.load(d + "/T_dust.npy"), td)
    path = neb.write_dust_ir(str(tmp_path / "dusty"))
    rows = np.loadtxt(path)
    assert rows.shape == (240, 2)
    np.testing.assert_allclose(rows[:, 1], lnu, rtol=1e-6)
    head = open(path).read().splitlines()[1]
    assert head.startswith("# L_abs(dust) =") and "ratio =" in head
    neb.close()
