"""Parity at the benchmark sizes: the headline H II region on the full
128^3 grid (FP32 segments, FP64 tallies, metal energy moments, diffuse Milne
packets, the coherent walk, the per-lane thermal solve) and the dusty
clumpy nebula on its full octree of about 3e6 leaves, each against the FP64
oracle with fewer packets so the oracle finishes.

Transport: the same packets on both sides (Sobol launch, Philox scattering
streams), so the rates differ by the FP32 segment arithmetic and, for a few
leaves, by diffuse packets that start in a neighbouring leaf (the device's
prefix sum of the leaf luminosities rounds differently from the sequential
sum); bars on the leaves carrying 99.9 % of each rate and on the totals.
Thermal update: the device state and rates before the update go to the
oracle, whose bisection solves a sample of the leaves (every 4th leaf of
the ionized region and its front, 20000 others); T_e within 20 K and x_HII
within 1e-3 on every sampled leaf."""
import numpy as np
import pytest

from mochii_b200 import Nebula, configs, parse_namelist
from test_gpu_metals import close_rel

pytestmark = pytest.mark.gpu


def copy_inputs(neb, sim):
    sim.set_state({f: neb.get(f) for f in ("x_HI", "x_HeI", "x_HeII", "n_e", "T_e")})
    fields = ["gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI", "heat_HeI", "heat_HeII"]
    if neb.metal_shape()[0]:
        fields += ["gamma_metal", "heat_metal"]
    for f in fields:
        sim.set(f, np.ascontiguousarray(neb.get(f)).ravel())


def check_update(neb, sim, rng):
    x, g = neb.get("x_HI"), neb.get("gamma_HI")
    front = np.flatnonzero((x < 0.99) | (g > 0.0))   # the ionized region, its front and every lit leaf
    idx = np.unique(np.concatenate([front[::max(4, front.size // 20000)], rng.choice(x.size, 20000, replace=False)]))
    copy_inputs(neb, sim)
    ref = sim.thermal_cells(idx)
    neb.gas_thermal_update()
    dT = np.abs(neb.get("T_e")[idx] - ref[:, 0])
    dx = np.abs(neb.get("x_HI")[idx] - ref[:, 1])
    assert front.size > 1000
    assert dT.max() < 20.0, dT.max()
    assert dx.max() < 1e-3, dx.max()


def test_hii_metals_128_matches_oracle():
    from oracle import pyorc
    n = 128
    nl = configs.hii_metals(nphotons=100000, niter=1, n=n, precision="fp32")
    neb = Nebula(parse_namelist(nl))
    sim = pyorc.Sim(nl.replace("'fp32'", "'fp64'"))
    state = configs.prepared_state(n)
    for k, v in state.items():
        neb.set(k, v)
    neb.gas_opacity_fill()
    sim.set_state(state)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    assert neb.nleaf == n ** 3 and st.closure <= 5e-13 and st.diffuse_packets == sim.diffuse_count
    e, _ = sim.energy()
    assert abs(st.energy_emitted / e[0] - 1) < 1e-12
    assert abs(st.energy_absorbed / e[1] - 1) < 1e-5
    for f in ("gamma_HI", "heat_HI", "gamma_HeI", "gamma_HeII", "gamma_metal", "heat_metal"):
        g, o = neb.get(f), sim.get(f)
        ok, worst = close_rel(g, o, 5e-5, frac=0.999)
        assert ok, (f, worst)
        assert abs(g.sum() / o.sum() - 1) < 1e-4, f
    check_update(neb, sim, np.random.default_rng(1))
    neb.close()


def test_clumpy_dusty_full_octree_matches_oracle(tmp_path):
    from oracle import pyorc
    nl = configs.clumpy_dusty(str(tmp_path), nphotons=100000, precision="fp32")
    neb = Nebula(parse_namelist(nl))
    sim = pyorc.Sim(nl.replace("'fp32'", "'fp64'"))
    assert neb.nleaf == sim.nleaf > 2_900_000
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    e, seg = sim.energy()
    assert st.closure <= 5e-13 and abs(st.energy_emitted / e[0] - 1) < 1e-12
    assert abs(st.energy_absorbed / e[1] - 1) < 1e-4
    assert abs(st.scattered_segments / seg[1] - 1) < 5e-3
    for f in ("gamma_HI", "gamma_HeI", "heat_dust", "g0_fuv"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-3 * o.max()
        assert np.median(np.abs(g[big] / o[big] - 1)) < 1e-4, f
        assert abs(g.sum() / o.sum() - 1) < 1e-3, f
    check_update(neb, sim, np.random.default_rng(2))
    neb.close()
