"""The bracketed cell solver (thermal_solver = 'bracketed') against the
reference's algorithm in the CPU oracle (damped n_e fixed point, bisection on
log T over [te_min, te_max]), through the C ABI.

Both find the same roots: n_e where the electrons the cell releases equal
n_e, and T_e where net heating vanishes.  Bars as for the reference solve:
T_e within 20 K and x_HII within 1e-3 of the FP64 oracle on the same
tallies, n_e within 1e-6 relative at fixed T_e; and the bracketed solve
uses fewer net-rate evaluations than the bisection on the same state.
"""
import numpy as np
import pytest

from mochii_b200 import Nebula, configs, parse_namelist

pytestmark = pytest.mark.gpu


def with_solver(nl, solver):
    return nl.replace("/\n", f" par%thermal_solver = '{solver}'\n/\n")


def partial_state(n, L):
    d = 2 * L / n
    c = (np.arange(n) + 0.5) * d - L
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z).ravel()
    xHI = np.clip(1e-4 + (r / (0.7 * L)) ** 6, 1e-4, 1.0)
    xHeI = np.clip(1.5 * xHI, 0.0, 1.0)
    return {"x_HI": xHI, "x_HeI": xHeI, "x_HeII": 1.0 - xHeI}


def run_pair(orc, nl, n, iters, thermal=True):
    neb = Nebula(parse_namelist(with_solver(nl, "bracketed")))
    sim = orc.Sim(nl)
    L = parse_namelist(nl).xmax
    st = partial_state(n, L)
    for k, v in st.items():
        neb.set(k, v)
        sim.set(k, v)
    ne = neb.get("nH") * ((1 - st["x_HI"]) + 0.1 * st["x_HeII"])
    neb.set("n_e", ne)
    sim.set("n_e", ne)
    neb.gas_opacity_fill()
    out = []
    for _ in range(iters):
        neb.ionizing_field_and_rates()
        sim.transport_pass()
        if thermal:
            neb.gas_thermal_update()
            sim.thermal_update()
        else:
            neb.gas_equilibrium_update()
            sim.equilibrium_update()
        out.append(neb.last_metrics.rate_evaluations)
        yield neb, sim


@pytest.mark.parametrize("metals", [False, True])
def test_bracketed_thermal_matches_oracle_bisection(orc, metals):
    if metals:
        n = 12
        nl = configs.hii_metals(nphotons=40000, niter=3, n=n, precision="fp64", rs_factor=1.3, diffuse=False)
    else:
        n = 24
        nl = configs.hii_thermal(nphotons=60000, niter=3, n=n, precision="fp64", rs_factor=1.2)
    for neb, sim in run_pair(orc, nl, n, 3):
        tg, to = neb.get("T_e"), sim.get("T_e")
        assert np.max(np.abs(tg - to)) < 20.0, np.max(np.abs(tg - to))
        assert np.max(np.abs(neb.get("x_HI") - sim.get("x_HI"))) < 1e-3
    neb.close()


def test_bracketed_equilibrium_matches_oracle(orc):
    n = 16
    nl = configs.hii_metals(nphotons=60000, niter=3, n=n, precision="fp64", rs_factor=1.3, diffuse=False,
                            solve_te=False)
    for neb, sim in run_pair(orc, nl, n, 3, thermal=False):
        assert np.max(np.abs(neb.get("x_HI") - sim.get("x_HI"))) < 1e-3
        np.testing.assert_allclose(neb.get("n_e"), sim.get("n_e"), rtol=1e-6)
    neb.close()


def test_bracketed_solve_needs_fewer_evaluations():
    """Same tallies and state, the two solvers: evaluations of net(T) and
    the metal cascade sums, and the T_e they reach."""
    n = 24
    nl = configs.hii_metals(nphotons=100000, niter=3, n=n, precision="fp64", rs_factor=1.2, diffuse=False)
    res = {}
    for solver in ("bisection", "bracketed"):
        neb = Nebula(parse_namelist(with_solver(nl, solver)))
        for _ in range(2):
            neb.ionizing_field_and_rates()
            neb.gas_thermal_update()
        m = neb.last_metrics
        res[solver] = (m.rate_evaluations, m.metal_sum_calls, neb.get("T_e"))
        neb.close()
    assert res["bracketed"][0] < 0.7 * res["bisection"][0], (res["bracketed"][0], res["bisection"][0])
    assert res["bracketed"][1] < 0.7 * res["bisection"][1]
    assert np.max(np.abs(res["bracketed"][2] - res["bisection"][2])) < 20.0


def test_cell_layouts_agree():
    """The thermal solve with metals in its four layouts -- warp-uniform root
    loops ('lockstep'), per-lane root machines with the metal cache in shared
    memory ('lane', the default), each leaf's solve a state machine served
    by warp-wide evaluations ('flow'), one warp per leaf ('warp') -- make the
    same solves per leaf.  Separate runs accumulate the transport tallies
    in different atomic orders, so the rates differ in their last bits and a
    leaf's T_e can move by a fraction of a kelvin where net(T) is flat."""
    n = 16
    nl = with_solver(configs.hii_metals(nphotons=60000, niter=2, n=n, precision="fp64", rs_factor=1.3,
                                        diffuse=False), "bracketed")
    out = {}
    for layout in ("lockstep", "lane", "flow", "warp"):
        neb = Nebula(parse_namelist(nl.replace("/\n", f" par%cell_layout = '{layout}'\n/\n")))
        st = partial_state(n, parse_namelist(nl).xmax)
        for k, v in st.items():
            neb.set(k, v)
        neb.gas_opacity_fill()
        for _ in range(2):
            neb.ionizing_field_and_rates()
            neb.gas_thermal_update()
        out[layout] = (neb.get("T_e"), neb.get("x_HI"), neb.last_metrics.rate_evaluations)
        neb.close()
    for other in ("lane", "flow", "warp"):
        dT = np.abs(out[other][0] - out["lockstep"][0])
        assert np.median(dT) < 1e-6 and dT.max() < 1.0, (other, dT.max())
        assert np.max(np.abs(out[other][1] - out["lockstep"][1])) < 1e-5
        assert abs(out[other][2] / out["lockstep"][2] - 1) < 0.01


def test_lane_layout_refills_lanes():
    """The per-lane layout on more leaves than the device has lanes (each
    lane solves several leaves, claimed as it frees) and with the reference's
    one-way charge exchange (no H root iteration): the same solves as the
    lockstep layout, every leaf written once."""
    n = 44
    for cx in ("two_way", "one_way"):
        nl = with_solver(configs.hii_metals(nphotons=200000, niter=2, n=n, precision="fp64", rs_factor=1.3,
                                            diffuse=False), "bracketed")
        nl = nl.replace("/\n", f" par%charge_exchange = '{cx}'\n/\n")
        out = {}
        for layout in ("lockstep", "lane"):
            neb = Nebula(parse_namelist(nl.replace("/\n", f" par%cell_layout = '{layout}'\n/\n")))
            st = partial_state(n, parse_namelist(nl).xmax)
            for k, v in st.items():
                neb.set(k, v)
            neb.gas_opacity_fill()
            for _ in range(2):
                neb.ionizing_field_and_rates()
                neb.gas_thermal_update()
            m = neb.last_metrics
            out[layout] = (neb.get("T_e"), neb.get("x_HI"), m.rate_evaluations, m.cells_solved, m.metal_sum_calls,
                           neb.get("n_e"))
            neb.close()
        a_, b_ = out["lockstep"], out["lane"]
        assert b_[3] == a_[3] == n ** 3
        dT = np.abs(b_[0] - a_[0])
        assert np.median(dT) < 1e-6 and dT.max() < 1.0, (cx, dT.max())
        assert np.max(np.abs(b_[1] - a_[1])) < 1e-5
        # n_e where hydrogen is ionized, to the T root's tolerance (1e-5 in
        # ln T); in neutral leaves n_e ~ n_H (1 - x_HI) ~ 1e-9 n_H sits below
        # the H root's resolution and differs between root paths by percents
        ion = a_[1] < 0.99
        assert ion.sum() > 1000
        assert np.max(np.abs(b_[5][ion] / a_[5][ion] - 1)) < 1e-4
        # the same temperature trials; the per-lane H root starts from the
        # extrapolation of its last two n_e evaluations, so it needs fewer sums
        assert abs(b_[2] / a_[2] - 1) < 0.01 and b_[4] <= 1.01 * a_[4]


def test_metal_rate_table_matches_exact():
    """The thermal solve with the interpolated T table of the metal rate
    coefficients against every coefficient evaluated directly, on the same
    nebula: T_e and x_HI agree to the table's interpolation error (up to
    rate-bit differences between separate runs)."""
    n = 16
    nl = with_solver(configs.hii_metals(nphotons=60000, niter=2, n=n, precision="fp64", rs_factor=1.3,
                                        diffuse=False), "bracketed")
    out = {}
    for mode in ("table", "exact"):
        neb = Nebula(parse_namelist(nl.replace("/\n", f" par%metal_rates = '{mode}'\n/\n")))
        st = partial_state(n, parse_namelist(nl).xmax)
        for k, v in st.items():
            neb.set(k, v)
        neb.gas_opacity_fill()
        for _ in range(2):
            neb.ionizing_field_and_rates()
            neb.gas_thermal_update()
        out[mode] = (neb.get("T_e"), neb.get("x_HI"))
        neb.close()
    dT = np.abs(out["table"][0] - out["exact"][0])
    assert np.median(dT) < 1e-6 and dT.max() < 1.0, dT.max()
    assert np.max(np.abs(out["table"][1] - out["exact"][1])) < 1e-5


def test_autotune_picks_a_cell_tile_and_keeps_the_state():
    """The autotuner's thermal trials (lanes per block of the per-lane solve)
    restore the state they start from, and the solve with any tile gives the
    same leaves."""
    n = 20
    nl = with_solver(configs.hii_metals(nphotons=60000, niter=2, n=n, precision="fp32", rs_factor=1.3,
                                        diffuse=False), "bracketed")
    neb = Nebula(parse_namelist(nl))
    st = partial_state(n, parse_namelist(nl).xmax)
    for k, v in st.items():
        neb.set(k, v)
    neb.gas_opacity_fill()
    before = {f: neb.get(f) for f in ("x_HI", "x_HeI", "x_HeII", "T_e", "n_e")}
    t = neb.autotune(20000)
    assert t["lane_threads"] in (0, 192, 160, 128, 96) and t["thermal_ms"] > 0
    for f, v in before.items():
        assert np.array_equal(neb.get(f), v), f
    neb.close()
    # the same update with two cell tiles, each on a fresh nebula (the metal
    # stage weights of an opacity fill depend on the last pass's metal rates,
    # which the trial passes overwrite)
    out = {}
    for lanes in (0, 96):
        nb = Nebula(parse_namelist(nl))
        nb.set_tuning(t["lookahead"], t["walk_blocks_per_sm"], lanes)
        for k, v in st.items():
            nb.set(k, v)
        nb.gas_opacity_fill()
        nb.ionizing_field_and_rates()
        nb.gas_thermal_update()
        out[lanes] = (nb.get("T_e"), nb.get("x_HI"))
        nb.close()
    dT = np.abs(out[0][0] - out[96][0])
    assert np.median(dT) < 1e-6 and dT.max() < 1.0, dT.max()
    assert np.max(np.abs(out[0][1] - out[96][1])) < 1e-5
