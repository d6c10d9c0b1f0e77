"""Host-side pieces of bench.py and of the workload generators (no GPU):
the workloads, the batched-nebulae instances, the algorithmic bytes per
segment used by the roofline, and the launch count."""
import importlib.util
import os

import pytest

from mochii_b200 import configs, parse_namelist

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    """The library (parse_namelist runs its namelist reader on the host)."""
    from mochii_b200 import _lib
    from mochii_b200.build import build
    build()
    return _lib.load()


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_workloads_build_their_namelists(bench, lib):
    for name in ("hii_metals128", "stromgren64"):
        wl = bench.Workload(name, grid=16, packets=1000)
        p = parse_namelist(wl.make(1000, "fp32", 7))
        assert p.nx == 16 and p.nphotons == 1000 and p.qmc_seed == 7
    wl = bench.Workload("batch64")
    assert wl.count == 64 and wl.nphot == 2_000_000 and wl.thermal
    with pytest.raises(SystemExit):
        bench.Workload("no_such_workload")


def test_batch_instances_are_seeded_and_in_range(lib):
    a, pa = configs.batch_instances(count=64)
    b, pb = configs.batch_instances(count=64)
    assert a == b and pa == pb
    assert len(a) == 64 and all(32 <= p["n"] <= 128 for p in pa)
    assert all(10.0 <= p["nH"] <= 1000.0 and 3.0e4 <= p["tstar"] <= 5.0e4 and 1e48 <= p["Q"] <= 1e50 for p in pa)
    assert len({p["n"] for p in pa}) > 20   # uneven sizes
    nl = parse_namelist(a[0])
    assert nl.nphotons == 2_000_000 and nl.solve_te == 1 and nl.caseA == 1
    leaves = sum(p["n"] ** 3 for p in pa)
    assert 3e7 < leaves < 6e7


def test_bytes_per_segment(bench):
    m = bench.Workload("hii_metals128", grid=16, packets=1000)
    # 4 FP32 state words, 7 FP64 tallies (6 H/He + spectrum) read and written,
    # 6 metal moments: FP32 (8 B) with FP64 tallies, FP64 otherwise
    assert bench.bytes_per_segment(m, "fp32", "fp64") == 4 * 4 + 16 * 7 + 8 * 6
    assert bench.bytes_per_segment(m, "fp32", "compensated") == 4 * 4 + 16 * 7 + 16 * 6
    assert bench.bytes_per_segment(m, "fp64") == 8 * 4 + 16 * 7 + 16 * 6
    s = bench.Workload("stromgren64", grid=16, packets=1000)
    assert bench.bytes_per_segment(s, "fp64") == 8 * 2 + 16 * 3


def test_launch_count(bench):
    m = bench.Workload("hii_metals128", grid=16, packets=10_000_000)
    # 3 chunks of <= 4 Mi packets: keys + launch + walk each (coherent
    # order), rates, metal rates, balance, diffuse luminosities, one diffuse
    # chunk
    assert bench.launches_per_step(m, 1_000_000) == 3 * 3 + 2 + 2 + 2
    assert bench.launches_per_step(m, 1_000_000, coherent=False) == 2 * 3 + 2 + 2 + 2


def test_prepared_state_is_a_developed_hii_region():
    """The analytic start state both bench arms use: deterministic, an
    ionized sphere of about 18 % of the box, charge balance in n_e."""
    import numpy as np
    a, b = configs.prepared_state(32), configs.prepared_state(32)
    for k in a:
        assert np.array_equal(a[k], b[k])
    x = a["x_HI"]
    assert x.size == 32 ** 3 and 0.15 < np.mean(x < 0.5) < 0.21
    assert x.min() >= 1e-3 and x.max() <= 1.0
    assert np.allclose(a["n_e"], 100.0 * ((1 - x) + 0.1 * a["x_HeII"]))
    assert a["T_e"].min() >= 3e3 - 1e-6 and a["T_e"].max() <= 8e3 + 1e-6
    s = configs.prepared_state(16, front=1.0, he=False, T_in=1e4, T_out=1e4)
    assert set(s) == {"x_HI", "T_e", "n_e"} and np.all(s["T_e"] == 1e4)


def test_reference_arm_measures_the_same_workload(bench, lib):
    """The reference arm (the oracle port on the host) times a measured
    fraction of the same step from the same analytic state: its config is
    the device arm's, and the sample's packet count includes the diffuse
    packets, as the device arm counts them."""
    wl = bench.Workload("hii_metals128", grid=12, packets=20000)
    assert bench.config_of(wl) == bench.config_of(wl) and "analytic" in bench.config_of(wl)["state"]
    v, desc, t_step, pk = bench.cpu_reference(wl, 2, steps=1, warmup=1)
    assert v > 0 and t_step > 0
    assert pk > 20000 // wl.cpu_fraction()   # stellar plus diffuse packets
    assert abs(v * t_step - pk) < 1e-6 * pk
