"""Plane-parallel slab illumination on the device (source_geometry 'slab',
par%xy_periodic) against the oracle and the reference's slab gates
(tests/slab/check_slab.py):

* launch records of the slab emitter (emit_slab_qmc, ion_band_mod.f90:
  2183-2208) -- energies, bins and entry points bit-exact, directions within
  the last ulp of cos/sin -- for beams, Lambert faces and both faces lit;
* FP64 passes through the periodic walks (the DDA's index wrap and the
  octree walk's face wrap, raytrace_amr.f90:330-345, 473-481, 575-588) and
  the boundary tally (slab_bnd_add, jtally_mod.f90:76-86): rates and every
  mu bin to the last bits of the FP64 sums, the budget closing;
* with dust scattering, the reflected light of the scattered flights;
* the gates at the reference's 4e6 packets with FP32 segments: the normal
  and oblique transmission against the quadrature of the source spectrum
  through the column, the DDA and octree walks and the nx = 1 and nx = 2
  tiles agreeing to 1e-4, the budget closing to 1e-4 in the written
  <base>_slab_Imu.txt, and the grazing-ray step guard silent."""
import re

import numpy as np
import pytest

from mochii_b200 import Nebula, configs, parse_namelist
from test_oracle_dust import dusty
from test_oracle_slab import NMU, quad_transmission

pytestmark = pytest.mark.gpu

CASES = {
    "beam60": dict(theta=60.0, phi=30.0),
    "iso": dict(mode="isotropic"),
    "both": dict(faces="both", mode="isotropic", bot=("beam", 30.0, 1e-5)),
    "bottom": dict(faces="bottom", bot=("isotropic", 0.0, 2e-5)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_slab_launch_matches_oracle(orc, case):
    nl = configs.slab(nphotons=8192, **CASES[case])
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl, nthreads=1)
    n = 8192
    rec = neb.launch_records(0, n)
    ref = np.array([sim.photon(i) for i in range(n)])
    assert np.array_equal(rec[:, 6], ref[:, 6]) and np.array_equal(rec[:, 7], ref[:, 7])
    assert np.array_equal(rec[:, :3], ref[:, :3])
    np.testing.assert_allclose(rec[:, 3:6], ref[:, 3:6], rtol=0, atol=4e-16)
    neb.close()


@pytest.mark.parametrize("case,extra", [("beam60", {}), ("beam60", dict(car_walk="amr")), ("beam60", dict(nx=2)),
                                        ("iso", {}), ("iso", dict(car_walk="amr", nx=2)), ("both", {}),
                                        ("bottom", dict(nnu=8))])
def test_slab_pass_fp64_matches_oracle(orc, case, extra):
    kw = dict(CASES[case], **extra)
    nl = configs.slab(nphotons=50000, **kw)
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    e, _ = sim.energy()
    assert st.closure <= 5e-13 and abs(st.energy_absorbed / e[1] - 1) < 1e-12 and st.walk_kills == 0
    top, bot, lin, az = neb.slab_tally()
    otop, obot = sim.slab_tally(NMU)
    assert abs(lin / sim.ion_Ltot - 1) < 1e-14
    for g, o in ((top, otop), (bot, obot)):
        assert np.array_equal(g > 0, o > 0)
        np.testing.assert_allclose(g, o, rtol=1e-11, atol=0)
    assert abs((top.sum() + bot.sum() + st.energy_absorbed) / lin - 1) < 1e-11
    for f in ("gamma_HI", "heat_HI"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-6 * o.max()
        assert big.sum() > 10 and np.max(np.abs(g[big] / o[big] - 1)) < 1e-9, f
    neb.close()


def test_slab_scattering_reflects(orc):
    """Grains that scatter send part of the beam back out of the lit face:
    the scattered flights' z-face escapes (raytrace_amr.f90:407-413,
    655-660) against the oracle's."""
    nl = configs.slab(nphotons=50000, theta=30.0, nH=0.01, nnu=4)
    nl = dusty(nl.replace("par%dust_density_law = 'none'", "par%dust_density_law = 'global_dgr'"),
               scatter=True, dgr=2000.0)
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    top, bot, lin, _ = neb.slab_tally()
    otop, obot = sim.slab_tally(NMU)
    assert otop.sum() > 1e-3 * lin and st.scattered_segments > 0
    assert abs(top.sum() / otop.sum() - 1) < 1e-3 and abs(bot.sum() / obot.sum() - 1) < 1e-3
    assert np.count_nonzero(top) > NMU // 2   # reflected light spreads over mu
    neb.close()


def imu_fractions(path):
    frac = {}
    with open(path) as fh:
        for ln in fh:
            m = re.search(r"#\s*(L_\w+).*fraction\s*=\s*([-\d.Ee+]+)", ln)
            if m:
                frac[m.group(1)] = float(m.group(2))
    return frac


def gate_run(tmp_path, name, **kw):
    neb = Nebula(parse_namelist(configs.slab(nphotons=4_000_000, precision="fp32", **kw)))
    st = neb.ionizing_field_and_rates()
    assert st.walk_kills == 0   # the grazing-ray guard stays silent
    path = neb.write_slab_imu(str(tmp_path / name))
    top, bot, lin, az = neb.slab_tally()
    data = np.loadtxt(path)
    mu = (np.arange(NMU) + 0.5) / NMU
    np.testing.assert_allclose(data[:, 0], np.round(mu, 5))
    np.testing.assert_allclose(data[:, 2], bot / (az * 2 * np.pi * mu / NMU), rtol=1e-7)
    neb.close()
    return imu_fractions(path), bot.sum() / lin


def test_slab_gates_fp32(tmp_path):
    f0, T0 = gate_run(tmp_path, "ga_beam_n1_dda")
    assert abs(T0 - quad_transmission(1.0)) < 2e-3 and f0["L_escape_top"] < 1e-3
    f60, T60 = gate_run(tmp_path, "ga60_n1_dda", theta=60.0)
    assert abs(T60 - quad_transmission(0.5)) < 2e-3
    _, T60s = gate_run(tmp_path, "ga60_n1_sh", theta=60.0, car_walk="amr")
    _, T60n2 = gate_run(tmp_path, "ga60_n2_dda", theta=60.0, nx=2)
    assert abs(T60 - T60s) < 1e-4 and abs(T60 - T60n2) < 1e-4
    fi, _ = gate_run(tmp_path, "ga_iso_n1", mode="isotropic")
    fb, _ = gate_run(tmp_path, "ga_both", faces="both", bot=("beam", 0.0, 1e-5))
    for f in (f0, f60, fi, fb):
        assert abs(f["L_escape_top"] + f["L_escape_bottom"] + f["L_absorbed"] - 1.0) < 1e-4
    assert "L_reflected" in f0 and "L_reflected" not in fb
