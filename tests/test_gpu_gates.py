"""End-to-end gates of the thermal balance against the reference's own gates
and published results.

G2a (tests/g2a_thermal/g2a_thermal.in, check_g2a.py): a uniform n_H = 100
H/He sphere of 4 pc around a 40 kK star with Q(H) = 1e49 s^-1, case B, T_e
from heating = cooling, iterated to convergence on the level-6 octree.  The
gate is the reference's: the median |T_e / T_e,1D - 1| over the leaves with
0.3 < r < 2.8 pc and n_e > 0 below 1 %, where T_e,1D is the 1D
radial-marching reference of check_g2a.py restated in the oracle (pinned to
the reference's own script in test_oracle_golden.py) and read at each leaf
centre from the rates file the run writes.

HII40 (the Lexington benchmark): the reference publishes the mean electron
temperature weighted by n_p n_e, <T[NpNe]> = 8169 K, for its production
input (tests/continuous_energy/hii40_continuous.in: case A with the Milne
diffuse field and its He I excited channel, metal absorption, metal n_e and
heating), which the run here uses as it stands; the bar is 1 % (the
reference states 0.5 % against Cloudy; the Monte Carlo packets and the
convergence point differ between the two runs)."""
import json
import os

import numpy as np
import pytest

from mochii_b200 import configs, host, parse_namelist

pytestmark = pytest.mark.gpu


def test_g2a_thermal_gate_against_1d_reference(tmp_path):
    from oracle import pyorc
    par = parse_namelist(configs.g2a(str(tmp_path)))
    neb, hist = host.run(par, final_pass=False)
    d = neb.write_rates(os.path.join(str(tmp_path), "g2a"), converged=True, iterations=len(hist))
    neb.close()
    xyz = np.load(os.path.join(d, "LeafXYZ.npy"))
    te = np.load(os.path.join(d, "T_e.npy"))
    ne = np.load(os.path.join(d, "n_e.npy"))
    with open(os.path.join(d, "header.json")) as fh:
        assert json.load(fh)
    r = np.sqrt((xyz ** 2).sum(axis=0))
    ref = pyorc.thermal_1d(configs.ATOMIC_DIR)
    sel = (r > 0.3) & (r < 2.8) & (ne > 0)
    dev = te[sel] / np.interp(r[sel], ref[0], ref[4]) - 1.0
    print(f"G2a: median |dev| {np.median(np.abs(dev)):.4%}, mean {dev.mean():+.4%}, "
          f"{sel.sum()} leaves, {len(hist)} iterations")
    assert sel.sum() > 10000
    assert np.median(np.abs(dev)) < 0.01, (np.median(np.abs(dev)), dev.mean(), len(hist))


def test_hii40_production_mean_electron_temperature(tmp_path):
    par = parse_namelist(configs.hii40(str(tmp_path), production=True))
    neb, hist = host.run(par, final_pass=False)
    nH, x, ne, T = neb.get("nH"), neb.get("x_HI"), neb.get("n_e"), neb.get("T_e")
    gas = nH > 0
    w = (nH * (1.0 - x) * ne)[gas]
    t_mean = float(np.sum(T[gas] * w) / np.sum(w))
    neb.close()
    print(f"HII40: <T[NpNe]> = {t_mean:.1f} K after {len(hist)} iterations")
    assert len(hist) >= 5
    assert abs(t_mean / 8169.0 - 1.0) < 0.01, (t_mean, len(hist), hist[-1])
