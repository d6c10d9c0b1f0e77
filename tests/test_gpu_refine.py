"""Re-refinement of a context on the GPU (mochii_refine_front): the new
context holds the planned leaves with the remapped state, conserves the box
integrals the reference checks, and iterates; the driver runs the one
refinement event at par%refine_iter (main.f90:172-178) and keeps iterating
on the new grid."""
import os

import numpy as np
import pytest

from mochii_b200 import Nebula, amr, configs, host, parse_namelist

pytestmark = pytest.mark.gpu


def sphere(tmp_path, level=4, niter=4):
    """The G2a sphere (n_H = 100 within 4 pc, 40 kK star) on a coarse uniform
    octree, fixed-T ionisation balance, a few iterations."""
    nl = configs.g2a(str(tmp_path), nphotons=400000, niter=niter, level=level)
    nl = nl.replace(" par%solve_te = .true.\n", " par%solve_te = .false.\n")
    return nl


def integrals(neb):
    h = neb.get("leaf_half")
    v = (2.0 * h) ** 3
    nH, x1, x2, x3, ne, T = (neb.get(f) for f in ("nH", "x_HI", "x_HeI", "x_HeII", "n_e", "T_e"))
    y = 0.1
    return np.array([np.sum(nH * v), np.sum(nH * x1 * v), np.sum(nH * y * x2 * v), np.sum(nH * y * x3 * v),
                     np.sum(ne * v), np.sum((nH * (1 + y) + ne) * T * v)])


def test_refine_front_new_context(tmp_path):
    nl = sphere(tmp_path)
    par = parse_namelist(nl.replace("/\n", " par%refine_lbase = 3\n par%refine_lmax = 6\n/\n"))
    neb = Nebula(par)
    for _ in range(3):
        neb.ionizing_field_and_rates()
        neb.gas_equilibrium_update()
        neb.gas_opacity_fill()
    a = integrals(neb)
    out = str(tmp_path / "refined.txt")
    new = neb.refine_front(out)
    rows = np.loadtxt(out, skiprows=1, ndmin=2)
    assert new.nleaf == rows.shape[0] and new.nleaf != neb.nleaf
    assert rows[:, 3].max() == 6 and rows[:, 3].min() == 3
    for k, f in enumerate(("x_HI", "x_HeI", "x_HeII", "n_e", "T_e")):
        np.testing.assert_array_equal(new.get(f), rows[:, 5 + k])
    np.testing.assert_array_equal(new.get("nH"), rows[:, 4])
    b = integrals(new)
    assert np.max(np.abs(b / a - 1)) < 1e-8, (a, b)
    st = new.ionizing_field_and_rates()
    assert st.closure <= 5e-13 and st.direct_segments > 0
    new.gas_equilibrium_update()
    # the front leaves sit at refine_lmax: the partly ionised leaves are the finest ones
    x = new.get("x_HI")
    lev = np.round(np.log2(8.0 / (2 * new.get("leaf_half")))).astype(int)
    part = (x > 0.05) & (x < 0.95) & (new.get("nH") > 0)
    assert part.sum() > 0 and np.median(lev[part]) == 6
    new.close()
    neb.close()


def test_driver_refines_once_and_keeps_iterating(tmp_path):
    nl = sphere(tmp_path, niter=5)
    par = parse_namelist(nl.replace("/\n", " par%refine_front = .true.\n par%refine_iter = 2\n"
                                          " par%refine_lbase = 3\n par%refine_lmax = 5\n/\n"))
    neb, hist = host.run(par, final_pass=False)
    ev = [h for h in hist if "refined" in h]
    assert len(ev) == 1 and ev[0]["iter"] == 2
    assert ev[0]["refined"]["leaves_after"] == neb.nleaf != ev[0]["refined"]["leaves_before"]
    assert len(hist) >= 3 and all(h["closure"] <= 5e-13 for h in hist)
    neb.close()
