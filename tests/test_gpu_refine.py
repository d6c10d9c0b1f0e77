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


@pytest.mark.parametrize("grid", ["g2a", "irregular"])
def test_device_plan_equals_host_plan(tmp_path, grid):
    """The device plan (front flags, level-by-level build sorted into
    depth-first order, remap) writes the same leaf list as the host plan on
    the same tree and state, to the last bit of every remapped value."""
    from conftest import octree_leaf_list
    if grid == "g2a":
        nl = sphere(tmp_path)
        par = parse_namelist(nl.replace("/\n", " par%refine_lbase = 3\n par%refine_lmax = 6\n/\n"))
        neb = Nebula(par)
        for _ in range(2):
            neb.ionizing_field_and_rates()
            neb.gas_equilibrium_update()
            neb.gas_opacity_fill()
        lbase, lmax = 3, 6
    else:
        src = str(tmp_path / "leaves.txt")
        octree_leaf_list(src, 8.0, base_level=2, max_level=5, p_split=0.35, seed=11)
        nl = configs.on_octree(configs.hhe128(nphotons=1000, niter=1, n=8, precision="fp64"), src)
        par = parse_namelist(nl.replace("/\n", " par%refine_lbase = 2\n par%refine_lmax = 6\n/\n"))
        neb = Nebula(par)
        rows = np.loadtxt(src, skiprows=1, ndmin=2)
        r = np.sqrt((rows[:, :3] ** 2).sum(axis=1)) / 4.0
        xHI = np.clip(1.0 / (1.0 + np.exp(-(r - 0.5) / 0.08)), 1e-6, 1.0)
        xHeI = np.clip(1.5 * xHI, 0.0, 1.0)
        neb.set("x_HI", xHI)
        neb.set("x_HeI", xHeI)
        neb.set("x_HeII", 1.0 - xHeI)
        neb.set("n_e", rows[:, 4] * ((1.0 - xHI) + 0.1 * (1.0 - xHeI)))
        neb.set("T_e", 3e3 + 7e3 * (1.0 - xHI))
        lbase, lmax = 2, 6
    st = {k: neb.get(k) for k in ("nH", "x_HI", "x_HeI", "x_HeII", "n_e", "T_e")}
    dev = str(tmp_path / "device.txt")
    new = neb.refine_front(dev)
    hst = str(tmp_path / "host.txt")
    nn, nf, worst = host.refine_plan(par.amr_file.decode(), st, He_abund=par.He_abund, te_min=par.te_min,
                                     lbase=lbase, lmax=lmax, eps=par.refine_eps, dx=par.refine_dx, out_list=hst)
    assert nf > 10 and nn == new.nleaf and worst < 1e-8
    assert open(dev).read() == open(hst).read()
    new.close()
    neb.close()
