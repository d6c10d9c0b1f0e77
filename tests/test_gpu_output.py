"""The rates file (mochii_write_rates, gas_rates_write of gas_rates_mod.f90:
216-366 with species_write of species_mod.f90:873-916): every dataset of the
reference's file under its name, read back with numpy against the fields the
C ABI returns, J_nu against its definition from the spectrum tallies, and
the header keywords."""
import json
import os

import numpy as np
import pytest

from mochii_b200 import Nebula, configs, parse_namelist

pytestmark = pytest.mark.gpu


def test_rates_file_round_trip(tmp_path):
    n = 12
    nl = configs.hii_metals(nphotons=20000, niter=2, n=n, precision="fp32", diffuse=False)
    neb = Nebula(parse_namelist(nl))
    st = neb.ionizing_field_and_rates()
    neb.gas_thermal_update()
    m = neb.last_metrics
    out = neb.write_rates(os.path.join(tmp_path, "hii"), converged=False, iterations=1, final_dx=m.max_dx,
                          final_dte=m.max_dte)
    hdr = json.load(open(os.path.join(out, "header.json")))
    names = [d["EXTNAME"] for d in hdr["datasets"]]
    for want in ("Gamma_HI", "Gamma_HeI", "Gamma_HeII", "Heat_HI", "Heat_HeI", "Heat_HeII", "J_nu", "x_HI", "x_HeI",
                 "x_HeII", "n_e", "T_e", "E_bin", "dE_bin", "LeafXYZ", "LeafSize", "x_c_stages", "Gamma_o_stages",
                 "Heat_fe_stages"):
        assert want in names, want
    load = lambda k: np.load(os.path.join(out, k + ".npy"))   # noqa: E731
    for ext, f in (("Gamma_HI", "gamma_HI"), ("Heat_HeII", "heat_HeII"), ("x_HI", "x_HI"), ("T_e", "T_e"),
                   ("n_e", "n_e")):
        assert np.array_equal(load(ext), neb.get(f)), ext
    kw = hdr["keywords"]
    assert kw["NITERDON"]["value"] == 1 and kw["CONVERGD"]["value"] is False
    assert kw["FINALDX"]["value"] == m.max_dx and kw["QMCSEED"]["value"] == 12345
    assert abs(kw["L_ABS"]["value"] - st.energy_absorbed) <= 1e-12 * st.energy_emitted
    assert kw["NNU_BAND"]["value"] == neb.nnu_band
    # J_nu(nnu, nleaf) from jt_ion / (4 pi V dnu d2cm^2), bins geometric centres
    e = neb.get("eedge")
    assert np.allclose(load("E_bin"), np.sqrt(e[:-1] * e[1:]), rtol=1e-15)
    dnu = np.diff(e) * 1.602176634e-12 / 6.62607015e-27
    h = neb.get("leaf_half")
    p = parse_namelist(nl)
    jn = neb.get("jt_ion") / (4 * np.pi * (2 * h[:, None]) ** 3 * dnu[None, :] * p.distance2cm ** 2)
    J = load("J_nu")
    assert J.shape == (n ** 3, neb.nnu_band)
    np.testing.assert_allclose(J, jn, rtol=1e-12, atol=0)
    xyz, size = load("LeafXYZ"), load("LeafSize")
    assert xyz.shape == (3, n ** 3) and np.allclose(size, 2 * h)
    assert abs(xyz[0, 1] - xyz[0, 0] - size[0]) < 1e-12 * size[0]      # raster order: x fastest
    # the metal blocks are the C-ABI's leaf-major registry fields split by element
    ntr, nst = neb.metal_shape()
    gm, xm = neb.get("gamma_metal"), neb.get("x_metal")
    gc, xc = load("Gamma_c_stages"), load("x_c_stages")
    assert gc.shape == (n ** 3, 3) and xc.shape == (n ** 3, 4)
    assert np.array_equal(gc, gm[:, :3]) and np.array_equal(xc, xm[:, :4])
    assert np.allclose(xc.sum(axis=1), 1.0, atol=1e-9)
    neb.close()
