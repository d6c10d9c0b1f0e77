"""Peel-off imaging (the imaging pass of main.f90:234-235: ion_peel_mod.f90
with the optical-depth-only walks of raytrace_amr.f90:678-775) against the
FP64 oracle's restatement: observers by angle and by position, direct and
unattenuated images on the Cartesian grid, direct and scattered images on
the octree with grains and Henyey-Greenstein scattering (the same Philox
streams on both sides), the channels of the FUV band, and the image file."""
import json
import os

import numpy as np
import pytest

from mochii_b200 import MochiiError, Nebula, configs, parse_namelist

pytestmark = pytest.mark.gpu


def partial(n, L, neb, sim):
    d = 2 * L / n
    c = (np.arange(n) + 0.5) * d - L
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z).ravel()
    xHI = np.clip(1e-4 + (r / (0.6 * L)) ** 6, 1e-4, 1.0)
    neb.set("x_HI", xHI)
    neb.gas_opacity_fill()
    sim.set("x_HI", xHI)


def test_peel_car_grid_matches_oracle(orc):
    n = 24
    nl = configs.stromgren64(nphotons=20000, n=n).replace(
        "/\n", " par%ion_peel = .true.\n par%nxim = 41\n par%nyim = 37\n par%save_direc0 = .true.\n"
               " par%alpha(1) = 0.0, 30.0, 75.0\n par%beta(1) = 0.0, 60.0, 110.0\n/\n")
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    partial(n, parse_namelist(nl).xmax, neb, sim)
    st = neb.imaging_pass()
    sim.imaging_pass()
    assert st.closure <= 5e-13
    for which in ("direct", "direct0"):
        g, o = neb.image(which), sim.peel_image(which)
        assert g.shape == o.shape == (3, 1, 37, 41)
        # a central point source seen through gas alone: one lit pixel per observer
        assert o.sum() > 0 and [np.count_nonzero(o[k]) for k in range(3)] == [1, 1, 1]
        np.testing.assert_allclose(g, o, rtol=1e-9, atol=1e-12 * o.max(), err_msg=which)
    assert np.all(neb.image("scattered") == 0.0)
    # the observers the two sides derived
    for k in range(3):
        np.testing.assert_allclose(neb.image_observer(k), sim.peel_observer(k), rtol=1e-14, atol=1e-14)
    # a pass without with_peel leaves the images of the imaging pass alone
    img = neb.image("direct")
    neb.ionizing_field_and_rates()
    assert np.array_equal(neb.image("direct"), img)
    neb.close()


def test_peel_octree_dust_scattering_matches_oracle(orc, tmp_path):
    nl = configs.clumpy_dusty(str(tmp_path), nphotons=30000, base_level=4, max_level=6, field_n=64,
                              precision="fp64").replace(
        "/\n", " par%ion_peel = .true.\n par%nxim = 31\n par%nyim = 31\n"
               " par%obsx(1) = 0.0, 1.0\n par%obsy(1) = 0.0, 1.0\n par%obsz(1) = 1.0, 0.5\n/\n")
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    st = neb.imaging_pass()
    sim.imaging_pass()
    assert st.closure <= 5e-13
    for which in ("direct", "scattered"):
        g, o = neb.image(which), sim.peel_image(which)
        assert g.shape == o.shape == (2, 2, 31, 31)   # ionizing and FUV channels
        assert o.sum() > 0, which
        big = o > 1e-6 * o.max()
        assert np.median(np.abs(g[big] / o[big] - 1)) < 1e-9, which
        assert abs(g.sum() / o.sum() - 1) < 1e-6, which
    # the image file: surface brightness = contributions / (d2cm^2 x pixel solid angle)
    out = neb.write_image(os.path.join(tmp_path, "clumpy"))
    hdr = json.load(open(os.path.join(out, "header.json")))
    names = [d["EXTNAME"] for d in hdr["datasets"]]
    assert {"direct_ion_obs1", "scatt_fuv_obs2"} <= set(names)
    ob = neb.image_observer(1)
    fac = 1.0 / (neb.par.distance2cm ** 2 * (ob[7] * ob[8] * (np.pi / 180) ** 2))
    np.testing.assert_allclose(np.load(os.path.join(out, "scatt_fuv_obs2.npy")), neb.image("scattered")[1, 1] * fac,
                               rtol=1e-15)
    neb.close()


def test_imaging_pass_needs_observers():
    neb = Nebula(parse_namelist(configs.stromgren64(nphotons=1000, n=8)))
    with pytest.raises(MochiiError) as ei:
        neb.imaging_pass()
    assert ei.value.status == 1
    neb.close()


@pytest.mark.parametrize("kind", ["rec_car", "mixed_car", "sph_amr"])
def test_peel_external_field_matches_oracle(orc, tmp_path, kind):
    """External-field packets peel max(k_obs . n_in, 0) / pi about the inward
    normal of their entry surface (ion_peel_mod.f90:254-263): the box faces
    on the Cartesian grid, alone and composed with a point source, and the
    bounding sphere on the octree; direct and unattenuated images."""
    from conftest import octree_leaf_list
    nl = configs.hhe128(nphotons=20000, niter=1, n=16, precision="fp64")
    L = parse_namelist(nl).xmax
    if kind == "sph_amr":
        leaves = str(tmp_path / "leaves.txt")
        octree_leaf_list(leaves, 2.0 * L, base_level=3, max_level=5, seed=9)
        nl = configs.on_octree(nl, leaves)
        ext = f" par%source_geometry = 'external_sph'\n par%ext_intensity = 3.0e-3\n par%rmax = {0.8 * L}\n"
    elif kind == "rec_car":
        ext = " par%source_geometry = 'external_rec'\n par%ext_intensity = 3.0e-3\n"
    else:
        ext = " par%ext_intensity = 3.0e-3\n par%ext_geometry = 'rec'\n par%xs_point = 0.3\n"
    nl = nl.replace("/\n", ext + " par%ion_peel = .true.\n par%nxim = 33\n par%nyim = 29\n par%save_direc0 = .true.\n"
                                 " par%alpha(1) = 0.0, 40.0\n par%beta(1) = 0.0, 70.0\n/\n")
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    st = neb.imaging_pass()
    sim.imaging_pass()
    assert st.closure <= 5e-13
    for which in ("direct", "direct0"):
        g, o = neb.image(which), sim.peel_image(which)
        assert o.sum() > 0 and np.count_nonzero(o) > 50, which   # the field lights the whole box outline
        np.testing.assert_allclose(g, o, rtol=1e-9, atol=1e-12 * o.max(), err_msg=which)
    neb.close()
