"""The isotropic external radiation field (ion_band_mod.f90: the external
component of build_external_field_sampler, emit_external_rec_qmc,
emit_external_sph_qmc) against the oracle: the launched packets of an
external-only field through the box faces and through a bounding sphere, and
of a point source composed with the field -- energies and bins bit-exact,
entry points exact on the faces (the sphere's within the last bits of its
cos/sin), directions within the last ulp of cos/sin (a few ulp for the
sphere's frame), every packet inside the
box and heading inward -- the entering power pi J A, and the FP64 pass over
the same packets."""
import numpy as np
import pytest

from conftest import octree_leaf_list
from mochii_b200 import Nebula, configs, parse_namelist

pytestmark = pytest.mark.gpu

J = 3.0e-3   # band mean intensity [erg/s/cm^2/sr]


def ext_nl(kind, n=16, nphot=8192, leaves=None):
    base = configs.hhe128(nphotons=nphot, niter=1, n=n, precision="fp64")
    if leaves:
        base = configs.on_octree(base, leaves)
    L = parse_namelist(base).xmax
    if kind == "rec":
        extra = f" par%source_geometry = 'external_rec'\n par%ext_intensity = {J}\n par%ext_tstar = 3.0e4\n"
    elif kind == "sph":
        extra = (f" par%source_geometry = 'external_sph'\n par%ext_intensity = {J}\n par%rmax = {0.9 * L}\n")
    else:   # one point source composed with the field
        extra = (f" par%nsource = 1\n par%src_lum(1) = 1.0e38\n par%src_tstar(1) = 4.0e4\n"
                 f" par%src_x(1) = 0.0\n par%src_y(1) = 0.0\n par%src_z(1) = 0.0\n"
                 f" par%ext_intensity = {J}\n par%ext_geometry = 'rec'\n")
    return base.replace("/\n", extra + "/\n"), L


@pytest.fixture(scope="module")
def leaves(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("ext") / "leaves.txt")
    octree_leaf_list(path, 2.0 * configs.stromgren_radius_pc(Q=5.0e49), base_level=3, max_level=5, seed=5)
    return path


@pytest.mark.parametrize("kind,grid", [("rec", "car"), ("sph", "amr"), ("mixed", "car"), ("rec", "amr")])
def test_external_launch_matches_oracle(orc, leaves, kind, grid):
    nl, L = ext_nl(kind, leaves=leaves if grid == "amr" else None)
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl, nthreads=1)
    if grid == "amr":
        L = float(open(leaves).readline().split()[1]) / 2
    n = 4096
    rec = neb.launch_records(0, n)
    ref = np.array([sim.photon(i) for i in range(n)])
    assert np.array_equal(rec[:, 6], ref[:, 6]) and np.array_equal(rec[:, 7], ref[:, 7])
    tol = 0.0 if kind != "sph" else 1e-14 * L
    np.testing.assert_allclose(rec[:, :3], ref[:, :3], rtol=0, atol=tol)
    # cos/sin last ulp; the sphere's directions combine two cos/sin pairs in a frame
    np.testing.assert_allclose(rec[:, 3:6], ref[:, 3:6], rtol=0, atol=4e-16 if kind != "sph" else 1.2e-15)
    assert np.all(np.abs(rec[:, :3]) < L)
    if kind == "sph":   # entry on the sphere, the direction within the inward hemisphere
        assert np.all(-np.sum(rec[:, :3] * rec[:, 3:6], axis=1) > -1e-12 * L)
    else:               # entry on a face, the direction into the box across it
        ext = np.abs(rec[:, :3]).max(axis=1) > 0.99 * L
        assert ext.sum() > n // 4
        ax = np.argmax(np.abs(rec[ext, :3]), axis=1)
        rows = np.flatnonzero(ext)
        assert np.all(rec[rows, ax] * rec[rows, 3 + ax] <= 0.0)
    neb.close()


def test_external_field_power_and_pass(orc):
    nl, L = ext_nl("rec", nphot=20000)
    neb = Nebula(parse_namelist(nl))
    sim = orc.Sim(nl)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    d2cm = configs.PC2CM
    side = 2 * L * d2cm
    assert abs(st.energy_emitted / (np.pi * J * 6 * side * side) - 1) < 1e-12   # pi J A, no FUV
    assert abs(st.energy_emitted / sim.ion_Ltot - 1) < 1e-14
    e, _ = sim.energy()
    assert st.closure <= 5e-13 and abs(st.energy_absorbed / e[1] - 1) < 1e-10
    for f in ("gamma_HI", "gamma_HeI", "heat_HI"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-3 * o.max()
        assert big.sum() > 100 and np.median(np.abs(g[big] / o[big] - 1)) < 1e-9, f
    neb.close()
