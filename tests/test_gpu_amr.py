"""The octree path (grid_type = 'amr', a generic text leaf list) on the
device against the oracle, through the C ABI:

* leaf sequences of rays (amr_find_leaf, amr_cell_exit, amr_next_leaf of
  octree_mod.f90) bit-exact, including rays from cell corners and along the
  axes;
* the stellar transport pass in FP64 (raytrace_ion_to_edge_amr,
  raytrace_amr.f90:422-486): per-leaf Gamma and heating within 1e-9 of the
  oracle (the tallies are atomic sums in another order), the energy ledger
  within 1e-12, H only and H+He;
* per-leaf volumes in the rate normalisation, the diffuse emission and the
  convergence sums: the diffuse luminosity within 1e-12, diffuse launch
  points bit-exact, the equilibrium and thermal updates within the solver
  bars (x_HI 1e-3, T_e 20 K), FP32 transport within the Monte Carlo bar;
* a leaf list that is missing, or a grid_type = 'amr' without one, is an
  error.
"""
import numpy as np
import pytest

from conftest import octree_leaf_list
from mochii_b200 import Nebula, MochiiError, configs, parse_namelist

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def leaf_file(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("amr") / "leaves.txt")
    rs = configs.stromgren_radius_pc()
    octree_leaf_list(path, 2.0 * rs, base_level=3, max_level=6, p_split=0.3, seed=5)
    return path, 2.0 * rs


@pytest.fixture(scope="module")
def leaf_file_hii(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("amr") / "leaves_hii.txt")
    box = 2.0 * 1.3 * configs.stromgren_radius_pc(Q=5.0e49)
    octree_leaf_list(path, box, base_level=3, max_level=5, p_split=0.3, seed=9)
    return path


def test_octree_leaf_sequences_bit_exact(orc, leaf_file):
    path, box = leaf_file
    nl = configs.on_octree(configs.stromgren64(nphotons=1000, niter=1, precision="fp64"), path)
    sim = orc.Sim(nl)
    neb = Nebula(parse_namelist(nl))
    rng = np.random.default_rng(21)
    n = 4000
    o = rng.uniform(-0.5 * box, 0.5 * box, (n, 3))
    o[:200] = 0.0                                       # the centre: a corner of eight cells
    lat = box / 64.0                                    # lattice of the finest cells: faces and corners
    o[200:600] = np.round(o[200:600] / lat) * lat
    mu = rng.uniform(-1, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    k = np.column_stack([np.sqrt(1 - mu * mu) * np.cos(ph), np.sqrt(1 - mu * mu) * np.sin(ph), mu])
    ax = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], float)
    k[600:900] = ax[np.arange(300) % 6]
    k[900:1000] = np.array([1.0, 1.0, 0.0]) / np.sqrt(2.0)   # through cell edges
    rays = np.column_stack([o, k])
    lg, ng = neb.walk_leaves(rays, 400)
    lo, no = sim.walk_leaves(rays, 400)
    assert np.array_equal(ng, no)
    assert np.array_equal(lg, lo)
    assert ng.max() > 20
    neb.close()


@pytest.mark.parametrize("he", [False, True])
def test_octree_pass_fp64_matches_oracle(orc, leaf_file, he):
    path, _ = leaf_file
    base = configs.hhe128(nphotons=200000, niter=2, n=8, precision="fp64") if he else \
        configs.stromgren64(nphotons=200000, niter=2, precision="fp64")
    nl = configs.on_octree(base, path)
    sim = orc.Sim(nl)
    neb = Nebula(parse_namelist(nl))
    assert neb.nleaf == sim.nleaf
    np.testing.assert_array_equal(neb.get("nH"), sim.get("nH"))
    for it in range(2):
        st = neb.ionizing_field_and_rates()
        sim.transport_pass()
        e, _ = sim.energy()
        assert abs(st.energy_emitted / e[0] - 1) < 1e-12
        assert abs(st.energy_absorbed / e[1] - 1) < 1e-12
        for f in ("gamma_HI", "heat_HI") + (("gamma_HeI", "gamma_HeII", "heat_HeII") if he else ()):
            g, o = neb.get(f), sim.get(f)
            big = o > 1e-12 * o.max()
            assert np.max(np.abs(g[big] / o[big] - 1)) < 1e-9, (it, f)
        neb.gas_equilibrium_update()
        sim.equilibrium_update()
        np.testing.assert_allclose(neb.get("x_HI"), sim.get("x_HI"), rtol=1e-7, atol=1e-10)
    neb.close()


def test_octree_leaf_half_and_density_override(leaf_file):
    path, box = leaf_file
    nl = configs.on_octree(configs.stromgren64(nphotons=1000, niter=1, precision="fp64"), path,
                           density_from_file=False)
    neb = Nebula(parse_namelist(nl))
    d = np.loadtxt(path, skiprows=1)
    np.testing.assert_array_equal(neb.get("leaf_half"), 0.5 * box / 2.0 ** d[:, 3])
    np.testing.assert_array_equal(neb.get("nH"), np.full(len(d), 100.0))   # par%nH_const
    neb.close()


def test_octree_diffuse_and_thermal_match_oracle(orc, leaf_file_hii):
    nl = configs.on_octree(configs.hii_metals(nphotons=60000, niter=2, n=8, precision="fp64", rs_factor=1.3),
                           leaf_file_hii)
    sim = orc.Sim(nl)
    neb = Nebula(parse_namelist(nl))
    # diffuse emission on the starting state: per-leaf volumes enter the luminosity
    lum_o, n_o = sim.diffuse_build()
    nrec = min(n_o, 3000)
    rec, lum_g, n_g = neb.diffuse_records(0, nrec)
    assert abs(lum_g / lum_o - 1) < 1e-12 and n_g == n_o and n_o > 100
    ref = np.array([sim.diffuse_photon(i) for i in range(nrec)])
    same = np.all(rec[:, 3:6] == ref[:, :3], axis=1)   # launch points bit-exact (same leaf drawn)
    assert same.mean() > 0.999
    assert np.array_equal(rec[same, 7], ref[same, 7])
    for _ in range(2):
        st = neb.ionizing_field_and_rates()
        sim.transport_pass()
        assert st.closure <= 5e-13
        g, o = neb.get("gamma_HI"), sim.get("gamma_HI")
        big = o > 1e-3 * o.max()
        assert np.median(np.abs(g[big] / o[big] - 1)) < 1e-9
        neb.gas_thermal_update()
        sim.thermal_update()
        assert np.max(np.abs(neb.get("T_e") - sim.get("T_e"))) < 20.0
        assert np.max(np.abs(neb.get("x_HI") - sim.get("x_HI"))) < 1e-3
    neb.close()


def test_octree_fp32_transport_within_mc_noise(orc, leaf_file):
    path, _ = leaf_file
    base = configs.hhe128(nphotons=400000, niter=1, n=8, precision="fp64")
    sim = orc.Sim(configs.on_octree(base, path))
    sim.transport_pass()
    neb = Nebula(parse_namelist(configs.on_octree(base.replace("'fp64'", "'fp32'"), path)))
    neb.ionizing_field_and_rates()
    for f in ("gamma_HI", "heat_HI", "gamma_HeI"):
        g, o = neb.get(f), sim.get(f)
        big = o > 1e-2 * o.max()
        assert np.max(np.abs(g[big] / o[big] - 1)) < 3e-5, f   # same packets: FP32 rounding only
    neb.close()


def test_octree_errors(tmp_path):
    nl = configs.stromgren64(nphotons=1000, niter=1).replace("par%grid_type = 'car'", "par%grid_type = 'amr'")
    with pytest.raises(MochiiError, match="amr_file"):
        Nebula(parse_namelist(nl))
    missing = str(tmp_path / "none.txt")
    with pytest.raises(MochiiError, match="cannot open"):
        Nebula(parse_namelist(configs.on_octree(configs.stromgren64(nphotons=1000, niter=1), missing)))
    bad = tmp_path / "bad.txt"
    bad.write_text("3 1.0\n0.25 0.25 0.25 1 1.0\n")
    with pytest.raises(MochiiError, match="fewer leaf rows"):
        Nebula(parse_namelist(configs.on_octree(configs.stromgren64(nphotons=1000, niter=1), str(bad))))


def test_car_grid_amr_walk_matches_oracle(orc):
    """par%car_walk = 'amr': the namelist car grid walked by cell exits and
    car_next (raytrace_ion_to_edge_amr on the car grid) -- leaf sequences
    bit-exact and the FP64 pass within 1e-9 of the oracle's same walk."""
    nl = configs.hhe128(nphotons=200000, niter=1, n=20, precision="fp64").replace(
        "par%grid_type = 'car'", "par%grid_type = 'car'\n par%car_walk = 'amr'")
    sim = orc.Sim(nl)
    neb = Nebula(parse_namelist(nl))
    L = parse_namelist(nl).xmax
    rng = np.random.default_rng(4)
    o = rng.uniform(-L, L, (3000, 3))
    o[:100] = 0.0
    mu = rng.uniform(-1, 1, 3000)
    ph = rng.uniform(0, 2 * np.pi, 3000)
    k = np.column_stack([np.sqrt(1 - mu * mu) * np.cos(ph), np.sqrt(1 - mu * mu) * np.sin(ph), mu])
    k[100:400] = np.array([[1, 0, 0], [0, -1, 0], [0, 0, 1]], float)[np.arange(300) % 3]
    rays = np.column_stack([o, k])
    lg, ng = neb.walk_leaves(rays, 100)
    lo, no = sim.walk_leaves(rays, 100)
    assert np.array_equal(ng, no) and np.array_equal(lg, lo)
    st = neb.ionizing_field_and_rates()
    sim.transport_pass()
    e, _ = sim.energy()
    assert abs(st.energy_absorbed / e[1] - 1) < 1e-12
    for f in ("gamma_HI", "gamma_HeI", "heat_HeII"):
        g, o_ = neb.get(f), sim.get(f)
        big = o_ > 1e-12 * o_.max()
        assert np.max(np.abs(g[big] / o_[big] - 1)) < 1e-9, f
    neb.close()
