"""The oracle's octree (octree_mod.f90 restatement) against geometry computed
independently: the leaf sequence of a ray through the tree is the list of
leaves whose boxes the ray crosses with positive length, ordered by entry
distance (slab intersection of the ray with every leaf box).  Also the leaf
lists written by mochii_b200.amr: they tile the box exactly and come in
Morton order.
"""
import numpy as np
import pytest

from conftest import octree_leaf_list
from mochii_b200 import amr, configs


def slab_intervals(leaves, o, k):
    """Entry and exit distances of the ray o + t k through every leaf box."""
    c = leaves[:, :3]
    h = 0.5 * leaves[:, 5:6]
    lo, hi = c - h, c + h
    with np.errstate(divide="ignore", invalid="ignore"):
        ta = (lo - o) / k
        tb = (hi - o) / k
    t0 = np.minimum(ta, tb)
    t1 = np.maximum(ta, tb)
    for a in range(3):
        if k[a] == 0.0:
            inside = (o[a] >= lo[:, a]) & (o[a] < hi[:, a])
            t0[:, a] = np.where(inside, -np.inf, np.inf)
            t1[:, a] = np.where(inside, np.inf, -np.inf)
    return t0.max(axis=1), t1.min(axis=1)


@pytest.fixture(scope="module")
def tree(tmp_path_factory, orc):
    path = str(tmp_path_factory.mktemp("amr") / "leaves.txt")
    boxlen = 8.0
    nleaf = octree_leaf_list(path, boxlen, base_level=2, max_level=5, seed=11)
    d = np.loadtxt(path, skiprows=1)
    side = boxlen / 2.0 ** d[:, 3]
    leaves = np.column_stack([d[:, :3], d[:, 3], d[:, 4], side])
    nl = configs.on_octree(configs.stromgren64(nphotons=1000, niter=1, precision="fp64"), path)
    sim = orc.Sim(nl)
    return sim, leaves, boxlen, nleaf


def test_leaf_list_tiles_the_box_in_morton_order(tree):
    _, leaves, boxlen, nleaf = tree
    assert leaves.shape[0] == nleaf
    assert abs(np.sum(leaves[:, 5] ** 3) / boxlen ** 3 - 1.0) < 1e-12
    # Morton order: the lower corners on the finest lattice have increasing keys
    fine = 1 << 5
    ijk = np.round((leaves[:, :3] - 0.5 * leaves[:, 5:6] + 0.5 * boxlen) / boxlen * fine).astype(np.int64)
    key = amr._morton(ijk[:, 0], ijk[:, 1], ijk[:, 2], 5)
    assert np.all(np.diff(key.astype(np.int64)) > 0)


def test_generated_levels_and_density_model():
    x, y, z, lev, nH = amr.build_leaves(4.0, 1, 3, lambda x, y, z, L: x > 0, lambda x, y, z, L: 10.0 + x)
    # x > 0 half refined twice: 4 coarse leaves on the -x side, 4*8*8 fine ones on the +x side
    assert np.bincount(lev).tolist() == [0, 4, 0, 256]
    np.testing.assert_array_equal(nH, 10.0 + x)


def test_oracle_octree_walk_matches_slab_geometry(tree):
    sim, leaves, boxlen, _ = tree
    rng = np.random.default_rng(3)
    nray = 300
    o = rng.uniform(-0.49 * boxlen, 0.49 * boxlen, (nray, 3))
    o[:40] = 0.0   # from the box centre, a corner of eight base cells
    mu = rng.uniform(-1, 1, nray)
    ph = rng.uniform(0, 2 * np.pi, nray)
    k = np.column_stack([np.sqrt(1 - mu * mu) * np.cos(ph), np.sqrt(1 - mu * mu) * np.sin(ph), mu])
    k[40:46] = [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]]
    rays = np.column_stack([o, k])
    seq, ns = sim.walk_leaves(rays, 512)
    eps = 1e-9 * boxlen
    for r in range(nray):
        t0, t1 = slab_intervals(leaves, o[r], k[r])
        t0 = np.maximum(t0, 0.0)
        crossed = np.nonzero(t1 - t0 > eps)[0]
        expect = crossed[np.argsort(t0[crossed], kind="stable")]
        got = seq[r, :ns[r]]
        # leaves the walk touches for a vanishing length (an edge or corner) are not in the slab list
        got_long = got[(t1[got] - t0[got]) > eps]
        assert np.array_equal(got_long, expect), r
        assert np.all(t1[got] - t0[got] > -eps), r   # every visited leaf is on the ray


def test_uniform_octree_walk_equals_car_amr_walk(tmp_path, orc):
    """The octree walk on a uniform tree and the car grid walked as an octree
    (par%car_walk = 'amr') take the same exit faces from the same centres, so
    their leaf sequences agree bit for bit once the Morton leaf order is
    mapped to raster order."""
    boxlen, lev = 8.0, 4
    n = 1 << lev
    x, y, z, lv, nH = amr.build_leaves(boxlen, lev, lev, lambda *a: False, lambda x, y, z, L: np.full(np.shape(x), 50.0))
    path = str(tmp_path / "uniform.txt")
    amr.write_leaf_list(path, boxlen, x, y, z, lv, nH)
    ijk = np.floor((np.column_stack([x, y, z]) + 0.5 * boxlen) / (boxlen / n)).astype(int)
    raster = ijk[:, 0] + n * (ijk[:, 1] + n * ijk[:, 2])
    car = configs.stromgren64(nphotons=1000, niter=1, n=n).replace("par%xmax", "par%xmax = 4.0 !").replace(
        "par%ymax", "par%ymax = 4.0 !").replace("par%zmax", "par%zmax = 4.0 !")
    s_car = orc.Sim(car.replace("par%car_walk = 'dda'", "par%car_walk = 'amr'"))
    s_oct = orc.Sim(configs.on_octree(car, path))
    rng = np.random.default_rng(8)
    o = rng.uniform(-4, 4, (500, 3))
    o[:50] = 0.0
    mu = rng.uniform(-1, 1, 500)
    ph = rng.uniform(0, 2 * np.pi, 500)
    k = np.column_stack([np.sqrt(1 - mu * mu) * np.cos(ph), np.sqrt(1 - mu * mu) * np.sin(ph), mu])
    rays = np.column_stack([o, k])
    la, na = s_car.walk_leaves(rays, 200)
    lb, nb = s_oct.walk_leaves(rays, 200)
    assert np.array_equal(na, nb)
    mapped = np.where(lb >= 0, raster[np.maximum(lb, 0)], -1)
    assert np.array_equal(la, mapped)
