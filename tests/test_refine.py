"""Solution-driven I-front re-refinement (amr_refine_mod.f90), host part:
the library's plan (mochii_refine_plan, no device needed) against the
oracle's restatement on the same irregular octree and state -- the same new
leaves and remapped state to the last bit -- and the properties the
reference asserts: the seven conserved box integrals unchanged to 1e-8
(conservation_report), pure refinement reproducing the old leaf's state
(remap_leaf collapses to centre sampling), front leaves at refine_lmax and
the rest at refine_lbase or coarser leaves kept whole."""
import numpy as np
import pytest

from conftest import octree_leaf_list
from mochii_b200 import host


def read_list(path):
    rows = np.loadtxt(path, skiprows=1, ndmin=2)
    with open(path) as f:
        n, box = f.readline().split()
    assert rows.shape[0] == int(n)
    return rows, float(box)


def state_of(path, front_r=0.5, width=0.08, yHe=0.1):
    rows = np.loadtxt(path, skiprows=1, ndmin=2)
    with open(path) as f:
        box = float(f.readline().split()[1])
    r = np.sqrt((rows[:, :3] ** 2).sum(axis=1)) / (0.5 * box)
    nH = rows[:, 4]
    xHI = np.clip(1.0 / (1.0 + np.exp(-(r - front_r) / width)), 1e-6, 1.0)
    xHeI = np.clip(1.5 * xHI, 0.0, 1.0)
    xHeII = 1.0 - xHeI
    ne = nH * ((1.0 - xHI) + yHe * xHeII)
    Te = 3e3 + 7e3 * (1.0 - xHI)
    return {"nH": nH, "x_HI": xHI, "x_HeI": xHeI, "x_HeII": xHeII, "n_e": ne, "T_e": Te}


@pytest.mark.parametrize("lbase,lmax", [(3, 6), (2, 5)])
def test_plan_matches_oracle(orc, tmp_path, lbase, lmax):
    src = str(tmp_path / "leaves.txt")
    octree_leaf_list(src, 8.0, base_level=2, max_level=5, p_split=0.35, seed=11)
    st = state_of(src)
    rk = st["nH"] * 0.05 * 1.6e-21 * 3.0857e18
    out_g, out_o = str(tmp_path / "g.txt"), str(tmp_path / "o.txt")
    ng, fg, wg = host.refine_plan(src, st, rhokap=rk, lbase=lbase, lmax=lmax, out_list=out_g)
    no, fo, wo = orc.refine_plan(src, st, rhokap=rk, lbase=lbase, lmax=lmax, out_list=out_o)
    assert (ng, fg) == (no, fo) and fg > 20 and ng > 100
    assert wg < 1e-8 and wo < 1e-8
    assert open(out_g).read() == open(out_o).read()   # every leaf and remapped value, bit for bit
    rows, _ = read_list(out_g)
    assert rows[:, 3].min() >= lbase - 0 and rows[:, 3].max() == lmax


def test_pure_refinement_copies_the_old_leaf(tmp_path):
    """A uniform level-3 tree refined everywhere to level 4 (every leaf is a
    front leaf): each new leaf takes its parent's state."""
    from mochii_b200 import amr
    src = str(tmp_path / "u.txt")
    x, y, z, lev, nH = amr.build_leaves(4.0, 3, 3, lambda *a: None, lambda x, y, z, l: 100.0 + 10.0 * x)
    amr.write_leaf_list(src, 4.0, x, y, z, lev, nH)
    n = len(x)
    st = {"nH": nH, "x_HI": np.full(n, 0.5), "x_HeI": np.full(n, 0.3), "x_HeII": np.full(n, 0.6),
          "n_e": 0.5 * nH, "T_e": 8e3 + 100.0 * y}
    out = str(tmp_path / "r.txt")
    nn, nf, worst = host.refine_plan(src, st, lbase=3, lmax=4, out_list=out)
    assert nf == n and nn == 8 * n and worst < 1e-12
    rows, _ = read_list(out)
    # the parent of each new leaf: the old leaf whose cell contains its centre
    h_old = 4.0 / 2 ** 3 / 2
    for k in range(0, nn, 37):
        c = rows[k, :3]
        j = np.argmin(np.abs(np.stack([x, y, z], axis=1) - c).max(axis=1))
        assert np.abs(np.array([x[j], y[j], z[j]]) - c).max() < h_old
        assert rows[k, 4] == nH[j] and rows[k, 9] == st["T_e"][j] and rows[k, 5] == 0.5


def test_plan_refuses_bad_levels(tmp_path):
    src = str(tmp_path / "leaves.txt")
    octree_leaf_list(src, 8.0, base_level=2, max_level=4, seed=3)
    st = state_of(src)
    with pytest.raises(Exception):
        host.refine_plan(src, st, lbase=5, lmax=4, out_list=str(tmp_path / "x.txt"))
