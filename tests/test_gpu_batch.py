"""Batched nebulae (mochii_batch_*): several H II regions of different grid
sizes advanced together, one iteration recorded as one CUDA graph and
replayed, the thermal solves of all nebulae in one persistent launch.  Each
nebula's iteration equals its own standalone iteration (the transport tallies
are atomic sums in another order, so rates agree to 1e-12 and the solved
states to the balance's rounding), energy closure holds per nebula, and the
graph replays."""
import numpy as np
import pytest

from mochii_b200 import Batch, Nebula, MochiiError, configs, parse_namelist

pytestmark = pytest.mark.gpu


def nebulae(sizes, solve_te=True, layout="lockstep", solver=None):
    out = []
    for k, n in enumerate(sizes):
        nl = configs.hii_metals(nphotons=30000 + 10000 * k, niter=3, n=n, precision="fp64", rs_factor=1.2 + 0.1 * k,
                                diffuse=False, solve_te=solve_te)
        extra = f" par%cell_layout = '{layout}'\n" + (f" par%thermal_solver = '{solver}'\n" if solver else "")
        out.append(Nebula(parse_namelist(nl.replace("/\n", extra + "/\n"))))
    return out


@pytest.mark.parametrize("solve_te,layout", [(True, "lockstep"), (True, "lane"), (False, "lockstep")])
def test_batch_iteration_equals_standalone(solve_te, layout):
    sizes = (12, 16, 20)
    alone = nebulae(sizes, solve_te, layout)
    together = nebulae(sizes, solve_te, layout)
    batch = Batch(together)
    for it in range(3):
        st, m, ms = batch.iterate(solve_te=solve_te)
        assert ms > 0
        for k, neb in enumerate(alone):
            s1 = neb.ionizing_field_and_rates()
            if solve_te:
                neb.gas_thermal_update()
            else:
                neb.gas_equilibrium_update()
            m1 = neb.last_metrics
            assert st[k].closure <= 5e-13
            assert abs(st[k].energy_absorbed / s1.energy_absorbed - 1) < 1e-12
            assert st[k].direct_segments == s1.direct_segments
            g_b, g_a = together[k].get("gamma_HI"), neb.get("gamma_HI")
            big = g_a > 1e-12 * g_a.max()
            assert np.max(np.abs(g_b[big] / g_a[big] - 1)) < 1e-9
            dT = np.abs(together[k].get("T_e") - neb.get("T_e"))
            assert np.median(dT) < 1e-6 and dT.max() < 1.0, (it, k, dT.max())
            assert np.max(np.abs(together[k].get("x_HI") - neb.get("x_HI"))) < 1e-5
            assert m[k].cells_solved == m1.cells_solved
    batch.close()
    for neb in alone + together:
        neb.close()


def test_batch_refuses_the_diffuse_field():
    nl = configs.hii_metals(nphotons=10000, niter=1, n=8, precision="fp64", diffuse=True)
    neb = Nebula(parse_namelist(nl))
    with pytest.raises(MochiiError) as ei:
        Batch([neb])
    assert ei.value.status == 8
    neb.close()


def test_packet_chunk_splits_the_pass():
    """par%packet_chunk bounds the per-launch record buffers: a pass in
    chunks of 4096 packets scores what a pass in one chunk scores."""
    nl = configs.hii_metals(nphotons=30000, niter=1, n=16, precision="fp64", diffuse=False)
    one = Nebula(parse_namelist(nl))
    many = Nebula(parse_namelist(nl.replace("/\n", " par%packet_chunk = 4096\n/\n")))
    s1, s2 = one.ionizing_field_and_rates(), many.ionizing_field_and_rates()
    assert s1.direct_segments == s2.direct_segments
    assert abs(s1.energy_absorbed / s2.energy_absorbed - 1) < 1e-12
    for f in ("gamma_HI", "heat_HeI"):
        a, b = one.get(f), many.get(f)
        big = a > 1e-12 * a.max()
        assert np.max(np.abs(b[big] / a[big] - 1)) < 1e-9, f
    one.close()
    many.close()


def test_batch_refuses_a_changed_context():
    """A recorded batch graph holds each context's launch shapes and
    buffers: after mochii_set_nphotons on a batched context the next
    iterate is refused (MOCHII_ERR_BAD_PARAM) before any launch, the
    context's tallies are untouched, and a new batch runs."""
    nebs = nebulae((8, 10))
    batch = Batch(nebs)
    batch.iterate()
    g0 = nebs[0].get("gamma_HI")
    nebs[0].set_nphotons(50000)
    with pytest.raises(MochiiError) as ei:
        batch.iterate()
    assert ei.value.status == 1
    assert np.array_equal(nebs[0].get("gamma_HI"), g0)
    batch.close()
    batch = Batch(nebs)
    st, _, _ = batch.iterate()
    assert st[0].packets == 50000
    batch.close()
    for neb in nebs:
        neb.close()


def test_batch_with_learned_warm_start_equals_standalone():
    """The learned warm start recorded into the batch iteration (each
    nebula's inference after its pass, the batched thermal launch from the
    predictions) solves each nebula as its own warm-started update does."""
    from mochii_b200.mlp import WarmStartMLP
    train = nebulae((12,), layout="lane", solver="bracketed")[0]
    X, Y = [], []
    for _ in range(3):
        train.ionizing_field_and_rates()
        X.append(WarmStartMLP.features(train))
        train.gas_thermal_update()
        Y.append(WarmStartMLP.targets(train, X[-1]))
    train.close()
    mlp = WarmStartMLP(seed=1)
    mlp.train(np.concatenate(X), np.concatenate(Y), epochs=10, batch=512, lr=2e-3, seed=2)
    sizes = (12, 16)
    alone = nebulae(sizes, layout="lane", solver="bracketed")
    together = nebulae(sizes, layout="lane", solver="bracketed")
    batch = Batch(together)
    batch.set_warm_start(mlp)
    for it in range(2):
        st, m, _ = batch.iterate()
        for k, neb in enumerate(alone):
            neb.ionizing_field_and_rates()
            mlp.warm_start(neb)
            neb.gas_thermal_update()
            dT = np.abs(together[k].get("T_e") - neb.get("T_e"))
            assert np.median(dT) < 1e-6 and dT.max() < 1.0, (it, k, dT.max())
            assert m[k].warm_accepted == neb.last_metrics.warm_accepted
            assert abs(m[k].rate_evaluations / neb.last_metrics.rate_evaluations - 1) < 0.01
    batch.close()
    for neb in alone + together:
        neb.close()
    mlp.close()
