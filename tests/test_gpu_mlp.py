"""The warm-start MLP: its BF16 tensor-core forward and backward kernels
against the FP64 numpy oracle (with the same BF16 rounding points), training
by the device Adam kernels, and what the trained network gains as the warm
start of the thermal solve.

Bars: gradients per layer within 1e-2 relative (norm) of the oracle's,
predictions within 1e-2 (the FP32 accumulation order and BF16 ties are the
only differences); training lowers the loss; the warm-started bracketed solve
reaches T_e within 20 K of the reference bisection with fewer net-rate
evaluations than the solve started from the previous iteration's T_e.
"""
import numpy as np
import pytest

from mochii_b200 import Nebula, configs, parse_namelist
from mochii_b200.mlp import DIMS, WarmStartMLP
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def batch(n, seed=0):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 16), dtype=np.float32)
    X[:, :12] = rng.normal(0, 1, (n, 12))
    Y = np.stack([rng.uniform(0, 1, n), rng.uniform(0, .5, n), rng.uniform(0, .5, n), rng.normal(0, 1, n)],
                 axis=1).astype(np.float32)
    return X, Y


def split(v):
    out, o = [], 0
    for l in range(4):
        no, ni = DIMS[l + 1], DIMS[l]
        out.append((v[o:o + no * ni], v[o + no * ni:o + no * ni + no]))
        o += no * ni + no
    return out


def test_gradients_match_oracle():
    mlp = WarmStartMLP(seed=7)
    X, Y = batch(512, 1)
    p = mlp.params()
    g, loss = mlp.gradients(X, Y)
    go = mlp_ref.gradients(p.astype(np.float64), X.astype(np.float64), Y.astype(np.float64))
    assert abs(loss - mlp_ref.loss(p, X, Y)) < 1e-3 * max(loss, 1e-6)
    for l, ((gw, gb), (ow, ob)) in enumerate(zip(split(g), split(go))):
        assert np.linalg.norm(gw - ow) <= 1e-2 * np.linalg.norm(ow), l
        assert np.linalg.norm(gb - ob) <= 1e-2 * np.linalg.norm(ob) + 1e-12, l
    mlp.close()


def test_predictions_match_oracle():
    mlp = WarmStartMLP(seed=11)
    X, _ = batch(3000, 2)
    pred = mlp.predict(X)
    _, _, out = mlp_ref.forward(mlp.params().astype(np.float64), X.astype(np.float64))
    po = mlp_ref.head(out)
    np.testing.assert_allclose(pred[:, :3], po[:, :3], atol=1e-2)
    np.testing.assert_allclose(np.log10(pred[:, 3]), 4.0 + (X[:, 11] + po[:, 3]) / 4.0, atol=1e-2)
    mlp.close()


def test_training_lowers_the_loss():
    rng = np.random.default_rng(5)
    X, _ = batch(65536, 3)
    # a smooth synthetic target of the features
    s = 1 / (1 + np.exp(-X[:, 0] - 0.5 * X[:, 1]))
    Y = np.stack([s, 0.3 * s, 0.2 * (1 - s), np.tanh(X[:, 2])], axis=1).astype(np.float32)
    mlp = WarmStartMLP(seed=3)
    losses = mlp.train(X, Y, epochs=8, batch=2048, lr=2e-3, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.2 * losses[0], losses
    mlp.close()


def nebula(solver, seed, n=24, nphot=100000):
    nl = configs.hii_metals(nphotons=nphot, niter=8, n=n, precision="fp32", seed=seed, rs_factor=1.2, diffuse=False)
    return Nebula(parse_namelist(nl.replace("/\n", f" par%thermal_solver = '{solver}'\n/\n")))


def test_warm_start_gain():
    """Train on the plain solver's pairs, then the same iterations of a
    nebula with another launch seed: bracketed solve from the previous T_e
    against bracketed solve from the MLP's T_e, and the reference bisection."""
    X, Y = [], []
    neb = nebula("bisection", 12345)
    for _ in range(6):
        neb.ionizing_field_and_rates()
        X.append(WarmStartMLP.features(neb))
        neb.gas_thermal_update()
        Y.append(WarmStartMLP.targets(neb, X[-1]))
    neb.close()
    X, Y = np.concatenate(X), np.concatenate(Y)
    mlp = WarmStartMLP(seed=1)
    losses = mlp.train(X, Y, epochs=30, batch=2048, lr=2e-3, seed=2)
    assert losses[-1] < losses[0]
    runs = {}
    for mode in ("bisection", "previous", "mlp"):
        neb = nebula("bisection" if mode == "bisection" else "bracketed", 777)
        evals = []
        for it in range(4):
            neb.ionizing_field_and_rates()
            if mode == "mlp":
                mlp.warm_start(neb)
            neb.gas_thermal_update()
            evals.append(neb.last_metrics.rate_evaluations)
        runs[mode] = (np.array(evals), neb.get("T_e"), neb.get("x_HI"))
        neb.close()
    tb, tp, tm = runs["bisection"][1], runs["previous"][1], runs["mlp"][1]
    assert np.max(np.abs(tm - tb)) < 20.0 and np.max(np.abs(tp - tb)) < 20.0
    assert np.max(np.abs(runs["mlp"][2] - runs["bisection"][2])) < 1e-3
    # the first iteration starts from T_e = te_fixed without the network
    assert runs["mlp"][0].sum() < runs["previous"][0].sum() < runs["bisection"][0].sum(), \
        {k: v[0].tolist() for k, v in runs.items()}
    mlp.close()


def test_warm_started_update_matches_oracle_on_every_leaf(orc):
    """One thermal update warm-started by the trained MLP (residual gate, then
    the bracketed search from the prediction) against the reference's
    bisection in the FP64 oracle on the same inputs -- the device state and
    rates before the update copied into the oracle -- on every leaf of a
    nebula with diffuse packets: T_e within 20 K and x_HII within 1e-3 (the
    north-star bars); gate acceptances are counted and bounded by the leaves."""
    X, Y = [], []
    neb = nebula("bisection", 12345, n=20, nphot=80000)
    for _ in range(5):
        neb.ionizing_field_and_rates()
        X.append(WarmStartMLP.features(neb))
        neb.gas_thermal_update()
        Y.append(WarmStartMLP.targets(neb, X[-1]))
    neb.close()
    mlp = WarmStartMLP(seed=1)
    mlp.train(np.concatenate(X), np.concatenate(Y), epochs=30, batch=2048, lr=2e-3, seed=2)
    n = 20
    nl = configs.hii_metals(nphotons=80000, niter=8, n=n, precision="fp32", seed=4242, rs_factor=1.2, diffuse=True)
    neb = Nebula(parse_namelist(nl.replace("/\n", " par%thermal_solver = 'bracketed'\n/\n")))
    sim = orc.Sim(nl.replace("'fp32'", "'fp64'"))
    for it in range(3):
        neb.ionizing_field_and_rates()
        for f in ("x_HI", "x_HeI", "x_HeII", "n_e", "T_e"):
            sim.set(f, neb.get(f))
        for f in ("gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI", "heat_HeI", "heat_HeII", "gamma_metal",
                  "heat_metal"):
            sim.set(f, np.ascontiguousarray(neb.get(f)).ravel())
        ref = sim.thermal_cells(np.arange(n ** 3))
        mlp.warm_start(neb)
        neb.gas_thermal_update()
        m = neb.last_metrics
        assert 0 <= m.warm_accepted <= m.cells_solved
        dT = np.abs(neb.get("T_e") - ref[:, 0])
        dx = np.abs(neb.get("x_HI") - ref[:, 1])
        assert dT.max() < 20.0, (it, dT.max())
        assert dx.max() < 1e-3, (it, dx.max())
    neb.close()
    mlp.close()
