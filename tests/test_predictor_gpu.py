"""Learned work predictor: CUDA gradients vs a CPU model, training, exactness of the
learned scheduler, and what the network gains over the degree order it replaces."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F, H = 8, 32


def unpack(p):
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def cpu_forward_backward(p, X, T):
    """Reference model in float64: forward, MSE loss and its gradient."""
    W1, b1, W2, b2, W3, b3 = (np.asarray(a, np.float64) for a in unpack(p))
    X = X.astype(np.float64)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ W3 + b3
    n = X.shape[0]
    err = y - T
    dy = 2 * err / n
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = np.outer(dy, W3) * (z2 > 0)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    gW1 = dz1.T @ X
    gb1 = dz1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return y, (err ** 2).mean(), grad


def test_gradients_and_inference_match_cpu(dm, gpu):
    pr = dm.Predictor(seed=3)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(3000, F)).astype(np.float32)
    T = rng.normal(size=3000).astype(np.float32)
    p = pr.get_params()
    assert p.size == 1377
    y_cpu, loss_cpu, g_cpu = cpu_forward_backward(p, X, T)
    y_gpu = pr.predict(X)
    assert np.allclose(y_gpu, y_cpu, rtol=1e-4, atol=1e-4)
    g_gpu, loss_gpu = pr.gradients(X, T)
    assert abs(loss_gpu - loss_cpu) <= 1e-4 * max(1.0, loss_cpu)
    assert np.allclose(g_gpu, g_cpu, rtol=1e-3, atol=1e-5)
    # finite differences on a few coordinates through the GPU forward pass
    for i in (0, 300, 1000, 1376):
        e = np.zeros_like(p)
        e[i] = 1e-2
        pr.set_params(p + e)
        lp = np.mean((pr.predict(X).astype(np.float64) - T) ** 2)
        pr.set_params(p - e)
        lm = np.mean((pr.predict(X).astype(np.float64) - T) ** 2)
        assert abs((lp - lm) / 2e-2 - g_cpu[i]) <= 2e-2 * max(1.0, abs(g_cpu[i]))
    pr.set_params(p)


def _dataset(dm, name, seeds, ks):
    from dumato_b200 import workloads

    Xs, Ts = [], []
    for s in seeds:
        g = workloads.make(name, s)
        for k in ks:
            X, T, m = dm.subtree_log(g, k)
            Xs.append(X[m])
            Ts.append(T[m])
    return np.concatenate(Xs), np.concatenate(Ts)


def test_training_lowers_loss_and_beats_degree_order(dm, gpu):
    from scipy.stats import spearmanr

    from dumato_b200 import workloads

    Xtr, Ttr = _dataset(dm, "rmat100k", [2, 3], [4, 5, 6])
    pr = dm.Predictor(seed=1)
    loss0 = float(np.mean((pr.predict(Xtr) - Ttr) ** 2))
    loss = pr.train(Xtr, Ttr, epochs=40, batch=512, lr=3e-3)
    assert loss < 0.5 * loss0
    # held-out graph (seed 1), k = 6
    g = workloads.make("rmat100k", 1)
    X, T, m = dm.subtree_log(g, 6)
    pred = pr.predict(X[m])
    mae = float(np.mean(np.abs(pred - T[m])))
    mae_mean = float(np.mean(np.abs(T[m].mean() - T[m])))
    assert mae < 0.6 * mae_mean
    rho_net = spearmanr(pred, T[m]).correlation
    rho_deg = spearmanr(X[m][:, 5], T[m]).correlation  # the plain order: DAG out-degree
    print(f"held-out k=6: MAE(log subtree) {mae:.3f} (mean predictor {mae_mean:.3f}); "
          f"rank correlation with true cost: network {rho_net:.3f}, out-degree {rho_deg:.3f}")
    assert rho_net > rho_deg


@pytest.mark.parametrize("k", [5, 6])
def test_learned_schedule_is_exact(dm, orc, gpu, k):
    from dumato_b200 import workloads

    Xtr, Ttr = _dataset(dm, "rmat100k", [2], [4, 5])
    pr = dm.Predictor(seed=2)
    pr.train(Xtr, Ttr, epochs=20, batch=512, lr=3e-3)
    g = workloads.make("rmat100k", 1)
    plain, _ = dm.count_cliques(g, k)
    learned, st = dm.count_cliques(g, k, dm.Options(scheduler=dm.SCHED_LEARNED, predictor=pr.handle))
    assert learned == plain
    assert st.tasks > 0
    # motifs through the learned schedule
    d = dm.Dictionary.generate(3)
    a, _ = dm.count_motifs(g, 3, d)
    b, _ = dm.count_motifs(g, 3, d, dm.Options(scheduler=dm.SCHED_LEARNED, predictor=pr.handle))
    assert np.array_equal(a, b)


def test_learned_schedule_on_device_every_path(dm, orc, gpu):
    """The device schedule (inference, bucketed longest-first order, splits, eager-donation
    flags) is exact on every clique path, on shards, and for motifs; every learned call
    pays its own scheduling (reported in prep_ms)."""
    from dumato_b200 import workloads

    Xtr, Ttr = _dataset(dm, "rmat100k", [3], [4, 5, 6])
    pr = dm.Predictor(seed=4)
    pr.train(Xtr, Ttr, epochs=20, batch=512, lr=3e-3)
    g = workloads.make("rmat100k", 1)
    og = orc.OracleGraph.from_pairs(*g.edges())
    L = dict(scheduler=dm.SCHED_LEARNED, predictor=pr.handle)
    for k in (4, 6, 7):
        want = orc.clique_dag_bytes(og, k)[0]
        for extra in ({}, {"mode": dm.MODE_REBUILD}, {"staging": dm.STAGE_LOADS}, {"mode": dm.MODE_LIST},
                      {"test_flags": dm.TEST_EAGER_DONATION}):
            got, st = dm.count_cliques(g, k, dm.Options(**L, **extra))
            assert got == want, (k, extra)
            assert st.prep_ms > 0
        parts = [dm.count_cliques(g, k, dm.Options(**L, rank=r, world_size=3))[0] for r in range(3)]
        assert sum(parts) == want
    d = dm.Dictionary.generate(3)
    a, _ = dm.count_motifs(g, 3, d)
    shards = [dm.count_motifs(g, 3, d, dm.Options(**L, rank=r, world_size=2))[0] for r in range(2)]
    assert np.array_equal(a, shards[0] + shards[1])
