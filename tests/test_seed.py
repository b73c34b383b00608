"""Learned chemistry seed: the network's tensor-core kernels against the NumPy
oracle (loss, gradient, prediction), the oracle's own gradient against finite
differences, and what a trained network gains over the plain point-implicit
update on the same states (the ablation)."""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W
from oracle import e4_seed_oracle as SO


def unit_norm():
    norm = np.zeros(SO.NNORM)
    norm[8:16] = 1.0
    norm[22:28] = 1.0
    norm[28] = 1.0e-9
    norm[29] = 1.0e-3
    return norm


def test_bf16_rounding_ties_to_even():
    ulp = 2.0 ** -7
    assert SO.bf16(1.0) == 1.0
    assert SO.bf16(1.0 + 0.5 * ulp) == 1.0                 # tie -> even
    assert SO.bf16(1.0 + 1.5 * ulp) == 1.0 + 2 * ulp       # tie -> even
    assert SO.bf16(1.0 + 0.6 * ulp) == 1.0 + ulp
    assert SO.bf16(-3.0) == -3.0


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    params = SO.init_params(11).astype(np.float64)
    X = rng.normal(size=(24, 8))
    Y = rng.normal(size=(24, 6))
    loss, g = SO.loss_grad(params, X, Y, mirror=False)
    idx = rng.choice(SO.NPARAM, 60, replace=False)
    idx = np.concatenate([idx, [0, 511, 512, 9279, 9280, 9285]])  # W1, b1, W4, b4 ends
    eps = 1.0e-6
    for q in idx:
        p1 = params.copy()
        p1[q] += eps
        p2 = params.copy()
        p2[q] -= eps
        fd = (SO.loss_grad(p1, X, Y, mirror=False)[0] - SO.loss_grad(p2, X, Y, mirror=False)[0]) / (2 * eps)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g).max()), (q, fd, g[q])


@pytest.mark.gpu
def test_seed_loss_and_gradient_match_oracle(e4lib):
    from eilmer4_b200.simcore import Simulation
    rng = np.random.default_rng(3)
    params = SO.init_params(5)
    X = rng.normal(size=(1000, 8)).astype(np.float32)
    Y = rng.normal(size=(1000, 6)).astype(np.float32)
    with Simulation.from_workload(W.sod_2d(16, 4)) as sim:
        sim.seed_set(params, unit_norm())
        loss, g = sim.seed_loss_grad(X, Y)
        p_back, _ = sim.seed_get()
    assert np.array_equal(p_back, params)
    loss_o, g_o = SO.loss_grad(params, X, Y, mirror=True)
    assert abs(loss - loss_o) <= 1e-5 * loss_o, (loss, loss_o)
    # per tensor: W1 b1 W2 b2 W3 b3 W4 b4
    bounds = np.cumsum([0, 512, 64, 4096, 64, 4096, 64, 384, 6])
    for a, b in zip(bounds[:-1], bounds[1:]):
        scale = np.abs(g_o[a:b]).max()
        err = np.abs(g[a:b] - g_o[a:b]).max()
        assert err <= 5e-3 * scale, (a, b, err, scale)
    cos = float(g @ g_o / (np.linalg.norm(g) * np.linalg.norm(g_o)))
    assert cos > 0.99999, cos


@pytest.mark.gpu
def test_seed_prediction_matches_oracle(e4lib):
    from eilmer4_b200.simcore import Simulation
    rng = np.random.default_rng(4)
    params = SO.init_params(6)
    norm = unit_norm()
    norm[0:8] = [8.3, 11.0, 0.7, 0.2, 0.02, 0.01, 0.02, -15.0]
    norm[8:16] = [0.3, 1.0, 0.05, 0.05, 0.01, 0.01, 0.01, 1.0]
    norm[16:22] = [0.0, -5.0, 3.0, 2.0, 4.0, -3.0]
    norm[22:28] = [10.0, 12.0, 11.0, 9.0, 12.0, 8.0]
    n = 777   # not a multiple of the 16-row warp tile
    y = np.array([0.74, 0.2, 0.02, 0.01, 0.03]) + 0.01 * rng.random((n, 5))
    rows = np.column_stack([2500.0 + 5000.0 * rng.random(n), 1e4 + 1e5 * rng.random(n), y,
                            1e-7 * (1.0 + rng.random(n))])
    with Simulation.from_workload(W.sod_2d(16, 4)) as sim:
        sim.seed_set(params, norm)
        out = sim.seed_predict(rows)
    ref = SO.predict(params, norm, rows, mirror=True)
    s = np.concatenate([np.full(5, norm[28]), [norm[29]]])
    zg = np.arcsinh(out / s)
    zo = np.arcsinh(ref / s)
    assert np.all(np.isfinite(zg))
    assert np.abs(zg - zo).max() <= 2e-2 * max(1.0, np.abs(zo).max()), np.abs(zg - zo).max()


@pytest.mark.gpu
def test_trained_seed_saves_newton_iterations_at_equal_result(e4lib):
    """Ablation on the high-enthalpy channel: after 60 steps, the chemistry
    update of the same states with and without the trained network.  The
    seeded update needs fewer Newton iterations and gives the same mass
    fractions to 1e-6."""
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel_hot(ni=128, nj=64)
    with Simulation.from_workload(wl, reacting=True) as sim:
        for _ in range(3):
            sim.run(20)
            _, dt, _ = sim.state()
            sim.seed_collect([0], dt, 100000, seed=sim.state()[2])
        assert sim.seed_dataset() > 100000
        rep = sim.seed_train(epochs=6, batch=1024, lr=2e-3, seed=1)
        assert rep["val_loss"] < 0.2, rep
        prim, _ = sim.download(0)
        _, dt, _ = sim.state()
        results = {}
        for seeded in (False, True):
            sim.upload(0, prim)
            sim.seed_enable(seeded)
            sim.chemistry_counters(reset=True)
            sim.chemistry_step([0], dt)
            cells, newton, recovered, active = sim.chemistry_counters(reset=True)
            out, _ = sim.download(0)
            results[seeded] = (out, cells, newton, active)
    (p0, c0, n0, a0), (p1, c1, n1, a1) = results[False], results[True]
    assert c0 == c1 and c0 > 1000 and a0 == a1 and a0 > 50
    assert n0 > 0, "the plain update must do some Newton work on this workload"
    assert np.abs(p1[8:] - p0[8:]).max() <= 1e-6
    assert np.abs(p1[5] - p0[5]).max() <= 1e-3 * p0[5].max()
    assert n1 < 0.75 * n0, (n0, n1)
