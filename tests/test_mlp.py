"""Learned selector network: the numpy oracle against finite differences (CPU),
and the engine's CUDA forward/backward, training and inference kernels against
the oracle (GPU)."""
import numpy as np
import pytest

import indigo2suite_b200 as i2
from oracle import mlp_oracle as mo


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, mo.F)).astype(np.float32) * 3 + 1
    T = rng.normal(10, 2, (n, mo.O)).astype(np.float32)
    M = (rng.random((n, mo.O)) < 0.8).astype(np.float32)
    M[:, 2] = 1
    return X, T, M


def _params(seed=3):
    p = mo.init_params(seed)
    rng = np.random.default_rng(seed + 1)
    p[mo.OFF_MU:mo.OFF_SD] = rng.normal(0, 1, mo.F)
    p[mo.OFF_SD:mo.OFF_W1] = rng.uniform(0.5, 2.0, mo.F)
    p[mo.OFF_B1:mo.OFF_W2] = rng.normal(0, 0.1, mo.H)
    return p.astype(np.float32)


def test_param_count_matches_engine():
    assert i2.mlp_param_count() == mo.NPARAMS


def test_oracle_gradient_matches_finite_differences():
    X, T, M = _data(40, 1)
    p = _params().astype(np.float64)
    _, g = mo.loss_grad(p, X, T, M)
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(np.arange(mo.OFF_W1, mo.NPARAMS), 60, replace=False)])
    eps = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        fd = (mo.loss_grad(pp, X, T, M)[0] - mo.loss_grad(pm, X, T, M)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)), (k, fd, g[k])
    assert np.all(g[:mo.OFF_W1] == 0)


@pytest.mark.gpu
def test_device_loss_and_gradient_match_oracle(gpu):
    # fp32 kernels vs float64 oracle: relative tolerance 1e-4 on the loss, and
    # |g - g_ref| <= 1e-4 * max|g_ref| + 1e-6 on the gradient
    for n, seed in ((1, 5), (31, 6), (32, 7), (333, 8), (2048, 9)):
        X, T, M = _data(n, seed)
        p = _params(seed)
        loss, g = i2.mlp_loss_grad(p, X, T, M)
        rloss, rg = mo.loss_grad(p, X, T, M)
        assert abs(loss - rloss) <= 1e-4 * abs(rloss) + 1e-6, (n, loss, rloss)
        tol = 1e-4 * np.abs(rg).max() + 1e-6
        assert np.abs(g - rg).max() <= tol, (n, np.abs(g - rg).max(), tol)


@pytest.mark.gpu
def test_device_training_reduces_loss_and_inference_matches_oracle(gpu):
    # a learnable target: the per-variant "time" is a fixed random function of x
    rng = np.random.default_rng(11)
    X = rng.normal(0, 1, (4000, mo.F)).astype(np.float32)
    Wt = rng.normal(0, 1, (mo.F, mo.O))
    T = (np.tanh(X @ Wt) * 3 + 10).astype(np.float32)
    M = np.ones_like(T)
    p0 = mo.init_params(1)
    l0 = mo.loss_grad(np.concatenate([X.mean(0), X.std(0), p0[mo.OFF_W1:]]), X, T, M)[0]
    p, loss = i2.mlp_train(p0, X, T, M, epochs=60, batch=256, lr=3e-3, seed=2)
    assert loss < 0.2 * l0, (loss, l0)
    np.testing.assert_allclose(p[:mo.OFF_SD], X.mean(0), rtol=1e-4, atol=1e-4)
    # inference: device argmin equals the oracle's except where the two best
    # predictions are within fp32 rounding of each other
    choice = i2.mlp_predict(p, X[:500], allowed_mask=0b11110111)
    y = mo.forward(p, X[:500])[-1]
    ref = mo.predict(p, X[:500], allowed_mask=0b11110111)
    mism = np.flatnonzero(choice != ref)
    for r in mism:
        assert abs(y[r, choice[r]] - y[r, ref[r]]) < 1e-4
    assert len(mism) <= 2
    assert not np.any(choice == 3)


def test_union_find_time_is_scaled_to_one_iterations_share():
    from indigo2suite_b200 import selector

    uf = selector.UF
    times = np.full((3, i2.I2_NUM_VARIANTS), -1.0)
    times[:, 2] = [10.0, 20.0, 30.0]  # the followed style
    times[:, uf] = [60.0, 40.0, 100.0]
    recs = [{"variant": 2}] * 3
    out = selector._union_find_equivalent(recs, times)
    # remaining after k: 50, 30, 0 -> uf scaled by f/(f+rest): 10/60, 20/50, 30/30
    np.testing.assert_allclose(out[:, uf], [10.0, 16.0, 100.0])
    np.testing.assert_array_equal(out[:, 2], times[:, 2])
    # union-find is preferred exactly when it beats finishing along the trajectory
    assert out[0, uf] <= out[0, 2] and out[1, uf] < out[1, 2] and out[2, uf] > out[2, 2]
