"""The radiance-cache oracle (oracle/radiance_cache.py) checked on its own, on CPU: its
backward pass against central finite differences of the same network in float64, its BF16
rounding helper against torch, and its configuration rules."""
import numpy as np
import pytest

import radiance_cache as rc


def small_cache(seed=0, log2_table=10, min_res=4, max_res=64):
    rng = np.random.default_rng(seed)
    res = rc.resolutions(min_res, max_res)
    grid = rng.uniform(-1, 1, (rc.LEVELS, 1 << log2_table, 2)).astype(np.float16).view(np.uint16)
    mlp = rc.bf16_bits(rng.uniform(-0.3, 0.3, rc.WEIGHTS).astype(np.float32))
    c = rc.Cache(res, log2_table, [-1, -1, -1], [1, 1, 1], grid, mlp)
    return c, rng


def random_records(rng, n, lo=-1.2, hi=1.2):
    r = np.zeros((n, 16), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3))
    r[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    r[:, 9] = rng.uniform(0, 1, n)
    r[:, 10:16] = rng.uniform(0, 1, (n, 6))
    return r


def test_resolutions_are_geometric():
    res = rc.resolutions(16, 2048)
    assert res[0] == 16 and res[-1] == 2048
    assert all(b > a for a, b in zip(res, res[1:]))
    assert rc.dense_mask(res, 1 << 19) == 0b11111  # 16, 22, 30, 42, 58: (n+1)^3 <= 2^19


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(1).normal(size=10000).astype(np.float32) * 10.0 ** np.random.default_rng(2).integers(
        -20, 20, 10000)
    ours = rc.bf16_round(x)
    theirs = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(ours, theirs)


def test_encoding_features_interpolate_corners():
    c, rng = small_cache()
    recs = random_records(rng, 50)
    x32 = rc.encode(c, recs)
    x64 = rc.encode64(c, recs)
    np.testing.assert_allclose(x32, x64, rtol=1e-5, atol=1e-6)
    assert np.all(x32[:, 57] == 1.0) and np.all(x32[:, 58:] == 0.0)
    # tent encoding of each direction component sums to 1 in [-1, 1]
    for a in range(3):
        np.testing.assert_allclose(x32[:, 32 + 5 * a:37 + 5 * a].sum(1), 1.0, rtol=1e-6)


def test_backward_matches_finite_differences():
    c, rng = small_cache(seed=3)
    n = 24
    recs = random_records(rng, n)
    targets = rng.uniform(0.1, 2.0, (n, 3))
    Ws = [w.copy() for w in c.W]
    grid = c.grid.astype(np.float64)
    c.grid = grid
    x = rc.encode64(c, recs)
    a, y = rc.forward(Ws, x, rounded=False)
    loss, gy = rc.loss_and_grad(y, targets, rounded=False)
    den = y[:, :3] ** 2 + 0.01
    dW, g_in = rc.backward(Ws, a, gy, rounded=False)
    gg = rc.grid_grad(c, recs, g_in)
    eps = 1e-6
    # weights
    for _ in range(40):
        l = int(rng.integers(0, 5))
        o = int(rng.integers(0, 3 if l == 4 else 64))
        i = int(rng.integers(0, 64))
        Wp = [w.copy() for w in Ws]
        Wm = [w.copy() for w in Ws]
        Wp[l][o, i] += eps
        Wm[l][o, i] -= eps
        num = (rc.loss_unrounded_full(c, Wp, grid, recs, targets, den) - rc.loss_unrounded_full(c, Wm, grid, recs, targets, den)) / (
            2 * eps)
        assert abs(num - dW[l][o, i]) <= 1e-5 * max(1.0, abs(num)), (l, o, i, num, dW[l][o, i])
    # grid entries touched by the batch
    touched = np.argwhere(np.abs(gg).sum(-1) > 0)
    for k in rng.choice(len(touched), 40, replace=False):
        l, e = touched[k]
        f = int(rng.integers(0, 2))
        gp = grid.copy()
        gm = grid.copy()
        gp[l, e, f] += eps
        gm[l, e, f] -= eps
        num = (rc.loss_unrounded_full(c, Ws, gp, recs, targets, den) - rc.loss_unrounded_full(c, Ws, gm, recs, targets, den)) / (
            2 * eps)
        assert abs(num - gg[l, e, f]) <= 1e-5 * max(1.0, abs(num)), (l, e, f, num, gg[l, e, f])


def test_adam_first_step_moves_by_learning_rate():
    p = np.array([1.0, -2.0, 0.5, 0.0], np.float32)
    g = np.array([0.3, -1e-3, 0.0, 5.0], np.float32)
    p2, m2, v2 = rc.adam(p, np.zeros(4), np.zeros(4), g, 1e-2, 0.9, 0.99, 1e-15, 1)
    np.testing.assert_allclose(p2, [0.99, -1.99, 0.5, -0.01], rtol=1e-6)
    p3, _, _ = rc.adam(p, np.zeros(4), np.zeros(4), g, 1e-2, 0.9, 0.99, 1e-15, 1, active=g != 0)
    assert p3[2] == 0.5 and p3[0] == p2[0]
