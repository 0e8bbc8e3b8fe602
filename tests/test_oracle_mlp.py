"""The MLP oracle (float64) pinned by central finite differences and known bfloat16 roundings."""
import numpy as np

from oracle import mlp_ref as M


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, M.NF)) * np.array([0.3, 0.5, 1.0, 0.4, 0.6, 0.02, 0.02, 2.0]) + 0.5
    y = (rng.random(n) < 0.4).astype(np.float64)
    return x, y


def test_gradient_matches_finite_differences():
    x, y = _data(64, 1)
    p = M.init_params(x.mean(0), x.std(0), seed=3).astype(np.float64)
    p[M.OFF_B1:M.OFF_W2] = 0.05   # keep ReLU kinks away from the probes
    p[M.OFF_B2:M.OFF_W3] = 0.05
    _, g = M.grad(p, x, y)
    rng = np.random.default_rng(5)
    idx = np.r_[rng.choice(M.N_TRAIN, 60, replace=False), M.OFF_B3]
    eps = 1e-6
    for i in idx:
        a, b = p.copy(), p.copy()
        a[i] += eps
        b[i] -= eps
        fd = (M.loss(a, x, y) - M.loss(b, x, y)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding_known_values():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, 3.14159265, -2.5e-3, 65504.0], np.float32)
    want = np.array([1.0, 1.0, 1.0078125, 1.0078125, 3.140625, -0.0025024414, 65536.0])
    np.testing.assert_allclose(M.bf16(v), want, rtol=0, atol=1e-9)


def test_adam_step_moves_against_gradient():
    x, y = _data(128, 2)
    p = M.init_params(x.mean(0), x.std(0), seed=4).astype(np.float64)
    l0, g = M.grad(p, x, y)
    p1, _, _ = M.adam(p, np.zeros(M.N_TRAIN), np.zeros(M.N_TRAIN), g, 1, 1e-3)
    assert M.loss(p1, x, y) < l0
