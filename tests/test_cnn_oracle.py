"""CPU checks of the learned-correction oracle: its float64 backpropagation
against central finite differences, and its BF16 rounding helper."""
import numpy as np

from oracle import cnn_oracle as C


def small_problem(seed=0, B=1, H=4, W=5):
    rng = np.random.default_rng(seed)
    p = C.init_params(seed, zero_last=False).astype(np.float64)
    x = np.zeros((B, H, W, 16))
    x[..., :5] = rng.standard_normal((B, H, W, 5)) * 0.3
    base = rng.standard_normal((B, H, W)) * 0.02
    target = base + rng.standard_normal((B, H, W)) * 0.001
    return p, x, base, target


def test_bf16_rounding_ties_to_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e-3], dtype=np.float32)
    r = C.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0  # tie -> even (mantissa ...0)
    assert r[2] == 1.0 + 4 * 2 ** -8  # tie -> even (mantissa ...10)
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) < 3.0e-3 * 2 ** -8


def test_parameter_count_and_layout():
    assert C.param_count() == 9 * 16 * 32 + 32 + 6 * (9 * 32 * 32 + 32) + 9 * 32 * 16 + 16
    p = np.arange(C.param_count(), dtype=np.float32)
    (w0, b0) = C.split(p)[0]
    assert w0.shape == (32, 9, 16) and w0[1, 0, 0] == 9 * 16 and b0[0] == 9 * 16 * 32


def test_backprop_matches_finite_differences():
    mu = 0.0193
    p, x, base, target = small_problem()
    loss, g = C.loss_and_grads(p, x, base, target, mu, bf16_mode=False)
    rng = np.random.default_rng(1)
    # a few parameters of every layer, avoiding padded (always-zero) channels
    idx = []
    o = 0
    for l, (ci, co) in enumerate(zip(C.CIN, C.COUT)):
        ci_r = 5 if l == 0 else ci
        co_r = 1 if l == 7 else co
        for _ in range(3):
            c, t, i = rng.integers(co_r), rng.integers(9), rng.integers(ci_r)
            idx.append(o + (c * 9 + t) * ci + i)
        idx.append(o + 9 * ci * co + rng.integers(co_r))
        o += 9 * ci * co + co

    def f(pp):
        pred, _, _ = C.forward(pp, x, base, mu, bf16_mode=False)
        e = (pred - target) / mu
        return np.mean(e * e)

    for k in idx:
        h = 1e-6 * max(abs(p[k]), 1e-2)
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        num = (f(pp) - f(pm)) / (2 * h)
        assert abs(num - g[k]) <= 1e-5 * max(abs(g[k]), 1e-3 * abs(loss)), (k, num, g[k])
