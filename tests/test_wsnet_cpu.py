"""The CPU restatement of the warm-start network (the checker of the device
kernels) checked against finite differences of its own loss, in float64
without BF16 rounding, and its BF16 rounding against known values."""

import numpy as np

import oracle.wsnet as W


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 3.140625, 1e-30], dtype=np.float32)
    r = W.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                     # tie -> even
    assert r[2] == 1.0 + 4 * 2 ** -8       # tie -> even (up)
    assert r[3] == -2.5 and r[4] == 0.0 and r[5] == 3.140625
    assert abs(r[6] - 1e-30) <= 1e-30 * 2 ** -8


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(size=W.NPARAM) * 0.3
    X = rng.normal(size=(40, 16))
    X[:, 13:] = 0
    T = rng.normal(size=(40, 2))
    inv = 1.0 / 40
    loss, g = W.gradients(p, X, T, inv, exact=True)
    idx = np.concatenate([rng.choice(np.arange(a, b), size=min(6, b - a), replace=False)
                          for a, b in ((0, 1024), (1024, 5120), (5120, 9216), (9216, 9344), (9344, 9408),
                                       (9408, 9472), (9472, 9536), (9536, 9538))])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (W.gradients(pp, X, T, inv, exact=True)[0] - W.gradients(pm, X, T, inv, exact=True)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
