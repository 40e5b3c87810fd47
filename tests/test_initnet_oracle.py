"""The FP64 restatement of the learned initialiser's network (oracle/netoracle.py) against finite
differences: the checker of the GPU gradients is itself checked."""
import numpy as np


def test_network_oracle_gradient_matches_finite_differences():
    from oracle import netoracle as N
    rng = np.random.default_rng(3)
    n = sum(27 * ci * co + co for ci, co, _, _ in N.LAYERS)
    params = rng.standard_normal(n) * 0.15
    x = rng.random((1, 8, 8, 8, 2))
    t = rng.standard_normal((1, 2, 2, 2, 3)) * 0.5
    _, loss, g = N.forward_backward(params, x, t, round=False)
    # a few parameters of every layer, central differences in FP64
    offs, o = [], 0
    for ci, co, _, _ in N.LAYERS:
        offs.append((o, 27 * ci * co + co))
        o += 27 * ci * co + co
    h = 1e-5
    for o, size in offs:
        for j in rng.choice(size, 3, replace=False):
            p = params.copy()
            p[o + j] += h
            lp = N.forward_backward(p, x, t, round=False)[1]
            p[o + j] -= 2 * h
            lm = N.forward_backward(p, x, t, round=False)[1]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[o + j]) <= 1e-6 + 1e-4 * abs(fd), (o, j, fd, g[o + j])


def test_network_oracle_rounding_is_bf16():
    from oracle import netoracle as N
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, -3.140625, 1e-3])
    r = N.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie rounds to even
    assert r[2] == 1.0 + 2 ** -6 or r[2] == 1.0 + 2 ** -7
    assert abs(r[4] - 1e-3) / 1e-3 < 2 ** -8
