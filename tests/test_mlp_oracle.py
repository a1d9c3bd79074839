"""The CPU MLP oracle against finite differences (CPU only)."""

import numpy as np

from oracle import mlp as om


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    W = [rng.standard_normal((128, 64)) * 0.1, rng.standard_normal((64, 64)) * 0.1, rng.standard_normal((64, 64)) * 0.1]
    b = [rng.standard_normal(64) * 0.1 for _ in range(3)]
    x = rng.standard_normal((7, 128))
    t = rng.standard_normal((7, 64))
    loss, gW, gb = om.loss_and_grads(x, t, W, b, bf16=False)
    for layer, (i, j) in [(0, (3, 5)), (1, (10, 2)), (2, (63, 0))]:
        e = 1e-6
        Wp = [w.copy() for w in W]
        Wp[layer][i, j] += e
        Wm = [w.copy() for w in W]
        Wm[layer][i, j] -= e
        lp = om.loss_and_grads(x, t, Wp, b, bf16=False)[0]
        lm = om.loss_and_grads(x, t, Wm, b, bf16=False)[0]
        assert abs((lp - lm) / (2 * e) - gW[layer][i, j]) <= 1e-6 * max(1.0, abs(gW[layer][i, j]))
    bp = [v.copy() for v in b]
    bp[1][7] += 1e-6
    bm = [v.copy() for v in b]
    bm[1][7] -= 1e-6
    fd = (om.loss_and_grads(x, t, W, bp, bf16=False)[0] - om.loss_and_grads(x, t, W, bm, bf16=False)[0]) / 2e-6
    assert abs(fd - gb[1][7]) <= 1e-6


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.1415927], dtype=np.float32)
    r = om.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway rounds to even mantissa
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-7
