"""The surrogate network's CPU restatement checked on its own (no GPU):
the analytic gradient of the float64 network against central finite
differences of its loss."""
import numpy as np

from oracle import nn_oracle as nn


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0.0, 0.3, nn.NPARAM)
    X = rng.uniform(-1, 1, (32, 4))
    Y = rng.uniform(-1, 1, (32, 2))
    loss, g = nn.loss_grad(p, X, Y, bf=False)
    idx = rng.choice(nn.NPARAM, 60, replace=False)
    idx = np.concatenate([idx, [nn.P_B1, nn.P_B2, nn.P_B3, nn.P_B3 + 1, nn.P_W3]])
    h = 1e-6
    for k in idx:
        q = p.copy()
        q[k] += h
        lp, _ = nn.loss_grad(q, X, Y, bf=False)
        q[k] -= 2 * h
        lm, _ = nn.loss_grad(q, X, Y, bf=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, 1.0 + 3 * 2 ** -8, -2.5, 0.0],
                 np.float32)
    r = nn.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # half-way: ties to the even neighbour
    assert r[2] == 1.0                      # below half-way
    assert r[3] == 1.0 + 2 ** -7            # above half-way
    assert r[4] == 1.0 + 2 ** -6            # half-way between odd and even: up to even
    assert r[5] == -2.5 and r[6] == 0.0
