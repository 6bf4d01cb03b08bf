"""The float64 oracle of the warm-start MLP: its backward pass agrees with
central finite differences of its own loss (plain float64 network)."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, size=M.NPARAM)
    norm = np.zeros(96)
    norm[M.XI:M.XI + M.DIN] = 1.0
    norm[M.YS:96] = 1.0
    X = rng.normal(size=(7, M.DIN))
    T = rng.normal(size=(7, M.USED))
    loss, g = M.forward_backward(p, norm, X, T, rounded=False)
    h = 1e-6
    for block, (a, b) in {"W1": (M.OW1, M.OB1), "b1": (M.OB1, M.OW2), "W2": (M.OW2, M.OB2),
                          "b3": (M.OB3, M.OW4), "W4": (M.OW4, M.OB4), "b4": (M.OB4, M.NPARAM)}.items():
        for i in rng.choice(np.arange(a, b), size=4, replace=False):
            e = np.zeros(M.NPARAM)
            e[i] = h
            fd = (M.forward_backward(p + e, norm, X, T, rounded=False)[0]
                  - M.forward_backward(p - e, norm, X, T, rounded=False)[0]) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (block, i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-5], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0               # tie to even
    assert r[2] == 1.0 + 2 ** -7                      # above the tie rounds up
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-5) <= 3.0e-5 * 2 ** -8
