"""The CPU oracle of the learned split: its analytic gradient against central
finite differences (without the BF16 rounding, which makes the loss
piecewise constant in the weights), and its loss invariances."""
import numpy as np

from oracle import learned


def _problem(seed=0, m=300, d=12, k=5, nodes=3):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((m, d))
    node = rng.integers(0, nodes, size=m)
    nbr = rng.integers(0, m, size=(m, k))
    nbr[rng.random((m, k)) < 0.1] = -1
    W1 = rng.standard_normal((learned.HIDDEN, d)) / np.sqrt(d)
    b1 = rng.standard_normal(learned.HIDDEN) * 0.1
    w2 = rng.standard_normal(learned.HIDDEN) / 8
    return X, W1, b1, w2, 0.3, node, nbr


def test_gradient_matches_finite_differences():
    X, W1, b1, w2, b2, node, nbr = _problem()
    L, dW1, db1, dw2, db2 = learned.loss_and_grad(X, W1, b1, w2, b2, node, nbr, rounded=False)
    rng = np.random.default_rng(1)
    h = 1e-6
    for _ in range(8):
        i, j = rng.integers(0, W1.shape[0]), rng.integers(0, W1.shape[1])
        Wp, Wm = W1.copy(), W1.copy()
        Wp[i, j] += h
        Wm[i, j] -= h
        fd = (learned.loss_and_grad(X, Wp, b1, w2, b2, node, nbr, False)[0] -
              learned.loss_and_grad(X, Wm, b1, w2, b2, node, nbr, False)[0]) / (2 * h)
        assert abs(fd - dW1[i, j]) <= 1e-6 + 1e-5 * abs(fd)
    for i in range(0, learned.HIDDEN, 13):
        for arr, grad in ((b1, db1), (w2, dw2)):
            p, q = arr.copy(), arr.copy()
            p[i] += h
            q[i] -= h
            args_p = (X, W1, p, w2, b2) if arr is b1 else (X, W1, b1, p, b2)
            args_q = (X, W1, q, w2, b2) if arr is b1 else (X, W1, b1, q, b2)
            fd = (learned.loss_and_grad(*args_p, node, nbr, False)[0] -
                  learned.loss_and_grad(*args_q, node, nbr, False)[0]) / (2 * h)
            assert abs(fd - grad[i]) <= 1e-6 + 1e-5 * abs(fd)
    assert abs(db2) < 1e-9  # the loss does not depend on a common shift of f


def test_loss_is_scale_invariant_in_the_output_layer():
    X, W1, b1, w2, b2, node, nbr = _problem(seed=3)
    L1 = learned.loss_and_grad(X, W1, b1, w2, b2, node, nbr, False)[0]
    L2 = learned.loss_and_grad(X, W1, b1, 4 * w2, b2 + 5, node, nbr, False)[0]
    assert abs(L1 - L2) <= 1e-4 * L1  # up to the variance floor eps


def test_bf16_round_ties_to_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e-39], np.float32)
    r = learned.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.015625)
    assert r[3] == -2.5
