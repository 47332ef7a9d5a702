"""The NumPy restatement of the refine-flag forecaster pinned by central
finite differences (FP64, roundings off): the gradient it returns is the
derivative of the loss it returns."""
import numpy as np

import net_ref


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((3, 4, 18, 18))
    y = np.array([1.0, 0.0, 1.0])
    p = rng.standard_normal(net_ref.NPARAM) * 0.2
    net_ref.EXACT = True
    try:
        _, g, _ = net_ref.loss_and_grad(p, x, y, pos_weight=2.0)
        idx = np.concatenate([rng.integers(a, b, 4) for a, b in (
            (net_ref.O_W1, net_ref.O_B1), (net_ref.O_B1, net_ref.O_W2), (net_ref.O_W2, net_ref.O_B2),
            (net_ref.O_W3, net_ref.O_B3), (net_ref.O_B3, net_ref.O_WD), (net_ref.O_WD, net_ref.O_BD))]
                              + [[net_ref.O_BD]])
        h = 1e-6
        for i in idx:
            q = p.copy()
            q[i] += h
            lp = net_ref.loss_and_grad(q, x, y, 2.0)[0]
            q[i] -= 2 * h
            lm = net_ref.loss_and_grad(q, x, y, 2.0)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])
    finally:
        net_ref.EXACT = False
