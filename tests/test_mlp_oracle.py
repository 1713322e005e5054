"""The MLP oracle's hand-written backpropagation against central finite
differences (CPU), so it can serve as the checker of the GPU training kernels."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init_params(3).astype(np.float64)
    X = rng.normal(0, 1, (17, M.IN))
    y = (rng.random(17) < 0.3).astype(np.float64)
    loss, g = M.loss_and_grad(p, X, y, pos_weight=4.0)
    idx = rng.choice(M.NPARAM, 60, replace=False)
    idx = np.concatenate([idx, [M.NPARAM - 1, 0]])
    h = 1e-6
    for i in idx:
        e = np.zeros(M.NPARAM)
        e[i] = h
        lp, _ = M.loss_and_grad(p + e, X, y, 4.0)
        lm, _ = M.loss_and_grad(p - e, X, y, 4.0)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])
    assert loss > 0


def test_param_count_matches_abi():
    from zuikakucfd_b200 import _native
    assert M.NPARAM == _native.MLP_NPARAM == 3457
