"""The cost model's CPU restatement (oracle/mlp_oracle.py) against central
finite differences, so that it can serve as the gradient check of the
library's CUDA forward/backward kernels (tests/test_gpu_model.py)."""
import numpy as np

import mlp_oracle as M


def test_param_count_matches_header():
    assert M.param_count() == 1638


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    w = M.init(3)
    x = rng.uniform(0, 1, (17, M.F))
    t = rng.uniform(5, 11, (17, M.P))
    mask = rng.integers(0, 2, (17, M.P)).astype(np.uint8)
    mask[0, 0] = 1
    loss, g = M.loss_and_grad(w, x, t, mask)
    assert loss > 0
    idx = rng.choice(w.size, size=60, replace=False)
    eps = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        num = (M.loss_and_grad(wp, x, t, mask)[0] - M.loss_and_grad(wm, x, t, mask)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])


def test_oracle_masked_entries_do_not_contribute():
    rng = np.random.default_rng(1)
    w = M.init(5)
    x = rng.uniform(0, 1, (4, M.F))
    t = rng.uniform(5, 11, (4, M.P))
    mask = np.zeros((4, M.P), np.uint8)
    mask[:, 2] = 1
    l1, g1 = M.loss_and_grad(w, x, t, mask)
    t2 = t.copy()
    t2[:, 0] += 100
    l2, g2 = M.loss_and_grad(w, x, t2, mask)
    assert l1 == l2 and np.array_equal(g1, g2)
