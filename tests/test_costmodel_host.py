"""The cost model's CPU oracle and the autotuner's host logic (no GPU).

The oracle (oracle/mlp_oracle.py) is pinned against central finite
differences here; the GPU kernels are then checked against the oracle in
tests/test_gpu_autotune.py.
"""

import numpy as np

from oracle import mlp_oracle as MO
from pureumfpack.autotune import NFEAT, NIN, LaunchTable, _design


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin, h = 5, 7
    p = rng.standard_normal(MO.nparams(nin, h)) * 0.5
    X = rng.standard_normal((40, nin))
    Y = rng.standard_normal(40)
    _, g = MO.loss_grad(p, X, Y, nin, h)
    eps = 1e-6
    fd = np.empty_like(p)
    for q in range(len(p)):
        e = np.zeros_like(p)
        e[q] = eps
        fd[q] = (MO.loss_grad(p + e, X, Y, nin, h)[0] - MO.loss_grad(p - e, X, Y, nin, h)[0]) / (2 * eps)
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-9)


def test_table_cost_best_and_design():
    feats = np.arange(3 * NFEAT, dtype=np.float32).reshape(3, NFEAT)
    t = LaunchTable(feats, np.array([[1.0, 2.0], [5.0, 3.0], [4.0, 4.5]]), np.array([1, 1, 1]))
    np.testing.assert_array_equal(t.best, [1, 2, 1])
    assert t.cost(t.best) == 8.0 and t.cost(t.rule) == 10.0 and t.cost([2, 2, 2]) == 9.5
    X = _design(feats)
    assert X.shape == (6, NIN)
    np.testing.assert_array_equal(X[0, NFEAT:], [1, 0])
    np.testing.assert_array_equal(X[1, NFEAT:], [0, 1])
    np.testing.assert_array_equal(X[2, :NFEAT], feats[1])
