"""The CPU restatement of the learned sensor (oracle/mlp.py) checked on its own (CPU only):
back-propagation against central finite differences, and the modal features on fields whose
modal content is known."""
import numpy as np

from oracle import mlp as omlp
from oracle import oracle as O
from horses2d_b200 import mesh as hmesh


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(omlp.N_PARAMS) * 0.3
    X = rng.standard_normal((64, 16))
    t = (rng.random(64) > 0.5).astype(float)
    w = rng.random(64) + 0.5
    _, g = omlp.loss_grad(p, X, t, w)
    eps = 1e-6
    for k in rng.choice(omlp.N_PARAMS, 40, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        fd = (omlp.loss_grad(pp, X, t, w)[0] - omlp.loss_grad(pm, X, t, w)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-7 + 1e-6 * abs(g[k])


def test_modal_features_of_known_fields():
    orc = O.Oracle(hmesh.cartesian(2, 1, 0.0, 2.0, 0.0, 1.0), 3, nodes=O.LG, bcs=hmesh.periodic_bcs_cartesian())
    X = orc.coords()
    xi = X[:4, 0]
    x, y = X[:, 0] - np.floor(X[:, 0]), X[:, 1]
    # rho = 1 + 0.1 x (xi-linear in each element), p = 1: energy only in modes (0,0) and (1,0) of rho
    Q = np.stack([1.0 + 0.1 * x, 0 * x, 0 * x, 2.5 + 0 * x], 1)
    f, s = omlp.element_features(Q.reshape(2, 16, 4), xi)
    assert np.all(f[:, 2:4] == -10.0) and np.all(f[:, 5:8] == -10.0)      # rho: xi index 2, 3; eta index >= 1
    assert np.all(f[:, 1] > -4.0)                                           # rho: xi index 1 carries the slope
    assert np.all(f[:, 9:12] == -10.0) and np.all(f[:, 13:16] == -10.0)    # p uniform
    assert np.all(s < -10.0)                                                # no energy in the top modes
    # a cubic in eta puts energy in the top eta mode
    Q3 = np.stack([1.0 + 0.1 * y ** 3, 0 * x, 0 * x, 2.5 + 0 * x], 1)
    f3, s3 = omlp.element_features(Q3.reshape(2, 16, 4), xi)
    assert np.all(f3[:, 7] > -6.0) and np.all(s3 > -6.0)
