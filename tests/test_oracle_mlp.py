"""The CPU oracle of the learned predictor (oracle/mlp.py) checked on its own: its
analytic gradient against central finite differences (FP64, no BF16 rounding), its BF16
rounding against the bit pattern rule, and the neighbour order of its features."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import mlp as M  # noqa: E402


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    B = 12
    X = rng.normal(0.0, 1.0, (B, M.MI))
    T = rng.normal(0.0, 0.3, (B, 3))
    P = M.init_params(seed=1, out_scale=1.0).astype(np.float64)
    loss, G, _ = M.loss_and_grad(X, T, P, exact=True)
    h = 1e-6
    for i in rng.choice(M.NPARAM, 40, replace=False).tolist() + [M.OB4, M.OB4 + 2, M.OW4 + 5, M.OB1 + 3]:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (M.loss_and_grad(X, T, Pp, exact=True)[0] - M.loss_and_grad(X, T, Pm, exact=True)[0]) / (2 * h)
        assert abs(fd - G[i]) <= 1e-6 * max(1.0, abs(G[i])) + 1e-9, (i, fd, G[i])


def test_bf16_rounding():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265, 1e-30], dtype=np.float32)
    r = M.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0                   # tie to even
    assert r[2] == np.float32(1.0 + 4 * 2 ** -8)         # tie to even, upwards
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-7
    assert (r.view(np.uint32) & 0xFFFF == 0).all()


def test_feature_neighbours():
    shape = (4, 3, 2)
    N = 24
    x0 = np.zeros((3, N))
    x1 = np.zeros((3, N))
    x1[0] = np.arange(N, dtype=float)                    # psi = k, so d = k / VT
    f = M.features(shape, x1, x0, 1.0, np.zeros(4), 1.0, np.zeros(N), 0.0, np.zeros(N, int), np.zeros(N, int))
    k = 1 + 4 * (1 + 3 * 1)                               # (i, j, l) = (1, 1, 1)
    assert list(f[k, 0:7]) == [k, k - 1, k + 1, k - 4, k + 4, k - 12, k]   # z+ missing: repeats k
    assert f[0, 1] == 0 and f[0, 3] == 0 and f[0, 5] == 0                  # minus sides at the corner
