"""CPU checks of the learned-preconditioner oracle: its analytic gradient
matches central finite differences, and an untrained (Jacobi-initialised)
parameter vector yields M = diag(A)^-1."""
import numpy as np

from bksp_b200 import problems as P
from oracle import mlp


def _init(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(5256)
    W1, b1, W2, b2, W3, b3 = mlp.unpack(p)   # views
    W1[...] = rng.uniform(-0.8, 0.8, W1.shape)
    W2[...] = rng.uniform(-0.3, 0.3, W2.shape)
    W3[...] = rng.uniform(-0.1, 0.1, W3.shape)
    b1[...] = 0.05
    b2[...] = 0.05
    b3[mlp.C] = 1.0
    return p


def test_slots_of_stencils():
    rp, c, v, n = P.convdiff3d(5)
    se = mlp.slots(rp, c, n)
    i = 2 + 5 * (2 + 5 * 2)            # interior point: all 7 slots
    assert (se[i, :7] >= 0).all() and se[i, 7] == -1
    assert c[se[i, 3]] == i and c[se[i, 2]] == i - 1 and c[se[i, 4]] == i + 1
    assert c[se[i, 0]] == i - 25 and c[se[i, 6]] == i + 25
    rp, c, v, n = P.poisson2d(6)
    se = mlp.slots(rp, c, n)
    assert (se[:, 0] == -1).all() and (se[:, 6] == -1).all()


def test_gradient_matches_finite_differences():
    rp, c, v, n = P.convdiff2d(7)
    rng = np.random.default_rng(1)
    Z = rng.choice([-1.0, 1.0], size=(3, n))
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp))
    A[rows, c] = v
    AZ = Z @ A.T
    p = _init(2)
    loss, g = mlp.loss_grad(p, rp, c, v, n, Z, AZ)
    idx = np.r_[0:5, 512:517, 700:705, 4672:4677, 5248:5256]
    eps = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        fd = (mlp.loss_grad(pp, rp, c, v, n, Z, AZ)[0]
              - mlp.loss_grad(pm, rp, c, v, n, Z, AZ)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_untrained_model_is_jacobi():
    rp, c, v, n = P.convdiff3d(4)
    p = np.zeros(5256)
    p[-8 + mlp.C] = 1.0
    mv = mlp.spai_values(p, rp, c, v, n)
    rows = np.repeat(np.arange(n), np.diff(rp))
    diag = c == rows
    assert np.allclose(mv[diag], 1.0 / v[diag]) and np.all(mv[~diag] == 0)
