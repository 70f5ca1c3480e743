"""CPU checks of the synthetic workload generators."""
import numpy as np
import scipy.sparse as sp

from bksp_b200 import problems as P


def test_gaussian_random_field_statistics():
    g = P.gaussian_random_field(48, 7)
    assert abs(g.mean()) < 1e-12 and abs(g.var() - 1.0) < 1e-9
    # correlation length 0.1 on the unit cube: neighbours (h = 1/48) are
    # strongly correlated, points half the cube apart are not
    c1 = np.corrcoef(g[:-1].ravel(), g[1:].ravel())[0, 1]
    c24 = np.corrcoef(g[:24].ravel(), g[24:].ravel())[0, 1]
    assert c1 > 0.8 and abs(c24) < 0.2
    assert np.array_equal(g, P.gaussian_random_field(48, 7))


def test_kappa_diffusion_operator():
    rp, c, v, n = P.kappa_diffusion3d(9, 3)
    assert n == 729
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    assert abs(A - A.T).max() == 0.0                 # symmetric
    assert np.all(np.diff(rp) <= 7)
    d = A.diagonal()
    off = np.asarray(abs(A).sum(axis=1)).ravel() - d
    assert np.all(d >= off - 1e-12)                  # diagonally dominant
    assert np.any(d > off + 1e-9)                    # strictly on boundary rows
    assert np.linalg.eigvalsh(A.toarray()).min() > 0  # positive definite
    # columns ascend within each row (the C-ABI's diagonal form needs it)
    for i in range(n):
        assert np.all(np.diff(c[rp[i]:rp[i + 1]]) > 0)


def test_kappa_batch_sizes():
    out = P.kappa_batch(count=3, lo=4, hi=6)
    for rp, c, v, n, b in out:
        L = round(n ** (1 / 3))
        assert L ** 3 == n and 4 <= L <= 6 and b.shape == (n,)
