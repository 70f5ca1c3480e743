"""Direct GPU tests of the block kernels against FP64 NumPy: the SpMM
(bksp_gpu_dcsrmm: diagonal form for stencil operators, CSR otherwise) and
the block Gram / update kernel (through myqr's Cholesky QR), for block
widths 1, 5 and 16 (the diagonal form needs a width divisible by its
16-byte vector, 2 doubles: 1 and 5 run the CSR kernel even on a stencil),
row counts that are not multiples of the 32-row tile, and an operator large
enough that every CTA walks many tiles."""
import numpy as np
import pytest
import scipy.sparse as sp

from bksp_b200 import problems as P

pytestmark = pytest.mark.gpu


def _random_csr(n, per_row, seed):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), per_row)
    cols = rng.integers(0, n, n * per_row)
    A = sp.csr_matrix((rng.uniform(-1, 1, n * per_row), (rows, cols)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A


@pytest.mark.parametrize("s", [1, 5, 16])
@pytest.mark.parametrize("kind", ["stencil", "random"])
@pytest.mark.parametrize("n_grid", [13, 70])
def test_spmm_matches_numpy(gpu, s, kind, n_grid):
    B = gpu
    if kind == "stencil":
        rp, c, v, n = P.convdiff3d(n_grid)
        A = sp.csr_matrix((v, c, rp), shape=(n, n))
    else:
        n = n_grid ** 3 + 7                     # not a multiple of 32
        A = _random_csr(n, 9, n_grid)
    rng = np.random.default_rng(s)
    Bm = rng.standard_normal((n, s))
    C0 = rng.standard_normal((n, s))
    C = C0.copy()
    rc = B.dcsrmm(B.CsrMatrix(A.indptr, A.indices, A.data), Bm, C, alpha=-0.75, beta=0.5)
    assert rc == 0
    ref = 0.5 * C0 - 0.75 * (A @ Bm)
    err = np.abs(C - ref).max() / np.abs(ref).max()
    assert err <= 1e-14, err


def test_spmm_symmetric_mirror(gpu):
    B = gpu
    rp, c, v, n = P.poisson3d(9)
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    Bm = np.random.default_rng(3).standard_normal((n, 16))
    C = np.zeros((n, 16))
    assert B.dcsrmm(B.CsrMatrix(lrp, lc, lv, symmetric=True), Bm, C, trans="s") == 0
    assert np.abs(C - A @ Bm).max() <= 1e-14 * np.abs(A @ Bm).max()


@pytest.mark.parametrize("s", [1, 5, 16])
@pytest.mark.parametrize("m", [37, 1000, 200003])
def test_block_gram_update_through_qr(gpu, s, m):
    """myqr runs the block kernel's Gram products and s-by-s updates (three
    Cholesky-QR passes): Q orthonormal, Q R = V, R upper triangular."""
    B = gpu
    V = np.random.default_rng(m + s).standard_normal((m, s))
    Q, R, info = B.myqr(V)
    assert info == 0
    assert np.abs(Q.T @ Q - np.eye(s)).max() <= 1e-12
    assert np.abs(Q @ R - V).max() <= 1e-12 * np.abs(V).max()
    assert np.allclose(np.tril(R, -1), 0.0)
    assert (np.diag(R) > 0).all()


@pytest.mark.parametrize("fp32", [False, True])
def test_spmm_kernels_bit_identical_and_autotuned(gpu, fp32):
    """The diagonal-form and CSR block products add each row's entries in
    the same order with the same rounding, so they agree bit for bit; the
    autotuned launch (either of them) gives the same block."""
    import torch
    rp, c, v, n = P.convdiff3d(48)
    G = gpu.GpuMatrix(gpu.CsrMatrix(rp, c, v), gpu.FP32)
    assert len(G.diagonals()) == 7
    dt = torch.float32 if fp32 else torch.float64
    X = torch.rand(n * 16, dtype=dt, device="cuda") * 2 - 1
    outs = []
    for kern in (0, 1, -1):
        Y = torch.full_like(X, float("nan"))
        G.spmm(16, X.data_ptr(), Y.data_ptr(), fp32, kern)
        torch.cuda.synchronize()
        outs.append(Y.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    ref = A @ X.cpu().numpy().astype(np.float64).reshape(n, 16)
    np.testing.assert_allclose(outs[0].reshape(n, 16), ref,
                               rtol=1e-4 if fp32 else 1e-12, atol=1e-4 if fp32 else 1e-12)
    G.close()
