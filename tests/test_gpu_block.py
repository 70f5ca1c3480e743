"""GPU parity of the block methods (dblcg, dblbicgstab, dblbicgstabl) and of
the thin QR (myqr) against the compiled reference's golden outputs and the
CPU oracle."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import hist_close, iters_close
from bksp_b200 import problems as P
from oracle import solvers as S

pytestmark = pytest.mark.gpu


def _col_res(A, B, X):
    return [float(np.linalg.norm(B[:, j] - A @ X[:, j]) / np.linalg.norm(B[:, j]))
            for j in range(B.shape[1])]


def test_block_cg_known_answer(gpu, testmats, golden):
    L = gpu.CsrMatrix(testmats["bfwb_rowptr"], testmats["bfwb_col"],
                      testmats["bfwb_val"], symmetric=True)
    Af = S.full_symmetric(sp.csr_matrix(
        (testmats["bfwb_val"], testmats["bfwb_col"], testmats["bfwb_rowptr"]),
        shape=(L.n, L.n)))
    B = np.zeros((L.n, 16)); B[np.arange(16), np.arange(16)] = 1.0
    X = np.zeros((L.n, 16))
    with gpu.record(hist_cap=1000) as st:
        ret = gpu.dblcg(L, B, 1e-14, 500, X)
    g = golden["testc/blcg"]
    assert iters_close(ret, g["ret"], rel=0.1), (ret, g["ret"])
    hist_close(st["hist"], g["hist"], k=15, rtol=1e-5, floor=1e-6)
    assert abs(np.linalg.norm(X) - g["xnorm"]) < 1e-6 * g["xnorm"]
    assert max(_col_res(Af, B, X)) < 1e-10


@pytest.mark.parametrize("key,l", [("testc/blbicgstab", None),
                                   ("testc/blbicgstabl6", 6)])
def test_block_bicgstab_known_answers(gpu, testmats, golden, key, l):
    A = gpu.CsrMatrix(testmats["pde_rowptr"], testmats["pde_col"], testmats["pde_val"])
    As = sp.csr_matrix((testmats["pde_val"], testmats["pde_col"],
                        testmats["pde_rowptr"]), shape=(A.n, A.n))
    B = testmats["pde_B"]
    X = np.zeros_like(B)
    if l is None:
        ret = gpu.dblbicgstab(A, B, 1e-14, 500, X)
    else:
        ret = gpu.dblbicgstabl(A, B, l, 1e-14, 500, X)
    g = golden[key]
    # At tol 1e-14 the reference itself moves (93 vs 87, 15 vs 16) with its
    # BLAS thread count.
    assert iters_close(ret, g["ret"], rel=0.15, abs_=3), (ret, g["ret"])
    assert max(_col_res(As, B, X)) < 1e-9


@pytest.mark.parametrize("key,method", [("cfg3/blcg_p12", "cg"),
                                        ("cfg3/blbicgstab_p12", "bs"),
                                        ("cfg3/blbicgstabl2_p12", "bsl")])
def test_block_seeded_configs(gpu, golden, key, method):
    rp, c, v, n = P.poisson3d(12)
    Af = sp.csr_matrix((v, c, rp), shape=(n, n))
    Bm = np.random.default_rng(2).standard_normal((n, 16))
    X = np.zeros((n, 16))
    with gpu.record(hist_cap=3000) as st:
        if method == "cg":
            lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
            ret = gpu.dblcg(gpu.CsrMatrix(lrp, lc, lv, symmetric=True), Bm, 1e-10, 2000, X)
        elif method == "bs":
            ret = gpu.dblbicgstab(gpu.CsrMatrix(rp, c, v), Bm, 1e-10, 2000, X)
        else:
            ret = gpu.dblbicgstabl(gpu.CsrMatrix(rp, c, v), Bm, 2, 1e-10, 2000, X)
    g = golden[key]
    assert iters_close(ret, g["ret"]), (ret, g["ret"])
    hist_close(st["hist"], g["hist"], floor=1e-8, rtol=1e-5)
    assert max(_col_res(Af, Bm, X)) <= 10 * max(max(g["true_res_cols"]), 1e-12)


def test_myqr(gpu):
    rng = np.random.default_rng(3)
    for m, n in ((1000, 16), (300, 5), (64, 1)):
        V = rng.standard_normal((m, n))
        V[:, -1] += 1e3 * V[:, 0]            # ill-conditioned columns
        Q, R, info = gpu.myqr(V)
        assert info == 0
        assert np.allclose(np.triu(R), R)
        assert np.all(np.diag(R) > 0)
        np.testing.assert_allclose(Q @ R, V, atol=1e-11 * np.abs(V).max())
        np.testing.assert_allclose(Q.T @ Q, np.eye(n), atol=1e-13)
        Qn, Rn = np.linalg.qr(V)
        sgn = np.sign(np.diag(Rn))
        np.testing.assert_allclose(R, sgn[:, None] * Rn, rtol=1e-9, atol=1e-10)


# ------------------------------------------- mixed-precision block solves

@pytest.mark.parametrize("method", ["blcg", "blbicgstabl2"])
def test_mixed_block_reaches_fp64_target(gpu, method):
    """The block configuration's operator (3D Poisson, 24^3 here) with 16
    Gaussian right-hand sides (seed 2): FP64 refinement around FP32 inner
    solves brings every column's FP64 true relative residual to 1e-8, and
    the solution agrees with the FP64 block solve."""
    B_ = gpu
    rp, c, v, n = P.poisson3d(24)
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    Bm = np.random.default_rng(2).standard_normal((n, 16))
    X = np.zeros((n, 16))
    with B_.record() as st:
        if method == "blcg":
            ret = B_.dblcg_mixed(B_.CsrMatrix(lrp, lc, lv, symmetric=True), Bm, X)
        else:
            ret = B_.dblbicgstabl_mixed(B_.CsrMatrix(rp, c, v), Bm, 2, X)
    assert ret >= 0, ret
    res = _col_res(A, Bm, X)
    assert max(res) <= 1e-8, max(res)
    assert abs(st["true_res"] - max(res)) <= 1e-9
    X64 = np.zeros((n, 16))
    if method == "blcg":
        B_.dblcg(B_.CsrMatrix(lrp, lc, lv, symmetric=True), Bm, 1e-10, 5000, X64)
    else:
        B_.dblbicgstabl(B_.CsrMatrix(rp, c, v), Bm, 2, 1e-10, 5000, X64)
    assert np.linalg.norm(X - X64) <= 1e-6 * np.linalg.norm(X64)


def test_mixed_block_cg_refuses_unsymmetric_type(gpu):
    B_ = gpu
    rp, c, v, n = P.poisson3d(6)
    Bm = np.ones((n, 4))
    X = np.zeros((n, 4))
    assert B_.dblcg_mixed(B_.CsrMatrix(rp, c, v), Bm, X) == B_.INVALID_MATRIX_TYPE
