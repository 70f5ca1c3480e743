"""GPU parity of the shifted methods (dshbicg, dshbicgstabl) against the
compiled reference's golden outputs and the CPU oracle: iteration index,
residual history, the seed's and every shift's FP64 true residual."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import hist_close, iters_close
from bksp_b200 import problems as P
from oracle import solvers as S

pytestmark = pytest.mark.gpu


def _pde(B, tm):
    A = B.CsrMatrix(tm["pde_rowptr"], tm["pde_col"], tm["pde_val"])
    As = sp.csr_matrix((tm["pde_val"], tm["pde_col"], tm["pde_rowptr"]),
                       shape=(A.n, A.n))
    return A, As


def _shift_res(As, b, x, sig):
    n = b.size
    return [S.true_residual(As, b, x[(k + 1) * n:(k + 2) * n], s)
            for k, s in enumerate(sig)]


@pytest.mark.parametrize("key,l,maxit", [("testc/shbicg", None, 500),
                                         ("testc/shbicgstabl1", 1, 200)])
def test_shifted_known_answers(gpu, testmats, golden, key, l, maxit):
    A, As = _pde(gpu, testmats)
    n = A.n
    b = np.zeros(n); b[0] = 1.0
    sig = np.array([0.0, 0.2, 0.4, 0.8])
    x = np.zeros(n * 5)
    with gpu.record(hist_cap=1000) as st:
        if l is None:
            ret = gpu.dshbicg(A, b, sig, 1e-14, maxit, x)
        else:
            ret = gpu.dshbicgstabl(A, b, l, sig, 1e-14, maxit, x)
    g = golden[key]
    assert iters_close(ret, g["ret"], rel=0.08), (ret, g["ret"])
    hist_close(st["hist"], g["hist"], floor=1e-6)
    assert S.true_residual(As, b, x[:n]) < 1e-12
    res = _shift_res(As, b, x, sig)
    assert max(res) < 100 * max(max(g["true_res_shifts"]), 1e-15), res


@pytest.mark.parametrize("key,l", [("cfg4/shbicg_cd48", None),
                                   ("cfg4/shbicgstabl4_cd48", 4)])
def test_shifted_seeded_config(gpu, golden, key, l):
    rp, c, v, n = P.convdiff2d(48)
    As = sp.csr_matrix((v, c, rp), shape=(n, n))
    A = gpu.CsrMatrix(rp, c, v)
    b = P.uniform(n, 3)
    sig = P.log_shifts(32)
    x = np.zeros(n * 33)
    with gpu.record(hist_cap=5000) as st:
        if l is None:
            ret = gpu.dshbicg(A, b, sig, 1e-10, 2000, x)
        else:
            ret = gpu.dshbicgstabl(A, b, l, sig, 1e-10, 2000, x)
    g = golden[key]
    assert iters_close(ret, g["ret"]), (ret, g["ret"])
    hist_close(st["hist"], g["hist"], floor=1e-8)
    res = _shift_res(As, b, x, sig)
    assert max(res) <= 10 * max(g["true_res_shifts"]), (max(res), max(g["true_res_shifts"]))


def test_shifted_matches_oracle_solution(gpu):
    rp, c, v, n = P.convdiff2d(20)
    As = sp.csr_matrix((v, c, rp), shape=(n, n))
    A = gpu.CsrMatrix(rp, c, v)
    b = P.uniform(n, 9)
    sig = np.array([0.001, 0.1, 1.0])
    for l in (2, 3):
        x = np.zeros(n * 4)
        ret = gpu.dshbicgstabl(A, b, l, sig, 1e-11, 500, x)
        ret_o, x_o, _ = S.shbicgstabl(As, b, l, sig, 1e-11, 500)
        assert iters_close(ret, ret_o)
        np.testing.assert_allclose(x, x_o, atol=1e-7 * np.abs(x_o).max())
    # BiCG's residual norm is erratic near the stopping level, so the index
    # at which it first dips below tol moves with rounding (dot-product
    # summation order); the solutions agree to the requested accuracy.
    x = np.zeros(n * 4)
    ret = gpu.dshbicg(A, b, sig, 1e-11, 500, x)
    ret_o, x_o, _ = S.shbicg(As, b, sig, 1e-11, 500)
    assert iters_close(ret, ret_o, rel=0.1, abs_=3)
    np.testing.assert_allclose(x, x_o, atol=1e-6 * np.abs(x_o).max())


def test_mixed_shifted_reaches_fp64_target_on_every_shift(gpu):
    """The shifted configuration at reduced size (2D convection-diffusion
    96^2, 32 shifts 1e-3..1, b ~ U[-1,1] seed 3): FP32 shift vectors plus
    per-shift polishing bring the seed and every shifted solution to an FP64
    true relative residual of 1e-8, close to the FP64 shifted solve's."""
    B = gpu
    rp, c, v, n = P.convdiff2d(96)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 3)
    sig = P.log_shifts(32)
    x = np.zeros(33 * n)
    with B.record() as st:
        ret = B.dshbicgstabl_mixed(B.CsrMatrix(rp, c, v), b, 4, sig, x)
    assert ret >= 0, ret
    nb = np.linalg.norm(b)
    res = [np.linalg.norm(b - A @ x[:n]) / nb] + [
        np.linalg.norm(b - (A @ x[(k + 1) * n:(k + 2) * n] + s * x[(k + 1) * n:(k + 2) * n])) / nb
        for k, s in enumerate(sig)]
    assert max(res) <= 1e-8, max(res)
    assert abs(st["true_res"] - max(res)) <= 1e-9
    x64 = np.zeros(33 * n)
    B.dshbicgstabl(B.CsrMatrix(rp, c, v), b, 4, sig, 1e-10, 5000, x64)
    for k in range(33):
        seg = slice(k * n, (k + 1) * n)
        assert np.linalg.norm(x[seg] - x64[seg]) <= 1e-6 * np.linalg.norm(x64[seg])
