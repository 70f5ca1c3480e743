"""The CPU oracle (NumPy restatement) against the golden outputs of the
compiled reference: iteration counts, residual histories, true residuals."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import hist_close, iters_close
from bksp_b200 import problems as P
from oracle import solvers as S


def _pde(tm):
    n = tm["pde_rowptr"].size - 1
    return sp.csr_matrix((tm["pde_val"], tm["pde_col"], tm["pde_rowptr"]), shape=(n, n))


def _bfwb(tm):
    n = tm["bfwb_rowptr"].size - 1
    L = sp.csr_matrix((tm["bfwb_val"], tm["bfwb_col"], tm["bfwb_rowptr"]), shape=(n, n))
    return S.full_symmetric(L)


def _hist_close(h, ref, k=20, rtol=1e-6, floor=1e-6):
    hist_close(h, ref, k=k, rtol=rtol, floor=floor)


def test_oracle_cg_cr_on_bfwb398(testmats, golden):
    A = _bfwb(testmats)
    n = A.shape[0]
    b = np.zeros(n); b[0] = 1.0
    for name, fn in (("testc/cg", S.cg), ("testc/cr", S.cr)):
        ret, x, h = fn(A, b, 1e-14, 500)
        g = golden[name]
        assert ret == g["ret"]
        assert abs(np.linalg.norm(x) - g["xnorm"]) < 1e-6 * g["xnorm"]
        _hist_close(h, g["hist"])


def test_oracle_blcg_on_bfwb398(testmats, golden):
    A = _bfwb(testmats)
    n = A.shape[0]
    B = np.zeros((n, 16)); B[np.arange(16), np.arange(16)] = 1.0
    ret, X, h = S.blcg(A, B, 1e-14, 500)
    g = golden["testc/blcg"]
    assert iters_close(ret, g["ret"])
    _hist_close(h, g["hist"], k=10, rtol=1e-5)


@pytest.mark.parametrize("key,fn,args,rel", [
    ("testc/bicg", S.bicg, (), 0.05),
    ("testc/bicgstab", S.bicgstab, (), 0.06),
    ("testc/bicgstabl4", lambda A, b, t, m: S.bicgstabl(A, b, 4, t, m), (), 0.05),
])
def test_oracle_single_on_pde2961(testmats, golden, key, fn, args, rel):
    A = _pde(testmats)
    n = A.shape[0]
    b = np.zeros(n); b[0] = 1.0
    ret, x, h = fn(A, b, 1e-14, 500)
    g = golden[key]
    assert iters_close(ret, g["ret"], rel=rel)
    _hist_close(h, g["hist"])


def test_oracle_block_on_pde2961(testmats, golden):
    A = _pde(testmats)
    B = testmats["pde_B"]
    ret, X, h = S.blbicgstab(A, B, 1e-14, 500)
    assert iters_close(ret, golden["testc/blbicgstab"]["ret"], rel=0.1)
    ret, X, h = S.blbicgstabl(A, B, 6, 1e-14, 500)
    assert iters_close(ret, golden["testc/blbicgstabl6"]["ret"], rel=0.1)


def test_oracle_shifted_on_pde2961(testmats, golden):
    A = _pde(testmats)
    n = A.shape[0]
    b = np.zeros(n); b[0] = 1.0
    sig = np.array([0.0, 0.2, 0.4, 0.8])
    ret, x, h = S.shbicg(A, b, sig, 1e-14, 500)
    g = golden["testc/shbicg"]
    assert ret == g["ret"]
    for k, s in enumerate(sig):
        assert S.true_residual(A, b, x[(k + 1) * n:(k + 2) * n], s) < 1e-13
    ret, x, h = S.shbicgstabl(A, b, 1, sig, 1e-14, 200)
    assert iters_close(ret, golden["testc/shbicgstabl1"]["ret"])


def test_oracle_seeded_configs(golden):
    rp, c, v, n = P.poisson2d(64)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 0)
    ret, x, h = S.cg(A, b, 1e-10, 10000)
    g = golden["cfg1/cg_poisson64"]
    assert iters_close(ret, g["ret"])
    _hist_close(h, g["hist"])
    rp, c, v, n = P.convdiff3d(24)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = A @ P.uniform(n, 1)
    for l in (1, 2, 4):
        ret, x, h = S.bicgstabl(A, b, l, 1e-10, 2000)
        g = golden[f"cfg2/bicgstabl{l}_cd24"]
        assert iters_close(ret, g["ret"]), (l, ret, g["ret"])
        _hist_close(h, g["hist"])
    rp, c, v, n = P.convdiff2d(48)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 3)
    sig = P.log_shifts(32)
    ret, x, h = S.shbicgstabl(A, b, 4, sig, 1e-10, 2000)
    g = golden["cfg4/shbicgstabl4_cd48"]
    assert iters_close(ret, g["ret"])
    worst = max(S.true_residual(A, b, x[(k + 1) * n:(k + 2) * n], s) for k, s in enumerate(sig))
    assert worst < 10 * max(g["true_res_shifts"])


def test_oracle_blocks_seeded(golden):
    rp, c, v, n = P.poisson3d(12)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    B = np.random.default_rng(2).standard_normal((n, 16))
    ret, X, h = S.blcg(A, B, 1e-10, 2000)
    assert iters_close(ret, golden["cfg3/blcg_p12"]["ret"])
    ret, X, h = S.blbicgstabl(A, B, 2, 1e-10, 2000)
    assert iters_close(ret, golden["cfg3/blbicgstabl2_p12"]["ret"])
    ret, X, h = S.blbicgstab(A, B, 1e-10, 2000)
    assert iters_close(ret, golden["cfg3/blbicgstab_p12"]["ret"])


def test_horner_and_comb():
    from math import comb
    for l in (1, 2, 4):
        om = np.linspace(0.3, 1.1, l)
        h = S.horner(om, l, 0.25)
        assert h.shape == (l + 1,)
    assert S.comb(5, 2) == comb(5, 2) and S.comb(2, 5) == 0
