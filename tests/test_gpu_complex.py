"""GPU parity of the complex methods (zbicg, zbicgstabl, zshbicgstabl,
zblbicgstabl, zqreco) and the complex SpMV against the compiled reference
(oracle/_ref, golden fixtures in tests/golden/reference_z.json) and the
complex oracle (oracle/zsolvers.py), through the C-ABI."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, hist_close, iters_close
from bksp_b200 import problems as P
from oracle import ref as R
from oracle import zsolvers as Z

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(GOLDEN, "reference_z.json")))
PROBLEMS = {"cd2d24": (P.complex_convdiff2d, 24),
            "cd3d10": (P.complex_convdiff3d, 10)}


def problem(gpu, tag):
    gen, nx = PROBLEMS[tag]
    rp, c, v, n = gen(nx)
    return gpu.ZCsrMatrix(rp, c, v), sp.csr_matrix((v, c, rp), shape=(n, n)), n


def random_complex_csr(n, per_row, seed, long_row=True):
    """Unsorted columns, empty rows, one long row (> the 2048-entry tile)
    when long_row (the tile kernel then serves it: its sliced-ELL copy would
    be mostly padding)."""
    g = np.random.default_rng(seed)
    counts = g.integers(0, per_row + 1, n)
    counts[n // 3] = 0
    if long_row:
        counts[n // 2] = 3000
    rp = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(counts, out=rp[1:])
    col = g.integers(0, n, int(rp[-1])).astype(np.int32)
    val = g.standard_normal(int(rp[-1])) + 1j * g.standard_normal(int(rp[-1]))
    return rp, col, val


@pytest.mark.parametrize("trans", ["n", "t"])
@pytest.mark.parametrize("long_row", [True, False])
def test_zspmv_bit_identical_to_reference(gpu, trans, long_row):
    """Tile kernel (long_row: a 3000-entry row) and sliced-ELL kernel."""
    n = 5000
    rp, col, val = random_complex_csr(n, 12, 4, long_row)
    x = P.complex_uniform(n, 9)
    A = gpu.ZCsrMatrix(rp, col, val)
    y = gpu.zcsrmv(A, x, trans)
    yr = R.zspmv(R.ZMatrix(rp, col, val, n), x, trans == "t")
    mask = np.ones(n, bool)
    if trans == "n" and long_row:
        mask[n // 2] = False      # strided CTA sum for a row over the tile
        assert abs(y[n // 2] - yr[n // 2]) <= 1e-12 * np.abs(yr).max()
    assert np.array_equal(y[mask].view(np.float64), yr[mask].view(np.float64))


@pytest.mark.parametrize("tag", sorted(PROBLEMS))
def test_zbicg_matches_reference(gpu, tag):
    A, As, n = problem(gpu, tag)
    b = P.complex_uniform(n, 3)
    x = np.zeros(n, complex)
    with gpu.record(hist_cap=2000) as st:
        ret = gpu.zbicg(A, b, 1e-10, 1000, x)
    g = GOLD[f"zbicg/{tag}"]
    assert iters_close(ret, g["ret"], rel=0.05, abs_=2), (ret, g["ret"])
    hist_close(st["hist"], g["hist"], k=30, rtol=1e-6)
    assert Z.true_residual(As, b, x) <= 10 * max(g["true_res"], 1e-12)


@pytest.mark.parametrize("tag", sorted(PROBLEMS))
@pytest.mark.parametrize("l", [1, 2, 4, 8])
def test_zbicgstabl_matches_oracle(gpu, tag, l):
    A, As, n = problem(gpu, tag)
    b = P.complex_uniform(n, 3)
    x = np.zeros(n, complex)
    with gpu.record(hist_cap=2000) as st:
        ret = gpu.zbicgstabl(A, b, l, 1e-10, 1000, x)
    r2, x2, h2 = Z.zbicgstabl(As, b, l, 1e-10, 1000)
    assert iters_close(ret, r2, rel=0.1, abs_=1), (ret, r2)
    hist_close(st["hist"], h2, k=8, rtol=1e-6)
    if l in (1, 2, 4):   # the reference's shifted seed is the same recurrence
        hist_close(st["hist"], GOLD[f"zshbicgstabl{l}/{tag}"]["hist"], k=6,
                   rtol=1e-6)
    assert ret >= 0 and Z.true_residual(As, b, x) < 1e-9


@pytest.mark.parametrize("tag", sorted(PROBLEMS))
@pytest.mark.parametrize("l", [1, 2, 4])
def test_zshbicgstabl_matches_reference(gpu, tag, l):
    A, As, n = problem(gpu, tag)
    b = P.complex_uniform(n, 3)
    sig = P.complex_shifts(4)
    x = np.zeros(n * 5, complex)
    with gpu.record(hist_cap=2000) as st:
        ret = gpu.zshbicgstabl(A, b, l, sig, 1e-10, 1000, x)
    g = GOLD[f"zshbicgstabl{l}/{tag}"]
    assert iters_close(ret, g["ret"], rel=0.05, abs_=1), (ret, g["ret"])
    hist_close(st["hist"], g["hist"], k=8, rtol=1e-6)
    assert Z.true_residual(As, b, x[:n]) <= 10 * max(g["true_res_seed"], 1e-12)
    for k, s in enumerate(sig):
        tr = Z.true_residual(As, b, x[(k + 1) * n:(k + 2) * n], s)
        assert tr <= 10 * max(g["true_res_shifts"][k], 1e-12), (k, tr)


def test_zshbicgstabl_many_shifts(gpu):
    """128 shifts (the limit): every shifted solution to the seed's level."""
    A, As, n = problem(gpu, "cd2d24")
    b = P.complex_uniform(n, 3)
    sig = P.complex_shifts(128, -4.0, 0.3)
    x = np.zeros(n * 129, complex)
    ret = gpu.zshbicgstabl(A, b, 2, sig, 1e-10, 1000, x)
    assert ret >= 0
    r2, x2, _ = Z.zshbicgstabl(As, b, 2, sig[:8], 1e-10, 1000)
    assert iters_close(ret, r2, rel=0.05, abs_=1)
    worst = max(Z.true_residual(As, b, x[(k + 1) * n:(k + 2) * n], s)
                for k, s in enumerate(sig))
    assert worst < 1e-8


@pytest.mark.parametrize("tag", sorted(PROBLEMS))
@pytest.mark.parametrize("l", [1, 2, 4])
def test_zblbicgstabl_matches_reference(gpu, tag, l, capfd):
    A, As, n = problem(gpu, tag)
    rng = np.random.default_rng(7)
    B = rng.uniform(-1, 1, (n, 4)) + 1j * rng.uniform(-1, 1, (n, 4))
    X = np.zeros((n, 4), complex)
    with gpu.record(hist_cap=2000) as st:
        ret = gpu.zblbicgstabl(A, B, l, 1e-10, 1000, X)
    g = GOLD[f"zblbicgstabl{l}/{tag}"]
    assert abs(ret - g["ret"]) <= max(2, 0.15 * g["ret"]), (ret, g["ret"])
    hist_close(st["hist"], g["hist"], k=2 if l == 4 else 4, rtol=1e-6)
    # The test stops on the whole block (||xi||_F / ||B||_F < tol), so a
    # column's residual is bounded by the tolerance scaled to its share of
    # ||B||_F, or sits near the reference's where that iterated further.
    for j in range(4):
        cn = np.linalg.norm(B[:, j])
        tr = np.linalg.norm(B[:, j] - As @ X[:, j]) / cn
        bound = max(10 * g["true_res_cols"][j], 10 * 1e-10 * np.linalg.norm(B) / cn)
        assert tr <= bound, (j, tr, bound)
    out = capfd.readouterr().out
    assert f"Block BiCGSTAB({l}) has converged at:" in out


def test_zblbicgstabl_block_width_16(gpu):
    A, As, n = problem(gpu, "cd3d10")
    rng = np.random.default_rng(8)
    B = rng.standard_normal((n, 16)) + 1j * rng.standard_normal((n, 16))
    X = np.zeros((n, 16), complex)
    ret = gpu.zblbicgstabl(A, B, 2, 1e-10, 1000, X)
    r2, X2, _ = Z.zblbicgstabl(As, B, 2, 1e-10, 1000)
    assert abs(ret - r2) <= max(2, 0.15 * r2), (ret, r2)
    res = np.linalg.norm(B - As @ X) / np.linalg.norm(B)
    assert ret >= 0 and res < 1e-9


def test_zqreco(gpu):
    rng = np.random.default_rng(3)
    V = rng.standard_normal((3000, 6)) + 1j * rng.standard_normal((3000, 6))
    Q, Rm, info = gpu.zqreco(V)
    assert info == 0
    assert np.allclose(Q.conj().T @ Q, np.eye(6), atol=1e-12)
    assert np.allclose(Q @ Rm, V, atol=1e-12 * np.abs(V).max())
    assert np.allclose(np.tril(Rm, -1), 0)
    d = np.diag(Rm)
    assert np.all(d.real > 0) and np.allclose(d.imag, 0)
    # LAPACK's R differs by the sign of each row (its diagonal is real too).
    Qr, Rr = Z.zqreco(V)
    sgn = np.sign(np.diag(Rr).real)
    assert np.allclose(Rm, sgn[:, None] * Rr, atol=1e-10 * np.abs(Rr).max())
