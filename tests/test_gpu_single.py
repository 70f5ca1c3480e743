"""GPU parity of the single-right-hand-side methods (through the C-ABI)
against the compiled reference's golden outputs and the CPU oracle."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import hist_close, iters_close
from bksp_b200 import problems as P
from oracle import solvers as S

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)


def _spmv(B, A, trans, x):
    B.lib.bksp_gpu_dcsrmv.argtypes = [C.c_void_p, C.c_char, _dp, _dp]
    y = np.zeros(A.n)
    x = np.ascontiguousarray(x, dtype=np.float64)
    rc = B.lib.bksp_gpu_dcsrmv(C.addressof(A.s), trans, x.ctypes.data_as(_dp),
                               y.ctypes.data_as(_dp))
    assert rc == 0
    return y


def _row_sums_sequential(rp, c, v, x):
    """y_i = ((0 + a_0 x_0) + a_1 x_1) + ... with FP64 rounding per step,
    the reference's dcsrgemm0 order (src/matvec.c:19-27)."""
    n = rp.size - 1
    y = np.zeros(n)
    L = np.diff(rp)
    prod = v * x[c]
    acc = np.zeros(n)
    for k in range(L.max()):
        m = L > k
        acc[m] = acc[m] + prod[rp[:-1][m] + k]
    return acc


def test_spmv_bit_exact_vs_reference_order(gpu, testmats):
    rp, c, v = testmats["pde_rowptr"], testmats["pde_col"], testmats["pde_val"]
    A = gpu.CsrMatrix(rp, c, v)
    x = np.random.default_rng(5).uniform(-1, 1, A.n)
    y = _spmv(gpu, A, b"n", x)
    assert np.array_equal(y, _row_sums_sequential(rp, c, v, x))
    # A^T: rows of the transpose in original row order (scatter order).
    At = sp.csr_matrix((v, c, rp), shape=(A.n, A.n)).T.tocsr()
    yt = _spmv(gpu, A, b"t", x)
    np.testing.assert_allclose(yt, At @ x, rtol=1e-13, atol=1e-13)
    # Mirrored one-triangle operator.
    Ls = gpu.CsrMatrix(testmats["bfwb_rowptr"], testmats["bfwb_col"],
                       testmats["bfwb_val"], symmetric=True)
    Lf = S.full_symmetric(sp.csr_matrix(
        (testmats["bfwb_val"], testmats["bfwb_col"], testmats["bfwb_rowptr"]),
        shape=(Ls.n, Ls.n)))
    xs = np.random.default_rng(6).uniform(-1, 1, Ls.n)
    np.testing.assert_allclose(_spmv(gpu, Ls, b"s", xs), Lf @ xs, rtol=1e-12,
                               atol=1e-20)


@pytest.mark.parametrize("variant", range(8))
def test_spmv_variants_bit_exact(gpu, testmats, variant):
    """Every SpMV kernel variant sums rows in the reference's order."""
    import torch
    rng = np.random.default_rng(variant)
    cases = [(testmats["pde_rowptr"], testmats["pde_col"], testmats["pde_val"])]
    n = 3000                                   # ragged rows, some long
    lens = rng.integers(0, 40, n)
    lens[[5, 77]] = [3000, 2049]
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    cases.append((rp.astype(np.int32), rng.integers(0, n, rp[-1]).astype(np.int32),
                  rng.uniform(-1, 1, rp[-1])))
    # Large enough that every CTA of the persistent kernels walks several
    # row blocks (more row blocks than the grid cap of 148 * 8 CTAs).
    rp3, c3, v3, n3 = P.convdiff3d(72)
    assert (n3 + 255) // 256 > 148 * 8
    cases.append((rp3, c3, v3))
    for rp, c, v in cases:
        G = gpu.GpuMatrix(gpu.CsrMatrix(rp, c, v), gpu.FP32)
        assert G.variant(variant) == variant
        x = rng.uniform(-1, 1, G.n)
        ref = _row_sums_sequential(rp, c, v, x)
        xd = torch.from_numpy(x).cuda()
        yd = torch.zeros(G.n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        G.spmv(xd.data_ptr(), yd.data_ptr(), False)
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        short = np.diff(rp) <= 2048
        assert np.array_equal(y[short], ref[short])
        np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-12)
        x32 = torch.from_numpy(x.astype(np.float32)).cuda()
        y32 = torch.zeros(G.n, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        G.spmv(x32.data_ptr(), y32.data_ptr(), True)
        torch.cuda.synchronize()
        ref32 = sp.csr_matrix((v.astype(np.float32), c, rp), shape=(G.n, G.n)) @ x.astype(np.float32)
        np.testing.assert_allclose(y32.cpu().numpy(), ref32, rtol=2e-5, atol=2e-4)
        G.close()


@pytest.mark.parametrize("nx", [48, 128])
def test_spmv_sell_bit_exact_on_permuted_operator(gpu, nx):
    """The sliced-ELL kernel on operators without a diagonal form (the 3D
    convection-diffusion stencil under a random symmetric permutation;
    128^3 is the benchmark size): FP64 bit-identical to the reference's row
    order, with and without the residual / dot epilogue; FP32 close."""
    import torch
    rp, c, v, n = P.permuted(*P.convdiff3d(nx))
    G = gpu.GpuMatrix(gpu.CsrMatrix(rp, c, v), gpu.FP32)
    assert G.diagonals() == []
    assert G.variant(8) == 8
    x = np.random.default_rng(11).uniform(-1, 1, n)
    ref = _row_sums_sequential(rp, c, v, x)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    G.spmv(xd.data_ptr(), yd.data_ptr(), False)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), ref)
    x32 = torch.from_numpy(x.astype(np.float32)).cuda()
    y32 = torch.zeros(n, dtype=torch.float32, device="cuda")
    G.spmv(x32.data_ptr(), y32.data_ptr(), True)
    torch.cuda.synchronize()
    ref32 = sp.csr_matrix((v.astype(np.float32), c, rp), shape=(n, n)) @ x.astype(np.float32)
    np.testing.assert_allclose(y32.cpu().numpy(), ref32, rtol=2e-5, atol=2e-4)
    # The residual epilogue (b - A x and dots) through a solve: the same
    # converged result as on the tile kernel.
    b = torch.from_numpy(P.uniform(n, 3)).cuda()
    rets = []
    for var in (8, 0):
        G.variant(var)
        xs = torch.zeros_like(b)
        ret, st = G.solve(gpu.BICGSTABL, b.data_ptr(), xs.data_ptr(), 1e-10, 2000, l=2)
        rets.append(ret)
        As = sp.csr_matrix((v, c, rp), shape=(n, n))
        assert S.true_residual(As, b.cpu().numpy(), xs.cpu().numpy()) < 1e-9
    assert iters_close(rets[0], rets[1], rel=0.05, abs_=1), rets
    G.close()


def test_diagonal_form_detection(gpu, testmats):
    """Operators on <= 8 diagonals with ascending rows get a diagonal form."""
    G = gpu.GpuMatrix(gpu.CsrMatrix(testmats["pde_rowptr"], testmats["pde_col"],
                                    testmats["pde_val"]))
    assert G.diagonals() == [-47, -1, 0, 1, 47]
    assert G.variant() == 7          # small operator with a diagonal form
    G.close()
    rp, c, v, n = P.convdiff3d(12)
    G = gpu.GpuMatrix(gpu.CsrMatrix(rp, c, v), gpu.FP32)
    assert G.diagonals() == [-144, -12, -1, 0, 1, 12, 144]
    G.close()
    # 165 diagonals: none.
    G = gpu.GpuMatrix(gpu.CsrMatrix(testmats["bfwb_rowptr"], testmats["bfwb_col"],
                                    testmats["bfwb_val"]))
    assert G.diagonals() == []
    G.close()
    # A row listing its columns out of order: none (the diagonal order would
    # not be the row's summation order).
    rp2, c2, v2 = rp.copy(), c.copy(), v.copy()
    k = rp2[100]
    c2[k], c2[k + 1] = c2[k + 1], c2[k]
    v2[k], v2[k + 1] = v2[k + 1], v2[k]
    G = gpu.GpuMatrix(gpu.CsrMatrix(rp2, c2, v2))
    assert G.diagonals() == []
    G.close()


def test_dia_tail_unaligned_and_missing_entries(gpu):
    """Diagonal kernel: odd n (tail rows), rows missing diagonals, an
    explicitly stored zero, and result vectors that are not 16-byte aligned
    (which fall back to the tile kernel) -- all bit-exact."""
    import torch
    rp, c, v, n = P.convdiff2d(37)          # n = 1369, odd
    rng = np.random.default_rng(11)
    v = v.copy()
    v[rng.integers(0, v.size, 50)] = 0.0    # stored zeros stay stored
    G = gpu.GpuMatrix(gpu.CsrMatrix(rp, c, v), gpu.FP32)
    assert len(G.diagonals()) == 5
    G.variant(7)
    x = rng.uniform(-1, 1, n)
    ref = _row_sums_sequential(rp, c, v, x)
    xd = torch.from_numpy(x).cuda()
    for shift in (0, 1):
        yb = torch.full((n + 1,), 7.0, dtype=torch.float64, device="cuda")
        y = yb[shift:shift + n]
        torch.cuda.synchronize()
        G.spmv(xd.data_ptr(), y.data_ptr(), False)
        torch.cuda.synchronize()
        assert np.array_equal(y.cpu().numpy(), ref)
        # Nothing written outside the n results.
        out = yb.cpu().numpy()
        assert out[n if shift == 0 else 0] == 7.0
    G.close()


@pytest.mark.parametrize("nrows,rowlen", [(1, 5000), (3, 2049), (700, 0), (1000, 1)])
def test_spmv_ragged_and_long_rows(gpu, nrows, rowlen):
    rng = np.random.default_rng(nrows)
    n = max(nrows, 64)
    lens = rng.integers(0, 12, n)
    lens[:nrows] = rowlen
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    c = rng.integers(0, n, rp[-1]).astype(np.int32)
    v = rng.uniform(-1, 1, rp[-1])
    A = gpu.CsrMatrix(rp.astype(np.int32), c, v)
    x = rng.uniform(-1, 1, n)
    y = _spmv(gpu, A, b"n", x)
    ref = sp.csr_matrix((v, c, rp), shape=(n, n)) @ x
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-12)
    short = lens <= 2048
    assert np.array_equal(y[short], _row_sums_sequential(rp, c, v, x)[short])


def _pde(gpu, tm):
    A = gpu.CsrMatrix(tm["pde_rowptr"], tm["pde_col"], tm["pde_val"])
    As = sp.csr_matrix((tm["pde_val"], tm["pde_col"], tm["pde_rowptr"]),
                       shape=(A.n, A.n))
    return A, As


def test_cg_cr_known_answers(gpu, testmats, golden):
    Ls = gpu.CsrMatrix(testmats["bfwb_rowptr"], testmats["bfwb_col"],
                       testmats["bfwb_val"], symmetric=True)
    Af = S.full_symmetric(sp.csr_matrix(
        (testmats["bfwb_val"], testmats["bfwb_col"], testmats["bfwb_rowptr"]),
        shape=(Ls.n, Ls.n)))
    b = np.zeros(Ls.n); b[0] = 1.0
    for key, fn in (("testc/cg", gpu.bksp_dcg), ("testc/cr", gpu.dcr)):
        g = golden[key]
        x = np.zeros(Ls.n)
        with gpu.record(hist_cap=1000) as st:
            ret = fn(Ls, b, 1e-14, 500, x)
        assert iters_close(ret, g["ret"]), (key, ret, g["ret"])
        assert abs(np.linalg.norm(x) - g["xnorm"]) < 1e-6 * g["xnorm"]
        assert S.true_residual(Af, b, x) < 10 * max(g["true_res"], 1e-15)
        hist_close(st["hist"], g["hist"], floor=1e-6)


@pytest.mark.parametrize("key,call", [
    ("testc/bicg", lambda B, A, b, x: B.dbicg(A, b, 1e-14, 500, x)),
    ("testc/bicgstab", lambda B, A, b, x: B.dbicgstab(A, b, 1e-14, 500, x)),
    ("testc/bicgstabl4", lambda B, A, b, x: B.dbicgstabl(A, b, 4, 1e-14, 500, x)),
])
def test_nonsymmetric_known_answers(gpu, testmats, golden, key, call):
    A, As = _pde(gpu, testmats)
    b = np.zeros(A.n); b[0] = 1.0
    x = np.zeros(A.n)
    with gpu.record(hist_cap=1000) as st:
        ret = call(gpu, A, b, x)
    g = golden[key]
    # tol 1e-14 sits at the rounding floor of this problem: the reference
    # itself moves by several iterations with its BLAS thread count.
    assert iters_close(ret, g["ret"], rel=0.08), (key, ret, g["ret"])
    assert S.true_residual(As, b, x) < 1e-12
    hist_close(st["hist"], g["hist"], floor=1e-6)


def test_seeded_configs_match_reference(gpu, golden):
    rp, c, v, n = P.poisson2d(64)
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    Af = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 0)
    for key, fn in (("cfg1/cg_poisson64", gpu.bksp_dcg), ("cfg1/cr_poisson64", gpu.dcr)):
        x = np.zeros(n)
        with gpu.record(hist_cap=20000) as st:
            ret = fn(gpu.CsrMatrix(lrp, lc, lv, symmetric=True), b, 1e-10, 10000, x)
        g = golden[key]
        assert iters_close(ret, g["ret"]), (key, ret, g["ret"])
        hist_close(st["hist"], g["hist"], floor=1e-8)
        assert S.true_residual(Af, b, x) < 1e-9
    rp, c, v, n = P.convdiff3d(24)
    Af = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = Af @ P.uniform(n, 1)
    A = gpu.CsrMatrix(rp, c, v)
    runs = [(f"cfg2/bicgstabl{l}_cd24",
             (lambda l: lambda x: gpu.dbicgstabl(A, b, l, 1e-10, 2000, x))(l))
            for l in (1, 2, 4)]
    runs += [("cfg2/bicgstab_cd24", lambda x: gpu.dbicgstab(A, b, 1e-10, 2000, x)),
             ("cfg2/bicg_cd24", lambda x: gpu.dbicg(A, b, 1e-10, 2000, x))]
    for key, run in runs:
        x = np.zeros(n)
        with gpu.record(hist_cap=5000) as st:
            ret = run(x)
        g = golden[key]
        assert iters_close(ret, g["ret"]), (key, ret, g["ret"])
        hist_close(st["hist"], g["hist"], floor=1e-8)
        assert S.true_residual(Af, b, x) < 1e-9


def test_initial_guess_and_budget(gpu):
    rp, c, v, n = P.convdiff3d(10)
    Af = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = Af @ P.uniform(n, 1)
    A = gpu.CsrMatrix(rp, c, v)
    x0 = P.uniform(n, 7)
    ret_o, x_o, _ = S.bicgstabl(Af, b, 2, 1e-10, 500, x0=x0)
    x = x0.copy()
    ret = gpu.dbicgstabl(A, b, 2, 1e-10, 500, x)
    assert iters_close(ret, ret_o)
    np.testing.assert_allclose(x, x_o, atol=1e-8)
    # Budget exhausted -> NOT_CONVERGED; no iteration -> first index.
    x = np.zeros(n)
    assert gpu.dbicgstabl(A, b, 2, 1e-10, 2, x) == gpu.NOT_CONVERGED
    x = np.zeros(n)
    assert gpu.dbicgstab(A, b, 1e-10, 0, x) == 0
    assert np.all(x == 0)
    Ls = gpu.CsrMatrix(*P.lower_triangle(*P.poisson2d(8))[:3], symmetric=True)
    assert gpu.dcr(Ls, np.ones(64), 1e-10, 1, np.zeros(64)) == 1


def test_nan_breakdown_is_divergence(gpu):
    # A zero matrix gives alpha = 0/0 in the first iteration.
    n = 64
    rp = np.arange(n + 1, dtype=np.int32)
    A = gpu.CsrMatrix(rp, np.arange(n, dtype=np.int32), np.zeros(n))
    x = np.zeros(n)
    assert gpu.dbicgstab(A, np.ones(n), 1e-10, 50, x) == gpu.DIVERGENCE


def test_structure_scan_rejects_bad_columns(gpu, testmats):
    """Column indices outside [0, n) are found by the GPU structure scan and
    rejected with INVALID_PARAMETERS, by the handle API and by bksp.h calls;
    a zero diagonal entry makes a Jacobi-preconditioned solve unavailable."""
    import torch
    rp, c, v = testmats["pde_rowptr"], testmats["pde_col"], testmats["pde_val"]
    n = rp.size - 1
    for bad in (-1, n, n + 1000):
        c2 = c.copy()
        c2[rp[n // 2] + 1] = bad
        A = gpu.CsrMatrix(rp, c2, v)
        with pytest.raises(RuntimeError):
            gpu.GpuMatrix(A)
        x = np.zeros(n)
        assert gpu.dbicgstab(A, np.ones(n), 1e-10, 100, x) == -3
    rows = np.repeat(np.arange(n), np.diff(rp))
    v2 = v.copy()
    v2[np.flatnonzero(c == rows)[7]] = 0.0
    G = gpu.GpuMatrix(gpu.CsrMatrix(rp, c, v2), gpu.FP32)
    bd = torch.ones(n, dtype=torch.float64, device="cuda")
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ret, _ = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), l=2, target=1e-8, precond=1)
    assert ret == -3
    G.close()


def test_spmv_bit_exact_at_benchmark_size(gpu):
    """The benchmark operator itself (3D convection-diffusion 128^3, 2.1 M
    rows): every SpMV variant the autotuner may pick reproduces the
    reference's row order bit for bit in FP64."""
    import torch
    rp, c, v, n = P.convdiff3d(128)
    x = np.random.default_rng(9).uniform(-1, 1, n)
    ref = _row_sums_sequential(rp, c, v, x)
    G = gpu.GpuMatrix(gpu.CsrMatrix(rp, c, v))
    assert len(G.diagonals()) == 7
    xd = torch.from_numpy(x).cuda()
    for variant in (7, 0, 6):
        G.variant(variant)
        yd = torch.zeros(n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        G.spmv(xd.data_ptr(), yd.data_ptr(), False)
        torch.cuda.synchronize()
        assert np.array_equal(yd.cpu().numpy(), ref), variant
    G.close()
