"""The reference's MATLAB front-ends (matlab/*.c: bicg, bicgstabl,
blbicgstabl, shbicgstabl), compiled unchanged against include/bksp.h and
libbksp.so by tests/mex/Makefile, called through the MATLAB-API stand-in
(tests/mex/mexshim.c) with MATLAB-layout sparse matrices (compressed
columns, separate real and imaginary parts): each returns what the
library's own C-ABI call returns on the same system, real and complex."""
import ctypes as C
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT
from bksp_b200 import problems as P
from oracle import solvers as S
from oracle import zsolvers as Z

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "tests", "mex", "_build")
_dp = C.POINTER(C.c_double)
_sz = C.POINTER(C.c_size_t)


@pytest.fixture(scope="module")
def mex(gpu):
    if not os.path.exists(os.path.join(BUILD, "bicg.so")):
        pytest.fail("MEX front-ends not built: make -C tests/mex")
    shim = C.CDLL(os.path.join(BUILD, "libmexshim.so"), mode=C.RTLD_GLOBAL)
    shim.shim_dense.restype = C.c_void_p
    shim.shim_dense.argtypes = [C.c_size_t, C.c_size_t, _dp, _dp]
    shim.shim_sparse.restype = C.c_void_p
    shim.shim_sparse.argtypes = [C.c_size_t, C.c_size_t, _sz, _sz, _dp, _dp]
    shim.shim_call.restype = C.c_int
    shim.shim_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                               C.c_int, C.POINTER(C.c_void_p)]
    shim.shim_error.restype = C.c_char_p
    for f in ("mxGetPr", "mxGetPi"):
        getattr(shim, f).restype = _dp
        getattr(shim, f).argtypes = [C.c_void_p]
    for f in ("mxGetM", "mxGetN"):
        getattr(shim, f).restype = C.c_size_t
        getattr(shim, f).argtypes = [C.c_void_p]
    fns = {}
    for name in ("bicg", "bicgstabl", "blbicgstabl", "shbicgstabl"):
        L = C.CDLL(os.path.join(BUILD, f"{name}.so"))
        fns[name] = C.cast(L.mexFunction, C.c_void_p).value
    return shim, fns


def _d(a):
    a = np.asfortranarray(a)
    return a.ctypes.data_as(_dp), a


def mx_dense(shim, a):
    a = np.asarray(a)
    if a.ndim == 1:
        a = a[:, None]
    re = np.asfortranarray(a.real, dtype=np.float64)
    im = np.asfortranarray(a.imag, dtype=np.float64) if np.iscomplexobj(a) else None
    return shim.shim_dense(a.shape[0], a.shape[1], re.ctypes.data_as(_dp),
                           im.ctypes.data_as(_dp) if im is not None else None)


def mx_sparse(shim, A):
    A = sp.csc_matrix(A)
    A.sort_indices()
    jc = A.indptr.astype(np.uint64)
    ir = A.indices.astype(np.uint64)
    re = np.ascontiguousarray(A.data.real, dtype=np.float64)
    im = np.ascontiguousarray(A.data.imag, dtype=np.float64) if np.iscomplexobj(A.data) else None
    return shim.shim_sparse(A.shape[0], A.shape[1], jc.ctypes.data_as(_sz),
                            ir.ctypes.data_as(_sz), re.ctypes.data_as(_dp),
                            im.ctypes.data_as(_dp) if im is not None else None)


def call(mex, name, *args):
    shim, fns = mex
    prhs = (C.c_void_p * len(args))(*args)
    plhs = (C.c_void_p * 1)()
    rc = shim.shim_call(fns[name], 1, plhs, len(args), prhs)
    assert rc == 0, shim.shim_error()
    out = plhs[0]
    m, n = shim.mxGetM(out), shim.mxGetN(out)
    re = np.ctypeslib.as_array(shim.mxGetPr(out), shape=(m * n,)).copy()
    pi = shim.mxGetPi(out)
    if pi:
        re = re + 1j * np.ctypeslib.as_array(pi, shape=(m * n,))
    return re.reshape((m, n), order="F")


def scalar(mex, v):
    return mx_dense(mex[0], np.array([[float(v)]]))


def test_mex_bicg_real_and_complex(gpu, mex, capfd):
    rp, c, v, n = P.convdiff2d(24)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 3)
    x = call(mex, "bicg", mx_sparse(mex[0], A), mx_dense(mex[0], b),
             scalar(mex, 1e-10), scalar(mex, 500))[:, 0]
    xr = np.zeros(n)
    ret = gpu.dbicg(gpu.CsrMatrix(rp, c, v), b, 1e-10, 500, xr)
    assert np.array_equal(x, xr) and ret >= 0
    assert f"converged at iteration {ret}" in capfd.readouterr().out
    zr, zc, zv, zn = P.complex_convdiff2d(24)
    Az = sp.csr_matrix((zv, zc, zr), shape=(zn, zn))
    bz = P.complex_uniform(zn, 3)
    xz = call(mex, "bicg", mx_sparse(mex[0], Az), mx_dense(mex[0], bz),
              scalar(mex, 1e-10), scalar(mex, 500))[:, 0]
    xzr = np.zeros(zn, complex)
    retz = gpu.zbicg(gpu.ZCsrMatrix(zr, zc, zv), bz, 1e-10, 500, xzr)
    assert retz >= 0 and np.array_equal(xz, xzr)
    assert Z.true_residual(Az, bz, xz) < 1e-9


@pytest.mark.parametrize("cplx", [False, True])
def test_mex_bicgstabl(gpu, mex, cplx):
    gen = P.complex_convdiff2d if cplx else P.convdiff2d
    rp, c, v, n = gen(24)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.complex_uniform(n, 3) if cplx else P.uniform(n, 3)
    x = call(mex, "bicgstabl", mx_sparse(mex[0], A), mx_dense(mex[0], b),
             scalar(mex, 4), scalar(mex, 1e-10), scalar(mex, 500))[:, 0]
    if cplx:
        xr = np.zeros(n, complex)
        ret = gpu.zbicgstabl(gpu.ZCsrMatrix(rp, c, v), b, 4, 1e-10, 500, xr)
    else:
        xr = np.zeros(n)
        ret = gpu.dbicgstabl(gpu.CsrMatrix(rp, c, v), b, 4, 1e-10, 500, xr)
    assert ret >= 0 and np.array_equal(x, xr)


@pytest.mark.parametrize("cplx", [False, True])
def test_mex_shbicgstabl(gpu, mex, cplx):
    gen = P.complex_convdiff2d if cplx else P.convdiff2d
    rp, c, v, n = gen(24)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.complex_uniform(n, 3) if cplx else P.uniform(n, 3)
    sig = P.complex_shifts(4) if cplx else P.log_shifts(4)
    X = call(mex, "shbicgstabl", mx_sparse(mex[0], A), mx_dense(mex[0], b),
             scalar(mex, 2), mx_dense(mex[0], sig), scalar(mex, 1e-10),
             scalar(mex, 500))
    assert X.shape == (n, 5)
    if cplx:
        xr = np.zeros(n * 5, complex)
        ret = gpu.zshbicgstabl(gpu.ZCsrMatrix(rp, c, v), b, 2, sig, 1e-10, 500, xr)
    else:
        xr = np.zeros(n * 5)
        ret = gpu.dshbicgstabl(gpu.CsrMatrix(rp, c, v), b, 2, sig, 1e-10, 500, xr)
    assert ret >= 0 and np.array_equal(X.reshape(-1, order="F"), xr)
    tr = (Z.true_residual if cplx else S.true_residual)
    assert max(tr(A, b, X[:, k + 1], s) for k, s in enumerate(sig)) < 1e-9


@pytest.mark.parametrize("cplx", [False, True])
def test_mex_blbicgstabl(gpu, mex, cplx, capfd):
    gen = P.complex_convdiff2d if cplx else P.convdiff2d
    rp, c, v, n = gen(24)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    rng = np.random.default_rng(7)
    B = rng.uniform(-1, 1, (n, 4))
    if cplx:
        B = B + 1j * rng.uniform(-1, 1, (n, 4))
    X = call(mex, "blbicgstabl", mx_sparse(mex[0], A), mx_dense(mex[0], B),
             scalar(mex, 2), scalar(mex, 1e-10), scalar(mex, 500))
    Xr = np.zeros((n, 4), complex if cplx else float)
    if cplx:
        ret = gpu.zblbicgstabl(gpu.ZCsrMatrix(rp, c, v), B, 2, 1e-10, 500, Xr)
    else:
        ret = gpu.dblbicgstabl(gpu.CsrMatrix(rp, c, v), B, 2, 1e-10, 500, Xr)
    assert ret >= 0 and np.array_equal(X, Xr)
    assert np.linalg.norm(B - A @ X) / np.linalg.norm(B) < 1e-9
    assert "Block BiCGSTAB(2) has converged at:" in capfd.readouterr().out


def test_mex_argument_errors_return_to_matlab(gpu, mex):
    shim = mex[0]
    rp, c, v, n = P.convdiff2d(8)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    prhs = (C.c_void_p * 3)(mx_sparse(shim, A), mx_dense(shim, np.ones(n)),
                            scalar(mex, 1e-8))
    plhs = (C.c_void_p * 1)()
    assert shim.shim_call(mex[1]["bicg"], 1, plhs, 3, prhs) == 1
    assert b"Four inputs required" in shim.shim_error()
