"""Host-side checks of libbksp.so that need no GPU: every function the
public headers declare is exported, argument validation, the Matrix Market
reader and the dense helpers."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import bksp_b200 as B
from conftest import ROOT

HEADERS = ["include/bksp.h", "include/bksp_gpu.h"]


def _declared():
    names = set()
    for h in HEADERS:
        src = open(os.path.join(ROOT, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"static inline[^{]*\{[^}]*\}", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([a-z_][\w]*)\s*\(", src, re.M):
            name = m.group(1)
            if name not in ("if", "return", "sizeof", "defined"):
                names.add(name)
    return names


def test_headers_declare_the_bksp_api():
    names = _declared()
    for f in ["bksp_dcg", "dcr", "dbicg", "dbicgstab", "dbicgstabl", "dblcg",
              "dblbicgstab", "dblbicgstabl", "dshbicg", "dshbicgstabl",
              "read_matrix_market", "myqr", "dmat_create", "darray2dmat",
              "dmat_free", "dvec2mat"]:
        assert f in names, f


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(B.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_arguments_are_rejected_without_gpu_work():
    # Matrix type checks happen before any device call.
    rp = np.array([0, 1, 2], np.int32)
    A = B.CsrMatrix(rp, np.array([0, 1], np.int32), np.array([1.0, 1.0]))
    x = np.zeros(2)
    assert B.bksp_dcg(A, np.ones(2), 1e-8, 10, x) == B.INVALID_MATRIX_TYPE
    assert B.dcr(A, np.ones(2), 1e-8, 10, x) == B.INVALID_MATRIX_TYPE
    assert B.dbicgstabl(A, np.ones(2), 0, 1e-8, 10, x) == B.INVALID_PARAMETERS
    assert B.dbicgstabl(A, np.ones(2), 99, 1e-8, 10, x) == B.INVALID_PARAMETERS
    # Row pointer inconsistent with the entry arrays: the Python wrapper
    # refuses to build it; the C entry points reject a dspmat whose nnz
    # disagrees with row[n].
    with pytest.raises(ValueError):
        B.CsrMatrix(np.array([0, 1, 3], np.int32), np.array([0, 1], np.int32),
                    np.array([1.0, 1.0]))
    bad = B.CsrMatrix(rp, np.array([0, 1], np.int32), np.array([1.0, 1.0]))
    bad._nnz.value = 3
    assert B.dbicg(bad, np.ones(2), 1e-8, 10, x) == B.INVALID_PARAMETERS


def test_read_matrix_market_matches_reference_reader(tmp_path, testmats):
    # Write pde2961 back out (general) and bfwb398 (symmetric triangle) and
    # read them with the library: same CSR, entries in file order.
    for name, sym in (("pde", False), ("bfwb", True)):
        rp, c, v = (testmats[f"{name}_rowptr"], testmats[f"{name}_col"],
                    testmats[f"{name}_val"])
        n = rp.size - 1
        rows = np.repeat(np.arange(n), np.diff(rp))
        p = tmp_path / f"{name}.mtx"
        with open(p, "w") as f:
            f.write("%%MatrixMarket matrix coordinate real "
                    + ("symmetric" if sym else "general") + "\n% comment\n")
            f.write(f"{n} {n} {rp[-1]}\n")
            for i, j, a in zip(rows, c, v):
                f.write(f"{i + 1} {j + 1} {float(a)!r}\n")
        r2, c2, v2, n2, t2 = B.read_matrix_market(str(p))
        assert n2 == n and t2 == ("symmetric" if sym else "unsymmetric")
        assert np.array_equal(r2, rp) and np.array_equal(c2, c)
        assert np.array_equal(v2, v)
    with pytest.raises(OSError):
        B.read_matrix_market(str(tmp_path / "missing.mtx"))


def test_dense_helpers():
    d = B.lib.dmat_create
    d.restype = C.POINTER(B.DMat)
    d.argtypes = [C.c_int, C.c_int]
    m = d(5, 3).contents
    assert (m.row_size, m.col_size) == (5, 3)
    vals = np.ctypeslib.as_array(m.value, shape=(15,))
    assert np.all(vals == 0.0)
    x = np.arange(5, dtype=np.float64)
    B.lib.dvec2mat.argtypes = [C.POINTER(C.c_double), C.c_int, C.POINTER(B.DMat)]
    B.lib.dvec2mat(x.ctypes.data_as(C.POINTER(C.c_double)), 1, C.byref(m))
    # reference src/util.c:57-67 writes value[i * col_size + m]
    assert [vals[i * 3 + 1] for i in range(5)] == list(x)


def test_read_matrix_market_edge_cases(tmp_path):
    """CRLF line ends, blank lines, signs and exponents parse; malformed entry
    lines (bad index, extra token, wrong count) are rejected."""
    ok = ("%%MatrixMarket matrix coordinate real general\r\n% c\r\n\r\n3 3 3\r\n"
          "1 1 +2.5e0\r\n\r\n3 2 -1E-3\r\n2 3 4\r\n")
    (tmp_path / "ok.mtx").write_text(ok)
    rp, c, v, n, t = B.read_matrix_market(str(tmp_path / "ok.mtx"))
    assert n == 3 and t == "unsymmetric"
    assert list(rp) == [0, 1, 2, 3] and list(c) == [0, 2, 1]
    assert list(v) == [2.5, 4.0, -1e-3]
    pat = "%%MatrixMarket matrix coordinate pattern symmetric\n2 2 2\n1 1\n2 1\n"
    (tmp_path / "pat.mtx").write_text(pat)
    rp, c, v, n, t = B.read_matrix_market(str(tmp_path / "pat.mtx"))
    assert t == "symmetric" and list(v) == [1.0, 1.0]
    for body in ("3 3 1\n4 1 2.0\n", "3 3 1\n1 1 2.0 7\n", "3 3 2\n1 1 2.0\n",
                 "3 3 1\n1 x 2.0\n"):
        (tmp_path / "bad.mtx").write_text(
            "%%MatrixMarket matrix coordinate real general\n" + body)
        with pytest.raises(OSError):
            B.read_matrix_market(str(tmp_path / "bad.mtx"))
    # a file large enough to be parsed by several threads
    rng = np.random.default_rng(0)
    n = 60000
    rows = rng.integers(0, n, 400000)
    cols = rng.integers(0, n, 400000)
    vals = rng.standard_normal(400000)
    with open(tmp_path / "big.mtx", "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n{n} {n} {rows.size}\n")
        f.writelines(f"{i + 1} {j + 1} {float(x)!r}\n" for i, j, x in zip(rows, cols, vals))
    rp, c, v, n2, _ = B.read_matrix_market(str(tmp_path / "big.mtx"))
    order = np.argsort(rows, kind="stable")
    assert np.array_equal(c, cols[order]) and np.array_equal(v, vals[order])
    assert np.array_equal(np.diff(rp), np.bincount(rows, minlength=n))


def test_complex_api_is_declared():
    names = _declared()
    for f in ["zbicg", "zbicgstabl", "zblbicgstabl", "zshbicgstabl",
              "zread_matrix_market", "zqreco", "zmat_create", "zmat_free",
              "bksp_gpu_zcsrmv"]:
        assert f in names, f


def test_zread_matrix_market_matches_reference_reader(tmp_path):
    """Complex files: the library's reader and the reference's
    (src/read_matrix.c:176-301, through oracle/_ref) give the same CSR with
    entries in file order within each row; real files are refused."""
    from oracle import ref as R
    rng = np.random.default_rng(5)
    n, nz = 300, 2000
    rows = rng.integers(0, n, nz)
    cols = rng.integers(0, n, nz)
    vals = rng.standard_normal(nz) + 1j * rng.standard_normal(nz)
    p = tmp_path / "z.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix coordinate complex general\n% c\n")
        f.write(f"{n} {n} {nz}\n")
        for i, j, a in zip(rows, cols, vals):
            f.write(f"{i + 1} {j + 1} {float(a.real)!r} {float(a.imag)!r}\n")
    rp, c, v, n2, t = B.zread_matrix_market(str(p))
    assert n2 == n and t == "unsymmetric"
    L = R._zlib()
    L.zread_matrix_market.argtypes = [C.c_char_p]
    L.zread_matrix_market.restype = C.POINTER(R.ZSpMat)
    m = L.zread_matrix_market(os.fsencode(str(p))).contents
    rr = np.ctypeslib.as_array(m.row, shape=(n + 1,))
    cr = np.ctypeslib.as_array(m.col, shape=(nz,))
    vr = np.ctypeslib.as_array(m.value, shape=(2 * nz,))
    assert np.array_equal(rp, rr) and np.array_equal(c, cr)
    assert np.array_equal(v.real, vr[0::2]) and np.array_equal(v.imag, vr[1::2])
    (tmp_path / "real.mtx").write_text(
        "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 2.0\n")
    with pytest.raises(OSError):
        B.zread_matrix_market(str(tmp_path / "real.mtx"))


def test_complex_invalid_arguments_are_rejected_without_gpu_work():
    rp = np.array([0, 1, 2], np.int32)
    A = B.ZCsrMatrix(rp, np.array([0, 1], np.int32), np.array([1.0, 1.0j]))
    x = np.zeros(2, complex)
    b = np.ones(2, complex)
    assert B.zbicgstabl(A, b, 0, 1e-8, 10, x) == B.INVALID_PARAMETERS
    assert B.zbicgstabl(A, b, 9, 1e-8, 10, x) == B.INVALID_PARAMETERS
    assert B.zshbicgstabl(A, b, 0, [0.1], 1e-8, 10, np.zeros(4, complex)) == \
        B.INVALID_PARAMETERS
    assert B.zshbicgstabl(A, b, 2, np.zeros(129), 1e-8, 10,
                          np.zeros(2 * 130, complex)) == B.INVALID_PARAMETERS
    Bm = np.ones((2, 17), complex)
    assert B.zblbicgstabl(A, Bm, 2, 1e-8, 10, np.zeros((2, 17), complex)) == \
        B.INVALID_PARAMETERS
    bad = B.ZCsrMatrix(rp, np.array([0, 1], np.int32), np.array([1.0, 1.0j]))
    bad._nnz.value = 3
    assert B.zbicg(bad, b, 1e-8, 10, x) == B.INVALID_PARAMETERS
    assert B.lib.zqreco(2, 17, None, None) == B.INVALID_PARAMETERS


def test_zmat_helpers():
    f = B.lib.zmat_create
    f.restype = C.POINTER(B.ZMat)
    f.argtypes = [C.c_int, C.c_int]
    m = f(4, 3)
    assert (m.contents.row_size, m.contents.col_size) == (4, 3)
    vals = np.ctypeslib.as_array(m.contents.value, shape=(24,))
    assert np.all(vals == 0.0)
    B.lib.zmat_free.argtypes = [C.POINTER(B.ZMat)]
    assert B.lib.zmat_free(m) == 0


def test_mex_front_ends_link_and_check_arguments_without_gpu():
    """The reference's MATLAB front-ends, compiled unchanged against
    include/bksp.h and libbksp.so (tests/mex/Makefile), load and report
    argument errors back to the caller (MATLAB-API stand-in
    tests/mex/mexshim.c); their solves run in tests/test_gpu_mex.py."""
    build = os.path.join(ROOT, "tests", "mex", "_build")
    if not os.path.exists(os.path.join(build, "bicg.so")):
        pytest.skip("MEX front-ends not built (no reference sources here)")
    shim = C.CDLL(os.path.join(build, "libmexshim.so"), mode=C.RTLD_GLOBAL)
    shim.shim_dense.restype = C.c_void_p
    shim.shim_dense.argtypes = [C.c_size_t, C.c_size_t, C.POINTER(C.c_double),
                                C.POINTER(C.c_double)]
    shim.shim_call.restype = C.c_int
    shim.shim_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                               C.c_int, C.POINTER(C.c_void_p)]
    shim.shim_error.restype = C.c_char_p
    one = np.ones(4)
    dense = shim.shim_dense(2, 2, one.ctypes.data_as(C.POINTER(C.c_double)), None)
    vec = shim.shim_dense(2, 1, one.ctypes.data_as(C.POINTER(C.c_double)), None)
    sc = shim.shim_dense(1, 1, one.ctypes.data_as(C.POINTER(C.c_double)), None)
    for name, nargs in (("bicg", 4), ("bicgstabl", 5), ("shbicgstabl", 6),
                        ("blbicgstabl", 5)):
        L = C.CDLL(os.path.join(build, f"{name}.so"))
        fn = C.cast(L.mexFunction, C.c_void_p).value
        plhs = (C.c_void_p * 1)()
        few = (C.c_void_p * 1)(dense)
        assert shim.shim_call(fn, 1, plhs, 1, few) == 1
        assert b"BKSP:" in shim.shim_error()
        args = (C.c_void_p * nargs)(*([dense, vec] + [sc] * (nargs - 2)))
        if name != "blbicgstabl":   # the block front-end checks sizes only
            assert shim.shim_call(fn, 1, plhs, nargs, args) == 1
            assert b"sparse square matrix" in shim.shim_error(), name
