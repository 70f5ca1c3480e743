"""ctypes binding of the reference implementation built by ``oracle/Makefile``.

TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline; never product).

The reference's C API (include/bksp.h:12-27 structs, :60-103 entry points)
is bound verbatim.  ``call()`` wraps one solver call: it builds the
``dspmat``/``dmat`` structs from NumPy arrays, records the ``cblas_dnrm2``
values the solver produces (see nrm2_log.c) and returns
``(ret, x, norms)``.
"""
import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libbksp_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class DSpMat(C.Structure):
    """Mirror of ``dspmat`` (include/bksp.h:12-21): pointer-to-int sizes."""
    _fields_ = [("row", _ip), ("col", _ip), ("nnz", _ip),
                ("row_size", _ip), ("col_size", _ip), ("value", _dp),
                ("format", C.c_char_p), ("type", C.c_char_p)]


class DMat(C.Structure):
    """Mirror of ``dmat`` (include/bksp.h:23-27), column-major values."""
    _fields_ = [("row_size", C.c_int), ("col_size", C.c_int), ("value", _dp)]


_lib = None
_lock = threading.Lock()


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference oracle not built: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        sp, mp = C.POINTER(DSpMat), C.POINTER(DMat)
        d, i = C.c_double, C.c_int
        sig = {
            "bksp_dcg": [sp, _dp, d, i, _dp],
            "dcr": [sp, _dp, d, i, _dp],
            "dbicg": [sp, _dp, d, i, _dp],
            "dbicgstab": [sp, _dp, d, i, _dp],
            "dbicgstabl": [sp, _dp, i, d, i, _dp],
            "dblcg": [sp, mp, d, i, mp],
            "dblbicgstab": [sp, mp, d, i, mp],
            "dblbicgstabl": [sp, mp, i, d, i, mp],
            "dshbicg": [sp, _dp, _dp, i, d, i, _dp],
            "dshbicgstabl": [sp, _dp, i, _dp, i, d, i, _dp],
            "dcsrgemm0": [C.c_char, i, i, _dp, _ip, _ip, i, _dp, _dp],
            "dcsrsymm0": [C.c_char, i, i, _dp, _ip, _ip, i, _dp, _dp],
            "myqr": [i, i, _dp, _dp],
            "dhorner": [_dp, i, d, _dp],
            "comb": [i, i],
        }
        for name, argt in sig.items():
            f = getattr(L, name)
            f.argtypes = argt
            f.restype = C.c_int
        L.read_matrix_market.argtypes = [C.c_char_p]
        L.read_matrix_market.restype = sp
        L.oracle_nrm2_log_begin.argtypes = [_dp, C.c_int]
        L.oracle_nrm2_log_end.restype = C.c_int
        _lib = L
    return _lib


class Matrix:
    """Keeps the NumPy buffers of a ``dspmat`` alive while C uses them."""

    def __init__(self, rowptr, col, val, n, symmetric=False):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self._nnz = C.c_int(int(self.col.size))
        self._n = C.c_int(int(n))
        self._m = C.c_int(int(n))
        self.s = DSpMat(self.rowptr.ctypes.data_as(_ip),
                        self.col.ctypes.data_as(_ip), C.pointer(self._nnz),
                        C.pointer(self._n), C.pointer(self._m),
                        self.val.ctypes.data_as(_dp), b"csr",
                        b"symmetric" if symmetric else b"unsymmetric")

    @property
    def ptr(self):
        return C.byref(self.s)


def read_matrix_market(path):
    """Reference Matrix-Market reader (src/read_matrix.c:38-120) -> arrays."""
    m = lib().read_matrix_market(os.fsencode(path)).contents
    n = m.row_size[0]
    nnz = m.nnz[0]
    rowptr = np.ctypeslib.as_array(m.row, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(m.col, shape=(nnz,)).copy()
    val = np.ctypeslib.as_array(m.value, shape=(nnz,)).copy()
    return rowptr, col, val, n, m.type.decode()


def _vec(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def call(name, A, *args, log_cap=1 << 20):
    """Run reference solver ``name`` on Matrix ``A``.

    ``args`` follow the C signature after the matrix; NumPy 1-D arrays become
    ``double*`` (copied, so the caller's arrays are untouched) and 2-D arrays
    become column-major ``dmat``.  Returns ``(ret, outputs, norms)`` where
    ``outputs`` are the (possibly modified) array arguments in order and
    ``norms`` every ``cblas_dnrm2`` value the call produced.
    """
    L = lib()
    cargs, outs, keep = [], [], []
    for a in args:
        if isinstance(a, np.ndarray) and a.ndim == 2:
            buf = np.asfortranarray(a, dtype=np.float64).copy(order="F")
            dm = DMat(buf.shape[0], buf.shape[1], buf.ctypes.data_as(_dp))
            keep.append((buf, dm))
            outs.append(buf)
            cargs.append(C.byref(dm))
        elif isinstance(a, np.ndarray):
            buf = _vec(a).copy()
            keep.append(buf)
            outs.append(buf)
            cargs.append(buf.ctypes.data_as(_dp))
        else:
            cargs.append(a)
    log = np.zeros(log_cap)
    with _lock:
        L.oracle_nrm2_log_begin(log.ctypes.data_as(_dp), log_cap)
        ret = getattr(L, name)(A.ptr, *cargs)
        cnt = L.oracle_nrm2_log_end()
    return ret, outs, log[:min(cnt, log_cap)].copy()


def spmv(A, x, trans=False):
    """Reference sparse kernel ``dcsrgemm0`` (src/matvec.c:11-53), y = A x."""
    x = _vec(x)
    y = np.zeros(A._n.value)
    lib().dcsrgemm0(b"t" if trans else b"n", A._n.value, 1,
                    A.val.ctypes.data_as(_dp), A.rowptr.ctypes.data_as(_ip),
                    A.col.ctypes.data_as(_ip), A._nnz.value,
                    x.ctypes.data_as(_dp), y.ctypes.data_as(_dp))
    return y


def symv(A, x):
    """Reference ``dcsrsymm0`` (src/matvec.c:100-127) on a one-triangle CSR."""
    x = _vec(x)
    y = np.zeros(A._n.value)
    lib().dcsrsymm0(b"l", A._n.value, 1, A.val.ctypes.data_as(_dp),
                    A.rowptr.ctypes.data_as(_ip), A.col.ctypes.data_as(_ip),
                    A._nnz.value, x.ctypes.data_as(_dp),
                    y.ctypes.data_as(_dp))
    return y


def dhorner(gamma, l, sigma):
    out = np.zeros(l + 1)
    g = _vec(gamma)
    lib().dhorner(g.ctypes.data_as(_dp), l, sigma, out.ctypes.data_as(_dp))
    return out


# ------------------------------------------------------------ complex API

class ZSpMat(C.Structure):
    """Mirror of ``zspmat`` (include/bksp.h:115-124): complex values as
    interleaved (re, im) doubles."""
    _fields_ = [("row", _ip), ("col", _ip), ("nnz", _ip),
                ("row_size", _ip), ("col_size", _ip), ("value", _dp),
                ("format", C.c_char_p), ("type", C.c_char_p)]


class ZMat(C.Structure):
    """Mirror of ``zmat`` (include/bksp.h:126-130), column-major."""
    _fields_ = [("row_size", C.c_int), ("col_size", C.c_int), ("value", _dp)]


class ZMatrix:
    """Keeps the NumPy buffers of a ``zspmat`` alive while C uses them."""

    def __init__(self, rowptr, col, val, n):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.complex128)
        self._nnz = C.c_int(int(self.col.size))
        self._n = C.c_int(int(n))
        self._m = C.c_int(int(n))
        self.s = ZSpMat(self.rowptr.ctypes.data_as(_ip),
                        self.col.ctypes.data_as(_ip), C.pointer(self._nnz),
                        C.pointer(self._n), C.pointer(self._m),
                        self.val.ctypes.data_as(_dp), b"csr", b"unsymmetric")

    @property
    def ptr(self):
        return C.byref(self.s)


_zsig_done = False


def _zlib():
    global _zsig_done
    L = lib()
    if not _zsig_done:
        zp, zm = C.POINTER(ZSpMat), C.POINTER(ZMat)
        d, i = C.c_double, C.c_int
        sig = {
            "zbicg": [zp, _dp, d, i, _dp],
            "zbicgstabl": [zp, _dp, i, d, i, _dp],
            "zblbicgstabl": [zp, zm, i, d, i, zm],
            "zshbicgstabl": [zp, _dp, i, _dp, i, d, i, _dp],
            "zcsrgemm0": [C.c_char, i, i, _dp, _ip, _ip, i, _dp, _dp],
            "zqreco": [i, i, _dp, _dp],
        }
        for name, argt in sig.items():
            f = getattr(L, name)
            f.argtypes = argt
            f.restype = C.c_int
        _zsig_done = True
    return L


def zcall(name, A, *args, log_cap=1 << 20):
    """Run complex reference solver ``name`` on ZMatrix ``A``.

    Like ``call``: 1-D arrays become ``double _Complex*`` (copied), 2-D
    arrays column-major ``zmat``; returns ``(ret, outputs, norms)`` with
    every ``cblas_dznrm2`` / ``cblas_dnrm2`` value of the call."""
    L = _zlib()
    cargs, outs, keep = [], [], []
    for a in args:
        if isinstance(a, np.ndarray) and a.ndim == 2:
            buf = np.asfortranarray(a, dtype=np.complex128).copy(order="F")
            zm = ZMat(buf.shape[0], buf.shape[1], buf.ctypes.data_as(_dp))
            keep.append((buf, zm))
            outs.append(buf)
            cargs.append(C.byref(zm))
        elif isinstance(a, np.ndarray):
            buf = np.ascontiguousarray(a, dtype=np.complex128).copy()
            keep.append(buf)
            outs.append(buf)
            cargs.append(buf.ctypes.data_as(_dp))
        else:
            cargs.append(a)
    log = np.zeros(log_cap)
    with _lock:
        L.oracle_nrm2_log_begin(log.ctypes.data_as(_dp), log_cap)
        ret = getattr(L, name)(A.ptr, *cargs)
        cnt = L.oracle_nrm2_log_end()
    return ret, outs, log[:min(cnt, log_cap)].copy()


def zspmv(A, x, trans=False):
    """Reference ``zcsrgemm0`` (src/matvec.c:55-98): y = A x, or A^H x."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros(A._n.value, dtype=np.complex128)
    _zlib().zcsrgemm0(b"t" if trans else b"n", A._n.value, 1,
                      A.val.ctypes.data_as(_dp), A.rowptr.ctypes.data_as(_ip),
                      A.col.ctypes.data_as(_ip), A._nnz.value,
                      x.ctypes.data_as(_dp), y.ctypes.data_as(_dp))
    return y
