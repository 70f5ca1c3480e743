"""bksp_b200 -- Python host binding of libbksp.so, the B200 (sm_100a) build
of the bksp Krylov-solver C API.

The functions below mirror ``bksp.h`` one to one (same names, argument
order and meaning, same return codes), taking NumPy arrays where the C API
takes host pointers:

* ``bksp_dcg, dcr, dbicg, dbicgstab, dbicgstabl`` -- single right-hand side;
  ``x`` is updated in place and the bksp return code is returned;
* ``dblcg, dblbicgstab, dblbicgstabl`` -- ``B``/``X`` are n-by-s arrays
  (passed to C column-major, as ``dmat``);
* ``dshbicg, dshbicgstabl`` -- ``x`` has ``n * (len(sigma) + 1)`` entries,
  seed first.

There is no CPU fallback: importing this module loads the CUDA library and
raises if it has not been built (``python -c "import __graft_entry__ as g;
g.build()"`` or ``make -C bksp_b200/csrc``).
"""
import contextlib
import ctypes as C
import os

import numpy as np

NOT_CONVERGED = -1
DIVERGENCE = -2
INVALID_PARAMETERS = -3
INVALID_MATRIX_TYPE = -4

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbksp.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class DSpMat(C.Structure):
    """``dspmat``: 0-based CSR with pointer-to-int size fields."""
    _fields_ = [("row", _ip), ("col", _ip), ("nnz", _ip),
                ("row_size", _ip), ("col_size", _ip), ("value", _dp),
                ("format", C.c_char_p), ("type", C.c_char_p)]


class DMat(C.Structure):
    """``dmat``: column-major dense block."""
    _fields_ = [("row_size", C.c_int), ("col_size", C.c_int), ("value", _dp)]


class Stats(C.Structure):
    """``bksp_gpu_stats`` (bksp_gpu.h)."""
    _fields_ = [("hist", _dp), ("hist_cap", C.c_int), ("hist_len", C.c_int),
                ("ret", C.c_int), ("solve_ms", C.c_double),
                ("total_ms", C.c_double), ("true_res", C.c_double),
                ("launches", C.c_longlong), ("inner_iters", C.c_int),
                ("sweeps", C.c_int), ("alg_bytes", C.c_longlong)]


class MixedOpts(C.Structure):
    """``bksp_gpu_mixed_opts`` (bksp_gpu.h)."""
    _fields_ = [("l", C.c_int), ("target", C.c_double), ("max_iter", C.c_int),
                ("precond", C.c_int), ("model", C.c_void_p),
                ("delta", C.c_double), ("period", C.c_int),
                ("fallback", C.c_int)]


class ZSpMat(C.Structure):
    """``zspmat`` (include/bksp.h): complex values, interleaved (re, im)."""
    _fields_ = [("row", _ip), ("col", _ip), ("nnz", _ip),
                ("row_size", _ip), ("col_size", _ip), ("value", _dp),
                ("format", C.c_char_p), ("type", C.c_char_p)]


class ZMat(C.Structure):
    """``zmat``: column-major complex values."""
    _fields_ = [("row_size", C.c_int), ("col_size", C.c_int), ("value", _dp)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"bksp_b200: CUDA library {LIB_PATH} is not built; run "
            "`make -C bksp_b200/csrc` (there is no CPU fallback)")
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
        "myqr": [i, i, _dp, _dp],
    }
    for name, argt in sig.items():
        f = getattr(L, name)
        f.argtypes = argt
        f.restype = C.c_int
    zp, zm = C.POINTER(ZSpMat), C.POINTER(ZMat)
    zsig = {
        "zbicg": [zp, _dp, d, i, _dp],
        "zbicgstabl": [zp, _dp, i, d, i, _dp],
        "zblbicgstabl": [zp, zm, i, d, i, zm],
        "zshbicgstabl": [zp, _dp, i, _dp, i, d, i, _dp],
        "zqreco": [i, i, _dp, _dp],
    }
    for name, argt in zsig.items():
        f = getattr(L, name)
        f.argtypes = argt
        f.restype = C.c_int
    L.bksp_gpu_zcsrmv.argtypes = [zp, C.c_char, _dp, _dp]
    L.bksp_gpu_zcsrmv.restype = i
    L.zread_matrix_market.argtypes = [C.c_char_p]
    L.zread_matrix_market.restype = zp
    L.bksp_gpu_dcsrmm.argtypes = [sp, C.c_char, i, d, _dp, d, _dp]
    L.bksp_gpu_dcsrmm.restype = i
    L.read_matrix_market.argtypes = [C.c_char_p]
    L.read_matrix_market.restype = sp
    L.bksp_gpu_record.argtypes = [C.POINTER(Stats)]
    L.bksp_gpu_record.restype = None
    L.bksp_gpu_version.restype = C.c_char_p
    vp = C.c_void_p
    L.bksp_gpu_matrix_create.argtypes = [sp, i, C.POINTER(vp)]
    L.bksp_gpu_matrix_destroy.argtypes = [vp]
    L.bksp_gpu_matrix_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.bksp_gpu_solve.argtypes = [vp, i, i, vp, vp, d, i, vp, C.POINTER(Stats)]
    L.bksp_gpu_spmv.argtypes = [vp, i, vp, vp, vp]
    L.bksp_gpu_matrix_variant.argtypes = [vp, i]
    L.bksp_gpu_spmm.argtypes = [vp, i, i, i, vp, vp, vp]
    L.bksp_gpu_matrix_diagonals.argtypes = [vp, C.POINTER(C.c_int)]
    L.bksp_gpu_read_matrix_market.argtypes = [C.c_char_p, i, C.POINTER(vp)]
    L.bksp_gpu_matrix_csr.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]
    L.bksp_gpu_true_residual.argtypes = [vp, vp, vp, vp]
    L.bksp_gpu_true_residual.restype = d
    L.bksp_gpu_device_count.restype = i
    L.bksp_gpu_solve_mixed.argtypes = [vp, vp, vp, C.POINTER(MixedOpts), vp,
                                       C.POINTER(Stats)]
    L.bksp_dbicgstabl_mixed.argtypes = [sp, _dp, C.POINTER(MixedOpts), _dp]
    L.bksp_gpu_cg_mixed.argtypes = [vp, vp, vp, C.POINTER(MixedOpts), vp,
                                    C.POINTER(Stats)]
    L.bksp_dcg_mixed.argtypes = [sp, _dp, C.POINTER(MixedOpts), _dp]
    L.bksp_dblcg_mixed.argtypes = [sp, mp, C.POINTER(MixedOpts), mp]
    L.bksp_dshbicgstabl_mixed.argtypes = [sp, _dp, _dp, i, C.POINTER(MixedOpts), _dp]
    L.bksp_dblbicgstabl_mixed.argtypes = [sp, mp, C.POINTER(MixedOpts), mp]
    L.bksp_gpu_solve_mixed_batch.argtypes = [C.POINTER(vp), C.POINTER(vp),
                                             C.POINTER(vp), i,
                                             C.POINTER(MixedOpts), i,
                                             C.POINTER(Stats)]
    L.bksp_gpu_solve_batch.argtypes = [C.POINTER(vp), i, i, C.POINTER(vp),
                                       C.POINTER(vp), i, d, i, i,
                                       C.POINTER(Stats)]
    L.bksp_gpu_persist_status.argtypes = [C.POINTER(C.c_int)]
    L.bksp_gpu_persist_status.restype = i
    L.bksp_gpu_persist_debug.argtypes = [C.c_longlong, i]
    L.bksp_gpu_persist_debug.restype = None
    L.bksp_gpu_loop_mode.argtypes = [i]
    L.bksp_gpu_loop_mode.restype = i
    L.bksp_gpu_spai_create.argtypes = [C.c_uint, C.POINTER(vp)]
    L.bksp_gpu_spai_destroy.argtypes = [vp]
    L.bksp_gpu_spai_params.argtypes = [vp, C.POINTER(C.c_float), i]
    L.bksp_gpu_spai_train.argtypes = [vp, C.POINTER(vp), i, i, i, C.c_float,
                                      C.c_uint, C.POINTER(d)]
    L.bksp_gpu_spai_loss_grad.argtypes = [vp, vp, C.POINTER(C.c_float), i,
                                          C.c_uint, C.POINTER(d),
                                          C.POINTER(C.c_float)]
    L.bksp_gpu_spai_save.argtypes = [vp, C.c_char_p]
    L.bksp_gpu_spai_load.argtypes = [C.c_char_p, C.POINTER(vp)]
    return L


lib = _load()


class CsrMatrix:
    """A ``dspmat`` over NumPy buffers (kept alive by this object).

    ``symmetric=True`` sets type "symmetric": the arrays then hold one
    triangle and the operator mirrors the off-diagonal entries.
    """

    def __init__(self, rowptr, col, val, n=None, symmetric=False):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        nnz = int(self.rowptr[-1]) if self.rowptr.size else 0
        if self.rowptr.ndim != 1 or self.rowptr.size < 2:
            raise ValueError("rowptr must hold n + 1 >= 2 entries")
        if self.col.shape != (nnz,) or self.val.shape != (nnz,):
            raise ValueError(f"col and val must hold rowptr[-1] = {nnz} entries "
                             f"(got {self.col.shape}, {self.val.shape})")
        n = self.rowptr.size - 1 if n is None else int(n)
        self.n = n
        self.symmetric = bool(symmetric)
        self._nnz = C.c_int(int(self.col.size))
        self._n = C.c_int(n)
        self._m = C.c_int(n)
        self.s = DSpMat(self.rowptr.ctypes.data_as(_ip),
                        self.col.ctypes.data_as(_ip), C.pointer(self._nnz),
                        C.pointer(self._n), C.pointer(self._m),
                        self.val.ctypes.data_as(_dp), b"csr",
                        b"symmetric" if symmetric else b"unsymmetric")

    @property
    def ptr(self):
        return C.byref(self.s)


def _vec(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


def _dmat(a):
    buf = np.asfortranarray(a, dtype=np.float64)
    return buf, DMat(buf.shape[0], buf.shape[1], buf.ctypes.data_as(_dp))


def _inplace(x):
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64
            and x.flags.c_contiguous):
        raise TypeError("x must be a C-contiguous float64 array (updated in place)")
    return x.ctypes.data_as(_dp)


def bksp_dcg(A, b, tol, max_iter, x):
    b = _vec(b)
    return lib.bksp_dcg(A.ptr, b.ctypes.data_as(_dp), tol, max_iter, _inplace(x))


def dcr(A, b, tol, max_iter, x):
    b = _vec(b)
    return lib.dcr(A.ptr, b.ctypes.data_as(_dp), tol, max_iter, _inplace(x))


def dbicg(A, b, tol, max_iter, x):
    b = _vec(b)
    return lib.dbicg(A.ptr, b.ctypes.data_as(_dp), tol, max_iter, _inplace(x))


def dbicgstab(A, b, tol, max_iter, x):
    b = _vec(b)
    return lib.dbicgstab(A.ptr, b.ctypes.data_as(_dp), tol, max_iter,
                         _inplace(x))


def dbicgstabl(A, b, l, tol, max_iter, x):
    b = _vec(b)
    return lib.dbicgstabl(A.ptr, b.ctypes.data_as(_dp), l, tol, max_iter,
                          _inplace(x))


def _block(fn, A, B, args, X):
    Bf, Bm = _dmat(B)
    Xf, Xm = _dmat(X)
    ret = fn(A.ptr, C.byref(Bm), *args, C.byref(Xm))
    X[...] = Xf
    return ret


def dblcg(A, B, tol, max_iter, X):
    """X (n-by-s NumPy array) is updated in place."""
    return _block(lib.dblcg, A, B, (tol, max_iter), X)


def dblbicgstab(A, B, tol, max_iter, X):
    return _block(lib.dblbicgstab, A, B, (tol, max_iter), X)


def dblbicgstabl(A, B, l, tol, max_iter, X):
    return _block(lib.dblbicgstabl, A, B, (l, tol, max_iter), X)


def dshbicg(A, b, sigma, tol, max_iter, x):
    b = _vec(b)
    s = _vec(sigma)
    return lib.dshbicg(A.ptr, b.ctypes.data_as(_dp), s.ctypes.data_as(_dp),
                       int(s.size), tol, max_iter, _inplace(x))


def dshbicgstabl(A, b, l, sigma, tol, max_iter, x):
    b = _vec(b)
    s = _vec(sigma)
    return lib.dshbicgstabl(A.ptr, b.ctypes.data_as(_dp), l,
                            s.ctypes.data_as(_dp), int(s.size), tol,
                            max_iter, _inplace(x))


def dcsrmm(A, Bm, C, alpha=1.0, beta=0.0, trans="n"):
    """C = beta C + alpha A B on the GPU (bksp_gpu_dcsrmm); C (n-by-s) is
    updated in place."""
    Bf = np.asfortranarray(Bm, dtype=np.float64)
    Cf = np.asfortranarray(C, dtype=np.float64)
    rc = lib.bksp_gpu_dcsrmm(A.ptr, trans.encode(), Bf.shape[1], float(alpha),
                             Bf.ctypes.data_as(_dp), float(beta),
                             Cf.ctypes.data_as(_dp))
    C[...] = Cf
    return rc


def myqr(V):
    """Thin QR of an m-by-n array; returns (Q, R, info)."""
    Vf = np.asfortranarray(V, dtype=np.float64).copy(order="F")
    m, n = Vf.shape
    R = np.zeros((n, n), order="F")
    info = lib.myqr(m, n, Vf.ctypes.data_as(_dp), R.ctypes.data_as(_dp))
    return Vf, R, info


def read_matrix_market(path):
    """Returns (rowptr, col, val, n, type) from the library's reader."""
    p = lib.read_matrix_market(os.fsencode(path))
    if not p:
        raise OSError(f"cannot read Matrix Market file {path}")
    m = p.contents
    n = m.row_size[0]
    nnz = m.nnz[0]
    rowptr = np.ctypeslib.as_array(m.row, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(m.col, shape=(nnz,)).copy() if nnz else np.zeros(0, np.int32)
    val = np.ctypeslib.as_array(m.value, shape=(nnz,)).copy() if nnz else np.zeros(0)
    return rowptr, col, val, n, m.type.decode()


# ------------------------------------------------------------- complex

class ZCsrMatrix:
    """A ``zspmat`` over NumPy buffers (values complex128)."""

    def __init__(self, rowptr, col, val, n=None):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.complex128)
        nnz = int(self.rowptr[-1]) if self.rowptr.size else 0
        if self.rowptr.ndim != 1 or self.rowptr.size < 2:
            raise ValueError("rowptr must hold n + 1 >= 2 entries")
        if self.col.shape != (nnz,) or self.val.shape != (nnz,):
            raise ValueError(f"col and val must hold rowptr[-1] = {nnz} entries")
        n = self.rowptr.size - 1 if n is None else int(n)
        self.n = n
        self._nnz = C.c_int(int(self.col.size))
        self._n = C.c_int(n)
        self._m = C.c_int(n)
        self.s = ZSpMat(self.rowptr.ctypes.data_as(_ip),
                        self.col.ctypes.data_as(_ip), C.pointer(self._nnz),
                        C.pointer(self._n), C.pointer(self._m),
                        self.val.ctypes.data_as(_dp), b"csr", b"unsymmetric")

    @property
    def ptr(self):
        return C.byref(self.s)


def _zinplace(x):
    if not (isinstance(x, np.ndarray) and x.dtype == np.complex128
            and x.flags.c_contiguous):
        raise TypeError("x must be a C-contiguous complex128 array (updated in place)")
    return x.ctypes.data_as(_dp)


def _zvec(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def zbicg(A, b, tol, max_iter, x):
    b = _zvec(b)
    return lib.zbicg(A.ptr, b.ctypes.data_as(_dp), tol, max_iter, _zinplace(x))


def zbicgstabl(A, b, l, tol, max_iter, x):
    b = _zvec(b)
    return lib.zbicgstabl(A.ptr, b.ctypes.data_as(_dp), l, tol, max_iter,
                          _zinplace(x))


def zshbicgstabl(A, b, l, sigma, tol, max_iter, x):
    """x: n * (len(sigma) + 1) complex entries, seed first, in place."""
    b = _zvec(b)
    s = _zvec(sigma)
    return lib.zshbicgstabl(A.ptr, b.ctypes.data_as(_dp), l,
                            s.ctypes.data_as(_dp), int(s.size), tol, max_iter,
                            _zinplace(x))


def zblbicgstabl(A, B, l, tol, max_iter, X):
    """X (n-by-s complex) is updated in place."""
    Bf = np.asfortranarray(B, dtype=np.complex128)
    Xf = np.asfortranarray(X, dtype=np.complex128)
    bm = ZMat(Bf.shape[0], Bf.shape[1], Bf.ctypes.data_as(_dp))
    xm = ZMat(Xf.shape[0], Xf.shape[1], Xf.ctypes.data_as(_dp))
    rc = lib.zblbicgstabl(A.ptr, C.byref(bm), l, tol, max_iter, C.byref(xm))
    X[...] = Xf
    return rc


def zcsrmv(A, x, trans="n"):
    """y = A x ('n') or A^H x ('t') on the GPU (bksp_gpu_zcsrmv)."""
    x = _zvec(x)
    y = np.zeros(A.n, dtype=np.complex128)
    rc = lib.bksp_gpu_zcsrmv(A.ptr, trans.encode(), x.ctypes.data_as(_dp),
                             y.ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError(f"bksp_gpu_zcsrmv failed ({rc})")
    return y


def zqreco(V):
    """Thin QR of an m-by-n complex array; returns (Q, R, info)."""
    Vf = np.asfortranarray(V, dtype=np.complex128).copy(order="F")
    m, n = Vf.shape
    R = np.zeros((n, n), dtype=np.complex128, order="F")
    info = lib.zqreco(m, n, Vf.ctypes.data_as(_dp), R.ctypes.data_as(_dp))
    return Vf, R, info


def zread_matrix_market(path):
    """Returns (rowptr, col, val, n, type) from the complex reader."""
    p = lib.zread_matrix_market(os.fsencode(path))
    if not p:
        raise OSError(f"cannot read complex Matrix Market file {path}")
    m = p.contents
    n = m.row_size[0]
    nnz = m.nnz[0]
    rowptr = np.ctypeslib.as_array(m.row, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(m.col, shape=(nnz,)).copy()
    raw = np.ctypeslib.as_array(m.value, shape=(2 * nnz,)).copy()
    return rowptr, col, raw[0::2] + 1j * raw[1::2], n, m.type.decode()


@contextlib.contextmanager
def record(hist_cap=0):
    """Collect ``bksp_gpu_stats`` of the bksp calls made inside the block.

    Yields a dict filled on exit: ``ret``, ``hist`` (convergence-test values,
    one per iteration), ``solve_ms``, ``total_ms``.
    """
    buf = np.zeros(max(int(hist_cap), 1))
    st = Stats(buf.ctypes.data_as(_dp), int(hist_cap), 0, 0, 0.0, 0.0, 0.0,
               0, 0, 0)
    out = {}
    lib.bksp_gpu_record(C.byref(st))
    try:
        yield out
    finally:
        lib.bksp_gpu_record(None)
        out["ret"] = st.ret
        out["hist_len"] = st.hist_len
        out["hist"] = buf[:min(st.hist_len, int(hist_cap))].copy()
        out["solve_ms"] = st.solve_ms
        out["total_ms"] = st.total_ms
        out["true_res"] = st.true_res
        out["launches"] = st.launches
        out["alg_bytes"] = st.alg_bytes
        out["inner_iters"] = st.inner_iters
        out["sweeps"] = st.sweeps


def version():
    return lib.bksp_gpu_version().decode()


# ------------------------------------------------------ device-resident API

MIRROR, FP32, TRANSPOSE = 1, 2, 4
CG, CR, BICG, BICGSTAB, BICGSTABL, BICGSTABL_FAST = 1, 2, 3, 4, 5, 6


class GpuMatrix:
    """``bksp_gpu_matrix``: an operator uploaded once and kept in HBM."""

    def __init__(self, A, flags=0, _handle=None):
        if _handle is not None:
            h = _handle
        else:
            h = C.c_void_p()
            rc = lib.bksp_gpu_matrix_create(A.ptr, int(flags), C.byref(h))
            if rc != 0:
                raise RuntimeError(f"bksp_gpu_matrix_create failed ({rc})")
        self.h = h
        n, nnz = C.c_int(), C.c_int()
        lib.bksp_gpu_matrix_info(h, C.byref(n), C.byref(nnz))
        self.n, self.nnz = n.value, nnz.value

    @classmethod
    def from_matrix_market(cls, path, flags=0):
        """bksp_gpu_read_matrix_market: a .mtx file straight into GPU memory
        (rows sorted and, with MIRROR, the triangle mirrored on the GPU)."""
        h = C.c_void_p()
        rc = lib.bksp_gpu_read_matrix_market(os.fsencode(path), int(flags), C.byref(h))
        if rc != 0:
            raise OSError(f"cannot load Matrix Market file {path} ({rc})")
        return cls(None, _handle=h)

    def csr(self):
        """The operator's CSR as stored on the device: (rowptr, col, val)."""
        rp = np.zeros(self.n + 1, np.int32)
        col = np.zeros(max(self.nnz, 1), np.int32)
        val = np.zeros(max(self.nnz, 1))
        rc = lib.bksp_gpu_matrix_csr(self.h, rp.ctypes.data_as(_ip),
                                     col.ctypes.data_as(_ip), val.ctypes.data_as(_dp))
        if rc != 0:
            raise RuntimeError("bksp_gpu_matrix_csr failed")
        return rp, col[:self.nnz], val[:self.nnz]

    def close(self):
        if self.h:
            lib.bksp_gpu_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve_mixed(self, b_ptr, x_ptr, l=4, target=1e-8, max_iter=10000,
                    precond=0, model=None, delta=0.0, period=0, fallback=1,
                    stream=None, hist_cap=0, method="bicgstabl"):
        """Mixed-precision BiCGSTAB(l) (method="cg": preconditioned CG,
        bksp_gpu_cg_mixed) on device vectors; (ret, stats)."""
        o = MixedOpts(l, target, max_iter, precond,
                      model.h if model is not None else None, delta, period,
                      fallback)
        buf = np.zeros(max(int(hist_cap), 1))
        st = Stats(buf.ctypes.data_as(_dp), int(hist_cap), 0, 0, 0.0, 0.0,
                   0.0, 0, 0, 0)
        fn = lib.bksp_gpu_cg_mixed if method == "cg" else lib.bksp_gpu_solve_mixed
        ret = fn(self.h, b_ptr, x_ptr, C.byref(o), stream, C.byref(st))
        return ret, {"ret": st.ret, "hist": buf[:min(st.hist_len, hist_cap)].copy(),
                     "iters": st.hist_len, "solve_ms": st.solve_ms,
                     "true_res": st.true_res, "launches": st.launches,
                     "alg_bytes": st.alg_bytes,
                     "inner_iters": st.inner_iters,
                     "sweeps": st.sweeps // 1000,
                     "replacements": st.sweeps % 1000}

    def solve(self, method, b_ptr, x_ptr, tol, max_iter, l=0, stream=None,
              hist_cap=0):
        """Device pointers b, x (n doubles).  Returns (ret, stats dict)."""
        buf = np.zeros(max(int(hist_cap), 1))
        st = Stats(buf.ctypes.data_as(_dp), int(hist_cap), 0, 0, 0.0, 0.0,
                   0.0, 0, 0, 0)
        ret = lib.bksp_gpu_solve(self.h, method, l, b_ptr, x_ptr, tol,
                                 max_iter, stream, C.byref(st))
        return ret, {"ret": st.ret, "hist": buf[:min(st.hist_len, hist_cap)].copy(),
                     "hist_len": st.hist_len, "solve_ms": st.solve_ms,
                     "true_res": st.true_res, "launches": st.launches,
                     "alg_bytes": st.alg_bytes,
                     "inner_iters": st.inner_iters, "sweeps": st.sweeps}

    SPMV_VARIANTS = {0: "tile", 1: "tma", 2: "vec4", 3: "vec8", 4: "vec16",
                     5: "vec32", 6: "wtile", 7: "dia", 8: "sell"}

    def diagonals(self):
        """Column offsets of the operator's diagonal form ([] when none)."""
        off = (C.c_int * 8)()
        nd = lib.bksp_gpu_matrix_diagonals(self.h, off)
        if nd < 0:
            raise RuntimeError("bksp_gpu_matrix_diagonals failed")
        return list(off[:nd])

    def variant(self, v=-1):
        """Query (v < 0) or set the SpMV kernel variant; returns it."""
        return lib.bksp_gpu_matrix_variant(self.h, int(v))

    def spmv(self, x_ptr, y_ptr, fp32=False, stream=None):
        rc = lib.bksp_gpu_spmv(self.h, int(bool(fp32)), x_ptr, y_ptr, stream)
        if rc != 0:
            raise RuntimeError("bksp_gpu_spmv failed")

    def spmm(self, s, X_ptr, Y_ptr, fp32=False, kernel=-1, stream=None):
        """Y = A X for row-major device blocks (n x s); kernel -1 autotuned,
        0 diagonal form, 1 CSR."""
        rc = lib.bksp_gpu_spmm(self.h, int(fp32), int(s), int(kernel), X_ptr,
                               Y_ptr, stream)
        if rc != 0:
            raise RuntimeError(f"bksp_gpu_spmm failed ({rc})")

    def true_residual(self, b_ptr, x_ptr, stream=None):
        return lib.bksp_gpu_true_residual(self.h, b_ptr, x_ptr, stream)


PRECOND_NONE, PRECOND_JACOBI, PRECOND_LEARNED = 0, 1, 2


class SpaiModel:
    """``bksp_gpu_spai_model``: the learned SPAI preconditioner's MLP."""

    def __init__(self, seed=0, path=None):
        h = C.c_void_p()
        if path is not None:
            rc = lib.bksp_gpu_spai_load(os.fsencode(path), C.byref(h))
        else:
            rc = lib.bksp_gpu_spai_create(int(seed), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"spai model creation failed ({rc})")
        self.h = h
        self.nparams = lib.bksp_gpu_spai_nparams()

    def close(self):
        if self.h:
            lib.bksp_gpu_spai_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        assert lib.bksp_gpu_spai_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), 0) == 0
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        assert lib.bksp_gpu_spai_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), 1) == 0

    def train(self, systems, epochs=20, probes=8, lr=1e-3, seed=1):
        arr = (C.c_void_p * len(systems))(*[s.h for s in systems])
        loss = C.c_double(0.0)
        rc = lib.bksp_gpu_spai_train(self.h, arr, len(systems), int(epochs),
                                     int(probes), float(lr), int(seed),
                                     C.byref(loss))
        if rc != 0:
            raise RuntimeError(f"spai training failed ({rc})")
        return loss.value

    def train_logged(self, systems, probe_systems, rounds=4, epochs=25,
                     probes=8, lr=1e-3, seed=1, l=2, target=1e-8):
        """Training with logged iteration counts: `rounds` rounds of
        `epochs` epochs of the ||(I - M A) Z||_F loss (train); after each
        round the learned mixed BiCGSTAB(l) solves every probe system
        ((CsrMatrix, b) pairs held out from `systems`) to the FP64 target
        and its iteration counts are logged.  The gradient comes from the
        loss (iteration counts are not differentiable); the logged counts
        pick the round whose parameters the model keeps (fewest total
        iterations; a round with a failed solve is never picked).  Returns
        {"best_round", "rounds": [{"loss", "iters"}, ...]}."""
        log, best, best_total, best_p = [], -1, None, None
        for r in range(rounds):
            loss = self.train(systems, epochs=epochs, probes=probes, lr=lr,
                              seed=seed + r)
            iters = []
            for A, b in probe_systems:
                x = np.zeros(A.n)
                ret = dbicgstabl_mixed(A, b, x, l=l, target=target,
                                       precond=PRECOND_LEARNED, model=self,
                                       fallback=0)
                iters.append(int(ret))
            log.append({"loss": float(loss), "iters": iters})
            if min(iters) >= 0 and (best_total is None or sum(iters) < best_total):
                best, best_total, best_p = r, sum(iters), self.params()
        if best_p is not None:
            self.set_params(best_p)
        return {"best_round": best, "rounds": log}

    def loss_grad(self, A, Z=None, probes=8, seed=1):
        """Loss and gradient; Z: (probes, n) float32 or None (seeded)."""
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_double(0.0)
        zp = None
        if Z is not None:
            Z = np.ascontiguousarray(Z, dtype=np.float32)
            probes = Z.shape[0]
            zp = Z.ctypes.data_as(C.POINTER(C.c_float))
        rc = lib.bksp_gpu_spai_loss_grad(self.h, A.h, zp, int(probes), int(seed),
                                         C.byref(loss),
                                         g.ctypes.data_as(C.POINTER(C.c_float)))
        if rc != 0:
            raise RuntimeError(f"spai loss/grad failed ({rc})")
        return loss.value, g

    def save(self, path):
        if lib.bksp_gpu_spai_save(self.h, os.fsencode(path)) != 0:
            raise OSError(f"cannot write {path}")


def dbicgstabl_mixed(A, b, x, l=4, target=1e-8, max_iter=10000, precond=0,
                     model=None, fallback=1):
    """Host-array mixed-precision solve (bksp_dbicgstabl_mixed)."""
    b = _vec(b)
    o = MixedOpts(l, target, max_iter, precond,
                  model.h if model is not None else None, 0.0, 0, fallback)
    return lib.bksp_dbicgstabl_mixed(A.ptr, b.ctypes.data_as(_dp), C.byref(o),
                                     _inplace(x))


def dcg_mixed(A, b, x, target=1e-8, max_iter=10000, precond=0, model=None,
              fallback=1):
    """Host-array mixed-precision preconditioned CG (bksp_dcg_mixed); A is
    a "symmetric" CsrMatrix holding one triangle, as for bksp_dcg."""
    b = _vec(b)
    o = MixedOpts(0, target, max_iter, precond,
                  model.h if model is not None else None, 0.0, 0, fallback)
    return lib.bksp_dcg_mixed(A.ptr, b.ctypes.data_as(_dp), C.byref(o),
                              _inplace(x))


def dblcg_mixed(A, B, X, target=1e-8, max_iter=10000, inner_tol=0.0):
    """bksp_dblcg_mixed: Block CG, FP64 refinement around FP32 inner solves
    (inner relative residual inner_tol, 0: 1e-4); X (n-by-s) updated in
    place."""
    o = MixedOpts(0, target, max_iter, 0, None, inner_tol, 0, 0)
    return _block(lib.bksp_dblcg_mixed, A, B, (C.byref(o),), X)


def dblbicgstabl_mixed(A, B, l, X, target=1e-8, max_iter=10000, inner_tol=0.0):
    """bksp_dblbicgstabl_mixed: Block BiCGSTAB(l), as dblcg_mixed."""
    o = MixedOpts(l, target, max_iter, 0, None, inner_tol, 0, 0)
    return _block(lib.bksp_dblbicgstabl_mixed, A, B, (C.byref(o),), X)


def dshbicgstabl_mixed(A, b, l, sigma, x, target=1e-8, max_iter=10000):
    """bksp_dshbicgstabl_mixed: FP32 shift vectors, FP64 per-shift
    polishing; x (n * (len(sigma) + 1), seed first) updated in place."""
    b = _vec(b)
    s = _vec(sigma)
    o = MixedOpts(l, target, max_iter, 0, None, 0.0, 0, 0)
    return lib.bksp_dshbicgstabl_mixed(A.ptr, b.ctypes.data_as(_dp),
                                       s.ctypes.data_as(_dp), int(s.size),
                                       C.byref(o), _inplace(x))


def _batch_args(mats, bs, xs):
    n = len(mats)
    if len(bs) != n or len(xs) != n:
        raise ValueError("one b and one x per matrix")
    A = (C.c_void_p * n)(*[m.h for m in mats])
    B = (C.c_void_p * n)(*[int(p) for p in bs])
    X = (C.c_void_p * n)(*[int(p) for p in xs])
    st = (Stats * n)()
    return n, A, B, X, st


def _batch_stats(st):
    return [{"ret": s.ret, "hist_len": s.hist_len, "true_res": s.true_res,
             "launches": s.launches, "alg_bytes": s.alg_bytes,
             "iters": s.hist_len,
             "inner_iters": s.inner_iters, "sweeps": s.sweeps,
             "solve_ms": s.solve_ms} for s in st]


def solve_mixed_batch(mats, bs, xs, l=4, target=1e-8, max_iter=10000,
                      precond=0, model=None, delta=0.0, period=0, fallback=1,
                      workers=0):
    """bksp_gpu_solve_mixed_batch: mixed-precision BiCGSTAB(l) on every
    (GpuMatrix, b, x) of the lists (device pointers, ready before the call,
    x in/out); workers>=0: that many host threads (0: 8), one graph loop
    per system; workers<0: all systems in one persistent launch.  Returns
    (ret, per-system stats)."""
    n, A, B, X, st = _batch_args(mats, bs, xs)
    o = MixedOpts(l, target, max_iter, precond,
                  model.h if model is not None else None, delta, period,
                  fallback)
    ret = lib.bksp_gpu_solve_mixed_batch(A, B, X, n, C.byref(o), int(workers), st)
    return ret, _batch_stats(st)


def solve_batch(mats, method, bs, xs, tol, max_iter, l=4, workers=0):
    """bksp_gpu_solve_batch: an FP64 method (CG ... BICGSTABL_FAST) on every
    system of the lists; returns (ret, per-system stats)."""
    n, A, B, X, st = _batch_args(mats, bs, xs)
    ret = lib.bksp_gpu_solve_batch(A, int(method), int(l), B, X, n, float(tol),
                                   int(max_iter), int(workers), st)
    return ret, _batch_stats(st)


def persist_status():
    """(status, grid) of this thread's last persistent batch: status 0 ok,
    1 a grid-barrier wait ran out, 2 launch failure."""
    g = C.c_int(0)
    st = lib.bksp_gpu_persist_status(C.byref(g))
    return st, g.value


def persist_debug(spin_limit=0, absent_cta=-1):
    """Test hook of the persistent batch's bounded barrier waits."""
    lib.bksp_gpu_persist_debug(int(spin_limit), int(absent_cta))


@contextlib.contextmanager
def loop_mode(mode):
    """Run this thread's single-system solves with iteration loop `mode`
    (0 CUDA-graph loop, 1 persistent launch) inside the block."""
    prev = lib.bksp_gpu_loop_mode(int(mode))
    try:
        yield
    finally:
        lib.bksp_gpu_loop_mode(prev)
