"""bksp_gpu_true_residual_noalloc -- the residual entry point for callers
that cannot allocate device memory (a host application whose own pool owns
the GPU's memory, or a latency-critical loop that cannot take cudaMalloc's
device-wide synchronisation).  Its scratch is a static device array, so this
checks it against the allocating bksp_gpu_true_residual on the same inputs,
twice in a row (the shared array keeps the previous call's contents), and
that an operator larger than the array's row limit is refused.

Kept in a file pytest collects last, so a stop-at-first-failure run has
already run every other test if this one fails."""
import ctypes as C

import numpy as np
import pytest

from bksp_b200 import problems as P

pytestmark = pytest.mark.gpu


def _noalloc(B):
    f = B.lib.bksp_gpu_true_residual_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_double)]
    f.restype = C.c_int
    return f


def test_noalloc_residual_matches_allocating_entry_point(gpu):
    import torch
    B = gpu
    rp, c, v, n = P.convdiff3d(40)
    A = B.GpuMatrix(B.CsrMatrix(rp, c, v))
    rng = np.random.default_rng(11)
    b = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    x = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    torch.cuda.synchronize()
    f = _noalloc(B)
    ref = A.true_residual(b.data_ptr(), x.data_ptr())
    assert np.isfinite(ref) and ref > 0
    for _ in range(2):
        out = C.c_double(-1.0)
        rc = f(A.h, b.data_ptr(), x.data_ptr(), None, C.byref(out))
        assert rc == 0
        assert abs(out.value - ref) <= 1e-12 * ref, (out.value, ref)
    # A second operator / vectors through the same scratch.
    rp2, c2, v2, n2 = P.poisson2d(50)
    A2 = B.GpuMatrix(B.CsrMatrix(rp2, c2, v2))
    b2 = torch.from_numpy(rng.uniform(-1, 1, n2)).cuda()
    x2 = torch.zeros(n2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    out = C.c_double(-1.0)
    assert f(A2.h, b2.data_ptr(), x2.data_ptr(), None, C.byref(out)) == 0
    assert abs(out.value - 1.0) <= 1e-12     # x = 0: ||b|| / ||b||
    A.close()
    A2.close()


def test_noalloc_on_caller_stream_and_second_thread(gpu):
    """A caller-supplied stream, and a call from a thread whose library
    stream is created by that call, give the allocating entry point's
    value."""
    import threading

    import torch
    B = gpu
    rp, c, v, n = P.convdiff3d(24)
    A = B.GpuMatrix(B.CsrMatrix(rp, c, v))
    rng = np.random.default_rng(12)
    b = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    x = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    torch.cuda.synchronize()
    ref = A.true_residual(b.data_ptr(), x.data_ptr())
    f = _noalloc(B)
    s = torch.cuda.Stream()
    for _ in range(2):
        out = C.c_double(-1.0)
        assert f(A.h, b.data_ptr(), x.data_ptr(), C.c_void_p(s.cuda_stream),
                 C.byref(out)) == 0
        assert abs(out.value - ref) <= 1e-12 * ref, (out.value, ref)
    got = {}

    def worker():
        torch.cuda.set_device(0)
        o = C.c_double(-1.0)
        got["rc"] = f(A.h, b.data_ptr(), x.data_ptr(), None, C.byref(o))
        got["res"] = o.value

    t = threading.Thread(target=worker)
    t.start()
    t.join()
    assert got["rc"] == 0
    assert abs(got["res"] - ref) <= 1e-12 * ref, (got, ref)
    A.close()


def test_noalloc_rejects_operators_beyond_its_limit(gpu):
    import torch
    B = gpu
    n = (1 << 20) + 1
    rp = np.arange(n + 1, dtype=np.int32)
    A = B.GpuMatrix(B.CsrMatrix(rp, np.arange(n, dtype=np.int32), np.ones(n)))
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    out = C.c_double(-1.0)
    rc = _noalloc(B)(A.h, b.data_ptr(), b.data_ptr(), None, C.byref(out))
    assert rc == B.INVALID_PARAMETERS
    assert out.value == -1.0
    A.close()
