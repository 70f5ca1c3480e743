"""GPU tests of the batched solves (bksp_gpu_solve_mixed_batch,
bksp_gpu_solve_batch) on kappa-diffusion systems of different sizes:
every system converges to the FP64 target, and the batch gives exactly the
single-system results."""
import numpy as np
import pytest
import scipy.sparse as sp

from bksp_b200 import problems as P
from oracle import solvers as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems(gpu):
    B = gpu
    out = []
    for i, L in enumerate((10, 13, 16, 12, 19, 14)):
        rp, c, v, n = P.kappa_diffusion3d(L, 50 + i)
        b = np.random.default_rng(80 + i).standard_normal(n)
        A = sp.csr_matrix((v, c, rp), shape=(n, n))
        out.append((B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32), A, b, rp, c, v))
    yield out
    for s in out:
        s[0].close()


@pytest.fixture(scope="module")
def kmodel(gpu):
    B = gpu
    mats = [B.GpuMatrix(B.CsrMatrix(*P.kappa_diffusion3d(L, 900 + L)[:3]), B.FP32)
            for L in (10, 12, 14)]
    model = B.SpaiModel(seed=2)
    model.train(mats, epochs=60, probes=8, lr=3e-3, seed=3)
    yield model
    for m in mats:
        m.close()
    model.close()


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.mark.parametrize("precond", [1, 2])
def test_mixed_batch_matches_single_solves(gpu, systems, kmodel, precond):
    import torch
    B = gpu
    bs = [_dev(torch, s[2]) for s in systems]
    xs = [torch.zeros_like(b) for b in bs]
    torch.cuda.synchronize()
    ret, st = B.solve_mixed_batch([s[0] for s in systems],
                                  [b.data_ptr() for b in bs],
                                  [x.data_ptr() for x in xs], l=2, target=1e-8,
                                  precond=precond, model=kmodel, workers=3)
    assert ret == 0, [s["ret"] for s in st]
    for (G, A, b, *_), x, s in zip(systems, xs, st):
        xh = x.cpu().numpy()
        assert s["ret"] >= 0
        assert S.true_residual(A, b, xh) <= 1e-8
        # the same system alone
        x1 = torch.zeros_like(x)
        torch.cuda.synchronize()
        r1, _ = G.solve_mixed(_dev(torch, b).data_ptr(), x1.data_ptr(), l=2,
                              target=1e-8, precond=precond, model=kmodel)
        torch.cuda.synchronize()
        assert r1 == s["ret"]
        assert np.array_equal(x1.cpu().numpy(), xh)


def test_fp64_batch_jacobi_scaled(gpu, systems):
    """FP64 BiCGSTAB(2) on the right-Jacobi-scaled systems A D^-1 y = b,
    x = D^-1 y (the plain comparator of the batched workload)."""
    import torch
    B = gpu
    mats, bs, xs, dinv = [], [], [], []
    for (_, A, b, rp, c, v) in systems:
        d = A.diagonal()
        vs = v / d[c]                       # column scaling
        mats.append(B.GpuMatrix(B.CsrMatrix(rp, c, vs)))
        bs.append(_dev(torch, b))
        xs.append(torch.zeros_like(bs[-1]))
        dinv.append(1.0 / d)
    torch.cuda.synchronize()
    ret, st = B.solve_batch(mats, B.BICGSTABL_FAST, [b.data_ptr() for b in bs],
                            [x.data_ptr() for x in xs], 1e-9, 5000, l=2, workers=4)
    assert ret == 0, [s["ret"] for s in st]
    for (_, A, b, *_), x, di in zip(systems, xs, dinv):
        xh = x.cpu().numpy() * di
        assert S.true_residual(A, b, xh) <= 1e-8
    for m in mats:
        m.close()


def test_batch_rejects_missing_operand(gpu, systems):
    import ctypes as C
    B = gpu
    G = systems[0][0]
    A = (C.c_void_p * 2)(G.h, None)
    b = (C.c_void_p * 2)(1, 1)
    x = (C.c_void_p * 2)(1, 1)
    o = B.MixedOpts(2, 1e-8, 100, 0, None, 0.0, 0, 0)
    assert B.lib.bksp_gpu_solve_mixed_batch(A, b, x, 2, C.byref(o), 2, None) == -3
    assert B.lib.bksp_gpu_solve_mixed_batch(A, b, x, 0, C.byref(o), 2, None) == 0
