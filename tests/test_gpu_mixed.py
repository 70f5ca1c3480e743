"""GPU tests of the mixed-precision solve and the learned SPAI
preconditioner: FP64 target reached and checked on the host, error against
an FP64 oracle solve, the MLP gradient against the NumPy oracle, what the
trained network gains over the unpreconditioned and Jacobi solves, the
stagnation fallback and checkpoint files."""
import numpy as np
import pytest
import scipy.sparse as sp

from bksp_b200 import problems as P
from oracle import mlp
from oracle import solvers as S

pytestmark = pytest.mark.gpu


def _system(gen, nx, seed=1):
    rp, c, v, n = gen(nx)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = A @ P.uniform(n, seed)
    return rp, c, v, n, A, b


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    return torch


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.fixture(scope="module")
def trained(gpu):
    """A model trained briefly on small 3D convection-diffusion systems."""
    B = gpu
    mats = [B.GpuMatrix(B.CsrMatrix(*P.convdiff3d(nx)[:3]), B.FP32) for nx in (12, 16)]
    model = B.SpaiModel(seed=3)
    loss0 = model.loss_grad(mats[1], probes=8, seed=5)[0]
    loss = model.train(mats, epochs=150, probes=8, lr=3e-3, seed=7)
    yield model, loss0, loss
    for m in mats:
        m.close()


def test_spai_gradient_matches_oracle(gpu):
    B = gpu
    rp, c, v, n = P.convdiff2d(18)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    model = B.SpaiModel(seed=11)
    rng = np.random.default_rng(4)
    p = model.params().astype(np.float64)
    W1, b1, W2, b2, W3, b3 = mlp.unpack(p)
    W3[...] = rng.uniform(-0.2, 0.2, W3.shape)      # exercise every layer
    b1[...] = rng.uniform(-0.1, 0.1, b1.shape)
    model.set_params(p.astype(np.float32))
    p32 = model.params().astype(np.float64)
    Z = rng.choice([-1.0, 1.0], size=(4, n)).astype(np.float32)
    loss_g, g_g = model.loss_grad(G, Z=Z)
    A32 = sp.csr_matrix((v.astype(np.float32).astype(np.float64), c, rp), shape=(n, n))
    AZ = (A32 @ Z.astype(np.float64).T).T
    loss_o, g_o = mlp.loss_grad(p32, rp, c, v, n, Z.astype(np.float64), AZ)
    assert abs(loss_g - loss_o) <= 1e-4 * loss_o
    assert np.linalg.norm(g_g - g_o) <= 1e-3 * np.linalg.norm(g_o)
    G.close()


@pytest.mark.parametrize("precond", [0, 1])
def test_mixed_reaches_fp64_target(gpu, torch_cuda, precond):
    B, torch = gpu, torch_cuda
    rp, c, v, n, A, b = _system(P.convdiff3d, 24)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    bd, xd = _dev(torch, b), torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), l=4, target=1e-8,
                            precond=precond, hist_cap=1000)
    x = xd.cpu().numpy()
    assert ret >= 0, st
    tr = S.true_residual(A, b, x)
    assert tr <= 1e-8 and abs(tr - st["true_res"]) <= 1e-3 * tr + 1e-15
    ret_o, x_o, _ = S.bicgstabl(A, b, 4, 1e-12, 1000)
    assert np.linalg.norm(x - x_o) <= 1e-6 * np.linalg.norm(x_o)
    assert st["replacements"] >= 1
    G.close()


def test_learned_preconditioner_gains(gpu, torch_cuda, trained):
    B, torch = gpu, torch_cuda
    model, loss0, loss = trained
    assert loss < 0.8 * loss0, (loss0, loss)
    rp, c, v, n, A, b = _system(P.convdiff3d, 32)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    bd = _dev(torch, b)
    its = {}
    for name, pc, md in (("none", 0, None), ("jacobi", 1, None),
                         ("learned", 2, model)):
        xd = torch.zeros(n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), l=4, target=1e-8,
                                precond=pc, model=md, fallback=0)
        assert ret >= 0, (name, st)
        assert S.true_residual(A, b, xd.cpu().numpy()) <= 1e-8
        its[name] = st["iters"]
    # What the trained network buys: fewer outer iterations than the same
    # solve without it (Jacobi is a no-op on this constant-diagonal matrix).
    assert its["learned"] <= 0.8 * its["none"], its
    G.close()


def test_fallback_on_broken_model(gpu, torch_cuda):
    B, torch = gpu, torch_cuda
    rp, c, v, n, A, b = _system(P.convdiff3d, 16)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    bad = B.SpaiModel(seed=1)
    p = bad.params()
    p[-8:] = np.nan                         # output bias NaN -> M is NaN
    bad.set_params(p)
    bd = _dev(torch, b)
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), precond=2, model=bad,
                            fallback=0)
    assert ret == B.DIVERGENCE
    xd.zero_()
    torch.cuda.synchronize()
    ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), precond=2, model=bad,
                            fallback=1)
    assert ret >= 0 and st["sweeps"] == 2
    assert S.true_residual(A, b, xd.cpu().numpy()) <= 1e-8
    G.close()


def test_checkpoint_roundtrip_and_host_api(gpu, trained, tmp_path):
    B = gpu
    model = trained[0]
    path = str(tmp_path / "spai.bin")
    model.save(path)
    loaded = B.SpaiModel(path=path)
    assert np.array_equal(loaded.params(), model.params())
    rp, c, v, n, A, b = _system(P.convdiff3d, 20)
    x = np.zeros(n)
    ret = B.dbicgstabl_mixed(B.CsrMatrix(rp, c, v), b, x, l=4, target=1e-8,
                             precond=2, model=loaded)
    assert ret >= 0 and S.true_residual(A, b, x) <= 1e-8


@pytest.mark.parametrize("fast", [False, True])
def test_one_pass_mr_matches_mgs(gpu, torch_cuda, golden, fast):
    """BiCGSTAB(l) with the one-pass (Gram) minimal-residual step follows the
    reference's iteration as closely as the MGS form does."""
    B, torch = gpu, torch_cuda
    rp, c, v, n, A, b = _system(P.convdiff3d, 24)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    bd = _dev(torch, b)
    for l in (1, 2, 4):
        xd = torch.zeros(n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ret, st = G.solve(B.BICGSTABL_FAST if fast else B.BICGSTABL,
                          bd.data_ptr(), xd.data_ptr(), 1e-10, 2000, l=l,
                          hist_cap=500)
        gk = golden[f"cfg2/bicgstabl{l}_cd24"]
        assert abs(ret - gk["ret"]) <= 2, (l, ret, gk["ret"])
        k = min(10, len(gk["hist"]))
        np.testing.assert_allclose(st["hist"][:k], gk["hist"][:k], rtol=1e-6)
        assert S.true_residual(A, b, xd.cpu().numpy()) < 1e-9
    G.close()


@pytest.mark.parametrize("precond", [0, 1, 2])
def test_mixed_solve_same_with_diagonal_form(gpu, torch_cuda, trained, precond):
    """The diagonal-form SpMV sums each row in the CSR order, so a mixed
    solve (A and M products) gives bit-identical results with either kernel."""
    B, torch = gpu, torch_cuda
    model = trained[0]
    rp, c, v, n, A, b = _system(P.convdiff3d, 20)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    assert len(G.diagonals()) == 7
    bd = _dev(torch, b)
    out = []
    for variant in (0, 7):
        G.variant(variant)
        xd = torch.zeros(n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), l=4, target=1e-8,
                                precond=precond, model=model)
        out.append((ret, st["true_res"], xd.cpu().numpy()))
    assert out[0][0] == out[1][0] >= 0
    assert out[0][1] == out[1][1] <= 1e-8
    assert np.array_equal(out[0][2], out[1][2])
    G.close()


# ------------------------------------------------- mixed-precision CG

@pytest.fixture(scope="module")
def poisson_model(gpu):
    """A model trained on small 2D Poisson systems (the CG configuration's
    family)."""
    B = gpu
    mats = [B.GpuMatrix(B.CsrMatrix(*P.poisson2d(nx)[:3]), B.FP32) for nx in (16, 24, 32)]
    model = B.SpaiModel(seed=5)
    model.train(mats, epochs=150, probes=8, lr=3e-3, seed=9)
    yield model
    for m in mats:
        m.close()
    model.close()


@pytest.mark.parametrize("precond", [0, 1, 2])
def test_mixed_cg_reaches_fp64_target(gpu, torch_cuda, poisson_model, precond):
    """The 2D Poisson 64^2 system (b ~ U[-1,1], seed 0): mixed CG reaches an
    FP64 true relative residual of 1e-8, with the solution within 1e-6 of
    the FP64 oracle solve; the symmetrised learned preconditioner needs
    fewer iterations than none."""
    B, torch = gpu, torch_cuda
    rp, c, v, n = P.poisson2d(64)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 0)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    bd, xd = _dev(torch, b), torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), target=1e-8,
                            precond=precond, model=poisson_model,
                            hist_cap=2000, method="cg")
    x = xd.cpu().numpy()
    assert ret >= 0, st
    assert S.true_residual(A, b, x) <= 1e-8
    assert abs(st["true_res"] - S.true_residual(A, b, x)) <= 1e-10
    ref = sp.linalg.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - ref) <= 1e-6 * np.linalg.norm(ref)
    assert st["replacements"] >= 1
    if precond == 0:
        ret_o, _, _ = S.cg(A, b, 1e-8, 10000)
        # FP32 vectors with replacement: close to the FP64 iteration count
        assert abs(ret - ret_o) <= max(3, 0.1 * ret_o), (ret, ret_o)
    G.close()


def test_mixed_cg_learned_gains(gpu, torch_cuda, poisson_model):
    B, torch = gpu, torch_cuda
    rp, c, v, n = P.poisson2d(64)
    b = P.uniform(n, 0)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    its = {}
    for pc in (0, 2):
        bd, xd = _dev(torch, b), torch.zeros(n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), target=1e-8,
                                precond=pc, model=poisson_model, method="cg")
        assert ret >= 0
        its[pc] = ret
    assert its[2] <= 0.8 * its[0], its
    G.close()


def test_mixed_cg_host_arrays_and_matrix_type(gpu, poisson_model):
    """bksp_dcg_mixed takes bksp_dcg's one-triangle "symmetric" matrix and
    gives the device call's result; an "unsymmetric" matrix is refused as
    bksp_dcg refuses it."""
    B = gpu
    rp, c, v, n = P.poisson2d(48)
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 4)
    x = np.zeros(n)
    ret = B.dcg_mixed(B.CsrMatrix(lrp, lc, lv, symmetric=True), b, x,
                      precond=B.PRECOND_LEARNED, model=poisson_model)
    assert ret >= 0
    assert S.true_residual(A, b, x) <= 1e-8
    x2 = np.zeros(n)
    assert B.dcg_mixed(B.CsrMatrix(rp, c, v), b, x2) == B.INVALID_MATRIX_TYPE


@pytest.mark.parametrize("precond", [0, 2])
def test_mixed_cg_fused_matches_unfused(gpu, torch_cuda, poisson_model, precond):
    """The two-launch CG iteration (vector updates fused into the diagonal
    products) against the four-launch one: the same iteration counts within
    two, both at the FP64 target, and fewer launches."""
    import os
    import subprocess
    import sys
    B, torch = gpu, torch_cuda
    rp, c, v, n = P.poisson2d(96)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 5)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    bd, xd = _dev(torch, b), torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ret, st = G.solve_mixed(bd.data_ptr(), xd.data_ptr(), target=1e-8,
                            precond=precond, model=poisson_model, method="cg")
    x = xd.cpu().numpy()
    assert ret >= 0 and S.true_residual(A, b, x) <= 1e-8
    G.close()
    # The unfused iteration in a child process (BKSP_GPU_FUSE=0 is read once).
    code = (
        "import sys, numpy as np, torch; sys.path.insert(0, %r)\n"
        "import bksp_b200 as B\nfrom bksp_b200 import problems as P\n"
        "rp, c, v, n = P.poisson2d(96)\n"
        "mats = [B.GpuMatrix(B.CsrMatrix(*P.poisson2d(k)[:3]), B.FP32) for k in (16, 24, 32)]\n"
        "m = B.SpaiModel(seed=5); m.train(mats, epochs=150, probes=8, lr=3e-3, seed=9)\n"
        "G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)\n"
        "b = torch.from_numpy(P.uniform(n, 5)).cuda(); x = torch.zeros_like(b)\n"
        "r, s = G.solve_mixed(b.data_ptr(), x.data_ptr(), target=1e-8, precond=%d, model=m, method='cg')\n"
        "print(r, s['launches'])\n" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))), precond))
    out = subprocess.run([sys.executable, "-c", code], env=dict(os.environ, BKSP_GPU_FUSE="0"),
                         capture_output=True, text=True, timeout=300)
    r0, l0 = [int(t) for t in out.stdout.split()[-2:]]
    assert r0 >= 0 and abs(r0 - ret) <= 2, (r0, ret)
    assert st["launches"] < l0, (st["launches"], l0)


def test_training_with_logged_iteration_counts(gpu):
    """SpaiModel.train_logged: the loss drives training; the learned solve's
    iteration counts on held-out systems are logged after every round and
    pick the parameters kept (the round with the fewest total iterations),
    which then reproduce that round's counts."""
    from bksp_b200 import problems as P
    train = [gpu.GpuMatrix(gpu.CsrMatrix(*P.kappa_diffusion3d(L, 1000 + i)[:3]), gpu.FP32)
             for i, L in enumerate((12, 14, 16, 18))]
    probe = []
    for i, L in enumerate((16, 20)):
        rp, c, v, n = P.kappa_diffusion3d(L, 5000 + i)
        probe.append((gpu.CsrMatrix(rp, c, v), np.random.default_rng(i).standard_normal(n)))
    model = gpu.SpaiModel(seed=3)
    log = model.train_logged(train, probe, rounds=3, epochs=10, probes=4,
                             lr=3e-3, seed=7, l=2)
    assert len(log["rounds"]) == 3
    totals = [sum(r["iters"]) for r in log["rounds"]]
    assert all(min(r["iters"]) >= 0 for r in log["rounds"])
    assert log["best_round"] == int(np.argmin(totals))
    again = []
    for A, b in probe:
        x = np.zeros(A.n)
        again.append(gpu.dbicgstabl_mixed(A, b, x, l=2, target=1e-8,
                                          precond=gpu.PRECOND_LEARNED,
                                          model=model, fallback=0))
    assert again == log["rounds"][log["best_round"]]["iters"]
    for m in train:
        m.close()
