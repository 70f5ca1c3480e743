"""Regenerates the golden fixtures of the parity tests (run in a container
that has the reference sources; the outputs are committed).

    make -C oracle && OPENBLAS_NUM_THREADS=1 python tests/golden/make_golden.py
    OPENBLAS_NUM_THREADS=8 OMP_NUM_THREADS=8 python tests/golden/make_golden.py --full
    OPENBLAS_NUM_THREADS=1 python tests/golden/make_golden.py --complex
    python tests/golden/make_golden.py --thread-spread

* ``testmats.npz`` -- the reference's two test matrices (testmat/bfwb398.mtx,
  symmetric, one triangle; testmat/pde2961.mtx, general) as read by the
  reference's own reader (src/read_matrix.c), plus the 2961x16 right-hand
  side block its driver draws with LAPACKE_dlarnv(seed {1,0,3,2})
  (tests/test.c:70-75).
* ``reference.json`` -- outputs of the compiled reference (oracle/_ref)
  with OpenBLAS on one thread: return value, norm of the solution, FP64 true
  residual and the per-iteration convergence-test history, for the calls of
  tests/test.c and for small seeded configurations of the benchmark problems
  (bksp_b200.problems).
* ``reference_full.json`` (``--full``) -- the same records at the full sizes
  of the block and shifted benchmark configurations (3D Poisson 64^3 with 16
  right-hand sides; 2D convection-diffusion 1024^2 with 32 shifts).
* ``--thread-spread`` adds to ``reference_full.json`` the return value of
  the block configurations' reference solves under OpenBLAS at 1, 2, 3, 4,
  6 and 8 threads (each in a child process): the reference's own spread of
  iteration counts, which comes from the order its threaded dgemm sums the
  Gram products in.
* ``reference_z.json`` (``--complex``) -- the complex solvers zbicg,
  zshbicgstabl and zblbicgstabl on seeded complex problems
  (bksp_b200.problems.complex_*).  zbicgstabl is not recorded: its unit
  coefficient is a real ``double`` read as a complex scalar
  (src/bicgstabl.c:147, 178, 196), so its result depends on stack contents.
"""
import ctypes as C
import json
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref as R          # noqa: E402
from oracle import solvers as S      # noqa: E402
from bksp_b200 import problems as P  # noqa: E402

def reference_dir():
    """The reference's source tree: BKSP_REFERENCE, else the location
    oracle/Makefile builds from."""
    d = os.environ.get("BKSP_REFERENCE")
    if not d:
        import subprocess
        d = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"),
                            "print-ref"], capture_output=True, text=True,
                           check=True).stdout.strip()
    return d


REF_TESTMAT = os.path.join(reference_dir(), "testmat")


def dlarnv_block(n, s):
    lib = C.CDLL(os.path.join(os.path.dirname(R.LIB_PATH), "libbksp_ref.so"))
    f = lib.LAPACKE_dlarnv
    f.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double)]
    seed = (C.c_int * 4)(1, 0, 3, 2)
    out = np.zeros(n * s)
    f(1, seed, n * s, out.ctypes.data_as(C.POINTER(C.c_double)))
    bb = out.reshape(s, n).T.copy()        # column-major n x s
    for i in range(s):
        bb[i, i] = 1.0                      # test.c:73-75: bb[(n+1) i] = 1
    return bb


def csr(rp, c, v, n):
    return sp.csr_matrix((v, c, rp), shape=(n, n))


def hist_of(norms):
    # first dnrm2 is ||b|| (||B||_F); then one per convergence test
    if len(norms) == 0:
        return []
    return list(np.asarray(norms[1:]) / norms[0])


def record(out, key, A_ref, Aop, b, name, args, kind="single", sigma=None):
    ret, outs, norms = R.call(name, A_ref, *args)
    xs = outs[-1]
    rec = {"ret": int(ret), "xnorm": float(np.linalg.norm(xs))}
    if kind == "single":
        rec["hist"] = hist_of(norms)
        rec["true_res"] = S.true_residual(Aop, b, xs)
    elif kind == "block":
        h = hist_of(norms)
        if name == "dblbicgstabl":
            h = h[:-1]                      # last dnrm2: printed true residual
        rec["hist"] = h
        Bm = args[0]
        rec["true_res_cols"] = [float(np.linalg.norm(Bm[:, j] - Aop @ xs[:, j])
                                      / np.linalg.norm(Bm[:, j]))
                                for j in range(Bm.shape[1])]
    elif kind == "shift":
        n = b.size
        rec["hist"] = hist_of(norms)
        rec["true_res_seed"] = S.true_residual(Aop, b, xs[:n])
        rec["true_res_shifts"] = [S.true_residual(Aop, b, xs[(k + 1) * n:(k + 2) * n], s)
                                  for k, s in enumerate(sigma)]
    out[key] = rec
    print(f"{key:28s} ret={ret}")


def main():
    out = {}
    rp2, c2, v2, n2, t2 = R.read_matrix_market(f"{REF_TESTMAT}/bfwb398.mtx")
    rp, c, v, n, t = R.read_matrix_market(f"{REF_TESTMAT}/pde2961.mtx")
    assert t2 == "symmetric" and t == "unsymmetric"
    BB = dlarnv_block(n, 16)
    np.savez_compressed(os.path.join(HERE, "testmats.npz"),
                        bfwb_rowptr=rp2, bfwb_col=c2, bfwb_val=v2,
                        pde_rowptr=rp, pde_col=c, pde_val=v, pde_B=BB)
    A2r = R.Matrix(rp2, c2, v2, n2, symmetric=True)
    A2 = S.full_symmetric(csr(rp2, c2, v2, n2))
    Ar = R.Matrix(rp, c, v, n)
    A = csr(rp, c, v, n)
    b2 = np.zeros(n2); b2[0] = 1.0
    b = np.zeros(n); b[0] = 1.0
    # ---- the calls of tests/test.c
    record(out, "testc/cg", A2r, A2, b2, "bksp_dcg", (b2, 1e-14, 500, np.zeros(n2)))
    record(out, "testc/cr", A2r, A2, b2, "dcr", (b2, 1e-14, 500, np.zeros(n2)))
    I16 = np.zeros((n2, 16)); I16[np.arange(16), np.arange(16)] = 1.0
    record(out, "testc/blcg", A2r, A2, None, "dblcg", (I16, 1e-14, 500, np.zeros((n2, 16))), kind="block")
    record(out, "testc/bicg", Ar, A, b, "dbicg", (b, 1e-14, 500, np.zeros(n)))
    record(out, "testc/bicgstab", Ar, A, b, "dbicgstab", (b, 1e-14, 500, np.zeros(n)))
    record(out, "testc/bicgstabl4", Ar, A, b, "dbicgstabl", (b, 4, 1e-14, 500, np.zeros(n)))
    record(out, "testc/blbicgstab", Ar, A, None, "dblbicgstab", (BB, 1e-14, 500, np.zeros((n, 16))), kind="block")
    record(out, "testc/blbicgstabl6", Ar, A, None, "dblbicgstabl", (BB, 6, 1e-14, 500, np.zeros((n, 16))), kind="block")
    sig = np.array([0.0, 0.2, 0.4, 0.8])
    record(out, "testc/shbicg", Ar, A, b, "dshbicg", (b, sig, 4, 1e-14, 500, np.zeros(5 * n)), kind="shift", sigma=sig)
    record(out, "testc/shbicgstabl1", Ar, A, b, "dshbicgstabl", (b, 1, sig, 4, 1e-14, 200, np.zeros(5 * n)), kind="shift", sigma=sig)
    # ---- small seeded versions of the benchmark configurations
    rp, c, v, n = P.poisson2d(64)
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    Af = csr(rp, c, v, n)
    b = P.uniform(n, 0)
    record(out, "cfg1/cg_poisson64", R.Matrix(lrp, lc, lv, n, symmetric=True), Af, b,
           "bksp_dcg", (b, 1e-10, 10000, np.zeros(n)))
    record(out, "cfg1/cr_poisson64", R.Matrix(lrp, lc, lv, n, symmetric=True), Af, b,
           "dcr", (b, 1e-10, 10000, np.zeros(n)))
    rp, c, v, n = P.convdiff3d(24)
    Af = csr(rp, c, v, n)
    b = Af @ P.uniform(n, 1)
    Ar = R.Matrix(rp, c, v, n)
    for l in (1, 2, 4):
        record(out, f"cfg2/bicgstabl{l}_cd24", Ar, Af, b, "dbicgstabl", (b, l, 1e-10, 2000, np.zeros(n)))
    record(out, "cfg2/bicgstab_cd24", Ar, Af, b, "dbicgstab", (b, 1e-10, 2000, np.zeros(n)))
    record(out, "cfg2/bicg_cd24", Ar, Af, b, "dbicg", (b, 1e-10, 2000, np.zeros(n)))
    rp, c, v, n = P.poisson3d(12)
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    Af = csr(rp, c, v, n)
    Bm = np.random.default_rng(2).standard_normal((n, 16))
    record(out, "cfg3/blcg_p12", R.Matrix(lrp, lc, lv, n, symmetric=True), Af, None,
           "dblcg", (Bm, 1e-10, 2000, np.zeros((n, 16))), kind="block")
    record(out, "cfg3/blbicgstabl2_p12", R.Matrix(rp, c, v, n), Af, None,
           "dblbicgstabl", (Bm, 2, 1e-10, 2000, np.zeros((n, 16))), kind="block")
    record(out, "cfg3/blbicgstab_p12", R.Matrix(rp, c, v, n), Af, None,
           "dblbicgstab", (Bm, 1e-10, 2000, np.zeros((n, 16))), kind="block")
    rp, c, v, n = P.convdiff2d(48)
    Af = csr(rp, c, v, n)
    b = P.uniform(n, 3)
    sig = P.log_shifts(32)
    Ar = R.Matrix(rp, c, v, n)
    record(out, "cfg4/shbicgstabl4_cd48", Ar, Af, b, "dshbicgstabl",
           (b, 4, sig, 32, 1e-10, 2000, np.zeros(33 * n)), kind="shift", sigma=sig)
    record(out, "cfg4/shbicg_cd48", Ar, Af, b, "dshbicg",
           (b, sig, 32, 1e-10, 2000, np.zeros(33 * n)), kind="shift", sigma=sig)
    with open(os.path.join(HERE, "reference.json"), "w") as f:
        json.dump(out, f, indent=1)


def main_full():
    """Full-size configurations (minutes of CPU each), written to
    reference_full.json: shifted BiCGSTAB(4) with 32 shifts on the 2D
    convection-diffusion 1024^2 operator, and Block CG / Block BiCGSTAB(2)
    with 16 right-hand sides on the 3D Poisson 64^3 operator."""
    out = {"threads": os.environ.get("OPENBLAS_NUM_THREADS", "default")}
    rp, c, v, n = P.poisson3d(64)
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    Af = csr(rp, c, v, n)
    Bm = np.random.default_rng(2).standard_normal((n, 16))
    record(out, "cfg3/blcg_p64", R.Matrix(lrp, lc, lv, n, symmetric=True), Af, None,
           "dblcg", (Bm, 1e-8, 5000, np.zeros((n, 16))), kind="block")
    record(out, "cfg3/blbicgstabl2_p64", R.Matrix(rp, c, v, n), Af, None,
           "dblbicgstabl", (Bm, 2, 1e-8, 5000, np.zeros((n, 16))), kind="block")
    rp, c, v, n = P.convdiff2d(1024)
    Af = csr(rp, c, v, n)
    b = P.uniform(n, 3)
    sig = P.log_shifts(32)
    record(out, "cfg4/shbicgstabl4_cd1024", R.Matrix(rp, c, v, n), Af, b,
           "dshbicgstabl", (b, 4, sig, 32, 1e-8, 5000, np.zeros(33 * n)),
           kind="shift", sigma=sig)
    with open(os.path.join(HERE, "reference_full.json"), "w") as f:
        json.dump(out, f, indent=1)


def zrecord(out, key, Aref, Aop, b, name, args, kind, sigma=None):
    from oracle import zsolvers as Z
    ret, outs, norms = R.zcall(name, Aref, *args)
    xs = outs[-1]
    h = hist_of(norms)
    rec = {"ret": int(ret), "xnorm": float(np.linalg.norm(xs))}
    if kind == "single":
        rec["hist"] = h
        rec["true_res"] = Z.true_residual(Aop, b, xs)
    elif kind == "block":
        Bm = args[0]
        rec["hist"] = h[:-1]                # last norm: printed true residual
        rec["true_res_cols"] = [float(np.linalg.norm(Bm[:, j] - Aop @ xs[:, j])
                                      / np.linalg.norm(Bm[:, j]))
                                for j in range(Bm.shape[1])]
    else:
        n = b.size
        rec["hist"] = h
        rec["true_res_seed"] = Z.true_residual(Aop, b, xs[:n])
        rec["true_res_shifts"] = [Z.true_residual(Aop, b, xs[(k + 1) * n:(k + 2) * n], sg)
                                  for k, sg in enumerate(sigma)]
    out[key] = rec
    print(f"{key:28s} ret={ret}")


def main_complex():
    out = {"threads": os.environ.get("OPENBLAS_NUM_THREADS", "default")}
    for tag, gen, nx in (("cd2d24", P.complex_convdiff2d, 24),
                         ("cd3d10", P.complex_convdiff3d, 10)):
        rp, c, v, n = gen(nx)
        Aop = csr(rp, c, v, n)
        Ar = R.ZMatrix(rp, c, v, n)
        b = P.complex_uniform(n, 3)
        zrecord(out, f"zbicg/{tag}", Ar, Aop, b, "zbicg",
                (b, 1e-10, 1000, np.zeros(n, complex)), "single")
        sig = P.complex_shifts(4)
        for l in (1, 2, 4):
            zrecord(out, f"zshbicgstabl{l}/{tag}", Ar, Aop, b, "zshbicgstabl",
                    (b, l, sig, 4, 1e-10, 1000, np.zeros(5 * n, complex)),
                    "shift", sigma=sig)
        rng = np.random.default_rng(7)
        Bm = rng.uniform(-1, 1, (n, 4)) + 1j * rng.uniform(-1, 1, (n, 4))
        for l in (1, 2, 4):
            zrecord(out, f"zblbicgstabl{l}/{tag}", Ar, Aop, None, "zblbicgstabl",
                    (Bm, l, 1e-10, 1000, np.zeros((n, 4), complex)), "block")
    with open(os.path.join(HERE, "reference_z.json"), "w") as f:
        json.dump(out, f, indent=1)


SPREAD_THREADS = (1, 2, 3, 4, 6, 8)


def spread_child(which):
    """One block solve at 64^3 in this process; prints its return value."""
    rp, c, v, n = P.poisson3d(64)
    Bm = np.random.default_rng(2).standard_normal((n, 16))
    if which == "blcg":
        lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
        ret = R.call("dblcg", R.Matrix(lrp, lc, lv, n, symmetric=True),
                     Bm, 1e-8, 5000, np.zeros((n, 16)))[0]
    else:
        ret = R.call("dblbicgstabl", R.Matrix(rp, c, v, n),
                     Bm, 2, 1e-8, 5000, np.zeros((n, 16)))[0]
    print(json.dumps({"ret": int(ret)}))


def main_spread():
    import subprocess
    path = os.path.join(HERE, "reference_full.json")
    with open(path) as f:
        out = json.load(f)
    for key, which in (("cfg3/blcg_p64", "blcg"), ("cfg3/blbicgstabl2_p64", "blbicgstabl2")):
        spread = {}
        for th in SPREAD_THREADS:
            env = dict(os.environ, OPENBLAS_NUM_THREADS=str(th), OMP_NUM_THREADS=str(th))
            r = subprocess.run([sys.executable, os.path.abspath(__file__),
                                "--spread-child", which], env=env,
                               capture_output=True, text=True, check=True)
            spread[str(th)] = json.loads(r.stdout.strip().splitlines()[-1])["ret"]
            print(key, th, spread[str(th)], flush=True)
        out[key]["ret_by_threads"] = spread
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if "--spread-child" in sys.argv[1:]:
        spread_child(sys.argv[sys.argv.index("--spread-child") + 1])
    elif "--thread-spread" in sys.argv[1:]:
        main_spread()
    elif "--full" in sys.argv[1:]:
        main_full()
    elif "--complex" in sys.argv[1:]:
        main_complex()
    else:
        main()
