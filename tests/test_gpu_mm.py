"""GPU Matrix Market loader (bksp_gpu_read_matrix_market) against the host
reader: the same CSR, entry for entry, for general and symmetric files,
entries in file order (including a file whose entries are shuffled), and
the mirrored operator of a symmetric file with its rows in column order."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import solvers as S

pytestmark = pytest.mark.gpu


def _write(path, rp, c, v, sym, order=None):
    n = rp.size - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    idx = np.arange(rows.size) if order is None else order
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real "
                + ("symmetric" if sym else "general") + "\n% comment\n")
        f.write(f"{n} {n} {rows.size}\n")
        for k in idx:
            f.write(f"{rows[k] + 1} {c[k] + 1} {float(v[k])!r}\n")


@pytest.mark.parametrize("name,sym", [("pde", False), ("bfwb", True)])
@pytest.mark.parametrize("shuffle", [False, True])
def test_gpu_loader_matches_host_reader(gpu, testmats, tmp_path, name, sym, shuffle):
    B = gpu
    rp, c, v = (testmats[f"{name}_rowptr"], testmats[f"{name}_col"],
                testmats[f"{name}_val"])
    order = np.random.default_rng(3).permutation(c.size) if shuffle else None
    p = tmp_path / f"{name}.mtx"
    _write(p, rp, c, v, sym, order)
    hrp, hc, hv, n, _ = B.read_matrix_market(str(p))
    G = B.GpuMatrix.from_matrix_market(str(p))
    grp, gc, gv = G.csr()
    assert np.array_equal(grp, hrp) and np.array_equal(gc, hc) and np.array_equal(gv, hv)
    G.close()
    if sym:
        # mirrored: the full operator, each row in ascending column order
        Gm = B.GpuMatrix.from_matrix_market(str(p), B.MIRROR | B.FP32)
        mrp, mc, mv = Gm.csr()
        full = S.full_symmetric(sp.csr_matrix((hv, hc, hrp), shape=(n, n))).tocsr()
        full.sort_indices()
        assert np.array_equal(mrp, full.indptr) and np.array_equal(mc, full.indices)
        assert np.array_equal(mv, full.data)
        # and it solves like the handle built from host arrays
        Gh = B.GpuMatrix(B.CsrMatrix(hrp, hc, hv, symmetric=True), B.MIRROR | B.FP32)
        assert np.array_equal(Gh.csr()[1], mc)
        Gh.close()
        Gm.close()


def test_gpu_loader_rejects_bad_files(gpu, tmp_path):
    B = gpu
    bad = {"rect.mtx": "%%MatrixMarket matrix coordinate real general\n3 4 1\n1 1 2.0\n",
           "range.mtx": "%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 2.0\n",
           "count.mtx": "%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 2.0\n",
           "cplx.mtx": "%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n"}
    for fname, text in bad.items():
        (tmp_path / fname).write_text(text)
        with pytest.raises(OSError):
            B.GpuMatrix.from_matrix_market(str(tmp_path / fname))
    with pytest.raises(OSError):
        B.GpuMatrix.from_matrix_market(str(tmp_path / "missing.mtx"))
