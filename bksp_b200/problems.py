"""Seeded synthetic linear systems with the shapes of the solver benchmarks.

All generators return SciPy-free plain CSR arrays ``(rowptr, col, val, n)``
(int32 / int32 / float64, columns ascending within each row) so they feed
both the C-ABI (``dspmat``) and NumPy/SciPy checkers.

Stencil scaling is h^2-scaled (2D Poisson: diagonal 4, off-diagonals -1).
Upwind convection with cell Peclet number 0.5 and diffusion 1 gives
grid-independent coefficients:

* 3D convection-diffusion, velocity (1, 0.5, 0.25): diagonal 7.75,
  x- -2, x+ -1, y- -1.5, y+ -1, z- -1.25, z+ -1;
* 2D convection-diffusion: diagonal 5.5, x- -2, x+ -1, y- -1.5, y+ -1.

Grid index is ``x + nx*(y + ny*z)``; Dirichlet boundaries drop the
off-grid neighbours.
"""
import numpy as np

# (dx, dy, dz, coefficient) in ascending linear-offset order.
STENCIL_POISSON2D = [(0, -1, 0, -1.0), (-1, 0, 0, -1.0), (0, 0, 0, 4.0),
                     (1, 0, 0, -1.0), (0, 1, 0, -1.0)]
STENCIL_CONVDIFF2D = [(0, -1, 0, -1.5), (-1, 0, 0, -2.0), (0, 0, 0, 5.5),
                      (1, 0, 0, -1.0), (0, 1, 0, -1.0)]
STENCIL_POISSON3D = [(0, 0, -1, -1.0), (0, -1, 0, -1.0), (-1, 0, 0, -1.0),
                     (0, 0, 0, 6.0), (1, 0, 0, -1.0), (0, 1, 0, -1.0),
                     (0, 0, 1, -1.0)]
STENCIL_CONVDIFF3D = [(0, 0, -1, -1.25), (0, -1, 0, -1.5), (-1, 0, 0, -2.0),
                      (0, 0, 0, 7.75), (1, 0, 0, -1.0), (0, 1, 0, -1.0),
                      (0, 0, 1, -1.0)]


def stencil_csr(stencil, nx, ny, nz=1):
    """Assemble a constant-coefficient stencil on an nx*ny*nz Dirichlet grid."""
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)
    k = len(stencil)
    cols = np.empty((n, k), dtype=np.int64)
    vals = np.empty((n, k), dtype=np.float64)
    mask = np.empty((n, k), dtype=bool)
    for s, (dx, dy, dz, c) in enumerate(stencil):
        xx, yy, zz = x + dx, y + dy, z + dz
        mask[:, s] = ((xx >= 0) & (xx < nx) & (yy >= 0) & (yy < ny)
                      & (zz >= 0) & (zz < nz))
        cols[:, s] = xx + nx * (yy + ny * zz)
        vals[:, s] = c
    counts = mask.sum(axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    col = cols[mask].astype(np.int32)
    val = vals[mask]
    return rowptr.astype(np.int32), col, val, n


def lower_triangle(rowptr, col, val, n):
    """One-triangle ("symmetric" in bksp) storage: entries with col <= row."""
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    keep = col <= rows
    counts = np.bincount(rows[keep], minlength=n)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    return rp.astype(np.int32), col[keep].copy(), val[keep].copy(), n


def poisson2d(nx):
    return stencil_csr(STENCIL_POISSON2D, nx, nx)


def convdiff2d(nx):
    return stencil_csr(STENCIL_CONVDIFF2D, nx, nx)


def poisson3d(nx):
    return stencil_csr(STENCIL_POISSON3D, nx, nx, nx)


def convdiff3d(nx):
    return stencil_csr(STENCIL_CONVDIFF3D, nx, nx, nx)


def complex_convdiff2d(nx, seed=11, lo=0.2, hi=1.0):
    """Complex non-Hermitian test operator: the 2D convection-diffusion
    stencil plus a seeded imaginary absorption on the diagonal,
    A = convdiff2d + i diag(d), d_i ~ U(lo, hi).  Values complex128."""
    rowptr, col, val, n = convdiff2d(nx)
    d = np.random.default_rng(seed).uniform(lo, hi, n)
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    v = val.astype(np.complex128)
    v[col == rows] += 1j * d
    return rowptr, col, v, n


def complex_convdiff3d(nx, seed=11, lo=0.2, hi=1.0):
    """3D counterpart of ``complex_convdiff2d``."""
    rowptr, col, val, n = convdiff3d(nx)
    d = np.random.default_rng(seed).uniform(lo, hi, n)
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    v = val.astype(np.complex128)
    v[col == rows] += 1j * d
    return rowptr, col, v, n


def complex_uniform(n, seed):
    """Seeded complex vector, real and imaginary parts U(-1, 1)."""
    g = np.random.default_rng(seed)
    return g.uniform(-1.0, 1.0, n) + 1j * g.uniform(-1.0, 1.0, n)


def complex_shifts(count=8, lo=-3.0, hi=0.0, angle=0.25 * np.pi):
    """sigma_k = 10^(lo + (hi-lo) k/(count-1)) e^{i angle}."""
    return log_shifts(count, lo, hi) * np.exp(1j * angle)


def permuted(rowptr, col, val, n, seed=21):
    """P A P^T for a seeded random permutation P, columns ascending within
    each row: the same operator without a diagonal form (a stand-in for an
    unstructured matrix of the same size and row lengths)."""
    perm = np.random.default_rng(seed).permutation(n)    # new index of row i
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    r2 = perm[rows]
    c2 = perm[col]
    order = np.lexsort((c2, r2))
    counts = np.bincount(r2, minlength=n)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    return (rp.astype(np.int32), c2[order].astype(np.int32),
            np.asarray(val)[order].copy(), n)


def csr_matvec(rowptr, col, val, x):
    """y = A x in float64 (host helper for building right-hand sides)."""
    n = rowptr.size - 1
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    return np.bincount(rows, weights=val * x[col], minlength=n)


def uniform(n, seed):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


def log_shifts(count=32, lo=-3.0, hi=0.0):
    """sigma_k = 10^(lo + (hi-lo) k/(count-1)), k = 0..count-1."""
    return 10.0 ** (lo + (hi - lo) * np.arange(count) / (count - 1))


def gaussian_random_field(L, seed, corr=0.1, var=1.0):
    """Stationary Gaussian random field on the L^3 cell centres of the unit
    cube with covariance var * exp(-r^2 / (2 corr^2)), by spectral sampling:
    white noise filtered in Fourier space with the square root of the
    covariance's spectral density (periodic FFT, then normalised to zero
    mean and variance `var`)."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((L, L, L))
    k = 2.0 * np.pi * np.fft.fftfreq(L, d=1.0 / L)
    kz = 2.0 * np.pi * np.fft.rfftfreq(L, d=1.0 / L)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    filt = np.exp(-0.25 * corr * corr * k2)   # sqrt of exp(-corr^2 k^2 / 2)
    g = np.fft.irfftn(np.fft.rfftn(noise) * filt, s=(L, L, L), axes=(0, 1, 2))
    g -= g.mean()
    s = g.std()
    return g * (np.sqrt(var) / s if s > 0 else 0.0)


def kappa_diffusion3d(L, seed):
    """-div(kappa grad u) = f on an L^3 cell-centred grid of the unit cube,
    Dirichlet u = 0 on the boundary, 7-point finite volumes (h^2-scaled):
    face coefficient = harmonic mean 2 k_i k_j / (k_i + k_j) between
    neighbouring cells, 2 k_i on a boundary face; kappa = exp(g) with g a
    Gaussian random field (correlation length 0.1, variance 1, seed).
    Symmetric positive definite.  Returns (rowptr, col, val, n)."""
    kap = np.exp(gaussian_random_field(L, seed)).reshape(-1)   # index x + L(y + L z)
    n = L ** 3
    idx = np.arange(n, dtype=np.int64)
    x = idx % L
    y = (idx // L) % L
    z = idx // (L * L)
    # neighbours in ascending linear-offset order: z-, y-, x-, (diag), x+, y+, z+
    nbr = [(0, 0, -1), (0, -1, 0), (-1, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]
    cols = np.empty((n, 7), dtype=np.int64)
    vals = np.zeros((n, 7), dtype=np.float64)
    mask = np.ones((n, 7), dtype=bool)
    diag = np.zeros(n)
    slot = [0, 1, 2, 4, 5, 6]
    for (dx, dy, dz), s in zip(nbr, slot):
        xx, yy, zz = x + dx, y + dy, z + dz
        inside = (xx >= 0) & (xx < L) & (yy >= 0) & (yy < L) & (zz >= 0) & (zz < L)
        j = np.where(inside, xx + L * (yy + L * zz), 0)
        kf = np.where(inside, 2.0 * kap * kap[j] / (kap + kap[j]), 2.0 * kap)
        diag += kf
        cols[:, s] = j
        vals[:, s] = -kf
        mask[:, s] = inside
    cols[:, 3] = idx
    vals[:, 3] = diag
    counts = mask.sum(axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    return rowptr.astype(np.int32), cols[mask].astype(np.int32), vals[mask], n


def kappa_batch_edges(count=64, seed=4, lo=32, hi=96):
    """Edge lengths L_i ~ U{lo..hi} (seed) of the batched workload."""
    return np.random.default_rng(seed).integers(lo, hi + 1, count)


def kappa_batch(count=64, seed=4, lo=32, hi=96, field_seed0=5, indices=None):
    """The batched workload: `count` kappa-diffusion systems with edge
    lengths L ~ U{lo..hi} (seed), field seeds field_seed0 + i, right-hand
    sides f ~ N(0, 1) (seed field_seed0 + i + 10000).  Returns a list of
    (rowptr, col, val, n, b) for all systems, or for `indices` only (the
    same systems as in the full batch)."""
    Ls = kappa_batch_edges(count, seed, lo, hi)
    out = []
    for i, L in enumerate(Ls):
        if indices is not None and i not in indices:
            continue
        rp, c, v, n = kappa_diffusion3d(int(L), field_seed0 + i)
        b = np.random.default_rng(field_seed0 + i + 10000).standard_normal(n)
        out.append((rp, c, v, n, b))
    return out
