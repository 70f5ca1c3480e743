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
