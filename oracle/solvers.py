"""NumPy FP64 restatement of the reference's real Krylov solvers.

TEST INFRASTRUCTURE ONLY: this is the checker, never the product path.

Each function follows one reference routine statement by statement (cited by
file:line of aldente39/bksp) and returns ``(ret, x, hist)``:

* ``ret``  -- the reference's return convention: the 0-based index of the
  iteration whose convergence test passed, ``-1`` (NOT_CONVERGED) otherwise,
  ``-4`` (INVALID_MATRIX_TYPE) for a non-"symmetric" matrix given to the
  symmetric-only methods;
* ``x``    -- the solution (``X`` n-by-s for the block methods; for the
  shifted methods ``x[0:n]`` is the seed and ``x[(k+1)n:(k+2)n]`` solves
  ``(A + sigma_k I) x = b``);
* ``hist`` -- the value the convergence test compared with ``tol`` at each
  iteration (recursive residual norm / ||b||, or the block methods'
  ``||C||_F / ||B||_F`` and ``||xi||_F / ||B||_F``).

Matrices are SciPy CSR.  ``Asym`` arguments of the symmetric methods hold one
triangle, as the reference stores "symmetric" matrices; ``full_symmetric``
mirrors it the way ``dcsrsymm0`` (src/matvec.c:100-127) does.
"""
import math

import numpy as np
import scipy.sparse as sp

NOT_CONVERGED = -1
DIVERGENCE = -2
INVALID_PARAMETERS = -3
INVALID_MATRIX_TYPE = -4


def full_symmetric(L):
    """Full operator of a one-triangle CSR: off-diagonals mirrored once."""
    L = sp.csr_matrix(L)
    d = sp.diags(L.diagonal())
    return sp.csr_matrix(L + L.T - d)


def _finish(error, tol, idx):
    # Every solver ends with `if (error >= tol) return NOT_CONVERGED;
    # return i;` (e.g. src/cg.c:67-70).  A NaN error is not >= tol, so the
    # reference would return the loop index there; the restatement keeps that.
    return NOT_CONVERGED if error >= tol else idx


def cg(A, b, tol, max_iter, x0=None, symmetric=True):
    """bksp_dcg, src/cg.c:6-71 (A is the full operator)."""
    if not symmetric:
        return INVALID_MATRIX_TYPE, None, []           # cg.c:9-11
    n = b.size
    x = np.zeros(n) if x0 is None else x0.astype(float).copy()
    r = b - A @ x                                       # cg.c:23-27
    p = r.copy()                                        # cg.c:28
    r_dot_old = r @ r                                   # cg.c:29
    fnb = np.linalg.norm(b)                             # cg.c:30
    error, hist, i = 0.0, [], 0
    for i in range(max_iter):                           # cg.c:33
        t = A @ p                                       # cg.c:35
        alpha = r_dot_old / (t @ p)                     # cg.c:39
        x += alpha * p                                  # cg.c:42
        r -= alpha * t                                  # cg.c:45
        r_dot = r @ r                                   # cg.c:48
        beta = r_dot / r_dot_old                        # cg.c:49
        r_dot_old = r_dot
        p = beta * p + r                                # cg.c:53-54
        error = np.linalg.norm(r) / fnb                 # cg.c:56
        hist.append(error)
        if error < tol:
            break
    else:
        i = max_iter
    return _finish(error, tol, i), x, hist


def cr(A, b, tol, max_iter, x0=None, symmetric=True):
    """dcr, src/cr.c:6-80.  The loop index starts at 1 (cr.c:37)."""
    if not symmetric:
        return INVALID_MATRIX_TYPE, None, []
    n = b.size
    x = np.zeros(n) if x0 is None else x0.astype(float).copy()
    r = b - A @ x                                       # cr.c:24-27
    p = r.copy()
    t = A @ r                                           # cr.c:30
    ap = t.copy()                                       # cr.c:32
    r_dot_old = r @ t                                   # cr.c:33
    norm_b = np.linalg.norm(b)
    error, hist, i = 0.0, [], 1
    i = 1
    while i < max_iter:                                 # cr.c:37
        alpha = r_dot_old / (ap @ ap)                   # cr.c:39
        x += alpha * p
        r -= alpha * ap
        t = A @ r                                       # cr.c:48
        r_dot = r @ t
        beta = r_dot / r_dot_old
        r_dot_old = r_dot
        p = beta * p + r                                # cr.c:57-58
        ap = beta * ap + t                              # cr.c:61-62
        error = np.linalg.norm(r) / norm_b
        hist.append(error)
        if error < tol:
            break
        i += 1
    return _finish(error, tol, i), x, hist


def bicg(A, b, tol, max_iter, x0=None):
    """dbicg, src/bicg.c:7-88 (uses A^T for the shadow recurrence)."""
    n = b.size
    AT = sp.csr_matrix(A.T)
    x = np.zeros(n) if x0 is None else x0.astype(float).copy()
    r = b - A @ x                                       # bicg.c:20-24
    sr = r.copy()
    p, s_p = r.copy(), sr.copy()
    r_dot_old = r @ sr                                  # bicg.c:28
    norm_b = np.linalg.norm(b)
    error, hist, i = 0.0, [], 0
    for i in range(max_iter):
        ap = A @ p                                      # bicg.c:34
        atp = AT @ s_p                                  # bicg.c:38
        alpha = r_dot_old / (ap @ s_p)                  # bicg.c:42
        x += alpha * p
        r -= alpha * ap
        sr -= alpha * atp                               # bicg.c:51
        r_dot = r @ sr
        beta = r_dot / r_dot_old
        r_dot_old = r_dot
        p = beta * p + r
        s_p = beta * s_p + sr                           # bicg.c:63-64
        error = np.linalg.norm(r) / norm_b
        hist.append(error)
        if error < tol:
            break
    else:
        i = max_iter
    return _finish(error, tol, i), x, hist


def bicgstab(A, b, tol, max_iter, x0=None):
    """dbicgstab, src/bicgstab.c:5-72."""
    n = b.size
    x = np.zeros(n) if x0 is None else x0.astype(float).copy()
    r = b - A @ x                                       # bicgstab.c:22-26
    p, rs = r.copy(), r.copy()
    norm_b = np.linalg.norm(b)
    rho = rs @ r                                        # bicgstab.c:30
    error, hist, i = 0.0, [], 0
    for i in range(max_iter):
        ap = A @ p                                      # bicgstab.c:34
        alpha = rho / (rs @ ap)
        s = r - alpha * ap                              # bicgstab.c:38-39
        as_ = A @ s                                     # bicgstab.c:41
        omega = (as_ @ s) / (as_ @ as_)                 # bicgstab.c:43
        x += alpha * p
        x += omega * s
        r = s - omega * as_                             # bicgstab.c:48-49
        rho_new = rs @ r
        beta = alpha / omega * rho_new / rho            # bicgstab.c:52
        rho = rho_new
        p = beta * (p - omega * ap) + r                 # bicgstab.c:55-57
        error = np.linalg.norm(r) / norm_b
        hist.append(error)
        if error < tol:
            break
    else:
        i = max_iter
    return _finish(error, tol, i), x, hist


def bicgstabl(A, b, l, tol, max_iter, x0=None):
    """dbicgstabl (Sleijpen-Fokkema BiCGSTAB(l)), src/bicgstabl.c:13-138."""
    n = b.size
    x = np.zeros(n) if x0 is None else x0.astype(float).copy()
    r = [np.zeros(n) for _ in range(l + 1)]
    p = [np.zeros(n) for _ in range(l + 1)]
    omega = np.zeros(l + 1)
    omega[l] = 1.0                                      # bicgstabl.c:39
    omega_d = np.zeros(l + 1)
    omega_dd = np.zeros(l + 1)
    sigma = np.zeros(l + 1)
    tau = np.zeros((l + 1) * (l + 1))
    r[0] = b - A @ x                                    # bicgstabl.c:45-49
    p[0] = r[0].copy()
    rs = r[0].copy()
    fnb = np.linalg.norm(b)
    alpha, gamma0 = 0.0, 1.0
    error, hist, m = 0.0, [], 0
    for m in range(max_iter):                           # bicgstabl.c:54
        gamma0 = -omega[l] * gamma0                     # bicgstabl.c:57
        for j in range(l):                              # BiCG part :59-80
            gamma1 = rs @ r[j]
            beta = -alpha * gamma1 / gamma0
            gamma0 = gamma1
            for i in range(j + 1):
                p[i] = beta * p[i] + r[i]               # :64-67
            p[j + 1] = A @ p[j]                         # :68
            alpha = gamma1 / (rs @ p[j + 1])            # :71
            for i in range(j + 1):
                r[i] = r[i] - alpha * p[i + 1]          # :73-75
            r[j + 1] = A @ r[j]                         # :76
            x += alpha * p[0]                           # :79
        for j in range(1, l + 1):                       # MR part :84-91
            for i in range(1, j):
                tau[i * l + j] = (r[j] @ r[i]) / sigma[i]
                r[j] = r[j] - tau[i * l + j] * r[i]
            sigma[j] = r[j] @ r[j]
            omega_d[j] = (r[0] @ r[j]) / sigma[j]
        omega[l] = omega_d[l]                           # :93
        for j in range(l - 1, 0, -1):                   # :95-101
            t = 0.0
            for i in range(j + 1, l + 1):
                t += tau[j * l + i] * omega[i]
            omega[j] = omega_d[j] - t
        for j in range(1, l):                           # :103-109
            t = 0.0
            for i in range(j + 1, l):
                t += tau[j * l + i] * omega[i + 1]
            omega_dd[j] = omega[j + 1] + t
        x += omega[1] * r[0]                            # update :113-120
        r[0] = r[0] - omega_d[l] * r[l]
        p[0] = p[0] - omega[l] * p[l]
        for i in range(1, l):
            p[0] = p[0] - omega[i] * p[i]
            r[0] = r[0] - omega_d[i] * r[i]
            x += omega_dd[i] * r[i]
        error = np.linalg.norm(r[0]) / fnb              # :122
        hist.append(error)
        if error < tol:
            break
    else:
        m = max_iter
    return _finish(error, tol, m), x, hist


def _myqr(V):
    """myqr, src/myqr.c:4-39: LAPACK dgeqrf + dorgqr, explicit thin Q and R."""
    Q, R = np.linalg.qr(V, mode="reduced")
    return Q, R


def blcg(A, B, tol, max_iter, X0=None, symmetric=True):
    """dblcg (Block CG, residual orthogonalised), src/blcg.c:15-119.

    Keeps the reference's initialisation: P = V and beta = I before the first
    direction update P = V + P beta^T (blcg.c:59-71), so the first direction
    block is 2V.
    """
    if not symmetric:
        return INVALID_MATRIX_TYPE, None, []
    m, s = B.shape
    X = np.zeros((m, s)) if X0 is None else X0.astype(float).copy()
    V = B - A @ X                                       # blcg.c:54-57
    V, C = _myqr(V)                                     # :58
    P = V.copy()
    fnb = np.linalg.norm(B)
    beta = np.eye(s)                                    # :61-63
    error, hist, i = 0.0, [], 0
    for i in range(max_iter):
        P = V + P @ beta.T                              # :68-71
        AP = A @ P                                      # :74
        alpha = np.linalg.inv(P.T @ AP)                 # :78-82
        X += P @ (alpha @ C)                            # :85-88
        V = V - AP @ alpha                              # :91-92
        V, beta = _myqr(V)                              # :95
        C = beta @ C                                    # :98-100
        error = np.linalg.norm(C) / fnb                 # :102
        hist.append(error)
        if error < tol:
            break
    else:
        i = max_iter
    return _finish(error, tol, i), X, hist


def blbicgstab(A, B, tol, max_iter, X0=None):
    """dblbicgstab (direction block orthogonalised), src/blbicgstab.c:13-123."""
    m, s = B.shape
    X = np.zeros((m, s)) if X0 is None else X0.astype(float).copy()
    R = B - A @ X                                       # :49-52
    P, Rs = R.copy(), R.copy()
    fnb = np.linalg.norm(B)
    error, hist, i = 0.0, [], 0
    for i in range(max_iter):
        V = A @ P                                       # :61
        G = Rs.T @ V                                    # :65
        alpha = np.linalg.solve(G, Rs.T @ R)            # :67-69
        R = R - V @ alpha                               # :72-73
        T = A @ R                                       # :76
        omega = np.vdot(T, R) / np.vdot(T, T)           # :80-81
        X += P @ alpha + omega * R                      # :84-86
        R = R - omega * T                               # :89
        beta = np.linalg.solve(G, -(Rs.T @ T))          # :92-94
        P = (P - omega * V) @ beta + R                  # :97-101
        P, _ = _myqr(P)                                 # :104
        error = np.linalg.norm(R) / fnb                 # :106
        hist.append(error)
        if error < tol:
            break
    else:
        i = max_iter
    return _finish(error, tol, i), X, hist


def blbicgstabl(A, B, l, tol, max_iter, X0=None):
    """dblbicgstabl (Block BiCGSTAB(l)-RH), src/blbicgstabl.c:16-252.

    Keeps the reference's start V0 = B + A X0 (blbicgstabl.c:83-86: the SpMM
    with alpha = -1 is followed by a further scaling by -1), which equals the
    residual only for X0 = 0.
    """
    m, s = B.shape
    X = np.zeros((m, s)) if X0 is None else X0.astype(float).copy()
    alpha = np.zeros((s, s))
    xi = np.zeros((s, s))
    gamma0 = np.eye(s)
    omega = np.zeros(l + 1)
    omega[l] = 1.0                                      # :38
    omega_d = np.zeros(l + 1)
    sigma = np.zeros(l + 1)
    tau = np.zeros((l + 1) * (l + 1))
    P = [np.zeros((m, s)) for _ in range(l + 1)]
    V = [np.zeros((m, s)) for _ in range(l + 1)]
    V[0] = B + A @ X                                    # :83-87
    V[0], xi = _myqr(V[0])                              # :88
    P[0] = V[0].copy()
    Rs = V[0].copy()
    fnb = np.linalg.norm(B)
    t = np.zeros((s, s))
    error, hist, it = 0.0, [], 0
    for it in range(max_iter):
        gamma0 = -omega[l] * gamma0                     # :98
        for j in range(l):
            gamma1 = Rs.T @ V[j]                        # :102-103
            beta = -alpha @ np.linalg.solve(gamma0, gamma1)   # :104-107
            gamma0 = gamma1.copy()
            for i in range(j + 1):
                P[i] = P[i] @ beta + V[i]               # :111-116
            P[j + 1] = A @ P[j]                         # :117
            alpha = np.linalg.solve(Rs.T @ P[j + 1], gamma1)  # :121-124
            for i in range(j + 1):
                if i == 0:
                    tmp = P[0] @ alpha                  # :129-130
                    V[0] = V[0] - A @ tmp               # :131-132
                    V[0], t = _myqr(V[0])               # :135
                    X += tmp @ xi                       # :138-139
                    xi = t @ xi                         # :142-144
                    t = np.linalg.inv(t)                # :147-148
                else:
                    V[i] = (V[i] - P[i + 1] @ alpha) @ t   # :151-155
            V[j + 1] = A @ V[j]                         # :159
        R = [V[i] @ xi for i in range(l + 1)]           # :163-166
        for j in range(1, l + 1):                       # MR part :170-178
            for i in range(1, j):
                tau[i * l + j] = np.vdot(R[j], R[i]) / sigma[i]
                R[j] = R[j] - tau[i * l + j] * R[i]
            sigma[j] = np.vdot(R[j], R[j])
            omega_d[j] = np.vdot(R[0], R[j]) / sigma[j]
        omega[l] = omega_d[l]
        for j in range(l - 1, 0, -1):                   # :181-187
            tl = 0.0
            for i in range(j + 1, l + 1):
                tl += tau[j * l + i] * omega[i]
            omega[j] = omega_d[j] - tl
        tmp = np.zeros((m, s))                          # update :198-207
        for i in range(1, l + 1):
            tmp += omega[i] * V[i - 1]
            P[0] = P[0] - omega[i] * P[i]
        V[0] = V[0] - A @ tmp
        X += tmp @ xi
        error = np.linalg.norm(xi) / fnb                # :209
        hist.append(error)
        if error < tol or math.isnan(error):
            break
    else:
        it = max_iter
    return _finish(error, tol, it), X, hist


def shbicg(A, b, sigma, tol, max_iter, x0=None):
    """dshbicg (shifted BiCG), src/shbicg.c:5-129.  x has n*(nsigma+1)."""
    n = b.size
    ns = len(sigma)
    AT = sp.csr_matrix(A.T)
    x = np.zeros(n * (ns + 1)) if x0 is None else x0.astype(float).copy()
    xs = x[:n]
    r = b - A @ xs                                      # :21-25
    sr = r.copy()
    p = np.zeros(n)
    s_p = np.zeros(n)
    fnb = np.linalg.norm(b)
    alpha_old, rho_old = 1.0, 1.0
    pi = np.ones(ns)
    pi_old = np.ones(ns)
    p_sh = np.zeros((ns, n))
    error, hist, i = 0.0, [], 0
    for i in range(max_iter):
        rho = r @ sr                                    # :52
        beta = -rho / rho_old
        p = -beta * p + r                               # :56-57
        s_p = -beta * s_p + sr                          # :60-61
        ap = A @ p
        atp = AT @ s_p
        alpha = rho / (ap @ sr)                         # :72
        xs += alpha * p
        pi_new = np.empty(ns)
        for k in range(ns):                             # :78-96
            pi_new[k] = ((1 + alpha * sigma[k]) * pi[k]
                         + alpha * beta / alpha_old * (pi_old[k] - pi[k]))
            beta_sh = (pi_old[k] / pi[k]) * (pi_old[k] / pi[k]) * beta
            alpha_sh = pi[k] / pi_new[k] * alpha
            p_sh[k] = -beta_sh * p_sh[k] + (1.0 / pi[k]) * r
            x[(k + 1) * n:(k + 2) * n] += alpha_sh * p_sh[k]
        r = r - alpha * ap
        sr = sr - alpha * atp
        alpha_old = alpha
        rho_old = rho
        pi_old = pi.copy()
        pi = pi_new
        error = np.linalg.norm(r) / fnb
        hist.append(error)
        if error < tol:
            break
    else:
        i = max_iter
    return _finish(error, tol, i), x, hist


def horner(omega, l, sigma):
    """dhorner, src/util_shift.c:5-27."""
    out = np.zeros(l + 1)
    out[l] = -omega[l - 1]
    for i in range(l - 1, 0, -1):
        out[i] = -sigma * out[i + 1] - omega[i - 1]
    out[0] = -sigma * out[1] + 1.0
    for i in range(1, l):
        for j in range(l - 1, i - 1, -1):
            out[j] += -sigma * out[j + 1]
    for i in range(1, l + 1):
        out[i] = -out[i] / out[0]
    return out


def comb(n, r):
    """comb, src/util_shift.c:55-63 (binomial coefficient)."""
    if n < 0 or r < 0 or n < r:
        return 0
    return math.comb(n, r)


def shbicgstabl(A, b, l, sigma, tol, max_iter, x0=None):
    """dshbicgstabl (shifted BiCGSTAB(l)), src/shbicgstabl.c:7-285."""
    n = b.size
    ns = len(sigma)
    x = np.zeros(n * (ns + 1)) if x0 is None else x0.astype(float).copy()
    xs = x[:n]
    r = [np.zeros(n) for _ in range(l + 1)]
    p = [np.zeros(n) for _ in range(l + 1)]
    omega = np.zeros(l)
    omega[l - 1] = 1.0                                  # :25
    omega_d = np.zeros(l)
    omega_dd = np.zeros(l)
    s = np.zeros(l)
    tau = np.zeros(l * l)
    r[0] = b - A @ xs                                   # :32-36
    p[0] = r[0].copy()
    rs = r[0].copy()
    norm_b = np.linalg.norm(b)
    alpha, alpha_old, rho_old = 0.0, 1.0, 1.0
    pi = np.ones(ns)
    pi_old = np.ones(ns)
    theta = np.ones(ns)
    p_sh = np.zeros((ns, l + 1, n))
    M = np.zeros((ns, l * l))                           # :70-81
    for k in range(ns):
        for j in range(l):
            for i in range(j + 1):
                M[k, j * l + i] = sigma[k] ** (j - i) * comb(j, i)
    alpha_sh = np.zeros(ns)
    error, hist, it = 0.0, [], 0
    for it in range(max_iter):
        rho_old = -omega[l - 1] * rho_old               # :88
        for j in range(l):
            rho = r[j] @ rs                             # :91
            beta = alpha * rho / rho_old
            for i in range(j + 1):
                p[i] = -beta * p[i] + r[i]              # :95-98
            p[j + 1] = A @ p[j]                         # :101
            alpha = rho / (rs @ p[j + 1])               # :105
            xs += alpha * p[0]                          # :108
            pi_new = np.empty(ns)
            for k in range(ns):                         # :111-134
                pi_new[k] = ((1.0 + alpha * sigma[k]) * pi[k]
                             + alpha * beta / alpha_old * (pi_old[k] - pi[k]))
                beta_sh = (pi_old[k] / pi[k]) * (pi_old[k] / pi[k]) * beta
                alpha_sh[k] = pi[k] / pi_new[k] * alpha
                for i in range(j + 1):
                    p_sh[k, i] = (-beta_sh * p_sh[k, i]
                                  + (1.0 / (pi[k] * theta[k])) * r[i])
                p_sh[k, j + 1] = r[j] * (1.0 / pi[k])   # :129-130
                x[(k + 1) * n:(k + 2) * n] += alpha_sh[k] * p_sh[k, 0]
            for i in range(j + 1):
                r[i] = r[i] - alpha * p[i + 1]          # :137-139
            r[j + 1] = A @ r[j]                         # :142
            for k in range(ns):                         # :146-153
                v = p_sh[k, j + 1] + (-1.0 / pi_new[k]) * r[j]
                v = v * (1.0 / (theta[k] * alpha_sh[k]))
                p_sh[k, j + 1] = v - sigma[k] * p_sh[k, j]
            alpha_old = alpha
            rho_old = rho
            pi_old = pi.copy()
            pi = pi_new
        for j in range(l):                              # MR part :166-173
            for i in range(j):
                tau[i * l + j] = (r[j + 1] @ r[i + 1]) / s[i]
                r[j + 1] = r[j + 1] - tau[i * l + j] * r[i + 1]
            s[j] = r[j + 1] @ r[j + 1]
            omega_d[j] = (r[0] @ r[j + 1]) / s[j]
        omega[l - 1] = omega_d[l - 1]
        for j in range(l - 2, -1, -1):                  # :177-183
            tl = 0.0
            for i in range(j + 1, l):
                tl += tau[j * l + i] * omega[i]
            omega[j] = omega_d[j] - tl
        for j in range(l - 1):                          # :185-191
            tl = 0.0
            for i in range(j + 1, l - 1):
                tl += tau[j * l + i] * omega[i + 1]
            omega_dd[j] = omega[j + 1] + tl
        xs += omega[0] * r[0]                           # :194-199
        p[0] = p[0] - omega[l - 1] * p[l]
        for i in range(1, l):
            p[0] = p[0] - omega[i - 1] * p[i]
            xs += omega_dd[i - 1] * r[i]
        for k in range(ns):                             # :202-237
            h = horner(omega, l, sigma[k])
            psi = h[0]
            om_sh = h[1:]
            e_sh = theta[k] * pi[k]
            theta[k] = theta[k] * psi
            om_sh_d = np.zeros(l)
            for j in range(l):
                acc = 0.0
                for i in range(j, l):
                    acc += M[k, i * l + j] * om_sh[i]
                om_sh_d[j] = acc
            om_sh_dd = np.zeros(l)
            for j in range(l - 1):
                acc = 0.0
                for i in range(j + 1, l - 1):
                    acc += tau[j * l + i] * om_sh_d[i + 1]
                om_sh_dd[j] = om_sh_d[j + 1] + acc
            xk = x[(k + 1) * n:(k + 2) * n]
            xk += (om_sh_d[0] / e_sh) * r[0]
            p_sh[k, 0] = p_sh[k, 0] - omega[l - 1] * p_sh[k, l]
            for i in range(1, l):
                p_sh[k, 0] = p_sh[k, 0] - omega[i - 1] * p_sh[k, i]
                xk += (om_sh_dd[i - 1] / e_sh) * r[i]
            p_sh[k, 0] = p_sh[k, 0] * (1.0 / psi)
        for i in range(1, l + 1):                       # :240-242
            r[0] = r[0] - omega_d[i - 1] * r[i]
        error = np.linalg.norm(r[0]) / norm_b
        hist.append(error)
        if error < tol:
            break
    else:
        it = max_iter
    return _finish(error, tol, it), x, hist


def true_residual(A, b, x, sigma=0.0):
    """||b - (A + sigma I) x|| / ||b|| (tests/test.c:8-49)."""
    return float(np.linalg.norm(b - A @ x - sigma * x) / np.linalg.norm(b))
