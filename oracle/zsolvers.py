"""NumPy complex128 restatement of the reference's complex Krylov solvers.

TEST INFRASTRUCTURE ONLY: this is the checker, never the product path.

Each function follows one reference routine statement by statement (cited
by file:line of aldente39/bksp) and returns ``(ret, x, hist)`` with the
conventions of ``oracle/solvers.py``: ``ret`` the 0-based index of the
iteration whose convergence test passed or -1, ``x`` the solution (n-by-s
``X`` for the block method; for the shifted method ``x[(k+1)n:(k+2)n]``
solves ``(A + sigma_k I) x = b``), ``hist`` the value compared with ``tol``
at each iteration.

Conventions of the reference's complex kernels, kept here:

* ``cblas_zdotc_sub(n, x, 1, y, 1, &d)`` is ``d = sum conj(x_i) y_i``
  (``np.vdot(x, y)``);
* ``zcsrgemm0`` 't' multiplies by the CONJUGATE transpose
  (src/matvec.c:74-90: ``conj(A[k]) * B[j]``), so zbicg's shadow product is
  ``A^H sp``;
* the block method's Gram products are ``cblas_zgemm(CblasTrans, ...)``:
  plain transposes, ``Rs^T V`` (src/blbicgstabl.c:343-344, 363-364);
* ``zqreco`` is LAPACK ``zgeqrf`` + ``zungqr`` (src/myqr.c:41-76), as
  ``np.linalg.qr``.

One departure: zbicgstabl declares its unit coefficient as a real
``double one = 1`` (src/bicgstabl.c:147) and passes its address where
``cblas_zaxpy`` reads a complex scalar (:178, :196), so the imaginary part of
that coefficient is whatever 8 bytes follow ``one`` on the stack.  The
restatement uses the intended coefficient 1 + 0i; the golden fixtures pin
the compiled reference only where its result agrees with it.

Kept as the reference computes it: zblbicgstabl accumulates the MR
back-substitution sum in a real ``double t_local`` (src/blbicgstabl.c:259,
:426-430), so only the real parts of tau_ij omega_i enter omega_j.
"""
import math

import numpy as np

NOT_CONVERGED = -1


def _finish(error, tol, idx):
    return NOT_CONVERGED if error >= tol else idx


def zbicg(A, b, tol, max_iter, x0=None):
    """zbicg, src/bicg.c:91-177 (A: SciPy CSR, complex)."""
    n = b.size
    x = np.zeros(n, complex) if x0 is None else x0.astype(complex).copy()
    AH = A.conj().T.tocsr()
    tmp = b - A @ x                                     # bicg.c:108-111
    r = tmp.copy()                                      # :112
    sr = tmp.copy()                                     # :113
    p = r.copy()                                        # :114
    sp = sr.copy()                                      # :115
    r_dot_old = np.vdot(sr, r)                          # :116
    norm_b = np.linalg.norm(b)                          # :117
    error, hist, i = 0.0, [], 0
    for i in range(max_iter):                           # :120
        ap = A @ p                                      # :122-123
        atp = AH @ sp                                   # :126-127 ('t' = A^H)
        alpha = r_dot_old / np.vdot(sp, ap)             # :130-131
        x += alpha * p                                  # :136
        r = r - alpha * ap                              # :139
        sr = sr - np.conj(alpha) * atp                  # :142
        r_dot = np.vdot(sr, r)                          # :145
        beta = r_dot / r_dot_old                        # :146
        r_dot_old = r_dot                               # :148
        p = beta * p + r                                # :151-152
        sp = np.conj(beta) * sp + sr                    # :155-156
        error = np.linalg.norm(r) / norm_b              # :158
        hist.append(error)
        if error < tol:
            break
    else:
        i = max_iter
    return _finish(error, tol, i), x, hist


def zbicgstabl(A, b, l, tol, max_iter, x0=None):
    """zbicgstabl, src/bicgstabl.c:141-276 (unit coefficient 1 + 0i)."""
    n = b.size
    x = np.zeros(n, complex) if x0 is None else x0.astype(complex).copy()
    r = [np.zeros(n, complex) for _ in range(l + 1)]
    p = [np.zeros(n, complex) for _ in range(l + 1)]
    omega = np.zeros(l + 1, complex)
    omega[l] = 1.0                                      # :169
    omega_d = np.zeros(l + 1, complex)
    omega_dd = np.zeros(l + 1, complex)
    sigma = np.zeros(l + 1, complex)
    tau = np.zeros((l + 1) * (l + 1), complex)
    r[0] = b - A @ x                                    # :175-179
    p[0] = r[0].copy()                                  # :180
    rs = r[0].copy()                                    # :181
    fnb = np.linalg.norm(b)                             # :182
    alpha, gamma0 = 0j, 1 + 0j                          # :150-151
    error, hist, m = 0.0, [], 0
    for m in range(max_iter):                           # :185
        gamma0 = -omega[l] * gamma0                     # :187
        for j in range(l):                              # BiCG part :189-212
            gamma1 = np.vdot(rs, r[j])                  # :190
            beta = -alpha * gamma1 / gamma0             # :191
            gamma0 = gamma1                             # :192
            for i in range(j + 1):                      # :194-197
                p[i] = beta * p[i] + r[i]
            p[j + 1] = A @ p[j]                         # :198-199
            alpha = gamma1 / np.vdot(rs, p[j + 1])      # :201-202
            for i in range(j + 1):                      # :204-207
                r[i] = r[i] - alpha * p[i + 1]
            r[j + 1] = A @ r[j]                         # :208-209
            x += alpha * p[0]                           # :211
        for j in range(1, l + 1):                       # MR part :216-226
            for i in range(1, j):
                tau[j * l + i] = np.vdot(r[i], r[j]) / sigma[i]
                r[j] = r[j] - tau[j * l + i] * r[i]
            sigma[j] = np.vdot(r[j], r[j])              # :223
            omega_d[j] = np.vdot(r[j], r[0]) / sigma[j]  # :224-225
        omega[l] = omega_d[l]                           # :228
        for j in range(l - 1, 0, -1):                   # :230-236
            t = 0j
            for i in range(j + 1, l + 1):
                t += tau[i * l + j] * omega[i]
            omega[j] = omega_d[j] - t
        for j in range(1, l):                           # :238-244
            t = 0j
            for i in range(j + 1, l):
                t += tau[i * l + j] * omega[i + 1]
            omega_dd[j] = omega[j + 1] + t
        x += omega[1] * r[0]                            # update :247-258
        r[0] = r[0] - omega_d[l] * r[l]
        p[0] = p[0] - omega[l] * p[l]
        for i in range(1, l):
            p[0] = p[0] - omega[i] * p[i]
            r[0] = r[0] - omega_d[i] * r[i]
            x += omega_dd[i] * r[i]
        error = np.linalg.norm(r[0]) / fnb              # :260
        hist.append(error)
        if error < tol:
            break
    else:
        m = max_iter
    return _finish(error, tol, m), x, hist


def zqreco(V):
    """zqreco, src/myqr.c:41-76: LAPACK zgeqrf + zungqr, thin Q and R."""
    Q, R = np.linalg.qr(V, mode="reduced")
    return Q, R


def zblbicgstabl(A, B, l, tol, max_iter, X0=None):
    """zblbicgstabl (complex Block BiCGSTAB(l)), src/blbicgstabl.c:255-486.

    Keeps the reference's start V0 = B + A X0 (:321-324: the SpMM with
    alpha = -1 followed by a scaling by -1), the residual only for X0 = 0.
    """
    m, s = B.shape
    X = np.zeros((m, s), complex) if X0 is None else X0.astype(complex).copy()
    alpha = np.zeros((s, s), complex)
    gamma0 = np.eye(s, dtype=complex)                   # :287-289
    omega = np.zeros(l, complex)
    omega[l - 1] = 1.0                                  # :279
    omega_d = np.zeros(l, complex)
    sigma = np.zeros(l, complex)
    tau = np.zeros(l * l, complex)
    P = [np.zeros((m, s), complex) for _ in range(l + 1)]
    V = [np.zeros((m, s), complex) for _ in range(l + 1)]
    V[0] = B + A @ X                                    # :321-325
    V[0], xi = zqreco(V[0])                             # :326
    P[0] = V[0].copy()                                  # :327
    Rs = V[0].copy()                                    # :328
    fnb = np.linalg.norm(B)                             # :333
    t = np.zeros((s, s), complex)
    error, hist, it = 0.0, [], 0
    for it in range(max_iter):                          # :336
        gamma0 = -omega[l - 1] * gamma0                 # :338-339
        for j in range(l):
            gamma1 = Rs.T @ V[j]                        # :343-344
            beta = alpha @ np.linalg.solve(gamma0, gamma1)   # :345-348
            gamma0 = gamma1.copy()                      # :349
            for i in range(j + 1):                      # :352-357
                P[i] = V[i] - P[i] @ beta
            P[j + 1] = A @ P[j]                         # :358-359
            alpha = np.linalg.solve(Rs.T @ P[j + 1], gamma1)  # :362-365
            for i in range(j + 1):
                if i == 0:
                    tmp = P[0] @ alpha                  # :370-371
                    V[0] = V[0] - A @ tmp               # :372-373
                    V[0], t = zqreco(V[0])              # :376
                    X += tmp @ xi                       # :379-381
                    xi = t @ xi                         # :384-386
                    t = np.linalg.inv(t)                # :389-390
                else:
                    V[i] = (V[i] - P[i + 1] @ alpha) @ t   # :393-397
            V[j + 1] = A @ V[j]                         # :401-402
        R = [V[i] @ xi for i in range(l + 1)]           # :405-408
        for j in range(l):                              # MR part :412-422
            for i in range(j):
                tau[j * l + i] = np.vdot(R[i + 1], R[j + 1]) / sigma[i]
                R[j + 1] = R[j + 1] - tau[j * l + i] * R[i + 1]
            sigma[j] = np.vdot(R[j + 1], R[j + 1])      # :419
            omega_d[j] = np.vdot(R[j + 1], R[0]) / sigma[j]   # :420-421
        omega[l - 1] = omega_d[l - 1]                   # :423
        for j in range(l - 2, -1, -1):                  # :425-431
            # t_local is a real double (:259), so each complex product
            # adds only its real part (C's complex -> real conversion).
            tl = 0.0
            for i in range(j + 1, l):
                tl = (tl + tau[i * l + j] * omega[i]).real
            omega[j] = omega_d[j] - tl
        tmp = np.zeros((m, s), complex)                 # update :442-452
        for i in range(l):
            tmp += omega[i] * V[i]
            P[0] = P[0] - omega[i] * P[i + 1]
        V[0] = V[0] - A @ tmp
        X += tmp @ xi
        error = np.linalg.norm(xi) / fnb                # :454
        hist.append(error)
        if error < tol or math.isnan(error):
            break
    else:
        it = max_iter
    return _finish(error, tol, it), X, hist


def zhorner(omega, l, sigma):
    """zhorner, src/util_shift.c:28-50."""
    out = np.zeros(l + 1, complex)
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


def zshbicgstabl(A, b, l, sigma, tol, max_iter, x0=None):
    """zshbicgstabl (complex shifted BiCGSTAB(l)), src/shbicgstabl.c:288-592.

    ``x0`` is the caller's x: the seed's initial guess in its first n
    entries, then each shifted system's (:362 points the shifted solutions
    into the caller's array and adds to them; any missing tail is zero)."""
    n = b.size
    ns = len(sigma)
    sigma = np.asarray(sigma, complex)
    x = np.zeros(n * (ns + 1), complex)
    if x0 is not None:
        x[:x0.size] = x0
    xs = x[:n]
    r = [np.zeros(n, complex) for _ in range(l + 1)]
    p = [np.zeros(n, complex) for _ in range(l + 1)]
    omega = np.zeros(l, complex)
    omega[l - 1] = 1.0                                  # :316
    omega_d = np.zeros(l, complex)
    omega_dd = np.zeros(l, complex)
    s_ = np.zeros(l, complex)
    tau = np.zeros(l * l, complex)
    r[0] = b - A @ xs                                   # :322-326
    p[0] = r[0].copy()
    rs = r[0].copy()
    norm_b = np.linalg.norm(b)                          # :329
    alpha, alpha_old, rho_old = 0j, 1 + 0j, 1 + 0j      # :330-332
    pi = np.ones(ns, complex)                           # :361-367
    pi_old = np.ones(ns, complex)
    theta = np.ones(ns, complex)
    pi_new = np.zeros(ns, complex)
    alpha_s = np.zeros(ns, complex)
    ps = [[np.zeros(n, complex) for _ in range(l + 1)] for _ in range(ns)]
    M = np.zeros((ns, l * l), complex)                  # :378-384
    for k in range(ns):
        for j in range(l):
            for i in range(j + 1):
                M[k, j * l + i] = sigma[k] ** (j - i) * math.comb(j, i)
    error, hist, it = 0.0, [], 0
    for it in range(max_iter):                          # :388
        rho_old = -omega[l - 1] * rho_old               # :391
        for j in range(l):
            rho = np.vdot(rs, r[j])                     # :394
            beta = alpha * rho / rho_old                # :395
            for i in range(j + 1):                      # :398-402
                p[i] = -beta * p[i] + r[i]
            p[j + 1] = A @ p[j]                         # :405-406
            alpha = rho / np.vdot(rs, p[j + 1])         # :409-410
            xs += alpha * p[0]                          # :413
            for k in range(ns):                         # :416-442
                pi_new[k] = ((1.0 + alpha * sigma[k]) * pi[k]
                             + alpha * beta / alpha_old * (pi_old[k] - pi[k]))
                beta_s = (pi_old[k] / pi[k]) * (pi_old[k] / pi[k]) * beta
                alpha_s[k] = pi[k] / pi_new[k] * alpha
                for i in range(j + 1):
                    ps[k][i] = (-beta_s * ps[k][i]
                                + (1.0 / (pi[k] * theta[k])) * r[i])
                ps[k][j + 1] = (1.0 / pi[k]) * r[j]
                x[(k + 1) * n:(k + 2) * n] += alpha_s[k] * ps[k][0]
            for i in range(j + 1):                      # :445-448
                r[i] = r[i] - alpha * p[i + 1]
            r[j + 1] = A @ r[j]                         # :451-452
            for k in range(ns):                         # :455-463
                ps[k][j + 1] = ps[k][j + 1] - (1.0 / pi_new[k]) * r[j]
                ps[k][j + 1] = (1.0 / (theta[k] * alpha_s[k])) * ps[k][j + 1]
                ps[k][j + 1] = ps[k][j + 1] - sigma[k] * ps[k][j]
            alpha_old = alpha                           # :466-471
            rho_old = rho
            pi_old = pi.copy()
            pi = pi_new.copy()
        for j in range(l):                              # MR part :477-487
            for i in range(j):
                tau[j * l + i] = np.vdot(r[i + 1], r[j + 1]) / s_[i]
                r[j + 1] = r[j + 1] - tau[j * l + i] * r[i + 1]
            s_[j] = np.vdot(r[j + 1], r[j + 1])
            omega_d[j] = np.vdot(r[j + 1], r[0]) / s_[j]
        omega[l - 1] = omega_d[l - 1]                   # :489
        for j in range(l - 2, -1, -1):                  # :491-497
            t = 0j
            for i in range(j + 1, l):
                t += tau[i * l + j] * omega[i]
            omega[j] = omega_d[j] - t
        for j in range(l - 1):                          # :499-505
            t = 0j
            for i in range(j + 1, l - 1):
                t += tau[i * l + j] * omega[i + 1]
            omega_dd[j] = omega[j + 1] + t
        xs += omega[0] * r[0]                           # :508-515
        p[0] = p[0] - omega[l - 1] * p[l]
        for i in range(1, l):
            p[0] = p[0] - omega[i - 1] * p[i]
            xs += omega_dd[i - 1] * r[i]
        for k in range(ns):                             # :518-557
            h = zhorner(omega, l, sigma[k])
            psi = h[0]
            om_s = h[1:l + 1]
            e = theta[k] * pi[k]
            theta[k] = theta[k] * psi
            om_sd = np.zeros(l, complex)
            for j in range(l):
                acc = 0j
                for i in range(j, l):
                    acc += M[k, i * l + j] * om_s[i]
                om_sd[j] = acc
            om_sdd = np.zeros(l, complex)
            for j in range(l - 1):
                acc = 0j
                for i in range(j + 1, l - 1):
                    acc += tau[i * l + j] * om_sd[i + 1]
                om_sdd[j] = om_sd[j + 1] + acc
            xk = x[(k + 1) * n:(k + 2) * n]
            xk += (om_sd[0] / e) * r[0]
            ps[k][0] = ps[k][0] - omega[l - 1] * ps[k][l]
            for i in range(1, l):
                ps[k][0] = ps[k][0] - omega[i - 1] * ps[k][i]
                xk += (om_sdd[i - 1] / e) * r[i]
            ps[k][0] = (1.0 / psi) * ps[k][0]
        for i in range(1, l + 1):                       # :560-563
            r[0] = r[0] - omega_d[i - 1] * r[i]
        error = np.linalg.norm(r[0]) / norm_b           # :565
        hist.append(error)
        if error < tol:
            break
    else:
        it = max_iter
    return _finish(error, tol, it), x, hist


def true_residual(A, b, x, sigma=0.0):
    """||b - (A + sigma I) x|| / ||b|| in complex128."""
    return float(np.linalg.norm(b - A @ x - sigma * x) / np.linalg.norm(b))
