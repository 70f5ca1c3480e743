"""NumPy FP64 restatement of the learned SPAI preconditioner's model --
TEST INFRASTRUCTURE ONLY (the checker of the GPU forward / backward
kernels).  The learned preconditioner has no reference counterpart; this is
the mathematics the kernels implement:

* slots: the operator's distinct diagonal offsets, the diagonal in slot 3,
  negative offsets in slots 2, 1, 0 (nearest first), positive ones in
  slots 4..7 (nearest first);
* features f_i[s] = a_{i,j_s} / a_ii, except f_i[3] = (sum_j a_ij) / a_ii;
* MLP o = W3 relu(W2 relu(W1 f + b1) + b2) + b3, m_{i,j_s} = o_s / a_ii;
* loss L = ||Z - M (A Z)||_F^2 / (n * probes)  (= ||(I - M A) Z||_F^2 scaled).

Parameters are one flat vector: W1[64][8], b1[64], W2[64][64], b2[64],
W3[8][64], b3[8].
"""
import numpy as np

S, H, C = 8, 64, 3


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * S].reshape(H, S); o += H * S
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + S * H].reshape(S, H); o += S * H
    b3 = p[o:o + S]; o += S
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def slots(rowptr, col, n):
    """(n, 8) CSR entry index of each slot (-1 absent), or None."""
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    off = col.astype(np.int64) - rows
    u = np.unique(off)
    if u.size > S or 0 not in u:
        return None
    neg = sorted([x for x in u if x < 0], reverse=True)
    pos = sorted([x for x in u if x > 0])
    if len(neg) > C or len(pos) > S - 1 - C:
        return None
    m = {0: C}
    m.update({o_: C - 1 - r for r, o_ in enumerate(neg)})
    m.update({o_: C + 1 + r for r, o_ in enumerate(pos)})
    se = -np.ones((n, S), dtype=np.int64)
    for k in range(col.size - 1, -1, -1):     # first entry of a slot wins
        se[rows[k], m[off[k]]] = k
    return se


def features(rowptr, col, val, n):
    se = slots(rowptr, col, n)
    d = val[se[:, C]]
    di = np.where(d != 0, 1.0 / d, 0.0)
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    rowsum = np.bincount(rows, weights=val, minlength=n)
    f = np.where(se >= 0, val[np.maximum(se, 0)] * di[:, None], 0.0)
    f[:, C] = rowsum * di
    return se, f, di


def loss_grad(p, rowptr, col, val, n, Z, AZ):
    """Loss and gradient of the flat parameter vector p (FP64).

    Z, AZ: (probes, n) arrays.  Follows the GPU kernel's conventions."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    se, f, di = features(rowptr, col, val, n)
    z1 = f @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    o = h2 @ W3.T + b3
    present = se >= 0
    cj = np.where(present, col[np.maximum(se, 0)], 0)
    m = np.where(present, o * di[:, None], 0.0)
    k = Z.shape[0]
    scale = 1.0 / (n * k)
    Wg = AZ[:, cj] * present[None, :, :]          # (k, n, S)
    R = Z - np.einsum("ns,kns->kn", m, Wg)         # (k, n)
    loss = scale * np.sum(R * R)
    dm = -2.0 * np.einsum("kn,kns->ns", R, Wg)
    dout = np.where(present, dm * di[:, None], 0.0) * scale
    gW3 = dout.T @ h2
    gb3 = dout.sum(0)
    dh2 = (dout @ W3) * (z2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (z1 > 0)
    gW1 = dh1.T @ f
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def spai_values(p, rowptr, col, val, n):
    """M's values on A's pattern for parameters p."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    se, f, di = features(rowptr, col, val, n)
    h1 = np.maximum(f @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    o = h2 @ W3.T + b3
    mv = np.zeros(col.size)
    present = se >= 0
    mv[se[present]] = (o * di[:, None])[present]
    return mv
