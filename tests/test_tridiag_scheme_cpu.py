"""The exchange scheme of libgwb's cluster and grid tridiagonalisation
kernels (``k_sytrd_cluster``, ``k_sytrd_grid`` in ``csrc/tridiag.cu``),
restated in numpy on the CPU with the kernels' data layout: CTA c keeps the
rows c, c + G, ...; per column every CTA forms w of the previous reflector,
the column and the reflector from the gathered (p, raw) pairs; the pass over
its rows fuses the previous reflector's rank-2 update with the current
product; the gathered values are double-buffered by the parity of the
column. A part of the columns reduced this way and written back (the grid
kernel's hand-off), then the rest (the cluster kernel), must give
Q^T A Q = T with Q from the stored reflectors.

The CTAs run one after another here. That is how an earlier form of the grid
kernel showed its fault on the CPU: it read column 0 from global memory in
the first column's step while CTA 0 already wrote the reflector into it; the
kernels read column 0 before any CTA writes.
"""

import numpy as np
import pytest


def _reflector(col, j):
    alpha = col[j + 1]
    s = float(np.sum(col[j + 2:] ** 2))
    tau, beta, scl = 0.0, alpha, 0.0
    if s > 0.0:
        beta = -np.copysign(np.sqrt(alpha * alpha + s), alpha)
        tau = (beta - alpha) / beta
        scl = 1.0 / (alpha - beta)
    return tau, beta, scl


def _reduce(A, t0, t1, G, late_col0=False):
    """Columns t0 .. t1 - 1 of A (full, symmetric, up to date from t0 on) by
    the scheme with G CTAs; the reflector vectors go below the subdiagonal of
    their columns, and the trailing part at t1 is written back brought up to
    date (when t1 < m - 1). ``late_col0`` plants a fault: each CTA takes
    column 0 from the matrix in the first column's step, after CTA 0 may
    have stored reflector 0 there. Returns d, e, tau of those columns."""
    m = A.shape[0]
    n, ncols = m - t0, t1 - t0
    T = A[t0:, t0:]
    nl = (n + G - 1) // G
    rows = [np.array([T[:, c + li * G] if c + li * G < n else np.zeros(n) for li in range(nl)]) for c in range(G)]
    col0 = T[:, 0].copy()  # read before any CTA writes reflector 0 into it
    v = [np.zeros((2, n)) for _ in range(G)]
    w = [np.zeros(n) for _ in range(G)]
    pr = np.zeros((2, n, 2))
    part = np.zeros((2, G))
    d, e, tau_out = np.zeros(m), np.zeros(m), np.zeros(m)
    tau_prev = 0.0
    for j in range(ncols):
        q, qp = j & 1, (j & 1) ^ 1
        taus = []
        for c in range(G):  # R(j), the same in every CTA
            vj, vq = v[c][q], v[c][qp]
            if j > 0:
                K = part[qp].sum() * 0.5 * tau_prev
                wj = pr[qp, j, 0] - K * vq[j]
                w[c][j:] = pr[qp, j:, 0] - K * vq[j:]
                col = np.zeros(n)
                col[j:] = pr[qp, j:, 1] - vq[j:] * wj - w[c][j:] * vq[j]
            else:
                col = T[:, 0].copy() if late_col0 else col0
            tau, beta, scl = _reflector(col, j)
            vj[j + 1] = 1.0
            vj[j + 2:] = col[j + 2:] * scl
            taus.append(tau)
            if c == 0:
                T[j + 2:, j] = vj[j + 2:]
                d[t0 + j], e[t0 + j], tau_out[t0 + j] = col[j], beta, tau
        kb = j + 1
        new_pr, new_part = np.zeros((n, 2)), np.zeros(G)
        for c in range(G):  # F(j)
            vj, vq = v[c][q], v[c][qp]
            for li in range(nl):
                i = c + li * G
                if i < kb or i >= n:
                    continue
                row = rows[c][li]
                if j > 0:
                    row[kb:] -= vq[i] * w[c][kb:] + w[c][i] * vq[kb:]
                new_pr[i, 1] = row[kb]
                p = taus[c] * float(np.dot(row[kb:], vj[kb:]))
                new_pr[i, 0] = p
                new_part[c] += p * vj[i]
        pr[q], part[q] = new_pr, new_part
        tau_prev = taus[0]
    J = ncols
    qp = (J - 1) & 1
    K = part[qp].sum() * 0.5 * tau_prev
    if J >= n - 1:  # to the end: the last diagonal element
        vq = v[0][qp]
        wl = pr[qp, n - 1, 0] - K * vq[n - 1]
        d[t0 + n - 1] = pr[qp, n - 1, 1] - 2.0 * vq[n - 1] * wl
        return d, e, tau_out
    for c in range(G):  # write-back of the trailing part at J
        vq = v[c][qp]
        wv = np.zeros(n)
        wv[J:] = pr[qp, J:, 0] - K * vq[J:]
        for li in range(nl):
            i = c + li * G
            if J <= i < n:
                T[J:, i] = rows[c][li][J:] - vq[i] * wv[J:] - wv[i] * vq[J:]
    return d, e, tau_out


def _q_of(A, tau):
    m = A.shape[0]
    Q = np.eye(m)
    for j in range(m - 1):
        v = np.zeros(m)
        v[j + 1] = 1.0
        v[j + 2:] = A[j + 2:, j]
        Q -= tau[j] * np.outer(Q @ v, v)
    return Q


@pytest.mark.parametrize("m,split,G1,G2", [(2, 0, 4, 4), (3, 0, 4, 4), (17, 0, 16, 16), (60, 20, 7, 4),
                                           (120, 37, 13, 8), (90, 0, 5, 16)])
def test_exchange_scheme_tridiagonalises(m, split, G1, G2):
    """Columns [0, split) with G1 CTAs and a write-back, then the rest with
    G2 CTAs: Q^T A Q = T and Q orthogonal to round-off."""
    rng = np.random.default_rng(m)
    a = rng.standard_normal((m, m))
    a = 0.5 * (a + a.T) + np.diag(np.linspace(-5.0, 80.0, m))
    A = a.copy()
    d, e, tau = np.zeros(m), np.zeros(m), np.zeros(m)
    if split > 0:
        d1, e1, t1 = _reduce(A, 0, split, G1)
        d[:split], e[:split], tau[:split] = d1[:split], e1[:split], t1[:split]
    d2, e2, t2 = _reduce(A, split, m - 1, G2)
    d[split:], e[split:], tau[split:] = d2[split:], e2[split:], t2[split:]
    Q = _q_of(A, tau)
    T = np.diag(d) + np.diag(e[:m - 1], 1) + np.diag(e[:m - 1], -1)
    scale = float(np.abs(np.linalg.eigvalsh(a)).max())
    assert np.abs(Q.T @ a @ Q - T).max() <= 1e-13 * scale
    assert np.abs(Q.T @ Q - np.eye(m)).max() <= 1e-13


def test_reading_column_zero_late_breaks_the_scheme():
    """The fault of the first grid-kernel form, planted in this CPU
    restatement: when the CTAs after CTA 0 take column 0 from the matrix
    once CTA 0 has stored reflector 0 in it, Q^T A Q is no longer T."""
    m, G = 40, 5
    rng = np.random.default_rng(1)
    a = rng.standard_normal((m, m))
    a = 0.5 * (a + a.T) + np.diag(np.linspace(-5.0, 80.0, m))
    A = a.copy()
    d, e, tau = _reduce(A, 0, m - 1, G, late_col0=True)
    Q = _q_of(A, tau)
    T = np.diag(d) + np.diag(e[:m - 1], 1) + np.diag(e[:m - 1], -1)
    assert np.abs(Q.T @ a @ Q - T).max() > 1e-3 * float(np.abs(np.linalg.eigvalsh(a)).max())
