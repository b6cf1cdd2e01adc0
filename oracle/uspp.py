"""Oracle overlap apply and dense generalized eigenproblem, float64 numpy
(test infrastructure only).

Restates gradwave ``scf/uspp_batch.py:69-73`` (``BatchedHS.s``):

    S c = (c + sum_pq |beta_p> q_pq <beta_q|c>) * mask,
    b = conj(p) . c over G, then (b q) p,

and, for cells small enough to hold the whole sphere, the lowest eigenpairs of
H x = eps S x by dense diagonalisation (scipy's ``eigh(H, S)``), H built
column by column from the oracle H apply. That is the exact answer the
reference's ``davidson_gen_batched`` (``scf/uspp_batch.py:99-233``) converges
to, independent of any Davidson schedule.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg


def s_apply(p, q, mask, c) -> np.ndarray:
    p = np.asarray(p, dtype=np.complex128)
    c = np.asarray(c, dtype=np.complex128)
    b = np.matmul(c, np.swapaxes(np.conj(p), 1, 2))           # (nk, nb, nproj)
    out = c + np.matmul(b @ np.asarray(q, dtype=np.complex128), p)
    return out * np.asarray(mask, dtype=bool)[:, None, :]


def dense_generalized(orc, p, q, npw, nbands: int, chunk: int = 256) -> np.ndarray:
    """Lowest ``nbands`` eigenvalues of H x = eps S x per k, (nk, nbands).

    ``orc`` is an ``oracle.ham.OracleHamiltonian``; the sphere of k holds the
    first ``npw[k]`` slots of the padded layout."""
    p = np.asarray(p, dtype=np.complex128)
    nk, _, m = p.shape
    out = np.zeros((nk, nbands))
    for k in range(nk):
        n = int(npw[k])
        h = np.zeros((n, n), dtype=np.complex128)
        s_mat = np.zeros((n, n), dtype=np.complex128)
        mask = np.zeros((nk, m), dtype=bool)
        mask[k, :n] = True
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            cols = np.zeros((nk, e - s, m), dtype=np.complex128)
            cols[k, np.arange(e - s), np.arange(s, e)] = 1.0
            # row b of an apply is the operator on the unit vector e_(s+b)
            h[:, s:e] = orc.apply(cols)[k, :, :n].T
            s_mat[:, s:e] = s_apply(p, q, mask, cols)[k, :, :n].T
        h = 0.5 * (h + h.conj().T)
        s_mat = 0.5 * (s_mat + s_mat.conj().T)
        out[k] = scipy.linalg.eigh(h, s_mat, eigvals_only=True, subset_by_index=[0, nbands - 1])
    return out
