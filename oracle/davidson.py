"""Oracle batched block Davidson, float64 numpy (test infrastructure only).

Restates gradwave ``solvers/davidson.py:528-774`` (``davidson_batched``, the
synchronous path with the default Householder-QR orthonormalisation) and its
helpers ``_orthonormalize_b`` (``:406-457``):

* max_dim = min(max_dim_factor * nb, min_k npw)                       (:572)
* v = orthonormalise(x0); hv = H v                                     (:624-625)
* per round: s = v^H hv, Hermitised, eigh; x = u^T v, hx = u^T hv;
  r = hx - eps x; rn = |r|                                              (:648-657)
* stop when max rn < tol                                                (:691-694)
* n_add = max_k #(rn > tol); worst-n_add residuals per k               (:698,729-730)
* TPA filter with t_band = <x|T|x>, rows unit-normalised               (:732-743)
* restart: QR of x, hx <- R^-T hx, keep d                               (:745-759)
* else: project d against v twice, QR, append d and H d                 (:760-763)

One deliberate difference: the rank-repair jitter for (near-)zero rows uses
numpy's generator instead of torch's (``:452-456``); it only fires on
rank-deficient blocks, which the parity cases do not produce.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.linalg

from .precond import teter_b


@dataclass
class OracleResult:
    eigenvalues: np.ndarray      # (nk, nb)
    eigenvectors: np.ndarray     # (nk, nb, npw)
    n_iter: int
    residual_norms: np.ndarray   # (nk, nb)
    n_apply: int
    history: list


def _qr_rows(x: np.ndarray):
    """Row-orthonormal q and triangular r with x^T = q^T r (batched)."""
    q, r = np.linalg.qr(np.swapaxes(x, -1, -2), mode="reduced")
    return np.swapaxes(q, -1, -2), r


def orthonormalize_b(v, mask, against=None):
    def project(x):
        if against is not None and against.shape[1]:
            for _ in range(2):
                x = x - (x @ np.conj(np.swapaxes(against, -1, -2))) @ against
        return x

    v = project(v * mask[:, None, :])
    rn = np.linalg.norm(v, axis=-1, keepdims=True)
    bad = rn < 1e-8
    if bad.any():
        rng = np.random.default_rng(v.shape[1] + 7919)
        jit = rng.standard_normal(v.shape) + 1j * rng.standard_normal(v.shape)
        v = project((v + bad * jit) * mask[:, None, :])
    q, _ = _qr_rows(v)
    return q


def davidson_rounds(h_apply, x0, t, mask, tol=1e-9, max_iter=40, max_dim_factor=4, keep_history=False):
    """The solve as a generator: yields ``(it, eig, rn)`` after every
    Rayleigh-Ritz round (the point where the reference appends to its
    ``history_out``, ``solvers/davidson.py:688-690``) and returns the
    ``OracleResult``. A caller can time the rounds one by one."""
    x0 = np.asarray(x0, dtype=np.complex128)
    t = np.asarray(t, dtype=np.float64)
    mask = np.asarray(mask, dtype=bool)
    nk, nb, m = x0.shape
    max_dim = min(max_dim_factor * nb, int(mask.sum(axis=1).min()))
    n_apply = 0

    def H(z):
        nonlocal n_apply
        n_apply += z.shape[0] * z.shape[1]
        return h_apply(z)

    v = orthonormalize_b(x0, mask)
    hv = H(v)
    history = []
    eig = np.zeros((nk, nb))
    x = v[:, :nb]
    rn = np.full((nk, nb), np.inf)
    for it in range(1, max_iter + 1):
        s = np.conj(v) @ np.swapaxes(hv, -1, -2)
        s = 0.5 * (s + np.conj(np.swapaxes(s, -1, -2)))
        w, u = np.linalg.eigh(s)
        u = u[:, :, :nb]
        eig = w[:, :nb].real
        ut = np.ascontiguousarray(np.swapaxes(u, 1, 2))
        x = ut @ v                                   # x_a = sum_j u_ja v_j
        hx = ut @ hv
        r = hx - eig[..., None] * x
        rn = np.linalg.norm(r, axis=-1)
        if keep_history:
            history.append((it, rn.copy(), eig.copy()))
        yield it, eig, rn
        if rn.max() < tol:
            return OracleResult(eig, x, it, rn, n_apply, history)
        n_add = int((rn > tol).sum(axis=1).max())
        sel = np.argsort(-rn, axis=1, kind="stable")[:, :n_add]
        r_sel = np.take_along_axis(r, sel[..., None], axis=1)
        t_band = ((x.real ** 2 + x.imag ** 2) * t[:, None, :]).sum(axis=-1)   # <x|T|x>
        d = teter_b(r_sel, t, np.take_along_axis(t_band, sel, axis=1))
        dn = np.linalg.norm(d, axis=-1, keepdims=True)
        d = np.where(dn > 1e-300, d / np.maximum(dn, 1e-300), d)
        if v.shape[1] + n_add > max_dim:
            x_orth, rmat = _qr_rows(x)
            hx_orth = np.stack([scipy.linalg.solve_triangular(rmat[k].T, hx[k], lower=True)
                                for k in range(nk)])
            d = orthonormalize_b(d, mask, against=x_orth)
            v = np.concatenate([x_orth, d], axis=1)
            hv = np.concatenate([hx_orth, H(d)], axis=1)
        else:
            d = orthonormalize_b(d, mask, against=v)
            v = np.concatenate([v, d], axis=1)
            hv = np.concatenate([hv, H(d)], axis=1)
    return OracleResult(eig, x, max_iter, rn, n_apply, history)


def davidson_batched(h_apply, x0, t, mask, tol=1e-9, max_iter=40, max_dim_factor=4,
                     keep_history=False) -> OracleResult:
    gen = davidson_rounds(h_apply, x0, t, mask, tol=tol, max_iter=max_iter, max_dim_factor=max_dim_factor,
                          keep_history=keep_history)
    while True:
        try:
            next(gen)
        except StopIteration as stop:
            return stop.value


def band_energy(eig: np.ndarray, kweights: np.ndarray, nocc: int) -> float:
    """sum_k w_k sum_{n < nocc} 2 eps_nk [eV]: the band-energy check of a solve."""
    return float(2.0 * np.sum(np.asarray(kweights)[:, None] * np.asarray(eig)[:, :nocc]))
