"""Oracle Hamiltonian apply, float64 numpy (test infrastructure only).

Restates gradwave ``core/batch.py:480-505`` (``BatchedHamiltonian.apply``):

    H c = T c + local(c) + nonlocal(c), then masked.

* kinetic: ``t * c`` (``core/batch.py:489``);
* local: scatter the sphere into the box with padded slots sent to a trash
  cell one past the box (``core/batch.py:277-279,416-417``), inverse FFT
  normalised by 1/N, multiply by v(r), forward FFT unnormalised, gather the
  sphere (``core/batch.py:420-428``) - i.e. the convolution with
  V(G) = fftn(v)/N of ``core/fftbox.py`` conventions;
* nonlocal: b = conj(p) . c over G, out += b D p (``core/batch.py:499-500,590-595``);
* final ``* mask`` (``core/batch.py:505``).
"""

from __future__ import annotations

import os

import numpy as np
import scipy.fft


def _workers() -> int:
    return int(os.environ.get("GWB_ORACLE_THREADS", os.cpu_count() or 1))


class OracleHamiltonian:
    def __init__(self, mask, flat_idx, t, shape, v_eff_r, p, dij):
        self.mask = np.asarray(mask, dtype=bool)
        self.flat_idx = np.asarray(flat_idx, dtype=np.int64)
        self.t = np.asarray(t, dtype=np.float64)
        self.shape = tuple(int(s) for s in shape)
        self.n = int(np.prod(self.shape))
        self.v = np.asarray(v_eff_r, dtype=np.float64).reshape(self.shape)
        self.p = np.asarray(p, dtype=np.complex128)
        self.pc = np.conj(self.p)
        self.dij = np.asarray(dij, dtype=np.float64)
        self.idx_scatter = np.where(self.mask, self.flat_idx, self.n)
        self.n_apply = 0   # band*k applies, the reference's hpsi tally

    def local(self, c: np.ndarray, chunk: int = 8) -> np.ndarray:
        """Band chunks of ``chunk`` boxes at a time (the same arithmetic as one
        batched transform; a chunk's boxes stay in cache)."""
        nk, nb, m = c.shape
        out = np.zeros_like(c)
        box = np.zeros((min(chunk, max(nb, 1)), self.n + 1), dtype=np.complex128)
        for k in range(nk):
            for b0 in range(0, nb, chunk):
                b1 = min(nb, b0 + chunk)
                bx = box[: b1 - b0]
                bx[:] = 0.0
                bx[:, self.idx_scatter[k]] = c[k, b0:b1]
                psi = scipy.fft.ifftn(bx[:, :self.n].reshape(b1 - b0, *self.shape), axes=(-3, -2, -1),
                                      workers=_workers(), overwrite_x=False)
                psi *= self.v
                vg = scipy.fft.fftn(psi, axes=(-3, -2, -1), workers=_workers(), overwrite_x=True)
                out[k, b0:b1] = vg.reshape(b1 - b0, self.n)[:, self.flat_idx[k]]
        return out

    def nonlocal_(self, c: np.ndarray) -> np.ndarray:
        if self.p.shape[1] == 0:
            return np.zeros_like(c)
        b = np.matmul(c, np.swapaxes(self.pc, 1, 2))          # (nk, nb, nproj)
        return np.matmul(b @ self.dij, self.p)                # (nk, nb, npw)

    def apply(self, c: np.ndarray) -> np.ndarray:
        c = np.asarray(c, dtype=np.complex128)
        self.n_apply += c.shape[0] * c.shape[1]
        out = self.t[:, None, :] * c + self.local(c) + self.nonlocal_(c)
        return out * self.mask[:, None, :]


def from_cell(ci) -> OracleHamiltonian:
    """Oracle operator for a ``gradwave_b200.cells.CellInputs``."""
    bk = ci.bk
    return OracleHamiltonian(bk.mask.numpy(), bk.flat_idx.numpy(), bk.t.numpy(), ci.shape,
                             ci.v_eff_r.numpy(), ci.p.numpy(), bk.dij_full.numpy())
