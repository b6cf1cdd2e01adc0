"""Oracle electron density, float64 numpy (test infrastructure only).

Restates gradwave ``core/batch.py:562-587`` (``density_b``) with
``g_to_r_b`` (``core/batch.py:208-216``):

    psi_kb(r) = sum_G c_kb(G) exp(iG.r): scatter-add of the sphere coefficients
                into the box at ``flat_idx`` (padded slots at their index,
                0), then the unnormalised inverse FFT (ifftn times N);
    rho(r)    = sum_k sum_b kweights[k] occ[k, b] |psi_kb(r)|^2 / volume.
"""

from __future__ import annotations

import numpy as np
import scipy.fft


def density_b(coeffs, occ, kweights, flat_idx, shape, volume) -> np.ndarray:
    c = np.asarray(coeffs, dtype=np.complex128)
    nk, nb, _ = c.shape
    shape = tuple(int(s) for s in shape)
    n = int(np.prod(shape))
    w = np.asarray(kweights, dtype=np.float64)[:, None] * np.asarray(occ, dtype=np.float64)
    rho = np.zeros(shape, dtype=np.float64)
    for k in range(nk):
        box = np.zeros((nb, n), dtype=np.complex128)
        for b in range(nb):
            np.add.at(box[b], np.asarray(flat_idx[k], dtype=np.int64), c[k, b])
        psi = scipy.fft.ifftn(box.reshape(nb, *shape), axes=(-3, -2, -1)) * n
        rho += np.einsum("b,bxyz->xyz", w[k], psi.real ** 2 + psi.imag ** 2)
    return rho / float(volume)
