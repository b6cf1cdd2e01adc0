"""Oracle Gamma-point apply on the half sphere, float64 numpy (test
infrastructure only).

Restates gradwave ``core/gamma.py:150-203`` by its definition: the half
vector is expanded to the Hermitian-symmetric full sphere
(``half_to_full``: each point reads its representative's slot, conjugated
for the -G member), the full complex apply of ``oracle.ham`` acts on it
(``core/batch.py:480-505``, equal to the reference's real-FFT local term on
such vectors), and the representatives are read back (``full_to_half``).
"""

from __future__ import annotations

import numpy as np

from oracle.ham import OracleHamiltonian


def gamma_apply(orc: OracleHamiltonian, src_half, conj_full, rep_full, chalf) -> np.ndarray:
    c = np.asarray(chalf, dtype=np.complex128)
    full = c[:, np.asarray(src_half)]
    full = np.where(np.asarray(conj_full, dtype=bool)[None, :], full.conj(), full)
    out = orc.apply(full[None])[0]
    return out[:, np.asarray(rep_full)]
