"""Oracle Teter-Payne-Allan preconditioner (test infrastructure only).

Restates gradwave ``solvers/precond.py:20-39`` (``teter_b``): with
x = T_G / max(T_band, 1e-12), the filter is
K = (27 + 18x + 12x^2 + 8x^3) / (27 + 18x + 12x^2 + 8x^3 + 16x^4), formed in
float64 and multiplied into the residual.
"""

from __future__ import annotations

import numpy as np


def teter_coeff(t_g: np.ndarray, t_band: np.ndarray) -> np.ndarray:
    """(nk, nsel, npw) coefficient from t_g (nk, npw) and t_band (nk, nsel)."""
    x = t_g[:, None, :] / np.maximum(t_band[..., None], 1e-12)
    x2 = x * x
    num = 27.0 + 18.0 * x + 12.0 * x2 + 8.0 * x2 * x
    return num / (num + 16.0 * x2 * x2)


def teter_b(residual: np.ndarray, t_g: np.ndarray, t_band: np.ndarray) -> np.ndarray:
    return residual * teter_coeff(np.asarray(t_g, np.float64), np.asarray(t_band, np.float64))
