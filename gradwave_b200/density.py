"""Electron density of a band block on the B200 path (drop-in for gradwave's
``density_b``, ``core/batch.py:562-587``).

    rho(r) = sum_k w_k sum_n f_kn |psi_kn(r)|^2 / volume,
    psi_kn(r) = sum_G c_kn(G) exp(iG.r)      (``g_to_r_b``, ``core/batch.py:208-216``)

on the (n0, n1, n2) box in float64, in libgwb.so (``gwb_ham_density``): the
sphere-pruned inverse FFT kernels of the Hamiltonian apply followed by a
pencil kernel that accumulates f |psi|^2 per k in a fixed order (no atomics),
then one sum over k. The band chunking that bounds the dense-grid memory is
the handle's (the reference chunks by a dense-grid budget too).

Padded plane-wave slots must be zero, as they are in the solver's
eigenvectors (the reference would add them to the G = 0 component).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


class _GeometryHandle:
    """A libgwb.so handle with the geometry of a ``BatchedK`` only (the density
    needs no kinetic, potential or projector tables)."""

    def __init__(self, bk, shape, device):
        nk, npw_max = bk.mask.shape
        npw = np.ascontiguousarray(bk.npw.detach().cpu().numpy().astype(np.int64))
        flat = np.ascontiguousarray(bk.flat_idx.detach().cpu().numpy().astype(np.int64))
        geom = _lib.Geometry()
        geom.nk, geom.npw_max, geom.nproj = int(nk), int(npw_max), 0
        for a in range(3):
            geom.n[a] = int(shape[a])
        geom.npw = npw.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        geom.flat_idx = flat.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        h = ctypes.c_void_p()
        _lib.call("gwb_ham_create", ctypes.byref(geom), int(device.index or 0), ctypes.byref(h))
        self._h = h
        self.device = device
        self.nk, self.npw_max = int(nk), int(npw_max)
        self.shape = tuple(int(s) for s in shape)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize(self.device)
                _lib.load().gwb_ham_destroy(h)
            except Exception:
                pass
            self._h = None


_HANDLES: dict = {}


def density_from_handle(handle, nk: int, npw_max: int, shape, coeffs: torch.Tensor, occ: torch.Tensor,
                        kweights: torch.Tensor, volume: float) -> torch.Tensor:
    """rho (n0, n1, n2) float64 from a libgwb.so handle of matching geometry."""
    _lib.require_cuda(coeffs, "coeffs")
    if coeffs.dim() != 3 or coeffs.shape[0] != nk or coeffs.shape[2] != npw_max:
        raise ValueError(f"expected coeffs of shape ({nk}, nb, {npw_max}), got {tuple(coeffs.shape)}")
    nb = int(coeffs.shape[1])
    if tuple(occ.shape) != (nk, nb):
        raise ValueError(f"occ must be ({nk}, {nb}), got {tuple(occ.shape)}")
    dev = coeffs.device
    c = coeffs.contiguous()
    w = (torch.as_tensor(kweights, dtype=torch.float64, device=dev)[:, None]
         * torch.as_tensor(occ, dtype=torch.float64, device=dev)).contiguous()
    rho = torch.empty(tuple(int(s) for s in shape), dtype=torch.float64, device=dev)
    _lib.call("gwb_ham_density", handle, c.data_ptr(), nb * npw_max, nb, _lib.io_dtype(c), w.data_ptr(), nb,
              1.0 / float(volume), rho.data_ptr(), _lib.stream_ptr(dev))
    return rho


def density_b(coeffs: torch.Tensor, occ: torch.Tensor, kweights: torch.Tensor, bk, shape, volume: float
              ) -> torch.Tensor:
    """rho(r) on the dense grid [e/A^3], the reference's ``density_b``
    signature (gradwave ``core/batch.py:562-587``); the handle for ``bk`` and
    ``shape`` is built once and cached."""
    dev = coeffs.device
    key = (id(bk), tuple(int(s) for s in shape), dev.index)
    h = _HANDLES.get(key)
    if h is None or h[1] is not bk:
        h = (_GeometryHandle(bk, shape, dev), bk)
        _HANDLES[key] = h
    g = h[0]
    return density_from_handle(g._h, g.nk, g.npw_max, g.shape, coeffs, occ, kweights, volume)
