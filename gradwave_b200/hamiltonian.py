"""Drop-in replacement of gradwave's ``BatchedHamiltonian`` on the B200 path.

Same constructor and ``apply`` contract as the reference
(gradwave ``core/batch.py:238-258,480-505``):

    h = BatchedHamiltonian(bk, shape, v_eff_r, p)
    out = h.apply(c)          # (nk, nb, npw_max) -> H c, padded slots 0

``apply`` computes in the dtype of its input (complex64 -> float32 arithmetic,
complex128 -> float64), as the reference's dtype-matched tables do
(``core/batch.py:306-331``). ``apply_fp32`` additionally offers float32
arithmetic on complex128 storage (the fp32-expansion applies of the mixed
solver). The work runs in libgwb.so through the torch custom op
``gwb::ham_apply``; internal scratch is owned by the operator and persists
across calls (like the reference's persistent scatter box).

Not supported (out of scope of this path): DFT+U terms (``hub_q``/``hub_dij``)
and the USPP dual grid (``smooth``); passing them raises.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from . import ops  # noqa: F401  (registers torch.ops.gwb.*)
from .telemetry import opcount

_TALLY = {"on": False, "count": 0}


def reset_happly_tally() -> None:
    """Zero and enable the band*k apply counter (gradwave ``core/batch.py:114-123``)."""
    _TALLY["on"] = True
    _TALLY["count"] = 0


def happly_tally() -> int:
    return _TALLY["count"]


class BatchedHamiltonian:
    def __init__(self, bk, shape, v_eff_r, p, hub_q=None, hub_dij=None, smooth=None):
        if hub_q is not None or hub_dij is not None:
            raise NotImplementedError("DFT+U terms are not part of the B200 band-solve path")
        if smooth is not None:
            raise NotImplementedError("the USPP dual grid is not part of the B200 band-solve path")
        if not torch.cuda.is_available():
            raise RuntimeError("BatchedHamiltonian needs a CUDA device (no CPU fallback)")
        self.bk = bk
        self.shape = tuple(int(s) for s in shape)
        dev = bk.mask.device if bk.mask.is_cuda else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        nk, npw_max = bk.mask.shape
        self.nk, self.npw_max = int(nk), int(npw_max)
        self.nproj = int(p.shape[1])
        npw = np.ascontiguousarray(bk.npw.detach().cpu().numpy().astype(np.int64))
        flat = np.ascontiguousarray(bk.flat_idx.detach().cpu().numpy().astype(np.int64))
        geom = _lib.Geometry()
        geom.nk, geom.npw_max, geom.nproj = self.nk, self.npw_max, self.nproj
        for a in range(3):
            geom.n[a] = self.shape[a]
        geom.npw = npw.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        geom.flat_idx = flat.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        handle = ctypes.c_void_p()
        _lib.call("gwb_ham_create", ctypes.byref(geom), int(dev.index or 0), ctypes.byref(handle))
        self._h = handle
        self.handle = int(handle.value)
        # device copies of the tables (kept alive for the handle's copies)
        self.mask = bk.mask.to(dev)
        self.t = bk.t.to(dev, torch.float64).contiguous()
        self.v_eff_r = torch.as_tensor(v_eff_r).to(dev, torch.float64).contiguous()
        self.p = torch.as_tensor(p).to(dev, torch.complex128).contiguous()
        self.dij = bk.dij_full.to(dev, torch.float64).contiguous()
        with torch.cuda.device(dev):
            s = _lib.stream_ptr(dev)
            _lib.call("gwb_ham_set_kinetic", self._h, self.t.data_ptr(), s)
            _lib.call("gwb_ham_set_potential", self._h, self.v_eff_r.data_ptr(), s)
            _lib.call("gwb_ham_set_projectors", self._h, self.p.data_ptr() if self.nproj else None,
                      self.dij.data_ptr() if self.nproj else None, s)
        from .autotune import apply_tuning
        self.tuning = apply_tuning(self._h, "complex", self.shape, self.nproj)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize(self.device)
                _lib.load().gwb_ham_destroy(h)
            except Exception:
                pass
            self._h = None

    def _count(self, c: torch.Tensor) -> None:
        n = int(c.shape[0]) * int(c.shape[1])
        if _TALLY["on"]:
            _TALLY["count"] += n
        opcount.bump("hpsi", n)
        opcount.bump("fft", 2)

    def _check(self, c: torch.Tensor) -> None:
        if c.dim() != 3 or c.shape[0] != self.nk or c.shape[2] != self.npw_max:
            raise ValueError(f"expected c of shape ({self.nk}, nb, {self.npw_max}), got {tuple(c.shape)}")
        if c.device != self.device:
            raise ValueError(f"c is on {c.device}, the operator on {self.device}")

    def apply(self, c: torch.Tensor) -> torch.Tensor:
        """H c in the arithmetic of c's dtype; mask preserved."""
        self._check(c)
        self._count(c)
        prec = _lib.GWB_FP64 if c.dtype == torch.complex128 else _lib.GWB_FP32
        return torch.ops.gwb.ham_apply(self.handle, c, prec)

    def apply_fp32(self, c: torch.Tensor) -> torch.Tensor:
        """H c with float32 arithmetic whatever the storage dtype of c."""
        self._check(c)
        self._count(c)
        return torch.ops.gwb.ham_apply(self.handle, c, _lib.GWB_FP32)

    def apply_into(self, src_ptr: int, src_kstride: int, dst_ptr: int, dst_kstride: int, nrows: int,
                   prec: int, n_rows_counted: int | None = None) -> None:
        """H on nrows complex128 rows per k read at src (k blocks src_kstride
        elements apart) written to dst: the in-place form the Davidson basis
        uses (``gwb_ham_apply_strided``)."""
        n = self.nk * nrows if n_rows_counted is None else n_rows_counted
        if _TALLY["on"]:
            _TALLY["count"] += n
        opcount.bump("hpsi", n)
        opcount.bump("fft", 2)
        _lib.call("gwb_ham_apply_strided", self._h, src_ptr, src_kstride, dst_ptr, dst_kstride, nrows,
                  _lib.GWB_C128, prec, _lib.stream_ptr(self.device))

    def _count_rows(self, n: int) -> None:
        if _TALLY["on"]:
            _TALLY["count"] += n
        opcount.bump("hpsi", n)

    def _native_workspace(self, nbytes: int) -> torch.Tensor:
        """Device workspace of the native Davidson driver, kept across solves."""
        ws = getattr(self, "_ws", None)
        if ws is None or ws.numel() < nbytes:
            ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._ws = ws
        return ws

    def k_slice(self, start: int, end: int) -> "BatchedHamiltonian":
        """The Hamiltonian of the k-points [start, end) (its own handle and
        scratch, cached): the unit of the k-group solves, which run
        concurrently on separate streams."""
        cache = self.__dict__.setdefault("_kslices", {})
        key = (int(start), int(end))
        if key not in cache:
            from .sharding import slice_batched
            cache[key] = BatchedHamiltonian(slice_batched(self.bk, start, end), self.shape, self.v_eff_r,
                                            self.p[start:end])
        return cache[key]

    def density(self, coeffs: torch.Tensor, occ: torch.Tensor, kweights: torch.Tensor,
                volume: float) -> torch.Tensor:
        """rho(r) = sum_k w_k sum_n f_kn |psi_kn(r)|^2 / volume on this
        operator's box, float64 (gradwave ``core/batch.py:562-587``,
        ``density_b``), with this handle's geometry and scratch."""
        from .density import density_from_handle
        self._check(coeffs)
        return density_from_handle(self._h, self.nk, self.npw_max, self.shape, coeffs, occ, kweights, volume)

    def scratch_bytes(self) -> int:
        return int(_lib.load().gwb_ham_scratch_bytes(self._h))
