"""Split-precision complex products on the tensor cores (host side of
``gwb_tc_planes`` / ``gwb_zgemm_tc``).

A ``PlaneSet`` holds a batch of complex matrices as four BF16 planes per
batch entry (re_hi, re_lo, im_hi, im_lo; x = hi + lo to about 2^-17 |x|), the
operand format of the tcgen05 kernels. ``zgemm_tc`` computes
C = alpha A op(B) + beta C in float64 complex from two plane sets with FP32
accumulation (error about 2^-15 sum_k |a_ik||b_kj|).
"""

from __future__ import annotations

import torch

from . import _lib

OP_N, OP_H = 0, 2


class PlaneSet:
    """(nk, 4, rows_cap, ld) BF16 planes of an nk-batch of complex matrices
    with up to rows_cap rows of up to ``cols`` columns (ld = cols rounded up to
    a multiple of 8)."""

    def __init__(self, nk: int, rows_cap: int, cols: int, device):
        self.nk, self.rows_cap, self.cols = int(nk), int(rows_cap), int(cols)
        self.ld = (self.cols + 7) // 8 * 8
        self.t = torch.zeros(self.nk, 4, self.rows_cap, self.ld, dtype=torch.bfloat16, device=device)

    def write(self, src: torch.Tensor, rows: int, row0: int = 0, src_ld: int | None = None,
              src_kstride: int | None = None, offset: int = 0, conj: bool = False, stream: int | None = None,
              cols: int | None = None):
        """Planes of rows [row0, row0 + rows) from rows [0, rows) of the
        complex tensor ``src`` (its storage from element ``offset``; row stride
        ``src_ld``, batch stride ``src_kstride``, default: src's own); ``cols``
        columns (default: the set's), the rest of each plane row zeroed."""
        _lib.require_cuda(src, "plane source")
        if src.dtype not in (torch.complex64, torch.complex128):
            raise TypeError(f"plane source must be complex64/complex128, got {src.dtype}")
        esz = src.element_size()
        ld = src.shape[-1] if src_ld is None else src_ld
        ks = (src.stride(0) if src.dim() == 3 else 0) if src_kstride is None else src_kstride
        c = self.cols if cols is None else int(cols)
        if c > self.cols:
            raise ValueError(f"{c} columns exceed the plane set's {self.cols}")
        _lib.call("gwb_tc_planes", self.nk, int(rows), c, src.data_ptr() + offset * esz, int(ld), int(ks),
                  _lib.io_dtype(src), 1 if conj else 0, self.t.data_ptr(), self.ld, self.rows_cap, int(row0),
                  _lib.stream_ptr(src.device) if stream is None else stream)


_WORK: dict = {}
_STATUS: dict = {}


def status_flag(device) -> torch.Tensor:
    """The device int the tensor-core kernels set to GWB_ERR_TIMEOUT when a
    bounded wait runs out (one per device, zeroed by ``check_status``)."""
    key = torch.device(device).index
    if key not in _STATUS:
        _STATUS[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _STATUS[key]


def check_status(device) -> None:
    """Raise if a tensor-core kernel on ``device`` reported a timed-out wait."""
    st = status_flag(device)
    v = int(st.item())
    if v != 0:
        st.zero_()
        raise _lib.GwbError(v, "tensor-core GEMM: a bounded pipeline wait ran out")


def _work(device, nbytes: int) -> torch.Tensor:
    key = torch.device(device).index
    w = _WORK.get(key)
    if w is None or w.numel() < nbytes:
        w = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
        _WORK[key] = w
    return w


def work_bytes(op_b: int, M: int, N: int, K: int, batch: int) -> int:
    """Bytes of partial-sum scratch ``zgemm_tc`` uses for these sizes."""
    return int(_lib.load().gwb_zgemm_tc_work_bytes(op_b, M, N, K, batch))


def zgemm_tc(op_b: int, M: int, N: int, K: int, A: PlaneSet, B: PlaneSet, C: torch.Tensor, ldc: int, strideC: int,
             alpha: complex = 1.0, beta: complex = 0.0, c_offset: int = 0, stream: int | None = None,
             status: torch.Tensor | None = None, work: torch.Tensor | None = None) -> None:
    """C = alpha A op(B) + beta C (per batch entry; complex128 C with row
    stride ``ldc`` and batch stride ``strideC``, from element ``c_offset``).
    op_b = OP_H: B holds N rows of length K; OP_N: B holds K rows of length N.
    A timed-out pipeline wait ORs GWB_ERR_TIMEOUT into ``status`` (an int32
    device tensor; default: the per-device flag read by ``check_status``).
    ``work``: partial-sum scratch (default: a per-device buffer; callers that
    run products concurrently on several streams pass their own)."""
    if C.dtype != torch.complex128:
        raise TypeError("zgemm_tc writes complex128")
    if A.nk != B.nk:
        raise ValueError("plane sets of different batch sizes")
    dev = C.device
    if work is None:
        work = _work(dev, work_bytes(op_b, M, N, K, A.nk))
    alpha, beta = complex(alpha), complex(beta)
    _lib.call("gwb_zgemm_tc", op_b, int(M), int(N), int(K), alpha.real, alpha.imag, A.t.data_ptr(), A.ld,
              A.rows_cap, B.t.data_ptr(), B.ld, B.rows_cap, beta.real, beta.imag, C.data_ptr() + 16 * c_offset,
              int(ldc), int(strideC), A.nk, work.data_ptr(), work.numel(),
              (status_flag(dev) if status is None else status).data_ptr(),
              _lib.stream_ptr(dev) if stream is None else stream)
