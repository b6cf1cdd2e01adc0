"""Float64-accurate real products on the int8 tensor cores (host side of
``gwb_oz_*``, the Ozaki scheme's first form with int8 slices, and of
``gwb_crt_*``, its second form with residues and the Chinese remainder
theorem; both on tcgen05 kind::i8).

Second form (``ResidueSet``, ``crt_gemm``, ``CrtMatmul``): a row is scaled to
integers below 2^p and held as n int8 residues (n = 18: p = 60); a product
is n exact int8 GEMMs, one per modulus, and a double-double reconstruction.
Its error is about 2^-p-1 of the row maxima (256x below the first form's
with 8 slices) and it costs n int8 products instead of s(s+1)/2, each on
M 128 x N 256 tiles.

First form:

A ``SliceSet`` holds up to ``rows_cap`` rows of length up to ``k_cap`` as s
int8 planes (about 7 bits each, rounded to nearest, per-row power-of-two
scales), the operand format of
``oz_gemm``. Rows are written either from rows of a float64 matrix
(``split_rows``, optionally multiplied column by column by ``fold``) or from
the columns of one (``split_cols``: the transposed layout that a product
C = A B needs for its B, with one scale per source row in ``kscale``).

    oz_gemm(M, N, K, A, B, C)   C = alpha A[:M] B[:N]^T + beta C   (float64)

The error of an element is about 2^-7s of the row maxima of both operands
times sqrt(K): with s = 8 (36 int8 products per float64 product) that is the
level of a float64 GEMM of the same shape.
"""

from __future__ import annotations

import torch

from . import _lib

# 8 slices keep the products at float64 level also for the residuals of the
# Davidson: the error of a product is relative to the row maxima of its
# operands, so in X = U^T V and HX = U^T HV every plane wave carries about
# 2^-56 of the row maxima (2^-49 with 7 slices, which puts a floor near
# 1e-10 eV under the residual norms of the 216-atom cell)
DEFAULT_SLICES = 8


class SliceSet:
    def __init__(self, rows_cap: int, k_cap: int, device, s: int = DEFAULT_SLICES):
        if s not in (6, 7, 8):
            raise ValueError("slice count must be 6, 7 or 8")
        self.s, self.rows_cap = int(s), int(rows_cap)
        self.ldk = max(64, (int(k_cap) + 63) // 64 * 64)
        self.device = torch.device(device)
        self.q = torch.zeros(self.s, self.rows_cap, self.ldk, dtype=torch.int8, device=self.device)
        self.scale = torch.ones(self.rows_cap, dtype=torch.float64, device=self.device)
        self.kscale = torch.ones(self.ldk, dtype=torch.float64, device=self.device)

    def split_rows(self, src: torch.Tensor, rows: int | None = None, row0: int = 0, fold: torch.Tensor | None = None,
                   stream: int | None = None) -> None:
        """Rows [row0, row0 + rows) from the rows of the float64 matrix
        ``src`` (2-D, unit column stride; K = its width), each times ``fold``
        column by column when given; columns K..ldk-1 are zeroed."""
        _check(src)
        n = int(src.shape[0]) if rows is None else int(rows)
        K = int(src.shape[1])
        if K > self.ldk:
            raise ValueError(f"rows of {K} exceed the slice set's {self.ldk}")
        if fold is not None and (fold.dtype != torch.float64 or not fold.is_contiguous() or fold.numel() < K):
            raise ValueError("fold must be a contiguous float64 vector of at least K values")
        _lib.call("gwb_oz_split_rows", self.s, n, K, src.data_ptr(), int(src.stride(0)),
                  None if fold is None else fold.data_ptr(), self.q.data_ptr(), self.ldk, self.rows_cap, int(row0),
                  self.scale.data_ptr(), _stream(src) if stream is None else stream)

    def split_cols(self, src: torch.Tensor, k0: int = 0, stream: int | None = None) -> None:
        """Columns [k0, k0 + src.shape[0]) of every row r < src.shape[1] from
        the float64 matrix ``src`` (krows x R, unit column stride): row r of
        the set holds column r of src, scaled per source row (``kscale``)."""
        _check(src)
        krows, R = int(src.shape[0]), int(src.shape[1])
        if R > self.rows_cap or k0 + krows > self.ldk:
            raise ValueError("columns beyond the slice set")
        _lib.call("gwb_oz_split_cols", self.s, krows, R, src.data_ptr(), int(src.stride(0)), self.q.data_ptr(),
                  self.ldk, self.rows_cap, int(k0), self.kscale.data_ptr(),
                  _stream(src) if stream is None else stream)


def _check(src: torch.Tensor) -> None:
    _lib.require_cuda(src, "slice source")
    if src.dtype != torch.float64 or src.dim() != 2 or src.stride(1) != 1:
        raise TypeError("slice source must be a 2-D float64 tensor with unit column stride")


def _stream(t: torch.Tensor) -> int:
    return _lib.stream_ptr(t.device)


_WORK: dict = {}
_STATUS: dict = {}


def status_flag(device) -> torch.Tensor:
    """The device int the Ozaki kernels set to GWB_ERR_TIMEOUT when a bounded
    wait runs out (one per device; ``check_status`` reads and clears it)."""
    key = torch.device(device).index
    if key not in _STATUS:
        _STATUS[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _STATUS[key]


def check_status(device) -> None:
    st = status_flag(device)
    v = int(st.item())
    if v != 0:
        st.zero_()
        raise _lib.GwbError(v, "int8 tensor-core product: a bounded pipeline wait ran out")


def _work(device, nbytes: int) -> torch.Tensor:
    key = torch.device(device).index
    w = _WORK.get(key)
    if w is None or w.numel() < nbytes:
        w = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
        _WORK[key] = w
    return w


def oz_gemm(M: int, N: int, K: int, A: SliceSet, B: SliceSet, C: torch.Tensor, alpha: float = 1.0,
            beta: float = 0.0, a_row0: int = 0, b_row0: int = 0, b_scaled: bool = True,
            stream: int | None = None, status: torch.Tensor | None = None, work: torch.Tensor | None = None) -> None:
    """C = alpha A[a_row0:a_row0+M] B[b_row0:b_row0+N]^T + beta C over K
    columns (C a 2-D float64 tensor with unit column stride). ``b_scaled``:
    B's rows carry their own scales (written by ``split_rows``); False for a
    B written by ``split_cols``, whose scales were folded into A. The
    columns K..ceil(K/64)*64-1 of A must be zero (``split_rows`` leaves them
    so)."""
    if A.s != B.s:
        raise ValueError("slice sets of different slice counts")
    if C.dtype != torch.float64 or C.dim() != 2 or C.stride(1) != 1:
        raise TypeError("C must be a 2-D float64 tensor with unit column stride")
    dev = C.device
    if work is None:
        work = _work(dev, int(_lib.load().gwb_oz_work_bytes(M, N, K)))
    _lib.call("gwb_oz_gemm", A.s, int(M), int(N), int(K), A.q.data_ptr(), A.ldk, A.rows_cap, int(a_row0),
              A.scale.data_ptr(), B.q.data_ptr(), B.ldk, B.rows_cap, int(b_row0),
              B.scale.data_ptr() if b_scaled else None, float(alpha), float(beta), C.data_ptr(), int(C.stride(0)),
              work.data_ptr(), work.numel(), (status_flag(dev) if status is None else status).data_ptr(),
              _lib.stream_ptr(dev) if stream is None else stream)


DEFAULT_MODULI = 18


class ResidueSet:
    """Up to ``rows_cap`` rows of length up to ``k_cap`` as n int8 residue
    planes with one float64 scale per row (``gwb_crt_split_rows`` /
    ``gwb_crt_split_cols``)."""

    def __init__(self, rows_cap: int, k_cap: int, device, n: int = DEFAULT_MODULI):
        if n not in (16, 18, 20):
            raise ValueError("modulus count must be 16, 18 or 20")
        self.s, self.rows_cap = int(n), int(rows_cap)
        self.ldk = max(64, (int(k_cap) + 63) // 64 * 64)
        self.device = torch.device(device)
        self.q = torch.zeros(self.s, self.rows_cap, self.ldk, dtype=torch.int8, device=self.device)
        self.scale = torch.ones(self.rows_cap, dtype=torch.float64, device=self.device)
        self.kscale = torch.ones(self.ldk, dtype=torch.float64, device=self.device)

    def split_rows(self, src: torch.Tensor, rows: int | None = None, row0: int = 0, fold: torch.Tensor | None = None,
                   stream: int | None = None) -> None:
        """Rows [row0, row0 + rows) from the rows of the float64 matrix
        ``src`` (2-D, unit column stride), each times ``fold`` column by
        column when given; columns K..ldk-1 are zeroed."""
        _check(src)
        n = int(src.shape[0]) if rows is None else int(rows)
        K = int(src.shape[1])
        if K > self.ldk:
            raise ValueError(f"rows of {K} exceed the residue set's {self.ldk}")
        if fold is not None and (fold.dtype != torch.float64 or not fold.is_contiguous() or fold.numel() < K):
            raise ValueError("fold must be a contiguous float64 vector of at least K values")
        _lib.call("gwb_crt_split_rows", self.s, n, K, src.data_ptr(), int(src.stride(0)),
                  None if fold is None else fold.data_ptr(), self.q.data_ptr(), self.ldk, self.rows_cap, int(row0),
                  self.scale.data_ptr(), _stream(src) if stream is None else stream)

    def split_cols(self, src: torch.Tensor, k0: int = 0, stream: int | None = None) -> None:
        """Columns [k0, k0 + src.shape[0]) of every row r < src.shape[1] from
        the float64 matrix ``src`` (krows x R, unit column stride): row r of
        the set holds column r of src, scaled per source row (``kscale``)."""
        _check(src)
        krows, R = int(src.shape[0]), int(src.shape[1])
        if R > self.rows_cap or k0 + krows > self.ldk:
            raise ValueError("columns beyond the residue set")
        _lib.call("gwb_crt_split_cols", self.s, krows, R, src.data_ptr(), int(src.stride(0)), self.q.data_ptr(),
                  self.ldk, self.rows_cap, int(k0), self.kscale.data_ptr(), self.scale.data_ptr(),
                  _stream(src) if stream is None else stream)


def crt_gemm(M: int, N: int, K: int, A: ResidueSet, B: ResidueSet, C: torch.Tensor, alpha: float = 1.0,
             beta: float = 0.0, a_row0: int = 0, b_row0: int = 0, stream: int | None = None,
             status: torch.Tensor | None = None, work: torch.Tensor | None = None) -> None:
    """C = alpha A[a_row0:a_row0+M] B[b_row0:b_row0+N]^T + beta C over K
    columns (C a 2-D float64 tensor with unit column stride); K <= 2^19."""
    if A.s != B.s:
        raise ValueError("residue sets of different modulus counts")
    if C.dtype != torch.float64 or C.dim() != 2 or C.stride(1) != 1:
        raise TypeError("C must be a 2-D float64 tensor with unit column stride")
    dev = C.device
    if work is None:
        work = _work(dev, int(_lib.load().gwb_crt_work_bytes(A.s, M, N, K)))
    _lib.call("gwb_crt_gemm", A.s, int(M), int(N), int(K), A.q.data_ptr(), A.ldk, A.rows_cap, int(a_row0),
              A.scale.data_ptr(), B.q.data_ptr(), B.ldk, B.rows_cap, int(b_row0), B.scale.data_ptr(), float(alpha),
              float(beta), C.data_ptr(), int(C.stride(0)), work.data_ptr(), work.numel(),
              (status_flag(dev) if status is None else status).data_ptr(),
              _lib.stream_ptr(dev) if stream is None else stream)


class OzMatmul:
    """Float64 products of the Davidson shapes on the int8 tensor cores,
    with the slice sets kept per operand role and grown as needed:

    * ``nt(a, b, out)``: out = a b^T (a: M x K, b: N x K rows);
    * ``nn(a, b, out)``: out = a b (a: M x K, b: K x N rows), through the
      transposed slices of b with b's row scales folded into a.
    ``alpha``/``beta`` as in a GEMM."""

    set_type = SliceSet

    def __init__(self, device, s: int = DEFAULT_SLICES):
        self.device, self.s = torch.device(device), int(s)
        self.sets: dict = {}

    def new_set(self, rows: int, k: int):
        return self.set_type(rows, k, self.device, self.s)

    def _set(self, key: str, rows: int, k: int):
        st = self.sets.get(key)
        if st is None or st.rows_cap < rows or st.ldk < k:
            rc = max(rows, st.rows_cap if st else 0)
            kc = max(k, st.ldk if st else 0)
            st = self.new_set(rc, kc)
            self.sets[key] = st
        return st

    def gemm(self, M, N, K, A, B, out, alpha=1.0, beta=0.0, a_row0=0, b_row0=0, b_scaled=True) -> None:
        oz_gemm(M, N, K, A, B, out, alpha, beta, a_row0=a_row0, b_row0=b_row0, b_scaled=b_scaled)

    def nt(self, a: torch.Tensor, b: torch.Tensor, out: torch.Tensor, alpha: float = 1.0, beta: float = 0.0,
           same: bool = False) -> torch.Tensor:
        M, K = a.shape
        N = b.shape[0]
        sa = self._set("nt_a", M, K)
        sa.split_rows(a)
        if same:
            sb = sa
        else:
            sb = self._set("nt_b", N, K)
            sb.split_rows(b)
        self.gemm(M, N, K, sa, sb, out, alpha, beta)
        return out

    def nn(self, a: torch.Tensor, b: torch.Tensor, out: torch.Tensor, alpha: float = 1.0,
           beta: float = 0.0) -> torch.Tensor:
        M, K = a.shape
        N = b.shape[1]
        sb = self._set("nn_b", N, K)
        sb.split_cols(b)
        sa = self._set("nn_a", M, K)
        sa.split_rows(a, fold=sb.kscale)
        self.gemm(M, N, K, sa, sb, out, alpha, beta, b_scaled=False)
        return out


class CrtMatmul(OzMatmul):
    """``OzMatmul`` on residue sets: the same ``nt`` / ``nn`` / ``gemm``
    calls through ``crt_gemm`` (the B scales of a transposed set are 2^-p
    and always applied)."""

    set_type = ResidueSet

    def __init__(self, device, n: int = DEFAULT_MODULI):
        super().__init__(device, n)

    def gemm(self, M, N, K, A, B, out, alpha=1.0, beta=0.0, a_row0=0, b_row0=0, b_scaled=True) -> None:
        crt_gemm(M, N, K, A, B, out, alpha, beta, a_row0=a_row0, b_row0=b_row0)
