"""Batched block Davidson on the B200 path (drop-in for gradwave's
``davidson_batched``, ``solvers/davidson.py:528-774``).

Same algorithm and contract as the reference:

* uniform subspace over all k, max_dim = min(max_dim_factor * nb, min_k npw);
* Rayleigh-Ritz with the subspace matrix s = v^H H v in float64;
* the n_add worst residuals per k (n_add = max_k #(|r| > tol)), TPA-filtered
  and unit-normalised, projected twice against the basis and orthonormalised;
* restart when the basis would exceed max_dim, re-orthonormalising the Ritz
  block and transforming its images by the same triangular factor;
* ``hit max_iter`` is not an error: the last Ritz pairs come back.

What differs is where it runs: every step is a libgwb.so kernel or cuBLAS
GEMM on the device, the basis lives in preallocated (nk, max_dim, npw)
buffers (new rows are written in place, H applies land directly in the image
buffer), the subspace matrix is updated incrementally (only the new columns
are formed, ``gwb_subspace_insert``), and orthonormalisation is CholQR2
(float64 Gram, Cholesky, triangular inverse; the reference's own optional
path, ``solvers/davidson.py:195-222``) with the reference's jitter + QR
fallback on breakdown.

Modes:
  ``mode="fp64"``     every apply in float64 (plain TPA Davidson).
  ``mode="fp32exp"``  expansion applies in float32 arithmetic, every
                      convergence decision certified with a float64 apply and
                      a float64 nb x nb Rayleigh-Ritz, float64 hand-off after
                      the first failed certification - the reference's
                      fp32-expansion mode (``solvers/davidson.py:226-308,
                      581-687``).
  ``mode="mixed"``    as fp32exp, but a round that shrinks the residual by less
                      than 30 % counts as a float32 stall only once the
                      residual is within 100x of the float32 floor (early
                      rounds stagnate without any precision limit).
In both float32-expansion modes the first of the two projection passes of
the expansion block, D -= (D V^H) V, runs as split-precision BF16 products on
the tensor cores (``gradwave_b200.tc``, error ~1e-6 of the unit input rows)
against a BF16 plane copy of the basis kept current row block by row block;
the float64 projection pass and float64 CholQR2 that follow remove that
error, so the block is orthonormal and orthogonal to the basis to float64
round-off as before. A block in which some row keeps less than 1e-2 of its
norm is redone in float64 (``GWB_TC_PROJECT=0`` keeps every step in float64;
``GWB_TC_STEPS`` selects steps, including an optional tensor-core
Cholesky-QR round).
``precond`` is ``"teter"`` or an object with ``apply_into(...)`` (the learned
preconditioner, ``gradwave_b200.learned``), which falls back to TPA per band.
"""

from __future__ import annotations

import contextlib
import logging
import math
import os
from dataclasses import dataclass, field

import torch

from . import _lib
from .telemetry import opcount

logger = logging.getLogger(__name__)

_FP32_CERT_FLOOR_EPS = 32 * torch.finfo(torch.float32).eps
_FP32_CERT_STALL = 0.7
_N, _T, _H = 0, 1, 2


@dataclass
class BatchedDavidsonResult:
    eigenvalues: torch.Tensor      # (nk, nb) ascending [eV]
    eigenvectors: torch.Tensor     # (nk, nb, npw_max), padded slots zero
    n_iter: int
    residual_norms: torch.Tensor   # (nk, nb)
    n_apply_low: int = 0
    n_apply_full: int = 0
    info: dict = field(default_factory=dict)


def _ptr(t: torch.Tensor, offset_elems: int = 0) -> int:
    return t.data_ptr() + offset_elems * t.element_size()


_NH_WORK: dict = {}


def _nh_work(dev) -> torch.Tensor:
    w = _NH_WORK.get(dev)
    if w is None:
        w = torch.empty(24 << 20, dtype=torch.uint8, device=dev)
        _NH_WORK[dev] = w
    return w


# A B^H products with at most this many outputs per batch entry go to the
# split-K kernel (which fills the GPU where cuBLAS's output tiles cannot);
# larger outputs to cuBLAS ZGEMM
_NH_MAX_OUT = 160 * 160


def zgemm(opA, opB, M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, batch, alpha=1.0, beta=0.0,
          a_off=0, b_off=0, c_off=0, stream=None, work=None):
    """Row-major batched complex128 GEMM (offsets in elements): A B^H products
    with a small output go to the split-K kernel gwb_zgemm_nh (partial sums in
    ``work``, default a per-device buffer), the rest to cuBLAS through
    gwb_zgemm."""
    s = _lib.stream_ptr(C.device) if stream is None else stream
    a = complex(alpha)
    b = complex(beta)
    w = _nh_work(C.device) if work is None else work
    if opA == _N and opB == _H and M * N <= _NH_MAX_OUT and M * N * batch * 16 <= w.numel():
        _lib.call("gwb_zgemm_nh", M, N, K, a.real, a.imag, _ptr(A, a_off), lda, sA, _ptr(B, b_off), ldb, sB,
                  b.real, b.imag, _ptr(C, c_off), ldc, sC, batch, w.data_ptr(), w.numel(), s)
        return
    _lib.call("gwb_zgemm", opA, opB, M, N, K, a.real, a.imag, _ptr(A, a_off), lda, sA, _ptr(B, b_off), ldb,
              sB, b.real, b.imag, _ptr(C, c_off), ldc, sC, batch, s)


class _PhaseTimer:
    """CUDA-event timing of the solver phases (``GWB_PROFILE=1``): events are
    recorded on the solve stream and read once at the end."""

    def __init__(self, on: bool):
        self.on = on
        self.events = []

    @contextlib.contextmanager
    def __call__(self, name: str):
        if not self.on:
            yield
            return
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record()
        try:
            yield
        finally:
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record()
            self.events.append((name, e0, e1))

    def summary(self) -> dict:
        if not self.events:
            return {}
        torch.cuda.synchronize()
        out: dict = {}
        for name, e0, e1 in self.events:
            out[name] = out.get(name, 0.0) + e0.elapsed_time(e1)
        return {k: round(v, 4) for k, v in sorted(out.items(), key=lambda kv: -kv[1])}


class _Workspace:
    """Device buffers of one solve (allocated once, reused every round)."""

    def __init__(self, nk, nb, npw, max_dim, dev, heev_max):
        c = dict(dtype=torch.complex128, device=dev)
        self.V = torch.zeros(nk, max_dim, npw, **c)
        self.HV = torch.zeros(nk, max_dim, npw, **c)
        self.S = torch.zeros(nk, max_dim, max_dim, **c)
        self.X = torch.zeros(nk, nb, npw, **c)
        self.HX = torch.zeros(nk, nb, npw, **c)
        self.R = torch.zeros(nk, nb, npw, **c)
        self.D = torch.zeros(nk, nb, npw, **c)
        self.D2 = torch.zeros(nk, nb, npw, **c)
        self.C = torch.zeros(nk * max_dim * max_dim, **c)
        self.G = torch.zeros(nk, nb, nb, **c)
        self.Linv = torch.zeros(nk, nb, nb, **c)
        self.rn = torch.zeros(nk, nb, dtype=torch.float64, device=dev)
        self.stats = torch.zeros(4, dtype=torch.float64, device=dev)
        self.flags = torch.zeros(1, dtype=torch.int32, device=dev)
        self.sel = torch.zeros(nk, nb, dtype=torch.int32, device=dev)
        self.info = torch.zeros(nk, dtype=torch.int32, device=dev)
        self.heev_info = torch.zeros(nk, dtype=torch.int32, device=dev)
        self.eig = torch.zeros(nk, nb, dtype=torch.float64, device=dev)
        hm = min(max_dim, heev_max)
        self.U = torch.zeros(nk, max(hm, nb), nb, **c)
        self.Z = torch.zeros(nk, int(_lib.load().gwb_heev_scratch_doubles(hm)), dtype=torch.float64, device=dev)
        self.Gs = torch.zeros(nk, nb, nb, **c)


class _Solver:
    def __init__(self, h_apply, x0, t, mask, tol, max_iter, max_dim_factor, mode, precond, history_out):
        if not x0.is_cuda:
            raise RuntimeError("davidson_batched (B200 path) needs CUDA tensors: there is no CPU fallback")
        if mode not in ("fp64", "fp32exp", "mixed"):
            raise ValueError(f"mode must be 'fp64', 'fp32exp' or 'mixed', got {mode!r}")
        self.h_apply = h_apply
        self.ham = getattr(h_apply, "__self__", None)
        if self.ham is not None and not hasattr(self.ham, "apply_into"):
            self.ham = None
        self.out_dtype = x0.dtype
        self.nk, self.nb, self.npw = (int(s) for s in x0.shape)
        self.dev = x0.device
        self.mask = mask.to(self.dev)
        self.t = t.to(self.dev, torch.float64).contiguous()
        self.tol = float(tol)
        self.max_iter = int(max_iter)
        self.max_dim = min(max_dim_factor * self.nb, int(self.mask.sum(dim=1).min()))
        if self.max_dim < self.nb:
            raise ValueError(f"basis of {self.max_dim} cannot hold {self.nb} bands")
        # a complex64 block is a low-precision draft: float32 applies throughout
        self.fp32_exp = mode in ("fp32exp", "mixed") and x0.dtype == torch.complex128
        self.mode = mode
        self.all_fp32 = x0.dtype == torch.complex64
        self.precond = precond
        self.history_out = history_out
        self.heev_max = int(_lib.load().gwb_heev_max_dim())
        self.ws = _Workspace(self.nk, self.nb, self.npw, self.max_dim, self.dev, self.heev_max)
        self.n_low = 0
        self.n_full = 0
        self.n_restart = 0
        self.n_cert = 0
        self.n_fallback_qr = 0
        self.n_repair = 0
        self.n_rollback = 0
        self.n_tc_fallback = 0
        self.breakdown = False
        self.mask_u8 = self.mask.to(torch.uint8).contiguous()
        self.stream = _lib.stream_ptr(self.dev)
        # scratch owned by this solve, so that solves on other streams (k
        # groups) never share it: split-K partial sums, tensor-core partials
        self.nh_work = torch.empty(24 << 20, dtype=torch.uint8, device=self.dev)
        self.tc_work = None
        self.x0 = x0
        self.prof = _PhaseTimer(os.environ.get("GWB_PROFILE", "0") == "1")
        # tensor-core first projection pass (float32-expansion modes): BF16
        # planes of the basis V, of the expansion block D and of D V^H
        self.tc = None
        self.tc_steps = _tc_steps() if mode in ("fp32exp", "mixed") and x0.dtype == torch.complex128 else frozenset()
        if self.tc_steps:
            from .tc import PlaneSet
            self.tc = (PlaneSet(self.nk, self.max_dim, self.npw, self.dev),
                       PlaneSet(self.nk, self.nb, self.npw, self.dev),
                       PlaneSet(self.nk, self.nb, self.max_dim, self.dev))

    # -- primitives -----------------------------------------------------------
    def zgemm(self, *args, **kw):
        kw.setdefault("work", self.nh_work)
        kw.setdefault("stream", self.stream)
        zgemm(*args, **kw)

    def apply_block(self, src: torch.Tensor, src_off: int, src_ks: int, nrows: int, dst: torch.Tensor,
                    dst_off: int, dst_ks: int, low: bool):
        """H on nrows rows of src (k stride src_ks) into dst rows (k stride dst_ks)."""
        n = self.nk * nrows
        if low:
            self.n_low += n
        else:
            self.n_full += n
        prec = _lib.GWB_FP32 if (low or self.all_fp32) else _lib.GWB_FP64
        if self.ham is not None:
            self.ham.apply_into(_ptr(src, src_off), src_ks, _ptr(dst, dst_off), dst_ks, nrows, prec,
                                n_rows_counted=n)
            return
        # generic callable: contiguous copy in, result copied out
        blk = src.view(-1)[src_off:].as_strided((self.nk, nrows, self.npw), (src_ks, self.npw, 1)).clone()
        if prec == _lib.GWB_FP32:
            out = self.h_apply(blk.to(torch.complex64)).to(torch.complex128)
        else:
            out = self.h_apply(blk)
        dview = dst.view(-1)[dst_off:].as_strided((self.nk, nrows, self.npw), (dst_ks, self.npw, 1))
        dview.copy_(out)

    def cholqr2(self, Y: torch.Tensor, n: int, Ytmp: torch.Tensor, Z: torch.Tensor | None = None,
                Ztmp: torch.Tensor | None = None, sync: bool = True, passes: int = 2):
        """Orthonormalise the first n rows of Y (nk, >=n, npw) in place by
        ``passes`` (default two) rounds of float64 Gram -> Cholesky -> L^-1 (Z,
        if given, gets the same row transform). With sync, a Cholesky breakdown
        is checked on the host and reported as False (Y untouched by the
        failing round); without, it only sets bit 1 of ws.flags, read with the
        next round's statistics."""
        ws, nk, npw = self.ws, self.nk, self.npw
        ys, zs = Y.shape[1] * npw, None if Z is None else Z.shape[1] * npw
        for _ in range(passes):
            self.zgemm(_N, _H, n, n, npw, Y, npw, ys, Y, npw, ys, ws.G, n, n * n, nk, stream=self.stream)
            if not self.chol_inv(n, sync):
                return False
            self.zgemm(_N, _N, n, npw, n, ws.Linv, n, n * n, Y, npw, ys, Ytmp, npw, Ytmp.shape[1] * npw, nk,
                  stream=self.stream)
            Y[:, :n].copy_(Ytmp[:, :n])
            if Z is not None:
                self.zgemm(_N, _N, n, npw, n, ws.Linv, n, n * n, Z, npw, zs, Ztmp, npw, Ztmp.shape[1] * npw, nk,
                      stream=self.stream)
                Z[:, :n].copy_(Ztmp[:, :n])
        return True

    def v_rows_changed(self, r0: int, r1: int):
        """Refresh the BF16 planes of basis rows [r0, r1) (tensor-core pass)."""
        if self.tc is not None and self.tc_steps & {"nh", "nn"} and r1 > r0:
            md, npw = self.max_dim, self.npw
            self.tc[0].write(self.ws.V, r1 - r0, row0=r0, src_ld=npw, src_kstride=md * npw, offset=r0 * npw,
                             stream=self.stream)

    def project_tc(self, n: int, m: int) -> bool:
        """D -= (D V^H) V over the first m basis rows as split-BF16
        tensor-core products (error ~1e-6 of the unit input rows; a float64
        pass follows). A row that keeps less than 1e-2 of its norm would be
        dominated by that error (near-converged bands whose corrections lie
        almost in the basis), so then the whole block is redone with the
        float64 pass from a saved copy (checked on the host). False if so."""
        from .tc import OP_H, OP_N, work_bytes, zgemm_tc
        pv, pd, pc = self.tc
        ws, npw = self.ws, self.npw
        ds = ws.D.shape[1] * npw
        need = work_bytes(OP_H, n, m, npw, self.nk)
        if self.tc_work is None or self.tc_work.numel() < need:
            self.tc_work = torch.empty(max(need, 1 << 20), dtype=torch.uint8, device=self.dev)
        md = self.max_dim
        ws.D2[:, :n].copy_(ws.D[:, :n])
        if "nh" in self.tc_steps:
            pd.write(ws.D, n, src_ld=npw, src_kstride=ds, stream=self.stream)
            zgemm_tc(OP_H, n, m, npw, pd, pv, ws.C, m, n * m, stream=self.stream, status=ws.flags,
                     work=self.tc_work)
        else:
            self.zgemm(_N, _H, n, m, npw, ws.D, npw, ds, ws.V, npw, md * npw, ws.C, m, n * m, self.nk)
        if "nn" in self.tc_steps:
            pc.write(ws.C, n, src_ld=m, src_kstride=n * m, cols=m, stream=self.stream)
            zgemm_tc(OP_N, n, npw, m, pc, pv, ws.D, npw, ds, alpha=-1.0, beta=1.0, stream=self.stream,
                     status=ws.flags, work=self.tc_work)
        else:
            self.zgemm(_N, _N, n, npw, m, ws.C, m, n * m, ws.V, npw, md * npw, ws.D, npw, ds, self.nk, alpha=-1.0,
                       beta=1.0)
        if float(torch.linalg.vector_norm(ws.D[:, :n], dim=-1).min()) < 1e-2:
            ws.D[:, :n].copy_(ws.D2[:, :n])
            self.project_out(ws.D, n, m, passes=1)
            self.n_tc_fallback += 1
            return False
        return True

    def chol_inv(self, n: int, sync: bool) -> bool:
        """ws.Linv[:n, :n] = L^-1 for the Cholesky factor L of ws.G (both as
        (nk, n, n) with ld n). Up to 64 columns the libgwb.so kernel (the Gram
        matrix in shared memory, one CTA per k); above that cuSOLVER's Cholesky
        and triangular solve (the one-CTA kernel is latency-bound there: 49 ms
        against 2 ms at n = 480). With sync a breakdown returns False; without,
        it sets bit 1 of ws.flags."""
        ws, nk = self.ws, self.nk
        if n <= 64:
            _lib.call("gwb_chol_inv", nk, n, _ptr(ws.G), n, n * n, _ptr(ws.Linv), n * n, _ptr(ws.info),
                      None if sync else _ptr(ws.flags), self.stream)
            return not sync or int(ws.info.max()) == 0
        G = ws.G.view(-1)[: nk * n * n].view(nk, n, n)
        L, info = torch.linalg.cholesky_ex(G)
        Li = ws.Linv.view(-1)[: nk * n * n].view(nk, n, n)
        eye = torch.eye(n, dtype=G.dtype, device=G.device).expand(nk, n, n)
        Li.copy_(torch.linalg.solve_triangular(L, eye, upper=False))
        if sync:
            return int(info.max()) == 0
        ws.flags.bitwise_or_((info.amax() != 0).to(torch.int32) * 2)
        return True

    def cholqr_tc(self, n: int) -> bool:
        """One Cholesky-QR round of D[:, :n] as split-BF16 tensor-core products:
        Gram D D^H (FP32-accumulated, summed in float64), float64 Cholesky and
        triangular inverse, D <- L^-1 D. Leaves D nearly orthonormal (to about
        1e-6 kappa(D)^2) for the float64 round that follows; False, with D
        untouched, when the Cholesky breaks down (checked on the host)."""
        from .tc import OP_H, OP_N, work_bytes, zgemm_tc
        _, pd, pc = self.tc
        ws, nk, npw = self.ws, self.nk, self.npw
        ds = ws.D.shape[1] * npw
        need = work_bytes(OP_H, n, n, npw, nk)
        if self.tc_work is None or self.tc_work.numel() < need:
            self.tc_work = torch.empty(max(need, 1 << 20), dtype=torch.uint8, device=self.dev)
        # unit rows first, so the FP32-accumulated Gram matrix resolves every
        # row to the same relative accuracy
        blk = ws.D[:, :n]
        blk.div_(torch.linalg.vector_norm(blk, dim=-1, keepdim=True))
        pd.write(ws.D, n, src_ld=npw, src_kstride=ds, stream=self.stream)
        zgemm_tc(OP_H, n, n, npw, pd, pd, ws.G, n, n * n, stream=self.stream, status=ws.flags, work=self.tc_work)
        if not self.chol_inv(n, sync=True):
            self.n_tc_fallback += 1
            return False
        # unit rows: 1 / L_ii is the inverse distance of row i from the span
        # of the rows before it; above 100 the BF16 error of the block,
        # amplified by L^-1, would swamp the new directions
        Li = ws.Linv.view(-1)[: nk * n * n].view(nk, n, n)
        if float(torch.diagonal(Li, dim1=-2, dim2=-1).abs().max()) > 1e2:
            self.n_tc_fallback += 1
            return False
        pc.write(ws.Linv, n, src_ld=n, src_kstride=n * n, cols=n, stream=self.stream)
        zgemm_tc(OP_N, n, npw, n, pc, pd, ws.D, npw, ds, stream=self.stream, status=ws.flags, work=self.tc_work)
        return True

    def project_out(self, Dblk: torch.Tensor, n: int, m: int, passes: int = 2):
        """D -= (D V^H) V over the first m basis rows (float64 GEMMs)."""
        ws, nk, npw, md = self.ws, self.nk, self.npw, self.max_dim
        ds = Dblk.shape[1] * npw
        for _ in range(passes):
            self.zgemm(_N, _H, n, m, npw, Dblk, npw, ds, ws.V, npw, md * npw, ws.C, m, n * m, nk,
                  stream=self.stream)
            self.zgemm(_N, _N, n, npw, m, ws.C, m, n * m, ws.V, npw, md * npw, Dblk, npw, ds, nk, alpha=-1.0,
                  beta=1.0, stream=self.stream)

    def orthonormalize_new(self, n: int, m: int, safe: bool = False):
        """Rows D[:, :n] -> orthonormal, orthogonal to V[:, :m] (reference
        ``_orthonormalize_b``, gradwave solvers/davidson.py:406-457).

        Default (no host synchronisation): projection, device rank repair of
        vanished rows, second projection, CholQR2; a breakdown is only flagged
        and the caller rolls the expansion back. ``safe``: the reference's
        order with host checks - two projections, seeded jitter of vanished
        rows, re-projection, CholQR2 with Householder QR on breakdown."""
        ws = self.ws
        D = ws.D
        D[:, :n].mul_(self.mask[:, None, :])
        if not safe:
            if m:
                if self.tc_steps & {"nh", "nn"}:
                    self.project_tc(n, m)
                else:
                    self.project_out(D, n, m, passes=1)
            _lib.call("gwb_row_repair", self.nk, n, self.npw, _ptr(D), D.shape[1] * self.npw,
                      _ptr(self.mask_u8), 1e-8, _ptr(ws.flags), self.stream)
            # tensor-core Cholesky-QR round before the float64 projection, so
            # that the float64 pass still sets the orthogonality to the basis;
            # one float64 Cholesky-QR round then finishes the block
            tc_round = "chol" in self.tc_steps and self.cholqr_tc(n)
            if m:
                self.project_out(D, n, m, passes=1)
            self.cholqr2(D, n, ws.D2, sync=False, passes=1 if tc_round else 2)
            return
        if m:
            self.project_out(D, n, m)
        if self.cholqr2(D, n, ws.D2):
            return
        self.n_fallback_qr += 1
        blk = D[:, :n]
        bad = torch.linalg.vector_norm(blk, dim=-1, keepdim=True) < 1e-8
        if bool(bad.any()):
            gen = torch.Generator(device="cpu").manual_seed(n + 7919)
            noise = torch.randn(self.nk, n, self.npw, 2, generator=gen, dtype=torch.float64)
            jit = torch.view_as_complex(noise).to(self.dev)
            blk.add_(bad * jit).mul_(self.mask[:, None, :])
            if m:
                self.project_out(D, n, m)
        q, _ = torch.linalg.qr(D[:, :n].transpose(-1, -2), mode="reduced")
        D[:, :n].copy_(q.transpose(-1, -2))

    def rayleigh_ritz(self, m: int, m0: int):
        """Update s (new columns m0..m-1), eigensolve, Ritz block X/HX, residuals."""
        ws, nk, npw, nb, md = self.ws, self.nk, self.npw, self.nb, self.max_dim
        nnew = m - m0
        if nnew > 0:
            with self.prof("subspace_gemm"):
                self.zgemm(_N, _H, m, nnew, npw, ws.V, npw, md * npw, ws.HV, npw, md * npw, ws.C, nnew, m * nnew, nk,
                      b_off=m0 * npw, stream=self.stream)
                _lib.call("gwb_subspace_insert", nk, m, m0, _ptr(ws.C), _ptr(ws.S), md, md * md, self.stream)
        with self.prof("eigh"):
            eig, u, ldu = self.eigh(m)
        with self.prof("ritz_gemm"):
            self.zgemm(_T, _N, nb, npw, m, u, ldu, m * ldu, ws.V, npw, md * npw, ws.X, npw, nb * npw, nk,
                  stream=self.stream)
            self.zgemm(_T, _N, nb, npw, m, u, ldu, m * ldu, ws.HV, npw, md * npw, ws.HX, npw, nb * npw, nk,
                  stream=self.stream)
        with self.prof("residual"):
            self.residuals(eig)
        return eig

    def eigh(self, m: int, S=None, lds=None):
        """Lowest nb eigenpairs of the Hermitian matrices S[:, :m, :m]:
        eigenvalues (nk, nb) and a row-major block U (nk, m, ldu) whose first nb
        columns are the eigenvectors. The batched libgwb.so eigensolver runs
        for m <= gwb_heev_max_dim(); larger subspaces use cuSOLVER (through
        torch.linalg.eigh). A QL failure is flagged in ws.info and caught by the
        next statistics read."""
        ws, nk, nb = self.ws, self.nk, self.nb
        S = ws.S if S is None else S
        lds = self.max_dim if lds is None else lds
        opcount.bump("eigh")
        if m <= self.heev_max:
            _lib.call("gwb_heev_lowest", nk, m, nb, _ptr(S), lds, S.shape[1] * S.shape[2], _ptr(ws.eig),
                      _ptr(ws.U), _ptr(ws.Z), _ptr(ws.heev_info), self.stream)
            return ws.eig[:, :nb], ws.U, nb
        w, u = torch.linalg.eigh(S[:, :m, :m])
        return w[:, :nb].contiguous(), u.contiguous(), m

    def residuals(self, eig):
        ws, nk, nb, npw = self.ws, self.nk, self.nb, self.npw
        _lib.call("gwb_residual", nk, nb, npw, _ptr(ws.X), nb * npw, _ptr(ws.HX), nb * npw, _ptr(eig), nb,
                  _ptr(ws.R), nb * npw, _ptr(ws.rn), self.stream)

    def certify(self):
        """Float64 refresh of the Ritz block (reference ``_certify_fp64``,
        gradwave solvers/davidson.py:287-308)."""
        ws, nk, nb, npw = self.ws, self.nk, self.nb, self.npw
        self.n_cert += 1
        self.apply_block(ws.X, 0, nb * npw, nb, ws.HX, 0, nb * npw, low=False)
        self.zgemm(_N, _H, nb, nb, npw, ws.X, npw, nb * npw, ws.HX, npw, nb * npw, ws.G, nb, nb * nb, nk,
              stream=self.stream)
        s = ws.G.conj()
        ws.Gs.copy_(0.5 * (s + s.conj().transpose(-1, -2)))
        eig, u, ldu = self.eigh(nb, ws.Gs, nb)
        eig = eig.clone()
        self.zgemm(_T, _N, nb, npw, nb, u, ldu, nb * ldu, ws.X, npw, nb * npw, ws.D2, npw, nb * npw, nk,
              stream=self.stream)
        ws.X.copy_(ws.D2)
        self.zgemm(_T, _N, nb, npw, nb, u, ldu, nb * ldu, ws.HX, npw, nb * npw, ws.D2, npw, nb * npw, nk,
              stream=self.stream)
        ws.HX.copy_(ws.D2)
        self.residuals(eig)
        return eig

    def read_stats(self):
        """(max |r|, n_add) from the device in one small read; raises if the
        eigensolver flagged a QL failure this round."""
        _lib.call("gwb_conv_stats", self.nk, self.nb, _ptr(self.ws.rn), self.tol, _ptr(self.ws.stats),
                  self.stream)
        ws = self.ws
        ws.stats[2] = ws.heev_info.max()
        ws.stats[3] = ws.flags[0]
        ws.flags.zero_()
        st = ws.stats.tolist()
        if st[2] != 0:
            raise _lib.GwbError(_lib.GWB_ERR_NOT_CONVERGED, "subspace eigensolver: QL iteration limit")
        flags = int(st[3])
        if flags & _lib.GWB_ERR_TIMEOUT:
            raise _lib.GwbError(_lib.GWB_ERR_TIMEOUT, "tensor-core projection: a bounded pipeline wait ran out")
        if flags & 1:
            self.n_repair += 1
        self.breakdown = bool(flags & 2)
        return st[0], int(st[1])

    # -- the solve --------------------------------------------------------------
    def run(self) -> BatchedDavidsonResult:
        ws, nk, nb, npw, md = self.ws, self.nk, self.nb, self.npw, self.max_dim
        ws.D[:, :nb].copy_(self.x0.to(torch.complex128))
        self.orthonormalize_new(nb, 0, safe=True)
        ws.V[:, :nb].copy_(ws.D[:, :nb])
        self.v_rows_changed(0, nb)
        self.apply_block(ws.V, 0, md * npw, nb, ws.HV, 0, md * npw, low=self.fp32_exp)
        # m: basis rows in use; m0: first column of s not formed yet (0 = rebuild)
        m, m0 = nb, 0
        m_prev = m
        safe_next = False
        cert_floor = _FP32_CERT_FLOOR_EPS * max(float(self.t.max()), 1.0) if self.fp32_exp else 0.0
        prev_rnmax = math.inf
        eig = None
        it = 0
        while it < self.max_iter:
            it += 1
            eig = self.rayleigh_ritz(m, m0)
            m0 = m
            with self.prof("stats_sync"):
                rnmax, n_add = self.read_stats()
            if self.breakdown:
                # the last expansion block lost rank in CholQR2: drop it, redo
                # this round on the previous basis, orthonormalise safely
                self.n_rollback += 1
                m = m0 = m_prev
                safe_next = True
                it -= 1
                continue
            if self.fp32_exp:
                gated = self.mode == "fp32exp" or rnmax < 100.0 * cert_floor
                stalled = it > 1 and rnmax > _FP32_CERT_STALL * prev_rnmax and gated
                prev_rnmax = rnmax
                if rnmax < max(self.tol, cert_floor) or stalled:
                    with self.prof("certify"):
                        eig = self.certify()
                        rnmax, n_add = self.read_stats()
                    if rnmax >= self.tol:
                        # hand-off: collapse to the certified block with exact
                        # images and continue with float64 expansion applies
                        ws.V[:, :nb].copy_(ws.X)
                        ws.HV[:, :nb].copy_(ws.HX)
                        self.v_rows_changed(0, nb)
                        m, m0 = nb, 0
                        self.fp32_exp = False
            if self.history_out is not None:
                self.history_out.append((it, ws.rn.cpu().clone(), eig.cpu().clone()))
            if rnmax < self.tol:
                return self.result(eig, it)
            with self.prof("precond"):
                _lib.call("gwb_select_worst", nk, nb, _ptr(ws.rn), n_add, _ptr(ws.sel), self.stream)
                self.precondition(n_add, eig)
            if m + n_add > md:
                # restart: re-orthonormalise the Ritz block, images by the same
                # transform (no re-application), keep the new directions
                self.n_restart += 1
                with self.prof("restart"):
                    restart_ok = self.cholqr2(ws.X, nb, ws.D2, ws.HX, ws.R)
                if not restart_ok:
                    q, r = torch.linalg.qr(ws.X.transpose(-1, -2), mode="reduced")
                    ws.X.copy_(q.transpose(-1, -2))
                    ws.HX.copy_(torch.linalg.solve_triangular(r.transpose(-1, -2), ws.HX, upper=False))
                ws.V[:, :nb].copy_(ws.X)
                ws.HV[:, :nb].copy_(ws.HX)
                self.v_rows_changed(0, nb)
                m, m0 = nb, 0
            with self.prof("orthonormalize"):
                self.orthonormalize_new(n_add, m, safe=safe_next)
                safe_next = False
                ws.V[:, m:m + n_add].copy_(ws.D[:, :n_add])
                self.v_rows_changed(m, m + n_add)
            with self.prof("apply"):
                self.apply_block(ws.V, m * npw, md * npw, n_add, ws.HV, m * npw, md * npw, low=self.fp32_exp)
            m_prev = m
            m += n_add
        if self.fp32_exp:
            eig = self.certify()
        if logger.isEnabledFor(logging.DEBUG):
            logger.debug("batched Davidson hit max_iter=%d (max res=%.3e > tol=%.1e)", self.max_iter,
                         float(ws.rn.max()), self.tol)
        return self.result(eig, self.max_iter)

    def precondition(self, n_add: int, eig: torch.Tensor):
        """D[:, :n_add] = preconditioned, unit-normalised worst residuals."""
        ws, nk, nb, npw = self.ws, self.nk, self.nb, self.npw
        if self.precond is None or (isinstance(self.precond, str) and self.precond == "teter"):
            _lib.call("gwb_precond_teter", nk, nb, n_add, npw, _ptr(ws.X), nb * npw, _ptr(ws.R), nb * npw,
                      _ptr(self.t), _ptr(ws.sel), _ptr(ws.D), nb * npw, self.stream)
        else:
            self.precond.apply_into(self, n_add, eig)

    def result(self, eig, it) -> BatchedDavidsonResult:
        ws = self.ws
        x = ws.X.clone()
        if self.out_dtype != torch.complex128:
            x = x.to(self.out_dtype)
        info = {"n_restart": self.n_restart, "n_cert": self.n_cert, "n_fallback_qr": self.n_fallback_qr,
                "tc_projection": self.tc is not None, "tc_steps": sorted(self.tc_steps),
                "n_tc_fallback": self.n_tc_fallback,
                "n_repair": self.n_repair, "n_rollback": self.n_rollback,
                "max_dim": self.max_dim, "phase_ms": self.prof.summary()}
        return BatchedDavidsonResult(eig.clone(), x, it, ws.rn.clone(), self.n_low, self.n_full, info)


def _native_solve(ham, x0, t, mask, tol, max_iter, max_dim, mode, time_applies=False, model=None
                  ) -> BatchedDavidsonResult | None:
    """The whole solve inside libgwb.so (``gwb_davidson_solve`` through the
    custom op ``gwb::davidson_solve``); None when the library reports a
    breakdown it does not repair (the host driver retries)."""
    from .ops import SOLVE_MODES, SOLVE_STATS, SOLVE_TIME_APPLIES
    try:
        eig, vec, rn, stats = torch.ops.gwb.davidson_solve(
            ham.handle, x0.contiguous(), t, mask, float(tol), int(max_iter), int(max_dim), SOLVE_MODES[mode],
            SOLVE_TIME_APPLIES if time_applies else 0, model)
    except Exception as e:  # the dispatcher may re-wrap the library's GwbError
        if getattr(e, "status", None) == _lib.GWB_ERR_BREAKDOWN or f"libgwb status {_lib.GWB_ERR_BREAKDOWN} " in str(e):
            logger.debug("native Davidson: %s; retrying on the host driver", e)
            return None
        raise
    st = dict(zip(SOLVE_STATS, stats.tolist()))
    n_low, n_full = int(st["n_apply_low"]), int(st["n_apply_full"])
    ham._count_rows(n_low + n_full)
    info = {"n_restart": int(st["n_restart"]), "n_cert": int(st["n_cert"]), "n_repair": int(st["n_repair"]),
            "n_rollback": int(st["n_rollback"]), "max_dim": max_dim, "native": True,
            "n_apply_calls": int(st["n_apply_calls"]), "n_tpa_fallback": int(st["n_tpa_fallback"])}
    if time_applies:
        info["apply_ms"] = float(st["apply_ms"])
    return BatchedDavidsonResult(eig, vec, int(st["n_iter"]), rn, n_low, n_full, info)


_TC_STEP_NAMES = ("nh", "nn", "chol")


def _tc_steps() -> frozenset:
    """Steps of the float32-expansion modes' orthonormalisation that run as
    tensor-core products: ``nh`` the coefficients D V^H of the first
    projection pass, ``nn`` its update D -= C V, ``chol`` the first
    Cholesky-QR round. ``GWB_TC_PROJECT=0`` turns all off; ``GWB_TC_STEPS`` (a
    comma list) picks a subset. The default is the projection pass (nh, nn):
    the tensor-core Cholesky-QR round perturbs the new directions by the BF16
    error amplified by L^-1, and on the 64-atom cell that let one band stall
    just above tolerance until the next restart (192-235 rounds against 64-75
    without it), for a saving of two n x n x npw products per round."""
    if os.environ.get("GWB_TC_PROJECT", "1") == "0":
        return frozenset()
    if os.environ.get("GWB_TC_PROJECT", "1") != "1":
        raise ValueError("GWB_TC_PROJECT must be 0 or 1")
    v = os.environ.get("GWB_TC_STEPS")
    if v is None:
        return frozenset(("nh", "nn"))
    steps = frozenset(x.strip() for x in v.split(",") if x.strip())
    if not steps <= set(_TC_STEP_NAMES):
        raise ValueError(f"GWB_TC_STEPS must name steps among {_TC_STEP_NAMES}")
    return steps


def _k_groups(default: int) -> int:
    """Number of concurrent k-groups of a solve (``GWB_KGROUPS``, else
    ``default``)."""
    v = os.environ.get("GWB_KGROUPS")
    if v is None:
        return default
    try:
        return max(1, int(v))
    except ValueError:
        raise ValueError("GWB_KGROUPS must be a positive integer") from None


def _solve_grouped(ham, x0, t, mask, tol, max_iter, max_dim_factor, mode, groups, *, native, time_applies=False,
                   model=None, precond="teter"):
    """The k-points split into contiguous groups balanced by plane-wave count,
    each solved from its own host thread on its own CUDA stream, by the native
    driver (``native``) or by the host driver. Every k is an independent
    eigenproblem, so the groups need no communication; running them side by
    side lets one group's latency-bound steps (the per-k subspace eigensolver)
    overlap another group's bandwidth-bound applies and products on the same
    GPU. Each group keeps the reference's uniform-subspace rule inside itself.
    None when a native group reports an unrepaired breakdown (the caller
    retries on the host)."""
    import threading
    from .sharding import shard_range_weighted
    nk, nb = int(x0.shape[0]), int(x0.shape[1])
    g_n = min(groups, nk)
    cost = mask.sum(dim=1).to("cpu", torch.float64).numpy()
    ranges = [shard_range_weighted(cost, g, g_n) for g in range(g_n)]
    dev = x0.device
    main = torch.cuda.current_stream(dev)
    streams = ham.__dict__.setdefault("_group_streams", {})
    for g in range(g_n):
        if g not in streams:
            streams[g] = torch.cuda.Stream(device=dev)
    subs = [ham.k_slice(s, e) for s, e in ranges]
    results: list = [None] * g_n
    errors: list = [None] * g_n

    def work(g):
        try:
            s, e = ranges[g]
            with torch.cuda.device(dev), torch.cuda.stream(streams[g]), torch.no_grad():
                if native:
                    md = min(max_dim_factor * nb, int(mask[s:e].sum(dim=1).min()))
                    results[g] = _native_solve(subs[g], x0[s:e], t[s:e], mask[s:e], tol, max_iter, md, mode,
                                               time_applies=time_applies, model=model)
                else:
                    results[g] = _Solver(subs[g].apply, x0[s:e], t[s:e], mask[s:e], tol, max_iter, max_dim_factor,
                                         mode, precond, None).run()
        except BaseException as exc:  # re-raised on the caller's thread
            errors[g] = exc

    if not native:
        # torch loads its CUDA linear-algebra backend lazily on the first call,
        # which must not happen from several threads at once
        a = torch.eye(2, dtype=torch.complex128, device=dev)
        torch.linalg.eigh(a)
        torch.linalg.qr(a)
        torch.linalg.solve_triangular(torch.linalg.cholesky_ex(a)[0], a, upper=False)
    for g in range(g_n):
        streams[g].wait_stream(main)
    threads = [threading.Thread(target=work, args=(g,)) for g in range(g_n)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    for g in range(g_n):
        main.wait_stream(streams[g])
    for exc in errors:
        if exc is not None:
            raise exc
    if any(r is None for r in results):
        return None
    for r in results:  # the group outputs are read on the caller's stream from here on
        for x in (r.eigenvalues, r.eigenvectors, r.residual_norms):
            x.record_stream(main)
    info = {"native": native, "k_groups": g_n, "max_dim": max(r.info["max_dim"] for r in results)}
    for key in ("n_restart", "n_cert", "n_repair", "n_rollback", "n_apply_calls", "apply_ms", "n_fallback_qr",
                "n_tc_fallback"):
        if key in results[0].info:
            info[key] = sum(r.info[key] for r in results)
    if "tc_projection" in results[0].info:
        info["tc_projection"] = results[0].info["tc_projection"]
    if results[0].info.get("phase_ms"):
        # per-phase event times summed over the groups (which overlap in time)
        ph: dict = {}
        for r in results:
            for k, v in r.info.get("phase_ms", {}).items():
                ph[k] = round(ph.get(k, 0.0) + v, 4)
        info["phase_ms"] = dict(sorted(ph.items(), key=lambda kv: -kv[1]))
    return BatchedDavidsonResult(torch.cat([r.eigenvalues for r in results]),
                                 torch.cat([r.eigenvectors for r in results]),
                                 max(r.n_iter for r in results),
                                 torch.cat([r.residual_norms for r in results]),
                                 sum(r.n_apply_low for r in results), sum(r.n_apply_full for r in results), info)


def davidson_batched(h_apply, x0, t, mask, tol: float = 1e-9, max_iter: int = 40, max_dim_factor: int = 4,
                     sync_free: bool = False, history_out=None, *, mode: str = "fp64",
                     precond="teter") -> BatchedDavidsonResult:
    """Batched block Davidson (see module docstring).

    When ``h_apply`` is ``BatchedHamiltonian.apply`` of this package, the
    block is complex128, the preconditioner is TPA, no history is requested and
    the basis fits the batched eigensolver, the whole solve runs natively in
    libgwb.so (``gwb_davidson_solve``); otherwise this module's host driver
    runs the same steps kernel by kernel. ``GWB_NATIVE=0`` forces the host
    driver. ``sync_free`` is accepted for signature parity and ignored (every
    round reads four device scalars, like the reference's synchronous path)."""
    if mode not in ("fp64", "fp32exp", "mixed"):
        raise ValueError(f"mode must be 'fp64', 'fp32exp' or 'mixed', got {mode!r}")
    with torch.no_grad():
        ham = getattr(h_apply, "__self__", None)
        max_dim = min(max_dim_factor * int(x0.shape[1]), int(mask.sum(dim=1).min()))
        native = (os.environ.get("GWB_NATIVE", "1") != "0" and ham is not None
                  and getattr(h_apply, "__func__", None) is getattr(type(ham), "apply", None)
                  and hasattr(ham, "_native_workspace") and x0.is_cuda and x0.dtype == torch.complex128
                  and (precond is None or (isinstance(precond, str) and precond == "teter")
                       or hasattr(precond, "params"))
                  and history_out is None and int(x0.shape[1]) <= max_dim <= int(_lib.load().gwb_heev_max_dim()))
        nk = int(x0.shape[0])
        if native:
            time_applies = os.environ.get("GWB_TIME_APPLIES", "0") == "1"
            model = getattr(precond, "params", None)
            # one group by default: two concurrent groups were ~5 % faster on
            # si8 but change the rounds' trajectory (each group keeps its own
            # uniform subspace), and in one such trajectory the learned fp64
            # solve missed an eigenvalue by 0.72 eV
            groups = _k_groups(1)
            if groups > 1 and nk > 1 and hasattr(ham, "k_slice"):
                res = _solve_grouped(ham, x0, t, mask, tol, max_iter, max_dim_factor, mode, groups, native=True,
                                     time_applies=time_applies, model=model)
            else:
                res = _native_solve(ham, x0, t, mask, tol, max_iter, max_dim, mode, time_applies=time_applies,
                                    model=model)
            if res is not None:
                return res
        # host driver: a basis beyond the batched eigensolver goes to cuSOLVER,
        # one matrix at a time, so by default every k (up to 8) gets its own
        # group and the eigensolves of different k overlap
        own_apply = ham is not None and getattr(h_apply, "__func__", None) is getattr(type(ham), "apply", None)
        groups = _k_groups(min(nk, 8) if max_dim > int(_lib.load().gwb_heev_max_dim()) else 1)
        if (groups > 1 and nk > 1 and own_apply and hasattr(ham, "k_slice") and history_out is None
                and x0.is_cuda and x0.dtype == torch.complex128):
            res = _solve_grouped(ham, x0, t, mask, tol, max_iter, max_dim_factor, mode, groups, native=False,
                                 precond=precond)
            if res is not None:
                return res
        if not bool(torch.isfinite(torch.view_as_real(x0) if x0.is_complex() else x0).all()):
            raise _lib.GwbError(_lib.GWB_ERR_NONFINITE, "the start block holds a non-finite value")
        return _Solver(h_apply, x0, t, mask, tol, max_iter, max_dim_factor, mode, precond, history_out).run()


LOW = torch.complex64  # the draft dtype of the two-stage schedule


def mixed_precision_solve(x0, tol, crossover, mixed_precision, *, full, make_stages):
    """Draft -> polish scaffold (gradwave ``solvers/_ms.py:26-52``): a single
    full-precision solve when mixed precision is off, x0 is already complex64
    or crossover >= tol; otherwise draft at complex64 to ``crossover`` and
    polish at x0's precision to ``tol`` from the drafted vectors."""
    if (not mixed_precision) or x0.dtype == LOW or crossover >= tol:
        return full()
    hi = x0.dtype
    draft, polish = make_stages()
    d = draft(x0.to(LOW))
    return polish(d.eigenvectors.to(hi))


def davidson_batched_ms(h_apply, x0, t, mask, tol: float = 1e-9, max_iter: int = 40, max_dim_factor: int = 4,
                        crossover: float = 1e-5, mixed_precision: bool = True) -> BatchedDavidsonResult:
    """Two-stage Davidson (gradwave ``solvers/davidson.py:778-812``): a
    complex64 draft (float32 applies) to ``crossover``, then a full-precision
    polish to ``tol`` warm-started from it."""

    def solve(x, tl):
        return davidson_batched(h_apply, x, t, mask, tol=tl, max_iter=max_iter, max_dim_factor=max_dim_factor)

    return mixed_precision_solve(x0, tol, crossover, mixed_precision,
                                 full=lambda: solve(x0, tol),
                                 make_stages=lambda: (lambda xlo: solve(xlo, crossover),
                                                      lambda x1: solve(x1, tol)))
