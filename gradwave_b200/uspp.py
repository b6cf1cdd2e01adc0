"""Generalized (USPP/PAW) band solve H x = eps S x on the B200 path: drop-in
for gradwave's ``scf/uspp_batch.py`` (``BatchedHS``, ``davidson_gen_batched``).

The overlap S = 1 + sum_pq |beta_p> q_pq <beta_q| shares the projector
contraction <beta|c> with the nonlocal part of H. ``BatchedHS`` therefore
keeps one libgwb handle holding D and q, and ``gwb_ham_apply_hs`` returns H c
and S c from a single pass: the FFT local term into the H output, one becp
contraction, then a projector sweep that adds (becp D) P to H c and writes
c + (becp q) P as S c (masked).

``davidson_gen_batched`` is a host driver over the package's own kernels. It
keeps the reference's order of steps, which fixes its eigenpairs:

1. the subspace pencil (V HV^H, V SV^H), grown by its new columns only
   (split-K products and ``gwb_subspace_insert``);
2. the Cholesky factor of the overlap block with its inverse
   (``gwb_chol_inv``). While it breaks down the oldest basis rows leave the
   window, down to nbands + 1 rows, then a 1e-10 diagonal shift (an
   indefinite S on a truncated sphere, ``scf/uspp_batch.py:155-185``);
3. the reduced matrix L^-1 H L^-H from two split-K products, its lowest
   eigenpairs (``gwb_heev_lowest``) and the pencil's vectors L^-H U;
4. the Ritz block X, HX, SX and the residuals HX - eps SX (``gwb_residual``
   with SX in place of X);
5. the worst max_k #(|r| > tol) residuals of every k (``gwb_select_worst``),
   TPA-filtered with the band's kinetic energy and unit-normalised
   (``gwb_precond_teter``);
6. past the basis cap, a restart to the Ritz block made orthonormal in the
   standard metric (two Cholesky-QR rounds) with HX and SX carried by the
   same triangular factors (no re-application);
7. the new directions orthogonalised in the standard metric: mask, two
   projections against the window, device rank repair of vanished rows,
   Cholesky-QR twice;
8. one fused H/S apply of the new rows straight into the image buffers.

The basis and both image blocks live in preallocated (nk, max_dim, npw)
buffers. The host reads three small values per round: the Cholesky status,
the convergence statistics and the rank-repair flag.
"""

from __future__ import annotations

import torch

from . import _lib
from .basis import BatchedK
from .davidson import _H, _N, _T, _ptr, zgemm
from .hamiltonian import BatchedHamiltonian


class BatchedHS:
    """H and S of all k on one handle: ``h(c)``, ``s(c)`` and ``hs(c)``
    (both from one pass), in the arithmetic of c's dtype. ``dscr`` is the
    screened D that replaces the bare one; ``q_full`` the (nproj, nproj)
    augmentation matrix (real symmetric; a complex array must have a zero
    imaginary part). DFT+U, the dual grid and meta-GGA raise."""

    def __init__(self, bk, shape, v_eff_r, p, dscr, q_full, hub_sphi=None, hub_d=None, smooth=None,
                 metagga_v=None):
        if hub_sphi is not None or hub_d is not None or smooth is not None or metagga_v is not None:
            raise NotImplementedError("DFT+U, the dual grid and meta-GGA are not part of the B200 band-solve path")
        q = torch.as_tensor(q_full)
        if q.is_complex():
            if float(q.imag.abs().max()) != 0.0:
                raise ValueError("the augmentation matrix q must be real")
            q = q.real
        self.bk = bk
        self.shape = tuple(int(s) for s in shape)
        bks = BatchedK(bk.npw, bk.mask, bk.flat_idx, bk.kpg, bk.t, bk.proj_phase_free, bk.proj_atom_index,
                       torch.as_tensor(dscr, dtype=torch.float64))
        self.ham = BatchedHamiltonian(bks, self.shape, v_eff_r, p)
        dev = self.ham.device
        nproj = self.ham.nproj
        if tuple(q.shape) != (nproj, nproj):
            raise ValueError(f"q must be ({nproj}, {nproj}), got {tuple(q.shape)}")
        self.q = q.to(dev, torch.float64).contiguous()
        self.mask = bk.mask.to(dev)
        self.t = bk.t.to(dev, torch.float64).contiguous()
        with torch.cuda.device(dev):
            _lib.call("gwb_ham_set_overlap", self.ham._h, self.q.data_ptr() if nproj else None,
                      _lib.stream_ptr(dev))

    @property
    def device(self):
        return self.ham.device

    def h(self, c: torch.Tensor) -> torch.Tensor:
        return self.ham.apply(c)

    def s(self, c: torch.Tensor) -> torch.Tensor:
        return self.hs(c)[1]

    def hs(self, c: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """(H c, S c) from one pass, masked, in the arithmetic of c's dtype."""
        self.ham._check(c)
        c = c.contiguous()
        out_h, out_s = torch.empty_like(c), torch.empty_like(c)
        nb = int(c.shape[1])
        ks = nb * self.ham.npw_max
        prec = _lib.GWB_FP64 if c.dtype == torch.complex128 else _lib.GWB_FP32
        self.ham._count_rows(self.ham.nk * nb)
        _lib.call("gwb_ham_apply_hs", self.ham._h, c.data_ptr(), ks, out_h.data_ptr(), ks, out_s.data_ptr(), ks, nb,
                  _lib.io_dtype(c), prec, _lib.stream_ptr(self.device))
        return out_h, out_s

    def hs_into(self, src, src_off: int, src_ks: int, hdst, sdst, dst_off: int, dst_ks: int, nrows: int) -> None:
        """H and S of nrows complex128 rows per k of ``src`` (k blocks src_ks
        elements apart, from element src_off) into ``hdst`` / ``sdst`` rows
        (k stride dst_ks, from element dst_off), float64."""
        self.ham._count_rows(self.ham.nk * nrows)
        _lib.call("gwb_ham_apply_hs", self.ham._h, _ptr(src, src_off), src_ks, _ptr(hdst, dst_off), dst_ks,
                  _ptr(sdst, dst_off), dst_ks, nrows, _lib.GWB_C128, _lib.GWB_FP64, _lib.stream_ptr(self.device))


class _GenSolver:
    """Buffers and steps of one generalized solve (see the module docstring)."""

    def __init__(self, hs: BatchedHS, x0: torch.Tensor, nbands: int, tol: float, max_iter: int,
                 max_dim_factor: int):
        self.hs = hs
        self.dev = hs.device
        self.nk, self.nb0, self.npw = (int(s) for s in x0.shape)
        self.nb = int(nbands)
        if self.nb0 < self.nb:
            raise ValueError(f"x0 holds {self.nb0} rows, fewer than nbands = {self.nb}")
        self.tol, self.max_iter = float(tol), int(max_iter)
        self.md = min(int(hs.bk.npw.min()), max(max_dim_factor * self.nb, self.nb + 24))
        if self.md < self.nb0:
            raise ValueError(f"basis of {self.md} cannot hold the {self.nb0} start rows")
        nk, npw, md, nb = self.nk, self.npw, self.md, self.nb
        c = dict(dtype=torch.complex128, device=self.dev)
        self.V = torch.zeros(nk, md, npw, **c)
        self.HV = torch.zeros(nk, md, npw, **c)
        self.SV = torch.zeros(nk, md, npw, **c)
        nrow = max(nb, self.nb0)
        self.X = torch.zeros(nk, nb, npw, **c)
        self.HX = torch.zeros(nk, nb, npw, **c)
        self.SX = torch.zeros(nk, nb, npw, **c)
        self.R = torch.zeros(nk, nb, npw, **c)
        self.D = torch.zeros(nk, nrow, npw, **c)
        self.T = torch.zeros(nk, nrow, npw, **c)     # row-transform target
        self.Hs = torch.zeros(nk, md, md, **c)
        self.Ss = torch.zeros(nk, md, md, **c)
        self.C = torch.zeros(nk * md * md, **c)      # product scratch
        self.G = torch.zeros(nk, md, md, **c)        # Cholesky input / factor
        self.Li = torch.zeros(nk, md, md, **c)       # inverse factor
        self.A = torch.zeros(nk, md, md, **c)
        self.Y = torch.zeros(nk, md, nb, **c)
        self.heev_max = int(_lib.load().gwb_heev_max_dim())
        hm = min(md, self.heev_max)
        self.U = torch.zeros(nk, max(hm, nb), nb, **c)
        self.Z = torch.zeros(nk, int(_lib.load().gwb_heev_scratch_doubles(hm)), dtype=torch.float64, device=self.dev)
        self.eig = torch.zeros(nk, nb, dtype=torch.float64, device=self.dev)
        self.rn = torch.zeros(nk, nb, dtype=torch.float64, device=self.dev)
        self.stats = torch.zeros(4, dtype=torch.float64, device=self.dev)
        self.info = torch.zeros(nk, dtype=torch.int32, device=self.dev)
        self.heev_info = torch.zeros(nk, dtype=torch.int32, device=self.dev)
        self.flags = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.sel = torch.zeros(nk, nb, dtype=torch.int32, device=self.dev)
        self.mask = hs.mask
        self.mask_u8 = self.mask.to(torch.uint8).contiguous()
        self.stream = _lib.stream_ptr(self.dev)
        self.work = torch.empty(24 << 20, dtype=torch.uint8, device=self.dev)

    def gemm(self, *a, **kw):
        kw.setdefault("work", self.work)
        kw.setdefault("stream", self.stream)
        zgemm(*a, **kw)

    # -- pencil ----------------------------------------------------------------
    def insert_columns(self, m: int, m0: int) -> None:
        """Columns m0..m-1 (and mirrored rows) of V HV^H and V SV^H."""
        nk, npw, md = self.nk, self.npw, self.md
        nnew = m - m0
        if nnew <= 0:
            return
        for img, mat in ((self.HV, self.Hs), (self.SV, self.Ss)):
            self.gemm(_N, _H, m, nnew, npw, self.V, npw, md * npw, img, npw, md * npw, self.C, nnew, m * nnew, nk,
                      b_off=m0 * npw)
            _lib.call("gwb_subspace_insert", nk, m, m0, _ptr(self.C), _ptr(mat), md, md * md, self.stream)

    def chol(self, src: torch.Tensor, lo: int, n: int, shift: float = 0.0) -> bool:
        """Lower Cholesky factor and its inverse of src[:, lo:lo+n, lo:lo+n]
        (+ shift on the diagonal) into G / Li (ld n); False on a breakdown."""
        g = self.G.view(-1)[: self.nk * n * n].view(self.nk, n, n)
        g.copy_(src[:, lo:lo + n, lo:lo + n])
        if shift:
            g.diagonal(dim1=-2, dim2=-1).add_(shift)
        _lib.call("gwb_chol_inv", self.nk, n, _ptr(self.G), n, n * n, _ptr(self.Li), n * n, _ptr(self.info), None,
                  self.stream)
        return int(self.info.max()) == 0

    def reduced_eigs(self, lo: int, n: int):
        """Lowest nb eigenpairs of L^-1 H L^-H and the pencil's vectors
        Y = L^-H U (nk, n, nb)."""
        nk, nb, md = self.nk, self.nb, self.md
        nn = n * n
        # C = L^-1 H (H Hermitian: H = H^H, an A B^H product), A = C L^-H
        self.gemm(_N, _H, n, n, n, self.Li, n, nn, self.Hs, md, md * md, self.C, n, nn, nk, b_off=lo * md + lo)
        self.gemm(_N, _H, n, n, n, self.C, n, nn, self.Li, n, nn, self.A, n, nn, nk)
        a = self.A.view(-1)[: nk * nn].view(nk, n, n)
        if n <= self.heev_max:
            _lib.call("gwb_heev_lowest", nk, n, nb, _ptr(self.A), n, nn, _ptr(self.eig), _ptr(self.U), _ptr(self.Z),
                      _ptr(self.heev_info), self.stream)
            u, ldu = self.U, nb
        else:
            w, uu = torch.linalg.eigh(a)
            self.eig.copy_(w[:, :nb])
            u, ldu = uu.contiguous(), n
        self.gemm(_H, _N, n, nb, n, self.Li, n, nn, u, ldu, n * ldu, self.Y, nb, n * nb, nk)

    def ritz(self, lo: int, n: int) -> None:
        nk, nb, npw, md = self.nk, self.nb, self.npw, self.md
        for src, dst in ((self.V, self.X), (self.HV, self.HX), (self.SV, self.SX)):
            self.gemm(_T, _N, nb, npw, n, self.Y, nb, n * nb, src, npw, md * npw, dst, npw, nb * npw, nk,
                      b_off=lo * npw)
        _lib.call("gwb_residual", nk, nb, npw, _ptr(self.SX), nb * npw, _ptr(self.HX), nb * npw, _ptr(self.eig), nb,
                  _ptr(self.R), nb * npw, _ptr(self.rn), self.stream)

    # -- orthonormalisation -------------------------------------------------------
    def rows_transform(self, blk: torch.Tensor, n: int) -> None:
        """blk[:, :n] <- Li blk[:, :n] (Li: n x n, ld n)."""
        nk, npw = self.nk, self.npw
        bs = blk.shape[1] * npw
        self.gemm(_N, _N, n, npw, n, self.Li, n, n * n, blk, npw, bs, self.T, npw, self.T.shape[1] * npw, nk)
        blk[:, :n].copy_(self.T[:, :n])

    def cholqr(self, blk: torch.Tensor, n: int, carried=()) -> bool:
        """One Cholesky-QR round of the rows blk[:, :n] in the standard
        metric; the blocks in ``carried`` get the same row transform."""
        nk, npw = self.nk, self.npw
        bs = blk.shape[1] * npw
        self.gemm(_N, _H, n, n, npw, blk, npw, bs, blk, npw, bs, self.G, n, n * n, nk)
        _lib.call("gwb_chol_inv", nk, n, _ptr(self.G), n, n * n, _ptr(self.Li), n * n, _ptr(self.info), None,
                  self.stream)
        if int(self.info.max()) != 0:
            return False
        for b in (blk, *carried):
            self.rows_transform(b, n)
        return True

    def project(self, n: int, lo: int, m: int) -> None:
        """D[:, :n] -= (D V^H) V over the window rows [lo, m)."""
        nk, npw, md = self.nk, self.npw, self.md
        w = m - lo
        if w <= 0:
            return
        ds = self.D.shape[1] * npw
        self.gemm(_N, _H, n, w, npw, self.D, npw, ds, self.V, npw, md * npw, self.C, w, n * w, nk, b_off=lo * npw)
        self.gemm(_N, _N, n, npw, w, self.C, w, n * w, self.V, npw, md * npw, self.D, npw, ds, nk, alpha=-1.0,
                  beta=1.0, b_off=lo * npw)

    def orthonormalize_new(self, n: int, lo: int, m: int) -> None:
        """Rows D[:, :n]: masked, orthogonal to the window, orthonormal."""
        self.D[:, :n].mul_(self.mask[:, None, :])
        self.project(n, lo, m)
        self.project(n, lo, m)
        self.flags.zero_()
        _lib.call("gwb_row_repair", self.nk, n, self.npw, _ptr(self.D), self.D.shape[1] * self.npw,
                  _ptr(self.mask_u8), 1e-8, _ptr(self.flags), self.stream)
        if int(self.flags.item()) & 1:  # repaired rows: orthogonalise them too
            self.project(n, lo, m)
            self.project(n, lo, m)
        for _ in range(2):
            if not self.cholqr(self.D, n):
                # dependent rows: repair at a coarser threshold and retry once
                _lib.call("gwb_row_repair", self.nk, n, self.npw, _ptr(self.D), self.D.shape[1] * self.npw,
                          _ptr(self.mask_u8), 1e-4, _ptr(self.flags), self.stream)
                self.project(n, lo, m)
                self.project(n, lo, m)
                if not self.cholqr(self.D, n):
                    raise _lib.GwbError(_lib.GWB_ERR_BREAKDOWN, "Cholesky-QR of the new directions broke down")

    def apply_rows(self, r0: int, n: int) -> None:
        md, npw = self.md, self.npw
        self.hs.hs_into(self.V, r0 * npw, md * npw, self.HV, self.SV, r0 * npw, md * npw, n)

    def compact(self, lo: int, m: int) -> None:
        """Move the window rows [lo, m) to the front of the buffers."""
        for buf in (self.V, self.HV, self.SV):
            buf[:, : m - lo].copy_(buf[:, lo:m].clone())

    # -- the solve -------------------------------------------------------------------
    def run(self, x0: torch.Tensor):
        nk, nb, npw = self.nk, self.nb, self.npw
        nb0 = self.nb0
        self.D[:, :nb0].copy_(x0)
        self.orthonormalize_new(nb0, 0, 0)
        self.V[:, :nb0].copy_(self.D[:, :nb0])
        self.apply_rows(0, nb0)
        lo, m, m0 = 0, nb0, 0
        for _ in range(self.max_iter):
            self.insert_columns(m, m0)
            m0 = m
            n = m - lo
            while not self.chol(self.Ss, lo, n) and n > nb + 1:
                lo += 1   # the oldest row leaves the window
                n -= 1
            if int(self.info.max()) != 0 and not self.chol(self.Ss, lo, n, shift=1e-10):
                raise _lib.GwbError(_lib.GWB_ERR_BREAKDOWN, "overlap of the basis is not positive definite")
            self.reduced_eigs(lo, n)
            self.ritz(lo, n)
            _lib.call("gwb_conv_stats", nk, nb, _ptr(self.rn), self.tol, _ptr(self.stats), self.stream)
            rmax, n_add = self.stats[:2].tolist()
            if rmax < self.tol:
                break
            n_add = int(n_add)
            _lib.call("gwb_select_worst", nk, nb, _ptr(self.rn), n_add, _ptr(self.sel), self.stream)
            _lib.call("gwb_precond_teter", nk, nb, n_add, npw, _ptr(self.X), nb * npw, _ptr(self.R), nb * npw,
                      _ptr(self.hs.t), _ptr(self.sel), _ptr(self.D), self.D.shape[1] * npw, self.stream)
            if n + n_add > self.md:
                # restart: the Ritz block orthonormal in the standard metric,
                # its images carried by the same triangular transforms
                for _ in range(2):
                    if not self.cholqr(self.X, nb, carried=(self.HX, self.SX)):
                        raise _lib.GwbError(_lib.GWB_ERR_BREAKDOWN, "Cholesky-QR of the Ritz block broke down")
                self.V[:, :nb].copy_(self.X)
                self.HV[:, :nb].copy_(self.HX)
                self.SV[:, :nb].copy_(self.SX)
                lo, m, m0 = 0, nb, 0
            elif m + n_add > self.md:
                self.compact(lo, m)
                lo, m, m0 = 0, m - lo, 0
            self.orthonormalize_new(n_add, lo, m)
            self.V[:, m:m + n_add].copy_(self.D[:, :n_add])
            self.apply_rows(m, n_add)
            m += n_add
        return self.eig.clone(), self.X.clone()


@torch.no_grad()
def davidson_gen_batched(hs: BatchedHS, x0: torch.Tensor, nbands: int, tol: float, max_iter: int = 60,
                         max_dim_factor: int = 4):
    """Block Davidson for H x = eps S x over (nk, ., npw_max) blocks
    (gradwave ``scf/uspp_batch.py:99-233``); returns (eig (nk, nbands) on the
    device, x (nk, nbands, npw_max)): the Ritz vectors of the pencil over a
    standard-orthonormal basis, S-normalised by the reduction (callers that
    need another normalisation apply it). Runs to ``tol`` (eV) on the largest
    residual |Hx - eps Sx| or ``max_iter`` rounds."""
    if not x0.is_cuda:
        raise RuntimeError("davidson_gen_batched (B200 path) needs CUDA tensors: there is no CPU fallback")
    solver = _GenSolver(hs, x0.to(hs.device, torch.complex128), nbands, tol, max_iter, max_dim_factor)
    eig, x = solver.run(x0.to(hs.device, torch.complex128))
    return eig, x.to(x0.dtype)
