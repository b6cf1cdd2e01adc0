"""Gamma-point real-wavefunction path on the B200 (drop-in for gradwave's
``core/gamma.py``: ``build_gamma_basis``, ``GammaHamiltonian``,
``davidson_gamma`` and the real embedding).

At k = 0 the eigenstates can be taken real, c(-G) = conj(c(G)), so one member
of each {G, -G} pair plus the real G = 0 coefficient carries the band. The
half sphere is stored with G = 0 first and, for the others, the member whose
Miller index is lexicographically positive in the order (m3, m2, m1) - the
reference's layout, kept alike so half vectors pass between the two
(``core/gamma.py:70-147``). The solver works in the real embedding
phi = (Re c0, sqrt2 Re c1, sqrt2 Im c1, ...), where the full-sphere inner
product is the plain dot product (``core/gamma.py:215-250``).

What is B200-specific is the apply: ``gwb_gamma_apply`` packs two real bands
into one complex row z = c_a + i c_b, runs the complex apply kernels on it
(FFTs, V(r), kinetic, nonlocal) and unpacks both images through the G / -G
symmetry. nb bands cost ceil(nb/2) complex rows: the halving of FFT work the
reference gets from rfftn/irfftn, here without a separate real-FFT kernel,
and the nonlocal term halves with it. The subspace algebra runs in real
float64 (cuBLAS DGEMM, cuSOLVER symmetric eigensolver, Householder QR), as
the reference's ``davidson_gamma`` runs the single-k ``davidson``
(``solvers/davidson.py:330-395``) in the embedding.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from . import ops  # noqa: F401  (registers torch.ops.gwb.*)
from .constants import HBAR2_2M

_R2 = 2.0 ** 0.5


@dataclass
class GammaBasis:
    shape: tuple[int, int, int]
    t_half: torch.Tensor         # (nhalf,) HBAR2_2M |G|^2 on the half sphere
    metric_w: torch.Tensor       # (nhalf,) 1 at G = 0, else 2
    full_flat_idx: torch.Tensor  # (npw,) sphere -> box flat index
    rep_full_idx: torch.Tensor   # (nhalf,) half slot -> full-sphere index
    src_half: torch.Tensor       # (npw,) full-sphere point -> its half slot
    conj_full: torch.Tensor      # (npw,) bool: the point is the conjugate of its representative
    partner_rep: torch.Tensor    # (nhalf,) full-sphere index of -G of each representative
    t_full: torch.Tensor         # (npw,) kinetic on the full sphere

    @property
    def nhalf(self) -> int:
        return int(self.t_half.shape[0])

    @property
    def npw(self) -> int:
        return int(self.src_half.shape[0])


def build_gamma_basis(sphere, shape, device=None) -> GammaBasis:
    """Half-sphere maps of a k = 0 sphere (``basis.GSphere``: ``miller``,
    ``kpg2``, ``flat_idx``). Raises when the sphere is not closed under
    G -> -G (k is not Gamma)."""
    n1, n2, n3 = (int(s) for s in shape)
    miller = np.asarray(sphere.miller, dtype=np.int64)
    npw = miller.shape[0]
    dev = torch.device("cpu") if device is None else torch.device(device)

    def flat(m):
        return ((m[:, 0] % n1) * n2 + (m[:, 1] % n2)) * n3 + (m[:, 2] % n3)

    where = np.full(n1 * n2 * n3, -1, dtype=np.int64)
    where[flat(miller)] = np.arange(npw)
    partner = where[flat(-miller)]
    if np.any(partner < 0):
        raise ValueError("the Gamma path needs a sphere closed under G -> -G (k must be Gamma)")
    zero = np.all(miller == 0, axis=1)
    if int(zero.sum()) != 1:
        raise ValueError("a Gamma sphere holds exactly one G = 0")
    m1, m2, m3 = miller[:, 0], miller[:, 1], miller[:, 2]
    positive = (m3 > 0) | ((m3 == 0) & (m2 > 0)) | ((m3 == 0) & (m2 == 0) & (m1 > 0))
    rep = np.concatenate([np.flatnonzero(zero), np.flatnonzero(positive)])
    nhalf = rep.shape[0]
    if 2 * nhalf - 1 != npw:
        raise ValueError(f"half sphere of {nhalf} does not pair up {npw} points")
    slot = np.full(npw, -1, dtype=np.int64)
    slot[rep] = np.arange(nhalf)
    is_rep = zero | positive
    src = np.where(is_rep, slot, slot[partner])
    kin = HBAR2_2M * np.asarray(sphere.kpg2, dtype=np.float64)
    w = np.full(nhalf, 2.0)
    w[0] = 1.0

    def t(a, dt):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)

    return GammaBasis(shape=(n1, n2, n3), t_half=t(kin[rep], torch.float64), metric_w=t(w, torch.float64),
                      full_flat_idx=t(np.asarray(sphere.flat_idx), torch.int64), rep_full_idx=t(rep, torch.int64),
                      src_half=t(src, torch.int64), conj_full=t(~is_rep, torch.bool),
                      partner_rep=t(partner[rep], torch.int64), t_full=t(kin, torch.float64))


def half_to_full(gb: GammaBasis, chalf: torch.Tensor) -> torch.Tensor:
    """(nb, nhalf) -> (nb, npw) Hermitian-symmetric full sphere."""
    c = chalf[:, gb.src_half.to(chalf.device)]
    return torch.where(gb.conj_full.to(chalf.device)[None, :], c.conj(), c)


def full_to_half(gb: GammaBasis, cfull: torch.Tensor) -> torch.Tensor:
    """(nb, npw) -> (nb, nhalf); lossless for a Hermitian-symmetric row."""
    return cfull[:, gb.rep_full_idx.to(cfull.device)]


def metric_inner(gb: GammaBasis, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Real Gram <a_m|b_n> = Re[a0* b0] + 2 sum_{G>0} Re[a* b] (nb, nb)."""
    return torch.einsum("mp,np->mn", a.conj(), gb.metric_w.to(b.device) * b).real


def embed_real(gb: GammaBasis, chalf: torch.Tensor) -> torch.Tensor:
    """(nb, nhalf) complex -> (nb, 2 nhalf - 1) real, dot product = metric."""
    nb = chalf.shape[0]
    phi = torch.empty(nb, 2 * gb.nhalf - 1, dtype=torch.float64, device=chalf.device)
    phi[:, 0] = chalf[:, 0].real
    phi[:, 1::2] = _R2 * chalf[:, 1:].real
    phi[:, 2::2] = _R2 * chalf[:, 1:].imag
    return phi


def unembed_real(gb: GammaBasis, phi: torch.Tensor) -> torch.Tensor:
    """Inverse of ``embed_real``."""
    nb = phi.shape[0]
    c = torch.empty(nb, gb.nhalf, dtype=torch.complex128, device=phi.device)
    c[:, 0] = phi[:, 0].to(torch.complex128)
    c[:, 1:] = torch.complex(phi[:, 1::2], phi[:, 2::2]) / _R2
    return c


def kinetic_phi(gb: GammaBasis) -> torch.Tensor:
    """The kinetic diagonal in the embedding (2 nhalf - 1,)."""
    t = torch.empty(2 * gb.nhalf - 1, dtype=torch.float64, device=gb.t_half.device)
    t[0] = gb.t_half[0]
    t[1::2] = gb.t_half[1:]
    t[2::2] = gb.t_half[1:]
    return t


class GammaHamiltonian:
    """H at Gamma on the half sphere (``core/gamma.py:161-203``):
    ``GammaHamiltonian(gb, v_eff_r, p, dij).apply(chalf)``, p the full-sphere
    projectors (nproj, npw). ``apply_phi`` is the same operator in the real
    embedding (what the solver uses), ``prec`` float64 or float32
    arithmetic."""

    def __init__(self, gb: GammaBasis, v_eff_r, p, dij, device=None):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.gb, self.device, self.shape = gb, dev, gb.shape
        npw, nhalf = gb.npw, gb.nhalf
        p = torch.as_tensor(p).to(dev, torch.complex128).reshape(1, -1, npw).contiguous()
        self.nproj = int(p.shape[1])
        flat = np.ascontiguousarray(gb.full_flat_idx.cpu().numpy().astype(np.int64))
        npw_arr = np.array([npw], dtype=np.int64)
        geom = _lib.Geometry()
        geom.nk, geom.npw_max, geom.nproj = 1, npw, self.nproj
        for a in range(3):
            geom.n[a] = int(gb.shape[a])
        geom.npw = npw_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        geom.flat_idx = flat.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        h = ctypes.c_void_p()
        _lib.call("gwb_ham_create", ctypes.byref(geom), int(dev.index or 0), ctypes.byref(h))
        self._h = h
        self.t = gb.t_full.to(dev).reshape(1, npw).contiguous()
        self.v = torch.as_tensor(v_eff_r).to(dev, torch.float64).contiguous()
        self.p = p
        self.dij = torch.as_tensor(dij).to(dev, torch.float64).contiguous()
        with torch.cuda.device(dev):
            s = _lib.stream_ptr(dev)
            _lib.call("gwb_ham_set_kinetic", self._h, self.t.data_ptr(), s)
            _lib.call("gwb_ham_set_potential", self._h, self.v.data_ptr(), s)
            _lib.call("gwb_ham_set_projectors", self._h, self.p.data_ptr() if self.nproj else None,
                      self.dij.data_ptr() if self.nproj else None, s)
        from .autotune import apply_tuning
        self.tuning = apply_tuning(self._h, "gamma", self.shape, self.nproj)
        # float64 applies from 128 projectors: the nonlocal term in the real
        # embedding as two float64 GEMMs (a second handle without projectors
        # gives T + V_loc). At k = 0 the projectors are Hermitian-symmetric
        # (P(-G) = conj P(G): real functions in real space), so their embedded
        # rows pi_p give <P_p|c> = pi_p . phi for every real band and the term
        # sum_pq P_p D_pq <P_q|c> embeds as (becp D) Pi: one real product per
        # real band where the complex row costs a complex one per band pair.
        self._h_loc = None
        self.pi = None
        if self.nproj >= 128 and os.environ.get("GWB_GAMMA_REAL_NL", "1") != "0":
            geom.nproj = 0
            hl = ctypes.c_void_p()
            _lib.call("gwb_ham_create", ctypes.byref(geom), int(dev.index or 0), ctypes.byref(hl))
            self._h_loc = hl
            with torch.cuda.device(dev):
                s = _lib.stream_ptr(dev)
                _lib.call("gwb_ham_set_kinetic", hl, self.t.data_ptr(), s)
                _lib.call("gwb_ham_set_potential", hl, self.v.data_ptr(), s)
                _lib.call("gwb_ham_set_projectors", hl, None, None, s)
            apply_tuning(hl, "gamma", self.shape, self.nproj)
            rep = gb.rep_full_idx.to(dev)
            self.pi = embed_real(gb, p[0][:, rep]).contiguous()     # (nproj, 2 nhalf - 1)
        i32 = dict(dtype=torch.int32, device=dev)
        self.src_half = gb.src_half.to(**i32).contiguous()
        self.conj_full = gb.conj_full.to(dev, torch.uint8).contiguous()
        self.rep_full = gb.rep_full_idx.to(**i32).contiguous()
        self.partner_rep = gb.partner_rep.to(**i32).contiguous()
        self.t_phi = kinetic_phi(gb).to(dev)
        self._work = None
        self.n_apply = 0
        self.timing: list | None = None   # (start event, end event, bands, prec) per apply when a list
        assert nhalf * 2 - 1 == npw

    def apply_times(self) -> dict:
        """Totals of the applies recorded since ``timing`` was set to a list
        (call after the stream has been synchronised): launches, milliseconds
        and real bands, per arithmetic precision."""
        out = {"calls": 0, "ms": 0.0, "bands": 0, "bands_fp32": 0, "bands_fp64": 0}
        for e0, e1, nb, prec in self.timing or []:
            out["calls"] += 1
            out["ms"] += e0.elapsed_time(e1)
            out["bands"] += nb
            out["bands_fp32" if prec == _lib.GWB_FP32 else "bands_fp64"] += nb
        return out

    def __del__(self):
        for name in ("_h", "_h_loc"):
            h = getattr(self, name, None)
            if h is not None and h.value:
                try:
                    torch.cuda.synchronize(self.device)
                    _lib.load().gwb_ham_destroy(h)
                except Exception:
                    pass
                setattr(self, name, None)

    def apply_phi(self, phi: torch.Tensor, prec: int = _lib.GWB_FP64) -> torch.Tensor:
        """H on real embedded rows (nb, 2 nhalf - 1) float64 -> same shape."""
        _lib.require_cuda(phi, "phi")
        nb = int(phi.shape[0])
        phi = phi.contiguous()  # row-major rows for the kernels (solver blocks may come transposed)
        out = torch.empty(phi.shape, dtype=torch.float64, device=phi.device)
        if nb == 0:
            return out
        need = int(_lib.load().gwb_gamma_work_bytes(nb, self.gb.npw))
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.uint8, device=self.device)
        ev = None
        if self.timing is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
        real_nl = prec == _lib.GWB_FP64 and self._h_loc is not None
        _lib.call("gwb_gamma_apply", self._h_loc if real_nl else self._h, nb, self.gb.nhalf, self.gb.npw,
                  phi.data_ptr(), phi.shape[1], out.data_ptr(), out.shape[1], self.src_half.data_ptr(),
                  self.conj_full.data_ptr(), self.rep_full.data_ptr(), self.partner_rep.data_ptr(), prec,
                  self._work.data_ptr(), self._work.numel(), _lib.stream_ptr(self.device))
        nphi = 2 * self.gb.nhalf - 1
        if real_nl:
            becp = phi[:, :nphi] @ self.pi.T
            out[:, :nphi].addmm_(becp @ self.dij, self.pi)
        if ev is not None:
            ev[1].record()
            self.timing.append((ev[0], ev[1], nb, prec))
        if out.shape[1] > nphi:  # padded rows (the solver's even width) keep their pad at zero
            out[:, nphi:] = 0.0
        self.n_apply += nb
        return out

    def apply(self, chalf: torch.Tensor) -> torch.Tensor:
        """H on half-sphere rows (nb, nhalf) complex -> (nb, nhalf)."""
        return unembed_real(self.gb, self.apply_phi(embed_real(self.gb, chalf.to(self.device))))


@dataclass
class GammaDavidsonResult:
    eigenvalues: torch.Tensor   # (nb,) ascending [eV]
    eigenvectors: torch.Tensor  # (nb, nhalf) metric-orthonormal half-sphere rows
    n_iter: int
    residual_norms: torch.Tensor  # (nb,)
    phase_ms: dict | None = None  # CUDA-event times per step (GWB_PROFILE=1)
    n_tpa_fallback: int = 0       # bands the learned preconditioner's stall rule sent to TPA
    info: dict | None = None      # rounds per phase, hand-off residual


class _OwnEigh:
    """The lowest eigenpairs of the subspace matrix by libgwb's own
    eigensolver (``gwb_sy_lowest``: tridiagonalisation across the GPU,
    multisection, inverse iteration, back-transform), with its workspace kept
    between calls. ``lowest(s, n)`` returns (w, ut): n ascending eigenvalues
    and the eigenvectors as the rows of ut (n x m). A bounded wait that ran
    out is reported by ``check()`` (one read per solve)."""

    def __init__(self, dev):
        self.dev = dev
        self.work = None
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    def lowest(self, s: torch.Tensor, n: int):
        m = int(s.shape[0])
        a = s.contiguous().clone()  # symmetric: row-major is column-major; overwritten
        need = int(_lib.load().gwb_sy_lowest_work_bytes(m, n))
        if self.work is None or self.work.numel() < need:
            self.work = torch.empty(need, dtype=torch.uint8, device=self.dev)
        w = torch.empty(n, dtype=torch.float64, device=self.dev)
        ut = torch.empty(n, m, dtype=torch.float64, device=self.dev)
        _lib.call("gwb_sy_lowest", m, n, a.data_ptr(), m, w.data_ptr(), ut.data_ptr(), m, self.work.data_ptr(),
                  self.work.numel(), self.status.data_ptr(), _lib.stream_ptr(self.dev))
        return w, ut

    def check(self) -> None:
        v = int(self.status.item())
        if v != 0:
            self.status.zero_()
            raise _lib.GwbError(v, "subspace eigensolver: a bounded grid barrier ran out")


def _orthonormalize(v: torch.Tensor, against: torch.Tensor | None = None) -> torch.Tensor:
    """Two projection passes against ``against``, Householder QR of the rows,
    rows with |R_ii| <= 1e-10 dropped (gradwave ``solvers/davidson.py:319-326``)."""
    if against is not None and against.shape[0]:
        v = v - (v @ against.T) @ against
        v = v - (v @ against.T) @ against
    q, r = torch.linalg.qr(v.T, mode="reduced")
    keep = r.diagonal().abs() > 1e-10
    return q.T[keep]


class _TcProjection:
    """Products of the float32 phase of the mixed schedule on the tensor
    cores. The solver keeps its real rows at an even width, so a row is also
    a complex row of half the length, and for such rows Re(A B^H) is exactly
    the real product A B^T, and a real coefficient matrix times complex rows
    gives the real product's even and odd columns as its real and imaginary
    parts: the split-BF16 complex kernels (``gradwave_b200.tc``, error about
    1e-6 of sum_k |a||b|) then compute

    * ``project``: the coefficients D V^T and the update D -= C V;
    * ``subspace``: the new columns V HV_new^T of the subspace matrix;
    * ``ritz``: the Ritz vectors U^T V and their images U^T HV.

    The BF16 planes of the basis and of its images are kept current row block
    by row block. In the float32 phase the applies themselves carry ~1e-7
    relative error, and every convergence decision is made after a float64
    certification of a re-orthonormalised block. A row that keeps less than
    1e-2 of its unit norm in ``project`` would be dominated by the products'
    error, so then the block is redone in float64 (the complex path's rule)."""

    def __init__(self, max_dim: int, nb: int, npad: int, dev):
        from .tc import PlaneSet
        self.nc = npad // 2
        self.pv = PlaneSet(1, max_dim, self.nc, dev)
        self.ph = PlaneSet(1, max_dim, self.nc, dev)
        self.pt = PlaneSet(1, nb, self.nc, dev)
        self.pc = PlaneSet(1, nb, max_dim, dev)
        self.n_fallback = 0

    def _cx(self, t: torch.Tensor) -> torch.Tensor:
        return torch.view_as_complex(t.view(t.shape[0], self.nc, 2))

    def rows(self, v: torch.Tensor, hv: torch.Tensor | None, r0: int, r1: int) -> None:
        if r1 > r0:
            self.pv.write(self._cx(v), r1 - r0, row0=r0, src_ld=self.nc, src_kstride=0, offset=r0 * self.nc)
            if hv is not None:
                self.ph.write(self._cx(hv), r1 - r0, row0=r0, src_ld=self.nc, src_kstride=0, offset=r0 * self.nc)

    def project(self, t: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
        from .tc import OP_H, OP_N, zgemm_tc
        n, m = t.shape[0], v.shape[0]
        t = t.contiguous()
        keep = t.clone()
        tc = self._cx(t)
        self.pt.write(tc, n, src_ld=self.nc, src_kstride=0)
        c = torch.empty(n, m, dtype=torch.complex128, device=t.device)
        zgemm_tc(OP_H, n, m, self.nc, self.pt, self.pv, c, m, n * m)
        c.imag.zero_()
        self.pc.write(c, n, src_ld=m, src_kstride=0, cols=m)
        zgemm_tc(OP_N, n, self.nc, m, self.pc, self.pv, tc, self.nc, n * self.nc, alpha=-1.0, beta=1.0)
        if float(torch.linalg.vector_norm(t, dim=1).min()) < 1e-2:
            self.n_fallback += 1
            return keep - (keep @ v.T) @ v
        return t

    def subspace(self, hv_new: torch.Tensor, m: int, m0: int) -> torch.Tensor:
        """V[:m] HV[m0:m]^T (m x (m - m0)); hv_new = HV[m0:m]. From m0 = 0
        (after a restart) the kept planes of both serve directly."""
        from .tc import OP_H, zgemm_tc
        if m0 == 0:
            c = torch.empty(m, m, dtype=torch.complex128, device=hv_new.device)
            zgemm_tc(OP_H, m, m, self.nc, self.pv, self.ph, c, m, m * m)
            return c.real
        n = hv_new.shape[0]
        self.pt.write(self._cx(hv_new.contiguous()), n, src_ld=self.nc, src_kstride=0)
        c = torch.empty(n, m, dtype=torch.complex128, device=hv_new.device)
        zgemm_tc(OP_H, n, m, self.nc, self.pt, self.pv, c, m, n * m)
        return c.real.T

    def ritz(self, ut: torch.Tensor, m: int):
        """(U^T V[:m], U^T HV[:m]) for the real coefficients ut (n x m)."""
        from .tc import OP_N, zgemm_tc
        n = ut.shape[0]
        self.pc.write(ut.to(torch.complex128), n, src_ld=m, src_kstride=0, cols=m)
        out = []
        for planes in (self.pv, self.ph):
            o = torch.empty(n, 2 * self.nc, dtype=torch.float64, device=ut.device)
            zgemm_tc(OP_N, n, self.nc, m, self.pc, planes, self._cx(o), self.nc, n * self.nc)
            out.append(o)
        return out[0], out[1]


class _Products:
    """The float64 products of the Gamma solver: cuBLAS DGEMM (through torch)
    or, with ``oz``, the int8 tensor-core products of ``gradwave_b200.oz``
    (the Ozaki scheme, 8 slices: float64-level error relative to the rows'
    maxima). ``nt(a, b)`` = a b^T, ``nn(a, b)`` = a b, ``sub_nn(t, c, b)``:
    t -= c b in place.

    ``attach(V, HV)`` registers the solver's basis buffers: their slices are
    then kept current by ``rows_changed(r0, r1)`` (only the rows that
    changed are sliced again), and a product whose operand is a prefix
    ``V[:m]`` or ``HV[:m]`` reads the kept slices instead of slicing it."""

    def __init__(self, dev=None, oz: bool | str = False):
        self.om = None
        self.V = self.HV = None
        self.valid = 0
        if oz == "crt":
            from .oz import CrtMatmul
            self.om = CrtMatmul(dev)
        elif oz:
            from .oz import OzMatmul
            self.om = OzMatmul(dev)

    def attach(self, V: torch.Tensor, HV: torch.Tensor) -> None:
        if self.om is None:
            return
        rows, npad = V.shape
        self.V, self.HV = V, HV
        self.v_rows = self.om.new_set(rows, npad)   # rows of V (a b^T operands)
        self.v_cols = self.om.new_set(npad, rows)   # V^T: the B of  . @ V
        self.hv_cols = self.om.new_set(npad, rows)  # HV^T: the B of . @ HV
        self.valid = 0

    def rows_changed(self, r0: int, r1: int) -> None:
        """Rows [r0, r1) of V and HV were written; rows before r0 are as
        they were when last sliced."""
        if self.V is None or r1 <= r0:
            return
        self.v_rows.split_rows(self.V[r0:r1], row0=r0)
        self.v_cols.split_cols(self.V[r0:r1], k0=r0)
        self.hv_cols.split_cols(self.HV[r0:r1], k0=r0)
        self.valid = r1

    def _prefix(self, t: torch.Tensor, base) -> bool:
        return (base is not None and t.dim() == 2 and t.data_ptr() == base.data_ptr()
                and t.stride() == base.stride() and t.shape[1] == base.shape[1] and t.shape[0] <= self.valid)

    @staticmethod
    def _rows(a: torch.Tensor) -> torch.Tensor:
        return a if a.stride(-1) == 1 else a.contiguous()

    def nt(self, a: torch.Tensor, b: torch.Tensor, same: bool = False) -> torch.Tensor:
        if self.om is None or a.shape[0] == 0 or b.shape[0] == 0:
            return a @ b.T
        a = self._rows(a)
        b = a if same else self._rows(b)
        out = torch.empty(a.shape[0], b.shape[0], dtype=torch.float64, device=a.device)
        if not same and self._prefix(a, self.V):      # V[:m] b^T
            sb = self.om._set("nt_b", b.shape[0], b.shape[1])
            sb.split_rows(b)
            self.om.gemm(a.shape[0], b.shape[0], a.shape[1], self.v_rows, sb, out)
            return out
        if not same and self._prefix(b, self.V):      # a V[:m]^T
            sa = self.om._set("nt_a", a.shape[0], a.shape[1])
            sa.split_rows(a)
            self.om.gemm(a.shape[0], b.shape[0], a.shape[1], sa, self.v_rows, out)
            return out
        return self.om.nt(a, b, out, same=same)

    def _nn_into(self, a: torch.Tensor, b: torch.Tensor, out: torch.Tensor, alpha: float, beta: float) -> None:
        for base, cols in ((self.V, getattr(self, "v_cols", None)), (self.HV, getattr(self, "hv_cols", None))):
            if self._prefix(b, base):
                m = b.shape[0]
                sa = self.om._set("nn_a", a.shape[0], m)
                sa.split_rows(a.contiguous(), fold=cols.kscale)
                self.om.gemm(a.shape[0], b.shape[1], m, sa, cols, out, alpha, beta, b_scaled=False)
                return
        self.om.nn(a.contiguous(), self._rows(b), out, alpha, beta)

    def nn(self, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        if self.om is None or a.shape[0] == 0 or b.shape[0] == 0:
            return a @ b
        out = torch.empty(a.shape[0], b.shape[1], dtype=torch.float64, device=a.device)
        self._nn_into(a, b, out, 1.0, 0.0)
        return out

    def sub_nn(self, t: torch.Tensor, c: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        if self.om is None or t.stride(-1) != 1:
            return t.addmm_(c, b, alpha=-1.0)
        self._nn_into(c, b, t, -1.0, 1.0)
        return t


_CUBLAS = _Products()


def _project_out(t: torch.Tensor, basis: torch.Tensor, mm: _Products = _CUBLAS) -> torch.Tensor:
    """t -= (t basis^T) basis, in place (one float64 product pair)."""
    if basis.shape[0]:
        mm.sub_nn(t, mm.nt(t, basis), basis)
    return t


def _cholqr(y: torch.Tensor, mm: _Products = _CUBLAS):
    """Cholesky-QR of the rows of y: L = chol(y y^T), y <- L^-1 y, with the
    triangular inverse formed once (n x n) and applied as one product. Returns
    None when the Gram matrix is not numerically positive definite (a row kept
    less than 1e-8 of its unit norm)."""
    L, info = torch.linalg.cholesky_ex(mm.nt(y, y, same=True))
    if int(info.max()) != 0 or float(torch.diagonal(L).min()) <= 1e-8:
        return None
    eye = torch.eye(L.shape[0], dtype=L.dtype, device=L.device)
    return mm.nn(torch.linalg.solve_triangular(L, eye, upper=False), y)


def _cholqr_images(x: torch.Tensor, hx: torch.Tensor, mm: _Products = _CUBLAS):
    """Cholesky-QR of the rows of x in float64 (twice; Householder QR if that
    breaks down), with the same triangular transform applied to their images
    hx, so that the pair stays (block, H block)."""
    for _ in range(2):
        L, info = torch.linalg.cholesky_ex(mm.nt(x, x, same=True))
        if int(info.max()) != 0 or float(torch.diagonal(L).min()) <= 1e-8:
            q, r = torch.linalg.qr(x.T, mode="reduced")
            rinv = torch.linalg.solve_triangular(r, torch.eye(r.shape[0], dtype=r.dtype, device=r.device),
                                                 upper=True)
            return q.T.contiguous(), mm.nn(rinv.T.contiguous(), hx)
        li = torch.linalg.solve_triangular(L, torch.eye(L.shape[0], dtype=L.dtype, device=L.device), upper=False)
        x, hx = mm.nn(li, x), mm.nn(li, hx)
    return x, hx


def _expand(t: torch.Tensor, v: torch.Tensor, tcp: _TcProjection | None = None,
            locked: torch.Tensor | None = None, mm: _Products = _CUBLAS, low: bool = False) -> torch.Tensor:
    """New directions from preconditioned residuals: unit rows, two
    projections against the orthonormal basis v (and the locked rows, which
    are orthogonal to v), then Cholesky-QR; Householder QR dropping rows that
    kept less than 1e-8 of their norm when Cholesky-QR breaks down.

    The reference's single-k Davidson orthonormalises the raw preconditioned
    residuals with an absolute 1e-10 rank threshold (``solvers/davidson.py:
    319-326,383``); their norm is of the order of the tolerance itself, so
    below ~1e-8 eV rows of round-off survive, the basis loses orthogonality and
    the solve stalls or diverges (on si216 at 1e-9 eV: residual 2e-2 after 300
    rounds). Unit rows and a relative threshold, as the batched Davidson does
    (``:406-457``), remove that floor. The second Cholesky-QR round is skipped
    when the first already left the Gram matrix within 1e-13 of the identity
    (it would change the rows by that much).

    ``low`` (the float32 phase, with ``tcp``): both projection passes on the
    tensor cores, each followed by a float64 Cholesky-QR. The first pass
    leaves components along v of ~1e-6 that the Cholesky-QR may amplify by
    the block's condition number; the second pass brings them back to ~1e-6
    of unit rows, and the second Cholesky-QR (of a nearly orthonormal block)
    restores orthonormality among the new rows. The basis of the float32
    phase is thus orthonormal to ~1e-6, the level of its float32 applies. A
    block whose Cholesky factorisation breaks down takes the float64 path
    below."""
    t = t / torch.linalg.vector_norm(t, dim=1, keepdim=True).clamp_min(1e-300)
    lk = locked if locked is not None else v[:0]
    if low and tcp is not None and lk.shape[0] == 0:
        y = _cholqr(tcp.project(t, v), mm)
        y2 = _cholqr(tcp.project(y, v), mm) if y is not None else None
        if y2 is not None:
            return y2
    _project_out(t, lk, mm)
    t = tcp.project(t, v) if tcp is not None else _project_out(t, v, mm)
    _project_out(_project_out(t, lk, mm), v, mm)
    y = _cholqr(t, mm)
    if y is not None:
        g = mm.nt(y, y, same=True)
        g.diagonal().sub_(1.0)
        if float(g.abs().max()) < 1e-13:
            return y
        y2 = _cholqr(y, mm)
        if y2 is not None:
            return y2
    q, r = torch.linalg.qr(t.T, mode="reduced")
    t = q.T[r.diagonal().abs() > 1e-8]
    if t.shape[0] == 0:
        return t
    _project_out(_project_out(t, lk, mm), v, mm)
    q, _ = torch.linalg.qr(t.T, mode="reduced")
    return q.T.contiguous()


def _teter(residual: torch.Tensor, t_g: torch.Tensor, t_band: torch.Tensor) -> torch.Tensor:
    """TPA filter (gradwave ``solvers/precond.py:8-18``)."""
    x = t_g[None, :] / torch.clamp(t_band[:, None], min=1e-12)
    x2 = x * x
    num = 27.0 + 18.0 * x + 12.0 * x2 + 8.0 * x2 * x
    return residual * (num / (num + 16.0 * x2 * x2))


def _half_rows(phi: torch.Tensor, nhalf: int) -> torch.Tensor:
    """Embedded real rows -> half-sphere complex rows scaled by sqrt(w_G):
    c'_0 = phi_0, c'_G = phi_2G-1 + i phi_2G (w_G = 2 off G = 0). Their plain
    sums over the half sphere are the full-sphere sums, so a kernel that reads
    complex rows (the band's kinetic energy, residual amplitudes) sees the
    same numbers as on the full sphere."""
    c = torch.empty(phi.shape[0], nhalf, dtype=torch.complex128, device=phi.device)
    c[:, 0] = phi[:, 0]
    c[:, 1:] = torch.complex(phi[:, 1:2 * nhalf - 1:2], phi[:, 2:2 * nhalf - 1:2])
    return c


def _embed_rows(c: torch.Tensor, npad: int) -> torch.Tensor:
    """Inverse of ``_half_rows`` (zero pad column(s))."""
    nhalf = c.shape[1]
    phi = torch.zeros(c.shape[0], npad, dtype=torch.float64, device=c.device)
    phi[:, 0] = c[:, 0].real
    phi[:, 1:2 * nhalf - 1:2] = c[:, 1:].real
    phi[:, 2:2 * nhalf - 1:2] = c[:, 1:].imag
    return phi


class _LearnedGamma:
    """The learned preconditioner on the Gamma path: the network on the
    tcgen05 tensor cores (``gwb_precond_learned_gamma``), reading the
    selected bands' embedded real rows as their sqrt(w)-scaled half-sphere
    rows and writing the result in the same embedding, with the stall rule
    of the complex solver (a band
    whose residual has not improved on its best by 10 % for 3 rounds keeps
    TPA from then on; ``gwb_stall_update``; GWB_STALL_RATIO and
    GWB_STALL_PATIENCE change the 0.9 and the 3). Its per-band state follows
    the active Ritz block through locking."""

    def __init__(self, model, nb: int, t_half: torch.Tensor, dev):
        import os
        self.params = model.params.to(dev)
        # the stall rule's ratio and patience (GWB_STALL_RATIO, GWB_STALL_PATIENCE)
        self.ratio = float(os.environ.get("GWB_STALL_RATIO", "0.9"))
        self.patience = int(os.environ.get("GWB_STALL_PATIENCE", "3"))
        self.t_half = t_half.to(dev, torch.float64).reshape(1, -1).contiguous()
        self.best = torch.full((nb,), float("inf"), dtype=torch.float64, device=dev)
        self.count = torch.zeros(nb, dtype=torch.uint8, device=dev)
        self.tpa_only = torch.zeros(nb, dtype=torch.uint8, device=dev)
        self._work = None

    def keep(self, mask: torch.Tensor) -> None:
        self.best, self.count, self.tpa_only = self.best[mask], self.count[mask], self.tpa_only[mask]

    def n_fallback(self) -> int:
        return int(self.tpa_only.sum())

    def __call__(self, x: torch.Tensor, r: torch.Tensor, rn: torch.Tensor, eig: torch.Tensor,
                 sel: torch.Tensor, npad: int) -> torch.Tensor:
        n_all = int(rn.shape[0])
        rn = rn.contiguous()
        _lib.call("gwb_stall_update", rn.data_ptr(), self.best.data_ptr(), self.count.data_ptr(),
                  self.tpa_only.data_ptr(), n_all, self.ratio, self.patience, _lib.stream_ptr(rn.device))
        nhalf = int(self.t_half.shape[1])
        x, r, eig = x.contiguous(), r.contiguous(), eig.contiguous()
        sl = sel.to(torch.int32).contiguous()
        n = int(sl.shape[0])
        d = torch.empty(n, npad, dtype=torch.float64, device=x.device)
        need = int(_lib.load().gwb_precond_learned_gamma_work_bytes(n, nhalf))
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.uint8, device=x.device)
        # the embedded rows in place: no gather, no complex copies
        _lib.call("gwb_precond_learned_gamma", self.params.data_ptr(), n_all, n, nhalf, npad, x.data_ptr(),
                  x.stride(0), r.data_ptr(), r.stride(0), self.t_half.data_ptr(), eig.data_ptr(), sl.data_ptr(),
                  self.tpa_only.data_ptr(), d.data_ptr(), npad, self._work.data_ptr(), self._work.numel(),
                  _lib.stream_ptr(x.device))
        return d


class _Locked:
    """Converged Ritz pairs taken out of the active Rayleigh-Ritz: rows,
    images, eigenvalues and residual norms, in preallocated buffers."""

    def __init__(self, cap: int, npad: int, dev):
        self.x = torch.empty(cap, npad, dtype=torch.float64, device=dev)
        self.hx = torch.empty(cap, npad, dtype=torch.float64, device=dev)
        self.eig = torch.empty(cap, dtype=torch.float64, device=dev)
        self.rn = torch.empty(cap, dtype=torch.float64, device=dev)
        self.n = 0

    def add(self, x, hx, eig, rn) -> None:
        k = int(x.shape[0])
        self.x[self.n:self.n + k] = x
        self.hx[self.n:self.n + k] = hx
        self.eig[self.n:self.n + k] = eig
        self.rn[self.n:self.n + k] = rn
        self.n += k

    def rows(self) -> torch.Tensor:
        return self.x[:self.n]

    def merge(self, eig, x, rn):
        """Locked and active wanted pairs together, ascending."""
        if self.n == 0:
            return eig, x, rn
        e = torch.cat([self.eig[:self.n], eig])
        order = torch.argsort(e)
        return e[order], torch.cat([self.x[:self.n], x])[order], torch.cat([self.rn[:self.n], rn])[order]


@torch.no_grad()
def davidson_gamma(ham: GammaHamiltonian, x0: torch.Tensor, tol: float = 1e-9, max_iter: int = 40,
                   max_dim_factor: int = 4, mode: str = "fp64", lock: bool | None = None,
                   n_buffer: int = 0, buffer_tol: float = 1e-2, precond="teter") -> GammaDavidsonResult:
    """Real-symmetric block Davidson on the half sphere
    (``core/gamma.py:261-290``): the single-k Davidson of the reference
    (``solvers/davidson.py:330-395``: Rayleigh-Ritz on the whole subspace,
    TPA on every unconverged residual, restart to [Ritz block, new
    directions]) in the real embedding, every step on the device. Two rules
    follow the reference's batched Davidson instead of its single-k one: the
    new directions are unit-normalised and rank-checked relative to their norm
    (``_expand``), and a restart keeps the Ritz block's images HX rather than
    applying H again (``solvers/davidson.py:745-759``), since [X, T] is
    already orthonormal with X = U^T V and HX = U^T HV.

    ``mode="mixed"``: the expansion applies run in float32 arithmetic until
    the largest residual reaches the float32 floor (32 eps_f32 max T) or stalls
    within 100x of it; then the Ritz block is certified with a float64 apply and
    a float64 nb x nb Rayleigh-Ritz, and unless that meets ``tol`` the basis
    collapses to the certified block and the solve continues in float64 (the
    complex path's mixed rule, ``davidson.py``; gradwave
    ``solvers/davidson.py:226-308``). Every convergence decision is made on
    float64 residuals.

    ``lock`` (default: on in the mixed mode, off in float64 mode, which keeps
    the reference's rules): at a restart, wanted Ritz pairs whose float64
    residual is within ``tol`` leave the active Rayleigh-Ritz for good. The
    restarted basis holds only the unconverged Ritz vectors and the new
    directions, so the eigensolve and the Ritz products of the rounds that
    follow (often only a few stragglers left) run on a basis a fraction of
    the size; the cap stays the reference's max_dim, so stragglers keep
    their history. New directions are also projected against the locked
    rows. A locked pair's coupling to the active space is its residual
    (<= tol), so the active pairs move by O(tol^2/gap). Locking happens only
    on float64 residuals, never in the float32 phase.

    ``n_buffer`` extra Ritz pairs ride along above the wanted ones (started on
    the next embedded coordinates, seeded noise where those repeat a start
    direction): they keep the wanted block's upper edge away
    from the first unwanted eigenvalue, are expanded only while their residual
    exceeds ``buffer_tol`` (eV) and are neither tested nor returned.

    ``precond``: ``"teter"`` (TPA) or a ``learned.LearnedPreconditioner``
    (the network on the half-sphere rows, TPA for bands whose residual
    stalls). With ``GWB_OZ=1`` the float64 products run on the int8 tensor
    cores (``gradwave_b200.oz``) instead of cuBLAS."""
    if mode not in ("fp64", "mixed"):
        raise ValueError(f"mode must be 'fp64' or 'mixed', got {mode!r}")
    if n_buffer < 0:
        raise ValueError(f"n_buffer must be >= 0, got {n_buffer}")
    import os
    from .davidson import _PhaseTimer
    prof = _PhaseTimer(os.environ.get("GWB_PROFILE", "0") == "1")
    lock = (mode == "mixed") if lock is None else bool(lock)
    gb, dev = ham.gb, ham.device
    phi0 = embed_real(gb, x0.to(dev, torch.complex128))
    nwant, nphi = phi0.shape
    n_buffer = min(int(n_buffer), nphi - nwant)
    if n_buffer:
        # buffer starts: unit vectors on the embedded coordinates nwant ...
        # nwant + n_buffer - 1. Those that repeat a direction of x0 (with the
        # identity start, every other one) are dropped by the orthonormalisation
        # and replaced by seeded noise rows below. On si216 this mixed start
        # converged in 32 rounds, plane-wave starts on the next half-sphere
        # slots in 38.
        extra = torch.zeros(n_buffer, nphi, dtype=torch.float64, device=dev)
        extra[torch.arange(n_buffer), torch.arange(nwant, nwant + n_buffer)] = 1.0
        phi0 = torch.cat([phi0, extra])
    nb = nwant + n_buffer

    # the reference's basis cap, for the whole block (buffer bands included)
    max_dim = max(min(max_dim_factor * nb, nphi), nb + 1)
    # the active basis and its images live in preallocated buffers; a restart
    # to [Ritz block, new directions] needs up to 2 nb rows
    rows = max(max_dim, 2 * nb)
    # rows are kept at an even width (one zero pad column), so that a real row
    # is also a complex row for the tensor-core products
    npad = nphi + (nphi & 1)
    phi0 = torch.nn.functional.pad(phi0, (0, npad - nphi))
    t_phi = torch.nn.functional.pad(ham.t_phi, (0, npad - nphi))
    tcp = _TcProjection(rows, nb, npad, dev) if (mode == "mixed" and dev.type == "cuda"
                                                 and os.environ.get("GWB_TC_PROJECT", "1") != "0") else None
    # float64 products: cuBLAS DGEMM; with GWB_OZ=crt the int8 tensor-core
    # products through residues (18 moduli), with GWB_OZ=1 through 8 int8
    # slices (measured on this path: no faster than DGEMM at these shapes,
    # and a residual floor just above 1e-10 eV on the 216-atom cell)
    oz_mode = os.environ.get("GWB_OZ", "0")
    mm = _Products(dev, oz=("crt" if oz_mode == "crt" else oz_mode == "1") if dev.type == "cuda" else False)
    # the float32 phase's subspace, Ritz and projection products on the
    # tensor cores (GWB_TC_LOW=0: only the first projection pass there) while
    # the largest residual stays above GWB_TC_SWITCH (default 30) times the
    # float32 floor; below it the basis collapses to the Ritz block made
    # orthonormal in float64 and the float32 phase continues on float64
    # products, so that the hand-off block is as good as without them
    tc_low_on = tcp is not None and os.environ.get("GWB_TC_LOW", "1") != "0"
    tc_switch = float(os.environ.get("GWB_TC_SWITCH", "30"))
    eig32 = os.environ.get("GWB_TC_EIG32", "0") == "1"
    # the subspace eigensolves from m = 128 on libgwb's own eigensolver
    # (GWB_OWN_EIGH=0: cuSOLVER through torch.linalg.eigh). Measured on the
    # 216-atom cell: 378 ms of eigensolves against cuSOLVER's 376 ms, 23
    # rounds each.
    own_eigh = _OwnEigh(dev) if dev.type == "cuda" and os.environ.get("GWB_OWN_EIGH", "1") != "0" else None
    info = {"rounds_tc": 0, "rounds_f32": 0, "rounds_f64": 0, "handoff_rn_ev": None, "m": []}
    v0 = _orthonormalize(phi0.clone())
    if v0.shape[0] < nb:  # degenerate start: pad with seeded noise (``:345-350``)
        gen = torch.Generator(device="cpu").manual_seed(1234)
        pad = torch.randn(nb - v0.shape[0], nphi, generator=gen, dtype=torch.float64).to(dev)
        pad = torch.nn.functional.pad(pad, (0, npad - nphi))
        v0 = torch.cat([v0, _orthonormalize(pad, against=v0)])
    V = torch.empty(rows, npad, dtype=torch.float64, device=dev)
    HV = torch.empty(rows, npad, dtype=torch.float64, device=dev)
    m = nb
    V[:m] = v0
    low = mode == "mixed"
    f32, f64 = _lib.GWB_FP32, _lib.GWB_FP64
    cert_floor = 32.0 * float(torch.finfo(torch.float32).eps) * max(float(t_phi.max()), 1.0)
    prev = float("inf")
    HV[:m] = ham.apply_phi(V[:m], prec=f32 if low else f64)
    if tcp is not None:
        tcp.rows(V, HV, 0, m)
    mm.attach(V, HV)
    mm.rows_changed(0, m)
    locked = _Locked(nwant, npad, dev)
    learned = None
    if not (precond is None or (isinstance(precond, str) and precond == "teter")):
        if not hasattr(precond, "params"):
            raise ValueError("precond must be 'teter' or a learned.LearnedPreconditioner")
        learned = _LearnedGamma(precond, nb, gb.t_half, dev)
    # the subspace matrix grows by the new columns only (m0: rows already in it)
    S = torch.zeros(rows, rows, dtype=torch.float64, device=dev)
    m0 = 0

    def certify(x):
        """Float64 apply of the Ritz block and its nb x nb Rayleigh-Ritz
        (gradwave ``solvers/davidson.py:281-308``). After a float32 phase on
        the tensor cores the block is first made orthonormal in float64
        (Cholesky-QR twice; Householder QR if that breaks down)."""
        if tc_low_on and tc_active:
            y = _cholqr(x, mm)
            y = _cholqr(y, mm) if y is not None else None
            if y is None:
                q, _ = torch.linalg.qr(x.T, mode="reduced")
                y = q.T.contiguous()
            x = y
        hx = ham.apply_phi(x, prec=f64)
        g = mm.nt(x, hx)
        if own_eigh is not None and g.shape[0] >= 128:
            w2, u2t = own_eigh.lowest(0.5 * (g + g.T), g.shape[0])
        else:
            w2, u2 = torch.linalg.eigh(0.5 * (g + g.T))
            u2t = u2.T
        x, hx = mm.nn(u2t, x), mm.nn(u2t, hx)
        r = hx - w2[:, None] * x
        return x, hx, w2, r, torch.linalg.vector_norm(r, dim=1)

    def finish(eig, x, rn, nw_a, it):
        if own_eigh is not None:
            own_eigh.check()
        e, xx, r = locked.merge(eig[:nw_a], x[:nw_a], rn[:nw_a])
        return GammaDavidsonResult(e, unembed_real(gb, xx[:, :nphi]), it, r, prof.summary(),
                                   0 if learned is None else learned.n_fallback(), info)

    def phase(name):
        """Phase timer; the float32 phase's share is reported as name/f32."""
        return prof(name + ("/f32" if low else ""))

    tc_active = tc_low_on and low
    it = 0
    for it in range(1, max_iter + 1):
        nb_a = nb - locked.n      # active Ritz block
        nw_a = nwant - locked.n   # wanted pairs still in it
        v, hv = V[:m], HV[:m]
        tc_low = low and tc_active
        info["rounds_tc" if tc_low else ("rounds_f32" if low else "rounds_f64")] += 1
        info["m"].append(m)
        with phase("subspace_gemm"):
            blk = tcp.subspace(hv[m0:m], m, m0) if tc_low else mm.nt(v, hv[m0:m])  # (m, m - m0)
            S[:m, m0:m] = blk
            S[m0:m, :m0] = blk[:m0].T
            S[m0:m, m0:m] = 0.5 * (blk[m0:] + blk[m0:].T)
            m0 = m
            s = S[:m, :m]
        with phase("eigh"):
            if own_eigh is not None and m >= 128:
                eig, ut = own_eigh.lowest(s, nb_a)
            else:
                if tc_low and eig32:
                    # the tensor-core rounds carry ~1e-6 errors: a float32
                    # eigensolve (6-11 % faster in cuSOLVER) is accurate enough
                    w, u = torch.linalg.eigh(s.float())
                    w, u = w.double(), u.double()
                else:
                    w, u = torch.linalg.eigh(s)
                eig = w[:nb_a]
                ut = u[:, :nb_a].T
        with phase("ritz_gemm"):
            if tc_low:
                x, hx = tcp.ritz(ut.contiguous(), m)
            else:
                x = mm.nn(ut, v)
                hx = mm.nn(ut, hv)
        with phase("residual"):
            r = hx - eig[:, None] * x
            rn = torch.linalg.vector_norm(r, dim=1)
            rmax = float(rn[:nw_a].max())
        if tc_low and rmax < tc_switch * cert_floor:
            # leave the tensor-core products: the Ritz block, orthonormal in
            # float64, becomes the basis (its float32 images transformed alike)
            with phase("restart"):
                xo, hxo = _cholqr_images(x.contiguous(), hx.contiguous(), mm)
                V[:nb_a] = xo
                HV[:nb_a] = hxo
                m, m0 = nb_a, 0
                x, hx = V[:nb_a], HV[:nb_a]
                v, hv = V[:m], HV[:m]
                r = hx - eig[:, None] * x
                rn = torch.linalg.vector_norm(r, dim=1)
                rmax = float(rn[:nw_a].max())
                tcp.rows(V, None, 0, m)
                mm.rows_changed(0, m)
                tc_active = False
        if low:
            stalled = it > 1 and rmax > 0.7 * prev and rmax < 100.0 * cert_floor
            prev = rmax
            if rmax < max(tol, cert_floor) or rmax <= tol or stalled:
                with prof("certify"):
                    x, hx, eig, r, rn = certify(x)
                    rmax = float(rn[:nw_a].max())
                info["handoff_rn_ev"] = rmax
                if rmax >= tol:  # hand-off: float64 from the certified block on
                    low = False
                    tc_active = False
                    V[:nb_a] = x
                    HV[:nb_a] = hx
                    m, m0 = nb_a, 0
                    x, hx = V[:nb_a], HV[:nb_a]
                    v, hv = V[:m], HV[:m]
                    if tcp is not None:
                        tcp.rows(V, HV, 0, m)
                    mm.rows_changed(0, m)
        with phase("residual"):
            unconv = rn > tol
            if n_buffer:
                unconv[nw_a:] = rn[nw_a:] > max(tol, buffer_tol)
            done = rmax <= tol
        if done:
            return finish(eig, x, rn, nw_a, it)
        with phase("precondition"):
            if learned is not None:
                pr = learned(x, r, rn, eig, torch.nonzero(unconv).flatten(), npad)
            else:
                t_band = (x * x * t_phi[None, :]).sum(dim=1)
                pr = _teter(r[unconv], t_phi, t_band[unconv])
            pr[:, nphi:] = 0.0  # the pad column is not a coordinate of the operator
        with phase("orthonormalize"):
            t = _expand(pr, v, tcp, locked.rows(), mm, low=low and tc_active)
        if t.shape[0] == 0:  # no independent direction left
            if low:
                x, hx, eig, r, rn = certify(x)
            return finish(eig, x, rn, nw_a, it)
        with phase("apply"):
            ht = ham.apply_phi(t, prec=f32 if low else f64)
        with phase("restart"):
            nt = int(t.shape[0])
            lockable = (rn[:nw_a] <= tol) if (lock and not low) else None
            n_lock = int(lockable.sum()) if lockable is not None else 0
            if m + nt > max_dim:
                # restart: [Ritz block, t]; t is orthogonal to all of v and to
                # the locked rows. Wanted pairs within tol are locked first.
                keep = torch.ones(nb_a, dtype=torch.bool, device=dev)
                if n_lock:
                    keep[:nw_a] = ~lockable
                    if learned is not None:
                        learned.keep(keep)
                    locked.add(x[:nw_a][lockable], hx[:nw_a][lockable], eig[:nw_a][lockable],
                               rn[:nw_a][lockable])
                xk, hxk = x[keep], hx[keep]   # copies (x may alias V rows)
                k = int(xk.shape[0])
                V[:k] = xk
                HV[:k] = hxk
                # the active Ritz block is now the kept rows
                x, hx, eig, rn = V[:k], HV[:k], eig[keep], rn[keep]
                r0, m, m0 = 0, k, 0
            else:
                r0 = m
            V[m:m + nt] = t
            HV[m:m + nt] = ht
            m += nt
            if tcp is not None:
                tcp.rows(V, HV if (low and tc_active) else None, r0, m)
            mm.rows_changed(r0, m)
    if low:  # out of rounds in float32: certify what there is
        x, hx, eig, r, rn = certify(x)
    return finish(eig, x, rn, nwant - locked.n, max_iter)


def gamma_start(gb: GammaBasis, nb: int, device=None) -> torch.Tensor:
    """Identity start on the lowest-|G|^2 half-sphere slots (the
    ``scf/loop.py:705-706`` cold start restricted to real states)."""
    x0 = torch.zeros(nb, gb.nhalf, dtype=torch.complex128, device=device)
    x0[torch.arange(nb), torch.arange(nb)] = 1.0
    return x0
