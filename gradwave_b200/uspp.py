"""Generalized (USPP/PAW) band solve H x = eps S x on the B200 path (drop-in for
gradwave's ``scf/uspp_batch.py``: ``BatchedHS`` and ``davidson_gen_batched``).

* ``BatchedHS(bk, shape, v_eff_r, p, dscr, q_full)``: ``h`` is this package's
  ``BatchedHamiltonian`` apply (the libgwb.so kernels) with the screened
  D ``dscr`` in place of the bare one; ``s`` is S c = c + sum_pq |beta_p>
  q_pq <beta_q|c>, masked: one more projector contraction, as two batched
  cuBLAS products (``scf/uspp_batch.py:27-73``).
* ``davidson_gen_batched``: the reference's generalized block Davidson
  (``scf/uspp_batch.py:99-233``), step for step, with every step on the
  device:
  - subspace matrices v^H H v and v^H S v in float64;
  - Cholesky of the overlap; while it fails (an indefinite S on a truncated
    sphere) drop the oldest basis vectors, else a 1e-10 shift;
  - the reduction L^-1 H L^-H (the Hermitian form), eigh, back-solve
    L^-H u;
  - Ritz blocks x, Hx, Sx and residuals Hx - eps Sx;
  - uniform expansion across k: the worst max_k #(|r| > tol) residuals;
  - TPA scaled by the band kinetic energy, rows unit-normalised;
  - a restart re-orthonormalises the Ritz block in the standard metric and
    carries Hx, Sx by the triangular factor;
  - orthonormalisation in the standard metric: mask, two projections,
    seeded noise for vanished rows, then CholQR2 with a Householder QR
    fallback (the reference's Householder QR by default, same span).
  The reference ships the small subspace solves to the CPU to avoid cuSOLVER's
  host reads; here they stay on the GPU (one host read per round, the
  Cholesky status).
"""

from __future__ import annotations

import torch

from .basis import BatchedK
from .hamiltonian import BatchedHamiltonian


class BatchedHS:
    def __init__(self, bk, shape, v_eff_r, p, dscr, q_full, hub_sphi=None, hub_d=None, smooth=None,
                 metagga_v=None):
        if hub_sphi is not None or hub_d is not None or smooth is not None or metagga_v is not None:
            raise NotImplementedError("DFT+U, the dual grid and meta-GGA are not part of the B200 band-solve path")
        self.bk = bk
        self.shape = tuple(int(s) for s in shape)
        bks = BatchedK(bk.npw, bk.mask, bk.flat_idx, bk.kpg, bk.t, bk.proj_phase_free, bk.proj_atom_index,
                       torch.as_tensor(dscr, dtype=torch.float64))
        self.ham = BatchedHamiltonian(bks, self.shape, v_eff_r, p)
        dev = self.ham.device
        self.p = torch.as_tensor(p).to(dev, torch.complex128).contiguous()
        self.p_conj_t = self.p.conj().transpose(-1, -2).contiguous()  # (nk, npw, nproj)
        self.q = torch.as_tensor(q_full).to(dev, torch.complex128).contiguous()
        self.mask = bk.mask.to(dev)
        self.t = bk.t.to(dev, torch.float64)

    def h(self, c: torch.Tensor) -> torch.Tensor:
        return self.ham.apply(c)

    def s(self, c: torch.Tensor) -> torch.Tensor:
        """S c = (c + (c P^H) q P) * mask, in the dtype of c."""
        dt = c.dtype
        b = torch.matmul(c, self.p_conj_t.to(dt))                 # (nk, nb, nproj)
        out = c + torch.matmul(torch.matmul(b, self.q.to(dt)), self.p.to(dt))
        return out * self.mask[:, None, :]


def _teter_b(r: torch.Tensor, t: torch.Tensor, t_band: torch.Tensor) -> torch.Tensor:
    """Batched TPA filter (gradwave ``solvers/precond.py:20-39``)."""
    x = t.double()[:, None, :] / torch.clamp(t_band.double()[..., None], min=1e-12)
    x2 = x * x
    num = 27.0 + 18.0 * x + 12.0 * x2 + 8.0 * x2 * x
    return r * (num / (num + 16.0 * x2 * x2)).to(r.real.dtype)


def _orthonormal_rows(x: torch.Tensor) -> torch.Tensor:
    """Rows of x (nk, j, npw) orthonormal per k: CholQR2, Householder QR when a
    Cholesky breaks down."""
    y = x
    for _ in range(2):
        g = torch.matmul(y, y.conj().transpose(-1, -2))
        L, info = torch.linalg.cholesky_ex(g)
        if int(info.max()) != 0:
            q, _ = torch.linalg.qr(x.transpose(-1, -2), mode="reduced")
            return q.transpose(-1, -2)
        y = torch.linalg.solve_triangular(L, y, upper=False)
    return y


def _orthonormalize_b(v: torch.Tensor, mask: torch.Tensor, against: torch.Tensor | None = None) -> torch.Tensor:
    """Mask, two projections against ``against``, seeded noise in rows that
    vanished (norm < 1e-8) followed by a re-projection, orthonormal rows
    (gradwave ``solvers/davidson.py:406-457``)."""

    def project(x):
        if against is not None and against.shape[1]:
            for _ in range(2):
                x = x - torch.matmul(torch.matmul(x, against.conj().transpose(-1, -2)), against)
        return x

    v = project(v * mask[:, None, :])
    bad = torch.linalg.vector_norm(v, dim=-1, keepdim=True) < 1e-8
    if bool(bad.any()):
        gen = torch.Generator(device="cpu").manual_seed(v.shape[1] + 7919)
        noise = torch.view_as_complex(torch.randn(*v.shape, 2, generator=gen, dtype=torch.float64))
        v = project((v + bad * noise.to(v.device).to(v.dtype)) * mask[:, None, :])
    return _orthonormal_rows(v)


def _sym(a: torch.Tensor) -> torch.Tensor:
    return 0.5 * (a + a.conj().transpose(-1, -2))


@torch.no_grad()
def davidson_gen_batched(hs: BatchedHS, x0: torch.Tensor, nbands: int, tol: float, max_iter: int = 60,
                         max_dim_factor: int = 4):
    """Block Davidson for H x = eps S x over (nk, ., npw_max) blocks; returns
    (eig (nk, nbands), x (nk, nbands, npw_max)), x Ritz-rotated from a
    standard-orthonormal basis (not S-normalised), as the reference."""
    nk, _, npw = x0.shape
    mask = hs.mask
    x0 = x0.to(mask.device)
    max_dim = min(int(hs.bk.npw.min()), max(max_dim_factor * nbands, nbands + 24))
    v = _orthonormalize_b(x0, mask)
    hv, sv = hs.h(v), hs.s(v)
    eig = x = None
    for _ in range(max_iter):
        while True:
            vc = v.conj()
            h_sub = _sym(torch.matmul(vc, hv.transpose(-1, -2)).to(torch.complex128))
            s_sub = _sym(torch.matmul(vc, sv.transpose(-1, -2)).to(torch.complex128))
            L, info = torch.linalg.cholesky_ex(s_sub)
            bad = int(info.max()) > 0
            if not bad or v.shape[1] <= nbands + 1:
                break
            v, hv, sv = v[:, 1:], hv[:, 1:], sv[:, 1:]  # drop the oldest direction
        if bad:
            eye = torch.eye(s_sub.shape[-1], dtype=s_sub.dtype, device=s_sub.device)
            L = torch.linalg.cholesky(s_sub + 1e-10 * eye)
        a = torch.linalg.solve_triangular(L, h_sub, upper=False)
        a = torch.linalg.solve_triangular(L, a.conj().transpose(-1, -2), upper=False).conj().transpose(-1, -2)
        w, u = torch.linalg.eigh(_sym(a))
        u = torch.linalg.solve_triangular(L.conj().transpose(-1, -2), u, upper=True)
        eig = w[:, :nbands].real
        ur = u[:, :, :nbands].transpose(-1, -2).to(x0.dtype)
        x, hx, sx = torch.matmul(ur, v), torch.matmul(ur, hv), torch.matmul(ur, sv)
        r = hx - eig[..., None].to(x0.dtype) * sx
        rn = torch.linalg.vector_norm(r, dim=-1)
        if float(rn.max()) < tol:
            return eig, x
        n_add = int((rn > tol).sum(dim=1).max())
        sel = torch.argsort(rn, dim=1, descending=True)[:, :n_add]
        r_sel = torch.gather(r, 1, sel[..., None].expand(-1, -1, npw))
        t_band = torch.einsum("kbg,kg,kbg->kb", x.conj(), hs.t.to(x.dtype), x).real
        d = _teter_b(r_sel, hs.t.to(r_sel.real.dtype), torch.gather(t_band, 1, sel))
        dn = torch.linalg.vector_norm(d, dim=-1, keepdim=True)
        d = torch.where(dn > 1e-300, d / dn.clamp_min(1e-300), d)
        if v.shape[1] + n_add > max_dim:
            q, rm = torch.linalg.qr(x.transpose(-1, -2), mode="reduced")
            rt = rm.transpose(-1, -2)
            v = q.transpose(-1, -2).contiguous()
            hv = torch.linalg.solve_triangular(rt, hx, upper=False)
            sv = torch.linalg.solve_triangular(rt, sx, upper=False)
        d = _orthonormalize_b(d, mask, against=v)
        v = torch.cat([v, d], dim=1)
        hv = torch.cat([hv, hs.h(d)], dim=1)
        sv = torch.cat([sv, hs.s(d)], dim=1)
    return eig, x
