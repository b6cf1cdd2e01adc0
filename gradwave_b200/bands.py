"""Non-SCF band structure at a frozen potential on the B200 path (gradwave
``postscf/bands.py:39-111``, ``band_structure``).

The reference's driver, step for step:

* the path's k-points go through the k-batched solver in chunks of at most
  24, fewer when nbands x box x 16 bytes of dense boxes would pass a 1.5 GB
  budget (``postscf/bands.py:64-66``);
* per chunk: spheres, projector tables and projectors at those k
  (``:72-83``), the Hamiltonian with the frozen V_eff(r), an identity cold
  start on the lowest-|k+G|^2 plane waves, and a Davidson solve to
  ``diago_tol`` with ``max_iter`` 80 (``:84-89``; the reference calls
  ``davidson_batched_ms`` with mixed precision off, i.e. one float64 solve);
* the energy reference: the reference reads the Fermi level or the valence
  band maximum from the SCF result (``:97-108``). Here the cells are
  insulators with fixed occupations and there is no SCF result, so the
  default reference is the valence-band maximum of the path itself (the
  highest eigenvalue of band nocc); a caller with an SCF result passes its
  own.

``k_path`` stands in for ASE's ``bandpath`` (ASE is not a dependency of this
path): straight segments between special points, sampled in proportion to
their reciprocal-space length, with the cumulative path coordinate and the
special-point labels.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .cells import CellInputs, at_kpoints


@dataclass
class BandStructure:
    kpts_frac: np.ndarray                       # (nkpath, 3)
    eigenvalues: np.ndarray                     # (nkpath, nbands) [eV], not referenced
    reference: float                            # valence-band maximum (or the caller's) [eV]
    labels: list[tuple[int, str]] | None = None  # (index, label) special points
    x: np.ndarray | None = None                 # path coordinate [1/A]
    n_iter: list[int] | None = None             # Davidson rounds per chunk


def chunk_size(nbands: int, box_points: int) -> int:
    """k-points per batched solve (gradwave ``postscf/bands.py:64-66``)."""
    return max(1, min(24, int(1.5e9 / (nbands * box_points * 16))))


def k_path(cell: np.ndarray, points: list[tuple[str, list[float]]], npoints: int):
    """(kpts_frac (n, 3), x (n,), labels [(index, label)]) along straight
    segments between the special points (fractional coordinates of the
    reciprocal lattice of ``cell``, rows = lattice vectors), ``npoints`` in
    total, each segment sampled in proportion to its length; the special
    points themselves are on the path."""
    if len(points) < 2:
        raise ValueError("a path needs at least two special points")
    if npoints < len(points):
        raise ValueError(f"{npoints} points cannot hold {len(points)} special points")
    recip = 2.0 * np.pi * np.linalg.inv(np.asarray(cell, dtype=np.float64)).T
    frac = np.array([p[1] for p in points], dtype=np.float64)
    seg = np.linalg.norm(np.diff(frac @ recip, axis=0), axis=1)
    total = float(seg.sum())
    # interior samples per segment, largest remainders first
    inner = npoints - len(points)
    share = seg / total * inner if total > 0 else np.full(len(seg), inner / len(seg))
    n_in = np.floor(share).astype(int)
    for i in np.argsort(-(share - n_in))[: inner - int(n_in.sum())]:
        n_in[i] += 1
    kpts, labels = [frac[0]], [(0, points[0][0])]
    for s in range(len(seg)):
        for j in range(1, n_in[s] + 2):
            kpts.append(frac[s] + (frac[s + 1] - frac[s]) * j / (n_in[s] + 1))
        labels.append((len(kpts) - 1, points[s + 1][0]))
    kpts = np.array(kpts)
    x = np.concatenate([[0.0], np.cumsum(np.linalg.norm(np.diff(kpts @ recip, axis=0), axis=1))])
    return kpts, x, labels


@torch.no_grad()
def band_structure(ci: CellInputs, kpts_frac, nbands: int | None = None, diago_tol: float = 1e-9,
                   max_iter: int = 80, chunk: int | None = None, reference: float | None = None,
                   mode: str = "fp64", precond="teter", device=None) -> BandStructure:
    """Eigenvalues along ``kpts_frac`` at the cell's frozen potential
    (gradwave ``postscf/bands.py:39-111``); see the module docstring."""
    from .davidson import davidson_batched
    from .hamiltonian import BatchedHamiltonian
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    kpts = np.asarray(kpts_frac, dtype=np.float64).reshape(-1, 3)
    nb = int(nbands or ci.nbands)
    n_box = int(np.prod(ci.shape))
    ch = chunk_size(nb, n_box) if chunk is None else int(chunk)
    eigs = np.empty((len(kpts), nb))
    rounds = []
    for lo in range(0, len(kpts), ch):
        hi = min(lo + ch, len(kpts))
        cp = at_kpoints(ci, kpts[lo:hi])
        bk = cp.bk.to(dev)
        h = BatchedHamiltonian(bk, cp.shape, cp.v_eff_r, cp.p)
        x0 = cp.identity_start(nb).to(dev)
        res = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=diago_tol, max_iter=max_iter, mode=mode,
                               precond=precond)
        eigs[lo:hi] = res.eigenvalues.cpu().numpy()
        rounds.append(int(res.n_iter))
    if reference is None:
        nocc = ci.nocc()
        reference = float(eigs[:, nocc - 1].max()) if nocc <= nb else float("nan")
    return BandStructure(kpts_frac=kpts, eigenvalues=eigs, reference=float(reference), n_iter=rounds)


def bands_along_path(ci: CellInputs, points: list[tuple[str, list[float]]], npoints: int = 120,
                     nbands: int | None = None, **kw) -> BandStructure:
    """Band structure along the special points (the role of gradwave's
    ``bands_along_ase_path``, ``postscf/bands.py:113-120``)."""
    kpts, x, labels = k_path(ci.cell, points, npoints)
    bs = band_structure(ci, kpts, nbands=nbands, **kw)
    bs.x, bs.labels = x, labels
    return bs
