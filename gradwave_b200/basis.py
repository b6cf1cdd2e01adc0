"""Plane-wave basis set-up for the band solve: FFT box, G-spheres, k-meshes,
Kleinman-Bylander projector tables and the padded per-k batch.

This is the host-side set-up that feeds the device path once per geometry. It
mirrors the reference's set-up API so a caller can hand the same objects to
either implementation:

* ``build_fft_grid``     - gradwave ``grids.py:68-126``
* ``build_gsphere``      - gradwave ``grids.py:145-184``
* ``monkhorst_pack``     - gradwave ``kpoints.py:15-54``
* ``ylm_real``           - gradwave ``core/ylm.py:45-118`` (QE m order)
* ``build_projector_data`` - gradwave ``core/hamiltonian.py:46-105``
* ``build_batched``      - gradwave ``core/batch.py:174-205``
* ``projectors_b``       - gradwave ``core/batch.py:229-235``

Conventions that the device kernels depend on (and that must match the
reference bit for bit, because they decide which box cell a coefficient lands
in):

* box index of Miller triple m is ``(m0 % n0)*n1*n2 + (m1 % n1)*n2 + (m2 % n2)``;
* sphere order is ascending |k+G|^2 (rounded to 1e-10), ties broken by the
  Miller triple (m0, m1, m2) lexicographically;
* padded slots of a batch carry flat index 0, kinetic 0, projector 0 and
  mask False.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from .constants import HBAR2_2M


def reciprocal_cell(cell: np.ndarray) -> np.ndarray:
    """Rows b_i with a_i . b_j = 2 pi delta_ij (cell rows a_i in A)."""
    return 2.0 * np.pi * np.linalg.inv(np.asarray(cell, dtype=np.float64)).T


def good_fft_size(n: int) -> int:
    """Smallest m >= n whose prime factors are all in {2, 3, 5, 7}."""
    m = int(n)
    while True:
        r = m
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def gmax_from_ecut(ecut: float) -> float:
    """Radius of the wavefunction sphere |k+G| <= sqrt(ecut / (hbar^2/2m))."""
    return math.sqrt(ecut / HBAR2_2M)


@dataclass(frozen=True)
class FFTGrid:
    cell: np.ndarray          # (3, 3) rows a_i [A]
    shape: tuple[int, int, int]
    miller: np.ndarray        # (n0, n1, n2, 3) signed Miller index of each box cell
    g_cart: np.ndarray        # (n0, n1, n2, 3) Cartesian G [1/A]

    @property
    def volume(self) -> float:
        return float(abs(np.linalg.det(self.cell)))

    @property
    def n_points(self) -> int:
        return int(np.prod(self.shape))


def build_fft_grid(cell, ecut: float, shape_override=None) -> FFTGrid:
    """Dense box that holds the density sphere |G| <= 2 G_max, or the pinned
    ``shape_override`` (the reference's ``grids.py:93-95``)."""
    cell = np.asarray(cell, dtype=np.float64)
    b = reciprocal_cell(cell)
    if shape_override is not None:
        shape = tuple(int(n) for n in shape_override)
    else:
        g2max = 2.0 * gmax_from_ecut(ecut)
        shape = tuple(
            good_fft_size(2 * int(np.floor(g2max * np.linalg.norm(cell[i]) / (2 * np.pi))) + 1)
            for i in range(3))
    axes = [np.rint(np.fft.fftfreq(n, d=1.0 / n)).astype(np.int64) for n in shape]
    m = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)
    return FFTGrid(cell=cell, shape=shape, miller=m, g_cart=m @ b)


@dataclass(frozen=True)
class GSphere:
    k_frac: np.ndarray        # (3,)
    miller: np.ndarray        # (npw, 3) int64
    kpg: np.ndarray           # (npw, 3) [1/A]
    kpg2: np.ndarray          # (npw,) [1/A^2]
    flat_idx: np.ndarray      # (npw,) int64 box index

    @property
    def npw(self) -> int:
        return int(self.miller.shape[0])


def build_gsphere(grid: FFTGrid, ecut: float, k_frac) -> GSphere:
    """All G with (hbar^2/2m)|k+G|^2 <= ecut as box indices of ``grid``."""
    cell = grid.cell
    b = reciprocal_cell(cell)
    k_frac = np.asarray(k_frac, dtype=np.float64)
    gmax = gmax_from_ecut(ecut)
    reach = [int(np.floor(gmax * np.linalg.norm(cell[i]) / (2 * np.pi) + 1)) + 1 for i in range(3)]
    cand = np.stack(np.meshgrid(*[np.arange(-r, r + 1) for r in reach], indexing="ij"),
                    axis=-1).reshape(-1, 3)
    kpg = (cand + k_frac) @ b
    kpg2 = np.einsum("ij,ij->i", kpg, kpg)
    inside = HBAR2_2M * kpg2 <= ecut * (1 + 1e-12)
    mm, kpg, kpg2 = cand[inside], kpg[inside], kpg2[inside]
    n0, n1, n2 = grid.shape
    for axis, n in enumerate(grid.shape):
        if np.any(np.abs(mm[:, axis]) > n // 2):
            raise RuntimeError("wavefunction sphere does not fit the FFT box")
    flat = (mm[:, 0] % n0) * (n1 * n2) + (mm[:, 1] % n1) * n2 + (mm[:, 2] % n2)
    order = np.lexsort((mm[:, 2], mm[:, 1], mm[:, 0], np.round(kpg2, 10)))
    return GSphere(k_frac=k_frac, miller=mm[order].astype(np.int64), kpg=kpg[order],
                   kpg2=kpg2[order], flat_idx=flat[order].astype(np.int64))


def monkhorst_pack(mesh, shift=(0, 0, 0), time_reversal: bool = True):
    """Gamma-centred (QE-shift) mesh folded to (-1/2, 1/2], optionally halved
    by k ~ -k. Returns (k_frac (nk, 3), weights (nk,)) with weights summing to 1."""
    mesh = np.asarray(mesh, dtype=np.int64)
    shift = np.asarray(shift, dtype=np.float64)
    if mesh.shape != (3,) or np.any(mesh < 1):
        raise ValueError(f"bad k-mesh {mesh}")
    if not np.all(np.isin(shift, (0.0, 1.0))):
        raise ValueError("shift components must be 0 or 1")

    def fold(x):
        return -((0.5 - x) % 1.0 - 0.5)

    axes = [(np.arange(n) + 0.5 * s) / n for n, s in zip(mesh, shift)]
    k = fold(np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3))
    w = np.full(len(k), 1.0 / len(k))
    if not time_reversal:
        return k, w
    index: dict[tuple, int] = {}
    ks, ws = [], []
    for ki, wi in zip(k, w):
        partner = tuple(np.round(fold(-ki), 9))
        if partner in index:
            ws[index[partner]] += wi
            continue
        index[tuple(np.round(ki, 9))] = len(ks)
        ks.append(ki)
        ws.append(wi)
    return np.array(ks), np.array(ws)


# Real spherical harmonics, QE m order within each l: 0, +1, -1, +2, -2, ...
# Normalisation: integral over the unit sphere of Y_lm^2 = 1.
def ylm_real(lmax: int, g: np.ndarray) -> np.ndarray:
    """(..., (lmax+1)^2) real harmonics at directions g (zero vectors give the
    q -> 0 limit: Y_00 only)."""
    if lmax > 2:
        raise ValueError("ylm_real supports l <= 2 (s, p, d channels)")
    g = np.asarray(g, dtype=np.float64)
    n2 = np.einsum("...i,...i->...", g, g)
    zero = n2 < 1e-28
    norm = np.sqrt(np.where(zero, 1.0, n2))
    u = np.where(zero[..., None], 0.0, g / norm[..., None])
    x, y, z = u[..., 0], u[..., 1], u[..., 2]
    r2 = x * x + y * y + z * z
    out = [np.full(x.shape, 0.5 / math.sqrt(math.pi))]
    if lmax >= 1:
        c1 = math.sqrt(3.0 / (4.0 * math.pi))
        out += [c1 * z, c1 * x, c1 * y]
    if lmax >= 2:
        c20 = math.sqrt(5.0 / math.pi) / 4.0
        c21 = math.sqrt(15.0 / math.pi) / 2.0
        c22 = math.sqrt(15.0 / math.pi) / 4.0
        out += [c20 * (3.0 * z * z - r2), c21 * x * z, c21 * y * z,
                c22 * (x * x - y * y), c21 * x * y]
    return np.stack(out, axis=-1)


@dataclass
class ProjectorData:
    atom_index: np.ndarray        # (nproj,) atom of each projector column
    f_ylm_phase_free: np.ndarray  # (nproj, npw) complex (4pi/sqrt(V)) (-i)^l Y_lm F(|k+G|)
    kpg: np.ndarray               # (npw, 3)
    dij_full: np.ndarray          # (nproj, nproj) real, block diagonal over atoms


_MINUS_I_POW = (1.0 + 0.0j, -1.0j, -1.0 + 0.0j)


def build_projector_data(sphere: GSphere, species_of_atom, beta_tables, beta_ls,
                         dij_species, volume: float) -> ProjectorData:
    """m-expanded projector columns for one k-point. Column order: atoms in
    order; per atom its channels in order; per channel m in QE order. The D
    block couples (i, m) with (j, m) for channels of equal l."""
    lmax = max((max(ls) for ls in beta_ls if ls), default=0)
    y = ylm_real(lmax, sphere.kpg)
    pref = 4.0 * math.pi / math.sqrt(volume)
    cols, atoms, blocks = [], [], []
    for a, s in enumerate(species_of_atom):
        ls = list(beta_ls[s])
        tab = np.asarray(beta_tables[s])
        offs = np.concatenate([[0], np.cumsum([2 * l + 1 for l in ls])]).astype(int)
        for i, l in enumerate(ls):
            for mc in range(2 * l + 1):
                cols.append(pref * _MINUS_I_POW[l] * (tab[i] * y[:, l * l + mc]))
                atoms.append(a)
        blk = np.zeros((offs[-1], offs[-1]))
        dsp = np.asarray(dij_species[s], dtype=np.float64)
        for i, li in enumerate(ls):
            for j, lj in enumerate(ls):
                if li == lj:
                    for mc in range(2 * li + 1):
                        blk[offs[i] + mc, offs[j] + mc] = dsp[i, j]
        blocks.append(blk)
    nproj = len(cols)
    dfull = np.zeros((nproj, nproj))
    o = 0
    for blk in blocks:
        dfull[o:o + blk.shape[0], o:o + blk.shape[0]] = blk
        o += blk.shape[0]
    f = (np.stack(cols).astype(np.complex128) if cols
         else np.zeros((0, sphere.npw), dtype=np.complex128))
    return ProjectorData(atom_index=np.asarray(atoms, dtype=np.int64), f_ylm_phase_free=f,
                         kpg=sphere.kpg, dij_full=dfull)


@dataclass
class BatchedK:
    """Padded per-k tables (the reference's ``BatchedK``, ``core/batch.py:126-171``).

    Tensors live on the CPU after ``build_batched``; ``to(device)`` moves them."""
    npw: torch.Tensor             # (nk,) int64
    mask: torch.Tensor            # (nk, npw_max) bool
    flat_idx: torch.Tensor        # (nk, npw_max) int64, 0 in padding
    kpg: torch.Tensor             # (nk, npw_max, 3) float64
    t: torch.Tensor               # (nk, npw_max) float64 kinetic, 0 in padding
    proj_phase_free: torch.Tensor  # (nk, nproj, npw_max) complex128
    proj_atom_index: torch.Tensor  # (nproj,) int64
    dij_full: torch.Tensor        # (nproj, nproj) float64

    @property
    def nk(self) -> int:
        return int(self.npw.shape[0])

    @property
    def npw_max(self) -> int:
        return int(self.mask.shape[1])

    def to(self, device) -> "BatchedK":
        return BatchedK(*(getattr(self, f).to(device) for f in (
            "npw", "mask", "flat_idx", "kpg", "t", "proj_phase_free",
            "proj_atom_index", "dij_full")))


def build_batched(spheres, proj_data) -> BatchedK:
    nk = len(spheres)
    npw = np.array([s.npw for s in spheres], dtype=np.int64)
    m = int(npw.max())
    nproj = proj_data[0].f_ylm_phase_free.shape[0] if proj_data else 0
    mask = np.zeros((nk, m), dtype=bool)
    flat = np.zeros((nk, m), dtype=np.int64)
    kpg = np.zeros((nk, m, 3))
    t = np.zeros((nk, m))
    pf = np.zeros((nk, nproj, m), dtype=np.complex128)
    for ik, (s, pd) in enumerate(zip(spheres, proj_data, strict=True)):
        n = s.npw
        mask[ik, :n] = True
        flat[ik, :n] = s.flat_idx
        kpg[ik, :n] = s.kpg
        t[ik, :n] = HBAR2_2M * s.kpg2
        if nproj:
            pf[ik, :, :n] = pd.f_ylm_phase_free
    return BatchedK(
        npw=torch.from_numpy(npw), mask=torch.from_numpy(mask), flat_idx=torch.from_numpy(flat),
        kpg=torch.from_numpy(kpg), t=torch.from_numpy(t), proj_phase_free=torch.from_numpy(pf),
        proj_atom_index=torch.from_numpy(proj_data[0].atom_index if nproj
                                         else np.zeros(0, dtype=np.int64)),
        dij_full=torch.from_numpy(proj_data[0].dij_full if nproj else np.zeros((0, 0))))


def projectors_b(bk: BatchedK, positions) -> torch.Tensor:
    """Full projectors p = f_ylm_phase_free * exp(-i (k+G) . tau_atom), (nk, nproj, npw_max)."""
    if bk.proj_phase_free.shape[1] == 0:
        return bk.proj_phase_free
    pos = torch.as_tensor(np.asarray(positions, dtype=np.float64), device=bk.kpg.device)
    arg = torch.einsum("kgi,ai->kga", bk.kpg, pos)
    phase = torch.exp(torch.complex(torch.zeros_like(arg), -arg))
    return bk.proj_phase_free * phase[:, :, bk.proj_atom_index].permute(0, 2, 1)
