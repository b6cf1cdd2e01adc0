"""Seeded synthetic diamond-Si cells: the inputs of every band-solve workload.

Each named cell (``data/cells.json``) becomes the full input set of one band
solve: FFT box, per-k G-spheres, the padded batch, the real local potential
v(r) on the box, the m-expanded Kleinman-Bylander projectors and the identity
start block. Set-up runs on the host with numpy, once per geometry.

Workloads (sizes are those the reference's own sphere builder gives):

==============  ======  ====  =====  =========  ======  =====
name            atoms   ecut  box    k-points   npw     bands
==============  ======  ====  =====  =========  ======  =====
si2_fcc         2       30Ry  24^3   Gamma      749     8
si8_cubic       8       40Ry  36^3   10 IBZ     ~4620   24
si64_cubic      64      40Ry  72^3   4 IBZ      ~36950  160
si8_perturbed   8       40Ry  36^3   36 (TR)    ~4620   24
si216_vacancy   216     30Ry  96^3   Gamma      80797   480
==============  ======  ====  =====  =========  ======  =====

The box is pinned (the reference's ``shape_override``, ``grids.py:78,93-95``);
the wavefunction sphere fits in every pinned box.
"""

from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from .basis import (BatchedK, FFTGrid, GSphere, build_batched, build_fft_grid,
                    build_gsphere, build_projector_data, monkhorst_pack, projectors_b)
from .constants import RY_EV

_SPEC = json.loads((Path(__file__).parent / "data" / "cells.json").read_text())

_FCC_PRIM = np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]])
_DIAMOND_CUBIC_FRAC = np.array([
    [0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25]])


def cell_names() -> list[str]:
    return list(_SPEC["cells"])


def _ibz_oh(n: int):
    """Irreducible k of an n x n x n Gamma-centred mesh of a simple-cubic
    lattice under O_h: k = (i, j, l)/n with n/2 >= i >= j >= l >= 0, weighted by
    the size of each star in the full mesh."""
    pts, wts = [], []
    half = n // 2
    full = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    canon = np.sort(np.minimum(full % n, (-full) % n), axis=1)[:, ::-1]
    for i in range(half + 1):
        for j in range(i + 1):
            for l in range(j + 1):
                star = int(np.sum(np.all(canon == (i, j, l), axis=1)))
                pts.append(np.array([i, j, l], dtype=np.float64) / n)
                wts.append(star / n ** 3)
    return np.array(pts), np.array(wts)


def _kpoints(kind: str):
    if kind == "gamma":
        return np.zeros((1, 3)), np.ones(1)
    if kind == "ibz444_oh":
        return _ibz_oh(4)
    if kind == "ibz222_oh":
        return _ibz_oh(2)
    if kind == "mp444_tr":
        return monkhorst_pack((4, 4, 4))
    raise ValueError(f"unknown k-point set {kind!r}")


def _structure(spec: dict, rng: np.random.Generator | None):
    a = float(spec["a"])
    if spec["lattice"] == "fcc":
        cell = a / 2 * _FCC_PRIM
        frac = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])
    else:
        s = int(spec["supercell"])
        cell = np.eye(3) * a * s
        shifts = np.stack(np.meshgrid(*[np.arange(s)] * 3, indexing="ij"), -1).reshape(-1, 3)
        frac = ((shifts[:, None, :] + _DIAMOND_CUBIC_FRAC[None]) / s).reshape(-1, 3)
    pos = frac @ cell
    if rng is not None and "strain" in spec:
        eps = rng.uniform(-spec["strain"], spec["strain"], size=3)
        cell = cell @ np.diag(1.0 + eps)
        pos = frac @ cell + rng.normal(0.0, spec["displacement_sigma"], size=pos.shape)
    return cell, pos


def local_potential(grid: FFTGrid, positions: np.ndarray, A: float, sigma: float,
                    extra_gaussians=()) -> np.ndarray:
    """v(r) on the box, real, [eV]: the Fourier series of
    V(G) = sum_a exp(-i G.tau_a) A exp(-sigma^2 G^2 / 2) / Omega over every box G,
    plus optional periodic Gaussian bumps (height h [eV], width s [A], centre R)."""
    g = grid.g_cart
    g2 = np.einsum("...i,...i->...", g, g)
    vol = grid.volume
    sfac = np.zeros(grid.shape, dtype=np.complex128)
    for tau in positions:
        sfac += np.exp(-1j * (g @ tau))
    vg = sfac * (A * np.exp(-0.5 * sigma ** 2 * g2) / vol)
    for h, s, centre in extra_gaussians:
        vg += h * (2 * math.pi * s * s) ** 1.5 / vol * np.exp(-0.5 * s * s * g2) \
            * np.exp(-1j * (g @ centre))
    n = grid.n_points
    return np.ascontiguousarray(np.real(np.fft.ifftn(vg) * n))


@dataclass
class CellInputs:
    name: str
    cell: np.ndarray
    positions: np.ndarray
    ecut: float                  # eV
    grid: FFTGrid
    spheres: list[GSphere]
    kpoints: np.ndarray
    kweights: np.ndarray
    bk: BatchedK
    v_eff_r: torch.Tensor        # (n0, n1, n2) float64 [eV]
    p: torch.Tensor              # (nk, nproj, npw_max) complex128
    nbands: int
    meta: dict = field(default_factory=dict)

    @property
    def shape(self) -> tuple[int, int, int]:
        return self.grid.shape

    def identity_start(self, nb: int | None = None) -> torch.Tensor:
        """Identity block on the lowest-|k+G|^2 plane waves (the reference's
        ``scf/loop.py:705-706`` cold start)."""
        nb = self.nbands if nb is None else nb
        x0 = torch.zeros(self.bk.nk, nb, self.bk.npw_max, dtype=torch.complex128)
        idx = torch.arange(nb)
        x0[:, idx, idx] = 1.0
        return x0

    def nocc(self) -> int:
        return 2 * len(self.positions)   # 4 valence electrons per Si, 2 per band


def _projector_tables(spheres, positions, volume):
    """Per-k projector data of the analytic s + p Kleinman-Bylander channels
    (the recipe every cell uses)."""
    sp = _SPEC["species"]["Si"]
    rc = float(sp["rc"])
    pds = []
    for s in spheres:
        q = np.sqrt(s.kpg2)
        tab = np.stack([np.exp(-0.5 * (q * rc) ** 2), q * rc * np.exp(-0.5 * (q * rc) ** 2)])
        pds.append(build_projector_data(s, [0] * len(positions), [tab], [[0, 1]], [np.diag(sp["D"])], volume))
    return pds


def at_kpoints(ci: CellInputs, kpoints_frac, kweights=None) -> CellInputs:
    """The same cell, box and frozen potential at other k-points (fractional
    coordinates): spheres, batched tables and projectors rebuilt, weights
    uniform unless given (the non-SCF set-up of gradwave
    ``postscf/bands.py:68-85``)."""
    kfr = np.asarray(kpoints_frac, dtype=np.float64).reshape(-1, 3)
    kw = np.full(len(kfr), 1.0 / len(kfr)) if kweights is None else np.asarray(kweights, dtype=np.float64)
    spheres = [build_gsphere(ci.grid, ci.ecut, k) for k in kfr]
    bk = build_batched(spheres, _projector_tables(spheres, ci.positions, ci.grid.volume))
    p = projectors_b(bk, ci.positions)
    return CellInputs(name=f"{ci.name}@path", cell=ci.cell, positions=ci.positions, ecut=ci.ecut, grid=ci.grid,
                      spheres=spheres, kpoints=kfr, kweights=kw, bk=bk, v_eff_r=ci.v_eff_r, p=p,
                      nbands=ci.nbands, meta=dict(ci.meta))


def make_cell(name: str, seed: int = 0) -> CellInputs:
    """Build one workload. ``seed`` only matters for seeded variants
    (displaced/strained cells, vacancy placement)."""
    spec = _SPEC["cells"][name]
    sp = _SPEC["species"]["Si"]
    rng = np.random.default_rng(seed) if ("strain" in spec or "vacancies" in spec) else None
    cell, pos = _structure(spec, rng if "strain" in spec else None)
    ecut = float(spec["ecut_ry"]) * RY_EV
    grid = build_fft_grid(cell, ecut, shape_override=spec["fft"])
    kfr, kw = _kpoints(spec["kpoints"])
    spheres = [build_gsphere(grid, ecut, k) for k in kfr]
    bk = build_batched(spheres, _projector_tables(spheres, pos, grid.volume))
    extra = []
    meta = {}
    if "vacancies" in spec:
        sites = rng.choice(len(pos), size=int(spec["vacancies"]), replace=False)
        for site in sites:
            h = rng.uniform(*spec["vacancy_height"])
            w = rng.uniform(*spec["vacancy_width"])
            extra.append((h, w, pos[site]))
        meta["vacancy_sites"] = [int(s) for s in sites]
    v = local_potential(grid, pos, float(sp["A"]), float(sp["sigma"]), extra)
    p = projectors_b(bk, pos)
    return CellInputs(name=name, cell=cell, positions=pos, ecut=ecut, grid=grid, spheres=spheres,
                      kpoints=kfr, kweights=kw, bk=bk, v_eff_r=torch.from_numpy(v), p=p,
                      nbands=int(spec["nbands"]), meta=meta)
