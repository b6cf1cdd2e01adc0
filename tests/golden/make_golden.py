"""Generate the golden fixtures of the band-solve path from the reference itself.

Runs the reference (gradwave, pure Python + torch, float64) on the seeded cells
of ``gradwave_b200/data/cells.json`` and writes small ``.npz`` fixtures next to
this script. The reference cannot travel to the GPU machine, so its outputs do.

The reference's package ``__init__`` pulls in ``ase`` (absent here); the hot-path
modules are imported through a namespace shim that bypasses it.

What is recorded, per case:
  * set-up: npw per k and the box index of every sphere point, kinetic and
    projector fingerprints, all from the reference's own builders
    (``grids.py:68-184``, ``core/hamiltonian.py:46-105``, ``core/batch.py:174-235``);
  * apply: ``BatchedHamiltonian.apply`` (``core/batch.py:480-505``) on a seeded
    random block - in full for small cases, else as projections on seeded
    random vectors (size-independent checksums);
  * solve: ``davidson_batched`` (``solvers/davidson.py:528-774``) from the
    identity start at tol 1e-10 eV: eigenvalues, residual norms, rounds, applies;
  * density: ``density_b`` (``core/batch.py:562-587``) on a seeded block;
  * Gamma path: the half-sphere layout, ``GammaHamiltonian.apply`` and
    ``davidson_gamma`` (``core/gamma.py``);
  * generalized USPP/PAW solve: ``BatchedHS.s`` and ``davidson_gen_batched``
    (``scf/uspp_batch.py``) with a synthetic augmentation matrix q.

Usage: python tests/golden/make_golden.py [small|big|all|density|gamma|uspp] --ref <gradwave>/src
       (or set GWB_REFERENCE_SRC instead of --ref)
"""

from __future__ import annotations

import argparse
import os
import sys
import time
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from gradwave_b200.cells import make_cell  # noqa: E402

TOL = 1e-10
GAMMA_TOL = 1e-6


def shim(ref_src: str):
    mod = types.ModuleType("gradwave")
    mod.__path__ = [os.path.join(ref_src, "gradwave")]
    sys.modules["gradwave"] = mod


def random_block(seed: int, nk: int, nb: int, npw: int) -> np.ndarray:
    """The seeded test block (every slot random, padding included)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))


def checksums(out: np.ndarray, seed: int, nvec: int = 4) -> np.ndarray:
    """Projections of ``out`` on seeded random vectors, then |out|^2."""
    rng = np.random.default_rng(seed + 1000)
    vals = []
    for _ in range(nvec):
        w = rng.standard_normal(out.shape) + 1j * rng.standard_normal(out.shape)
        vals.append(np.vdot(w, out))
    vals.append(np.vdot(out, out))
    return np.array(vals)


def reference_setup(ci):
    """Rebuild the cell's set-up with the reference's own builders."""
    from gradwave.core.batch import build_batched, projectors_b
    from gradwave.core.hamiltonian import build_projector_data
    from gradwave.grids import build_fft_grid, build_gsphere

    grid = build_fft_grid(ci.cell, ci.ecut, shape_override=ci.shape)
    sph = [build_gsphere(grid, ci.ecut, k) for k in ci.kpoints]
    from gradwave_b200.cells import _SPEC
    sp = _SPEC["species"]["Si"]
    rc = float(sp["rc"])
    pds = []
    for s in sph:
        q = torch.sqrt(s.kpg2)
        tab = torch.stack([torch.exp(-0.5 * (q * rc) ** 2), q * rc * torch.exp(-0.5 * (q * rc) ** 2)])
        pds.append(build_projector_data(s, [0] * len(ci.positions), [tab], [[0, 1]],
                                        [torch.diag(torch.tensor(sp["D"], dtype=torch.float64))],
                                        grid.volume))
    bk = build_batched(sph, pds)
    p = projectors_b(bk, torch.as_tensor(ci.positions))
    return grid, bk, p


def run_case(name: str, seed_cell: int, apply_nb: int, full_apply: bool, solve: bool,
             fp32_expansion: bool = False) -> dict:
    from gradwave.core.batch import BatchedHamiltonian
    from gradwave.solvers.davidson import davidson_batched

    ci = make_cell(name, seed=seed_cell)
    grid, bk, p = reference_setup(ci)
    assert grid.shape == ci.shape
    rec: dict = {"npw": bk.npw.numpy()}
    # set-up parity: exact integer tables, float fingerprints
    assert torch.equal(bk.flat_idx, ci.bk.flat_idx), f"{name}: flat_idx differs"
    assert torch.equal(bk.mask, ci.bk.mask)
    rec["flat_idx"] = bk.flat_idx.numpy().astype(np.int32)
    rec["t_sum"] = np.array([float(bk.t.sum()), float((bk.t ** 2).sum())])
    rec["p_chk"] = checksums(p.numpy(), 7)
    rec["dij"] = bk.dij_full.numpy()
    v = ci.v_eff_r
    h = BatchedHamiltonian(bk, grid.shape, v, p)
    nk, npw = bk.mask.shape
    c = torch.from_numpy(random_block(11, nk, apply_nb, npw))
    t0 = time.perf_counter()
    out = h.apply(c).numpy()
    rec["apply_seconds"] = np.array(time.perf_counter() - t0)
    rec["apply_chk"] = checksums(out, 11)
    if full_apply:
        rec["apply_out"] = out
    if solve:
        if fp32_expansion:
            os.environ["GRADWAVE_FP32_EXPANSION"] = "on"
        try:
            x0 = ci.identity_start()
            t0 = time.perf_counter()
            res = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=TOL, max_iter=200)
            rec["solve_seconds"] = np.array(time.perf_counter() - t0)
        finally:
            os.environ.pop("GRADWAVE_FP32_EXPANSION", None)
        rec["eigenvalues"] = res.eigenvalues.numpy()
        rec["residual_norms"] = res.residual_norms.numpy()
        rec["n_iter"] = np.array(res.n_iter)
        rec["n_apply"] = np.array([res.n_apply_low, res.n_apply_full])
        rec["kweights"] = ci.kweights
    return rec


def density_case(name: str, nb: int, seed: int, full: bool) -> dict:
    """``density_b`` (``core/batch.py:562-587``) on a seeded block with zero
    padding and seeded occupations in [0, 2]; the full rho for small boxes,
    else checksums (sum, sum of squares, projections on seeded vectors)."""
    from gradwave.core.batch import density_b

    ci = make_cell(name)
    grid, bk, _ = reference_setup(ci)
    nk, npw = bk.mask.shape
    c = random_block(seed, nk, nb, npw) * bk.mask.numpy()[:, None, :]
    occ = np.random.default_rng(seed + 1).uniform(0.0, 2.0, (nk, nb))
    kw = np.asarray(ci.kweights, dtype=np.float64)
    rho = density_b(torch.from_numpy(c), torch.from_numpy(occ), torch.from_numpy(kw), bk, grid.shape,
                    grid.volume).numpy()
    rec = {"nb": np.array(nb), "seed": np.array(seed), "occ": occ, "kweights": kw, "volume": np.array(grid.volume),
           "rho_chk": density_checksums(rho, seed)}
    if full:
        rec["rho"] = rho
    return rec


def gamma_case(name: str, nb_apply: int, seed: int, solve: bool) -> dict:
    """The Gamma real path (``core/gamma.py``): the half-sphere layout,
    ``GammaHamiltonian.apply`` on a seeded half block (G = 0 real), and
    ``davidson_gamma`` from the identity start on the lowest half-sphere
    slots at tol 1e-6 eV. (The reference's real-embedding Davidson has a
    residual floor near 1e-9 eV on si2: at tol 1e-8 its QR rank reveal empties
    the expansion block with residuals near 3e-6, at 1e-10 it stalls for 200
    rounds; its eigenvalues stay within 2e-8 eV of the complex solve.)"""
    from gradwave.core.gamma import GammaHamiltonian, build_gamma_basis, davidson_gamma
    from gradwave.grids import build_gsphere

    ci = make_cell(name)
    grid, bk, p = reference_setup(ci)
    assert bk.mask.shape[0] == 1
    gb = build_gamma_basis(build_gsphere(grid, ci.ecut, [0.0, 0.0, 0.0]), grid.shape)
    gh = GammaHamiltonian(gb, ci.v_eff_r, p[0], bk.dij_full)
    rng = np.random.default_rng(seed)
    ch = rng.standard_normal((nb_apply, gb.nhalf)) + 1j * rng.standard_normal((nb_apply, gb.nhalf))
    ch[:, 0] = ch[:, 0].real
    out = gh.apply(torch.from_numpy(ch)).numpy()
    rec = {"rep_full_idx": gb.rep_full_idx.numpy().astype(np.int32), "seed": np.array(seed),
           "nb_apply": np.array(nb_apply), "apply_chk": checksums(out, seed)}
    if gb.nhalf <= 2000:
        rec["apply_out"] = out
    if solve:
        nb = ci.nbands
        x0 = torch.zeros(nb, gb.nhalf, dtype=torch.complex128)
        x0[torch.arange(nb), torch.arange(nb)] = 1.0
        t0 = time.perf_counter()
        res = davidson_gamma(gh, x0, tol=GAMMA_TOL, max_iter=200)
        rec["solve_seconds"] = np.array(time.perf_counter() - t0)
        rec["eigenvalues"] = res.eigenvalues.numpy()
        rec["residual_norms"] = res.residual_norms.numpy()
        rec["n_iter"] = np.array(res.n_iter)
    return rec


def uspp_q(natoms: int, seed: int) -> np.ndarray:
    """Synthetic augmentation matrix for the generalized problem: per atom a
    seeded symmetric positive 4 x 4 block on its (s, p_y, p_z, p_x) projector
    columns, scaled to norm 0.3, so that S = 1 + sum q |beta><beta| is
    positive definite."""
    rng = np.random.default_rng(seed)
    q = np.zeros((4 * natoms, 4 * natoms))
    for a in range(natoms):
        m = rng.standard_normal((4, 4))
        blk = m @ m.T
        q[4 * a:4 * a + 4, 4 * a:4 * a + 4] = 0.3 * blk / np.linalg.norm(blk, 2)
    return q


def uspp_case(name: str, seed: int) -> dict:
    """The generalized USPP/PAW band solve (``scf/uspp_batch.py``):
    ``BatchedHS`` with the cell's D as the screened D and a synthetic q, its S
    apply on a seeded block, and ``davidson_gen_batched`` from the identity
    start at tol 1e-10 eV."""
    from gradwave.scf.uspp_batch import BatchedHS, davidson_gen_batched

    ci = make_cell(name)
    grid, bk, p = reference_setup(ci)
    q = uspp_q(len(ci.positions), seed)
    assert q.shape[0] == p.shape[1]
    hs = BatchedHS(bk, grid.shape, ci.v_eff_r, p, bk.dij_full, torch.from_numpy(q))
    nk, npw = bk.mask.shape
    c = torch.from_numpy(random_block(seed, nk, 2, npw))
    rec = {"q": q, "seed": np.array(seed), "s_chk": checksums(hs.s(c).numpy(), seed)}
    x0 = ci.identity_start()
    t0 = time.perf_counter()
    eig, x = davidson_gen_batched(hs, x0, ci.nbands, tol=TOL, max_iter=200)
    rec["solve_seconds"] = np.array(time.perf_counter() - t0)
    rec["eigenvalues"] = eig.numpy()
    return rec


def density_checksums(rho: np.ndarray, seed: int, nvec: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed + 2000)
    vals = [rho.sum(), (rho * rho).sum()]
    for _ in range(nvec):
        vals.append(float((rng.standard_normal(rho.shape) * rho).sum()))
    return np.array(vals)


def synthetic_case(seed: int = 2, nk: int = 4, npw: int = 80, nb: int = 8) -> dict:
    """Dense random Hermitian operator with a kinetic-like diagonal; isolates
    the eigensolver from the FFT."""
    from gradwave.solvers.davidson import davidson_batched

    rng = np.random.default_rng(seed)
    diag = np.linspace(1.0, 100.0, npw)
    h = np.zeros((nk, npw, npw), dtype=np.complex128)
    for k in range(nk):
        a = rng.standard_normal((npw, npw)) + 1j * rng.standard_normal((npw, npw))
        h[k] = 0.5 * (a + a.conj().T) + np.diag(diag)
    ht = torch.from_numpy(h)
    x0 = torch.from_numpy(rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw)))
    mask = torch.ones(nk, npw, dtype=torch.bool)
    t = torch.from_numpy(np.broadcast_to(diag, (nk, npw)).copy())
    res = davidson_batched(lambda c: torch.einsum("kij,kbj->kbi", ht.to(c.dtype), c),
                           x0, t, mask, tol=1e-9, max_iter=100)
    return {"h": h, "x0": x0.numpy(), "t": t.numpy(), "eigenvalues": res.eigenvalues.numpy(),
            "residual_norms": res.residual_norms.numpy(), "n_iter": np.array(res.n_iter),
            "exact": np.linalg.eigvalsh(h)[:, :nb]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("which", nargs="?", default="small",
                    choices=["small", "big", "all", "density", "gamma", "uspp"])
    ap.add_argument("--ref", default=os.environ.get("GWB_REFERENCE_SRC"),
                    help="the reference's source directory (the one holding the gradwave package); "
                         "or set GWB_REFERENCE_SRC")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set GWB_REFERENCE_SRC")
    shim(args.ref)
    torch.set_num_threads(os.cpu_count() or 1)
    jobs = []
    if args.which in ("small", "all"):
        jobs += [
            ("si2_fcc", lambda: run_case("si2_fcc", 0, 8, True, True)),
            ("si8_cubic", lambda: run_case("si8_cubic", 0, 2, False, True)),
            ("si8_cubic_fp32exp", lambda: run_case("si8_cubic", 0, 1, False, True, fp32_expansion=True)),
            ("si8_perturbed", lambda: run_case("si8_perturbed", 1, 2, False, False)),
            ("synthetic", synthetic_case),
        ]
    if args.which in ("density", "all"):
        jobs += [
            ("density_si2_fcc", lambda: density_case("si2_fcc", 6, 21, True)),
            ("density_si8_cubic", lambda: density_case("si8_cubic", 5, 22, False)),
            ("density_si64_cubic", lambda: density_case("si64_cubic", 3, 23, False)),
        ]
    if args.which in ("uspp", "all"):
        jobs += [
            ("uspp_si2_fcc", lambda: uspp_case("si2_fcc", 41)),
            ("uspp_si8_cubic", lambda: uspp_case("si8_cubic", 42)),
        ]
    if args.which in ("gamma", "all"):
        jobs += [
            ("gamma_si2_fcc", lambda: gamma_case("si2_fcc", 5, 31, True)),
            ("gamma_si216_vacancy", lambda: gamma_case("si216_vacancy", 2, 32, False)),
        ]
    if args.which in ("big", "all"):
        jobs += [
            ("si64_cubic", lambda: run_case("si64_cubic", 0, 2, False, True)),
            ("si216_vacancy", lambda: run_case("si216_vacancy", 0, 1, False, True)),
        ]
    for tag, fn in jobs:
        t0 = time.perf_counter()
        rec = fn()
        np.savez_compressed(HERE / f"{tag}.npz", **rec)
        extra = ""
        if "n_iter" in rec:
            extra = f" n_iter={int(rec['n_iter'])} max_res={float(np.max(rec['residual_norms'])):.2e}"
        print(f"{tag}: {time.perf_counter() - t0:.1f}s{extra}", flush=True)


if __name__ == "__main__":
    main()
