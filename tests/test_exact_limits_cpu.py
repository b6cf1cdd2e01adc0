"""Exactly solvable limits, on the CPU: the host-side basis builders
(``gradwave_b200.basis``: FFT box, G-sphere, batched tables) and the oracle
apply + Davidson (``oracle/ham.py``, ``oracle/davidson.py``) against analytic
spectra, with no pseudopotential and no reference code. The cases are those
of gradwave ``tests/unit/test_exact_limits.py:51-100``:

* empty lattice: with V = 0 the spectrum at any k is hbar^2 |k+G|^2 / 2m, on a
  triclinic cell at a generic k so that no symmetry hides an index or
  convention error (1e-9 eV);
* cosine potential V(x) = 2 q u cos(2 pi x / a), u = hbar^2/2m (pi/a)^2: the
  band edges at Gamma and X are Mathieu characteristic values (scipy
  ``mathieu_a/b``): Gamma carries a_0, b_2, a_2, ..., X carries b_1, a_1, b_3,
  ... (1e-7 eV). The transverse lengths are 1.2 A so that transverse
  excitations sit ~100 eV up.
"""

import numpy as np
import pytest

from gradwave_b200.basis import ProjectorData, build_batched, build_fft_grid, build_gsphere
from gradwave_b200.constants import HBAR2_2M, RY_EV as RY
from oracle.davidson import davidson_batched
from oracle.ham import OracleHamiltonian


def _operator(cell, ecut, k_frac, v_of_shape):
    """Sphere, batched tables and oracle operator T + V at one k (no projectors)."""
    grid = build_fft_grid(np.asarray(cell, dtype=np.float64), ecut)
    sph = build_gsphere(grid, ecut, k_frac)
    pd = ProjectorData(atom_index=np.zeros(0, dtype=np.int64),
                       f_ylm_phase_free=np.zeros((0, sph.npw), dtype=np.complex128),
                       kpg=sph.kpg, dij_full=np.zeros((0, 0)))
    bk = build_batched([sph], [pd])
    h = OracleHamiltonian(bk.mask.numpy(), bk.flat_idx.numpy(), bk.t.numpy(), grid.shape,
                          v_of_shape(grid.shape), np.zeros((1, 0, sph.npw), dtype=np.complex128),
                          np.zeros((0, 0)))
    return grid, sph, bk, h


def _solve(cell, ecut, k_frac, v_of_shape, nb, seed=0, tol=1e-11):
    """Lowest nb eigenvalues of T + V at one k, seeded random start scaled by
    1/(1 + T) as in the reference's test."""
    grid, sph, bk, h = _operator(cell, ecut, k_frac, v_of_shape)
    rng = np.random.default_rng(seed)
    x0 = rng.standard_normal((1, nb, sph.npw)) + 1j * rng.standard_normal((1, nb, sph.npw))
    x0 = x0 / (1.0 + HBAR2_2M * sph.kpg2)
    x0 /= np.linalg.norm(x0, axis=-1, keepdims=True)
    res = davidson_batched(h.apply, x0, bk.t.numpy(), bk.mask.numpy(), tol=tol, max_iter=200)
    assert float(res.residual_norms.max()) < tol
    return res.eigenvalues[0], sph


def test_empty_lattice_free_electron_bands():
    cell = [[3.1, 0.0, 0.0], [0.4, 2.7, 0.0], [0.2, -0.3, 3.3]]  # triclinic
    k = (0.31, 0.17, -0.23)                                      # generic k
    nb = 12
    eigs, sph = _solve(cell, 30 * RY, k, lambda shape: np.zeros(shape), nb)
    exact = np.sort(HBAR2_2M * sph.kpg2)[:nb]
    assert np.abs(eigs - exact).max() < 1e-9
    # the sphere order is |k+G|^2 ascending (the reference's lexsort), so the
    # exact spectrum is also the sphere's first nb kinetic energies
    assert np.array_equal(np.sort(sph.kpg2)[:nb], sph.kpg2[:nb])


A_X, L_T, Q = 3.0, 1.2, 1.5
UNIT = HBAR2_2M * (np.pi / A_X) ** 2     # Mathieu energy scale [eV]
E_CAP = 80.0                             # below the first transverse excitation (~104 eV)


def _v_cos(shape):
    x = np.arange(shape[0]) / shape[0]
    return np.broadcast_to((2.0 * Q * UNIT * np.cos(2.0 * np.pi * x))[:, None, None], shape).copy()


def test_cosine_potential_mathieu_bands():
    special = pytest.importorskip("scipy.special")
    a, L, q, unit, e_cap, v_cos = A_X, L_T, Q, UNIT, E_CAP, _v_cos
    cases = {
        (0.0, 0.0, 0.0): [special.mathieu_a(0, q), special.mathieu_b(2, q), special.mathieu_a(2, q),
                          special.mathieu_b(4, q), special.mathieu_a(4, q)],
        (0.5, 0.0, 0.0): [special.mathieu_b(1, q), special.mathieu_a(1, q), special.mathieu_b(3, q),
                          special.mathieu_a(3, q)],
    }
    cell = np.diag([a, L, L])
    for k, chars in cases.items():
        exact = np.array([unit * c for c in chars])
        exact = exact[exact < e_cap]
        assert len(exact) >= 4
        eigs, _ = _solve(cell, 60 * RY, k, v_cos, len(exact) + 2)
        err = np.abs(eigs[:len(exact)] - exact).max()
        assert err < 1e-7, f"k={k}: max |E - Mathieu| = {err:.2e} eV"


def test_gamma_path_mathieu_band_edges():
    """The Gamma real path (``gradwave_b200.gamma``: half-sphere maps, the
    real embedding, ``davidson_gamma`` in float64 and with locking and
    buffer bands) driven by the oracle Gamma apply on the cosine-potential
    cell: the Gamma band edges a_0, b_2, a_2, b_4, a_4 to 1e-7 eV."""
    special = pytest.importorskip("scipy.special")
    import torch
    from gradwave_b200 import gamma as G
    from oracle.gamma import gamma_apply
    grid, sph, bk, h = _operator(np.diag([A_X, L_T, L_T]), 60 * RY, (0.0, 0.0, 0.0), _v_cos)
    gb = G.build_gamma_basis(sph, grid.shape)

    class _Ham:
        device = torch.device("cpu")

        def apply_phi(self, phi, prec=None):
            nphi = 2 * gb.nhalf - 1
            ch = G.unembed_real(gb, phi[:, :nphi].contiguous()).numpy()
            out = gamma_apply(h, gb.src_half.numpy(), gb.conj_full.numpy(), gb.rep_full_idx.numpy(), ch)
            return torch.nn.functional.pad(G.embed_real(gb, torch.from_numpy(out)), (0, phi.shape[1] - nphi))

    ham = _Ham()
    ham.gb, ham.t_phi = gb, G.kinetic_phi(gb)
    exact = np.array([UNIT * c for c in (special.mathieu_a(0, Q), special.mathieu_b(2, Q),
                                         special.mathieu_a(2, Q), special.mathieu_b(4, Q),
                                         special.mathieu_a(4, Q))])
    exact = exact[exact < E_CAP]
    nb = len(exact) + 2
    for kw in ({}, {"lock": True, "n_buffer": 2}):
        res = G.davidson_gamma(ham, G.gamma_start(gb, nb), tol=1e-10, max_iter=200, **kw)
        assert float(res.residual_norms.max()) < 1e-10
        err = np.abs(res.eigenvalues.numpy()[:len(exact)] - exact).max()
        assert err < 1e-7, f"{kw}: max |E - Mathieu| = {err:.2e} eV"
