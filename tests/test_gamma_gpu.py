"""The Gamma-point real path on the GPU against the reference.

* The apply (two real bands per complex row of the apply kernels, unpacked by
  the G / -G symmetry) against the reference's own ``GammaHamiltonian.apply``
  on seeded half blocks: si2 in full (odd nb, so one row pairs with a zero
  partner), si216 by checksums; float64 1e-11 relative, float32 3e-6.
* ``davidson_gamma`` (real-symmetric Davidson in the embedding) against the
  complex float64 reference solves of the same Gamma-only cells: eigenvalues
  within 1e-8 Ha. The reference's own real-embedding solver has a residual
  floor near 1e-9 eV, so the solves here stop at 1e-6 eV (eigenvalue error
  ~ residual^2 / gap) and, for si2, the round count is compared with the
  reference's at the same tolerance.
"""

import numpy as np
import pytest
import torch

from tests.conftest import load_golden
from tests.golden.make_golden import checksums

pytestmark = pytest.mark.gpu

HA = 27.211386245988


def _gamma(name, dev):
    from gradwave_b200.cells import make_cell
    from gradwave_b200.gamma import GammaHamiltonian, build_gamma_basis
    ci = make_cell(name)
    gb = build_gamma_basis(ci.spheres[0], ci.shape)
    return ci, gb, GammaHamiltonian(gb, ci.v_eff_r, ci.p[0], ci.bk.dij_full, device=dev)


def _block(g, gb):
    rng = np.random.default_rng(int(g["seed"]))
    nb = int(g["nb_apply"])
    ch = rng.standard_normal((nb, gb.nhalf)) + 1j * rng.standard_normal((nb, gb.nhalf))
    ch[:, 0] = ch[:, 0].real
    return ch


@pytest.mark.parametrize("name", ["si2_fcc", "si216_vacancy"])
def test_gamma_apply_matches_reference(cuda_device, name):
    from gradwave_b200 import _lib
    from gradwave_b200.gamma import embed_real, unembed_real
    g = load_golden(f"gamma_{name}")
    ci, gb, gh = _gamma(name, cuda_device)
    ch = torch.from_numpy(_block(g, gb)).to(cuda_device)
    out = gh.apply(ch).cpu().numpy()
    if "apply_out" in g:
        assert np.abs(out - g["apply_out"]).max() / np.abs(g["apply_out"]).max() < 1e-11
    chk = checksums(out, int(g["seed"]))
    assert np.abs(chk - g["apply_chk"]).max() / np.abs(g["apply_chk"]).max() < 1e-11
    # G = 0 stays real; float32 arithmetic within the float32 bar
    assert float(out[:, 0].imag.__abs__().max()) == 0.0
    o32 = unembed_real(gb, gh.apply_phi(embed_real(gb, ch), prec=_lib.GWB_FP32)).cpu().numpy()
    assert np.abs(o32 - out).max() / np.abs(out).max() < 3e-6


def test_gamma_davidson_si2_matches_reference(cuda_device):
    from gradwave_b200.gamma import davidson_gamma, gamma_start, metric_inner
    gg = load_golden("gamma_si2_fcc")
    gc = load_golden("si2_fcc")
    ci, gb, gh = _gamma("si2_fcc", cuda_device)
    res = davidson_gamma(gh, gamma_start(gb, ci.nbands, cuda_device), tol=1e-6, max_iter=200)
    eig = res.eigenvalues.cpu().numpy()
    assert float(res.residual_norms.max()) < 1e-6
    assert np.abs(eig - gc["eigenvalues"][0]).max() < 1e-8 * HA
    assert np.abs(eig - gg["eigenvalues"]).max() < 1e-8 * HA
    assert res.n_iter <= int(gg["n_iter"]) + 3
    gram = metric_inner(gb, res.eigenvectors, res.eigenvectors)
    assert float((gram - torch.eye(ci.nbands, dtype=gram.dtype, device=gram.device)).abs().max()) < 1e-12


@pytest.mark.parametrize("mode,tol,nbuf", [("fp64", 1e-6, 0), ("fp64", 1e-10, 0), ("mixed", 1e-10, 0),
                                           ("mixed", 1e-10, 32)])
def test_gamma_davidson_si216_matches_complex_reference(cuda_device, mode, tol, nbuf):
    """si216 on the Gamma path, float64 and mixed (float32 expansion applies,
    its first rounds on split-BF16 tensor-core products, float64
    certification and hand-off, converged pairs locked), with and without
    buffer bands, to 1e-6 and 1e-10 eV."""
    from gradwave_b200.gamma import davidson_gamma, gamma_start
    gc = load_golden("si216_vacancy")
    ci, gb, gh = _gamma("si216_vacancy", cuda_device)
    res = davidson_gamma(gh, gamma_start(gb, ci.nbands, cuda_device), tol=tol, max_iter=200, mode=mode,
                         n_buffer=nbuf)
    eig = res.eigenvalues.cpu().numpy()
    assert float(res.residual_norms.max()) < tol
    assert np.abs(eig - gc["eigenvalues"][0]).max() < 1e-8 * HA
    if mode == "mixed":
        # the float32 phase ran its first rounds on the tensor-core products
        # and handed a float64-orthonormal block to the float64 phase
        assert res.info["rounds_tc"] > 0 and res.info["rounds_f64"] > 0


def test_gamma_apply_accepts_transposed_blocks(cuda_device):
    """Solver blocks can come out of a triangular solve with transposed
    strides; the apply reads and writes row-major whatever the input layout."""
    ci, gb, gh = _gamma("si2_fcc", cuda_device)
    g = torch.Generator(device="cpu").manual_seed(3)
    phi = torch.randn(2 * gb.nhalf - 1, 6, generator=g, dtype=torch.float64).to(cuda_device).T
    assert not phi.is_contiguous()
    assert torch.equal(gh.apply_phi(phi), gh.apply_phi(phi.contiguous()))
