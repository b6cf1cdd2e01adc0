"""Parity of the device Davidson with the reference's float64 ``davidson_batched``.

Golden eigenvalues come from the reference itself at tol 1e-10 eV on the same
seeded cells (``tests/golden/make_golden.py``). The bar of the band solve is
eigenvalues within 1e-8 Ha = 2.72e-7 eV of the reference and band energy
within 1e-6 Ha/cell = 2.72e-5 eV; the float64 path is held to 1e-9 eV here.
"""

import numpy as np
import pytest
import torch

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu

HA = 27.211386245988
EIG_TOL_HA = 1e-8 * HA          # 2.72e-7 eV
BAND_E_TOL = 1e-6 * HA          # per cell


def _cell_ham(name, seed=0):
    from gradwave_b200.cells import make_cell
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    ci = make_cell(name, seed=seed)
    dev = torch.device("cuda", 0)
    bk = ci.bk.to(dev)
    return ci, bk, BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)


def _band_energy(eig, w, nocc):
    return float(2.0 * np.sum(np.asarray(w)[:, None] * np.asarray(eig)[:, :nocc]))


def test_synthetic_operator_generic_apply(cuda_device):
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("synthetic")
    h = torch.from_numpy(g["h"]).to(cuda_device)

    def apply(c):
        return torch.einsum("kij,kbj->kbi", h.to(c.dtype), c)

    x0 = torch.from_numpy(g["x0"]).to(cuda_device)
    t = torch.from_numpy(g["t"]).to(cuda_device)
    mask = torch.ones(t.shape, dtype=torch.bool, device=cuda_device)
    res = davidson_batched(apply, x0, t, mask, tol=1e-9, max_iter=100)
    assert float(res.residual_norms.max()) < 1e-9
    assert np.abs(res.eigenvalues.cpu().numpy() - g["exact"]).max() < 1e-9
    assert np.abs(res.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < 1e-10


def test_si2_fp64_matches_reference(cuda_device):
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("si2_fcc")
    ci, bk, h = _cell_ham("si2_fcc")
    res = davidson_batched(h.apply, ci.identity_start().to(cuda_device), bk.t, bk.mask, tol=1e-10,
                           max_iter=200)
    eig = res.eigenvalues.cpu().numpy()
    assert float(res.residual_norms.max()) < 1e-10
    assert np.abs(eig - g["eigenvalues"]).max() < 1e-9
    # at tol 1e-10 eV (~2e-13 of |H|) the last rounds run at float64 round-off,
    # so the round count moves with last-bit differences; it must stay close
    assert res.n_iter <= int(1.3 * int(g["n_iter"])) + 3


def test_si8_fp64_matches_reference_and_certified(cuda_device):
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("si8_cubic")
    ci, bk, h = _cell_ham("si8_cubic")
    res = davidson_batched(h.apply, ci.identity_start().to(cuda_device), bk.t, bk.mask, tol=1e-10,
                           max_iter=200)
    eig = res.eigenvalues.cpu().numpy()
    assert np.abs(eig - g["eigenvalues"]).max() < 1e-9
    nocc = ci.nocc()
    assert abs(_band_energy(eig, ci.kweights, nocc) - _band_energy(g["eigenvalues"], ci.kweights, nocc)) \
        < 1e-3 * BAND_E_TOL
    # returned residual norms equal an independent float64 recompute; rows orthonormal
    x = res.eigenvectors
    hx = h.apply(x)
    rn = torch.linalg.vector_norm(hx - res.eigenvalues[..., None] * x, dim=-1)
    assert float((rn - res.residual_norms).abs().max()) < 1e-11
    gram = torch.einsum("kag,kbg->kab", x.conj(), x)
    eye = torch.eye(ci.nbands, dtype=torch.complex128, device=cuda_device)
    assert float((gram - eye).abs().max()) < 1e-10
    # padded slots stay zero
    assert float(x[~bk.mask[:, None, :].expand_as(x)].abs().max()) == 0.0


def test_si8_fp32_expansion_within_bar(cuda_device):
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("si8_cubic")
    ci, bk, h = _cell_ham("si8_cubic")
    res = davidson_batched(h.apply, ci.identity_start().to(cuda_device), bk.t, bk.mask, tol=1e-10,
                           max_iter=200, mode="fp32exp")
    eig = res.eigenvalues.cpu().numpy()
    assert float(res.residual_norms.max()) < 1e-10
    assert np.abs(eig - g["eigenvalues"]).max() < EIG_TOL_HA
    assert res.n_apply_low > 0 and res.n_apply_full > 0


def test_native_and_host_driver_agree(cuda_device, monkeypatch):
    """The native driver (one libgwb.so call) and the host driver (kernel by
    kernel from Python) run the same algorithm: same eigenpairs."""
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("si8_cubic")
    ci, bk, h = _cell_ham("si8_cubic")
    x0 = ci.identity_start().to(cuda_device)
    monkeypatch.setenv("GWB_KGROUPS", "1")  # one group on both drivers: the same algorithm step for step
    for mode in ("fp64", "fp32exp"):
        native = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=200, mode=mode)
        assert native.info.get("native")
        monkeypatch.setenv("GWB_NATIVE", "0")
        monkeypatch.setenv("GWB_TC_PROJECT", "0")  # both passes in float64, as the native driver
        host = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=200, mode=mode)
        monkeypatch.delenv("GWB_NATIVE")
        monkeypatch.delenv("GWB_TC_PROJECT")
        assert not host.info.get("native")
        for res in (native, host):
            assert float(res.residual_norms.max()) < 1e-10
            assert np.abs(res.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < 1e-9
        assert abs(native.n_iter - host.n_iter) <= 3


@pytest.mark.parametrize("mode,steps", [("fp32exp", None), ("mixed", None), ("mixed", "nh,nn,chol")])
def test_tensor_core_projection_pass_keeps_parity(cuda_device, monkeypatch, mode, steps):
    """The float32-expansion modes of the host driver run the first projection
    pass (and, when selected, a first Cholesky-QR round) as split-BF16
    tensor-core products; the float64 steps after them remove their error:
    same eigenvalues as the reference, an orthonormal block, and about the
    same number of rounds as with every step in float64."""
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("si8_cubic")
    ci, bk, h = _cell_ham("si8_cubic")
    x0 = ci.identity_start().to(cuda_device)
    monkeypatch.setenv("GWB_NATIVE", "0")
    if steps is not None:
        monkeypatch.setenv("GWB_TC_STEPS", steps)
    runs = {}
    for tc in ("1", "0"):
        monkeypatch.setenv("GWB_TC_PROJECT", tc)
        runs[tc] = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=200, mode=mode)
    res = runs["1"]
    assert res.info["tc_projection"] and not runs["0"].info["tc_projection"]
    assert set(res.info["tc_steps"]) == ({"nh", "nn", "chol"} if steps else {"nh", "nn"})
    assert float(res.residual_norms.max()) < 1e-10
    assert np.abs(res.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < EIG_TOL_HA
    x = res.eigenvectors
    gram = x @ x.conj().transpose(-1, -2)
    eye = torch.eye(gram.shape[-1], dtype=gram.dtype, device=gram.device)
    assert float((gram - eye).abs().max()) < 1e-12
    assert res.n_iter <= runs["0"].n_iter + 5


def test_registry_adapters_and_two_stage(cuda_device):
    """Registry contract (reference solvers/registry.py) and the complex64
    draft -> complex128 polish schedule (reference davidson_batched_ms)."""
    from gradwave_b200 import registry
    from gradwave_b200.davidson import davidson_batched_ms
    g = load_golden("si8_cubic")
    ci, bk, h = _cell_ham("si8_cubic")
    x0 = ci.identity_start().to(cuda_device)
    with pytest.raises(ValueError):
        registry.register("davidson", registry.davidson_adapter)
    with pytest.raises(ValueError, match="registered"):
        registry.get("nope")
    for name in ("davidson", "davidson_fp32exp", "davidson_mixed"):
        r = registry.get(name)(h.apply, x0, bk.t, bk.mask, tol=1e-10, nbands=ci.nbands, max_iter=200)
        assert isinstance(r, registry.EigResult)
        assert np.abs(r.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < EIG_TOL_HA
        assert r.diagnostics["hit_max_iter"] is False
    r = registry.get("davidson")(h.apply, x0, bk.t, bk.mask, tol=1e-10, nbands=ci.nbands, max_iter=3)
    assert r.diagnostics["hit_max_iter"] is True and r.n_iter == 3
    ms = davidson_batched_ms(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=200, crossover=1e-4)
    assert float(ms.residual_norms.max()) < 1e-10
    assert np.abs(ms.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < 1e-9


@pytest.mark.parametrize("groups", [2, 3, 5])
def test_k_group_solves_match_reference(cuda_device, monkeypatch, groups):
    """The k-points split into groups solved concurrently on separate streams
    (GWB_KGROUPS) give the reference's eigenvalues, certified residuals and
    orthonormal rows, for float64, the float32-expansion mode and the learned
    mixed mode (groups of different subspace sizes run at the same time)."""
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("si8_cubic")
    ci, bk, h = _cell_ham("si8_cubic")
    x0 = ci.identity_start().to(cuda_device)
    from gradwave_b200 import learned
    monkeypatch.setenv("GWB_KGROUPS", str(groups))
    cases = [("fp64", "teter", 1e-9), ("fp32exp", "teter", EIG_TOL_HA)]
    if learned.available():
        cases.append(("mixed", learned.LearnedPreconditioner.load(device=cuda_device), EIG_TOL_HA))
    for mode, pc, tol_eig in cases:
        res = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=200, mode=mode, precond=pc)
        assert res.info.get("k_groups") == groups
        assert float(res.residual_norms.max()) < 1e-10
        assert np.abs(res.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < tol_eig
        x = res.eigenvectors
        gram = torch.einsum("kag,kbg->kab", x.conj(), x)
        eye = torch.eye(ci.nbands, dtype=torch.complex128, device=cuda_device)
        assert float((gram - eye).abs().max()) < 1e-10


@pytest.mark.parametrize("name,mode", [("si64_cubic", "mixed"), ("si64_cubic", "fp64"), ("si216_vacancy", "mixed")])
def test_large_cells_match_reference(cuda_device, name, mode):
    """The 64-atom (4 k, 160 bands, basis up to 640) and 216-atom (Gamma, 480
    bands, basis up to 1920) cells: host driver with cuSOLVER subspace
    eigensolves, k-groups on their own streams, the tensor-core projection and
    Cholesky-QR rounds in the mixed mode. Eigenvalues within 1e-8 Ha of the
    reference's own float64 Davidson, band energy within 1e-6 Ha/cell."""
    from gradwave_b200.davidson import davidson_batched
    g = load_golden(name)
    ci, bk, h = _cell_ham(name)
    res = davidson_batched(h.apply, ci.identity_start().to(cuda_device), bk.t, bk.mask, tol=1e-10, max_iter=300,
                           mode=mode)
    eig = res.eigenvalues.cpu().numpy()
    assert float(res.residual_norms.max()) < 1e-10
    assert np.abs(eig - g["eigenvalues"]).max() < EIG_TOL_HA
    nocc = ci.nocc()
    assert abs(_band_energy(eig, ci.kweights, nocc) - _band_energy(g["eigenvalues"], ci.kweights, nocc)) < BAND_E_TOL
    if mode == "mixed":
        assert res.info.get("tc_projection")
