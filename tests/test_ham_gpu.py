"""Parity of the CUDA Hamiltonian apply (through the C ABI) with the reference.

Golden values come from the reference's own ``BatchedHamiltonian.apply``
(gradwave ``core/batch.py:480-505``) run on the same seeded inputs
(``tests/golden/make_golden.py``); the float64 oracle is checked alongside.

Tolerances: float64 arithmetic 1e-11 relative to the largest output element;
float32 arithmetic 3e-6 relative (fp32 FFT round-off grows like eps*log N).
"""

import numpy as np
import pytest
import torch

from tests.conftest import load_golden
from tests.golden.make_golden import checksums, random_block

pytestmark = pytest.mark.gpu

TOL64 = 1e-11
TOL32 = 3e-6


def _ham(name, seed=0):
    from gradwave_b200.cells import make_cell
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    ci = make_cell(name, seed=seed)
    dev = torch.device("cuda", 0)
    return ci, BatchedHamiltonian(ci.bk.to(dev), ci.shape, ci.v_eff_r, ci.p)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_apply_si2_full_vs_reference(cuda_device):
    g = load_golden("si2_fcc")
    ci, h = _ham("si2_fcc")
    c = random_block(11, ci.bk.nk, 8, ci.bk.npw_max)
    out = h.apply(torch.from_numpy(c).to(cuda_device)).cpu().numpy()
    assert _rel(out, g["apply_out"]) < TOL64
    out32 = h.apply(torch.from_numpy(c).to(cuda_device, torch.complex64)).cpu().numpy()
    assert _rel(out32, g["apply_out"]) < TOL32
    out32b = h.apply_fp32(torch.from_numpy(c).to(cuda_device)).cpu().numpy()
    assert _rel(out32b, g["apply_out"]) < TOL32


@pytest.mark.parametrize("name,seed", [("si8_cubic", 0), ("si8_perturbed", 1)])
def test_apply_checksums_vs_reference(cuda_device, name, seed):
    g = load_golden(name)
    ci, h = _ham(name, seed)
    assert np.array_equal(ci.bk.npw.numpy(), g["npw"])
    c = random_block(11, ci.bk.nk, 2, ci.bk.npw_max)   # random padding too
    out = h.apply(torch.from_numpy(c).to(cuda_device)).cpu().numpy()
    chk = checksums(out, 11)
    ref = g["apply_chk"]
    assert np.abs(chk - ref).max() / np.abs(ref).max() < TOL64
    # padded slots come out exactly zero
    assert np.all(out[~ci.bk.mask.numpy()[:, None, :].repeat(2, 1)] == 0)


def test_apply_vs_oracle_and_hermitian(cuda_device):
    from oracle.ham import from_cell
    ci, h = _ham("si8_cubic")
    orc = from_cell(ci)
    rng = np.random.default_rng(5)
    nb = 5
    c = (rng.standard_normal((ci.bk.nk, nb, ci.bk.npw_max))
         + 1j * rng.standard_normal((ci.bk.nk, nb, ci.bk.npw_max))) * ci.bk.mask.numpy()[:, None, :]
    ref = orc.apply(c)
    out = h.apply(torch.from_numpy(c).to(cuda_device)).cpu().numpy()
    assert _rel(out, ref) < TOL64
    # <a|H b> == conj(<b|H a>) per k
    a, b = c[:, :1], c[:, 1:2]
    ha = h.apply(torch.from_numpy(a.copy()).to(cuda_device)).cpu().numpy()
    hb = h.apply(torch.from_numpy(b.copy()).to(cuda_device)).cpu().numpy()
    lhs = np.einsum("kbg,kbg->k", a.conj(), hb)
    rhs = np.einsum("kbg,kbg->k", b.conj(), ha).conj()
    assert np.abs(lhs - rhs).max() / np.abs(lhs).max() < 1e-12


def test_apply_band_chunking_invariant(cuda_device, monkeypatch):
    """The L2-sized band chunking of the scratch must not change results."""
    ci, h = _ham("si8_cubic")
    rng = np.random.default_rng(9)
    c = torch.from_numpy(rng.standard_normal((ci.bk.nk, 7, ci.bk.npw_max))
                         + 1j * rng.standard_normal((ci.bk.nk, 7, ci.bk.npw_max))).to(cuda_device)
    full = h.apply(c)
    monkeypatch.setenv("GWB_W_BUDGET_MB", "1")
    ci2, h2 = _ham("si8_cubic")
    chunked = h2.apply(c)
    assert torch.equal(full, chunked)


def test_apply_si64_checksums_and_tensor_core_nonlocal(cuda_device):
    """The 64-atom cell (72^3 box, 256 projectors): float64 checksums against
    the reference, and the float32 apply, whose nonlocal term runs as
    split-BF16 tensor-core products from 128 projectors up, within the float32
    bar of the float64 result; no pipeline wait ran out."""
    import ctypes
    from gradwave_b200 import _lib
    g = load_golden("si64_cubic")
    ci, h = _ham("si64_cubic")
    assert np.array_equal(ci.bk.npw.numpy(), g["npw"])
    c = random_block(11, ci.bk.nk, 2, ci.bk.npw_max)
    out = h.apply(torch.from_numpy(c).to(cuda_device)).cpu().numpy()
    ref = g["apply_chk"]
    assert np.abs(checksums(out, 11) - ref).max() / np.abs(ref).max() < TOL64
    rng = np.random.default_rng(3)
    nb = 6
    cm = (rng.standard_normal((ci.bk.nk, nb, ci.bk.npw_max))
          + 1j * rng.standard_normal((ci.bk.nk, nb, ci.bk.npw_max))) * ci.bk.mask.numpy()[:, None, :]
    x = torch.from_numpy(cm).to(cuda_device)
    o64 = h.apply(x).cpu().numpy()
    o32 = h.apply_fp32(x).cpu().numpy()
    assert _rel(o32, o64) < TOL32
    assert np.all(o32[~ci.bk.mask.numpy()[:, None, :].repeat(nb, 1)] == 0)
    st = ctypes.c_int(-1)
    _lib.call("gwb_ham_tc_status", h._h, ctypes.byref(st))
    assert st.value == 0
