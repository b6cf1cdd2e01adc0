"""The electron density on the GPU (``gwb_ham_density``) against the
reference's own ``density_b`` (gradwave ``core/batch.py:562-587``).

Golden values come from the reference on seeded blocks with zero padding and
seeded occupations (``tests/golden/make_golden.py density``): the full rho
for the 2-atom cell, checksums for the 8- and 64-atom cells (72^3 box, the
shared-memory pencil kernel). The arithmetic is float64, so the bar is
1e-11 relative. Size-independent checks: Parseval (sum_r rho * volume / N =
sum w f |c|^2), band-chunking invariance, complex64 storage.
"""

import numpy as np
import pytest
import torch

from tests.conftest import load_golden
from tests.golden.make_golden import density_checksums, random_block

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _inputs(name, dev):
    from gradwave_b200.cells import make_cell
    g = load_golden(f"density_{name}")
    ci = make_cell(name)
    nb, seed = int(g["nb"]), int(g["seed"])
    c = random_block(seed, ci.bk.nk, nb, ci.bk.npw_max) * ci.bk.mask.numpy()[:, None, :]
    return g, ci, torch.from_numpy(c).to(dev), torch.from_numpy(g["occ"]).to(dev), \
        torch.from_numpy(g["kweights"]).to(dev)


@pytest.mark.parametrize("name", ["si2_fcc", "si8_cubic", "si64_cubic"])
def test_density_matches_reference(cuda_device, name):
    from gradwave_b200.density import density_b
    g, ci, c, occ, kw = _inputs(name, cuda_device)
    bk = ci.bk.to(cuda_device)
    rho = density_b(c, occ, kw, bk, ci.shape, float(g["volume"])).cpu().numpy()
    chk = density_checksums(rho, int(g["seed"]))
    assert np.abs(chk - g["rho_chk"]).max() / np.abs(g["rho_chk"]).max() < TOL
    if "rho" in g:
        assert np.abs(rho - g["rho"]).max() / np.abs(g["rho"]).max() < TOL
    # Parseval: sum_r |psi(r)|^2 = N sum_G |c(G)|^2
    n = int(np.prod(ci.shape))
    w = (kw[:, None] * occ).cpu().numpy()
    expect = float((w * (c.abs() ** 2).sum(-1).cpu().numpy()).sum())
    assert abs(rho.sum() * float(g["volume"]) / n - expect) / expect < 1e-12


def test_density_chunking_storage_and_operator(cuda_device, monkeypatch):
    """Band chunks of the scratch do not change the result (bit for bit:
    every element sums its bands in the same order); complex64 storage is
    read into float64 FFTs; ``BatchedHamiltonian.density`` equals
    ``density_b``."""
    from gradwave_b200.density import density_b
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    g, ci, c, occ, kw = _inputs("si8_cubic", cuda_device)
    bk = ci.bk.to(cuda_device)
    vol = float(g["volume"])
    full = density_b(c, occ, kw, bk, ci.shape, vol)
    monkeypatch.setenv("GWB_W_BUDGET_MB", "1")  # read at every call: one band per chunk here
    chunked = density_b(c, occ, kw, bk, ci.shape, vol)
    assert torch.equal(full, chunked)
    monkeypatch.delenv("GWB_W_BUDGET_MB")
    c64 = c.to(torch.complex64)
    r64 = density_b(c64, occ, kw, bk, ci.shape, vol)
    ref = density_b(c64.to(torch.complex128), occ, kw, bk, ci.shape, vol)
    assert torch.equal(r64, ref)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
    assert torch.equal(h.density(c, occ, kw, vol), full)
