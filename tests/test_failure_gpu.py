"""Failure paths of the band solve on the GPU, in forms that fault nothing:
every failure is made on the host (bad input data, a withheld load, a
corrupted network) and must come back as a status the host reads, with the
CUDA context still usable afterwards.

* a non-finite start block: GWB_ERR_NONFINITE from the native solver (checked
  before any kernel uses the block) and from the host driver;
* a rank-deficient start block (two equal rows): repaired and converged to
  the reference's eigenvalues (gradwave solvers/davidson.py:406-457 jitters
  such rows);
* a learned preconditioner whose network is corrupted: the stall rule
  reverts the affected bands to TPA inside the solve and the solve still
  converges to the reference's eigenvalues;
* a tensor-core product whose producer withholds one K step's load: the
  consumer's bounded wait (set to about a millisecond) runs out,
  GWB_ERR_TIMEOUT comes back through the status word, and the next product
  on the same context is correct.
"""

import numpy as np
import pytest
import torch

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


def _si2(dev):
    from gradwave_b200.cells import make_cell
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    ci = make_cell("si2_fcc")
    bk = ci.bk.to(dev)
    return ci, bk, BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)


def test_nonfinite_start_block(cuda_device, monkeypatch):
    from gradwave_b200 import _lib
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.ops import SOLVE_MODES
    ci, bk, h = _si2(cuda_device)
    x0 = ci.identity_start().to(cuda_device)
    x0[0, 3, 5] = float("nan")
    with pytest.raises(Exception, match="status 3"):
        torch.ops.gwb.davidson_solve(h.handle, x0, bk.t, bk.mask, 1e-10, 50, 32, SOLVE_MODES["fp64"], 0, None)
    monkeypatch.setenv("GWB_NATIVE", "0")
    with pytest.raises(_lib.GwbError) as e:
        davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=50)
    assert e.value.status == _lib.GWB_ERR_NONFINITE
    # the context is still usable
    x0[0, 3, 5] = 0.0
    r = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=200)
    assert float(r.residual_norms.max()) < 1e-10


def test_rank_deficient_start_block(cuda_device):
    from gradwave_b200.davidson import davidson_batched
    g = load_golden("si2_fcc")
    ci, bk, h = _si2(cuda_device)
    x0 = ci.identity_start().to(cuda_device)
    x0[:, 1] = x0[:, 0]                      # two equal rows: rank nb - 1
    r = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=200)
    assert float(r.residual_norms.max()) < 1e-10
    assert np.abs(r.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < 1e-9


def test_corrupted_network_falls_back_to_tpa(cuda_device):
    """Output weights drawn at a large scale make exp(o) a random factor of up
    to e^3 either way at every plane wave: the preconditioned directions are
    poor, the stall rule sends the bands that stop improving to TPA, and the
    solve still ends at the reference's eigenvalues."""
    from gradwave_b200 import learned
    from gradwave_b200.cells import make_cell
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    g = load_golden("si8_cubic")
    ci = make_cell("si8_cubic")
    bk = ci.bk.to(cuda_device)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
    p = learned.init_params(0)
    hid, nin = learned.HID, learned.NIN
    w4 = hid * nin + hid + 2 * (hid * hid + hid)
    p[w4:w4 + hid] = np.random.default_rng(5).standard_normal(hid).astype(np.float32) * 20.0
    pc = learned.LearnedPreconditioner(p, device=cuda_device)
    x0 = ci.identity_start().to(cuda_device)
    r = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=300, mode="fp64", precond=pc)
    assert r.info.get("native") and r.info["n_tpa_fallback"] > 0
    assert float(r.residual_norms.max()) < 1e-10
    assert np.abs(r.eigenvalues.cpu().numpy() - g["eigenvalues"]).max() < 1e-9


def test_tensor_core_wait_runs_out(cuda_device):
    from gradwave_b200 import _lib
    from gradwave_b200.tc import OP_H, PlaneSet, zgemm_tc
    gen = torch.Generator(device="cpu").manual_seed(3)
    nk, n, m, k = 1, 100, 60, 512
    A = torch.randn(nk, n, k, dtype=torch.complex128, generator=gen).to(cuda_device)
    B = torch.randn(nk, m, k, dtype=torch.complex128, generator=gen).to(cuda_device)
    pa, pb = PlaneSet(nk, n, k, cuda_device), PlaneSet(nk, m, k, cuda_device)
    pa.write(A, n)
    pb.write(B, m)
    C = torch.zeros(nk, n, m, dtype=torch.complex128, device=cuda_device)
    status = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    lib = _lib.load()
    try:
        _lib.check(lib.gwb_tc_set_wait_limit(2_000_000))     # ~1 ms of SM clock
        _lib.check(lib.gwb_tc_test_withhold(0))
        zgemm_tc(OP_H, n, m, k, pa, pb, C, m, n * m, status=status)
        torch.cuda.synchronize()
        assert int(status.item()) & _lib.GWB_ERR_TIMEOUT
    finally:
        _lib.check(lib.gwb_tc_test_withhold(-1))
        _lib.check(lib.gwb_tc_set_wait_limit(4_000_000_000))
    status.zero_()
    zgemm_tc(OP_H, n, m, k, pa, pb, C, m, n * m, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref = A @ B.conj().transpose(-1, -2)
    bound = A.abs() @ B.abs().transpose(-1, -2)
    assert float(((C - ref).abs() / bound).max()) < 4e-5
