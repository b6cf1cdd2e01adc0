"""The torch custom ops of the path (``gwb::davidson_solve``,
``gwb::precond_apply``) against the oracle and the reference's goldens.

* ``davidson_solve`` on the 2-atom cell: eigenvalues within 1e-9 eV of the
  reference's own float64 Davidson (``tests/golden/si2_fcc.npz``), residuals
  below tol, the stats vector consistent with the result.
* ``precond_apply`` without weights: the TPA rows of the selected bands equal
  the float64 oracle's ``teter_b`` (gradwave ``solvers/precond.py:20-39``),
  unit-normalised, to 1e-12; with the untrained network (zero output layer,
  K = TPA exactly) the learned path gives the same rows to float32 accuracy.
"""

import numpy as np
import pytest
import torch

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


def test_davidson_solve_op_matches_reference(cuda_device):
    from gradwave_b200.cells import make_cell
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    from gradwave_b200.ops import SOLVE_MODES, SOLVE_STATS
    g = load_golden("si2_fcc")
    ci = make_cell("si2_fcc")
    bk = ci.bk.to(cuda_device)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
    x0 = ci.identity_start().to(cuda_device)
    eig, vec, rn, stats = torch.ops.gwb.davidson_solve(h.handle, x0, bk.t, bk.mask, 1e-10, 200, 32,
                                                        SOLVE_MODES["fp64"], 0, None)
    st = dict(zip(SOLVE_STATS, stats.tolist()))
    assert np.abs(eig.cpu().numpy() - g["eigenvalues"]).max() < 1e-9
    assert float(rn.max()) < 1e-10 and st["max_residual"] < 1e-10
    assert st["hit_max_iter"] == 0 and 0 < st["n_iter"] < 200
    pad = vec[~bk.mask[:, None, :].expand_as(vec)]
    assert vec.shape == x0.shape and (pad.numel() == 0 or float(pad.abs().max()) == 0.0)


def test_precond_apply_op(cuda_device):
    from gradwave_b200 import learned
    from oracle.precond import teter_b
    rng = np.random.default_rng(9)
    nk, nb, npw, n_add = 2, 7, 700, 4
    x = rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))
    r = rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))
    t = np.abs(rng.standard_normal((nk, npw))) * 40.0
    eig = rng.standard_normal((nk, nb))
    sel = np.stack([rng.permutation(nb)[:n_add] for _ in range(nk)]).astype(np.int32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device)
    d = torch.ops.gwb.precond_apply(T(x), T(r), T(t), T(sel), T(eig), None, None).cpu().numpy()
    xs = np.take_along_axis(x, sel[..., None].astype(np.int64), axis=1)
    rs = np.take_along_axis(r, sel[..., None].astype(np.int64), axis=1)
    tb = np.einsum("kbg,kg,kbg->kb", xs.conj(), t, xs).real
    ref = teter_b(rs, t, tb)
    ref /= np.linalg.norm(ref, axis=-1, keepdims=True)
    assert np.abs(d - ref).max() < 1e-12
    params = torch.from_numpy(learned.init_params(0)).to(cuda_device)
    dl = torch.ops.gwb.precond_apply(T(x), T(r), T(t), T(sel), T(eig), params, None).cpu().numpy()
    assert np.abs(dl - ref).max() < 1e-5
