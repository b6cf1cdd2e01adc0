"""Learned preconditioner kernels against the float64 oracle (oracle/mlp.py).

* forward and gradient of the training kernel vs the oracle with the same
  BF16 rounding (float32 accumulation: 1e-2 relative in norm, with a few
  activations allowed to round to the neighbouring BF16 value);
* Adam step vs numpy;
* a zero output layer makes the learned step exactly TPA;
* training on solver-logged pairs lowers the held-out loss below TPA's;
* with the committed weights (trained on 8-atom cells), the held-out
  64-atom cell converges to the reference's eigenvalues in fewer rounds with
  the network than with TPA.
"""

import json

import numpy as np
import pytest
import torch

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu

HA = 27.211386245988


def _rand_params(seed):
    from oracle import mlp
    rng = np.random.default_rng(seed)
    p = mlp.init_params(seed)
    p[-(mlp.HID + 1):] = rng.standard_normal(mlp.HID + 1) * 0.3
    return p


def test_forward_and_gradient_vs_oracle(cuda_device):
    from gradwave_b200 import learned
    from oracle import mlp
    rng = np.random.default_rng(1)
    n = 777
    p = _rand_params(2)
    u = rng.standard_normal((n, 4)) * 0.8
    y = rng.standard_normal(n)
    w = rng.uniform(0, 1, n)
    w /= w.sum()
    P = torch.from_numpy(p.astype(np.float32)).to(cuda_device)
    U = torch.from_numpy(u.astype(np.float32)).to(cuda_device)
    out = learned.forward(P, U).cpu().numpy()
    o_ref, _ = mlp.forward(p.astype(np.float32).astype(np.float64), u.astype(np.float32).astype(np.float64))
    assert np.abs(out - o_ref).max() <= 2e-2 * max(1.0, np.abs(o_ref).max())
    loss, grad = learned.loss_grad(P, U, torch.from_numpy(y.astype(np.float32)).to(cuda_device),
                                   torch.from_numpy(w.astype(np.float32)).to(cuda_device))
    l_ref, g_ref = mlp.loss_grad(p.astype(np.float32).astype(np.float64), u.astype(np.float32).astype(np.float64),
                                 y.astype(np.float32).astype(np.float64), w.astype(np.float32).astype(np.float64))
    g = grad.cpu().numpy()
    assert abs(float(loss.item()) - l_ref) <= 1e-2 * l_ref
    assert np.linalg.norm(g - g_ref) <= 1e-2 * np.linalg.norm(g_ref)


def test_adam_step(cuda_device):
    import ctypes
    from gradwave_b200 import _lib, learned
    rng = np.random.default_rng(3)
    npar = learned.nparam()
    p = rng.standard_normal(npar).astype(np.float32)
    g = rng.standard_normal(npar).astype(np.float32)
    m = rng.standard_normal(npar).astype(np.float32) * 0.1
    v = np.abs(rng.standard_normal(npar)).astype(np.float32) * 0.1
    T = lambda a: torch.from_numpy(a.copy()).to(cuda_device)
    P, G, M, V = T(p), T(g), T(m), T(v)
    _lib.call("gwb_mlp_adam", P.data_ptr(), G.data_ptr(), M.data_ptr(), V.data_ptr(), 3, ctypes.c_float(1e-3),
              ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), _lib.stream_ptr(cuda_device))
    m2 = 0.9 * m + 0.1 * g
    v2 = 0.999 * v + 0.001 * g * g
    p2 = p - 1e-3 * (m2 / (1 - 0.9 ** 3)) / (np.sqrt(v2 / (1 - 0.999 ** 3)) + 1e-8)
    assert np.abs(P.cpu().numpy() - p2).max() < 1e-5


def test_zero_output_layer_is_tpa(cuda_device):
    from gradwave_b200 import _lib, learned
    rng = np.random.default_rng(5)
    nk, nb, npw, n_add = 2, 5, 300, 3
    x = rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))
    r = rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))
    t = np.abs(rng.standard_normal((nk, npw))) * 40
    eig = rng.standard_normal((nk, nb))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device)
    X, R, Tt, E = T(x), T(r), T(t), T(eig)
    sel = torch.tensor([[0, 3, 1], [4, 2, 0]], dtype=torch.int32, device=cuda_device)
    D1 = torch.zeros_like(X)
    D2 = torch.zeros_like(X)
    s = _lib.stream_ptr(cuda_device)
    _lib.call("gwb_precond_teter", nk, nb, n_add, npw, X.data_ptr(), nb * npw, R.data_ptr(), nb * npw,
              Tt.data_ptr(), sel.data_ptr(), D1.data_ptr(), nb * npw, s)
    P = torch.from_numpy(learned.init_params(0)).to(cuda_device)
    W = torch.empty(_lib.load().gwb_precond_learned_work_bytes(nk, n_add, npw), dtype=torch.uint8, device=cuda_device)
    _lib.call("gwb_precond_learned", P.data_ptr(), nk, nb, n_add, npw, X.data_ptr(), nb * npw, R.data_ptr(),
              nb * npw, Tt.data_ptr(), E.data_ptr(), sel.data_ptr(), None, D2.data_ptr(), nb * npw, W.data_ptr(),
              W.numel(), s)
    assert float((D1 - D2).abs().max()) < 1e-13


def test_training_on_logged_rows_beats_tpa(cuda_device):
    """Solver-logged rows of one perturbed cell; 300 Adam steps of the
    alignment objective lower the held-out loss below TPA's."""
    from gradwave_b200 import learned
    F, R, E, M = learned.collect_rows([("si8_perturbed", 11)], rows_per_round=24)
    assert F.shape[0] > 500 and torch.isfinite(F[M]).all()
    res = learned.train_alignment(F, R, E, M, steps=300, batch_rows=32, lr=3e-3)
    assert res.val_loss < res.val_loss_tpa


def test_alignment_gradient_matches_finite_difference(cuda_device):
    """dL/do from the band sums against a finite difference of the loss in o."""
    from gradwave_b200 import learned
    rng = np.random.default_rng(9)
    nrow, npw = 3, 50
    F = torch.from_numpy(rng.standard_normal((nrow, npw, 4)).astype(np.float32)).to(cuda_device)
    F[..., 0] = F[..., 0].abs()
    R = torch.from_numpy((rng.standard_normal((nrow, npw)) + 1j * rng.standard_normal((nrow, npw)))
                         .astype(np.complex64)).to(cuda_device)
    E = torch.from_numpy((rng.standard_normal((nrow, npw)) + 1j * rng.standard_normal((nrow, npw)))
                         .astype(np.complex64)).to(cuda_device)
    M = torch.ones(nrow, npw, dtype=torch.bool, device=cuda_device)
    P = torch.from_numpy(learned.init_params(0)).to(cuda_device)
    P[-65:] = torch.from_numpy(rng.standard_normal(65).astype(np.float32) * 0.1).to(cuda_device)
    L0, do = learned.alignment_loss(P, F, R, E, M, dout=True)
    # perturb the output bias b4: dL/db4 = sum_i dL/do_i (the step is far
    # above the BF16 spacing of b4, which the forward pass rounds to)
    h = 5e-2
    Pp, Pm = P.clone(), P.clone()
    Pp[-1] += h
    Pm[-1] -= h
    fd = (learned.alignment_loss(Pp, F, R, E, M) - learned.alignment_loss(Pm, F, R, E, M)) / (2 * h)
    assert abs(fd - float(do.sum())) <= 5e-2 * abs(fd) + 1e-6


def test_committed_network_gains_on_heldout_cell(cuda_device):
    """What the trained network gains: the committed weights were trained on
    rows logged from solves of seeded displaced and strained 8-atom cells
    only; applied to the 64-atom cell (4 k, 160 bands, basis 640: held out),
    the mixed solve with the network needs fewer Davidson rounds than the same
    solve with TPA, and both end within 1e-8 Ha of the reference's float64
    eigenvalues and 1e-6 Ha/cell in band energy."""
    from gradwave_b200 import learned
    from gradwave_b200.cells import make_cell
    from gradwave_b200.davidson import davidson_batched
    from gradwave_b200.hamiltonian import BatchedHamiltonian
    if not learned.available():
        pytest.skip("no trained weights committed")
    g = load_golden("si64_cubic")
    ci = make_cell("si64_cubic")
    bk = ci.bk.to(cuda_device)
    h = BatchedHamiltonian(bk, ci.shape, ci.v_eff_r, ci.p)
    x0 = ci.identity_start().to(cuda_device)
    lp = learned.LearnedPreconditioner.load(device=cuda_device)
    rl = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=300, mode="mixed", precond=lp)
    rt = davidson_batched(h.apply, x0, bk.t, bk.mask, tol=1e-10, max_iter=300, mode="mixed")
    nocc = ci.nocc()
    w = np.asarray(ci.kweights)
    for r in (rl, rt):
        eig = r.eigenvalues.cpu().numpy()
        assert float(r.residual_norms.max()) < 1e-10
        assert np.abs(eig - g["eigenvalues"]).max() < 1e-8 * HA
        be = 2.0 * float(np.sum(w[:, None] * (eig[:, :nocc] - g["eigenvalues"][:, :nocc])))
        assert abs(be) < 1e-6 * HA
    print(json.dumps({"learned_iters": rl.n_iter, "tpa_iters": rt.n_iter,
                      "learned_applies": rl.n_apply_low + rl.n_apply_full,
                      "tpa_applies": rt.n_apply_low + rt.n_apply_full}))
    assert rl.n_iter < rt.n_iter


@pytest.fixture(params=[1, 0], ids=["tcgen05", "mma_sync"])
def precond_kernel(request):
    """Both inference kernels of gwb_precond_learned."""
    from gradwave_b200 import _lib
    _lib.call("gwb_precond_set_kernel", request.param)
    yield request.param
    _lib.call("gwb_precond_set_kernel", 1)


def test_tensor_core_inference_matches_reference_forward(cuda_device, precond_kernel):
    """The tensor-core inference paths of gwb_precond_learned (tcgen05 and
    mma.sync) against features + the CUDA-core forward + TPA, on random
    parameters; 1000 plane waves per row leave a ragged last tile."""
    from gradwave_b200 import _lib, learned
    rng = np.random.default_rng(21)
    nk, nb, npw, n_add = 2, 4, 1000, 3
    x = rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))
    r = (rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))) * rng.uniform(0, 2, npw)
    t = np.abs(rng.standard_normal((nk, npw))) * 60
    eig = rng.standard_normal((nk, nb)) * 5
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device)
    X, R, Tt, E = T(x), T(r), T(t), T(eig)
    sel = torch.tensor([[1, 0, 3], [2, 3, 0]], dtype=torch.int32, device=cuda_device)
    p = learned.init_params(4)
    p[-65:] = rng.standard_normal(65).astype(np.float32) * 0.2
    P = torch.from_numpy(p).to(cuda_device)
    s = _lib.stream_ptr(cuda_device)
    D = torch.zeros_like(X)
    W = torch.empty(_lib.load().gwb_precond_learned_work_bytes(nk, n_add, npw), dtype=torch.uint8, device=cuda_device)
    _lib.call("gwb_precond_learned", P.data_ptr(), nk, nb, n_add, npw, X.data_ptr(), nb * npw, R.data_ptr(),
              nb * npw, Tt.data_ptr(), E.data_ptr(), sel.data_ptr(), None, D.data_ptr(), nb * npw, W.data_ptr(),
              W.numel(), s)
    F = torch.empty(nk, n_add, npw, 4, dtype=torch.float32, device=cuda_device)
    _lib.call("gwb_precond_features", nk, nb, n_add, npw, X.data_ptr(), nb * npw, R.data_ptr(), nb * npw,
              Tt.data_ptr(), E.data_ptr(), sel.data_ptr(), F.data_ptr(), s)
    o = learned.forward(P, F.reshape(-1, 4)).view(nk, n_add, npw).double().clamp(-3, 3)
    sl = sel.long().cpu().numpy()
    xs = np.take_along_axis(x, sl[..., None], 1)
    rs = np.take_along_axis(r, sl[..., None], 1)
    tb = np.einsum("kag,kg,kag->ka", xs.conj(), t, xs).real
    xx = t[:, None, :] / tb[..., None]
    pp = 27 + 18 * xx + 12 * xx ** 2 + 8 * xx ** 3
    tpa = pp / (pp + 16 * xx ** 4)
    ref = rs * tpa * np.exp(o.cpu().numpy())
    ref /= np.linalg.norm(ref, axis=-1, keepdims=True)
    got = D.cpu().numpy()[:, :n_add]
    assert np.abs(got - ref).max() <= 2e-2 * np.abs(ref).max()


def test_stall_rule(cuda_device):
    from gradwave_b200 import _lib
    n = 3
    best = torch.full((n,), float("inf"), dtype=torch.float64, device=cuda_device)
    cnt = torch.zeros(n, dtype=torch.uint8, device=cuda_device)
    tpa = torch.zeros(n, dtype=torch.uint8, device=cuda_device)
    s = _lib.stream_ptr(cuda_device)
    # band 0 improves every round, band 1 stagnates, band 2 improves once then stagnates
    seq = [[1.0, 1.0, 1.0], [0.5, 0.99, 0.5], [0.2, 0.98, 0.49], [0.1, 0.97, 0.48], [0.05, 0.96, 0.47]]
    for row in seq:
        rn = torch.tensor(row, dtype=torch.float64, device=cuda_device)
        _lib.call("gwb_stall_update", rn.data_ptr(), best.data_ptr(), cnt.data_ptr(), tpa.data_ptr(), n, 0.9, 3, s)
    torch.cuda.synchronize()
    assert tpa.tolist() == [0, 1, 1]


def test_gamma_embedded_rows_match_half_rows(cuda_device):
    """gwb_precond_learned_gamma on the Gamma path's embedded real rows equals
    the complex-row kernel on the same rows as sqrt(w)-scaled half-sphere rows
    (gamma._half_rows / _embed_rows), including a band kept on TPA and a
    ragged last tile; the pad coordinates come back zero."""
    from gradwave_b200 import _lib, learned
    from gradwave_b200.gamma import _embed_rows, _half_rows
    rng = np.random.default_rng(31)
    nb, nhalf = 6, 777
    nphi = 2 * nhalf - 1
    npad = nphi + 1
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device)
    x = rng.standard_normal((nb, npad))
    r = rng.standard_normal((nb, npad)) * rng.uniform(0, 2, npad)
    x[:, nphi:] = 0.0
    r[:, nphi:] = 0.0
    X, R = T(x), T(r)
    th = T(np.abs(rng.standard_normal(nhalf)) * 60)
    eig = T(rng.standard_normal(nb) * 5)
    sel = torch.tensor([4, 0, 2, 5], dtype=torch.int32, device=cuda_device)
    tpa = torch.zeros(nb, dtype=torch.uint8, device=cuda_device)
    tpa[2] = 1
    p = learned.init_params(7)
    p[-65:] = rng.standard_normal(65).astype(np.float32) * 0.2
    P = torch.from_numpy(p).to(cuda_device)
    n = int(sel.shape[0])
    D = torch.full((n, npad), 7.0, dtype=torch.float64, device=cuda_device)
    W = torch.empty(int(_lib.load().gwb_precond_learned_gamma_work_bytes(n, nhalf)), dtype=torch.uint8,
                    device=cuda_device)
    s = _lib.stream_ptr(cuda_device)
    _lib.call("gwb_precond_learned_gamma", P.data_ptr(), nb, n, nhalf, npad, X.data_ptr(), npad, R.data_ptr(), npad,
              th.data_ptr(), eig.data_ptr(), sel.data_ptr(), tpa.data_ptr(), D.data_ptr(), npad, W.data_ptr(),
              W.numel(), s)
    sl = sel.long()
    xs, rs = _half_rows(X[sl], nhalf), _half_rows(R[sl], nhalf)
    idx = torch.arange(n, dtype=torch.int32, device=cuda_device).reshape(1, n)
    ref = torch.ops.gwb.precond_apply(xs[None], rs[None], th.reshape(1, -1), idx, eig[sl].reshape(1, n), P,
                                      tpa[sl].reshape(1, n))
    ref = _embed_rows(ref[0], npad)
    torch.cuda.synchronize()
    assert float((D - ref).abs().max()) <= 1e-12
    assert float(D[:, nphi:].abs().max()) == 0.0
    assert torch.allclose(torch.linalg.vector_norm(D, dim=1), torch.ones(n, dtype=torch.float64,
                                                                         device=cuda_device), atol=1e-12)
