"""Device kernels of the Davidson steps against numpy float64 on small cases:
Cholesky + triangular inverse (shared-memory and global versions), the TPA
preconditioner, the residual and the worst-residual selection."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 7, 24, 64, 65, 100])
def test_chol_inv(cuda_device, n):
    from gradwave_b200 import _lib
    rng = np.random.default_rng(n)
    nk = 3
    a = rng.standard_normal((nk, n, n + 5)) + 1j * rng.standard_normal((nk, n, n + 5))
    g = a @ a.conj().transpose(0, 2, 1)
    G = torch.from_numpy(g.copy()).to(cuda_device)
    Linv = torch.zeros(nk, n, n, dtype=torch.complex128, device=cuda_device)
    info = torch.full((nk,), -1, dtype=torch.int32, device=cuda_device)
    _lib.call("gwb_chol_inv", nk, n, G.data_ptr(), n, n * n, Linv.data_ptr(), n * n, info.data_ptr(), None,
              _lib.stream_ptr(cuda_device))
    torch.cuda.synchronize()
    assert np.all(info.cpu().numpy() == 0)
    L = np.tril(G.cpu().numpy())
    Li = Linv.cpu().numpy()
    for k in range(nk):
        ref = np.linalg.cholesky(g[k])
        assert np.abs(L[k] - ref).max() <= 1e-10 * np.abs(ref).max()
        assert np.abs(Li[k] @ ref - np.eye(n)).max() <= 1e-10
        assert np.abs(np.triu(Li[k], 1)).max() == 0.0


def test_chol_breakdown_flag(cuda_device):
    from gradwave_b200 import _lib
    n, nk = 6, 2
    g = np.stack([np.eye(n), np.eye(n)]).astype(np.complex128)
    g[1, 3, 3] = -1.0
    G = torch.from_numpy(g).to(cuda_device)
    Linv = torch.zeros(nk, n, n, dtype=torch.complex128, device=cuda_device)
    info = torch.zeros(nk, dtype=torch.int32, device=cuda_device)
    flag = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    _lib.call("gwb_chol_inv", nk, n, G.data_ptr(), n, n * n, Linv.data_ptr(), n * n, info.data_ptr(),
              flag.data_ptr(), _lib.stream_ptr(cuda_device))
    torch.cuda.synchronize()
    assert info.tolist() == [0, 4]
    assert int(flag.item()) & 2


def test_precond_residual_select(cuda_device):
    from gradwave_b200 import _lib
    from oracle.precond import teter_b
    rng = np.random.default_rng(4)
    nk, nb, npw, n_add = 3, 6, 500, 4
    x = rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))
    hx = rng.standard_normal((nk, nb, npw)) + 1j * rng.standard_normal((nk, nb, npw))
    eig = rng.standard_normal((nk, nb))
    t = np.abs(rng.standard_normal((nk, npw))) * 50
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device)
    X, HX, E, Tt = T(x), T(hx), T(eig), T(t)
    R = torch.zeros_like(X)
    rn = torch.zeros(nk, nb, dtype=torch.float64, device=cuda_device)
    s = _lib.stream_ptr(cuda_device)
    _lib.call("gwb_residual", nk, nb, npw, X.data_ptr(), nb * npw, HX.data_ptr(), nb * npw, E.data_ptr(), nb,
              R.data_ptr(), nb * npw, rn.data_ptr(), s)
    r_ref = hx - eig[..., None] * x
    assert np.abs(R.cpu().numpy() - r_ref).max() < 1e-13
    assert np.abs(rn.cpu().numpy() - np.linalg.norm(r_ref, axis=-1)).max() < 1e-12
    sel = torch.zeros(nk, n_add, dtype=torch.int32, device=cuda_device)
    _lib.call("gwb_select_worst", nk, nb, rn.data_ptr(), n_add, sel.data_ptr(), s)
    sel_ref = np.argsort(-np.linalg.norm(r_ref, axis=-1), axis=1, kind="stable")[:, :n_add]
    assert np.array_equal(sel.cpu().numpy(), sel_ref)
    D = torch.zeros(nk, nb, npw, dtype=torch.complex128, device=cuda_device)
    _lib.call("gwb_precond_teter", nk, nb, n_add, npw, X.data_ptr(), nb * npw, R.data_ptr(), nb * npw,
              Tt.data_ptr(), sel.data_ptr(), D.data_ptr(), nb * npw, s)
    tband = np.einsum("kbg,kg,kbg->kb", x.conj(), t, x).real
    rsel = np.take_along_axis(r_ref, sel_ref[..., None], 1)
    d_ref = teter_b(rsel, t, np.take_along_axis(tband, sel_ref, 1))
    d_ref /= np.linalg.norm(d_ref, axis=-1, keepdims=True)
    assert np.abs(D.cpu().numpy()[:, :n_add] - d_ref).max() < 1e-12


@pytest.mark.parametrize("M,N,K,batch", [(96, 24, 4645, 10), (7, 3, 100, 2), (640, 160, 37073, 1), (24, 24, 33, 4)])
def test_zgemm_nh_split_k(cuda_device, M, N, K, batch):
    from gradwave_b200 import _lib
    rng = np.random.default_rng(M + N)
    a = rng.standard_normal((batch, M, K)) + 1j * rng.standard_normal((batch, M, K))
    b = rng.standard_normal((batch, N, K)) + 1j * rng.standard_normal((batch, N, K))
    c0 = rng.standard_normal((batch, M, N)) + 1j * rng.standard_normal((batch, M, N))
    A, B, C = (torch.from_numpy(x).to(cuda_device) for x in (a, b, c0))
    work = torch.empty(24 << 20, dtype=torch.uint8, device=cuda_device)
    _lib.call("gwb_zgemm_nh", M, N, K, 0.5, 0.25, A.data_ptr(), K, M * K, B.data_ptr(), K, N * K, -1.0, 0.0,
              C.data_ptr(), N, M * N, batch, work.data_ptr(), work.numel(), _lib.stream_ptr(cuda_device))
    ref = (0.5 + 0.25j) * a @ b.conj().transpose(0, 2, 1) - c0
    assert np.abs(C.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
