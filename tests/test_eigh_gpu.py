"""The batched float64 Hermitian eigensolver (gwb_heev_lowest) against LAPACK.

Cases: random Hermitian matrices with exactly degenerate clusters (Davidson
subspaces of Si have 2- and 3-fold degenerate Ritz values), a diagonal matrix
(zero off-diagonal: reflector skips), m = 1 and 2, and the largest supported m.
Tolerances: eigenvalues 1e-12 relative to the spectral radius, residual
|A y - lambda y| 1e-12 relative, orthonormality 1e-12.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _run(S: np.ndarray, nb: int):
    from gradwave_b200 import _lib
    nk, m, _ = S.shape
    dev = torch.device("cuda", 0)
    St = torch.from_numpy(S).to(dev)
    eig = torch.zeros(nk, nb, dtype=torch.float64, device=dev)
    U = torch.zeros(nk, m, nb, dtype=torch.complex128, device=dev)
    Z = torch.zeros(nk, m * m, dtype=torch.float64, device=dev)
    info = torch.full((nk,), -1, dtype=torch.int32, device=dev)
    _lib.call("gwb_heev_lowest", nk, m, nb, St.data_ptr(), m, m * m, eig.data_ptr(), U.data_ptr(),
              Z.data_ptr(), info.data_ptr(), _lib.stream_ptr(dev))
    torch.cuda.synchronize()
    return eig.cpu().numpy(), U.cpu().numpy(), info.cpu().numpy()


def _random_herm(rng, m, degenerate=True):
    x = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
    q, _ = np.linalg.qr(x)
    ev = np.sort(rng.uniform(-50, 400, m))
    if degenerate and m >= 8:
        ev[2:5] = ev[2]
        ev[6:8] = ev[6]
    h = (q * ev) @ q.conj().T
    return 0.5 * (h + h.conj().T)


@pytest.mark.parametrize("m,nb", [(1, 1), (2, 2), (3, 2), (13, 5), (24, 24), (57, 20), (96, 24), (97, 24), (112, 40)])
def test_heev_matches_lapack(cuda_device, m, nb):
    from gradwave_b200 import _lib
    assert m <= _lib.load().gwb_heev_max_dim()
    rng = np.random.default_rng(m)
    S = np.stack([_random_herm(rng, m) for _ in range(5)])
    eig, U, info = _run(S, nb)
    assert np.all(info == 0)
    scale = np.abs(np.linalg.eigvalsh(S)).max()
    ref = np.linalg.eigvalsh(S)[:, :nb]
    assert np.abs(eig - ref).max() <= 1e-12 * scale
    for k in range(S.shape[0]):
        r = S[k] @ U[k] - U[k] * eig[k]
        assert np.abs(r).max() <= 1e-12 * scale
        assert np.abs(U[k].conj().T @ U[k] - np.eye(nb)).max() <= 1e-12


def test_heev_diagonal_and_tridiagonal(cuda_device):
    rng = np.random.default_rng(3)
    m = 40
    d = rng.uniform(-5, 5, m)
    diag = np.diag(d).astype(np.complex128)[None]
    eig, U, info = _run(diag, 10)
    assert info[0] == 0
    assert np.abs(eig[0] - np.sort(d)[:10]).max() < 1e-13
    tri = np.diag(d) + np.diag(rng.standard_normal(m - 1) * 1j, -1)
    tri = (tri + tri.conj().T - np.diag(np.diag(tri))).astype(np.complex128)[None]
    tri[0] = 0.5 * (tri[0] + tri[0].conj().T)
    eig, U, info = _run(tri, 10)
    assert np.abs(eig[0] - np.linalg.eigvalsh(tri[0])[:10]).max() < 1e-12
