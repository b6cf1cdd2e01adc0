"""The batched float64 Hermitian eigensolver (gwb_heev_lowest) against LAPACK.

Cases: random Hermitian matrices with exactly degenerate clusters (Davidson
subspaces of Si have 2- and 3-fold degenerate Ritz values), a diagonal matrix
(zero off-diagonal: reflector skips), m = 1 and 2, and the largest supported m.
Tolerances: eigenvalues 1e-12 relative to the spectral radius, residual
|A y - lambda y| 1e-12 relative, orthonormality 1e-12.
"""


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
    Z = torch.zeros(nk, _lib.load().gwb_heev_scratch_doubles(m), dtype=torch.float64, device=dev)
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


def test_heev_fast_path_and_ql_fallback(cuda_device):
    """Typical Davidson shapes run on the bisection/inverse-iteration path (no
    QL fallback); m = nb = 112 does not fit its pool and runs QL; both agree
    with LAPACK."""
    from gradwave_b200 import _lib
    rng = np.random.default_rng(7)
    n0 = _lib.heev_ql_count()
    for m, nb in [(24, 24), (48, 24), (72, 24), (96, 24), (36, 24)]:
        S = np.stack([_random_herm(rng, m) for _ in range(3)])
        eig, U, info = _run(S, nb)
        assert np.all(info == 0)
        assert np.abs(eig - np.linalg.eigvalsh(S)[:, :nb]).max() <= 1e-12 * np.abs(np.linalg.eigvalsh(S)).max()
    assert _lib.heev_ql_count() == n0
    S = np.stack([_random_herm(rng, 112) for _ in range(2)])
    eig, U, info = _run(S, 112)
    assert np.all(info == 0)
    assert _lib.heev_ql_count() == n0 + 2
    scale = np.abs(np.linalg.eigvalsh(S)).max()
    assert np.abs(eig - np.linalg.eigvalsh(S)).max() <= 1e-12 * scale
    for k in range(2):
        assert np.abs(S[k] @ U[k] - U[k] * eig[k]).max() <= 1e-12 * scale


def test_heev_tight_clusters_and_wilkinson(cuda_device):
    """Eigenvalues split by 1e-12 relative, a 1e-9 pair, and the Wilkinson
    W21+ matrix (pairs agreeing to 1e-14): eigenvalues, residuals and
    orthonormality at the LAPACK level."""
    rng = np.random.default_rng(11)
    m, nb = 64, 16
    x = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
    q, _ = np.linalg.qr(x)
    ev = np.sort(rng.uniform(0, 10, m))
    ev[1], ev[2] = ev[0] + 1e-12, ev[0] + 2e-12
    ev[10] = ev[9] * (1 + 1e-9)
    h = (q * ev) @ q.conj().T
    w = np.diag(np.abs(np.arange(21) - 10.0)) + np.diag(np.ones(20), 1) + np.diag(np.ones(20), -1)
    for S, nbk in [(0.5 * (h + h.conj().T), nb), (w.astype(np.complex128), 21)]:
        eig, U, info = _run(S[None], nbk)
        assert info[0] == 0
        scale = np.abs(np.linalg.eigvalsh(S)).max()
        assert np.abs(eig[0] - np.linalg.eigvalsh(S)[:nbk]).max() <= 1e-12 * scale
        assert np.abs(S @ U[0] - U[0] * eig[0]).max() <= 1e-12 * scale
        assert np.abs(U[0].conj().T @ U[0] - np.eye(nbk)).max() <= 1e-12
