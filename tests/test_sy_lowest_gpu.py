"""libgwb's own dense symmetric eigensolver (``gwb_sytrd``, ``gwb_sy_lowest``)
against LAPACK (numpy's eigh / eigvalsh):

* the tridiagonalisation: the eigenvalues of (d, e) are those of A, and the
  reflectors in LAPACK's storage rebuild Q with Q^T A Q = T (small m);
* the lowest nev eigenpairs at odd and even m up to the Davidson subspace
  sizes (641, 1920): eigenvalues, residuals |A u - lambda u| and the
  orthonormality of U, all at float64 round-off of |A|;
* exact degenerate clusters (a triple, a sextuple), a pair 1e-13 apart, the
  Wilkinson matrices W21+ and W201+ (pairs equal to ~1e-14), and a block
  diagonal matrix (reflectors with tau = 0);
* each with the four forms of the tridiagonalisation: cooperative panels,
  the opt-in shared-memory-resident grid kernel and the cluster; without the
  cluster; without the grid kernel (the default); the cooperative launch
  alone (``gwb_sytrd_set_grid``, ``gwb_sytrd_set_cluster``); 1920 passes
  through all three launches in the first form.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[(1, -1), (1, 0), (0, -1), (0, 0)], ids=["grid+cluster", "grid", "cluster", "coop"])
def cluster(request):
    """The forms of the tridiagonalisation: cooperative panels, then the
    shared-memory-resident grid kernel (opt-in), then one thread-block
    cluster; without the cluster; without the grid kernel (the default);
    the cooperative launch alone."""
    from gradwave_b200 import _lib
    grid, cl = request.param
    _lib.call("gwb_sytrd_set_grid", grid)
    _lib.call("gwb_sytrd_set_cluster", cl)
    yield request.param
    _lib.call("gwb_sytrd_set_grid", 0)
    _lib.call("gwb_sytrd_set_cluster", -1)


def _sytrd(a, dev):
    from gradwave_b200 import _lib
    m = a.shape[0]
    A = torch.from_numpy(a.copy()).to(dev)
    d = torch.empty(m, dtype=torch.float64, device=dev)
    e = torch.empty(max(m - 1, 1), dtype=torch.float64, device=dev)
    tau = torch.empty(m, dtype=torch.float64, device=dev)
    w = torch.empty(int(_lib.load().gwb_sytrd_work_bytes(m)), dtype=torch.uint8, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call("gwb_sytrd", m, A.data_ptr(), m, d.data_ptr(), e.data_ptr(), tau.data_ptr(), w.data_ptr(), w.numel(),
              st.data_ptr(), _lib.stream_ptr(dev))
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return A.cpu().numpy(), d.cpu().numpy(), e.cpu().numpy()[: m - 1], tau.cpu().numpy()


def _lowest(a, nev, dev):
    from gradwave_b200 import _lib
    m = a.shape[0]
    A = torch.from_numpy(a.copy()).to(dev)
    w = torch.empty(nev, dtype=torch.float64, device=dev)
    ut = torch.empty(nev, m, dtype=torch.float64, device=dev)
    wk = torch.empty(int(_lib.load().gwb_sy_lowest_work_bytes(m, nev)), dtype=torch.uint8, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call("gwb_sy_lowest", m, nev, A.data_ptr(), m, w.data_ptr(), ut.data_ptr(), m, wk.data_ptr(), wk.numel(),
              st.data_ptr(), _lib.stream_ptr(dev))
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return w.cpu().numpy(), ut.cpu().numpy().T


def _rand(m, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((m, m))
    return 0.5 * (a + a.T) * 0.05 + np.diag(np.linspace(-5.0, 80.0, m))


def _with_spectrum(lam, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((len(lam), len(lam))))
    a = (q * lam) @ q.T
    return 0.5 * (a + a.T)


def _wilkinson(m):
    k = (m - 1) // 2
    return np.diag(np.abs(np.arange(m) - k).astype(np.float64)) + np.diag(np.ones(m - 1), 1) + np.diag(np.ones(m - 1), -1)


def _check(a, nev, dev):
    w, u = _lowest(a, nev, dev)
    ref = np.linalg.eigvalsh(a)
    scale = float(np.abs(ref).max())
    assert np.abs(w - ref[:nev]).max() <= 1e-13 * scale
    assert np.abs(a @ u - u * w).max() <= 1e-12 * scale
    assert np.abs(u.T @ u - np.eye(nev)).max() <= 1e-12


@pytest.mark.parametrize("m", [2, 3, 9, 17, 200, 700, 1100])
def test_tridiagonalisation_rebuilds_q(cuda_device, cluster, m):
    """Q^T A Q = T with Q rebuilt from the stored reflectors; 700 and 1100
    hand the trailing part from the grid kernel (or the cooperative launch)
    to the cluster."""
    a = _rand(m, m)
    A, d, e, tau = _sytrd(a, cuda_device)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    Q = np.eye(m)
    for j in range(m - 1):  # column j of the column-major output is row j of the array
        v = np.zeros(m)
        v[j + 1] = 1.0
        v[j + 2:] = A[j, j + 2:]
        Q -= tau[j] * np.outer(Q @ v, v)
    scale = float(np.abs(np.linalg.eigvalsh(a)).max())
    assert np.abs(Q.T @ a @ Q - T).max() <= 1e-13 * scale
    assert np.abs(Q.T @ Q - np.eye(m)).max() <= 1e-13


@pytest.mark.parametrize("m,nev", [(2, 2), (3, 3), (50, 50), (600, 300), (641, 320), (1920, 496)])
def test_lowest_pairs_random(cuda_device, cluster, m, nev):
    _check(_rand(m, m + 1), nev, cuda_device)


def test_lowest_pairs_degenerate_clusters(cuda_device, cluster):
    m = 700
    lam = np.linspace(-5.0, 80.0, m)
    lam[10:13] = lam[10]
    lam[40:46] = lam[40]
    lam[100:102] = lam[100] + np.array([0.0, 1e-13])
    _check(_with_spectrum(lam, 3), 300, cuda_device)


@pytest.mark.parametrize("m", [21, 201])
def test_wilkinson(cuda_device, cluster, m):
    _check(_wilkinson(m), m, cuda_device)


def test_block_diagonal_needs_no_reflection(cuda_device, cluster):
    a = np.zeros((300, 300))
    a[:120, :120] = _rand(120, 7)
    a[120:, 120:] = _rand(180, 8) + 3.0 * np.eye(180)
    A, d, e, tau = _sytrd(a, cuda_device)
    assert np.abs(np.sort(np.linalg.eigvalsh(np.diag(d) + np.diag(e, 1) + np.diag(e, -1)))
                  - np.linalg.eigvalsh(a)).max() <= 1e-12 * np.abs(a).max()
    _check(a, 300, cuda_device)
