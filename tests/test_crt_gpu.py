"""Float64-accurate products on the int8 tensor cores through residues
(``gradwave_b200.oz``: ``ResidueSet``, ``crt_gemm``, ``CrtMatmul``) against
float64 products of numpy with long-double accumulation.

* the residue planes rebuild every row: the centred residues of each element
  agree, modulo every m_t, with the nearest integer to x / scale; the scales
  are 2^(e - p) with 2^e the power of two above the row maximum; pad columns
  are zero;
* A B^T for ragged sizes (partial tiles in M, N and K), K split across CTAs,
  alpha/beta, offset rows, and each modulus count: the error of every
  element stays within the conversion bound
  2^-p (max|a_i| sum|b_j| + max|b_j| sum|a_i|) plus the reference's rounding;
* A B through the transposed residues of B, written in two column blocks
  (as the Davidson basis grows), with B's row scales folded into A;
* K = 0 leaves beta C; a non-finite row gives NaN in its products; the
  workspace size is checked.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rows(rng, n, k, decay=12.0, amp=1.0):
    d = np.exp(-np.linspace(0.0, decay, k))
    return rng.standard_normal((n, k)) * d * amp


def _exact(a, b):
    return (a.astype(np.longdouble) @ b.T.astype(np.longdouble)).astype(np.float64)


def _bound(a, b, p):
    """Conversion bound of C = A B^T per element, plus float64 rounding."""
    ma, mb = np.abs(a).max(axis=1), np.abs(b).max(axis=1)
    sa, sb = np.abs(a).sum(axis=1), np.abs(b).sum(axis=1)
    conv = 2.0 ** -p * (ma[:, None] * sb[None, :] + mb[None, :] * sa[:, None])
    return 2.0 * conv + 4e-16 * (np.abs(a) @ np.abs(b).T)


def test_split_rows_rebuilds_the_rows(cuda_device):
    from gradwave_b200 import _lib
    from gradwave_b200.oz import ResidueSet
    n = 18
    p = int(_lib.load().gwb_crt_bits(n))
    rng = np.random.default_rng(1)
    a = _rows(rng, 21, 1000, amp=5.0)
    a[3] = 0.0
    st = ResidueSet(24, 1000, cuda_device, n=n)
    st.split_rows(torch.from_numpy(a).to(cuda_device), row0=2)
    torch.cuda.synchronize()
    q = st.q.cpu().numpy().astype(np.int64)[:, 2:23]
    sc = st.scale.cpu().numpy()[2:23]
    mods = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181][:n]
    mx = np.abs(a).max(axis=1)
    nz = mx > 0
    assert np.all(sc[nz] * 2.0 ** p > mx[nz]) and np.all(sc[nz] * 2.0 ** p <= 2 * mx[nz])
    assert np.all(np.log2(sc) == np.round(np.log2(sc)))
    xi = [[int(np.rint(v / s)) for v in row] for row, s in zip(a, sc)]
    for t, m in enumerate(mods):
        assert np.abs(q[t]).max() <= 128
        for r in (0, 3, 7, 20):
            for k in (0, 1, 499, 999):
                assert (int(q[t, r, k]) - xi[r][k]) % m == 0
    assert np.all(q[:, :, 1000:] == 0)


@pytest.mark.parametrize("n,M,N,K", [(18, 200, 300, 20011), (18, 130, 70, 4099), (16, 64, 64, 80000),
                                     (20, 257, 129, 777), (18, 128, 256, 64), (18, 1, 1, 1)])
def test_product_nt(cuda_device, n, M, N, K):
    from gradwave_b200 import _lib
    from gradwave_b200.oz import ResidueSet, check_status, crt_gemm
    p = int(_lib.load().gwb_crt_bits(n))
    rng = np.random.default_rng(M + N + K)
    a = _rows(rng, M, K)
    b = _rows(rng, N, K, amp=300.0)
    sa, sb = ResidueSet(M + 3, K, cuda_device, n=n), ResidueSet(N, K, cuda_device, n=n)
    sa.split_rows(torch.from_numpy(a).to(cuda_device), row0=3)
    sb.split_rows(torch.from_numpy(b).to(cuda_device))
    c0 = rng.standard_normal((M, N))
    c = torch.from_numpy(c0.copy()).to(cuda_device)
    crt_gemm(M, N, K, sa, sb, c, alpha=-0.5, beta=2.0, a_row0=3)
    check_status(cuda_device)
    ref = -0.5 * _exact(a, b) + 2.0 * c0
    err = np.abs(c.cpu().numpy() - ref)
    assert np.all(err <= 0.5 * _bound(a, b, p) + 4e-16 * np.abs(2.0 * c0) + 1e-300), float(err.max())


def test_product_large_k_split(cuda_device):
    """K = 80,798 (the 216-atom cell's embedded basis): split across CTAs."""
    from gradwave_b200 import _lib
    from gradwave_b200.oz import CrtMatmul, check_status
    p = int(_lib.load().gwb_crt_bits(18))
    rng = np.random.default_rng(7)
    a = _rows(rng, 300, 80798)
    b = _rows(rng, 200, 80798, amp=40.0)
    cm = CrtMatmul(cuda_device, n=18)
    c = torch.empty(300, 200, dtype=torch.float64, device=cuda_device)
    cm.nt(torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device), c)
    check_status(cuda_device)
    err = np.abs(c.cpu().numpy() - _exact(a, b))
    assert np.all(err <= _bound(a, b, p)), float(err.max())
    g = torch.empty(300, 300, dtype=torch.float64, device=cuda_device)
    at = torch.from_numpy(a).to(cuda_device)
    cm.nt(at, at, g, same=True)
    check_status(cuda_device)
    gerr = np.abs(g.cpu().numpy() - _exact(a, a))
    assert np.all(gerr <= _bound(a, a, p)), float(gerr.max())


def test_product_nn_transposed_blocks(cuda_device):
    """C = A B with B (K x N) written as transposed residues in two blocks of
    rows, B's per-row scales folded into A."""
    from gradwave_b200 import _lib
    from gradwave_b200.oz import ResidueSet, check_status, crt_gemm
    p = int(_lib.load().gwb_crt_bits(18))
    rng = np.random.default_rng(11)
    M, K, N = 90, 700, 5000
    a = rng.standard_normal((M, K))
    b = _rows(rng, K, N, decay=8.0) * np.exp(rng.uniform(-3, 3, (K, 1)))
    sb = ResidueSet(N, 1024, cuda_device, n=18)
    bt = torch.from_numpy(b).to(cuda_device)
    sb.split_cols(bt[:300], k0=0)
    sb.split_cols(bt[300:], k0=300)
    sa = ResidueSet(M, K, cuda_device, n=18)
    sa.split_rows(torch.from_numpy(a).to(cuda_device), fold=sb.kscale)
    c = torch.empty(M, N, dtype=torch.float64, device=cuda_device)
    crt_gemm(M, N, K, sa, sb, c)
    check_status(cuda_device)
    ref = (a.astype(np.longdouble) @ b.astype(np.longdouble)).astype(np.float64)
    ks = sb.kscale.cpu().numpy()[:K]
    af = a * ks[None, :]
    bs = b / ks[:, None]
    ma = np.abs(af).max(axis=1)
    conv = 2.0 ** -p * (ma[:, None] * np.abs(bs).sum(axis=0)[None, :] + np.abs(af) @ np.ones((K, N)))
    err = np.abs(c.cpu().numpy() - ref)
    assert np.all(err <= 2 * conv + 4e-16 * (np.abs(a) @ np.abs(b))), float(err.max())


def test_zero_k_nan_rows_and_workspace(cuda_device):
    from gradwave_b200 import _lib
    from gradwave_b200.oz import ResidueSet, check_status, crt_gemm
    rng = np.random.default_rng(3)
    sa, sb = ResidueSet(8, 256, cuda_device), ResidueSet(8, 256, cuda_device)
    c0 = rng.standard_normal((8, 8))
    c = torch.from_numpy(c0.copy()).to(cuda_device)
    crt_gemm(8, 8, 0, sa, sb, c, beta=3.0)
    check_status(cuda_device)
    assert np.allclose(c.cpu().numpy(), 3.0 * c0, rtol=0, atol=0)
    a = rng.standard_normal((8, 256))
    a[5, 17] = np.nan
    b = rng.standard_normal((8, 256))
    sa.split_rows(torch.from_numpy(a).to(cuda_device))
    sb.split_rows(torch.from_numpy(b).to(cuda_device))
    crt_gemm(8, 8, 256, sa, sb, c)
    check_status(cuda_device)
    out = c.cpu().numpy()
    assert np.all(np.isnan(out[5])) and np.all(np.isfinite(np.delete(out, 5, axis=0)))
    need = int(_lib.load().gwb_crt_work_bytes(18, 8, 8, 256))
    small = torch.empty(max(need - 16, 16), dtype=torch.uint8, device=cuda_device)
    with pytest.raises(_lib.GwbError):
        crt_gemm(8, 8, 256, sa, sb, c, work=small)
    with pytest.raises(_lib.GwbError):
        crt_gemm(8, 8, (1 << 19) + 64, ResidueSet(8, (1 << 19) + 64, cuda_device), sb, c)


def test_gamma_solve_on_residue_products(cuda_device, monkeypatch):
    """The 216-atom Gamma solve (mixed, locking, 16 buffer bands) with every
    float64 product of the solver on the residue products: converged to
    1e-10 eV, eigenvalues within 1e-8 Ha of the reference's complex float64
    solve."""
    from tests.conftest import load_golden
    from tests.test_gamma_gpu import HA, _gamma
    from gradwave_b200.gamma import davidson_gamma, gamma_start
    monkeypatch.setenv("GWB_OZ", "crt")
    gc = load_golden("si216_vacancy")
    ci, gb, gh = _gamma("si216_vacancy", cuda_device)
    res = davidson_gamma(gh, gamma_start(gb, ci.nbands, cuda_device), tol=1e-10, max_iter=200, mode="mixed",
                         n_buffer=16)
    assert float(res.residual_norms.max()) < 1e-10
    assert np.abs(res.eigenvalues.cpu().numpy() - gc["eigenvalues"][0]).max() < 1e-8 * HA
