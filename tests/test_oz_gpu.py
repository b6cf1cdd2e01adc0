"""Float64-accurate products on the int8 tensor cores (``gradwave_b200.oz``)
against float64 products of numpy (long-double accumulation as the exact
reference).

* the slices (rounded to nearest, |q| <= 64) rebuild every element to 2^-7s
  of its row's scale, the pad columns are zero, the scales are powers of two
  above the row maxima;
* A B^T (both forms of operand), ragged sizes, split K, alpha/beta, rows
  taken from an offset: error within 1e-13 (7 slices) and 1e-15 (8 slices)
  of max|a| max|b| K-scaled, i.e. at the level of a float64 GEMM, on rows of
  plane-wave-like coefficients decaying over six decades;
* A B through the transposed slices of B with B's row scales folded into A:
  error within 1e-13 of sum_k |a_mk| max_n |b_kn| (7 slices).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rows(rng, n, k, decay=12.0, amp=1.0):
    d = np.exp(-np.linspace(0.0, decay, k))
    a = rng.standard_normal((n, k)) * d * amp
    return a


def _exact(a, b):
    return (a.astype(np.longdouble) @ b.T.astype(np.longdouble)).astype(np.float64)


def test_split_rows_rebuilds_the_rows(cuda_device):
    from gradwave_b200.oz import SliceSet
    rng = np.random.default_rng(1)
    a = _rows(rng, 37, 1000, amp=5.0)
    a[3] = 0.0
    st = SliceSet(40, 1000, cuda_device, s=7)
    st.split_rows(torch.from_numpy(a).to(cuda_device), row0=2)
    torch.cuda.synchronize()
    q = st.q.cpu().numpy().astype(np.float64)[:, 2:39]
    sc = st.scale.cpu().numpy()[2:39]
    rebuilt = sum(q[p] * 2.0 ** (-6 - 7 * p) for p in range(7)) * sc[:, None]
    assert np.all(np.abs(rebuilt[:, :1000] - a) <= 2.0 ** -49 * sc[:, None])
    assert np.abs(q).max() <= 64
    assert np.all(q[:, :, 1000:] == 0)
    mx = np.abs(a).max(axis=1)
    nz = mx > 0
    assert np.all(sc[nz] > mx[nz]) and np.all(sc[nz] <= 2 * mx[nz]) and sc[3] == 1.0
    assert np.all(np.log2(sc) == np.round(np.log2(sc)))


@pytest.mark.parametrize("s,M,N,K,bound", [(7, 200, 90, 20011, 1e-13), (8, 130, 70, 4099, 1e-15),
                                           (7, 64, 64, 80000, 1e-13), (6, 257, 129, 777, 1e-11)])
def test_product_nt(cuda_device, s, M, N, K, bound):
    from gradwave_b200.oz import SliceSet, oz_gemm
    rng = np.random.default_rng(M + N + K)
    a = _rows(rng, M, K)
    b = _rows(rng, N, K, amp=300.0)
    sa, sb = SliceSet(M + 3, K, cuda_device, s=s), SliceSet(N, K, cuda_device, s=s)
    sa.split_rows(torch.from_numpy(a).to(cuda_device), row0=3)
    sb.split_rows(torch.from_numpy(b).to(cuda_device))
    c0 = rng.standard_normal((M, N))
    C = torch.from_numpy(c0.copy()).to(cuda_device)
    status = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    oz_gemm(M, N, K, sa, sb, C, alpha=-1.0, beta=0.5, a_row0=3, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref = 0.5 * c0 - _exact(a, b)
    scale = np.abs(a).max(axis=1)[:, None] * np.abs(b).max(axis=1)[None, :] * np.sqrt(K)
    err = np.abs(C.cpu().numpy() - ref) / scale
    assert err.max() < bound


def test_product_nn_and_reuse(cuda_device):
    from gradwave_b200.oz import OzMatmul
    rng = np.random.default_rng(7)
    M, K, N = 130, 700, 3001
    a = rng.standard_normal((M, K))
    b = _rows(rng, K, N)                       # K rows of N, decaying along N
    b *= np.exp(rng.uniform(-8, 2, size=(K, 1)))  # rows of very different size
    om = OzMatmul(cuda_device, s=7)
    out = torch.zeros(M, N, dtype=torch.float64, device=cuda_device)
    A, B = torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device)
    om.nn(A, B, out)
    ref = (a.astype(np.longdouble) @ b.astype(np.longdouble)).astype(np.float64)
    # the error is relative to the row maxima of b (its per-row scales), not
    # to each element: scale[m, n] = sum_k |a_mk| max_n' |b_kn'|
    scale = np.abs(a) @ np.abs(b).max(axis=1, keepdims=True)
    assert (np.abs(out.cpu().numpy() - ref) / scale).max() < 1e-13
    # the same object again with other shapes (slice sets grow), and nt with a == b
    g = torch.zeros(M, M, dtype=torch.float64, device=cuda_device)
    om.nt(A, A, g, same=True)
    refg = _exact(a, a)
    assert np.abs(g.cpu().numpy() - refg).max() < 1e-13 * np.abs(refg).max()

