"""Split-precision complex products on the tensor cores (gwb_tc_planes,
gwb_zgemm_tc) against float64 torch products of the same operands.

The planes are checked bit for bit against torch's own round-to-nearest BF16
conversion. The products are checked entry by entry against the bound
|C - AB| <= 4e-5 sum_k |a_ik||b_kj| (the hi/lo split represents each operand
to about 2^-17 relative, the dropped lo*lo term is 2^-18, accumulation is in
FP32), for both forms (A B^H over long K with split-K partial sums, and A B
with B read MN-major), ragged sizes, alpha/beta, complex64 sources and
batches.
"""

import pytest
import torch

from gradwave_b200 import _lib
from gradwave_b200.tc import OP_H, OP_N, PlaneSet, check_status, zgemm_tc

pytestmark = pytest.mark.gpu

TOL = 4e-5


def _rand(shape, dev, seed, dtype=torch.complex128):
    g = torch.Generator(device="cpu").manual_seed(seed)
    re = torch.randn(*shape, generator=g, dtype=torch.float64)
    im = torch.randn(*shape, generator=g, dtype=torch.float64)
    return torch.complex(re, im).to(dtype).to(dev)


def _planes(x, rows_cap=None):
    nk, rows, cols = x.shape
    p = PlaneSet(nk, rows if rows_cap is None else rows_cap, cols, x.device)
    p.write(x, rows)
    return p


def test_planes_split_exactly(cuda_device):
    x = _rand((3, 37, 45), cuda_device, 1)
    p = _planes(x, rows_cap=40)
    for q, part in enumerate((x.real, x.imag)):
        hi = part.float().to(torch.bfloat16)
        lo = (part - hi.double()).float().to(torch.bfloat16)
        assert torch.equal(p.t[:, 2 * q, :37, :45].view(torch.int16), hi.view(torch.int16))
        assert torch.equal(p.t[:, 2 * q + 1, :37, :45].view(torch.int16), lo.view(torch.int16))
    assert int(p.t[:, :, :, 45:].abs().max()) == 0  # padded columns zero
    rel = ((p.t[:, 0].double() + p.t[:, 1].double())[:, :37, :45] - x.real).abs().max() / x.real.abs().max()
    assert float(rel) < 2 ** -15


def _check(C, ref, bound):
    err = (C - ref).abs()
    assert torch.isfinite(C).all()
    worst = float((err / bound).max())
    assert worst < TOL, f"error / (|A||B|) = {worst:.3e}"


@pytest.mark.parametrize("nk,M,N,K", [(10, 24, 96, 4640), (1, 130, 257, 1001), (2, 1, 1, 1), (1, 300, 600, 20000),
                                      (3, 129, 128, 33)])
def test_a_bh_matches_float64(cuda_device, nk, M, N, K):
    A = _rand((nk, M, K), cuda_device, 2)
    B = _rand((nk, N, K), cuda_device, 3)
    C = torch.zeros(nk, M, N, dtype=torch.complex128, device=cuda_device)
    zgemm_tc(OP_H, M, N, K, _planes(A), _planes(B), C, N, M * N)
    torch.cuda.synchronize()
    check_status(cuda_device)
    ref = A @ B.conj().transpose(-1, -2)
    _check(C, ref, A.abs() @ B.abs().transpose(-1, -2))


@pytest.mark.parametrize("nk,M,N,K", [(10, 24, 4640, 96), (1, 130, 1001, 257), (2, 1, 1, 1), (1, 200, 9000, 640)])
def test_a_b_update_matches_float64(cuda_device, nk, M, N, K):
    # D -= C V: the basis update of the projection pass (alpha -1, beta 1)
    A = _rand((nk, M, K), cuda_device, 4)
    B = _rand((nk, K, N), cuda_device, 5)
    D0 = _rand((nk, M, N), cuda_device, 6)
    D = D0.clone()
    zgemm_tc(OP_N, M, N, K, _planes(A), _planes(B), D, N, M * N, alpha=-1.0, beta=1.0)
    torch.cuda.synchronize()
    check_status(cuda_device)
    _check(D, D0 - A @ B, A.abs() @ B.abs())


def test_strided_output_complex64_source_and_row_offsets(cuda_device):
    # A from complex64 storage; B planes written in two row blocks; C a
    # sub-block of a larger strided buffer with complex alpha and beta
    nk, M, N, K = 2, 40, 70, 300
    A = _rand((nk, M, K), cuda_device, 7, torch.complex64)
    B = _rand((nk, N, K), cuda_device, 8)
    pb = PlaneSet(nk, 96, K, cuda_device)
    pb.write(B[:, :50].contiguous(), 50, row0=0)
    pb.write(B[:, 50:].contiguous(), N - 50, row0=50)
    big = _rand((nk, M + 5, N + 9), cuda_device, 9)
    ref = 0.5j * (A.to(torch.complex128) @ B.conj().transpose(-1, -2)) + (1 - 2j) * big[:, 2:2 + M, 3:3 + N]
    C = big.clone()
    zgemm_tc(OP_H, M, N, K, _planes(A), pb, C, N + 9, (M + 5) * (N + 9), alpha=0.5j, beta=1 - 2j,
             c_offset=2 * (N + 9) + 3)
    torch.cuda.synchronize()
    check_status(cuda_device)
    bound = 0.5 * A.abs().double() @ B.abs().transpose(-1, -2) + 1e-30
    _check(C[:, 2:2 + M, 3:3 + N], ref, bound)
    # untouched outside the block
    mask = torch.ones_like(big, dtype=torch.bool)
    mask[:, 2:2 + M, 3:3 + N] = False
    assert torch.equal(C[mask], big[mask])


def test_bad_arguments_are_rejected(cuda_device):
    p = PlaneSet(1, 8, 8, cuda_device)
    C = torch.zeros(1, 8, 8, dtype=torch.complex128, device=cuda_device)
    with pytest.raises(_lib.GwbError):
        zgemm_tc(OP_H, 8, 8, 16, p, p, C, 8, 64)  # K beyond the planes' columns
    with pytest.raises(_lib.GwbError):
        zgemm_tc(1, 8, 8, 8, p, p, C, 8, 64)  # transpose without conjugation is not a form
