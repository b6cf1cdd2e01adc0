"""Host logic of the Gamma real path on seeded random cells (CPU): the
half-sphere maps of ``build_gamma_basis`` (gradwave ``core/gamma.py:70-147``),
the real embedding and its metric (``core/gamma.py:215-250``), and the rule
that a sphere not closed under G -> -G is refused."""

import numpy as np
import pytest
import torch

from gradwave_b200 import gamma as G
from gradwave_b200.basis import build_fft_grid, build_gsphere


def _cells(n=4, seed=7):
    rng = np.random.default_rng(seed)
    for _ in range(n):
        cell = np.diag(rng.uniform(2.5, 4.5, 3)) + rng.uniform(-0.4, 0.4, (3, 3)) * (1 - np.eye(3))
        yield cell, float(rng.uniform(150.0, 300.0))


@pytest.mark.parametrize("cell,ecut", list(_cells()))
def test_half_sphere_maps(cell, ecut):
    grid = build_fft_grid(cell, ecut)
    sph = build_gsphere(grid, ecut, (0.0, 0.0, 0.0))
    gb = G.build_gamma_basis(sph, grid.shape)
    m = sph.miller
    rep = gb.rep_full_idx.numpy()
    src = gb.src_half.numpy()
    conj = gb.conj_full.numpy()
    partner = gb.partner_rep.numpy()
    assert gb.npw == 2 * gb.nhalf - 1 and np.all(m[rep[0]] == 0)
    # every full-sphere point maps to the slot of itself or of -G
    assert np.array_equal(src[rep], np.arange(gb.nhalf))
    for i in range(gb.npw):
        r = rep[src[i]]
        if conj[i]:
            assert i != r and np.all(m[i] == -m[r])
        else:
            assert i == r
    # the partner of each representative is its -G point
    assert np.array_equal(m[partner], -m[rep])
    # representatives: G = 0, then (m3, m2, m1) lexicographically positive
    for mm in m[rep[1:]]:
        assert mm[2] > 0 or (mm[2] == 0 and (mm[1] > 0 or (mm[1] == 0 and mm[0] > 0)))
    # the half-sphere kinetic energies are those of the representatives
    assert np.allclose(gb.t_half.numpy(), gb.t_full.numpy()[rep])


@pytest.mark.parametrize("cell,ecut", list(_cells(2, seed=3)))
def test_embedding_round_trip_and_metric(cell, ecut):
    grid = build_fft_grid(cell, ecut)
    sph = build_gsphere(grid, ecut, (0.0, 0.0, 0.0))
    gb = G.build_gamma_basis(sph, grid.shape)
    g = torch.Generator().manual_seed(1)
    nb = 5
    ch = torch.complex(torch.randn(nb, gb.nhalf, generator=g, dtype=torch.float64),
                       torch.randn(nb, gb.nhalf, generator=g, dtype=torch.float64))
    ch[:, 0] = ch[:, 0].real.to(ch.dtype)   # a real state has a real G = 0 coefficient
    phi = G.embed_real(gb, ch)
    assert phi.shape == (nb, 2 * gb.nhalf - 1)
    assert torch.allclose(G.unembed_real(gb, phi), ch, rtol=0, atol=1e-15)
    # plain dot products of the embedding = the full-sphere inner products
    full = G.half_to_full(gb, ch)
    gram_full = (full.conj() @ full.T).real
    assert torch.allclose(phi @ phi.T, gram_full, rtol=1e-13, atol=1e-12)
    assert torch.allclose(G.metric_inner(gb, ch, ch), gram_full, rtol=1e-13, atol=1e-12)
    # a full Hermitian-symmetric row goes back losslessly
    assert torch.allclose(G.full_to_half(gb, full), ch, rtol=0, atol=0)
    # the kinetic diagonal of the embedding repeats each slot for Re and Im
    t = G.kinetic_phi(gb)
    assert torch.equal(t[1::2], gb.t_half[1:]) and torch.equal(t[2::2], gb.t_half[1:])


def test_sphere_off_gamma_is_refused():
    cell = np.diag([3.0, 3.3, 3.7])
    grid = build_fft_grid(cell, 200.0)
    sph = build_gsphere(grid, 200.0, (0.25, 0.0, 0.0))
    with pytest.raises(ValueError):
        G.build_gamma_basis(sph, grid.shape)
