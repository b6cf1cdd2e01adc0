"""k-point sharding of the band solve across ranks (one process per GPU).

Each k-point's band solve is an independent eigenproblem, so N ranks solve N
disjoint, contiguous k-ranges with no communication inside the solve, and the
eigenvalues and residual norms are gathered once at the end, in rank order, to
the global k order. This is the reference's k-point data parallelism
(gradwave ``distributed.py:155-164`` ``shard_range``, ``:167-224``
``shard_system``, ``:440-452`` ``gather_cat``) with the process group on NCCL
for CUDA tensors and gloo for CPU ones.

``shard_range`` keeps the reference's split (as even as possible by count;
the first ``n % world_size`` ranks get one more). ``shard_range_weighted``
balances contiguous ranges by a per-k cost (npw_k: the apply, the subspace
products and the orthonormalisation all scale with it).
"""

from __future__ import annotations

from typing import Callable, Sequence

import numpy as np
import torch


def shard_range(n: int, rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous ``[start, end)`` of ``n`` k-points for ``rank``
    (gradwave ``distributed.py:155-164``)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside a world of {world_size}")
    base, rem = divmod(n, world_size)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def shard_range_weighted(cost: Sequence[float], rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous ``[start, end)`` whose summed cost is closest to an equal
    share: rank r ends at the first k where the running cost reaches
    (r+1)/world_size of the total. Every rank gets at least one k-point
    (raises when there are fewer k-points than ranks)."""
    c = np.asarray(cost, dtype=np.float64)
    n = int(c.shape[0])
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside a world of {world_size}")
    if n < world_size:
        raise ValueError(f"{n} k-points cannot give each of {world_size} ranks one")
    cum = np.cumsum(c)
    bounds = [0]
    for r in range(1, world_size):
        target = cum[-1] * r / world_size
        b = int(np.searchsorted(cum, target, side="left")) + 1
        # keep at least one k per rank on both sides
        b = max(b, bounds[-1] + 1)
        b = min(b, n - (world_size - r))
        bounds.append(b)
    bounds.append(n)
    return bounds[rank], bounds[rank + 1]


def slice_batched(bk, start: int, end: int):
    """The k-range ``[start, end)`` of a ``BatchedK`` (per-k tables sliced,
    geometry-global fields kept; gradwave ``distributed.py:167-224``)."""
    from .basis import BatchedK
    sl = slice(start, end)
    return BatchedK(bk.npw[sl], bk.mask[sl], bk.flat_idx[sl], bk.kpg[sl], bk.t[sl],
                    bk.proj_phase_free[sl], bk.proj_atom_index, bk.dij_full)


def gather_cat(local: torch.Tensor, world_size: int, group=None, dim: int = 0) -> torch.Tensor:
    """All-gather ``local`` from every rank (shapes may differ along ``dim``)
    and concatenate in rank order (gradwave ``distributed.py:440-452``).
    Sizes go first, then zero-padded payloads, so one code path serves gloo
    (CPU tensors) and NCCL (CUDA tensors)."""
    import torch.distributed as dist
    if world_size == 1:
        return local
    local = local.contiguous()
    n_local = torch.tensor([local.shape[dim]], dtype=torch.int64, device=local.device)
    sizes = [torch.zeros_like(n_local) for _ in range(world_size)]
    dist.all_gather(sizes, n_local, group=group)
    sizes = [int(s.item()) for s in sizes]
    n_max = max(sizes)
    pad_shape = list(local.shape)
    pad_shape[dim] = n_max
    padded = torch.zeros(pad_shape, dtype=local.dtype, device=local.device)
    padded.narrow(dim, 0, local.shape[dim]).copy_(local)
    parts = [torch.empty_like(padded) for _ in range(world_size)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p.narrow(dim, 0, s) for p, s in zip(parts, sizes)], dim=dim)


def solve_sharded(solve: Callable[[int, int], tuple[torch.Tensor, torch.Tensor]], nk: int, rank: int,
                  world_size: int, group=None, cost: Sequence[float] | None = None):
    """Run ``solve(start, end) -> (eigenvalues (n_loc, nb), residual_norms
    (n_loc, nb))`` on this rank's k-range and return the global
    ``(eigenvalues, residual_norms, (start, end))``, gathered in k order on
    every rank. ``cost`` (per k) selects the weighted split."""
    start, end = (shard_range_weighted(cost, rank, world_size) if cost is not None
                  else shard_range(nk, rank, world_size))
    if start == end:
        raise ValueError(f"rank {rank} would get zero of {nk} k-points (world size {world_size})")
    eig, rn = solve(start, end)
    return gather_cat(eig, world_size, group), gather_cat(rn, world_size, group), (start, end)
