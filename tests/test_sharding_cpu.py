"""k-point sharding across ranks, on CPU with gloo (world size 2).

The split keeps the reference's contract (gradwave ``distributed.py:155-164``:
contiguous, as even as possible, rank-order concatenation restores the global
k order); the weighted split balances per-k cost. The two-rank test solves
each rank's k-range of the synthetic operator golden with the float64 oracle
and checks the gathered eigenvalues against the reference's own.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from gradwave_b200.sharding import gather_cat, shard_range, shard_range_weighted, solve_sharded


def test_shard_range_matches_reference_split():
    for n in (1, 4, 10, 36):
        for ws in range(1, min(n, 8) + 1):
            ranges = [shard_range(n, r, ws) for r in range(ws)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [e - s for s, e in ranges]
            assert max(sizes) - min(sizes) <= 1
            assert sizes == sorted(sizes, reverse=True)  # first n % ws ranks get one more
    with pytest.raises(ValueError):
        shard_range(4, 4, 4)


def test_weighted_split_balances_cost():
    rng = np.random.default_rng(0)
    cost = rng.integers(1000, 1100, size=10).astype(float)
    cost[3] = 9000.0  # one heavy k
    for ws in (2, 3, 4):
        ranges = [shard_range_weighted(cost, r, ws) for r in range(ws)]
        assert ranges[0][0] == 0 and ranges[-1][1] == len(cost)
        assert all(a[1] == b[0] and a[1] > a[0] for a, b in zip(ranges, ranges[1:]))
        loads = [cost[s:e].sum() for s, e in ranges]
        # contiguous ranges: no rank exceeds the fair share by more than one k's cost
        assert max(loads) <= cost.sum() / ws + cost.max()
    with pytest.raises(ValueError):
        shard_range_weighted(cost[:2], 0, 3)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, ws, port, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle.davidson import davidson_batched
        from tests.conftest import load_golden
        g = load_golden("synthetic")
        h, x0, t = g["h"], g["x0"], g["t"]

        def solve(start, end):
            hk = h[start:end]
            res = davidson_batched(lambda c: np.einsum("kij,kbj->kbi", hk, c), x0[start:end], t[start:end],
                                   np.ones(t[start:end].shape, bool), tol=1e-9, max_iter=100)
            return torch.from_numpy(res.eigenvalues), torch.from_numpy(res.residual_norms)

        eig, rn, rng_ = solve_sharded(solve, h.shape[0], rank, ws, cost=[1.0, 1.0, 3.0, 1.0])
        # a ragged gather: rank r contributes r + 1 rows
        rag = gather_cat(torch.full((rank + 1, 2), float(rank)), ws)
        out_q.put((rank, eig.numpy(), rn.numpy(), rng_, rag.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_k_sharded_solve_matches_reference():
    from tests.conftest import load_golden
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = load_golden("synthetic")
    ranges = {}
    for rank, eig, rn, rng_, rag in results:
        ranges[rank] = rng_
        assert eig.shape == g["eigenvalues"].shape
        assert np.abs(eig - g["eigenvalues"]).max() < 1e-10
        assert np.abs(eig - g["exact"]).max() < 1e-9
        assert rn.max() < 1e-9
        assert rag.tolist() == [[0.0, 0.0], [1.0, 1.0], [1.0, 1.0]]
    # weighted split of cost [1, 1, 3, 1] (running cost 1, 2, 5, 6; half is 3):
    # rank 0 takes k 0..2, rank 1 takes k 3
    assert ranges[0] == (0, 3) and ranges[1] == (3, 4)
