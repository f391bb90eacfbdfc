"""The bench's multi-rank logic on CPU with the gloo backend, world size 2 (no GPU).

bench.py runs one replica (or its share of the 48-run sweep) per rank with no collective
in the step; the only collectives are the MAX reductions of the device times
(`max_over_ranks`) and the barriers around the timed region.  The sweep split
(`partition_by_cost`) is computed by every rank without communication; here the ranks
exchange their shares to check that together they cover every run once and balance the
cost.  The reference arm prints from rank 0 only.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "sma-dft_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import smadft
        runs = bench.sweep_params(smadft)
        costs = [n ** 3 * (6 if model == smadft.NOADV else 32) for model, n, _, _ in runs]
        mine = bench.partition_by_cost(costs, world, rank)
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        mx = bench.max_over_ranks(torch, dist, [1.5 + rank, 10.0 - rank], "cpu")

        class Args:
            gpus, steps = world, 3
        ref_rc = bench.run_reference_arm(Args, rank, world) if rank != 0 else 0
        dist.barrier()
        q.put((rank, shares, costs, mx, ref_rc))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_the_sweep_and_reduce_times():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {r: (shares, costs, mx, rc) for r, shares, costs, mx, rc in out}
    shares, costs = by_rank[0][0], by_rank[0][1]
    assert by_rank[1][0] == shares                      # every rank computes the same split
    union = sorted(i for s in shares for i in s)
    assert union == list(range(len(costs)))             # each run exactly once
    loads = [sum(costs[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(costs)        # greedy balance bound
    for r in range(world):
        assert by_rank[r][2] == [2.5, 10.0]             # element-wise maximum on every rank
    assert by_rank[1][3] == 0                           # the reference arm: rank 1 exits quietly
