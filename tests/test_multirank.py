"""Multi-rank bench plumbing on CPU: two `gloo` ranks combine their timed regions the way
`bench.py --gpus N` does under torchrun (maximum time over ranks, sum of leaf cell-updates), split a
batch of trees between them without communicating (each computes its own share), and the reference
arm lets every rank but rank 0 exit without work."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms, upd = bench.reduce_ranks(10.0 + rank, 100.0 * (rank + 1), world)
        out.put((rank, ms, upd))
    finally:
        dist.destroy_process_group()


def test_reduce_ranks_takes_max_time_and_sum_of_updates():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, upd in got:
        assert ms == 11.0 and upd == 300.0


def test_reference_arm_idles_on_nonzero_ranks(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        gpus, steps, warmup, base_level, levels = 2, 1, 3, 3, 1

    bench.bench_reference(A(), rank=1, world=2)
    assert capsys.readouterr().out == ""


def _batch_rank(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dacti_b200 import cases
        from dacti_b200.batch import my_trees, tree_work
        batch = cases.riemann_batch(12, seed=3)
        work = [tree_work(c) for c in batch]
        mine = my_trees(work, rank, world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        out.put((rank, got, work))
    finally:
        dist.destroy_process_group()


def test_batch_split_between_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(2)]
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (_, a, work), (_, b, _) = sorted(res, key=lambda t: t[0])
    assert a == b                                     # both ranks see the same split
    assert sorted(a[0] + a[1]) == list(range(12)) and not set(a[0]) & set(a[1])
    loads = [sum(work[i] for i in part) for part in a]
    assert abs(loads[0] - loads[1]) <= max(work)
