"""The multi-rank side of bench.py on CPU: two gloo ranks (one process
each, rendezvous on 127.0.0.1) reduce their timings by max and their work
by sum, the way `bench.py --gpus N` does over NCCL; each rank's shard is
its own seeded workload; the reference arm does its work on rank 0 only."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # per-rank shard: cells and pairs differ between ranks
        queries, buf, offs, lens = bench.workload(rank, n_targets=200)
        cells = float(sum(len(x) for x in queries)) * float(lens.sum())
        t, w = bench.over_ranks(world, [10.0 + rank, 3.0 - rank], [cells, len(queries) * len(lens)], "cpu")
        q.put((rank, t, w, cells, int(buf[: 64].astype("int64").sum())))
    finally:
        dist.destroy_process_group()


def test_over_ranks_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    got = [q.get(timeout=240) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    cells = [g[3] for g in got]
    for rank, t, w, _, _ in got:
        assert t == [11.0, 3.0]                          # max over ranks, on every rank
        assert w == [cells[0] + cells[1], 2 * 5 * 200]   # sum over ranks
    assert cells[0] != cells[1]                          # each rank has its own shard
    assert got[0][4] != got[1][4]


def test_over_ranks_single_process_is_identity():
    assert bench.over_ranks(1, [2.5, 4], [7, 8], "cpu") == ([2.5, 4.0], [7.0, 8.0])


def test_reference_arm_other_ranks_do_no_work(capsys):
    class A:
        n_targets, cpu_seconds, gpus, steps, warmup = 10, 1.0, 2, 1, 1
    bench.run_reference(A(), 1, 2)
    assert capsys.readouterr().out == ""
