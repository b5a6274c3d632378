"""Multi-rank host logic of bench.py on CPU, with gloo and world size 2: the
max-over-ranks time reduction and the whole-job throughput of the replica runs, and
the reference arm's rank-0-only behaviour under torchrun.  The data path itself has
no collective (every rank solves its own configuration), so this is all the N > 1
path adds."""
import os
import socket
from datetime import timedelta

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench

        total_ms = 1000.0 + 250.0 * rank  # the slower rank sets the job time
        m = bench.max_over_ranks(total_ms, world)
        q.put((rank, m, bench.sec_per_rhs(m, 3, 12, world)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_throughput_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=120) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.terminate()
    assert all(p.exitcode == 0 for p in procs)
    for rank, m, spr in res:
        assert m == 1250.0
        assert spr == pytest.approx(1.25 / (3 * 12 * 2))


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.sec_per_rhs(1200.0, 3, 12, 1) == pytest.approx(1.2 / 36)


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.main(["--impl", "reference"]) == 0
    assert capsys.readouterr().out == ""
