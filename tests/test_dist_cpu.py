"""bench.py's multi-GPU arithmetic (independent replicas, max over ranks) on
CPU ranks over gloo, world_size 2 -- no GPU involved."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = 10.0 * (rank + 1)                 # rank 1 is the slow one
    mx = bench.max_over_ranks(ms, world)
    bench.barrier(world)
    rate = bench.whole_job_rate(1000, world, mx, steps=5)
    out.put((rank, mx, rate))
    dist.destroy_process_group()


def test_replicas_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]          # every rank sees the slowest time
    # 2 ranks x 1000 elements per step, 5 steps in 20 ms -> 2000 / 4 ms
    assert res[0][2] == pytest.approx(2 * 1000 / (20.0 / 5 / 1e3))


def test_reference_arm_only_rank0_prints(capsys, monkeypatch):
    sys.path.insert(0, REPO)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup = 1, 3
    bench.run_reference(A())
    assert capsys.readouterr().out == ""
