"""bench.py's multi-rank logic on the CPU (gloo, world size 2).

Each rank of `bench.py --gpus N` advances its own lattice; the job's time is
the slowest rank's (max over ranks, taken by an all-reduce) and the value is
all ranks' site-updates over that time. These tests run the same helpers in
two gloo processes on 127.0.0.1, with ranks that report different times,
and check the reference arm's rule that only rank 0 does work.
"""
import multiprocessing as mp
import os
import socket

import bench


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import bench as b
    r, w, _ = b.dist_setup(world, backend="gloo", timeout_s=60)
    ms = 10.0 + 5.0 * r                # rank 1 is the slow one
    b.barrier(w)
    m = b.max_over_ranks(ms, w)
    v = b.whole_job_rate(4096 * 4096, w, 20, m)
    b.barrier(w)
    q.put((r, w, m, v))
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    for _, _, m, v in out:
        assert m == 15.0
        assert abs(v - 4096 * 4096 * 2 * 20 / 0.015) < 1e-6 * v


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.whole_job_rate(100, 1, 10, 1000.0) == 1000.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        model, size, steps, warmup, gpus = "lyotropic", 64, 1, 1, 2
    assert bench.run_reference(A()) == 0
    assert capsys.readouterr().out == ""
