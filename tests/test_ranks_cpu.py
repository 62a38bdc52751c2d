"""The N-rank plumbing of bench.py on CPU: two gloo ranks run the same calls
the GPU replicas make over NCCL (barrier, max of the elapsed time, close), and
the reference arm returns at once on every rank but 0."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch

    import bench

    r = bench.Ranks("gloo", torch.device("cpu"))
    assert (r.world, r.rank, r.root) == (world, rank, rank == 0)
    r.barrier()
    ms = 10.0 + 5.0 * rank  # this rank's elapsed time per step
    m = r.max(ms)
    r.barrier()
    r.close()
    q.put((rank, m, bench.job_rate(world, m)))


@pytest.mark.parametrize("world", [2])
def test_ranks_reduce_max_elapsed_time_over_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    slowest = 10.0 + 5.0 * (world - 1)
    for rank, m, rate in got:
        assert m == slowest  # every rank sees the slowest rank's time
        assert rate == pytest.approx(world * 1000.0 / slowest)  # the whole job's steps/s


def test_single_rank_needs_no_process_group(monkeypatch):
    import torch

    import bench

    for k in ("RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    r = bench.Ranks("gloo", torch.device("cpu"))
    assert r.dist is None and r.root and r.max(3.5) == 3.5
    r.barrier()
    r.close()


def test_reference_arm_runs_on_rank_0_only(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.run_reference(type("A", (), {"res": 32, "ppc": 8, "steps": 1, "warmup": 0, "gpus": 2})()) == 0
    assert capsys.readouterr().out == ""  # no line, no work
