"""The N > 1 host path of bench.py: one replica per rank, no data-path
collective, a barrier and the max over ranks of the timed region.  Run as two
gloo ranks on the CPU (the GPU pool gives one GPU per call)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    g = bench.Group(world, rank, backend="gloo", timeout_s=60)
    g.barrier()
    slowest = g.max(10.0 + rank)          # per-rank timed region, ms
    value = bench.whole_job_mlups(1_000_000, 100, world, slowest / 1e3)
    g.barrier()
    g.close()
    q.put((rank, slowest, value))


def test_two_replicas_reduce_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]
    # 2 ranks x 1e6 cells x 100 steps over the slower rank's 11 ms
    assert out[0][2] == pytest.approx(2 * 1e6 * 100 / 0.011 / 1e6)


def test_reference_arm_other_ranks_exit(monkeypatch, capsys):
    """Under torchrun only rank 0 times the reference; others return 0."""
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = type("A", (), dict(steps=3, warmup=3, cpu_steps=1, config="c1", gpus=2))()
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""
