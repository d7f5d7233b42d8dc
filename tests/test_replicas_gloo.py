"""The N > 1 path on CPU: two gloo ranks on 127.0.0.1.

bench.py runs N independent replicas (no data-path collective); the only
collectives are a barrier and a max over ranks of the timed duration.  These
tests drive that plumbing with real processes, without a GPU.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from self_b200 import replicas as R
    r, w, _ = R.init("gloo", timeout_s=60)
    assert (r, w) == (rank, world)
    R.barrier()
    t_max = R.max_over_ranks(10.0 + rank)  # rank 1 is the slowest
    total = R.sum_over_ranks(rank + 1)
    share = R.deal(7, rank, world)
    shares = [None] * world
    import torch.distributed as dist
    dist.all_gather_object(shares, share)
    out[rank] = (t_max, total, shares, R.aggregate_rate(100.0, w, t_max))
    R.finalize()


def test_two_gloo_ranks_max_sum_and_deal():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        t_max, total, shares, rate = res[r]
        assert t_max == 11.0 and total == 3.0
        assert sorted(i for s in shares for i in s) == list(range(7))  # every instance on exactly one rank
        assert rate == pytest.approx(200.0 / 11.0)


def test_deal_and_rate_single_process():
    from self_b200 import replicas as R
    assert R.deal(5, 0, 1) == [0, 1, 2, 3, 4]
    assert R.deal(5, 2, 3) == [2]
    with pytest.raises(ValueError):
        R.deal(5, 3, 3)
    assert R.max_over_ranks(4.5) == 4.5  # no process group: identity
    with pytest.raises(ValueError):
        R.aggregate_rate(1.0, 1, 0.0)


def test_bench_reference_arm_under_torchrun_two_ranks():
    """rank 0 alone runs the CPU reference arm and prints one JSON line; rank 1 exits 0 without work."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
