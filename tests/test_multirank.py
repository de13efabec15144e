"""The replica path of bench.py on two CPU ranks (gloo): timings reduce to the
slowest rank, throughputs to the slowest rank times the rank count, and the
whole-job rate counts every rank's units."""
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        times = bench.reduce_over_ranks([10.0 + rank, 5.0 * (rank + 1)], device="cpu")
        rates = bench.reduce_over_ranks([100.0 - rank], op="min", device="cpu")
        rate = bench.replica_rate(1000, 4, times[0], world)
        dist.barrier()
        out.put((rank, times, rates, rate))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, times, rates, rate in got:
        assert times == [11.0, 10.0]          # max over ranks, element-wise
        assert rates == [99.0]                # min over ranks
        assert rate == pytest.approx(2 * 1000 * 4 / (11.0 / 1e3))


def test_single_process_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks([3.0, 4.0], device="cpu") == [3.0, 4.0]
    assert bench.replica_rate(10, 2, 1000.0, 1) == pytest.approx(20.0)


def _bench(env_extra, *args):
    import subprocess
    import sys
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_runs_on_rank_zero_only():
    import json
    args = ("--impl", "reference", "--workload", "p1", "--steps", "1", "--warmup", "1")
    other = _bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, *args)
    assert other.returncode == 0 and other.stdout.strip() == ""
    first = _bench({"RANK": "0", "WORLD_SIZE": "2", "LOCAL_RANK": "0"}, *args)
    assert first.returncode == 0, first.stderr[-2000:]
    lines = [ln for ln in first.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["value"] > 0 and out["unit"] == "nnz/s"
    assert out["cpu_baseline"]["value"] == out["value"] and out["cpu_baseline"]["kind"] in ("port", "reference")
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["e2e"]["d2h_bytes_per_step"] == 0
