"""The multi-process path of bench.py, on the CPU (gloo, world size 2,
rendezvous on 127.0.0.1).

* Ranks combine their step times by maximum (one all-reduce that every rank
  takes) and the job rate counts every rank's units over the slowest rank's
  time: the contract's `value` for N replicas.
* The reference arm launched by torch.distributed.run with two ranks prints
  exactly one JSON line, from rank 0, and every rank exits 0.
"""
import datetime
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took 1 + r ms for one stage and 5 - r ms for another
        vals = bench.max_over_ranks([1.0 + rank, 5.0 - rank], dist, "cpu")
        dist.barrier()
        out.put((rank, vals))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: [2.0, 5.0], 1: [2.0, 5.0]}
    sys.path.insert(0, ROOT)
    import bench
    # 1,000 units on each of 2 ranks, slowest rank 2 ms
    assert bench.job_rate(1000, 2, 2.0) == 1_000_000.0
    assert bench.max_over_ranks([3.0, 4.0], None, "cpu") == [3.0, 4.0]


def test_reference_arm_under_torchrun_prints_one_line_from_rank_0():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-seconds", "1", "--workload", "small"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"
    # the arm processes whole bounces: its step time covers every query
    assert d["ms_per_step"] > 0 and abs(d["value"] * d["ms_per_step"] * 1e-3 - 65536) < 1.0
