"""The multi-rank host logic of bench.py on the CPU (world_size 2, gloo, 127.0.0.1): the element loop
has no data-path collective (every rank runs its own replica), so a run of N ranks reports the
largest rank time and N times the per-rank work; the reference arm prints from rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [3.5, 7.25][rank]                         # rank 1 is the slow one
        ms = bench.max_over_ranks(local_ms, world, "cpu")
        rate = bench.whole_job_rate(1000, world, ms * 1e-3)
        with open(os.path.join(out, f"r{rank}.json"), "w") as f:
            json.dump({"ms": ms, "rate": rate}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_on_two_gloo_ranks(tmp_path):
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    for r in range(2):
        d = json.load(open(tmp_path / f"r{r}.json"))
        assert d["ms"] == 7.25                                 # every rank sees the slowest rank's time
        assert abs(d["rate"] - 2 * 1000 / 7.25e-3) < 1e-6     # both ranks' work over that time


def test_reference_arm_prints_from_rank_zero_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "3", "--nx", "8"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
