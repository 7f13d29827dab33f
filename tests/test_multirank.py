"""The N > 1 path of bench.py on CPU: two ranks over gloo (no GPU).

Each rank times its own tile; the whole-job value uses the slowest rank's time
(max over ranks with the same collective order on every rank), and under torchrun
the reference arm runs on rank 0 alone while the other ranks exit 0 silently.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    assert bench.rank_env() == (rank, world, rank)
    # rank r "took" 10 (r + 1) ms for 4 steps of its tile
    total = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
    again = bench.max_over_ranks(-1.0 * rank, dist, "cpu")
    dist.barrier()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"total": total, "again": again,
                   "value": bench.job_throughput(world, 4, total)}, f)
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r = [json.load(open(tmp_path / f"r{i}.json")) for i in range(2)]
    assert r[0] == r[1]
    assert r[0]["total"] == 20.0 and r[0]["again"] == 0.0
    assert r[0]["value"] == pytest.approx(2 * 4 / 0.020)


def test_single_process_helpers():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.job_throughput(1, 20, 100.0) == pytest.approx(200.0)


def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched like the multi-GPU runs: rank 0 prints one
    JSON line, rank 1 does no work and exits 0 (small size so the CPU oracle is quick)."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--size", "128",
           "--kernels", "2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
