"""bench.py's multi-rank path on CPU: two gloo ranks on 127.0.0.1 (replicas; only the timing and counts are
reduced), and the reference arm under torchrun (rank 0 prints the one JSON line, the others exit 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, local, ws = bench.dist_setup()
    assert (r, ws) == (rank, 2)
    # rank 0: 1000 pairs in 2.0 s of device time; rank 1: 3000 pairs in 4.0 s -> 4000 pairs / 4 s
    value, tot_ms = bench.aggregate([2000.0, 4000.0][rank], [1000.0, 3000.0][rank], ws)
    bench.barrier(ws)
    with open(os.path.join(out, f"r{rank}.json"), "w") as f:
        json.dump({"value": value, "ms": tot_ms}, f)
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_max_time_and_total_units(tmp_path):
    mp.start_processes(_rank, args=(free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    got = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert got[0] == got[1] == {"value": 1000.0, "ms": 4000.0}


def test_reference_arm_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(free_port()), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--seeds", "20000", "--cpu-sample-s", "0.5"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["higher_is_better"] is True
