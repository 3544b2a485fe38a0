"""bench.py's multi-rank path on CPU: two gloo ranks on 127.0.0.1 (replicas; only the timing and counts are
reduced), the reference arm under torchrun (rank 0 prints the one JSON line, the others exit 0), and the exchange of
the sharded cluster (each rank's forest gathered in rank order)."""
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
    """The reference arm under torchrun: rank 0 alone runs the reference engine's driver and prints one line (here,
    without a GPU, the line says the driver is unavailable); rank 1 exits cleanly."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(free_port()), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--seeds", "20000"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" not in d:
        assert d["n_gpus"] == 2 and d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference" and d["higher_is_better"] is True


def _forest(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "postgis-cuda_b200"))
    import numpy as np
    import torch.distributed as dist
    from gsj import dist as gd
    dist.init_process_group("gloo", rank=rank, world_size=2)
    rng = np.random.default_rng(rank)
    n = 1000
    root = np.arange(n, dtype=np.uint32)   # a forest: each i points at a smaller index of its component (a root)
    for i in rng.choice(n, 300, replace=False):
        root[i] = rng.integers(0, i + 1)
    for i in range(n):                     # flattened to component minima, as gsj_cluster returns them
        root[i] = root[root[i]]
    parts = gd.gather_forests(root)
    np.save(os.path.join(out, f"f{rank}.npy"), np.stack(parts))
    dist.destroy_process_group()


def test_cluster_forests_gathered_in_rank_order(tmp_path):
    """The one exchange of the sharded cluster on two gloo ranks: every rank receives every rank's forest, in rank
    order; joining them (union-find restated here) gives the components of all the ranks' edges."""
    import numpy as np
    mp.start_processes(_forest, args=(free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    a, b = np.load(tmp_path / "f0.npy"), np.load(tmp_path / "f1.npy")
    assert np.array_equal(a, b) and a.shape == (2, 1000)
    par = list(range(1000))

    def find(x):
        while par[x] != x:
            par[x] = par[par[x]]
            x = par[x]
        return x
    for forest in a:
        for i, r in enumerate(forest):
            x, y = find(i), find(int(r))
            if x != y:
                par[max(x, y)] = min(x, y)
    merged = [find(i) for i in range(1000)]
    # independently: connected components of the edges (i, root_f[i]) of both forests by breadth-first search,
    # labelled by their smallest member
    adj = [[] for _ in range(1000)]
    for forest in a:
        for i, r in enumerate(forest):
            adj[i].append(int(r)); adj[int(r)].append(i)
    comp = [-1] * 1000
    for s in range(1000):
        if comp[s] < 0:
            todo, members = [s], []
            comp[s] = s
            while todo:
                x = todo.pop()
                members.append(x)
                for y in adj[x]:
                    if comp[y] < 0:
                        comp[y] = s; todo.append(y)
            m = min(members)
            for x in members:
                comp[x] = m
    assert merged == comp
    assert len(set(merged)) < min(len(set(a[0].tolist())), len(set(a[1].tolist())))
