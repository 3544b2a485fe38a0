"""The reference engine's own file driver, run as a checker and as the timed reference arm (GPU box).

Test and measurement infrastructure, not product. ``oracle/_ref/harness`` is landstats-us/postgis-cuda
engine/harness.cu, unmodified, compiled for sm_100a by ``oracle/build_ref.sh`` (git-ignored; it travels to the GPU box
with the tree). This module runs it on .gset/.pset files written by ``gsj.gen`` and reads back what it prints and
writes:

- the stats line (engine/harness.cu:75-77 for joins, :121-123 buffer joins, :148-149 points x polygons buffer joins,
  :174-176 points in polygons, :200-202 clusters): phase times (upload, bvh, traverse, refine, compact, d2h) and
  counts (cand, gpu_hits, rows, clusters);
- the ``--out`` CSV (engine/harness.cu:78-86, :124-127, :150-153, :177-184, :203): rows ``landrecid,"sid",t,area``
  with ``%.17g`` areas, ``landrecid,"sid",t,relate`` with the 9-character DE-9IM matrix, or ``id,cluster`` with dense
  cluster numbers in order of first row.

Self-joins in the harness write every unordered pair in both orders (the mirrored row carries the transposed matrix)
and the diagonal once (engine/harness.cu:54-65).
"""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "harness")

_NUM = re.compile(r"\b(upload|bvh|traverse|refine|compact|d2h|union-find)=([\d.]+)ms")
_CNT = re.compile(r"\b(cand|gpu_hits|rows|clusters|pairs|heavy|edges)=(\d+)")
_CELL = np.zeros(256, np.uint32)
_CELL[ord("F")], _CELL[ord("0")], _CELL[ord("1")], _CELL[ord("2")] = 0, 1, 2, 3


def available() -> bool:
    return os.access(HARNESS, os.X_OK)


def run(args, reps=1, out_csv=None, timeout=1800, env=None):
    """Runs the harness; returns {'ms': {phase: ms}, 'count': {name: n}, 'stdout': text} of its last stats line."""
    cmd = [HARNESS, *map(str, args), "--reps", str(reps)] + (["--out", out_csv] if out_csv else [])
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=timeout,
                       env=None if env is None else {**os.environ, **env})
    if r.returncode:
        raise RuntimeError(f"harness {' '.join(cmd[1:])} exited {r.returncode}: {r.stdout[-800:]}")
    stats = [ln for ln in r.stdout.splitlines() if _NUM.search(ln) and _CNT.search(ln)]
    if not stats:
        raise RuntimeError(f"harness printed no stats line: {r.stdout[-800:]}")
    ln = stats[-1]
    return {"ms": {k: float(v) for k, v in _NUM.findall(ln)}, "count": {k: int(v) for k, v in _CNT.findall(ln)}, "stdout": r.stdout}


def gpu_ms(res) -> float:
    """The GPU phases both engines report for a join: traverse + refine + compact (the reference's JoinStats)."""
    return sum(res["ms"].get(k, 0.0) for k in ("traverse", "refine", "compact"))


def de9im_codes(mats: np.ndarray) -> np.ndarray:
    """9-character DE-9IM strings (cells II IB IE BI BB BE EI EB EE) -> 2-bit-per-cell codes (F 0, '0' 1, '1' 2, '2' 3)."""
    b = np.frombuffer(b"".join(m.encode() if isinstance(m, str) else m for m in mats), np.uint8).reshape(-1, 9)
    v = _CELL[b]
    return (v << (2 * np.arange(9, dtype=np.uint32))).sum(axis=1).astype(np.uint32)


def read_pairs_csv(path):
    """(pairs uint32[n, 2], payload): payload = float64 areas, or uint32 DE-9IM codes for a relate CSV."""
    import pandas as pd
    head = open(path).readline().strip().split(",")
    df = pd.read_csv(path, dtype={0: np.uint32, 1: np.uint32, 2: str, 3: (str if head[3] == "relate" else np.float64)},
                     keep_default_na=False, float_precision="round_trip")
    pairs = np.stack([df.iloc[:, 0].to_numpy(np.uint32), df.iloc[:, 1].to_numpy(np.uint32)], axis=1)
    col = df.iloc[:, 3]
    payload = de9im_codes(col.to_numpy()) if head[3] == "relate" else col.to_numpy(np.float64)
    return pairs, payload


def read_cluster_csv(path) -> np.ndarray:
    import pandas as pd
    df = pd.read_csv(path, dtype={0: np.uint64, 1: np.uint32})
    lab = np.empty(len(df), np.uint32)
    lab[df.iloc[:, 0].to_numpy(np.int64)] = df.iloc[:, 1].to_numpy(np.uint32)
    return lab


def dense_labels(root: np.ndarray) -> np.ndarray:
    """Cluster numbers as the harness writes them: dense, in order of each component's first row."""
    _, first, inv = np.unique(root, return_index=True, return_inverse=True)
    rank = np.empty(len(first), np.uint32)
    rank[np.argsort(first, kind="stable")] = np.arange(len(first), dtype=np.uint32)
    return rank[inv]


def upper_rows(pairs, payload=None):
    """The rows of a self-join with a <= b (drops the mirrored copies the harness writes), sorted by (a, b)."""
    k = pairs[:, 0] <= pairs[:, 1]
    p = pairs[k]
    i = np.lexsort(p.T[::-1])
    return (p[i], None if payload is None else payload[k][i])


def sorted_rows(pairs, payload=None):
    i = np.lexsort(pairs.T[::-1])
    return pairs[i], (None if payload is None else payload[i])
