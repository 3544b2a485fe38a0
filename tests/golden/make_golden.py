#!/usr/bin/env python3
"""Golden vectors from the reference engine itself.

The reference (landstats-us/postgis-cuda) ships no tests or fixtures, so its own file driver
(engine/harness.cu, built unmodified for sm_100a by oracle/build_ref.sh into oracle/_ref/harness) is run on small
seeded synthetic layers; its CSV outputs are folded into tests/golden/*.npz, which pin the CPU oracle in the
CPU-only tests.

  make_golden.py inputs DIR              write the input layers (.gset/.pset + .ids) and cases.json into DIR
  make_golden.py run DIR HARNESS         run the reference harness on every case (GPU box), CSVs into DIR
  make_golden.py collect DIR             fold DIR/*.csv into tests/golden/<case>.npz (+ input checksums)
"""
from __future__ import annotations

import csv
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "postgis-cuda_b200"))
from gsj import gen  # noqa: E402

SMALL_BOX = (-118.30, 33.95, -118.20, 34.05)   # 0.1 deg x 0.1 deg


def layers():
    """name -> (kind, builder). Every builder is seeded: identical bytes on every run."""
    return {
        "zonesA": ("gset", lambda: gen.voronoi(2000, gen.LA_BOX, 0, vmin=6, vmax=40)),
        "zonesB": ("gset", lambda: gen.voronoi(50, gen.LA_BOX, 1, vmin=4, vmax=4)),
        "parcels": ("gset", lambda: gen.layer_parcels(3000, SMALL_BOX, seed=5)),
        "points": ("pset", lambda: gen.points(5000, SMALL_BOX, 3)),
        "parcels2": ("gset", lambda: gen.layer_parcels(2000, SMALL_BOX, seed=6)),
    }


# case -> (P layer, R layer, harness flags)
CASES = {
    "ab_area": ("zonesA", "zonesB", ["--area"]),
    "aa_area": ("zonesA", "zonesA", ["--area"]),
    "pp_relate": ("parcels", "parcels", ["--relate"]),
    "pp_area_sub32": ("parcels", "parcels", ["--area", "--subdiv", "32"]),
    "pp_relate_sub32": ("parcels", "parcels", ["--relate", "--subdiv", "32"]),
    "pb_relate": ("parcels", "zonesB", ["--relate"]),
    "pts_pip": ("points", "parcels", []),
    "pts_pip_sub32": ("points", "parcels", ["--subdiv-b", "32"]),
    "cluster": ("parcels", "parcels", ["--cluster"]),
    "cluster_sub32": ("parcels", "parcels", ["--cluster", "--subdiv", "32"]),
    "pp_dwithin5": ("parcels", "parcels", ["--dwithin", "5"]),
    "pp_dwithin5_sub32": ("parcels", "parcels", ["--dwithin", "5", "--subdiv", "32"]),
    "pts_dwithin5": ("points", "parcels", ["--dwithin", "5"]),
    "pp_erode1": ("parcels", "parcels", ["--erode", "1"]),
    "pp_erode1_sub32": ("parcels", "parcels", ["--erode", "1", "--subdiv", "32"]),
    "pts_erode1": ("points", "parcels", ["--erode", "1"]),
    "pq_area": ("parcels", "parcels2", ["--area"]),
    "pq_relate": ("parcels", "parcels2", ["--relate"]),
    "pq_erode1": ("parcels", "parcels2", ["--erode", "1"]),
    "pq_erode1_3": ("parcels", "parcels2", ["--erode", "1,3"]),
    "pq_erode5": ("parcels", "parcels2", ["--erode", "5"]),
    "pq_erode1_sub32": ("parcels", "parcels2", ["--erode", "1", "--subdiv", "32"]),
    "pq_dwithin5": ("parcels", "parcels2", ["--dwithin", "5"]),
    "pts_erode3_sub32": ("points", "parcels", ["--erode", "3", "--subdiv-b", "32"]),
}


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def cmd_inputs(d):
    os.makedirs(d, exist_ok=True)
    sums = {}
    for name, (kind, build) in layers().items():
        p = os.path.join(d, f"{name}.{kind}")
        obj = build()
        if kind == "gset":
            gen.write_gset(p, obj)
        else:
            gen.write_pset(p, obj)
        sums[name] = sha(p)
    json.dump({"inputs": sums, "cases": CASES}, open(os.path.join(d, "cases.json"), "w"), indent=1)


def cmd_run(d, harness):
    log = open(os.path.join(d, "harness.log"), "w")
    ok = True
    for case, (pa, pb, flags) in CASES.items():
        ka = "pset" if pa == "points" else "gset"
        a = os.path.join(d, f"{pa}.{ka}")
        b = os.path.join(d, f"{pb}.gset")
        out = os.path.join(d, f"{case}.csv")
        cmd = [harness, a, b, *flags, "--reps", "1", "--out", out]
        log.write("$ " + " ".join(cmd) + "\n"); log.flush()
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
        log.write(r.stdout + f"[exit {r.returncode}]\n"); log.flush()
        ok = ok and r.returncode == 0
    return 0 if ok else 1


def cmd_collect(d):
    meta = json.load(open(os.path.join(d, "cases.json")))
    for case, (pa, pb, flags) in CASES.items():
        p = os.path.join(d, f"{case}.csv")
        if not os.path.exists(p):
            print("missing", p)
            continue
        rows = list(csv.reader(open(p)))
        head, body = rows[0], rows[1:]
        out = {"inputs_sha256": np.array([meta["inputs"][pa], meta["inputs"][pb]])}
        if head[0] == "id":   # cluster: id, label
            out["label"] = np.array([int(r[1]) for r in body], np.uint32)
        else:
            out["pairs"] = np.array([[int(r[0]), int(r[1])] for r in body], np.uint32).reshape(-1, 2)
            if head[3] == "relate":
                out["relate"] = np.array([r[3] for r in body])
            else:
                out["area"] = np.array([float(r[3]) for r in body], np.float64)
        np.savez_compressed(os.path.join(HERE, f"{case}.npz"), **out)
        print(case, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    c = sys.argv[1]
    if c == "inputs":
        cmd_inputs(sys.argv[2])
    elif c == "run":
        sys.exit(cmd_run(sys.argv[2], sys.argv[3]))
    elif c == "collect":
        cmd_collect(sys.argv[2])
    else:
        print(__doc__)
        sys.exit(2)
