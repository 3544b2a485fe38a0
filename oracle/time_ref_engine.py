"""Times the reference engine's own file driver and this engine on identical seeded layers (GPU box).

Test and measurement infrastructure, not product: it runs ``oracle/_ref/harness`` (landstats-us/postgis-cuda
engine/harness.cu, unmodified, built for sm_100a by ``oracle/build_ref.sh``) and the gsj C ABI on the same inputs
and prints one markdown table of GPU phase times (traverse + refine + compact, the harness's own stats fields,
engine/harness.cu:75 / :126; best of ``--reps``) and result counts.

  python oracle/time_ref_engine.py [--reps 3] [--cases relate,area2m,area,dwithin,erode,cluster] [--big]

Self-join semantics follow the harness: unordered pairs (engine/harness.cu:54, :105) and, for erosion, no
geometry's pair with itself (need_self all zero for a layer without duplicate geometries, engine/harness.cu:108-115;
the daemon's self_pairs 'distinct', daemon/gpujoind.cu:445-449). ``--big`` adds the 20M-parcel erosion and
cluster layers (~10 GB of .gset files under the scratch directory).
"""
import argparse
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "postgis-cuda_b200"))
import gsj  # noqa: E402
from gsj import gen  # noqa: E402

HARNESS = os.path.join(HERE, "_ref", "harness")
BOX = (-119.0, 33.0, -117.0, 35.0)
PHASE = re.compile(r"traverse=([\d.]+)ms refine=([\d.]+)ms compact=([\d.]+)ms")
COUNT = re.compile(r"(gpu_hits|clusters|rows)=(\d+)")


def harness(args, reps):
    r = subprocess.run([HARNESS, *args, "--reps", str(reps)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=1800)
    if r.returncode:
        raise RuntimeError(f"harness {' '.join(args)} exited {r.returncode}: {r.stdout[-500:]}")
    line = [ln for ln in r.stdout.splitlines() if PHASE.search(ln)][-1]
    t = sum(float(x) for x in PHASE.search(line).groups())
    return t, dict((k, int(v)) for k, v in COUNT.findall(line))


def ours(fn, reps):
    best, out = None, None
    for _ in range(reps + 1):   # first call warms up (module load, pools)
        n, st = fn()
        t = st["traverse_ms"] + st["refine_ms"] + st["compact_ms"]
        best = t if out is not None and (best is None or t < best) else best
        out = n
    return best, out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--cases", default="relate,area2m,area,dwithin,erode,cluster")
    ap.add_argument("--big", action="store_true")
    ap.add_argument("--dir", default=None)
    a = ap.parse_args()
    if not os.path.exists(HARNESS):
        sys.exit("oracle/_ref/harness is missing: build it with oracle/build_ref.sh where the reference sources are")
    cases = a.cases.split(",")
    d = a.dir or tempfile.mkdtemp(prefix="gsj_refcmp_")
    os.makedirs(d, exist_ok=True)
    eng = gsj.Engine(0)
    rows = []

    def add(name, ref, mine, what):
        (tr, cr), (to, co) = ref, mine
        rows.append((name, tr, to, tr / to if to else float("nan"), cr, co, what))
        print(f"{name}: reference {tr:.2f} ms ({cr}), ours {to:.2f} ms ({co})", flush=True)

    if "relate" in cases or "area2m" in cases:
        p = os.path.join(d, "parcels2m.gset")
        ps = gen.layer_parcels(2_000_000, BOX, seed=0)
        gen.write_gset(p, ps)
        L = eng.upload_polygons(ps)
        if "relate" in cases:
            t, c = harness([p, p, "--relate"], a.reps)
            mine = ours(lambda: (lambda r: (len(r.pairs), r.stats))(eng.join(L, L, want_area=False, want_relate=True, upper=True)), a.reps)
            add("relate self-join, 2M parcels (4-256 v)", (t, c.get("gpu_hits")), mine, "intersecting pairs")
        if "area2m" in cases:
            t, c = harness([p, p, "--area"], a.reps)
            mine = ours(lambda: (lambda r: (len(r.pairs), r.stats))(eng.join(L, L, want_area=True, upper=True)), a.reps)
            add("intersects + area self-join, 2M parcels", (t, c.get("gpu_hits")), mine, "intersecting pairs")
        L.free()
    if "area" in cases:
        pa, pb = os.path.join(d, "zones20k.gset"), os.path.join(d, "zones50.gset")
        A, B = gen.layer_cfg_parcels_small(20000, seed=0), gen.layer_cfg_zones(50, seed=1)
        gen.write_gset(pa, A)
        gen.write_gset(pb, B)
        LA, LB = eng.upload_polygons(A), eng.upload_polygons(B)
        t, c = harness([pa, pb, "--area"], a.reps)
        mine = ours(lambda: (lambda r: (len(r.pairs), r.stats))(eng.join(LA, LB, want_area=True)), a.reps)
        add("intersects + area, 20k zones x 50 zones", (t, c.get("gpu_hits")), mine, "intersecting pairs")
        LA.free()
        LB.free()
    if "dwithin" in cases:
        box = (-119.0, 33.0, -118.0, 34.0)
        pp, pg = os.path.join(d, "points1m.pset"), os.path.join(d, "parcels1m.gset")
        xy, R = gen.points(1_000_000, box, 7), gen.layer_parcels(1_000_000, box, seed=0)
        gen.write_pset(pp, xy)
        gen.write_gset(pg, R)
        LP, LR = eng.upload_points(xy), eng.upload_polygons(R)
        t, c = harness([pp, pg, "--dwithin", "5"], a.reps)
        mine = ours(lambda: (lambda r: (len(r[0]), r[1]))(eng.points_dwithin(LP, LR, 5.0)), a.reps)
        add("ST_DWithin 5 m, 1M points x 1M parcels", (t, c.get("gpu_hits")), mine, "pairs within 5 m")
        LP.free()
        LR.free()
    sizes = [2_000_000] + ([20_000_000] if a.big else [])
    for n in sizes:
        if "erode" not in cases and "cluster" not in cases:
            break
        side = 2.0 * (n / 2e6) ** 0.5
        p = os.path.join(d, f"cfg5_{n}.gset")
        ps = gen.layer_cfg5(n, (-119.0, 33.0, -119.0 + side, 33.0 + side), seed=0)
        gen.write_gset(p, ps)
        L = eng.upload_polygons(ps)
        tag = f"{n / 1e6:g}M parcels (~30 v)"
        if "erode" in cases:
            t, c = harness([p, p, "--erode", "1"], a.reps)
            none = np.zeros(L.info["nparent"], np.uint8)
            mine = ours(lambda: (lambda r: (len(r[0]), r[1]))(eng.erode(L, L, 1.0, 1.0, same=True, need_self=none)), a.reps)
            add(f"buffer(-1 m) x buffer(-1 m) self-join (distinct), {tag}", (t, c.get("gpu_hits")), mine, "pairs")
        if "cluster" in cases:
            t, c = harness([p, p, "--cluster"], a.reps)
            mine = ours(lambda: (lambda r: (int(np.unique(r[0]).size), r[1]))(eng.cluster(L)), a.reps)
            add(f"ST_ClusterIntersecting, {tag}", (t, c.get("clusters")), mine, "clusters")
        L.free()
        os.remove(p)
    print()
    print("| workload | reference engine (ms) | gsj (ms) | speed-up | reference count | gsj count | counted |")
    print("|---|---|---|---|---|---|---|")
    for name, tr, to, sp, cr, co, what in rows:
        print(f"| {name} | {tr:.2f} | {to:.2f} | {sp:.2f}x | {cr} | {co} | {what} |")


if __name__ == "__main__":
    main()
