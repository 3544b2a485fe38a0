#!/usr/bin/env python3
"""Benchmark: DE-9IM relate self-join of 2M synthetic parcels on one B200 (per rank).

Workload (the configuration the headline metric is quoted on): Voronoi cells of 2M jittered-grid seeds in a
2 x 2 degree lon/lat box (lon -119..-117, lat 33..35), 4-256 vertices per ring (log-uniform), 5% MultiPolygons
with 2-4 parts, 2% with one interior hole; gpu_relate self-join, each unordered pair once (diagonal included);
the filtered refinement (candidate edge-pair lists) vs the plain FP64 kernels, pair sets and DE-9IM compared;
plus the serving leg (gsjd under a Poisson request stream, p50/p99 latency).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--op relate|area|dwithin|erode|cluster]

--op selects the other configurations of the same metric family (one JSON line each): area = intersects + area of
20k Voronoi zones (6-40 vertices) x 50 zones; dwithin = 1M parcels x 1M points, ST_DWithin(geography, 5 m);
erode = ST_Intersects(ST_Buffer(a, -1 m), ST_Buffer(b, -1 m)) self-join and cluster = ST_ClusterIntersecting, both
on a parcel layer with ~30 vertices per ring (20M parcels by default; --seeds to change).

A step is one full self-join of the resident layer. value = intersecting pairs / device time (CUDA events on the
engine's stream; the rows reach pinned host buffers every step). e2e = the same join through the C ABI from pinned
host buffers: upload (H2D) + LBVH build + join + result D2H, every step. N > 1 (torchrun): every rank joins its own
2M-parcel layer (seed = rank), no data-path collective; value = all ranks' pairs / max-over-ranks time (weak
scaling). After the timed steps the filtered and the plain variant's rows are compared with each other and, row by
row, with the reference engine's own driver run on the same layer (pair_diffs_vs_reference, code_diffs_vs_reference).

--impl reference runs the reference engine itself (landstats-us/postgis-cuda engine/harness.cu, unmodified, built
for sm_100a into oracle/_ref/harness) on the same seeded layer on this GPU: value = its intersecting pairs / its GPU
phase time (traverse + refine + compact, its own stats) of the last of warmup + steps repetitions; e2e = the same
pairs / its upload + BVH + join + D2H time. The CPU FP64 oracle stays the cpu_baseline of this arm's line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "postgis-cuda_b200"))

BOX = (-119.0, 33.0, -117.0, 35.0)
N_SEEDS = 2_000_000
METRIC = "join pairs/s (DE-9IM relate self-join, filtered FP64 refinement)"
# B200 FP64 (non-tensor) peak per GPU from NVIDIA's HGX B200 specification (296 TFLOPS for 8 GPUs); no measured copy
FP64_PEAK_TFLOPS = 37.0
# algorithmic FP64 work of the reference's refinement per local edge pair (i, j): the contact test's 4 orientations
# x 10 flops, plus ~30 flops of the Green's-theorem / relate pass (edge_contrib_loc, engine.cuh:416-515)
FLOPS_PER_EDGE_PAIR = 70.0
WORKLOAD = "relate self-join, 2M jittered-grid Voronoi parcels, 2x2 deg, 4-256 vertices/ring, 5% multipolygons, 2% holes"


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.lines, self.p = gpu, [], None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=lambda: self.lines.extend(self.p.stdout), daemon=True)
            self.t.start()
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.t.join(2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        import torch
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return rank, local, ws


def allreduce_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate(ms_local: float, units_local: float, ws: int):
    """Whole-job rate over replicas: units of all ranks / the slowest rank's device time. (value, max ms)."""
    tot_ms = allreduce_max(ms_local, ws)
    units = allreduce_sum(units_local, ws)
    return units / (tot_ms / 1000.0), tot_ms


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def sub_layer(ps, box):
    """Geometries of ps whose vertices all lie inside box (re-indexed), a spatially bounded sample."""
    from gsj.gen import PolygonSet
    gro, rvo, xy = ps.gro.astype(np.int64), ps.rvo.astype(np.int64), ps.xy
    v0, v1 = rvo[gro[:-1]], rvo[gro[1:]]
    vmin = np.minimum.reduceat(xy, v0, axis=0)
    vmax = np.maximum.reduceat(xy, v0, axis=0)
    sel = np.nonzero((vmin[:, 0] >= box[0]) & (vmin[:, 1] >= box[1]) & (vmax[:, 0] <= box[2]) & (vmax[:, 1] <= box[3]))[0]
    ngro, nrvo, nxy = [0], [0], []
    for g in sel:
        for r in range(gro[g], gro[g + 1]):
            nxy.append(xy[rvo[r]:rvo[r + 1]])
            nrvo.append(nrvo[-1] + rvo[r + 1] - rvo[r])
        ngro.append(len(nrvo) - 1)
    return PolygonSet(np.array(ngro, np.uint64), np.array(nrvo, np.uint64), np.concatenate(nxy))


def cpu_sample(ps, target_s):
    """A corner sub-box of the layer sized so the CPU oracle's relate self-join takes about target_s here."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    frac = 0.06
    while True:
        w = (BOX[2] - BOX[0]) * frac
        sub = sub_layer(ps, (BOX[0], BOX[1], BOX[0] + w, BOX[1] + w))
        S = O.OSet(sub)
        t = time.perf_counter()
        O.join(S, S, O.params(0, 1), upper=True)
        dt = time.perf_counter() - t
        if dt >= target_s / 3 or frac >= 1.0:
            return S, sub, w
        frac = min(1.0, frac * (target_s / max(dt, 0.02)) ** 0.5)


def cpu_time(S):
    import pyoracle as O
    t = time.perf_counter()
    p, a, c, nc = O.join(S, S, O.params(0, 1), upper=True)
    dt = time.perf_counter() - t
    return len(p), dt


def cpu_oracle_rate(ps, target_s=15.0):
    """The CPU FP64 oracle (OpenMP, all host threads) on a bounded spatial sample: pairs/s."""
    S, sub, w = cpu_sample(ps, target_s)
    n, dt = cpu_time(S)
    return n / dt, dict(pairs=n, seconds=dt, parcels=sub.n, box_deg=w, threads=os.cpu_count())


# Serving: resident 10M Voronoi polygons (4-512 vertices, log-uniform) + 5M points; a seeded Poisson stream of 50 req/s,
# each a join of 10^2-10^6 query polygons (log-uniform) of mixed type; then the same requests by closed-loop clients
# (the daemon at saturation). SERVE_SMALL is a scaled-down copy for quick runs (--serve-small).
SERVE = dict(name="cfg4", resident=10_000_000, box=(-120.0, 32.0, -115.5, 36.5), vmin=4, vmax=512, points=5_000_000, rate=50.0,
             requests=1100, warmup=100, sizes=(1e2, 1e6), queries=24, closed_clients=8, closed_s=15.0)
SERVE_SMALL = dict(name="cfg4 scaled down", resident=1_000_000, box=(-119.0, 33.0, -117.6, 34.4), vmin=4, vmax=512, points=500_000,
                   rate=50.0, requests=300, warmup=30, sizes=(1e2, 1e5), queries=12, closed_clients=8, closed_s=8.0)


def serving_schedule(rng, qpoly, n, rate):
    """Poisson arrivals at rate; ops: intersects+area 50%, relate 20%, dwithin 5 m 20%, point in polygon 10% (the query
    polygons against the resident points)."""
    lines, t = [], 0.0
    for _ in range(n):
        t += rng.exponential(1.0 / rate)
        u, q = rng.random(), rng.choice(qpoly)
        if u < 0.5:
            lines.append(f"{t:.6f}\tJOIN\t{q}\tresident\t1\tall")
        elif u < 0.7:
            lines.append(f"{t:.6f}\tRELATE\t{q}\tresident\t\tall")
        elif u < 0.9:
            lines.append(f"{t:.6f}\tDWITHIN\t{q}\tresident\tdwithin\t5\t0\tall")
        else:
            lines.append(f"{t:.6f}\tJOIN\t{q}\tpoints\t0\tall")
    return "\n".join(lines) + "\n"


SERVE_ARMS = (   # name -> gsjd flags; the same daemon, schedule and priming, only the refinement differs; each arm's
    # refinement launch shape is chosen by the autotuner when the resident layer is loaded
    ("filtered", ["--refine", "filtered", "--tune", "1"]),
    ("plain", ["--refine", "plain", "--tune", "1"]),
)


def serving_leg(cfg, workers=4):
    """gsjd serving the request stream against the resident layers, filtered and plain FP64 refinement on the same
    schedule, each after an untimed priming pass over the schedule's distinct requests; then closed-loop clients."""
    import shutil
    import tempfile
    from gsj import client as C
    from gsj import daemon as D
    from gsj import gen
    from gsj._build import lib_path
    d = tempfile.mkdtemp(prefix="gsjd_bench_")
    try:
        t0 = time.time()
        box = cfg["box"]
        area = (box[2] - box[0]) * (box[3] - box[1])
        params = dict(jitter_grid=True, jitter=0.4, vmin=cfg["vmin"], vmax=cfg["vmax"], log_uniform=True)
        res_layer = gen.voronoi(cfg["resident"], box, 0, **params)
        n_res, nv_res = res_layer.n, res_layer.nv
        gen.write_gset(os.path.join(d, "resident.gset"), res_layer)
        del res_layer
        gen.write_pset(os.path.join(d, "points.pset"), gen.points(cfg["points"], box, 7))
        rng = np.random.default_rng(42)
        density = cfg["resident"] / area
        qpoly, qsizes = [], []
        lo, hi = cfg["sizes"]
        for i in range(cfg["queries"]):
            n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
            side = min(box[2] - box[0], (n / density) ** 0.5)
            x0 = rng.uniform(box[0], box[2] - side)
            y0 = rng.uniform(box[1], box[3] - side)
            gen.write_gset(os.path.join(d, f"q{i}.gset"), gen.voronoi(max(n, 4), (x0, y0, x0 + side, y0 + side), 1000 + i, **params))
            qpoly.append(f"q{i}")
            qsizes.append(max(n, 4))
        sched = os.path.join(d, "schedule.tsv")
        open(sched, "w").write(serving_schedule(rng, qpoly, cfg["requests"], cfg["rate"]))
        distinct = sorted({ln.split("\t", 1)[1] for ln in open(sched).read().splitlines() if ln})
        prime = os.path.join(d, "prime.tsv")
        open(prime, "w").write("".join(f"{0.05 * (i // 4):.3f}\t{req}\n" for i, req in enumerate(distinct)))
        prep_s = time.time() - t0
        out = {}
        for mode, flags in SERVE_ARMS:
            sock = os.path.join(d, f"gsjd_{mode}.sock")
            log = open(os.path.join(d, f"gsjd_{mode}.log"), "w")
            p = D.start(sock, d, workers=workers, threads=max(4, (os.cpu_count() or 8) // 2), log=log, extra=flags)
            try:
                cl = C.Client(sock)
                tl = time.time()
                cl.load("resident", "resident.gset", dedup=False)
                cl.load("points", "points.pset")
                for q in qpoly:
                    cl.load(q, q + ".gset", dedup=False)
                load_s = time.time() - tl
                # untimed priming: every distinct request of the schedule once, 4 at a time, so each context has grown
                # its scratch for the largest requests before the measured replay (steady-state serving)
                subprocess.run([lib_path("gsjd_loadgen"), "--socket", sock, "--schedule", prime], capture_output=True, text=True, timeout=1800)
                r = subprocess.run([lib_path("gsjd_loadgen"), "--socket", sock, "--schedule", sched, "--warmup", str(cfg["warmup"])],
                                   capture_output=True, text=True, timeout=3600)
                res = json.loads(r.stdout.strip().splitlines()[-1])
                res["rows_per_s"] = res["rows"] / res["span_s"]
                res["load_s"] = round(load_s, 1)
                r = subprocess.run([lib_path("gsjd_loadgen"), "--socket", sock, "--schedule", sched, "--closed", str(cfg["closed_clients"]),
                                    "--duration", str(cfg["closed_s"])], capture_output=True, text=True, timeout=3600)
                res["saturated"] = json.loads(r.stdout.strip().splitlines()[-1])
                out[mode] = res
            finally:
                D.stop(p)
                log.close()
            if mode in out:   # the launch shape the daemon's autotuner chose when the resident layer was loaded
                tl = [ln.strip() for ln in open(os.path.join(d, f"gsjd_{mode}.log")) if "tune resident:" in ln]
                out[mode]["autotuner"] = tl[-1].split("tune resident: ", 1)[1] if tl else None
        out["pairs_per_s_saturated"] = {m: out[m]["saturated"]["rows_per_s"] for m, _ in SERVE_ARMS}
        out["p99_ratio_plain_over_filtered"] = out["plain"]["p99_ms"] / out["filtered"]["p99_ms"] if out["filtered"]["p99_ms"] else None
        out["saturated_ratio_filtered_over_plain"] = (out["pairs_per_s_saturated"]["filtered"] / out["pairs_per_s_saturated"]["plain"]
                                                     if out["pairs_per_s_saturated"]["plain"] else None)
        out["config"] = {"workload": cfg["name"], "resident_polygons": int(n_res), "resident_vertices": int(nv_res),
                         "resident_points": cfg["points"], "vertices_per_ring": f"{cfg['vmin']}-{cfg['vmax']} log-uniform",
                         "box_deg": list(box), "rate_per_s": cfg["rate"], "requests": cfg["requests"], "warmup_requests": cfg["warmup"],
                         "query_sizes": f"log-uniform {lo:g}-{hi:g} polygons", "query_layers": cfg["queries"],
                         "query_polygons_total": int(sum(qsizes)),
                         "mix": "join+area 50%, relate 20%, dwithin 5 m 20%, point in polygon 10% (query polygons x resident points)",
                         "workers": workers, "closed_clients": cfg["closed_clients"], "closed_s": cfg["closed_s"],
                         "rows": "rows are pairs (no duplicate geometries in these layers)", "prep_s": round(prep_s, 1)}
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_op(args, rank, local, ws):
    """The other configurations: one JSON line with the same keys as the headline."""
    import torch
    import gsj
    from gsj import gen
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    torch.cuda.set_device(local)
    eng = gsj.Engine(local)
    ext = torch.cuda.ExternalStream(eng.stream_handle(), device=local)
    op = args.op
    # cluster across GPUs: one layer, each rank its probe shard, forests all-gathered and joined (gsj.dist)
    cl_shard = op == "cluster" and args.shard and ws > 1
    t0 = time.time()
    pts = None
    if op == "area":
        A, B = gen.layer_cfg_parcels_small(20000, seed=rank), gen.layer_cfg_zones(50, seed=1)
        workload = "intersects + area, 20k Voronoi zones (6-40 vertices, LA box) x 50 zones"
        metric, unit = "join pairs/s (intersects + area, filtered FP64 refinement)", "pairs/s"
    elif op == "dwithin":
        box = (-119.0, 33.0, -118.0, 34.0)
        A, B = None, gen.layer_parcels(1_000_000, box, seed=rank)
        pts = gen.points(1_000_000, box, 7 + rank)
        workload = "ST_DWithin(geography, 5 m): 1M uniform points x 1M jittered-grid parcels, 1x1 deg"
        metric, unit = "join pairs/s (points x parcels ST_DWithin 5 m)", "pairs/s"
    else:
        n = args.seeds or 20_000_000
        side = 2.0 * (n / 2e6) ** 0.5
        box = (-119.0, 33.0, -119.0 + side, 33.0 + side)
        A = B = gen.layer_cfg5(n, box, seed=0 if cl_shard else rank)
        if op == "erode":
            workload = f"ST_Intersects(ST_Buffer(a,-1m), ST_Buffer(b,-1m)) self-join (self_pairs all), {n / 1e6:g}M parcels, ~30 vertices/ring"
            metric, unit = "join pairs/s (negative-buffer intersects self-join, ra = rb = 1 m)", "pairs/s"
        else:
            workload = f"ST_ClusterIntersecting, {n / 1e6:g}M parcels, ~30 vertices/ring"
            metric, unit = "parcels/s (ST_ClusterIntersecting)", "parcels/s"
    t_gen = time.time() - t0
    LA = eng.upload_polygons(A) if A is not None else None
    LB = LA if B is A else eng.upload_polygons(B)
    LP = eng.upload_points(pts) if pts is not None else None

    def run(mode):
        if op == "area":
            r = eng.join(LA, LB, want_area=True, want_relate=False, refine_mode=mode)
            return len(r.pairs), r.stats
        if op == "dwithin":
            p, st = eng.points_dwithin(LP, LB, 5.0, refine_mode=mode)   # warp / thread per (point, parcel)
            return len(p), st
        if op == "erode":   # self_pairs 'all': a parcel's pair with itself is kept when its eroded form is not empty
            p, st = eng.erode(LA, LA, 1.0, 1.0, same=True, refine_mode=mode)
            return len(p), st
        if cl_shard:
            from gsj import dist as gd
            root, st = gd.cluster_sharded(eng, LA, refine_mode=mode)
            return (len(root) if rank == 0 else 0), st   # the layer counted once
        root, st = eng.cluster(LA, refine_mode=mode)
        return len(root), st

    def timed(mode):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            e0.record()
        units, st = run(mode)
        with torch.cuda.stream(ext):
            e1.record()
        e1.synchronize()
        return units, st, e0.elapsed_time(e1)

    modes = [(n, m) for n, m in (("filtered", gsj.GSJ_REFINE_FILTERED), ("plain", gsj.GSJ_REFINE_PLAIN)) if n in args.arms.split(",")]
    res = {}
    for name, mode in modes:
        for _ in range(args.warmup):
            timed(mode)
        barrier(ws)
        torch.cuda.synchronize()
        ms, units, stats = [], 0, []
        with Clocks(local) as clk:
            for _ in range(args.steps):
                u, st, t = timed(mode)
                ms.append(t); units += u; stats.append(st)
        torch.cuda.synchronize()
        barrier(ws)
        res[name] = dict(ms=ms, units=units, stats=stats, clocks=clk.summary())
    f = res["filtered"]
    value, tot_ms = aggregate(float(np.sum(f["ms"])), float(f["units"]), ws)
    # end to end through the C ABI from host buffers: upload (+ LBVH) + the op + the rows back
    e2e_ms, e2e_units = [], 0
    h2d = sum(int(x.nbytes) for x in ([A.gro, A.rvo, A.xy] if A is not None else []) + ([B.gro, B.rvo, B.xy] if B is not A else []) +
              ([pts] if pts is not None else []))
    for i in range(1 + args.steps):
        t = time.perf_counter()
        xa = eng.upload_polygons(A) if A is not None else None
        xb = xa if B is A else eng.upload_polygons(B)
        xp = eng.upload_points(pts) if pts is not None else None
        if op == "area":
            u = len(eng.join(xa, xb, want_area=True).pairs)
        elif op == "dwithin":
            u = len(eng.points_dwithin(xp, xb, 5.0)[0])
        elif op == "erode":
            u = len(eng.erode(xa, xa, 1.0, 1.0, same=True)[0])
        elif cl_shard:
            from gsj import dist as gd
            root_all = gd.cluster_sharded(eng, xa)[0]
            u = len(root_all) if rank == 0 else 0   # the layer counted once
        else:
            u = len(eng.cluster(xa)[0])
        for x in {id(v): v for v in (xa, xb, xp) if v is not None}.values():
            x.free()
        if i:
            e2e_ms.append((time.perf_counter() - t) * 1000.0); e2e_units += u
    e2e_value, e2e_tot = aggregate(float(np.sum(e2e_ms)), float(e2e_units), ws)
    st = f["stats"]
    pk = peaks()
    hbm = pk.get("hbm_gbs", 6650.0)
    trav_ms = float(np.mean([s_["traverse_ms"] for s_ in st]))
    nq = (LP.info["n"] if LP is not None else LA.info["n"])
    trav_bytes = float(np.mean([s_["node_visits"] for s_ in st]) * 48 + nq * 20 + np.mean([s_["candidates"] for s_ in st]) * 8)
    # the dominant kernel, refinement: algorithmic bytes = both geometries' vertices per candidate pair (layer means)
    ref_ms = float(np.mean([s_["refine_ms"] for s_ in st]))
    nv_a = 1.0 if A is None else len(A.xy) / A.n
    nv_b = len(B.xy) / B.n
    ref_bytes = float(np.mean([s_["candidates"] for s_ in st])) * 16.0 * (nv_a + nv_b)
    ref_kernel = {"area": "k_refine<filtered>", "dwithin": "k_pt_dwithin_warp",
                  "erode": "k_refine<filtered> (pass 1) + k_erode_main/tiles", "cluster": "k_refine<filtered> (cluster rounds)"}[op]
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        t = time.perf_counter()
        if op == "area":   # CPU-runnable in full
            OA, OB = O.OSet(A), O.OSet(B)
            n_cpu = len(O.join(OA, OB, O.params(1, 0))[0]); sample = "the whole workload"
        elif op == "dwithin":
            k = 50_000
            n_cpu = len(O.pt_dwithin(pts[:k], O.OSet(B), 5.0)); sample = f"the first {k} points against the whole layer"
        else:
            w = 0.1 * (box[2] - box[0])
            sub = sub_layer(A, (box[0], box[1], box[0] + w, box[1] + w))
            S = O.OSet(sub)
            if op == "erode":
                n_cpu = len(O.erode(S, S, 1.0, 1.0, same=True))
            else:
                O.cluster(S, sub.n); n_cpu = sub.n
            sample = f"{sub.n} parcels in a {w:.3f} deg corner sub-box"
        dt = time.perf_counter() - t
        cpu = {"value": n_cpu / dt, "unit": unit, "cores": os.cpu_count(), "kind": "port",
               "sample": f"CPU FP64 oracle (OpenMP) on {sample} ({dt:.1f} s)"}
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "strong" if cl_shard else "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Voronoi parcels / uniform points)",
        "config": {"workload": workload, "units_per_step": int(f["units"] / args.steps), "candidates": int(st[0]["candidates"]),
                   "parallelism": (f"probe shards x{ws}, forests all-gathered and joined" if cl_shard else f"replicas x{ws}"),
                   "gen_s": round(t_gen, 1)},
        "phases_ms": {k: float(np.mean([s_[k] for s_ in st])) for k in ("traverse_ms", "refine_ms", "compact_ms", "copy_ms")},
        "e2e": {"value": e2e_value, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(8 * e2e_units / max(1, args.steps)),
                "ms_per_step": e2e_tot / args.steps},
        "roofline": {"kernel": ref_kernel, "bound": "hbm", "achieved": ref_bytes / (ref_ms / 1000.0) / 1e9 if ref_ms > 0 else None,
                     "peak": hbm, "unit": "GB/s", "frac": ref_bytes / (ref_ms / 1000.0) / 1e9 / hbm if ref_ms > 0 else None, "traffic": None,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in pk else "fallback",
                     "note": "bytes = candidates x both geometries' mean vertex bytes; the kernels are FP64/latency-bound, not HBM-bound"
                             + ("; the cluster rounds refine a subset of the candidates" if op == "cluster" else ""),
                     # the polygon refinement's FP64 work, as on the headline line: 70 flops per local edge pair, counted in the kernels
                     "fp64": ({"achieved_tflops": ep * FLOPS_PER_EDGE_PAIR / (ref_ms / 1000.0) / 1e12,
                               "frac": ep * FLOPS_PER_EDGE_PAIR / (ref_ms / 1000.0) / 1e12 / FP64_PEAK_TFLOPS, "peak_tflops": FP64_PEAK_TFLOPS,
                               "edge_pairs_per_step": ep,
                               "what": "the refine phase's time includes the erosion tests" if op == "erode" else "the refine phase"}
                              if (ep := float(np.mean([s_.get("edge_pairs", 0) for s_ in st]))) > 0 and ref_ms > 0 else None)},
        "roofline_traversal": {"kernel": "k_traverse", "bound": "hbm",
                               "achieved": trav_bytes / (trav_ms / 1000.0) / 1e9 if trav_ms > 0 else None, "peak": hbm, "unit": "GB/s",
                               "frac": trav_bytes / (trav_ms / 1000.0) / 1e9 / hbm if trav_ms > 0 else None},
        "gpu_launches": int(sum(s_["launches"] for s_ in st)),
        "clocks": f["clocks"],
        "cpu_baseline": cpu,
    }
    if "plain" in res:
        pv, pms = aggregate(float(np.sum(res["plain"]["ms"])), float(res["plain"]["units"]), ws)
        line["plain_fp64"] = {"value": pv, "ms_per_step": pms / args.steps, "speedup_filtered": (pms / tot_ms) if tot_ms > 0 else None,
                              "same_units": res["plain"]["units"] == f["units"]}
    if op in ("erode", "cluster") and ws == 1 and not cl_shard:
        line["non_degenerate"] = non_degenerate_leg(eng, ext, op, n, box, LA, args)
    if rank == 0:
        print(json.dumps(line), flush=True)


def non_degenerate_leg(eng, ext, op, n, box, LA, args):
    """Beside the cfg5 numbers, the same op on inputs whose answer is not trivial on a tiling (where neighbours only
    touch): erosion of the layer against an independently seeded layer of the same size (interiors overlap, so
    eroded pairs survive), and clustering of a layer whose parcels are 55 % shrunk (components of every size).
    Filtered variant, the same warm-up and step counts."""
    import torch
    from gsj import gen
    if op == "erode":
        other = gen.layer_cfg5(n, box, seed=1)
        L2 = eng.upload_polygons(other)
        work = f"erosion (1 m) of the layer against an independently seeded {n / 1e6:g}M-parcel layer"
        run = lambda: eng.erode(LA, L2, 1.0, 1.0, same=False)[0]
        count = len
        unit = "pairs"
    else:
        shr = gen.shrunk(gen.layer_cfg5(n, box, seed=3), seed=3)
        L2 = eng.upload_polygons(shr)
        work = f"ST_ClusterIntersecting of {n / 1e6:g}M parcels, 55 % of them shrunk (components of every size)"
        run = lambda: eng.cluster(L2)[0]
        count = lambda root: int(len(np.unique(root)))
        unit = "components"
    ms, last = [], None
    for i in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            e0.record()
        r = run()
        with torch.cuda.stream(ext):
            e1.record()
        e1.synchronize()
        if i >= args.warmup:
            ms.append(e0.elapsed_time(e1)); last = r
    units = count(last)   # outside the timed region
    L2.free()
    out = {"workload": work, "ms_per_step": float(np.mean(ms)), unit: units}
    out["value"] = (units if op == "erode" else n) / (float(np.mean(ms)) / 1000.0)
    out["unit"] = "pairs/s" if op == "erode" else "parcels/s"
    return out


def reference_check(ps, filt, tmpdir):
    """Row-by-row comparison with the reference engine's own driver on the same layer (checker, untimed)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refharness as RH
    from gsj import gen
    if not RH.available():
        return {"available": False, "why": "oracle/_ref/harness is not built"}
    g = os.path.join(tmpdir, "parcels.gset")
    gen.write_gset(g, ps)
    out = os.path.join(tmpdir, "reference_rows.csv")
    t = time.time()
    r = RH.run([g, g, "--relate"], reps=1, out_csv=out)
    rows, codes = RH.read_pairs_csv(out)
    os.remove(out)
    want_p, want_c = RH.upper_rows(rows, codes)
    got_p, got_c = RH.sorted_rows(filt.pairs, filt.code)
    same = got_p.shape == want_p.shape and np.array_equal(got_p, want_p)
    if same:
        pair_diffs, code_diffs = 0, int((got_c != want_c).sum())
    else:
        a, b = set(map(tuple, got_p.tolist())), set(map(tuple, want_p.tolist()))
        pair_diffs, code_diffs = len(a ^ b), None
    return {"available": True, "pair_diffs": pair_diffs, "code_diffs": code_diffs, "reference_rows": int(len(rows)),
            "reference_pairs": int(len(want_p)), "reference_phases_ms": r["ms"], "seconds": round(time.time() - t, 1)}


def run_reference(args, rank, ws):
    """--impl reference: the reference engine's own driver (unmodified, sm_100a) on the same seeded layer and GPU."""
    import shutil
    import tempfile
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refharness as RH
    from gsj import gen
    if rank != 0:
        return
    if not RH.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/harness (the reference engine's driver) is not built"}), flush=True)
        return
    if args.op != "relate":
        run_reference_op(args, RH)
        return
    ps = gen.layer_parcels(args.seeds, BOX, seed=0)
    d = tempfile.mkdtemp(prefix="gsj_ref_")
    # The driver reports its phase times for its last repetition only, and its repetitions slow down after the first
    # few in one process (refine 0.52 s in the first, 2.1 s in the eighth on the same B200). Each measured step is
    # therefore one driver process with two repetitions, the second (warm) one reported; at most 5 such steps.
    runs = max(1, min(args.steps, 5))
    try:
        g = os.path.join(d, "parcels.gset")
        gen.write_gset(g, ps)
        with Clocks(0) as clk:
            rs = [RH.run([g, g, "--relate"], reps=2) for _ in range(runs)]
    except (RuntimeError, OSError, subprocess.TimeoutExpired) as e:   # e.g. no usable CUDA device for the driver
        why = str(e).strip().splitlines()[-1][:300] if str(e).strip() else type(e).__name__
        print(json.dumps({"impl": "reference", "unavailable": f"the reference engine's driver did not run: {why}"}), flush=True)
        return
    finally:
        shutil.rmtree(d, ignore_errors=True)
    gms = [RH.gpu_ms(r) for r in rs]
    k = int(np.argsort(gms)[len(gms) // 2])   # the median step
    r = rs[k]
    ms = gms[k]
    pairs = r["count"]["gpu_hits"]
    value = pairs / (ms / 1000.0)
    e2e_ms = r["ms"]["upload"] + r["ms"]["bvh"] + ms + r["ms"].get("d2h", 0.0)
    reps = 2
    h2d = int(ps.gro.nbytes + ps.rvo.nbytes + ps.xy.nbytes)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Voronoi parcels; the reference's parcel datasets are private)",
            "config": {"workload": WORKLOAD, "parcels": int(ps.n), "vertices": int(ps.nv), "candidates": int(r["count"]["cand"]),
                       "pairs_per_step": int(pairs), "parallelism": "replicas x1 (own layer per rank)", "l2": "inputs > L2 (2.2 GB resident layer)"},
            "reference_engine": {"driver": "landstats-us/postgis-cuda engine/harness.cu, unmodified, nvcc -arch=sm_100a",
                                 "command": "harness parcels.gset parcels.gset --relate --reps %d" % reps, "processes": runs,
                                 "phases_ms": r["ms"], "counts": r["count"], "gpu_ms_per_process": gms,
                                 "timing": "the driver's own stats of its second (warm) repetition: GPU phases traverse + refine + "
                                           "compact; the median over the processes"},
            "e2e": {"value": pairs / (e2e_ms / 1000.0), "unit": "pairs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(pairs * 12),
                    "ms_per_step": e2e_ms, "what": "upload (host prep + H2D) + BVH + join + D2H, the driver's own timers"},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"the reference engine's driver on this box's GPU (host threads for its prep: {os.cpu_count()}); "
                                       f"relate self-join of {ps.n} parcels, the warm repetition, median of {runs} processes"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_reference_op(args, RH):
    """--impl reference --op X: the reference engine's driver on the layers `--op X` uses (rank 0's seeds). area: cfg1's
    20k zones x 50 zones; dwithin: 1M points x 1M parcels at 5 m; cluster: the cfg5 layer; erode: the cfg5 layer against
    an independently seeded one (the driver's self-join drops a geometry's pair with itself, so the two-layer form is
    the one both engines define alike: the `non_degenerate` leg of `--op erode`). value = units / its GPU phase time
    (traverse + refine + compact) of the warm repetition, median over up to 5 (cfg5: 3) driver processes."""
    import shutil
    import tempfile
    from gsj import gen
    op = args.op
    d = tempfile.mkdtemp(prefix="gsj_refop_")
    try:
        if op == "area":
            A, B = gen.layer_cfg_parcels_small(20000, seed=0), gen.layer_cfg_zones(50, seed=1)
            fa, fb = os.path.join(d, "a.gset"), os.path.join(d, "b.gset")
            gen.write_gset(fa, A); gen.write_gset(fb, B)
            cmd, unit, key, work = [fa, fb, "--area"], "pairs/s", "gpu_hits", "intersects + area, 20k Voronoi zones x 50 zones"
        elif op == "dwithin":
            box = (-119.0, 33.0, -118.0, 34.0)
            fp, fb = os.path.join(d, "p.pset"), os.path.join(d, "b.gset")
            gen.write_pset(fp, gen.points(1_000_000, box, 7)); gen.write_gset(fb, gen.layer_parcels(1_000_000, box, seed=0))
            cmd, unit, key, work = [fp, fb, "--dwithin", "5"], "pairs/s", "rows", "ST_DWithin 5 m, 1M points x 1M parcels"
        else:
            n = args.seeds or 20_000_000
            side = 2.0 * (n / 2e6) ** 0.5
            box = (-119.0, 33.0, -119.0 + side, 33.0 + side)
            fa = os.path.join(d, "a.gset")
            la = gen.layer_cfg5(n, box, seed=0)
            gen.write_gset(fa, la)
            n = int(la.n)   # parcels of the layer (the seeds' cells)
            del la
            if op == "erode":
                fb = os.path.join(d, "b.gset")
                gen.write_gset(fb, gen.layer_cfg5(n, box, seed=1))
                cmd, unit, key = [fa, fb, "--erode", "1"], "pairs/s", "rows"
                work = f"erosion (1 m) of a {n / 1e6:g}M-parcel layer against an independently seeded one"
            else:
                cmd, unit, key = [fa, fa, "--cluster"], "parcels/s", None
                work = f"ST_ClusterIntersecting, {n / 1e6:g}M parcels"
        runs = max(1, min(args.steps, 5 if op in ("area", "dwithin") else 3))
        with Clocks(0) as clk:
            rs = [RH.run(cmd, reps=2, timeout=3600) for _ in range(runs)]
    except (RuntimeError, OSError, subprocess.TimeoutExpired) as e:
        why = str(e).strip().splitlines()[-1][:300] if str(e).strip() else type(e).__name__
        print(json.dumps({"impl": "reference", "unavailable": f"the reference engine's driver did not run: {why}"}), flush=True)
        return
    finally:
        shutil.rmtree(d, ignore_errors=True)
    # GPU phases as the driver reports them; clustering adds its union-find (gsj's cluster time includes its own)
    gms = [RH.gpu_ms(r) + (r["ms"].get("union-find", 0.0) if op == "cluster" else 0.0) for r in rs]
    k = int(np.argsort(gms)[len(gms) // 2])
    r, ms = rs[k], gms[k]
    units = r["count"][key] if key else n
    line = {"impl": "reference", "metric": f"{unit} ({op})", "value": units / (ms / 1000.0), "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded Voronoi parcels / uniform points)", "config": {"workload": work, "units_per_step": int(units)},
            "reference_engine": {"driver": "landstats-us/postgis-cuda engine/harness.cu, unmodified, nvcc -arch=sm_100a",
                                 "command": "harness " + " ".join(os.path.basename(x) if x.endswith("set") else x for x in cmd) + " --reps 2",
                                 "processes": runs, "phases_ms": r["ms"], "counts": r["count"], "gpu_ms_per_process": gms},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seeds", type=int, default=None, help="parcels (default 2M; 20M for --op erode / cluster)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-s", type=float, default=0.0, help="CPU seconds per reference-arm step (0: sized from --steps)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-latency leg (gsjd under a Poisson request stream)")
    ap.add_argument("--no-reference-check", action="store_true", help="skip the row-by-row comparison with the reference engine's driver")
    ap.add_argument("--serve-small", action="store_true", help="the serving leg on a scaled-down copy of its workload (quick runs)")
    ap.add_argument("--no-tune", action="store_true", help="skip the refinement autotuner: the default launch shape (profiling)")
    ap.add_argument("--op", default="relate", choices=["relate", "area", "dwithin", "erode", "cluster"])
    ap.add_argument("--arms", default="filtered,plain", help="refinement variants an --op run times (filtered first; for profiling one)")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: every rank joins the same layer, each its shard of the probes (strong scaling) instead of its own layer")
    args = ap.parse_args()
    if args.seeds is None and args.op == "relate":
        args.seeds = N_SEEDS
    rank, local, ws = dist_setup()
    if args.impl == "reference":
        run_reference(args, rank, ws)
        barrier(ws)
        return
    if args.op != "relate":
        run_op(args, rank, local, ws)
        barrier(ws)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    import gsj
    from gsj import gen

    torch.cuda.set_device(local)
    eng = gsj.Engine(local)
    ext = torch.cuda.ExternalStream(eng.stream_handle(), device=local)
    t0 = time.time()
    shard = dict(shard=rank, nshards=ws) if (args.shard and ws > 1) else {}
    ps = gen.layer_parcels(args.seeds, BOX, seed=0 if shard else rank)
    t_gen = time.time() - t0
    # pinned host copies for the end-to-end leg
    pin = {k: torch.from_numpy(np.ascontiguousarray(getattr(ps, k))).pin_memory() for k in ("gro", "rvo", "xy")}
    hps = gen.PolygonSet(pin["gro"].numpy(), pin["rvo"].numpy(), pin["xy"].numpy())
    L = eng.upload_polygons(hps)

    def timed_join(mode):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            e0.record()
        r = eng.join(L, L, want_area=False, want_relate=True, upper=True, refine_mode=mode, collect=False, **shard)
        with torch.cuda.stream(ext):
            e1.record()
        e1.synchronize()
        return r, e0.elapsed_time(e1)

    # untimed: the refinement autotuner picks the filtered variant's launch shape on a sample of this join's
    # candidate pairs; the plain variant runs with the default shape (the reference's fixed scheme)
    default_shape = eng.refine_shape
    tune = ({"best": default_shape, "start_ms": None, "best_ms": None, "sample_pairs": 0, "shapes_tried": 0} if args.no_tune else
            eng.tune_refine(L, L, want_area=False, want_relate=True, refine_mode=gsj.GSJ_REFINE_FILTERED, max_pairs=1 << 21))
    for _ in range(args.warmup):
        timed_join(gsj.GSJ_REFINE_FILTERED)
    res = {}
    for mode, name in ((gsj.GSJ_REFINE_FILTERED, "filtered"), (gsj.GSJ_REFINE_PLAIN, "plain")):
        eng.refine_shape = tune["best"] if name == "filtered" else default_shape
        if name == "plain":
            timed_join(mode)   # warm this variant too
        barrier(ws)
        torch.cuda.synchronize()
        ms, pairs, stats = [], 0, []
        with Clocks(local) as clk:
            for _ in range(args.steps):
                r, t = timed_join(mode)
                ms.append(t); pairs += r.stats["hits"]; stats.append(r.stats)
        torch.cuda.synchronize()
        barrier(ws)
        res[name] = dict(ms=ms, pairs=pairs, stats=stats, clocks=clk.summary())
    eng.refine_shape = tune["best"]
    # checks (untimed): the rows of both variants, compared with each other and with the reference engine's
    a = eng.join(L, L, want_area=False, want_relate=True, upper=True, refine_mode=gsj.GSJ_REFINE_FILTERED, **shard)
    b = eng.join(L, L, want_area=False, want_relate=True, upper=True, refine_mode=gsj.GSJ_REFINE_PLAIN, **shard)
    ia, ib = np.lexsort(a.pairs.T[::-1]), np.lexsort(b.pairs.T[::-1])
    same_pairs = a.pairs.shape == b.pairs.shape and np.array_equal(a.pairs[ia], b.pairs[ib])
    pair_diffs = 0 if same_pairs else len(set(map(tuple, a.pairs.tolist())) ^ set(map(tuple, b.pairs.tolist())))
    code_diffs = int((a.code[ia] != b.code[ib]).sum()) if same_pairs else None
    refcheck = None
    if rank == 0 and not shard and not args.no_reference_check:
        import shutil
        import tempfile
        d = tempfile.mkdtemp(prefix="gsj_refcheck_")
        try:
            refcheck = reference_check(ps, a, d)
        finally:
            shutil.rmtree(d, ignore_errors=True)
    del b

    # end-to-end through the C ABI from pinned host buffers: upload + LBVH + join + D2H of the rows
    e2e_ms, e2e_pairs, e2e_parts = [], 0, []
    for i in range(1 + args.steps):
        t = time.perf_counter()
        Lx = eng.upload_polygons(hps)   # returns after the layer and its LBVH are on the device
        t1 = time.perf_counter()
        r = eng.join(Lx, Lx, want_area=False, want_relate=True, upper=True, **shard)
        t2 = time.perf_counter()
        Lx.free()
        dt = (time.perf_counter() - t) * 1000.0
        if i:
            e2e_ms.append(dt); e2e_pairs += len(r.pairs)
            e2e_parts.append(((t1 - t) * 1000.0, (t2 - t1) * 1000.0))
    h2d = int(ps.gro.nbytes + ps.rvo.nbytes + ps.xy.nbytes)
    d2h = int(len(r.pairs) * 12)

    f = res["filtered"]
    value, tot_ms = aggregate(float(np.sum(f["ms"])), float(f["pairs"]), ws)
    plain_value, plain_ms = aggregate(float(np.sum(res["plain"]["ms"])), float(res["plain"]["pairs"]), ws)
    e2e_value, e2e_tot = aggregate(float(np.sum(e2e_ms)), float(e2e_pairs), ws)
    pk = peaks()
    st = f["stats"]
    refine_ms = float(np.mean([s["refine_ms"] for s in st]))
    trav_ms = float(np.mean([s["traverse_ms"] for s in st]))
    hbm = pk.get("hbm_gbs", 6650.0)
    # roofline of the dominant kernel (refinement), FP64-bound: algorithmic flops = the local edge pairs (na x nb per
    # refined pair, counted by the kernels) x FLOPS_PER_EDGE_PAIR; its HBM figure = both geometries' vertices per pair
    edge_pairs = float(np.mean([s["edge_pairs"] for s in st]))
    flops = edge_pairs * FLOPS_PER_EDGE_PAIR
    cand = eng.candidates(L, L, upper=True)
    nvg = (ps.rvo[ps.gro[1:]] - ps.rvo[ps.gro[:-1]]).astype(np.int64)
    alg_bytes = float(16 * (nvg[cand[:, 0]] + nvg[cand[:, 1]]).sum() + len(cand) * (8 + 1 + 32 + 4 + 2 * 40))
    # traversal: 48-byte node records visited + probe box and order id + written pairs (mostly served from L2)
    trav_bytes = float(np.mean([s_["node_visits"] for s_ in st]) * 48 + ps.n * (16 + 4) + len(cand) * 8)
    traffic = None
    try:
        for ln in open(os.path.join(ROOT, "profiles", "traffic_per_launch.txt")):
            k, v = ln.split()[:2]
            if k == "k_refine":   # DRAM bytes per candidate pair from one ncu pass over this join, times its candidate pairs
                traffic = float(v) * float(st[0]["candidates"])
    except OSError:
        pass
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, info = cpu_oracle_rate(ps)
        cpu = {"value": v, "unit": "pairs/s", "cores": info["threads"], "kind": "port",
               "sample": f"CPU FP64 oracle, relate self-join of {info['parcels']} parcels in a {info['box_deg']:.3f} deg corner sub-box "
                         f"({info['pairs']} pairs, {info['seconds']:.1f} s)"}
    lat = sorted(f["ms"])
    serving = None
    if rank == 0 and not args.no_serve:
        serving = serving_leg(SERVE_SMALL if args.serve_small else SERVE)
    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "strong" if shard else "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Voronoi parcels; the reference's parcel datasets are private)",
        "config": {"workload": WORKLOAD, "parcels": int(L.info["n"]), "vertices": int(L.info["nv"]), "candidates": int(st[0]["candidates"]),
                   "pairs_per_step": int(st[0]["hits"]),
                   "parallelism": f"probe shards x{ws} (one layer, R replicated)" if shard else f"replicas x{ws} (own layer per rank)",
                   "l2": "inputs > L2 (2.2 GB resident layer)"},
        "gen_s": round(t_gen, 2),
        "refine_shape": {"filtered": tune["best"], "plain": default_shape, "autotuner": {k: tune[k] for k in ("start_ms", "best_ms", "sample_pairs", "shapes_tried")},
                         "what": "launch shape of the refinement's two size bins; the filtered one chosen by gsj_tune_refine (untimed)"},
        "latency_ms": ({"p50": serving["filtered"]["p50_ms"], "p99": serving["filtered"]["p99_ms"],
                        "plain_p50": serving["plain"]["p50_ms"], "plain_p99": serving["plain"]["p99_ms"],
                        "what": "gsjd serving the request stream, arrival to end of result stream"} if serving else None),
        "step_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "serving": serving,
        "plain_fp64": {"value": plain_value, "ms_per_step": plain_ms / args.steps,
                       "latency_ms": {"p50": float(np.percentile(res["plain"]["ms"], 50)), "p99": float(np.percentile(res["plain"]["ms"], 99))},
                       "speedup_filtered": value / plain_value},
        "pair_diffs_filtered_vs_plain": pair_diffs, "code_diffs_filtered_vs_plain": code_diffs,
        "pair_diffs_vs_reference": (refcheck or {}).get("pair_diffs"), "code_diffs_vs_reference": (refcheck or {}).get("code_diffs"),
        "reference_check": refcheck,
        "phases_ms": {k: float(np.mean([s[k] for s in st])) for k in ("traverse_ms", "refine_ms", "compact_ms", "copy_ms")},
        "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_tot / args.steps,
                "parts_ms": {"upload_and_lbvh": float(np.mean([a for a, _ in e2e_parts])),
                             "join_and_rows_to_host": float(np.mean([b for _, b in e2e_parts])),
                             "what": "host clock: gsj_layer_upload_polygons (H2D of the arrays, device prep, LBVH), then gsj_join with the "
                                     "rows copied out of the library's pinned buffers"}},
        "roofline": {"kernel": "k_refine<1> + k_refine_self + k_refine_scratch<1> (the refinement graph)", "bound": "fp64", "achieved": flops / (refine_ms / 1000.0) / 1e12,
                     "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": flops / (refine_ms / 1000.0) / 1e12 / FP64_PEAK_TFLOPS,
                     "traffic": traffic, "peak_source": "B200 FP64 specification (HGX B200: 296 TFLOPS / 8 GPUs); not measured here",
                     "work": {"edge_pairs_per_launch": edge_pairs, "flops_per_edge_pair": FLOPS_PER_EDGE_PAIR,
                              "what": "local edge pairs na x nb of every refined pair (the reference's brute-force unit), counted in the kernels"},
                     "hbm": {"achieved_gbs": alg_bytes / (refine_ms / 1000.0) / 1e9, "peak_gbs": hbm,
                             "frac": alg_bytes / (refine_ms / 1000.0) / 1e9 / hbm,
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in pk else "fallback",
                             "bytes": "both geometries' vertices per candidate pair + per-pair outputs"}},
        "roofline_traversal": {"kernel": "k_traverse", "bound": "l2/hbm latency", "what": "visited LBVH node bytes per second (mostly L2 hits)",
                               "achieved": trav_bytes / (trav_ms / 1000.0) / 1e9, "unit": "GB/s", "hbm_peak": hbm,
                               "node_bytes_over_hbm_peak": trav_bytes / (trav_ms / 1000.0) / 1e9 / hbm},
        "gpu_launches": int(sum(s["launches"] for s in st)),
        "clocks": f["clocks"],
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(ws)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
