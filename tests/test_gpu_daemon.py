"""gsjd end to end on the GPU: layers loaded from files over the wire protocol, every op's rows against the CPU
oracle expanded by the reference daemon's row rules (oracle/rows.py), the reference engine's golden outputs, stats
mode, concurrent requests and a client that goes away mid-stream."""
import concurrent.futures as cf
import math
import socket
import struct

import numpy as np
import pytest

import gsj
import make_golden as MG
import pgcopy
import pyoracle as O
import rows as RR
from gsj import client as C
from gsj import daemon as D
from gsj import gen
from gsj.gen import PolygonSet

pytestmark = pytest.mark.gpu
DE9_INTERIOR = 1 | 3 << 12 | 2 << 14 | 3 << 16
DE9_BOUNDARY = 1 << 2 | 3 << 12 | 2 << 14 | 3 << 16


def with_duplicates(ps, idx):
    """ps with copies of geometries idx appended (identical coordinates: dedup groups)."""
    gro, rvo, xy = list(ps.gro), list(ps.rvo), [ps.xy]
    nv = len(ps.xy)
    for g in idx:
        r0, r1 = int(ps.gro[g]), int(ps.gro[g + 1])
        v0 = int(ps.rvo[r0])
        for r in range(r0, r1):
            rvo.append(nv + int(ps.rvo[r + 1]) - v0)
        nv += int(ps.rvo[r1]) - v0
        xy.append(ps.xy[v0:int(ps.rvo[r1])])
        gro.append(len(rvo) - 1)
    return PolygonSet(np.array(gro, np.uint64), np.array(rvo, np.uint64), np.concatenate(xy))


class Env:
    pass


@pytest.fixture(scope="module")
def env(tmp_path_factory):
    e = Env()
    d = tmp_path_factory.mktemp("gsjd")
    e.dir = d
    L = {k: b() for k, (kind, b) in MG.layers().items()}
    e.golden = L
    rng = np.random.default_rng(11)
    base = L["parcels"]
    e.dups = rng.choice(base.n, 150, replace=False)
    e.parcels = with_duplicates(base, e.dups)
    e.pids = [f"p{g}" for g in range(e.parcels.n)]
    pgcopy.write_copy(str(d / "parcels.copy"), pgcopy.polygonset_rows(e.parcels, e.pids, reverse_every=5))
    e.u, e.moff, e.midx = gsj.dedup(e.parcels)
    gen.write_gset(str(d / "parcels2.gset"), L["parcels2"])
    gen.write_gset(str(d / "gparcels.gset"), base)
    gen.write_gset(str(d / "zonesA.gset"), L["zonesA"])
    gen.write_pset(str(d / "points.pset"), L["points"])
    e.sock = str(d / "gsjd.sock")
    e.log = open(d / "gsjd.log", "w")
    e.proc = D.start(e.sock, str(d), workers=3, log=e.log)
    e.cl = C.Client(e.sock)
    e.info = {
        "parcels": e.cl.load("parcels", "parcels.copy"),
        "parcels_sub": e.cl.load("parcels_sub", "parcels.copy", subdivide=32),
        "parcels2": e.cl.load("parcels2", "parcels2.gset"),
        "gparcels": e.cl.load("gparcels", "gparcels.gset", dedup=False),
        "zonesA": e.cl.load("zonesA", "zonesA.gset", dedup=False),
        "points": e.cl.load("points", "points.pset"),
    }
    e.O = {"u": O.OSet(e.u), "p2": O.OSet(L["parcels2"])}
    yield e
    D.stop(e.proc)
    e.log.close()


def rowset(rows):
    return {(a, b): v for a, b, v in rows}


def expect_pairs(pairs, vals, ma, mb, ida, idb, same, distinct, tr=None):
    out = {}
    for ra, rb, i, t in RR.expand(pairs, ma, mb, same, distinct):
        v = vals[i] if vals is not None else None
        if tr is not None and t:
            v = tr(v)
        out[(ida[ra], idb[rb])] = v
    return out


def test_load_and_layers(env):
    i = env.info["parcels"]
    assert i["rows"] == env.parcels.n and i["distinct"] == env.u.n and i["dedup"] is True and i["kind"] == "polygon"
    assert env.info["parcels_sub"]["gpu_geoms"] > env.info["parcels_sub"]["distinct"] == env.u.n
    assert env.info["points"]["kind"] == "point" and env.info["points"]["rows"] == len(env.golden["points"])
    names = [x["layer"] for x in env.cl.list()]
    assert {"parcels", "parcels2", "points"} <= set(names)
    st = env.cl.status()
    assert st["cc"] == "10.0" and st["workers"] == 3 and "parcels" in st["layers"]


@pytest.mark.parametrize("distinct", [False, True])
def test_join_self(env, distinct):
    rows, st = env.cl.join("parcels", "parcels", want_area=True, self_pairs="distinct" if distinct else "all")
    p, a, c, _ = O.join(env.O["u"], env.O["u"], O.params(1, 0), upper=True)
    m = (env.moff, env.midx)
    want = expect_pairs(p, a, m, m, env.pids, env.pids, True, distinct)
    got = rowset(rows)
    assert len(rows) == len(got) == st["rows"]
    assert got.keys() == want.keys()
    assert all(got[k] == want[k] for k in want)   # areas bit-identical to the oracle's
    s_rows, s_st = env.cl.join("parcels", "parcels", want_area=True, self_pairs="distinct" if distinct else "all", stats_only=True)
    assert s_rows == [] and s_st["rows"] == len(rows) and s_st["stats_only"] is True
    assert math.isclose(s_st["area_sum"], sum(v for _, _, v in rows), rel_tol=1e-5)


def test_join_two_layers_and_subdivided(env):
    rows, st = env.cl.join("parcels", "parcels2", want_area=False, self_pairs="all")
    p, a, c, _ = O.join(env.O["u"], env.O["p2"], O.params(1, 0))
    want = expect_pairs(p, None, (env.moff, env.midx), (None, None), env.pids, [str(i) for i in range(env.golden["parcels2"].n)], False, False)
    got = rowset(rows)
    assert got.keys() == want.keys() and all(math.isnan(v) for v in got.values())
    sub, _ = env.cl.join("parcels_sub", "parcels2", want_area=True, self_pairs="all")
    assert rowset(sub).keys() == want.keys()


def test_points(env):
    pts = env.golden["points"]
    p, w, _ = O.pip(pts, env.O["u"])
    pid = [str(i) for i in range(len(pts))]
    rows, st = env.cl.join("points", "parcels", want_area=True)
    want = expect_pairs(p, None, (None, None), (env.moff, env.midx), pid, env.pids, False, False)
    assert rowset(rows).keys() == want.keys() and all(v == 0.0 for _, _, v in rows)
    rows, st = env.cl.join("parcels", "points", want_area=False)   # swapped: (polygon id, point id)
    assert {(b, a) for a, b, _ in rows} == set(want.keys())
    codes = np.where(w == 2, DE9_BOUNDARY, DE9_INTERIOR)
    rel, _ = env.cl.relate("parcels", "points")
    wantr = {(b, a): O.de9im_str(O.de9im_transpose(int(v))) for (a, b), v in expect_pairs(p, codes, (None, None), (env.moff, env.midx), pid, env.pids, False, False).items()}
    assert rowset(rel) == wantr


@pytest.mark.parametrize("pattern,distinct", [("", False), ("", True), ("T*T***T**", True), ("2FFF1FFF2", False)])
def test_relate_self(env, pattern, distinct):
    rows, st = env.cl.relate("parcels", "parcels", pattern, "distinct" if distinct else "all")
    p, a, c, _ = O.join(env.O["u"], env.O["u"], O.params(0, 1), upper=True)
    m = (env.moff, env.midx)
    want = expect_pairs(p, c, m, m, env.pids, env.pids, True, distinct, tr=O.de9im_transpose)
    want = {k: O.de9im_str(int(v)) for k, v in want.items() if not pattern or O.de9im_match(int(v), pattern)}
    assert rowset(rows) == want and len(rows) == len(want)


def test_cluster(env):
    rows, st = env.cl.cluster("parcels")
    root = O.cluster(env.O["u"], env.u.n)
    lab = RR.cluster_labels(root, env.moff, env.midx, env.parcels.n)
    assert [r[0] for r in rows] == env.pids and [r[1] for r in rows] == lab and st["clusters"] == len(set(lab))


def test_dwithin_and_buffer(env):
    m = (env.moff, env.midx)
    ids2 = [str(i) for i in range(env.golden["parcels2"].n)]
    rows, _ = env.cl.dwithin("parcels", "parcels", 5.0, "distinct")
    p, _ = O.dwithin(env.O["u"], env.O["u"], 5.0, same=True)
    assert set(rowset(rows)) == set(expect_pairs(p, None, m, m, env.pids, env.pids, True, True))
    rows, _ = env.cl.intersects_buffered("parcels", "parcels2", 2.0, 3.0)   # both >= 0: dwithin(5)
    p, _ = O.dwithin(env.O["u"], env.O["p2"], 5.0)
    assert set(rowset(rows)) == set(expect_pairs(p, None, m, (None, None), env.pids, ids2, False, False))
    rows, _ = env.cl.intersects_buffered("parcels", "parcels2", -1.0, -3.0)
    p = O.erode(env.O["u"], env.O["p2"], 1.0, 3.0)
    assert set(rowset(rows)) == set(expect_pairs(p, None, m, (None, None), env.pids, ids2, False, False)) and len(rows) > 0
    need = (np.diff(env.moff) > 1).astype(np.uint8)
    rows, _ = env.cl.intersects_buffered("parcels", "parcels", -1.0, -1.0, "distinct")
    p = O.erode(env.O["u"], env.O["u"], 1.0, 1.0, same=True, need_self=need)
    want = set(expect_pairs(p, None, m, m, env.pids, env.pids, True, True))
    n0 = env.golden["parcels"].n   # copies of geometry g were appended as rows n0 + k: their self pairs are needed
    assert set(rowset(rows)) == want and any((f"p{g}", f"p{n0 + k}") in want for k, g in enumerate(env.dups))
    pts = env.golden["points"]
    pid = [str(i) for i in range(len(pts))]
    rows, _ = env.cl.intersects_buffered("parcels", "points", -3.0, 0.0)   # swapped, polygon side eroded
    p = O.pt_erode(pts, env.O["u"], 3.0)
    assert {(b, a) for a, b, _ in rows} == set(expect_pairs(p, None, (None, None), m, pid, env.pids, False, False))
    with pytest.raises(C.GspError, match="negative buffer"):
        env.cl.intersects_buffered("points", "parcels", -1.0, -1.0)
    with pytest.raises(C.GspError, match="opposite sign"):
        env.cl.intersects_buffered("parcels", "parcels2", -1.0, 1.0)
    _, st = env.cl.dwithin("parcels", "parcels2", 5.0, stats_only=True)
    assert st["stats_only"] is True and st["rows"] > 0


def test_reference_golden_rows(env):
    """Self-join rows ("all") of the reference harness: relate codes and areas on layers loaded as files."""
    rows, _ = env.cl.relate("gparcels", "gparcels", "", "all")
    g = np.load(f"{MG.HERE}/pp_relate.npz")
    want = {(str(a), str(b)): r for (a, b), r in zip(g["pairs"].tolist(), g["relate"].tolist())}
    assert rowset(rows) == want
    rows, _ = env.cl.join("zonesA", "zonesA", want_area=True, self_pairs="all")
    g = np.load(f"{MG.HERE}/aa_area.npz")
    got = rowset(rows)
    want = {(str(a), str(b)): v for (a, b), v in zip(g["pairs"].tolist(), g["area"].tolist())}
    assert got.keys() == want.keys()
    big = [k for k, v in want.items() if abs(v) > 1e-12]
    assert max(abs(got[k] - want[k]) / abs(want[k]) for k in big) <= 1e-9


def same_value(a, b):
    """Row payloads equal bit for bit (areas as float64 words, NaN for rows without an area; DE-9IM strings)."""
    if isinstance(a, float) and isinstance(b, float):
        return struct.pack("<d", a) == struct.pack("<d", b) or (math.isnan(a) and math.isnan(b))
    return a == b


def test_concurrent_requests(env):
    """Each result is the same alone and in the mix: the same rows with the same areas and DE-9IM matrices, bit for
    bit, whether a request runs by itself or while 15 others of every kind run on the device beside it."""
    calls = [lambda: env.cl.join("parcels", "parcels2", True, "all"), lambda: env.cl.relate("parcels", "parcels", "", "distinct"),
             lambda: env.cl.dwithin("parcels", "parcels2", 5.0), lambda: env.cl.join("points", "parcels", False),
             lambda: env.cl.relate("parcels", "parcels2", "", "all"), lambda: env.cl.join("parcels2", "parcels", True, "all")]
    serial = [rowset(f()[0]) for f in calls]
    assert all(len(r) > 0 for r in serial)
    with cf.ThreadPoolExecutor(12) as ex:
        futs = [ex.submit(calls[i % len(calls)]) for i in range(4 * len(calls))]
        for i, f in enumerate(futs):
            got, ref = rowset(f.result()[0]), serial[i % len(calls)]
            assert got.keys() == ref.keys()
            assert all(same_value(got[k], ref[k]) for k in ref)


def test_client_gone_and_drop(env):
    s = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
    s.connect(env.sock)
    s.sendall(C.encode_request(C.OP_JOIN, ["parcels", "parcels", "1", "all"]))
    s.recv(16)
    s.close()   # mid-stream
    rows, st = env.cl.join("parcels", "parcels2", True)
    assert st["rows"] == len(rows) > 0
    env.cl.load("tmp", "parcels2.gset")
    assert env.cl.drop("tmp") is True and env.cl.drop("tmp") is False
    with pytest.raises(C.GspError, match="no such layer"):
        env.cl.join("tmp", "parcels")
    with pytest.raises(C.GspError, match="point x point"):
        env.cl.join("points", "points")
    with pytest.raises(C.GspError, match="pattern"):
        env.cl.relate("parcels", "parcels", "T*T", "all")


def test_stream_batches_same_rows(env):
    """The same rows (pairs, bit-identical areas, DE-9IM strings) for every streamed op from: one batch encoded on the
    device (the default), probe batches of 64 query geometries encoded on the host by a sender thread while the
    engine refines the next batch, and one batch encoded on the host."""
    def norm(rows):
        return sorted(tuple(-1.0 if isinstance(x, float) and math.isnan(x) else x for x in r) for r in rows)

    res, procs = {}, []
    try:
        for sb, flags in ((0, []), (64, ["--stream-batch", "64"]), (1, ["--gpu-encode", "0"])):
            sock = str(env.dir / f"gsjd_sb{sb}.sock")
            log = open(env.dir / f"gsjd_sb{sb}.log", "w")
            procs.append((D.start(sock, str(env.dir), workers=2, log=log, extra=flags), log))
            cl = C.Client(sock)
            cl.load("parcels", "parcels.copy")
            cl.load("parcels_sub", "parcels.copy", subdivide=32)
            cl.load("parcels2", "parcels2.gset")
            cl.load("points", "points.pset")
            res[sb] = [norm(rows) for rows, _ in (
                cl.join("parcels", "parcels", True, "all"), cl.join("parcels", "parcels", False, "distinct"),
                cl.join("parcels_sub", "parcels2", True), cl.join("points", "parcels", False),
                cl.join("parcels", "points", True), cl.relate("parcels", "parcels", "", "all"),
                cl.relate("points", "parcels_sub", "", "all"), cl.dwithin("parcels", "parcels2", 5.0),
                cl.dwithin("points", "parcels", 5.0), cl.intersects_buffered("parcels", "parcels2", 2.0, 1.0),
                cl.intersects_buffered("parcels", "parcels", -1.0, -1.0, "distinct"))]
    finally:
        for p, log in procs:
            D.stop(p)
            log.close()
    assert env.info["points"]["rows"] > 64 * 8 and env.info["parcels"]["rows"] > 64 * 8   # many batches
    for a, b, c in zip(res[0], res[64], res[1]):
        assert a == b == c and len(a) > 0


def test_snapshots_restore_layers(env, tmp_path):
    """--snapshot-dir: a restarted daemon restores every loaded layer (deduplicated, subdivided, points) from its
    snapshot, without the source files, and answers with the same rows; a dropped layer is not restored."""
    snap = tmp_path / "snap"
    snap.mkdir()

    def start(tag):
        log = open(env.dir / f"gsjd_snap_{tag}.log", "w")
        sock = str(env.dir / f"gsjd_snap_{tag}.sock")
        return D.start(sock, str(env.dir), workers=2, log=log, extra=["--snapshot-dir", str(snap)]), log, C.Client(sock)

    def info(cl):
        return sorted((x["layer"], x["kind"], x["rows"], x["distinct"], x["gpu_geoms"], x["dedup"]) for x in cl.list())

    def queries(cl):   # NaN payloads (dwithin rows) compared as a marker: NaN != NaN
        return [sorted(tuple(-1.0 if isinstance(v, float) and math.isnan(v) else v for v in r) for r in rows) for rows, _ in (cl.join("parcels", "parcels", True, "all"), cl.join("parcels_sub", "parcels2", True),
                                             cl.relate("points", "parcels", "", "all"), cl.dwithin("parcels", "parcels2", 5.0))]

    p, log, cl = start("a")
    try:
        cl.load("parcels", "parcels.copy")
        cl.load("parcels_sub", "parcels.copy", subdivide=32)
        cl.load("parcels2", "parcels2.gset")
        cl.load("points", "points.pset")
        cl.load("gone", "parcels2.gset")
        want = queries(cl)
        assert cl.drop("gone") is True
        layers = info(cl)
    finally:
        D.stop(p)
        log.close()
    assert len(list(snap.glob("*.gsnap"))) == 4
    p, log, cl = start("b")
    try:
        assert info(cl) == layers and [x[0] for x in layers] == ["parcels", "parcels2", "parcels_sub", "points"]
        assert queries(cl) == want and all(len(w) > 0 for w in want)
    finally:
        D.stop(p)
        log.close()


def test_tune_at_load_same_rows(env):
    """--tune 1: loading a polygon layer of >= 100k geometries runs the refinement autotuner (logged) and every
    context takes the chosen launch shape; the rows are the same as without it."""
    big = gen.layer_parcels(120_000, (-118.6, 33.7, -118.0, 34.3), seed=21)
    gen.write_gset(str(env.dir / "big.gset"), big)
    logp = env.dir / "gsjd_tune.log"
    log = open(logp, "w")
    sock = str(env.dir / "gsjd_tune.sock")
    p = D.start(sock, str(env.dir), workers=2, log=log, extra=["--tune", "1"])
    try:
        cl = C.Client(sock)
        cl.load("big", "big.gset", dedup=False)
        got = sorted(cl.join("big", "big", True, "distinct")[0])
        got_rel = sorted(cl.relate("big", "big", "", "distinct")[0])
    finally:
        D.stop(p)
        log.close()
    env.cl.load("big", "big.gset", dedup=False)
    try:
        want = sorted(env.cl.join("big", "big", True, "distinct")[0])
        want_rel = sorted(env.cl.relate("big", "big", "", "distinct")[0])
    finally:
        env.cl.drop("big")
    text = logp.read_text()
    assert "tune big: shape run=4 runs=32 " in text, text[-2000:]   # the block-lifetime fields stay at their defaults
    assert got == want and got_rel == want_rel and len(want) > 100_000
