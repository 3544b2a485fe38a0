"""The serving daemon's host side without a GPU: row rules against the oracle restatement of gpujoind.cu, layer
files (binary COPY with EWKB, .gset/.pset), and the wire protocol (framing limits, auth, errors, no-GPU LOAD)."""
import os
import socket
import struct

import numpy as np
import pytest

import pgcopy
import rows as R
from gsj import client as C
from gsj import daemon as D
from gsj import gen


def random_members(rng, n_rows):
    """A dedup-style member map: distinct geometries in first-occurrence order, some with several rows."""
    rep = np.arange(n_rows)
    for i in range(1, n_rows):
        if rng.random() < 0.3:
            rep[i] = rep[rng.integers(0, i)]
    first = {}
    for i in range(n_rows):
        first.setdefault(rep[i], len(first))
    groups = [[] for _ in first]
    for i in range(n_rows):
        groups[first[rep[i]]].append(i)
    moff = np.cumsum([0] + [len(g) for g in groups]).astype(np.uint64)
    midx = np.array([r for g in groups for r in g], np.uint32)
    return moff, midx


@pytest.mark.parametrize("same,distinct,dedup", [(False, False, False), (False, False, True), (True, False, False), (True, False, True),
                                                 (True, True, False), (True, True, True)])
def test_row_rules(same, distinct, dedup):
    rng = np.random.default_rng(7)
    ma = random_members(rng, 40) if dedup else (None, None)
    nA = 40 if ma[0] is None else len(ma[0]) - 1
    if same:
        mb, nB = ma, nA
        pairs = np.array([(a, b) for a in range(nA) for b in range(a, nA) if rng.random() < 0.2], np.uint32)
    else:
        mb = random_members(rng, 25) if dedup else (None, None)
        nB = 25 if mb[0] is None else len(mb[0]) - 1
        pairs = np.array([(a, b) for a in range(nA) for b in range(nB) if rng.random() < 0.2], np.uint32)
    rows, src, tr = D.expand_rows(pairs, same, distinct, *ma, *mb)
    want = R.expand(pairs, ma, mb, same, distinct)
    assert [(int(a), int(b), int(s), bool(t)) for (a, b), s, t in zip(rows, src, tr)] == [(a, b, i, t) for a, b, i, t in want]
    assert D.count_rows(pairs, same, distinct, ma[0], mb[0]) == len(want) == sum(R.row_count(int(a), int(b), ma, mb, same, distinct) for a, b in pairs)
    if same and distinct:
        assert all(a < b for a, b in rows.tolist())
    if same and not distinct:   # "all" is symmetric
        s = set(map(tuple, rows.tolist()))
        assert all((b, a) in s for a, b in s)


def test_cluster_labels():
    rng = np.random.default_rng(3)
    moff, midx = random_members(rng, 60)
    nd = len(moff) - 1
    root = np.array([min(g, int(rng.integers(0, g + 1))) for g in range(nd)], np.uint32)
    root = np.array([root[r] if root[r] <= g else g for g, r in enumerate(root)], np.uint32)
    lab, k = D.cluster_labels(root, 60, moff, midx)
    want = R.cluster_labels(root, moff, midx, 60)
    assert lab.tolist() == want and k == len(set(want))
    lab, k = D.cluster_labels(np.array([0, 0, 2, 2, 0], np.uint32), 5)
    assert lab.tolist() == [0, 0, 1, 1, 0] and k == 2


def square(x0, y0, s, ccw=True):
    r = [(x0, y0), (x0 + s, y0), (x0 + s, y0 + s), (x0, y0 + s), (x0, y0)]
    return r if ccw else r[::-1]


def test_copy_file_loader(tmp_path):
    P = pgcopy
    shell_cw = square(0, 0, 1, ccw=False)             # shell given CW: the loader makes it CCW
    hole_ccw = square(0.25, 0.25, 0.5, ccw=True)      # hole given CCW: made CW
    rows = [
        ("a", P.ewkb_polygon([shell_cw, hole_ccw])),
        ("b", P.ewkb_polygon([square(2, 0, 1)], le=False, flags=P.SRID)),                     # big endian + SRID
        ("c", P.ewkb_polygon([square(4, 0, 1)], flags=P.Z | P.SRID, dims=3)),               # EWKB Z
        ("d", P.ewkb_polygon([square(6, 0, 1)], iso=3000, dims=4)),                          # ISO ZM
        ("e", P.ewkb_multi([P.ewkb_polygon([square(8, 0, 1)]), P.ewkb_polygon([square(10, 0, 1, ccw=False)])])),
        ("f", P.ewkb_multi([P.ewkb_polygon([square(12, 0, 1)]), P.ewkb_line([(0, 0), (1, 1)])], kind=7)),   # line inside: wrong type
        (None, P.ewkb_polygon([square(14, 0, 1)])),                                          # null id
        ("h", None),                                                                         # null geometry
        ("i", P.ewkb_polygon([[(0, 0), (1, 0), (0, 0)]])),                                   # only a degenerate ring: empty
        ("j", P.ewkb_point(1.0, 2.0)),                                                       # a point in a polygon layer
        ("k", P.ewkb_multi([P.ewkb_polygon([square(16, 0, 1)]), P.ewkb_polygon([[(0, 0), (1, 1), (0, 0)]])], kind=7)),
        ("l", P.ewkb_line([(0, 0), (1, 1)])),
        ("m", b"\x01\x03"),                                                                  # truncated
    ]
    path = str(tmp_path / "t.copy")
    P.write_copy(path, rows)
    f = D.LayerFile(path)
    info = f.info
    assert info["is_points"] == 0 and info["rows"] == 13
    assert (info["skipped_null"], info["skipped_type"], info["skipped_empty"]) == (2, 4, 1)
    assert f.ids == ["a", "b", "c", "d", "e", "k"]
    assert info["n"] == 6 and info["nr"] == 8 and len(f.gro) == 7
    ring = lambda r: f.xy[f.rvo[r]:f.rvo[r + 1]]
    assert P.signed_area2(ring(0)) > 0 and P.signed_area2(ring(1)) < 0            # shell CCW, hole CW
    assert np.array_equal(ring(0), np.array(shell_cw[::-1]))
    assert np.array_equal(ring(2), np.array(square(2, 0, 1))) and np.array_equal(ring(3), np.array(square(4, 0, 1)))
    assert list(f.gro) == [0, 2, 3, 4, 5, 7, 8]
    assert P.signed_area2(ring(6)) > 0                                            # second polygon of e made CCW
    f.close()
    # a point layer: the first kind fixes the layer; polygons are then wrong type
    P.write_copy(path, [("p1", P.ewkb_point(1.5, 2.5)), ("p2", P.ewkb_polygon([square(0, 0, 1)])), ("p3", P.ewkb_point(3.0, 4.0)),
                        ("p4", struct.pack("<BIdd", 1, 1, float("nan"), float("nan")))])
    f = D.LayerFile(path)
    assert f.info["is_points"] == 1 and f.ids == ["p1", "p3"] and f.xy.tolist() == [[1.5, 2.5], [3.0, 4.0]]
    assert (f.info["skipped_type"], f.info["skipped_empty"]) == (1, 1)
    f.close()


def test_copy_roundtrip_of_generated_layer(tmp_path):
    ps = gen.layer_parcels(300, (-118.3, 33.95, -118.25, 34.0), seed=2)
    path = str(tmp_path / "parcels.copy")
    pgcopy.write_copy(path, pgcopy.polygonset_rows(ps, reverse_every=3))
    f = D.LayerFile(path)
    assert f.info["n"] == ps.n and np.array_equal(f.gro, ps.gro) and np.array_equal(f.rvo, ps.rvo)
    assert np.array_equal(f.xy, ps.xy)   # orientation restored exactly
    assert f.ids == [str(g) for g in range(ps.n)]


def test_gset_pset_files(tmp_path):
    ps = gen.voronoi(50, gen.LA_BOX, 1, vmin=4, vmax=8)
    gen.write_gset(str(tmp_path / "z.gset"), ps)
    f = D.LayerFile(str(tmp_path / "z.gset"))
    assert f.info["n"] == ps.n and np.array_equal(f.xy, ps.xy) and f.ids[:3] == ["0", "1", "2"]
    pts = gen.points(100, gen.LA_BOX, 1)
    gen.write_pset(str(tmp_path / "p.pset"), pts)
    os.remove(str(tmp_path / "p.pset.ids"))
    f = D.LayerFile(str(tmp_path / "p.pset"))
    assert f.info["is_points"] == 1 and np.array_equal(f.xy, pts) and f.ids[-1] == "99"
    (tmp_path / "bad.gset").write_bytes(b"GSET\x01\x00\x00\x00" + b"\x05" * 10)
    with pytest.raises(OSError, match="truncated"):
        D.LayerFile(str(tmp_path / "bad.gset"))


# ---- the protocol, daemon running without a GPU ----
@pytest.fixture
def daemon(tmp_path):
    tok = tmp_path / "token"
    tok.write_text("s3cret\n")
    sock = str(tmp_path / "gsjd.sock")
    data = tmp_path / "data"
    data.mkdir()
    log = open(tmp_path / "gsjd.log", "w")
    p = D.start(sock, str(data), token_file=str(tok), workers=1, log=log)
    yield sock, data, tmp_path
    D.stop(p)
    log.close()


def raw(sock, payload: bytes) -> bytes:
    s = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
    s.settimeout(30)
    s.connect(sock)
    s.sendall(payload)
    out = b""
    try:
        while True:
            b = s.recv(65536)
            if not b:
                break
            out += b
    except ConnectionResetError:   # closed with request bytes still unread
        pass
    s.close()
    return out


def test_protocol_limits_and_auth(daemon):
    sock, data, tmp = daemon
    assert raw(sock, struct.pack("<III", 0x12345678, C.OP_LIST, 1) + struct.pack("<I", 0)) == b""   # bad magic: closed
    assert raw(sock, struct.pack("<III", C.GSP_MAGIC, C.OP_LIST, 65)) == b""                          # > 64 args: closed
    assert raw(sock, struct.pack("<III", C.GSP_MAGIC, C.OP_LIST, 1) + struct.pack("<I", (64 << 20) + 1)) == b""   # arg > 64 MiB
    bad = C.Client(sock, token="wrong")
    with pytest.raises(C.GspError, match="authentication failed"):
        bad.list()
    cl = C.Client(sock, token="s3cret")
    assert cl.list() == [] and cl.drop("nothing") is False
    r = raw(sock, C.encode_request(99, [], "s3cret"))
    assert struct.unpack("<I", r[:4])[0] == C.GSP_ERR and b"unknown op" in r
    with pytest.raises(C.GspError, match="no such layer: a"):
        cl.join("a", "b")
    with pytest.raises(C.GspError, match="LOAD_QUERY"):
        cl.load_query("q", "select 1")
    with pytest.raises(C.GspError, match="row filter"):
        cl.load("x", "f.copy", filter="id > 3")
    with pytest.raises(C.GspError, match="inside the data directory"):
        cl.load("x", str(tmp / "token"))
    with pytest.raises(C.GspError, match="cannot open"):
        cl.load("x", "missing.copy")
    with pytest.raises(C.GspError, match="LOAD needs 7 args"):
        cl.json_call(C.OP_LOAD, ["x"])


def test_load_without_gpu_fails_loudly(daemon):
    sock, data, tmp = daemon
    pgcopy.write_copy(str(data / "t.copy"), [("a", pgcopy.ewkb_polygon([square(0, 0, 1)]))])
    cl = C.Client(sock, token="s3cret")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(C.GspError, match="no usable CUDA device"):
        cl.load("t", "t.copy")
    with pytest.raises(C.GspError, match="no usable CUDA device"):
        cl.status()
    assert cl.list() == []


def test_daemon_library_exports_gsjd_h():
    import ctypes
    import re
    from conftest import ROOT
    names = re.findall(r"\b(gsjd_[a-z_]+)\s*\(", open(os.path.join(ROOT, "include", "gsjd.h")).read())
    assert len(set(names)) >= 10
    L = ctypes.CDLL(D.lib_path("libgsjd.so"))
    assert [n for n in set(names) if not hasattr(L, n)] == []
