"""Row encoding on the device (gsj_encode_rows): the gpujoind frames decoded back into rows equal the rows the
reference daemon's rules give (oracle/rows.py), for every mode, with and without dedup members, self-joins in both
self_pairs rules, DE-9IM patterns, swapped point rows, many frames, and empty results."""
import math
import struct

import numpy as np
import pytest

import gsj
import rows as RR

pytestmark = pytest.mark.gpu
PT_INTERIOR = 1 | 3 << 12 | 2 << 14 | 3 << 16
PT_BOUNDARY = 1 << 2 | 3 << 12 | 2 << 14 | 3 << 16


def decode(buf, plen):
    """[(id_a, id_b, payload bytes)] of a frame stream; checks every frame is non-empty and ends exactly."""
    out, o = [], 0
    while o < len(buf):
        (n,) = struct.unpack_from("<I", buf, o)
        o += 4
        assert n > 0
        for _ in range(n):
            (la,) = struct.unpack_from("<H", buf, o); o += 2
            a = buf[o:o + la]; o += la
            (lb,) = struct.unpack_from("<H", buf, o); o += 2
            b = buf[o:o + lb]; o += lb
            out.append((a, b, buf[o:o + plen])); o += plen
    assert o == len(buf)
    return out


def de9(code):
    return "".join("F012"[(code >> (2 * k)) & 3] for k in range(9)).encode()


def match(code, pat):
    return gsj.de9im_match(code, pat) if pat else True


def make_members(rng, n_geoms, extra):
    """moff / midx: every geometry one row, `extra` geometries with 1-3 more rows (identical copies)."""
    groups = [[g] for g in range(n_geoms)]
    nxt = n_geoms
    for g in rng.choice(n_geoms, extra, replace=False):
        for _ in range(int(rng.integers(1, 4))):
            groups[g].append(nxt); nxt += 1
    moff = np.zeros(n_geoms + 1, np.uint64)
    moff[1:] = np.cumsum([len(x) for x in groups])
    return moff, np.array([r for gg in groups for r in gg], np.uint32), nxt


@pytest.fixture(scope="module")
def sets(engine):
    rng = np.random.default_rng(5)
    moff, midx, nrows = make_members(rng, 300, 40)
    ids = [f"r{r}x{'y' * int(rng.integers(0, 9))}".encode() for r in range(nrows)]
    pids = [f"pt{k}".encode() for k in range(500)]
    return dict(rng=rng, moff=moff, midx=midx, ids=ids, pids=pids, D=engine.rowset(ids, moff, midx), U=engine.rowset(ids[:300]),
                PT=engine.rowset(pids))


@pytest.mark.parametrize("members", [False, True])
@pytest.mark.parametrize("same,distinct", [(False, False), (True, False), (True, True)])
def test_pair_rows(engine, sets, members, same, distinct):
    rng, ids = sets["rng"], sets["ids"]
    S = sets["D"] if members else sets["U"]
    m = (sets["moff"], sets["midx"]) if members else (None, None)
    pairs = rng.integers(0, 300, (2000, 2)).astype(np.uint32)
    if same:
        pairs = np.sort(pairs, axis=1)   # the engine reports each unordered pair once
        pairs[::97, 1] = pairs[::97, 0]  # and geometries with themselves
    area = rng.random(len(pairs))
    area[::13] = 0.0
    buf, n = engine.encode_rows(S, S, gsj.GSJ_ENC_PAIRS, pairs, area=area, same=same, distinct=distinct)
    want = [(ids[ra], ids[rb], struct.pack("<d", area[i])) for ra, rb, i, t in RR.expand(pairs, m, m, same, distinct)]
    got = decode(buf, 8)
    assert n == len(want) and sorted(got) == sorted(want)
    # no area array: NaN payloads
    buf, n = engine.encode_rows(S, S, gsj.GSJ_ENC_PAIRS, pairs, same=same, distinct=distinct)
    assert all(math.isnan(struct.unpack("<d", r[2])[0]) for r in decode(buf, 8)) and n == len(want)


@pytest.mark.parametrize("pattern", ["", "T*T***T**", "FF*F0****", "212101212"])
@pytest.mark.parametrize("same,distinct", [(False, False), (True, False), (True, True)])
def test_relate_rows(engine, sets, pattern, same, distinct):
    rng, ids, S = sets["rng"], sets["ids"], sets["D"]
    m = (sets["moff"], sets["midx"])
    pairs = rng.integers(0, 300, (1500, 2)).astype(np.uint32)
    if same:
        pairs = np.sort(pairs, axis=1)
        pairs[::50, 1] = pairs[::50, 0]
    codes = rng.integers(0, 4, (len(pairs), 9))
    code = (codes << (2 * np.arange(9))).sum(axis=1).astype(np.uint32)
    code[::7] = 0x2DA0A   # a fixed, non-symmetric matrix now and then
    buf, n = engine.encode_rows(S, S, gsj.GSJ_ENC_RELATE, pairs, code=code, same=same, distinct=distinct, pattern=pattern)
    want = []
    for ra, rb, i, t in RR.expand(pairs, m, m, same, distinct):
        c = gsj.de9im_transpose(int(code[i])) if t else int(code[i])
        if match(c, pattern):
            want.append((ids[ra], ids[rb], de9(c)))
    got = decode(buf, 9)
    assert n == len(want) and sorted(got) == sorted(want)


@pytest.mark.parametrize("swapped", [False, True])
@pytest.mark.parametrize("relate,pattern", [(False, ""), (True, ""), (True, "0********")])
def test_point_rows(engine, sets, swapped, relate, pattern):
    rng, ids, pids = sets["rng"], sets["ids"], sets["pids"]
    m = (sets["moff"], sets["midx"])
    pairs = np.stack([rng.integers(0, 500, 3000), rng.integers(0, 300, 3000)], axis=1).astype(np.uint32)
    where = rng.integers(1, 3, len(pairs)).astype(np.uint8)
    mode = gsj.GSJ_ENC_POINT_RELATE if relate else gsj.GSJ_ENC_POINTS
    buf, n = engine.encode_rows(sets["PT"], sets["D"], mode, pairs, where=where if relate else None, swapped=swapped, point_value=0.0,
                                pattern=pattern)
    want = []
    for i, (p, g) in enumerate(pairs):
        for rb in RR.members(*m, int(g)):
            if relate:
                c = PT_BOUNDARY if where[i] == 2 else PT_INTERIOR
                if swapped:
                    c = gsj.de9im_transpose(c)
                if not match(c, pattern):
                    continue
                pay = de9(c)
            else:
                pay = struct.pack("<d", 0.0)
            want.append((ids[rb], pids[p], pay) if swapped else (pids[p], ids[rb], pay))
    got = decode(buf, 9 if relate else 8)
    assert n == len(want) and sorted(got) == sorted(want)


def test_many_frames_and_empty(engine, sets):
    rng, ids = sets["rng"], sets["ids"]
    pairs = rng.integers(0, 300, (200000, 2)).astype(np.uint32)
    area = rng.random(len(pairs))
    buf, n = engine.encode_rows(sets["U"], sets["U"], gsj.GSJ_ENC_PAIRS, pairs, area=area)
    got = decode(buf, 8)
    assert n == len(pairs) == len(got)
    assert got[:3] == [(ids[int(a)], ids[int(b)], struct.pack("<d", area[i])) for i, (a, b) in enumerate(pairs[:3])]   # pair order kept
    frames, o = 0, 0
    while o < len(buf):   # frames of whole pairs, each at most ~1 MiB
        (k,) = struct.unpack_from("<I", buf, o)
        start = o
        o += 4
        for _ in range(k):
            (la,) = struct.unpack_from("<H", buf, o); o += 2 + la
            (lb,) = struct.unpack_from("<H", buf, o); o += 2 + lb + 8
        assert o - start <= (1 << 20) + 4
        frames += 1
    assert frames > 1
    # a pattern nothing matches: no rows, no frames (an empty frame would end the stream)
    code = np.zeros(1000, np.uint32)
    buf, n = engine.encode_rows(sets["U"], sets["U"], gsj.GSJ_ENC_RELATE, pairs[:1000], code=code, pattern="T********")
    assert n == 0 and buf == b""
    buf, n = engine.encode_rows(sets["U"], sets["U"], gsj.GSJ_ENC_PAIRS, pairs[:0])
    assert n == 0 and buf == b""


def test_bad_arguments(engine, sets):
    with pytest.raises(gsj.GsjError):
        engine.encode_rows(sets["U"], sets["U"], gsj.GSJ_ENC_PAIRS, np.array([[300, 0]], np.uint32))   # geometry out of range
    with pytest.raises(gsj.GsjError):
        engine.encode_rows(sets["U"], sets["U"], gsj.GSJ_ENC_RELATE, np.array([[0, 0]], np.uint32), code=np.zeros(1, np.uint32),
                           pattern="T*")


def test_long_ids_are_cut_like_the_host_encoder(engine):
    """An id longer than a u16 length can say is sent as its first 65535 bytes (FrameWriter::id does the same)."""
    ids = [b"a" * 70000, b"b", b"c" * 65535]
    S = engine.rowset(ids)
    pairs = np.array([[0, 1], [2, 0], [1, 1]], np.uint32)
    buf, n = engine.encode_rows(S, S, gsj.GSJ_ENC_PAIRS, pairs, area=np.array([1.0, 2.0, 3.0]))
    got = decode(buf, 8)
    assert n == 3 and [(len(a), len(b)) for a, b, _ in got] == [(65535, 1), (65535, 65535), (1, 1)]
