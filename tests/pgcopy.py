"""Test helper: PostgreSQL binary COPY files of (id text, geometry EWKB) rows, the stream the reference daemon
reads from COPY ... TO STDOUT (FORMAT binary) (daemon/loader.h) and that gsjd LOADs from files."""
import struct

import numpy as np

SIG = b"PGCOPY\n\xff\r\n\x00"
Z, M, SRID = 0x80000000, 0x40000000, 0x20000000


def ewkb_polygon(rings, le=True, flags=0, srid=4326, dims=2, iso=0):
    """rings: list of [(x, y), ...]; extra dims filled with 7.0."""
    e = "<" if le else ">"
    t = 3 + iso
    if flags & SRID:
        head = struct.pack(e + "BII", 1 if le else 0, t | flags, srid)
    else:
        head = struct.pack(e + "BI", 1 if le else 0, t | flags)
    body = [struct.pack(e + "I", len(rings))]
    for r in rings:
        body.append(struct.pack(e + "I", len(r)))
        for x, y in r:
            body.append(struct.pack(e + "dd", x, y) + struct.pack(e + "d", 7.0) * (dims - 2))
    return head + b"".join(body)


def ewkb_multi(parts, kind=6, le=True):
    e = "<" if le else ">"
    return struct.pack(e + "BII", 1 if le else 0, kind, len(parts)) + b"".join(parts)


def ewkb_point(x, y, le=True):
    e = "<" if le else ">"
    return struct.pack(e + "BIdd", 1 if le else 0, 1, x, y)


def ewkb_line(pts, le=True):
    e = "<" if le else ">"
    return struct.pack(e + "BII", 1 if le else 0, 2, len(pts)) + b"".join(struct.pack(e + "dd", x, y) for x, y in pts)


def write_copy(path, rows):
    """rows: [(id str or None, ewkb bytes or None)]."""
    out = [SIG, struct.pack(">II", 0, 0)]
    for rid, g in rows:
        out.append(struct.pack(">h", 2))
        for f in (None if rid is None else rid.encode(), g):
            out.append(struct.pack(">i", -1) if f is None else struct.pack(">i", len(f)) + f)
    out.append(struct.pack(">h", -1))
    open(path, "wb").write(b"".join(out))


def signed_area2(pts):
    a = np.asarray(pts, np.float64)
    a = a - a[0]
    return float(np.sum(a[:-1, 0] * a[1:, 1] - a[1:, 0] * a[:-1, 1]))


def polygonset_rows(ps, ids=None, reverse_every=0):
    """Rows of a PolygonSet as POLYGON / MULTIPOLYGON EWKB (a CCW ring opens a polygon, CW rings are its holes).
    reverse_every=k reverses every k-th ring's orientation so the loader must restore it."""
    rows, k = [], 0
    for g in range(ps.n):
        polys = []
        for r in range(int(ps.gro[g]), int(ps.gro[g + 1])):
            pts = [tuple(p) for p in ps.xy[ps.rvo[r]:ps.rvo[r + 1]]]
            if signed_area2(pts) > 0 or not polys:
                polys.append([])
            k += 1
            if reverse_every and k % reverse_every == 0:
                pts = pts[::-1]
            polys[-1].append(pts)
        g_wkb = ewkb_polygon(polys[0]) if len(polys) == 1 else ewkb_multi([ewkb_polygon(p) for p in polys])
        rows.append((str(g) if ids is None else ids[g], g_wkb))
    return rows


def as_array(rings):
    return np.array([p for r in rings for p in r], np.float64)
