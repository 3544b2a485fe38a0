"""Hand-made polygon sets for known-answer tests (closed rings, shells CCW, holes CW)."""
import numpy as np

from gsj.gen import PolygonSet

X0, Y0 = -118.25, 34.05   # a lon/lat origin, so coordinates have realistic magnitudes


def square(x0, y0, s):
    return [(x0, y0), (x0 + s, y0), (x0 + s, y0 + s), (x0, y0 + s), (x0, y0)]


def cw(r):
    return list(reversed(r))


def make_set(geoms):
    """geoms: list of geometries; a geometry is a list of rings; a ring is a list of (dx, dy) offsets in degrees."""
    gro, rvo, xy = [0], [0], []
    for g in geoms:
        for r in g:
            xy.extend((X0 + x, Y0 + y) for x, y in r)
            rvo.append(len(xy))
        gro.append(len(rvo) - 1)
    return PolygonSet(np.array(gro, np.uint64), np.array(rvo, np.uint64), np.array(xy, np.float64).reshape(-1, 2))


S = 0.001
# probe geometries (A side) and build geometries (B side) with their expected DE-9IM relate(A, B) and area
CASES = [
    ("touch_edge", [square(0, 0, S)], [square(S, 0, S)], "FF2F11212", 0.0),
    ("touch_corner", [square(0, 0, S)], [square(S, S, S)], "FF2F01212", 0.0),
    ("overlap", [square(0, 0, S)], [square(S / 2, S / 2, S)], "212101212", (S / 2) ** 2),
    ("equal", [square(0, 0, S)], [square(0, 0, S)], "2FFF1FFF2", S * S),
    ("within", [square(S / 4, S / 4, S / 2)], [square(0, 0, S)], "2FF1FF212", (S / 2) ** 2),
    ("contains", [square(0, 0, S)], [square(S / 4, S / 4, S / 2)], "212FF1FF2", (S / 2) ** 2),
    ("in_hole", [square(S * 0.4, S * 0.4, S * 0.2)], [square(0, 0, S), cw(square(S / 4, S / 4, S / 2))], None, 0.0),
    ("fills_hole", [square(S / 4, S / 4, S / 2)], [square(0, 0, S), cw(square(S / 4, S / 4, S / 2))], "FF2F1F212", 0.0),
]
