"""Negative-buffer joins on the GPU against the CPU oracle: ST_Intersects(ST_Buffer(a, -ra), ST_Buffer(b, -rb)) for
polygon pairs and points in ST_Buffer(b, -r), whole and subdivided layers, asymmetric radii, and the overflow passes
(quadrant tiles, then unlimited per-warp lists) on dense rings."""
import numpy as np
import pytest

import gsj
import pyoracle as O
import shapes
from gsj import gen

pytestmark = pytest.mark.gpu
BOX = (-118.3, 33.95, -118.1, 34.15)


def as_set(p):
    return set(map(tuple, np.asarray(p).reshape(-1, 2).tolist()))


def circle(cx, cy, r, n):
    t = np.linspace(0, 2 * np.pi, n, endpoint=False)
    pts = [(cx + r * np.cos(a) / np.cos(np.radians(34.05)), cy + r * np.sin(a)) for a in t]
    return pts + [pts[0]]


@pytest.fixture(scope="module")
def layers(engine):
    hs = {"parcels": gen.layer_parcels(20000, BOX, seed=5), "parcels2": gen.layer_parcels(15000, BOX, seed=6),
          "zones": gen.voronoi(50, gen.LA_BOX, 1, vmin=4, vmax=4)}
    hs["sub"] = gsj.subdivide(hs["parcels"], 24)
    hs["sub2"] = gsj.subdivide(hs["parcels2"], 32)
    return {k: (engine.upload_polygons(v), O.OSet(v), v) for k, v in hs.items()}


@pytest.mark.parametrize("r", [0.0, 1.0, 5.0])
def test_erode_self(engine, layers, r):
    L, S, ps = layers["parcels"]
    none = np.zeros(ps.n, np.uint8)
    for ns in (None, none):
        g, st = engine.erode(L, L, r, r, same=True, need_self=ns)
        o = O.erode(S, S, r, r, same=True, need_self=ns)
        assert as_set(g) == as_set(o)


@pytest.mark.parametrize("a,b,ra,rb", [("parcels", "parcels2", 1.0, 1.0), ("parcels", "parcels2", 1.0, 3.0), ("parcels2", "parcels", 0.0, 5.0),
                                       ("parcels", "zones", 2.0, 800.0), ("zones", "parcels2", 50.0, 0.5), ("sub", "sub2", 1.0, 1.0),
                                       ("sub", "parcels2", 3.0, 1.0), ("parcels2", "sub", 5.0, 5.0)])
def test_erode_two_layers(engine, layers, a, b, ra, rb):
    g, st = engine.erode(layers[a][0], layers[b][0], ra, rb)
    o = O.erode(layers[a][1], layers[b][1], ra, rb)
    assert as_set(g) == as_set(o) and len(o) > 0


def test_erode_subdivided_self(engine, layers):
    L, S, ps = layers["sub"]
    g, st = engine.erode(L, L, 1.0, 1.0, same=True)
    o = O.erode(S, S, 1.0, 1.0, same=True)
    assert as_set(g) == as_set(o)


def test_erode_overflow_passes(engine):
    """Rings of thousands of vertices overflow the 64-edge lists: tiles split until they fit or reach the radius,
    then unlimited lists."""
    A = shapes.make_set([[circle(0, 0, 0.01, 3000)], [circle(0.03, 0, 0.008, 2500)]])
    B = shapes.make_set([[circle(0.012, 0.004, 0.01, 2800)], [circle(0.04, 0.01, 0.012, 64)]])
    GA, GB = engine.upload_polygons(A), engine.upload_polygons(B)
    for ra, rb in ((50.0, 50.0), (300.0, 300.0), (300.0, 40.0), (900.0, 900.0)):
        g, st = engine.erode(GA, GB, ra, rb)
        o = O.erode(O.OSet(A), O.OSet(B), ra, rb)
        assert as_set(g) == as_set(o)
        if ra == 50.0:
            assert st["heavy"] > 0 and len(o) == 3


@pytest.mark.parametrize("mode", [gsj.GSJ_REFINE_PLAIN, gsj.GSJ_REFINE_FILTERED])   # thread / warp per (point, piece)
@pytest.mark.parametrize("r", [0.0, 1.0, 3.0, 25.0])
def test_points_erode(engine, layers, r, mode):
    pts = gen.points(30000, BOX, 3)
    pts = np.concatenate([pts, layers["parcels"][2].xy[::131]])   # boundary points
    P = engine.upload_points(pts)
    for k in ("parcels", "sub"):
        g, st = engine.points_erode(P, layers[k][0], r, refine_mode=mode)
        o = O.pt_erode(pts, layers[k][1], r)
        assert as_set(g) == as_set(o) and len(o) > 0


def test_erode_reference_golden(engine):
    """The GPU against the reference engine's own outputs on the golden layers (no oracle in between)."""
    import make_golden as MG
    L = {k: b() for k, (kind, b) in MG.layers().items()}

    def golden(case):
        return as_set(np.load(f"{MG.HERE}/{case}.npz")["pairs"])

    P, Q = engine.upload_polygons(L["parcels"]), engine.upload_polygons(L["parcels2"])
    for case, ra, rb in (("pq_erode1", 1.0, 1.0), ("pq_erode1_3", 1.0, 3.0), ("pq_erode5", 5.0, 5.0)):
        assert as_set(engine.erode(P, Q, ra, rb)[0]) == golden(case), case
    SP, SQ = engine.upload_polygons(gsj.subdivide(L["parcels"], 32)), engine.upload_polygons(gsj.subdivide(L["parcels2"], 32))
    assert as_set(engine.erode(SP, SQ, 1.0, 1.0)[0]) == golden("pq_erode1_sub32")
    none = np.zeros(L["parcels"].n, np.uint8)
    g = engine.erode(P, P, 1.0, 1.0, same=True, need_self=none)[0]
    assert as_set(g) == golden("pp_erode1")
    pts = engine.upload_points(L["points"])
    for mode in (gsj.GSJ_REFINE_PLAIN, gsj.GSJ_REFINE_FILTERED):
        assert as_set(engine.points_erode(pts, P, 1.0, refine_mode=mode)[0]) == golden("pts_erode1")
        assert as_set(engine.points_erode(pts, SP, 3.0, refine_mode=mode)[0]) == golden("pts_erode3_sub32")
        assert as_set(engine.dwithin(P, Q, 5.0, refine_mode=mode)[0]) == golden("pq_dwithin5")
