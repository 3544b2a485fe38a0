"""Distance joins on the GPU against the CPU oracle: ST_DWithin(geography) for polygon pairs and points."""
import numpy as np
import pytest

import gsj
import pyoracle as O
from gsj import gen

pytestmark = pytest.mark.gpu
BOX = (-118.3, 33.95, -118.1, 34.15)


def as_set(p):
    return set(map(tuple, np.asarray(p).tolist()))


@pytest.fixture(scope="module")
def layers(engine):
    hs = {"parcels": gen.layer_parcels(20000, BOX, seed=5), "parcels2": gen.layer_parcels(15000, BOX, seed=6),
          "zones": gen.voronoi(50, gen.LA_BOX, 1, vmin=4, vmax=4)}
    return {k: (engine.upload_polygons(v), O.OSet(v), v) for k, v in hs.items()}


MODES = [gsj.GSJ_REFINE_PLAIN, gsj.GSJ_REFINE_FILTERED]   # lane per A edge / queued edge pairs


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("d", [0.0, 5.0, 40.0])
def test_dwithin_self(engine, layers, d, mode):
    L, S, _ = layers["parcels"]
    g, st = engine.dwithin(L, L, d, same=True, refine_mode=mode)
    o, nc = O.dwithin(S, S, d, same=True)
    assert as_set(g) == as_set(o) and st["candidates"] == nc


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("a,b,d", [("parcels", "parcels2", 5.0), ("parcels2", "zones", 1000.0), ("zones", "parcels", 25.0)])
def test_dwithin_two_layers(engine, layers, a, b, d, mode):
    g, st = engine.dwithin(layers[a][0], layers[b][0], d, refine_mode=mode)
    o, nc = O.dwithin(layers[a][1], layers[b][1], d)
    assert as_set(g) == as_set(o) and len(o) > 0


@pytest.mark.parametrize("mode", [gsj.GSJ_REFINE_PLAIN, gsj.GSJ_REFINE_FILTERED])   # thread / warp per (point, piece)
@pytest.mark.parametrize("d", [0.0, 5.0, 100.0])
def test_points_dwithin(engine, layers, d, mode):
    pts = gen.points(30000, BOX, 3)
    ps = layers["parcels"][2]
    pts = np.concatenate([pts, ps.xy[::131]])   # boundary points
    g, st = engine.points_dwithin(engine.upload_points(pts), layers["parcels"][0], d, refine_mode=mode)
    o = O.pt_dwithin(pts, layers["parcels"][1], d)
    assert as_set(g) == as_set(o) and len(o) > 0
