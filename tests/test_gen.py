"""Synthetic Voronoi layers: determinism, exact tiling, orientation, shared vertices."""
import hashlib

import numpy as np
import pytest

from gsj import gen


def ring_areas(ps):
    out = []
    for r in range(ps.nr):
        v = ps.xy[ps.rvo[r]:ps.rvo[r + 1]]
        v = v - v[0]
        out.append(0.5 * np.sum(v[:-1, 0] * v[1:, 1] - v[1:, 0] * v[:-1, 1]))
    return np.array(out)


def digest(ps):
    h = hashlib.sha256()
    for a in (ps.gro, ps.rvo, ps.xy):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("builder", [lambda: gen.voronoi(3000, gen.LA_BOX, 0, vmin=6, vmax=40),
                                     lambda: gen.layer_parcels(4000, (-118.3, 33.95, -118.2, 34.05), seed=7)])
def test_tiles_box_exactly(builder):
    ps = builder()
    assert ps.stats["inconsistent"] == 0
    rings_closed = np.all(ps.xy[ps.rvo[:-1]] == ps.xy[ps.rvo[1:] - 1], axis=1)
    assert rings_closed.all()
    a = ring_areas(ps)
    # shells CCW (positive), holes CW (negative): first ring of every geometry is a shell
    first = ps.gro[:-1]
    assert (a[first] > 0).all()
    box = ps.xy.min(0), ps.xy.max(0)
    assert abs(a.sum() - np.prod(box[1] - box[0])) < 1e-12


def test_deterministic():
    assert digest(gen.layer_parcels(3000, (-118.3, 33.95, -118.2, 34.05), seed=5)) == \
        digest(gen.layer_parcels(3000, (-118.3, 33.95, -118.2, 34.05), seed=5))
    assert digest(gen.voronoi(500, gen.LA_BOX, 1)) != digest(gen.voronoi(500, gen.LA_BOX, 2))


def test_parcel_mix():
    ps = gen.layer_parcels(20000, (-118.5, 33.8, -118.2, 34.1), seed=3)
    rl = np.diff(ps.rvo.astype(np.int64))
    assert rl.min() >= 4 and 40 < rl.mean() < 80            # log-uniform 4..256 targets: mean ~60
    assert 0.02 < ps.stats["multipolygons"] / 20000 < 0.08
    assert 0.01 < ps.stats["holes"] / 20000 < 0.03


def test_shared_vertices_are_bit_identical():
    """Neighbouring cells reuse the exact same doubles along their common edge."""
    ps = gen.voronoi(400, gen.LA_BOX, 4, vmin=10, vmax=30)
    seen = {}
    for g in range(ps.n):
        v = ps.xy[ps.rvo[ps.gro[g]]:ps.rvo[ps.gro[g + 1]]]
        for p in map(tuple, v[:-1]):
            seen.setdefault(p, set()).add(g)
    shared = sum(1 for s in seen.values() if len(s) >= 2)
    assert shared > 2 * ps.n   # interior vertices are shared by 2-3 cells


def test_gset_roundtrip(tmp_path):
    ps = gen.layer_parcels(1000, (-118.3, 33.95, -118.25, 34.0), seed=2)
    p = tmp_path / "x.gset"
    gen.write_gset(str(p), ps)
    q = gen.read_gset(str(p))
    assert np.array_equal(ps.gro, q.gro) and np.array_equal(ps.rvo, q.rvo) and np.array_equal(ps.xy, q.xy)
    assert len(open(str(p) + ".ids").read().split()) == ps.n
