"""CUDA engine (through the C ABI) against the CPU FP64 oracle: bit-exact pair sets, flags, areas, DE-9IM."""
import numpy as np
import pytest

import gsj
import pyoracle as O
import shapes
from gsj import gen

pytestmark = pytest.mark.gpu
MODES = [gsj.GSJ_REFINE_PLAIN, gsj.GSJ_REFINE_FILTERED, gsj.GSJ_REFINE_FILTERED_FP32]
SMALL_BOX = (-118.30, 33.95, -118.20, 34.05)


def srt(p, *vals):
    i = np.lexsort((p[:, 1], p[:, 0]))
    return (p[i],) + tuple(None if v is None else v[i] for v in vals)


@pytest.fixture(scope="module")
def layers(engine):
    hs = {
        "zonesA": gen.voronoi(20000, gen.LA_BOX, 0, vmin=6, vmax=40),
        "zonesB": gen.voronoi(50, gen.LA_BOX, 1, vmin=4, vmax=4),
        "parcels": gen.layer_parcels(20000, (-118.3, 33.95, -118.1, 34.15), seed=5),
        "parcels2": gen.layer_parcels(15000, (-118.3, 33.95, -118.1, 34.15), seed=6),
        "one": gen.voronoi(1, gen.LA_BOX, 9, vmin=40, vmax=40),
    }
    return {k: (engine.upload_polygons(v), O.OSet(v), v) for k, v in hs.items()}


PAIRS = [("zonesA", "zonesB", False), ("zonesA", "zonesA", True), ("parcels", "parcels", True), ("parcels", "parcels2", False),
         ("parcels2", "zonesB", False), ("one", "parcels", False), ("parcels", "one", False)]


@pytest.mark.parametrize("a,b,upper", PAIRS)
def test_candidates(engine, layers, a, b, upper):
    g = srt(engine.candidates(layers[a][0], layers[b][0], upper=upper))[0]
    o = O.candidates(layers[a][1], layers[b][1], upper=upper)
    assert np.array_equal(g, o)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("a,b,upper", PAIRS)
def test_refine_pairs_bitexact(engine, layers, a, b, upper, mode):
    cand = O.candidates(layers[a][1], layers[b][1], upper=upper)
    for rel in (False, True):
        f, ar, ev, evb = engine.refine_pairs(layers[a][0], layers[b][0], cand, want_area=True, want_relate=rel, refine_mode=mode)
        of, oa, oe, ob = O.refine_pairs(layers[a][1], layers[b][1], cand, O.params(1, int(rel)))
        assert np.array_equal(f, of)
        assert np.array_equal(ar, oa)            # same rounding order: bit-identical areas
        if rel:
            assert np.array_equal(ev, oe) and np.array_equal(evb, ob)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("a,b,upper", PAIRS)
def test_join_bitexact(engine, layers, a, b, upper, mode):
    for area, rel in ((True, False), (False, True), (True, True)):
        r = engine.join(layers[a][0], layers[b][0], want_area=area, want_relate=rel, upper=upper, refine_mode=mode)
        p, oa, oc, nc = O.join(layers[a][1], layers[b][1], O.params(int(area), int(rel)), upper=upper)
        gp, ga, gc = srt(r.pairs, r.area, r.code)
        assert np.array_equal(gp, p)
        if area:
            assert np.array_equal(ga, oa)
        if rel:
            assert np.array_equal(gc, oc)
        assert r.stats["candidates"] == nc and r.stats["launches"] >= 3


def test_area_tiles_box(engine, layers):
    r = engine.join(layers["zonesA"][0], layers["zonesB"][0])
    assert abs(r.area.sum() - 0.25) < 1e-12


@pytest.mark.parametrize("name,a,b,rel,area", shapes.CASES)
def test_known_answers_gpu(engine, name, a, b, rel, area):
    A, B = engine.upload_polygons(shapes.make_set([a])), engine.upload_polygons(shapes.make_set([b]))
    r = engine.join(A, B, want_area=True, want_relate=True)
    if rel is None:
        assert len(r.pairs) == 0
        return
    assert len(r.pairs) == 1 and gsj.de9im_str(int(r.code[0])) == rel
    assert abs(r.area[0] - area) <= 1e-9 * max(area, 1e-12) + 1e-20


def test_batches_give_same_rows(engine, layers):
    L = layers["parcels"][0]
    whole = engine.join(L, L, want_area=True, want_relate=True, upper=True)
    parts = engine.join(L, L, want_area=True, want_relate=True, upper=True, batch_q=3000)
    assert parts.stats["batches"] > 1
    a, b = srt(whole.pairs, whole.area, whole.code), srt(parts.pairs, parts.area, parts.code)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("mode", MODES)   # thread / warp per (point, piece)
def test_points_in_polygons(engine, layers, mode):
    pts = gen.points(50000, (-118.3, 33.95, -118.1, 34.15), 3)
    # include vertices and edge midpoints (boundary cases) of the parcels
    ps = layers["parcels"][2]
    extra = np.concatenate([ps.xy[::97], 0.5 * (ps.xy[:-1:89] + ps.xy[1::89])])
    pts = np.concatenate([pts, extra])
    gp, gw, st = engine.join_points(engine.upload_points(pts), layers["parcels"][0], refine_mode=mode)
    op, ow, nc = O.pip(pts, layers["parcels"][1])
    gp, gw = srt(gp, gw)
    assert np.array_equal(gp, op) and np.array_equal(gw, ow)
    assert (ow == 2).sum() > 100 and st["candidates"] == nc


def test_cluster(engine, layers):
    for k in ("parcels", "zonesA"):
        root, st = engine.cluster(layers[k][0])
        assert np.array_equal(root, O.cluster(layers[k][1], layers[k][1].n))
    # two separate groups of squares
    geoms = [[shapes.square(i * shapes.S, 0, shapes.S)] for i in range(3)] + [[shapes.square(10 * shapes.S + i * shapes.S, 0, shapes.S)] for i in range(2)]
    root, _ = engine.cluster(engine.upload_polygons(shapes.make_set(geoms)))
    assert root.tolist() == [0, 0, 0, 3, 3]


def shrunk_parcels(n, box, seed, frac=0.55, f=0.9):
    """Parcels with a seeded fraction shrunk toward their bbox centre: components of every size."""
    return gen.shrunk(gen.layer_parcels(n, box, seed=seed), seed, frac, f)


@pytest.mark.parametrize("mode", MODES)
def test_cluster_many_components(engine, mode):
    """More than 65536 candidates (the filtered cluster then refines in rounds that skip pairs already connected)
    and components of every size: roots equal the oracle's, for the whole layer and for its pieces."""
    ps = shrunk_parcels(40000, (-118.3, 33.95, -118.1, 34.15), seed=11)
    want = O.cluster(O.OSet(ps), ps.n)
    sizes = np.unique(want, return_counts=True)[1]
    assert (sizes >= 2).sum() > 500 and (sizes >= 100).sum() > 5
    root, st = engine.cluster(engine.upload_polygons(ps), refine_mode=mode)
    assert st["candidates"] > 1 << 16 and np.array_equal(root, want)
    sub = gsj.subdivide(ps, 12)
    root, st = engine.cluster(engine.upload_polygons(sub), ps.n, refine_mode=mode)
    assert st["candidates"] > 1 << 16 and np.array_equal(root, O.cluster(O.OSet(sub), ps.n))


def test_bad_arguments_are_errors(engine, layers):
    with pytest.raises(gsj.GsjError):
        engine.join(layers["parcels"][0], engine.upload_points(np.zeros((3, 2))))
    with pytest.raises(gsj.GsjError):
        engine.refine_pairs(layers["one"][0], layers["one"][0], np.array([[0, 5]], np.uint32))


@pytest.fixture(scope="module")
def pieces(engine):
    import gsj
    a = gsj.subdivide(gen.layer_parcels(8000, (-118.3, 33.95, -118.2, 34.05), seed=5), 24)
    b = gsj.subdivide(gen.voronoi(50, gen.LA_BOX, 1, vmin=40, vmax=80), 16)
    return {k: (engine.upload_polygons(v), O.OSet(v), v) for k, v in (("a", a), ("b", b))}


@pytest.mark.parametrize("mode", MODES)
def test_subdivided_join_bitexact(engine, pieces, mode):
    for (x, y, upper) in (("a", "a", True), ("a", "b", False)):
        for area, rel in ((True, False), (False, True)):
            r = engine.join(pieces[x][0], pieces[y][0], want_area=area, want_relate=rel, upper=upper, refine_mode=mode)
            p, oa, oc, nc = O.join(pieces[x][1], pieces[y][1], O.params(int(area), int(rel)), upper=upper)
            gp, ga, gc = srt(r.pairs, r.area, r.code)
            assert np.array_equal(gp, p)
            if area:
                assert np.array_equal(ga, oa)
            if rel:
                assert np.array_equal(gc, oc)


def test_subdivided_points_cluster_dwithin(engine, pieces):
    pts = gen.points(20000, (-118.3, 33.95, -118.2, 34.05), 8)
    op, ow, _ = O.pip(pts, pieces["a"][1])
    for mode in MODES:
        gp, gw, _ = engine.join_points(engine.upload_points(pts), pieces["a"][0], refine_mode=mode)
        gp, gw = srt(gp, gw)
        assert np.array_equal(gp, op) and np.array_equal(gw, ow)
    root, _ = engine.cluster(pieces["a"][0])
    assert np.array_equal(root, O.cluster(pieces["a"][1], pieces["a"][0].info["nparent"]))
    g, _ = engine.dwithin(pieces["a"][0], pieces["a"][0], 5.0, same=True)
    o, _ = O.dwithin(pieces["a"][1], pieces["a"][1], 5.0, same=True)
    assert set(map(tuple, g.tolist())) == set(map(tuple, o.tolist()))


@pytest.mark.parametrize("morton", [False, True])
def test_dedup_gpu_matches_oracle(engine, morton):
    """gsj_dedup_gpu gives the oracle's arrays bit for bit: distinct set, member offsets and indices."""
    import test_gpu_daemon as TD
    base = gen.layer_parcels(30000, (-118.3, 33.95, -118.2, 34.05), seed=4)
    rng = np.random.default_rng(5)
    ps = TD.with_duplicates(base, rng.choice(base.n, 3000, replace=True))   # groups of 2+ copies, some repeated
    hu, hmo, hmi = O.dedup(ps, morton=morton)
    gu, gmo, gmi = engine.dedup(ps, morton=morton)
    assert np.array_equal(hmo, gmo) and np.array_equal(hmi, gmi)
    assert np.array_equal(hu.gro, gu.gro) and np.array_equal(hu.rvo, gu.rvo) and np.array_equal(hu.xy.view(np.uint64), gu.xy.view(np.uint64))
    assert hu.n < ps.n


def degenerate_geometries():
    """Hand-made troublesome rings (degree offsets around shapes.X0, shapes.Y0)."""
    S = 0.001
    sq = shapes.square
    g = []
    g.append([[(0, 0), (S, 0), (S, 0), (S, S), (0, S), (0, S), (0, 0)]])                        # repeated vertices
    g.append([[(S, 0), (2 * S, 0), (2 * S, S / 2), (3 * S, S / 2), (2 * S, S / 2), (2 * S, S), (S, S), (S, 0)]])   # spike
    g.append([[(0, S), (S / 3, S), (2 * S / 3, S), (S, S), (S, 2 * S), (0, 2 * S), (0, S)]])    # collinear run on a shared edge
    g.append([[(0, 0), (3 * S, 1e-12), (0, 2e-12), (0, 0)]])                                    # sliver
    g.append([sq(S, S, S)])                                                                     # touches others at points / edges
    g.append([sq(-S, -S, 4 * S), shapes.cw(sq(0, 0, 2 * S)), sq(S / 2, S / 2, S / 2)])          # hole with an island inside
    g.append([sq(0, 0, S)])                                                                     # duplicate of an existing square
    g.append([sq(0, 0, S)])
    g.append([[(S / 2, 0), (S, S / 2), (S / 2, S), (0, S / 2), (S / 2, 0)]])                   # diamond in a square
    g.append([[(0, 0), (S, 0), (S, S), (0, 0)], [(2 * S, 0), (3 * S, 0), (3 * S, S), (2 * S, 0)]])   # multipolygon
    g.append([[(-S, S / 2), (4 * S, S / 2), (4 * S, S / 2 + 1e-9), (-S, S / 2 + 1e-9), (-S, S / 2)]])  # long thin bar across
    big = [(S * np.cos(t), S * np.sin(t)) for t in np.linspace(0, 2 * np.pi, 400, endpoint=False)]
    g.append([big + [big[0]]])                                                                  # heavy ring (> 128 edges)
    return g


@pytest.mark.parametrize("mode", MODES)
def test_degenerate_inputs_bitexact(engine, mode):
    ps = shapes.make_set(degenerate_geometries())
    L, S = engine.upload_polygons(ps), O.OSet(ps)
    for area, rel in ((True, False), (False, True), (True, True)):
        r = engine.join(L, L, want_area=area, want_relate=rel, upper=True, refine_mode=mode)
        p, oa, oc, nc = O.join(S, S, O.params(int(area), int(rel)), upper=True)
        gp, ga, gc = srt(r.pairs, r.area, r.code)
        assert np.array_equal(gp, p) and len(p) > 10
        if area:
            assert np.array_equal(ga, oa)
        if rel:
            assert np.array_equal(gc, oc)
    cand = O.candidates(S, S, upper=True)
    f, ar, ev, evb = engine.refine_pairs(L, L, cand, want_area=True, want_relate=True, refine_mode=mode)
    of, oa, oe, ob = O.refine_pairs(S, S, cand, O.params(1, 1))
    assert np.array_equal(f, of) and np.array_equal(ar, oa) and np.array_equal(ev, oe) and np.array_equal(evb, ob)
    root, _ = engine.cluster(L)
    assert np.array_equal(root, O.cluster(S, ps.n))
    pts = np.concatenate([ps.xy, ps.xy[::3] + 1e-7, np.array([[shapes.X0 + 0.0005, shapes.Y0 + 0.0005]])])   # vertices, near-vertices
    gp, gw, _ = engine.join_points(engine.upload_points(pts), L, refine_mode=mode)
    op_, ow, _ = O.pip(pts, S)
    gp, gw = srt(gp, gw)
    assert np.array_equal(gp, op_) and np.array_equal(gw, ow)


def test_empty_and_tiny_layers(engine):
    one = shapes.make_set([[shapes.square(0, 0, 0.001)]])
    L = engine.upload_polygons(one)
    r = engine.join(L, L, upper=True)
    assert len(r.pairs) == 1 and r.area[0] > 0
    far = shapes.make_set([[shapes.square(1.0, 1.0, 0.001)]])
    assert len(engine.join(L, engine.upload_polygons(far)).pairs) == 0
    with pytest.raises(gsj.GsjError):
        engine.upload_polygons(gen.PolygonSet(np.zeros(1, np.uint64), np.zeros(1, np.uint64), np.zeros((0, 2))))


@pytest.mark.parametrize("maxv", [12, 24, 64])
def test_subdivide_gpu_matches_oracle(engine, maxv):
    """gsj_subdivide_gpu gives the oracle's pieces bit for bit: order, rings, vertices, cut flags, parents."""
    layers = [gen.layer_parcels(20000, (-118.3, 33.95, -118.2, 34.05), seed=5), gen.voronoi(50, gen.LA_BOX, 1, vmin=40, vmax=80),
              shapes.make_set(degenerate_geometries())]
    for ps in layers:
        h = O.subdivide(ps, maxv)
        g = engine.subdivide(ps, maxv)
        assert g.n == h.n and np.array_equal(g.gro, h.gro) and np.array_equal(g.rvo, h.rvo)
        assert np.array_equal(g.xy.view(np.uint64), h.xy.view(np.uint64))
        assert np.array_equal(g.parent, h.parent) and np.array_equal(g.syn, h.syn)


@pytest.mark.parametrize("nshards", [2, 3, 8])
def test_probe_shards_partition_the_join(engine, layers, pieces, nshards):
    """Probe shards (one per GPU in a multi-GPU run) partition the join: their union is the whole result, values equal."""
    cases = [(layers["parcels"][0], layers["parcels"][0], True), (layers["parcels"][0], layers["parcels2"][0], False),
             (pieces["a"][0], pieces["a"][0], True), (pieces["a"][0], pieces["b"][0], False)]
    for P, R, upper in cases:
        full = engine.join(P, R, want_area=True, want_relate=True, upper=upper)
        parts = [engine.join(P, R, want_area=True, want_relate=True, upper=upper, shard=k, nshards=nshards) for k in range(nshards)]
        fp, fa, fc = srt(full.pairs, full.area, full.code)
        sp, sa, sc = srt(np.concatenate([x.pairs for x in parts]), np.concatenate([x.area for x in parts]), np.concatenate([x.code for x in parts]))
        assert np.array_equal(fp, sp) and np.array_equal(fa, sa) and np.array_equal(fc, sc)
    pts = gen.points(40000, (-118.3, 33.95, -118.1, 34.15), 9)
    L = engine.upload_points(pts)
    fp, fw, _ = engine.join_points(L, layers["parcels"][0])
    parts = [engine.join_points(L, layers["parcels"][0], shard=k, nshards=nshards) for k in range(nshards)]
    a, aw = srt(fp, fw)
    b, bw = srt(np.concatenate([x[0] for x in parts]), np.concatenate([x[1] for x in parts]))
    assert np.array_equal(a, b) and np.array_equal(aw, bw)


@pytest.mark.parametrize("mode", MODES)
def test_cluster_probe_shards_merge(engine, mode):
    """Clustering across GPUs, on one: the clusters of 3 probe shards (each finds its own intersecting pairs) joined
    by gsj_cluster_merge equal the single-pass roots, on a layer with components of every size and on its pieces."""
    ps = shrunk_parcels(30000, (-118.3, 33.95, -118.15, 34.1), seed=12)
    for layer, nparent in ((ps, ps.n), (gsj.subdivide(ps, 16), ps.n)):
        L = engine.upload_polygons(layer)
        whole, _ = engine.cluster(L, nparent, refine_mode=mode)
        forests = [engine.cluster(L, nparent, refine_mode=mode, shard=k, nshards=3)[0] for k in range(3)]
        assert not any(np.array_equal(f, whole) for f in forests)   # each shard alone misses connections
        assert np.array_equal(engine.cluster_merge(forests), whole)
        assert np.array_equal(whole, O.cluster(O.OSet(layer), nparent))
