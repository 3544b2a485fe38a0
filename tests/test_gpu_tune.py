"""Refinement launch shapes and the autotuner (gsj_set_refine_shape, gsj_tune_refine) on the GPU.

A shape moves pairs between the two size bins (shared-memory lists up to bin_edges local edges per side, global
scratch above) and changes how warps take pairs; it never changes a decision. So every shape must give the oracle's
pair sets, areas and DE-9IM codes bit for bit, including shapes that send nearly every pair to the scratch bin.
"""
import numpy as np
import pytest

import gsj
import pyoracle as O
from gsj import gen

pytestmark = pytest.mark.gpu
MODES = [gsj.GSJ_REFINE_PLAIN, gsj.GSJ_REFINE_FILTERED, gsj.GSJ_REFINE_FILTERED_FP32]
SHAPES = [
    {},                                                    # the default shape
    {"run": 1, "runs": 1},                                 # one pair per fetch, one fetch per warp: the largest grid
    {"run": 16, "runs": 4096},                             # few long-lived warps
    {"bin_edges": 8, "scratch_warps_per_sm": 1},           # nearly every pair in the scratch bin, few scratch warps
    {"bin_edges": 32, "scratch_warps_per_sm": 64},
    {"run": 2, "runs": 8, "bin_edges": 96, "scratch_warps_per_sm": 8},
]


def srt(p, *vals):
    i = np.lexsort((p[:, 1], p[:, 0]))
    return (p[i],) + tuple(None if v is None else v[i] for v in vals)


@pytest.fixture(scope="module")
def layers(engine):
    hs = {
        "parcels": gen.layer_parcels(20000, (-118.3, 33.95, -118.1, 34.15), seed=5),
        "parcels2": gen.layer_parcels(15000, (-118.3, 33.95, -118.1, 34.15), seed=6),
        "zonesA": gen.voronoi(20000, gen.LA_BOX, 0, vmin=6, vmax=40),
        "zonesB": gen.voronoi(50, gen.LA_BOX, 1, vmin=4, vmax=4),
    }
    return {k: (engine.upload_polygons(v), O.OSet(v)) for k, v in hs.items()}


@pytest.fixture
def shaped(engine):
    start = engine.refine_shape
    yield engine
    engine.refine_shape = start


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("a,b,upper", [("parcels", "parcels", True), ("parcels", "parcels2", False), ("zonesA", "zonesB", False)])
def test_every_shape_gives_the_oracle_rows(shaped, layers, a, b, upper, mode):
    p, oa, oc, _ = O.join(layers[a][1], layers[b][1], O.params(1, 1), upper=upper)
    default = shaped.refine_shape
    heavy = {}
    for sh in SHAPES:
        shaped.refine_shape = {**default, **sh}
        r = shaped.join(layers[a][0], layers[b][0], want_area=True, want_relate=True, upper=upper, refine_mode=mode)
        gp, ga, gc = srt(r.pairs, r.area, r.code)
        assert np.array_equal(gp, p), f"shape {sh}: pair sets differ from the oracle"
        assert np.array_equal(ga, oa), f"shape {sh}: areas differ from the oracle"
        assert np.array_equal(gc, oc), f"shape {sh}: DE-9IM codes differ from the oracle"
        heavy[str(sh)] = r.stats["heavy"]
    # bin_edges 8 sends most contact pairs of the parcel layers to the scratch bin
    if a.startswith("parcels"):
        assert heavy[str(SHAPES[3])] > 10 * max(1, heavy[str(SHAPES[0])])


def test_shape_rejects_out_of_range(shaped):
    for bad in ({"run": 0}, {"run": 65}, {"runs": 0}, {"bin_edges": 7}, {"bin_edges": 129}, {"scratch_warps_per_sm": 65}):
        with pytest.raises(gsj.GsjError) as e:
            shaped.refine_shape = bad
        assert e.value.code == 1
    assert shaped.refine_shape == {"run": 4, "runs": 32, "bin_edges": 128, "scratch_warps_per_sm": 32}


def test_tuner_picks_a_shape_and_keeps_the_rows(shaped, layers):
    P = layers["parcels"][0]
    before = shaped.join(P, P, want_area=True, want_relate=True, upper=True)
    t = shaped.tune_refine(P, P, want_area=True, want_relate=True, max_pairs=20000)
    assert t["sample_pairs"] == 20000 and t["shapes_tried"] >= 11
    assert 0 < t["best_ms"] <= t["start_ms"]
    assert shaped.refine_shape == t["best"]
    after = shaped.join(P, P, want_area=True, want_relate=True, upper=True)
    gp, ga, gc = srt(before.pairs, before.area, before.code)
    hp, ha, hc = srt(after.pairs, after.area, after.code)
    assert np.array_equal(gp, hp) and np.array_equal(ga, ha) and np.array_equal(gc, hc)


def test_tuner_small_sample_takes_every_pair(shaped, layers):
    A, B = layers["zonesA"][0], layers["zonesB"][0]
    nc = len(shaped.candidates(A, B))
    t = shaped.tune_refine(A, B, max_pairs=10 * nc)
    assert t["sample_pairs"] == nc


def test_tuner_keeps_named_fields(shaped, layers):
    P = layers["parcels"][0]
    shaped.refine_shape = {"runs": 16, "run": 2}
    t = shaped.tune_refine(P, P, max_pairs=20000, keep=("runs", "run"))
    assert t["best"]["runs"] == 16 and t["best"]["run"] == 2
    assert t["shapes_tried"] <= 1 + 3 + 4
