"""Pair-level parity with the reference engine at the benchmarked sizes, on non-degenerate inputs (GPU box).

The reference's own file driver (landstats-us/postgis-cuda engine/harness.cu, unmodified, built for sm_100a into
oracle/_ref/harness by oracle/build_ref.sh) runs on the same seeded layers and writes every result row
(engine/harness.cu:78-86, :124-127, :150-153, :203); gsj's rows must be the same set, with the same DE-9IM matrices,
the same cluster numbering, and areas within 1e-9 relative (the reference build contracts multiply-adds, gsj does
not; absolute 1e-15 deg^2 for areas that cancel to ~0 on shared boundaries). Both refinement variants are checked.

Layers: the headline relate self-join of 2M parcels; 2M parcels against an independently seeded 2M-parcel layer
(interiors overlap: non-zero areas, every DE-9IM cell in play); 1M points x 1M parcels ST_DWithin 5 m; erosion of
two independently seeded 2M-parcel layers (pairs survive 1 m erosion); ST_ClusterIntersecting of 2M parcels of
which a seeded 55 % are shrunk, so the intersects graph falls into components of every size.
"""
import os

import numpy as np
import pytest

import gsj
import refharness as RH
from gsj import gen

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not RH.available(), reason="oracle/_ref/harness is not built (oracle/build_ref.sh)")]
MODES = [gsj.GSJ_REFINE_FILTERED, gsj.GSJ_REFINE_PLAIN]
BOX = (-119.0, 33.0, -117.0, 35.0)
BOX1 = (-119.0, 33.0, -118.0, 34.0)


@pytest.fixture(scope="module")
def tmp(tmp_path_factory):
    return tmp_path_factory.mktemp("refscale")


@pytest.fixture(scope="module")
def parcels(tmp):
    ps = gen.layer_parcels(2_000_000, BOX, seed=0)
    p = str(tmp / "parcels2m.gset")
    gen.write_gset(p, ps)
    return ps, p


@pytest.fixture(scope="module")
def parcels_b(tmp):
    ps = gen.layer_parcels(2_000_000, BOX, seed=1)
    p = str(tmp / "parcels2m_b.gset")
    gen.write_gset(p, ps)
    return ps, p


def assert_areas(got, want):
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-15)


def test_relate_self_join_2m(engine, tmp, parcels):
    ps, p = parcels
    out = str(tmp / "relate_self.csv")
    res = RH.run([p, p, "--relate"], out_csv=out)
    rows, codes = RH.read_pairs_csv(out)
    os.remove(out)
    want_p, want_c = RH.upper_rows(rows, codes)
    n_diag = int((want_p[:, 0] == want_p[:, 1]).sum())
    assert len(rows) == 2 * len(want_p) - n_diag == res["count"]["rows"]   # mirrored rows + the diagonal once
    L = engine.upload_polygons(ps)
    for mode in MODES + [gsj.GSJ_REFINE_FILTERED_FP32]:
        r = engine.join(L, L, want_area=False, want_relate=True, upper=True, refine_mode=mode)
        got_p, got_c = RH.sorted_rows(r.pairs, r.code)
        assert np.array_equal(got_p, want_p), f"mode {mode}: pair sets differ from the reference"
        assert np.array_equal(got_c, want_c), f"mode {mode}: {(got_c != want_c).sum()} DE-9IM matrices differ"
    assert len(want_p) > 7_000_000
    L.free()


def test_area_and_relate_two_layers_2m(engine, tmp, parcels, parcels_b):
    (pa, fa), (pb, fb) = parcels, parcels_b
    LA, LB = engine.upload_polygons(pa), engine.upload_polygons(pb)
    out = str(tmp / "ab_area.csv")
    RH.run([fa, fb, "--area"], out_csv=out)
    want_p, want_a = RH.sorted_rows(*RH.read_pairs_csv(out))
    os.remove(out)
    out = str(tmp / "ab_relate.csv")
    RH.run([fa, fb, "--relate"], out_csv=out)
    rel_p, rel_c = RH.sorted_rows(*RH.read_pairs_csv(out))
    os.remove(out)
    assert np.array_equal(rel_p, want_p)
    for mode in MODES:
        r = engine.join(LA, LB, want_area=True, want_relate=True, refine_mode=mode)
        got_p, got_a = RH.sorted_rows(r.pairs, r.area)
        _, got_c = RH.sorted_rows(r.pairs, r.code)
        assert np.array_equal(got_p, want_p), f"mode {mode}: pair sets differ from the reference"
        assert_areas(got_a, want_a)
        assert np.array_equal(got_c, rel_c), f"mode {mode}: {(got_c != rel_c).sum()} DE-9IM matrices differ"
    assert len(want_p) > 8_000_000 and (want_a > 0).mean() > 0.5    # interiors overlap
    LA.free(); LB.free()


def test_points_dwithin_1m_x_1m(engine, tmp):
    xy, ps = gen.points(1_000_000, BOX1, 7), gen.layer_parcels(1_000_000, BOX1, seed=0)
    fp, fg, out = str(tmp / "points1m.pset"), str(tmp / "parcels1m.gset"), str(tmp / "pts_dwithin.csv")
    gen.write_pset(fp, xy)
    gen.write_gset(fg, ps)
    RH.run([fp, fg, "--dwithin", "5"], out_csv=out)
    want, _ = RH.sorted_rows(RH.read_pairs_csv(out)[0])
    LP, LR = engine.upload_points(xy), engine.upload_polygons(ps)
    for mode in MODES:
        got, _ = RH.sorted_rows(engine.points_dwithin(LP, LR, 5.0, refine_mode=mode)[0])
        assert np.array_equal(got, want), f"mode {mode}: pair sets differ from the reference"
    assert len(want) > 1_000_000
    LP.free(); LR.free()


def test_erode_two_layers_2m(engine, tmp):
    A, B = gen.layer_cfg5(2_000_000, BOX, seed=0), gen.layer_cfg5(2_000_000, BOX, seed=1)
    fa, fb, out = str(tmp / "cfg5a.gset"), str(tmp / "cfg5b.gset"), str(tmp / "erode.csv")
    gen.write_gset(fa, A)
    gen.write_gset(fb, B)
    RH.run([fa, fb, "--erode", "1"], out_csv=out)
    want, _ = RH.sorted_rows(RH.read_pairs_csv(out)[0])
    LA, LB = engine.upload_polygons(A), engine.upload_polygons(B)
    for mode in MODES:
        got, _ = RH.sorted_rows(engine.erode(LA, LB, 1.0, 1.0, refine_mode=mode)[0])
        assert np.array_equal(got, want), f"mode {mode}: pair sets differ from the reference"
    assert len(want) > 1_000_000
    LA.free(); LB.free()


def test_cluster_many_components_2m(engine, tmp):
    ps = gen.shrunk(gen.layer_cfg5(2_000_000, BOX, seed=3), seed=3)
    f, out = str(tmp / "shrunk2m.gset"), str(tmp / "cluster.csv")
    gen.write_gset(f, ps)
    RH.run([f, f, "--cluster"], out_csv=out)
    want = RH.read_cluster_csv(out)
    sizes = np.unique(want, return_counts=True)[1]
    assert len(want) == ps.n and (sizes >= 2).sum() > 20_000 and (sizes >= 100).sum() > 10
    L = engine.upload_polygons(ps)
    for mode in MODES:
        root, _ = engine.cluster(L, refine_mode=mode)
        assert np.array_equal(RH.dense_labels(root), want), f"mode {mode}: cluster numbering differs from the reference"
    L.free()
