"""The CPU FP64 oracle: known answers and golden vectors of the reference engine (engine/harness.cu run on a B200)."""
import numpy as np
import pytest

import make_golden as MG
import pyoracle as O
import shapes

PT_INTERIOR = 1 | 3 << 12 | 2 << 14 | 3 << 16
PT_BOUNDARY = 1 << 2 | 3 << 12 | 2 << 14 | 3 << 16


@pytest.mark.parametrize("name,a,b,rel,area", shapes.CASES)
def test_known_answers(name, a, b, rel, area):
    A, B = O.OSet(shapes.make_set([a])), O.OSet(shapes.make_set([b]))
    p, ar, code, nc = O.join(A, B, O.params(1, 1))
    if rel is None:
        assert len(p) == 0
        return
    assert len(p) == 1 and O.de9im_str(int(code[0])) == rel
    assert abs(ar[0] - area) <= 1e-9 * max(area, 1e-12) + 1e-20


def test_de9im_helpers():
    for c in [PT_INTERIOR, PT_BOUNDARY, 0x3FFFF, 0]:
        assert O.de9im_transpose(O.de9im_transpose(c)) == c
    assert O.de9im_str(PT_INTERIOR) == "0FFFFF212" and O.de9im_str(PT_BOUNDARY) == "F0FFFF212"
    code = int(sum(v << (2 * k) for k, v in enumerate([3, 0, 3, 0, 2, 2, 3, 2, 3])))   # 2F2F11212
    assert O.de9im_match(code, "T*T***T**") and not O.de9im_match(code, "T*F**F***") and O.de9im_match(code, "2f2F1121*")


@pytest.fixture(scope="module")
def golden_layers():
    return {k: b() for k, (kind, b) in MG.layers().items()}


def sorted_rows(p, v):
    i = np.lexsort((p[:, 1], p[:, 0]))
    return p[i], v[i]


def mirror(p, v, tr=None):
    """Self-join rows as the reference harness writes them: both orders, the diagonal once."""
    off = p[:, 0] != p[:, 1]
    pm = np.concatenate([p, p[off][:, ::-1]])
    vm = np.concatenate([v, np.array([tr(int(x)) for x in v[off]], dtype=v.dtype) if tr else v[off]])
    return pm, vm


def check_pairs(case, p, v, kind):
    g = np.load(f"{MG.HERE}/{case}.npz")
    gp, gv = sorted_rows(g["pairs"], g[kind])
    p, v = sorted_rows(p, v)
    assert np.array_equal(p, gp), f"{case}: pair sets differ"
    if kind == "area":
        # relative 1e-9 where the area is meaningful (> 1e-12 deg^2, ~0.01 m^2); touching pairs carry rounding
        # noise of ~1e-20 deg^2 in both engines, bounded absolutely
        big = np.abs(gv) > 1e-12
        rel = np.abs(v - gv)[big] / np.abs(gv[big])
        assert rel.max(initial=0) <= 1e-9, f"{case}: area rel err {rel.max()}"
        assert np.abs(v - gv).max(initial=0) <= 1e-18
    else:
        assert list(map(O.de9im_str, map(int, v))) == list(gv), f"{case}: DE-9IM differs"


def test_golden_inputs_unchanged(golden_layers, tmp_path):
    from gsj import gen
    for case in ("ab_area", "pp_relate", "pts_pip"):
        pa, pb, _ = MG.CASES[case]
        want = np.load(f"{MG.HERE}/{case}.npz")["inputs_sha256"]
        for name, w in zip((pa, pb), want):
            kind = MG.layers()[name][0]
            path = str(tmp_path / f"{name}.{kind}")
            (gen.write_gset if kind == "gset" else gen.write_pset)(path, golden_layers[name])
            assert MG.sha(path) == w


def test_golden_area_join(golden_layers):
    A, B = O.OSet(golden_layers["zonesA"]), O.OSet(golden_layers["zonesB"])
    p, a, c, _ = O.join(A, B, O.params(1, 0))
    check_pairs("ab_area", p, a, "area")
    assert abs(a.sum() - 0.25) < 1e-12          # both layers tile the same 0.5 x 0.5 deg box
    p, a, c, _ = O.join(A, A, O.params(1, 0), upper=True)
    check_pairs("aa_area", *mirror(p, a), "area")


def test_golden_relate(golden_layers):
    P, B = O.OSet(golden_layers["parcels"]), O.OSet(golden_layers["zonesB"])
    p, a, c, _ = O.join(P, P, O.params(0, 1), upper=True)
    check_pairs("pp_relate", *mirror(p, c, O.de9im_transpose), "relate")
    p, a, c, _ = O.join(P, B, O.params(0, 1))
    check_pairs("pb_relate", p, c, "relate")


def test_golden_pip_and_cluster(golden_layers):
    P = O.OSet(golden_layers["parcels"])
    p, w, _ = O.pip(golden_layers["points"], P)
    check_pairs("pts_pip", p, np.where(w == 2, PT_BOUNDARY, PT_INTERIOR).astype(np.uint32), "relate")
    root = O.cluster(P, P.n)
    first, lab = {}, []
    for r in root.tolist():
        lab.append(first.setdefault(r, len(first)))
    assert np.array_equal(np.array(lab), np.load(f"{MG.HERE}/cluster.npz")["label"])


def test_golden_dwithin(golden_layers):
    P = O.OSet(golden_layers["parcels"])
    p, nc = O.dwithin(P, P, 5.0, same=True)
    off = p[:, 0] != p[:, 1]
    pm = np.concatenate([p, p[off][:, ::-1]])
    g = np.load(f"{MG.HERE}/pp_dwithin5.npz")["pairs"]
    assert set(map(tuple, pm.tolist())) == set(map(tuple, g.tolist()))
    g = np.load(f"{MG.HERE}/pts_dwithin5.npz")["pairs"]
    p = O.pt_dwithin(golden_layers["points"], P, 5.0)
    assert set(map(tuple, p.tolist())) == set(map(tuple, g.tolist()))


@pytest.fixture(scope="module")
def sub32(golden_layers):
    return O.subdivide(golden_layers["parcels"], 32)


def test_subdivision_matches_reference_pieces(golden_layers, sub32):
    """The oracle's pieces give the reference engine's subdivided results (same cut points, cut flags); the GPU
    subdivision is checked against these pieces bit for bit in the GPU tests."""
    assert sub32.n == 11203 and int(sub32.parent.max()) == golden_layers["parcels"].n - 1
    S = O.OSet(sub32)
    p, a, c, _ = O.join(S, S, O.params(1, 0), upper=True)
    check_pairs("pp_area_sub32", *mirror(p, a), "area")
    p, a, c, _ = O.join(S, S, O.params(0, 1), upper=True)
    check_pairs("pp_relate_sub32", *mirror(p, c, O.de9im_transpose), "relate")
    p, w, _ = O.pip(golden_layers["points"], S)
    check_pairs("pts_pip_sub32", p, np.where(w == 2, PT_BOUNDARY, PT_INTERIOR).astype(np.uint32), "relate")
    root = O.cluster(S, golden_layers["parcels"].n)
    first, lab = {}, []
    for r in root.tolist():
        lab.append(first.setdefault(r, len(first)))
    assert np.array_equal(np.array(lab), np.load(f"{MG.HERE}/cluster_sub32.npz")["label"])
    p, _ = O.dwithin(S, S, 5.0, same=True)
    off = p[:, 0] != p[:, 1]
    assert set(map(tuple, np.concatenate([p, p[off][:, ::-1]]).tolist())) == set(map(tuple, np.load(f"{MG.HERE}/pp_dwithin5_sub32.npz")["pairs"].tolist()))


def test_subdivision_preserves_area(sub32, golden_layers):
    def area(ps):
        tot = 0.0
        for r in range(ps.nr):
            v = ps.xy[ps.rvo[r]:ps.rvo[r + 1]] - ps.xy[ps.rvo[r]]
            tot += 0.5 * np.sum(v[:-1, 0] * v[1:, 1] - v[1:, 0] * v[:-1, 1])
        return tot
    assert abs(area(sub32) - area(golden_layers["parcels"])) < 1e-12
    assert sub32.syn.sum() > 0 and np.diff(sub32.parent.astype(np.int64)).min() >= 0


def test_dedup_members():
    import gsj
    from gsj import gen
    ps = gen.voronoi(300, gen.LA_BOX, 3)
    # stack copies of geometries 5 and 7 (condo-style duplicates) at the end
    sel = [5, 7, 5]
    gro, rvo, xy = list(ps.gro), list(ps.rvo), [ps.xy]
    for g in sel:
        for r in range(ps.gro[g], ps.gro[g + 1]):
            v = ps.xy[ps.rvo[r]:ps.rvo[r + 1]]
            xy.append(v); rvo.append(rvo[-1] + len(v))
        gro.append(len(rvo) - 1)
    dup = gen.PolygonSet(np.array(gro, np.uint64), np.array(rvo, np.uint64), np.concatenate(xy))
    u, moff, midx = O.dedup(dup)
    assert u.n == ps.n and list(midx[moff[5]:moff[6]]) == [5, 300, 302] and list(midx[moff[7]:moff[8]]) == [7, 301]
    um, moffm, midxm = O.dedup(dup, morton=True)
    assert um.n == ps.n and sorted(np.diff(moffm).tolist()) == sorted(np.diff(moff).tolist())


def rowset(p):
    return set(map(tuple, np.asarray(p).reshape(-1, 2).tolist()))


def self_rows(p):
    off = p[:, 0] != p[:, 1]
    return rowset(np.concatenate([p, p[off][:, ::-1]]))


def test_golden_erode(golden_layers, sub32):
    """ST_Intersects(ST_Buffer(a, -1 m), ST_Buffer(b, -1 m)) and points in ST_Buffer(b, -1 m), whole and subdivided."""
    P = O.OSet(golden_layers["parcels"])
    none = np.zeros(golden_layers["parcels"].n, np.uint8)   # the harness's need_self without dedup: no self rows
    p = O.erode(P, P, 1.0, 1.0, same=True, need_self=none)
    assert self_rows(p) == rowset(np.load(f"{MG.HERE}/pp_erode1.npz")["pairs"])
    S = O.OSet(sub32)
    p = O.erode(S, S, 1.0, 1.0, same=True, need_self=none)
    assert self_rows(p) == rowset(np.load(f"{MG.HERE}/pp_erode1_sub32.npz")["pairs"])
    p = O.pt_erode(golden_layers["points"], P, 1.0)
    assert rowset(p) == rowset(np.load(f"{MG.HERE}/pts_erode1.npz")["pairs"])


def test_golden_two_layer_cases(golden_layers):
    """Two overlapping parcel layers (different seeds): area, DE-9IM, eroded intersects with equal and unequal radii,
    the subdivided erosion, dwithin, and points in subdivided eroded parcels."""
    import gsj
    P, Q = O.OSet(golden_layers["parcels"]), O.OSet(golden_layers["parcels2"])
    p, a, c, _ = O.join(P, Q, O.params(1, 0))
    check_pairs("pq_area", p, a, "area")
    p, a, c, _ = O.join(P, Q, O.params(0, 1))
    check_pairs("pq_relate", p, c, "relate")
    for case, ra, rb in (("pq_erode1", 1.0, 1.0), ("pq_erode1_3", 1.0, 3.0), ("pq_erode5", 5.0, 5.0)):
        assert rowset(O.erode(P, Q, ra, rb)) == rowset(np.load(f"{MG.HERE}/{case}.npz")["pairs"]), case
    SP = O.OSet(O.subdivide(golden_layers["parcels"], 32))
    SQ = O.OSet(O.subdivide(golden_layers["parcels2"], 32))
    assert rowset(O.erode(SP, SQ, 1.0, 1.0)) == rowset(np.load(f"{MG.HERE}/pq_erode1_sub32.npz")["pairs"])
    p, _ = O.dwithin(P, Q, 5.0)
    assert rowset(p) == rowset(np.load(f"{MG.HERE}/pq_dwithin5.npz")["pairs"])
    p = O.pt_erode(golden_layers["points"], SP, 3.0)
    assert rowset(p) == rowset(np.load(f"{MG.HERE}/pts_erode3_sub32.npz")["pairs"])
