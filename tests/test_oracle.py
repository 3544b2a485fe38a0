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
        big = np.abs(gv) > 1e-18
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
