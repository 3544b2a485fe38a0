"""The certified FP32 sign filter of the orientation test (csrc/geom.cuh orient_sign32), restated with numpy float32
arithmetic and checked against exact rational arithmetic: whenever the filter decides a sign, it is the sign of the
exact determinant of the FP64 differences and the sign the FP64 routine (the reference's compensated orient,
engine/engine.cuh:283-289) returns; undecided cases fall back to that routine. The GPU parity tests check the device
code itself, bit for bit, in the GSJ_REFINE_FILTERED_FP32 mode.
"""
from fractions import Fraction

import numpy as np

U_BOUND = np.float32(3.6e-7)   # 6 x 2^-24, rounded up
TINY = np.float32(1e-30)


def orient64(ax, ay, bx, by, cx, cy):
    """The FP64 routine: a = bx-ax, b = cy-ay, c = by-ay, d = cx-ax; w = c*d; e = fma(-c, d, w); f = fma(a, b, -w);
    f + e. fma is emulated exactly with rationals (one rounding of the exact value)."""
    a, b, c, d = bx - ax, cy - ay, by - ay, cx - ax
    w = c * d
    e = float(Fraction(w) - Fraction(c) * Fraction(d))
    f = float(Fraction(a) * Fraction(b) - Fraction(w))
    return f + e, (a, b, c, d)


def sign_filter32(a, b, c, d):
    """orient_sign32's FP32 stage on the FP64 differences: +1 / -1 when decided, None when the FP64 routine decides."""
    p = np.float32(a) * np.float32(b)
    q = np.float32(c) * np.float32(d)
    ap, aq = abs(p), abs(q)
    if ap >= TINY and aq >= TINY:
        det = p - q
        bound = U_BOUND * (ap + aq)
        if det > bound:
            return 1
        if det < -bound:
            return -1
    return None


def exact_sign(a, b, c, d):
    v = Fraction(a) * Fraction(b) - Fraction(c) * Fraction(d)
    return (v > 0) - (v < 0)


def cases(rng, n):
    """Triples near a line (the hard cases), shared vertices, tiny and large offsets, in a parcel-sized local frame."""
    out = []
    for k in range(n):
        ax, ay = rng.uniform(0, 2e-3, 2)
        bx, by = ax + rng.uniform(-1e-3, 1e-3), ay + rng.uniform(-1e-3, 1e-3)
        t = rng.uniform(-0.5, 1.5)
        cx, cy = ax + t * (bx - ax), ay + t * (by - ay)
        kind = k % 5
        if kind == 0:   # on the line up to rounding
            pass
        elif kind == 1:   # a tiny perpendicular offset (near-degenerate)
            eps = 10.0 ** rng.uniform(-22, -8)
            cx, cy = cx - eps * (by - ay), cy + eps * (bx - ax)
        elif kind == 2:   # a shared vertex: exactly degenerate
            cx, cy = bx, by
        elif kind == 3:   # far from the line
            cx, cy = cx + rng.uniform(-1e-3, 1e-3), cy + rng.uniform(-1e-3, 1e-3)
        else:   # coordinates differing in the last bits only
            cx, cy = np.nextafter(ax, 1.0), np.nextafter(ay, -1.0)
        out.append((ax, ay, bx, by, cx, cy))
    return out


def test_filter_decisions_are_certified():
    rng = np.random.default_rng(0)
    decided = 0
    for ax, ay, bx, by, cx, cy in cases(rng, 6000):
        o, (a, b, c, d) = orient64(ax, ay, bx, by, cx, cy)
        s = sign_filter32(a, b, c, d)
        if s is None:
            continue
        decided += 1
        assert s == exact_sign(a, b, c, d)
        assert s == ((o > 0) - (o < 0)) and o != 0
    assert decided > 2000   # the far and most of the offset cases are decided in FP32


def test_degenerate_cases_fall_back():
    # exact zeros (shared vertices, collinear runs) and products too small for normal floats are left to FP64
    assert sign_filter32(1e-3, 0.0, 2e-3, 5e-4) is None
    assert sign_filter32(0.0, 0.0, 0.0, 0.0) is None
    assert sign_filter32(1e-20, 1e-20, 3e-4, 4e-4) is None
    assert sign_filter32(1e-3, 2e-3, 2e-3, 1e-3) is None   # equal products: det 0
