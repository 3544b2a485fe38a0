"""ctypes binding of the CPU FP64 oracle (oracle.cpp) - TEST INFRASTRUCTURE ONLY.

Imported by tests/, by ``__graft_entry__.smoke()`` and by the bench's cpu_baseline leg / reference arm, never by
the engine. Builds ``oracle/_build/liboracle.so`` with ``make -C oracle`` when it is missing.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None

u32p = ctypes.POINTER(ctypes.c_uint32)
f64p = ctypes.POINTER(ctypes.c_double)
u8p = ctypes.POINTER(ctypes.c_uint8)


class Params(ctypes.Structure):
    _fields_ = [("tol_rel", ctypes.c_double), ("eps_par", ctypes.c_double), ("tol_abs", ctypes.c_double),
                ("want_area", ctypes.c_int), ("want_relate", ctypes.c_int), ("snap_half_ulp", ctypes.c_int)]


def params(want_area=1, want_relate=0, snap_half_ulp=0, tol_rel=1e-12, eps_par=1e-7, tol_abs=1e-11) -> Params:
    return Params(tol_rel, eps_par, tol_abs, want_area, want_relate, snap_half_ulp)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE], check=True)
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.orc_set_create.restype = vp
        L.orc_set_create.argtypes = [ctypes.c_uint64] * 3 + [vp] * 5
        L.orc_set_free.argtypes = [vp]
        L.orc_set_bbox.argtypes = [vp, vp]
        L.orc_candidates.restype = ctypes.c_int64
        L.orc_candidates.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(u32p)]
        L.orc_candidates_bb.restype = ctypes.c_int64
        L.orc_candidates_bb.argtypes = [vp, ctypes.c_uint64, vp, ctypes.c_int, ctypes.POINTER(u32p)]
        L.orc_refine_pairs.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.POINTER(Params), vp, vp, vp, vp, ctypes.c_int]
        L.orc_join.restype = ctypes.c_int64
        L.orc_join.argtypes = [vp, vp, ctypes.POINTER(Params), ctypes.c_int, ctypes.c_int, ctypes.POINTER(u32p), ctypes.POINTER(f64p),
                               ctypes.POINTER(u32p), ctypes.POINTER(ctypes.c_int64)]
        L.orc_de9im_code.restype = ctypes.c_uint32
        L.orc_de9im_code.argtypes = [vp, ctypes.c_uint32, ctypes.c_double, ctypes.c_double]
        L.orc_de9im_transpose.restype = ctypes.c_uint32
        L.orc_de9im_transpose.argtypes = [ctypes.c_uint32]
        L.orc_de9im_match.restype = ctypes.c_int
        L.orc_de9im_match.argtypes = [ctypes.c_uint32, ctypes.c_char_p]
        L.orc_blen.restype = ctypes.c_double
        L.orc_blen.argtypes = [vp, ctypes.c_uint32]
        L.orc_pip.restype = ctypes.c_int64
        L.orc_pip.argtypes = [vp, ctypes.c_uint64, vp, ctypes.c_int, ctypes.POINTER(u32p), ctypes.POINTER(u8p), ctypes.POINTER(ctypes.c_int64)]
        L.orc_cluster.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(Params), ctypes.c_int, vp]
        for name in ("orc_dwithin",):
            if hasattr(L, name):
                f = getattr(L, name)
                f.restype = ctypes.c_int64
                f.argtypes = [vp, vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(u32p), ctypes.POINTER(ctypes.c_int64)]
        for name in ("orc_pt_dwithin", "orc_pt_erode"):
            if hasattr(L, name):
                f = getattr(L, name)
                f.restype = ctypes.c_int64
                f.argtypes = [vp, ctypes.c_uint64, vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(u32p)]
        if hasattr(L, "orc_erode"):
            L.orc_erode.restype = ctypes.c_int64
            L.orc_erode.argtypes = [vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(u32p)]
        u64pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_uint64))
        L.orc_subdivide.restype = ctypes.c_int64
        L.orc_subdivide.argtypes = [ctypes.c_uint64, vp, vp, vp, ctypes.c_int, u64pp, u64pp, ctypes.POINTER(f64p), ctypes.POINTER(u32p),
                                    ctypes.POINTER(u8p), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.orc_dedup.restype = ctypes.c_int64
        L.orc_dedup.argtypes = [ctypes.c_uint64, vp, vp, vp, ctypes.c_int, u64pp, u64pp, ctypes.POINTER(f64p), u64pp, ctypes.POINTER(u32p),
                                ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.orc_free.argtypes = [vp]
        _lib = L
    return _lib


def _take(ptr, count, dtype, shape=None):
    if count == 0:
        lib().orc_free(ptr)
        return np.zeros(shape if shape is not None else (0,), dtype=dtype)
    a = np.ctypeslib.as_array(ptr, (count,)).copy().astype(dtype, copy=False)
    lib().orc_free(ptr)
    return a.reshape(shape) if shape is not None else a


class OSet:
    """A polygon set prepared by the oracle (upload_set semantics)."""

    def __init__(self, ps, parent=None, syn=None):
        self.gro = np.ascontiguousarray(ps.gro, dtype=np.uint64)
        self.rvo = np.ascontiguousarray(ps.rvo, dtype=np.uint64)
        self.xy = np.ascontiguousarray(ps.xy, dtype=np.float64)
        parent = parent if parent is not None else getattr(ps, "parent", None)
        syn = syn if syn is not None else getattr(ps, "syn", None)
        self.parent = None if parent is None else np.ascontiguousarray(parent, dtype=np.uint32)
        self.syn = None if syn is None else np.ascontiguousarray(syn, dtype=np.uint8)
        self.n = len(self.gro) - 1
        self.h = lib().orc_set_create(self.n, len(self.rvo) - 1, len(self.xy), self.gro.ctypes.data, self.rvo.ctypes.data,
                                      self.xy.ctypes.data, None if self.parent is None else self.parent.ctypes.data,
                                      None if self.syn is None else self.syn.ctypes.data)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_set_free(self.h)
            self.h = None

    def bbox(self) -> np.ndarray:
        bb = np.empty((self.n, 4), dtype=np.float32)
        lib().orc_set_bbox(self.h, bb.ctypes.data)
        return bb

    def blen(self, p: int) -> float:
        return lib().orc_blen(self.h, p)


def candidates(P: OSet, R: OSet, upper=False) -> np.ndarray:
    out = u32p()
    n = lib().orc_candidates(P.h, R.h, int(upper), ctypes.byref(out))
    return _take(out, 2 * n, np.uint32, (n, 2))


def candidates_bb(qbb: np.ndarray, R: OSet, upper=False) -> np.ndarray:
    qbb = np.ascontiguousarray(qbb, dtype=np.float32)
    out = u32p()
    n = lib().orc_candidates_bb(qbb.ctypes.data, len(qbb), R.h, int(upper), ctypes.byref(out))
    return _take(out, 2 * n, np.uint32, (n, 2))


def refine_pairs(P: OSet, R: OSet, pairs: np.ndarray, rp: Params, nthreads=0):
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    n = len(pairs)
    flag = np.zeros(n, np.uint8); area = np.zeros(n, np.float64); ev = np.zeros((n, 4), np.float64); evb = np.zeros(n, np.uint32)
    lib().orc_refine_pairs(P.h, R.h, pairs.ctypes.data, n, ctypes.byref(rp), flag.ctypes.data, area.ctypes.data, ev.ctypes.data,
                           evb.ctypes.data, nthreads)
    return flag, area, ev, evb


def join(P: OSet, R: OSet, rp: Params, upper=False, nthreads=0):
    """Parent pairs (sorted by a, b), areas, DE-9IM codes, candidate count."""
    op, oa, oc, nc = u32p(), f64p(), u32p(), ctypes.c_int64()
    n = lib().orc_join(P.h, R.h, ctypes.byref(rp), int(upper), nthreads, ctypes.byref(op), ctypes.byref(oa), ctypes.byref(oc), ctypes.byref(nc))
    return _take(op, 2 * n, np.uint32, (n, 2)), _take(oa, n, np.float64), _take(oc, n, np.uint32), nc.value


def pip(pts: np.ndarray, R: OSet, nthreads=0):
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    op, ow, nc = u32p(), u8p(), ctypes.c_int64()
    n = lib().orc_pip(pts.ctypes.data, len(pts), R.h, nthreads, ctypes.byref(op), ctypes.byref(ow), ctypes.byref(nc))
    return _take(op, 2 * n, np.uint32, (n, 2)), _take(ow, n, np.uint8), nc.value


def cluster(P: OSet, nparent: int, nthreads=0) -> np.ndarray:
    root = np.empty(nparent, np.uint32)
    rp = params(0, 0)
    lib().orc_cluster(P.h, nparent, ctypes.byref(rp), nthreads, root.ctypes.data)
    return root


def dwithin(P: OSet, R: OSet, d: float, same=False, nthreads=0):
    op, nc = u32p(), ctypes.c_int64()
    n = lib().orc_dwithin(P.h, R.h, d, int(same), nthreads, ctypes.byref(op), ctypes.byref(nc))
    return _take(op, 2 * n, np.uint32, (n, 2)), nc.value


def pt_dwithin(pts, R: OSet, d: float, nthreads=0):
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    op = u32p()
    n = lib().orc_pt_dwithin(pts.ctypes.data, len(pts), R.h, d, nthreads, ctypes.byref(op))
    return _take(op, 2 * n, np.uint32, (n, 2))


def pt_erode(pts, R: OSet, r: float, nthreads=0):
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    op = u32p()
    n = lib().orc_pt_erode(pts.ctypes.data, len(pts), R.h, r, nthreads, ctypes.byref(op))
    return _take(op, 2 * n, np.uint32, (n, 2))


def erode(P: OSet, R: OSet, ra: float, rb: float, same=False, need_self=None, nthreads=0):
    op = u32p()
    ns = None if need_self is None else np.ascontiguousarray(need_self, dtype=np.uint8)
    n = lib().orc_erode(P.h, R.h, ra, rb, int(same), None if ns is None else ns.ctypes.data, nthreads, ctypes.byref(op))
    return _take(op, 2 * n, np.uint32, (n, 2))


def _host_set(ps):
    return (np.ascontiguousarray(ps.gro, np.uint64), np.ascontiguousarray(ps.rvo, np.uint64), np.ascontiguousarray(ps.xy, np.float64))


def subdivide(ps, maxv: int):
    """Pieces of at most ~maxv vertices (a PolygonSet-like object with .parent and .syn), restated on the CPU."""
    from gsj.gen import PolygonSet
    gro, rvo, xy = _host_set(ps)
    u64 = ctypes.POINTER(ctypes.c_uint64)
    og, orv, oxy, opar, osyn = u64(), u64(), f64p(), u32p(), u8p()
    nr, nv = ctypes.c_uint64(), ctypes.c_uint64()
    n = lib().orc_subdivide(len(gro) - 1, gro.ctypes.data, rvo.ctypes.data, xy.ctypes.data, int(maxv), ctypes.byref(og), ctypes.byref(orv),
                            ctypes.byref(oxy), ctypes.byref(opar), ctypes.byref(osyn), ctypes.byref(nr), ctypes.byref(nv))
    return PolygonSet(_take(og, n + 1, np.uint64), _take(orv, nr.value + 1, np.uint64), _take(oxy, 2 * nv.value, np.float64, (nv.value, 2)),
                      parent=_take(opar, n, np.uint32), syn=_take(osyn, nv.value, np.uint8))


def dedup(ps, morton=False):
    """(distinct PolygonSet, moff, midx), restated on the CPU."""
    from gsj.gen import PolygonSet
    gro, rvo, xy = _host_set(ps)
    u64 = ctypes.POINTER(ctypes.c_uint64)
    og, orv, oxy, omo, omi = u64(), u64(), f64p(), u64(), u32p()
    nr, nv = ctypes.c_uint64(), ctypes.c_uint64()
    n = lib().orc_dedup(len(gro) - 1, gro.ctypes.data, rvo.ctypes.data, xy.ctypes.data, int(morton), ctypes.byref(og), ctypes.byref(orv),
                        ctypes.byref(oxy), ctypes.byref(omo), ctypes.byref(omi), ctypes.byref(nr), ctypes.byref(nv))
    u = PolygonSet(_take(og, n + 1, np.uint64), _take(orv, nr.value + 1, np.uint64), _take(oxy, 2 * nv.value, np.float64, (nv.value, 2)))
    return u, _take(omo, n + 1, np.uint64), _take(omi, len(gro) - 1, np.uint32)


def de9im_str(code: int) -> str:
    return "".join("F012"[(code >> (2 * k)) & 3] for k in range(9))


def de9im_transpose(code: int) -> int:
    return lib().orc_de9im_transpose(code)


def de9im_match(code: int, pat: str) -> bool:
    return bool(lib().orc_de9im_match(code, pat.encode()))
