"""Synthetic parcel layers (Voronoi cells with shared vertices) and points, via libgsjgen.so.

The layouts follow the reference's flat polygon set (engine/gset.h:5-11): ``gro`` u64[n+1] geometry -> first
ring, ``rvo`` u64[nr+1] ring -> first vertex, ``xy`` f64[nv, 2], closed rings, shells CCW, holes CW.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

from ._build import lib_path


class _Params(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("x0", ctypes.c_double), ("y0", ctypes.c_double), ("x1", ctypes.c_double),
                ("y1", ctypes.c_double), ("seed", ctypes.c_uint64), ("jitter_grid", ctypes.c_int), ("jitter", ctypes.c_double),
                ("vmin", ctypes.c_int), ("vmax", ctypes.c_int), ("log_uniform", ctypes.c_int), ("mp_frac", ctypes.c_double),
                ("mp_parts_min", ctypes.c_int), ("mp_parts_max", ctypes.c_int), ("hole_frac", ctypes.c_double)]


class _Set(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("nr", ctypes.c_uint64), ("nv", ctypes.c_uint64),
                ("gro", ctypes.POINTER(ctypes.c_uint64)), ("rvo", ctypes.POINTER(ctypes.c_uint64)),
                ("xy", ctypes.POINTER(ctypes.c_double)), ("n_mp", ctypes.c_uint64), ("n_holes", ctypes.c_uint64),
                ("n_inconsistent", ctypes.c_uint64)]


_lib = None


def _gen():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(lib_path("libgsjgen.so"))
        _lib.gsjgen_voronoi.argtypes = [ctypes.POINTER(_Params), ctypes.POINTER(_Set)]
        _lib.gsjgen_free.argtypes = [ctypes.POINTER(_Set)]
        _lib.gsjgen_points.argtypes = [ctypes.c_uint64] + [ctypes.c_double] * 4 + [ctypes.c_uint64, ctypes.c_void_p]
        _lib.gsjgen_write_gset.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Set)]
        _lib.gsjgen_write_pset.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_void_p]
        _lib.gsjgen_read_gset.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Set)]
    return _lib


@dataclasses.dataclass
class PolygonSet:
    """Host polygon set; ``parent``/``syn`` are set for subdivided layers (piece -> geometry, cut-edge flags)."""
    gro: np.ndarray
    rvo: np.ndarray
    xy: np.ndarray
    parent: np.ndarray | None = None
    syn: np.ndarray | None = None
    stats: dict = dataclasses.field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.gro) - 1

    @property
    def nr(self) -> int:
        return len(self.rvo) - 1

    @property
    def nv(self) -> int:
        return len(self.xy)


def _from_c(s: _Set) -> PolygonSet:
    gro = np.ctypeslib.as_array(s.gro, (s.n + 1,)).copy()
    rvo = np.ctypeslib.as_array(s.rvo, (s.nr + 1,)).copy()
    xy = np.ctypeslib.as_array(s.xy, (max(1, 2 * s.nv),))[: 2 * s.nv].copy().reshape(-1, 2)
    return PolygonSet(gro, rvo, xy, stats=dict(multipolygons=s.n_mp, holes=s.n_holes, inconsistent=s.n_inconsistent))


def voronoi(n, box, seed, *, jitter_grid=False, jitter=0.4, vmin=6, vmax=40, log_uniform=False,
            mp_frac=0.0, mp_parts=(2, 4), hole_frac=0.0) -> PolygonSet:
    p = _Params(n, box[0], box[1], box[2], box[3], seed, int(jitter_grid), jitter, vmin, vmax, int(log_uniform),
                mp_frac, mp_parts[0], mp_parts[1], hole_frac)
    s = _Set()
    rc = _gen().gsjgen_voronoi(ctypes.byref(p), ctypes.byref(s))
    if rc:
        raise RuntimeError(f"gsjgen_voronoi failed ({rc})")
    try:
        return _from_c(s)
    finally:
        _gen().gsjgen_free(ctypes.byref(s))


def points(n, box, seed) -> np.ndarray:
    xy = np.empty((n, 2), dtype=np.float64)
    _gen().gsjgen_points(n, box[0], box[1], box[2], box[3], seed, xy.ctypes.data)
    return xy


def write_gset(path: str, ps: PolygonSet) -> None:
    s = _Set(ps.n, ps.nr, ps.nv, ps.gro.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
             ps.rvo.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ps.xy.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, 0, 0)
    if _gen().gsjgen_write_gset(os.fsencode(path), ctypes.byref(s)):
        raise OSError(f"cannot write {path}")


def write_pset(path: str, xy: np.ndarray) -> None:
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    if _gen().gsjgen_write_pset(os.fsencode(path), len(xy), xy.ctypes.data):
        raise OSError(f"cannot write {path}")


def read_gset(path: str) -> PolygonSet:
    s = _Set()
    if _gen().gsjgen_read_gset(os.fsencode(path), ctypes.byref(s)):
        raise OSError(f"cannot read {path}")
    try:
        return _from_c(s)
    finally:
        _gen().gsjgen_free(ctypes.byref(s))


# ---- the layers the benchmarks and tests are quoted on (seeded; identical bytes on every run) -------------
LA_BOX = (-118.5, 33.8, -118.0, 34.3)


def layer_cfg_parcels_small(n=20000, seed=0) -> PolygonSet:
    """Voronoi cells of uniform seeds in the LA box, edges subdivided so rings have ~6-40 vertices."""
    return voronoi(n, LA_BOX, seed, vmin=6, vmax=40)


def layer_cfg_zones(n=50, seed=1) -> PolygonSet:
    """Large raw Voronoi cells over the same box (the 'soils/counties' side of the small config)."""
    return voronoi(n, LA_BOX, seed, vmin=4, vmax=4)


def layer_cfg5(n, box, seed=0) -> PolygonSet:
    """Jittered-grid parcels with ~30 vertices per ring (uniform 6-54), 5% MultiPolygons (2-4 parts), 2% holes."""
    return voronoi(n, box, seed, jitter_grid=True, jitter=0.4, vmin=6, vmax=54, log_uniform=False,
                   mp_frac=0.05, mp_parts=(2, 4), hole_frac=0.02)


def layer_parcels(n, box, seed=0) -> PolygonSet:
    """Jittered-grid parcels, 4-256 vertices per ring (log-uniform), 5% MultiPolygons (2-4 parts), 2% holes."""
    return voronoi(n, box, seed, jitter_grid=True, jitter=0.4, vmin=4, vmax=256, log_uniform=True,
                   mp_frac=0.05, mp_parts=(2, 4), hole_frac=0.02)


def shrunk(ps: PolygonSet, seed: int, frac=0.55, f=0.9) -> PolygonSet:
    """A seeded fraction ``frac`` of the geometries shrunk by ``f`` toward their bbox centre. Only neighbours that both
    keep their size touch, so the intersects graph of a tiling falls into components of every size (site
    percolation): the clustering workload with many components."""
    shrink = np.random.default_rng(seed).random(ps.n) < frac
    v0 = ps.rvo[ps.gro[:-1]].astype(np.int64)
    cnt = np.diff(np.append(v0, ps.nv))
    lo = np.minimum.reduceat(ps.xy, v0, axis=0)
    hi = np.maximum.reduceat(ps.xy, v0, axis=0)
    c = np.repeat(0.5 * (lo + hi), cnt, axis=0)
    m = np.repeat(shrink, cnt)
    xy = ps.xy.copy()
    xy[m] = c[m] + f * (xy[m] - c[m])
    return PolygonSet(ps.gro, ps.rvo, xy)
