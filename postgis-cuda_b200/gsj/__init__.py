"""Python binding of the gsj C ABI (include/gsj.h) over ctypes.

The engine is ``_build/libgsj.so`` (hand-written sm_100a kernels + C++ host drivers). This module only moves
host arrays in and out; every join runs in the library. There is no CPU fallback: without a CUDA device (or
without the built library) the calls raise.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from ._build import lib_path

GSJ_REFINE_PLAIN = 0
GSJ_REFINE_FILTERED = 1
GSJ_REFINE_FILTERED_FP32 = 2   # the filtered variant with certified FP32 sign filters in front of its orientation tests

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p

JOIN_SINK = ctypes.CFUNCTYPE(ctypes.c_int, _vp, _u32p, _f64p, _u32p, ctypes.c_uint64)
POINTS_SINK = ctypes.CFUNCTYPE(ctypes.c_int, _vp, _u32p, _u8p, ctypes.c_uint64)
PAIRS_SINK = ctypes.CFUNCTYPE(ctypes.c_int, _vp, _u32p, ctypes.c_uint64)
BYTES_SINK = ctypes.CFUNCTYPE(ctypes.c_int, _vp, _u8p, ctypes.c_uint64, ctypes.c_uint64)
GSJ_ENC_PAIRS, GSJ_ENC_RELATE, GSJ_ENC_POINTS, GSJ_ENC_POINT_RELATE = 0, 1, 2, 3


class EncodeSpec(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("same", ctypes.c_int), ("distinct", ctypes.c_int), ("swapped", ctypes.c_int),
                ("point_value", ctypes.c_double), ("pattern", ctypes.c_char * 10)]


class RefineParams(ctypes.Structure):
    _fields_ = [("tol_rel", ctypes.c_double), ("eps_par", ctypes.c_double), ("tol_abs", ctypes.c_double),
                ("want_area", ctypes.c_int), ("want_relate", ctypes.c_int), ("snap_half_ulp", ctypes.c_int)]


class JoinOpts(ctypes.Structure):
    _fields_ = [("batch_q", ctypes.c_uint32), ("max_pairs", ctypes.c_uint64), ("upper", ctypes.c_int), ("no_agg", ctypes.c_int),
                ("refine_mode", ctypes.c_int), ("cancel", ctypes.POINTER(ctypes.c_int)), ("shard", ctypes.c_uint32), ("nshards", ctypes.c_uint32)]


class JoinStats(ctypes.Structure):
    _fields_ = [("traverse_ms", ctypes.c_double), ("refine_ms", ctypes.c_double), ("compact_ms", ctypes.c_double),
                ("copy_ms", ctypes.c_double), ("candidates", ctypes.c_uint64), ("hits", ctypes.c_uint64), ("heavy", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("launches", ctypes.c_uint64), ("node_visits", ctypes.c_uint64),
                ("edge_pairs", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RefineShape(ctypes.Structure):
    _fields_ = [("run", ctypes.c_int), ("runs", ctypes.c_int), ("bin_edges", ctypes.c_int), ("scratch_warps_per_sm", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneResult(ctypes.Structure):
    _fields_ = [("best", RefineShape), ("start_ms", ctypes.c_double), ("best_ms", ctypes.c_double), ("sample_pairs", ctypes.c_uint64),
                ("shapes_tried", ctypes.c_uint32)]


class LayerInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("nr", ctypes.c_uint64), ("nv", ctypes.c_uint64), ("nparent", ctypes.c_uint32),
                ("is_points", ctypes.c_int), ("max_geom_edges", ctypes.c_uint32), ("device_bytes", ctypes.c_uint64)]


class GsjError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gsj error {code}: {msg}")
        self.code = code


_lib = None

# exported symbols with their ctypes signatures (restype, argtypes)
SIGNATURES = {
    "gsj_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "gsj_ctx_destroy": (None, [_vp]),
    "gsj_last_error": (ctypes.c_char_p, [_vp]),
    "gsj_ctx_stream": (_vp, [_vp]),
    "gsj_device_query": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "gsj_ctx_create_prio": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    "gsj_dedup_gpu": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _vp, _vp, _vp, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "gsj_subdivide_gpu": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _vp, _vp, _vp, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "gsj_ctx_mem_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int)]),
    "gsj_layer_upload_polygons": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _vp, _vp, _vp, _vp, _vp,
                                                 ctypes.POINTER(_vp)]),
    "gsj_layer_upload_points": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp, ctypes.POINTER(_vp)]),
    "gsj_layer_free": (None, [_vp, _vp]),
    "gsj_layer_get_info": (ctypes.c_int, [_vp, ctypes.POINTER(LayerInfo)]),
    "gsj_refine_params_default": (None, [ctypes.POINTER(RefineParams)]),
    "gsj_join_opts_default": (None, [ctypes.POINTER(JoinOpts)]),
    "gsj_join": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(RefineParams), ctypes.POINTER(JoinOpts), JOIN_SINK, _vp, ctypes.POINTER(JoinStats)]),
    "gsj_join_points": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(JoinOpts), POINTS_SINK, _vp, ctypes.POINTER(JoinStats)]),
    "gsj_cluster": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, ctypes.POINTER(JoinOpts), _vp, ctypes.POINTER(JoinStats)]),
    "gsj_cluster_merge": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp]),
    "gsj_dwithin": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(JoinOpts), PAIRS_SINK, _vp,
                                   ctypes.POINTER(JoinStats)]),
    "gsj_erode": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, ctypes.POINTER(JoinOpts), PAIRS_SINK,
                                 _vp, ctypes.POINTER(JoinStats)]),
    "gsj_points_dwithin": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.POINTER(JoinOpts), PAIRS_SINK, _vp, ctypes.POINTER(JoinStats)]),
    "gsj_points_erode": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.POINTER(JoinOpts), PAIRS_SINK, _vp, ctypes.POINTER(JoinStats)]),
    "gsj_candidates": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, PAIRS_SINK, _vp]),
    "gsj_refine_pairs": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_uint64, ctypes.POINTER(RefineParams), ctypes.c_int, _vp, _vp, _vp, _vp]),
    "gsj_refine_pairs_noalloc": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_uint64, ctypes.POINTER(RefineParams), _vp, _vp, _vp, _vp]),
    "gsj_get_refine_shape": (ctypes.c_int, [_vp, ctypes.POINTER(RefineShape)]),
    "gsj_set_refine_shape": (ctypes.c_int, [_vp, ctypes.POINTER(RefineShape)]),
    "gsj_tune_refine": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(RefineParams), ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                       ctypes.POINTER(TuneResult)]),
    "gsj_subdivide": (ctypes.c_int, [ctypes.c_uint64] * 3 + [_vp] * 3 + [ctypes.c_int] + [ctypes.POINTER(ctypes.c_uint64)] * 3 +
                      [ctypes.POINTER(_vp)] * 5),
    "gsj_dedup": (ctypes.c_int, [ctypes.c_uint64] * 3 + [_vp] * 3 + [ctypes.c_int] + [ctypes.POINTER(ctypes.c_uint64)] * 3 +
                  [ctypes.POINTER(_vp)] * 5),
    "gsj_host_free": (None, [_vp]),
    "gsj_rowset_upload": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp, _vp, ctypes.c_uint64, _vp, _vp, ctypes.POINTER(_vp)]),
    "gsj_rowset_free": (None, [_vp]),
    "gsj_encode_rows": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(EncodeSpec), _vp, _vp, _vp, _vp, ctypes.c_uint64, BYTES_SINK, _vp,
                                       ctypes.POINTER(ctypes.c_uint64)]),
    "gsj_de9im_str": (None, [ctypes.c_uint32, ctypes.c_char_p]),
    "gsj_de9im_transpose": (ctypes.c_uint32, [ctypes.c_uint32]),
    "gsj_de9im_match": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_char_p]),
}


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(lib_path("libgsj.so"))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def refine_params(want_area=True, want_relate=False, snap_half_ulp=False) -> RefineParams:
    p = RefineParams()
    lib().gsj_refine_params_default(ctypes.byref(p))
    p.want_area, p.want_relate, p.snap_half_ulp = int(want_area), int(want_relate), int(snap_half_ulp)
    return p


def join_opts(upper=False, no_agg=False, refine_mode=GSJ_REFINE_FILTERED, batch_q=0, shard=0, nshards=1) -> JoinOpts:
    o = JoinOpts()
    lib().gsj_join_opts_default(ctypes.byref(o))
    o.upper, o.no_agg, o.refine_mode, o.batch_q = int(upper), int(no_agg), int(refine_mode), int(batch_q)
    o.shard, o.nshards = int(shard), int(nshards)
    return o


def de9im_str(code: int) -> str:
    b = ctypes.create_string_buffer(10)
    lib().gsj_de9im_str(code, b)
    return b.raw[:9].decode()


def de9im_transpose(code: int) -> int:
    return lib().gsj_de9im_transpose(code)


def de9im_match(code: int, pattern: str) -> bool:
    return bool(lib().gsj_de9im_match(code, pattern.encode()))


_COPY_POOL = None


def _copy_out(ptr, count, dtype):
    """count elements from a host pointer the library owns only during a sink call, into a new numpy array. Large
    arrays are copied in 8 slices on a small thread pool (ctypes.memmove releases the GIL), so a sink's copy of a
    few hundred MB of rows is not one thread's memcpy."""
    global _COPY_POOL
    out = np.empty(count, dtype)
    nbytes = out.nbytes
    src = ctypes.cast(ptr, ctypes.c_void_p).value
    if nbytes < (8 << 20):
        if nbytes:
            ctypes.memmove(out.ctypes.data, src, nbytes)
        return out
    if _COPY_POOL is None:
        import concurrent.futures
        _COPY_POOL = concurrent.futures.ThreadPoolExecutor(max_workers=8, thread_name_prefix="gsj-copy")
    step = ((nbytes + 7) // 8 + 63) & ~63
    dst = out.ctypes.data
    futs = [_COPY_POOL.submit(ctypes.memmove, dst + o, src + o, min(step, nbytes - o)) for o in range(0, nbytes, step)]
    for f in futs:
        f.result()
    return out


def _join_chunks(chunks, dtype):
    """The batches' arrays as one (a single batch is returned as it is, without another copy)."""
    if not chunks:
        return np.zeros(0, dtype)
    return chunks[0] if len(chunks) == 1 else np.concatenate(chunks)


def _take(ptr, count, dtype):
    a = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dtype))), (max(count, 1),))[:count].copy()
    lib().gsj_host_free(ptr)
    return a


def subdivide(ps, maxv: int):
    """Pieces of at most ~maxv vertices (gsj_subdivide, on the current CUDA device): a PolygonSet with .parent and .syn set."""
    from .gen import PolygonSet
    gro = np.ascontiguousarray(ps.gro, np.uint64); rvo = np.ascontiguousarray(ps.rvo, np.uint64); xy = np.ascontiguousarray(ps.xy, np.float64)
    n, nr, nv = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    ptrs = [_vp() for _ in range(5)]
    rc = lib().gsj_subdivide(len(gro) - 1, len(rvo) - 1, len(xy), gro.ctypes.data, rvo.ctypes.data, xy.ctypes.data, int(maxv),
                             ctypes.byref(n), ctypes.byref(nr), ctypes.byref(nv), *[ctypes.byref(p) for p in ptrs])
    if rc:
        raise GsjError(rc, "gsj_subdivide failed")
    return PolygonSet(_take(ptrs[0], n.value + 1, np.uint64), _take(ptrs[1], nr.value + 1, np.uint64),
                      _take(ptrs[2], 2 * nv.value, np.float64).reshape(-1, 2), parent=_take(ptrs[3], n.value, np.uint32),
                      syn=_take(ptrs[4], nv.value, np.uint8))


def dedup(ps, morton=False):
    """(distinct PolygonSet, moff, midx) (gsj_dedup, on the current CUDA device)."""
    from .gen import PolygonSet
    gro = np.ascontiguousarray(ps.gro, np.uint64); rvo = np.ascontiguousarray(ps.rvo, np.uint64); xy = np.ascontiguousarray(ps.xy, np.float64)
    n, nr, nv = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    ptrs = [_vp() for _ in range(5)]
    rc = lib().gsj_dedup(len(gro) - 1, len(rvo) - 1, len(xy), gro.ctypes.data, rvo.ctypes.data, xy.ctypes.data, int(morton),
                         ctypes.byref(n), ctypes.byref(nr), ctypes.byref(nv), *[ctypes.byref(p) for p in ptrs])
    if rc:
        raise GsjError(rc, "gsj_dedup failed")
    u = PolygonSet(_take(ptrs[0], n.value + 1, np.uint64), _take(ptrs[1], nr.value + 1, np.uint64),
                   _take(ptrs[2], 2 * nv.value, np.float64).reshape(-1, 2))
    return u, _take(ptrs[3], n.value + 1, np.uint64), _take(ptrs[4], len(gro) - 1, np.uint32)


class _RowsetHandle:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            lib().gsj_rowset_free(self.h)
            self.h = None


@dataclasses.dataclass
class JoinResult:
    pairs: np.ndarray          # (n, 2) uint32: (P parent, R parent)
    area: np.ndarray | None    # (n,) float64
    code: np.ndarray | None    # (n,) uint32 DE-9IM codes
    stats: dict


class Layer:
    def __init__(self, eng: "Engine", handle, keep=()):
        self.eng, self.h = eng, handle
        self._keep = keep
        info = LayerInfo()
        lib().gsj_layer_get_info(handle, ctypes.byref(info))
        self.info = {k: getattr(info, k) for k, _ in LayerInfo._fields_}

    @property
    def n(self):
        return self.info["n"]

    def free(self):
        if self.h:
            lib().gsj_layer_free(self.eng.ctx, self.h)
            self.h = None

    def __del__(self):
        try:
            if self.h and self.eng.ctx:
                self.free()
        except Exception:
            pass


class Engine:
    """One gsj context on a CUDA device."""

    def __init__(self, device: int = 0):
        h = _vp()
        rc = lib().gsj_ctx_create(device, ctypes.byref(h))
        if rc:
            raise GsjError(rc, "cannot create a context (no CUDA device?)")
        self.ctx = h
        self.device = device

    def close(self):
        if self.ctx:
            lib().gsj_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise GsjError(rc, lib().gsj_last_error(self.ctx).decode(errors="replace"))

    def stream_handle(self) -> int:
        """cudaStream_t of the context (all its kernels run there), e.g. for torch.cuda.ExternalStream."""
        return lib().gsj_ctx_stream(self.ctx)

    def dedup(self, ps, morton=False):
        """(distinct PolygonSet, moff, midx) computed on this context's GPU (gsj_dedup_gpu): the same arrays as dedup()."""
        from .gen import PolygonSet
        gro = np.ascontiguousarray(ps.gro, np.uint64); rvo = np.ascontiguousarray(ps.rvo, np.uint64); xy = np.ascontiguousarray(ps.xy, np.float64)
        n, nr, nv = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        ptrs = [_vp() for _ in range(5)]
        self._check(lib().gsj_dedup_gpu(self.ctx, len(gro) - 1, len(rvo) - 1, len(xy), gro.ctypes.data, rvo.ctypes.data, xy.ctypes.data, int(morton),
                                        ctypes.byref(n), ctypes.byref(nr), ctypes.byref(nv), *[ctypes.byref(p) for p in ptrs]))
        u = PolygonSet(_take(ptrs[0], n.value + 1, np.uint64), _take(ptrs[1], nr.value + 1, np.uint64),
                       _take(ptrs[2], 2 * nv.value, np.float64).reshape(-1, 2))
        return u, _take(ptrs[3], n.value + 1, np.uint64), _take(ptrs[4], len(gro) - 1, np.uint32)

    def subdivide(self, ps, maxv: int):
        """Pieces of at most ~maxv vertices computed on this context's GPU (gsj_subdivide_gpu): the same arrays as subdivide()."""
        from .gen import PolygonSet
        gro = np.ascontiguousarray(ps.gro, np.uint64); rvo = np.ascontiguousarray(ps.rvo, np.uint64); xy = np.ascontiguousarray(ps.xy, np.float64)
        n, nr, nv = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        ptrs = [_vp() for _ in range(5)]
        self._check(lib().gsj_subdivide_gpu(self.ctx, len(gro) - 1, len(rvo) - 1, len(xy), gro.ctypes.data, rvo.ctypes.data, xy.ctypes.data, int(maxv),
                                            ctypes.byref(n), ctypes.byref(nr), ctypes.byref(nv), *[ctypes.byref(p) for p in ptrs]))
        return PolygonSet(_take(ptrs[0], n.value + 1, np.uint64), _take(ptrs[1], nr.value + 1, np.uint64),
                          _take(ptrs[2], 2 * nv.value, np.float64).reshape(-1, 2), parent=_take(ptrs[3], n.value, np.uint32),
                          syn=_take(ptrs[4], nv.value, np.uint8))

    def mem_info(self):
        f, t, s = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int()
        self._check(lib().gsj_ctx_mem_info(self.ctx, ctypes.byref(f), ctypes.byref(t), ctypes.byref(s)))
        return f.value, t.value, s.value

    # ---- layers ----
    def upload_polygons(self, ps, parent=None, syn=None) -> Layer:
        gro = np.ascontiguousarray(ps.gro, dtype=np.uint64)
        rvo = np.ascontiguousarray(ps.rvo, dtype=np.uint64)
        xy = np.ascontiguousarray(ps.xy, dtype=np.float64)
        parent = parent if parent is not None else getattr(ps, "parent", None)
        syn = syn if syn is not None else getattr(ps, "syn", None)
        par = None if parent is None else np.ascontiguousarray(parent, dtype=np.uint32)
        sy = None if syn is None else np.ascontiguousarray(syn, dtype=np.uint8)
        h = _vp()
        self._check(lib().gsj_layer_upload_polygons(self.ctx, len(gro) - 1, len(rvo) - 1, len(xy), gro.ctypes.data, rvo.ctypes.data,
                                                     xy.ctypes.data, None if par is None else par.ctypes.data,
                                                     None if sy is None else sy.ctypes.data, ctypes.byref(h)))
        return Layer(self, h)

    def upload_points(self, xy) -> Layer:
        xy = np.ascontiguousarray(xy, dtype=np.float64)
        h = _vp()
        self._check(lib().gsj_layer_upload_points(self.ctx, len(xy), xy.ctypes.data, ctypes.byref(h)))
        return Layer(self, h)

    # ---- joins ----
    def join(self, P: Layer, R: Layer, want_area=True, want_relate=False, upper=False, no_agg=False,
             refine_mode=GSJ_REFINE_FILTERED, batch_q=0, snap_half_ulp=False, shard=0, nshards=1, collect=True) -> JoinResult:
        """collect=False: the rows reach the library's pinned host buffers batch by batch as usual but are not copied
        into numpy arrays (pairs/area/code are None; stats['hits'] counts them)."""
        rp = refine_params(want_area, want_relate, snap_half_ulp)
        o = join_opts(upper, no_agg, refine_mode, batch_q, shard, nshards)
        chunks_p, chunks_a, chunks_c = [], [], []

        def sink(user, pairs, area, code, n):
            if not collect:
                return 0
            chunks_p.append(_copy_out(pairs, n * 2, np.uint32))
            if area:
                chunks_a.append(_copy_out(area, n, np.float64))
            if code:
                chunks_c.append(_copy_out(code, n, np.uint32))
            return 0

        cb = JOIN_SINK(sink)
        st = JoinStats()
        self._check(lib().gsj_join(self.ctx, P.h, R.h, ctypes.byref(rp), ctypes.byref(o), cb, None, ctypes.byref(st)))
        if not collect:
            return JoinResult(None, None, None, st.as_dict())
        pairs = _join_chunks(chunks_p, np.uint32).reshape(-1, 2)
        area = _join_chunks(chunks_a, np.float64) if want_area else None
        code = _join_chunks(chunks_c, np.uint32) if want_relate else None
        return JoinResult(pairs, area, code, st.as_dict())

    def join_points(self, pts: Layer, R: Layer, batch_q=0, shard=0, nshards=1, refine_mode=GSJ_REFINE_FILTERED):
        o = join_opts(batch_q=batch_q, shard=shard, nshards=nshards, refine_mode=refine_mode)
        cp, cw = [], []

        def sink(user, pairs, where, n):
            cp.append(np.ctypeslib.as_array(pairs, (n * 2,)).copy())
            cw.append(np.ctypeslib.as_array(where, (n,)).copy())
            return 0

        cb = POINTS_SINK(sink)
        st = JoinStats()
        self._check(lib().gsj_join_points(self.ctx, pts.h, R.h, ctypes.byref(o), cb, None, ctypes.byref(st)))
        pairs = np.concatenate(cp).reshape(-1, 2) if cp else np.zeros((0, 2), np.uint32)
        where = np.concatenate(cw) if cw else np.zeros(0, np.uint8)
        return pairs, where, st.as_dict()

    def cluster(self, P: Layer, nparent: int | None = None, refine_mode=GSJ_REFINE_FILTERED, shard=0, nshards=1):
        nparent = P.info["nparent"] if nparent is None else nparent
        root = np.empty(nparent, np.uint32)
        st = JoinStats()
        o = join_opts(refine_mode=refine_mode, shard=shard, nshards=nshards)
        self._check(lib().gsj_cluster(self.ctx, P.h, nparent, ctypes.byref(o), root.ctypes.data, ctypes.byref(st)))
        return root, st.as_dict()

    def cluster_merge(self, roots) -> np.ndarray:
        """Roots of the union of the given forests (probe-shard clusters of one layer): gsj_cluster_merge."""
        r = np.ascontiguousarray(np.stack([np.asarray(x, np.uint32) for x in roots]), np.uint32)
        out = np.empty(r.shape[1], np.uint32)
        self._check(lib().gsj_cluster_merge(self.ctx, r.shape[1], r.shape[0], r.ctypes.data, out.ctypes.data))
        return out

    def _pairs_call(self, fn, *args, opts=None):
        chunks = []

        def sink(user, pairs, n):
            chunks.append(np.ctypeslib.as_array(pairs, (n * 2,)).copy())
            return 0

        cb = PAIRS_SINK(sink)
        st = JoinStats()
        o = opts if opts is not None else join_opts()
        self._check(fn(self.ctx, *args, ctypes.byref(o), cb, None, ctypes.byref(st)))
        pairs = np.concatenate(chunks).reshape(-1, 2) if chunks else np.zeros((0, 2), np.uint32)
        return pairs, st.as_dict()

    def dwithin(self, P: Layer, R: Layer, d: float, same=False, upper=None, refine_mode=GSJ_REFINE_FILTERED):
        o = join_opts(upper=same if upper is None else upper, refine_mode=refine_mode)
        return self._pairs_call(lib().gsj_dwithin, P.h, R.h, float(d), int(same), opts=o)

    def erode(self, P: Layer, R: Layer, ra: float, rb: float, same=False, need_self=None, refine_mode=GSJ_REFINE_FILTERED):
        ns = None if need_self is None else np.ascontiguousarray(need_self, dtype=np.uint8)
        o = join_opts(upper=same, refine_mode=refine_mode)
        return self._pairs_call(lib().gsj_erode, P.h, R.h, float(ra), float(rb), int(same), None if ns is None else ns.ctypes.data, opts=o)

    def points_dwithin(self, pts: Layer, R: Layer, d: float, refine_mode=GSJ_REFINE_FILTERED):
        return self._pairs_call(lib().gsj_points_dwithin, pts.h, R.h, float(d), opts=join_opts(refine_mode=refine_mode))

    def points_erode(self, pts: Layer, R: Layer, r: float, refine_mode=GSJ_REFINE_FILTERED):
        return self._pairs_call(lib().gsj_points_erode, pts.h, R.h, float(r), opts=join_opts(refine_mode=refine_mode))

    # ---- row encoding on the device (the daemon's result frames) ----
    def rowset(self, ids, moff=None, midx=None):
        """Device row ids (list of bytes) and optional dedup members (moff[n_geoms + 1], midx) for encode_rows."""
        blob = b"".join(ids)
        off = np.zeros(len(ids) + 1, np.uint64)
        off[1:] = np.cumsum([len(x) for x in ids])
        mo = None if moff is None else np.ascontiguousarray(moff, np.uint64)
        mi = None if midx is None else np.ascontiguousarray(midx, np.uint32)
        n_geoms = len(ids) if mo is None else len(mo) - 1
        h = _vp()
        bb = ctypes.create_string_buffer(blob, max(1, len(blob)))
        self._check(lib().gsj_rowset_upload(self.ctx, n_geoms, None if mo is None else mo.ctypes.data, None if mi is None else mi.ctypes.data,
                                            len(ids), bb, off.ctypes.data, ctypes.byref(h)))
        return _RowsetHandle(h)

    def encode_rows(self, P, Q, mode, pairs, area=None, code=None, where=None, same=False, distinct=False, swapped=False, point_value=0.0,
                    pattern=""):
        """(stream bytes, rows) of gsj_encode_rows."""
        pairs = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
        a = None if area is None else np.ascontiguousarray(area, np.float64)
        c = None if code is None else np.ascontiguousarray(code, np.uint32)
        w = None if where is None else np.ascontiguousarray(where, np.uint8)
        sp = EncodeSpec(mode, int(same), int(distinct), int(swapped), float(point_value), pattern.encode())
        chunks = []

        def sink(user, b, nb, nr):
            chunks.append(ctypes.string_at(b, nb))
            return 0

        cb = BYTES_SINK(sink)
        rows = ctypes.c_uint64()
        self._check(lib().gsj_encode_rows(self.ctx, P.h, Q.h, ctypes.byref(sp), pairs.ctypes.data, None if a is None else a.ctypes.data,
                                          None if c is None else c.ctypes.data, None if w is None else w.ctypes.data, len(pairs), cb, None,
                                          ctypes.byref(rows)))
        return b"".join(chunks), rows.value

    # ---- parity / diagnostics ----
    def candidates(self, P: Layer, R: Layer, upper=False) -> np.ndarray:
        chunks = []

        def sink(user, pairs, n):
            chunks.append(np.ctypeslib.as_array(pairs, (n * 2,)).copy())
            return 0

        cb = PAIRS_SINK(sink)
        self._check(lib().gsj_candidates(self.ctx, P.h, R.h, int(upper), cb, None))
        return np.concatenate(chunks).reshape(-1, 2) if chunks else np.zeros((0, 2), np.uint32)

    @property
    def refine_shape(self) -> dict:
        """The context's refinement launch shape (gsj_get_refine_shape): run, runs, bin_edges, scratch_warps_per_sm."""
        sh = RefineShape()
        self._check(lib().gsj_get_refine_shape(self.ctx, ctypes.byref(sh)))
        return sh.as_dict()

    @refine_shape.setter
    def refine_shape(self, shape: dict):
        sh = RefineShape(**{**self.refine_shape, **shape})
        self._check(lib().gsj_set_refine_shape(self.ctx, ctypes.byref(sh)))

    def tune_refine(self, P: Layer, R: Layer, want_area=True, want_relate=False, refine_mode=GSJ_REFINE_FILTERED, upper=None, max_pairs=0,
                    keep=()) -> dict:
        """Runs the refinement autotuner (gsj_tune_refine) on P x R's candidate pairs and sets the chosen shape on this
        context; keep names shape fields left as they are. Returns {'best': shape, 'start_ms', 'best_ms', 'sample_pairs',
        'shapes_tried'}."""
        rp = refine_params(want_area, want_relate)
        r = TuneResult()
        up = (P is R) if upper is None else bool(upper)
        bits = {"run": 1, "runs": 2, "bin_edges": 4, "scratch_warps_per_sm": 8}
        mask = sum(bits[k] for k in keep)
        self._check(lib().gsj_tune_refine(self.ctx, P.h, R.h, ctypes.byref(rp), refine_mode, int(up), int(max_pairs), mask, ctypes.byref(r)))
        return {"best": r.best.as_dict(), "start_ms": r.start_ms, "best_ms": r.best_ms, "sample_pairs": r.sample_pairs, "shapes_tried": r.shapes_tried}

    def refine_pairs(self, P: Layer, R: Layer, pairs, want_area=True, want_relate=False, refine_mode=GSJ_REFINE_FILTERED, snap_half_ulp=False):
        pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
        n = len(pairs)
        flag = np.zeros(n, np.uint8); area = np.zeros(n); ev = np.zeros((n, 4)); evb = np.zeros(n, np.uint32)
        rp = refine_params(want_area, want_relate, snap_half_ulp)
        self._check(lib().gsj_refine_pairs(self.ctx, P.h, R.h, pairs.ctypes.data, n, ctypes.byref(rp), refine_mode, flag.ctypes.data,
                                           area.ctypes.data, ev.ctypes.data, evb.ctypes.data))
        return flag, area, ev, evb
