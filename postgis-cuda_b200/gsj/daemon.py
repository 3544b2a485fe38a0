"""The serving daemon's host rules through its C ABI (include/gsjd.h), and a helper to run gsjd."""
from __future__ import annotations

import ctypes
import os
import subprocess
import time

import numpy as np

from ._build import BUILD_DIR, lib_path

_lib = None
_vp = ctypes.c_void_p


class FileInfo(ctypes.Structure):
    _fields_ = [("is_points", ctypes.c_int), ("rows", ctypes.c_uint64), ("skipped_null", ctypes.c_uint64),
                ("skipped_type", ctypes.c_uint64), ("skipped_empty", ctypes.c_uint64), ("n", ctypes.c_uint64),
                ("nr", ctypes.c_uint64), ("nv", ctypes.c_uint64)]


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(lib_path("libgsjd.so"))   # builds the package (libgsj.so, libgsjd.so, gsjd) when missing
        u64p, u32p, u8p = ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint8)
        L.gsjd_expand_rows.restype = ctypes.c_int
        L.gsjd_expand_rows.argtypes = [ctypes.c_uint64, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, u64p,
                                       ctypes.POINTER(u32p), ctypes.POINTER(u64p), ctypes.POINTER(u8p)]
        L.gsjd_count_rows.restype = ctypes.c_uint64
        L.gsjd_count_rows.argtypes = [ctypes.c_uint64, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]
        L.gsjd_cluster_labels.restype = ctypes.c_uint32
        L.gsjd_cluster_labels.argtypes = [ctypes.c_uint32, _vp, ctypes.c_uint64, _vp, _vp, _vp]
        L.gsjd_file_open.restype = ctypes.c_int
        L.gsjd_file_open.argtypes = [ctypes.c_char_p, ctypes.POINTER(_vp), ctypes.c_char_p, ctypes.c_size_t]
        L.gsjd_file_get_info.restype = None
        L.gsjd_file_get_info.argtypes = [_vp, ctypes.POINTER(FileInfo)]
        L.gsjd_file_arrays.restype = None
        L.gsjd_file_arrays.argtypes = [_vp, ctypes.POINTER(u64p), ctypes.POINTER(u64p), ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        L.gsjd_file_id.restype = ctypes.c_void_p
        L.gsjd_file_id.argtypes = [_vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_size_t)]
        L.gsjd_file_close.restype = None
        L.gsjd_file_close.argtypes = [_vp]
        L.gsjd_free.restype = None
        L.gsjd_free.argtypes = [_vp]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def expand_rows(pairs, same, distinct, moff_a=None, midx_a=None, moff_b=None, midx_b=None):
    """(rows[k, 2], src[k], transposed[k]) of the daemon's row rules for engine pairs[n, 2]."""
    pairs = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
    conv = [None if a is None else np.ascontiguousarray(a, t) for a, t in
            ((moff_a, np.uint64), (midx_a, np.uint32), (moff_b, np.uint64), (midx_b, np.uint32))]
    n = ctypes.c_uint64()
    rows, src, tr = ctypes.POINTER(ctypes.c_uint32)(), ctypes.POINTER(ctypes.c_uint64)(), ctypes.POINTER(ctypes.c_uint8)()
    if lib().gsjd_expand_rows(len(pairs), _ptr(pairs), int(same), int(distinct), *map(_ptr, conv), ctypes.byref(n),
                              ctypes.byref(rows), ctypes.byref(src), ctypes.byref(tr)):
        raise ValueError("gsjd_expand_rows: bad arguments")
    k = n.value
    try:
        r = np.ctypeslib.as_array(rows, (2 * k,)).reshape(-1, 2).copy() if k else np.zeros((0, 2), np.uint32)
        s = np.ctypeslib.as_array(src, (k,)).copy() if k else np.zeros(0, np.uint64)
        t = np.ctypeslib.as_array(tr, (k,)).copy() if k else np.zeros(0, np.uint8)
    finally:
        for p in (rows, src, tr):
            lib().gsjd_free(ctypes.cast(p, _vp))
    return r, s, t


def count_rows(pairs, same, distinct, moff_a=None, moff_b=None):
    pairs = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
    ma = None if moff_a is None else np.ascontiguousarray(moff_a, np.uint64)
    mb = None if moff_b is None else np.ascontiguousarray(moff_b, np.uint64)
    return int(lib().gsjd_count_rows(len(pairs), _ptr(pairs), int(same), int(distinct), _ptr(ma), _ptr(mb)))


def cluster_labels(root, rows, moff=None, midx=None):
    root = np.ascontiguousarray(root, np.uint32)
    mo = None if moff is None else np.ascontiguousarray(moff, np.uint64)
    mi = None if midx is None else np.ascontiguousarray(midx, np.uint32)
    out = np.zeros(rows, np.uint32)
    k = lib().gsjd_cluster_labels(len(root), _ptr(root), rows, _ptr(mo), _ptr(mi), out.ctypes.data)
    return out, int(k)


class LayerFile:
    """A layer file as the daemon's LOAD reads it (binary COPY of (id, EWKB), .gset, .pset)."""

    def __init__(self, path: str):
        self.h = None
        h, err = _vp(), ctypes.create_string_buffer(512)
        if lib().gsjd_file_open(os.fsencode(path), ctypes.byref(h), err, 512):
            raise OSError(err.value.decode())
        self.h = h
        info = FileInfo()
        lib().gsjd_file_get_info(h, ctypes.byref(info))
        self.info = {k: getattr(info, k) for k, _ in FileInfo._fields_}
        g, r, x = ctypes.POINTER(ctypes.c_uint64)(), ctypes.POINTER(ctypes.c_uint64)(), ctypes.POINTER(ctypes.c_double)()
        lib().gsjd_file_arrays(h, ctypes.byref(g), ctypes.byref(r), ctypes.byref(x))
        n, nr, nv = info.n, info.nr, info.nv
        self.xy = np.ctypeslib.as_array(x, (2 * nv,)).reshape(-1, 2).copy() if nv else np.zeros((0, 2))
        self.gro = None if info.is_points else np.ctypeslib.as_array(g, (n + 1,)).copy()
        self.rvo = None if info.is_points else np.ctypeslib.as_array(r, (nr + 1,)).copy()
        self.ids = []
        for i in range(n):
            ln = ctypes.c_size_t()
            p = lib().gsjd_file_id(h, i, ctypes.byref(ln))
            self.ids.append(ctypes.string_at(p, ln.value).decode() if ln.value else "")

    def close(self):
        if self.h:
            lib().gsjd_file_close(self.h)
            self.h = None

    def __del__(self):
        self.close()


def start(socket_path: str, data_dir: str, token_file: str | None = None, workers: int = 2, threads: int = 8, log=None,
          extra=()) -> subprocess.Popen:
    """Start gsjd and wait until its socket accepts connections."""
    cmd = [lib_path("gsjd"), "--socket", socket_path, "--data-dir", data_dir, "--workers", str(workers),
           "--threads", str(threads), *extra]
    if token_file:
        cmd += ["--token-file", token_file]
    p = subprocess.Popen(cmd, stdout=log or subprocess.DEVNULL, stderr=log or subprocess.DEVNULL)
    import socket as _s
    for _ in range(200):
        if p.poll() is not None:
            raise RuntimeError(f"gsjd exited with {p.returncode}")
        try:
            s = _s.socket(_s.AF_UNIX, _s.SOCK_STREAM)
            s.connect(socket_path)
            s.close()
            return p
        except OSError:
            time.sleep(0.05)
    p.kill()
    raise RuntimeError("gsjd did not start listening")


def stop(p: subprocess.Popen):
    if p.poll() is None:
        p.terminate()
        try:
            p.wait(10)
        except subprocess.TimeoutExpired:
            p.kill()
            p.wait()
