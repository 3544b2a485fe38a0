"""Client of the gpujoind wire protocol (include/gsp_protocol.h), for gsjd or the reference's gpujoind.

The calls mirror the gpu_spatial extension's SQL functions (ext/gpu_spatial.c): gpu_load / gpu_drop / gpu_status /
gpu_layers, gpu_join (+ stats), gpu_relate, gpu_cluster_intersecting, gpu_dwithin and gpu_intersects_buffered.
"""
from __future__ import annotations

import json
import math
import socket
import struct

GSP_MAGIC = 0x52505347
GSP_OK, GSP_ERR, GSP_FRAME_ERR = 0, 1, 0xFFFFFFFF
OP_LOAD, OP_LOAD_QUERY, OP_DROP, OP_LIST, OP_STATUS, OP_JOIN, OP_CLUSTER, OP_RELATE, OP_DWITHIN = range(1, 10)


class GspError(RuntimeError):
    """The daemon answered with an error (before or during a result stream)."""


class _Reader:
    def __init__(self, s: socket.socket):
        self.s, self.buf, self.pos = s, b"", 0

    def read(self, n: int) -> bytes:
        while len(self.buf) - self.pos < n:
            chunk = self.s.recv(1 << 20)
            if not chunk:
                raise ConnectionError("connection closed by the daemon")
            self.buf = self.buf[self.pos:] + chunk
            self.pos = 0
        out = self.buf[self.pos:self.pos + n]
        self.pos += n
        return out

    def u32(self) -> int:
        return struct.unpack("<I", self.read(4))[0]

    def text(self) -> str:
        return self.read(self.u32()).decode("utf-8", "replace")


def encode_request(op: int, args, token: str = "") -> bytes:
    parts = [struct.pack("<III", GSP_MAGIC, op, len(args) + 1)]
    for a in [token, *args]:
        b = a.encode() if isinstance(a, str) else bytes(a)
        parts.append(struct.pack("<I", len(b)) + b)
    return b"".join(parts)


class Client:
    def __init__(self, unix_path: str | None = "/tmp/gpujoind.sock", tcp: tuple[str, int] | None = None, token: str = "",
                 timeout: float | None = 600.0):
        self.unix_path, self.tcp, self.token, self.timeout = unix_path, tcp, token, timeout

    def connect(self) -> socket.socket:
        if self.tcp:
            s = socket.create_connection(self.tcp, timeout=self.timeout)
        else:
            s = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
            s.settimeout(self.timeout)
            s.connect(self.unix_path)
        return s

    def _open(self, op: int, args):
        s = self.connect()
        s.sendall(encode_request(op, args, self.token))
        r = _Reader(s)
        st = r.u32()
        if st != GSP_OK:
            msg = r.text()
            s.close()
            raise GspError(msg)
        return s, r

    def json_call(self, op: int, args=()):
        s, r = self._open(op, list(args))
        try:
            return json.loads(r.text())
        finally:
            s.close()

    def stream_call(self, op: int, args, row):
        """Rows parsed by row(reader) until the end of the stream; returns (rows, stats dict)."""
        s, r = self._open(op, list(args))
        try:
            rows = []
            while True:
                n = r.u32()
                if n == GSP_FRAME_ERR:
                    raise GspError(r.text())
                if n == 0:
                    return rows, json.loads(r.text())
                for _ in range(n):
                    rows.append(row(r))
        finally:
            s.close()

    # ---- layers (gpu_load, gpu_drop, gpu_status, gpu_layers) ----
    def load(self, layer: str, path: str, subdivide: int = 0, dedup: bool = True, id_col: str = "id", geom_col: str = "geom",
             filter: str = ""):
        return self.json_call(OP_LOAD, [layer, path, id_col, geom_col, filter, str(subdivide), "1" if dedup else "0"])

    def load_query(self, layer: str, sql: str, subdivide: int = 0, dedup: bool = True):
        return self.json_call(OP_LOAD_QUERY, [layer, sql, str(subdivide), "1" if dedup else "0"])

    def drop(self, layer: str) -> bool:
        return self.json_call(OP_DROP, [layer])

    def list(self):
        return self.json_call(OP_LIST)

    def status(self):
        return self.json_call(OP_STATUS)

    # ---- joins ----
    @staticmethod
    def _id(r: _Reader) -> str:
        return r.read(struct.unpack("<H", r.read(2))[0]).decode("utf-8", "replace")

    def _pair_row(self, r: _Reader):
        a, b = self._id(r), self._id(r)
        return a, b, struct.unpack("<d", r.read(8))[0]

    def join(self, a: str, b: str, want_area: bool = True, self_pairs: str = "all", stats_only: bool = False):
        args = [a, b, "1" if want_area else "0", self_pairs] + (["stats"] if stats_only else [])
        return self.stream_call(OP_JOIN, args, self._pair_row)

    def relate(self, a: str, b: str, pattern: str = "", self_pairs: str = "all"):
        return self.stream_call(OP_RELATE, [a, b, pattern, self_pairs], lambda r: (self._id(r), self._id(r), r.read(9).decode()))

    def cluster(self, layer: str):
        return self.stream_call(OP_CLUSTER, [layer], lambda r: (self._id(r), struct.unpack("<I", r.read(4))[0]))

    def dwithin(self, a: str, b: str, dist: float, self_pairs: str = "all", stats_only: bool = False):
        args = [a, b, "dwithin", repr(float(dist)), "0", self_pairs] + (["stats"] if stats_only else [])
        return self.stream_call(OP_DWITHIN, args, self._pair_row)

    def intersects_buffered(self, a: str, b: str, buf_a: float, buf_b: float, self_pairs: str = "all", stats_only: bool = False):
        args = [a, b, "buffer", repr(float(buf_a)), repr(float(buf_b)), self_pairs] + (["stats"] if stats_only else [])
        return self.stream_call(OP_DWITHIN, args, self._pair_row)


def is_nan(x: float) -> bool:
    return isinstance(x, float) and math.isnan(x)
