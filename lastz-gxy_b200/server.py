"""Serving loop over resident position tables (gxy_server_* in include/gxy_seed.h)."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, lib


class Server:
    """Keeps tables resident, admits queries by free device memory and runs them in overlapping batches."""

    def __init__(self, tables: Sequence, matrix, params, max_device_bytes: int = 8 << 30, max_units: int = 4096,
                 max_streams: int = 2, max_batch_units: int = 256, both_strands: bool = True,
                 max_batch_bases: int = 16 << 20, big_bases: int = 1 << 20, max_big_inflight: int = 1,
                 warm_bases: int = 0):
        from . import _params_c
        self.ctx = tables[0].ctx
        self._tables = list(tables)
        th = (C.c_void_p * len(tables))(*[t.h for t in tables])
        p = _params_c(matrix, params)
        o = _lib.ServerOptsC(max_device_bytes, max_units, max_streams, max_batch_units, 1 if both_strands else 0,
                              max_batch_bases, big_bases, max_big_inflight, 0, warm_bases)
        h = C.c_void_p()
        check(lib().gxy_server_create(self.ctx.h, len(tables), th, C.byref(p), C.byref(o), C.byref(h)))
        self.h = h

    def submit(self, table: int, query) -> int:
        s = query.c_struct()
        rid = C.c_uint64()
        check(lib().gxy_server_submit(self.h, table, C.byref(s), C.byref(rid)))
        return rid.value

    def wait(self, request_id: int, timeout_ms: int = 600000):
        """Returns (plus_hsps, minus_hsps, latency_ms) or raises on timeout."""
        from . import _take_buf
        plus, minus = _lib.HspBufC(), _lib.HspBufC()
        lat = C.c_double()
        check(lib().gxy_server_wait(self.h, request_id, timeout_ms, C.byref(plus), C.byref(minus), C.byref(lat)))
        return _take_buf(plus), _take_buf(minus), lat.value

    def wait_status(self, request_id: int, timeout_ms: int = 600000):
        """Like wait(), but returns (status, plus, minus, latency_ms) instead of
        raising when the request completed with an error status."""
        from . import _take_buf
        plus, minus = _lib.HspBufC(), _lib.HspBufC()
        lat = C.c_double()
        st = lib().gxy_server_wait(self.h, request_id, timeout_ms, C.byref(plus), C.byref(minus), C.byref(lat))
        if st != _lib.GXY_OK:
            return st, None, None, lat.value
        return st, _take_buf(plus), _take_buf(minus), lat.value

    def cancel(self, request_id: int) -> None:
        check(lib().gxy_server_cancel(self.h, request_id))

    def inject_fault(self, request_id: int, status: int) -> None:
        """Test hook: batches holding this request fail with `status` before any device work."""
        check(lib().gxy_server_inject_fault(self.h, request_id, status))

    def stats(self) -> dict:
        s = _lib.ServerStatsC()
        check(lib().gxy_server_get_stats(self.h, C.byref(s)))
        return {"submitted": s.submitted, "completed": s.completed, "batches": s.batches,
                "max_inflight_units": s.max_inflight_units, "bytes_in_use": s.bytes_in_use, "reruns": s.reruns,
                "busy_ms": s.busy_ms, "failed": s.failed, "canceled": s.canceled, "isolated": s.isolated,
                "mem_refreshes": s.mem_refreshes}

    def close(self) -> None:
        if self.h:
            check(lib().gxy_server_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
