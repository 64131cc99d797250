"""Continuous-batching retrieval server over the C ABI (rbw_server_*): query images in (host
descriptors), top-k database documents out, lookup and scoring batched on the GPU."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import Vocabulary, _check, load_library


class ServerOptions(C.Structure):
    _fields_ = [("max_batch_queries", C.c_uint32), ("max_inflight_batches", C.c_uint32),
                ("max_batch_descriptors", C.c_uint64), ("hbm_budget_bytes", C.c_uint64),
                ("max_results", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("max_inflight_seen", C.c_uint32), ("mean_batch_requests", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("queue_p99_ms", C.c_double), ("launch_p99_ms", C.c_double), ("device_p99_ms", C.c_double),
                ("queue_max_ms", C.c_double), ("launch_max_ms", C.c_double), ("device_max_ms", C.c_double)]


class Server:
    """Answers query images with their top-k documents.  Requests submitted while batches are on
    the GPU join the next batch; batches are admitted while their device-memory estimate fits
    the budget.  The vocabulary and database must outlive the server."""

    def __init__(self, voc: Vocabulary, db, max_results: int = 100, max_batch_queries: int = 256,
                 max_inflight_batches: int = 3, max_batch_descriptors: int = 1 << 21,
                 hbm_budget_bytes: int = 0) -> None:
        self._lib = load_library()
        o = ServerOptions()
        self._lib.rbw_server_options_default(C.byref(o))
        o.max_results = max_results
        o.max_batch_queries = max_batch_queries
        o.max_inflight_batches = max_inflight_batches
        o.max_batch_descriptors = max_batch_descriptors
        o.hbm_budget_bytes = hbm_budget_bytes
        self.voc, self.db, self.k = voc, db, max_results
        h = C.c_void_p()
        _check(self._lib.rbw_server_create(voc.handle, db._h, C.byref(o), C.byref(h)))
        self._h = h

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.rbw_server_destroy(h)
            self._h = None

    def __del__(self) -> None:
        self.close()

    def submit(self, desc: np.ndarray) -> int:
        """desc: host uint8 [n, 128].  Returns the request id at once."""
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        rid = C.c_uint64()
        n = desc.shape[0] if desc.ndim == 2 else 0
        _check(self._lib.rbw_server_submit(self._h, desc.ctypes.data, n, C.byref(rid)))
        return rid.value

    def wait(self, rid: int, timeout_s: Optional[float] = None) -> Tuple[np.ndarray, np.ndarray, float]:
        """(documents, scores, latency in ms) of a request; raises RbwError(RBW_ERR_TIMEOUT)
        when it is not done within timeout_s (the request can be waited for again)."""
        docs = np.empty(self.k, np.uint32)
        scores = np.empty(self.k, np.float32)
        n = C.c_uint32()
        lat = C.c_double()
        t = -1 if timeout_s is None else int(timeout_s * 1e6)
        _check(self._lib.rbw_server_wait(self._h, rid, t, docs.ctypes.data, scores.ctypes.data, self.k, C.byref(n),
                                         C.byref(lat)))
        return docs[: n.value].copy(), scores[: n.value].copy(), lat.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(self._lib.rbw_server_get_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def batch_bytes(self, n_desc: int, n_requests: int) -> int:
        """Device bytes the server reserves for a batch (what hbm_budget_bytes is counted in)."""
        b = C.c_uint64()
        _check(self._lib.rbw_server_batch_bytes(self._h, n_desc, n_requests, C.byref(b)))
        return b.value

    def reset_stats(self) -> None:
        _check(self._lib.rbw_server_reset_stats(self._h))
