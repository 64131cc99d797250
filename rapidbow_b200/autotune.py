"""Autotuner for the library's launch parameters, with a per-device cache file.

The reference sizes its assign grid from an occupancy query (kmeans.cu:307-322); here the
candidates of each tunable parameter are timed on the caller's own workload (CUDA events around
the library's kernels, rbw_timing_*) and the fastest is kept, per (parameter, branch factor,
tree levels, descriptor-count bucket = floor(log2(n))):

    assign_ctas_per_sm      uint8 k-means assign, CTAs per SM: 2..8         (default 6)
    assign_f32_ctas_per_sm  float-center assign, CTAs per SM: 1..3          (default 3)
    scatter_rows            lookup regroup scatter of more than 1,024 bins, rows per thread:
                            8|16|32 (default 16)
    lookup_schedule         tensor-core lookup schedule of algo "auto": 1 level pairs in two
                            accumulator buffers, 2 the three-slot ring (default 1)
    assign_sums             uint8 k-means center sums: 1 shared atomics, 2 a second MMA per
                            tile (default 1; with 2 at most 4 CTAs per SM)
    db_shard_tables         DataBase inverted file: 1 one CSR per 2,560-document shard while
                            small, 2 one CSR (default 1; its bucket counts documents)

Cache file (JSON): {"format": "rapidbow_b200 tuning cache", "version": 1,
"device": {"name": ..., "sms": ...}, "entries": [{"param", "B", "L", "bucket", "value",
"ms", "default_ms", "candidates": {value: ms}}]}.  Its path is $RBW_TUNING_CACHE, else
~/.cache/rapidbow_b200/tuning-<device>.json.  `Autotuner.apply()` hands every entry of the
file to the library (rbw_tuning_set), so later builds and lookups of matching shapes use it.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import re
from typing import Callable, Dict, Iterable, List, Optional

import numpy as np

from . import _check, load_library

PARAMS = {"assign_ctas_per_sm": 0, "assign_f32_ctas_per_sm": 1, "scatter_rows": 2, "db_shard_tables": 3,
          "lookup_schedule": 4, "assign_sums": 5}
DEFAULTS = {"assign_ctas_per_sm": 6, "assign_f32_ctas_per_sm": 3, "scatter_rows": 16, "db_shard_tables": 1,
            "lookup_schedule": 1, "assign_sums": 1}
CANDIDATES = {"assign_ctas_per_sm": (2, 3, 4, 5, 6, 7, 8), "assign_f32_ctas_per_sm": (1, 2, 3), "scatter_rows": (8, 16, 32),
              "db_shard_tables": (1, 2), "lookup_schedule": (1, 2), "assign_sums": (1, 2)}
FORMAT = "rapidbow_b200 tuning cache"
VERSION = 1


def bucket(n: int) -> int:
    """floor(log2(max(n, 1))): the descriptor-count bucket of a workload."""
    return max(int(n), 1).bit_length() - 1


def set_value(param: str, B: int, L: int, bkt: int, value: int) -> None:
    """Stores one value in the library (0 removes the entry)."""
    _check(load_library().rbw_tuning_set(PARAMS[param], B, L, bkt, value))


def get_value(param: str, B: int, L: int, n: int) -> int:
    """The value a launch of n descriptors would use."""
    v = C.c_uint32()
    _check(load_library().rbw_tuning_get(PARAMS[param], B, L, n, C.byref(v)))
    return v.value


def clear() -> None:
    _check(load_library().rbw_tuning_clear())


def choose(timings: Dict[int, float]) -> int:
    """The fastest candidate; ties go to the smaller value."""
    return min(sorted(timings), key=lambda v: timings[v])


def _slug(name: str) -> str:
    return re.sub(r"[^A-Za-z0-9]+", "-", name).strip("-").lower() or "device"


def default_cache_path(device_name: str) -> str:
    env = os.environ.get("RBW_TUNING_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "rapidbow_b200", f"tuning-{_slug(device_name)}.json")


class Autotuner:
    """Times candidates, keeps the best per key, and saves/loads/applies the cache file."""

    def __init__(self, device_name: str, sms: int, path: Optional[str] = None) -> None:
        self.device = {"name": device_name, "sms": int(sms)}
        self.path = path or default_cache_path(device_name)
        self.entries: List[dict] = []

    @classmethod
    def for_current_device(cls, path: Optional[str] = None) -> "Autotuner":
        import torch

        p = torch.cuda.get_device_properties(torch.cuda.current_device())
        return cls(p.name, p.multi_processor_count, path)

    # ---------------------------------------------------------------- cache
    def load(self) -> bool:
        """Reads the cache file if it exists and was written for this device."""
        if not os.path.exists(self.path):
            return False
        with open(self.path) as fh:
            d = json.load(fh)
        if d.get("format") != FORMAT or d.get("version") != VERSION or d.get("device") != self.device:
            return False
        self.entries = [e for e in d.get("entries", []) if e.get("param") in PARAMS]
        return True

    def save(self) -> str:
        os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump({"format": FORMAT, "version": VERSION, "device": self.device, "entries": self.entries}, fh,
                      indent=1, sort_keys=True)
        os.replace(tmp, self.path)
        return self.path

    def apply(self) -> int:
        """Hands every cached entry to the library; returns how many."""
        for e in self.entries:
            set_value(e["param"], e["B"], e["L"], e["bucket"], e["value"])
        return len(self.entries)

    def lookup(self, param: str, B: int, L: int, n: int) -> Optional[dict]:
        b = bucket(n)
        for e in self.entries:
            if e["param"] == param and e["B"] == B and e["L"] == L and e["bucket"] == b:
                return e
        return None

    def record(self, param: str, B: int, L: int, n: int, timings: Dict[int, float]) -> dict:
        """Keeps the fastest of `timings` (value -> ms) for the key and sets it in the library."""
        best = choose(timings)
        e = {"param": param, "B": int(B), "L": int(L), "bucket": bucket(n), "value": int(best),
             "ms": float(timings[best]), "default_ms": float(timings.get(DEFAULTS[param], float("nan"))),
             "candidates": {str(k): float(v) for k, v in sorted(timings.items())}}
        self.entries = [x for x in self.entries
                        if not (x["param"] == param and x["B"] == e["B"] and x["L"] == e["L"]
                                and x["bucket"] == e["bucket"])]
        self.entries.append(e)
        set_value(param, B, L, e["bucket"], best)
        return e

    # ---------------------------------------------------------------- tuning
    def tune(self, param: str, B: int, L: int, n: int, measure: Callable[[], float],
             candidates: Optional[Iterable[int]] = None) -> dict:
        """Sets each candidate, calls measure() (ms of the kernel being tuned) and records the best."""
        timings = {}
        b = bucket(n)
        for v in (candidates or CANDIDATES[param]):
            set_value(param, B, L, b, v)
            timings[int(v)] = float(measure())
        return self.record(param, B, L, n, timings)

    def tune_build(self, desc, B: int, L: int, float_centers: bool = False, repeats: int = 2, **build_kw) -> dict:
        """Tunes the assign kernel on a build of `desc` (CUDA uint8 [n, 128]); the build itself is
        the workload, timed by the library's assign-kernel events.  uint8 centers: the center sums
        (shared atomics or the tensor core) first, then the CTAs per SM for the chosen sums;
        returns the second entry, with the first under "sums"."""
        from . import build_vocabulary, timing_enable, timing_read, timing_reset

        n = desc.shape[0]

        def measure() -> float:
            build_vocabulary(desc, B, nb_levels=L, float_centers=float_centers, **build_kw)  # warm-up
            timing_reset()
            timing_enable(True)
            for _ in range(repeats):
                build_vocabulary(desc, B, nb_levels=L, float_centers=float_centers, **build_kw)
            timing_enable(False)
            return timing_read("kmeans_assign")[0] / repeats

        if float_centers:
            return self.tune("assign_f32_ctas_per_sm", B, 0, n, measure)
        sums = self.tune("assign_sums", B, 0, n, measure)
        e = self.tune("assign_ctas_per_sm", B, 0, n, measure,
                      candidates=[v for v in CANDIDATES["assign_ctas_per_sm"] if sums["value"] == 1 or v <= 4])
        return dict(e, sums=sums)

    def tune_lookup(self, voc, desc, repeats: int = 3) -> dict:
        """Tunes the tensor-core schedule of algo "auto" on lookups of `desc` through `voc`, timed
        by the library's pass events."""
        import torch

        from . import timing_enable, timing_read, timing_reset

        out = torch.empty(desc.shape[0], dtype=torch.int32, device=desc.device)

        def measure() -> float:
            voc.lookup(desc, out)
            torch.cuda.synchronize()
            timing_reset()
            timing_enable(True)
            for _ in range(repeats):
                voc.lookup(desc, out)
            torch.cuda.synchronize()
            timing_enable(False)
            return timing_read("lookup_pass_tc")[0] / repeats

        return self.tune("lookup_schedule", voc.branch_factor, voc.nb_levels, desc.shape[0], measure)

    def tune_lookup_regroup(self, voc, desc, repeats: int = 3) -> dict:
        """Tunes the scatter of regroups of more than 1,024 bins (trees with B^(2p+2) > 1,024 at a
        pass boundary) on lookups of `desc`, timed by the library's regroup events."""
        import torch

        from . import timing_enable, timing_read, timing_reset

        out = torch.empty(desc.shape[0], dtype=torch.int32, device=desc.device)

        def measure() -> float:
            voc.lookup(desc, out)
            torch.cuda.synchronize()
            timing_reset()
            timing_enable(True)
            for _ in range(repeats):
                voc.lookup(desc, out)
            torch.cuda.synchronize()
            timing_enable(False)
            return timing_read("lookup_regroup")[0] / repeats

        return self.tune("scatter_rows", voc.branch_factor, voc.nb_levels, desc.shape[0], measure)

    def tune_database(self, voc, doc_ids, leaves, offsets, query_leaves, query_offsets, max_results: int,
                      repeats: int = 3) -> dict:
        """Tunes the inverted-file layout (one CSR per document shard or one CSR) on batched queries
        (CUDA uint32 leaves, uint64 offsets) against a database of the given documents (host
        arrays, DataBase.add_docs form), timed by the library's scoring events.  The layout is
        chosen when the index is built, so each candidate builds its own database."""
        import torch

        from . import timing_enable, timing_read, timing_reset
        from .database import DataBase

        n_docs = int(np.asarray(doc_ids).size)

        def measure() -> float:
            db = DataBase(voc)
            db.add_docs(doc_ids, leaves, offsets)
            db.query_batched(query_leaves, query_offsets, max_results)  # builds the index
            torch.cuda.synchronize()
            timing_reset()
            timing_enable(True)
            for _ in range(repeats):
                db.query_batched(query_leaves, query_offsets, max_results)
            torch.cuda.synchronize()
            timing_enable(False)
            del db
            return timing_read("score")[0] / repeats

        return self.tune("db_shard_tables", voc.branch_factor, voc.nb_levels, n_docs, measure)
