"""Mirror of rbow::IDataBase (RapidBoW.h:92-107) over the C ABI (device-resident inverted file)."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import RBW_ERR_UNSUPPORTED, RbwError, Vocabulary, _check, _dev_ptr, _stream_ptr, load_library


class DataBase:
    """Inverted file over the leaf words of a vocabulary, scored with hierarchical tf-idf L1
    distances (DataBase.cpp:39-197).  Leaf indices are host arrays, as in the reference."""

    def __init__(self, voc: Vocabulary) -> None:
        self._lib = load_library()
        if getattr(self._lib, "rbw_db_create", None) is None:
            raise RbwError(RBW_ERR_UNSUPPORTED, "this build has no DataBase entry points")
        self.voc = voc  # the DataBase keeps a non-owning reference (DataBase.h:43-45)
        h = C.c_void_p()
        _check(self._lib.rbw_db_create(voc.handle, C.byref(h)))
        self._h = h

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.rbw_db_destroy(h)
            self._h = None

    def get_vocabulary(self) -> Vocabulary:
        return self.voc

    def add_doc(self, idx_doc: int, leaves: np.ndarray) -> None:
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        _check(self._lib.rbw_db_add(self._h, idx_doc, leaves.ctypes.data, leaves.size))

    def add_docs(self, doc_ids: np.ndarray, leaves: np.ndarray, offsets: np.ndarray) -> None:
        """Adds many documents at once: doc i owns leaves[offsets[i]:offsets[i+1]]."""
        doc_ids = np.ascontiguousarray(doc_ids, dtype=np.uint32)
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        _check(self._lib.rbw_db_add_batch(self._h, doc_ids.ctypes.data, leaves.ctypes.data, offsets.ctypes.data,
                                          doc_ids.size))

    def query(self, leaves: np.ndarray, max_results: int, with_scores: bool = False):
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        docs = np.empty(max(max_results, 1), np.uint32)
        scores = np.empty(max(max_results, 1), np.float32)
        n = C.c_uint32()
        _check(self._lib.rbw_db_query(self._h, leaves.ctypes.data, leaves.size, max_results, docs.ctypes.data,
                                      scores.ctypes.data, C.byref(n)))
        k = n.value
        return (docs[:k].copy(), scores[:k].copy()) if with_scores else docs[:k].copy()

    def query_and_add_doc(self, idx_doc: int, leaves: np.ndarray, max_results: int) -> np.ndarray:
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        docs = np.empty(max(max_results, 1), np.uint32)
        scores = np.empty(max(max_results, 1), np.float32)
        n = C.c_uint32()
        _check(self._lib.rbw_db_query_and_add(self._h, idx_doc, leaves.ctypes.data, leaves.size, max_results,
                                              docs.ctypes.data, scores.ctypes.data, C.byref(n)))
        return docs[: n.value].copy()

    def query_batched(self, leaves, offsets, max_results: int, stream=None) -> Tuple[object, object, object]:
        """One launch scoring many queries.  leaves: CUDA int32/uint32 tensor; offsets: CUDA int64
        tensor [nq + 1].  Returns (docs [nq, k] int32, scores [nq, k] float32, counts [nq] int32)."""
        import torch

        nq = offsets.numel() - 1
        k = max_results
        docs = torch.empty((nq, max(k, 1)), dtype=torch.int32, device=leaves.device)
        scores = torch.empty((nq, max(k, 1)), dtype=torch.float32, device=leaves.device)
        counts = torch.empty(nq, dtype=torch.int32, device=leaves.device)
        _check(self._lib.rbw_db_query_batched(self._h, _dev_ptr(leaves), _dev_ptr(offsets), nq, k, _dev_ptr(docs),
                                              _dev_ptr(scores), _dev_ptr(counts), _stream_ptr(stream)))
        return docs, scores, counts

    def info(self) -> Tuple[int, int]:
        nd, npost = C.c_uint32(), C.c_uint64()
        _check(self._lib.rbw_db_info(self._h, C.byref(nd), C.byref(npost)))
        return nd.value, npost.value

    def segments(self) -> Tuple[int, int]:
        """Documents in the (main, delta) segments of the device index, after an update."""
        m, d = C.c_uint32(), C.c_uint32()
        _check(self._lib.rbw_db_segments(self._h, C.byref(m), C.byref(d)))
        return m.value, d.value

    def doc_rcp(self, doc: int) -> float:
        v = C.c_float()
        _check(self._lib.rbw_db_doc_rcp(self._h, doc, C.byref(v)))
        return v.value

    def word_postings(self) -> np.ndarray:
        """Subtree posting counts of every word ([levelBeg(L) * B] uint64), as the skip rule uses them."""
        B, L = self.voc.branch_factor, self.voc.nb_levels
        n = sum(B ** lv for lv in range(L)) * B
        out = np.empty(n, np.uint64)
        _check(self._lib.rbw_db_word_postings(self._h, out.ctypes.data))
        return out

    def set_word_postings(self, counts: Optional[np.ndarray]) -> None:
        """Counts for the skip rule in place of this database's own (None: its own again)."""
        if counts is None:
            _check(self._lib.rbw_db_set_word_postings(self._h, None))
            return
        c = np.ascontiguousarray(counts, np.uint64)
        _check(self._lib.rbw_db_set_word_postings(self._h, c.ctypes.data))

    def postings(self, leaf: int) -> np.ndarray:
        n = C.c_uint32()
        _check(self._lib.rbw_db_postings(self._h, leaf, None, 0, C.byref(n)))
        out = np.empty(n.value, np.uint32)
        _check(self._lib.rbw_db_postings(self._h, leaf, out.ctypes.data, n.value, C.byref(n)))
        return out


def create_database(voc: Vocabulary) -> DataBase:
    """rbow::createDataBase (RapidBoW.h:107)."""
    return DataBase(voc)
