"""Test infrastructure only: ctypes access to the two checkers.

* ``Oracle``   -- liborc.so, the C++ restatement of the reference algorithm (rbw_oracle.cpp).
* ``Reference``-- _ref/libref_rbow.so, the unmodified reference sources built by oracle/Makefile.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs import this module,
and only to check results or to time the CPU baseline.  The product never calls it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liborc.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_rbow.so")

INIT_REFERENCE, INIT_KMEANSPP, INIT_INJECTED = 0, 1, 2

u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def level_beg(B: int, level: int) -> int:
    acc = 0
    for _ in range(level):
        acc = acc * B + 1
    return acc


def build_oracle(reference_dir: str | None = None) -> None:
    """Compile liborc.so, and the reference checker when the reference sources are given
    (``reference_dir``, else the environment variable RBW_REFERENCE_DIR) and present."""
    import subprocess

    subprocess.run(["make", "-C", HERE, "orc"], check=True, capture_output=True)
    ref = reference_dir or os.environ.get("RBW_REFERENCE_DIR", "")
    if ref and os.path.isdir(ref):
        subprocess.run(["make", "-C", HERE, "ref", "REF=" + ref], check=True, capture_output=True)


class Oracle:
    _lib = None

    def __init__(self) -> None:
        if Oracle._lib is None:
            if not os.path.exists(ORC_PATH):
                build_oracle()
            lib = C.CDLL(ORC_PATH)
            lib.orc_level_beg.restype = C.c_uint64
            lib.orc_level_beg.argtypes = [C.c_uint32, C.c_uint32]
            lib.orc_lookup.restype = None
            lib.orc_lookup.argtypes = [u8p, C.c_uint32, C.c_uint32, u8p, C.c_uint64, u32p, C.c_uint32]
            lib.orc_kmeans_assign.restype = None
            lib.orc_kmeans_assign.argtypes = [u8p, u32p, C.c_uint32, u8p, C.c_uint32, u8p, u32p, u64p, u32p]
            lib.orc_kmeans_update.restype = None
            lib.orc_kmeans_update.argtypes = [u32p, u64p, C.c_uint32, u8p]
            lib.orc_kmeanspp_init.restype = C.c_uint32
            lib.orc_kmeanspp_init.argtypes = [u8p, u32p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                                              C.c_uint64, u32p]
            lib.orc_build_vocabulary.restype = C.c_int
            lib.orc_build_vocabulary.argtypes = [u8p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                                 C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p,
                                                 u8p, u32p, f32p, u32p, u32p]
            lib.orc_dist64.restype = C.c_double
            lib.orc_dist64.argtypes = [u8p, f32p]
            lib.orc_lookup_f32.restype = None
            lib.orc_lookup_f32.argtypes = [f32p, C.c_uint32, C.c_uint32, u8p, C.c_uint64, u32p, C.c_uint32]
            lib.orc_build_vocabulary_f32.restype = C.c_int
            lib.orc_build_vocabulary_f32.argtypes = [u8p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                                     C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p,
                                                     f32p, u32p, f32p, u32p, u32p, f64p, f64p, C.c_uint32]
            lib.orc_db_create.restype = C.c_void_p
            lib.orc_db_create.argtypes = [C.c_uint32, C.c_uint32, f32p]
            lib.orc_db_destroy.restype = None
            lib.orc_db_destroy.argtypes = [C.c_void_p]
            lib.orc_db_add.restype = C.c_int
            lib.orc_db_add.argtypes = [C.c_void_p, C.c_uint32, u32p, C.c_uint32]
            lib.orc_db_doc_rcp.restype = C.c_float
            lib.orc_db_doc_rcp.argtypes = [C.c_void_p, C.c_uint32]
            lib.orc_db_query.restype = C.c_uint32
            lib.orc_db_query.argtypes = [C.c_void_p, u32p, C.c_uint32, C.c_uint32, C.c_int, u32p, f64p,
                                         C.c_uint32]
            lib.orc_db_word_postings.restype = None
            lib.orc_db_word_postings.argtypes = [C.c_void_p, u64p]
            lib.orc_db_set_word_postings.restype = None
            lib.orc_db_set_word_postings.argtypes = [C.c_void_p, C.c_void_p]
            lib.orc_db_postings.restype = C.c_uint32
            lib.orc_db_postings.argtypes = [C.c_void_p, C.c_uint32, u32p, C.c_uint32]
            Oracle._lib = lib
        self.lib = Oracle._lib

    # ---------------------------------------------------------------- lookup
    def lookup(self, centers: np.ndarray, B: int, L: int, desc: np.ndarray, threads: int = 1) -> np.ndarray:
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        out = np.empty(desc.shape[0], dtype=np.uint32)
        self.lib.orc_lookup(np.ascontiguousarray(centers, dtype=np.uint8).reshape(-1), B, L,
                            desc.reshape(-1), desc.shape[0], out, threads)
        return out

    # ---------------------------------------------------------------- k-means
    def kmeans_assign(self, desc, members, centers, B, assign):
        members = np.ascontiguousarray(members, dtype=np.uint32)
        assign = np.ascontiguousarray(assign, dtype=np.uint8).copy()
        counts = np.zeros(B, dtype=np.uint32)
        sums = np.zeros(B * 128, dtype=np.uint64)
        changed = np.zeros(1, dtype=np.uint32)
        self.lib.orc_kmeans_assign(np.ascontiguousarray(desc, dtype=np.uint8).reshape(-1), members,
                                   members.size, np.ascontiguousarray(centers, dtype=np.uint8).reshape(-1),
                                   B, assign, counts, sums, changed)
        return assign, counts, sums.reshape(B, 128), int(changed[0])

    def kmeans_update(self, counts, sums, centers):
        centers = np.ascontiguousarray(centers, dtype=np.uint8).copy()
        B = centers.shape[0]
        self.lib.orc_kmeans_update(np.ascontiguousarray(counts, dtype=np.uint32),
                                   np.ascontiguousarray(sums, dtype=np.uint64).reshape(-1), B,
                                   centers.reshape(-1))
        return centers

    def kmeanspp_init(self, desc, members, B, seed, level, node):
        members = np.ascontiguousarray(members, dtype=np.uint32)
        out = np.empty(B, dtype=np.uint32)
        n = self.lib.orc_kmeanspp_init(np.ascontiguousarray(desc, dtype=np.uint8).reshape(-1), members,
                                       members.size, B, seed, level, node, out)
        return out, int(n)

    def build_vocabulary(self, desc, nb_doc, B, L, max_iter=1000, init=INIT_REFERENCE, seed=0, injected=None):
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        nodes = level_beg(B, L)
        centers = np.empty((nodes, B, 128), dtype=np.uint8)
        masks = np.empty(nodes, dtype=np.uint32)
        weights = np.empty((nodes, B), dtype=np.float32)
        occ = np.empty((nodes, B), dtype=np.uint32)
        iters = np.empty(nodes, dtype=np.uint32)
        inj = None
        if injected is not None:
            injected = np.ascontiguousarray(injected, dtype=np.uint32)
            inj = injected.ctypes.data_as(C.c_void_p)
        rc = self.lib.orc_build_vocabulary(desc.reshape(-1), desc.shape[0], nb_doc, B, L, max_iter, init, seed,
                                           inj, centers.reshape(-1), masks, weights.reshape(-1),
                                           occ.reshape(-1), iters)
        if rc != 0:
            raise ValueError("oracle build rejected its input")
        return dict(centers=centers, masks=masks, weights=weights, occ=occ, iters=iters)

    # ---------------------------------------------------------------- float-center mode
    def dist64(self, x: np.ndarray, c: np.ndarray) -> float:
        return float(self.lib.orc_dist64(np.ascontiguousarray(x, dtype=np.uint8),
                                         np.ascontiguousarray(c, dtype=np.float32)))

    def lookup_f32(self, centers: np.ndarray, B: int, L: int, desc: np.ndarray, threads: int = 1) -> np.ndarray:
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        out = np.empty(desc.shape[0], dtype=np.uint32)
        self.lib.orc_lookup_f32(np.ascontiguousarray(centers, dtype=np.float32).reshape(-1), B, L,
                                desc.reshape(-1), desc.shape[0], out, threads)
        return out

    def build_vocabulary_f32(self, desc, nb_doc, B, L, max_iter=1000, init=INIT_REFERENCE, seed=0, injected=None,
                             threads: int = 1):
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        nodes = level_beg(B, L)
        centers = np.empty((nodes, B, 128), dtype=np.float32)
        masks = np.empty(nodes, dtype=np.uint32)
        weights = np.empty((nodes, B), dtype=np.float32)
        occ = np.empty((nodes, B), dtype=np.uint32)
        iters = np.empty(nodes, dtype=np.uint32)
        first = np.empty(L, dtype=np.float64)
        last = np.empty(L, dtype=np.float64)
        inj = None
        if injected is not None:
            injected = np.ascontiguousarray(injected, dtype=np.uint32)
            inj = injected.ctypes.data_as(C.c_void_p)
        rc = self.lib.orc_build_vocabulary_f32(desc.reshape(-1), desc.shape[0], nb_doc, B, L, max_iter, init, seed,
                                               inj, centers.reshape(-1), masks, weights.reshape(-1),
                                               occ.reshape(-1), iters, first, last, threads)
        if rc != 0:
            raise ValueError("oracle build rejected its input")
        return dict(centers=centers, masks=masks, weights=weights, occ=occ, iters=iters, inertia_first=first,
                    inertia_last=last)

    # ---------------------------------------------------------------- DataBase
    def db(self, B: int, L: int, weights: np.ndarray) -> "OracleDb":
        return OracleDb(self, B, L, weights)


class OracleDb:
    def __init__(self, orc: Oracle, B: int, L: int, weights: np.ndarray) -> None:
        self.lib = orc.lib
        self.B, self.L = B, L
        self._w = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1)
        self.h = self.lib.orc_db_create(B, L, self._w)

    def __del__(self) -> None:
        if getattr(self, "h", None):
            self.lib.orc_db_destroy(self.h)
            self.h = None

    def add(self, doc: int, leaves: np.ndarray) -> None:
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        if self.lib.orc_db_add(self.h, doc, leaves, leaves.size) != 0:
            raise RuntimeError("Duplicate document index")

    def doc_rcp(self, doc: int) -> float:
        return float(self.lib.orc_db_doc_rcp(self.h, doc))

    def word_postings(self) -> np.ndarray:
        out = np.empty(level_beg(self.B, self.L) * self.B, dtype=np.uint64)
        self.lib.orc_db_word_postings(self.h, out)
        return out

    def set_word_postings(self, counts) -> None:
        if counts is None:
            self.lib.orc_db_set_word_postings(self.h, None)
            return
        self._ext = np.ascontiguousarray(counts, dtype=np.uint64)
        self.lib.orc_db_set_word_postings(self.h, self._ext.ctypes.data_as(C.c_void_p))

    def postings(self, leaf: int) -> np.ndarray:
        n = self.lib.orc_db_postings(self.h, leaf, np.empty(0, np.uint32), 0)
        out = np.empty(n, dtype=np.uint32)
        self.lib.orc_db_postings(self.h, leaf, out, n)
        return out

    def query(self, leaves: np.ndarray, max_results: int, mode: int = 0, capacity: int = 1 << 22):
        """All touched documents sorted by (score, doc); mode 0 = reference arithmetic, 1 = FP64."""
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        docs = np.empty(capacity, dtype=np.uint32)
        scores = np.empty(capacity, dtype=np.float64)
        n = self.lib.orc_db_query(self.h, leaves, leaves.size, max_results, mode, docs, scores, capacity)
        n = min(n, capacity)
        return docs[:n].copy(), scores[:n].copy()


class Reference:
    """The reference itself (oracle/_ref/libref_rbow.so).  DataBase calls run on the CPU; the
    vocabulary, lookup and k-means-kernel calls need a GPU."""

    _lib = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_PATH)

    def __init__(self) -> None:
        if Reference._lib is None:
            lib = C.CDLL(REF_PATH)
            lib.ref_last_error.restype = C.c_char_p
            lib.ref_hostvoc_create.restype = C.c_void_p
            lib.ref_hostvoc_create.argtypes = [C.c_uint32, f32p]
            lib.ref_hostvoc_destroy.argtypes = [C.c_void_p]
            lib.ref_db_create.restype = C.c_void_p
            lib.ref_db_create.argtypes = [C.c_void_p]
            lib.ref_db_destroy.argtypes = [C.c_void_p]
            lib.ref_db_add.restype = C.c_int
            lib.ref_db_add.argtypes = [C.c_void_p, C.c_uint32, u32p, C.c_uint32]
            lib.ref_db_query.restype = C.c_int
            lib.ref_db_query.argtypes = [C.c_void_p, u32p, C.c_uint32, C.c_uint32, u32p, u32p]
            lib.ref_db_query_batch.restype = C.c_int
            lib.ref_db_query_batch.argtypes = [C.c_void_p, u32p, u64p, C.c_uint32, C.c_uint32, u32p, u32p,
                                               C.c_uint32]
            lib.ref_build_vocabulary.restype = C.c_int
            lib.ref_build_vocabulary.argtypes = [u8p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                                 C.c_uint32, C.POINTER(C.POINTER(C.c_uint8)),
                                                 C.POINTER(C.c_uint64)]
            lib.ref_free.argtypes = [C.c_void_p]
            lib.ref_lookup.restype = C.c_int
            lib.ref_lookup.argtypes = [u8p, C.c_uint64, u8p, C.c_uint32, u32p]
            lib.ref_lookup_device_timed.restype = C.c_int
            lib.ref_lookup_device_timed.argtypes = [u8p, C.c_uint64, u8p, C.c_uint32, u32p, C.c_uint32,
                                                    C.POINTER(C.c_float)]
            lib.ref_kmeans_task.restype = C.c_int
            lib.ref_kmeans_task.argtypes = [u32p, C.c_uint32, C.c_uint32, u32p, u8p, u32p, u32p, u32p, C.c_int]
            Reference._lib = lib
        self.lib = Reference._lib

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def db(self, L: int, weights: np.ndarray) -> "ReferenceDb":
        return ReferenceDb(self, L, weights)

    def build_vocabulary(self, desc: np.ndarray, nb_doc: int, L: int, max_iter: int = 0,
                         check_interval: int = 4) -> bytes:
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        blob = C.POINTER(C.c_uint8)()
        size = C.c_uint64()
        self._check(self.lib.ref_build_vocabulary(desc.reshape(-1), desc.shape[0], nb_doc, L, max_iter,
                                                  check_interval, C.byref(blob), C.byref(size)))
        data = bytes(C.string_at(blob, size.value))
        self.lib.ref_free(blob)
        return data

    def lookup(self, blob: bytes, desc: np.ndarray) -> np.ndarray:
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        out = np.empty(desc.shape[0], dtype=np.uint32)
        b = np.frombuffer(blob, dtype=np.uint8).copy()
        self._check(self.lib.ref_lookup(b, b.size, desc.reshape(-1), desc.shape[0], out))
        return out

    def lookup_device_timed(self, blob: bytes, desc: np.ndarray, iters: int = 5):
        """(leaf IDs, ms per launch) of the reference lookup kernel on descriptors already in
        device memory (launches bracketed by CUDA events; the copy in is not timed)."""
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        out = np.empty(desc.shape[0], dtype=np.uint32)
        b = np.frombuffer(blob, dtype=np.uint8).copy()
        ms = C.c_float()
        self._check(self.lib.ref_lookup_device_timed(b, b.size, desc.reshape(-1), desc.shape[0], out, iters,
                                                     C.byref(ms)))
        return out, float(ms.value)

    def kmeans_task(self, tiles_words, nb_desc, centers_words, assign, do_update):
        tiles_words = np.ascontiguousarray(tiles_words, dtype=np.uint32)
        centers_words = np.ascontiguousarray(centers_words, dtype=np.uint32).copy()
        assign = np.ascontiguousarray(assign, dtype=np.uint8).copy()
        counts = np.zeros(16, dtype=np.uint32)
        sums = np.zeros(2048, dtype=np.uint32)
        changed = np.zeros(1, dtype=np.uint32)
        self._check(self.lib.ref_kmeans_task(tiles_words.reshape(-1), tiles_words.size // 1024, nb_desc,
                                             centers_words.reshape(-1), assign, counts, sums, changed,
                                             int(do_update)))
        return centers_words, assign, counts, sums, int(changed[0])


class ReferenceDb:
    def __init__(self, ref: Reference, L: int, weights: np.ndarray) -> None:
        self.ref = ref
        self.lib = ref.lib
        self._w = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1)
        self.voc = self.lib.ref_hostvoc_create(L, self._w)
        self.h = self.lib.ref_db_create(self.voc)

    def __del__(self) -> None:
        if getattr(self, "h", None):
            self.lib.ref_db_destroy(self.h)
            self.lib.ref_hostvoc_destroy(self.voc)
            self.h = None

    def add(self, doc: int, leaves: np.ndarray) -> None:
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        self.ref._check(self.lib.ref_db_add(self.h, doc, leaves, leaves.size))

    def query(self, leaves: np.ndarray, k: int) -> np.ndarray:
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        out = np.empty(max(k, 1), dtype=np.uint32)
        n = np.zeros(1, dtype=np.uint32)
        self.ref._check(self.lib.ref_db_query(self.h, leaves, leaves.size, k, out, n))
        return out[: int(n[0])].copy()

    def query_batch(self, leaves: np.ndarray, offsets: np.ndarray, k: int, threads: int):
        leaves = np.ascontiguousarray(leaves, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        nq = offsets.size - 1
        out = np.zeros((nq, max(k, 1)), dtype=np.uint32)
        n = np.zeros(nq, dtype=np.uint32)
        self.ref._check(self.lib.ref_db_query_batch(self.h, leaves, offsets, nq, k, out.reshape(-1), n, threads))
        return out, n


# ------------------------------------------------------------------ layout conversions
def centers_to_reference_nodes(centers: np.ndarray) -> np.ndarray:
    """[nodes][16][128] uint8 -> reference Node bytes (uint32[32 words][16 centers] per node)."""
    nodes = centers.shape[0]
    c = centers.reshape(nodes, 16, 32, 4)          # node, center, word, byte
    return np.ascontiguousarray(c.transpose(0, 2, 1, 3)).reshape(nodes, 2048)


def reference_nodes_to_centers(nodes_bytes: np.ndarray) -> np.ndarray:
    nodes = nodes_bytes.shape[0]
    c = nodes_bytes.reshape(nodes, 32, 16, 4)      # node, word, center, byte
    return np.ascontiguousarray(c.transpose(0, 2, 1, 3)).reshape(nodes, 16, 128)


def parse_reference_blob(blob: bytes):
    """Vocabulary blob (Vocabulary.cpp:175-198): u32 L | Node x levelBeg(L) | u16 mask x .. | f32[16] x .."""
    b = np.frombuffer(blob, dtype=np.uint8)
    L = int(b[:4].view(np.uint32)[0])
    nodes = level_beg(16, L)
    off = 4
    nb = b[off: off + nodes * 2048].reshape(nodes, 2048)
    off += nodes * 2048
    masks = b[off: off + nodes * 2].view(np.uint16).astype(np.uint32)
    off += nodes * 2
    weights = b[off: off + nodes * 64].view(np.float32).reshape(nodes, 16)
    return L, reference_nodes_to_centers(nb), masks, weights.copy()
