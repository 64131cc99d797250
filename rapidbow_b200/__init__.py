"""RapidBoW-B200: B200-native vocabulary-tree hot path behind the reference's API.

Python mirror of the reference's public interface (RapidBoW.h:60-107) over the C ABI in
include/rapidbow_b200.h:

    rbow::buildVocabulary        -> build_vocabulary(...)            -> Vocabulary
    rbow::deserializeVocabulary  -> deserialize_vocabulary(blob)     -> Vocabulary
    IVocabulary::lookUp          -> Vocabulary.lookup(desc, out)     (device buffers, async)
    IVocabulary::serialize       -> Vocabulary.serialize()           -> bytes
    rbow::createDataBase         -> create_database(voc)             -> DataBase
    IDataBase::addDoc / query / queryAndAddDoc -> DataBase.add_doc / query / query_and_add_doc
    (no counterpart)             -> Server(voc, db): continuous-batching retrieval serving

Errors raise RbwError (the reference throws std::runtime_error).  The compiled library must be
present: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

__all__ = ["RbwError", "Vocabulary", "DataBase", "Server", "build_vocabulary", "deserialize_vocabulary", "create_database",
           "load_library", "LIB_PATH", "SIFT_ATTR"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librapidbow_b200.so")

RBW_OK, RBW_ERR_INVALID_ARG, RBW_ERR_UNSUPPORTED, RBW_ERR_OUT_OF_MEMORY, RBW_ERR_CUDA, RBW_ERR_TIMEOUT, \
    RBW_ERR_INVALID_BLOB, RBW_ERR_DUPLICATE, RBW_ERR_INTERNAL = range(9)
LOOKUP_ALGOS = {"auto": 0, "tensor_u8": 1, "simt_f32": 2, "tensor_u8_warpnode": 3, "tensor_u8_ring": 4}
INIT_MODES = {"reference": 0, "kmeans++": 1, "injected": 2}
DATA_BINARY, DATA_UINT8 = 0, 1
DIST_HAMMING, DIST_L1, DIST_L2 = 0, 1, 2


class DescAttr(C.Structure):
    _fields_ = [("data_type", C.c_int32), ("distance_type", C.c_int32), ("nb_dims", C.c_uint64)]


SIFT_ATTR = (DATA_UINT8, DIST_L2, 128)


class BuildOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_uint32), ("check_interval", C.c_uint32), ("init_mode", C.c_uint32),
                ("flags", C.c_uint32), ("seed", C.c_uint64), ("injected_init", C.c_void_p)]


class BuildStats(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("iterations", C.c_uint32 * 16), ("inertia_first", C.c_double * 16),
                ("inertia_last", C.c_double * 16), ("refined", C.c_uint64 * 16), ("assignments", C.c_uint64 * 16),
                ("seconds", C.c_double)]


BUILD_IEEE_DIVISION, BUILD_FLOAT_CENTERS = 1, 2


class RbwError(RuntimeError):
    def __init__(self, status: int, message: str) -> None:
        super().__init__(message)
        self.status = status


_lib: Optional[C.CDLL] = None


def load_library() -> C.CDLL:
    """Loads librapidbow_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RbwError(RBW_ERR_INTERNAL, f"{LIB_PATH} is missing; run rapidbow_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32
    pp = C.POINTER(C.c_void_p)
    sig = {
        "rbw_last_error": (C.c_char_p, []),
        "rbw_version": (C.c_char_p, []),
        "rbw_build_options_default": (None, [C.POINTER(BuildOptions)]),
        "rbw_voc_build": (C.c_int, [DescAttr, u32, vp, u32, u32, u32, C.POINTER(BuildOptions), vp, pp]),
        "rbw_voc_from_host": (C.c_int, [u32, u32, vp, vp, vp, pp]),
        "rbw_voc_lookup": (C.c_int, [vp, vp, u32, vp, vp]),
        "rbw_voc_lookup_ex": (C.c_int, [vp, vp, u64, vp, i32, vp, C.POINTER(u32)]),
        "rbw_voc_lookup_host": (C.c_int, [vp, vp, u64, vp, i32, C.POINTER(u32)]),
        "rbw_voc_serialize": (C.c_int, [vp, vp, u64, C.POINTER(u64)]),
        "rbw_voc_deserialize": (C.c_int, [vp, u64, pp]),
        "rbw_voc_info": (C.c_int, [vp, C.POINTER(DescAttr), C.POINTER(u32), C.POINTER(u32), C.POINTER(u64)]),
        "rbw_voc_level_weights": (C.c_int, [vp, u32, C.POINTER(C.POINTER(C.c_float))]),
        "rbw_voc_get_tree": (C.c_int, [vp, vp, vp, vp]),
        "rbw_voc_lookup_scratch_bytes": (C.c_int, [vp, u64, C.POINTER(u64)]),
        "rbw_voc_device_errors": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32)]),
        "rbw_voc_destroy": (None, [vp]),
        "rbw_voc_lookup_noalloc": (C.c_int, [vp, vp, u32, vp, vp]),
        "rbw_voc_from_host_f32": (C.c_int, [u32, u32, vp, vp, vp, pp]),
        "rbw_voc_center_type": (C.c_int, [vp, C.POINTER(i32)]),
        "rbw_voc_get_centers_f32": (C.c_int, [vp, vp]),
        "rbw_voc_build_stats": (C.c_int, [vp, C.POINTER(BuildStats)]),
        "rbw_voc_refined_lookups": (C.c_int, [vp, C.POINTER(u64)]),
        "rbw_kmeans_shard_create": (C.c_int, [vp, u32, u32, u32, vp, pp]),
        "rbw_kmeans_shard_destroy": (None, [vp]),
        "rbw_kmeans_shard_level": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32)]),
        "rbw_kmeans_shard_node_counts": (C.c_int, [vp, vp]),
        "rbw_kmeans_shard_member_rows": (C.c_int, [vp, vp, vp, u32, vp]),
        "rbw_kmeans_shard_desc_rows": (C.c_int, [vp, vp, u32, vp]),
        "rbw_kmeans_shard_set_centers": (C.c_int, [vp, vp]),
        "rbw_kmeans_shard_assign": (C.c_int, [vp, vp, vp, vp, vp]),
        "rbw_kmeans_shard_update": (C.c_int, [vp, vp, vp, vp]),
        "rbw_kmeans_shard_get_centers": (C.c_int, [vp, vp]),
        "rbw_kmeans_shard_next_level": (C.c_int, [vp, vp]),
        "rbw_init_picker_create": (C.c_int, [pp]),
        "rbw_init_picker_destroy": (None, [vp]),
        "rbw_init_picker_level": (C.c_int, [vp, u32, vp, u32, vp, vp]),
        "rbw_idf_weights": (C.c_int, [u32, vp, u64, vp]),
        "rbw_tuning_set": (C.c_int, [u32, u32, u32, u32, u32]),
        "rbw_tuning_get": (C.c_int, [u32, u32, u32, u64, C.POINTER(u32)]),
        "rbw_tuning_clear": (C.c_int, []),
        "rbw_timing_enable": (None, [i32]),
        "rbw_timing_reset": (C.c_int, []),
        "rbw_timing_read": (C.c_int, [u32, C.POINTER(C.c_double), C.POINTER(u64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _bind_optional(lib)
    _lib = lib
    return lib


def _bind_optional(lib: C.CDLL) -> None:
    """DataBase entry points (present once the scoring kernels are built in)."""
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32
    pp = C.POINTER(C.c_void_p)
    sig = {
        "rbw_db_create": (C.c_int, [vp, pp]),
        "rbw_db_destroy": (None, [vp]),
        "rbw_db_add": (C.c_int, [vp, u32, vp, u32]),
        "rbw_db_add_batch": (C.c_int, [vp, vp, vp, vp, u32]),
        "rbw_db_query": (C.c_int, [vp, vp, u32, u32, vp, vp, C.POINTER(u32)]),
        "rbw_db_query_and_add": (C.c_int, [vp, u32, vp, u32, u32, vp, vp, C.POINTER(u32)]),
        "rbw_db_query_batched": (C.c_int, [vp, vp, vp, u32, u32, vp, vp, vp, vp]),
        "rbw_db_info": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u64)]),
        "rbw_db_segments": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32)]),
        "rbw_db_doc_rcp": (C.c_int, [vp, u32, C.POINTER(C.c_float)]),
        "rbw_db_postings": (C.c_int, [vp, u32, vp, u32, C.POINTER(u32)]),
        "rbw_db_word_postings": (C.c_int, [vp, vp]),
        "rbw_db_set_word_postings": (C.c_int, [vp, vp]),
        "rbw_db_query_batched_host_offsets": (C.c_int, [vp, vp, vp, vp, u32, u32, vp, vp, vp, vp]),
        "rbw_server_options_default": (None, [vp]),
        "rbw_server_create": (C.c_int, [vp, vp, vp, pp]),
        "rbw_server_destroy": (None, [vp]),
        "rbw_server_submit": (C.c_int, [vp, vp, u32, C.POINTER(u64)]),
        "rbw_server_wait": (C.c_int, [vp, u64, C.c_int64, vp, vp, u32, C.POINTER(u32), C.POINTER(C.c_double)]),
        "rbw_server_get_stats": (C.c_int, [vp, vp]),
        "rbw_server_reset_stats": (C.c_int, [vp]),
        "rbw_server_batch_bytes": (C.c_int, [vp, u64, u32, C.POINTER(u64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name, None)
        if f is not None:
            f.restype = res
            f.argtypes = args


def _check(rc: int) -> None:
    if rc != RBW_OK:
        raise RbwError(rc, load_library().rbw_last_error().decode())


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _dev_ptr(t) -> int:
    """Device pointer of a torch CUDA tensor (contiguous)."""
    if not t.is_cuda:
        raise RbwError(RBW_ERR_INVALID_ARG, "expected a CUDA tensor")
    if not t.is_contiguous():
        raise RbwError(RBW_ERR_INVALID_ARG, "expected a contiguous tensor")
    return t.data_ptr()


class Vocabulary:
    """Mirror of rbow::IVocabulary (RapidBoW.h:60-71)."""

    def __init__(self, handle: int) -> None:
        self._h = C.c_void_p(handle)
        self._lib = load_library()

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.rbw_voc_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- attributes (RapidBoW.h:63-65)
    def _info(self):
        a, b, l, n = DescAttr(), C.c_uint32(), C.c_uint32(), C.c_uint64()
        _check(self._lib.rbw_voc_info(self._h, C.byref(a), C.byref(b), C.byref(l), C.byref(n)))
        return (a.data_type, a.distance_type, a.nb_dims), b.value, l.value, n.value

    def get_descriptor_attributes(self):
        return self._info()[0]

    @property
    def branch_factor(self) -> int:
        return self._info()[1]

    @property
    def nb_levels(self) -> int:
        return self._info()[2]

    @property
    def nb_nodes(self) -> int:
        return self._info()[3]

    def level_weights(self, level: int) -> np.ndarray:
        """getLevelWeights (RapidBoWInternal.h:26-31): float[levelSize(level)][B] (a copy)."""
        p = C.POINTER(C.c_float)()
        _check(self._lib.rbw_voc_level_weights(self._h, level, C.byref(p)))
        B = self.branch_factor
        n = (B ** level) * B
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(B ** level, B).copy()

    @property
    def float_centers(self) -> bool:
        """True for a float-center vocabulary (RBW_CENTERS_FLOAT32)."""
        v = C.c_int32()
        _check(self._lib.rbw_voc_center_type(self._h, C.byref(v)))
        return v.value == 1

    def centers_f32(self) -> np.ndarray:
        """fp32 centers [nodes][B][128] of a float-center vocabulary."""
        c = np.empty((self.nb_nodes, self.branch_factor, 128), np.float32)
        _check(self._lib.rbw_voc_get_centers_f32(self._h, c.ctypes.data))
        return c

    def build_stats(self) -> dict:
        """Statistics of the build (iterations, FP64 inertia, FP64 re-scored assignments per level)."""
        s = BuildStats()
        _check(self._lib.rbw_voc_build_stats(self._h, C.byref(s)))
        L = s.levels
        return {"levels": L, "iterations": list(s.iterations[:L]), "inertia_first": list(s.inertia_first[:L]),
                "inertia_last": list(s.inertia_last[:L]), "refined": list(s.refined[:L]),
                "assignments": list(s.assignments[:L]), "seconds": s.seconds}

    def refined_lookups(self) -> int:
        """Lookup descriptors re-scored in FP64 since the last call (float centers)."""
        v = C.c_uint64()
        _check(self._lib.rbw_voc_refined_lookups(self._h, C.byref(v)))
        return v.value

    def tree(self):
        """(centers [nodes][B][128] uint8, masks [nodes] uint32, weights [nodes][B] float32)."""
        B, nodes = self.branch_factor, self.nb_nodes
        c = np.empty((nodes, B, 128), np.uint8)
        m = np.empty(nodes, np.uint32)
        w = np.empty((nodes, B), np.float32)
        _check(self._lib.rbw_voc_get_tree(self._h, c.ctypes.data, m.ctypes.data, w.ctypes.data))
        return c, m, w

    # -- lookup (RapidBoW.h:66-68)
    def lookup(self, desc, out=None, algo: str = "auto", stream=None) -> "object":
        """Leaf index of every descriptor row; desc is a CUDA uint8 tensor [n, 128].  Returns an
        int32 CUDA tensor holding the uint32 leaf indices.  Asynchronous on `stream`."""
        import torch

        n = desc.shape[0]
        if desc.dtype != torch.uint8 or (n and desc.shape[1] != 128):
            raise RbwError(RBW_ERR_INVALID_ARG, "descriptors must be uint8 [n, 128]")
        if out is None:
            out = torch.empty(n, dtype=torch.int32, device=desc.device)
        k = C.c_uint32()
        _check(self._lib.rbw_voc_lookup_ex(self._h, _dev_ptr(desc) if n else None, n,
                                           _dev_ptr(out) if n else None, LOOKUP_ALGOS[algo],
                                           _stream_ptr(stream), C.byref(k)))
        self.last_kernels = k.value
        return out

    def lookup_noalloc(self, desc, out, stream=None):
        """Lookup whose working memory is the library's fixed per-GPU array (no allocation;
        see rbw_voc_lookup_noalloc for the limits).  desc: CUDA uint8 [n, 128]; out: CUDA int32 [n]."""
        n = desc.shape[0]
        _check(self._lib.rbw_voc_lookup_noalloc(self._h, _dev_ptr(desc) if n else None, n,
                                                _dev_ptr(out) if n else None, _stream_ptr(stream)))
        return out

    def lookup_host(self, desc: np.ndarray, algo: str = "auto") -> np.ndarray:
        """Host-to-host lookUp (copies in, looks up, copies out).  Synchronous."""
        desc = np.ascontiguousarray(desc, dtype=np.uint8)
        out = np.empty(desc.shape[0], np.uint32)
        k = C.c_uint32()
        _check(self._lib.rbw_voc_lookup_host(self._h, desc.ctypes.data, desc.shape[0], out.ctypes.data,
                                             LOOKUP_ALGOS[algo], C.byref(k)))
        self.last_kernels = k.value
        return out

    def lookup_host_ptr(self, desc_ptr: int, n: int, out_ptr: int, algo: str = "auto") -> int:
        k = C.c_uint32()
        _check(self._lib.rbw_voc_lookup_host(self._h, desc_ptr, n, out_ptr, LOOKUP_ALGOS[algo], C.byref(k)))
        return k.value

    def scratch_bytes(self, n: int) -> int:
        b = C.c_uint64()
        _check(self._lib.rbw_voc_lookup_scratch_bytes(self._h, n, C.byref(b)))
        return b.value

    def device_errors(self):
        code, where = C.c_uint32(), C.c_uint32()
        _check(self._lib.rbw_voc_device_errors(self._h, C.byref(code), C.byref(where)))
        return code.value, where.value

    # -- persistence (RapidBoW.h:69,90)
    def serialize(self) -> bytes:
        size = C.c_uint64()
        _check(self._lib.rbw_voc_serialize(self._h, None, 0, C.byref(size)))
        buf = (C.c_uint8 * size.value)()
        _check(self._lib.rbw_voc_serialize(self._h, buf, size.value, C.byref(size)))
        return bytes(buf)


TIMED_KERNELS = {"lookup_pass_tc": 0, "lookup_simt_f32": 1, "lookup_regroup": 2, "kmeans_assign": 3,
                 "kmeans_update": 4, "score": 5, "index": 6, "score_prep": 7, "score_merge": 8}


def timing_enable(on: bool) -> None:
    """Brackets this library's kernel launches with CUDA events (see rbw_timing_enable)."""
    load_library().rbw_timing_enable(1 if on else 0)


def timing_reset() -> None:
    _check(load_library().rbw_timing_reset())


def timing_read(kernel: str):
    """(total milliseconds, launches) of the completed launches of one kernel since the reset."""
    ms, n = C.c_double(), C.c_uint64()
    _check(load_library().rbw_timing_read(TIMED_KERNELS[kernel], C.byref(ms), C.byref(n)))
    return ms.value, n.value


def build_vocabulary(descriptors, branch_factor: int = 16, nb_doc: int = 1, nb_levels: int = 4, stream=None,
                     max_iterations: int = 1000, check_interval: int = 4, init: str = "reference", seed: int = 0,
                     injected: Optional[np.ndarray] = None, attr=SIFT_ATTR,
                     ieee_division: bool = False, float_centers: bool = False) -> Vocabulary:
    """rbow::buildVocabulary (RapidBoW.h:82-88); descriptors is a CUDA uint8 tensor [n, 128].
    ieee_division=True rounds centers with the correctly rounded quotient instead of the
    reference's fast-math division; float_centers=True keeps fp32 centers (split-bf16 distances
    with an FP64 re-score near ties, see RBW_BUILD_FLOAT_CENTERS)."""
    lib = load_library()
    o = BuildOptions()
    lib.rbw_build_options_default(C.byref(o))
    o.max_iterations = max_iterations
    o.check_interval = check_interval
    o.init_mode = INIT_MODES[init]
    o.seed = seed
    o.flags = (BUILD_IEEE_DIVISION if ieee_division else 0) | (BUILD_FLOAT_CENTERS if float_centers else 0)
    keep = None
    if injected is not None:
        keep = np.ascontiguousarray(injected, dtype=np.uint32)
        o.injected_init = keep.ctypes.data
    h = C.c_void_p()
    n = descriptors.shape[0]
    _check(lib.rbw_voc_build(DescAttr(*attr), branch_factor, _dev_ptr(descriptors), n, nb_doc, nb_levels,
                             C.byref(o), _stream_ptr(stream), C.byref(h)))
    del keep
    return Vocabulary(h.value)


def vocabulary_from_host(branch_factor: int, nb_levels: int, centers: np.ndarray, masks: np.ndarray,
                         weights: np.ndarray) -> Vocabulary:
    lib = load_library()
    centers = np.ascontiguousarray(centers, dtype=np.uint8)
    masks = np.ascontiguousarray(masks, dtype=np.uint32)
    weights = np.ascontiguousarray(weights, dtype=np.float32)
    h = C.c_void_p()
    _check(lib.rbw_voc_from_host(branch_factor, nb_levels, centers.ctypes.data, masks.ctypes.data,
                                 weights.ctypes.data, C.byref(h)))
    return Vocabulary(h.value)


def vocabulary_from_host_f32(branch_factor: int, nb_levels: int, centers: np.ndarray, masks: np.ndarray,
                             weights: np.ndarray) -> Vocabulary:
    """A float-center vocabulary from fp32 centers [nodes][B][128]."""
    lib = load_library()
    centers = np.ascontiguousarray(centers, dtype=np.float32)
    masks = np.ascontiguousarray(masks, dtype=np.uint32)
    weights = np.ascontiguousarray(weights, dtype=np.float32)
    h = C.c_void_p()
    _check(lib.rbw_voc_from_host_f32(branch_factor, nb_levels, centers.ctypes.data, masks.ctypes.data,
                                     weights.ctypes.data, C.byref(h)))
    return Vocabulary(h.value)


def deserialize_vocabulary(blob: bytes) -> Vocabulary:
    """rbow::deserializeVocabulary (RapidBoW.h:90)."""
    lib = load_library()
    buf = (C.c_uint8 * len(blob)).from_buffer_copy(blob)
    h = C.c_void_p()
    _check(lib.rbw_voc_deserialize(buf, len(blob), C.byref(h)))
    return Vocabulary(h.value)


from .database import DataBase, create_database  # noqa: E402
from .server import Server  # noqa: E402
