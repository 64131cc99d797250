"""Multi-GPU hot path: a hierarchical k-means build over descriptors sharded across ranks, and an
inverted file sharded by documents with a merged top-k.  No counterpart in the reference, which
runs on one GPU (Vocabulary.cpp:32-121) and one host DataBase (DataBase.cpp:39-197).

One process per GPU with torch.distributed (NCCL between GPUs; gloo works too, through host
copies).  Every rank runs the same steps in the same order:

Build (`build_vocabulary_sharded`): rank r holds descriptors [offset_r, offset_r + n_r) of the
whole set.  Per level, the node sizes are all-gathered and the initial centers chosen from them
(the reference's picks over the whole set, or injected descriptor indices); the rank owning each
picked row contributes it to an all-reduce.  Per Lloyd step every rank assigns its own members
(rbw_kmeans_shard_assign), the per-node sums [nodes][16][128], counts [nodes][16] and change
counts [nodes] are all-reduced, and every rank applies the same update, so the centers stay
identical on all ranks.  Child sizes are all-reduced into the occurrence counts of the idf
weights.  The result equals the one-GPU build with IEEE rounding of the center quotient, byte
for byte.

Database (`ShardedDataBase`): rank r holds some of the documents.  The reference's skip rule
(a non-leaf word is scored only while its subtree holds fewer than 16 + 4k postings,
DataBase.cpp:125) counts the postings of the whole database, so `sync()` all-reduces every
shard's subtree posting counts and installs the sum in each shard.  A query runs on every shard
and the per-shard top-k lists are all-gathered and merged by (score, document id), which gives
exactly the top-k of one database holding every document.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _check, _dev_ptr, _stream_ptr, load_library

INVALID = 0xFFFFFFFF


def _level_beg(B: int, level: int) -> int:
    acc = 0
    for _ in range(level):
        acc = acc * B + 1
    return acc


# ------------------------------------------------------------------ collectives
def _dist():
    import torch.distributed as dist

    return dist


def _coll_device(group):
    """Device of tensors handed to collectives: CUDA for NCCL, CPU otherwise."""
    import torch

    dist = _dist()
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")


def _all_reduce_(t, group):
    """In-place sum over ranks of a tensor on any device (copied through the collective device)."""
    dist = _dist()
    dev = _coll_device(group)
    if t.device == dev:
        dist.all_reduce(t, group=group)
        return t
    tmp = t.to(dev)
    dist.all_reduce(tmp, group=group)
    t.copy_(tmp)
    return t


def _all_reduce_np(a: np.ndarray, group) -> np.ndarray:
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a).astype(np.int64))
    _all_reduce_(t, group)
    return t.numpy()


def _all_gather_np(a: np.ndarray, group) -> np.ndarray:
    """[world, *a.shape] of equally shaped int64 arrays."""
    import torch

    dist = _dist()
    dev = _coll_device(group)
    t = torch.from_numpy(np.ascontiguousarray(a).astype(np.int64)).to(dev)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return np.stack([o.cpu().numpy() for o in out])


# ------------------------------------------------------------------ build
class CudaShardEngine:
    """This rank's descriptors on its GPU, driven through rbw_kmeans_shard_*."""

    def __init__(self, desc, B: int, L: int, stream=None) -> None:
        import torch

        if desc.dtype != torch.uint8 or desc.dim() != 2 or desc.shape[1] != 128:
            raise ValueError("descriptors must be a CUDA uint8 tensor [n, 128]")
        self._lib = load_library()
        self.desc, self.B, self.L = desc, B, L
        self.n_local = int(desc.shape[0])
        self.device = desc.device
        self._stream = stream
        h = C.c_void_p()
        _check(self._lib.rbw_kmeans_shard_create(_dev_ptr(desc) if self.n_local else None, self.n_local, B, L,
                                                 _stream_ptr(stream), C.byref(h)))
        self._h = h

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.rbw_kmeans_shard_destroy(h)
            self._h = None

    def _nodes(self) -> int:
        nb = C.c_uint32()
        _check(self._lib.rbw_kmeans_shard_level(self._h, None, C.byref(nb)))
        return nb.value

    def node_counts(self) -> np.ndarray:
        out = np.empty(self._nodes(), np.uint32)
        _check(self._lib.rbw_kmeans_shard_node_counts(self._h, out.ctypes.data))
        return out

    def member_rows(self, nodes: np.ndarray, pos: np.ndarray) -> np.ndarray:
        nodes = np.ascontiguousarray(nodes, np.uint32)
        pos = np.ascontiguousarray(pos, np.uint32)
        out = np.empty((nodes.size, 128), np.uint8)
        _check(self._lib.rbw_kmeans_shard_member_rows(self._h, nodes.ctypes.data, pos.ctypes.data, nodes.size,
                                                      out.ctypes.data))
        return out

    def desc_rows(self, idx: np.ndarray) -> np.ndarray:
        idx = np.ascontiguousarray(idx, np.uint32)
        out = np.empty((idx.size, 128), np.uint8)
        _check(self._lib.rbw_kmeans_shard_desc_rows(self._h, idx.ctypes.data, idx.size, out.ctypes.data))
        return out

    def set_centers(self, centers: np.ndarray) -> None:
        c = np.ascontiguousarray(centers, np.uint8)
        _check(self._lib.rbw_kmeans_shard_set_centers(self._h, c.ctypes.data))

    def buffers(self, nb: int):
        import torch

        z = dict(device=self.device)
        return (torch.zeros(nb, dtype=torch.int32, **z), torch.zeros((nb, 16, 128), dtype=torch.int64, **z),
                torch.zeros((nb, 16), dtype=torch.int32, **z), torch.zeros(nb, dtype=torch.int32, **z))

    def assign(self, last, sums, counts, changed) -> None:
        _check(self._lib.rbw_kmeans_shard_assign(self._h, _dev_ptr(last), _dev_ptr(sums), _dev_ptr(counts),
                                                 _dev_ptr(changed)))

    def update(self, sums, counts, changed) -> None:
        _check(self._lib.rbw_kmeans_shard_update(self._h, _dev_ptr(sums), _dev_ptr(counts), _dev_ptr(changed)))

    def get_centers(self) -> np.ndarray:
        out = np.empty((self._nodes(), self.B, 128), np.uint8)
        _check(self._lib.rbw_kmeans_shard_get_centers(self._h, out.ctypes.data))
        return out

    def next_level(self) -> np.ndarray:
        out = np.empty(self._nodes() * self.B, np.uint32)
        _check(self._lib.rbw_kmeans_shard_next_level(self._h, out.ctypes.data))
        return out


class InitPicker:
    """The reference's initial picks (kmeans.cpp:141-196) from node sizes, one engine per build."""

    def __init__(self) -> None:
        self._lib = load_library()
        h = C.c_void_p()
        _check(self._lib.rbw_init_picker_create(C.byref(h)))
        self._h = h

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.rbw_init_picker_destroy(h)
            self._h = None

    def level(self, B: int, counts: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        counts = np.ascontiguousarray(counts, np.uint32)
        pos = np.empty((counts.size, B), np.uint32)
        nv = np.empty(counts.size, np.uint32)
        _check(self._lib.rbw_init_picker_level(self._h, B, counts.ctypes.data, counts.size, pos.ctypes.data,
                                               nv.ctypes.data))
        return pos, nv


def idf_weights(nb_doc: int, occ: np.ndarray) -> np.ndarray:
    """Node weights from occurrence counts (Vocabulary.cpp:103-108), as the library computes them."""
    occ = np.ascontiguousarray(occ, np.uint32).reshape(-1)
    out = np.empty(occ.size, np.float32)
    _check(load_library().rbw_idf_weights(nb_doc, occ.ctypes.data, occ.size, out.ctypes.data))
    return out


def _mask(n_valid: int) -> int:
    return 0xFFFFFFFF if n_valid >= 32 else (1 << int(n_valid)) - 1


def build_vocabulary_sharded(engine, B: int, L: int, nb_doc: int, group=None, init: str = "reference",
                             injected: Optional[np.ndarray] = None, max_iterations: int = 1000,
                             check_interval: int = 4):
    """Collective build over every rank's `engine` (ranks hold consecutive descriptor ranges, in
    rank order).  Returns (centers [levelBeg(L)][B][128] uint8, masks [levelBeg(L)] uint32,
    weights [levelBeg(L)][B] float32), identical on every rank."""
    import torch

    dist = _dist()
    rank = dist.get_rank(group)
    if init not in ("reference", "injected"):
        raise ValueError("sharded builds take the reference init or injected descriptor indices")
    if max_iterations < 1:
        raise ValueError("max_iterations must be positive")
    sizes = _all_gather_np(np.array([engine.n_local]), group)[:, 0]
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    n_total = int(offsets[-1])
    if n_total < B or nb_doc == 0:
        raise ValueError("Insufficient descriptors")  # Vocabulary.cpp:38-44
    nodes_total = _level_beg(B, L)
    if init == "injected":
        injected = np.ascontiguousarray(injected, np.uint32).reshape(nodes_total, B)
        bad = (injected != INVALID) & (injected >= n_total)
        if bad.any():
            raise ValueError("injected index out of range")
    centers_all = np.zeros((nodes_total, B, 128), np.uint8)
    masks = np.zeros(nodes_total, np.uint32)
    occ = np.zeros((nodes_total, B), np.uint32)
    picker = InitPicker() if init == "reference" else None
    check = max(1, check_interval)
    for level in range(L):
        nb = B ** level
        lb = _level_beg(B, level)
        cnt_r = _all_gather_np(engine.node_counts(), group)  # [world, nb]
        n_g = cnt_r.sum(0)
        first = np.concatenate([np.zeros((1, nb), np.int64), np.cumsum(cnt_r, 0)])  # [world + 1, nb]
        # ---- initial centers: the picked rows, contributed by the ranks that own them
        rows = np.zeros((nb, B, 128), np.int64)
        invalid = np.zeros((nb, B), bool)
        if init == "reference":
            pos, nv = picker.level(B, n_g)
            node_of = np.repeat(np.arange(nb), B).reshape(nb, B)
            # an empty node reads the first member of the next non-empty node (kmeans.cpp:179-186)
            nxt = np.full(nb, -1, np.int64)
            following = -1
            for g in range(nb - 1, -1, -1):
                nxt[g] = following
                if n_g[g] > 0:
                    following = g
            for g in np.nonzero(n_g == 0)[0]:
                if nxt[g] < 0:
                    invalid[g] = True
                else:
                    node_of[g] = nxt[g]
                    pos[g] = 0
            for g in range(nb):
                masks[lb + g] = _mask(nv[g])
            lo = first[rank][node_of]
            mine = (~invalid) & (pos >= lo) & (pos < lo + cnt_r[rank][node_of])
            if mine.any():
                got = engine.member_rows(node_of[mine].astype(np.uint32), (pos[mine] - lo[mine]).astype(np.uint32))
                rows[mine] = got
        else:
            inj = injected[lb: lb + nb]
            invalid = inj == INVALID
            for g in range(nb):
                k = 0
                for b in range(B):
                    if inj[g, b] != INVALID and b == k:
                        k += 1
                masks[lb + g] = _mask(k)
            mine = (~invalid) & (inj >= offsets[rank]) & (inj < offsets[rank + 1])
            if mine.any():
                rows[mine] = engine.desc_rows((inj[mine] - offsets[rank]).astype(np.uint32))
        rows = _all_reduce_np(rows, group)
        init_c = rows.astype(np.uint8)
        init_c[invalid] = 0xFF
        engine.set_centers(init_c)
        # ---- Lloyd steps: local assign, all-reduce, identical update everywhere
        last, sums, counts, changed = engine.buffers(nb)
        last.fill_(-1)
        for it in range(max_iterations):
            sums.zero_()
            counts.zero_()
            changed.zero_()
            engine.assign(last, sums, counts, changed)
            _all_reduce_(sums, group)
            _all_reduce_(counts, group)
            _all_reduce_(changed, group)
            engine.update(sums, counts, changed)
            last.copy_(changed)
            if ((it + 1) % check == 0 or it + 1 == max_iterations) and not bool(torch.any(changed != 0)):
                break
        centers_all[lb: lb + nb] = engine.get_centers()
        occ[lb: lb + nb] = _all_reduce_np(engine.next_level(), group).reshape(nb, B).astype(np.uint32)
    weights = idf_weights(nb_doc, occ).reshape(nodes_total, B)
    return centers_all, masks, weights


# ------------------------------------------------------------------ database
class ShardedDataBase:
    """One rank's shard of an inverted file (any object with add_doc / query(leaves, k,
    with_scores=True) / word_postings() / set_word_postings(counts), e.g. rapidbow_b200.DataBase),
    queried collectively."""

    def __init__(self, db, group=None) -> None:
        self.db = db
        self.group = group

    def add_doc(self, idx_doc: int, leaves: np.ndarray) -> None:
        self.db.add_doc(idx_doc, leaves)

    def sync(self) -> None:
        """Collective: installs the subtree posting counts summed over all shards in this shard's
        skip rule.  Call after documents were added to any shard, before querying."""
        counts = _all_reduce_np(np.asarray(self.db.word_postings(), np.uint64).astype(np.int64), self.group)
        self.db.set_word_postings(counts.astype(np.uint64))

    def query(self, leaves: np.ndarray, max_results: int) -> Tuple[np.ndarray, np.ndarray]:
        """Collective: (document ids, scores) of the max_results best documents over all shards,
        ascending by (score, document id)."""
        k = int(max_results)
        if k == 0:
            return np.zeros(0, np.uint32), np.zeros(0, np.float32)
        d, s = self.db.query(leaves, k, with_scores=True)
        docs = np.full(k, INVALID, np.int64)
        scores = np.full(k, np.inf, np.float64)
        docs[: d.size] = d
        scores[: s.size] = s
        g_docs = _all_gather_np(docs, self.group).reshape(-1)
        g_bits = _all_gather_np(scores.view(np.int64), self.group).reshape(-1).view(np.float64)
        valid = g_docs != INVALID
        order = np.lexsort((g_docs[valid], g_bits[valid]))[:k]
        return g_docs[valid][order].astype(np.uint32), g_bits[valid][order].astype(np.float32)
