"""Generates the golden fixtures in this folder by running the reference itself.

The reference library is compiled from its own sources into oracle/_ref/libref_rbow.so
(oracle/Makefile, target ``ref``).  Its vocabulary build, lookup and k-means kernels need a CUDA
device; its DataBase runs on the CPU.  Run on a GPU machine from the repository root:

    python tests/golden/make_golden.py --out tests/golden

Fixtures (numpy .npz, all inputs seeded and stored):
  voc_b16_l2.npz      reference build (default settings) of a 16-ary, 2-level tree from 2000
                      synthetic SIFT-like descriptors, and the reference lookup of 1000 queries
  lookup_b16_l3.npz   reference lookup of 1000 queries through a seeded random 16-ary, 3-level
                      tree (tests.helpers.random_tree(16, 3, seed), rebuilt by the reader)
  kmeans_task.npz     the reference's assign-center kernel (and center update) on four tasks of
                      478, 15, 39 and 134 random descriptors (the shapes of the reference's
                      KMeansAssignCenterTest.random)
  db_b16_l3.npz       the reference DataBase: 150 documents added, 24 queries at k = 10 and 50
"""
import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import Reference, centers_to_reference_nodes, level_beg  # noqa: E402
from tests.helpers import edge_descriptors, random_tree  # noqa: E402


def sift_like_np(n, seed, n_components=64):
    """Small numpy SIFT-like generator: gamma(0.5) around mixture means, L2-normalise, clip at
    0.2, renormalise, scale by 512, clamp to 255."""
    rng = np.random.default_rng(seed)
    means = rng.gamma(0.5, 1.0, size=(n_components, 128))
    comp = rng.integers(0, n_components, size=n)
    x = means[comp] * rng.gamma(0.5, 2.0, size=(n, 128))
    x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
    x = np.minimum(x, 0.2)
    x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
    return np.clip(np.rint(x * 512), 0, 255).astype(np.uint8)


def reference_blob(centers, masks, weights, L):
    nodes = centers.shape[0]
    return (np.array([L], np.uint32).tobytes() + centers_to_reference_nodes(centers).tobytes()
            + masks.astype(np.uint16).tobytes() + weights.astype(np.float32).reshape(nodes, 16).tobytes())


def to_reference_tiles(desc):
    """Descriptors [n][128] -> the reference's kmeans tiles [n/32][32 words][32 descriptors]
    (reformatDesc.cu), padded with all-ones descriptors."""
    n = desc.shape[0]
    nt = (n + 31) // 32
    w = np.full((nt * 32, 32), 0xFFFFFFFF, np.uint32)
    w[:n] = desc.view(np.uint32).reshape(n, 32)
    return np.ascontiguousarray(w.reshape(nt, 32, 32).transpose(0, 2, 1))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    ref = Reference()

    # 1. build + lookup
    train = sift_like_np(2000, seed=1)
    blob = ref.build_vocabulary(train, nb_doc=50, L=2)
    queries = np.concatenate([sift_like_np(900, seed=2), edge_descriptors(train[:256].reshape(16, 16, 128), 100, 3)])
    leaves = ref.lookup(blob, queries)
    np.savez_compressed(os.path.join(args.out, "voc_b16_l2.npz"), train=train, nb_doc=np.uint32(50),
                        blob=np.frombuffer(blob, np.uint8), queries=queries, leaves=leaves)

    # 2. lookup through a seeded random 3-level tree (duplicate centers: ties)
    seed = 1234
    centers, masks, weights = random_tree(16, 3, seed)
    q3 = edge_descriptors(centers, 1000, seed=5)
    leaves3 = ref.lookup(reference_blob(centers, masks, weights, 3), q3)
    np.savez_compressed(os.path.join(args.out, "lookup_b16_l3.npz"), tree_seed=np.uint32(seed), queries=q3,
                        leaves=leaves3)

    # 3. k-means assign / update tasks
    rng = np.random.default_rng(77)
    tasks = {}
    for t, n in enumerate((478, 15, 39, 134)):
        desc = rng.integers(0, 256, size=(n, 128), dtype=np.uint8)
        cidx = np.minimum(np.arange(16), n - 1)
        centers_t = desc[cidx]
        prev = rng.integers(0, 16, size=n, dtype=np.uint8)
        tiles = to_reference_tiles(desc)
        assign_in = np.zeros(tiles.shape[0] * 32, np.uint8)
        assign_in[:n] = prev
        cw = centers_to_reference_nodes(centers_t[None])[0].view(np.uint32)
        _, assign, counts, sums, changed = ref.kmeans_task(tiles, n, cw, assign_in, do_update=False)
        new_cw = ref.kmeans_task(tiles, n, cw, assign_in, do_update=True)[0]
        new_centers = (np.frombuffer(new_cw.tobytes(), np.uint8).reshape(32, 16, 4)
                       .transpose(1, 0, 2).reshape(16, 128))
        tasks.update({f"t{t}_desc": desc, f"t{t}_centers": centers_t, f"t{t}_prev": prev,
                      f"t{t}_assign": assign[:n], f"t{t}_counts": counts, f"t{t}_sums": sums.reshape(128, 16).T.copy(),
                      f"t{t}_changed": np.uint32(changed), f"t{t}_updated": new_centers})
    np.savez_compressed(os.path.join(args.out, "kmeans_task.npz"), **tasks)

    # 4. DataBase
    rng = np.random.default_rng(99)
    n_leaves = 16 ** 3
    _, _, w = random_tree(16, 3, 4321)
    pop = 1.0 / np.arange(1, n_leaves + 1) ** 0.8
    pop = pop[rng.permutation(n_leaves)]
    pop /= pop.sum()
    docs = [rng.choice(n_leaves, size=int(s), p=pop).astype(np.uint32)
            for s in np.exp(rng.uniform(np.log(10), np.log(300), 150))]
    ids = (rng.permutation(150) * 7 + 3).astype(np.uint32)
    rdb = ref.db(3, w)
    for i, d in zip(ids, docs):
        rdb.add(int(i), d)
    queries_db = []
    for j in range(24):
        base = docs[int(rng.integers(0, 150))]
        q = np.concatenate([base[rng.random(base.size) < 0.6],
                            rng.integers(0, n_leaves, size=base.size // 3 + 1, dtype=np.uint32)]).astype(np.uint32)
        queries_db.append(q)
    out = {"weights": w, "doc_ids": ids, "doc_leaves": np.concatenate(docs),
           "doc_offsets": np.concatenate([[0], np.cumsum([d.size for d in docs])]).astype(np.uint64),
           "query_leaves": np.concatenate(queries_db),
           "query_offsets": np.concatenate([[0], np.cumsum([q.size for q in queries_db])]).astype(np.uint64)}
    for k in (10, 50):
        res = np.full((len(queries_db), k), 0xFFFFFFFF, np.uint32)
        cnt = np.zeros(len(queries_db), np.uint32)
        for j, q in enumerate(queries_db):
            r = rdb.query(q, k)
            res[j, : r.size] = r
            cnt[j] = r.size
        out[f"k{k}_results"] = res
        out[f"k{k}_counts"] = cnt
    np.savez_compressed(os.path.join(args.out, "db_b16_l3.npz"), **out)
    print("golden fixtures written to", args.out)


if __name__ == "__main__":
    main()
