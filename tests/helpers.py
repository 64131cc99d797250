"""Shared test inputs: random trees with deliberate ties, and descriptor sets with edge cases."""
import numpy as np

from oracle.pyoracle import level_beg


def random_tree(B: int, L: int, seed: int, dup_rate: float = 0.1, data=None):
    """Centers [levelBeg(L)][B][128] (random bytes, or rows of `data`), with some duplicate
    centers inside nodes so the lowest-index tie rule is exercised."""
    rng = np.random.default_rng(seed)
    nodes = level_beg(B, L)
    if data is not None:
        idx = rng.integers(0, data.shape[0], size=nodes * B)
        centers = data[idx].reshape(nodes, B, 128).copy()
    else:
        centers = rng.integers(0, 256, size=(nodes, B, 128), dtype=np.uint8)
    dup = rng.random((nodes, B)) < dup_rate
    for n, b in zip(*np.nonzero(dup)):
        if b + 1 < B:
            centers[n, b + 1] = centers[n, b]
    masks = np.full(nodes, (1 << B) - 1, dtype=np.uint32)
    weights = rng.uniform(0.01, 3.0, size=(nodes, B)).astype(np.float32)
    return centers, masks, weights


def edge_descriptors(centers: np.ndarray, n: int, seed: int, data=None) -> np.ndarray:
    """n descriptors: random bytes, copies of centers (exact ties with duplicates), all-zero,
    all-255, and (optionally) rows of `data`."""
    rng = np.random.default_rng(seed)
    out = rng.integers(0, 256, size=(n, 128), dtype=np.uint8)
    flat = centers.reshape(-1, 128)
    k = n // 4
    if k:
        out[:k] = flat[rng.integers(0, flat.shape[0], size=k)]
    if n > 8:
        out[k: k + 2] = 0
        out[k + 2: k + 4] = 255
    if data is not None and n > 16:
        m = n // 3
        out[-m:] = data[rng.integers(0, data.shape[0], size=m)]
    perm = rng.permutation(n)
    return np.ascontiguousarray(out[perm])
