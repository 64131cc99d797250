"""The k-means++ kernel (kmeansPPKernel in rapidbow_b200/csrc/kmeans.cu) makes Floyd's sampling
draws in parallel: thread m draws t_m = out_m mod (j_m + 1) from the counter-based SplitMix64
stream, and whether
step m inserts j_m (t_m already taken) follows from the draws alone, except for t_m = j_r with
r < m, where it also depends on step r: found_m = local_m or found_r, resolved by eight rounds of
pointer jumping.  This restates that formulation in Python and checks it against the sequential
algorithm of the oracle (orc_kmeanspp_init) on many streams, including node sizes just above the
256-member sample, where the j_r case is most frequent.  The GPU parity tests pin the kernel
itself against the oracle's builds."""
import random

import pytest

M64 = (1 << 64) - 1
GAMMA = 0x9E3779B97F4A7C15
S = 256


def _out(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def _sequential(n, s):
    pos = []
    for j in range(n - S, n):
        s = (s + GAMMA) & M64
        t = _out(s) % (j + 1)
        pos.append(j if t in pos else t)
    return sorted(pos), s


def _parallel(n, s0):
    base = n - S
    t = [_out((s0 + (m + 1) * GAMMA) & M64) % (base + m + 1) for m in range(S)]
    found, link = [False] * S, [-1] * S
    for m in range(S):
        q0 = 0
        if t[m] >= base:
            r = t[m] - base
            q0 = min(r, m)
            if r < m:
                link[m] = r
        found[m] = any(t[q] == t[m] for q in range(q0, m))
    for _ in range(8):
        nf, nl = found[:], link[:]
        for m in range(S):
            if link[m] >= 0:
                nf[m] = found[m] or found[link[m]]
                nl[m] = link[link[m]]
        found, link = nf, nl
    pos = [base + m if found[m] else t[m] for m in range(S)]
    assert len(set(pos)) == S
    return sorted(pos), (s0 + S * GAMMA) & M64


@pytest.mark.parametrize("seed", range(4))
def test_parallel_floyd_equals_sequential(seed):
    rng = random.Random(seed)
    sizes = [257, 258, 260, 300, 384, 511, 512, 1000, 4096, 10 ** 6] + [rng.randint(257, 3000) for _ in range(30)]
    for n in sizes:
        s0 = rng.getrandbits(64)
        assert _parallel(n, s0) == _sequential(n, s0), (n, s0)
