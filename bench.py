#!/usr/bin/env python
"""Headline benchmark: vocabulary-tree lookup of 10M fresh SIFT-like descriptors through a
65,536-word tree (branching 16, depth 4) trained on 2M descriptors, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one lookup of the rank's 10M descriptors (inputs resident in HBM, 1.28 GB > L2, so
no flush is needed).  N > 1 runs one process per GPU (torchrun) with the tree replicated and
10M descriptors per rank (weak scaling, no collective on the data path).  Rank 0 prints one
JSON line (the headline).  On one GPU the other workloads follow, one line each, prefixed with
"# <name> " so that the headline stays the only JSON line: the vocabulary builds (200,000
descriptors B=16 L=3; 10M descriptors B=10 L=6), batched inverted-file scoring (20,000 images)
and serving (100,000 images, Poisson arrivals).  The reference has no CPU lookup;
`--impl reference` times the CPU restatement of its kernel (the oracle, all host threads) on the
same workload shape.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "tree-lookup desc/s (65,536 words, bit-exact IDs): split-BF16 vs FP32, 1×B200"
UNIT = "desc/s"
B, L = 16, 4
N_TRAIN = 2_000_000
N_LOOKUP = 10_000_000
BYTES_PER_DESC = 132  # 128 B read + 4 B leaf written (algorithmic, per descriptor per pass)
# DRAM bytes per descriptor of one lookupPassTc launch: dram__bytes_read.sum + dram__bytes_write.sum
# of an ncu capture of a 2M-descriptor lookup (B=16, L=4; both pass launches averaged).  Traffic
# grows in proportion to the descriptors, so it is scaled to the timed launch.
LOOKUP_PASS_DRAM_BYTES_PER_DESC = 136.6
# DRAM bytes of one scoring launch (queryPrepKernel + scoreKernel: 2.6 MB + 1.388 GB read,
# 3.9 MB written) on the seeded 20,000-image database with 256 queries, top-50, from an ncu
# capture of that workload.
SCORE_DRAM_BYTES_20K_IMAGES = 1_394_930_000
WORKLOAD = ("lookup of 10M fresh SIFT-like descriptors per GPU through a 65,536-word tree "
            "(B=16, L=4) trained on 2M descriptors (k-means++ init, 10 Lloyd iterations)")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=N_LOOKUP)
    p.add_argument("--algo", default="auto", choices=["auto", "tensor_u8", "tensor_u8_warpnode", "tensor_u8_ring"],
                   help="tensor-core lookup variant of the timed steps (auto = the library's default)")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-scoring", action="store_true", help="skip the inverted-file scoring workload")
    p.add_argument("--db-docs", type=int, default=20000, help="images in the scoring database")
    p.add_argument("--no-build", action="store_true", help="skip the vocabulary-build workloads")
    p.add_argument("--no-serving", action="store_true",
                   help="skip the serving workload (1M-word tree, 100,000 images, Poisson arrivals)")
    p.add_argument("--no-ref-gpu", action="store_true", help="skip the reference's own GPU lookup kernel")
    p.add_argument("--no-tune", action="store_true", help="skip autotuning (built-in launch parameters)")
    p.add_argument("--serving-docs", type=int, default=100_000)
    p.add_argument("--serving-rate", type=float, default=2000.0, help="arrivals per second")
    p.add_argument("--serving-seconds", type=float, default=5.0)
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()

    def summary(self):
        rows = []
        try:
            with open(self.file.name) as fh:
                for line in fh:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def allreduce_max(world, x: float) -> float:
    """Max over ranks (timings are reported as the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(n_threads: int, target_s: float, seed: int = 4242):
    """Times the oracle (CPU restatement of vocTreeLookUp.cu, integer distances) with
    n_threads host threads on a bounded sample of the same workload shape."""
    import numpy as np

    from oracle.pyoracle import Oracle
    from rapidbow_b200.synth import sift_like
    from oracle.pyoracle import level_beg

    global _CPU_POOL
    orc = Oracle()
    if _CPU_POOL is None:
        rng = np.random.default_rng(seed)
        pool = sift_like(131_072, seed=seed).numpy()
        nodes = level_beg(B, L)
        centers = pool[rng.integers(0, pool.shape[0], size=nodes * B)].reshape(nodes, B, 128)
        # 2M-descriptor sample: the generated pool tiled (work per descriptor is data-independent)
        _CPU_POOL = (centers, np.ascontiguousarray(np.tile(pool, (16, 1))))
    centers, sample = _CPU_POOL
    done, t0 = 0, time.perf_counter()
    while True:
        orc.lookup(centers, B, L, sample, threads=n_threads)
        done += sample.shape[0]
        dt = time.perf_counter() - t0
        if dt >= target_s:
            break
    return done / dt, done, dt


_CPU_POOL = None


def run_reference(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    vals = []
    n_last = 0
    for _ in range(max(args.warmup, 0)):
        cpu_baseline(threads, min(args.cpu_seconds, 3.0) / 4)
    for _ in range(args.steps):
        v, n, _ = cpu_baseline(threads, args.cpu_seconds / max(args.steps, 1))
        vals.append(v)
        n_last = n
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": n_last / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD, "note": "the reference has no CPU lookup; its kernel restated on CPU "
                   "(oracle, exact integer distances) on a bounded sample per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n_last} descriptors per step through a B=16 L=4 tree"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import rapidbow_b200 as rbw
    from rapidbow_b200.synth import sift_like

    dev = torch.device("cuda", local)
    n = args.n
    train = sift_like(N_TRAIN, seed=1, device=dev)
    voc = rbw.build_vocabulary(train, B, nb_doc=1000, nb_levels=L, init="kmeans++", seed=7, max_iterations=10)
    del train
    desc = sift_like(n, seed=1000 + rank, device=dev)
    out = torch.empty(n, dtype=torch.int32, device=dev)
    ref32 = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(algo, steps, warmup, kernel_name=None):
        for _ in range(warmup):
            voc.lookup(desc, out if algo != "simt_f32" else ref32, algo=algo)
        torch.cuda.synchronize(dev)
        barrier(world)
        torch.cuda.synchronize(dev)
        if kernel_name:
            rbw.timing_reset()
            rbw.timing_enable(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        e0.record(stream)
        for _ in range(steps):
            voc.lookup(desc, out if algo != "simt_f32" else ref32, algo=algo)
            launches += voc.last_kernels
        e1.record(stream)
        torch.cuda.synchronize(dev)
        rbw.timing_enable(False)
        barrier(world)
        ms = e0.elapsed_time(e1) / steps
        kern = None
        if kernel_name:
            kern = rbw.timing_read(kernel_name)
            timed.regroup = rbw.timing_read("lookup_regroup")
        return allreduce_max(world, ms), launches, kern

    # autotuning (before the timed region): the tensor-core schedule of algo "auto", on this lookup
    tuned = None
    if not args.no_tune:
        from rapidbow_b200.autotune import Autotuner

        e = Autotuner.for_current_device().tune_lookup(voc, desc)
        tuned = {"param": "lookup_schedule", "value": e["value"], "default": 1, "tuned_ms": e["ms"],
                 "default_ms": e["default_ms"], "candidates_ms": e["candidates"],
                 "kernel": "tensor-core pass (1 = level pairs in two buffers, 2 = three-slot ring), per launch"}
    with ClockSampler(local) as clocks:
        ms, launches, (k_ms, k_n) = timed(args.algo, args.steps, args.warmup, "lookup_pass_tc")
    regroup_ms, regroup_n = timed.regroup
    clk = clocks.summary()
    ms_simt, _, (s_ms, s_n) = timed("simt_f32", max(3, args.steps // 4), 2, "lookup_simt_f32")
    # exactness on the bench data: tensor-core IDs == FP32 kernel IDs
    same = bool(torch.equal(out, ref32))
    code, where = voc.device_errors()

    value = world * n / (ms / 1e3)
    fp32_value = world * n / (ms_simt / 1e3)
    ring = args.algo == "tensor_u8_ring" or (args.algo == "auto" and tuned is not None and tuned["value"] == 2)
    pass_kernel = "lookupPassRing" if ring else "lookupPassTc"
    hbm_peak, peak_kind = peaks()
    k_avg_ms = k_ms / max(k_n, 1)
    achieved = n * BYTES_PER_DESC / (k_avg_ms / 1e3) / 1e9
    traffic = LOOKUP_PASS_DRAM_BYTES_PER_DESC * n

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD, "descriptors_per_gpu": n, "branching": B, "levels": L,
                   "parallelism": f"dp{world} (tree replicated, descriptors sharded)",
                   "l2": "inputs 1.28 GB per GPU > 126 MB L2, no flush needed", "algo": args.algo},
        "gpu_launches": launches,
        "bit_exact_vs_fp32_kernel": same,
        "refined_descriptors": 0,
        "fp32_simt": {"value": fp32_value, "unit": UNIT, "ms_per_step": ms_simt,
                      "speedup": value / fp32_value, "kernel": "lookupSimtF32"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_kind,
                     "kernel": pass_kernel, "launch_ms": k_avg_ms, "launches_per_step": k_n / args.steps,
                     "algorithmic_bytes_per_launch": n * BYTES_PER_DESC},
        "whole_lookup_hbm_frac": (n * BYTES_PER_DESC / (ms / 1e3) / 1e9) / hbm_peak,
        "regroup": {"ms_per_step": regroup_ms / args.steps, "regroups_per_step": regroup_n / args.steps,
                    "kernels": "regroupHist + regroupScan + buildTiles + regroupScatter",
                    "algorithmic_bytes": 8 * n,
                    "achieved_gbs": 8 * n / (regroup_ms / max(regroup_n, 1) / 1e3) / 1e9 if regroup_n else None},
        "clocks": clk,
        "device_errors": [code, where],
    }
    if tuned is not None:
        line["autotune"] = tuned

    if rank == 0 and world == 1 and not args.no_ref_gpu:
        line["ref_gpu_kernel"] = ref_gpu_lookup(voc, desc, out, value)

    if not args.no_e2e:
        # end to end through the C ABI: pinned host in, pinned host out, every step.
        host_desc = torch.empty((n, 128), dtype=torch.uint8, pin_memory=True)
        host_desc.copy_(desc)
        host_out = torch.empty(n, dtype=torch.int32, pin_memory=True)
        e_steps = max(3, min(args.steps, 10))
        voc.lookup_host_ptr(host_desc.data_ptr(), n, host_out.data_ptr())
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(e_steps):
            voc.lookup_host_ptr(host_desc.data_ptr(), n, host_out.data_ptr())
        e_s = allreduce_max(world, (time.perf_counter() - t0) / e_steps)
        same_e2e = bool(torch.equal(host_out, out.cpu()))
        line["e2e"] = {"value": world * n / e_s, "unit": UNIT, "h2d_bytes_per_step": n * 128,
                       "d2h_bytes_per_step": n * 4, "ms_per_step": e_s * 1e3, "steps": e_steps,
                       "timer": "host wall clock around the synchronous C-ABI call", "matches_device": same_e2e}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, sn, dt = cpu_baseline(threads, args.cpu_seconds)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{sn} descriptors through a B=16 L=4 tree in {dt:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        return  # the other workloads are single-GPU workloads
    del desc, out, ref32
    torch.cuda.empty_cache()
    if not args.no_build:
        for name, res in build_bench(args, dev, rank).items():
            sub_line(name, res)
    if not args.no_scoring:
        sub_line("scoring", scoring_bench(args, voc, dev, world, rank))
    if not args.no_serving:
        del voc
        torch.cuda.empty_cache()
        sub_line("serving", serving_bench(args, dev, rank))


def sub_line(name, res):
    """One line per further workload after the headline, prefixed so that it does not parse as
    the headline JSON."""
    print(f"# {name} " + json.dumps(res), flush=True)


def ref_gpu_build(host_desc):
    """The reference's own GPU build (buildVocabulary: kernel_kmeansAssignCenter and
    kernel_kmeansUpdateCenters, compiled for sm_100a from its sources into oracle/_ref) of the same
    200,000 descriptors into a B=16, L=3 tree, capped at 10 Lloyd iterations with its own random
    init and convergence poll every 4 iterations: median host wall time of 3 builds (the
    descriptors are copied in inside each call, about 26 MB)."""
    from oracle.pyoracle import Reference

    if not Reference.available():
        return {"unavailable": "reference library not built"}
    ref = Reference()
    ref.build_vocabulary(host_desc, 1000, 3, max_iter=10, check_interval=4)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        ref.build_vocabulary(host_desc, 1000, 3, max_iter=10, check_interval=4)
        times.append(time.perf_counter() - t0)
    return {"value": statistics.median(times), "unit": "s", "higher_is_better": False,
            "note": "reference init (random distinct picks), not k-means++; includes its 26 MB copy in"}


def ref_gpu_lookup(voc, desc, ours, ours_value):
    """The reference's own lookup kernel (kernel_VocTreeLookUp through IVocabulary::lookUp,
    compiled for sm_100a from its sources into oracle/_ref) on the same descriptors and tree:
    device time per launch from CUDA events, and whether its leaf IDs equal ours."""
    import numpy as np

    from oracle.pyoracle import Reference

    if not Reference.available() or voc.branch_factor != 16:
        return {"unavailable": "reference library not built or tree not 16-ary"}
    ref = Reference()
    host = desc.cpu().numpy()
    got, ms = ref.lookup_device_timed(voc.serialize(), host, iters=5)
    same = bool(np.array_equal(got, ours.cpu().numpy().view(np.uint32)))
    n = host.shape[0]
    return {"value": n / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "speedup": ours_value / (n / (ms / 1e3)),
            "kernel": "kernel_VocTreeLookUp (reference, dp4a SIMT, sm_100a)", "identical_leaf_ids": same}


SCORING_WORKLOAD = ("inverted-file retrieval: 20,000 images of log-uniform 500-4,000 SIFT-like descriptors "
                    "quantised on the 65,536-word tree; one batched launch scores 256 query images of uneven "
                    "size (half share 60% of their words with a database image), top-50 by L1 tf-idf score")


def scoring_bench(args, voc, dev, world, rank):
    """Device-resident DataBase: index build, then batches of 256 queries (top-50) scored in one
    launch, timed with CUDA events; the reference's own CPU DataBase timed on the same queries."""
    import numpy as np
    import torch

    import rapidbow_b200 as rbw
    from rapidbow_b200.synth import sift_like

    n_docs, nq, k = args.db_docs, 256, 50
    rng = np.random.default_rng(2024 + rank)
    sizes = np.exp(rng.uniform(np.log(500), np.log(4000), n_docs)).astype(np.int64)
    qsizes = np.exp(rng.uniform(np.log(500), np.log(4000), nq)).astype(np.int64)

    def quantise(total, seed0):
        leaves = torch.empty(total, dtype=torch.int32, device=dev)
        chunk = 1 << 22
        for i, beg in enumerate(range(0, total, chunk)):
            m = min(chunk, total - beg)
            voc.lookup(sift_like(m, seed=seed0 + i, device=dev), leaves[beg: beg + m])
        return leaves.cpu().numpy().view(np.uint32)

    doc_leaves = quantise(int(sizes.sum()), 50_000)
    fresh = quantise(int(qsizes.sum()), 90_000)
    torch.cuda.empty_cache()
    offs = np.zeros(n_docs + 1, np.uint64)
    offs[1:] = np.cumsum(sizes)
    queries, pos = [], 0
    for j, s in enumerate(qsizes):
        f = fresh[pos: pos + s]
        pos += s
        if j % 2 == 0:
            d = int(rng.integers(0, n_docs))
            base = doc_leaves[int(offs[d]): int(offs[d + 1])]
            m = min(base.size, int(0.6 * s))
            f = np.concatenate([rng.choice(base, m, replace=False), f[: s - m]])
        queries.append(f.astype(np.uint32))
    q_off = np.zeros(nq + 1, np.int64)
    q_off[1:] = np.cumsum([q.size for q in queries])
    q_host = torch.from_numpy(np.concatenate(queries).view(np.int32)).pin_memory()
    q_leaves = q_host.to(dev)
    q_offsets = torch.from_numpy(q_off).to(dev)

    db = rbw.DataBase(voc)
    ids = np.arange(n_docs, dtype=np.uint32)
    db.add_docs(ids, doc_leaves, offs)
    stream = torch.cuda.current_stream(dev)
    rbw.timing_reset()
    rbw.timing_enable(True)
    t0 = time.perf_counter()
    db.query_batched(q_leaves, q_offsets, k)  # brings the index up to date first
    torch.cuda.synchronize(dev)
    first_s = time.perf_counter() - t0
    rbw.timing_enable(False)
    index_ms, _ = rbw.timing_read("index")
    for _ in range(args.warmup):
        db.query_batched(q_leaves, q_offsets, k)
    torch.cuda.synchronize(dev)
    barrier(world)
    rbw.timing_reset()
    rbw.timing_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        docs, scores, counts = db.query_batched(q_leaves, q_offsets, k)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    rbw.timing_enable(False)
    ms = allreduce_max(world, e0.elapsed_time(e1) / args.steps)
    score_ms, score_n = rbw.timing_read("score")
    kern_ms = score_ms / max(score_n, 1)

    # algorithmic bytes: every (document, entry) pair of every leaf word of every query, 8 B
    # (4 B document + 4 B tf-derived entry); the accumulators stay on chip, and non-leaf levels
    # are skipped at this database size
    pair_cnt = np.zeros(voc.branch_factor ** voc.nb_levels, np.int64)
    doc_of = np.repeat(ids, sizes)
    uniq = np.unique(doc_of.astype(np.uint64) << np.uint64(32) | doc_leaves.astype(np.uint64))
    np.add.at(pair_cnt, (uniq & np.uint64(0xFFFFFFFF)).astype(np.int64), 1)
    pairs_read = int(sum(pair_cnt[np.unique(q)].sum() for q in queries))
    alg_bytes = pairs_read * 8
    hbm_peak, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9

    # end to end: pinned host query leaves in, results out, every batch
    e_steps = max(3, min(args.steps, 10))
    out_docs = torch.empty((nq, k), dtype=torch.int32, pin_memory=True)
    out_cnt = torch.empty(nq, dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(e_steps):
        ql = q_host.to(dev, non_blocking=True)
        d_, _, c_ = db.query_batched(ql, q_offsets, k)
        out_docs.copy_(d_, non_blocking=True)
        out_cnt.copy_(c_, non_blocking=True)
        torch.cuda.synchronize(dev)
    e_s = allreduce_max(world, (time.perf_counter() - t0) / e_steps)

    res = {
        "workload": SCORING_WORKLOAD, "docs": n_docs, "postings": int(sizes.sum()), "queries_per_batch": nq,
        "top_k": k, "value": world * nq / (ms / 1e3), "unit": "queries/s", "ms_per_batch": ms,
        "index_build_ms": index_ms, "first_batch_wall_ms": first_s * 1e3,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": score_traffic(n_docs), "peak_source": peak_kind,
                     "kernel": "queryPrepKernel + scoreKernel", "launch_ms": kern_ms,
                     "algorithmic_bytes_per_launch": alg_bytes, "posting_pairs_read": pairs_read},
        "e2e": {"value": world * nq / e_s, "unit": "queries/s", "h2d_bytes_per_step": int(q_host.numel()) * 4,
                "d2h_bytes_per_step": nq * k * 4 + nq * 4, "ms_per_step": e_s * 1e3, "steps": e_steps},
    }

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res["cpu_baseline"], res["parity_vs_cpu"] = scoring_cpu_baseline(
            voc, ids, doc_leaves, offs, queries, k, docs.cpu().numpy().view(np.uint32), counts.cpu().numpy(),
            args.cpu_seconds)
    return res


def build_bench(args, dev, rank):
    """Hierarchical k-means builds: 200,000 descriptors into a B=16, L=3 tree with a CPU
    baseline and an exactness check against the oracle, and 10M descriptors from a
    4,096-component Zipf(1.1) mixture into a B=10, L=6 tree.  Both: seeded k-means++ init, 10 Lloyd
    iterations.  The build API is synchronous; times are host wall clock around it."""
    import numpy as np
    import torch

    import rapidbow_b200 as rbw
    from oracle.pyoracle import INIT_KMEANSPP, Oracle
    from rapidbow_b200.synth import sift_like

    def timed_build(desc, B, L, reps, **kw):
        """Median wall time of `reps` builds (after one warm-up), then one more build with the
        per-kernel events on; returns (vocabulary, seconds, assign ms, update ms of that build)."""
        rbw.build_vocabulary(desc, B, nb_doc=1000, nb_levels=L, init="kmeans++", seed=7, max_iterations=10, **kw)
        times, built = [], []
        for _ in range(reps):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            built.append(rbw.build_vocabulary(desc, B, nb_doc=1000, nb_levels=L, init="kmeans++", seed=7,
                                              max_iterations=10, **kw))
            torch.cuda.synchronize(dev)
            times.append(time.perf_counter() - t0)
        built.clear()  # the vocabularies are freed outside the timed builds
        rbw.timing_reset()
        rbw.timing_enable(True)
        voc = rbw.build_vocabulary(desc, B, nb_doc=1000, nb_levels=L, init="kmeans++", seed=7, max_iterations=10,
                                   **kw)
        torch.cuda.synchronize(dev)
        rbw.timing_enable(False)
        a_ms, _ = rbw.timing_read("kmeans_assign")
        u_ms, _ = rbw.timing_read("kmeans_update")
        return voc, statistics.median(times), a_ms, u_ms

    out = {}
    c0 = sift_like(200_000, seed=11, device=dev)
    voc0, s0, assign_ms, update_ms = timed_build(c0, 16, 3, 5)
    out["b16_l3_200k"] = {
        "workload": "build: 200,000 SIFT-like descriptors, B=16, L=3 (4,096 words), k-means++ init, 10 Lloyd iterations",
        "value": s0, "unit": "s", "higher_is_better": False,
        # wall time without per-kernel events; kernel times from one further build with them on
        "assign_kernel_ms_per_build": assign_ms, "update_kernel_ms_per_build": update_ms,
    }
    if rank == 0 and not args.no_cpu_baseline:
        # exactness: the GPU build with IEEE center rounding equals the oracle's build
        host = c0.cpu().numpy()
        voc_ieee = rbw.build_vocabulary(c0, 16, nb_doc=1000, nb_levels=3, init="kmeans++", seed=7, max_iterations=10,
                                        ieee_division=True)
        t0 = time.perf_counter()
        ref = Oracle().build_vocabulary(host, 1000, 16, 3, max_iter=10, init=INIT_KMEANSPP, seed=7)
        cpu_s = time.perf_counter() - t0
        centers, masks, weights = voc_ieee.tree()
        out["b16_l3_200k"]["matches_oracle"] = bool(np.array_equal(centers, ref["centers"]) and
                                                    np.array_equal(masks, ref["masks"]))
        out["b16_l3_200k"]["cpu_baseline"] = {"value": cpu_s, "unit": "s", "cores": 1, "kind": "port",
                                              "sample": "the same build (oracle restatement, one thread)"}
        out["b16_l3_200k"]["ref_gpu_build"] = ref_gpu_build(host)
    del c0
    torch.cuda.empty_cache()
    c2 = sift_like(10_000_000, seed=2, n_components=4096, zipf=1.1, device=dev)
    wl2 = ("10M SIFT-like descriptors (4,096-component mixture, Zipf(1.1) weights), B=10, L=6 (1M words), "
           "k-means++ init, 10 Lloyd iterations")
    for key, fl in (("b10_l6_10m", False), ("b10_l6_10m_float", True)):
        tune = None
        if not args.no_tune:
            from rapidbow_b200.autotune import Autotuner

            e = Autotuner.for_current_device().tune_build(c2, 10, 6, float_centers=fl, repeats=1, nb_doc=1000,
                                                          init="kmeans++", seed=7, max_iterations=10)
            tune = {"param": e["param"], "value": e["value"], "tuned_assign_ms": e["ms"],
                    "default_assign_ms": e["default_ms"]}
            if "sums" in e:
                tune["sums"] = {"value": e["sums"]["value"], "candidates_ms": e["sums"]["candidates"],
                                "note": "1 = shared-memory atomics, 2 = a second MMA per tile"}
        voc2, s2, a_ms, u_ms = timed_build(c2, 10, 6, 3, float_centers=fl)
        res = {"workload": ("build (float centers: split-bf16 distances, FP64 re-score, FP64 inertia): " if fl
                            else "build (uint8 centers): ") + wl2,
               "value": s2, "unit": "s", "higher_is_better": False,
               "assign_kernel_ms_per_build": a_ms, "update_kernel_ms_per_build": u_ms,
               "note": "the reference supports B=16 only and cannot run this configuration",
               "build_call_s_last": voc2.build_stats()["seconds"]}
        if fl:
            st = voc2.build_stats()
            res["refined_descriptors"] = int(sum(st["refined"]))
            res["assignments"] = int(sum(st["assignments"]))
            res["inertia_first_last_by_level"] = [[a, b] for a, b in zip(st["inertia_first"], st["inertia_last"])]
        if tune:
            res["autotune"] = tune
        out[key] = res
        del voc2
    del c2
    torch.cuda.empty_cache()
    if rank == 0 and not args.no_cpu_baseline:
        out["b10_l4_1m_float_vs_fp64_oracle"] = float_build_check(dev)
    return out


def float_build_check(dev):
    """The float-center build against the FP64 oracle on 1M descriptors of the same generator
    (B=10, L=4, k-means++ init, 10 Lloyd iterations): maximum relative center error, identical
    occurrence counts (assignments), refined descriptors, and the oracle's time on all host
    threads."""
    import numpy as np
    import torch

    import rapidbow_b200 as rbw
    from oracle.pyoracle import INIT_KMEANSPP, Oracle
    from rapidbow_b200.synth import sift_like

    d = sift_like(1_000_000, seed=12, n_components=4096, zipf=1.1, device=dev)
    voc = rbw.build_vocabulary(d, 10, nb_doc=1000, nb_levels=4, init="kmeans++", seed=7, max_iterations=10,
                               float_centers=True)
    host = d.cpu().numpy()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = Oracle().build_vocabulary_f32(host, 1000, 10, 4, max_iter=10, init=INIT_KMEANSPP, seed=7, threads=threads)
    cpu_s = time.perf_counter() - t0
    got = voc.centers_f32().astype(np.float64)
    want = ref["centers"].astype(np.float64)
    rel = float(np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-30)))
    st = voc.build_stats()
    leaves = voc.lookup(d).cpu().numpy().view(np.uint32)
    return {"workload": "1M descriptors of the 4,096-component Zipf(1.1) generator, B=10, L=4, k-means++, 10 iterations",
            "max_relative_center_error": rel, "centers_bit_identical": bool(np.array_equal(got, want)),
            "identical_occurrences": bool(np.array_equal(voc.tree()[2], ref["weights"])),
            "word_ids_equal_fp64_lookup": bool(np.array_equal(leaves, Oracle().lookup_f32(ref["centers"], 10, 4, host,
                                                                                          threads=threads))),
            "refined_descriptors": int(sum(st["refined"])), "assignments": int(sum(st["assignments"])),
            "cpu_baseline": {"value": cpu_s, "unit": "s", "cores": threads, "kind": "port",
                             "sample": "the same build (FP64 oracle)"}}


SERVING_WORKLOAD = ("serving: 1M-word tree (B=10, L=6) trained on 10M SIFT-like descriptors from a 4,096-component "
                    "mixture with Zipf(1.1) weights (k-means++ init, 10 Lloyd iterations); device-resident database of "
                    "100,000 images of log-uniform 300-8,000 descriptors; query images of log-uniform 300-8,000 "
                    "descriptors arrive as a Poisson stream; lookup + scoring, top-100, continuous batching")


def serving_bench(args, dev, rank):
    """Build (B=10, L=6) timed, then a Poisson request stream through rapidbow_b200.Server.
    Database images are drawn from the leaf distribution of 8M looked-up descriptors (the
    posting-list shape of real lookups without generating 234M descriptors); query images are
    slices of a pool of fresh descriptors and go through the server's lookup."""
    import threading

    import numpy as np
    import torch

    import rapidbow_b200 as rbw
    from rapidbow_b200.synth import sift_like

    rng = np.random.default_rng(77 + rank)
    train = sift_like(10_000_000, seed=2, n_components=4096, zipf=1.1, device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    voc = rbw.build_vocabulary(train, 10, nb_doc=args.serving_docs, nb_levels=6, init="kmeans++", seed=11,
                               max_iterations=10)
    torch.cuda.synchronize(dev)
    build_s = time.perf_counter() - t0
    del train
    pool = sift_like(8_000_000, seed=3, n_components=4096, zipf=1.1, device=dev)
    leaf_pool = voc.lookup(pool).cpu().numpy().view(np.uint32)
    del pool
    sizes = np.exp(rng.uniform(np.log(300), np.log(8000), args.serving_docs)).astype(np.int64)
    doc_leaves = leaf_pool[rng.integers(0, leaf_pool.size, int(sizes.sum()))]
    offs = np.zeros(args.serving_docs + 1, np.uint64)
    offs[1:] = np.cumsum(sizes)
    db = rbw.DataBase(voc)
    db.add_docs(np.arange(args.serving_docs, dtype=np.uint32), doc_leaves, offs)
    del doc_leaves
    qpool = sift_like(4_000_000, seed=4, n_components=4096, zipf=1.1, device=dev).cpu().numpy()
    torch.cuda.empty_cache()
    srv = rbw.Server(voc, db, max_results=100)
    # warm-up (also builds the index): a few requests alone, then 0.25 s of the same Poisson
    # stream, so that buffers of every size the run will use exist before the timed region
    for _ in range(3):
        srv.wait(srv.submit(qpool[:2000]))
    warm_n = int(args.serving_rate * 0.25)
    warm_gaps = rng.exponential(1.0 / args.serving_rate, warm_n)
    warm_sizes = np.exp(rng.uniform(np.log(300), np.log(8000), warm_n)).astype(np.int64)
    warm_ids = []
    t_next = time.perf_counter()
    for i in range(warm_n):
        t_next += warm_gaps[i]
        while time.perf_counter() < t_next:
            pass
        warm_ids.append(srv.submit(qpool[i * 97 % (qpool.shape[0] - 8000):][: warm_sizes[i]]))
    for i in warm_ids:
        srv.wait(i)
    srv.reset_stats()

    def stream(seconds, timing):
        """A Poisson stream of `seconds`; returns (requests, elapsed s, sizes, server stats)."""
        n_req = int(args.serving_rate * seconds)
        gaps = rng.exponential(1.0 / args.serving_rate, n_req)
        qs = np.exp(rng.uniform(np.log(300), np.log(8000), n_req)).astype(np.int64)
        starts = rng.integers(0, qpool.shape[0] - 8000, n_req)
        ids = [0] * n_req

        def collector():
            for i in range(n_req):
                while ids[i] == 0:
                    time.sleep(0.0001)
                srv.wait(ids[i])

        col = threading.Thread(target=collector)
        srv.reset_stats()
        if timing:
            rbw.timing_reset()
            rbw.timing_enable(True)
        col.start()
        t_begin = time.perf_counter()
        t_next = t_begin
        for i in range(n_req):
            t_next += gaps[i]
            ahead = t_next - time.perf_counter()
            if ahead > 0.001:
                time.sleep(ahead - 0.0005)
            while time.perf_counter() < t_next:
                pass
            ids[i] = srv.submit(qpool[starts[i]: starts[i] + qs[i]])
        col.join()
        elapsed = time.perf_counter() - t_begin
        torch.cuda.synchronize(dev)
        rbw.timing_enable(False)
        return n_req, elapsed, qs, srv.stats()

    # latency and rate without per-kernel events; then one second with them for the kernel spans
    n_req, elapsed, qs, st = stream(args.serving_seconds, False)
    stream(1.0, True)
    kernels = {}
    for name in ("lookup_pass_tc", "lookup_regroup", "score"):
        ms, n = rbw.timing_read(name)
        kernels[name] = {"launches": n, "total_ms": ms, "mean_ms": ms / max(n, 1)}
    srv.close()
    return {"workload": SERVING_WORKLOAD, "build_s": build_s, "requests": n_req,
            "offered_rate_qps": args.serving_rate, "value": n_req / elapsed, "unit": "queries/s",
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
            "mean_batch_requests": st["mean_batch_requests"], "batches": st["batches"],
            "max_inflight_batches_seen": st["max_inflight_seen"], "descriptors_per_request_mean": float(qs.mean()),
            "latency_stages_ms": {k: st[k] for k in ("queue_p99_ms", "launch_p99_ms", "device_p99_ms", "queue_max_ms",
                                                      "launch_max_ms", "device_max_ms")},
            "db_postings": int(sizes.sum()), "gpu_event_ms_by_kernel_1s": kernels,
            "note": "latency = submit to result on the host, including the host-to-device copy of the descriptors; "
                    "measured without per-kernel events; kernel times are event spans of a further second "
                    "of the same stream, on streams that share the GPU"}


def score_traffic(n_docs):
    """DRAM bytes of one scoring launch (ncu capture of the same seeded 20,000-image workload);
    None for other sizes."""
    return float(SCORE_DRAM_BYTES_20K_IMAGES) if n_docs == 20000 else None


def scoring_cpu_baseline(voc, ids, doc_leaves, offs, queries, k, got_docs, got_counts, seconds):
    """The reference's DataBase (compiled from its sources, oracle/_ref) on all host threads, or
    the oracle's restatement of it when the reference library is absent."""
    import numpy as np

    from oracle.pyoracle import Oracle, Reference

    threads = os.cpu_count() or 1
    weights = np.concatenate([voc.level_weights(lv).reshape(-1) for lv in range(voc.nb_levels)])
    if Reference.available() and voc.branch_factor == 16:
        ref = Reference()
        cdb, kind = ref.db(voc.nb_levels, weights), "reference"
    else:
        cdb, kind = Oracle().db(voc.branch_factor, voc.nb_levels, weights), "port"
    for i, d in enumerate(ids):
        cdb.add(int(d), doc_leaves[int(offs[i]): int(offs[i + 1])])
    q_cat = np.concatenate(queries)
    q_off = np.zeros(len(queries) + 1, np.uint64)
    q_off[1:] = np.cumsum([q.size for q in queries])
    done, t0 = 0, time.perf_counter()
    want = want_n = None
    while True:
        if kind == "reference":
            want, want_n = cdb.query_batch(q_cat, q_off, k, threads)
        else:
            want = np.full((len(queries), k), 0xFFFFFFFF, np.uint32)
            want_n = np.zeros(len(queries), np.uint32)
            for j, q in enumerate(queries):
                r = cdb.query(q, k)[0][:k]
                want[j, : r.size] = r
                want_n[j] = r.size
        done += len(queries)
        dt = time.perf_counter() - t0
        if dt >= seconds / 2:
            break
    identical = same_set = 0
    for j in range(len(queries)):
        a = got_docs[j, : got_counts[j]]
        b = want[j, : want_n[j]]
        identical += int(np.array_equal(a, b))
        same_set += int(set(a.tolist()) == set(b.tolist()))
    base = {"value": done / dt, "unit": "queries/s", "cores": threads if kind == "reference" else 1,
            "kind": kind, "sample": f"{done} queries (top-{k}) against the same 20,000-image database in {dt:.1f} s"}
    parity = {"queries": len(queries), "identical_rankings": identical, "same_result_sets": same_set,
              "note": "equal scores may come in another order from the reference's unstable sort"}
    return base, parity


def main():
    args = parse()
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
