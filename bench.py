"""Benchmark: exact kNN queries/s at 1M x 128 reference rows, 100k queries, k=10.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = kneighbors of the whole 100,000-query batch against the fitted
1,000,000 x 128 float32 index (Gaussian mixture: 1,024 centres uniform in
[-1,1]^128, sigma 0.1; reference rows seed 2, queries seed 3), k = 10.  The
headline `value` is the bf16-screen + certified re-rank form with inputs
resident in HBM; the plain fp32 form is measured in the same run
(`plain_fp32`).  `e2e` goes through the public host API with pinned host
buffers (query upload and result download inside the timed region).

Multi-GPU (torchrun, one process per GPU): every rank holds a replica of the
index and answers its own 100,000 queries (weak scaling, no collective on the
data path); time is the max over ranks.

--impl reference times the reference's own CPU implementation of this path
(mlxlearn's exact native scan, compiled from the reference sources into
oracle/_ref) on the host cores, on bounded query samples.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests"))

METRIC = ("exact kNN queries/s at 1M×128 k=10: BF16-screen+certified vs FP32; % TC peak")
N_REF, N_QUERY, D, K = 1_000_000, 100_000, 128, 10
WORKLOAD = "knn_gauss_mixture_1Mx128_100kq_k10"
# Our kernels per kNN call: assign, bin_scan, scatter, gather (query grouping),
# prep_queries, screen_tc, certify, exact (fallback rows; no-op when none).
LAUNCHES_PER_STEP = 8
SCREEN_TRAFFIC_BYTES = 5.77e9


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["bf16_tflops"], p["bf16_tflops_sustained"], p["hbm_gbs"], "measured"
    except Exception:
        return 1590.0, 1400.0, 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_reference_time(X, Q, sample, threads, k=K):
    """Time the reference's own exact CPU kNN scan (oracle/_ref) on a query sample.

    Returns (queries/s, results (dist, idx), kind, cores).
    """
    import oracle
    from concurrent.futures import ThreadPoolExecutor

    ref = oracle.ref_native()
    Qs = np.ascontiguousarray(Q[:sample])
    dist = np.empty((sample, k), np.float64)
    idx = np.empty((sample, k), np.int64)
    if ref is not None:
        kind = "reference"
        chunks = np.array_split(np.arange(sample), threads)

        def run(rows):
            if len(rows):
                a, b = rows[0], rows[-1] + 1
                # reference: src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:362-418 (GIL released)
                ref.neighbors.query(X, Qs[a:b], k, False, 0, dist[a:b], idx[a:b])

        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(run, chunks))
        el = time.perf_counter() - t0
    else:
        kind = "port"
        t0 = time.perf_counter()
        dist, idx = oracle.knn(X, Qs, k, nthreads=threads)
        el = time.perf_counter() - t0
    return sample / el, (dist, idx), kind


def run_reference_arm(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from datasets import cfg2a

    X, Q = cfg2a(N_REF, N_QUERY, D)
    threads = os.cpu_count() or 1
    # 16 queries per host thread per call: enough to amortise the scan's
    # per-call work (the full batch is one call of 100k queries); ~4 s per step
    sample = max(threads, int(os.environ.get("B2K_REF_SAMPLE", "0")) or threads * 16)
    vals = []
    kind = "reference"
    for step in range(args.warmup + args.steps):
        qps, _, kind = cpu_reference_time(X, Q[(step * sample) % N_QUERY:], sample, threads)
        if step >= args.warmup:
            vals.append(qps)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * N_QUERY / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_ref": N_REF, "d": D, "n_query": N_QUERY, "k": K},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": kind,
                         "sample": f"{sample} queries per step of the {N_QUERY}-query batch; "
                                   "ms_per_step extrapolates to the full batch"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    from datasets import cfg2a
    from mlxlearn_b200 import _lib
    from mlxlearn_b200.index import build_index
    from mlxlearn_b200.sharding import max_over_ranks

    X, _ = cfg2a(N_REF, 1, D)
    # each rank answers its own query shard (weak scaling)
    from datasets import mixture

    C = np.random.default_rng(2).uniform(-1, 1, (1024, D))
    Q, _ = mixture(np.random.default_rng(3 + 1000 * rank), N_QUERY, C, 0.1)
    index = build_index(X, device=local)
    index._ensure_device()
    Qd = torch.from_numpy(Q).cuda()
    stream = torch.cuda.current_stream()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    def timed(mode, steps, warmup):
        stats = []
        for _ in range(warmup):
            index.query_device(Qd, K, mode=mode)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            index.query_device(Qd, K, mode=mode, stats=True)
            stats.append(index.last_stats)
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1) / steps
        if pg is not None:
            ms = max_over_ranks(ms)
        return ms, stats

    with ClockSampler(local) as clk:
        ms_bf16, st_bf16 = timed("bf16", args.steps, args.warmup)
    clocks = clk.summary()
    ms_fp32, st_fp32 = timed("fp32", max(1, min(2, args.steps)), 1)

    # e2e: public host API, pinned host buffers, copies inside the timed region
    Qh = torch.from_numpy(Q).pin_memory().numpy()
    out_i = torch.empty((N_QUERY, K), dtype=torch.int64).pin_memory().numpy()
    out_d = torch.empty((N_QUERY, K), dtype=torch.float64).pin_memory().numpy()
    for _ in range(max(1, args.warmup)):
        index.query(Qh, K, mode="bf16", out=(out_d, out_i))
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        index.query(Qh, K, mode="bf16", out=(out_d, out_i))
    barrier()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if pg is not None:
        e2e_s = max_over_ranks(e2e_s)

    result = None
    if rank == 0:
        tf_burst, tf_sust, hbm, peak_kind = peaks()
        flops = 2.0 * N_REF * D * N_QUERY
        screen_ms = statistics.median(s["screen_ms"] for s in st_bf16)
        achieved = flops / (screen_ms * 1e-3) / 1e12
        total_timed_s = ms_bf16 * args.steps / 1000.0
        peak = tf_sust if total_timed_s > 1.0 else tf_burst
        fp32_screen_ms = statistics.median(s["screen_ms"] for s in st_fp32)
        # DRAM bytes (read + write) of one screen launch, from the ncu capture in
        # profiles/screen_tc_knn_gauss1Mx128.txt (10k queries, scaled by tile pairs)
        traffic = os.environ.get("B2K_SCREEN_TRAFFIC_BYTES", SCREEN_TRAFFIC_BYTES)
        result = {
            "metric": METRIC,
            "value": ws * N_QUERY / (ms_bf16 / 1000.0),
            "unit": "queries/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_bf16,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16",
            "data": "synthetic: Gaussian mixture (1024 centres U[-1,1]^128, sigma 0.1), "
                    "seeds 2/3",
            "config": {"workload": WORKLOAD, "n_ref": N_REF, "d": D, "n_query": N_QUERY, "k": K,
                       "queries_per_gpu": N_QUERY, "parallelism": f"replicas x{ws}",
                       "l2": "inputs larger than L2 (bf16 index 256 MB, fp32 index 512 MB)"},
            "roofline": {"kernel": "screen_tc_kernel (bf16 tcgen05 distance tile)",
                         "bound": "tensor", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} "
                                        f"{'sustained' if peak == tf_sust else 'burst'} bf16",
                         "algorithmic_flops_per_launch": flops,
                         "traffic": None if traffic is None else float(traffic)},
            "plain_fp32": {"value": ws * N_QUERY / (ms_fp32 / 1000.0), "unit": "queries/s",
                           "ms_per_step": ms_fp32, "screen_ms": fp32_screen_ms,
                           "screen_tflops": flops / (fp32_screen_ms * 1e-3) / 1e12,
                           "bf16_speedup": ms_fp32 / ms_bf16},
            "screen_stats": {k: v for k, v in st_bf16[-1].items()},
            "e2e": {"value": ws * N_QUERY / e2e_s, "unit": "queries/s",
                    "h2d_bytes_per_step": int(Qh.nbytes),
                    "d2h_bytes_per_step": int(out_i.nbytes + out_d.nbytes)},
            "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "clocks": clocks,
        }
        # CPU baseline: the reference's exact CPU scan on a bounded sample, with
        # our answers for the same queries compared against it.
        threads = os.cpu_count() or 1
        # a bounded sample of about 10 s of CPU work: calls of 16 queries per
        # thread (amortising the scan's per-call work, as the full batch does)
        # until 10 s have passed (at most 30 calls)
        block = 16 * threads
        done, spent, first = 0, 0.0, None
        while spent < float(os.environ.get("B2K_CPU_SECONDS", "10")) and done < 30 * block:
            t_b = time.perf_counter()
            qps_b, res_b, kind = cpu_reference_time(X, Q[done:], block, threads)
            spent += time.perf_counter() - t_b
            if first is None:
                first = res_b
            done += block
        qps = done / spent
        sample = min(block, 64)  # parity: the first 64 queries of the first call
        rd, ri = first[0][:sample], first[1][:sample]
        od, oi = index.query(Q[:sample], K, mode="bf16")
        rel = np.max(np.abs(od - rd) / np.maximum(rd, 1e-300))
        result["cpu_baseline"] = {"value": qps, "unit": "queries/s", "cores": threads,
                                  "kind": kind,
                                  "sample": f"first {done} queries of the batch, k={K} "
                                            f"({spent:.1f} s of CPU work)"}
        result["parity_vs_cpu_reference"] = {"queries": sample,
                                             "indices_bit_exact": bool(np.array_equal(oi, ri)),
                                             "max_rel_dist_err": float(rel)}
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Secondary workloads (not the headline line): --workload pixels|radius|small
# ---------------------------------------------------------------------------

def _radius_threshold_tuple(d, R2):
    """(R2, f64_in, f64_out, prune_above, bulk_below) as the reference's
    radius extension takes it (src/mlxlearn/_kernels/radius_contract.py:129-153,
    radius_cpu.py:137-140)."""
    import math

    down = lambda v: math.nextafter(v, -math.inf)  # noqa: E731
    up = lambda v: math.nextafter(v, math.inf)  # noqa: E731
    u = 2.0 ** -53
    g = (d + 2) * u / (1.0 - (d + 2) * u)
    f_in = max(down(down(R2 * down(1.0 - 2.0 * g))), 0.0)
    f_out = up(up(R2 * up(1.0 + 2.0 * g)))
    prune = up(up(R2 * up(1.0 + 4.0 * g)))
    bulk = max(down(down(R2 * down(1.0 - 4.0 * g))), 0.0)
    return (float(R2), f_in, f_out, prune, bulk)


def _timed_wall(fn, steps, warmup):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        out = fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / steps, out


def run_secondary(args):
    import torch

    from mlxlearn_b200.index import build_index
    from mlxlearn_b200.neighbors import KNeighborsClassifier, NearestNeighbors
    from mlxlearn_b200.neighbors import RadiusNeighborsClassifier

    torch.cuda.set_device(0)
    threads = os.cpu_count() or 1
    line = {"metric": None, "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic", "workload_kind": "secondary"}
    import oracle

    ref = oracle.ref_native()
    if args.workload == "pixels":
        from datasets import cfg2b

        X, Q, y = cfg2b()
        k = 5
        clf = KNeighborsClassifier(n_neighbors=k).fit(X, y)
        Qd = torch.from_numpy(Q).cuda()
        ms = 1000 * _timed_wall(lambda: clf._index_.query_device(Qd, k, mode="bf16"),
                                args.steps, args.warmup)[0]
        e2e_s, pred = _timed_wall(lambda: clf.predict(Q), args.steps, args.warmup)
        st = clf._index_.query_device(Qd, k, mode="bf16", stats=True) and clf._index_.last_stats
        sample = min(len(Q), 4 * threads)
        rd = np.empty((sample, k)); ri = np.empty((sample, k), np.int64)
        t0 = time.perf_counter()
        _ref_knn_threads(ref, X, Q[:sample], k, rd, ri, threads)
        cpu_qps = sample / (time.perf_counter() - t0)
        od, oi = clf.kneighbors(Q[:sample])
        line.update({"metric": "KNeighborsClassifier(k=5).predict queries/s, 60k x 784 pixels",
                     "value": len(Q) / (ms / 1000), "ms_per_step": ms, "dtype": "bf16",
                     "config": {"workload": "knn_pixels_60000x784_10000q_k5"},
                     "e2e": {"value": len(Q) / e2e_s, "unit": "queries/s",
                             "api": "KNeighborsClassifier.predict (host arrays)"},
                     "screen_stats": st,
                     "cpu_baseline": {"value": cpu_qps, "unit": "queries/s", "cores": threads,
                                      "kind": "reference" if ref else "port",
                                      "sample": f"first {sample} queries"},
                     "parity_vs_cpu_reference": {"indices_bit_exact": bool(np.array_equal(oi, ri)),
                                                 "max_rel_dist_err": float(np.max(
                                                     np.abs(od - rd) / np.maximum(rd, 1e-300)))}})
    elif args.workload == "radius":
        from datasets import cfg3

        X, y, Q = cfg3()
        index = build_index(X)
        # radius: median 50th-neighbour distance over a 1000-query sample
        d50, _ = index.query(Q[:1000], 50)
        r = float(np.median(d50[:, -1]))
        clf = RadiusNeighborsClassifier(radius=r, outlier_label="most_frequent").fit(X, y)
        e2e_s, pred = _timed_wall(lambda: clf.predict(Q), args.steps, args.warmup)
        csr_s, parts = _timed_wall(lambda: clf._index_.query_radius_csr(Q, r),
                                   args.steps, args.warmup)
        p = parts[0]
        sample = min(len(Q), 16 * threads)
        t0 = time.perf_counter()
        ok = None
        if ref is not None:
            thr = _radius_threshold_tuple(X.shape[1], r * r)
            res = ref.radius.brute_query(X, np.ascontiguousarray(Q[:sample]), thr, 0, False, 1,
                                         threads)
            cpu_qps = sample / (time.perf_counter() - t0)
            nq, nnz = ref.radius.result_sizes(res)
            counts = np.empty(nq, np.int64)
            ref.radius.result_counts(res, counts)
            ip = np.zeros(nq + 1, np.int64)
            np.cumsum(counts, out=ip[1:])
            ix = np.empty(nnz, np.int64); dd = np.empty(nnz)
            ref.radius.result_fill_csr(res, ip, ix, dd, threads)
            ok = (bool(np.array_equal(ip, p.indptr[:sample + 1]))
                  and bool(np.array_equal(ix, p.indices[:ip[-1]]))
                  and bool(np.array_equal(dd, p.distances[:ip[-1]])))
        else:
            oracle.radius(X, Q[:sample], r)
            cpu_qps = sample / (time.perf_counter() - t0)
        line.update({"metric": "RadiusNeighborsClassifier.predict queries/s, 200k x 32",
                     "value": len(Q) / csr_s, "ms_per_step": 1000 * csr_s, "dtype": "bf16",
                     "config": {"workload": "radius_200000x32_50000q", "radius": r,
                                "median_neighbours": float(np.median(p.lengths())),
                                "zero_neighbour_queries": int((p.lengths() == 0).sum()),
                                "nnz": p.nnz,
                                "value_note": "query_radius_csr through the host C ABI "
                                              "(upload, screen, exact classify, CSR download)"},
                     "e2e": {"value": len(Q) / e2e_s, "unit": "queries/s",
                             "api": "RadiusNeighborsClassifier.predict (host arrays)"},
                     "cpu_baseline": {"value": cpu_qps, "unit": "queries/s", "cores": threads,
                                      "kind": "reference" if ref else "port",
                                      "sample": f"first {sample} queries, brute_query"},
                     "parity_vs_cpu_reference": {"csr_bit_exact": ok}})
    else:  # small: config 1
        from datasets import cfg1

        X, Q = cfg1()
        nn = NearestNeighbors(n_neighbors=5, algorithm="brute", metric="euclidean").fit(X)
        Qd = torch.from_numpy(Q).cuda()
        ms = 1000 * _timed_wall(lambda: nn._index_.query_device(Qd, 5), args.steps,
                                args.warmup)[0]
        e2e_s, (od, oi) = _timed_wall(lambda: nn.kneighbors(Q), args.steps, args.warmup)
        rd = np.empty((len(Q), 5)); ri = np.empty((len(Q), 5), np.int64)
        t0 = time.perf_counter()
        _ref_knn_threads(ref, X, Q, 5, rd, ri, threads)
        cpu_qps = len(Q) / (time.perf_counter() - t0)
        line.update({"metric": "NearestNeighbors(k=5).kneighbors queries/s, 10000 x 64",
                     "value": len(Q) / (ms / 1000), "ms_per_step": ms, "dtype": "auto",
                     "config": {"workload": "knn_gauss_10000x64_2000q_k5"},
                     "e2e": {"value": len(Q) / e2e_s, "unit": "queries/s",
                             "api": "NearestNeighbors.kneighbors (host arrays)"},
                     "cpu_baseline": {"value": cpu_qps, "unit": "queries/s", "cores": threads,
                                      "kind": "reference" if ref else "port",
                                      "sample": "all 2000 queries"},
                     "parity_vs_cpu_reference": {
                         "queries": len(Q), "indices_bit_exact": bool(np.array_equal(oi, ri)),
                         "max_rel_dist_err": float(np.max(np.abs(od - rd) /
                                                          np.maximum(rd, 1e-300)))}})
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """256 uneven problems (seed 5) as one planned batch vs one call per problem."""
    import torch

    from datasets import cfg4
    from mlxlearn_b200.batch import KnnBatch
    from mlxlearn_b200.index import build_index

    import oracle

    torch.cuda.set_device(0)
    threads = os.cpu_count() or 1
    problems = cfg4(problems=args.problems)
    total_q = sum(Q.shape[0] for _, Q, _ in problems)
    flops = sum(2.0 * X.shape[0] * Q.shape[0] * X.shape[1] for X, Q, _ in problems)
    t0 = time.perf_counter()
    indexes = [build_index(X) for X, _, _ in problems]
    for ix in indexes:
        ix._ensure_device()
    fit_s = time.perf_counter() - t0
    Qd = [torch.from_numpy(Q).cuda() for _, Q, _ in problems]
    items = [(ix, q, k) for ix, q, (_, _, k) in zip(indexes, Qd, problems)]
    t0 = time.perf_counter()
    batch = KnnBatch(items, autotune=not args.profile)
    plan_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    if args.profile:  # profiling driver: the batched runs only
        for _ in range(args.warmup + args.steps):
            batch.run()
        print(json.dumps({"profile": True, "stats": batch.finish()}), flush=True)
        batch.close()
        return 0
    for _ in range(args.warmup):
        batch.run()
    batch.finish()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            batch.run()
        ev1.record(stream)
        stats = batch.finish()
    ms = ev0.elapsed_time(ev1) / args.steps
    # one call per problem through the single-problem device API
    for ix, q, (_, _, k) in zip(indexes, Qd, problems):
        ix.query_device(q, k)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for ix, q, (_, _, k) in zip(indexes, Qd, problems):
        ix.query_device(q, k)
    torch.cuda.synchronize()
    one_s = time.perf_counter() - t0
    # e2e: pinned host queries in, results out, through the batch object
    Qh = [torch.from_numpy(Q).pin_memory() for _, Q, _ in problems]
    Dh = [torch.empty(d.shape, dtype=d.dtype).pin_memory() for d in batch.dist]
    Ih = [torch.empty(i.shape, dtype=i.dtype).pin_memory() for i in batch.idx]

    def e2e_step():
        for dst, src in zip(batch.queries, Qh):
            dst.copy_(src, non_blocking=True)
        batch.run()
        batch.finish()
        for dst, src in zip(Dh, batch.dist):
            dst.copy_(src, non_blocking=True)
        for dst, src in zip(Ih, batch.idx):
            dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()

    e2e_s = _timed_wall(e2e_step, args.steps, 1)[0]
    h2d = sum(q.numel() * 4 for q in Qh)
    d2h = sum(d.numel() * 8 for d in Dh) + sum(i.numel() * 8 for i in Ih)
    # parity + CPU baseline: the reference's exact scan on a few queries of every problem
    ref = oracle.ref_native()
    per = int(os.environ.get("B2K_BATCH_CPU_QUERIES", "4"))
    est_cpu_s, sample_q, exact, rel = 0.0, 0, True, 0.0
    for (X, Q, k), d, i in zip(problems, batch.dist, batch.idx):
        s = min(per, Q.shape[0])
        rd = np.empty((s, k)); ri = np.empty((s, k), np.int64)
        t1 = time.perf_counter()
        _ref_knn_threads(ref, X, Q[:s], k, rd, ri, min(threads, s))
        est_cpu_s += (time.perf_counter() - t1) * Q.shape[0] / s
        sample_q += s
        exact &= bool(np.array_equal(ri, i[:s].cpu().numpy()))
        od = d[:s].cpu().numpy()
        rel = max(rel, float(np.max(np.abs(od - rd) / np.maximum(rd, 1e-300))))
    tf_burst, tf_sust, hbm, peak_kind = peaks()
    achieved = flops / (ms * 1e-3) / 1e12
    line = {
        "metric": "batched uneven kNN: aggregate queries/s, 256 problems (one graph) vs one "
                  "call per problem",
        "value": total_q / (ms / 1000), "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16", "data": "synthetic: cfg4 recipe (seed 5)",
        "workload_kind": "secondary",
        "config": {"workload": f"knn_batch_{len(problems)}_uneven_seed5",
                   "problems": len(problems),
                   "queries": total_q, "flops": flops,
                   "l2": "operands 1.9 GB bf16, larger than L2"},
        "one_call_per_problem": {"value": total_q / one_s, "unit": "queries/s",
                                 "ms_per_step": 1000 * one_s,
                                 "batch_speedup": one_s / (ms / 1000)},
        "roofline": {"kernel": "whole batched run (prep, screens, certify, exact)",
                     "bound": "tensor", "achieved": achieved, "peak": tf_burst,
                     "unit": "TFLOP/s", "frac": achieved / tf_burst,
                     "peak_source": f"{peak_kind} burst bf16", "traffic": None},
        "batch_stats": stats, "fit_s": fit_s, "plan_s": plan_s,
        "e2e": {"value": total_q / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "cpu_baseline": {"value": total_q / est_cpu_s, "unit": "queries/s", "cores": threads,
                         "kind": "reference" if ref else "port",
                         "sample": f"first {per} queries of every problem, time scaled by "
                                   "each problem's query count"},
        "parity_vs_cpu_reference": {"queries": sample_q, "indices_bit_exact": exact,
                                    "max_rel_dist_err": rel},
        "clocks": clk.summary(),
    }
    batch.close()
    print(json.dumps(line), flush=True)
    return 0


def run_chamfer(args):
    """Differentiable kNN losses: 64 symmetric k=1 Chamfer terms on 8192 x 3
    clouds plus a self k=8 mean-distance term on 4096 x 64, forward + backward."""
    import torch

    from datasets import cfg5
    from mlxlearn_b200.autograd import chamfer_loss_batch, knn_distances

    import oracle

    torch.cuda.set_device(0)
    threads = os.cpu_count() or 1
    clouds, S = cfg5()
    # the 64 pairs as two [64, 8192, 3] tensors
    A = torch.from_numpy(np.stack([a for a, _ in clouds])).cuda().requires_grad_()
    B = torch.from_numpy(np.stack([b for _, b in clouds])).cuda().requires_grad_()
    Sd = torch.from_numpy(S).cuda().requires_grad_()
    pairs = sum(2 * a.shape[0] * b.shape[0] for a, b in clouds) + S.shape[0] * S.shape[0]

    def step():
        loss = chamfer_loss_batch(A, B)  # all 64 pairs in one search + one backward
        d8, _ = knn_distances(Sd, None, 8)
        loss = loss + d8.mean()
        loss.backward()
        return loss

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    step_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        loss = step()
        torch.cuda.synchronize()
        step_ms.append(1000 * (time.perf_counter() - t0))
    s = sum(step_ms) / len(step_ms) / 1000
    # CPU baseline: the reference's exact scan for the forward of two pairs
    # (both directions) and torch float64 autograd on the CPU for their backward
    ref = oracle.ref_native()
    t0 = time.perf_counter()
    cpu_pairs = 0
    for a, b in clouds[:2]:
        for P, Qr in ((a, b), (b, a)):
            dist = np.empty((len(P), 1)); idx = np.empty((len(P), 1), np.int64)
            _ref_knn_threads(ref, Qr, P, 1, dist, idx, threads)
            Pt = torch.from_numpy(P).double().requires_grad_()
            Qt = torch.from_numpy(Qr).double().requires_grad_()
            ((Pt - Qt[torch.from_numpy(idx[:, 0])]) ** 2).sum().backward()
            cpu_pairs += len(P) * len(Qr)
    cpu_s = time.perf_counter() - t0
    # parity of the forward: the two sampled pairs (both directions) through the
    # segment search against the reference's exact scan
    from mlxlearn_b200.autograd import knn_segments

    exact, err = True, 0.0
    for a, b in clouds[:2]:
        for P, Qr in ((a, b), (b, a)):
            gd, gi = knn_segments(torch.from_numpy(Qr).cuda(), torch.from_numpy(P).cuda(),
                                  [len(Qr)], [len(P)], 1)
            rdist = np.empty((len(Qr), 1)); ridx = np.empty((len(Qr), 1), np.int64)
            _ref_knn_threads(ref, P, Qr, 1, rdist, ridx, threads)
            exact &= bool(np.array_equal(gi.cpu().numpy(), ridx))
            gdv = gd.double().cpu().numpy()
            err = max(err, float(np.max(np.abs(gdv - rdist) / np.maximum(rdist, 1e-300))))
    line = {
        "metric": "differentiable kNN: (query, reference) pairs/s, forward + backward "
                  "(64 Chamfer k=1 pairs of 8192x3 + self k=8 on 4096x64)",
        "value": pairs / s, "unit": "pairs/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * s, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: cfg5 recipe (seed 6)", "workload_kind": "secondary",
        "config": {"workload": "knn_chamfer_64x8192x3_self4096x64", "pairs_per_step": pairs,
                   "api": "mlxlearn_b200.autograd (public), wall clock with device sync"},
        "loss": float(loss.item()), "step_ms": step_ms,
        "cpu_baseline": {"value": cpu_pairs / cpu_s, "unit": "pairs/s", "cores": threads,
                         "kind": "reference" if ref else "port",
                         "sample": "2 Chamfer pairs both ways: reference exact scan forward, "
                                   "torch float64 CPU autograd backward"},
        "parity_vs_cpu_reference": {"pairs": 4, "indices_bit_exact": exact,
                                    "max_rel_dist_err": err,
                                    "note": "forward k=1 of 2 Chamfer pairs, both directions; "
                                            "distances are float32 outputs of the autograd path"},
    }
    print(json.dumps(line), flush=True)
    return 0


def _ref_knn_threads(ref, X, Q, k, dist, idx, threads):
    """The reference's exact native kNN scan over query blocks in threads."""
    from concurrent.futures import ThreadPoolExecutor

    import oracle

    if ref is None:
        d, i = oracle.knn(X, Q, k, nthreads=threads)
        dist[:] = d
        idx[:] = i
        return
    Q = np.ascontiguousarray(Q)
    chunks = np.array_split(np.arange(len(Q)), threads)

    def run(rows):
        if len(rows):
            a, b = rows[0], rows[-1] + 1
            ref.neighbors.query(X, Q[a:b], k, False, 0, dist[a:b], idx[a:b])

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(run, chunks))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="knn",
                    choices=["knn", "pixels", "radius", "small", "batch", "chamfer"])
    ap.add_argument("--profile", action="store_true",
                    help="profiling driver: only the bf16 device-resident steps of the "
                         "headline workload (no fp32 leg, e2e or CPU baseline)")
    ap.add_argument("--mode", default="bf16", choices=["bf16", "fp32", "exact", "auto"],
                    help="screen form for --profile")
    ap.add_argument("--k", type=int, default=K, help="neighbours for --profile")
    ap.add_argument("--problems", type=int, default=256,
                    help="problem count of the batch workload (the benchmark uses 256)")
    ap.add_argument("--queries", type=int, default=N_QUERY,
                    help="query count for --profile (the headline uses 100,000)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "chamfer":
        return run_chamfer(args)
    if args.profile:
        return run_profile(args)
    if args.workload != "knn":
        return run_secondary(args)
    return run_ours(args)


def run_profile(args):
    """Screen + certify on the headline index, `--queries` queries, `--mode`."""
    import torch

    from datasets import cfg2a
    from mlxlearn_b200.index import build_index

    torch.cuda.set_device(0)
    X, Q = cfg2a(N_REF, args.queries, D)
    index = build_index(X)
    Qd = torch.from_numpy(Q).cuda()
    for _ in range(args.warmup):
        index.query_device(Qd, args.k, mode=args.mode)
    torch.cuda.synchronize()
    for _ in range(args.steps):
        index.query_device(Qd, args.k, mode=args.mode, stats=True)
    torch.cuda.synchronize()
    print(json.dumps({"profile": True, "queries": args.queries, "mode": args.mode, "k": args.k,
                      "stats": index.last_stats}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
