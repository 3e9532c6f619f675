"""Benchmark: exact kNN queries/s at 1M x 128 reference rows, 100k queries, k=10.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload all|knn|small|pixels|radius|batch|chamfer]

Headline (one step = kneighbors of the whole 100,000-query batch against the
fitted 1,000,000 x 128 float32 index; Gaussian mixture: 1,024 centres uniform
in [-1,1]^128, sigma 0.1; reference rows seed 2, queries seed 3; k = 10).
`value` is the bf16-screen + certified re-rank form with inputs resident in
HBM; the plain fp32 form is measured in the same run (`plain_fp32`); `e2e`
goes through the public host API with page-locked host buffers (query upload
and result download inside the timed region).  `cpu_baseline` is the
reference's own stock route, NearestNeighbors(algorithm='brute').kneighbors
from the installed reference package, on a bounded query sample; every query
it answers is compared with ours (`parity_vs_cpu_reference`).

The default run (N = 1) also measures the other four configurations and
nests their lines under `secondary`: config 1 (10k x 64, k = 5), config 2b
(60k x 784 integer pixels, k = 5), config 3 (radius classifier, 200k x 32),
config 4 (256 uneven problems in one graph) and config 5 (differentiable kNN:
Chamfer + self-kNN losses, forward and backward).  Each has its own roofline,
CPU baseline (the reference's stock estimators), e2e figure and parity.

Multi-GPU (torchrun, one process per GPU): every rank holds a replica of the
index and answers its own 100,000 queries (weak scaling, no collective on the
data path); time is the max over ranks.  Secondary configurations run at
N = 1 only.

--impl reference times the reference's own CPU implementation of this path:
mlxlearn's NearestNeighbors(n_neighbors=10, algorithm='brute').kneighbors
(installed into baseline/_ref by `make -C oracle refpkg`; its CPUIndex route
with the reference's native engines), one bounded query sample per step.
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
# Our kernels per kNN call (the ncu launch list of this workload): nonfinite
# check; assign, bin_scan, scatter, gather (query grouping); prep_queries;
# home_tiles and the seeding screen; the main screen; certify.  No exhaustive
# or second-pass launch when every row certifies.
LAUNCHES_PER_STEP = 10
# DRAM bytes (read + write) of one screen launch at the headline size: an ncu
# capture of the full 100,000-query launch (dram__bytes_read/write, one pass),
# summarised in profiles/screen_tc_knn_gauss1Mx128.txt
SCREEN_TRAFFIC_BYTES = 5.84e9
# FP32 CUDA-core rate (no measured figure): 148 SMs x 128 lanes x 2 FLOP x 1.965 GHz
FP32_NOMINAL_TFLOPS = 74.4
L2_FLUSH_BYTES = 256 << 20  # larger than the 126 MB L2


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["bf16_tflops"], p["bf16_tflops_sustained"], p["hbm_gbs"], "measured"
    except Exception:
        return 1590.0, 1400.0, 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region.

    Samples are stamped with the host clock as they arrive (every 50 ms);
    `begin()` / `end()` mark the timed region and `summary()` keeps the
    samples inside it (all samples when the region caught none)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the sampler is live before the caller's work starts
            deadline = time.perf_counter() + 3.0
            while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def begin(self):
        self.window = [time.perf_counter(), None]

    def end(self):
        if self.window is not None:
            # one more interval: the sample taken while the last step ran
            time.sleep(self.INTERVAL_MS / 1000.0)
            self.window[1] = time.perf_counter()

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        lines = self.lines
        in_window = False
        if self.window is not None and self.window[1] is not None:
            t0, t1 = self.window
            inside = [(t, ln) for t, ln in lines if t0 <= t <= t1]
            if inside:
                lines, in_window = inside, True
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, line in lines:
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
                "reasons": sorted(reasons), "samples": len(sm),
                "timed_region_only": in_window, "interval_ms": self.INTERVAL_MS}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------
# The reference's CPU path (checker and baseline only)
# ---------------------------------------------------------------------------

def reference_neighbors():
    """The reference's estimator module (installed package), or None."""
    from oracle import refpkg

    ref = refpkg.import_reference()
    return None if ref is None else ref.neighbors


def host_threads():
    """Host threads the reference's CPU path uses (its BLAS pool and native
    engines run on every core)."""
    n = os.cpu_count() or 1
    try:
        from threadpoolctl import threadpool_info

        blas = [p.get("num_threads", 0) for p in threadpool_info()]
        if blas:
            n = max(n, max(blas))
    except Exception:
        pass
    return n


def rel_err(ours, ref):
    ours = np.asarray(ours, np.float64)
    ref = np.asarray(ref, np.float64)
    if ours.size == 0:
        return 0.0
    return float(np.max(np.abs(ours - ref) / np.maximum(np.abs(ref), 1e-300)))


def stock_kneighbors(est, Q, block, seconds, max_queries):
    """kneighbors of the fitted reference estimator over consecutive blocks
    of `block` queries until `seconds` of CPU work or `max_queries`; returns
    (queries/s, dist, idx, queries answered)."""
    done, spent, ds, ix = 0, 0.0, [], []
    while spent < seconds and done < max_queries:
        t0 = time.perf_counter()
        d, i = est.kneighbors(Q[done:done + block])
        spent += time.perf_counter() - t0
        ds.append(d)
        ix.append(i)
        done += len(i)
    return done / spent, np.concatenate(ds), np.concatenate(ix), done


def native_kneighbors(X, Q, k, threads):
    """Fallback when the reference package is not installed: the reference's
    native exact scan (oracle/_ref), else the oracle port.  Returns
    (dist, idx, kind)."""
    from concurrent.futures import ThreadPoolExecutor

    import oracle

    ref = oracle.ref_native()
    if ref is None:
        d, i = oracle.knn(X, Q, k, nthreads=threads)
        return d, i, "port"
    Q = np.ascontiguousarray(Q)
    dist = np.empty((len(Q), k))
    idx = np.empty((len(Q), k), np.int64)
    chunks = np.array_split(np.arange(len(Q)), threads)

    def run(rows):
        if len(rows):
            a, b = rows[0], rows[-1] + 1
            # reference: src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:362-418 (GIL released)
            ref.neighbors.query(X, Q[a:b], k, False, 0, dist[a:b], idx[a:b])

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(run, chunks))
    return dist, idx, "reference"


def run_reference_arm(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from datasets import cfg2a

    X, Q = cfg2a(N_REF, N_QUERY, D)
    threads = host_threads()
    sample = int(os.environ.get("B2K_REF_SAMPLE", "256"))
    nb = reference_neighbors()
    if nb is not None:
        est = nb.NearestNeighbors(n_neighbors=K, algorithm="brute").fit(X)
        route = ("mlxlearn NearestNeighbors(n_neighbors=10, algorithm='brute').kneighbors "
                 "(installed reference, CPUIndex route with its native engines)")
    else:
        est, route = None, "mlxlearn's native exact scan (oracle/_ref)"
    times = []
    kind = "reference"
    for step in range(args.warmup + args.steps):
        Qs = Q[(step * sample) % N_QUERY:][:sample]
        t0 = time.perf_counter()
        if est is not None:
            est.kneighbors(Qs)
        else:
            _, _, kind = native_kneighbors(X, Qs, K, threads)
        el = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(el)
    step_s = statistics.median(times)
    value = sample / step_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * step_s, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_ref": N_REF, "d": D, "n_query": N_QUERY, "k": K,
                   "step": f"{sample} consecutive queries of the {N_QUERY}-query batch"},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": kind,
                         "sample": f"{sample} queries per step through {route}"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Device timing helpers
# ---------------------------------------------------------------------------

class L2Flush:
    """Writes a buffer larger than L2 between timed iterations."""

    def __init__(self, device):
        import torch

        self.buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)

    def __call__(self):
        self.buf.fill_(1.0)


def event_times(fn, steps, warmup, flush=None):
    """Per-step device times (ms) of fn on the current stream, each step
    bracketed by CUDA events; `flush` (untimed) runs before every step."""
    import torch

    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(steps):
        if flush is not None:
            flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def wall_times(fn, steps, warmup):
    """Per-step wall times (s) of a host-facing call that synchronises."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        out.append(time.perf_counter() - t0)
    return out


def tensor_roofline(kernel, flops, seconds, peak_tf, peak_kind, peak_name="burst bf16"):
    achieved = flops / seconds / 1e12
    return {"kernel": kernel, "bound": "tensor", "achieved": achieved, "peak": peak_tf,
            "unit": "TFLOP/s", "frac": achieved / peak_tf,
            "peak_source": f"{peak_kind} {peak_name}", "traffic": None}


# ---------------------------------------------------------------------------
# Headline
# ---------------------------------------------------------------------------

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
    from datasets import cfg2a, mixture
    from mlxlearn_b200.index import build_index
    from mlxlearn_b200.sharding import max_over_ranks

    X, _ = cfg2a(N_REF, 1, D)
    # each rank answers its own query shard (weak scaling)
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

    def timed(mode, steps, warmup, clk=None):
        stats = []
        for _ in range(warmup):
            index.query_device(Qd, K, mode=mode)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if clk is not None:
            clk.begin()
        ev0.record(stream)
        for _ in range(steps):
            index.query_device(Qd, K, mode=mode, stats=True)
            stats.append(index.last_stats)
        ev1.record(stream)
        barrier()
        if clk is not None:
            clk.end()
        ms = ev0.elapsed_time(ev1) / steps
        if pg is not None:
            ms = max_over_ranks(ms)
        return ms, stats

    with ClockSampler(local) as clk:
        ms_bf16, st_bf16 = timed("bf16", args.steps, args.warmup, clk)
    clocks = clk.summary()
    ms_fp32, st_fp32 = timed("fp32", max(1, min(2, args.steps)), 1)
    ms_tf32, st_tf32 = timed("tf32", max(1, min(5, args.steps)), 2)

    # e2e: public host API, page-locked host buffers, copies inside the timed region
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
        seed_ms = statistics.median(s["seed_ms"] for s in st_bf16)
        # the distance tile's launch: screen_ms spans the seeding pass (a launch
        # of the same kernel over each query tile's 16-tile home window, 2.6% of
        # the pairs again) and the main launch over all 2 n m d FLOPs
        main_ms = screen_ms - seed_ms
        total_timed_s = ms_bf16 * args.steps / 1000.0
        peak = tf_sust if total_timed_s > 1.0 else tf_burst
        roof = tensor_roofline("screen_tc_kernel main launch (bf16 tcgen05 distance tile)", flops,
                               main_ms * 1e-3, peak, peak_kind,
                               "sustained bf16" if peak == tf_sust else "burst bf16")
        roof["algorithmic_flops_per_launch"] = flops
        roof["launch_ms"] = main_ms
        roof["seeding_pass_ms"] = seed_ms
        roof["frac_incl_seeding_pass"] = flops / (screen_ms * 1e-3) / 1e12 / peak
        traffic = os.environ.get("B2K_SCREEN_TRAFFIC_BYTES", SCREEN_TRAFFIC_BYTES)
        roof["traffic"] = None if traffic is None else float(traffic)
        fp32_screen_ms = statistics.median(s["screen_ms"] for s in st_fp32)
        tf32_screen_ms = statistics.median(s["screen_ms"] for s in st_tf32)
        # no measured tf32 figure: kind::tf32 does half the FLOPs of kind::f16
        # per instruction at the same rate, so half the measured bf16 peak
        tf32_peak = tf_burst / 2
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
            "roofline": roof,
            "plain_fp32": {"value": ws * N_QUERY / (ms_fp32 / 1000.0), "unit": "queries/s",
                           "form": "fp32 CUDA-core screen (screen_simt_kernel) + the same "
                                   "certify pass",
                           "ms_per_step": ms_fp32, "screen_ms": fp32_screen_ms,
                           "screen_tflops": flops / (fp32_screen_ms * 1e-3) / 1e12,
                           "screen_frac_of_fp32_nominal":
                               flops / (fp32_screen_ms * 1e-3) / 1e12 / FP32_NOMINAL_TFLOPS,
                           "bf16_speedup": ms_fp32 / ms_bf16},
            "plain_tf32": {"value": ws * N_QUERY / (ms_tf32 / 1000.0), "unit": "queries/s",
                           "form": "tf32 tcgen05 screen (kind::tf32, operands rounded to tf32) "
                                   "+ the same certify pass",
                           "ms_per_step": ms_tf32, "screen_ms": tf32_screen_ms,
                           "screen_tflops": flops / (tf32_screen_ms * 1e-3) / 1e12,
                           "screen_frac_of_tf32_peak":
                               flops / (tf32_screen_ms * 1e-3) / 1e12 / tf32_peak,
                           "tf32_peak_source": f"half the {peak_kind} burst bf16 figure",
                           "candidates_per_query": st_tf32[-1]["candidates"] / N_QUERY,
                           "bf16_speedup": ms_tf32 / ms_bf16},
            "screen_stats": {k: v for k, v in st_bf16[-1].items()},
            "e2e": {"value": ws * N_QUERY / e2e_s, "unit": "queries/s",
                    "h2d_bytes_per_step": int(Qh.nbytes),
                    "d2h_bytes_per_step": int(out_i.nbytes + out_d.nbytes)},
            "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "clocks": clocks,
        }
        result.update(headline_cpu_baseline(X, Q, index))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if result is not None and ws == 1 and args.workload == "all":
        result["secondary"] = run_secondaries(args)
    if result is not None:
        print(json.dumps(result), flush=True)
    return 0


def headline_cpu_baseline(X, Q, index):
    """The reference's stock route on a bounded sample (~10 s of CPU work),
    and every query it answered compared with ours."""
    threads = host_threads()
    seconds = float(os.environ.get("B2K_CPU_SECONDS", "10"))
    nb = reference_neighbors()
    if nb is not None:
        est = nb.NearestNeighbors(n_neighbors=K, algorithm="brute").fit(X)
        qps, rd, ri, done = stock_kneighbors(est, Q, 256, seconds, 4096)
        kind, route = "reference", ("NearestNeighbors(n_neighbors=10, algorithm='brute')."
                                    "kneighbors, installed reference (CPUIndex route)")
    else:
        done = 16 * threads
        t0 = time.perf_counter()
        rd, ri, kind = native_kneighbors(X, Q[:done], K, threads)
        qps = done / (time.perf_counter() - t0)
        route = "the reference's native exact scan"
    od, oi = index.query(Q[:done], K, mode="bf16")
    return {
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": kind,
                         "sample": f"first {done} queries of the batch in blocks of 256 "
                                   f"through {route}"},
        "parity_vs_cpu_reference": {"queries": int(done),
                                    "indices_bit_exact": bool(np.array_equal(oi, ri)),
                                    "max_rel_dist_err": rel_err(od, rd)},
    }


# ---------------------------------------------------------------------------
# Secondary configurations (nested under "secondary"; --workload NAME alone)
# ---------------------------------------------------------------------------

def _steps(args, cap=10):
    return max(1, min(args.steps, cap)), max(3, min(args.warmup, 5))


def sec_small(args):
    """Config 1: NearestNeighbors(n_neighbors=5, brute) on 10,000 x 64 N(0,1)
    rows (seed 0), 2,000 queries (seed 1)."""
    import torch

    import oracle
    from datasets import cfg1
    from mlxlearn_b200.neighbors import NearestNeighbors

    X, Q = cfg1()
    k = 5
    steps, warmup = _steps(args)
    nn = NearestNeighbors(n_neighbors=k, algorithm="brute", metric="euclidean").fit(X)
    index = nn._index_
    Qd = torch.from_numpy(Q).cuda()
    flush = L2Flush(Qd.device)
    ms = statistics.median(event_times(lambda: index.query_device(Qd, k), steps, warmup, flush))
    index.query_device(Qd, k, stats=True)
    st = index.last_stats
    e2e_s = statistics.median(wall_times(lambda: nn.kneighbors(Q), steps, warmup))
    od, oi = nn.kneighbors(Q)
    tf_burst, _, _, peak_kind = peaks()
    line = {
        "metric": "NearestNeighbors(n_neighbors=5).kneighbors queries/s, 10000 x 64",
        "value": len(Q) / (ms / 1000), "unit": "queries/s", "ms_per_step": ms,
        "steps": steps, "warmup": warmup, "dtype": "bf16" if st["mode_used"] == 2 else "f32",
        "config": {"workload": "knn_gauss_10000x64_2000q_k5",
                   "l2": "inputs smaller than L2: L2 flushed (256 MB write) before every step"},
        "roofline": tensor_roofline("screen_tc_kernel (launch/latency bound at this size)",
                                    2.0 * X.shape[0] * X.shape[1] * len(Q),
                                    st["screen_ms"] * 1e-3, tf_burst, peak_kind),
        "e2e": {"value": len(Q) / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": Q.nbytes,
                "d2h_bytes_per_step": oi.nbytes + od.nbytes,
                "api": "NearestNeighbors.kneighbors (host arrays)"},
    }
    threads = host_threads()
    nb = reference_neighbors()
    ed, ei = oracle.knn(X, Q, k)
    if nb is not None:
        est = nb.NearestNeighbors(n_neighbors=k, algorithm="brute", metric="euclidean").fit(X)
        est.kneighbors(Q[:64])
        t0 = time.perf_counter()
        rd, ri = est.kneighbors(Q)
        cpu_s, kind = time.perf_counter() - t0, "reference"
    else:
        t0 = time.perf_counter()
        rd, ri, kind = native_kneighbors(X, Q, k, threads)
        cpu_s = time.perf_counter() - t0
    line["cpu_baseline"] = {"value": len(Q) / cpu_s, "unit": "queries/s", "cores": threads,
                            "kind": kind, "sample": "all 2000 queries, NearestNeighbors(brute)"
                                                    ".kneighbors of the installed reference"}
    line["parity"] = {"queries": len(Q), "indices_bit_exact_vs_reference":
                      bool(np.array_equal(oi, ri)),
                      "max_rel_dist_err_vs_reference": rel_err(od, rd),
                      "indices_bit_exact_vs_fp64_oracle": bool(np.array_equal(oi, ei)),
                      "max_rel_dist_err_vs_fp64_oracle": rel_err(od, ed)}
    return line


def sec_pixels(args):
    """Config 2b: 60,000 x 784 integer pixels, 10,000 queries, k = 5."""
    import torch

    import oracle
    from datasets import cfg2b
    from mlxlearn_b200.neighbors import KNeighborsClassifier

    X, Q, y = cfg2b()
    k = 5
    steps, warmup = _steps(args)
    clf = KNeighborsClassifier(n_neighbors=k).fit(X, y)
    index = clf._index_
    Qd = torch.from_numpy(Q).cuda()
    flush = L2Flush(Qd.device)
    # AUTO: integer pixels take the exact u8 screen (kind::i8, no certified band)
    ms = statistics.median(event_times(lambda: index.query_device(Qd, k), steps, warmup,
                                       flush))
    index.query_device(Qd, k, stats=True)
    st = index.last_stats
    # the certified bf16 screen on the same data, for comparison
    ms_bf16 = statistics.median(event_times(lambda: index.query_device(Qd, k, mode="bf16"),
                                            steps, warmup, flush))
    index.query_device(Qd, k, mode="bf16", stats=True)
    st_bf16 = index.last_stats
    e2e_s = statistics.median(wall_times(lambda: clf.predict(Q), steps, warmup))
    pred = clf.predict(Q)
    tf_burst, _, _, peak_kind = peaks()
    ops = 2.0 * X.shape[0] * X.shape[1] * len(Q)
    u8 = st["mode_used"] == 5
    roof = tensor_roofline(
        "screen_tc_kernel (u8 tcgen05 kind::i8 distance tile, exact)" if u8 else
        "screen_tc_kernel (bf16 tcgen05 distance tile)", ops, st["screen_ms"] * 1e-3,
        2 * tf_burst if u8 else tf_burst, peak_kind,
        "burst bf16 x 2 (the dense int8 tensor rate is twice bf16's; no int8 figure is "
        "measured)" if u8 else "burst bf16")
    if u8:
        roof["unit"] = "TOP/s"
    line = {
        "metric": "kneighbors queries/s (k=5), 60000 x 784 integer pixels; e2e = "
                  "KNeighborsClassifier.predict",
        "value": len(Q) / (ms / 1000), "unit": "queries/s", "ms_per_step": ms,
        "steps": steps, "warmup": warmup, "dtype": "u8" if u8 else "bf16",
        "config": {"workload": "knn_pixels_60000x784_10000q_k5",
                   "l2": "u8 operand 54 MB, bf16 operand 94 MB: L2 flushed (256 MB write) "
                         "before every step"},
        "roofline": roof,
        "screen_stats": st,
        "certified_bf16": {"value": len(Q) / (ms_bf16 / 1000), "unit": "queries/s",
                           "ms_per_step": ms_bf16, "screen_stats": st_bf16,
                           "form": "bf16 tcgen05 screen + certified re-rank on the same data"},
        # downloaded per step: float64 votes [m, classes] and int64 predictions [m]
        "e2e": {"value": len(Q) / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": Q.nbytes,
                "d2h_bytes_per_step": len(Q) * (len(clf.classes_) + 1) * 8,
                "api": "KNeighborsClassifier.predict (host arrays; votes on the device)"},
    }
    threads = host_threads()
    nb = reference_neighbors()
    sample = min(len(Q), int(os.environ.get("B2K_PIXELS_CPU_QUERIES", "2000")))
    od, oi = clf.kneighbors(Q[:sample])
    ed, ei = oracle.knn(X, Q[:200], k)
    if nb is not None:
        ref = nb.KNeighborsClassifier(n_neighbors=k).fit(X, y)
        ref.predict(Q[:64])
        t0 = time.perf_counter()
        rpred = ref.predict(Q[:sample])
        cpu_s, kind = time.perf_counter() - t0, "reference"
        rd, ri = ref.kneighbors(Q[:sample])
        pred_equal = bool(np.array_equal(pred[:sample], rpred))
    else:
        t0 = time.perf_counter()
        rd, ri, kind = native_kneighbors(X, Q[:sample], k, threads)
        cpu_s, pred_equal = time.perf_counter() - t0, None
    line["cpu_baseline"] = {"value": sample / cpu_s, "unit": "queries/s", "cores": threads,
                            "kind": kind, "sample": f"first {sample} queries, "
                                                    "KNeighborsClassifier(5).predict of the "
                                                    "installed reference"}
    line["parity"] = {"queries": sample, "indices_bit_exact_vs_reference":
                      bool(np.array_equal(oi, ri)),
                      "max_rel_dist_err_vs_reference": rel_err(od, rd),
                      "predictions_equal_reference": pred_equal,
                      "indices_bit_exact_vs_fp64_oracle_200q":
                          bool(np.array_equal(oi[:200], ei)),
                      "max_rel_dist_err_vs_fp64_oracle_200q": rel_err(od[:200], ed)}
    return line


def sec_radius(args):
    """Config 3: RadiusNeighborsClassifier on 200,000 x 32 (10-class mixture),
    50,000 queries, radius = median 50th-neighbour distance of 1,000 queries."""
    import oracle
    from datasets import cfg3
    from mlxlearn_b200.index import build_index
    from mlxlearn_b200.neighbors import RadiusNeighborsClassifier
    from mlxlearn_b200.radius_result import join_batches

    X, y, Q = cfg3()
    steps, warmup = _steps(args, cap=5)
    index = build_index(X)
    d50, _ = index.query(Q[:1000], 50)
    r = float(np.median(d50[:, -1]))
    clf = RadiusNeighborsClassifier(radius=r, outlier_label="most_frequent").fit(X, y)
    csr_s = statistics.median(wall_times(lambda: clf._index_.query_radius_csr(Q, r),
                                         steps, warmup))
    e2e_s = statistics.median(wall_times(lambda: clf.predict(Q), steps, warmup))
    pred = clf.predict(Q)
    ip, ix, dd = join_batches(clf._index_.query_radius_csr(Q, r))
    tf_burst, _, hbm, peak_kind = peaks()
    nnz = int(ip[-1])
    lengths = np.diff(ip)
    # HBM roofline of the whole call: the bf16 index streamed once by the
    # single screen pass plus 16 B per returned neighbour, over the call time
    moved = X.shape[0] * 64 + 16 * nnz
    line = {
        "metric": "radius neighbourhoods (CSR) queries/s, 200000 x 32; e2e = "
                  "RadiusNeighborsClassifier.predict",
        "value": len(Q) / csr_s, "unit": "queries/s", "ms_per_step": 1000 * csr_s,
        "steps": steps, "warmup": warmup, "dtype": "bf16",
        "config": {"workload": "radius_200000x32_50000q", "radius": r,
                   "median_neighbours": float(np.median(lengths)),
                   "zero_neighbour_queries": int((lengths == 0).sum()), "nnz": nnz,
                   "value_note": "query_radius_csr through the host C ABI (upload, one "
                                 "screen pass into capped lists, exact classify, CSR "
                                 "download)"},
        "roofline": {"kernel": "whole radius call", "bound": "tensor",
                     "achieved": 2.0 * X.shape[0] * X.shape[1] * len(Q) / csr_s / 1e12,
                     "peak": tf_burst, "unit": "TFLOP/s",
                     "frac": 2.0 * X.shape[0] * X.shape[1] * len(Q) / csr_s / 1e12 / tf_burst,
                     "peak_source": f"{peak_kind} burst bf16", "traffic": None,
                     "hbm_gbs_of_call": moved / csr_s / 1e9},
        # downloaded per step: int64 class codes and int64 neighbour counts [m]
        "e2e": {"value": len(Q) / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": Q.nbytes,
                "d2h_bytes_per_step": len(Q) * 2 * 8,
                "api": "RadiusNeighborsClassifier.predict (host arrays; class counts and "
                       "their argmax on the device)"},
    }
    threads = host_threads()
    nb = reference_neighbors()
    sample = min(len(Q), int(os.environ.get("B2K_RADIUS_CPU_QUERIES", "4000")))
    ip_s = ip[:sample + 1]
    ix_s, dd_s = ix[:ip_s[-1]], dd[:ip_s[-1]]
    eip, eix, edd = oracle.radius(X, Q[:500], r)
    oracle_ok = (bool(np.array_equal(ip[:501], eip)) and bool(np.array_equal(ix[:eip[-1]], eix))
                 and bool(np.array_equal(dd[:eip[-1]], edd)))
    if nb is not None:
        ref = nb.RadiusNeighborsClassifier(radius=r, outlier_label="most_frequent").fit(X, y)
        ref.predict(Q[:64])
        t0 = time.perf_counter()
        rpred = ref.predict(Q[:sample])
        cpu_s, kind = time.perf_counter() - t0, "reference"
        rd, ri = ref.radius_neighbors(Q[:sample])
        rl = np.array([len(a) for a in ri], np.int64)
        rip = np.concatenate([[0], np.cumsum(rl)])
        csr_ok = (bool(np.array_equal(rip, ip_s)) and
                  bool(np.array_equal(np.concatenate(ri), ix_s)))
        err = rel_err(dd_s, np.concatenate(rd))
        pred_equal = bool(np.array_equal(pred[:sample], rpred))
    else:
        t0 = time.perf_counter()
        rip, rix, rdd = oracle.radius(X, Q[:sample], r, nthreads=threads)
        cpu_s, kind = time.perf_counter() - t0, "port"
        csr_ok = bool(np.array_equal(rip, ip_s)) and bool(np.array_equal(rix, ix_s))
        err, pred_equal = rel_err(dd_s, rdd), None
    line["cpu_baseline"] = {"value": sample / cpu_s, "unit": "queries/s", "cores": threads,
                            "kind": kind, "sample": f"first {sample} queries, "
                                                    "RadiusNeighborsClassifier.predict of the "
                                                    "installed reference"}
    line["parity"] = {"queries": sample, "csr_indices_bit_exact_vs_reference": csr_ok,
                      "max_rel_dist_err_vs_reference": err,
                      "predictions_equal_reference": pred_equal,
                      "csr_bit_exact_vs_fp64_oracle_500q": oracle_ok}
    return line


def sec_batch(args):
    """Config 4: 256 uneven problems (seed 5) as one planned batch (one CUDA
    graph) vs one call per problem."""
    import torch

    from datasets import cfg4
    from mlxlearn_b200.batch import KnnBatch
    from mlxlearn_b200.index import build_index

    torch.cuda.set_device(0)
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
    if args.profile:  # profiling driver: the batched runs only
        for _ in range(args.warmup + args.steps):
            batch.run()
        out = {"profile": True, "stats": batch.finish()}
        batch.close()
        return out
    steps, warmup = _steps(args)
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        batch.run()
    batch.finish()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        clk.begin()
        ev0.record(stream)
        for _ in range(steps):
            batch.run()
        ev1.record(stream)
        stats = batch.finish()
        torch.cuda.synchronize()
        clk.end()
    ms = ev0.elapsed_time(ev1) / steps
    # one call per problem through the single-problem device API
    for ix, q, (_, _, k) in zip(indexes, Qd, problems):
        ix.query_device(q, k)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for ix, q, (_, _, k) in zip(indexes, Qd, problems):
        ix.query_device(q, k)
    torch.cuda.synchronize()
    one_s = time.perf_counter() - t0
    # e2e: page-locked host queries in, results out, through the batch object
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

    e2e_s = statistics.median(wall_times(e2e_step, steps, 1))
    h2d = sum(q.numel() * 4 for q in Qh)
    d2h = sum(d.numel() * 8 for d in Dh) + sum(i.numel() * 8 for i in Ih)
    # CPU baseline + parity: the reference's stock kneighbors on the first
    # queries of every problem, time scaled by each problem's query count
    threads = host_threads()
    nb = reference_neighbors()
    per = int(os.environ.get("B2K_BATCH_CPU_QUERIES", "4"))
    est_cpu_s, sample_q, exact, rel = 0.0, 0, True, 0.0
    kind = "reference"
    for (X, Q, k), d, i in zip(problems, batch.dist, batch.idx):
        s = min(per, Q.shape[0])
        if nb is not None:
            est = nb.NearestNeighbors(n_neighbors=k, algorithm="brute").fit(X)
            t1 = time.perf_counter()
            rd, ri = est.kneighbors(Q[:s])
            el = time.perf_counter() - t1
        else:
            t1 = time.perf_counter()
            rd, ri, kind = native_kneighbors(X, Q[:s], k, min(threads, s))
            el = time.perf_counter() - t1
        est_cpu_s += el * Q.shape[0] / s
        sample_q += s
        exact &= bool(np.array_equal(ri, i[:s].cpu().numpy()))
        rel = max(rel, rel_err(d[:s].cpu().numpy(), rd))
    tf_burst, tf_sust, hbm, peak_kind = peaks()
    line = {
        "metric": "batched uneven kNN: aggregate queries/s, 256 problems (one graph) vs one "
                  "call per problem",
        "value": total_q / (ms / 1000), "unit": "queries/s", "steps": steps, "warmup": warmup,
        "ms_per_step": ms, "dtype": "bf16", "data": "synthetic: cfg4 recipe (seed 5)",
        "config": {"workload": f"knn_batch_{len(problems)}_uneven_seed5",
                   "problems": len(problems), "queries": total_q, "flops": flops,
                   "l2": "operands 1.9 GB bf16, larger than L2"},
        "one_call_per_problem": {"value": total_q / one_s, "unit": "queries/s",
                                 "ms_per_step": 1000 * one_s,
                                 "batch_speedup": one_s / (ms / 1000)},
        "roofline": tensor_roofline("whole batched run (prep, screens, certify, exact)", flops,
                                    ms * 1e-3, tf_burst, peak_kind),
        "batch_stats": stats, "fit_s": fit_s, "plan_s": plan_s,
        "e2e": {"value": total_q / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "cpu_baseline": {"value": total_q / est_cpu_s, "unit": "queries/s", "cores": threads,
                         "kind": kind,
                         "sample": f"first {per} queries of every problem through the "
                                   "installed reference's NearestNeighbors(brute).kneighbors, "
                                   "time scaled by each problem's query count"},
        "parity": {"queries": sample_q, "indices_bit_exact_vs_reference": exact,
                   "max_rel_dist_err_vs_reference": rel},
        "clocks": clk.summary(),
    }
    batch.close()
    return line


def sec_chamfer(args):
    """Config 5: 64 symmetric k=1 Chamfer terms on 8192 x 3 clouds plus a self
    k=8 mean-distance term on 4096 x 64, forward + hand-written backward."""
    import torch

    from datasets import cfg5
    from mlxlearn_b200.autograd import chamfer_loss_batch, knn_distances, knn_segments

    torch.cuda.set_device(0)
    threads = host_threads()
    clouds, S = cfg5()
    steps, warmup = _steps(args)
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

    step_ms = [1000 * s for s in wall_times(step, steps, warmup)]
    loss = step()
    torch.cuda.synchronize()
    s = statistics.median(step_ms) / 1000
    # FP32 CUDA-core roofline of the forward scan: 3 d + 1 FLOP per pair (d = 3)
    cham_pairs = sum(2 * a.shape[0] * b.shape[0] for a, b in clouds)
    achieved = (cham_pairs * 10 + S.shape[0] ** 2 * 2 * S.shape[1]) / s / 1e12
    nb = reference_neighbors()
    cpu_pairs, cpu_s, exact, err = 0, 0.0, True, 0.0
    for a, b in clouds[:2]:
        for P, Qr in ((a, b), (b, a)):
            t0 = time.perf_counter()
            if nb is not None:
                rdist, ridx = nb.NearestNeighbors(n_neighbors=1, algorithm="brute").fit(
                    P).kneighbors(Qr)
                kind = "reference"
            else:
                rdist, ridx, kind = native_kneighbors(P, Qr, 1, threads)
            Pt = torch.from_numpy(P).double().requires_grad_()
            Qt = torch.from_numpy(Qr).double().requires_grad_()
            ((Qt - Pt[torch.from_numpy(ridx[:, 0])]) ** 2).sum().backward()
            cpu_s += time.perf_counter() - t0
            cpu_pairs += len(P) * len(Qr)
            gd, gi = knn_segments(torch.from_numpy(Qr).cuda(), torch.from_numpy(P).cuda(),
                                  [len(Qr)], [len(P)], 1)
            exact &= bool(np.array_equal(gi.cpu().numpy(), ridx))
            err = max(err, rel_err(gd.double().cpu().numpy(), rdist))
    return {
        "metric": "differentiable kNN: (query, reference) pairs/s, forward + backward "
                  "(64 Chamfer k=1 pairs of 8192x3 + self k=8 on 4096x64)",
        "value": pairs / s, "unit": "pairs/s", "steps": steps, "warmup": warmup,
        "ms_per_step": 1000 * s, "dtype": "f32",
        "data": "synthetic: cfg5 recipe (seed 6)",
        "config": {"workload": "knn_chamfer_64x8192x3_self4096x64", "pairs_per_step": pairs,
                   "api": "mlxlearn_b200.autograd (public), wall clock with device sync"},
        "roofline": {"kernel": "whole step (segment scans, backward)", "bound": "fp32 cores",
                     "achieved": achieved, "peak": FP32_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                     "frac": achieved / FP32_NOMINAL_TFLOPS,
                     "peak_source": "nominal fp32 CUDA-core rate at 1965 MHz (no measured "
                                    "figure)", "traffic": None},
        "e2e": {"value": pairs / s, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8,
                "note": "inputs stay on the device (a training loop's tensors); the loss "
                        "value is read back every step"},
        "loss": float(loss.item()), "step_ms": step_ms,
        "cpu_baseline": {"value": cpu_pairs / cpu_s, "unit": "pairs/s", "cores": threads,
                         "kind": kind,
                         "sample": "2 Chamfer pairs both ways: the installed reference's "
                                   "kneighbors forward, torch float64 CPU autograd backward"},
        "parity": {"pairs": 4, "indices_bit_exact_vs_reference": exact,
                   "max_rel_dist_err_vs_reference": err,
                   "note": "forward k=1 of 2 Chamfer pairs, both directions; distances are "
                           "float32 outputs of the autograd path"},
    }


SECONDARY = {"small": sec_small, "pixels": sec_pixels, "radius": sec_radius,
             "batch": sec_batch, "chamfer": sec_chamfer}


def run_secondaries(args):
    out = {}
    for name, fn in SECONDARY.items():
        t0 = time.perf_counter()
        try:
            out[name] = fn(args)
        except Exception as e:  # one configuration's failure must not hide the others
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = time.perf_counter() - t0
    return out


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="all", choices=["all", "knn", *SECONDARY])
    ap.add_argument("--profile", action="store_true",
                    help="profiling driver: only the device steps of the headline workload "
                         "(or of --workload batch)")
    ap.add_argument("--mode", default="bf16", choices=["bf16", "tf32", "fp32", "exact", "auto"],
                    help="screen form for --profile")
    ap.add_argument("--k", type=int, default=K, help="neighbours for --profile")
    ap.add_argument("--problems", type=int, default=256,
                    help="problem count of the batch workload (the benchmark uses 256)")
    ap.add_argument("--queries", type=int, default=N_QUERY,
                    help="query count for --profile (the headline uses 100,000)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload in SECONDARY:
        import torch

        torch.cuda.set_device(0)
        line = SECONDARY[args.workload](args)
        line.setdefault("n_gpus", 1)
        line.update({"higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                     "workload_kind": "secondary"})
        print(json.dumps(line), flush=True)
        return 0
    if args.profile:
        return run_profile(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
