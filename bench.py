#!/usr/bin/env python3
"""Benchmark of the certified exact epsilon-join on B200.

Headline workload (N=1): the high-dimensional R-S join, |R| = |S| = 500,000, d = 512,
rank-32 factor model + N(0, 0.1^2), rows L2-normalised, eps for ~8 neighbours,
BF16 tensor-core screen (the tuning table's choice; the same join with the FP16 screen is
timed beside it) + certified band + FP64 refinement, pair set bit-exact to the FP64 oracle.  This is the configuration the >= 5x target against the plain FP32
direct-difference GPU join is stated on.  Data are seeded synthetic arrays with
those shapes and distributions.

One step = one complete join through the library: index build (Morton sort, operand
and certificate metadata, tile statistics), candidate tile pairs, tensor-core screen,
FP64 refinement of the band, radix sort into canonical order and decoding into the
sorted (i, j) device arrays.  Inputs are resident in HBM (2 x 1 GiB FP32, larger than
the 126 MB L2, so no separate L2 flush is needed).

metric: distance evaluations per second (candidate pairs screened / step time),
        whole job over all ranks; ms_per_step is the join wall time.
e2e:    the same metric through the public API with host (pinned) inputs and host
        outputs: H2D of R and S and D2H of the (i, j) result inside the timed region.
parity: after the timed steps, complete result rows of a seeded sample of R rows are
        recomputed by the CPU oracle (FP64 sequential k, or exact int64) against all of S
        and compared key for key with the GPU result restricted to those rows, and every
        emitted pair's distance is recomputed by the oracle and checked against T.
configs: the default run (N=1) also measures the other four configurations (mixture,
        int14 self-join, ragged batch, 20k x 16 plain grid), each with its own timing,
        clocks, roofline, plain-GPU comparison, end-to-end time, CPU baseline and parity audit.
--impl reference: the reference's own exact CPU path (SciPy cdist 'sqeuclidean' on
        FP64-widened rows + <= T, all host cores) on a bounded row sample per step.
Multi-GPU: one process per GPU (torchrun), independent replicas of the workload
(the join is single-GPU by design); max step time over ranks; scaling "weak".
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "dist_evals_per_s"
UNIT = "pairs/s"
WORKLOADS = {
    "factor512": dict(fn="factor512", screen="bf16", mode="rs", audit_rows=1024),
    "mixture64": dict(fn="mixture64", screen="bf16x3", mode="rs", audit_rows=2048),
    "uniform16": dict(fn="uniform16", screen="plain", mode="upper", audit_rows=0),   # 0: exhaustive
    "int14x128": dict(fn="int14x128", screen="int8limb", mode="upper", audit_rows=2048),
    "ragged4096": dict(fn="ragged4096", screen="bf16x3", mode="rs", audit_rows=64),   # joins checked
}
SUB_CONFIGS = ["mixture64", "int14x128", "ragged4096", "uniform16"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="factor512")
    ap.add_argument("--screen", default=None, help="override the workload's screen (plain/bf16/fp16/int8limb)")
    ap.add_argument("--n", type=int, default=0, help="rows per side (0 = the configuration's size)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 GPU baseline run")
    ap.add_argument("--index-frame", default="auto", choices=["auto", "axes", "pca"],
                    help="cells the rows are sorted by before tiling (default: the library's choice)")
    ap.add_argument("--band-fp32", action="store_true", help="certified FP32 band stage before the FP64 terminal")
    ap.add_argument("--untuned", action="store_true",
                    help="library defaults instead of the committed tuning table's knobs for each configuration")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle audit after the timed steps")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the other 16-bit operand format's run on the headline join")
    ap.add_argument("--configs", default="auto", choices=["auto", "none"],
                    help="auto: a default single-GPU run also measures the other configurations")
    ap.add_argument("--sub-steps", type=int, default=5, help="timed steps of each other configuration")
    ap.add_argument("--cpu-rows", type=int, default=128, help="R rows in the CPU baseline sample")
    ap.add_argument("--ref-rows", type=int, default=48, help="R rows per step of --impl reference")
    return ap.parse_args()


def make_workload(name: str, n: int):
    from tensorjoin_variants_b200 import workloads as W

    spec = WORKLOADS[name]
    fn = getattr(W, spec["fn"])
    return fn(n=n) if n else fn()


# ---------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampler running during the timed region (reads settings only)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.idx = gpu_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # nvidia-smi's start-up (driver queries of every GPU) can hold up this process's CUDA calls
        # for hundreds of ms: let it write its first sample before the timed region begins
        t0 = time.time()
        while time.time() - t0 < 2.0 and self.proc.poll() is None:   # bounded: output may be buffered
            self.file.flush()
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.02)
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


def gpu_uuid() -> str:
    import torch

    try:
        return "GPU-" + str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
    except Exception:
        return str(torch.cuda.current_device())


def max_over_ranks(x: float, world: int, dist, device: str = "cuda") -> float:
    """The largest of every rank's `x` (all ranks call this at the same point)."""
    if world <= 1:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs"), "tflops": d.get("bf16_tflops"),
                "tflops_sustained": d.get("bf16_tflops_sustained"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "tflops": 1590.0, "tflops_sustained": 1400.0, "source": "fallback"}


_INT8_PEAK = None


def int8_peak_tops() -> dict:
    """Dense INT8 tensor throughput of this GPU, measured here: torch._int_mm (a cuBLAS int8 GEMM,
    int32 accumulate) at 8192^3, 10 timed launches after 3 warm-ups, CUDA events.  Only the
    denominator of the int8 screen's roofline fraction; the screen never calls it."""
    global _INT8_PEAK
    if _INT8_PEAK is not None:
        return _INT8_PEAK
    import torch

    n = 8192
    a = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda").t()
    for _ in range(3):
        torch._int_mm(a, b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    reps = 10
    for _ in range(reps):
        torch._int_mm(a, b)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    _INT8_PEAK = {"tops": 2.0 * n ** 3 / (ms / 1000.0) / 1e12, "ms": ms,
                  "source": "measured here: torch._int_mm int8 GEMM 8192^3, burst"}
    del a, b
    torch.cuda.empty_cache()
    return _INT8_PEAK


def committed_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/traffic.txt)."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload and not line.startswith("#"):
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------- oracle audit
def _keys_np(keys_t) -> np.ndarray:
    return keys_t.cpu().numpy().view(np.uint64)


def parity_audit(R: np.ndarray, S: np.ndarray | None, T, mode: str, keys: np.ndarray, rows: int,
                 seed: int = 2024) -> dict:
    """Audit one GPU result against the CPU oracle (outside every timed region).

    (i) complete rows: a seeded sample of `rows` R rows (all rows when rows == 0) joined by the
        oracle against all of S; the GPU keys that touch those rows must be exactly that set
        (self-joins: every pair with either end in the sample, i < j);
    (ii) every emitted pair: its distance recomputed by the oracle must be <= T.
    Pairs are canonical keys i * n_cols + j."""
    import oracle

    t0 = time.perf_counter()
    is_int = R.dtype == np.int16
    Sx = R if S is None else S
    n_cols = Sx.shape[0]
    nc = np.uint64(n_cols)
    gi = (keys // nc).astype(np.int64)
    gj = (keys % nc).astype(np.int64)
    rng = np.random.default_rng(seed)
    if rows <= 0 or rows >= R.shape[0]:
        sample = np.arange(R.shape[0], dtype=np.int64)
    else:
        sample = np.sort(rng.choice(R.shape[0], rows, replace=False)).astype(np.int64)
    sub = R[sample]
    part = oracle.join_i16(sub, Sx, int(T), "rs") if is_int else oracle.join_f32(sub, Sx, float(T), "rs")
    ii = sample[(part // nc).astype(np.int64)]
    jj = (part % nc).astype(np.int64)
    if mode == "rs":
        want = ii.astype(np.uint64) * nc + jj.astype(np.uint64)
        sel = np.isin(gi, sample)
    else:   # self-join (upper): the neighbours of a sampled point on either side of the diagonal
        keep = jj != ii
        lo, hi = np.minimum(ii[keep], jj[keep]), np.maximum(ii[keep], jj[keep])
        want = np.unique(lo.astype(np.uint64) * nc + hi.astype(np.uint64))
        sel = np.isin(gi, sample) | np.isin(gj, sample)
    got = np.unique(keys[sel])
    want = np.unique(want)
    missing = int(np.setdiff1d(want, got, assume_unique=True).size)
    extra = int(np.setdiff1d(got, want, assume_unique=True).size)
    d2 = oracle.pair_d2_mt(R, Sx, gi, gj)
    over = int(np.count_nonzero(d2 > T))
    dup = int(keys.size - np.unique(keys).size) if keys.size < (1 << 27) else None
    return {"rows_checked": int(sample.size), "pairs_checked": int(want.size), "emitted_rechecked": int(keys.size),
            "missing": missing, "extra": extra, "emitted_over_T": over, "duplicates": dup,
            "mismatches": missing + extra + over + (dup or 0),
            "oracle": ("exact int64" if is_int else "FP64 sequential-k") + f" C oracle, {oracle.default_threads()} "
                      "host threads", "seconds": round(time.perf_counter() - t0, 2)}


# ---------------------------------------------------------------------- reference arm
def reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    import oracle

    w = make_workload(args.workload, args.n)
    S = w.R if w.S is None else w.S
    rows = min(args.ref_rows, w.R.shape[0])
    procs = len(os.sched_getaffinity(0))
    rng = np.random.default_rng(7)
    sample = w.R[np.sort(rng.choice(w.R.shape[0], rows, replace=False))]
    pairs, secs, _ = oracle.scipy_rate(sample, S, w.T, procs, rows_per_task=2, repeats=args.warmup + args.steps,
                                       context="fork")
    timed = secs[args.warmup:]
    value = pairs / statistics.mean(timed)
    full_pairs = w.candidate_pairs_all
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.mean(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, args.screen, args.gpus, w),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": f"scipy.spatial.distance.cdist(R64, S64, 'sqeuclidean') <= T (the reference's "
                                   f"exact CPU path) on {rows} seeded R rows x all {len(S)} S rows per step, "
                                   f"{procs} processes; full join extrapolated: "
                                   f"{full_pairs / value:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(name: str, screen: str | None, gpus: int, w) -> dict:
    spec = WORKLOADS[name]
    S = w.R if w.S is None else w.S
    return {"workload": name, "n_rows": int(w.R.shape[0]), "n_cols": int(S.shape[0]),
            "d": int(w.R.shape[1]), "mode": spec["mode"], "screen": screen or spec["screen"],
            "eps": w.eps, "eps2": float(w.T), "target_degree": w.target_degree,
            "l2": "inputs larger than L2 (no flush needed)" if w.R.nbytes > (128 << 20)
            else "inputs smaller than L2: every step re-reads them from L2 (no flush); reported as is",
            "parallelism": f"replicas x{gpus}"}


def screen_roofline(screen: str, d: int, pairs: int, screen_ms: float, issued_ops: float, peaks: dict) -> dict:
    """Roofline of the screen kernel: algorithmic ops (2 d per pair; int8 limbs 8 d per pair, the count
    the scope table fixes) and the ops the kernel actually issues, each over the same kernel time."""
    secs = screen_ms / 1000.0
    if screen == "plain":
        ach = 2.0 * d * pairs / secs / 1e12
        return {"bound": "simt", "kernel": "plain_kernel", "achieved": ach, "peak": None, "unit": "TFLOP/s",
                "frac": None, "screen_ms": screen_ms, "flops_per_launch": 2.0 * d * pairs}
    if screen == "int8limb":
        p8 = int8_peak_tops()
        alg = 8.0 * d * pairs
        ach, iss = alg / secs / 1e12, issued_ops / secs / 1e12
        return {"bound": "tensor", "kernel": "screen_i8_kernel", "achieved": ach, "peak": p8["tops"],
                "unit": "TOP/s", "frac": ach / p8["tops"], "frac_algorithmic": ach / p8["tops"],
                "achieved_issued": iss, "frac_issued": iss / p8["tops"], "peak_source": p8["source"],
                "screen_ms": screen_ms, "ops_per_launch": alg, "issued_ops_per_launch": issued_ops}
    peak = peaks["tflops_sustained"]
    alg = 2.0 * d * pairs
    ach, iss = alg / secs / 1e12, issued_ops / secs / 1e12
    return {"bound": "tensor", "kernel": "screen_tc_kernel", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
            "frac": ach / peak, "frac_algorithmic": ach / peak, "achieved_issued": iss, "frac_issued": iss / peak,
            "peak_source": f"{peaks['source']} bf16_tflops_sustained (dense fp16 = bf16 rate)",
            "screen_ms": screen_ms, "flops_per_launch": alg, "issued_flops_per_launch": issued_ops}


def issued_screen_ops(screen: str, st: dict, d: int) -> float:
    """Tensor-core operations the screen issued: 2 d per screened pair (6 d with the hi/lo split; the
    int8-limb screen reports its own count, which depends on how many items needed the low limbs)."""
    if screen == "int8limb":
        return float(st.get("screen_ops_issued") or st["screen_ops"])
    return (6.0 if screen in ("bf16x3", "fp16x3") else 2.0) * d * st["pairs_screened"]


def cpu_baseline_leg(R: np.ndarray, S: np.ndarray, T, rows: int, full_pairs: int) -> dict:
    import oracle

    rows = min(rows, R.shape[0])
    rng = np.random.default_rng(7)
    sample = R[np.sort(rng.choice(R.shape[0], rows, replace=False))]
    procs = len(os.sched_getaffinity(0))
    cp, secs, _ = oracle.scipy_rate(sample.astype(np.float32), S.astype(np.float32), T, procs, rows_per_task=2,
                                    repeats=1, context="spawn")
    rate = cp / secs[0]
    return {"value": rate, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"scipy cdist sqeuclidean (the reference's exact CPU path), {rows} seeded R "
                      f"rows x all {len(S)} S rows, {procs} spawned processes, "
                      f"{secs[0]:.1f} s; full join extrapolated {full_pairs / rate:.0f} s"}


# ---------------------------------------------------------------------- tuned knobs
def tuned_knobs(args, R, S, T, mode: str, screen: str) -> tuple[dict, str | None]:
    """Knobs the committed B200 tuning table holds for this join and its fixed screen (tile shape,
    half-tile packing, chunking, cell frame, FP32 band stage); {} on a miss or with --untuned.
    --index-frame and --band-fp32 given on the command line win over the table."""
    from tensorjoin_variants_b200 import autotune

    kw: dict = {}
    key = None
    if not args.untuned:
        table = autotune.default_table()
        key = table.key_for(R, S, T, mode, screen)
        choice = table.lookup(key)
        if choice is not None and not choice.screen:
            kw = choice.kwargs()
    if args.index_frame != "auto":
        kw["index_frame"] = args.index_frame
    if args.band_fp32:
        kw["band_fp32"] = True
    return kw, key


def tuned_batch_knobs(args, joins, screen: str) -> tuple[dict, str | None]:
    """The same for a batch of joins (``autotune.Tuner.batch_key``)."""
    from tensorjoin_variants_b200 import autotune

    kw: dict = {}
    key = None
    if not args.untuned:
        table = autotune.default_table()
        key = table.batch_key(joins, screen)
        choice = table.lookup(key)
        if choice is not None and not choice.screen:
            kw = choice.kwargs()
            kw.pop("i8_four_products")
    if args.index_frame != "auto":
        kw["index_frame"] = args.index_frame
    if args.band_fp32:
        kw["band_fp32"] = True
    return kw, key


# ---------------------------------------------------------------------- one single-join configuration
def bench_single(name: str, args, steps: int, warmup: int, rank: int, world: int, dist, headline: bool) -> dict:
    import torch

    import tensorjoin_variants_b200 as tj
    from tensorjoin_variants_b200 import _lib

    spec = WORKLOADS[name]
    screen = (args.screen if headline else None) or spec["screen"]
    mode = spec["mode"]
    w = make_workload(name, args.n if headline else 0)
    R = torch.from_numpy(w.R).cuda()
    S = None if w.S is None else torch.from_numpy(w.S).cuda()
    T = w.T
    d = int(w.R.shape[1])

    knobs, tkey = tuned_knobs(args, R, S, T, mode, screen)

    def step():
        res = tj.join_result(R, S, eps2=T, mode=mode, screen=screen, **knobs)
        i, j = res.pairs()
        return res, i, j

    for _ in range(warmup):
        res, i, j = step()
        del res, i, j
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(gpu_uuid())
    clocks.start()
    launches0 = _lib.lib().tj_kernel_launches()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    stats = []
    count = 0
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for s_ in range(steps):
        res, i, j = step()
        stats.append(res.stats)
        count = res.count
        del res, i, j
        marks[s_].record(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = _lib.lib().tj_kernel_launches() - launches0
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / steps
    step_ms = [(ev0 if k == 0 else marks[k - 1]).elapsed_time(marks[k]) for k in range(steps)]
    ms = max_over_ranks(ms, world, dist)
    if world > 1:
        dist.barrier()
    st = stats[-1]
    pairs = st["pairs_screened"]
    value = world * pairs / (ms / 1000.0)
    peaks = measured_peaks()
    screen_ms = statistics.mean(s["ms_screen"] for s in stats)
    roofline = screen_roofline(screen, d, pairs, screen_ms, issued_screen_ops(screen, st, d), peaks)
    if headline:
        roofline["traffic"] = committed_traffic(roofline["kernel"], name)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"plain": "f32", "int8limb": "s8"}.get(screen, screen), "data": "synthetic",
        "config": workload_config(name, screen, world, w), "roofline": roofline, "clocks": clk,
        "gpu_launches": int(launches), "result_pairs": int(count), "step_ms": step_ms,
        "lib_ms_total": [s["ms_total"] for s in stats],
        "stats": {k: st[k] for k in (
            "pairs_all", "pairs_screened", "tile_pairs", "screen_accept", "band", "refine_accept", "rare_checks",
            "result_pairs", "retries", "ms_index", "ms_candidates", "ms_screen", "ms_refine", "ms_sort", "ms_total",
            "index_frame", "band_fp64")},
    }
    line["stats"]["refined_fraction"] = st["band"] / max(1, st["pairs_screened"])
    line["rates"] = {"all_pairs_equivalent_per_s": world * st["pairs_all"] / (ms / 1000.0),
                     "result_pairs_per_s": world * int(count) / (ms / 1000.0),
                     "pair_space_pruned_fraction": max(0.0, 1.0 - st["pairs_screened"] / max(1, st["pairs_all"]))}
    if screen not in ("plain", "int8limb"):   # screen error vs sequential FP64 on 64 sampled tile pairs
        rd = tj.join_result(R, S, eps2=T, mode=mode, screen=screen, screen_diag=True)
        sd = rd.stats
        line["screen_error"] = {"max_abs_err_d2": sd["screen_max_abs_err"],
                                "max_err_over_certified_radius": sd["screen_err_over_bound"],
                                "pairs_sampled": sd["screen_err_pairs"], "eps2": float(T),
                                "band_pairs": sd["band"], "refined_fraction": sd["band"] / max(1, sd["pairs_screened"])}
        del rd
    elif screen == "int8limb":
        line["screen_error"] = {"max_abs_err_d2": 0, "note": "exact integer screen (int8 limbs, INT64 recombination)"}

    # the GPU result once more, for the plain comparison and the oracle audit
    res = tj.join_result(R, S, eps2=T, mode=mode, screen=screen, **knobs)
    keys_t = res.keys()
    del res

    # plain FP32 direct-difference GPU join over the same candidate tile pairs (the baseline to beat)
    if not args.no_plain and screen != "plain":
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # int14 data run the plain path on exact FP32 copies (same predicate: d2 is exact in FP64)
        Rp = R.float() if R.dtype == torch.int16 else R
        Sp = None if S is None else (S.float() if S.dtype == torch.int16 else S)
        resp = tj.join_result(Rp, Sp, eps2=T, mode=mode, screen="plain")
        kp = resp.keys()
        e1.record(stream)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1)
        line["plain_gpu"] = {"ms_per_step": pms, "value": world * resp.stats["pairs_screened"] / (pms / 1000.0),
                             "speedup_of_tc_path": pms / ms, "identical_pair_set": bool(torch.equal(kp, keys_t)),
                             "ms_screen": resp.stats["ms_screen"],
                             "note": "one run; the same index, candidates, refinement and sort as the "
                                     "tensor-core path, only the screen differs"}
        del resp, kp, Rp, Sp

    # the other unsplit 16-bit operand format on the same join (FP16 against BF16): time, band, screen
    # error against sequential FP64 and whether the pair set is the same
    other = {"fp16": "bf16", "bf16": "fp16"}.get(screen)
    if headline and other and not args.no_compare:
        kwo = {k: v for k, v in knobs.items()}
        for _ in range(2):
            r_ = tj.join_result(R, S, eps2=T, mode=mode, screen=other, **kwo)
            del r_
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k_cmp = 3
        ost = []
        e0.record(stream)
        for _ in range(k_cmp):
            r_ = tj.join_result(R, S, eps2=T, mode=mode, screen=other, **kwo)
            ost.append(r_.stats)
            del r_
        e1.record(stream)
        torch.cuda.synchronize()
        oms = e0.elapsed_time(e1) / k_cmp
        ro = tj.join_result(R, S, eps2=T, mode=mode, screen=other, **kwo)
        same = bool(torch.equal(ro.keys(), keys_t))
        del ro
        rd = tj.join_result(R, S, eps2=T, mode=mode, screen=other, screen_diag=True)
        sd = rd.stats
        del rd
        line["screens_compared"] = {
            screen: {"ms_per_step": ms, "ms_screen": screen_ms, "band": st["band"],
                     "refined_fraction": st["band"] / max(1, st["pairs_screened"]),
                     "max_abs_err_d2": line.get("screen_error", {}).get("max_abs_err_d2")},
            other: {"ms_per_step": oms, "ms_screen": statistics.mean(s["ms_screen"] for s in ost),
                    "band": ost[-1]["band"], "refined_fraction": ost[-1]["band"] / max(1, ost[-1]["pairs_screened"]),
                    "max_abs_err_d2": sd["screen_max_abs_err"],
                    "max_err_over_certified_radius": sd["screen_err_over_bound"],
                    "identical_pair_set": same, "steps": k_cmp},
        }

    # end to end through the public API with host buffers (pinned inputs, host outputs)
    if not args.no_e2e:
        Rh = torch.from_numpy(w.R).pin_memory()
        Sh = None if w.S is None else torch.from_numpy(w.S).pin_memory()
        fn = (lambda: tj.join(Rh, Sh, eps2=T, screen=screen, **knobs)) if mode == "rs" else \
            (lambda: tj.self_join(Rh, eps2=T, mode=mode, screen=screen, **knobs))
        for _ in range(max(3, warmup)):   # warm-up: the pinned host buffers reach the allocator's cache
            ih, jh = fn()
        torch.cuda.synchronize()
        k_e2e = max(1, min(steps, 3))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d2h = 0
        for _ in range(k_e2e):   # each step's host outputs are dropped before the next step allocates its own
            ih, jh = fn()
            d2h = 16 * len(ih)
            del ih, jh
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / k_e2e
        ems = max_over_ranks(ems, world, dist)
        h2d = Rh.numel() * Rh.element_size() + (0 if Sh is None else Sh.numel() * Sh.element_size())
        line["e2e"] = {"value": world * pairs / (ems / 1000.0), "unit": UNIT, "ms_per_step": ems,
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "api": ("tensorjoin_variants_b200.join" if mode == "rs" else "tensorjoin_variants_b200.self_join")
                              + "(host pinned inputs) -> host (i, j)"}
        del Rh, Sh

    keys = _keys_np(keys_t)
    del keys_t, R, S
    torch.cuda.synchronize()
    if rank == 0 and world == 1 and not args.no_parity:
        line["parity"] = parity_audit(w.R, w.S, T, mode, keys, spec["audit_rows"])
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_leg(w.R, w.R if w.S is None else w.S, T, args.cpu_rows,
                                                w.candidate_pairs_all)
    return line


# ---------------------------------------------------------------------- config 5: batched ragged joins
def ragged_audit(joins, result, count: int, seed: int = 2025) -> dict:
    """`count` seeded joins of the batch, each checked exhaustively by the CPU oracle against the
    batch result's range for that join (local (i, j) keys i * |S| + j)."""
    import oracle

    t0 = time.perf_counter()
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(len(joins), size=min(count, len(joins)), replace=False))
    parts = result.split()
    mism, pairs, evals = 0, 0, 0
    worst = None
    for k in pick:
        R, S, e = joins[int(k)]
        Rn, Sn = R.cpu().numpy(), S.cpu().numpy()
        i, j = parts[int(k)]
        got = i.cpu().numpy().astype(np.uint64) * np.uint64(Sn.shape[0]) + j.cpu().numpy().astype(np.uint64)
        want = oracle.join_f32(Rn, Sn, e * e, "rs")
        bad = int(np.setdiff1d(got, want).size + np.setdiff1d(want, got).size) if not np.array_equal(got, want) else 0
        if bad and worst is None:
            worst = int(k)
        mism += bad
        pairs += int(want.size)
        evals += int(Rn.shape[0]) * int(Sn.shape[0])
    return {"joins_checked": int(len(pick)), "pairs_checked": pairs, "pair_evaluations": evals,
            "mismatches": mism, "first_bad_join": worst,
            "oracle": f"FP64 sequential-k C oracle, exhaustive per join, {oracle.default_threads()} host threads",
            "seconds": round(time.perf_counter() - t0, 2)}


def bench_ragged(args, steps: int, warmup: int, rank, world, dist, headline: bool) -> dict:
    import torch

    import tensorjoin_variants_b200 as tj
    from tensorjoin_variants_b200 import _lib
    from tensorjoin_variants_b200 import workloads as W

    screen = (args.screen if headline else None) or WORKLOADS["ragged4096"]["screen"]
    scale = (args.n / 11_800 if args.n else 1.0) if headline else 1.0   # --n sets the mean side length
    joins, classes = W.ragged4096_device(size_scale=scale)
    torch.cuda.synchronize()
    nj = len(joins)
    stream = torch.cuda.current_stream()

    knobs, tkey = tuned_batch_knobs(args, joins, screen)

    def step(scr):
        return tj.join_batched_result(joins, screen=scr, **knobs)

    for _ in range(warmup):
        r = step(screen)
        del r
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(gpu_uuid())
    clocks.start()
    l0 = _lib.lib().tj_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    stats = []
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for s_ in range(steps):
        r = step(screen)
        stats.append(r.stats)
        pairs_out = r.count
        del r
        marks[s_].record(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = _lib.lib().tj_kernel_launches() - l0
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / steps
    step_ms = [(e0 if k == 0 else marks[k - 1]).elapsed_time(marks[k]) for k in range(steps)]
    ms = max_over_ranks(ms, world, dist)
    st = stats[-1]
    pairs = st["pairs_screened"]
    peaks = measured_peaks()
    screen_ms = statistics.mean(s["ms_screen"] for s in stats)
    # algorithmic flops 2 d per pair summed over the joins' classes: from the library's count of
    # issued ops, which is 6 d per pair with the hi/lo split and 2 d without
    issued = statistics.mean(s["screen_ops"] for s in stats)
    alg = issued / 3.0 if screen in ("bf16x3", "fp16x3") else issued
    secs = screen_ms / 1000.0
    peak = peaks["tflops_sustained"] if screen != "plain" else None
    roof = {"bound": "tensor" if screen != "plain" else "simt", "kernel": "screen_tc_kernel",
            "achieved": alg / secs / 1e12, "peak": peak, "unit": "TFLOP/s",
            "frac": (alg / secs / 1e12) / peak if peak else None,
            "frac_algorithmic": (alg / secs / 1e12) / peak if peak else None,
            "achieved_issued": issued / secs / 1e12, "frac_issued": (issued / secs / 1e12) / peak if peak else None,
            "peak_source": f"{peaks['source']} bf16_tflops_sustained", "traffic": None,
            "screen_ms": screen_ms, "flops_per_launch": alg, "issued_flops_per_launch": issued}
    # per-join latency: a seeded sample of joins run one at a time through tj.join
    rng = np.random.default_rng(11)
    lat = []
    for k in rng.choice(nj, size=min(128, nj), replace=False):
        R, S, e = joins[int(k)]
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        i, j = tj.join(R, S, e, screen=screen)
        b.record(stream)
        torch.cuda.synchronize()
        lat.append(a.elapsed_time(b))
    line = {
        "metric": METRIC, "value": world * pairs / (ms / 1000.0), "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": screen, "data": "synthetic (seeded, drawn on the GPU)",
        "config": {"workload": "ragged4096", "joins": nj, "rows_r": int(sum(j[0].shape[0] for j in joins)),
                   "rows_s": int(sum(j[1].shape[0] for j in joins)), "dims": [8, 32, 128], "screen": screen,
                   "mean_side": 11_800 * scale, "l2": "inputs larger than L2 (no flush needed)",
                   "parallelism": f"replicas x{world}"},
        "roofline": roof, "clocks": clk, "gpu_launches": int(launches), "result_pairs": int(pairs_out),
        "step_ms": step_ms, "lib_ms_total": [s["ms_total"] for s in stats],
        "stage_ms_per_step": [{k[3:]: round(s[k], 3) for k in ("ms_index", "ms_candidates", "ms_screen", "ms_refine",
                                                               "ms_sort")} for s in stats],
        "batch": {"joins_per_s": nj / (ms / 1000.0), "ms_per_join_amortised": ms / nj,
                  "single_join_latency_ms_p50": float(np.percentile(lat, 50)),
                  "single_join_latency_ms_p99": float(np.percentile(lat, 99)), "latency_sample": len(lat)},
        "stats": {k: st[k] for k in ("pairs_all", "pairs_screened", "tile_pairs", "screen_accept", "band",
                                     "refine_accept", "result_pairs", "retries", "ms_index", "ms_candidates",
                                     "ms_screen", "ms_refine", "ms_sort", "ms_total", "band_fp64")},
    }
    line["stats"]["refined_fraction"] = st["band"] / max(1, st["pairs_screened"])
    if screen != "plain":   # sampled screen error against FP64, outside the timed region
        rd = tj.join_batched_result(joins, screen=screen, screen_diag=True)
        sd = rd.stats
        line["screen_error"] = {"max_abs_err_d2": sd["screen_max_abs_err"],
                                "max_err_over_certified_radius": sd["screen_err_over_bound"],
                                "pairs_sampled": sd["screen_err_pairs"], "band_pairs": sd["band"],
                                "refined_fraction": sd["band"] / max(1, sd["pairs_screened"])}
        del rd
    if screen != "plain":   # per-join spans inside one batched screen launch, and the CTAs' idle tail
        rt_ = tj.join_batched_result(joins, screen=screen, screen_times=True, **knobs)
        stt = rt_.stats
        line["batch"].update({"in_batch_join_span_ms_p50": stt["join_span_ms_p50"],
                              "in_batch_join_span_ms_p99": stt["join_span_ms_p99"],
                              "in_batch_join_span_ms_max": stt["join_span_ms_max"],
                              "screen_cta_tail_ms": stt["screen_cta_tail_ms"],
                              "screen_ms_with_stamps": stt["ms_screen"],
                              "note": "spans: first chunk start to last chunk end of each join inside the screen "
                                      "launch (%globaltimer, an untimed extra run); tail: spread of the CTAs' end "
                                      "times"})
        del rt_
    r = step(screen)
    if not args.no_plain and screen != "plain":
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rp = step("plain")
        b.record(stream)
        torch.cuda.synchronize()
        line["plain_gpu"] = {"ms_per_step": a.elapsed_time(b), "speedup_of_tc_path": a.elapsed_time(b) / ms,
                             "identical_pair_set": bool(torch.equal(rp.keys(), r.keys()))}
        del rp
    if not args.no_e2e:   # host-resident batch: every join's rows from pinned host memory, pairs back to the host
        # (each join's R and S are views of a few pinned host arrays, one per dimension class and side,
        # as a caller holding its batch in a few large arrays has them)
        pins = {X.untyped_storage().data_ptr(): X.cpu().pin_memory() for X in classes}

        def host_view(t):
            P = pins[t.untyped_storage().data_ptr()].view(-1)
            return P[t.storage_offset():t.storage_offset() + t.numel()].view(t.shape)

        hj = [(host_view(Rd), host_view(Sd), e) for Rd, Sd, e in joins]
        for _ in range(max(1, min(warmup, 2))):
            tj.join_batched_result(hj, screen=screen, **knobs).pairs()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        k_e2e = 2
        d2h = 0
        for _ in range(k_e2e):   # each step's host outputs are dropped before the next step allocates its own
            ih, jh = tj.join_batched_result(hj, screen=screen, **knobs).pairs()
            d2h = 16 * len(ih)
            del ih, jh
        b.record(stream)
        torch.cuda.synchronize()
        ems = a.elapsed_time(b) / k_e2e
        h2d = sum(P.numel() * 4 for P in pins.values())
        line["e2e"] = {"value": world * pairs / (ems / 1000.0), "unit": UNIT, "ms_per_step": ems,
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "api": "tensorjoin_variants_b200.join_batched_result(host pinned joins).pairs() -> host (i, j)"}
        del hj, pins
    if rank == 0 and world == 1 and not args.no_parity:
        line["parity"] = ragged_audit(joins, r, WORKLOADS["ragged4096"]["audit_rows"])
    if rank == 0 and world == 1 and not args.no_cpu:   # the reference's CPU path on one seeded join's rows
        k = int(np.random.default_rng(7).integers(nj))
        Rn, Sn, e = joins[k][0].cpu().numpy(), joins[k][1].cpu().numpy(), joins[k][2]
        cb = cpu_baseline_leg(Rn, Sn, e * e, args.cpu_rows, int(st["pairs_all"]))
        cb["sample"] += f" (join {k} of the batch; extrapolated to the batch's {int(st['pairs_all'])} pairs)"
        line["cpu_baseline"] = cb
    del r
    return line


# ---------------------------------------------------------------------- main
def main() -> None:
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch
    import torch.distributed as dist

    from tensorjoin_variants_b200 import _lib

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    if args.workload == "ragged4096":
        line = bench_ragged(args, args.steps, args.warmup, rank, world, dist, True)
    else:
        line = bench_single(args.workload, args, args.steps, args.warmup, rank, world, dist, True)
    # the other configurations under the same clock (default single-GPU run only)
    run_subs = args.configs == "auto" and world == 1 and args.workload == "factor512" and not args.n and \
        not args.screen
    if run_subs:
        subs = {}
        sub_steps, sub_warm = max(1, min(args.steps, args.sub_steps)), max(3, min(args.warmup, 3))
        for name in SUB_CONFIGS:
            _lib.lib().tj_pool_trim(0)
            torch.cuda.empty_cache()
            t0 = time.time()
            try:
                if name == "ragged4096":
                    rec = bench_ragged(args, sub_steps, sub_warm, rank, world, dist, False)
                else:
                    rec = bench_single(name, args, sub_steps, sub_warm, rank, world, dist, False)
            except Exception as exc:   # report the failure in the line; the headline stands
                rec = {"error": f"{type(exc).__name__}: {exc}"}
            rec["wall_s"] = round(time.time() - t0, 1)
            subs[name] = rec
        line["configs"] = subs
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
