"""Benchmark of the epsilon-join cardinality path on B200.

Workload (the configuration the headline metric is quoted on): self-join of
n = 1,000,000 points in d = 64, coordinates i.i.d. uniform [0,1) drawn from
seed 22 and stored as FP32, eps calibrated from the first 10,000 points so
that a point has ~32 neighbours (eps = 2.279504; grid pruning is ineffective,
every one of the n(n-1)/2 pairs is evaluated). A step is one complete join:
cell keys, EGO sort, stripe index, distance kernel, FP64 recheck of the band,
count read back.

Metric: pair-distance evaluations per second = n(n-1)/2 per step / step time.
`value` is measured on inputs already resident in device memory with CUDA
events on the stream the engine runs on; `e2e` through the public C-ABI call
with the input in pinned host memory (host->device copy and the count's
read-back inside the timed region, synchronous calls, host clock).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form tf32|fp16|bf16x3|plain]
    python bench.py --impl reference ...     (the reference's AVX-512 CPU path)

With N > 1 (torchrun), every rank runs its own replica of the workload on its
GPU (weak scaling, no data-path collective); rank 0 prints the line with the
maximum time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 1_000_000
DIM = 64
SEED = 22
NEIGHBOURS = 32
EPS_CALIBRATED = 2.279504  # calibrate_eps(first 10k points, n=1M, 32 neighbours); re-derived at start-up
METRIC = "pair-dist evals/s (self-join 1M x 64, exact count)"
UNIT = "pair-dist evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default=None, choices=["fp16", "tf32", "bf16x3", "plain", "auto"],
                    help="distance form (default: fp16 for the self-join and batch lines, auto for serving)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison step")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-variants", action="store_true", help="skip the other tensor-core forms")
    ap.add_argument("--no-serving", action="store_true", help="skip the shortened serving stream")
    ap.add_argument("--n", type=int, default=N_POINTS, help=argparse.SUPPRESS)
    ap.add_argument("--workload", default="selfjoin", choices=["selfjoin", "serving", "batch", "config"],
                    help="serving: the join-serving stream; config: one benchmark configuration "
                         "(--config) in every form (not the headline line)")
    ap.add_argument("--prefix", type=int, default=0,
                    help="--workload config: use only the first N points of each set (no count check)")
    ap.add_argument("--config", default="cfg4_self_4M_d28_gmm64_nbrs100",
                    help="configuration name for --workload config (hilbertjoin_b200.workloads.CONFIGS)")
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--baseline-requests", type=int, default=200)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload(n: int):
    from hilbertjoin_b200 import workloads as W
    x = W.uniform(n, DIM, SEED, dtype=np.float32)
    eps = W.calibrate_eps(x, N_POINTS, NEIGHBOURS)
    return x, eps


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def mark(self):
        """Start of the timed region: earlier samples are dropped."""
        try:
            self.out.flush()
            self.skip = len(open(self.out.name).read().strip().splitlines())
        except OSError:
            self.skip = 0

    def summary(self):
        try:
            self.out.flush()
            rows = [r.split(",") for r in open(self.out.name).read().strip().splitlines() if r.strip()]
            rows = rows[getattr(self, "skip", 0):]
        except OSError:
            rows = []
        finally:
            try:
                os.unlink(self.out.name)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and "Active" in r[5 + i] and "Not" not in r[5 + i]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# The reference's loops and tables assume whole 8-point blocks: for n % 8 != 0
# its self-term table (hilbertjoin/egojoin.h:178-195, n * blocks doubles,
# written at index (i/8 * blocks + k) * 8 + i%8) is overrun by
# (8 - n%8) * blocks doubles and the process dies. Samples are therefore cut
# to whole 64-point groups.
SAMPLE_ALIGN = 64
CAL_SAMPLE = 20_032


class RefSampler:
    """The reference's own CPU path (built from its sources in oracle/_ref) on
    a bounded sample of the workload: the first n_s points with the same eps
    (still the dense regime: every pair is evaluated). n_s is sized once from
    a calibration run so that one run takes about `budget_s` of ALGTIME; the
    faster of the reference's two KBLOCK builds (4 and 16; its FAQ recommends
    16 for uniform data) is used with every host core. If the sized run fails,
    the calibration sample stands. Without an AVX-512 host or a reference
    build, the oracle's brute-force C port is timed instead (kind "port")."""

    def __init__(self, x: np.ndarray, eps: float, budget_s: float):
        import oracle
        self.oracle = oracle
        self.x = x.astype(np.float64)
        self.eps = eps
        self.cores = os.cpu_count() or 1
        self.avx512 = oracle.host_has_avx512()
        self.kind = "port"
        self.note = ""
        self.kblock = None
        if oracle.pick_ref_binary(4, self.cores) is None:
            self.note = ("no AVX-512 on this host" if not self.avx512 else "reference build missing")
            self.n_s = 6016
            return
        best = None
        for kb in (4, 16):
            try:
                r = self._ref(CAL_SAMPLE, kb)
            except Exception as e:  # keep the other build
                self.note += f"KBLOCK={kb} calibration failed: {e}; "
                continue
            if best is None or r["alg_s"] < best[1]["alg_s"]:
                best = (kb, r)
        if best is None:
            self.n_s = 6016
            return
        self.kind, self.kblock = "reference", best[0]
        rate = (CAL_SAMPLE * (CAL_SAMPLE - 1) / 2) / max(best[1]["alg_s"], 1e-6)
        n_s = int(min(len(self.x), max(CAL_SAMPLE, np.sqrt(2 * rate * budget_s))))
        self.n_s = max(SAMPLE_ALIGN, n_s // SAMPLE_ALIGN * SAMPLE_ALIGN)
        try:
            self._ref(self.n_s, self.kblock)
        except Exception as e:
            self.note += f"sample of {self.n_s} failed ({e}); calibration sample kept; "
            self.n_s = CAL_SAMPLE

    def _ref(self, n_s: int, kb: int) -> dict:
        return self.oracle.ref_self_count(self.x[:n_s], self.eps, stripes=14, kblock=kb, threads=self.cores)

    def run(self) -> dict:
        n_s = self.n_s
        pairs = n_s * (n_s - 1) / 2
        if self.kind == "reference":
            r = self._ref(n_s, self.kblock)
            cores, dt, count = int(r["threads"]), r["alg_s"], r["count"]
            what = (f"test_ego_loop3_macro (reference built from its sources), KBLOCK={self.kblock}, "
                    f"NUM_THREADS={cores}, 14 stripes; time = its ALGTIME (sort + index + join)")
        else:
            t = time.perf_counter()
            count = self.oracle.self_count_brute(self.x[:n_s], self.eps, threads=self.cores)
            dt, cores = time.perf_counter() - t, self.cores
            what = f"FP64 brute-force C port of the path ({self.note.strip() or 'reference unavailable'})"
        return {"value": pairs / dt, "unit": UNIT, "cores": cores, "kind": self.kind,
                "sample": f"first {n_s} points of the workload, same eps (dense: {pairs:.3e} pairs); {what}",
                "host_cores": self.cores, "avx512f": self.avx512, "count": count, "alg_s": dt,
                "note": self.note.strip() or None}


CPU_KEYS = ("value", "unit", "cores", "kind", "sample", "host_cores", "avx512f", "note")


def cpu_baseline(x: np.ndarray, eps: float, budget_s: float = 8.0) -> dict:
    s = RefSampler(x, eps, budget_s)
    return s.run()


def roofline(form: str, kms: float, pairs: float, peaks: dict, peak_src: str) -> dict:
    """Algorithmic FLOP of the distance kernel per launch over its CUDA-event
    time, against the measured peak of the unit the form runs on."""
    if form == "plain":
        flops = 3.0 * DIM * pairs  # direct difference: sub + fma per dim and pair
        roof = {"bound": "fp64", "achieved": flops / (kms / 1e3) / 1e12, "peak": 37.0, "unit": "TFLOP/s",
                "peak_source": "datasheet FP64 37 TFLOP/s (assumption; no measured FP64 peak)"}
    else:
        flops = 2.0 * DIM * pairs  # Gram form: one multiply-add per dim and pair
        sustained = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops"))
        if form == "tf32":
            peak = sustained / 2.0
            src = f"{peak_src} bf16_tflops_sustained / 2 (TF32 dense = half of BF16)"
        elif form == "fp16":
            peak = sustained
            src = f"{peak_src} bf16_tflops_sustained (FP16 dense = BF16 dense)"
        else:
            peak = sustained / 3.0
            src = f"{peak_src} bf16_tflops_sustained / 3 (three BF16 products per algorithmic multiply-add)"
        roof = {"bound": "tensor", "achieved": flops / (kms / 1e3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                "peak_source": src}
    roof["frac"] = roof["achieved"] / roof["peak"]
    roof["kernel"] = "k_join_tc" if form != "plain" else "k_join_fp64"
    roof["kernel_ms"] = kms
    roof["algorithmic_flops_per_launch"] = flops
    roof["traffic"] = None
    return roof


def golden_count(n: int):
    """The FP64 oracle's count for the 1M x 64 workload (brute force over all
    pairs, tests/golden/config_counts.json), or None for other sizes."""
    p = os.path.join(ROOT, "tests", "golden", "config_counts.json")
    if n != N_POINTS or not os.path.exists(p):
        return None
    with open(p) as f:
        c = json.load(f)["configs"].get("cfg3_self_1M_d64_nbrs32")
    return None if c is None else int(c["oracle_count"])


def serving_summary(r):
    """Requests/s and p50/p99 of the shortened serving stream, and the target
    check: >= 3x the plain path's requests/s at an equal or lower p99."""
    if r is None:
        return None
    keys = ("requests", "requests_per_s", "p50_ms", "p99_ms", "offered_rate", "ok")
    out = {k: {kk: v.get(kk) for kk in keys if kk in v} for k, v in r.items() if isinstance(v, dict)}
    out["workload"] = r["workload"]
    out["form"] = r["form"]
    out["throughput_ratio_vs_plain"] = r["throughput_ratio_vs_plain"]
    same = r["open_loop_same_rate"]["p99_ms"]
    base = r["baseline_open_loop"]["p99_ms"]
    out["p99_at_plain_rate_ms"] = {"server": same, "plain_one_at_a_time": base}
    out["target_3x_at_le_p99"] = bool(r["throughput_ratio_vs_plain"] >= 3.0 and same <= base)
    return out


def run_reference(args):
    ws, rank, _ = dist_env()
    if ws > 1 and rank != 0:
        return
    x, eps = workload(N_POINTS)
    budget = max(1.5, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    try:
        sampler = RefSampler(x, eps, budget)
        steps = []
        for i in range(args.warmup + args.steps):
            r = sampler.run()
            if i >= args.warmup:
                steps.append(r)
    except Exception as e:  # the arm always prints its line
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU path failed: {e}"}), flush=True)
        return
    vals = [s["value"] for s in steps]
    v = statistics.median(vals)
    secs = [s["alg_s"] for s in steps]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "self-join 1M x 64 uniform FP32 (seed 22), eps for 32 "
                                            "neighbours; bounded CPU sample per step", "eps": eps,
                                            "sample_points": sampler.n_s},
            "cpu_baseline": dict({k: steps[-1][k] for k in CPU_KEYS}, value=v),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_serving(args):
    """The serving stream: throughput and p50/p99 latency of the tensor-core
    server (continuous batching across streams) next to the plain FP64 path
    serving one request at a time."""
    import torch
    torch.cuda.set_device(0)
    from hilbertjoin_b200 import serving
    r = serving.run_benchmark(n_requests=args.requests, form=args.form or "auto",
                              baseline_requests=args.baseline_requests)
    line = {"metric": "join-serving requests/s (p50/p99 latency)", "value": r["saturated"]["requests_per_s"],
            "unit": "requests/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": r["workload"], "form": r["form"]}, "serving": r}
    print(json.dumps(line), flush=True)


def run_batch(args):
    """Many joins in one persistent launch: jobs/s of single calls, of one
    planned batch, and of replays of a graph-captured batch run."""
    import torch
    torch.cuda.set_device(0)
    from hilbertjoin_b200 import batching
    r = batching.run_benchmark(form=args.form if args.form not in (None, "plain", "auto") else "fp16")
    line = {"metric": "batched joins/s (one persistent launch, graph replay)",
            "value": r["batch_replay"]["jobs_per_s"], "unit": "joins/s", "n_gpus": 1, "higher_is_better": True,
            "data": "synthetic", "config": {"workload": r["workload"], "form": r["form"]}, "batch": r}
    print(json.dumps(line), flush=True)


def run_config(args):
    """One benchmark configuration at its stated size, device-resident input:
    per form (--form, else all four) the whole-join time over --steps steps and
    the stage times, with the count checked against the oracle's fixture."""
    import torch
    torch.cuda.set_device(0)
    import hilbertjoin_b200 as hj
    from hilbertjoin_b200 import workloads as W
    a, b, eps = W.config_sets(args.config)
    if args.prefix:
        a = np.ascontiguousarray(a[:args.prefix])
        b = None if b is None else np.ascontiguousarray(b[:args.prefix])
    p = os.path.join(ROOT, "tests", "golden", "config_counts.json")
    want = None
    if os.path.exists(p) and not args.prefix:
        with open(p) as f:
            fx = json.load(f)["configs"].get(args.config)
        want = None if fx is None else int(fx["oracle_count"])
    ad = torch.from_numpy(a).cuda()
    bd = None if b is None else torch.from_numpy(b).cuda()
    stream = torch.cuda.current_stream()
    out = {}
    forms = [args.form] if args.form not in (None, "auto") else ["plain", "fp16", "tf32", "bf16x3"]
    for form in forms:
        def step():
            if bd is None:
                return hj.self_join_count(ad, eps, form=form, return_stats=True)
            return hj.join_count(ad, bd, eps, form=form, return_stats=True)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = [step() for _ in range(args.steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        counts = {c for c, _ in res}
        st = res[-1][1]
        if want is not None and counts != {want}:
            raise SystemExit(f"{args.config} {form}: count {counts} differs from the oracle's {want}")
        out[form] = {"ms_per_step": e0.elapsed_time(e1) / args.steps, "count": res[-1][0],
                     **{k: st[k] for k in ("sort_ms", "index_ms", "join_ms", "kernel_ms", "recheck_ms",
                                           "candidate_pairs", "work_items", "fp64_items", "band_pairs",
                                           "form_used", "kernel_launches")}}
    print(json.dumps({"workload": args.config, "prefix": args.prefix or None, "eps": eps,
                      "oracle_count_fixture": want, "forms": out}), flush=True)


def main():
    args = parse()
    if args.workload == "selfjoin":
        if args.form is None:
            args.form = "fp16"
        if args.form == "auto":
            args.form = "fp16"  # the 1M x 64 join is far above the small-join threshold
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "config":
        return run_config(args)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    import hilbertjoin_b200 as hj

    n = args.n
    x, eps = workload(n)
    if n == N_POINTS:
        assert abs(eps - EPS_CALIBRATED) < 1e-6, eps
    pairs = n * (n - 1) / 2
    xd = torch.from_numpy(x).to(dev)
    xh = torch.from_numpy(x).pin_memory()
    xh_np = xh.numpy()
    stream = torch.cuda.current_stream(dev)

    def step_dev(form):
        return hj.self_join_count(xd, eps, form=form, return_stats=True)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    props = torch.cuda.get_device_properties(dev)
    gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(dev.index)
    counts, kernel_ms, launches = [], [], []
    with ClockSampler(gpu_id) as clk:
        # warm-up (the sampler starts up meanwhile; its samples are kept only
        # from the timed region on)
        for _ in range(args.warmup):
            c0, st0 = step_dev(args.form)
        barrier()
        clk.mark()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            c, st = step_dev(args.form)
            counts.append(c)
            kernel_ms.append(st["kernel_ms"])
            launches.append(st["kernel_launches"])
        e1.record(stream)
        barrier()
    clocks = clk.summary()
    ms = e0.elapsed_time(e1) / args.steps
    if ws > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    assert len(set(counts)) == 1, counts
    value = pairs * ws / (ms / 1e3)

    # e2e: the public C-ABI call on pinned host memory (copy in, count out)
    for _ in range(1):
        hj.self_join_count(xh_np, eps, form=args.form)
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        ce = hj.self_join_count(xh_np, eps, form=args.form)
    barrier()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    if ws > 1:
        t = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    assert ce == counts[0]

    # the plain FP64 form on the same input: the tensor-core form's speed-up over it
    plain = None
    if not args.no_plain and args.form != "plain" and rank == 0:
        step_dev("plain")
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        cp, stp = step_dev("plain")
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        assert cp == counts[0], (cp, counts[0])
        plain = {"value": pairs / (pms / 1e3), "ms_per_step": pms, "kernel_ms": stp["kernel_ms"],
                 "count": cp}

    peaks, peak_src = load_peaks()
    kms = statistics.mean(kernel_ms)
    roof = roofline(args.form, kms, pairs, peaks, peak_src)
    # one-pass ncu capture of dram__bytes_read.sum + dram__bytes_write.sum on this exact
    # workload, summarised under profiles/ (the line "bytes_per_launch_full_size: N")
    tname = f"{roof['kernel']}_{args.form}_selfjoin_1Mx64_dram_traffic.md"
    tpath = os.path.join(ROOT, "profiles", tname)
    if args.n == N_POINTS and os.path.exists(tpath):
        m = re.search(r"^bytes_per_launch_full_size:\s*(\d+)", open(tpath).read(), re.M)
        if m:
            roof["traffic"] = int(m.group(1))
            roof["traffic_source"] = f"profiles/{tname}"

    # the other tensor-core forms the workload names (TF32, BF16 hi/lo three-product)
    # on the same device-resident input: whole-join time, kernel roofline, count
    variants = {}
    if rank == 0 and not args.no_variants:
        for form in ("tf32", "bf16x3", "fp16"):
            if form == args.form:
                continue
            step_dev(form)
            torch.cuda.synchronize()
            v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            vk, vc = [], []
            v0.record(stream)
            for _ in range(2):
                cv, stv = step_dev(form)
                vk.append(stv["kernel_ms"])
                vc.append(cv)
            v1.record(stream)
            torch.cuda.synchronize()
            assert set(vc) == {counts[0]}, (form, vc, counts[0])
            r = roofline(form, statistics.mean(vk), pairs, peaks, peak_src)
            vms = v0.elapsed_time(v1) / 2
            variants[form] = {"value": pairs / (vms / 1e3), "ms_per_step": vms, "kernel_ms": r["kernel_ms"],
                              "frac": r["frac"], "achieved_tflops": r["achieved"], "peak_tflops": r["peak"],
                              "count": vc[0], "band_pairs": stv["band_pairs"],
                              "band_fraction": stv["band_fraction"],
                              "max_abs_err_band": stv["max_abs_err_band"]}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(x, eps)
        except Exception as e:  # the baseline never blocks the GPU line
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}", "host_cores": os.cpu_count(), "avx512f": None, "note": None}
        cpu = {k: cpu.get(k) for k in CPU_KEYS}

    # the serving stream, shortened (same request mix): the default server next
    # to the plain FP64 path serving one request at a time
    serving_r = None
    if rank == 0 and ws == 1 and not args.no_serving:
        from hilbertjoin_b200 import serving
        serving_r = serving.run_benchmark(n_requests=400, form="auto", baseline_requests=100, batch_max=1)

    fixture = golden_count(n)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"tf32": "tf32", "fp16": "fp16", "bf16x3": "bf16x3", "plain": "f64"}[args.form],
            "data": "synthetic (seeded uniform, FP32)",
            "config": {"workload": f"self-join {n} x {DIM}, uniform [0,1) FP32 seed {SEED}, eps for {NEIGHBOURS} "
                                   f"neighbours (dense regime, all pairs evaluated)", "n": n, "d": DIM,
                       "eps": eps, "form": args.form, "count": counts[0],
                       "oracle_count_fixture": fixture,
                       "l2": "input 256 MB > 126 MB L2 (no flush needed)",
                       "parallelism": "replicas" if ws > 1 else "single GPU"},
            "e2e": {"value": pairs * ws / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(x.nbytes), "d2h_bytes_per_step": 8 + 8,
                    "ms_per_step": e2e_ms, "timing": "host clock around synchronous C-ABI calls"},
            "gpu_launches": int(sum(launches)),
            "roofline": roof,
            "cpu_baseline": cpu,
            "plain_fp64": plain,
            "vs_plain_fp64": (value / plain["value"]) if plain else None,
            "stats": {k: st0[k] for k in ("sort_ms", "index_ms", "join_ms", "recheck_ms", "band_pairs",
                                          "band_halfwidth_rel", "max_abs_err_band", "fp64_items",
                                          "candidate_pairs", "work_items")},
            "variants": variants or None,
            "serving": serving_summary(serving_r),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    # after the ranks have left the process group, so that none waits on a rank that stopped
    if fixture is not None and counts[0] != fixture:
        raise SystemExit(f"count {counts[0]} differs from the oracle's {fixture} for this workload")


if __name__ == "__main__":
    main()
