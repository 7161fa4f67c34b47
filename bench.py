"""Benchmark of the in-place 213 transpose on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one in-place 213 transpose of the workload tensor: fp32
(d1,d2,d3) = (8192,6144,4), 805 MB, values uniform[-1,1) from seed 0 (the large
fp32 configuration of the headline metric; the fp64 (7919,6151,2) tensor is
reported beside it).  `value` is the whole-job effective bandwidth
2 * bytes / time (GB/s) with the tensor resident in HBM; `e2e` is the same
metric through the public host-buffer call (pinned host memory copied in and
out inside every timed step).  Under torchrun every rank transposes its own
replica (no collective on the data path); the time is the max over ranks.

`--impl reference` times the reference's own CPU path (TensorUtil::seq_tt,
compiled from its sources into oracle/_ref/) on the host cores, one thread per
slice, on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

D1, D2, D3, EB = 8192, 6144, 4, 4
D1B, D2B, D3B, EBB = 7919, 6151, 2, 8
METRIC = "in-place 213 effective GB/s (2*bytes/time)"
UNIT = "GB/s"
PASSES = ("tile_swap", "segment_cycles", "row_gather", "col_gather", "band_transpose", "slice")
FALLBACK_PEAK = 6650.0


def workload_desc():
    return {"workload": f"in-place 213 transpose, fp32 (d1,d2,d3)=({D1},{D2},{D3}), "
                        f"{D1 * D2 * D3 * EB / 1e6:.1f} MB, uniform[-1,1) seed 0",
            "d1": D1, "d2": D2, "d3": D3, "elem_bytes": EB,
            "l2": "inputs larger than L2 (805 MB per tensor vs 126 MB L2); no flush needed"}


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """Samples SM clock and throttle reasons through NVML (read-only) while the
    timed region runs."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle",
               0x2: "applications_clocks_setting"}

    def __init__(self, index: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.ok = False
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self._t.join()

    def result(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "note": "NVML unavailable" if not self.ok else "no samples"}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------- helpers -------
def peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_PEAK, "fallback"


def ncu_traffic(pass_name: str):
    """Per-launch DRAM bytes of a pass from the committed ncu summary
    (profiles/traffic.json), scaled to this workload; None if absent."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            t = json.load(f)
        e = t[pass_name]
        return int(e["dram_bytes_per_launch"] * (D1 * D2 * D3 * EB) / e["tensor_bytes"])
    except Exception:
        return None


def init_dist(n_gpus, backend="nccl"):
    """One process per GPU under torchrun (RANK/LOCAL_RANK/WORLD_SIZE/MASTER_*
    from the environment); (None, 0, 1, 0) for a single process.  The CPU
    tests use backend "gloo"."""
    if n_gpus <= 1 or "RANK" not in os.environ:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist
    import datetime
    local = int(os.environ.get("LOCAL_RANK", 0))
    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist, dist.get_rank(), dist.get_world_size(), local


def max_over_ranks(dist, value: float, device="cuda") -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device="cuda"):
    if dist is not None:
        import torch
        t = torch.zeros(1, device=device)
        dist.all_reduce(t)
        if device == "cuda":
            torch.cuda.synchronize()


def whole_job_gbps(world: int, nbytes: int, steps: int, ms_max: float) -> float:
    """Effective 2 x bytes / time of all ranks' replicas, timed as the max
    over ranks (each rank transposes its own tensor of nbytes per step)."""
    return world * 2 * nbytes * steps / (ms_max * 1e-3) / 1e9


# ------------------------------------------------------------ our arm --------
def run_ours(args):
    import numpy as np
    import torch
    t213 = importlib.import_module("213transpose_b200")
    dist, rank, world, local = init_dist(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nbytes = D1 * D2 * D3 * EB
    gen = torch.Generator(device=dev).manual_seed(0)
    x = (torch.rand(D1 * D2 * D3, generator=gen, device=dev, dtype=torch.float32) * 2 - 1)
    stream = torch.cuda.current_stream(dev)

    def step():
        t213.transpose(x, D1, D2, D3)

    # warm-up (also builds and uploads the plan)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches_per_step = t213.plan_launches(D1, D2, D3, EB)
    desc = t213.describe(D1, D2, D3, EB)

    # timed region: K steps, CUDA events on the launching stream
    barrier(dist)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        a.record(stream)
        for _ in range(args.steps):
            step()
        b.record(stream)
        b.synchronize()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    ms_max = max_over_ranks(dist, ms)
    barrier(dist)

    # per-pass timing for the roofline (separate loop, events on the same stream)
    t213.pass_timing.reset()
    t213.pass_timing.enable(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    per = {p: t213.pass_timing.read(p) for p in PASSES}
    t213.pass_timing.enable(False)
    per = {k: v for k, v in per.items() if v[1] > 0}
    total_pass_ms = sum(v[0] for v in per.values())
    dom = max(per, key=lambda k: per[k][0])
    dom_ms = per[dom][0] / per[dom][1]
    peak, peak_kind = peak_gbs()
    achieved = 2 * nbytes / (dom_ms * 1e-3) / 1e9
    traffic = ncu_traffic(dom)

    # out-of-place comparison point: torch's transpose(-2, -1) copied into a
    # second buffer (one read and one write of every byte, twice the memory)
    oop = torch.empty_like(x)
    xv, ov = x.view(D3, D2, D1), oop.view(D3, D1, D2)
    for _ in range(args.warmup):
        ov.copy_(xv.transpose(1, 2))
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        ov.copy_(xv.transpose(1, 2))
    b.record(stream)
    b.synchronize()
    ms_oop = a.elapsed_time(b) / args.steps
    del oop, xv, ov
    torch.cuda.empty_cache()

    # the same tensor through the reference's own decomposition (C2R forced)
    c2r_plan = t213.describe(D1, D2, D3, EB, "c2r")
    for _ in range(args.warmup):
        t213.transpose_with_plan(x, D1, D2, D3, "c2r")
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        t213.transpose_with_plan(x, D1, D2, D3, "c2r")
    b.record(stream)
    b.synchronize()
    ms_c2r = max_over_ranks(dist, a.elapsed_time(b)) / args.steps

    # secondary tensor: fp64 (7919, 6151, 2)
    nb2 = D1B * D2B * D3B * EBB
    y = torch.empty(D1B * D2B * D3B, dtype=torch.float64, device=dev).uniform_(-1, 1, generator=gen)
    for _ in range(max(1, args.warmup)):
        t213.transpose(y, D1B, D2B, D3B)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        t213.transpose(y, D1B, D2B, D3B)
    b.record(stream)
    b.synchronize()
    ms_b = max_over_ranks(dist, a.elapsed_time(b))
    t213.pass_timing.reset()
    t213.pass_timing.enable(True)
    for _ in range(args.steps):
        t213.transpose(y, D1B, D2B, D3B)
    torch.cuda.synchronize()
    per_b = {p: t213.pass_timing.read(p) for p in PASSES}
    t213.pass_timing.enable(False)
    per_b = {k: v for k, v in per_b.items() if v[1] > 0}
    del y
    torch.cuda.empty_cache()

    # end to end through the public host-buffer call (pinned memory)
    e2e_steps = max(1, min(args.steps, 5))
    host = torch.empty(D1 * D2 * D3, dtype=torch.float32).pin_memory()
    host.copy_(x.cpu())
    t213.transpose_host(host, D1, D2, D3)  # warm-up
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        t213.transpose_host(host, D1, D2, D3)
    e2e_s = max_over_ranks(dist, time.perf_counter() - t0)

    del host
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()
    batched = serving = configs = None
    if world == 1 and not args.quick:
        del x
        torch.cuda.empty_cache()
        configs = configs_section(t213, torch, args.steps, args.warmup)
        batched = batched_section(t213, torch, stream)
        serving = serving_section(t213, torch)

    if rank == 0:
        value = whole_job_gbps(world, nbytes, args.steps, ms_max)
        n_passes = len(per)
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "index_arith": "u32",
            "data": "synthetic uniform[-1,1) fp32, seed 0",
            "config": dict(workload_desc(), plan=desc, parallelism=f"replicas x{world}"),
            "frac_of_8TBps": round(value / world / 8000.0, 4),
            "pass_count_GBps": round(n_passes * value, 1),
            "passes": {k: {"ms_per_launch": round(v[0] / v[1], 4), "share": round(v[0] / total_pass_ms, 3)}
                       for k, v in per.items()},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                         "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": 2 * nbytes},
            "forced_c2r": {"what": "the headline tensor through the reference's C2R decomposition (forced plan)",
                           "plan": c2r_plan, "ms": round(ms_c2r, 4),
                           "value": round(world * 2 * nbytes / (ms_c2r * 1e-3) / 1e9, 1), "unit": UNIT},
            "secondary": {"workload": f"fp64 (7919,6151,2) {nb2 / 1e6:.1f} MB",
                          "plan": t213.describe(D1B, D2B, D3B, EBB),
                          "value": round(world * 2 * nb2 * args.steps / (ms_b * 1e-3) / 1e9, 1), "unit": UNIT,
                          "roofline": {k: {"ms_per_launch": round(v[0] / v[1], 4),
                                           "achieved": round(2 * nb2 / (v[0] / v[1] * 1e-3) / 1e9, 1),
                                           "frac": round(2 * nb2 / (v[0] / v[1] * 1e-3) / 1e9 / peak, 4)}
                                       for k, v in per_b.items()}},
            "out_of_place_torch": {"what": "torch x.view(d3,d2,d1).transpose(1,2) copied into a second buffer "
                                           "(out of place: one sweep, 2x memory)",
                                   "ms": round(ms_oop, 4), "GBps": round(2 * nbytes / (ms_oop * 1e-3) / 1e9, 1),
                                   "in_place_vs_out_of_place_time": round((ms_max / args.steps) / ms_oop, 3)},
            "e2e": {"value": round(world * 2 * nbytes * e2e_steps / e2e_s / 1e9, 2), "unit": UNIT,
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "path": "t213_transpose_host (pinned host memory, slices pipelined over copy engines)"},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.result(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if configs:
            line["configs"] = configs
        if batched:
            line["batched"] = batched
        if serving:
            line["serving"] = serving
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ------------------------------------------------------- other configs -----
CONFIGS = [  # name, d1, d2, d3, element bytes
    ("fp32 (512,384,16)", 512, 384, 16, 4),
    ("fp32 (32,2^24,1)", 32, 1 << 24, 1, 4),
    ("fp32 (2^24,48,1)", 1 << 24, 48, 1, 4),
    ("int32 (3,2^22,8)", 3, 1 << 22, 8, 4),
    ("16B (1024,1024,1)", 1024, 1024, 1, 16),
]


def configs_section(t213, torch, steps, warmup):
    """The workload's other single-tensor configurations, device-resident,
    random bit patterns: the plain call timed with CUDA events over `steps`
    calls, and for tensors under 64 MB also one call captured in a CUDA graph
    and replayed (launch latency off the critical path)."""
    out = []
    for name, d1, d2, d3, eb in CONFIGS:
        n = d1 * d2 * d3 * eb
        x = torch.empty(n, dtype=torch.uint8, device="cuda")
        x.random_(0, 256, generator=torch.Generator(device="cuda").manual_seed(3))

        def call():
            t213.transpose(x, d1, d2, d3, elem_bytes=eb)

        def timed(fn):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            a.record(torch.cuda.current_stream())
            for _ in range(steps):
                fn()
            b.record(torch.cuda.current_stream())
            b.synchronize()
            return a.elapsed_time(b) / steps

        ms = timed(call)
        e = {"config": name, "plan": t213.describe(d1, d2, d3, eb), "MB": round(n / 1e6, 1), "ms": round(ms, 4),
             "GBps": round(2 * n / (ms * 1e-3) / 1e9, 1)}
        if n < (64 << 20):
            try:
                side = torch.cuda.Stream()
                with torch.cuda.stream(side):
                    call()  # plan and workspace for this stream, outside the capture
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=side):
                    call()
                msg = timed(g.replay)
                e["graph_ms"] = round(msg, 4)
                e["graph_GBps"] = round(2 * n / (msg * 1e-3) / 1e9, 1)
                del g
            except Exception as ex:  # capture is optional: report why it did not happen
                e["graph_error"] = str(ex)[:200]
        out.append(e)
        del x
        torch.cuda.empty_cache()
    return out


# ------------------------------------------------------ batched / serving ----
def batched_section(t213, torch, stream):
    """512 uneven tensors (d1,d2 log-uniform in [16,4096], d3 in {1,2,4,8},
    fp32/fp64/int32/16-byte, seed 1): one persistent graph-captured launch
    against the plain call looped over the same list."""
    w = importlib.import_module("213transpose_b200.workloads")
    shapes = w.batched_shapes(1, 512)
    gen = torch.Generator(device="cuda").manual_seed(1)
    bufs = []
    for d1, d2, d3, eb, _ in shapes:
        x = torch.empty(d1 * d2 * d3 * eb, dtype=torch.uint8, device="cuda")
        x.random_(0, 256, generator=gen)
        bufs.append(x)
    # the autotuner times every shape's plan families, block sizes and kernel
    # variants on scratch memory (outside the timed region); the batch and the
    # looped plain call then both run the tuned choices
    t0 = time.perf_counter()
    B = t213.Batch([(x, d1, d2, d3, eb) for x, (d1, d2, d3, eb, _) in zip(bufs, shapes)], tune=True)
    tune_s = time.perf_counter() - t0
    tuned = sum(1 for d1, d2, d3, eb, _ in shapes if t213.tuner.lookup(d1, d2, d3, eb) is not None)

    def tm(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            best = min(best, a.elapsed_time(b))
        return best

    tb, tl = tm(B.execute), tm(B.looped)
    status = B.status()
    tot = w.total_bytes(shapes)
    out = {"workload": "512 tensors, d1,d2 log-uniform [16,4096], d3 in {1,2,4,8}, fp32/fp64/int32/16B, seed 1",
           "total_GB": round(tot / 1e9, 3), "batched_ms": round(tb, 3), "looped_ms": round(tl, 3),
           "speedup_vs_looped": round(tl / tb, 3), "batched_GBps": round(2 * tot / tb / 1e6, 1),
           "looped_GBps": round(2 * tot / tl / 1e6, 1), "device_status": status, "desc": B.describe(),
           "autotuner": {"tuned_tensors": tuned, "tuning_s": round(tune_s, 1),
                         "searched": "plan family, block/band size, column/row/tile/cycle kernel variants"}}
    B.close()
    t213.tuner.clear()
    del bufs
    torch.cuda.empty_cache()
    return out


def serving_section(t213, torch):
    """Poisson 2000 req/s, request size log-uniform 1 KB - 2 GB, shapes/dtypes
    drawn as in the batched workload, 150 GB HBM budget; 2000 requests."""
    w = importlib.import_module("213transpose_b200.workloads")
    reqs = w.serving_requests(5, 2000)
    for i, r in enumerate(reqs):
        r["seed"] = 1 + i
    srv = t213.Server(hbm_budget_bytes=150 * 10**9, max_inflight=64, streams=8)
    srv.run(reqs[:50])  # warm-up: plans of the first shapes
    stats, sums, lat = srv.run(reqs)
    bad = sum(1 for r, s in list(zip(reqs, sums))[::40] if s != srv.expected_checksum(r))
    srv.close()
    torch.cuda.empty_cache()
    return {"workload": "Poisson 2000 req/s, log-uniform 1 KB-2 GB, 150 GB budget, 2000 requests",
            "completed": stats["completed"], "rejected": stats["rejected"],
            "p50_ms": round(stats["p50_ms"], 3), "p99_ms": round(stats["p99_ms"], 3),
            "mean_ms": round(stats["mean_ms"], 3), "max_ms": round(stats["max_ms"], 3),
            "cold_requests": stats["cold"], "p50_cold_ms": round(stats["p50_cold_ms"], 3),
            "p99_cold_ms": round(stats["p99_cold_ms"], 3), "p50_warm_ms": round(stats["p50_warm_ms"], 3),
            "p99_warm_ms": round(stats["p99_warm_ms"], 3),
            "group_launches": stats["group_launches"], "grouped_requests": stats["grouped_requests"],
            "throughput_GBps": round(stats["bytes_done"] / stats["wall_s"] / 1e9, 2),
            "requests_per_s": round(stats["completed"] / stats["wall_s"], 1),
            "peak_resident_GB": round(stats["peak_resident_bytes"] / 1e9, 2),
            "max_inflight": stats["max_inflight"],
            "latency_includes": "fill of the request tensor on the device (producer stand-in) + in-place transpose",
            "checksum_mismatches_of_50_sampled": bad}


# ----------------------------------------------------------- CPU baseline ----
def _ref_seq_tt():
    from oracle import oracle as O
    if not O.ref_available():
        return None, "port"
    return O, "reference"


def cpu_baseline_sample():
    """The reference's own CPU path (TensorUtil::seq_tt) on a bounded sample:
    one slice (d3=1) of the workload, one thread, best of two."""
    import numpy as np
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    x = O.uniform_f32(D1 * D2, 0)
    out = np.empty_like(x)
    best = 1e30
    for _ in range(2):
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_seq_tt_into(out, x, D1, D2, 1, EB)
        else:
            out = O.seq_tt(x.view(np.uint32), (D1, D2, 1))
        best = min(best, time.perf_counter() - t0)
    return {"value": round(2 * D1 * D2 * EB / best / 1e9, 3), "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"1 of {D3} slices ({D1}x{D2} fp32, {D1 * D2 * EB / 1e6:.0f} MB), TensorUtil::seq_tt, "
                      f"1 thread, best of 2; host has {os.cpu_count()} cores"}


def run_reference(args):
    """--impl reference: the reference's CPU implementation, all slices in
    parallel threads (one per slice, up to the host's cores)."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    threads = max(1, min(D3, os.cpu_count() or 1))
    slices = [O.uniform_f32(D1 * D2, k) for k in range(D3)]
    outs = [np.empty_like(s) for s in slices]

    def one(k):
        if kind == "reference":
            O.ref_seq_tt_into(outs[k], slices[k], D1, D2, 1, EB)
        else:
            O.seq_tt(slices[k].view(np.uint32), (D1, D2, 1))

    def step():
        ths = [threading.Thread(target=one, args=(k,)) for k in range(D3)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    nbytes = D1 * D2 * D3 * EB
    value = 2 * nbytes * args.steps / dt / 1e9
    sample = (f"full workload per step: {D3} slices of {D1}x{D2} fp32 in {threads} threads "
              f"(TensorUtil::seq_tt, one slice per thread); host has {os.cpu_count()} cores")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic uniform[-1,1) fp32", "config": workload_desc(),
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="skip the batched and serving sections")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
