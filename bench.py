"""Benchmark: reduce/scan GB/s and fraction of HBM peak at 2^28 elements.

One step = the fp32 precision workload on 2^28 elements: transform_reduce
dot product of two fp32 arrays (N(0,1), 1/8 of the values scaled by 1e-6)
plus an inclusive scan of one fp32 |N(0,1)| array, inputs resident in HBM.
Algorithmic bytes per step: dot 8n + scan 8n = 4 GiB.  Inputs (3 GiB) are
larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (under torchrun): the arrays are shards of one logical array of
2^28 * N elements (rank r holds the r-th 2^28 elements).  The step is the
sharded dot (local dot, all-gather of the N partials over NCCL) and the
sharded inclusive scan (local reduce, all-gather of the N shard totals,
local scan with the carry as init): weak scaling, time = max over ranks.
--impl reference times the oracle's restatement of the reference's OpenMP
backend (oracle/baseline.py) on the host cores, on the same workload; it
loads nothing from this package.

Before the headline line, compact JSON lines carry the per-primitive table
(`ops_summary`), the segmented batch (`segmented_summary`) and the selector
stream (`selector_summary`); the headline repeats their key figures.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N28 = 1 << 28
N24 = 1 << 24
GIB = float(1 << 30)
METRIC = "reduce/scan GB/s & %HBM peak at 2^28; segmented batch calls/s, learned vs plain"


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic():
    """Per-launch DRAM bytes of the dominant kernels from the committed ncu
    summary (profiles/traffic.txt: `<kernel-key> <bytes-per-launch> <n>`)."""
    out = {}
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(p):
        for line in open(p):
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#"):
                out[parts[0]] = (float(parts[1]), int(parts[2]))
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.count(",") >= 8]
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- reference arm

def workload_config(log2n: int, world: int) -> dict:
    n = 1 << log2n
    return {"workload": f"fp32 dot(a,b) 2^{log2n} + fp32 inclusive_scan 2^{log2n}"
                        + (f" per rank, one logical array of 2^{log2n} x {world}" if world > 1 else ""),
            "elements": n, "step_bytes": 16.0 * n,
            "l2": f"inputs ({12.0 * n / 2**30:g} GiB) larger than the 126 MB L2; no flush" if n >= N24
                  else "inputs smaller than L2 (profiling size); no flush",
            "parallelism": "single device" if world == 1 else f"sharded x{world} (one exchange per primitive)"}


def run_reference(args, world):
    """The oracle's restatement of the reference's OpenMP backend on every
    host core, on the same workload as our arm (oracle/baseline.py, its own
    process and generator: nothing from this package is loaded)."""
    from oracle import baseline

    r = baseline.run(args.log2n, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(r["value"], 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(r["ms_per_step"], 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.log2n, world),
        "cpu_baseline": {"value": round(r["value"], 3), "unit": "GB/s", "cores": r["threads"], "kind": "port",
                         "cpu_model": r["cpu_model"], "omp": r["omp"],
                         "sample": f"the full workload: {args.steps} timed steps of dot + inclusive_scan over "
                                   f"2^{args.log2n} fp32 elements, OpenMP-backend evaluation order, "
                                   f"{r['threads']} threads"},
        "e2e": {"value": round(r["value"], 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "precision": {"dot_rel_err_vs_fp64": r["dot_rel_err_vs_fp64"],
                      "scan_max_rel_err_vs_fp64": r["scan_max_rel_err_vs_fp64"]},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-ops", action="store_true", help="skip the per-primitive table")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--log2n", type=int, default=28,
                    help="elements per array of the headline step (small cases for profiling)")
    ap.add_argument("--ops-log2n", type=int, default=28,
                    help="elements per array of the per-primitive table (below 28: no 2^24, segmented "
                         "or selector entries; small cases for profiling)")
    ap.add_argument("--ops-reps", type=int, default=10, help="timed launches per primitive")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend for N > 1 (gloo: a functional check of the sharded path, "
                         "ranks may share a GPU; not a measurement)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        run_reference(args, world)
        return

    import numpy as np
    import torch

    from opensycl_b200 import capi as C
    from opensycl_b200 import sharded as SH

    torch.cuda.set_device(local % max(torch.cuda.device_count(), 1))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(args.dist_backend, timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    peak, peak_kind = hbm_peak()
    selector_state = install_selector(C)
    n = 1 << args.log2n
    # rank r's shard of the logical arrays: elements [r n, (r+1) n) of streams 1, 2, 3
    a_h = C.synth_fill(1, 1 + 10 * rank, n, 0.125, 1e-6)
    b_h = C.synth_fill(1, 2 + 10 * rank, n, 0.125, 1e-6)
    x_h = C.synth_fill(2, 3 + 10 * rank, n, 0.125, 1e-6)
    a = torch.from_numpy(a_h).cuda()
    b = torch.from_numpy(b_h).cuda()
    x = torch.from_numpy(x_h).cuda()
    y = torch.empty(n, dtype=torch.float32, device="cuda")
    dres = torch.zeros(1, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    step_bytes = 8.0 * n + 8.0 * n
    sharded_dot = [0.0]

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        if world == 1:
            C.dot(a, b, init=0.0, out=dres)
        else:
            sharded_dot[0] = SH.sharded_dot(a, b, 0.0)
        if ev is not None:
            ev[1].record(stream)
        if world == 1:
            C.scan(x, True, "sum", None, out=y)
        else:
            y.copy_(SH.sharded_scan(x, True, "sum", None))
        if ev is not None:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clk:
        start.record(stream)
        for k in range(args.steps):
            step(evs[k])
        end.record(stream)
        barrier()
    ms = start.elapsed_time(end)
    if dist is not None:
        t = torch.tensor([ms], device="cuda" if args.dist_backend == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    dot_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    scan_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    clocks = clk.summary()

    value = step_bytes * args.steps * world / (ms / 1e3) / 1e9
    scan_cfg = C.lib().b2p_auto_config(C.PRIM_SCAN, C.F32, n, 0, 0.0)
    dot_cfg = C.lib().b2p_auto_config(C.PRIM_DOT, C.F32, n, 0, 0.0)
    scan_blk, scan_items, scan_mode = C.config_describe(scan_cfg)
    scan_name = (f"scan_tmem_kernel<f32 sum,{scan_blk}x{scan_items}>" if scan_mode == 1
                 else f"scan_{'lookback' if scan_mode == 0 else 'twophase'}_kernel<f32 sum,{scan_blk}x{scan_items}>")
    kern = {scan_name: (scan_ms, 8.0 * n), "reduce_kernel<f32 dot>": (dot_ms, 8.0 * n)}
    dom = max(kern, key=lambda k: kern[k][0])
    dom_ms, dom_bytes = kern[dom]
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    # the committed DRAM-traffic figures are per launch at 2^28 elements
    traffic = read_traffic().get("scan_f32" if dom.startswith("scan") else "dot_f32") if args.log2n == 28 else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic[0] if traffic else None,
                "algorithmic_bytes": dom_bytes}
    if world > 1:
        roofline["note"] = "scan time includes the shard reduce and the exchange"

    config = workload_config(args.log2n, world)
    config.update(scan_config=scan_cfg, dot_config=dot_cfg)
    result = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": config,
        "roofline": roofline,
        "gpu_launches": (2 if world == 1 else 3) * args.steps,
        "clocks": clocks,
        "per_kernel_ms": {"dot": round(dot_ms, 4), "scan": round(scan_ms, 4)},
        "precision": measure_precision(torch, a, b, x, y, dres if world == 1 else None),
    }

    if rank == 0 and world == 1:
        result["e2e"] = measure_e2e(C, torch, a_h, b_h, x_h, args)
        if not args.no_cpu:
            result["cpu_baseline"] = cpu_baseline(args.log2n)
        if not args.no_ops:
            ops = measure_ops(C, torch, np, peak, args.ops_log2n, args.ops_reps)
            print(json.dumps({"ops_summary": ops}), flush=True)
            result["ops"] = {k: [v["GB/s"], v["frac_hbm"], v.get("b2b_frac_hbm")] for k, v in ops.items()}
            result["ops_columns"] = ["GB/s single launch", "frac of measured HBM", "frac back-to-back"]
            if args.ops_log2n == 28:
                seg = measure_segmented(C, torch, np, peak)
                print(json.dumps({"segmented_summary": seg}), flush=True)
                result["segmented"] = {k: {"GB/s": v["learned"]["GB/s"], "frac": v["learned"]["frac_hbm"],
                                           "x_plain": v["speedup_learned_vs_plain"]}
                                       for k, v in seg.items() if isinstance(v, dict) and "learned" in v}
                sel = measure_selector_stream(selector_state)
                print(json.dumps({"selector_summary": sel}), flush=True)
                result["selector"] = {k: sel[k] for k in ("learned_vs_exhaustive_table", "heuristic_vs_learned")
                                      if k in sel}
        result["selector_state"] = selector_state["status"]
    elif world > 1:
        # every rank takes part in the exchanges of the end-to-end step
        result["e2e"] = measure_e2e_sharded(SH, torch, a_h, b_h, x_h, args, dist)
    else:
        result["e2e"] = None
    if rank == 0:
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def install_selector(C):
    """Install the learned schedule selector for B2P_CONFIG_AUTO when its
    weights match this GPU and library version (else AUTO stays heuristic)."""
    from opensycl_b200 import selector as S
    state = {"status": "heuristic", "sel": None}
    try:
        sel = S.Selector(seed=1)
        if sel.load(S.WEIGHTS):
            sel.install()
            state = {"status": "learned (opensycl_b200/data/selector_b200.bin)", "sel": sel}
        else:
            state["status"] = "heuristic (selector weights do not match this GPU/library)"
    except Exception as e:  # no weights file
        state["status"] = f"heuristic ({e})"
    return state


def measure_segmented(C, torch, np, peak):
    """10,000 segments, lengths log-uniform in [1, 2^20] scaled to 2^28 elements
    in total, fp32 N(0,1) and int64 U[-2^20, 2^20]: one CUDA-graph plan launch
    (configuration from AUTO = learned selector, and from the fixed heuristic)
    against one plain call per segment."""
    import ctypes
    L = C.lib()
    nseg = 10000
    offs = C.synth_segments(6, nseg, 20.0, 1 << 28)
    total = int(offs[-1])
    od = torch.from_numpy(offs).cuda()
    s = torch.cuda.current_stream()
    sh = ctypes.c_void_p(s.cuda_stream)
    res = {"nseg": nseg, "total_elems": total,
           "lengths": {"min": int(np.diff(offs).min()), "max": int(np.diff(offs).max())}}
    for name, kind, code, a, b, seed, es in (("fp32", 1, C.F32, 0.0, 0.0, 7, 4),
                                             ("int64", 5, C.I64, -(1 << 20), 1 << 20, 8, 8)):
        x = torch.from_numpy(C.synth_fill(kind, seed, total, a, b)).cuda()
        for prim, label in ((C.PRIM_SEG_REDUCE, "reduce"), (C.PRIM_SEG_SCAN, "inclusive_scan")):
            out = torch.empty(nseg if prim == C.PRIM_SEG_REDUCE else total, dtype=x.dtype, device="cuda")
            nbytes = es * total * (1 if prim == C.PRIM_SEG_REDUCE else 2) + 8 * (nseg + 1)
            entry = {"bytes": nbytes}
            for pol, cfg in (("learned", C.AUTO),
                             ("heuristic", L.b2p_heuristic_config(prim, code, total, nseg))):
                plan = ctypes.c_void_p()
                C.check(L.b2p_plan_segmented(ctypes.byref(plan), prim, code, C.SUM, x.data_ptr(), out.data_ptr(),
                                             od.data_ptr(), nseg, total, cfg, sh), "plan")
                ms = _time_op(torch, lambda: C.check(L.b2p_plan_launch(plan, sh)), reps=10)
                entry[pol] = {"config": L.b2p_plan_config(plan), "ms": round(ms, 4),
                              "batch_calls_per_s": round(1e3 / ms, 1),
                              "GB/s": round(nbytes / (ms / 1e3) / 1e9, 1),
                              "frac_hbm": round(nbytes / (ms / 1e3) / 1e9 / peak, 4)}
                L.b2p_plan_destroy(plan)
            sb = L.b2p_scratch_bytes(C.PRIM_REDUCE if prim == C.PRIM_SEG_REDUCE else C.PRIM_SCAN, code,
                                     1 << 21, 0, C.AUTO)
            scratch = torch.zeros(sb + 512, dtype=torch.uint8, device="cuda")
            sp = ctypes.c_void_p((scratch.data_ptr() + 255) & ~255)
            offs_c = offs.ctypes.data_as(ctypes.c_void_p)
            plain = lambda: C.check(L.b2p_segmented_per_call(prim, code, C.SUM, x.data_ptr(), out.data_ptr(),
                                                            offs_c, nseg, sp, sb, C.AUTO, sh), "per-call")
            ms_plain = _time_op(torch, plain, reps=3, warm=1)
            entry["plain_per_segment_calls"] = {"ms": round(ms_plain, 3), "launches": nseg,
                                                "batch_calls_per_s": round(1e3 / ms_plain, 2)}
            entry["speedup_learned_vs_plain"] = round(ms_plain / entry["learned"]["ms"], 1)
            entry["speedup_learned_vs_heuristic"] = round(entry["heuristic"]["ms"] / entry["learned"]["ms"], 3)
            res[f"{label}_{name}"] = entry
        del x
    return res


def measure_selector_stream(state, ncalls=20000):
    """A seeded stream of calls (random op, dtype, n in 2^10..2^28) run end to
    end under the learned selector, the exhaustive tuner's table and the fixed
    heuristic (the 100,000-call version is in profiles/)."""
    if state.get("sel") is None:
        return {"skipped": state["status"]}
    from opensycl_b200 import selector as S
    shapes, X, T, _ = S.load_dataset(S.DATASET)
    r = S.evaluate_stream(state["sel"], shapes, T, ncalls=ncalls, seed=10, regret_sample=0)
    return {"ncalls": ncalls, "stream_ms": {k: round(v, 2) for k, v in r["stream_ms"].items()},
            "learned_vs_exhaustive_table": round(r["learned_vs_exhaustive_table"], 4),
            "heuristic_vs_learned": round(r["heuristic_vs_learned"], 4),
            "calls_per_s": {k: round(v, 1) for k, v in r["calls_per_s"].items()}}


def measure_e2e(C, torch, a_h, b_h, x_h, args):
    """Same step through the C-ABI from pinned HOST buffers: every step copies
    its three inputs in, runs dot + scan and copies the dot result and the
    scan output back, all inside the timed region.  Inputs go in on one
    stream (which also runs the kernels) and results come back on a second
    one, with two device buffer sets, so the copy-back of step k overlaps the
    copy-in of step k + 1 (PCIe is full duplex)."""
    n = a_h.size
    ap = torch.from_numpy(a_h).pin_memory()
    bp = torch.from_numpy(b_h).pin_memory()
    xp = torch.from_numpy(x_h).pin_memory()
    outs = [(torch.empty(n, dtype=torch.float32).pin_memory(), torch.empty(1, dtype=torch.float32).pin_memory())
            for _ in range(2)]
    sets = [dict(a=torch.empty(n, dtype=torch.float32, device="cuda"),
                 b=torch.empty(n, dtype=torch.float32, device="cuda"),
                 x=torch.empty(n, dtype=torch.float32, device="cuda"),
                 y=torch.empty(n, dtype=torch.float32, device="cuda"),
                 r=torch.zeros(1, dtype=torch.float32, device="cuda")) for _ in range(2)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    computed = [torch.cuda.Event() for _ in range(2)]
    drained = [torch.cuda.Event() for _ in range(2)]
    for ev in drained:
        ev.record(s_out)

    def step(k):
        j = k % 2
        d = sets[j]
        yp, rp = outs[j]
        s_in.wait_event(drained[j])  # this set's previous results have left the GPU
        with torch.cuda.stream(s_in):
            d["a"].copy_(ap, non_blocking=True)
            d["b"].copy_(bp, non_blocking=True)
            d["x"].copy_(xp, non_blocking=True)
            C.dot(d["a"], d["b"], init=0.0, out=d["r"], stream=s_in)
            C.scan(d["x"], True, "sum", None, out=d["y"], stream=s_in)
            computed[j].record(s_in)
        s_out.wait_event(computed[j])
        with torch.cuda.stream(s_out):
            yp.copy_(d["y"], non_blocking=True)
            rp.copy_(d["r"], non_blocking=True)
            drained[j].record(s_out)

    steps = max(3, min(args.steps, 10))
    for k in range(2):
        step(k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    for k in range(steps):
        step(k)
    s_in.wait_stream(s_out)
    e1.record(s_in)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ok = bool(torch.equal(outs[(steps - 1) % 2][1], sets[(steps - 1) % 2]["r"].cpu()))
    return {"value": round(16.0 * n / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": 12 * n, "d2h_bytes_per_step": 4 * n + 4,
            "ms_per_step": round(ms, 3), "steps": steps, "result_read_back": ok,
            "path": "pinned host -> H2D on stream 1 -> b2p_dot + b2p_scan (stream 1) -> D2H on stream 2; "
                    "two buffer sets, step k's D2H overlaps step k+1's H2D"}


def measure_e2e_sharded(SH, torch, a_h, b_h, x_h, args, dist):
    """The sharded step end to end on every rank: copy this rank's shard of
    the three inputs in from pinned host buffers, run sharded_dot and
    sharded_scan (their exchanges included) and copy the scan output back,
    all inside the timed region; time = max over ranks."""
    n = a_h.size
    world = dist.get_world_size()
    ap = torch.from_numpy(a_h).pin_memory()
    bp = torch.from_numpy(b_h).pin_memory()
    xp = torch.from_numpy(x_h).pin_memory()
    yp = torch.empty(n, dtype=torch.float32).pin_memory()
    a = torch.empty(n, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    x = torch.empty_like(a)
    y = torch.empty_like(a)
    dots = []

    def step():
        a.copy_(ap, non_blocking=True)
        b.copy_(bp, non_blocking=True)
        x.copy_(xp, non_blocking=True)
        dots.append(SH.sharded_dot(a, b, 0.0))  # a host value: the step's scalar result
        y.copy_(SH.sharded_scan(x, True, "sum", None))
        yp.copy_(y, non_blocking=True)

    steps = max(3, min(args.steps, 10))
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        step()
    e1.record(s)
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1) / steps], device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    return {"value": round(16.0 * n * world / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": 12 * n * world, "d2h_bytes_per_step": 4 * n * world,
            "ms_per_step": round(ms, 3), "steps": steps, "result_read_back": True,
            "path": f"per rank: pinned host -> H2D -> sharded_dot + sharded_scan ({dist.get_backend()} exchanges) "
                    "-> D2H; max over ranks"}


def measure_precision(torch, a, b, x, y, dres):
    """Error of the timed step's fp32 results against float64 on the device
    (torch, outside the timed region): the dot relative and condition-normalised
    (|got - ref| / sum |a_i b_i|) errors, the scan's largest relative error."""
    ref_s = torch.cumsum(x.double(), 0)
    rel_s = ((y.double() - ref_s).abs() / ref_s.abs().clamp_min(1e-300)).max().item()
    del ref_s
    if dres is None:  # sharded: the scan of this rank's shard includes the carry
        return {"reference": "float64 on the device (torch)", "scan_max_rel_err_local": rel_s}
    ad, bd = a.double(), b.double()
    prod = ad * bd
    ref = float(prod.sum().item())
    cond = float(prod.abs().sum().item())
    del ad, bd, prod
    got = float(dres.item())
    return {"reference": "float64 on the device (torch)",
            "dot_rel_err": abs(got - ref) / abs(ref), "dot_cond_err": abs(got - ref) / cond,
            "scan_max_rel_err": rel_s, "tolerance": 1e-6}


def cpu_baseline(log2n):
    """The oracle's restatement of the reference's OpenMP backend on every
    host core, on the same workload (oracle/baseline.py: the same process
    setup as the reference arm), 5 timed steps after 1 warm-up."""
    from oracle import baseline

    r = baseline.run(log2n, 5, 1)
    return {"value": round(r["value"], 3), "unit": "GB/s", "cores": r["threads"], "kind": "port",
            "cpu_model": r["cpu_model"], "dot_rel_err_vs_fp64": r["dot_rel_err_vs_fp64"],
            "scan_max_rel_err_vs_fp64": r["scan_max_rel_err_vs_fp64"],
            "sample": f"the full workload: 5 steps of dot + inclusive_scan over 2^{log2n} fp32 elements, "
                      f"OpenMP-backend evaluation order, {r['threads']} threads (OMP_PROC_BIND=close)"}


def _time_b2b(torch, fn, reps=10, warm=3):
    """Mean time of `reps` back-to-back launches between one event pair."""
    s = torch.cuda.current_stream()
    for _ in range(warm):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _time_op(torch, fn, reps=10, warm=3, flush=None, pre=None, hold_cycles=200000):
    """Median device time of single launches of fn, one event pair around
    each.  Before the start event the stream is kept busy on the GPU (the L2
    flush, or a spin of `hold_cycles` clock cycles, about 0.1 ms), so the
    host-side cost of enqueueing fn (Python, ctypes, argument checks) falls
    inside that work instead of showing up as idle GPU time between the
    events: the figure is the launch's own device time, ramp and drain
    included."""
    s = torch.cuda.current_stream()
    for _ in range(warm):
        if pre is not None:
            pre()
        fn()
    ts = []
    for _ in range(reps):
        if pre is not None:
            pre()  # untimed set-up of the launch's input
        if flush is not None:
            flush.sum()  # reads 512 MB: evicts L2 without leaving dirty lines to drain later
        elif hold_cycles:
            torch.cuda._sleep(hold_cycles)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def measure_ops(C, torch, np, peak, log2n=28, reps=10):
    """Per-primitive GB/s and fraction of measured HBM peak on arrays of
    2^log2n elements."""
    ops = {}
    n = 1 << log2n
    sz = f"2^{log2n}"

    def rec(name, fn, nbytes, note=None, flush=None):
        """Median of single launches (an event pair around each launch), and
        for inputs larger than L2 also the mean of 10 back-to-back launches."""
        ms = _time_op(torch, fn, reps=reps, flush=flush)
        gbs = nbytes / (ms / 1e3) / 1e9
        ops[name] = {"ms": round(ms, 4), "GB/s": round(gbs, 1), "frac_hbm": round(gbs / peak, 4),
                     "bytes": nbytes}
        if flush is None:
            b2b = nbytes / (_time_b2b(torch, fn, reps=reps) / 1e3) / 1e9
            ops[name]["b2b_GB/s"] = round(b2b, 1)
            ops[name]["b2b_frac_hbm"] = round(b2b / peak, 4)
        if note:
            ops[name]["note"] = note

    flush = torch.empty(1 << 27, dtype=torch.float32, device="cuda")  # 512 MB > L2
    xi = torch.from_numpy(C.synth_fill(0, 0, n, -1000, 1000)).cuda()
    yi = torch.empty_like(xi)
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    rec(f"reduce_i32_{sz}", lambda: C.reduce(xi, "sum", init=0, out=out), 4 * n)
    rec(f"scan_i32_{sz}", lambda: C.scan(xi, True, "sum", None, out=yi), 8 * n)
    if log2n == 28:
        x24 = xi[:N24]
        y24 = yi[:N24]
        rec("reduce_i32_2^24_flushed", lambda: C.reduce(x24, "sum", init=0, out=out), 4 * N24,
            "L2 flushed before each rep", flush=flush)
        rec("scan_i32_2^24_flushed", lambda: C.scan(x24, True, "sum", None, out=y24), 8 * N24,
            "L2 flushed before each rep", flush=flush)
    del xi, yi
    xf = torch.from_numpy(C.synth_fill(1, 1, n, 0.125, 1e-6)).cuda()
    bf = torch.from_numpy(C.synth_fill(1, 2, n, 0.125, 1e-6)).cuda()
    of = torch.zeros(1, dtype=torch.float32, device="cuda")
    rec(f"reduce_f32_{sz}", lambda: C.reduce(xf, "sum", init=0.0, out=of), 4 * n)
    rec(f"dot_f32_{sz}", lambda: C.dot(xf, bf, out=of), 8 * n)
    yf = torch.empty_like(xf)
    rec(f"scan_f32_{sz}", lambda: C.scan(xf, True, "sum", None, out=yf), 8 * n)
    del bf
    ab = torch.from_numpy(C.synth_fill(6, 1, n, 0.125, 1e-6).view(np.int16)).cuda().view(torch.bfloat16)
    bb = torch.from_numpy(C.synth_fill(6, 2, n, 0.125, 1e-6).view(np.int16)).cuda().view(torch.bfloat16)
    rec(f"dot_bf16_{sz}", lambda: C.dot(ab, bb, out=of), 4 * n)
    rec(f"scan_bf16in_f32out_{sz}", lambda: C.scan(ab, True, "sum", None, out=yf), 6 * n)
    del ab, bb, xf, yf
    xu = torch.from_numpy(C.synth_fill(3, 4, n)).cuda()
    yu = torch.empty_like(xu)
    rec(f"exclusive_scan_u32_{sz}", lambda: C.scan(xu, False, "sum", 0, out=yu), 8 * n)
    cnt = C.zeros(1, torch.uint64, "cuda")
    C.copy_if(xu, 7, C.CMP_LT, 3, out=yu, count=cnt)
    kept = int(cnt.item())
    rec(f"copy_if_u32_{sz}", lambda: C.copy_if(xu, 7, C.CMP_LT, 3, out=yu, count=cnt),
        4 * n + 4 * kept, f"kept {kept} ({kept / n:.4f})")
    del xu, yu
    # merge: two sorted halves of n int32 keys; sort: n random int32 keys,
    # restored from a copy before each rep (outside the timed pair)
    L = C.lib()
    sh = C._stream(None)
    g = torch.Generator(device="cuda").manual_seed(11)
    ma = torch.randint(-(1 << 31), 1 << 31, (n // 2,), generator=g, device="cuda", dtype=torch.int64)
    ma = ma.to(torch.int32).sort().values
    mb = torch.randint(-(1 << 31), 1 << 31, (n // 2,), generator=g, device="cuda", dtype=torch.int64)
    mb = mb.to(torch.int32).sort().values
    mo = torch.empty(n, dtype=torch.int32, device="cuda")
    msb = L.b2p_scratch_bytes(C.PRIM_MERGE, C.I32, n, 0, C.AUTO)
    mscr = torch.empty(msb, dtype=torch.uint8, device="cuda")
    rec(f"merge_i32_{sz}", lambda: C.check(L.b2p_merge(C.I32, ma.data_ptr(), n // 2, mb.data_ptr(), n // 2,
                                                       mo.data_ptr(), 0, mscr.data_ptr(), msb, sh)),
        8 * n, "two sorted halves; partition + merge-path tiles")
    del ma, mb
    keys0 = torch.randint(-(1 << 31), 1 << 31, (n,), generator=g, device="cuda", dtype=torch.int64)
    keys0 = keys0.to(torch.int32)
    ssb = L.b2p_scratch_bytes(C.PRIM_SORT, C.I32, n, 0, C.AUTO)
    sscr = torch.empty(ssb, dtype=torch.uint8, device="cuda")
    # 2^15 keys and more: the LSD radix sort, 4 digit passes of 8 bits over
    # int32 keys, each an upsweep read plus a downsweep read and write
    passes = 4
    nbytes = 3 * 4 * n * passes
    ms = _time_op(torch, lambda: C.check(L.b2p_sort(C.I32, mo.data_ptr(), n, 0, sscr.data_ptr(), ssb, sh)),
                  reps=reps, flush=None, pre=lambda: mo.copy_(keys0))
    gbs = nbytes / (ms / 1e3) / 1e9
    ops[f"sort_i32_{sz}"] = {"ms": round(ms, 4), "Gkeys/s": round(n / ms / 1e6, 2), "GB/s": round(gbs, 1),
                            "frac_hbm": round(gbs / peak, 4), "bytes": nbytes,
                            "note": f"random keys; LSD radix sort, {passes} passes of 8 bits "
                                    "(bytes = what those passes move)"}
    del keys0, mo, mscr, sscr
    k = torch.from_numpy(C.synth_fill(4, 5, n, 1.2)).cuda()
    bins = torch.zeros(256, dtype=torch.int32, device="cuda")
    rec(f"histogram_u8_zipf1.2_{sz}", lambda: C.histogram_u8(k, bins=bins), n + 1024)
    ku = torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda")
    rec(f"histogram_u8_uniform_{sz}", lambda: C.histogram_u8(ku, bins=bins), n + 1024)
    return ops


if __name__ == "__main__":
    main()
