"""ORACLE — test infrastructure only: the timed CPU baseline.

Times the oracle's restatement of the reference's OpenMP-backend evaluation
order (oracle.c: transform_reduce dot as 8-element work-items + 128-wide
trees, numeric.hpp:67-161; inclusive_scan as 16x1024-element tiles scanned
by one leader with a single write per element,
decoupled_lookback_scan.hpp:137-177) on the benchmark's headline workload:
an fp32 dot of two 2^log2n arrays and an fp32 inclusive scan of a third,
generated by the oracle's own copy of the seeded generator.

Run as a separate process so that every caller gets the same OpenMP
placement: the benchmark's reference arm and the CPU-baseline leg of its
GPU arm both launch it through ``run()``, with OMP_PROC_BIND=close,
OMP_PLACES=threads and OMP_NUM_THREADS = the CPUs this process may use.

    python -m oracle.baseline --log2n 28 --steps 20 --warmup 3

prints one JSON object: GB/s over the algorithmic bytes (16 bytes per
element: dot 8, scan 8), ms per step, threads, CPU model and the fp32
errors of the timed results against FP64.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def omp_env() -> dict:
    env = dict(os.environ)
    try:
        ncpu = len(os.sched_getaffinity(0))
    except AttributeError:
        ncpu = os.cpu_count() or 1
    env.update(OMP_NUM_THREADS=str(ncpu), OMP_PROC_BIND="close", OMP_PLACES="threads",
               OMP_WAIT_POLICY="active")
    return env


def run(log2n: int, steps: int, warmup: int, timeout: float = 900.0) -> dict:
    """Launch the baseline in a fresh process and return its JSON result."""
    cmd = [sys.executable, "-m", "oracle.baseline", "--log2n", str(log2n), "--steps", str(steps),
           "--warmup", str(warmup)]
    r = subprocess.run(cmd, cwd=ROOT, env=omp_env(), capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"oracle baseline failed: {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--log2n", type=int, default=28)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=1)
    args = ap.parse_args()

    import numpy as np

    sys.path.insert(0, ROOT)
    from oracle import oracle as O

    n = 1 << args.log2n
    a = O.synth_fill(1, 1, n, 0.125, 1e-6)
    b = O.synth_fill(1, 2, n, 0.125, 1e-6)
    x = O.synth_fill(2, 3, n, 0.125, 1e-6)
    y = np.zeros(n, dtype=np.float32)
    y[:] = 1.0  # pages mapped before timing, as a caller's output buffer would be

    def step():
        d = O.dot(O.F32, a, b, 0.0)
        O.scan(O.F32, O.SUM, True, x, out=y)
        return d

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        d = step()
    dt = time.perf_counter() - t0
    ref, cond = O.fp64_sum(O.F32, a, b)
    sref = O.fp64_scan(O.F32, True, x)
    rel_s = float(np.max(np.abs(y.astype(np.float64) - sref) / np.maximum(np.abs(sref), 1e-300)))
    print(json.dumps({
        "value": 16.0 * n * args.steps / dt / 1e9, "unit": "GB/s", "ms_per_step": dt / args.steps * 1e3,
        "steps": args.steps, "warmup": args.warmup, "elements": n, "threads": O.num_threads(),
        "omp": {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OMP_PROC_BIND", "OMP_PLACES")},
        "cpu_model": cpu_model(), "dot_rel_err_vs_fp64": abs(float(d) - ref) / abs(ref),
        "dot_cond_err": abs(float(d) - ref) / cond, "scan_max_rel_err_vs_fp64": rel_s,
    }), flush=True)


if __name__ == "__main__":
    main()
