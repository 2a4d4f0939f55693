"""Learned schedule selector: data collection, training and evaluation.

Pipeline (everything on the GPU goes through libb2p's C-ABI):

1. ``sample_shapes``: call shapes log-uniform over 2^10 .. 2^28 elements,
   random primitive (reduce, scan, copy_if, histogram; a quarter of the
   reduce/scan shapes segmented) and dtype (int32, int64, fp32, bf16).
2. ``collect``: the exhaustive autotuner (b2p_tune_shape) times every valid
   launch configuration of every shape (median of `reps` launches).
3. ``Selector.train``: the 11 -> 64 -> 64 -> 48 MLP is trained with the
   library's CUDA forward/backward/Adam kernels (b2p_selector_train).
4. ``evaluate_stream``: a seeded stream of calls with random op, dtype and
   size is executed end to end under three policies -- the learned selector,
   the exhaustive tuner's table (best configuration of the nearest tuned
   shape) and the fixed heuristic -- and per-call regret is measured on a
   sample of the calls by timing every configuration of their exact shape.

The selector only picks the launch configuration; results never depend on
it (integers are bit-exact for every configuration).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import time

import numpy as np

from . import capi as C

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")
DATASET = os.path.join(DATA, "tuning_b200.npz")
WEIGHTS = os.path.join(DATA, "selector_b200.bin")

DTYPES = [C.I32, C.I64, C.F32, C.BF16]
OPS = [C.PRIM_REDUCE, C.PRIM_SCAN, C.PRIM_COPY_IF, C.PRIM_HISTOGRAM]


def _rng(seed):
    return np.random.default_rng(seed)


def sample_shapes(count: int, seed: int = 9, lo: int = 10, hi: int = 28, seg_frac: float = 0.25):
    """Shapes as dicts {prim, dtype, n, nseg, cv}."""
    r = _rng(seed)
    out = []
    for _ in range(count):
        op = OPS[r.integers(len(OPS))]
        dt = DTYPES[r.integers(len(DTYPES))]
        n = int(round(2.0 ** r.uniform(lo, hi)))
        prim, nseg, cv = op, 0, 0.0
        if op == C.PRIM_COPY_IF and dt == C.BF16:
            dt = C.F32
        if op == C.PRIM_HISTOGRAM:
            dt = C.U32
        if op in (C.PRIM_REDUCE, C.PRIM_SCAN) and r.random() < seg_frac:
            prim = C.PRIM_SEG_REDUCE if op == C.PRIM_REDUCE else C.PRIM_SEG_SCAN
            nseg = int(min(n // 2, round(2.0 ** r.uniform(1, 14))))
            nseg = max(nseg, 2)
            cv = float(r.uniform(0.0, 3.0))
        out.append({"prim": prim, "dtype": dt, "n": n, "nseg": nseg, "cv": cv})
    return out


def features(shapes) -> np.ndarray:
    L = C.lib()
    X = np.zeros((len(shapes), C.SEL_FEATURES), dtype=np.float32)
    for i, s in enumerate(shapes):
        f = (ctypes.c_float * C.SEL_FEATURES)()
        C.check(L.b2p_selector_features(s["prim"], s["dtype"], s["n"], s["nseg"], s["cv"], f))
        X[i] = np.frombuffer(f, dtype=np.float32)
    return X


def tune(shape, reps: int = 5, seed: int = 1) -> np.ndarray:
    """Median time (ms) of every configuration for one shape (+inf = masked)."""
    L = C.lib()
    t = (ctypes.c_float * C.NUM_CONFIGS)()
    op = C.SUM
    C.check(L.b2p_tune_shape(shape["prim"], shape["dtype"], op, shape["n"], shape["nseg"],
                             shape["cv"], reps, seed, t), "b2p_tune_shape")
    return np.frombuffer(t, dtype=np.float32).copy()


def collect(shapes, reps: int = 5, progress=None) -> np.ndarray:
    T = np.full((len(shapes), C.NUM_CONFIGS), np.inf, dtype=np.float32)
    for i, s in enumerate(shapes):
        T[i] = tune(s, reps, seed=1000 + i)
        if progress and i % 100 == 0:
            progress(i, len(shapes))
    return T


def save_dataset(path, shapes, X, T, meta=None):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, X=X, T=T, shapes=json.dumps(shapes), meta=json.dumps(meta or {}))


def load_dataset(path=DATASET):
    d = np.load(path, allow_pickle=False)
    return json.loads(str(d["shapes"])), d["X"], d["T"], json.loads(str(d["meta"]))


class Selector:
    """Handle on a b2p_selector (weights live on the GPU)."""

    def __init__(self, seed: int = 1):
        self.L = C.lib()
        self.h = ctypes.c_void_p()
        C.check(self.L.b2p_selector_create(ctypes.byref(self.h), seed), "b2p_selector_create")

    def __del__(self):
        try:
            if self.h:
                self.L.b2p_selector_destroy(self.h)
        except Exception:
            pass

    @staticmethod
    def _fp(a):
        return np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(ctypes.POINTER(ctypes.c_float))

    def train(self, X, T, epochs=3000, lr=2e-3, ce_weight=0.05) -> float:
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = ctypes.c_float()
        C.check(self.L.b2p_selector_train(self.h, self._fp(X), self._fp(T), X.shape[0], epochs, lr,
                                          ce_weight, ctypes.byref(loss)), "b2p_selector_train")
        return float(loss.value)

    def grad(self, X, T, ce_weight=0.05):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = ctypes.c_float()
        g = np.zeros(self.L.b2p_selector_num_params(), dtype=np.float32)
        C.check(self.L.b2p_selector_grad(self.h, self._fp(X), self._fp(T), X.shape[0], ce_weight,
                                         ctypes.byref(loss),
                                         g.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return float(loss.value), g

    def predict(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros(X.shape[0], dtype=np.int32)
        C.check(self.L.b2p_selector_predict(self.h, self._fp(X), X.shape[0],
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out

    def params(self) -> np.ndarray:
        p = np.zeros(self.L.b2p_selector_num_params(), dtype=np.float32)
        C.check(self.L.b2p_selector_get_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        C.check(self.L.b2p_selector_set_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def save(self, path=WEIGHTS):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        C.check(self.L.b2p_selector_save(self.h, path.encode()), "b2p_selector_save")

    def load(self, path=WEIGHTS) -> bool:
        return self.L.b2p_selector_load(self.h, path.encode()) == C.OK

    def install(self):
        C.check(self.L.b2p_selector_install(self.h), "b2p_selector_install")


def masks_for(shapes) -> np.ndarray:
    L = C.lib()
    M = np.zeros((len(shapes), C.NUM_CONFIGS), dtype=bool)
    for i, s in enumerate(shapes):
        for c in range(C.NUM_CONFIGS):
            M[i, c] = bool(L.b2p_config_valid(s["prim"], s["dtype"], c))
    return M


def heuristic(shapes) -> np.ndarray:
    L = C.lib()
    return np.array([L.b2p_heuristic_config(s["prim"], s["dtype"], s["n"], s["nseg"]) for s in shapes],
                    dtype=np.int32)


def table_policy(train_shapes, train_T, shapes) -> np.ndarray:
    """The exhaustive tuner's table: best configuration of the nearest tuned
    shape with the same primitive and dtype (log2 n distance)."""
    best = np.argmin(train_T, axis=1)
    keys = {}
    for i, s in enumerate(train_shapes):
        keys.setdefault((s["prim"], s["dtype"]), []).append((math.log2(s["n"]), int(best[i])))
    out = []
    for s in shapes:
        cand = keys.get((s["prim"], s["dtype"]))
        if not cand:
            out.append(int(C.lib().b2p_heuristic_config(s["prim"], s["dtype"], s["n"], s["nseg"])))
            continue
        ln = math.log2(s["n"])
        out.append(min(cand, key=lambda c: abs(c[0] - ln))[1])
    return np.array(out, dtype=np.int32)


# --------------------------------------------------------------- evaluation

class StreamRunner:
    """Executes a stream of non-segmented calls on preallocated buffers."""

    def __init__(self, max_n: int):
        import torch
        self.torch = torch
        self.max_n = max_n
        self.buf_in = torch.empty(max_n * 8 + 256, dtype=torch.uint8, device="cuda")
        self.buf_out = torch.empty(max_n * 8 + 256, dtype=torch.uint8, device="cuda")
        self.buf_in.random_(0, 7)  # small integers / denormal-free floats
        self.small = torch.zeros(4096, dtype=torch.int64, device="cuda")
        L = C.lib()
        sb = max(L.b2p_scratch_bytes(p, d, max_n, 0, C.AUTO) for p in (0, 1, 2) for d in (0, 1, 4, 5))
        self.scratch = torch.zeros(sb + 512, dtype=torch.uint8, device="cuda")
        self.sp = ctypes.c_void_p((self.scratch.data_ptr() + 255) & ~255)
        self.sb = sb
        self.stream = torch.cuda.current_stream()
        self.sh = ctypes.c_void_p(self.stream.cuda_stream)
        self.L = L

    def call(self, s, cfg):
        L, n = self.L, s["n"]
        inp, out = self.buf_in.data_ptr(), self.buf_out.data_ptr()
        p = s["prim"]
        if p == C.PRIM_REDUCE:
            return L.b2p_reduce(s["dtype"], C.SUM, inp, n, self.small.data_ptr(), None, self.sp, self.sb, cfg, self.sh)
        if p == C.PRIM_SCAN:
            return L.b2p_scan(s["dtype"], C.SUM, 1, inp, out, n, None, self.sp, self.sb, cfg, self.sh)
        if p == C.PRIM_COPY_IF:
            return L.b2p_copy_if(s["dtype"], inp, out, n, 7, C.CMP_LT, 3, self.small.data_ptr(), self.sp,
                                 self.sb, cfg, self.sh)
        return L.b2p_histogram_u8(inp, n, self.small.data_ptr(), 256, cfg, self.sh)

    def run(self, shapes, cfgs) -> float:
        torch = self.torch
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for s, c in zip(shapes, cfgs):
            rc = self.call(s, int(c))
            if rc:
                raise C.B2PError(rc, "stream call")
        e1.record(self.stream)
        e1.synchronize()
        return e0.elapsed_time(e1)


def stream_shapes(count: int, seed: int = 10, lo=10, hi=28):
    return sample_shapes(count, seed=seed, lo=lo, hi=hi, seg_frac=0.0)


def evaluate_stream(sel: Selector, train_shapes, train_T, ncalls=100000, seed=10, regret_sample=200,
                    hi=28):
    shapes = stream_shapes(ncalls, seed, hi=hi)
    X = features(shapes)
    t0 = time.perf_counter()
    learned = sel.predict(X)
    t_predict = time.perf_counter() - t0
    pol = {"learned": learned, "exhaustive_table": table_policy(train_shapes, train_T, shapes),
           "heuristic": heuristic(shapes)}
    runner = StreamRunner(max(s["n"] for s in shapes))
    for name, cfgs in pol.items():  # warm-up
        runner.run(shapes[:200], cfgs[:200])
    times = {name: runner.run(shapes, cfgs) for name, cfgs in pol.items()}
    # per-call regret against the exhaustive tuner on the exact shape
    r = _rng(seed + 1)
    idx = r.choice(len(shapes), size=min(regret_sample, len(shapes)), replace=False)
    regret = {k: [] for k in pol}
    best_sum = {k: 0.0 for k in pol}
    opt_sum = 0.0
    for i in idx:
        t = tune(shapes[i], reps=5, seed=77 + int(i))
        tb = float(np.min(t))
        opt_sum += tb
        for k, cfgs in pol.items():
            tk = float(t[cfgs[i]])
            regret[k].append(tk / tb - 1.0)
            best_sum[k] += tk
    opt_sum = opt_sum or float("nan")
    return {
        "ncalls": ncalls, "seed": seed, "stream_ms": times,
        "learned_vs_exhaustive_table": times["learned"] / times["exhaustive_table"],
        "heuristic_vs_learned": times["heuristic"] / times["learned"],
        "calls_per_s": {k: ncalls / (v / 1e3) for k, v in times.items()},
        "predict_s_for_stream": t_predict,
        "regret_sample": len(idx),
        "mean_regret": {k: (float(np.mean(v)) if v else None) for k, v in regret.items()},
        "sample_time_vs_best": {k: best_sum[k] / opt_sum for k in pol},
    }


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="collect / train / evaluate the schedule selector")
    ap.add_argument("step", choices=["collect", "train", "eval", "all"])
    ap.add_argument("--shapes", type=int, default=2000)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--calls", type=int, default=100000)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--dataset", default=DATASET)
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--out", default=None, help="write the evaluation JSON here")
    ap.add_argument("--only-prims", default=None,
                    help="collect: re-time only the rows of these primitive ids (comma separated) in the "
                         "existing dataset, keeping the others")
    a = ap.parse_args(argv)
    if a.step == "collect" and a.only_prims:
        prims = {int(v) for v in a.only_prims.split(",")}
        shapes, X, T, meta = load_dataset(a.dataset)
        rows = [i for i, s in enumerate(shapes) if s["prim"] in prims]
        t0 = time.time()
        for k, i in enumerate(rows):
            T[i] = tune(shapes[i], a.reps, seed=1000 + i)
            if k % 50 == 0:
                print(f"re-tuned {k}/{len(rows)}", flush=True)
        meta = dict(meta, retuned={"prims": sorted(prims), "rows": len(rows), "seconds": time.time() - t0})
        save_dataset(a.dataset, shapes, X, T, meta)
        print("dataset", a.dataset, "re-tuned rows", len(rows), f"{time.time() - t0:.1f}s", flush=True)
        return
    if a.step in ("collect", "all"):
        shapes = sample_shapes(a.shapes, seed=9)
        X = features(shapes)
        t0 = time.time()
        T = collect(shapes, a.reps, progress=lambda i, n: print(f"tuned {i}/{n}", flush=True))
        save_dataset(a.dataset, shapes, X, T, {"reps": a.reps, "seconds": time.time() - t0,
                                               "gpu": _gpu_name()})
        print("dataset", a.dataset, T.shape, f"{time.time() - t0:.1f}s", flush=True)
    if a.step in ("train", "all"):
        shapes, X, T, _ = load_dataset(a.dataset)
        sel = Selector(seed=1)
        t0 = time.time()
        loss = sel.train(X, T, epochs=a.epochs)
        sel.save(a.weights)
        print("trained", f"loss={loss:.4f}", f"{time.time() - t0:.1f}s", flush=True)
    if a.step in ("eval", "all"):
        shapes, X, T, _ = load_dataset(a.dataset)
        sel = Selector(seed=1)
        if not sel.load(a.weights):
            sel.train(X, T, epochs=a.epochs)
        res = evaluate_stream(sel, shapes, T, ncalls=a.calls)
        print(json.dumps(res), flush=True)
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f, indent=1)


def _gpu_name():
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


if __name__ == "__main__":
    main()
