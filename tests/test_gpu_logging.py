"""The environment switches on a GPU: B2P_LOG_LEVEL call records (level 3:
one line per call with its configuration; level 4: timed on the stream),
B2P_CHECKED extent and offset checks, and B2P_SELECTOR.  Each case runs in
a child process (the switches are read once per process).  The checked-mode
cases pass a NULL scratch buffer: without the check the call stops at the
scratch check, with it at the extent or offset check, so neither launches
anything."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HEAD = r"""
import ctypes, sys
sys.path.insert(0, %r)
import numpy as np, torch
from opensycl_b200 import capi as C
L = C.lib()
""" % ROOT


def run(code, env_extra):
    env = {k: v for k, v in os.environ.items()
           if k not in ("B2P_LOG_LEVEL", "ACPP_DEBUG_LEVEL", "HIPSYCL_DEBUG_LEVEL", "B2P_CHECKED", "B2P_SELECTOR")}
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", HEAD + code], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout, r.stderr


CALLS = r"""
x = torch.ones(1 << 20, dtype=torch.float32, device="cuda")
out = torch.zeros(1, dtype=torch.float32, device="cuda")
C.reduce(x, "sum", init=0.0, out=out)
y = C.scan(x, True, "sum")
torch.cuda.synchronize()
print("SUM", float(out.item()), float(y[-1].item()))
"""


def test_level3_records_each_call_with_its_configuration():
    out, err = run(CALLS, {"B2P_LOG_LEVEL": "3"})
    assert "SUM 1048576.0 1048576.0" in out
    recs = [l for l in err.splitlines() if l.startswith("[b2p info]")]
    assert any(l.startswith("[b2p info] b2p_reduce dtype=f32 n=1048576 nseg=0 config=") and "status=0" in l
               for l in recs), err
    assert any(l.startswith("[b2p info] b2p_scan dtype=f32 n=1048576") for l in recs), err
    assert all("config=-1" not in l for l in recs), err


def test_level4_records_are_timed():
    out, err = run(CALLS, {"B2P_LOG_LEVEL": "4"})
    assert "SUM 1048576.0 1048576.0" in out
    recs = [l for l in err.splitlines() if l.startswith("[b2p verbose] b2p_reduce")]
    assert recs and " time=" in recs[0] and recs[0].endswith("GB/s"), err
    ms = float(recs[0].split(" time=")[1].split()[0])
    assert 0 < ms < 1000


CHECKED = r"""
x = torch.ones(1 << 20, dtype=torch.float32, device="cuda")
out = torch.zeros(1, dtype=torch.float32, device="cuda")
# far more elements than any allocation holds, and no scratch
print("REDUCE", L.b2p_reduce(C.F32, C.SUM, x.data_ptr(), 1 << 40, out.data_ptr(), None, None, 0, -1, None))
offs = torch.tensor([0, 10, 5, 20], dtype=torch.int64, device="cuda")  # not non-decreasing
o2 = torch.zeros(3, dtype=torch.float32, device="cuda")
print("SEG", L.b2p_segmented_reduce(C.F32, C.SUM, x.data_ptr(), offs.data_ptr(), 3, o2.data_ptr(), None, None, 0,
                                    -1, None))
"""


def test_checked_mode_rejects_extents_and_offsets():
    out, _ = run(CHECKED, {"B2P_CHECKED": "1"})
    assert "REDUCE %d" % 2 in out and "SEG %d" % 1 in out, out   # INVALID_PTR, INVALID_ARG
    out, _ = run(CHECKED, {})
    assert "REDUCE %d" % 6 in out and "SEG %d" % 6 in out, out   # ERR_SCRATCH


SELECT = r"""
import bench
shapes = [(C.PRIM_SCAN, C.F32, 1 << 26), (C.PRIM_REDUCE, C.I32, 1 << 18), (C.PRIM_COPY_IF, C.U32, 1 << 24),
          (C.PRIM_SCAN, C.BF16, 1 << 12), (C.PRIM_REDUCE, C.F32, 1 << 28)]
before = [L.b2p_auto_config(p, d, n, 0, 0.0) for p, d, n in shapes]
heur = [L.b2p_heuristic_config(p, d, n, 0) for p, d, n in shapes]
st = bench.install_selector(C)
after = [L.b2p_auto_config(p, d, n, 0, 0.0) for p, d, n in shapes]
print("BEFORE", before)
print("HEUR", heur)
print("AFTER", after)
"""


def parse(out, key):
    line = [l for l in out.splitlines() if l.startswith(key)][0]
    return [int(v) for v in line.split("[")[1].rstrip("]").split(",")]


def test_selector_environment():
    weights = os.path.join(ROOT, "opensycl_b200", "data", "selector_b200.bin")
    # default: AUTO is the heuristic until a table is installed, then the table
    out, _ = run(SELECT, {})
    learned = parse(out, "AFTER")
    assert parse(out, "BEFORE") == parse(out, "HEUR")
    # heuristic: the installed table is ignored
    out, _ = run(SELECT, {"B2P_SELECTOR": "heuristic"})
    assert parse(out, "AFTER") == parse(out, "HEUR")
    # a weights path: installed at the first AUTO call, without Python
    out, _ = run(SELECT, {"B2P_SELECTOR": weights})
    assert parse(out, "BEFORE") == learned
