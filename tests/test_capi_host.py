"""C-ABI checks that need no GPU: the library loads, exports every function
include/b2p.h declares, and its host-side logic (configuration table,
scratch sizing, validation, synthetic inputs) behaves."""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

from opensycl_b200 import capi as C

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def test_library_exports_every_declared_function():
    syms = subprocess.run(["nm", "-D", "--defined-only", C.LIB_PATH], capture_output=True,
                          text=True, check=True).stdout
    declared = C.header_functions()
    assert len(declared) >= 30
    missing = [f for f in declared if f" T {f}" not in syms]
    assert not missing, missing
    L = C.lib()
    for f in declared:
        assert hasattr(L, f)


def test_library_builds_for_sm100a_only():
    """Every translation unit is compiled with one -gencode target, sm_100a
    machine code (no PTX, no other architecture); the GPU-side check of the
    loaded kernels is tests/test_gpu_parity.py::test_kernels_are_sm100a."""
    from opensycl_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert not any("gencode" in f or "arch" in f for f in B.COMMON)


def test_config_table():
    seen = set()
    for c in range(C.NUM_CONFIGS):
        b, it, g = C.config_describe(c)
        assert b in (128, 256, 512, 1024) and it in (4, 8, 16, 32) and g in (0, 1, 2)
        seen.add((b, it, g))
    assert len(seen) == 48
    with pytest.raises(C.B2PError):
        C.config_describe(48)
    L = C.lib()
    # tiles above 8192 elements are masked for scans; reductions take all
    assert sum(L.b2p_config_valid(C.PRIM_SCAN, C.F32, c) for c in range(48)) == 39
    assert sum(L.b2p_config_valid(C.PRIM_REDUCE, C.F32, c) for c in range(48)) == 48
    for prim in (C.PRIM_REDUCE, C.PRIM_SCAN, C.PRIM_COPY_IF, C.PRIM_HISTOGRAM):
        c = L.b2p_heuristic_config(prim, C.F32, 1 << 20, 0)
        assert L.b2p_config_valid(prim, C.F32, c)
        a = L.b2p_auto_config(prim, C.F32, 1 << 20, 0, 0.0)
        assert L.b2p_config_valid(prim, C.F32, a)


def test_scratch_sizes():
    L = C.lib()
    prefix = 256 + 4 * 1024  # header + fixed arrival-counter block
    # reduce: one 16-byte word per run; runs bounded (2368..4736) for large n
    r28 = L.b2p_scratch_bytes(C.PRIM_REDUCE, C.F32, 1 << 28, 0, C.AUTO)
    assert prefix < r28 <= prefix + 16 * 4736 * 2
    assert L.b2p_scratch_bytes(C.PRIM_REDUCE, C.F32, 10, 0, C.AUTO) == prefix + 16
    # scan: one 16-byte word per tile and per chunk; AUTO covers the smallest tile (512)
    n = 1 << 20
    auto = L.b2p_scratch_bytes(C.PRIM_SCAN, C.F32, n, 0, C.AUTO)
    assert auto >= prefix + 16 * (n // 512)
    for c in range(48):
        b, it, _ = C.config_describe(c)
        got = L.b2p_scratch_bytes(C.PRIM_SCAN, C.F32, n, 0, c)
        assert prefix + 16 * (n // (b * it)) < got <= auto


def test_status_strings():
    L = C.lib()
    for s in range(9):
        assert len(L.b2p_status_string(s)) > 0


def test_synth_generator_pins():
    pins = GOLD["synth"]
    assert C.synth_fill(0, 0, 16, -1000, 1000).tolist() == pins["int32_seed0"]
    got = C.synth_fill(1, 1, 16, 0.125, 1e-6)
    assert np.array_equal(got, np.array(pins["fp32_seed1_frac0.125"], dtype=np.float32))
    assert C.synth_fill(3, 4, 16).tolist() == pins["uint32_seed4"]


def test_synth_distributions():
    x = C.synth_fill(1, 1, 1 << 20, 0.125, 1e-6)
    big = np.abs(x) > 1e-3
    assert 0.86 < big.mean() < 0.89          # 1/8 replaced by 1e-6 * N(0,1)
    assert abs(x[big].std() - 1.0) < 0.01
    z = C.synth_fill(4, 5, 1 << 20, 1.2)
    h = np.bincount(z, minlength=256) / z.size
    H = sum(r ** -1.2 for r in range(1, 257))
    assert abs(h[0] - 1 / H) < 0.005 and abs(h[1] - 2 ** -1.2 / H) < 0.005
    b = C.synth_fill(6, 1, 1000, 0.125, 1e-6)
    f = C.synth_fill(1, 1, 1000, 0.125, 1e-6)
    back = (b.astype(np.uint32) << 16).view(np.float32)
    assert np.all(np.abs(back - f) <= np.abs(f) * 2 ** -8)


def test_synth_segments_cap():
    offs = C.synth_segments(6, 10000, 20.0, 1 << 28)
    lens = np.diff(offs)
    assert offs[0] == 0 and offs[-1] <= 1 << 28 and offs[-1] > 0.99 * (1 << 28)
    assert lens.min() >= 1 and lens.max() <= 1 << 20


def test_calls_without_device_fail_cleanly():
    """On a machine without a GPU every compute entry point returns an error
    status instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("host-only check")
    L = C.lib()
    buf = np.zeros(64, dtype=np.float32)
    out = np.zeros(1, dtype=np.float32)
    p = buf.ctypes.data_as(ctypes.c_void_p)
    rc = L.b2p_reduce(C.F32, C.SUM, p, 64, out.ctypes.data_as(ctypes.c_void_p), None, p, 256, 0, None)
    assert rc != C.OK
    assert out[0] == 0
