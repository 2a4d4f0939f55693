"""Selector pieces that need no GPU: the feature encoding, the numpy
oracle's gradients (pinned by finite differences) and the data sampler."""
import ctypes

import numpy as np

from opensycl_b200 import capi as C
from opensycl_b200 import selector as S
from oracle import mlp as M


def test_feature_encoding():
    L = C.lib()
    f = (ctypes.c_float * 11)()
    assert L.b2p_selector_features(C.PRIM_SCAN, C.BF16, 1 << 20, 0, 0.0, f) == C.OK
    v = np.frombuffer(f, np.float32)
    assert abs(v[0] - 20 / 32) < 1e-6 and v[4] == 1 and v[6] == 1 and v[9] == 0 and v[10] == 0
    assert L.b2p_selector_features(C.PRIM_SEG_REDUCE, C.I64, 1 << 24, 1000, 2.0, f) == C.OK
    v = np.frombuffer(f, np.float32)
    assert v[2] == 1 and v[5] == 1 and v[9] > 0 and abs(v[10] - 0.5) < 1e-6
    assert L.b2p_selector_features(C.PRIM_HISTOGRAM, C.U32, 1 << 24, 0, 0.0, f) == C.OK
    v = np.frombuffer(f, np.float32)
    assert v[1:5].sum() == 0 and v[8] == 1


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(8048) * 0.2
    X = rng.random((6, 11))
    T = rng.random((6, 48)) + 0.1
    T[:, ::7] = np.inf
    _, g = M.loss_and_grad(p, X, T, 0.05)
    for k in rng.choice(8048, 40, replace=False):
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (M.loss_and_grad(p + e, X, T, 0.05)[0] - M.loss_and_grad(p - e, X, T, 0.05)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-5 + 1e-4 * abs(g[k])


def test_shape_sampler():
    sh = S.sample_shapes(500, seed=9)
    ns = np.array([s["n"] for s in sh])
    assert ns.min() >= 2 ** 10 and ns.max() <= 2 ** 28
    assert len({s["prim"] for s in sh}) == 6
    assert all(s["nseg"] >= 2 for s in sh if s["prim"] in (C.PRIM_SEG_REDUCE, C.PRIM_SEG_SCAN))
    assert sh == S.sample_shapes(500, seed=9)
    m = S.masks_for(sh[:50])
    assert m.any(axis=1).all()
    h = S.heuristic(sh[:50])
    assert all(m[i, h[i]] for i in range(50))
