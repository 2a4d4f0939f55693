"""Failure detection without a GPU fault: every look-back wait in the scan
and copy_if kernels is bounded.  A test hook makes one tile never publish
its status; its successors' waits run out after a short limit, the kernel
records B2P_ERR_TIMEOUT in the scratch error word and returns, and the
context stays usable for the next call.  No trap, no fault, no endless loop.
"""
import time

import numpy as np
import pytest
import torch

from opensycl_b200 import capi as C

pytestmark = pytest.mark.gpu


@pytest.fixture
def short_timeout():
    L = C.lib()
    old = L.b2p_set_wait_timeout_ns(200_000_000)  # 0.2 s
    yield
    L.b2p_debug_stall_tile(-1)
    L.b2p_set_wait_timeout_ns(old)


@pytest.mark.parametrize("prim", ["scan", "copy_if"])
# look-back kernel (128 x 4 tiles) / two-phase kernel (128 x 4) / pipelined
# TMEM-staged scan and copy_if (256 x 32 = 8192-element tiles), with one
# tile per block and with several (the rings of stages and TMEM slots wrap)
@pytest.mark.parametrize("config,stall,n", [(0, 37, 512 * 200), (16, 37, 512 * 200), (23, 5, 512 * 200),
                                            (23, 150, 8192 * 400 + 77)])
def test_stalled_tile_times_out_and_context_survives(dev, short_timeout, prim, config, stall, n):
    L = C.lib()
    x = torch.arange(n, dtype=torch.int32, device="cuda")
    C.device_error(clear=True)
    L.b2p_debug_stall_tile(stall)
    t0 = time.time()
    if prim == "scan":
        C.scan(x, True, "sum", None, config=config)
    else:
        C.copy_if(x, 1, C.CMP_EQ, 0, config=config)
    err = C.device_error(clear=True)
    dt = time.time() - t0
    L.b2p_debug_stall_tile(-1)
    assert err == C.ERR_TIMEOUT
    assert dt < 30.0
    # the same scratch and context keep working
    y = C.scan(x, True, "sum", None, config=config)
    ref = (np.cumsum(np.arange(n, dtype=np.int64)) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)
    assert np.array_equal(y.cpu().numpy(), ref)
    assert C.device_error(clear=True) == C.OK
