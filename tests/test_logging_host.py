"""Host-side checks of the library's environment switches (no GPU work):
B2P_LOG_LEVEL and the reference's ACPP_DEBUG_LEVEL / HIPSYCL_DEBUG_LEVEL
fallbacks (common/debug.hpp:14-21,61), error records on stderr, and the
exported log-level calls.  Each case runs in a child process because the
level is read once per process."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import ctypes, sys
sys.path.insert(0, %r)
from opensycl_b200 import capi as C
L = C.lib()
print("LEVEL", L.b2p_log_level())
# an invalid dtype is rejected before any device work; at level >= 1 the
# rejection is logged
L.b2p_merge(99, None, 1, None, 1, None, 0, None, 0, None)
L.b2p_set_log_level(0)
print("LEVEL", L.b2p_log_level())
L.b2p_merge(99, None, 1, None, 1, None, 0, None, 0, None)
""" % ROOT


def run_probe(env_extra):
    env = {k: v for k, v in os.environ.items()
           if k not in ("B2P_LOG_LEVEL", "ACPP_DEBUG_LEVEL", "HIPSYCL_DEBUG_LEVEL")}
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", PROBE], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    levels = [int(l.split()[1]) for l in r.stdout.splitlines() if l.startswith("LEVEL")]
    return levels, r.stderr


def test_exports():
    from opensycl_b200 import capi as C
    L = C.lib()
    assert hasattr(L, "b2p_log_level") and hasattr(L, "b2p_set_log_level")


@pytest.mark.parametrize("env,level", [({}, 2), ({"B2P_LOG_LEVEL": "3"}, 3), ({"ACPP_DEBUG_LEVEL": "1"}, 1),
                                       ({"HIPSYCL_DEBUG_LEVEL": "4"}, 4),
                                       ({"B2P_LOG_LEVEL": "0", "ACPP_DEBUG_LEVEL": "3"}, 0),
                                       ({"B2P_LOG_LEVEL": "x"}, 2)])
def test_level_from_environment(env, level):
    levels, err = run_probe(env)
    assert levels == [level, 0]
    lines = [l for l in err.splitlines() if l.startswith("[b2p")]
    if level >= 1:
        # one error record for the first rejected call, none after level 0
        assert len(lines) == 1 and lines[0].startswith("[b2p error] b2p_merge"), err
    else:
        assert not lines, err
