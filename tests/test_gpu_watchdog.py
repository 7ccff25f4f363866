"""The watchdog's error path on the device, without stalling any copy.

Every wait of the TMA kernels is bounded; one that runs out sets the env's
sticky error flag. bfb_watchdog_selftest queues one such wait on a barrier
that nothing completes, so the flag is set exactly as a stalled copy would
set it, with nothing left in flight. Every entry point that hands the field
back must then report BFB_ERR_WATCHDOG, and bfb_step_host must leave the
caller's host field unchanged.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
WATCHDOG = -6


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_watchdog_run_out_is_reported_everywhere(bfb, precision):
    rng = np.random.default_rng(3)
    shape, S = (16, 12, 8), 2
    rho = rng.random((*shape, S))
    env = bfb.Env(shape, S, precision=precision)
    env.set_coefficients([1e3, 1e4], [0.1, 0.01])
    env.set_field(rho)
    env.synchronize()  # healthy so far
    env.watchdog_selftest(64)
    with pytest.raises(bfb.BFBError) as e:
        env.synchronize()
    assert e.value.code == WATCHDOG
    host = rho.reshape(-1).copy()
    L = bfb.load_library()
    rc = L.bfb_step_host(env.h, ctypes.c_void_p(host.ctypes.data), 0.01, 1)
    assert rc == WATCHDOG
    assert np.array_equal(host, rho.reshape(-1))  # untouched
    for call in (env.get_field, env.get_field_raw, env.checksum, env.gradients):
        with pytest.raises(bfb.BFBError) as e:
            call()
        assert e.value.code == WATCHDOG
    env.close()
    # a fresh env on the same device is unaffected
    env2 = bfb.Env(shape, S, precision=precision)
    env2.set_field(rho)
    env2.synchronize()
    env2.close()
