"""Failure paths of the device, exercised without a GPU fault.

* A bounded wait that runs out: one warp waits on an mbarrier that nothing
  arrives at, with the same clock budget as every tensor-core completion and
  bulk-copy wait (about 2^31 clocks).  The call returns CHAPSIM_ERR_TIMEOUT
  after about a second, the error word is cleared, and the context keeps
  stepping.
* A non-finite field and a collapsing time step are reported by their codes
  (the host plants them: a NaN in an uploaded field, a tiny CFLGV).
"""
import math
import time

import numpy as np
import pytest

from chapsim import gpu
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu


def _channel():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 3, 0.1)
    c = gpu.ChannelTG(s)
    c.upload(Q, PR)
    c.set_dt(1e-3)
    return c, Q, PR


def test_bounded_wait_times_out_and_context_survives():
    c, Q, PR = _channel()
    t0 = time.perf_counter()
    rc = c.lib.chapsim_probe_wait_timeout(c.h)
    waited = time.perf_counter() - t0
    print("timeout after %.2f s" % waited)
    assert rc == -5  # CHAPSIM_ERR_TIMEOUT
    assert 0.1 < waited < 30.0
    dt, cfl = c.advance(3, 1e-3, 1e-6, 0.5)
    assert math.isfinite(dt) and math.isfinite(cfl)
    Q2, _ = c.download()
    assert np.isfinite(Q2).all()
    c.close()


def test_nan_and_dt_collapse_codes():
    c, Q, PR = _channel()
    Qn = Q.copy()
    Qn[0, 3, 5, 7] = float("nan")
    c.upload(Qn, PR)
    with pytest.raises(gpu.ChapsimError) as e:
        c.advance(1, 1e-3, 1e-6, 0.5)
    assert e.value.code == -2
    c.upload(Q, PR)
    with pytest.raises(gpu.ChapsimError) as e:
        c.advance(1, 1e-3, 1e-6, 1e-9)  # CFLGV so small that DT/DT0 < 0.01
    assert e.value.code == -3
    c.upload(Q, PR)
    c.set_dt(1e-3)
    c.advance(1, 1e-3, 1e-6, 0.5)  # the context is usable after both
    c.close()
