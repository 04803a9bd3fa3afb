"""Programmatic dependent launch of the step's kernels changes only when a
kernel's launch begins, not what it computes: every step kernel waits for
its predecessor before it touches memory.  The fields after ten steps are
bitwise those of plain launches, in both precisions and with either form of
the pressure stage (chained or fused plane transforms)."""
import math

import numpy as np
import pytest

from chapsim import gpu
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,force", [("fp64", 5), ("fp64", 13), ("mixed", 13), ("fp64", 2)])
def test_pdl_step_is_bitwise_the_plain_step(precision, force):
    s = channel_setup(128, 64, 64, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 23, 0.1)
    out = []
    for pdl in (False, True):
        c = gpu.ChannelTG(s, precision=precision, pdl=pdl)
        choice, _ = c.autotune(force=force)
        assert choice == force
        c.upload(Q, PR)
        c.set_dt(1e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(10, 0.02, 1e-6, 0.5)
        out.append(c.download() + (c.get_dt(),))
        c.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
