"""Pipelined host I/O of the periodic channel (chapsim_upload_fields_async,
chapsim_download_fields_async, chapsim_io_wait) against the blocking transfer
calls: a step taken from fields uploaded through the staging slots gives,
bitwise, the fields of the same step taken after chapsim_upload_fields, in
FP64 and in mixed precision; with three different inputs in flight (the H2D
copy of step s + 1's input issued before step s) every step's downloaded
result is that of its own input.
"""
import math

import numpy as np
import pytest

from chapsim import gpu
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu

L = M = N = 64
ARGS = (0.05, 1e-6, 0.5)  # DT0, DTMIN, CFLGV


def _inputs(n):
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    return s, [initial_field(s, 100 + i, 0.2) for i in range(n)]


def _blocking_step(s, Q, PR, precision):
    ch = gpu.ChannelTG(s, precision=precision)
    ch.upload(Q, PR)
    ch.set_dt(ARGS[0])
    ch.advance(1, *ARGS)
    out = ch.download()
    ch.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pipelined_steps_match_blocking_transfers(precision):
    s, ins = _inputs(3)
    want = [_blocking_step(s, Q, PR, precision) for Q, PR in ins]
    ch = gpu.ChannelTG(s, precision=precision)
    ch.upload(*ins[0])  # a first field set, replaced by the first staged upload
    ch.set_dt(ARGS[0])
    outs = [(np.empty_like(ins[0][0]), np.empty_like(ins[0][1])) for _ in ins]
    ch.upload_async(*ins[0])
    for k in range(len(ins)):
        if k + 1 < len(ins):
            ch.upload_async(*ins[k + 1])
        ch.set_dt(ARGS[0])
        ch.advance(1, *ARGS)
        ch.download_async(*outs[k])
    ch.io_wait()
    for k in range(len(ins)):
        for got, ref in zip(outs[k], want[k]):
            assert np.array_equal(got, ref), (precision, k)
    # a third upload with both slots full commits the older one at once
    ch.upload_async(*ins[1])
    ch.upload_async(*ins[2])
    ch.upload_async(*ins[0])
    ch.set_dt(ARGS[0])
    ch.advance(1, *ARGS)
    ch.io_wait()
    for got, ref in zip(ch.download(), want[2]):
        assert np.array_equal(got, ref), precision
    ch.close()


def test_pipelined_io_rejects_bad_arguments():
    s, ins = _inputs(1)
    ch = gpu.ChannelTG(s)
    with pytest.raises(ValueError):
        ch.upload_async(ins[0][0][:, :-1], ins[0][1])
    with pytest.raises(gpu.ChapsimError):
        ch._check(ch.lib.chapsim_upload_fields_async(ch.h, None, None))
    ch.close()
