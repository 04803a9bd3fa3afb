"""On-device statistics of the periodic channel (PP_MEAN_ZX_FLOW_TG,
PP_MEAN_T_TG, PP_MONITOR_TG) through the C ABI against the oracle.

Both advance the same seeded channel and take the statistics after every
step.  The fields agree to ~1e-13 after 10 steps; the plane sums are added
in a different order (tree vs the reference's I, K loop).  Bound: each array
within 1e-11 of the oracle, relative to the array's largest entry, for the
instantaneous and the time-averaged means and the monitor quantities.
"""
import math

import numpy as np
import pytest

from oracle import Oracle
from chapsim import gpu
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _pair(L, M, N, precision="fp64"):
    HX, HZ, STR2, REN = 2 * math.pi, math.pi, 2.0, 2800.0
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 1973, 0.1)
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=0.02, DTMIN=1e-6, CFLGV=0.5, threads=8)
    o.set_fields(Q, PR)
    o.substep(0)
    c = gpu.ChannelTG(s, precision=precision)
    c.upload(Q, PR)
    c.set_dt(0.02)
    c.SOLVERRK3_MOM_tg(0)
    return s, o, c


def _cmp(a, b, M, tol):
    ga, gb = gpu.ChannelTG.pp_split(a, M), gpu.ChannelTG.pp_split(b, M)
    worst = 0.0
    for name in ga:
        scale = max(np.abs(gb[name]).max(), 1e-300)
        e = np.abs(ga[name] - gb[name]).max() / scale
        worst = max(worst, e)
        assert e <= tol, (name, e)
    return worst


@pytest.mark.parametrize("shape", [(64, 64, 64), (96, 128, 64)])
def test_statistics_match_oracle(shape):
    L, M, N = shape
    s, o, c = _pair(L, M, N)
    avg_o, n_o = np.zeros(122 * M), 0
    for step in range(10):
        o.run_steps(1)
        c.advance(1, 0.02, 1e-6, 0.5)
        inst_o = o.pp_mean_zx_tg()
        n_o = o.pp_mean_t_tg(1, inst_o, avg_o, n_o)
        c.PP_MEAN_ZX_FLOW_TG()
        c.PP_MEAN_T_TG(1)
    inst_g, n_g = c.download_pp_means(False)
    avg_g, n_g2 = c.download_pp_means(True)
    assert n_g == n_g2 == n_o == 10
    print("instantaneous", _cmp(inst_g, inst_o, M, TOL), "averaged", _cmp(avg_g, avg_o, M, TOL))
    mon_o = o.pp_monitor_tg(inst_o, avg_o, 2800.0)
    mon_g = c.PP_MONITOR_TG(2800.0)
    for k, (name, v) in enumerate(mon_g.items()):
        assert abs(v - mon_o[k]) <= TOL * max(abs(mon_o[k]), 1e-3), (name, v, mon_o[k])
    c.close()
    o.close()


def test_statistics_restart_and_summing_average():
    L = M = N = 64
    s, o, c = _pair(L, M, N)
    c.advance(2, 0.02, 1e-6, 0.5)
    c.PP_MEAN_ZX_FLOW_TG()
    c.PP_MEAN_T_TG(1)
    c.PP_MEAN_T_TG(1)
    avg, n = c.download_pp_means(True)
    inst, _ = c.download_pp_means(False)
    assert n == 2 and np.abs(avg - inst).max() <= 1e-15 * np.abs(inst).max()  # the mean of two equal sets
    # restart: upload the averages into a fresh context, then a summing average adds inst/4
    c2 = gpu.ChannelTG(s)
    flat = np.ascontiguousarray(avg)
    ptrs, off = [], 0
    for _, w in gpu.PP_ARRAYS:
        ptrs.append(gpu._ptr(flat[off * M:(off + w) * M]))
        off += w
    c2._check(c2.lib.chapsim_upload_pp_means_tg(c2.h, 7, *ptrs))
    Qg, Pg = c.download()
    c2.upload(Qg, Pg)
    c2.PP_MEAN_ZX_FLOW_TG()
    c2.PP_MEAN_T_TG(2, pp_instn_sz=4)
    got, n2 = c2.download_pp_means(True)
    assert n2 == 8
    assert np.abs(got - (avg + 0.25 * inst)).max() <= 1e-14 * np.abs(avg).max()
    c.close()
    c2.close()


def test_statistics_mixed_precision_within_bound():
    """Mixed precision: the statistics of the FP32 fields stay within 1e-5 of the FP64 oracle's."""
    L = M = N = 64
    s, o, c = _pair(L, M, N, precision="mixed")
    o.run_steps(5)
    c.advance(5, 0.02, 1e-6, 0.5)
    c.PP_MEAN_ZX_FLOW_TG()
    inst_g, _ = c.download_pp_means(False)
    inst_o = o.pp_mean_zx_tg()
    ga, gb = gpu.ChannelTG.pp_split(inst_g, M), gpu.ChannelTG.pp_split(inst_o, M)
    for name in ("U1xzL", "U2xzL"):
        e = np.abs(ga[name] - gb[name]).max() / np.abs(gb[name]).max()
        assert e <= 1e-5, (name, e)
    c.close()


def test_statistics_rejected_on_main_domain():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    c = gpu.ChannelIO(s)
    with pytest.raises(gpu.ChapsimError):
        c.PP_MEAN_ZX_FLOW_TG()
    c.close()
