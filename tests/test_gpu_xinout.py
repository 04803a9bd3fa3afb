"""Main domain with inflow and outflow (iDomain = 3) on the GPU, through the C
ABI, against the oracle's restatement (tests/test_oracle_xinout.py pins that
restatement on the CPU).

A periodic TG context and the inflow/outflow main domain start from the same
fields as the oracle pair and step together (chapsim_advance_xinout): CFL of
both domains, one DT, TG substep then main-domain substep.  Compared after each
step: G, Q and PR of the main domain with their ghost columns, DT, U_OUTLET and
the outflow scaling, and the three divergence ranges of DIVGCK_io.  There is no
singular Poisson mode in this domain, so PR is compared as is.  Bounds: 1e-10
relative to each array's largest entry (the TG fields that feed the inlet agree
with the oracle's to about 1e-13 per step; the transforms and reductions sum in
other orders).
"""
import math

import numpy as np
import pytest

import oracle as orc
from oracle import Oracle, OracleXinout
from chapsim import gpu
from chapsim.mesh import channel_setup, xinout_setup
from chapsim.fields import initial_field, xinout_fields_from_tg

pytestmark = pytest.mark.gpu

HZ, STR2, REN = math.pi, 2.0, 2800.0
TOL = 1e-10


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _pair(LT, L, M, N, seed=41, dt0=1e-3, cflgv=0.5):
    DX = 2 * math.pi / 64
    st = channel_setup(LT, M, N, LT * DX, HZ, STR2, REN)
    Q, PR = initial_field(st, seed, 0.2)
    # oracle pair
    otg = Oracle(LT, M, N, LT * DX, HZ, STR2, REN, DT0=dt0, DTMIN=1e-6, CFLGV=cflgv, threads=8)
    otg.set_fields(Q, PR)
    otg.substep(0)
    Qt, PRt, _ = otg.get_fields()
    oio = OracleXinout(L, M, N, L * DX, HZ, STR2, REN, DT0=dt0, DTMIN=1e-6, CFLGV=cflgv, threads=8)
    G, P = xinout_fields_from_tg(Qt, L)
    ones = np.ones(oio.field_shape())
    oio.io_set_fields(G, P, ones, ones, ones)
    oio.set_dt(dt0)
    # device pair: the TG context restarts from the oracle's projected field
    tg = gpu.ChannelTG(st)
    tg.upload(Qt, PRt)
    tg.set_dt(dt0)
    io = gpu.ChannelXinout(xinout_setup(L, M, N, L * DX, HZ, STR2, REN), tg=tg)
    io.upload_io(G, P, ones, ones, ones)
    io.set_dt(dt0)
    return otg, oio, tg, io


def _compare(oio, io, M, L):
    Go, Qo, Po = oio.io_get_fields()
    Gg, Qg, Pg = io.download_io()
    out = {"G": rel(Gg[:, :, 1:M + 1], Go[:, :, 1:M + 1]), "Q": rel(Qg[:, :, 1:M + 1], Qo[:, :, 1:M + 1]),
           "P": rel(Pg[:, 1:M + 1, 1:L + 1], Po[:, 1:M + 1, 1:L + 1])}
    return out


@pytest.mark.parametrize("LT,L,M,N", [(32, 64, 32, 32), (64, 96, 64, 64), (32, 56, 64, 64)])
def test_coupled_steps_match_oracle(LT, L, M, N):
    otg, oio, tg, io = _pair(LT, L, M, N)
    for step in range(4):
        rc, cfl_dt = oio.xio_run_steps(otg, 1)
        assert rc == 0
        dt, cfl = io.advance(1, 1e-3, 1e-6, 0.5)
        assert abs(dt - oio.dt()) <= 1e-13 * oio.dt() and abs(tg.get_dt() - dt) == 0.0
        assert abs(cfl * dt - cfl_dt[0]) <= 1e-12 * cfl_dt[0]
        d = _compare(oio, io, M, L)
        uo, so = oio.xio_outlet_state()
        ug, sg = io.outlet_state()
        print(step, d, "U_OUTLET", ug, uo, "scaling", sg, so)
        assert max(d.values()) <= TOL, d
        assert abs(ug - uo) <= 1e-11 * abs(uo) and abs(sg - so) <= 1e-13
    dv_o, dv_g = oio.xio_divgck(), io.DIVGCK_io()
    print("divergence ranges", dv_g, dv_o)
    assert dv_g[0] < 1e-11 and dv_g[2] < 1e-11
    assert abs(dv_g[1] - dv_o[1]) <= 1e-8 * dv_o[1] + 1e-12
    # the TG context advanced with the common DT: its fields still match the oracle's
    Qtg, _ = tg.download()
    Qto, _, _ = otg.get_fields()
    assert rel(Qtg, Qto) <= TOL
    for h in (io, tg, oio, otg):
        h.close()


def test_substep_api_matches_coupled_advance():
    """chapsim_rk_substep_io on the inflow/outflow context after the TG context's own
    substep gives the fields of chapsim_advance_xinout with the same DT (bitwise)."""
    _, _, tg1, io1 = _pair(32, 64, 32, 32)
    _, _, tg2, io2 = _pair(32, 64, 32, 32)
    io1.advance(1, 1e-3, 1e-6, 0.5)
    dt = io1.get_dt()
    tg2.set_dt(dt)
    io2.set_dt(dt)
    for ns in (1, 2, 3):
        tg2.SOLVERRK3_MOM_tg(ns)
        io2.SOLVERRK3_MOM_io(ns)
    a, b = io1.download_io(), io2.download_io()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    for h in (io1, tg1, io2, tg2):
        h.close()


def test_inflow_outflow_contract_errors():
    s = xinout_setup(64, 32, 32, 2.0, HZ, STR2, REN)
    io = gpu.ChannelXinout(s)
    with pytest.raises(gpu.ChapsimError):
        io.advance(1, 1e-3, 1e-6, 0.5)  # no TG context attached
    other = gpu.ChannelTG(channel_setup(32, 64, 32, 1.0, HZ, STR2, REN))
    with pytest.raises(gpu.ChapsimError):
        io.attach(other)  # NCL2 differs
    mixed = gpu.ChannelTG(channel_setup(32, 32, 32, 1.0, HZ, STR2, REN), precision="mixed")
    with pytest.raises(gpu.ChapsimError):
        io.attach(mixed)  # the inlet is fed by an FP64 TG context
    with pytest.raises(gpu.ChapsimError):
        io._check(io.lib.chapsim_advance_tg(io.h, 1, 1e-3, 1e-6, 0.5, None, None))
    with pytest.raises(gpu.ChapsimError):
        gpu.ChannelXinout(s, precision="mixed")
    for h in (io, other, mixed):
        h.close()


def test_thermal_inflow_outflow_matches_oracle():
    """The same coupled case with the thermal solver on the main domain (TC7's setting: constant
    wall heat flux, explicit viscous terms): BC_TINLET_THERML, BC_COUTLET_ENEG_RK3, DrhoDtP in
    DIVG_io and in the outflow scaling.  Flow and thermal fields with their ghost columns within
    1e-10 after three steps, and U_OUTLET and the scaling to round-off."""
    from chapsim import thermo
    LT, L, M, N, qw = 32, 64, 32, 32, 0.5
    otg, oio, tg, io = _pair(LT, L, M, N)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / REN / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros(oio.field_shape())
    DH[:, 1:M + 1, :] = 1e-3 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L + 2))
    ot = orc.PropTable(tab.lists)
    oio.thermal_enable(ot, DH, qw, qw, cthecd)
    io.thermal_init(tab, DH, qw, qw, cthecd)
    r, nbad, _ = ot.update(np.array([0.0]))
    st = [float(r[k][0]) for k in ("T", "H", "D", "M", "K", "CP")]
    inlet = st + [st[2] * st[1]]
    oio.xio_thermal_inlet(inlet)
    io.thermal_inlet(inlet)
    for step in range(3):
        rc, cfl_dt = oio.xio_run_steps(otg, 1)
        assert rc == 0
        dt, cfl = io.advance(1, 1e-3, 1e-6, 0.5)
        assert abs(dt - oio.dt()) <= 1e-13 * oio.dt()
        d = _compare(oio, io, M, L)
        to, tg_ = oio.thermal_get(), io.download_thermal()
        for k in ("DH", "T", "D", "M", "K"):
            d[k] = rel(tg_[k][:, 1:M + 1], to[k][:, 1:M + 1])
        uo, so = oio.xio_outlet_state()
        ug, sg = io.outlet_state()
        print(step, d, "U_OUTLET", ug, uo, "scaling", sg, so)
        assert max(d.values()) <= TOL, d
        assert abs(ug - uo) <= 1e-11 * abs(uo) and abs(sg - so) <= 1e-12
    dv_o, dv_g = oio.xio_divgck(), io.DIVGCK_io()
    print("divergence ranges", dv_g, dv_o)
    assert dv_g[0] < 1e-11 and dv_g[2] < 1e-11
    for h in (io, tg, oio, otg):
        h.close()
