"""Main-domain statistics on the device (PP_MEAN_ZX_FLOW_Xperiodic_io,
src/processing/PP_MEAN_ZX.f90:311-796) against the oracle's restatement.

A set is per_row * M doubles: 141 flow sums per row, 360 with the thermal
solver (the module arrays in the order the reference zeroes them).  Each
array is compared relative to its own largest magnitude: 1e-11 on identical
fields (the device sums in a tree order, the oracle in the I, K loop), and
after three steps of both solvers (fields within 1e-10 of each other) for the
arrays that do not involve the pressure, whose mean the two Poisson solves
may pin differently.
"""
import math

import numpy as np
import pytest

import oracle as orc
from oracle import Oracle
from chapsim import gpu, thermo
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu

# (name, width) of the arrays of one set, in storage order
FLOW = [("U1", 3), ("P1", 1), ("G1", 3), ("UP", 3), ("U2", 6), ("UG", 6), ("U3", 10), ("UGU", 10), ("DVDL1", 9),
        ("DVDLP", 9), ("DVDL2", 81)]
THERMAL = [("T1", 1), ("D1", 1), ("H1", 1), ("M1", 1), ("T2", 1), ("D2", 1), ("H2", 1), ("DH", 1), ("PH", 1),
           ("DVDL1M", 9), ("DVDL1MH", 9), ("DVDL1MU", 27), ("DVDL2M", 81), ("UH", 3), ("GH", 3), ("U2DH", 6),
           ("DhDL1", 3), ("DhDLP", 3), ("DTDLK", 3), ("DTDLKU", 9), ("DTDLKDVDL", 27), ("DHDLMDVDL", 27)]
WITH_P = {"P1", "UP", "DVDLP", "PH", "DhDLP"}


def _split(flat, M, arrays):
    out, off = {}, 0
    for name, w in arrays:
        out[name] = flat[off * M:(off + w) * M].reshape(w, M)
        off += w
    assert off * M == flat.size
    return out


def _compare(got, ref, M, arrays, tol, skip=()):
    g, r = _split(got, M, arrays), _split(ref, M, arrays)
    worst = {}
    for name, _ in arrays:
        if name in skip:
            continue
        scale = max(float(np.abs(r[name]).max()), 1e-300)
        worst[name] = float(np.abs(g[name] - r[name]).max()) / scale
    print({k: "%.1e" % v for k, v in worst.items()})
    for k, v in worst.items():
        assert v <= tol, (k, v)


def _flow_case(L=64, M=64, N=32):
    HX, HZ, STR2, REN = 2 * math.pi, math.pi, 2.0, 2800.0
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    G, PR = initial_field(s, 41, 0.2)  # the momentum rho u
    rng = np.random.default_rng(8)
    RHO = 1.0 + 0.1 * rng.uniform(-1.0, 1.0, (N, M + 2, L))  # u = G / rho differs from G
    MU = 1.0 + 0.1 * rng.uniform(-1.0, 1.0, (N, M + 2, L))
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=8)
    o.io_set_fields(G, PR, RHO, RHO, MU)
    o.set_dt(1e-3)
    c = gpu.ChannelIO(s)
    c.upload_io(G, PR, RHO, RHO, MU)
    c.set_dt(1e-3)
    return s, o, c


def _thermal_case(L=64, M=64, N=32, qw=0.5):
    HX, HZ, STR2, REN = 2 * math.pi, math.pi, 2.0, 2800.0
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / REN / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((N, M + 2, L))
    DH[:, 1:M + 1, :] = 1e-2 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L))
    ones = np.ones((N, M + 2, L))
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=8)
    o.io_set_fields(Q, PR, ones, ones, ones)
    o.thermal_enable(orc.PropTable(tab.lists), DH, qw, qw, cthecd)
    o.set_dt(1e-3)
    c = gpu.ChannelIO(s)
    c.upload_io(Q, PR, ones, ones, ones)
    c.thermal_init(tab, DH, qw, qw, cthecd)
    c.set_dt(1e-3)
    return s, o, c


def test_flow_means_match_oracle():
    s, o, c = _flow_case()
    got = c.PP_MEAN_ZX_FLOW_Xperiodic_io()
    ref = o.pp_mean_zx_io()
    assert got.size == ref.size == 141 * s.M
    _compare(got, ref, s.M, FLOW, 1e-11)
    c.close()
    o.close()


@pytest.mark.parametrize("steps", [0, 3])
def test_thermal_means_match_oracle(steps):
    s, o, c = _thermal_case()
    if steps:
        o.io_run_steps(steps)
        c.advance(steps, 1e-3, 1e-6, 0.5)
    got = c.PP_MEAN_ZX_FLOW_Xperiodic_io()
    ref = o.pp_mean_zx_io()
    assert got.size == ref.size == 360 * s.M
    tol, skip = (1e-11, ()) if steps == 0 else (1e-9, WITH_P)
    _compare(got, ref, s.M, FLOW + THERMAL, tol, skip)
    c.close()
    o.close()


def test_means_need_a_main_domain_context():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    c = gpu.ChannelTG(s)
    with pytest.raises(gpu.ChapsimError):
        c._check(c.lib.chapsim_pp_mean_zx_io(c.h))
    c.close()
