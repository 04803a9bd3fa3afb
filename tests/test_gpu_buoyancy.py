"""Buoyancy (iGravity) and weighted pressure (iWeightedPre) of the main-domain
step on the GPU against the oracle (RHS_MOM_EXPLICIT_io,
src/RHS_MOM_EXPLICIT_io.f90:103-226; DIVG_io, src/DIVG.f90:78-82).

Starts from the reference's own TC8 step-100 fields with non-uniform
DENSITY0 / viscosities, so the buoyancy force D_STG * TALP*DT*F_A varies in
space; explicit and Crank-Nicolson schemes; 3 steps.  Tolerance: G, Q and P
within 1e-10 relative (max-norm), as for the other main-domain parity tests.
The heated case (thermal solver on, table-search properties) runs iGravity = 1
with the Crank-Nicolson scheme.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle as orc
from oracle import Oracle
from chapsim import gpu, thermo
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _tc8(golden_dir):
    d = np.load(os.path.join(golden_dir, "tc8_step100_fields.npz"))
    c = json.load(open(os.path.join(golden_dir, "tc8_setup.json")))["case"]
    L, M, N = c["NCL1"], c["NCL2"], c["NCL3"]
    G = np.zeros((3, N, M + 2, L))
    PR = np.zeros((N, M + 2, L))
    for comp, name in enumerate(("G1", "G2", "G3")):
        G[comp, :, 1:M + 1, :] = d[name].astype(np.float64)
    PR[:, 1:M + 1, :] = d["P"].astype(np.float64)
    k, j, i = np.meshgrid(np.arange(N), np.arange(M + 2), np.arange(L), indexing="ij")
    rho = 1.0 + 0.05 * np.sin(2 * np.pi * i / L) * np.cos(2 * np.pi * k / N) + 0.1 * np.cos(np.pi * j / (M + 2))
    mu0 = 1.0 + 0.1 * np.cos(2 * np.pi * i / L + 0.3) * np.sin(np.pi * j / (M + 2))
    return c, G, PR, rho, mu0, mu0 * 1.01


def _pair(c, G, PR, rho, mu0, mu, ivis):
    L, M, N = c["NCL1"], c["NCL2"], c["NCL3"]
    o = Oracle(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"], iFlowDriven=c["iFlowDriven"], Cf_Given=c["Cf_Given"],
               DT0=c["DT"], DTMIN=1e-6, CFLGV=c["CFLGV"], threads=8)
    o.io_set_fields(G, PR, rho, mu0, mu)
    o.io_set_vis_scheme(ivis)
    s = channel_setup(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"], c["iFlowDriven"], c["Cf_Given"])
    ch = gpu.ChannelIO(s, ivisscheme=ivis)
    ch.upload_io(G, PR, rho, mu0, mu)
    ch.set_dt(c["DT"])
    return o, ch


def _check(o, ch, M):
    Gg, Qg, Pg = ch.download_io()
    Go, Qo, Po = o.io_get_fields()
    errs = {}
    for comp, n in enumerate("uvw"):
        errs["G" + n] = rel(Gg[comp], Go[comp])
        errs["Q" + n] = rel(Qg[comp], Qo[comp])
    errs["P"] = rel(Pg[:, 1:M + 1], Po[:, 1:M + 1])
    print(errs)
    for k, e in errs.items():
        assert e <= TOL, (k, e, errs)


@pytest.mark.parametrize("ivis", [0, 1])
@pytest.mark.parametrize("igrav,fa", [(1, 0.8), (-1, -0.8), (-2, -0.5), (3, 0.3)])
def test_buoyancy_matches_oracle(golden_dir, ivis, igrav, fa):
    c, G, PR, rho, mu0, mu = _tc8(golden_dir)
    o, ch = _pair(c, G, PR, rho, mu0, mu, ivis)
    o.io_set_buoyancy(igrav, fa)
    ch.set_buoyancy(igrav, fa)
    assert o.io_run_steps(3)[0] == 0
    ch.advance(3, c["DT"], 1e-6, c["CFLGV"])
    _check(o, ch, c["NCL2"])


@pytest.mark.parametrize("ivis", [0, 1])
def test_weighted_pressure_matches_oracle(golden_dir, ivis):
    c, G, PR, rho, mu0, mu = _tc8(golden_dir)
    o, ch = _pair(c, G, PR, rho, mu0, mu, ivis)
    # the two layers differ here (the reference starts both at PR_io), so both are exercised
    pr0b = PR + 1e-3 * np.random.default_rng(2).standard_normal(PR.shape)
    o.io_set_weighted_pressure(PR, pr0b)
    ch.set_weighted_pressure(PR, pr0b)
    assert o.io_run_steps(3)[0] == 0
    ch.advance(3, c["DT"], 1e-6, c["CFLGV"])
    _check(o, ch, c["NCL2"])
    # turned off again, the step is the plain one on both sides
    o.io_set_weighted_pressure(None)
    ch.set_weighted_pressure(None)
    assert o.io_run_steps(1)[0] == 0
    ch.advance(1, c["DT"], 1e-6, c["CFLGV"])
    _check(o, ch, c["NCL2"])


def test_buoyancy_heated_channel_cn():
    L, M, N, qw = 64, 64, 32, 0.5
    HX, HZ, STR2, REN = 2 * math.pi, math.pi, 2.0, 2800.0
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / REN / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((N, M + 2, L))
    # a density spread of about 1 % (the wall-ghost extrapolation of rho*h must stay inside the table)
    DH[:, 1:M + 1, :] = 1e-2 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L))
    ones = np.ones((N, M + 2, L))
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=8)
    o.io_set_fields(Q, PR, ones, ones, ones)
    o.io_set_vis_scheme(1)
    o.thermal_enable(orc.PropTable(tab.lists), DH, qw, qw, cthecd)
    o.set_dt(1e-3)
    o.io_set_buoyancy(1, 1.5)
    ch = gpu.ChannelIO(s, ivisscheme=1)
    ch.upload_io(Q, PR, ones, ones, ones)
    ch.thermal_init(tab, DH, qw, qw, cthecd)
    ch.set_dt(1e-3)
    ch.set_buoyancy(1, 1.5)
    assert o.io_run_steps(3)[0] == 0
    ch.advance(3, 1e-3, 1e-6, 0.5)
    Gg, _, Pg = ch.download_io()
    Go, _, Po = o.io_get_fields()
    for comp in range(3):
        assert rel(Gg[comp][:, 1:M + 1], Go[comp][:, 1:M + 1]) <= TOL
    pg = Pg[:, 1:M + 1] - Pg[:, 1:M + 1].mean()
    po = Po[:, 1:M + 1] - Po[:, 1:M + 1].mean()
    assert rel(pg, po) <= TOL
    tg, to = ch.download_thermal(), o.thermal_get()
    for k in ("DH", "T", "D"):
        assert rel(tg[k], to[k]) <= TOL, k


def test_buoyancy_arguments():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    tg = gpu.ChannelTG(s)
    assert tg.lib.chapsim_set_buoyancy(tg.h, 1, 1.0) == -6  # the periodic (TG) domain has no buoyancy term
    io = gpu.ChannelIO(s)
    with pytest.raises(gpu.ChapsimError):
        io.set_buoyancy(4, 1.0)
    with pytest.raises(gpu.ChapsimError):
        io.set_buoyancy(1, float("nan"))
    io.set_buoyancy(0, 0.0)
