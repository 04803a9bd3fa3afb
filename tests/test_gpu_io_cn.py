"""Main-domain (IO) path with the Crank-Nicolson viscous scheme (iVisScheme = 1)
on the GPU, through the C ABI, against the oracle.

The right-hand side is VISCOUS_PAR_EXPLT_X/Y/Z_io + RHS_MOM_EXPLICIT_io's
VisImplicit branch; MOMFA_io's x, z and y sweeps use per-point coefficients
from Viscousity, MU_STG and D_STG; PRCALC_io subtracts BE * RHSLLPHI.  The
GPU solves each line with the warp Thomas/PCR hybrid, the oracle with the
reference's sequential recurrences, so agreement is to round-off: every
field within 1e-11 relative (max-norm) of the oracle after 5 steps
(thermal case 1e-10, as the explicit-scheme thermal test).
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

TOL = 1e-11


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
    return c, G, PR


def _variable_props(N, M2, L):
    k, j, i = np.meshgrid(np.arange(N), np.arange(M2), np.arange(L), indexing="ij")
    rho = 1.0 + 0.05 * np.sin(2 * np.pi * i / L) * np.cos(2 * np.pi * k / N) + 0.02 * np.cos(np.pi * j / M2)
    mu0 = 1.0 + 0.1 * np.cos(2 * np.pi * i / L + 0.3) * np.sin(np.pi * j / M2)
    mu = mu0 * (1.0 + 0.03 * np.sin(2 * np.pi * k / N + 0.7))
    return rho, mu0, mu


def _pair(c, G, PR, rho, mu0, mu, ivis=1):
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


def _check(o, ch, M, tol=TOL):
    Gg, Qg, Pg = ch.download_io()
    Go, Qo, Po = o.io_get_fields()
    errs = {}
    for comp, n in enumerate("uvw"):
        errs["G" + n] = rel(Gg[comp], Go[comp])
        errs["Q" + n] = rel(Qg[comp], Qo[comp])
    errs["P"] = rel(Pg[:, 1:M + 1], Po[:, 1:M + 1])
    print(errs)
    for k, e in errs.items():
        assert e <= tol, (k, e)
    return Gg


def test_cn_tc8_variable_properties(golden_dir):
    """5 steps from the reference's TC8 step-100 fields with non-uniform
    DENSITY0, Viscousity0 and a different Viscousity: exercises every
    per-point coefficient of the three sweeps and the wall rows."""
    c, G, PR = _tc8(golden_dir)
    N, M2, L = PR.shape
    rho, mu0, mu = _variable_props(N, M2, L)
    o, ch = _pair(c, G, PR, rho, mu0, mu)
    o.io_run_steps(5)
    ch.advance(5, c["DT"], 1e-6, c["CFLGV"])
    Gg = _check(o, ch, c["NCL2"])
    assert np.all(Gg[1][:, 1, :] == 0.0)  # v at the wall face stays zero


def test_cn_differs_from_explicit(golden_dir):
    """The scheme switch is live: after 5 steps the two schemes differ by far
    more than round-off, and by less than the truncation error."""
    c, G, PR = _tc8(golden_dir)
    N, M2, L = PR.shape
    rho, mu0, mu = _variable_props(N, M2, L)
    _, a = _pair(c, G, PR, rho, mu0, mu, ivis=1)
    _, b = _pair(c, G, PR, rho, mu0, mu, ivis=0)
    a.advance(5, c["DT"], 1e-6, c["CFLGV"])
    b.advance(5, c["DT"], 1e-6, c["CFLGV"])
    ga, _, _ = a.download_io()
    gb, _, _ = b.download_io()
    d = rel(ga, gb)
    print("CN vs explicit", d)
    assert 1e-9 < d < 1e-3


def test_cn_larger_grid_substeps():
    """192 x 128 x 96 (S = 6, 4, 3 in the three sweeps) from a seeded field, substep by substep."""
    L, M, N = 192, 128, 96
    c = {"NCL1": L, "NCL2": M, "NCL3": N, "HX": 4 * math.pi, "HZ": 4 * math.pi / 3, "STR2": 2.0, "REN": 2800.0,
         "iFlowDriven": 1, "Cf_Given": 8.18e-3, "DT": 1e-3, "CFLGV": 0.5}
    s = channel_setup(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"])
    Q, PR = initial_field(s, 21, 0.1)
    rho, mu0, mu = _variable_props(N, M + 2, L)
    o, ch = _pair(c, Q, PR, rho, mu0, mu)
    for ns in (1, 2, 3):
        o.set_dt(1e-3)
        o.io_substep(ns)
        ch.SOLVERRK3_MOM_io(ns)
    _check(o, ch, M)


def test_cn_constant_cf_forcing(golden_dir):
    """iFlowDriven = 2: the constant-Cf forcing enters the u right-hand side before the sweeps."""
    c, G, PR = _tc8(golden_dir)
    c = dict(c, iFlowDriven=2)
    N, M2, L = PR.shape
    rho, mu0, mu = _variable_props(N, M2, L)
    o, ch = _pair(c, G, PR, rho, mu0, mu)
    o.io_run_steps(3)
    ch.advance(3, c["DT"], 1e-6, c["CFLGV"])
    _check(o, ch, c["NCL2"])


def test_cn_heated_channel_matches_oracle():
    """Thermal solver on (table-search properties, wall heat flux) with the
    Crank-Nicolson momentum step: flow and thermal fields after 5 steps."""
    L, M, N, qw = 64, 64, 32, 0.5
    HX, HZ, STR2, REN = 2 * math.pi, math.pi, 2.0, 2800.0
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / REN / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((N, M + 2, L))
    DH[:, 1:M + 1, :] = 1e-3 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L))
    ones = np.ones((N, M + 2, L))
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=8)
    o.io_set_fields(Q, PR, ones, ones, ones)
    o.io_set_vis_scheme(1)
    ot = orc.PropTable(tab.lists)
    o.thermal_enable(ot, DH, qw, qw, cthecd)
    o.set_dt(1e-3)
    ch = gpu.ChannelIO(s, ivisscheme=1)
    ch.upload_io(Q, PR, ones, ones, ones)
    ch.thermal_init(tab, DH, qw, qw, cthecd)
    ch.set_dt(1e-3)
    rc, _ = o.io_run_steps(5)
    assert rc == 0
    ch.advance(5, 1e-3, 1e-6, 0.5)
    Gg, Qg, Pg = ch.download_io()
    Go, Qo, Po = o.io_get_fields()
    for comp in range(3):
        assert rel(Gg[comp][:, 1:M + 1], Go[comp][:, 1:M + 1]) <= 1e-10
    pg = Pg[:, 1:M + 1] - Pg[:, 1:M + 1].mean()
    po = Po[:, 1:M + 1] - Po[:, 1:M + 1].mean()
    assert rel(pg, po) <= 1e-10
    tg, to = ch.download_thermal(), o.thermal_get()
    for k in ("DH", "T", "D", "M"):
        assert rel(tg[k], to[k]) <= 1e-10, k
    # DIVGCK_io: the projection leaves div G + DrhoDtP at round-off, on both sides
    dg, do = ch.DIVGCK_io(), o.io_divgck()
    print("max |div G + drho/dt|", dg, do)
    assert dg <= 1e-11 and do <= 1e-11


def test_cn_option_rejected_outside_main_domain():
    """ivisscheme selects the main-domain scheme: the TG domain (always
    Crank-Nicolson, SOLVERRK3_MOM_tg) and unknown values are rejected."""
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    with pytest.raises(gpu.ChapsimError):
        gpu.ChannelTG(s, ivisscheme=1)
    with pytest.raises(gpu.ChapsimError):
        gpu.ChannelIO(s, ivisscheme=2)
    ok = gpu.ChannelIO(s, ivisscheme=1)
    ok.close()
