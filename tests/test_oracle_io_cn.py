"""CPU checks of the oracle's Crank-Nicolson main-domain step (iVisScheme = 1:
VISCOUS_PAR_EXPLT_*, RHS_MOM_EXPLICIT_io VisImplicit, MOMFA_io, PRCALC_io CN).

No test case shipped with the reference runs iVisScheme = 1 (every
readdata.ini sets iVisScheme = 0), so no reference output pins this scheme;
its shared parts (convection, pressure gradient, Poisson solve, correction)
are the ones the TC8 trajectory pins.  These checks pin what the scheme must
satisfy: consistency with the explicit scheme to truncation error, the
projection, the v wall face, and the identically-zero density correction.
"""
import json
import os

import numpy as np
import pytest

import oracle as orc
from oracle import Oracle
from chapsim import thermo
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field


def _tc8(golden_dir, ivis):
    d = np.load(os.path.join(golden_dir, "tc8_step100_fields.npz"))
    c = json.load(open(os.path.join(golden_dir, "tc8_setup.json")))["case"]
    L, M, N = c["NCL1"], c["NCL2"], c["NCL3"]
    G = np.zeros((3, N, M + 2, L))
    PR = np.zeros((N, M + 2, L))
    for comp, name in enumerate(("G1", "G2", "G3")):
        G[comp, :, 1:M + 1, :] = d[name].astype(np.float64)
    PR[:, 1:M + 1, :] = d["P"].astype(np.float64)
    k, j, i = np.meshgrid(np.arange(N), np.arange(M + 2), np.arange(L), indexing="ij")
    rho = 1.0 + 0.05 * np.sin(2 * np.pi * i / L) * np.cos(2 * np.pi * k / N) + 0.02 * np.cos(np.pi * j / (M + 2))
    mu = 1.0 + 0.1 * np.cos(2 * np.pi * i / L + 0.3) * np.sin(np.pi * j / (M + 2))
    o = Oracle(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"], iFlowDriven=c["iFlowDriven"], Cf_Given=c["Cf_Given"],
               DT0=c["DT"], DTMIN=1e-6, CFLGV=c["CFLGV"], threads=4)
    o.io_set_fields(G, PR, rho, mu, mu)
    o.io_set_vis_scheme(ivis)
    return o, c


def _div_g(o, c):
    """max |DIVG_io| of G (flow only: DrhoDt = 0) with the oracle's metrics"""
    G, _, _ = o.io_get_fields()
    s = channel_setup(c["NCL1"], c["NCL2"], c["NCL3"], c["HX"], c["HZ"], c["STR2"], c["REN"])
    M = c["NCL2"]
    dx = (np.roll(G[0], -1, axis=2) - G[0])[:, 1:M + 1] * s.DXI
    dy = (G[1][:, 2:M + 2] - G[1][:, 1:M + 1]) * s.DYFI[1:M + 1][None, :, None]
    dz = (np.roll(G[2], -1, axis=0) - G[2])[:, 1:M + 1] * s.DZI
    return float(np.abs(dx + dy + dz).max()), float(np.abs(G).max())


def test_cn_matches_explicit_to_truncation_error(golden_dir):
    a, c = _tc8(golden_dir, 1)
    b, _ = _tc8(golden_dir, 0)
    assert a.io_run_steps(5)[0] == 0 and b.io_run_steps(5)[0] == 0
    ga, _, _ = a.io_get_fields()
    gb, _, _ = b.io_get_fields()
    d = np.abs(ga - gb).max() / np.abs(gb).max()
    assert 1e-9 < d < 1e-4, d


def test_cn_projection_and_wall_face(golden_dir):
    o, c = _tc8(golden_dir, 1)
    assert o.io_run_steps(3)[0] == 0
    div, gmax = _div_g(o, c)
    assert div <= 1e-10 * gmax * c["NCL1"], div
    G, Q, _ = o.io_get_fields()
    assert np.all(G[1][:, 1, :] == 0.0) and np.all(Q[1][:, 1, :] == 0.0)


def test_cn_density_correction_is_identically_zero():
    """DENSITY_IMPLICIT_add right after DENSITY_Staggered gives DRHOI_STG = 0
    exactly, so the density-correction part of VISCOUS_PAR_EXPLT_* vanishes
    (the GPU does not compute it)."""
    import math
    L, M, N = 32, 32, 32
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 7, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / 2800.0 / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((N, M + 2, L))
    DH[:, 1:M + 1, :] = 1e-3 * np.random.default_rng(3).uniform(-1.0, 1.0, (N, M, L))
    ones = np.ones((N, M + 2, L))
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=4)
    o.io_set_fields(Q, PR, ones, ones, ones)
    o.io_set_vis_scheme(1)
    ot = orc.PropTable(tab.lists)
    o.thermal_enable(ot, DH, 2.0, 2.0, cthecd)
    o.set_dt(1e-3)
    assert o.io_run_steps(3)[0] == 0
    th = o.thermal_get()
    assert np.ptp(th["D"][:, 1:M + 1]) > 0.0  # the density really varies
    assert o.io_drhoi_maxabs() == 0.0
