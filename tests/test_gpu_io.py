"""Main-domain (IO) path with explicit viscous terms on the GPU, through the
C ABI, against the oracle and against the reference's own TC8 monitor log."""
import json
import math
import os

import numpy as np
import pytest

from oracle import Oracle
from chapsim import gpu
from chapsim.mesh import channel_setup

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-11


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def monitor(G, Q, RHO, M):
    """Uc, u'u'_c, u'v'_c, Gmaxx of PP_MONITOR_Xperiodic_io from x-z means at cell centres."""
    g1 = 0.5 * (G[0] + np.roll(G[0], -1, axis=2))[:, 1:M + 1, :]
    u1 = 0.5 * (Q[0] + np.roll(Q[0], -1, axis=2))[:, 1:M + 1, :]
    g2 = 0.5 * (G[1][:, 1:M + 1, :] + G[1][:, 2:M + 2, :])
    G1 = g1.mean(axis=(0, 2))
    G2 = g2.mean(axis=(0, 2))
    UG1 = (u1 * g1).mean(axis=(0, 2))
    UG2 = (u1 * g2).mean(axis=(0, 2))
    D1 = RHO[:, 1:M + 1, :].mean(axis=(0, 2))
    j = M // 2 - 1
    return {"Uc": G1[j] / D1[j], "UUc": UG1[j] - G1[j] ** 2 / D1[j], "UVc": UG2[j] - G1[j] * G2[j] / D1[j],
            "Gmaxx": np.abs(G1).max()}


@pytest.fixture(scope="module")
def tc8(golden_dir):
    d = np.load(os.path.join(golden_dir, "tc8_step100_fields.npz"))
    c = json.load(open(os.path.join(golden_dir, "tc8_setup.json")))["case"]
    mon = json.load(open(os.path.join(golden_dir, "tc8_monitor.json")))
    L, M, N = c["NCL1"], c["NCL2"], c["NCL3"]
    G = np.zeros((3, N, M + 2, L))
    PR = np.zeros((N, M + 2, L))
    for comp, name in enumerate(("G1", "G2", "G3")):
        G[comp, :, 1:M + 1, :] = d[name].astype(np.float64)
    PR[:, 1:M + 1, :] = d["P"].astype(np.float64)
    rho = np.full((N, M + 2, L), float(d["D"]))
    return c, mon, G, PR, rho, np.ones_like(rho), np.full_like(rho, float(d["M"]))


def _io_pair(c, G, PR, rho, mu0, mu, threads=8):
    L, M, N = c["NCL1"], c["NCL2"], c["NCL3"]
    o = Oracle(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"], iFlowDriven=c["iFlowDriven"], Cf_Given=c["Cf_Given"],
               DT0=c["DT"], DTMIN=1e-6, CFLGV=c["CFLGV"], threads=threads)
    o.io_set_fields(G, PR, rho, mu0, mu)
    s = channel_setup(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"], c["iFlowDriven"], c["Cf_Given"])
    ch = gpu.ChannelIO(s)
    ch.upload_io(G, PR, rho, mu0, mu)
    ch.set_dt(c["DT"])
    return o, ch


def test_io_tc8_reproduces_reference_monitor_on_gpu(tc8):
    """The GPU IO step restarted from the reference's step-100 fields reproduces
    the reference's monitor rows 101-119 to every printed digit, and matches
    the oracle field by field."""
    c, mon, G, PR, rho, mu0, mu = tc8
    cols = mon["columns"]
    rows = {int(r[0]): r for r in mon["rows"]}
    o, ch = _io_pair(c, G, PR, rho, mu0, mu)
    M = c["NCL2"]
    for step in range(101, 120):
        o.io_run_steps(1)
        dt, cfl = ch.advance(1, c["DT"], 1e-6, c["CFLGV"])
        Gg, Qg, Pg = ch.download_io()
        m = monitor(Gg, Qg, rho, M)
        r = rows[step]
        assert abs(cfl * dt - r[cols.index("CFL")]) <= 0.5e-5 * 1.0001
        for name in ("Uc", "UUc", "UVc"):
            ref = r[cols.index(name)]
            assert abs(m[name] - ref) <= 0.5 * 10.0 ** (math.floor(math.log10(abs(ref))) - 5) * 1.0001, (step, name)
        assert abs(m["Gmaxx"] - r[cols.index("Gmaxx")]) <= 0.5e-5 * 1.0001
        # DIVGCK_io: round-off, within twice the reference's logged MaxDiv of the row
        assert ch.DIVGCK_io() <= 2.0 * r[cols.index("MaxDiv")], (step, ch.DIVGCK_io())
    Go, Qo, Po = o.io_get_fields()
    for comp in range(3):
        assert rel(Gg[comp], Go[comp]) <= TOL_STEP
        assert rel(Qg[comp], Qo[comp]) <= TOL_STEP
    assert rel(Pg[:, 1:M + 1], Po[:, 1:M + 1]) <= TOL_STEP


def test_io_variable_properties_against_oracle(tc8):
    """Non-uniform DENSITY0 / Viscousity0 exercise the staggered-property and
    variable-viscosity terms; 5 steps from the TC8 fields."""
    c, mon, G, PR, rho, mu0, mu = tc8
    N, M2, L = rho.shape
    k, j, i = np.meshgrid(np.arange(N), np.arange(M2), np.arange(L), indexing="ij")
    rho_v = 1.0 + 0.05 * np.sin(2 * np.pi * i / L) * np.cos(2 * np.pi * k / N) + 0.02 * np.cos(np.pi * j / M2)
    mu_v = 1.0 + 0.1 * np.cos(2 * np.pi * i / L + 0.3) * np.sin(np.pi * j / M2)
    o, ch = _io_pair(c, G, PR, rho_v, mu_v, mu_v)
    o.io_run_steps(5)
    ch.advance(5, c["DT"], 1e-6, c["CFLGV"])
    Gg, Qg, Pg = ch.download_io()
    Go, Qo, Po = o.io_get_fields()
    Mc = c["NCL2"]
    for comp in range(3):
        assert rel(Gg[comp], Go[comp]) <= TOL_STEP
        assert rel(Qg[comp], Qo[comp]) <= TOL_STEP
    assert rel(Pg[:, 1:Mc + 1], Po[:, 1:Mc + 1]) <= TOL_STEP


def test_io_larger_grid_substeps():
    """128 x 96 x 64 main domain from a seeded field, substep by substep."""
    from chapsim.fields import initial_field
    L, M, N = 128, 96, 64
    c = {"NCL1": L, "NCL2": M, "NCL3": N, "HX": 4 * math.pi, "HZ": 4 * math.pi / 3, "STR2": 2.0, "REN": 2800.0,
         "iFlowDriven": 1, "Cf_Given": 8.18e-3, "DT": 1e-3, "CFLGV": 0.5}
    s = channel_setup(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"])
    Q, PR = initial_field(s, 21, 0.1)
    rho = np.ones((N, M + 2, L))
    o, ch = _io_pair(c, Q, PR, rho, rho, rho)
    for ns in (1, 2, 3):
        o.set_dt(1e-3)
        o.io_substep(ns)
        ch.SOLVERRK3_MOM_io(ns)
    Gg, Qg, Pg = ch.download_io()
    Go, Qo, Po = o.io_get_fields()
    for comp in range(3):
        assert rel(Gg[comp], Go[comp]) <= TOL_STEP
    assert rel(Pg[:, 1:M + 1], Po[:, 1:M + 1]) <= TOL_STEP


def test_io_context_rejects_tg_calls():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    ch = gpu.ChannelIO(s)
    with pytest.raises(gpu.ChapsimError):
        ch.SOLVERRK3_MOM_tg(1)
