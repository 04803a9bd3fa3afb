"""Thermal IO step on the GPU (SOLVERRK3_ENG_io with table-search properties,
DENSITY_TIME_DERIVATION, DENSITY_Staggered / MU_Staggered, then
SOLVERRK3_MOM_io) against the CPU oracle.

Heated channel with a constant heat flux on both walls and the seeded
2048-row synthetic table; the flow starts from the seeded perturbed
Poiseuille field.  Tolerance: every flow and thermal field within 1e-10
relative (max-norm) of the oracle after 5 steps.  The table search itself is
bitwise (see test_gpu_thermo.py); the remaining differences are the
round-off of the FP64 stencils and the Poisson solve.
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

TOL = 1e-10


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _case(L=64, M=64, N=32, qw=0.5):
    HX, HZ, STR2, REN = 2 * math.pi, math.pi, 2.0, 2800.0
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    prt0 = tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"]
    cthecd = 1.0 / REN / prt0
    rng = np.random.default_rng(5)
    DH = np.zeros((N, M + 2, L))
    DH[:, 1:M + 1, :] = 1e-3 * rng.uniform(-1.0, 1.0, (N, M, L))
    ones = np.ones((N, M + 2, L))
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=8)
    o.io_set_fields(Q, PR, ones, ones, ones)
    ot = orc.PropTable(tab.lists)
    o.thermal_enable(ot, DH, qw, qw, cthecd)
    o.set_dt(1e-3)
    c = gpu.ChannelIO(s)
    c.upload_io(Q, PR, ones, ones, ones)
    c.thermal_init(tab, DH, qw, qw, cthecd)
    c.set_dt(1e-3)
    return s, o, ot, c


def _compare(s, o, c, tol):
    M = s.M
    Gg, Qg, Pg = c.download_io()
    Go, Qo, Po = o.io_get_fields()
    errs = {}
    for i, n in enumerate("uvw"):
        errs["G" + n] = rel(Gg[i][:, 1:M + 1], Go[i][:, 1:M + 1])
        errs["Q" + n] = rel(Qg[i][:, 1:M + 1], Qo[i][:, 1:M + 1])
    pg = Pg[:, 1:M + 1] - Pg[:, 1:M + 1].mean()
    po = Po[:, 1:M + 1] - Po[:, 1:M + 1].mean()
    errs["P"] = rel(pg, po)
    tg = c.download_thermal()
    to = o.thermal_get()
    for k in ("DH", "H", "T", "D", "M", "K", "CP"):
        errs[k] = rel(tg[k], to[k])
    print(errs)
    for k, e in errs.items():
        assert e <= tol, (k, e)
    return tg


def test_thermal_start_matches_oracle():
    s, o, ot, c = _case()
    tg = _compare(s, o, c, 1e-14)
    # start-up properties are the table's at the given rho*h (bitwise)
    res, nbad, _ = ot.update(tg["DH"][:, 1:s.M + 1])
    assert nbad == 0
    assert np.array_equal(res["T"], tg["T"][:, 1:s.M + 1])
    c.close()


def test_thermal_five_steps_match_oracle():
    s, o, ot, c = _case()
    rc, cdt = o.io_run_steps(5)
    assert rc == 0
    c.advance(5, 1e-3, 1e-6, 0.5)
    tg = _compare(s, o, c, TOL)
    # the walls heat up: rho*h rises next to both walls
    M = s.M
    dh = tg["DH"][:, 1:M + 1].mean(axis=(0, 2))
    assert dh[0] > dh[M // 2] and dh[-1] > dh[M // 2]
    c.close()


def test_thermal_substeps_match_oracle_per_call():
    s, o, ot, c = _case(L=32, M=32, N=32)
    o.io_cfl()
    for ns in (1, 2, 3):
        assert o.thermal_substep(ns) == 0
        o.io_substep(ns)
        c.SOLVERRK3_MOM_io(ns)
    _compare(s, o, c, TOL)
    c.close()


def _wall_state(ot, dh):
    r, nbad, _ = ot.update(np.array([dh]))
    assert nbad == 0
    return [float(r[k][0]) for k in ("T", "H", "D", "M", "K")]


def test_isothermal_walls_match_oracle():
    """BC_Fixed_Temperature on both walls (iThermalWallType = 2, 2 as TC4 and TC6 set them):
    the wall state from the table at a hotter bottom and a cooler top rho*h, held in the
    ghost rows; the wall face of the energy equation keeps its conduction term.  Five
    steps against the oracle at the same tolerance; the wall rows hold the state exactly,
    and the fluid next to the hot wall heats up."""
    s, o, ot, c = _case()
    hot, cold = _wall_state(ot, 2e-3), _wall_state(ot, -2e-3)
    for w, st in ((0, hot), (1, cold)):
        o.thermal_set_isothermal(w, st)
        c.thermal_set_isothermal(w, st)
    t0 = _compare(s, o, c, 1e-14)["T"][:, 1:s.M + 1].mean(axis=(0, 2))
    rc, _ = o.io_run_steps(5)
    assert rc == 0
    c.advance(5, 1e-3, 1e-6, 0.5)
    tg = _compare(s, o, c, TOL)
    M = s.M
    assert np.all(tg["T"][:, 0] == hot[0]) and np.all(tg["T"][:, M + 1] == cold[0])
    dt_rows = tg["T"][:, 1:M + 1].mean(axis=(0, 2)) - t0
    assert dt_rows[0] > 0 > dt_rows[-1]  # the first rows warm at the hot wall and cool at the cold one
    # back to the constant heat flux on the top wall
    o.thermal_set_isothermal(1, None)
    c.thermal_set_isothermal(1, None)
    o.io_run_steps(2)
    c.advance(2, 1e-3, 1e-6, 0.5)
    _compare(s, o, c, TOL)
    c.close()
