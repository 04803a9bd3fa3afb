"""The oracle's main domain with inflow and outflow (iDomain = 3, TgFlowFlg),
checked on the CPU before it is trusted as the checker of the device path.

* FISHPACK_POIS3D_SIMPLE with BCX_io = (2, 1) (src/possion3d_fishpack.f90:
  48-137, 344-460): the solution satisfies FISHPACK's LPEROD = 4 discrete
  problem -- x(0) = x(2) at the inlet, x(L+1) = 0 at the outlet, periodic z,
  the AMPH/ACPH/APPH operator in y -- to round-off, and leaves the ghost
  columns at zero.
* The x roots restated by the host set-up (chapsim.mesh.xinout_setup) are the
  oracle's, bitwise.
* A coupled TG + main-domain run (src/SOLVE.f90:75-134): the inlet face u(1)
  is the TG domain's first u face (BC_TINLET_FLOW), the outflow scaling of
  CHK_MassConsv_io makes the outlet flux equal the inlet flux, and the
  projection leaves the cells 2..L-1 and L divergence-free to round-off.  The
  cell next to the inlet keeps a residual: FISHPACK's mirror condition
  x(0) = x(2) is not the one-sided condition of the fixed inlet face, and the
  reference has the same residual.
* With the thermal solver (BC_TINLET_THERML, BC_COUTLET_ENEG_RK3): the inlet
  column holds the inlet state, the heated walls raise the mean rho*h, and
  the cells 2..L stay divergence-free against DrhoDtP.
"""
import math

import numpy as np
import pytest

from oracle import Oracle, OracleXinout
from chapsim.mesh import channel_setup, xinout_setup
from chapsim.fields import initial_field, xinout_fields_from_tg

HZ, STR2, REN = math.pi, 2.0, 2800.0


def _operator_residual(o, rhs, ph):
    L, M, N = o.L, o.M, o.N
    s = o.scalars()
    A, B, C = o.y("AMPH")[:M], o.y("ACPH")[:M], o.y("APPH")[:M]
    p = ph[:, 1:M + 1, 1:L + 1]
    px = np.zeros((N, M, L + 2))
    px[:, :, 1:L + 1] = p
    px[:, :, 0] = p[:, :, 1]  # x(0) = x(2)
    lapx = (px[:, :, 2:] - 2 * px[:, :, 1:-1] + px[:, :, :-2]) * s["DXQI"]
    lapz = (np.roll(p, -1, 0) - 2 * p + np.roll(p, 1, 0)) * s["DZQI"]
    py = np.zeros((N, M + 2, L))
    py[:, 1:M + 1] = p
    lapy = A[None, :, None] * py[:, 0:M] + B[None, :, None] * py[:, 1:M + 1] + C[None, :, None] * py[:, 2:M + 2]
    scale = np.abs(rhs).max() * (1.0 + 4.0 * s["DXQI"] / np.abs(rhs).max())
    return np.abs(lapx + lapy + lapz - rhs[:, 1:M + 1, 1:L + 1]).max() / scale


@pytest.mark.parametrize("L,M,N", [(32, 32, 32), (48, 40, 24), (64, 32, 16)])
def test_cosine_poisson_solves_lperod4_problem(L, M, N):
    o = OracleXinout(L, M, N, L * 2 * math.pi / 64, HZ, STR2, REN, threads=4)
    rhs = np.zeros(o.field_shape())
    rhs[:, 1:M + 1, 1:L + 1] = np.random.default_rng(L + M).standard_normal((N, M, L))
    ph = o.xio_poisson(rhs)
    assert _operator_residual(o, rhs, ph) < 1e-13
    assert np.abs(ph[:, :, 0]).max() == 0.0 and np.abs(ph[:, :, L + 1]).max() == 0.0
    o.close()


def test_host_roots_equal_oracle_roots():
    s = xinout_setup(96, 32, 48, 3.0, HZ, STR2, REN)
    o = OracleXinout(96, 32, 48, 3.0, HZ, STR2, REN)
    assert np.array_equal(s.AK1, o.akx()) and np.array_equal(s.AK3, o.akz())
    assert s.iFlowDriven == 0
    o.close()


def coupled_case(LT=32, L=64, M=32, N=32, seed=41, threads=8):
    """A TG domain after its NS = 0 projection and a main domain started from it."""
    DX = 2 * math.pi / 64
    st = channel_setup(LT, M, N, LT * DX, HZ, STR2, REN)
    tg = Oracle(LT, M, N, LT * DX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=threads)
    Q, PR = initial_field(st, seed, 0.2)
    tg.set_fields(Q, PR)
    tg.substep(0)
    Qt, _, _ = tg.get_fields()
    io = OracleXinout(L, M, N, L * DX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=threads)
    G, P = xinout_fields_from_tg(Qt, L)
    ones = np.ones(io.field_shape())
    io.io_set_fields(G, P, ones, ones, ones)
    io.set_dt(1e-3)
    return tg, io


def test_coupled_run_inlet_outlet_and_projection():
    tg, io = coupled_case()
    L, M, N = io.L, io.M, io.N
    rc, cfl_dt = io.xio_run_steps(tg, 4)
    assert rc == 0 and np.all(cfl_dt > 0)
    assert io.dt() == tg.dt()
    G, Q, P = io.io_get_fields()
    Qt, _, _ = tg.get_fields()
    assert np.isfinite(G).all() and np.isfinite(P).all()
    # inlet: the ghost column is the TG domain's last column, the inlet face its first u face
    assert np.array_equal(Q[:, :, 1:M + 1, 0], Qt[:, :, 1:M + 1, -1])
    assert np.array_equal(G[0, :, 1:M + 1, 1], Qt[0, :, 1:M + 1, 0])
    # outflow scaling: after BC_COUTLET the outlet flux matched the inlet flux; the scaling factor
    # stays within round-off-sized steps of 1 for this near-periodic start
    u_out, scaling = io.xio_outlet_state()
    assert 0.5 < u_out < 1.5 and abs(scaling - 1.0) < 1e-4
    div = io.xio_divgck()
    assert div[0] < 1e-12 and div[2] < 1e-12, div  # cells 2..L-1 and L
    assert div[1] < 1e-2, div  # cells 0..1: the inlet cell's residual
    tg.close()
    io.close()


def thermal_case(LT=32, L=64, M=32, N=32, qw=0.5, threads=8):
    """The coupled flow case plus the thermal solver on the main domain: the seeded synthetic
    table, rho*h perturbed by 1e-3 (interior and both ghost columns), the inlet state from the
    table at rho*h = 0, a constant heat flux on both walls."""
    import oracle as orc
    from chapsim import thermo
    tg, io = coupled_case(LT, L, M, N, threads=threads)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / REN / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros(io.field_shape())
    DH[:, 1:M + 1, :] = 1e-3 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L + 2))
    ot = orc.PropTable(tab.lists)
    io.thermal_enable(ot, DH, qw, qw, cthecd)
    r, nbad, _ = ot.update(np.array([0.0]))
    assert nbad == 0
    st = [float(r[k][0]) for k in ("T", "H", "D", "M", "K", "CP")]
    inlet = st + [st[2] * st[1]]
    io.xio_thermal_inlet(inlet)
    return tg, io, ot, tab, DH, cthecd, inlet


def test_thermal_inflow_outflow_oracle_run():
    """BC_TINLET_THERML holds the inlet column at the inlet state, BC_COUTLET_ENEG_RK3 carries
    rho*h out, the heated walls raise the mean rho*h, and the interior stays divergence-free
    against DrhoDtP (DIVGCK_io adds it)."""
    tg, io, ot, tab, DH, cthecd, inlet = thermal_case()
    L, M = io.L, io.M
    rc, _ = io.xio_run_steps(tg, 3)
    assert rc == 0
    th = io.thermal_get()
    # rows 1..M of the inlet column (BC_WALL_THERMAL then re-extrapolates its wall rows)
    assert np.all(th["DH"][:, 1:M + 1, 0] == inlet[6]) and np.all(th["T"][:, 1:M + 1, 0] == inlet[0])
    assert np.isfinite(th["DH"]).all()
    assert th["DH"][:, 1:M + 1, 1:L + 1].mean() > DH[:, 1:M + 1, 1:L + 1].mean()
    div = io.xio_divgck()
    assert div[0] < 1e-11 and div[2] < 1e-11, div
    tg.close()
    io.close()
