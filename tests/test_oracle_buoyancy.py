"""CPU pins of the oracle's buoyancy (iGravity) and weighted-pressure
(iWeightedPre) terms of RHS_MOM_EXPLICIT_io (src/RHS_MOM_EXPLICIT_io.f90:103-226)
and DIVG_io (src/DIVG.f90:78-82).

No reference output exercises either option (the shipped cases that set
iGravity = 1 are thermal runs whose output is not shipped; every case sets
iWeightedPre = 0), so these checks pin properties the terms must have:
* with uniform density a buoyancy force along x (the flow direction) is a
  uniform body force, which the constant-mass-flux forcing DPGRNS takes
  out again: the fields equal the run without gravity to round-off;
* with uniform density a buoyancy force along y is hydrostatic: the
  velocity is unchanged and the pressure gains F_A * y (plus a constant);
* with PR0 equal to PR the weighted gradient is the plain one, so the first
  substep differs only through DIVG_io's factor 1/(1/4 + eps): the pressure
  increment is that factor times the unweighted one.
"""
import math

import numpy as np

from oracle import Oracle
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

L, M, N = 32, 32, 16
HX, HZ, STR2, REN = 2 * math.pi, math.pi, 2.0, 2800.0
EPS = 0.001


def _case(ivis=0):
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 91, 0.1)
    PR = PR + 0.01 * np.random.default_rng(4).standard_normal(PR.shape)
    ones = np.ones_like(PR)
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=4)
    o.io_set_fields(Q, PR, ones, ones, ones)
    o.io_set_vis_scheme(ivis)
    o.set_dt(1e-3)
    return s, o, PR


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_streamwise_buoyancy_with_uniform_density_is_taken_by_the_mass_flux_forcing():
    for ivis in (0, 1):
        _, a, _ = _case(ivis)
        _, b, _ = _case(ivis)
        b.io_set_buoyancy(1, 0.37)
        assert a.io_run_steps(3)[0] == 0 and b.io_run_steps(3)[0] == 0
        ga, _, pa = a.io_get_fields()
        gb, _, pb = b.io_get_fields()
        assert rel(gb[:, :, 1:M + 1], ga[:, :, 1:M + 1]) < 1e-12, ivis
        da = pa[:, 1:M + 1] - pa[:, 1:M + 1].mean()
        db = pb[:, 1:M + 1] - pb[:, 1:M + 1].mean()
        assert rel(db, da) < 1e-9, ivis


def test_wall_normal_buoyancy_with_uniform_density_is_hydrostatic():
    s, a, _ = _case(0)
    _, b, _ = _case(0)
    fa = -0.21
    b.io_set_buoyancy(-2, fa)
    assert a.io_run_steps(3)[0] == 0 and b.io_run_steps(3)[0] == 0
    ga, _, pa = a.io_get_fields()
    gb, _, pb = b.io_get_fields()
    assert rel(gb[:, :, 1:M + 1], ga[:, :, 1:M + 1]) < 1e-10
    dp = (pb - pa)[:, 1:M + 1]
    y = s.YCC[1:M + 1][None, :, None]
    hyd = fa * y
    d = (dp - dp.mean()) - (hyd - hyd.mean())
    assert float(np.abs(d).max()) < 1e-10 * float(np.abs(hyd).max()) + 1e-12


def test_buoyancy_acts_on_its_component_only_with_variable_density():
    # a density that varies in y: the x force is no longer uniform and changes the flow
    s, a, _ = _case(0)
    _, b, PR = _case(0)
    k, j, i = np.meshgrid(np.arange(N), np.arange(M + 2), np.arange(L), indexing="ij")
    rho = 1.0 + 0.2 * np.cos(np.pi * (j - 0.5) / M)
    for o in (a, b):
        G, _, P = o.io_get_fields()
        o.io_set_fields(G, P, rho, np.ones_like(rho), np.ones_like(rho))
        o.set_dt(1e-3)
    b.io_set_buoyancy(1, 0.5)
    assert a.io_run_steps(2)[0] == 0 and b.io_run_steps(2)[0] == 0
    ga, _, _ = a.io_get_fields()
    gb, _, _ = b.io_get_fields()
    assert rel(gb[0][:, 1:M + 1], ga[0][:, 1:M + 1]) > 1e-6
    assert b.io_divgck() < 1e-11


def test_weighted_pressure_scales_the_first_pressure_increment():
    _, a, P0 = _case(0)
    _, b, _ = _case(0)
    b.io_set_weighted_pressure(P0, P0)
    a.io_substep(1)
    b.io_substep(1)
    _, _, pa = a.io_get_fields()
    _, _, pb = b.io_get_fields()
    inc_a = (pa - P0)[:, 1:M + 1]
    inc_b = (pb - P0)[:, 1:M + 1]
    assert rel(inc_b, inc_a / (0.25 + EPS)) < 1e-10


def test_weighted_pressure_off_restores_the_plain_step():
    _, a, P0 = _case(0)
    _, b, _ = _case(0)
    b.io_set_weighted_pressure(P0, P0)
    b.io_set_weighted_pressure(None)
    assert a.io_run_steps(2)[0] == 0 and b.io_run_steps(2)[0] == 0
    ga, _, pa = a.io_get_fields()
    gb, _, pb = b.io_get_fields()
    assert np.array_equal(ga, gb) and np.array_equal(pa, pb)
