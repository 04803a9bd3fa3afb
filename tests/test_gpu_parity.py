"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Acceptance (plain FP64 path): every field within 1e-11 relative (max-norm
of the difference over the max-norm of the oracle field) after 10 steps,
and max|div u| <= 1e-12.  Line solvers and the Poisson solve alone are held
to 1e-12."""
import math

import numpy as np
import pytest

import oracle as orc
from oracle import Oracle
from chapsim import gpu
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field, bulk_velocity

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-11
TOL_OP = 1e-12


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _pair(L, M, N, HX, HZ, STR2, REN, seed=1973, dt0=1e-3, cflgv=0.5, fix=False, threads=8):
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, seed, 0.1)
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=dt0, CFLGV=cflgv, threads=threads)
    o.set_fix_v_wall_row(fix)
    o.set_fields(Q, PR)
    c = gpu.ChannelTG(s, fix_v_wall_row=fix)
    c.upload(Q, PR)
    c.set_dt(dt0)
    return s, o, c


def _cmp_fields(o, c, tol):
    Qo, PRo, H0o = o.get_fields()
    Qg, PRg, H0g = c.download(want_h0=True)
    M = c.M
    errs = {
        "U": rel(Qg[0], Qo[0]), "V": rel(Qg[1], Qo[1]), "W": rel(Qg[2], Qo[2]),
        "P": rel(PRg[:, 1:M + 1], PRo[:, 1:M + 1]),
        "H0": rel(H0g, H0o[:, :, 1:M + 1, :]),
    }
    for k, v in errs.items():
        assert v <= tol, (k, v, errs)
    return errs


# ----------------------------------------------------------------- line solvers
@pytest.mark.parametrize("n", [32, 64, 96, 128, 192, 256, 384, 48, 20])
def test_tdmaiji_cyc(n):
    rng = np.random.default_rng(n)
    jsz = 37
    A = -rng.uniform(0.0, 0.4, (jsz, n))
    C = -rng.uniform(0.0, 0.4, (jsz, n))
    B = 1.0 - A - C + rng.uniform(0.0, 0.2, (jsz, n))
    R = rng.standard_normal((jsz, n))
    got = gpu.tdmaiji_cyc(A, B, C, R)
    for j in range(jsz):
        ref = orc.tdma_cyc(A[j], B[j], C[j], R[j])
        assert rel(got[j], ref) <= TOL_OP


@pytest.mark.parametrize("n", [32, 64, 96, 128, 192, 256, 384, 40])
def test_tdmaijj_noncyc_with_bc(n):
    rng = np.random.default_rng(100 + n)
    isz = 45
    A = -rng.uniform(0.0, 0.4, (n, isz))
    C = -rng.uniform(0.0, 0.4, (n, isz))
    B = 1.0 - A - C + rng.uniform(0.0, 0.2, (n, isz))
    R = rng.standard_normal((n, isz))
    BCJ = rng.standard_normal((2, isz))
    got = gpu.tdmaijj_noncyc(A, B, C, R, BCJ)
    for i in range(isz):
        r = R[:, i].copy()
        r[0] -= A[0, i] * BCJ[0, i]
        r[-1] -= C[-1, i] * BCJ[1, i]
        a = A[:, i].copy(); a[0] = 0.0
        c = C[:, i].copy(); c[-1] = 0.0
        ref = orc.tdma_noncyc(a, B[:, i], c, r)
        assert rel(got[:, i], ref) <= TOL_OP


# ----------------------------------------------------------------- Poisson
@pytest.mark.parametrize("shape", [(64, 64, 64), (96, 64, 192), (128, 96, 64), (32, 32, 32), (256, 32, 384), (384, 64, 256)])
def test_fft99_poisson(shape):
    L, M, N = shape
    s = channel_setup(L, M, N, 4 * math.pi, 4 * math.pi / 3, 2.0, 2800.0)
    o = Oracle(L, M, N, 4 * math.pi, 4 * math.pi / 3, 2.0, 2800.0, threads=8)
    c = gpu.ChannelTG(s)
    rng = np.random.default_rng(L + M + N)
    rhs = rng.standard_normal((N, M, L))
    full = np.zeros((N, M + 2, L))
    full[:, 1:M + 1, :] = rhs
    ref = o.poisson(full)
    got = c.FFT99_POIS3D_periodicxz(rhs)
    assert rel(got[:, 1:M + 1], ref[:, 1:M + 1]) <= TOL_OP
    c.close()


# ----------------------------------------------------------------- full step
def test_projection_substep_ns0():
    s, o, c = _pair(64, 64, 64, 2 * math.pi, math.pi, 2.0, 2800.0)
    o.substep(0)
    c.SOLVERRK3_MOM_tg(0)
    _cmp_fields(o, c, TOL_OP * 10)
    assert c.DIVGCK_tg() <= 1e-12


def test_c1_ten_steps():
    """64^3 channel, 2pi x 2 x pi, STR2 = 2, REN = 2800, CFL 0.5: 10 steps."""
    s, o, c = _pair(64, 64, 64, 2 * math.pi, math.pi, 2.0, 2800.0, dt0=2e-3, cflgv=0.5)
    o.substep(0)
    c.SOLVERRK3_MOM_tg(0)
    rc, dts = o.run_steps(10)
    assert rc == 0
    dt, cfl = c.advance(10, 2e-3, 1e-6, 0.5)
    assert abs(dt - dts[-1]) <= 1e-13 * dts[-1]
    _cmp_fields(o, c, TOL_STEP)
    assert c.DIVGCK_tg() <= 1e-12
    Qg, _ = c.download()
    assert abs(bulk_velocity(s, Qg) - 1.0) < 1e-9


def test_c2_shape_three_steps():
    """128^3 channel, 4pi x 2 x 4pi/3 (the benchmark configuration)."""
    s, o, c = _pair(128, 128, 128, 4 * math.pi, 4 * math.pi / 3, 2.0, 2800.0, dt0=2e-3, cflgv=0.5)
    o.substep(0)
    c.SOLVERRK3_MOM_tg(0)
    o.run_steps(3)
    c.advance(3, 2e-3, 1e-6, 0.5)
    _cmp_fields(o, c, TOL_STEP)
    assert c.DIVGCK_tg() <= 1e-12


@pytest.mark.parametrize("shape", [(96, 64, 192), (192, 96, 96), (32, 64, 32)])
def test_ragged_shapes(shape):
    L, M, N = shape
    s, o, c = _pair(L, M, N, 4 * math.pi, 4 * math.pi / 3, 2.0, 2800.0, seed=7, dt0=2e-3)
    o.substep(0)
    c.SOLVERRK3_MOM_tg(0)
    o.run_steps(4)
    c.advance(4, 2e-3, 1e-6, 0.5)
    _cmp_fields(o, c, TOL_STEP)


def test_fix_v_wall_row_option():
    s, o, c = _pair(64, 64, 64, 2 * math.pi, math.pi, 2.0, 2800.0, fix=True)
    o.substep(0)
    c.SOLVERRK3_MOM_tg(0)
    o.run_steps(3)
    c.advance(3, 1e-3, 1e-6, 0.5)
    _cmp_fields(o, c, TOL_STEP)


def test_constant_pressure_gradient_drive():
    L = M = N = 64
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, iFlowDriven=2, Cf_Given=8.18e-3)
    Q, PR = initial_field(s, 3, 0.1)
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, iFlowDriven=2, Cf_Given=8.18e-3, DT0=1e-3, threads=8)
    o.set_fields(Q, PR)
    c = gpu.ChannelTG(s)
    c.upload(Q, PR)
    c.set_dt(1e-3)
    o.substep(0); c.SOLVERRK3_MOM_tg(0)
    o.run_steps(3); c.advance(3, 1e-3, 1e-6, 0.5)
    _cmp_fields(o, c, TOL_STEP)


def test_graph_path_equals_per_call_path():
    s = channel_setup(64, 64, 64, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 11, 0.1)
    outs = []
    for use_graph in (True, False):
        c = gpu.ChannelTG(s)
        c.upload(Q, PR)
        c.set_dt(1e-3)
        c.SOLVERRK3_MOM_tg(0)
        if use_graph:
            c.advance(3, 1e-3, 1e-6, 0.5)
        else:
            for _ in range(3):
                c.step_begin(1e-3, 1e-6, 0.5)
                for ns in (1, 2, 3):
                    c.SOLVERRK3_MOM_tg(ns)
        outs.append(c.download())
        c.close()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


# ----------------------------------------------------------------- full size, size-independent properties
def test_full_size_c3_properties():
    """384 x 256 x 384 (Re_tau 395 box): one projection and two steps keep the
    field divergence-free and the bulk velocity at 1, and two runs agree bitwise."""
    L, M, N = 384, 256, 384
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 6875.0)
    Q, PR = initial_field(s, 1973, 0.1)
    outs = []
    for _ in range(2):
        c = gpu.ChannelTG(s)
        c.upload(Q, PR)
        c.set_dt(5e-4)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(2, 5e-4, 1e-6, 0.5)
        assert c.DIVGCK_tg() <= 1e-11
        Qg, PRg = c.download()
        assert abs(bulk_velocity(s, Qg) - 1.0) < 1e-9
        assert np.isfinite(Qg).all() and np.isfinite(PRg).all()
        outs.append(Qg)
        c.close()
    assert np.array_equal(outs[0], outs[1])


# ----------------------------------------------------------------- error paths (host-detected, no GPU fault)
def test_nan_field_reports_error():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 1, 0.1)
    Q[0, 3, 5, 7] = np.nan
    c = gpu.ChannelTG(s)
    c.upload(Q, PR)
    with pytest.raises(gpu.ChapsimError) as e:
        c.step_begin(1e-3, 1e-6, 0.5)
    assert e.value.code == -2


def test_dt_collapse_reports_error():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 1, 0.1)
    c = gpu.ChannelTG(s)
    c.upload(Q, PR)
    c.set_dt(1.0)
    with pytest.raises(gpu.ChapsimError) as e:
        c.advance(1, 1.0, 1e-9, 1e-4)
    assert e.value.code == -3


def test_bad_arguments():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    c = gpu.ChannelTG(s)
    with pytest.raises(gpu.ChapsimError):
        c.SOLVERRK3_MOM_tg(4)
    with pytest.raises(gpu.ChapsimError):
        c.set_dt(-1.0)
    with pytest.raises(ValueError):
        c.upload(np.zeros((3, 2, 2, 2)), np.zeros((2, 2, 2)))
