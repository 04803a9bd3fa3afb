"""Unit checks of the CPU oracle's building blocks (FFT, line solvers,
Poisson solve, projection) against independent numpy computations."""
import math

import numpy as np
import pytest

import oracle as orc_mod
from oracle import Oracle
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field, bulk_velocity


@pytest.mark.parametrize("n", [8, 12, 64, 96, 128, 192, 384, 30])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft_matches_numpy(n, sign):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    got = orc_mod.fft_complex(x, sign)
    ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


def _dense(A, B, C, cyclic):
    n = len(B)
    T = np.diag(B) + np.diag(A[1:], -1) + np.diag(C[:-1], 1)
    if cyclic:
        T[0, -1] = A[0]
        T[-1, 0] = C[-1]
    return T


@pytest.mark.parametrize("n", [5, 17, 64, 128])
def test_tdma_cyc(n):
    rng = np.random.default_rng(7 + n)
    A = -rng.uniform(0.1, 1.0, n)
    C = -rng.uniform(0.1, 1.0, n)
    B = 1.0 - A - C + rng.uniform(0.0, 0.5, n)
    R = rng.standard_normal(n)
    x = orc_mod.tdma_cyc(A, B, C, R)
    ref = np.linalg.solve(_dense(A, B, C, True), R)
    assert np.max(np.abs(x - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("n", [3, 16, 64, 129])
def test_tdma_noncyc(n):
    rng = np.random.default_rng(11 + n)
    A = -rng.uniform(0.1, 1.0, n)
    C = -rng.uniform(0.1, 1.0, n)
    B = 1.0 - A - C + rng.uniform(0.0, 0.5, n)
    R = rng.standard_normal(n)
    x = orc_mod.tdma_noncyc(A, B, C, R)
    ref = np.linalg.solve(_dense(A, B, C, False), R)
    assert np.max(np.abs(x - ref)) <= 1e-13 * np.max(np.abs(ref))


def _laplacian(s, phi):
    """Discrete operator of FFT99_POIS3D_periodicxz applied to phi (N, M+2, L)."""
    M = s.M
    p = phi[:, 1:M + 1, :]
    lap = (np.roll(p, -1, 2) - 2 * p + np.roll(p, 1, 2)) * s.DXQI + (np.roll(p, -1, 0) - 2 * p + np.roll(p, 1, 0)) * s.DZQI
    am, ac, ap = s.AMPH[1:M + 1], s.ACPH[1:M + 1], s.APPH[1:M + 1]
    pm = phi[:, 0:M, :]
    pp = phi[:, 2:M + 2, :]
    lap += am[None, :, None] * pm + ac[None, :, None] * p + ap[None, :, None] * pp
    return lap


@pytest.mark.parametrize("shape", [(32, 16, 24), (64, 32, 48)])
def test_poisson_residual(shape):
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    rng = np.random.default_rng(3)
    rhs = np.zeros((N, M + 2, L))
    rhs[:, 1:M + 1, :] = rng.standard_normal((N, M, L))
    phi = o.poisson(rhs)
    res = _laplacian(s, phi) - rhs[:, 1:M + 1, :]
    scale = np.abs(rhs).max()
    # every row but the pinned one is solved exactly; the pinned zero mode
    # leaves a residual that is constant over x and z in row j = 1
    assert np.abs(res[:, 1:, :]).max() <= 1e-10 * scale
    assert np.ptp(res[:, 0, :]) <= 1e-10 * scale
    assert np.abs(phi[:, 1, :].mean()) <= 1e-12 * np.abs(phi).max()


def test_projection_is_divergence_free():
    L, M, N = 32, 32, 32
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 1973, 0.1)
    assert abs(bulk_velocity(s, Q) - 1.0) < 1e-14
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, DT0=1e-3)
    o.set_fields(Q, PR)
    assert o.divgck() > 1.0
    o.substep(0)
    assert o.divgck() < 1e-12
    rc, dts = o.run_steps(3)
    assert rc == 0 and o.divgck() < 1e-12


def test_fix_v_wall_row_changes_only_v_path():
    """The reproduced quirk matters: zeroing row 1 of the v sweep changes v."""
    L, M, N = 32, 32, 32
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 5, 0.1)
    out = []
    for fix in (False, True):
        o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, DT0=1e-3)
        o.set_fix_v_wall_row(fix)
        o.set_fields(Q, PR)
        o.substep(0)
        o.substep(1)
        out.append(o.get_fields()[0])
    d = np.abs(out[0] - out[1])
    assert d[1].max() > 1e-12
