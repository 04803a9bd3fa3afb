"""CPU checks of the oracle's statistics routines (PP_MEAN_ZX_FLOW_TG,
PP_MEAN_T_TG, PP_MONITOR_TG) against independent numpy computations of the
same definitions on a seeded, stepped 32^3 channel."""
import math

import numpy as np
import pytest

from oracle import Oracle
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

L = M = N = 32


@pytest.fixture(scope="module")
def stepped():
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 11, 0.1)
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, DT0=0.02, DTMIN=1e-6, CFLGV=0.5, threads=4)
    o.set_fields(Q, PR)
    o.substep(0)
    o.run_steps(3)
    Qs, Ps, _ = o.get_fields()
    return s, o, Qs, Ps


def _split(flat):
    names = [("U1", 4), ("UP", 3), ("U2", 6), ("U3", 10), ("D1", 9), ("DP", 9), ("D2", 81)]
    out, off = {}, 0
    for n, w in names:
        out[n] = flat[off * M:(off + w) * M].reshape(w, M)
        off += w
    return out


def test_plane_means_match_numpy(stepped):
    s, o, Q, P = stepped
    got = _split(o.pp_mean_zx_tg())
    u, v, w = Q  # (N, M+2, L)
    js = slice(1, M + 1)
    U = np.stack([(u + np.roll(u, -1, axis=2))[:, js], (v[:, 1:M + 1] + v[:, 2:M + 2]),
                  (w + np.roll(w, -1, axis=0))[:, js]])        # cell-centred sums U_CCT
    p = P[:, js]
    mean = lambda a: a.mean(axis=(0, 2))  # noqa: E731

    def close(got_row, integrand, scale):
        # a plane mean carries round-off of the size of its summands, whatever the mean itself
        ref = scale * mean(integrand)
        return np.abs(got_row - ref).max() <= 1e-13 * scale * np.abs(integrand).max()

    for m in range(3):
        assert close(got["U1"][m], U[m], 0.5)
        assert close(got["UP"][m], U[m] * p, 0.5)
    assert close(got["U1"][3], p, 1.0)
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    for l, (a, b) in enumerate(pairs):
        assert close(got["U2"][l], U[a] * U[b], 0.25)
    trip = [(0, 0, 0), (0, 0, 1), (0, 0, 2), (0, 1, 1), (0, 1, 2), (0, 2, 2), (1, 1, 1), (1, 1, 2), (1, 2, 2), (2, 2, 2)]
    for l, (a, b, c) in enumerate(trip):
        assert close(got["U3"][l], U[a] * U[b] * U[c], 0.125)
    # du/dx at the cell centre and <du/dx>, with COG1(1,1) = DXI / (L N)
    dudx = (np.roll(u, -1, axis=2) - u)[:, js]
    assert close(got["D1"][0], dudx, s.DXI)
    # (dw/dz)^2 entry of DVDL2 (L1 = L2 = 9): the reference scales it by
    # COG2 = COG1(3,3)^2, which carries VL1313 = 1/(L N) twice (PP_MEAN_ZX.f90:82-93)
    dwdz = (np.roll(w, -1, axis=0) - w)[:, js]
    assert close(got["D2"][80], dwdz * dwdz, s.DZI ** 2 / (L * N))
    # symmetry of DVDL2 in (L1, L2)
    d2 = got["D2"].reshape(9, 9, M)
    assert np.array_equal(d2, d2.transpose(1, 0, 2))


def test_time_average_is_running_mean(stepped):
    s, o, Q, P = stepped
    sets, avg, n = [], np.zeros(122 * M), 0
    for _ in range(4):
        o.run_steps(1)
        inst = o.pp_mean_zx_tg()
        sets.append(inst)
        n = o.pp_mean_t_tg(1, inst, avg, n)
    assert n == 4
    ref = np.mean(sets, axis=0)
    assert np.abs(avg - ref).max() <= 1e-14 * np.abs(ref).max()
    summed, n2 = np.zeros(122 * M), 0
    for inst in sets:
        n2 = o.pp_mean_t_tg(2, inst, summed, n2, pp_instn_sz=4)
    assert np.abs(summed - ref).max() <= 1e-14 * np.abs(ref).max()


def test_monitor_quantities(stepped):
    s, o, Q, P = stepped
    inst = o.pp_mean_zx_tg()
    mon = o.pp_monitor_tg(inst, inst, 2800.0)
    g = _split(inst)
    js = M // 2 - 1
    assert mon[0] == g["U1"][0][js] and mon[1] == mon[0]
    assert mon[6] == g["U2"][0][js] - g["U1"][0][js] ** 2
    assert mon[14] == g["U1"][0][0] * s.DYFI[1] * 2.0 * 2.0 / 2800.0
    # U1mean: the bulk velocity, sum_j U1xzL(j,1)/DYFI(j) / DZI * NCL3 / Area_inlet; the
    # seeded start has U_b = 1 up to its perturbation, and the forcing holds it there
    ref = np.sum(g["U1"][0] / s.DYFI[1:M + 1]) / s.DZI * N / s.Area_inlet
    assert abs(mon[18] - ref) <= 1e-14 and abs(mon[18] - 1.0) <= 1e-6
    assert mon[19] == np.abs(g["U1"][0]).max()
