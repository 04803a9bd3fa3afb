"""Property-table set-up and the table-search oracle (CPU).

Pins of the restated CUBIC_SPLINE and search (the reference ships no output
of its table path): Forsythe-Malcolm-Moler end conditions reproduce any cubic
exactly, the spline passes through its knots, and the search returns the
reference's interval (I = N at the last knot).  The F7 assignment
(DENSITY <- mu spline, Viscousity <- kappa spline, THERMCONDT <- rho spline)
is checked at the knots, where each spline returns its own table column.
"""
import os

import numpy as np
import pytest

import oracle
from chapsim import thermo

# every 6th row of the reference's NIST_WATER_23.5MP.DAT (TC4), written by tests/golden/make_golden.py
NIST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nist_water_rows.npz")


@pytest.fixture(scope="module")
def synth():
    rows, T0 = thermo.synthetic_table()
    return rows, T0, thermo.SplineTable.from_rows(rows, T0)


def test_cubic_spline_reproduces_cubics():
    rng = np.random.default_rng(3)
    x = np.cumsum(rng.uniform(0.2, 1.0, 40))
    p = np.array([0.7, -1.3, 0.25, -0.04])          # y = p0 + p1 x + p2 x^2 + p3 x^3
    y = p[0] + x * (p[1] + x * (p[2] + x * p[3]))
    for b, c, d in (thermo.cubic_spline(x, y), oracle.cubic_spline(x, y)):
        np.testing.assert_allclose(b, p[1] + 2 * p[2] * x + 3 * p[3] * x**2, rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(c, p[2] + 3 * p[3] * x, rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(d, np.full_like(x, p[3]), rtol=1e-7)


def test_cubic_spline_host_equals_oracle_bitwise():
    rng = np.random.default_rng(11)
    for n in (2, 3, 4, 5, 17, 300):
        x = np.cumsum(rng.uniform(0.01, 1.0, n))
        y = rng.standard_normal(n)
        for a, b in zip(thermo.cubic_spline(x, y), oracle.cubic_spline(x, y)):
            assert np.array_equal(a, b), n


def test_search_interval_semantics():
    x = np.array([0.0, 1.0, 2.0, 3.0, 4.0])
    lib = oracle.lib()
    idx = [lib.orc_spline_index(5, oracle._p(x), u) for u in (0.0, 0.5, 1.0, 3.999, 4.0, 4.0 + 5e-9)]
    assert idx == [0, 0, 1, 3, 4, 4]


def test_synthetic_table_shape(synth):
    rows, T0, tab = synth
    assert rows.shape == (2048, 8)
    h, T, rho, mu, kap, cp = rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4], rows[:, 5], rows[:, 6]
    assert np.all(np.diff(h) > 0) and np.all(np.diff(T) > 0)
    assert np.all(np.diff(rho) < 0) and np.all(np.diff(mu) < 0) and np.all(np.diff(kap) < 0)
    base = min(cp[0], cp[-1])
    assert 7.5 < cp.max() / base < 8.0                   # peak 8x the baseline (sampled)
    above = h[cp - base >= 0.5 * (cp.max() - base)]
    fwhm = (above[-1] - above[0]) / (h[-1] - h[0])
    assert abs(fwhm - 0.03) < 0.002
    assert T[0] < T0 < T[-1]
    assert np.all(np.diff(tab.lists["DH"]) > 0)


def test_nondim_and_coefficients_equal_oracle(synth):
    rows, T0, tab = synth
    lists, ref = oracle.table_nondim(rows, T0)
    for k in thermo.LIST_NAMES:
        assert np.array_equal(lists[k], tab.lists[k]), k
    assert ref == tab.ref
    ot = oracle.PropTable(lists)
    for name in oracle.SPLINES:
        assert np.array_equal(np.array(tab.coef[name]), ot.coefs(name)), name


@pytest.mark.parametrize("fix_swap", [False, True])
def test_update_at_knots_returns_table_columns(synth, fix_swap):
    _, _, tab = synth
    ot = oracle.PropTable(tab.lists, fix_swap=fix_swap)
    L = tab.lists
    res, nbad, fb = ot.update(L["DH"])
    assert nbad == 0 and fb == -1
    assert np.array_equal(res["H"], L["H"]) and np.array_equal(res["T"], L["T"])
    assert np.array_equal(res["CP"], L["CP"])
    if fix_swap:
        want = {"D": L["D"], "M": L["M"], "K": L["K"]}
    else:
        want = {"D": L["M"], "M": L["K"], "K": L["D"]}
    for k, v in want.items():
        assert np.array_equal(res[k], v), k


def test_update_range_checks(synth):
    _, _, tab = synth
    ot = oracle.PropTable(tab.lists)
    lo, hi = tab.lists["DH"][0], tab.lists["DH"][-1]
    # within 1e-8 of the ends: accepted.  hi + 5e-9 passes the rho*h check but
    # maps to an h about 4e-8 beyond LIST_H (dh/d(rho h) ~ 8 there), where the
    # H-spline check stops, as in the reference.
    dh = np.array([0.5 * (lo + hi), hi + 1e-9, lo - 5e-9, hi + 5e-9, hi + 2e-8, 0.3 * lo + 0.7 * hi, lo - 3e-8])
    res, nbad, fb = ot.update(dh)
    assert nbad == 3 and fb == 3
    # interior values are smooth interpolants
    assert np.all(np.isfinite(res["T"][:3]))


def test_update_interpolates_smoothly(synth):
    """Between knots the interpolants of the swapped columns follow those columns."""
    rows, T0, tab = synth
    ot = oracle.PropTable(tab.lists, fix_swap=True)
    dh = thermo.table_field(rows, T0, (5000,), seed=5)
    res, nbad, _ = ot.update(dh)
    assert nbad == 0
    H = tab.lists["H"]
    for k in ("T", "D", "M", "K", "CP"):
        lin = np.interp(res["H"], H, tab.lists[k])
        scale = np.ptp(tab.lists[k])
        assert np.max(np.abs(res[k] - lin)) < 1e-3 * scale, k


def test_nist_table_setup_equals_oracle():
    fx = np.load(NIST)
    rows = fx["rows"]
    assert int(fx["n_full"]) == 11998 and rows.shape == (2000, 8)
    tab = thermo.SplineTable.from_rows(rows, 680.15)
    lists, ref = oracle.table_nondim(rows, 680.15)
    for k in thermo.LIST_NAMES:
        assert np.array_equal(lists[k], tab.lists[k]), k
    ot = oracle.PropTable(lists)
    for name in oracle.SPLINES:
        assert np.array_equal(np.array(tab.coef[name]), ot.coefs(name)), name
    # the reference state sits at T0 = 680.15 K inside the table; h is zero there
    assert abs(np.interp(1.0, tab.lists["T"], tab.lists["H"])) < 1e-3
    assert np.all(np.diff(tab.lists["DH"]) > 0)
