"""Pins the oracle's set-up stage (and the host set-up of the package) to the
reference's own outputs: the CHK_*.dat dumps of the TC8 case (64^3 channel,
STR2 = 3.75, HX = 6, HZ = 3, REN = 2800), extracted by tests/golden/make_golden.py."""
import json
import os

import numpy as np
import pytest

from oracle import Oracle
from chapsim.mesh import channel_setup


@pytest.fixture(scope="module")
def fx(golden_dir):
    with open(os.path.join(golden_dir, "tc8_setup.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def orc(fx):
    c = fx["case"]
    return Oracle(c["NCL1"], c["NCL2"], c["NCL3"], c["HX"], c["HZ"], c["STR2"], c["REN"])


def _close(a, b, digits):
    """Elementwise agreement with a value printed to `digits` significant digits."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    tol = 0.51 * 10.0 ** (1 - digits) * np.abs(b) + 1e-300
    return np.all(np.abs(a - b) <= np.maximum(tol, 1e-12 * np.abs(b).max()))


def test_mesh_y(orc, fx):
    assert _close(orc.y("YND"), fx["YND"], 8)
    assert _close(orc.y("YCC"), fx["YCC"], 8)
    assert _close(1.0 / orc.y("DYCI"), fx["inv_DYCI"], 8)
    assert _close(1.0 / orc.y("DYFI"), fx["inv_DYFI"], 8)
    assert _close(orc.y("DYCI"), fx["DYCI"], 6)


def test_y_weights(orc, fx):
    assert _close(orc.y("WFF"), fx["WFF"], 6)
    assert _close(orc.y("WFB"), fx["WFB"], 6)


def test_tdma_coefficients(orc, fx):
    for n in ("AMPH", "ACPH", "APPH"):
        assert _close(orc.y(n), fx[n], 8), n
    for idr in (1, 2, 3):
        for n in ("AMVR", "ACVR", "APVR"):
            ref = fx[f"{n}{idr}"]
            assert _close(orc.y(n, idr)[: len(ref)], ref, 8), (n, idr)


def test_poiseuille(orc, fx):
    assert _close(orc.y("Vini"), fx["Vini"], 8)


def test_xz_nodes(orc, fx):
    s = orc.scalars()
    xnd = np.arange(len(fx["XND"])) * s["DX"]
    znd = np.arange(len(fx["ZND"])) * s["DZ"]
    assert np.allclose(xnd, fx["XND"], rtol=0, atol=1e-15)
    assert np.allclose(znd, fx["ZND"], rtol=0, atol=1e-15)


def test_host_setup_equals_oracle_bitwise(fx):
    c = fx["case"]
    s = channel_setup(c["NCL1"], c["NCL2"], c["NCL3"], c["HX"], c["HZ"], c["STR2"], c["REN"])
    o = Oracle(c["NCL1"], c["NCL2"], c["NCL3"], c["HX"], c["HZ"], c["STR2"], c["REN"])
    M = c["NCL2"]
    sc = o.scalars()
    assert sc["VOLM"] == s.VOLM and sc["Area_inlet"] == s.Area_inlet
    assert sc["DXI"] == s.DXI and sc["DZQI"] == s.DZQI
    for name, arr, n in (("YND", s.YND, M + 1), ("DYFI", s.DYFI, M), ("DYCI", s.DYCI, M + 1), ("WFF", s.WFF, M + 1),
                         ("WFB", s.WFB, M + 1), ("AMPH", s.AMPH, M), ("ACPH", s.ACPH, M), ("APPH", s.APPH, M),
                         ("Vini", s.Vini, M)):
        assert np.array_equal(o.y(name)[:n], arr[1:n + 1]), name
    for idr in (1, 2, 3):
        assert np.array_equal(o.y("ACVR", idr), s.ACVR[idr, 1:M + 2])
        assert np.array_equal(o.y("AMVR", idr), s.AMVR[idr, 1:M + 2])
        assert np.array_equal(o.y("APVR", idr), s.APVR[idr, 1:M + 2])
