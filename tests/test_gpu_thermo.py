"""CUDA table-search property update against the CPU oracle (bitwise).

The kernel searches once for h on LIST_DH and once on LIST_H, where the
reference searches per spline call; the intervals are the same, and the
cubic is evaluated with explicitly rounded operations, so every output must
equal the oracle's to the last bit.  Tables up to 6144 rows are searched in
shared memory, larger ones in global memory; both paths are covered.
"""
import numpy as np
import pytest

import oracle as orc
from chapsim import gpu, thermo
from chapsim.mesh import channel_setup

pytestmark = pytest.mark.gpu

FIELDS = ("H", "T", "D", "M", "K", "CP")


@pytest.fixture(scope="module")
def chan():
    c = gpu.ChannelTG(channel_setup(32, 32, 32, 6.0, 3.0, 2.0, 2800.0))
    yield c
    c.close()


def _tables(n):
    rows, T0 = thermo.synthetic_table(n=n, seed=n)
    return rows, T0, thermo.SplineTable.from_rows(rows, T0)


def _points(rows, T0, tab, npts, seed):
    dh = thermo.table_field(rows, T0, (npts,), seed=seed, frac=(0.0, 1.0))
    L = tab.lists["DH"]
    knots = np.concatenate([L, 0.5 * (L[1:] + L[:-1]), [L[0] - 5e-9, L[-1] + 1e-9]])
    return np.concatenate([knots, dh])


@pytest.mark.parametrize("n_list", [2048, 8192])
@pytest.mark.parametrize("fix_swap", [False, True])
def test_points_bitwise_equal_oracle(chan, n_list, fix_swap):
    rows, T0, tab = _tables(n_list)
    chan.prop_table_init(tab, fix_swap=fix_swap)
    dh = _points(rows, T0, tab, 1 << 20, seed=n_list + fix_swap)
    got = chan.THERM_PROP_UPDATE_points(dh)
    want, nbad, _ = orc.PropTable(tab.lists, fix_swap=fix_swap).update(dh)
    assert nbad == 0
    for k in FIELDS:
        assert np.array_equal(got[k], want[k]), k


def test_heated_channel_size_bitwise(chan):
    """256 x 192 x 128 points (the heated-channel grid) against the oracle."""
    rows, T0, tab = _tables(2048)
    chan.prop_table_init(tab)
    dh = thermo.table_field(rows, T0, (128, 192, 256), seed=4)
    got = chan.THERM_PROP_UPDATE_points(dh)
    want, nbad, _ = orc.PropTable(tab.lists).update(dh)
    assert nbad == 0
    for k in FIELDS:
        assert np.array_equal(got[k], want[k]), k


def test_out_of_table_point_reports_table_range(chan):
    rows, T0, tab = _tables(2048)
    chan.prop_table_init(tab)
    dh = thermo.table_field(rows, T0, (4096,), seed=9)
    dh[1234] = tab.lists["DH"][-1] + 1e-6
    dh[3000] = tab.lists["DH"][0] - 1e-6
    with pytest.raises(gpu.ChapsimError) as e:
        chan.THERM_PROP_UPDATE_points(dh)
    assert e.value.code == -4 and "2 of 4096 points" in str(e.value) and "index 1234" in str(e.value)
    # the same context keeps working afterwards
    ok = chan.THERM_PROP_UPDATE_points(dh[:1000])
    want, _, _ = orc.PropTable(tab.lists).update(dh[:1000])
    assert np.array_equal(ok["T"], want["T"])


def test_table_checks(chan):
    rows, T0, tab = _tables(2048)
    bad = thermo.SplineTable(tab.lists)
    bad.lists = dict(tab.lists)
    dh = bad.lists["DH"].copy()
    dh[100] = dh[99]                                     # not strictly increasing
    bad.lists["DH"] = dh
    with pytest.raises(gpu.ChapsimError) as e:
        chan.prop_table_init(bad)
    assert e.value.code == -6
