"""Asynchronous field dumps in the reference's .D format and restarts from
them (WRT_INSTANT_VARS_TG / _FLOW_IO / _THERMAL_IO, ReStart_INSTANT_VARS_TG).

* A dump taken between steps holds the fields of that moment, bitwise, even
  when the caller writes the files after further steps: the snapshot is in
  stream order and the copy to the host overlaps the later steps.  Header:
  {L, M, N, ITERG}, {PhyTIME, REN, DT} with DT the device dt at the snapshot.
* Mixed precision: the files hold the FP32 fields widened to FP64.
* Thermal main domain: nine files, U V W P and T D H M K.
* A context restarted from the files advances exactly as the original one
  (bitwise): the first RK3 substep does not read CONVH0, and the file's DT
  seeds the dt rule.
"""
import math

import numpy as np
import pytest

from chapsim import gpu, thermo
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field, read_dfile

pytestmark = pytest.mark.gpu


def _tg(precision="fp64", shape=(64, 64, 32)):
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 11, 0.1)
    c = gpu.ChannelTG(s, precision=precision)
    c.upload(Q, PR)
    c.set_dt(1e-3)
    c.SOLVERRK3_MOM_tg(0)
    return s, c


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dump_holds_the_fields_of_its_moment(tmp_path, precision):
    s, c = _tg(precision)
    M = s.M
    c.advance(3, 0.02, 1e-6, 0.5)
    c.dump_begin()
    Q3, P3 = c.download()           # stream order: after the snapshot, before the next steps
    dt3 = c.get_dt()
    c.advance(4, 0.02, 1e-6, 0.5)   # the copy to the host overlaps these steps
    dt = c.dump_write(str(tmp_path / "DNS_perixz_INSTANT_T"), 3, 0.125, 2800.0)
    assert dt == dt3
    stem = tmp_path / ("DNS_perixz_INSTANT_T" + gpu.es15_9(0.125))
    for comp, x in enumerate("UVWP"):
        f, h = read_dfile(f"{stem}_{x}.D")
        ref = (Q3[comp] if comp < 3 else P3)[:, 1:M + 1, :]
        assert np.array_equal(f, ref), x
        assert (h["L"], h["M"], h["N"], h["ITERG"]) == (s.L, s.M, s.N, 3)
        assert (h["time"], h["REN"], h["DT"]) == (0.125, 2800.0, dt3)
    # the later steps really moved on
    Q7, _ = c.download()
    assert not np.array_equal(Q7[0], Q3[0])
    c.close()


def test_restart_from_dump_continues_bitwise(tmp_path):
    s, c = _tg()
    c.advance(4, 0.02, 1e-6, 0.5)
    stem = c.WRT_INSTANT_VARS(str(tmp_path) + "/", 4, 0.5, 2800.0)
    c.advance(5, 0.02, 1e-6, 0.5)
    Qa, Pa = c.download()
    r = gpu.ChannelTG(s)
    hdr = r.restart_from_dfiles(stem)
    assert hdr["ITERG"] == 4
    r.advance(5, 0.02, 1e-6, 0.5)
    Qb, Pb = r.download()
    M = s.M
    assert np.array_equal(Qa[:, :, 1:M + 1], Qb[:, :, 1:M + 1])
    assert np.array_equal(Pa[:, 1:M + 1], Pb[:, 1:M + 1])
    assert c.get_dt() == r.get_dt()
    c.close()
    r.close()


def test_restart_rejects_other_grids(tmp_path):
    s, c = _tg()
    stem = c.WRT_INSTANT_VARS(str(tmp_path) + "/", 0, 0.0, 2800.0)
    s2 = channel_setup(64, 64, 64, 2 * math.pi, math.pi, 2.0, 2800.0)
    r = gpu.ChannelTG(s2)
    with pytest.raises(ValueError):
        r.restart_from_dfiles(stem)
    with pytest.raises(gpu.ChapsimError):
        r.dump_write(str(tmp_path / "x"), 0, 0.0, 1.0)  # no dump in flight
    c.close()
    r.close()


def test_thermal_dump_writes_nine_files(tmp_path):
    L, M, N = 64, 64, 32
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / 2800.0 / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((N, M + 2, L))
    DH[:, 1:M + 1, :] = 1e-3 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L))
    ones = np.ones((N, M + 2, L))
    c = gpu.ChannelIO(s)
    c.upload_io(Q, PR, ones, ones, ones)
    c.thermal_init(tab, DH, 0.5, 0.5, cthecd)
    c.set_dt(1e-3)
    c.advance(2, 1e-3, 1e-6, 0.5)
    stem = c.WRT_INSTANT_VARS(str(tmp_path) + "/", 2, 0.002, 2800.0)
    tg = c.download_thermal()
    _, Qd, Pd = c.download_io()
    want = {"U": Qd[0], "V": Qd[1], "W": Qd[2], "P": Pd, "T": tg["T"], "D": tg["D"], "H": tg["H"], "M": tg["M"],
            "K": tg["K"]}
    for x, ref in want.items():
        f, h = read_dfile(f"{stem}_{x}.D")
        assert np.array_equal(f, ref[:, 1:M + 1, :]), x
    c.close()
