"""Dynamic pin of the oracle against the reference's own run.

TC8 (64^3 channel, main domain, explicit viscous terms, thermal solver not yet
active, DT = 1e-3) is restarted from the reference's step-100 fields and
advanced 19 steps.  The monitor columns that follow from the instantaneous
fields (CFL, centreline mean u, u'u', u'v', max of the mean mass-flux
profile) must equal the reference's log rows 101-119 to every printed digit
(monitor.io.2020.1217.1640.log, written by PP_MONITOR_Xperiodic_io,
src/processing/PP_SCN_MONITOR.f90:610-613).  The MaxDiv column (DIVGCK_io) is
round-off, 1.1e-14 to 1.4e-14 in the log; the oracle's must stay within twice
the logged value of each row."""
import json
import os

import numpy as np
import pytest

from oracle import Oracle


def _half_ulp(v, kind):
    if kind == "F9.5":
        return 0.5e-5 * 1.0001
    e = np.floor(np.log10(abs(v))) if v != 0 else 0.0
    return 0.5 * 10.0 ** (e - 5) * 1.0001  # ES13.5: 6 significant digits


@pytest.fixture(scope="module")
def tc8(golden_dir):
    d = np.load(os.path.join(golden_dir, "tc8_step100_fields.npz"))
    case = json.load(open(os.path.join(golden_dir, "tc8_setup.json")))["case"]
    mon = json.load(open(os.path.join(golden_dir, "tc8_monitor.json")))
    return d, case, mon


def test_tc8_restart_reproduces_monitor_rows_101_119(tc8):
    d, c, mon = tc8
    cols = mon["columns"]
    rows = {int(r[0]): r for r in mon["rows"]}
    L, M, N = c["NCL1"], c["NCL2"], c["NCL3"]
    o = Oracle(L, M, N, c["HX"], c["HZ"], c["STR2"], c["REN"], iFlowDriven=c["iFlowDriven"], Cf_Given=c["Cf_Given"],
               DT0=c["DT"], DTMIN=1e-6, CFLGV=c["CFLGV"], threads=os.cpu_count() or 1)
    G = np.zeros((3, N, M + 2, L))
    PR = np.zeros((N, M + 2, L))
    for comp, name in enumerate(("G1", "G2", "G3")):
        G[comp, :, 1:M + 1, :] = d[name].astype(np.float64)
    PR[:, 1:M + 1, :] = d["P"].astype(np.float64)
    # thermal solver inactive (t < timeThermoStart): uniform properties;
    # Viscousity0 keeps its allocation value 1 (src/MEMALLOCT.f90:199)
    rho = np.full((N, M + 2, L), float(d["D"]))
    o.io_set_fields(G, PR, rho, np.ones_like(rho), np.full_like(rho, float(d["M"])))
    m = o.io_monitor()
    r = rows[100]
    assert abs(m["Uc"] - r[cols.index("Uc")]) <= _half_ulp(r[cols.index("Uc")], "ES")
    checked = 0
    for step in range(101, 120):
        rc, cfl_dt = o.io_run_steps(1)
        assert rc == 0
        m = o.io_monitor()
        r = rows[step]
        pairs = [(cfl_dt[0], "CFL", "F9.5"), (m["Uc"], "Uc", "ES"), (m["UUc"], "UUc", "ES"), (m["UVc"], "UVc", "ES"),
                 (m["Gmaxx"], "Gmaxx", "F9.5")]
        for val, name, kind in pairs:
            ref = r[cols.index(name)]
            assert abs(val - ref) <= _half_ulp(ref, kind), (step, name, val, ref)
            checked += 1
        assert o.io_divgck() <= 2.0 * r[cols.index("MaxDiv")], (step, o.io_divgck())
    assert checked == 19 * 5
