"""Extract golden vectors from the reference's shipped outputs into small fixtures.

Run where a reference checkout exists, with its path in the environment
variable ``CHAPSIM_REFERENCE``.  The tests never read the reference tree: they
read only the fixtures this script writes.

Sources (all produced by the reference solver itself):
  test_cases_template/TC8_Channel_IO_thermal_LiquidWater/0_log_monitors/
    CHK_COORD_YND.dat      -- COORDJR (src/COORDJR.f90:301-311)
    CHK_COEF_YCL2ND.dat    -- MESH_YWEIGHT_FACTORS (src/COORDJR.f90:454-462)
    CHK_COEF_TDMA.dat      -- TDMA_COEF (src/TDMA_COEF.f90:287-330)
    CHK_INIL_Poiseuille.dat-- LAMPOISLPROF (src/LAMPOISLPROF.f90:63-69)
    CHK_COORD_XND/ZND.dat  -- COORDJR (src/COORDJR.f90:269-328)
    monitor.io.2020.1217.1640.log -- per-step monitor rows (PP_SCN_MONITOR)
  test_cases_template/TC8_.../readdata.ini -- the case parameters
  test_cases_template/TC4_Channel_IO_thermal_ScpWater/NIST_WATER_23.5MP.DAT
                         -- the property table read by the table path
                            (src/thermo_properties_table_searching.f90:1261),
                            every 6th row kept (nist_water_rows.npz)
"""
import json
import os
import re

import numpy as np

REF = os.environ.get("CHAPSIM_REFERENCE", "")
TC8 = os.path.join(REF, "test_cases_template", "TC8_Channel_IO_thermal_LiquidWater")
MON = os.path.join(TC8, "0_log_monitors")
NIST = os.path.join(REF, "test_cases_template", "TC4_Channel_IO_thermal_ScpWater", "NIST_WATER_23.5MP.DAT")
OUT = os.path.dirname(os.path.abspath(__file__))
NIST_STRIDE = 6


def write_nist():
    """Every NIST_STRIDE-th row of the reference's NIST water table (file order), float64."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(OUT)), "chapsim1.0_b200"))
    from chapsim import thermo
    rows = thermo.read_table(NIST)
    np.savez_compressed(os.path.join(OUT, "nist_water_rows.npz"), rows=rows[::NIST_STRIDE],
                        n_full=np.int64(rows.shape[0]), stride=np.int64(NIST_STRIDE))
    print("wrote", os.path.join(OUT, "nist_water_rows.npz"))


def _rows(path, ncols=None):
    rows = []
    for line in open(path):
        s = line.strip()
        if not s or s.startswith("#") or re.match(r"^[A-Za-z]", s):
            continue
        vals = [float(v.replace("D", "E")) for v in s.split()]
        if ncols is None or len(vals) == ncols:
            rows.append(vals)
    return rows


def _blocks_tdma(path):
    blocks, cur = [], None
    for line in open(path):
        s = line.strip()
        if s.startswith("#"):
            cur = []
            blocks.append(cur)
            continue
        if s:
            cur.append([float(v) for v in s.split()])
    return [np.array(b) for b in blocks]


def main():
    if not REF or not os.path.isdir(REF):
        raise SystemExit("set CHAPSIM_REFERENCE to the reference checkout")
    write_nist()
    fx = {}
    # CHK_COORD_YND: first block JND YND 1/DYCI YND+ ; second block JCL YCC 1/DYFI DYC+
    lines = open(os.path.join(MON, "CHK_COORD_YND.dat")).read().split("# JCL")
    nd = np.array(_rows_text(lines[0]))
    cl = np.array(_rows_text(lines[1]))
    fx["YND"] = nd[:, 1].tolist()
    fx["inv_DYCI"] = nd[:, 2].tolist()
    fx["YCC"] = cl[:, 1].tolist()
    fx["inv_DYFI"] = cl[:, 2].tolist()
    yc = np.array(_rows(os.path.join(MON, "CHK_COEF_YCL2ND.dat"), 4))
    fx["DYCI"] = yc[:, 1].tolist()
    fx["WFF"] = yc[:, 2].tolist()
    fx["WFB"] = yc[:, 3].tolist()
    b = _blocks_tdma(os.path.join(MON, "CHK_COEF_TDMA.dat"))
    fx["AMPH"], fx["ACPH"], fx["APPH"] = (b[0][:, c].tolist() for c in range(3))
    for idr in (1, 2, 3):
        fx[f"AMVR{idr}"], fx[f"ACVR{idr}"], fx[f"APVR{idr}"] = (b[idr][:, c].tolist() for c in range(3))
    ps = np.array(_rows(os.path.join(MON, "CHK_INIL_Poiseuille.dat"), 3))
    fx["Vini"] = ps[:, 2].tolist()
    zn = np.array(_rows(os.path.join(MON, "CHK_COORD_ZND.dat"), 2))
    fx["ZND"] = zn[:, 1].tolist()
    xn = np.array(_rows(os.path.join(MON, "CHK_COORD_XND.dat"), 2))
    fx["XND"] = xn[:, 1].tolist()
    ini = open(os.path.join(TC8, "readdata.ini")).read()

    def g(key):
        m = re.search(r"^" + key + r"=\s*([^\n#]+)", ini, re.M)
        return m.group(1).strip()

    fx["case"] = {
        "NCL1": int(g("NCL1_io")), "NCL2": int(g("NCL2")), "NCL3": int(g("NCL3")),
        "HX": float(g("HX_io")), "HZ": float(g("HZ")), "STR2": float(g("STR2")), "REN": float(g("REN")),
        "iFlowDriven": int(g("iFlowDriven")), "Cf_Given": float(g("Cf_Given")), "DT": float(g("DT")),
        "CFLGV": float(g("CFLGV")),
    }
    fx["printed_digits"] = {"CHK_COEF_TDMA": 8, "CHK_COORD_YND": 8, "CHK_COEF_YCL2ND": 6, "CHK_INIL_Poiseuille": 8}
    with open(os.path.join(OUT, "tc8_setup.json"), "w") as f:
        json.dump(fx, f, indent=0)
    # monitor rows (instantaneous columns), for the trajectory pin of the IO path
    cols = ["STEP", "PhyT", "CpuT", "CFL", "DT", "MaxDiv", "Uc", "Uct", "UUc", "UUct", "UVc", "UVct",
            "Cf_B", "Cf_Bt", "Cf_T", "Cf_Tt", "Gmean", "Gmaxx"]
    rows = []
    for line in open(os.path.join(MON, "monitor.io.2020.1217.1640.log")):
        s = line.split()
        if s and s[0].isdigit():
            rows.append([float(v) for v in s[: len(cols)]])
    with open(os.path.join(OUT, "tc8_monitor.json"), "w") as f:
        json.dump({"columns": cols, "rows": rows}, f)
    # step-100 restart fields of the same run (rho*u, rho*v, rho*w and p; the
    # thermal solver is not active yet, so D and M are uniform and stored as
    # scalars).  float32 keeps the fixture small; the monitor columns are
    # printed to 5-6 digits, far above the 1e-8 perturbation this introduces.
    raw = os.path.join(TC8, "1_instant_rawdata")
    fields = {}
    hdr = None
    for name in ("U", "V", "W", "P", "D", "M"):
        b = open(os.path.join(raw, f"DNS_perixz_INSTANT_T1.000000000E-01_{name}.D"), "rb").read()
        h = np.frombuffer(b[:16], "<i4")
        hdr = (h.tolist(), np.frombuffer(b[16:40], "<f8").tolist())
        L, M, N = (int(x) for x in h[:3])
        f = np.frombuffer(b[40:], "<f8").reshape(N, M, L)
        fields[name] = f
    np.savez_compressed(os.path.join(OUT, "tc8_step100_fields.npz"),
                        G1=fields["U"].astype(np.float32), G2=fields["V"].astype(np.float32),
                        G3=fields["W"].astype(np.float32), P=fields["P"].astype(np.float32),
                        D=np.float64(fields["D"].mean()), M=np.float64(fields["M"].mean()),
                        D_ptp=np.float64(np.ptp(fields["D"])), M_ptp=np.float64(np.ptp(fields["M"])),
                        header_int=np.array(hdr[0]), header_real=np.array(hdr[1]))
    print("wrote", os.path.join(OUT, "tc8_setup.json"), "tc8_monitor.json and tc8_step100_fields.npz")


def _rows_text(text):
    rows = []
    for line in text.splitlines():
        s = line.strip()
        if not s or s.startswith("#") or s.startswith(","):
            continue
        try:
            rows.append([float(v) for v in s.split()])
        except ValueError:
            continue
    return rows


if __name__ == "__main__":
    main()
