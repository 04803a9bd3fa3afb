"""Mixed-precision periodic-channel and main-domain steps (FP32 storage and stencils / CN
sweeps, FP32 spectrum with FP32 x and z transforms; FP64 y-solve of the
Poisson modes, divergence, projection and bulk-flux sums) against the FP64
oracle and the FP64 GPU step.

Tolerances, stated against FP64:
* after 10 steps on the 64^3 channel (dt = 1e-3) u, v, w are within 1e-5
  relative (max-norm difference over max-norm) of the FP64 oracle: FP32
  round-off (~6e-8 per operation) grown over 30 substeps;
* the pressure (compared modulo its mean) within 3e-3: storing the
  projected velocity in FP32 leaves a divergence of about eps32 |u| / dx,
  which the next projection removes, so the pressure picks up a correction
  of about eps32 |u| dx / (alpha dt) per substep, largest at small dt;
* max|div u| of the stored FP32 velocity, evaluated in FP64, stays below
  1e-5 (the projection is exact in FP64; storing the corrected velocity in
  FP32 leaves eps32 * |u| / dx);
* after 200 steps the plane-averaged mean velocity profile differs from the
  FP64 GPU run by less than 1 % of the bulk velocity, and the rms profiles of
  u', v', w' by less than 1 % of their peak.
"""
import numpy as np
import pytest

from oracle import Oracle
from chapsim import gpu
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field, bulk_velocity

pytestmark = pytest.mark.gpu

C1 = dict(L=64, M=64, N=64, HX=2 * np.pi, HZ=np.pi, STR2=2.0, REN=2800.0)


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _setup():
    s = channel_setup(C1["L"], C1["M"], C1["N"], C1["HX"], C1["HZ"], C1["STR2"], C1["REN"])
    Q, PR = initial_field(s, 1973, 0.1)
    return s, Q, PR


def test_upload_download_rounds_to_fp32():
    s, Q, PR = _setup()
    c = gpu.ChannelTG(s, precision="mixed")
    c.upload(Q, PR)
    Qd, PRd = c.download()
    M = s.M
    inner = (slice(None), slice(None), slice(1, M + 1), slice(None))
    np.testing.assert_array_equal(Qd[inner][0], Q[inner][0].astype(np.float32).astype(np.float64))
    np.testing.assert_array_equal(PRd[:, 1:M + 1], PR[:, 1:M + 1].astype(np.float32).astype(np.float64))
    c.close()


def test_mixed_vs_fp64_oracle_10_steps():
    s, Q, PR = _setup()
    o = Oracle(C1["L"], C1["M"], C1["N"], C1["HX"], C1["HZ"], C1["STR2"], C1["REN"], DT0=1e-3, CFLGV=0.5, threads=8)
    o.set_fields(Q, PR)
    c = gpu.ChannelTG(s, precision="mixed")
    c.upload(Q, PR)
    c.set_dt(1e-3)
    o.set_dt(1e-3)
    o.substep(0)
    c.SOLVERRK3_MOM_tg(0)
    rc, dts = o.run_steps(10)
    assert rc == 0
    dt, _ = c.advance(10, 1e-3, 1e-6, 0.5)
    assert abs(dt - dts[-1]) <= 1e-4 * dts[-1]
    Qg, PRg = c.download()
    Qo, PRo, _ = o.get_fields()
    M = s.M
    errs = {n: rel(Qg[i][:, 1:M + 1], Qo[i][:, 1:M + 1]) for i, n in enumerate("uvw")}
    pin = PRg[:, 1:M + 1] - PRg[:, 1:M + 1].mean()
    pon = PRo[:, 1:M + 1] - PRo[:, 1:M + 1].mean()
    errs["p"] = rel(pin, pon)
    print("mixed vs FP64 oracle after 10 steps:", errs)
    for k in "uvw":
        assert errs[k] <= 1e-5, (k, errs[k])
    assert errs["p"] <= 3e-3
    div = c.DIVGCK_tg()
    print("mixed max|div u|:", div)
    assert div <= 1e-5
    ub = bulk_velocity(s, Qg)
    assert abs(ub - bulk_velocity(s, Q)) <= 1e-6


def _profiles(s, Q):
    M = s.M
    u = Q[0][:, 1:M + 1, :]
    v = 0.5 * (Q[1][:, 1:M + 1, :] + Q[1][:, 2:M + 2, :])
    w = Q[2][:, 1:M + 1, :]
    mu = u.mean(axis=(0, 2))
    rms = [np.sqrt(((f - f.mean(axis=(0, 2), keepdims=True)) ** 2).mean(axis=(0, 2))) for f in (u, v, w)]
    return mu, rms


def test_mixed_statistics_track_fp64_200_steps():
    s, Q, PR = _setup()
    runs = {}
    for prec in ("fp64", "mixed"):
        c = gpu.ChannelTG(s, precision=prec)
        c.upload(Q, PR)
        c.set_dt(1e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(200, 0.02, 1e-6, 0.5)
        runs[prec] = c.download()[0]
        c.close()
    m64, r64 = _profiles(s, runs["fp64"])
    m32, r32 = _profiles(s, runs["mixed"])
    dmean = float(np.abs(m32 - m64).max())
    drms = [float(np.abs(a - b).max() / b.max()) for a, b in zip(r32, r64)]
    print("mean-profile diff / Ub:", dmean, "rms diffs / peak:", drms)
    assert dmean <= 1e-2
    assert max(drms) <= 1e-2


# ---------------------------------------------------------------- main (IO) domain
# Mixed precision of the main-domain step: FP32 storage of the flow fields G,
# Q, PR, EXPLT0, RHS, D_STG, MU_STG, DivU (stencils and Crank-Nicolson sweeps
# evaluated from them); FP64 properties, thermal fields, Poisson solve and
# projection.  Bounds against the FP64 oracle as for the periodic channel:
# G, Q within 1e-5, P (modulo its mean) within 3e-3, the thermal fields within
# 1e-5.

def _io_errs(o, c, M):
    Gg, Qg, Pg = c.download_io()
    Go, Qo, Po = o.io_get_fields()
    errs = {}
    for i, n in enumerate("uvw"):
        errs["G" + n] = rel(Gg[i][:, 1:M + 1], Go[i][:, 1:M + 1])
        errs["Q" + n] = rel(Qg[i][:, 1:M + 1], Qo[i][:, 1:M + 1])
    pg = Pg[:, 1:M + 1] - Pg[:, 1:M + 1].mean()
    po = Po[:, 1:M + 1] - Po[:, 1:M + 1].mean()
    errs["P"] = rel(pg, po)
    return errs


@pytest.mark.parametrize("ivis", [0, 1])
def test_mixed_main_domain_tc8_five_steps(golden_dir, ivis):
    """From the reference's TC8 step-100 fields with non-uniform properties."""
    import json
    import os
    d = np.load(os.path.join(golden_dir, "tc8_step100_fields.npz"))
    cs = json.load(open(os.path.join(golden_dir, "tc8_setup.json")))["case"]
    L, M, N = cs["NCL1"], cs["NCL2"], cs["NCL3"]
    G = np.zeros((3, N, M + 2, L))
    PR = np.zeros((N, M + 2, L))
    for comp, name in enumerate(("G1", "G2", "G3")):
        G[comp, :, 1:M + 1, :] = d[name].astype(np.float64)
    PR[:, 1:M + 1, :] = d["P"].astype(np.float64)
    k, j, i = np.meshgrid(np.arange(N), np.arange(M + 2), np.arange(L), indexing="ij")
    rho = 1.0 + 0.05 * np.sin(2 * np.pi * i / L) * np.cos(2 * np.pi * k / N) + 0.02 * np.cos(np.pi * j / (M + 2))
    mu = 1.0 + 0.1 * np.cos(2 * np.pi * i / L + 0.3) * np.sin(np.pi * j / (M + 2))
    o = Oracle(L, M, N, cs["HX"], cs["HZ"], cs["STR2"], cs["REN"], iFlowDriven=cs["iFlowDriven"],
               Cf_Given=cs["Cf_Given"], DT0=cs["DT"], DTMIN=1e-6, CFLGV=cs["CFLGV"], threads=8)
    o.io_set_fields(G, PR, rho, mu, mu)
    o.io_set_vis_scheme(ivis)
    s = channel_setup(L, M, N, cs["HX"], cs["HZ"], cs["STR2"], cs["REN"], cs["iFlowDriven"], cs["Cf_Given"])
    c = gpu.ChannelIO(s, ivisscheme=ivis, precision="mixed")
    c.upload_io(G, PR, rho, mu, mu)
    c.set_dt(cs["DT"])
    assert o.io_run_steps(5)[0] == 0
    c.advance(5, cs["DT"], 1e-6, cs["CFLGV"])
    errs = _io_errs(o, c, M)
    print("mixed main domain (TC8, iVisScheme %d) vs FP64 oracle:" % ivis, errs)
    for k2, v in errs.items():
        assert v <= (3e-3 if k2 == "P" else 1e-5), (k2, v)
    assert c.DIVGCK_io() <= 1e-4


def test_mixed_heated_channel_cn_five_steps():
    import oracle as orc
    from chapsim import thermo
    L, M, N, qw = 64, 64, 32, 0.5
    HX, HZ, STR2, REN = 2 * np.pi, np.pi, 2.0, 2800.0
    s = channel_setup(L, M, N, HX, HZ, STR2, REN)
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / REN / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((N, M + 2, L))
    DH[:, 1:M + 1, :] = 1e-2 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L))
    ones = np.ones((N, M + 2, L))
    o = Oracle(L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=8)
    o.io_set_fields(Q, PR, ones, ones, ones)
    o.io_set_vis_scheme(1)
    o.thermal_enable(orc.PropTable(tab.lists), DH, qw, qw, cthecd)
    o.set_dt(1e-3)
    c = gpu.ChannelIO(s, ivisscheme=1, precision="mixed")
    c.upload_io(Q, PR, ones, ones, ones)
    c.thermal_init(tab, DH, qw, qw, cthecd)
    c.set_dt(1e-3)
    assert o.io_run_steps(5)[0] == 0
    c.advance(5, 1e-3, 1e-6, 0.5)
    errs = _io_errs(o, c, M)
    tg, to = c.download_thermal(), o.thermal_get()
    for k2 in ("DH", "T", "D", "M"):
        errs[k2] = rel(tg[k2], to[k2])
    print("mixed heated channel (CN) vs FP64 oracle:", errs)
    for k2, v in errs.items():
        assert v <= (3e-3 if k2 == "P" else 1e-5), (k2, v)

