"""Mixed-precision periodic-channel step (FP32 storage and stencils / CN
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


def test_mixed_rejected_for_io_domain():
    s, _, _ = _setup()
    with pytest.raises(gpu.ChapsimError) as e:
        gpu.ChannelIO(s, precision="mixed")
    assert e.value.code == -6
