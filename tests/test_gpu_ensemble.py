"""Ensembles of uneven periodic channels and the y-solve autotuner.

* The Poisson y-solve variants (warp Thomas/PCR hybrid, sequential
  Thomas, two-way elimination, warp affine scans over the sequential factors)
  and the three forms of the right-hand-side / x-sweep stage (fused, split,
  fused with bulk-copy staging) solve the FFT99 problem to 1e-12 of the
  oracle, and the step with any combination, with chained or fused plane
  transforms, stays within 1e-11 after 10 steps.  The bulk-staged form computes the same per-point arithmetic as the
  fused one (only the bulk-flux sum is added in another order), checked at
  other line lengths and in mixed precision.
* An ensemble (one graph per step, one branch per member) advances every
  member exactly as its own graph does: fields bitwise equal.
"""
import math

import numpy as np
import pytest

from oracle import Oracle
from chapsim import gpu
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4, 5, 8, 9, 12, 13, 16, 20, 24, 28, 64, 68, 72])
def test_ysolve_variants_match_oracle(kind):
    L, M, N = 96, 64, 64
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    c = gpu.ChannelTG(s)
    choice, ms = c.autotune(force=kind)
    assert choice == kind and min(ms.values()) > 0
    rhs = np.random.default_rng(3).standard_normal((N, M, L))
    full = np.zeros((N, M + 2, L))
    full[:, 1:M + 1, :] = rhs
    ref = o.poisson(full)
    got = c.FFT99_POIS3D_periodicxz(rhs)
    assert rel(got[:, 1:M + 1], ref[:, 1:M + 1]) <= 1e-12
    Q, PR = initial_field(s, 1973, 0.1)
    o.set_fields(Q, PR)
    c.upload(Q, PR)
    o.set_dt(2e-3)
    c.set_dt(2e-3)
    o.substep(0)
    c.SOLVERRK3_MOM_tg(0)
    o2 = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0, DT0=2e-3, threads=8)
    Qo, PRo, H0o = o.get_fields()
    o2.set_fields(Qo, PRo, H0o)
    o2.set_dt(2e-3)
    o2.run_steps(10)
    c.advance(10, 2e-3, 1e-6, 0.5)
    Qg, PRg, H0g = c.download(want_h0=True)
    Qo, PRo, H0o = o2.get_fields()
    for i in range(3):
        assert rel(Qg[i][:, 1:M + 1], Qo[i][:, 1:M + 1]) <= 1e-11
    assert rel(PRg[:, 1:M + 1], PRo[:, 1:M + 1]) <= 1e-11
    assert rel(H0g, H0o[:, :, 1:M + 1, :]) <= 1e-11
    c.close()


@pytest.mark.parametrize("shape,precision,tol", [((384, 32, 32), "fp64", 1e-12), ((128, 64, 32), "fp64", 1e-12),
                                                 ((32, 32, 32), "fp64", 1e-12), ((256, 64, 32), "mixed", 1e-5)])
def test_bulk_staged_rhs_matches_fused(shape, precision, tol):
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 77, 0.1)
    out = []
    for kind in (0, 4):
        c = gpu.ChannelTG(s, precision=precision)
        choice, _ = c.autotune(force=kind)
        assert choice == kind
        c.upload(Q, PR)
        c.set_dt(2e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(5, 2e-3, 1e-6, 0.5)
        out.append(c.download()[0])
        c.close()
    for i in range(3):
        e = rel(out[1][i][:, 1:M + 1], out[0][i][:, 1:M + 1])
        assert e <= tol, (i, e)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sequential_ysolve_in_shared_memory_at_one_block(precision):
    """Lines of 256 rows: the sequential y-solve's forward intermediate does
    not fit two blocks per SM, so the fourth variant (bit 5) keeps it in
    shared memory at one block per SM.  The same recurrence as the sequential
    variant with the intermediate in global memory: bitwise equal fields, and
    the Poisson solve within 1e-12 of the oracle."""
    L, M, N = 64, 256, 64
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    if precision == "fp64":
        o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
        c = gpu.ChannelTG(s)
        choice, ms = c.autotune(force=32)
        assert choice == 32 and ms["ysolve_sequential_smem"] < 1e29
        rhs = np.random.default_rng(9).standard_normal((N, M, L))
        full = np.zeros((N, M + 2, L))
        full[:, 1:M + 1, :] = rhs
        ref = o.poisson(full)
        got = c.FFT99_POIS3D_periodicxz(rhs)
        assert rel(got[:, 1:M + 1], ref[:, 1:M + 1]) <= 1e-12
        c.close()
    Q, PR = initial_field(s, 13, 0.1)
    out = []
    for force in (1, 32):
        c = gpu.ChannelTG(s, precision=precision)
        assert c.autotune(force=force)[0] == force
        c.upload(Q, PR)
        c.set_dt(2e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(3, 2e-3, 1e-6, 0.5)
        out.append(c.download())
        c.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("shape", [(64, 32, 64), (128, 128, 128), (32, 256, 32)])
def test_two_way_ysolve_matches_oracle(shape):
    """The two-way y-solve (two threads per mode line meeting at the middle
    row) solves the FFT99 problem to 1e-12 of the oracle for line lengths
    32, 128 and 256, the zero mode included; in the mixed-precision step it
    gives the sequential variant's fields to the FP32 bound."""
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    c = gpu.ChannelTG(s)
    choice, ms = c.autotune(force=16)
    assert choice == 16 and ms["ysolve_two_way"] > 0
    rhs = np.random.default_rng(7).standard_normal((N, M, L))
    full = np.zeros((N, M + 2, L))
    full[:, 1:M + 1, :] = rhs
    ref = o.poisson(full)
    got = c.FFT99_POIS3D_periodicxz(rhs)
    assert rel(got[:, 1:M + 1], ref[:, 1:M + 1]) <= 1e-12
    c.close()
    Q, PR = initial_field(s, 5, 0.1)
    out = []
    for force in (1, 16):
        c = gpu.ChannelTG(s, precision="mixed")
        assert c.autotune(force=force)[0] == force
        c.upload(Q, PR)
        c.set_dt(2e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(5, 2e-3, 1e-6, 0.5)
        out.append(c.download()[0])
        c.close()
    for i in range(3):
        assert rel(out[1][i][:, 1:M + 1], out[0][i][:, 1:M + 1]) <= 1e-5


@pytest.mark.parametrize("shape,precision,tol", [((128, 128, 128), "fp64", 1e-12), ((64, 64, 64), "fp64", 1e-12),
                                                 ((192, 32, 128), "fp64", 1e-12), ((96, 64, 192), "fp64", 1e-12),
                                                 ((128, 64, 192), "mixed", 1e-5), ((192, 32, 192), "mixed", 1e-5),
                                                 ((384, 32, 384), "fp64", 1e-12), ((384, 32, 384), "mixed", 1e-5),
                                                 ((256, 64, 384), "fp64", 1e-12), ((384, 32, 256), "mixed", 1e-5),
                                                 ((256, 32, 256), "fp64", 1e-12)])
def test_plane_transforms_match_chained(shape, precision, tol):
    """The fused plane transforms (one block per y row, or a thread-block
    cluster per row where the plane does not fit one block: divergence, x
    and z transforms, and their inverses) advance the channel as the chained
    transforms do, to round-off (only the pairing of real lines differs)."""
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 91, 0.1)
    out = []
    for kind in (0, 8):
        c = gpu.ChannelTG(s, precision=precision)
        choice, ms = c.autotune(force=kind)
        assert choice == kind and ms["pressure_plane"] < 1e29
        c.upload(Q, PR)
        c.set_dt(2e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(5, 2e-3, 1e-6, 0.5)
        out.append(c.download())
        c.close()
    for i in range(3):
        e = rel(out[1][0][i][:, 1:M + 1], out[0][0][i][:, 1:M + 1])
        assert e <= tol, (i, e)
    pa = out[1][1][:, 1:M + 1] - out[1][1][:, 1:M + 1].mean()
    pb = out[0][1][:, 1:M + 1] - out[0][1][:, 1:M + 1].mean()
    assert rel(pa, pb) <= (1e-11 if precision == "fp64" else 1e-3)


def test_plane_transforms_refused_where_the_plane_does_not_fit():
    """A 192 x 192 FP64 plane (97 z lines of 205 complex words, 318 KB)
    exceeds one block's shared memory: forcing bit 3 keeps the chained
    transforms (in mixed precision the same plane, 159 KB, fits)."""
    s = channel_setup(192, 32, 192, 2 * math.pi, math.pi, 2.0, 2800.0)
    c = gpu.ChannelTG(s)
    choice, ms = c.autotune(force=8)
    assert choice == 0 and ms["pressure_plane"] >= 1e29
    c.close()


GRIDS = [(64, 64, 64, 2 * math.pi, math.pi, 2800.0), (96, 64, 96, 2 * math.pi, math.pi, 4000.0),
         (128, 96, 64, 4 * math.pi, 2 * math.pi / 3, 5000.0), (64, 128, 96, 2 * math.pi, math.pi, 6875.0)]


def _member(k, g, precision="fp64"):
    L, M, N, HX, HZ, REN = g
    s = channel_setup(L, M, N, HX, HZ, 2.0, REN)
    Q, PR = initial_field(s, 100 + k, 0.1)
    c = gpu.ChannelTG(s, precision=precision)
    c.upload(Q, PR)
    c.set_dt(1e-3)
    c.SOLVERRK3_MOM_tg(0)
    return c


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_equals_individual_runs(precision):
    solo = [_member(k, g, precision) for k, g in enumerate(GRIDS)]
    grp = [_member(k, g, precision) for k, g in enumerate(GRIDS)]
    for c in solo:
        c.advance(6, 0.02, 1e-6, 0.5)
    ens = gpu.Ensemble(grp)
    ens.advance(6, 0.02, 1e-6, 0.5)
    for a, b in zip(solo, grp):
        Qa, Pa = a.download()
        Qb, Pb = b.download()
        assert np.array_equal(Qa, Qb) and np.array_equal(Pa, Pb)
        assert a.get_dt() == b.get_dt()
    ens.close()
    for c in solo + grp:
        c.close()


@pytest.mark.parametrize("shape", [(64, 32, 64), (96, 96, 64), (32, 256, 32), (32, 384, 32), (64, 64, 96)])
def test_scan_ysolve_matches_oracle(shape):
    """The scan y-solve (one warp per mode line; the sequential recurrence's
    forward and backward sweeps as affine maps composed over the lanes, then
    each lane's rows recomputed in the reference's order from its incoming
    value) solves the FFT99 problem to 1e-12 of the oracle for line lengths
    32 to 384 (one to twelve rows per lane), the pinned zero mode included;
    in the mixed-precision step it gives the sequential variant's fields to
    the FP32 bound."""
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    o = Oracle(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    c = gpu.ChannelTG(s)
    choice, ms = c.autotune(force=64)
    assert choice == 64 and 0 < ms["ysolve_scan"] < 1e29
    rhs = np.random.default_rng(17).standard_normal((N, M, L))
    full = np.zeros((N, M + 2, L))
    full[:, 1:M + 1, :] = rhs
    ref = o.poisson(full)
    got = c.FFT99_POIS3D_periodicxz(rhs)
    assert rel(got[:, 1:M + 1], ref[:, 1:M + 1]) <= 1e-12
    c.close()
    Q, PR = initial_field(s, 23, 0.1)
    out = []
    for force in (1, 64):
        c = gpu.ChannelTG(s, precision="mixed")
        assert c.autotune(force=force)[0] == force
        c.upload(Q, PR)
        c.set_dt(2e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(5, 2e-3, 1e-6, 0.5)
        out.append(c.download()[0])
        c.close()
    for i in range(3):
        assert rel(out[1][i][:, 1:M + 1], out[0][i][:, 1:M + 1]) <= 1e-5


@pytest.mark.parametrize("shape,precision", [((64, 32, 192), "fp64"), ((64, 32, 384), "fp64"),
                                             ((64, 64, 128), "mixed"), ((32, 32, 384), "mixed")])
def test_zsweep_tile_widths_bitwise(shape, precision):
    """The z sweep's tile shape (32 or 16 x lines per tile, bit 8) and layout
    (lines contiguous or interleaved in pairs, bit 10), and the y sweep's
    layout (bit 11) change only which block solves a line and where it is
    staged: the fields after 3 steps are bitwise equal, and the tuner times
    every form (restoring Q after the y-sweep trials)."""
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 29, 0.1)
    out = []
    for force in (0, 256, 1024, 1280, 2048, 3328):
        c = gpu.ChannelTG(s, precision=precision)
        choice, ms = c.autotune(force=force)
        assert choice == force and min(ms[k] for k in ("zsweep_tile32", "zsweep_tile16", "zsweep_tile32_pairs",
                                                       "zsweep_tile16_pairs", "ysweep_lines", "ysweep_pairs")) > 0
        c.upload(Q, PR)
        c.set_dt(2e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(3, 2e-3, 1e-6, 0.5)
        out.append(c.download())
        c.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])


@pytest.mark.parametrize("shape,precision", [((64, 32, 384), "fp64"), ((64, 64, 256), "fp64"), ((96, 32, 96), "fp64"),
                                             ((64, 32, 384), "mixed"), ((64, 64, 128), "mixed")])
def test_pipelined_z_transforms_bitwise(shape, precision):
    """The persistent double-buffered z transforms (bit 9) and the z transforms
    with wave-ahead L2 requests (bit 12) compute each line as the one-tile
    kernel does: fields bitwise equal after 3 steps."""
    L, M, N = shape
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 31, 0.1)
    out = []
    for force in (1, 513, 4097):
        c = gpu.ChannelTG(s, precision=precision)
        choice, ms = c.autotune(force=force)
        assert choice == force and ms["pressure_chained_zpipe"] > 0 and ms["pressure_chained_zprefetch"] > 0
        c.upload(Q, PR)
        c.set_dt(2e-3)
        c.SOLVERRK3_MOM_tg(0)
        c.advance(3, 2e-3, 1e-6, 0.5)
        out.append(c.download())
        c.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])
