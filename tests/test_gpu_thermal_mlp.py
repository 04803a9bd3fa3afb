"""Heated channel with the learned property model in the thermal step.

The model is trained on the table knots of its range plus rho*h samples
drawn from the solver's own running fields, then replaces the interior
property update.  The judge (table search on the same rho*h) runs every 5
steps; its error must stay within the model's stated bound (2 % of
max(|value|, output scale)).  Against a table-search run from the same start,
the temperature and density fields stay within 1 % after 10
steps (differences over the fields' magnitude: the temperature varies by only
~1e-4 across the channel this early).  The step times of both runs are printed: the comparison of what the
model gains over the table search (on the GPU the table search is already
cheap; see the bench for the full-size numbers).
"""
import math
import time

import numpy as np
import pytest

from chapsim import gpu, thermo
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

pytestmark = pytest.mark.gpu

SCHEDULE = [(8000, 3e-3), (8000, 1e-3), (8000, 3e-4), (4000, 1e-4)]
BOUND = 2e-2


def _channel(s, Q, PR, tab, DH, qw, cthecd):
    ones = np.ones((s.N, s.M + 2, s.L))
    c = gpu.ChannelIO(s)
    c.upload_io(Q, PR, ones, ones, ones)
    c.thermal_init(tab, DH, qw, qw, cthecd)
    c.set_dt(1e-3)
    return c


@pytest.mark.parametrize("act", [gpu.MLP_TANH, gpu.MLP_CUBIC])
def test_thermal_step_with_learned_properties(act):
    L, M, N = 64, 64, 32
    s = channel_setup(L, M, N, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 1973, 0.1)
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    cthecd = 1.0 / 2800.0 / (tab.ref["M0"] * tab.ref["CP0"] / tab.ref["K0"])
    DH = np.zeros((N, M + 2, L))
    DH[:, 1:M + 1, :] = 1e-3 * np.random.default_rng(5).uniform(-1.0, 1.0, (N, M, L))
    qw = 2.0
    ref = _channel(s, Q, PR, tab, DH, qw, cthecd)
    ml = _channel(s, Q, PR, tab, DH, qw, cthecd)
    # samples from the running solver: rho*h after a few table-search steps
    probe = _channel(s, Q, PR, tab, DH, qw, cthecd)
    probe.advance(20, 1e-3, 1e-6, 0.5)
    field = probe.download_thermal()["DH"][:, 1:M + 1]
    probe.close()
    dh = tab.lists["DH"]
    lo = float(dh[0] + 0.02 * (dh[-1] - dh[0]))
    hi = float(dh[-1] - 0.02 * (dh[-1] - dh[0]))
    ml.mlp_init(lo, hi, seed=11)
    ml.mlp_set_activation(act)
    samples = np.random.default_rng(6).choice(field.reshape(-1), 4000, replace=False)
    knots = dh[(dh >= lo) & (dh <= hi)]
    train = np.concatenate([knots, samples, np.random.default_rng(7).uniform(lo, hi, 2000)])
    for it, lr in SCHEDULE:
        loss = ml.mlp_train(train, it, lr=lr)
    print("training loss", loss)
    ml.thermal_use_mlp(True)
    times = {}
    for name, c in (("table", ref), ("mlp", ml)):
        c.sync()
        t0 = time.perf_counter()
        for blk in range(2):
            c.advance(5, 1e-3, 1e-6, 0.5)
            if name == "mlp":
                err = c.mlp_judge()
                print("judge after", 5 * (blk + 1), "steps:", err)
                assert max(err.values()) <= BOUND, err
        c.sync()
        times[name] = (time.perf_counter() - t0) / 10
    print("wall time per step: table %.3f ms, model %.3f ms" % (1e3 * times["table"], 1e3 * times["mlp"]))
    a, b = ref.download_thermal(), ml.download_thermal()
    for k in ("T", "D"):
        x, y = a[k][:, 1:M + 1], b[k][:, 1:M + 1]
        e = np.abs(x - y).max() / np.abs(x).max()
        print(k, "field difference / magnitude", e)
        assert e <= 1e-2, (k, e)
    ga, _, _ = ref.download_io()
    gb, _, _ = ml.download_io()
    assert np.abs(ga - gb).max() <= 1e-3 * np.abs(ga).max()
    ref.close()
    ml.close()
