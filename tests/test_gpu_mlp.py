"""Learned property model on the GPU (tcgen05 layers with 16-bit operands,
FP32 accumulation) against the CPU oracle of the same network, and against
the table search it replaces.

* forward: model outputs for the same parameters agree with the oracle to
  1e-2 of each output's scale.  Inference takes the hardware tanh on FP16
  pairs (tanh.approx.f16x2) where the oracle takes libm's tanhf between the
  same FP16 roundings of the activation's input and result; both multiply
  the FP16 activations by the FP16-rounded weights.  The hardware
  approximation of the untrained network's 128 activations per point adds
  up to a few 1e-3 of an output's scale (6e-3 measured with BF16 operands);
  a layout or indexing fault would show as errors of order 1.  The trained
  model's accuracy is held to its own bound below;
* gradients of one pass agree with the oracle to 1e-2 of the largest entry
  of each parameter group (FP32 atomics and accumulation order vs FP64);
* outside the trained range the result is the table search, bitwise;
* after training, the judge's error stays below the bound stated in
  test_trained_model_accuracy.
"""
import numpy as np
import pytest

import oracle as orc
from chapsim import gpu, thermo
from chapsim.mesh import channel_setup

pytestmark = pytest.mark.gpu

FIELDS = ("H", "T", "D", "M", "K", "CP")
GROUPS = {"w1": (0, 64), "b1": (64, 128), "W2": (128, 4224), "b2": (4224, 4288), "W3": (4288, 4672), "b3": (4672, 4678)}


@pytest.fixture(scope="module")
def setup():
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    c = gpu.ChannelTG(channel_setup(32, 32, 32, 6.0, 3.0, 2.0, 2800.0))
    c.prop_table_init(tab)
    dh = tab.lists["DH"]
    lo, hi = float(dh[0] + 0.05 * (dh[-1] - dh[0])), float(dh[-1] - 0.05 * (dh[-1] - dh[0]))
    c.mlp_init(lo, hi, seed=7)
    yield c, tab, lo, hi
    c.close()


def test_forward_matches_oracle(setup):
    c, tab, lo, hi = setup
    p, nm = c.mlp_params()
    dh = np.random.default_rng(1).uniform(lo, hi, 5000)
    got = c.mlp_infer_points(dh)
    want = orc.mlp_forward(p, nm, dh)
    for m, k in enumerate(FIELDS):
        err = np.abs(got[k] - want[k]).max() / nm[8 + m]
        print(k, err)
        assert err <= 1e-2, (k, err)


def test_gradients_match_oracle(setup):
    c, tab, lo, hi = setup
    p, nm = c.mlp_params()
    dh = np.random.default_rng(2).uniform(lo, hi, 1000)
    g, loss = c.mlp_gradients(dh)
    ot = orc.PropTable(tab.lists)
    go, lo_ = orc.mlp_gradients(ot, p, nm, dh)
    assert lo_ >= 0 and abs(loss - lo_) <= 1e-3 * lo_
    for name, (a, b) in GROUPS.items():
        err = np.abs(g[a:b] - go[a:b]).max() / np.abs(go[a:b]).max()
        print(name, err)
        assert err <= 1e-2, (name, err)


def test_outside_range_is_table_search(setup):
    c, tab, lo, hi = setup
    dh = tab.lists["DH"]
    pts = np.concatenate([np.linspace(dh[0], lo * 0.999 + dh[0] * 0.001, 300), np.linspace(hi + 1e-9, dh[-1], 300)])
    pts = pts[(pts < lo) | (pts > hi)]
    got = c.mlp_infer_points(pts)
    want, nbad, _ = orc.PropTable(tab.lists).update(pts)
    assert nbad == 0
    for k in FIELDS:
        assert np.array_equal(got[k], want[k]), k


TRAIN_SCHEDULE = [(8000, 3e-3), (8000, 1e-3), (8000, 3e-4), (4000, 1e-4)]


def test_trained_model_accuracy(setup):
    """Trained on the table knots in range plus uniform samples (Adam, stepped
    learning rate); bound: 2 % of max(|value|, output scale) for every output
    over 20000 test points.  BF16 activations limit the attainable error to a
    few 1e-3."""
    import time
    c, tab, lo, hi = setup
    dh = tab.lists["DH"]
    knots = dh[(dh >= lo) & (dh <= hi)]
    train = np.concatenate([knots, np.random.default_rng(3).uniform(lo, hi, 6000)])
    loss0 = c.mlp_train(train, 1, lr=1e-3)
    t0 = time.perf_counter()
    for it, lr in TRAIN_SCHEDULE:
        loss = c.mlp_train(train, it, lr=lr)
    print("loss", loss0, "->", loss, "in %.2f s" % (time.perf_counter() - t0))
    assert loss < 1e-3 * loss0
    test = np.random.default_rng(4).uniform(lo, hi, 20000)
    got = c.mlp_infer_points(test)
    want, _, _ = orc.PropTable(tab.lists).update(test)
    p, nm = c.mlp_params()
    for m, k in enumerate(FIELDS):
        rel = np.abs(got[k] - want[k]) / np.maximum(np.abs(want[k]), nm[8 + m])
        print(k, rel.max())
        assert rel.max() <= 2e-2, (k, rel.max())


# ---- the clamped cubic activation (no special-function unit in inference) ----

@pytest.fixture(scope="module")
def setup_cubic():
    rows, T0 = thermo.synthetic_table()
    tab = thermo.SplineTable.from_rows(rows, T0)
    c = gpu.ChannelTG(channel_setup(32, 32, 32, 6.0, 3.0, 2.0, 2800.0))
    c.prop_table_init(tab)
    dh = tab.lists["DH"]
    lo, hi = float(dh[0] + 0.05 * (dh[-1] - dh[0])), float(dh[-1] - 0.05 * (dh[-1] - dh[0]))
    c.mlp_init(lo, hi, seed=7)
    c.mlp_set_activation(gpu.MLP_CUBIC)
    orc.mlp_set_activation(1)
    yield c, tab, lo, hi
    orc.mlp_set_activation(0)
    c.close()


def test_cubic_forward_matches_oracle(setup_cubic):
    """The FP16 pair arithmetic of the cubic is emulated exactly by the oracle; what is left is
    the order of the tensor-core sums, which can move an activation by one FP16 rounding."""
    c, tab, lo, hi = setup_cubic
    p, nm = c.mlp_params()
    dh = np.random.default_rng(1).uniform(lo, hi, 5000)
    got = c.mlp_infer_points(dh)
    want = orc.mlp_forward(p, nm, dh)
    for m, k in enumerate(FIELDS):
        err = np.abs(got[k] - want[k]).max() / nm[8 + m]
        print(k, err)
        assert err <= 2e-3, (k, err)


def test_cubic_gradients_match_oracle(setup_cubic):
    c, tab, lo, hi = setup_cubic
    p, nm = c.mlp_params()
    dh = np.random.default_rng(2).uniform(lo, hi, 1000)
    g, loss = c.mlp_gradients(dh)
    ot = orc.PropTable(tab.lists)
    go, lo_ = orc.mlp_gradients(ot, p, nm, dh)
    assert lo_ >= 0 and abs(loss - lo_) <= 1e-3 * lo_
    for name, (a, b) in GROUPS.items():
        err = np.abs(g[a:b] - go[a:b]).max() / np.abs(go[a:b]).max()
        print(name, err)
        assert err <= 1e-2, (name, err)


# measured bound of the cubic network over its whole trained range: 2 % of max(|value|, output
# scale) for H, T, D, M, K; cp reaches 2.2-2.4 % at its peak (the tanh network: 0.7 %), so cp is
# held to 3 % here.  In the running heated channel the judge reads within 2 % (bench variant).
CUBIC_BOUND = {"H": 2e-2, "T": 2e-2, "D": 2e-2, "M": 2e-2, "K": 2e-2, "CP": 3e-2}


def test_cubic_trained_model_accuracy(setup_cubic):
    """The same data and training schedule as the tanh model, bounds CUBIC_BOUND."""
    c, tab, lo, hi = setup_cubic
    dh = tab.lists["DH"]
    knots = dh[(dh >= lo) & (dh <= hi)]
    train = np.concatenate([knots, np.random.default_rng(3).uniform(lo, hi, 6000)])
    loss0 = c.mlp_train(train, 1, lr=1e-3)
    for it, lr in TRAIN_SCHEDULE:
        loss = c.mlp_train(train, it, lr=lr)
    print("loss", loss0, "->", loss)
    assert loss < 1e-3 * loss0
    test = np.random.default_rng(4).uniform(lo, hi, 20000)
    got = c.mlp_infer_points(test)
    want, _, _ = orc.PropTable(tab.lists).update(test)
    p, nm = c.mlp_params()
    for m, k in enumerate(FIELDS):
        rel = np.abs(got[k] - want[k]) / np.maximum(np.abs(want[k]), nm[8 + m])
        print(k, rel.max())
        assert rel.max() <= CUBIC_BOUND[k], (k, rel.max())
