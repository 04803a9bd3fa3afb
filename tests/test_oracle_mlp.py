"""The learned-model oracle (oracle/mlp_oracle.c), checked on the CPU before it
checks the tensor-core kernels.

* The clamped cubic activation c = clamp(z, -1, 1), h = c (3 - c^2) / 2: odd,
  saturating at +-1 with zero slope there, slope 3/2 at 0.
* The oracle's inference form with that activation equals a numpy restatement
  of the same FP16 pair arithmetic (x split into two FP16 parts, FP16 fused
  multiply-adds of the first layer, FP16 products and one-rounding fused
  multiply-add of the cubic, FP16 operands of the two products summed in
  FP64).
"""
import numpy as np

import oracle as orc

NP = orc.MLP_NPARAM
H = 64


def _params(seed):
    r = np.random.default_rng(seed)
    p = np.zeros(NP, np.float32)
    p[0:64] = r.uniform(-3, 3, 64)           # w1
    p[64:128] = r.uniform(-1, 1, 64)         # b1
    p[128:4224] = r.normal(0, 0.25, 4096)    # W2 (out, in)
    p[4224:4288] = r.uniform(-0.5, 0.5, 64)  # b2
    p[4288:4672] = r.normal(0, 0.2, 384)     # W3
    p[4672:4678] = r.uniform(-0.1, 0.1, 6)   # b3
    return p


def _cubic16(pre):
    c = np.clip(pre.astype(np.float64), -1.0, 1.0)
    c2 = (c * c).astype(np.float16).astype(np.float64)
    s = (c2 * -0.5 + 1.5).astype(np.float16).astype(np.float64)
    return (c * s).astype(np.float16).astype(np.float64)


def _forward_inf_cubic(p, norm, dh):
    lo, hi = float(np.float32(norm[0])), float(np.float32(norm[1]))
    x = np.float32(2.0 * (dh - lo) / (hi - lo) - 1.0)
    xh = np.float32(np.float16(x))
    xl = np.float32(np.float16(np.float32(x - xh)))
    w = p[0:64].astype(np.float16).astype(np.float64)
    b = p[64:128].astype(np.float16).astype(np.float64)
    inner = (w * float(xl) + b).astype(np.float16).astype(np.float64)
    pre = (w * float(xh) + inner).astype(np.float16)
    h1 = _cubic16(pre)
    W2 = p[128:4224].reshape(64, 64).astype(np.float16).astype(np.float64)
    a2 = W2 @ h1
    z2 = (a2.astype(np.float32) + p[4224:4288]).astype(np.float16)
    h2 = _cubic16(z2)
    W3 = p[4288:4672].reshape(6, 64).astype(np.float16).astype(np.float64)
    y = (W3 @ h2).astype(np.float32) + p[4672:4678]
    off, sc = np.float32(norm[2:8]), np.float32(norm[8:14])
    return (off + sc * y).astype(np.float64)


def test_cubic_activation_shape():
    z = np.linspace(-3, 3, 601)
    c = np.clip(z, -1, 1)
    h = c * (1.5 - 0.5 * c * c)
    assert np.allclose(h, -h[::-1]) and h.max() == 1.0 and h.min() == -1.0
    d = 1.5 * (1 - c * c)
    assert d[np.abs(z) >= 1].max() == 0.0 and abs(d[300] - 1.5) < 1e-15
    # C1 at the clamp points
    assert np.allclose(np.gradient(h, z)[np.abs(np.abs(z) - 1) < 0.02], 0.0, atol=0.05)


def test_cubic_inference_form_matches_numpy_restatement():
    p = _params(11)
    norm = np.array([0.1, 2.3] + [0.5] * 6 + [1.7] * 6)
    dh = np.random.default_rng(3).uniform(0.1, 2.3, 200)
    orc.mlp_set_activation(1)
    try:
        got = orc.mlp_forward(p, norm, dh)
    finally:
        orc.mlp_set_activation(0)
    want = np.array([_forward_inf_cubic(p, norm, v) for v in dh])  # (n, 6)
    for k, name in enumerate(["H", "T", "D", "M", "K", "CP"]):
        err = np.abs(got[name] - want[:, k]).max() / 1.7
        assert err <= 1e-6, (name, err)
