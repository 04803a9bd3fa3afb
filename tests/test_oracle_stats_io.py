"""The oracle's restatement of PP_MEAN_ZX_FLOW_Xperiodic_io
(src/processing/PP_MEAN_ZX.f90:311-796), checked on the CPU before it is
trusted as the checker of the device statistics.

* With unit density the momentum G equals the velocity, and the flow arrays
  the main-domain routine shares with PP_MEAN_ZX_FLOW_TG (:14-307) -- U1, UP,
  U2, U3, DVDL1, DVDLP, DVDL2 -- equal the periodic-domain restatement's on
  the same field (the TG routine scales its sums once at the end, the IO
  routine per point: rounding only), and G1, UG, UGU equal U1, U2, U3.  The
  one exception is the reference's own: PP_MEAN_ZX_FLOW_TG scales DVDL2 by
  COG2 = COG1 COG1 (:79-89, :280-289), which carries VL1313 twice, so its
  DVDL2 is the main domain's divided by NCL1 * NCL3.
* Closed forms on a uniform flow: the means are the values, the products
  their products, and every gradient and gradient product vanishes.
"""
import math

import numpy as np

from oracle import Oracle
from chapsim.mesh import channel_setup
from chapsim.fields import initial_field

FLOW = [("U1", 3), ("P1", 1), ("G1", 3), ("UP", 3), ("U2", 6), ("UG", 6), ("U3", 10), ("UGU", 10), ("DVDL1", 9),
        ("DVDLP", 9), ("DVDL2", 81)]
TG = [("U1", 3), ("P1", 1), ("UP", 3), ("U2", 6), ("U3", 10), ("DVDL1", 9), ("DVDLP", 9), ("DVDL2", 81)]
ARGS = (32, 32, 16, 2 * math.pi, math.pi, 2.0, 2800.0)


def _split(flat, M, arrays):
    out, off = {}, 0
    for name, w in arrays:
        out[name] = flat[off * M:(off + w) * M].reshape(w, M)
        off += w
    assert off * M == flat.size
    return out


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_io_means_match_periodic_restatement_at_unit_density():
    L, M, N = ARGS[:3]
    s = channel_setup(*ARGS)
    Q, PR = initial_field(s, 7, 0.2)
    ones = np.ones((N, M + 2, L))
    io = Oracle(*ARGS)
    io.io_set_fields(Q, PR, ones, ones, ones)
    tg = Oracle(*ARGS)
    tg.set_fields(Q, PR)
    a = _split(io.pp_mean_zx_io(), M, FLOW)
    b = _split(tg.pp_mean_zx_tg(), M, TG)
    b["DVDL2"] = b["DVDL2"] * (L * N)  # VL1313 twice in the periodic routine's COG2
    for name, _ in TG:
        assert _rel(a[name], b[name]) <= 1e-13, name
    assert _rel(a["G1"], a["U1"]) <= 1e-15
    assert _rel(a["UG"], a["U2"]) <= 1e-15
    assert _rel(a["UGU"], a["U3"]) <= 1e-15
    io.close()
    tg.close()


def test_io_means_of_a_uniform_flow():
    L, M, N = ARGS[:3]
    u, v, w, p = 0.7, 0.0, 0.3, 1.5  # v = 0: the walls impose it
    Q = np.zeros((3, N, M + 2, L))
    Q[0], Q[1], Q[2] = u, v, w
    PR = np.full((N, M + 2, L), p)
    ones = np.ones((N, M + 2, L))
    io = Oracle(*ARGS)
    io.io_set_fields(Q, PR, ones, ones, ones)
    a = _split(io.pp_mean_zx_io(), M, FLOW)
    vel = [u, v, w]
    assert np.allclose(a["U1"], np.array(vel)[:, None], rtol=1e-13, atol=0)
    assert np.allclose(a["P1"], p, rtol=1e-13, atol=0)
    assert np.allclose(a["UP"], (np.array(vel) * p)[:, None], rtol=1e-13, atol=0)
    pairs = [vel[m] * vel[n] for m in range(3) for n in range(m, 3)]
    assert np.allclose(a["U2"], np.array(pairs)[:, None], rtol=1e-13, atol=0)
    triples = [vel[m] * vel[n] * vel[h] for m in range(3) for n in range(m, 3) for h in range(n, 3)]
    assert np.allclose(a["U3"], np.array(triples)[:, None], rtol=1e-13, atol=0)
    # gradients vanish away from the walls (rows 2 .. M-1; the wall rows see the no-slip ghosts)
    for name in ("DVDL1", "DVDLP", "DVDL2"):
        assert np.abs(a[name][:, 1:M - 1]).max() <= 1e-12, name
    io.close()
