"""Host-side logic: seeded initial field, .D file format, error paths."""
import math
import os

import numpy as np
import pytest

from chapsim.mesh import channel_setup
from chapsim.fields import initial_field, bulk_velocity, read_dfile, write_dfile, uniform_pm1


def test_rng_deterministic_and_uniform():
    a = uniform_pm1(1973, 0, (8, 16, 32))
    b = uniform_pm1(1973, 0, (8, 16, 32))
    c = uniform_pm1(1974, 0, (8, 16, 32))
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.min() >= -1.0 and a.max() < 1.0 and abs(a.mean()) < 0.05


def test_initial_field_properties():
    s = channel_setup(32, 32, 32, 2 * math.pi, math.pi, 2.0, 2800.0)
    Q, PR = initial_field(s, 1973, 0.1)
    assert abs(bulk_velocity(s, Q) - 1.0) < 1e-14
    assert np.all(Q[:, :, 0, :] == 0) and np.all(Q[:, :, -1, :] == 0) and np.all(Q[1, :, 1, :] == 0)
    assert np.all(PR == 0)


def test_dfile_roundtrip(tmp_path):
    f = np.random.default_rng(0).standard_normal((6, 5, 4))
    p = tmp_path / "x.D"
    write_dfile(p, f, 100, 0.1, 2800.0, 1e-3)
    g, h = read_dfile(p)
    assert np.array_equal(f, g)
    assert (h["L"], h["M"], h["N"], h["ITERG"]) == (4, 5, 6, 100)
    assert os.path.getsize(p) == 40 + 8 * f.size


def test_dfile_truncated_and_bad_header(tmp_path):
    f = np.zeros((2, 2, 2))
    p = tmp_path / "t.D"
    write_dfile(p, f, 1, 0.0, 1.0, 1.0)
    b = open(p, "rb").read()
    open(p, "wb").write(b[:-8])
    with pytest.raises(ValueError):
        read_dfile(p)
    open(p, "wb").write(b[:20])
    with pytest.raises(ValueError):
        read_dfile(p)


def test_setup_rejects_odd_periodic_length():
    with pytest.raises(ValueError):
        channel_setup(31, 32, 32, 1.0, 1.0, 2.0, 100.0)
