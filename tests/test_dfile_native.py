""".D field files through the library's native reader and writer (host
functions of the C ABI: no GPU needed).

* The header layout is pinned by the reference's own step-100 TC8 files
  (DNS_perixz_INSTANT_T1.000000000E-01_*.D, their header kept in the golden
  fixture): the native writer produces exactly those 40 bytes, and the time
  string of the file name (ES15.9) is exactly the reference's.
* Native writer and the NumPy reader, and the NumPy writer and the native
  reader, round-trip bitwise; truncated files and headers that do not match
  the payload are rejected with CHAPSIM_ERR_BADARG.
"""
import os
import struct

import numpy as np
import pytest

from chapsim import gpu
from chapsim import fields


def test_header_bytes_match_the_reference_file(golden_dir, tmp_path):
    d = np.load(os.path.join(golden_dir, "tc8_step100_fields.npz"))
    hi = [int(x) for x in d["header_int"]]
    hr = [float(x) for x in d["header_real"]]
    L, M, N, it = hi
    f = d["G1"].astype(np.float64)
    p = tmp_path / "u.D"
    gpu.write_dfile(p, f, it, hr[0], hr[1], hr[2])
    b = p.read_bytes()
    assert b[:40] == struct.pack("<4i", *hi) + struct.pack("<3d", *hr)
    assert len(b) == 40 + 8 * L * M * N
    assert np.array_equal(np.frombuffer(b[40:], "<f8").reshape(N, M, L), f)


def test_file_name_time_string_is_the_references(golden_dir):
    d = np.load(os.path.join(golden_dir, "tc8_step100_fields.npz"))
    assert gpu.es15_9(float(d["header_real"][0])) == "1.000000000E-01"
    assert gpu.es15_9(0.0) == "0.000000000E+00"
    assert gpu.es15_9(12.5) == "1.250000000E+01"
    assert all(len(gpu.es15_9(t)) == 15 for t in (0.0, 1e-3, 0.1, 2.0, 99.5))


def test_native_and_numpy_round_trips(tmp_path):
    rng = np.random.default_rng(5)
    f = rng.standard_normal((6, 5, 8))
    gpu.write_dfile(tmp_path / "a.D", f, 42, 0.25, 2800.0, 1e-3)
    g, h = fields.read_dfile(tmp_path / "a.D")
    assert np.array_equal(g, f) and h == {"L": 8, "M": 5, "N": 6, "ITERG": 42, "time": 0.25, "REN": 2800.0,
                                          "DT": 1e-3}
    fields.write_dfile(tmp_path / "b.D", f, 7, 1.5, 180.0, 2e-4)
    g, h = gpu.read_dfile(tmp_path / "b.D")
    assert np.array_equal(g, f) and (h["L"], h["M"], h["N"], h["ITERG"]) == (8, 5, 6, 7)
    assert (h["time"], h["REN"], h["DT"]) == (1.5, 180.0, 2e-4)


def test_native_reader_rejects_bad_files(tmp_path):
    f = np.zeros((2, 3, 4))
    p = tmp_path / "c.D"
    gpu.write_dfile(p, f, 1, 0.0, 1.0, 1.0)
    b = p.read_bytes()
    (tmp_path / "short.D").write_bytes(b[:30])
    (tmp_path / "cut.D").write_bytes(b[:-8])
    (tmp_path / "dims.D").write_bytes(struct.pack("<4i", 4, 3, 3, 1) + b[16:])
    for name in ("short.D", "cut.D", "dims.D", "missing.D"):
        with pytest.raises(gpu.ChapsimError) as e:
            gpu.read_dfile(tmp_path / name)
        assert e.value.code == -6, name
