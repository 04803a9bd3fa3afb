"""chapsim_tdma_lines_noalloc: the line solves on caller-owned device arrays,
with the library's work vectors in its fixed device scratch array.

Checked against the host-array entry points chapsim_tdmaijj_noncyc and
chapsim_tdmaiji_cyc on consecutive calls of different shapes, so a call that
finds the previous call's contents in the shared scratch array is covered.
This file is collected last on purpose: it must pass both alone in a fresh
process and after every other GPU test has used the device.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12          # FP64 recurrences vs the warp Thomas/PCR path: rounding only
ERR_BADARG, ERR_NAN = -6, -2


def _lib():
    from chapsim import gpu
    return gpu.load_library()


def _system(rng, jsz, isz):
    A = rng.uniform(-1.0, 0.0, (jsz, isz))
    C = rng.uniform(-1.0, 0.0, (jsz, isz))
    B = 2.5 + rng.uniform(0.0, 1.0, (jsz, isz))
    R = rng.standard_normal((jsz, isz))
    return A, B, C, R


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float64)).to("cuda:0")


def _noalloc(A, B, C, R, bcj, cyclic):
    """Solves on device copies; lines along ISZ when cyclic (TDMAIJI), along JSZ otherwise (TDMAIJJ)."""
    import torch
    jsz, isz = R.shape
    if cyclic:
        nlines, ls, es, n = jsz, isz, 1, isz
    else:
        nlines, ls, es, n = isz, 1, isz, jsz
    dA, dB, dC, dR = (_dev(x) for x in (A, B, C, R))
    dbc = None if bcj is None else _dev(bcj)
    torch.cuda.synchronize()
    rc = _lib().chapsim_tdma_lines_noalloc(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), dR.data_ptr(),
                                           None if dbc is None else dbc.data_ptr(), nlines, ls, es, n,
                                           1 if cyclic else 0, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc, dR.cpu().numpy()


def _err():
    return _lib().chapsim_last_error_string(None).decode()


def _close(x, ref):
    scale = np.max(np.abs(ref))
    return np.max(np.abs(x - ref)) <= RTOL * scale


def test_noalloc_matches_existing_entry_points_on_consecutive_calls():
    from chapsim import gpu
    rng = np.random.default_rng(20261203)
    # call 1: non-cyclic along J with Dirichlet values, 200 lines of 128
    A1, B1, C1, R1 = _system(rng, 128, 200)
    bc1 = rng.standard_normal((2, 200))
    ref1 = gpu.tdmaijj_noncyc(A1, B1, C1, R1, bc1)
    rc, out1 = _noalloc(A1, B1, C1, R1, bc1, cyclic=False)
    assert rc == 0, _err()
    assert _close(out1, ref1)
    # call 2: cyclic along I, 300 lines of 96 (a different size: stale scratch from call 1)
    A2, B2, C2, R2 = _system(rng, 300, 96)
    ref2 = gpu.tdmaiji_cyc(A2, B2, C2, R2)
    rc, out2 = _noalloc(A2, B2, C2, R2, None, cyclic=True)
    assert rc == 0, _err()
    assert _close(out2, ref2)
    # call 3: the first system again, ragged length 70, no Dirichlet values
    A3, B3, C3, R3 = (x[:70] for x in (A1, B1, C1, R1))
    ref3 = gpu.tdmaijj_noncyc(A3, B3, C3, R3)
    rc, out3 = _noalloc(A3, B3, C3, R3, None, cyclic=False)
    assert rc == 0, _err()
    assert _close(out3, ref3)


def test_noalloc_rejects_oversize_and_host_pointers():
    import torch
    lib = _lib()
    t = torch.zeros(64, dtype=torch.float64, device="cuda:0")
    p = t.data_ptr()
    # 3 * 64 * 2^20 doubles of scratch is beyond the fixed 16 MiB array
    rc = lib.chapsim_tdma_lines_noalloc(p, p, p, p, None, 1 << 20, 64, 1, 64, 0, None)
    assert rc == ERR_BADARG and "exceeds the fixed limit" in _err()
    h = np.zeros(64)
    hp = h.ctypes.data_as(ctypes.c_void_p).value
    rc = lib.chapsim_tdma_lines_noalloc(hp, hp, hp, hp, None, 1, 64, 1, 64, 0, None)
    assert rc == ERR_BADARG and "device memory" in _err()


def test_noalloc_status_counter_is_cleared_between_calls():
    rng = np.random.default_rng(7)
    A, B, C, R = _system(rng, 64, 40)
    Rbad = R.copy()
    Rbad[:, 5] = np.nan          # line 5 (along J) has a non-finite right-hand side
    rc, _ = _noalloc(A, B, C, Rbad, None, cyclic=False)
    assert rc == ERR_NAN and "1 of 40 lines" in _err()
    from chapsim import gpu
    ref = gpu.tdmaijj_noncyc(A, B, C, R)
    rc, out = _noalloc(A, B, C, R, None, cyclic=False)
    assert rc == 0, _err()
    assert _close(out, ref)


def test_noalloc_strided_subblock_against_oracle():
    """Lines inside a larger caller-owned device array, with padded strides:
    rows of a (48, 80) block with line_stride 80 > n, and every other column
    of it (line_stride 2, elem_stride 80, neither 1 nor the line count).
    The solution matches the oracle's recurrences (TDMAIJI_CYC,
    src/TDMAIJI_CYC.f90:67-157; TDMAIJJ_nonCYC, src/TDMAIJJ_nonCYC.f90:67-123)
    and no entry outside the lines is read or written: the coefficient
    padding holds NaN and the right-hand side's padding a sentinel."""
    import torch
    import oracle as orc
    rng = np.random.default_rng(31)
    rows, cols = 48, 80
    cases = [
        # (first offset, nlines, line_stride, elem_stride, n, cyclic)
        (3 * cols + 5, 40, cols, 1, 60, True),
        (2 * cols + 1, 30, 2, cols, 45, False),
    ]
    for off, nl, ls, es, n, cyc in cases:
        idx = off + np.arange(nl)[:, None] * ls + np.arange(n)[None, :] * es
        assert idx.max() < rows * cols and len(np.unique(idx)) == idx.size
        coef = []
        for lo, hi in ((-1.0, 0.0), (2.5, 3.5), (-1.0, 0.0)):
            x = np.full(rows * cols, np.nan)
            x[idx] = rng.uniform(lo, hi, idx.shape)
            coef.append(x)
        r = np.full(rows * cols, 12345.0)
        r[idx] = rng.standard_normal(idx.shape)
        dA, dB, dC, dR = (_dev(x) for x in (*coef, r))
        torch.cuda.synchronize()
        o8 = 8 * off  # the sub-block starts `off` doubles into each array
        rc = _lib().chapsim_tdma_lines_noalloc(dA.data_ptr() + o8, dB.data_ptr() + o8, dC.data_ptr() + o8,
                                               dR.data_ptr() + o8, None, nl, ls, es, n, 1 if cyc else 0,
                                               torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert rc == 0, _err()
        out = dR.cpu().numpy()
        pad = np.ones(rows * cols, bool)
        pad[idx] = False
        assert np.all(out[pad] == 12345.0)
        for l in range(nl):
            a, b, c, rr = (x[idx[l]].copy() for x in (*coef, r))
            if cyc:
                ref = orc.tdma_cyc(a, b, c, rr)
            else:
                a[0] = 0.0
                c[-1] = 0.0
                ref = orc.tdma_noncyc(a, b, c, rr)
            assert _close(out[idx[l]], ref), (l, cyc)
