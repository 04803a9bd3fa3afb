"""Seeded initial fields and the reference's ``.D`` field-file format.

Initial field.  The reference draws its perturbation from gfortran's
intrinsic RNG re-seeded per grid point (src/INITIAL_FL_FLD_TG.f90:176-200,
src/processing/randomgen.f90:66-112); that stream is not reproducible
outside libgfortran, so it is replaced by SplitMix64 (Steele, Lea & Flood,
"Fast splittable pseudorandom number generators", OOPSLA 2014) keyed by
(seed, component, i, j, k).  The remaining steps follow random_FL_FLD_TG
(src/INITIAL_FL_FLD_TG.f90:13-104): perturbation of amplitude ``vper`` in
all three components, v = 0 on the wall face, subtraction of the x-z mean of
every component per y row (INITIAL_MEAN_TG), addition of the Poiseuille
profile Vini to u, and scaling of u to unit bulk velocity
(BULK_VELOCITY_TG :141-170).  The caller then runs the NS = 0 substep, the
projection of CALC_INITIALIZATION_tg (:109-139).

``.D`` files (src/processing/WRT_VARS_TG.f90, READ_INTP_3D_VARS.f90): a
40-byte header int32[4] {L, M, N, ITERG} + float64[3] {time, REN, DT},
then float64 (L, M, N) in Fortran order, no ghost planes.
"""
from __future__ import annotations

import struct

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 output function applied to a uint64 counter array."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def uniform_pm1(seed: int, comp: int, shape_nml) -> np.ndarray:
    """Uniform numbers in [-1, 1) for every (k, j, i) of a (N, M, L) block."""
    N, M, L = shape_nml
    k, j, i = np.meshgrid(np.arange(N, dtype=np.uint64), np.arange(M, dtype=np.uint64),
                          np.arange(L, dtype=np.uint64), indexing="ij")
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0x100000001B3)) & _M64
        key = (key ^ (np.uint64(comp) << np.uint64(56))) & _M64
        ctr = (key + ((k << np.uint64(40)) | (j << np.uint64(20)) | i)) & _M64
    r = splitmix64(splitmix64(ctr))
    u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)  # [0, 1)
    return 2.0 * u - 1.0


def initial_field(setup, seed: int = 1973, vper: float = 0.1):
    """Seeded perturbed-Poiseuille field (before the NS = 0 projection).

    Returns Q of shape (3, N, M+2, L) and PR of shape (N, M+2, L) (C order,
    i.e. Fortran Q_tg(L, 0:M+1, N, 3) and PR_tg(L, 0:M+1, N)).
    """
    L, M, N = setup.L, setup.M, setup.N
    Q = np.zeros((3, N, M + 2, L))
    for c in range(3):
        Q[c, :, 1:M + 1, :] = vper * uniform_pm1(seed, c, (N, M, L))
    Q[1, :, 1, :] = 0.0  # v on the bottom wall face
    # subtract the x-z mean of each component per y row
    for c in range(3):
        Q[c, :, 1:M + 1, :] -= Q[c, :, 1:M + 1, :].mean(axis=(0, 2), keepdims=True)
    Q[0, :, 1:M + 1, :] += setup.Vini[1:M + 1][None, :, None]
    Q[1, :, 1, :] = 0.0
    # unit bulk velocity
    dy = 1.0 / setup.DYFI[1:M + 1]
    ub = float((Q[0, :, 1:M + 1, :] * dy[None, :, None]).sum() / setup.DZI / (setup.Area_inlet * L))
    Q[0, :, 1:M + 1, :] /= ub
    # wall ghosts (BC_WALL_Q_tg)
    Q[:, :, 0, :] = 0.0
    Q[:, :, M + 1, :] = 0.0
    Q[1, :, 1, :] = 0.0
    PR = np.zeros((N, M + 2, L))
    return Q, PR


def bulk_velocity(setup, Q) -> float:
    """BULK_VELOCITY_TG (src/INITIAL_FL_FLD_TG.f90:141-170)."""
    M, L = setup.M, setup.L
    dy = 1.0 / setup.DYFI[1:M + 1]
    return float((Q[0, :, 1:M + 1, :] * dy[None, :, None]).sum() / setup.DZI / (setup.Area_inlet * L))


def write_dfile(path, field_nml, iterg: int, time: float, ren: float, dt: float):
    """Write one (N, M, L) C-order interior field as a reference .D file."""
    f = np.ascontiguousarray(field_nml, dtype="<f8")
    N, M, L = f.shape
    with open(path, "wb") as fh:
        fh.write(struct.pack("<4i", L, M, N, int(iterg)))
        fh.write(struct.pack("<3d", float(time), float(ren), float(dt)))
        fh.write(f.tobytes())


def read_dfile(path):
    """Read a reference .D file: returns (field (N, M, L), header dict)."""
    with open(path, "rb") as fh:
        b = fh.read()
    if len(b) < 40:
        raise ValueError(f"{path}: truncated header")
    L, M, N, it = struct.unpack("<4i", b[:16])
    t, ren, dt = struct.unpack("<3d", b[16:40])
    if min(L, M, N) <= 0 or len(b) != 40 + 8 * L * M * N:
        raise ValueError(f"{path}: header dims {L}x{M}x{N} do not match the payload")
    f = np.frombuffer(b[40:], dtype="<f8").reshape(N, M, L).copy()
    return f, {"L": L, "M": M, "N": N, "ITERG": it, "time": t, "REN": ren, "DT": dt}


def xinout_fields_from_tg(Q_tg, L_io: int):
    """Start fields of an inflow/outflow main domain (iDomain = 3) of L_io cells from a
    periodic TG velocity field (3, N, M+2, L_tg): the TG field repeated along x, with the
    ghost columns 0 and L_io + 1 (NCL1S:NCL1E) filled the same way.  Returns G of shape
    (3, N, M+2, L_io+2) (rho u with unit density) and a zero pressure (N, M+2, L_io+2).
    """
    Q_tg = np.asarray(Q_tg, np.float64)
    _, N, M2, LT = Q_tg.shape
    idx = [(i - 1) % LT for i in range(L_io + 2)]
    G = np.ascontiguousarray(Q_tg[:, :, :, idx])
    return G, np.zeros((N, M2, L_io + 2))
