"""Host-side property-table set-up for the table-search property update.

Restates, for callers without the Fortran host, the set-up the reference
does once per run before THERM_PROP_UPDATE can search the table:

* ``read_table`` reads the table file format of ``Property_Table_Nondimensionalization``
  (src/thermo_properties_table_searching.f90:1242-1263): one title line,
  N_LIST, then N_LIST rows of P, H, T, D, M, K, CP, B (SI units).
* ``nondimensionalize`` sorts by T (selection sort, :1265-1293), interpolates
  the reference state at T0 with ``BiSection_LIST_T`` (:808-839, :1297-1307)
  and scales the table (:1321-1330).
* ``cubic_spline`` is CUBIC_SPLINE (:842-936), Forsythe, Malcolm & Moler's
  spline with third-divided-difference end conditions.
* ``spline_table`` builds the DH->H spline and the H->T, D, M, K, CP splines
  of SPLINE_COEFFICIENTS_FOR_DH / _FOR_H (:972-1128), and checks that rho*h
  is monotone in T and in h as the reference does (:1016-1023).

All arithmetic is scalar IEEE FP64 in the reference's order, so the lists
and coefficients are bitwise those the Fortran set-up produces.

``synthetic_table`` writes a seeded 2048-row table in the same file format
for the heated-channel workload (monotone rho, mu, kappa, T in h; a
Lorentzian cp peak 8x the baseline with a FWHM of 3 % of the h range).
"""
from __future__ import annotations

import math

import numpy as np

COLUMNS = ["P", "H", "T", "D", "M", "K", "CP", "B"]
LIST_NAMES = ["H", "T", "D", "M", "K", "CP", "B", "DH"]
H_SPLINES = ["T", "D", "M", "K", "CP", "B"]


def read_table(path: str) -> np.ndarray:
    """Rows (N_LIST, 8) of the table file, in file order."""
    with open(path) as f:
        f.readline()
        n = int(f.readline().split()[0])
        rows = np.array([[float(v) for v in f.readline().split()[:8]] for _ in range(n)], np.float64)
    if rows.shape != (n, 8):
        raise ValueError(f"{path}: expected {n} rows of 8 values")
    return rows


def write_table(path: str, rows: np.ndarray, title: str = "#P(Mpa) H(J/KG) T(K) D(KG/M3) M(PA-S) K(W/M-K) "
                                                          "CP(J/KG-K) Beta(1/K)") -> None:
    with open(path, "w") as f:
        f.write(title + "\n")
        f.write(f"{rows.shape[0]}\n")
        for r in rows:
            f.write("\t".join(f"{v:.13E}" for v in r) + "\n")


def nondimensionalize(rows: np.ndarray, T0: float):
    """Sorted, scaled lists {H, T, D, M, K, CP, B, DH} and the reference state
    {H0, D0, K0, M0, CP0, B0} (dimensional)."""
    rows = np.asarray(rows, np.float64)
    n = rows.shape[0]
    H, T, D, M, K, CP, B = (rows[:, c].copy() for c in range(1, 8))
    for i in range(n):
        k = int(np.argmin(T[i:])) + i          # MINLOC: first minimum
        for a in (T, D, H, M, K, B, CP):
            a[i], a[k] = a[k], a[i]
    is_, ie = 1, n
    while ie - is_ > 1:
        im = is_ + (ie - is_) // 2
        if (T[is_ - 1] - T0) * (T[im - 1] - T0) > 0.0:
            is_ = im
        else:
            ie = im
    sfs = (T[ie - 1] - T0) / (T[ie - 1] - T[is_ - 1])
    sfe = 1.0 - sfs

    def ref(a):
        return sfe * a[ie - 1] + sfs * a[is_ - 1]

    H0, D0, K0, M0, CP0, B0 = ref(H), ref(D), ref(K), ref(M), ref(CP), ref(B)
    H = (H - H0) / T0 / CP0
    T = T / T0
    D = D / D0
    M = M / M0
    K = K / K0
    CP = CP / CP0
    B = B / B0
    DH = D * H
    return ({"H": H, "T": T, "D": D, "M": M, "K": K, "CP": CP, "B": B, "DH": DH},
            {"H0": H0, "D0": D0, "K0": K0, "M0": M0, "CP0": CP0, "B0": B0})


def cubic_spline(x, y):
    """CUBIC_SPLINE(N, X, Y, B, C, D) -> (B, C, D), scalar FP64 in the reference's order."""
    x = [float(v) for v in x]
    y = [float(v) for v in y]
    n = len(x)
    b, c, d = [0.0] * n, [0.0] * n, [0.0] * n
    if n < 2:
        return np.array(b), np.array(c), np.array(d)
    if n < 3:
        b[0] = (y[1] - y[0]) / (x[1] - x[0])
        b[1] = b[0]
        return np.array(b), np.array(c), np.array(d)
    nm1 = n - 1
    d[0] = x[1] - x[0]
    c[1] = (y[1] - y[0]) / d[0]
    for i in range(1, nm1):
        d[i] = x[i + 1] - x[i]
        b[i] = 2.0 * (d[i - 1] + d[i])
        c[i + 1] = (y[i + 1] - y[i]) / d[i]
        c[i] = c[i + 1] - c[i]
    b[0] = -d[0]
    b[n - 1] = -d[n - 2]
    c[0] = 0.0
    c[n - 1] = 0.0
    if n != 3:
        c[0] = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0])
        c[n - 1] = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4])
        c[0] = c[0] * d[0] * d[0] / (x[3] - x[0])
        c[n - 1] = -c[n - 1] * (d[n - 2] * d[n - 2]) / (x[n - 1] - x[n - 4])
    for i in range(1, n):
        t = d[i - 1] / b[i - 1]
        b[i] = b[i] - t * d[i - 1]
        c[i] = c[i] - t * c[i - 1]
    c[n - 1] = c[n - 1] / b[n - 1]
    for i in range(n - 2, -1, -1):
        c[i] = (c[i] - d[i] * c[i + 1]) / b[i]
    b[n - 1] = (y[n - 1] - y[nm1 - 1]) / d[nm1 - 1] + d[nm1 - 1] * (c[nm1 - 1] + 2.0 * c[n - 1])
    for i in range(nm1):
        b[i] = (y[i + 1] - y[i]) / d[i] - d[i] * (c[i + 1] + 2.0 * c[i])
        d[i] = (c[i + 1] - c[i]) / d[i]
        c[i] = 3.0 * c[i]
    c[n - 1] = 3.0 * c[n - 1]
    d[n - 1] = d[nm1 - 1]
    return np.array(b), np.array(c), np.array(d)


class SplineTable:
    """Nondimensional lists plus the spline coefficients the property update needs."""

    def __init__(self, lists: dict, ref: dict | None = None):
        self.lists = {k: np.ascontiguousarray(v, np.float64) for k, v in lists.items()}
        self.ref = ref or {}
        self.n = len(self.lists["H"])
        H, T, DH = self.lists["H"], self.lists["T"], self.lists["DH"]
        for i in range(1, self.n - 1):
            if ((DH[i] - DH[i - 1]) / (T[i] - T[i - 1])) * ((DH[i + 1] - DH[i]) / (T[i + 1] - T[i])) < 0.0:
                raise ValueError("the relation (rho * h) = FUNCTION (T) is not monotone")
            if ((DH[i] - DH[i - 1]) / (H[i] - H[i - 1])) * ((DH[i + 1] - DH[i]) / (H[i + 1] - H[i])) < 0.0:
                raise ValueError("the relation (rho * h) = FUNCTION (h) is not monotone")
        self.coef = {"DHH": cubic_spline(DH, H)}
        for name in H_SPLINES:
            self.coef["H" + name] = cubic_spline(H, self.lists[name])

    @classmethod
    def from_rows(cls, rows, T0):
        lists, ref = nondimensionalize(rows, T0)
        return cls(lists, ref)

    @classmethod
    def from_file(cls, path, T0):
        return cls.from_rows(read_table(path), T0)


def _lorentz_T(h, h_lo, h_pc, gamma, cp_b, T_lo):
    """T(h) = T_lo + integral of dh / cp with cp = cp_b (1 + 7 / (1 + u^2)), u = (h - h_pc) / gamma."""
    r8 = math.sqrt(8.0)

    def F(x):
        u = (x - h_pc) / gamma
        return gamma / cp_b * (u - 7.0 / r8 * np.arctan(u / r8))

    return T_lo + F(h) - F(h_lo)


def synthetic_table(n: int = 2048, seed: int = 2048, P: float = 23.5):
    """Seeded table rows (n, 8) in SI units, and a T0 inside it.

    h is uniform over [1.0e6, 2.6e6] J/kg.  cp has a Lorentzian peak of height
    8x its baseline and FWHM 3 % of the h range at a seeded pseudo-critical
    enthalpy h_pc; T(h) is the exact integral of dh/cp.  rho, mu and kappa fall
    monotonically, with most of the drop across the cp peak; beta follows cp.
    T0 lies above the peak (as for the reference's supercritical-water case),
    which keeps rho*h monotone in h.
    """
    rng = np.random.default_rng(seed)
    h_lo, h_hi = 1.0e6, 2.6e6
    span = h_hi - h_lo
    h_pc = h_lo + span * rng.uniform(0.42, 0.48)
    gamma = 0.5 * 0.03 * span
    cp_b = 5000.0 * rng.uniform(0.98, 1.02)
    T_lo = 600.0
    h = h_lo + span * np.arange(n, dtype=np.float64) / (n - 1)
    u = (h - h_pc) / gamma
    lor = 1.0 / (1.0 + u * u)
    cp = cp_b * (1.0 + 7.0 * lor)
    T = _lorentz_T(h, h_lo, h_pc, gamma, cp_b, T_lo)
    # monotone transition through the peak plus a linear background, both in [0, 1]
    s = 0.65 * (np.arctan(u / 3.0) / math.pi + 0.5) + 0.35 * (h - h_lo) / span
    s = (s - s[0]) / (s[-1] - s[0])
    rho = 720.0 - (720.0 - 110.0) * s
    mu = 9.0e-5 - (9.0e-5 - 2.8e-5) * s
    kap = 0.52 - (0.52 - 0.11) * s
    beta = 2.0e-3 * (1.0 + 7.0 * lor)
    rows = np.stack([np.full(n, P), h, T, rho, mu, kap, cp, beta], axis=1)
    # reference temperature above the pseudo-critical peak, where rho*h is monotone
    T0 = float(_lorentz_T(h_lo + 0.65 * span, h_lo, h_pc, gamma, cp_b, T_lo))
    return rows, T0


def table_field(rows, T0, shape, seed=1, frac=(0.05, 0.95)):
    """Seeded rho*h samples inside the nondimensional table range (for tests and benches)."""
    tab = SplineTable.from_rows(rows, T0)
    dh = tab.lists["DH"]
    lo, hi = dh.min(), dh.max()
    rng = np.random.default_rng(seed)
    return lo + (hi - lo) * rng.uniform(frac[0], frac[1], size=shape)
