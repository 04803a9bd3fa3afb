"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``chapsim_oracle.c``) is an FP64 restatement of CHAPSim's
periodic-channel time step (``src/SOLVERRK3_MOM_tg.f90`` and the routines it
calls).  It is used by ``tests/`` as the checker, by the smoke check, and by
the CPU-baseline leg of ``bench.py``.  The product library never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_chapsim.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    srcs = [os.path.join(_HERE, f) for f in ("chapsim_oracle.c", "thermo_oracle.c", "mlp_oracle.c")]
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(f) for f in srcs)
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [ctypes.c_int] + [ctypes.c_double] * 4
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_fix_v_wall_row.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_get_y.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_get_scalars.argtypes = [ctypes.c_void_p, _dp]
        L.orc_set_fields.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_get_fields.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_get_work.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_set_dt.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_get_dt.argtypes = [ctypes.c_void_p]
        L.orc_get_dt.restype = ctypes.c_double
        L.orc_substep.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_substep.restype = ctypes.c_int
        L.orc_cfl.argtypes = [ctypes.c_void_p]
        L.orc_cfl.restype = ctypes.c_double
        L.orc_step_dt.argtypes = [ctypes.c_void_p, _dp]
        L.orc_step_dt.restype = ctypes.c_int
        L.orc_run_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_run_steps.restype = ctypes.c_int
        L.orc_divgck.argtypes = [ctypes.c_void_p]
        L.orc_divgck.restype = ctypes.c_double
        L.orc_pp_mean_zx_tg.argtypes = [ctypes.c_void_p, _dp]
        L.orc_pp_mean_t_tg.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                       ctypes.POINTER(ctypes.c_int)]
        L.orc_pp_monitor_tg.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_double, _dp]
        L.orc_pp_io_per_row.argtypes = [ctypes.c_void_p]
        L.orc_pp_io_per_row.restype = ctypes.c_int
        L.orc_pp_mean_zx_io.argtypes = [ctypes.c_void_p, _dp]
        L.orc_poisson.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_fft_complex.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.orc_tdma_cyc.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp]
        L.orc_tdma_noncyc.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp]
        L.orc_io_enable.argtypes = [ctypes.c_void_p]
        L.orc_io_set_fields.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.orc_io_get_fields.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_io_substep.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_io_substep.restype = ctypes.c_int
        L.orc_io_cfl.argtypes = [ctypes.c_void_p]
        L.orc_io_cfl.restype = ctypes.c_double
        L.orc_io_run_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_io_run_steps.restype = ctypes.c_int
        L.orc_io_monitor.argtypes = [ctypes.c_void_p, _dp]
        L.orc_io_set_vis_scheme.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_io_set_buoyancy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.orc_io_set_weighted_pressure.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_io_divgck.argtypes = [ctypes.c_void_p]
        L.orc_io_divgck.restype = ctypes.c_double
        L.orc_io_drhoi_maxabs.argtypes = [ctypes.c_void_p]
        L.orc_io_drhoi_maxabs.restype = ctypes.c_double
        L.orc_thermal_enable.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _dp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double]
        L.orc_thermal_enable.restype = ctypes.c_int
        L.orc_thermal_substep.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_thermal_substep.restype = ctypes.c_int
        L.orc_thermal_get.argtypes = [ctypes.c_void_p, _dp]
        L.orc_thermal_set_isothermal.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_thermal_set_isothermal.restype = ctypes.c_int
        _fp = ctypes.POINTER(ctypes.c_float)
        L.orc_mlp_forward.argtypes = [_fp, _dp, ctypes.c_int, _dp, _dp]
        L.orc_mlp_gradients.argtypes = [ctypes.c_void_p, _fp, _dp, ctypes.c_int, _dp, _dp]
        L.orc_mlp_gradients.restype = ctypes.c_double
        L.orc_mlp_set_activation.argtypes = [ctypes.c_int]
        _ip = ctypes.POINTER(ctypes.c_int)
        L.orc_cubic_spline.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
        L.orc_spline_index.argtypes = [ctypes.c_int, _dp, ctypes.c_double]
        L.orc_spline_index.restype = ctypes.c_int
        L.orc_spline_eval.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, _dp]
        L.orc_spline_eval.restype = ctypes.c_int
        L.orc_table_nondim.argtypes = [ctypes.c_int, _dp, ctypes.c_double, _dp, _dp]
        L.orc_table_create.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        L.orc_table_create.restype = ctypes.c_void_p
        L.orc_table_destroy.argtypes = [ctypes.c_void_p]
        L.orc_table_coefs.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_table_extrema.argtypes = [ctypes.c_void_p, _ip]
        L.orc_prop_update.argtypes = [ctypes.c_void_p, ctypes.c_long, _dp, _dp, ctypes.POINTER(ctypes.c_long)]
        L.orc_prop_update.restype = ctypes.c_long
        L.orc_create_xinout.restype = ctypes.c_void_p
        L.orc_create_xinout.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 7
        L.orc_xio_substep.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.orc_xio_substep.restype = ctypes.c_int
        L.orc_xio_run_steps.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_xio_run_steps.restype = ctypes.c_int
        L.orc_xio_divgck.argtypes = [ctypes.c_void_p, _dp]
        L.orc_xio_outlet_state.argtypes = [ctypes.c_void_p, _dp]
        L.orc_xio_poisson.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_xio_akx.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_xio_akx.restype = ctypes.c_double
        L.orc_xio_akz.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_xio_akz.restype = ctypes.c_double
        L.orc_xio_thermal_inlet.argtypes = [ctypes.c_void_p, _dp]
        L.orc_xio_thermal_inlet.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class Oracle:
    """CPU FP64 periodic-channel solver (test checker).

    Fields use the reference layout: ``Q`` has shape (3, N, M+2, L) in C order,
    i.e. Fortran ``Q_tg(L, 0:M+1, N, 3)``; ``PR`` is (N, M+2, L).
    """

    Y_NAMES = {"YND": 0, "YCC": 1, "DYFI": 2, "DYCI": 3, "WFF": 4, "WFB": 5, "AMPH": 6, "ACPH": 7,
               "APPH": 8, "AMVR": 9, "ACVR": 10, "APVR": 11, "Vini": 12}

    def __init__(self, L, M, N, HX, HZ, STR2, REN, iFlowDriven=1, Cf_Given=8.18e-3, DT0=1e-3, DTMIN=1e-6,
                 CFLGV=0.5, threads=1):
        self.L, self.M, self.N = L, M, N
        self._lib = lib()
        self._h = self._lib.orc_create(L, M, N, HX, HZ, STR2, REN, iFlowDriven, Cf_Given, DT0, DTMIN, CFLGV)
        if not self._h:
            raise ValueError("invalid oracle grid")
        self._lib.orc_set_threads(self._h, int(threads))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.orc_destroy(self._h)
            self._h = None

    __del__ = close

    def set_fix_v_wall_row(self, flag: bool):
        self._lib.orc_set_fix_v_wall_row(self._h, int(bool(flag)))

    def y(self, name, idr=1):
        n = self.M + 1
        out = np.zeros(n, np.float64)
        self._lib.orc_get_y(self._h, self.Y_NAMES[name], idr, _p(out))
        if name in ("YCC", "DYFI", "AMPH", "ACPH", "APPH", "Vini"):
            return out[: self.M]
        return out

    def scalars(self):
        s = np.zeros(12, np.float64)
        self._lib.orc_get_scalars(self._h, _p(s))
        keys = ["DX", "DZ", "DXI", "DZI", "DXQI", "DZQI", "VOLM", "Area_inlet", "AMVR1", "APVRN", "CVISC", "DT"]
        return dict(zip(keys, s.tolist()))

    def field_shape(self):
        return (self.N, self.M + 2, self.L)

    def set_fields(self, Q, PR, H0=None):
        Q = np.ascontiguousarray(Q, np.float64)
        PR = np.ascontiguousarray(PR, np.float64)
        assert Q.shape == (3,) + self.field_shape() and PR.shape == self.field_shape()
        if H0 is None:
            self._lib.orc_set_fields(self._h, _p(Q), _p(PR), None)
        else:
            H0 = np.ascontiguousarray(H0, np.float64)
            self._lib.orc_set_fields(self._h, _p(Q), _p(PR), _p(H0))

    def get_fields(self):
        Q = np.zeros((3,) + self.field_shape())
        PR = np.zeros(self.field_shape())
        H0 = np.zeros((3,) + self.field_shape())
        self._lib.orc_get_fields(self._h, _p(Q), _p(PR), _p(H0))
        return Q, PR, H0

    def work(self, which):
        out = np.zeros(self.field_shape())
        self._lib.orc_get_work(self._h, {"DPH": 0, "RHSLLPHI": 1, "RHS": 2, "QTMP": 3}[which], _p(out))
        return out

    def set_dt(self, dt):
        self._lib.orc_set_dt(self._h, float(dt))

    def dt(self):
        return self._lib.orc_get_dt(self._h)

    def substep(self, ns):
        if self._lib.orc_substep(self._h, int(ns)) != 0:
            raise ValueError("bad substep index")

    def cfl(self):
        return self._lib.orc_cfl(self._h)

    def step_dt(self):
        dt = ctypes.c_double()
        rc = self._lib.orc_step_dt(self._h, ctypes.byref(dt))
        return dt.value, rc

    def run_steps(self, n):
        dts = np.zeros(max(n, 1))
        rc = self._lib.orc_run_steps(self._h, int(n), _p(dts))
        return rc, dts[:n]

    def divgck(self):
        return self._lib.orc_divgck(self._h)

    # ---- statistics of the periodic channel (POSTPROCESS_TG) ----
    # A set of x-z means is a flat array of 122*M doubles: U1xzL(M,4), UPxzL(M,3),
    # U2xzL(M,6), U3xzL(M,10), DVDL1xzL(M,3,3), DVDLPxzL(M,3,3), DVDL2xzL(M,9,9) (Fortran order).
    def pp_mean_zx_tg(self):
        out = np.zeros(122 * self.M)
        self._lib.orc_pp_mean_zx_tg(self._h, _p(out))
        return out

    def pp_mean_t_tg(self, tp, inst, avg, nstatis, pp_instn_sz=1):
        """PP_MEAN_T_TG: updates avg in place; returns the new NSTATIS."""
        n = ctypes.c_int(int(nstatis))
        self._lib.orc_pp_mean_t_tg(self.M, int(tp), int(pp_instn_sz), _p(inst), _p(avg), ctypes.byref(n))
        return n.value

    # ---- statistics of the main domain (PP_MEAN_ZX_FLOW_Xperiodic_io) ----
    # One set is a flat array of 141*M doubles (flow) or 360*M (with the thermal solver), the
    # module arrays in the order the reference zeroes them (Fortran order, j fastest).
    def pp_mean_zx_io(self):
        out = np.zeros(self._lib.orc_pp_io_per_row(self._h) * self.M)
        self._lib.orc_pp_mean_zx_io(self._h, _p(out))
        return out

    def pp_monitor_tg(self, inst, avg, ren):
        mon = np.zeros(20)
        self._lib.orc_pp_monitor_tg(self._h, _p(inst), _p(avg), float(ren), _p(mon))
        return mon

    # ---- IO (main-domain) path, explicit (iVisScheme 0) or Crank-Nicolson (1) viscous terms ----
    def io_set_vis_scheme(self, ivis):
        self._lib.orc_io_set_vis_scheme(self._h, int(ivis))

    def io_set_buoyancy(self, igravity, f_a):
        """thermal_gravity: the buoyancy term D_STG * TALP*DT*F_A on component |iGravity|."""
        self._lib.orc_io_set_buoyancy(self._h, int(igravity), float(f_a))

    def io_set_weighted_pressure(self, pr0_1=None, pr0_2=None):
        """iWeightedPre = 1 with the two PR0_io layers (padded (N, M+2, L)); None turns it off."""
        if pr0_1 is None:
            self._lib.orc_io_set_weighted_pressure(self._h, None, None)
            return
        a = np.ascontiguousarray(pr0_1, np.float64)
        b = np.ascontiguousarray(pr0_2 if pr0_2 is not None else pr0_1, np.float64)
        assert a.shape == self.field_shape() and b.shape == self.field_shape()
        self._lib.orc_io_set_weighted_pressure(self._h, _p(a), _p(b))

    def io_drhoi_maxabs(self):
        return self._lib.orc_io_drhoi_maxabs(self._h)

    def io_set_fields(self, G, PR, RHO, MU0, MU):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (G, PR, RHO, MU0, MU)]
        assert arrs[0].shape == (3,) + self.field_shape()
        self._lib.orc_io_set_fields(self._h, *[_p(a) for a in arrs])

    def io_get_fields(self):
        G = np.zeros((3,) + self.field_shape())
        Q = np.zeros((3,) + self.field_shape())
        PR = np.zeros(self.field_shape())
        self._lib.orc_io_get_fields(self._h, _p(G), _p(Q), _p(PR))
        return G, Q, PR

    def io_substep(self, ns):
        if self._lib.orc_io_substep(self._h, int(ns)) != 0:
            raise ValueError("bad substep or IO path not enabled")

    def io_divgck(self):
        return self._lib.orc_io_divgck(self._h)

    def io_cfl(self):
        return self._lib.orc_io_cfl(self._h)

    def io_run_steps(self, n):
        cdt = np.zeros(max(n, 1))
        rc = self._lib.orc_io_run_steps(self._h, int(n), _p(cdt))
        return rc, cdt[:n]

    def io_monitor(self):
        out = np.zeros(5)
        self._lib.orc_io_monitor(self._h, _p(out))
        return dict(zip(["Uc", "UUc", "UVc", "Gmaxx", "Gbulk"], out.tolist()))

    # ---- thermal solver of the IO domain (table-search properties) ----
    def thermal_enable(self, table, DH, qw_bot, qw_top, cthecd):
        """table: a PropTable; DH: padded (N, M+2, L) rho*h field (rows 1..M used)."""
        DH = np.ascontiguousarray(DH, np.float64)
        self._table = table
        rc = self._lib.orc_thermal_enable(self._h, table._h, _p(DH), float(qw_bot), float(qw_top), float(cthecd))
        if rc != 0:
            raise ValueError("thermal start-up failed (DH outside the property table)")

    def thermal_set_isothermal(self, wall, state=None):
        """BC_Fixed_Temperature on wall 0 (bottom) or 1 (top) with the wall state (T, H, D, M, K);
        None returns that wall to the constant heat flux."""
        v = None if state is None else np.ascontiguousarray(state, np.float64)
        if self._lib.orc_thermal_set_isothermal(self._h, int(wall), None if v is None else _p(v)) != 0:
            raise ValueError("thermal solver not enabled, bad wall, or a point outside the table")

    def thermal_substep(self, ns):
        return self._lib.orc_thermal_substep(self._h, int(ns))

    def thermal_get(self):
        out = np.zeros((7,) + self.field_shape())
        self._lib.orc_thermal_get(self._h, _p(out))
        return dict(zip(["DH", "H", "T", "D", "M", "K", "CP"], out))

    def poisson(self, rhs):
        rhs = np.ascontiguousarray(rhs, np.float64)
        out = np.zeros(self.field_shape())
        self._lib.orc_poisson(self._h, _p(rhs), _p(out))
        return out


class OracleXinout(Oracle):
    """Main domain of a TG + main-domain run (iDomain = 3) with inflow from a periodic TG
    domain and a convective outlet; explicit viscous terms; the thermal solver after
    ``thermal_enable`` and ``xio_thermal_inlet``.

    Fields carry the x ghost columns: shape (N, M+2, L+2) = Fortran (0:L+1, 0:M+1, N), i.e.
    ``NCL1S:NCL1E``.  The TG domain is an :class:`Oracle` with the same M, N and y mesh.
    """

    def __init__(self, L, M, N, HX, HZ, STR2, REN, DT0=1e-3, DTMIN=1e-6, CFLGV=0.5, threads=1):
        self.L, self.M, self.N = L, M, N
        self._lib = lib()
        self._h = self._lib.orc_create_xinout(L, M, N, HX, HZ, STR2, REN, DT0, DTMIN, CFLGV)
        if not self._h:
            raise ValueError("invalid oracle grid")
        self._lib.orc_set_threads(self._h, int(threads))

    def field_shape(self):
        return (self.N, self.M + 2, self.L + 2)

    def xio_substep(self, tg: Oracle, ns):
        if self._lib.orc_xio_substep(self._h, tg._h, int(ns)) != 0:
            raise ValueError("bad substep, TG domain mismatch or fields not set")

    def xio_run_steps(self, tg: Oracle, n):
        out = np.zeros(max(n, 1))
        rc = self._lib.orc_xio_run_steps(self._h, tg._h, int(n), _p(out))
        return rc, out[:n]

    def xio_divgck(self):
        out = np.zeros(3)
        self._lib.orc_xio_divgck(self._h, _p(out))
        return out

    def xio_outlet_state(self):
        """(U_OUTLET, CHK_Mass_CONSV0_SCALING) of the last substep."""
        out = np.zeros(2)
        self._lib.orc_xio_outlet_state(self._h, _p(out))
        return tuple(out.tolist())

    def xio_poisson(self, rhs):
        rhs = np.ascontiguousarray(rhs, np.float64)
        assert rhs.shape == self.field_shape()
        out = np.zeros(self.field_shape())
        self._lib.orc_xio_poisson(self._h, _p(rhs), _p(out))
        return out

    def xio_thermal_inlet(self, state7):
        """BC_TINLET_THERML's inlet state (T, H, D, M, K, CP, DH), applied at once and every substep."""
        v = np.ascontiguousarray(state7, np.float64)
        if self._lib.orc_xio_thermal_inlet(self._h, _p(v)) != 0:
            raise ValueError("thermal solver not enabled")

    def akx(self):
        return np.array([self._lib.orc_xio_akx(self._h, i) for i in range(1, self.L + 1)])

    def akz(self):
        return np.array([self._lib.orc_xio_akz(self._h, k) for k in range(self.N)])


def fft_complex(x: np.ndarray, sign: int) -> np.ndarray:
    re = np.ascontiguousarray(x.real, np.float64).copy()
    im = np.ascontiguousarray(x.imag, np.float64).copy()
    lib().orc_fft_complex(len(x), _p(re), _p(im), int(sign))
    return re + 1j * im


def tdma_cyc(A, B, C, R):
    R = np.array(R, np.float64)
    lib().orc_tdma_cyc(len(R), _p(np.ascontiguousarray(A, np.float64)), _p(np.ascontiguousarray(B, np.float64)),
                       _p(np.ascontiguousarray(C, np.float64)), _p(R))
    return R


def tdma_noncyc(A, B, C, R):
    R = np.array(R, np.float64)
    lib().orc_tdma_noncyc(len(R), _p(np.ascontiguousarray(A, np.float64)), _p(np.ascontiguousarray(B, np.float64)),
                          _p(np.ascontiguousarray(C, np.float64)), _p(R))
    return R


# ---- property update by table search (thermo_oracle.c) ----
SPLINES = ["DHH", "HT", "HD", "HM", "HK", "HCP", "HB"]
LIST_NAMES = ["H", "T", "D", "M", "K", "CP", "B", "DH"]


def cubic_spline(x, y):
    """CUBIC_SPLINE(N, X, Y, B, C, D); returns (B, C, D)."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    n = len(x)
    b, c, d = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().orc_cubic_spline(n, _p(x), _p(y), _p(b), _p(c), _p(d))
    return b, c, d


def table_nondim(raw, T0):
    """Property_Table_Nondimensionalization of raw (n, 8) rows; returns
    (lists dict H..DH, reference state dict H0, D0, K0, M0, CP0, B0)."""
    raw = np.ascontiguousarray(raw, np.float64)
    n = raw.shape[0]
    lists = np.zeros(8 * n)
    ref = np.zeros(6)
    lib().orc_table_nondim(n, _p(raw), float(T0), _p(lists), _p(ref))
    return ({k: lists[i * n:(i + 1) * n].copy() for i, k in enumerate(LIST_NAMES)},
            dict(zip(["H0", "D0", "K0", "M0", "CP0", "B0"], ref.tolist())))


class PropTable:
    """Table with its spline coefficients; update() is THERM_PROP_UPDATE_FROM_DH (table arm)."""

    def __init__(self, lists, fix_swap=False):
        self.n = len(lists["H"])
        self._buf = np.ascontiguousarray(np.concatenate([lists[k] for k in LIST_NAMES]), np.float64)
        self._h = lib().orc_table_create(self.n, _p(self._buf), int(bool(fix_swap)))
        if not self._h:
            raise ValueError("table needs at least 4 rows")

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_table_destroy(self._h)
            self._h = None

    __del__ = close

    def coefs(self, name):
        out = np.zeros(3 * self.n)
        lib().orc_table_coefs(self._h, SPLINES.index(name), _p(out))
        return out.reshape(3, self.n)

    def extrema(self):
        out = (ctypes.c_int * 4)()
        lib().orc_table_extrema(self._h, out)
        return dict(zip(["imin_h", "imax_h", "imin_dh", "imax_dh"], list(out)))

    def update(self, dh):
        """Returns (dict of H, T, D, M, K, CP arrays shaped like dh, number of
        out-of-range points, first out-of-range flat index or -1)."""
        dh = np.ascontiguousarray(dh, np.float64)
        flat = dh.reshape(-1)
        out = np.zeros(6 * flat.size)
        fb = ctypes.c_long(-1)
        nbad = lib().orc_prop_update(self._h, flat.size, _p(flat), _p(out), ctypes.byref(fb))
        res = {k: out[i * flat.size:(i + 1) * flat.size].reshape(dh.shape) for i, k in
               enumerate(["H", "T", "D", "M", "K", "CP"])}
        return res, nbad, fb.value


# ---- learned property model (mlp_oracle.c) ----
MLP_NPARAM = 64 + 64 + 64 * 64 + 64 + 6 * 64 + 6


def mlp_set_activation(act):
    """0: tanh, 1: the clamped cubic (applies to mlp_forward and mlp_gradients)."""
    lib().orc_mlp_set_activation(int(act))


def mlp_forward(params, norm, dh):
    p = np.ascontiguousarray(params, np.float32)
    nm = np.ascontiguousarray(norm, np.float64)
    dh = np.ascontiguousarray(dh, np.float64)
    out = np.zeros(6 * dh.size)
    lib().orc_mlp_forward(p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _p(nm), dh.size, _p(dh), _p(out))
    return dict(zip(["H", "T", "D", "M", "K", "CP"], out.reshape(6, dh.size)))


def mlp_gradients(table, params, norm, dh):
    p = np.ascontiguousarray(params, np.float32)
    nm = np.ascontiguousarray(norm, np.float64)
    dh = np.ascontiguousarray(dh, np.float64)
    g = np.zeros(MLP_NPARAM)
    loss = lib().orc_mlp_gradients(table._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _p(nm), dh.size,
                                   _p(dh), _p(g))
    return g, loss
