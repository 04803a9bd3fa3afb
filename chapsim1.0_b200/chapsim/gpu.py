"""ctypes binding of libchapsim_gpu.so and a host-side mirror of CHAPSim's
subroutine interface for the periodic-channel time step.

Method names follow the Fortran subroutines they replace; arguments keep the
reference's meaning (NS = RK substep 0..3, DT0/DTMIN/CFLGV from readdata.ini)
and a nonzero status raises :class:`ChapsimError`, the counterpart of
``CALL ERRHDL`` (src/WRTHDL.f90:48-63, log + STOP).  There is no CPU
fallback: if the CUDA library is missing, construction fails.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .mesh import ChannelSetup, channel_setup

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CHAPSIM_GPU_LIB", os.path.join(_HERE, "libchapsim_gpu.so"))

_dp = ctypes.POINTER(ctypes.c_double)

ERR_NAMES = {0: "CHAPSIM_OK", -1: "CHAPSIM_ERR_CUDA", -2: "CHAPSIM_ERR_NAN", -3: "CHAPSIM_ERR_DT_COLLAPSE",
             -4: "CHAPSIM_ERR_TABLE_RANGE", -5: "CHAPSIM_ERR_TIMEOUT", -6: "CHAPSIM_ERR_BADARG",
             -7: "CHAPSIM_ERR_NOMEM"}

MLP_TANH, MLP_CUBIC = 0, 1

EXPORTED = ["chapsim_gpu_init", "chapsim_gpu_finalize", "chapsim_last_error_string", "chapsim_upload_fields",
            "chapsim_download_fields", "chapsim_upload_fields_async", "chapsim_download_fields_async", "chapsim_io_wait", "chapsim_set_dt", "chapsim_get_dt", "chapsim_cfl_tg", "chapsim_step_begin",
            "chapsim_rk_substep_tg", "chapsim_advance_tg", "chapsim_divgck_tg", "chapsim_fft99_pois3d",
            "chapsim_tdmaiji_cyc", "chapsim_tdmaijj_noncyc", "chapsim_upload_io_fields",
            "chapsim_download_io_fields", "chapsim_rk_substep_io", "chapsim_cfl_io", "chapsim_profile_steps",
            "chapsim_get_stream",
            "chapsim_sync", "chapsim_launch_count", "chapsim_kernels_per_step", "chapsim_tdma_lines_noalloc",
            "chapsim_prop_table_init", "chapsim_therm_prop_update_points", "chapsim_thermal_init",
            "chapsim_download_thermal_fields", "chapsim_mlp_init", "chapsim_mlp_set_params", "chapsim_mlp_get_params",
            "chapsim_mlp_gradients", "chapsim_mlp_train", "chapsim_mlp_infer_points", "chapsim_thermal_use_mlp",
            "chapsim_mlp_judge", "chapsim_autotune", "chapsim_batch_create", "chapsim_batch_advance",
            "chapsim_set_buoyancy", "chapsim_upload_weighted_pressure",
            "chapsim_batch_get_stream", "chapsim_batch_destroy", "chapsim_pp_mean_zx_tg", "chapsim_pp_mean_t_tg",
            "chapsim_pp_monitor_tg", "chapsim_download_pp_means_tg", "chapsim_upload_pp_means_tg", "chapsim_divgck_io",
            "chapsim_pp_mean_zx_io", "chapsim_download_pp_means_io",
            "chapsim_write_dfile", "chapsim_read_dfile", "chapsim_dump_begin", "chapsim_dump_write",
            "chapsim_mlp_set_activation", "chapsim_probe_wait_timeout", "chapsim_thermal_set_isothermal", "chapsim_xinout_thermal_inlet", "chapsim_xinout_attach", "chapsim_advance_xinout", "chapsim_divgck_xinout", "chapsim_xinout_outlet_state"]

# the arrays of one set of x-z means (postprocess_info), their widths per y row
PP_ARRAYS = [("U1xzL", 4), ("UPxzL", 3), ("U2xzL", 6), ("U3xzL", 10), ("DVDL1xzL", 9), ("DVDLPxzL", 9), ("DVDL2xzL", 81)]
PP_MONITOR = ["U1c", "U1c_t", "U2c", "U2c_t", "U3c", "U3c_t", "uu", "uu_t", "uv", "uv_t", "vv", "vv_t", "ww", "ww_t",
              "Cf_bottom", "Cf_bottom_t", "Cf_top", "Cf_top_t", "U1mean", "U1maxx"]

KERNEL_SLOTS = ["k_cfl", "k_dt_factors"] + ["k_rhs_xsweep", "k_zsweep", "k_ysweep", "k_div_fftx", "k_fftz_fwd", "k_ysolve",
                                    "k_fftz_inv", "k_fftx_inv", "k_correct"] * 3


# (n1, n2) split of the supported FFT lengths (csrc/fft.cuh: fft4s_split)
FFT_SPLIT = {32: (4, 8), 64: (8, 8), 96: (12, 8), 128: (16, 8), 192: (16, 12), 256: (16, 16), 384: (16, 24)}


def plane_in_one_block(L, N, precision="fp64"):
    """True when the fused plane transforms of an (L, N) plane run as one block
    (k_div_fft2 / k_fft2_inv), False when they run as a thread-block cluster
    (k_div_fft2c / k_fft2c_inv): the rule of plane_fft_ok in csrc/chapsim_gpu.cu."""
    if L not in (64, 96, 128, 192) or N not in (64, 96, 128, 192):
        return False
    words = max((N // 2) * (L + FFT_SPLIT[L][1] + 1), (L // 2 + 1) * (N + FFT_SPLIT[N][1] + 1))
    return words * (16 if precision == "fp64" else 8) <= 220 * 1024


def step_kernel_slots(choice: int = 0, plane_cluster: bool = False):
    """Names of the kernels in the profiling slots of one periodic-channel step
    for the variant bits `choice` of chapsim_autotune.  The split right-hand
    side times k_rhs_point and k_xsweep in one slot; with the fused plane
    transforms (one block per row, or a cluster per row when plane_cluster)
    the two z-transform slots stay empty and are named None."""
    rhs = {0: "k_rhs_xsweep", 1: "k_rhs_point+k_xsweep", 2: "k_rhs_xsweep_bulk", 3: "k_rhs_xsweep"}[(choice >> 1) & 3]
    if choice & 1:
        ys = "k_ysolve_seq"
    elif choice & 16:
        ys = "k_ysolve_2w"
    elif choice & 32:
        ys = "k_ysolve_seq"
    elif choice & 64:
        ys = "k_ysolve_scan"
    else:
        ys = "k_ysolve_warp"
    if choice & 8 and plane_cluster:
        pre = ["k_div_fft2c", None, ys, None, "k_fft2c_inv"]
    elif choice & 8:
        pre = ["k_div_fft2", None, ys, None, "k_fft2_inv"]
    else:
        pre = ["k_div_fftx", "k_fftz_fwd", ys, "k_fftz_inv", "k_fftx_inv"]
    return ["k_cfl", "k_dt_factors"] + ([rhs, "k_zsweep", "k_ysweep"] + pre + ["k_correct"]) * 3


class ChapsimError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Grid(ctypes.Structure):
    _fields_ = [("ncl1", ctypes.c_int32), ("ncl2", ctypes.c_int32), ("ncl3", ctypes.c_int32),
                ("icase", ctypes.c_int32), ("idomain", ctypes.c_int32)]


class Coefs(ctypes.Structure):
    _fields_ = [("dxi", ctypes.c_double), ("dzi", ctypes.c_double), ("dxqi", ctypes.c_double),
                ("dzqi", ctypes.c_double), ("cvisc", ctypes.c_double), ("volm", ctypes.c_double),
                ("cf_given", ctypes.c_double), ("iflowdriven", ctypes.c_int32), ("pad0", ctypes.c_int32),
                ("dyfi", _dp), ("dyci", _dp), ("ycl2nd_wff", _dp), ("ycl2nd_wfb", _dp), ("amph", _dp),
                ("acph", _dp), ("apph", _dp), ("amvr", _dp), ("acvr", _dp), ("apvr", _dp), ("ak1", _dp),
                ("ak3", _dp), ("tgam", ctypes.c_double * 4), ("troh", ctypes.c_double * 4),
                ("talp", ctypes.c_double * 4), ("amvr1", ctypes.c_double), ("apvrn", ctypes.c_double)]


class PropTableC(ctypes.Structure):
    _fields_ = ([("n_list", ctypes.c_int32), ("fix_swap", ctypes.c_int32)] +
                [(f"list_{n}", _dp) for n in ("h", "t", "d", "m", "k", "cp", "dh")] +
                [(f"{s}_{c}", _dp) for s in ("dhh", "ht", "hd", "hm", "hk", "hcp") for c in ("b", "c", "d")])


PREC_FP64, PREC_MIXED = 0, 1
PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED}


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("fix_v_wall_row", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("ivisscheme", ctypes.c_int32), ("no_pdl", ctypes.c_int32), ("reserved", ctypes.c_int32 * 3)]


VIS_EXPLICIT, VIS_IMPLICIT = 0, 1


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libchapsim_gpu.so not built ({path}); run `make -C chapsim1.0_b200`")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.chapsim_gpu_init.argtypes = [ctypes.POINTER(Grid), ctypes.POINTER(Coefs), ctypes.POINTER(Opts),
                                   ctypes.POINTER(vp)]
    L.chapsim_gpu_finalize.argtypes = [vp]
    L.chapsim_last_error_string.argtypes = [vp]
    L.chapsim_last_error_string.restype = ctypes.c_char_p
    L.chapsim_upload_fields.argtypes = [vp, _dp, _dp, _dp]
    L.chapsim_download_fields.argtypes = [vp, _dp, _dp, _dp]
    L.chapsim_upload_fields_async.argtypes = [vp, _dp, _dp]
    L.chapsim_download_fields_async.argtypes = [vp, _dp, _dp]
    L.chapsim_io_wait.argtypes = [vp]
    L.chapsim_set_dt.argtypes = [vp, ctypes.c_double]
    L.chapsim_get_dt.argtypes = [vp, _dp]
    L.chapsim_cfl_tg.argtypes = [vp, _dp]
    L.chapsim_step_begin.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp]
    L.chapsim_rk_substep_tg.argtypes = [vp, ctypes.c_int32]
    L.chapsim_advance_tg.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp]
    L.chapsim_divgck_tg.argtypes = [vp, _dp]
    L.chapsim_fft99_pois3d.argtypes = [vp, _dp, _dp]
    L.chapsim_tdmaiji_cyc.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int32, ctypes.c_int32]
    L.chapsim_tdmaijj_noncyc.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int32, ctypes.c_int32]
    L.chapsim_prop_table_init.argtypes = [vp, ctypes.POINTER(PropTableC)]
    L.chapsim_therm_prop_update_points.argtypes = [vp, ctypes.c_int64] + [_dp] * 7
    L.chapsim_thermal_init.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.chapsim_download_thermal_fields.argtypes = [vp] + [_dp] * 7
    _fp = ctypes.POINTER(ctypes.c_float)
    L.chapsim_mlp_init.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_uint64]
    L.chapsim_mlp_set_params.argtypes = [vp, _fp]
    L.chapsim_mlp_get_params.argtypes = [vp, _fp, _dp]
    L.chapsim_mlp_gradients.argtypes = [vp, ctypes.c_int32, _dp, _fp, _dp]
    L.chapsim_mlp_train.argtypes = [vp, ctypes.c_int32, _dp, ctypes.c_int32, ctypes.c_float, _dp]
    L.chapsim_mlp_infer_points.argtypes = [vp, ctypes.c_int64] + [_dp] * 7
    L.chapsim_thermal_use_mlp.argtypes = [vp, ctypes.c_int32]
    L.chapsim_mlp_judge.argtypes = [vp, _dp]
    L.chapsim_autotune.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)]
    L.chapsim_divgck_io.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    i32 = ctypes.c_int32
    L.chapsim_write_dfile.argtypes = [ctypes.c_char_p, i32, i32, i32, i32, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, _dp]
    L.chapsim_read_dfile.argtypes = [ctypes.c_char_p, ctypes.POINTER(i32), _dp, _dp, ctypes.c_int64]
    L.chapsim_dump_begin.argtypes = [vp]
    L.chapsim_dump_write.argtypes = [vp, ctypes.c_char_p, i32, ctypes.c_double, ctypes.c_double, _dp]
    L.chapsim_pp_mean_zx_tg.argtypes = [vp]
    L.chapsim_pp_mean_t_tg.argtypes = [vp, ctypes.c_int32, ctypes.c_int32]
    L.chapsim_pp_monitor_tg.argtypes = [vp, ctypes.c_double, _dp]
    L.chapsim_download_pp_means_tg.argtypes = [vp, ctypes.c_int32] + [_dp] * 7 + [ctypes.POINTER(ctypes.c_int32)]
    L.chapsim_upload_pp_means_tg.argtypes = [vp, ctypes.c_int32] + [_dp] * 7
    L.chapsim_pp_mean_zx_io.argtypes = [vp]
    L.chapsim_download_pp_means_io.argtypes = [vp, _dp, ctypes.POINTER(ctypes.c_int32)]
    L.chapsim_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int32, ctypes.POINTER(vp)]
    L.chapsim_batch_advance.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.chapsim_batch_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.chapsim_batch_destroy.argtypes = [vp]
    L.chapsim_tdma_lines_noalloc.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_int32, ctypes.c_int32, vp]
    L.chapsim_upload_io_fields.argtypes = [vp, _dp, _dp, _dp, _dp, _dp]
    L.chapsim_download_io_fields.argtypes = [vp, _dp, _dp, _dp]
    L.chapsim_rk_substep_io.argtypes = [vp, ctypes.c_int32]
    L.chapsim_xinout_attach.argtypes = [vp, vp]
    L.chapsim_mlp_set_activation.argtypes = [vp, ctypes.c_int32]
    L.chapsim_probe_wait_timeout.argtypes = [vp]
    L.chapsim_thermal_set_isothermal.argtypes = [vp, ctypes.c_int32, _dp]
    L.chapsim_xinout_thermal_inlet.argtypes = [vp, _dp]
    L.chapsim_advance_xinout.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp,
                                         _dp]
    L.chapsim_divgck_xinout.argtypes = [vp, _dp]
    L.chapsim_xinout_outlet_state.argtypes = [vp, _dp]
    L.chapsim_cfl_io.argtypes = [vp, _dp]
    L.chapsim_set_buoyancy.argtypes = [vp, ctypes.c_int32, ctypes.c_double]
    L.chapsim_upload_weighted_pressure.argtypes = [vp, _dp, _dp]
    L.chapsim_profile_steps.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_float), ctypes.c_int32]
    L.chapsim_get_stream.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    L.chapsim_sync.argtypes = [vp]
    L.chapsim_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.chapsim_kernels_per_step.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    _lib = L
    return L


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _fortran_cols(arr_idr_j: np.ndarray, M: int) -> np.ndarray:
    """AMVR(1:NND2, 1:3) in Fortran order from a [IDR, j] 1-based table."""
    return np.ascontiguousarray(np.concatenate([arr_idr_j[c, 1:M + 2] for c in (1, 2, 3)]))


def _check_global(rc):
    if rc != 0:
        lib = load_library()
        raise ChapsimError(rc, lib.chapsim_last_error_string(None).decode())


DUMP_FLOW = ["U", "V", "W", "P"]
DUMP_THERMAL = ["T", "D", "H", "M", "K"]   # TEMPERATURE, DENSITY, ENTHALPY, Viscousity, THERMCONDT
DFILE_PREFIX = "DNS_perixz_INSTANT_T"


def es15_9(t):
    """PhyTIME as the reference's file names print it (Fortran ES15.9)."""
    return "%.9E" % float(t)


def write_dfile(path, field_nml, iterg, time, ren, dt):
    """Native .D writer (WRT_INSTANT_VARS_*): field given (N, M, L) C-order, i.e. Fortran (L, M, N)."""
    f = np.ascontiguousarray(field_nml, np.float64)
    N, M, L = f.shape
    _check_global(load_library().chapsim_write_dfile(str(path).encode(), L, M, N, int(iterg), float(time),
                                                     float(ren), float(dt), _ptr(f)))


def read_dfile(path):
    """Native .D reader: returns (field (N, M, L), header dict)."""
    lib = load_library()
    dims = (ctypes.c_int32 * 4)()
    reals = np.zeros(3)
    _check_global(lib.chapsim_read_dfile(str(path).encode(), dims, _ptr(reals), None, 0))
    L, M, N, it = list(dims)
    f = np.empty((N, M, L))
    _check_global(lib.chapsim_read_dfile(str(path).encode(), dims, _ptr(reals), _ptr(f), f.size))
    return f, {"L": L, "M": M, "N": N, "ITERG": it, "time": float(reals[0]), "REN": float(reals[1]),
               "DT": float(reals[2])}


def tdmaiji_cyc(A, B, C, R):
    """TDMAIJI_CYC on (ISZ, JSZ) arrays given as numpy (JSZ, ISZ) C-order (lines along ISZ)."""
    lib = load_library()
    R = np.ascontiguousarray(R, np.float64).copy()
    jsz, isz = R.shape
    arrs = [np.ascontiguousarray(x, np.float64) for x in (A, B, C)]
    _check_global(lib.chapsim_tdmaiji_cyc(_ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(R), isz, jsz))
    return R


def tdmaijj_noncyc(A, B, C, R, BCJ=None):
    """TDMAIJJ_nonCYC on (ISZ, JSZ) arrays given as numpy (JSZ, ISZ) C-order (lines along JSZ);
    BCJ is (2, ISZ) or None."""
    lib = load_library()
    R = np.ascontiguousarray(R, np.float64).copy()
    jsz, isz = R.shape
    arrs = [np.ascontiguousarray(x, np.float64) for x in (A, B, C)]
    bc = None if BCJ is None else np.ascontiguousarray(BCJ, np.float64)
    _check_global(lib.chapsim_tdmaijj_noncyc(_ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(R), _ptr(bc), jsz, isz))
    return R


class ChannelTG:
    """Device-resident periodic plane channel (CHAPSim TG domain).

    Fields use the reference layout: ``Q`` is numpy (3, N, M+2, L) C-order =
    Fortran ``Q_tg(L, 0:M+1, N, 3)``; ``PR`` is (N, M+2, L); ``CONVH0`` is
    (3, N, M, L) = ``CONVH0_tg(L, M, N, 3)``.
    """

    IDOMAIN = 1

    def __init__(self, setup: ChannelSetup, device: int = 0, fix_v_wall_row: bool = False, precision: str = "fp64",
                 ivisscheme: int = VIS_EXPLICIT, pdl: bool = True):
        """precision: "fp64" (every field and operation in FP64) or "mixed" (FP32
        velocity/pressure storage, stencils and CN sweeps; FP64 Poisson solve,
        projection and bulk-flux sums).  ivisscheme: iVisScheme of the main
        domain (0 explicit, 1 Crank-Nicolson); the TG domain accepts 0 only.
        pdl: launch the step's kernels with programmatic dependent launch."""
        self.lib = load_library()
        self.choice = 0  # variant bits in use (chapsim_autotune); the library starts with all zero
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.precision = precision
        self.s = setup
        L, M, N = setup.L, setup.M, setup.N
        self.L, self.M, self.N = L, M, N
        self._keep = {
            "dyfi": np.ascontiguousarray(setup.DYFI[1:M + 1]),
            "dyci": np.ascontiguousarray(setup.DYCI[1:M + 2]),
            "wff": np.ascontiguousarray(setup.WFF[1:M + 2]),
            "wfb": np.ascontiguousarray(setup.WFB[1:M + 2]),
            "amph": np.ascontiguousarray(setup.AMPH[1:M + 1]),
            "acph": np.ascontiguousarray(setup.ACPH[1:M + 1]),
            "apph": np.ascontiguousarray(setup.APPH[1:M + 1]),
            "amvr": _fortran_cols(setup.AMVR, M),
            "acvr": _fortran_cols(setup.ACVR, M),
            "apvr": _fortran_cols(setup.APVR, M),
            "ak1": np.ascontiguousarray(setup.AK1),
            "ak3": np.ascontiguousarray(setup.AK3),
        }
        k = self._keep
        cf = Coefs(setup.DXI, setup.DZI, setup.DXQI, setup.DZQI, setup.CVISC, setup.VOLM, setup.Cf_Given,
                   setup.iFlowDriven, 0, _ptr(k["dyfi"]), _ptr(k["dyci"]), _ptr(k["wff"]), _ptr(k["wfb"]),
                   _ptr(k["amph"]), _ptr(k["acph"]), _ptr(k["apph"]), _ptr(k["amvr"]), _ptr(k["acvr"]),
                   _ptr(k["apvr"]), _ptr(k["ak1"]), _ptr(k["ak3"]), (ctypes.c_double * 4)(*setup.TGAM),
                   (ctypes.c_double * 4)(*setup.TROH), (ctypes.c_double * 4)(*setup.TALP), setup.AMVR1, setup.APVRN)
        g = Grid(L, M, N, 1, self.IDOMAIN)
        o = Opts(device, int(bool(fix_v_wall_row)), PRECISIONS[precision], int(ivisscheme), int(not pdl))
        h = ctypes.c_void_p()
        rc = self.lib.chapsim_gpu_init(ctypes.byref(g), ctypes.byref(cf), ctypes.byref(o), ctypes.byref(h))
        if rc != 0:
            raise ChapsimError(rc, self.lib.chapsim_last_error_string(None).decode())
        self.h = h

    @classmethod
    def create(cls, L, M, N, HX, HZ, STR2, REN, iFlowDriven=1, Cf_Given=8.18e-3, **kw):
        return cls(channel_setup(L, M, N, HX, HZ, STR2, REN, iFlowDriven, Cf_Given), **kw)

    # -- plumbing -------------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            raise ChapsimError(rc, self.lib.chapsim_last_error_string(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.chapsim_gpu_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field_shape(self):
        return (self.N, self.M + 2, self.L)

    def upload(self, Q, PR, CONVH0=None):
        Q = np.ascontiguousarray(Q, np.float64)
        PR = np.ascontiguousarray(PR, np.float64)
        if Q.shape != (3,) + self.field_shape() or PR.shape != self.field_shape():
            raise ValueError("field shape mismatch")
        H = None
        if CONVH0 is not None:
            H = np.ascontiguousarray(CONVH0, np.float64)
            if H.shape != (3, self.N, self.M, self.L):
                raise ValueError("CONVH0 shape mismatch")
        self._check(self.lib.chapsim_upload_fields(self.h, _ptr(Q), _ptr(PR), _ptr(H)))

    def download(self, want_h0=False):
        Q = np.empty((3,) + self.field_shape())
        PR = np.empty(self.field_shape())
        H = np.empty((3, self.N, self.M, self.L)) if want_h0 else None
        self._check(self.lib.chapsim_download_fields(self.h, _ptr(Q), _ptr(PR), _ptr(H)))
        return (Q, PR, H) if want_h0 else (Q, PR)

    def upload_async(self, Q, PR):
        """Pipelined upload (chapsim_upload_fields_async): Q and PR, C-contiguous float64 arrays of
        the field shapes, preferably in pinned memory, stay unchanged until io_wait(); the next
        advance() starts from them."""
        if Q.shape != (3,) + self.field_shape() or PR.shape != self.field_shape():
            raise ValueError("field shape mismatch")
        self._check(self.lib.chapsim_upload_fields_async(self.h, _ptr(Q), _ptr(PR)))

    def download_async(self, Q, PR):
        """Pipelined download (chapsim_download_fields_async) of the current fields into Q and PR,
        complete after io_wait()."""
        if Q.shape != (3,) + self.field_shape() or PR.shape != self.field_shape():
            raise ValueError("field shape mismatch")
        self._check(self.lib.chapsim_download_fields_async(self.h, _ptr(Q), _ptr(PR)))

    def io_wait(self):
        self._check(self.lib.chapsim_io_wait(self.h))

    def set_dt(self, dt):
        self._check(self.lib.chapsim_set_dt(self.h, float(dt)))

    def get_dt(self):
        v = ctypes.c_double()
        self._check(self.lib.chapsim_get_dt(self.h, ctypes.byref(v)))
        return v.value

    def sync(self):
        self._check(self.lib.chapsim_sync(self.h))

    def launch_count(self):
        v = ctypes.c_uint64()
        self._check(self.lib.chapsim_launch_count(self.h, ctypes.byref(v)))
        return int(v.value)

    def kernels_per_step(self):
        v = ctypes.c_int32()
        self._check(self.lib.chapsim_kernels_per_step(self.h, ctypes.byref(v)))
        return int(v.value)

    # -- reference interface ---------------------------------------------------
    def CFL_tg(self):
        v = ctypes.c_double()
        self._check(self.lib.chapsim_cfl_tg(self.h, ctypes.byref(v)))
        return v.value

    def step_begin(self, DT0, DTMIN, CFLGV):
        dt, cfl = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.chapsim_step_begin(self.h, DT0, DTMIN, CFLGV, ctypes.byref(dt), ctypes.byref(cfl)))
        return dt.value, cfl.value

    def SOLVERRK3_MOM_tg(self, NS):
        self._check(self.lib.chapsim_rk_substep_tg(self.h, int(NS)))

    def advance(self, nsteps, DT0, DTMIN, CFLGV):
        dt, cfl = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.chapsim_advance_tg(self.h, int(nsteps), DT0, DTMIN, CFLGV, ctypes.byref(dt),
                                                ctypes.byref(cfl)))
        return dt.value, cfl.value

    # -- statistics (POSTPROCESS_TG) -----------------------------------------------
    def PP_MEAN_ZX_FLOW_TG(self):
        self._check(self.lib.chapsim_pp_mean_zx_tg(self.h))

    def PP_MEAN_T_TG(self, TP=1, pp_instn_sz=1):
        self._check(self.lib.chapsim_pp_mean_t_tg(self.h, int(TP), int(pp_instn_sz)))

    def PP_MONITOR_TG(self, REN):
        """dict of the monitor quantities (instantaneous and time-averaged, at j = NCL2/2), Cf and U1mean."""
        mon = np.zeros(20)
        self._check(self.lib.chapsim_pp_monitor_tg(self.h, float(REN), _ptr(mon)))
        return dict(zip(PP_MONITOR, mon.tolist()))

    def download_pp_means(self, averaged=False):
        """(flat set of 122*M doubles in the order of PP_ARRAYS, NSTATIS_TG)"""
        M = self.M
        flat = np.zeros(122 * M)
        ptrs, o = [], 0
        for _, w in PP_ARRAYS:
            ptrs.append(_ptr(flat[o * M:(o + w) * M]))
            o += w
        n = ctypes.c_int32()
        self._check(self.lib.chapsim_download_pp_means_tg(self.h, int(bool(averaged)), *ptrs, ctypes.byref(n)))
        return flat, n.value

    @staticmethod
    def pp_split(flat, M):
        """dict name -> numpy array of the Fortran shape (M, w) given as (w, M) (j fastest)."""
        out, o = {}, 0
        for name, w in PP_ARRAYS:
            out[name] = flat[o * M:(o + w) * M].reshape(w, M)
            o += w
        return out

    def kernel_slots(self):
        """Names of the kernels in the slots of one step, in the order
        chapsim_profile_steps reports them, for the variants in use."""
        return step_kernel_slots(self.choice, not plane_in_one_block(self.L, self.N, self.precision))

    def profile_steps(self, nsteps, DT0, DTMIN, CFLGV):
        """Per-kernel durations (ms, summed over nsteps) keyed by the name of the
        kernel that ran (empty slots are left out)."""
        slots = self.kernel_slots()
        n = len(slots)
        buf = (ctypes.c_float * n)()
        self._check(self.lib.chapsim_profile_steps(self.h, int(nsteps), DT0, DTMIN, CFLGV, buf, n))
        out = {}
        for name, v in zip(slots, buf):
            if name is not None:
                out[name] = out.get(name, 0.0) + float(v)
        return out

    def stream_handle(self):
        v = ctypes.c_void_p()
        self._check(self.lib.chapsim_get_stream(self.h, ctypes.byref(v)))
        return v.value or 0

    def dump_begin(self):
        """Snapshot U, V, W, P (and the thermal fields) now; the copy to the host
        overlaps the steps launched next (chapsim_dump_begin)."""
        self._check(self.lib.chapsim_dump_begin(self.h))

    def dump_write(self, path_prefix, iterg, time, ren):
        """Writes the snapshot as .D files <path_prefix><time ES15.9>_X.D; returns the
        snapshot's dt (chapsim_dump_write)."""
        dt = ctypes.c_double()
        self._check(self.lib.chapsim_dump_write(self.h, str(path_prefix).encode(), int(iterg), float(time),
                                                float(ren), ctypes.byref(dt)))
        return dt.value

    def WRT_INSTANT_VARS(self, file_path, iterg, time, ren, prefix=DFILE_PREFIX):
        """WRT_INSTANT_VARS_TG / _FLOW_IO (+ _THERMAL_IO): dump and write now; returns the file stem."""
        self.dump_begin()
        self.dump_write(str(file_path) + prefix, iterg, time, ren)
        return str(file_path) + prefix + es15_9(time)

    def restart_from_dfiles(self, stem):
        """ReStart_INSTANT_VARS_TG: reads <stem>_U.D, _V.D, _W.D, _P.D, uploads the
        fields (ghost planes zero, then the wall conditions of the upload) and the
        files' DT; returns the header of the U file."""
        M = self.M
        Q = np.zeros((3,) + self.field_shape())
        PR = np.zeros(self.field_shape())
        hdr = None
        for c, x in enumerate(DUMP_FLOW):
            f, h = read_dfile(f"{stem}_{x}.D")
            if (h["L"], h["M"], h["N"]) != (self.L, self.M, self.N):
                raise ValueError(f"{stem}_{x}.D: grid {h['L']}x{h['M']}x{h['N']} is not this context's")
            if c < 3:
                Q[c, :, 1:M + 1, :] = f
            else:
                PR[:, 1:M + 1, :] = f
            hdr = hdr or h
        self.upload(Q, PR)
        self.set_dt(hdr["DT"])
        return hdr

    def DIVGCK_tg(self):
        v = ctypes.c_double()
        self._check(self.lib.chapsim_divgck_tg(self.h, ctypes.byref(v)))
        return v.value

    def FFT99_POIS3D_periodicxz(self, rhs_nml):
        rhs = np.ascontiguousarray(rhs_nml, np.float64)
        if rhs.shape != (self.N, self.M, self.L):
            raise ValueError("RHSLLPHI shape mismatch")
        out = np.zeros(self.field_shape())
        self._check(self.lib.chapsim_fft99_pois3d(self.h, _ptr(rhs), _ptr(out)))
        return out


    # -- thermophysical properties (table search) --------------------------------
    def prop_table_init(self, table, fix_swap=False):
        """Uploads a ``chapsim.thermo.SplineTable`` (nondimensional lists and coefficients)."""
        li, co = table.lists, table.coef
        keep = {f"list_{n.lower()}": np.ascontiguousarray(li[n], np.float64)
                for n in ("H", "T", "D", "M", "K", "CP", "DH")}
        for s, key in (("dhh", "DHH"), ("ht", "HT"), ("hd", "HD"), ("hm", "HM"), ("hk", "HK"), ("hcp", "HCP")):
            for c, arr in zip("bcd", co[key]):
                keep[f"{s}_{c}"] = np.ascontiguousarray(arr, np.float64)
        t = PropTableC(n_list=table.n, fix_swap=int(bool(fix_swap)), **{k: _ptr(v) for k, v in keep.items()})
        self._check(self.lib.chapsim_prop_table_init(self.h, ctypes.byref(t)))
        self._prop_keep = keep

    def THERM_PROP_UPDATE_points(self, dh):
        """Table-search property update of host points; returns dict H, T, D, M, K, CP shaped like dh."""
        dh = np.ascontiguousarray(dh, np.float64)
        n = dh.size
        outs = {k: np.empty(dh.shape) for k in ("H", "T", "D", "M", "K", "CP")}
        self._check(self.lib.chapsim_therm_prop_update_points(self.h, n, _ptr(dh), *[_ptr(outs[k]) for k in
                                                                                      ("H", "T", "D", "M", "K", "CP")]))
        return outs


    # -- learned property model -------------------------------------------------
    MLP_NPARAM = 4678
    MLP_FIELDS = ("H", "T", "D", "M", "K", "CP")

    def mlp_init(self, dh_lo, dh_hi, seed=2024):
        """Random-initialised 1-64-64-6 MLP for rho*h in [dh_lo, dh_hi] (needs the property table)."""
        self._check(self.lib.chapsim_mlp_init(self.h, float(dh_lo), float(dh_hi), int(seed)))

    def mlp_set_activation(self, act):
        """Hidden-layer activation: MLP_TANH (default) or MLP_CUBIC, the clamped cubic
        c = clamp(z, -1, 1), h = c (3 - c^2) / 2.  Set it before training."""
        self._check(self.lib.chapsim_mlp_set_activation(self.h, int(act)))

    def mlp_params(self):
        p = np.zeros(self.MLP_NPARAM, np.float32)
        nm = np.zeros(14)
        self._check(self.lib.chapsim_mlp_get_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _ptr(nm)))
        return p, nm

    def mlp_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.chapsim_mlp_set_params(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def mlp_gradients(self, dh):
        dh = np.ascontiguousarray(dh, np.float64).reshape(-1)
        g = np.zeros(self.MLP_NPARAM, np.float32)
        loss = ctypes.c_double()
        self._check(self.lib.chapsim_mlp_gradients(self.h, dh.size, _ptr(dh), g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                   ctypes.byref(loss)))
        return g, loss.value

    def mlp_train(self, dh, iters, lr=2e-3):
        dh = np.ascontiguousarray(dh, np.float64).reshape(-1)
        loss = ctypes.c_double()
        self._check(self.lib.chapsim_mlp_train(self.h, dh.size, _ptr(dh), int(iters), float(lr), ctypes.byref(loss)))
        return loss.value

    def mlp_infer_points(self, dh):
        dh = np.ascontiguousarray(dh, np.float64)
        outs = {k: np.empty(dh.shape) for k in self.MLP_FIELDS}
        self._check(self.lib.chapsim_mlp_infer_points(self.h, dh.size, _ptr(dh), *[_ptr(outs[k]) for k in self.MLP_FIELDS]))
        return outs


    def autotune(self, force=-1):
        """Keeps the fastest y-solve, right-hand-side and pressure-stage variants for
        this grid, or forces them (bit 0: sequential y-solve; bits 1-2: right-hand
        sides 0 fused, 1 split, 2 fused with bulk-copy staging, 3 the wide fused
        form (16-byte loads: two points per lane in FP64, four in FP32); bit 3: fused plane
        transforms; bit 4: two-way y-solve; bit 5: sequential y-solve with its
        forward intermediate in shared memory at one block per SM; bit 6: warp
        affine scans over the sequential factors; bit 8: z-sweep tiles of 16
        lines instead of 32; bit 9: double-buffered persistent z transforms; bit 10:
        z-sweep tiles with the lines interleaved in pairs; bit 11: the same for the y sweep;
        bit 12: z transforms that request the next wave's tiles into L2);
        returns
        (choice bits, {variant: ms})."""
        ch = ctypes.c_int32()
        ms = (ctypes.c_float * 19)()
        self._check(self.lib.chapsim_autotune(self.h, int(force), ctypes.byref(ch), ms))
        self.choice = ch.value
        return ch.value, {"ysolve_warp_pcr": ms[0], "ysolve_sequential": ms[1], "rhs_fused": ms[2],
                          "rhs_split": ms[3], "rhs_bulk": ms[4], "pressure_chained": ms[5],
                          "pressure_plane": ms[6], "ysolve_two_way": ms[7], "ysolve_sequential_smem": ms[8],
                          "ysolve_scan": ms[9], "zsweep_tile32": ms[10], "zsweep_tile16": ms[11],
                          "pressure_chained_zpipe": ms[12], "rhs_fused_wide": ms[13],
                          "zsweep_tile32_pairs": ms[14], "zsweep_tile16_pairs": ms[15],
                          "ysweep_lines": ms[16], "ysweep_pairs": ms[17], "pressure_chained_zprefetch": ms[18]}


class Ensemble:
    """Independent periodic channels advanced together (one graph per step, one branch per member)."""

    def __init__(self, channels):
        self.lib = load_library()
        self.members = list(channels)
        arr = (ctypes.c_void_p * len(self.members))(*[c.h.value if hasattr(c.h, "value") else c.h
                                                      for c in self.members])
        h = ctypes.c_void_p()
        rc = self.lib.chapsim_batch_create(arr, len(self.members), ctypes.byref(h))
        if rc != 0:
            raise ChapsimError(rc, self.lib.chapsim_last_error_string(None).decode())
        self.h = h

    def advance(self, nsteps, DT0, DTMIN, CFLGV):
        rc = self.lib.chapsim_batch_advance(self.h, int(nsteps), DT0, DTMIN, CFLGV)
        if rc != 0:
            raise ChapsimError(rc, self.lib.chapsim_last_error_string(None).decode())

    def stream_handle(self):
        v = ctypes.c_void_p()
        self.lib.chapsim_batch_get_stream(self.h, ctypes.byref(v))
        return v.value or 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.chapsim_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ChannelIO(ChannelTG):
    """Device-resident x-periodic main-domain channel (CHAPSim IO domain) with
    explicit (``ivisscheme=0``) or Crank-Nicolson (``ivisscheme=1``) viscous
    terms; property fields fixed, or updated by the thermal solver.

    ``G`` is numpy (3, N, M+2, L) = Fortran ``G_io(L, 0:M+1, N, 3)`` (rho*u);
    ``RHO``, ``MU0``, ``MU`` are (N, M+2, L) = ``DENSITY0``, ``Viscousity0``,
    ``Viscousity``.  ``advance`` runs CFL_io, the dt rule and three
    SOLVERRK3_MOM_io substeps per step.
    """

    IDOMAIN = 2

    def __init__(self, setup, device: int = 0, ivisscheme: int = VIS_EXPLICIT, **kw):
        super().__init__(setup, device=device, ivisscheme=ivisscheme, **kw)
        self.ivisscheme = int(ivisscheme)
        self.thermal = False
        self.use_mlp = False

    def kernel_slots(self):
        mom = (["k_io_rhs_cn", "k_io_cn_xsweep", "k_io_cn_zysweep"] if self.ivisscheme
               else ["k_io_divu", "k_io_rhs", "k_io_massflux"])
        eng = (["k_eng_rhs", "k_mlp_infer" if self.use_mlp else "k_eng_props", "k_eng_bc", "k_drhodt", "k_io_props",
                "k_g0_velocity"] if self.thermal else [])
        sub = eng + mom + ["k_io_div_fftx", "k_fftz_fwd", "k_ysolve", "k_fftz_inv", "k_fftx_inv", "k_io_correct"]
        return ["k_io_cfl", "k_dt"] + sub * 3

    def upload_io(self, G, PR, RHO, MU0, MU):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (G, PR, RHO, MU0, MU)]
        if arrs[0].shape != (3,) + self.field_shape() or any(a.shape != self.field_shape() for a in arrs[1:]):
            raise ValueError("field shape mismatch")
        self._check(self.lib.chapsim_upload_io_fields(self.h, *[_ptr(a) for a in arrs]))

    def download_io(self):
        G = np.empty((3,) + self.field_shape())
        Q = np.empty((3,) + self.field_shape())
        PR = np.empty(self.field_shape())
        self._check(self.lib.chapsim_download_io_fields(self.h, _ptr(G), _ptr(Q), _ptr(PR)))
        return G, Q, PR

    def SOLVERRK3_MOM_io(self, NS):
        self._check(self.lib.chapsim_rk_substep_io(self.h, int(NS)))

    def set_buoyancy(self, iGravity, F_A):
        """thermal_gravity / RHS_MOM_EXPLICIT_io buoyancy: D_STG * TALP*DT*F_A on component |iGravity|."""
        self._check(self.lib.chapsim_set_buoyancy(self.h, int(iGravity), float(F_A)))

    def PP_MEAN_ZX_FLOW_Xperiodic_io(self):
        """Instantaneous x-z means of the main domain on the device; returns the set as a flat
        array of per_row * M doubles (141 per row, 360 with the thermal solver) in the module
        arrays' order (Fortran order, j fastest)."""
        self._check(self.lib.chapsim_pp_mean_zx_io(self.h))
        n = ctypes.c_int32()
        self._check(self.lib.chapsim_download_pp_means_io(self.h, None, ctypes.byref(n)))
        out = np.zeros(n.value * self.M)
        self._check(self.lib.chapsim_download_pp_means_io(self.h, _ptr(out), ctypes.byref(n)))
        return out

    def set_weighted_pressure(self, PR0_1=None, PR0_2=None):
        """iWeightedPre = 1 with the two PR0_io layers ((N, M+2, L), the second defaults to the first);
        None turns it off."""
        if PR0_1 is None:
            self._check(self.lib.chapsim_upload_weighted_pressure(self.h, None, None))
            return
        a = np.ascontiguousarray(PR0_1, np.float64)
        b = np.ascontiguousarray(PR0_2 if PR0_2 is not None else PR0_1, np.float64)
        if a.shape != self.field_shape() or b.shape != self.field_shape():
            raise ValueError("PR0 layers must have the padded field shape")
        self._check(self.lib.chapsim_upload_weighted_pressure(self.h, _ptr(a), _ptr(b)))

    def CFL_io(self):
        v = ctypes.c_double()
        self._check(self.lib.chapsim_cfl_io(self.h, ctypes.byref(v)))
        return v.value

    def DIVGCK_io(self):
        """MAXDIVGV_io: max |div G + DrhoDtP| over the interior."""
        v = ctypes.c_double()
        self._check(self.lib.chapsim_divgck_io(self.h, ctypes.byref(v)))
        return v.value

    # -- thermal solver (SOLVERRK3_ENG_io with table-search properties) ----------
    def thermal_init(self, table, DH, qw_bot, qw_top, cthecd, fix_swap=False):
        """Uploads the property table (chapsim.thermo.SplineTable) and starts the
        energy equation from the padded rho*h field DH (N, M+2, L)."""
        self.prop_table_init(table, fix_swap=fix_swap)
        DH = np.ascontiguousarray(DH, np.float64)
        if DH.shape != self.field_shape():
            raise ValueError("DH shape mismatch")
        self._check(self.lib.chapsim_thermal_init(self.h, _ptr(DH), float(qw_bot), float(qw_top), float(cthecd)))
        self.thermal = True

    def thermal_set_isothermal(self, wall, state=None):
        """BC_Fixed_Temperature on wall 0 (bottom) or 1 (top): state = (T, H, D, M, K) of the wall;
        None returns that wall to the constant heat flux."""
        v = None if state is None else np.ascontiguousarray(state, np.float64)
        self._check(self.lib.chapsim_thermal_set_isothermal(self.h, int(wall), _ptr(v)))

    def download_thermal(self):
        """dict DH, H, T, D, M, K, CP of padded fields."""
        names = ["DH", "H", "T", "D", "M", "K", "CP"]
        out = {k: np.empty(self.field_shape()) for k in names}
        self._check(self.lib.chapsim_download_thermal_fields(self.h, *[_ptr(out[k]) for k in names]))
        return out

    def thermal_use_mlp(self, enable=True):
        self._check(self.lib.chapsim_thermal_use_mlp(self.h, int(bool(enable))))
        self.use_mlp = bool(enable)

    def mlp_judge(self):
        """Largest |model - table| / max(|table|, output scale) per output over the interior fields."""
        e = np.zeros(6)
        self._check(self.lib.chapsim_mlp_judge(self.h, _ptr(e)))
        return dict(zip(self.MLP_FIELDS, e.tolist()))


class ChannelXinout(ChannelIO):
    """Main domain of a TG + main-domain run (CHAPSim iDomain = 3): inflow from a periodic
    :class:`ChannelTG` context (BC_TINLET_FLOW), a convective outlet (BC_COUTLET_MOM_RK3) and
    FISHPACK's x-cosine Poisson solve; explicit viscous terms, FP64; the thermal solver with
    ``thermal_init`` and ``thermal_inlet`` (BC_TINLET_THERML, BC_COUTLET_ENEG_RK3).

    ``setup`` comes from :func:`chapsim.mesh.xinout_setup`.  Fields carry the x ghost
    columns: ``G`` is (3, N, M+2, L+2) = Fortran ``G_io(0:L+1, 0:M+1, N, 3)``, ``PR``, ``RHO``,
    ``MU0``, ``MU`` are (N, M+2, L+2).  ``attach(tg)`` names the TG context that feeds the
    inlet; ``advance`` runs both domains' steps with their common DT.
    """

    IDOMAIN = 3

    def __init__(self, setup, tg: ChannelTG = None, device: int = 0, **kw):
        super().__init__(setup, device=device, ivisscheme=VIS_EXPLICIT, **kw)
        self.tg = None
        if tg is not None:
            self.attach(tg)

    def field_shape(self):
        return (self.N, self.M + 2, self.L + 2)

    def attach(self, tg: ChannelTG):
        self._check(self.lib.chapsim_xinout_attach(self.h, tg.h))
        self.tg = tg

    def kernel_slots(self):
        fft = self.L in (32, 64, 96, 128, 192, 256, 384)  # the cosine transforms through the FFT
        sub = ["k_xio_inlet", "k_xio_outlet_a", "k_xio_outlet_b", "k_xio_outlet_c", "k_io_divu", "k_io_rhs",
               "k_io_massflux", "k_xio_div_cosqf" if fft else "k_xio_div_dctx", "k_fftz_fwd", "k_xio_ysolve",
               "k_fftz_inv", "k_xio_cosqb" if fft else "k_xio_dctx_inv", "k_io_correct"]
        return ["k_io_cfl", "k_dt", "k_dt_pair"] + sub * 3

    def advance(self, nsteps, DT0, DTMIN, CFLGV):
        """nsteps steps of the TG + main-domain loop; returns (DT, CFLMM) of the last step."""
        dt, cfl = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.chapsim_advance_xinout(self.h, int(nsteps), DT0, DTMIN, CFLGV, ctypes.byref(dt),
                                                    ctypes.byref(cfl)))
        return dt.value, cfl.value

    def DIVGCK_io(self):
        """MAXDIVGV_io(1:3): max |div G| over the cells 2..L-1, 0..1 and L."""
        out = np.zeros(3)
        self._check(self.lib.chapsim_divgck_xinout(self.h, _ptr(out)))
        return out

    def thermal_inlet(self, state7):
        """BC_TINLET_THERML's inlet state (T, H, D, M, K, CP, DH) after thermal_init."""
        self._check(self.lib.chapsim_xinout_thermal_inlet(self.h, _ptr(np.ascontiguousarray(state7, np.float64))))

    def outlet_state(self):
        """(U_OUTLET, CHK_Mass_CONSV0_SCALING) of the last substep."""
        out = np.zeros(2)
        self._check(self.lib.chapsim_xinout_outlet_state(self.h, _ptr(out)))
        return float(out[0]), float(out[1])
