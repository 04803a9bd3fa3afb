"""Host-side set-up of the periodic plane channel.

In CHAPSim these quantities are computed once by the Fortran host before the
time loop and live in module variables; the B200 library receives them
through ``chapsim_gpu_init``.  This module restates those set-up routines so
that a Python caller can drive the library without the Fortran host:

  CONSPARA            src/CONSPARA.f90:54-73       DX, DZ, DXI, DZI, DXQI, DZQI
  COORDJR             src/COORDJR.f90:38-145       YND, YCC, DYFI, DYCI (channel)
  AREA_INOUTLET       src/COORDJR.f90:345-395      Area_inlet, VOLM_tg
  MESH_YWEIGHT_FACTORS src/COORDJR.f90:416-442     YCL2ND_WFF / _WFB
  TDMA_COEF           src/TDMA_COEF.f90:44-110     AMPH/ACPH/APPH, AMVR/ACVR/APVR
  LAMPOISLPROF        src/LAMPOISLPROF.f90:17-60   Vini (Poiseuille profile)
  CONS_RKCOEF         src/CONS_RKCOEF.f90:25-51    TGAM, TROH, TALP
  FFT99_ROOT          src/possion3d_FFT99.f90:140-202  AK1, AK3
  FFTPACK_ROOT        src/possion3d_fishpack.f90:48-137 XRT, YRT of the inflow/outflow
                      main domain (xinout_setup)

Arrays are returned 1-based as in Fortran (index 0 unused) unless noted.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class ChannelSetup:
    L: int
    M: int
    N: int
    HX: float
    HZ: float
    STR2: float
    REN: float
    iFlowDriven: int = 1
    Cf_Given: float = 8.18e-3
    # derived
    DX: float = 0.0
    DZ: float = 0.0
    DXI: float = 0.0
    DZI: float = 0.0
    DXQI: float = 0.0
    DZQI: float = 0.0
    CVISC: float = 0.0
    VOLM: float = 0.0
    Area_inlet: float = 0.0
    AMVR1: float = 0.0
    APVRN: float = 0.0
    YND: np.ndarray = field(default=None, repr=False)
    YCC: np.ndarray = field(default=None, repr=False)
    DYFI: np.ndarray = field(default=None, repr=False)
    DYCI: np.ndarray = field(default=None, repr=False)
    WFF: np.ndarray = field(default=None, repr=False)
    WFB: np.ndarray = field(default=None, repr=False)
    AMPH: np.ndarray = field(default=None, repr=False)
    ACPH: np.ndarray = field(default=None, repr=False)
    APPH: np.ndarray = field(default=None, repr=False)
    AMVR: np.ndarray = field(default=None, repr=False)  # (4, M+2): [IDR, j]
    ACVR: np.ndarray = field(default=None, repr=False)
    APVR: np.ndarray = field(default=None, repr=False)
    Vini: np.ndarray = field(default=None, repr=False)
    TGAM: np.ndarray = field(default=None, repr=False)
    TROH: np.ndarray = field(default=None, repr=False)
    TALP: np.ndarray = field(default=None, repr=False)
    AK1: np.ndarray = field(default=None, repr=False)  # 0-based kx
    AK3: np.ndarray = field(default=None, repr=False)  # 0-based kz


def channel_setup(L, M, N, HX, HZ, STR2, REN, iFlowDriven=1, Cf_Given=8.18e-3) -> ChannelSetup:
    if min(L, M, N) < 4 or L % 2 or N % 2:
        raise ValueError("grid too small or odd periodic length")
    s = ChannelSetup(L, M, N, float(HX), float(HZ), float(STR2), float(REN), int(iFlowDriven), float(Cf_Given))
    NND2 = M + 1
    PI = 2.0 * math.asin(1.0)
    # CONSPARA
    s.DX = s.HX / float(L)
    s.DXI = 1.0 / s.DX
    s.DXQI = s.DXI * s.DXI
    s.DZ = s.HZ / float(N)
    s.DZI = 1.0 / s.DZ
    s.DZQI = s.DZI * s.DZI
    s.CVISC = 1.0 / s.REN
    # COORDJR (channel)
    YND = np.zeros(M + 3)
    for J in range(1, NND2 + 1):
        X2 = float(J - 1) / float(NND2 - 1)
        YND[J] = math.tanh(s.STR2 * (X2 - 0.5)) / math.tanh(s.STR2 * 0.5)
    YCC = np.zeros(M + 3)
    DYFI = np.zeros(M + 3)
    DYCI = np.zeros(M + 3)
    for J in range(1, M + 1):
        YCC[J] = (YND[J] + YND[J + 1]) * 0.5
        DYFI[J] = 1.0 / (YND[J + 1] - YND[J])
    for J in range(2, NND2):
        DYCI[J] = 1.0 / ((YND[J + 1] - YND[J - 1]) * 0.5)
    DYCI[1] = 2.0 / (YND[2] - YND[1])
    DYCI[NND2] = 2.0 / (YND[NND2] - YND[M])
    # AREA_INOUTLET: naive running sums in the reference's loop order
    # (np.cumsum of a 1-D array accumulates sequentially, like the Fortran loop)
    t_area = 1.0 / 1.0 / DYFI[1:M + 1] / s.DZI
    s.Area_inlet = float(np.cumsum(np.concatenate([[0.0], np.repeat(t_area, N)]))[-1])
    t_vol = np.repeat(1.0 / 1.0 / DYFI[1:M + 1], L)
    vol = 0.0
    for _KC in range(N):
        vol = float(np.cumsum(np.concatenate([[vol], t_vol]))[-1])
    s.VOLM = vol
    # MESH_YWEIGHT_FACTORS
    WFF = np.zeros(M + 3)
    WFB = np.zeros(M + 3)
    for JC in range(2, M + 1):
        JM = JC - 1
        WFF[JC] = (YND[JC] - YCC[JM]) / (YCC[JC] - YCC[JM])
        WFB[JC] = (YCC[JC] - YND[JC]) / (YCC[JC] - YCC[JM])
    WFB[1], WFF[1] = 1.0, 0.0
    WFB[NND2], WFF[NND2] = 0.0, 1.0
    # TDMA_COEF (channel)
    AMPH = np.zeros(M + 3)
    ACPH = np.zeros(M + 3)
    APPH = np.zeros(M + 3)
    for JC in range(1, M + 1):
        JP = JC + 1
        AMPH[JC] = DYFI[JC] * DYCI[JC]
        APPH[JC] = DYFI[JC] * DYCI[JP]
        if JC == 1:
            AMPH[JC] = DYFI[JC] * DYCI[JC] * 0.5
        if JP == NND2:
            APPH[JC] = DYFI[JC] * DYCI[JP] * 0.5
    for JC in range(1, M + 1):
        ACPH[JC] = -(AMPH[JC] + APPH[JC])
    ACPH[1] = AMPH[1] + ACPH[1]
    AMPH[1] = 0.0
    ACPH[M] = APPH[M] + ACPH[M]
    APPH[M] = 0.0
    AMVR = np.zeros((4, M + 3))
    ACVR = np.zeros((4, M + 3))
    APVR = np.zeros((4, M + 3))
    for IDR in (1, 2, 3):
        if IDR in (1, 3):
            for JC in range(2, M):
                JP = JC + 1
                AMVR[IDR, JC] = DYFI[JC] * DYCI[JC]
                APVR[IDR, JC] = DYFI[JC] * DYCI[JP]
                ACVR[IDR, JC] = -(AMVR[IDR, JC] + APVR[IDR, JC])
            UCAJ = 4.0 / (2.0 / DYCI[2] + 1.0 / DYFI[1])
            AMVR[IDR, 1] = 0.0
            APVR[IDR, 1] = UCAJ * DYCI[2]
            ACVR[IDR, 1] = -UCAJ * (DYCI[2] + 2.0 * DYFI[1])
            s.AMVR1 = UCAJ * (2.0 * DYFI[1])
            UCAJ = 4.0 / (2.0 / DYCI[M] + 1.0 / DYFI[M])
            AMVR[IDR, M] = UCAJ * DYCI[M]
            APVR[IDR, M] = 0.0
            ACVR[IDR, M] = -UCAJ * (2.0 * DYFI[M] + DYCI[M])
            s.APVRN = UCAJ * (2.0 * DYFI[M])
        else:
            for JC in range(2, M + 1):
                JM = JC - 1
                AMVR[IDR, JC] = DYFI[JM] * DYCI[JC]
                APVR[IDR, JC] = DYFI[JC] * DYCI[JC]
                ACVR[IDR, JC] = -(AMVR[IDR, JC] + APVR[IDR, JC])
            AMVR[IDR, 1], APVR[IDR, 1], ACVR[IDR, 1] = 0.0, 0.0, 1.0
            AMVR[IDR, NND2], APVR[IDR, NND2], ACVR[IDR, NND2] = 0.0, 0.0, 1.0
    # LAMPOISLPROF (channel: a = 1, b = 0, PCOE = 3/2)
    Vini = np.zeros(M + 3)
    a, b, PCOE = (1.0 - (-1.0)) / 2.0, 0.0, 3.0 / 2.0
    for J in range(1, M + 1):
        if -1.0 < YCC[J] < 1.0:
            Vini[J] = (1.0 - ((YCC[J] - b) * (YCC[J] - b)) / a / a) * PCOE
    # CONS_RKCOEF
    TGAM = np.array([1.0, 8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0])
    TROH = np.array([0.0, 0.0, -17.0 / 60.0, -5.0 / 12.0])
    TALP = TGAM + TROH
    # FFT99_ROOT
    AK1 = np.zeros(L)
    AK3 = np.zeros(N)
    for K in range(1, N + 1):
        AN = float(K - 1) * 2.0 * PI if K <= N // 2 else -float(N - K + 1) * 2.0 * PI
        AK3[K - 1] = 2.0 * (1.0 - math.cos(AN / float(N))) * s.DZQI
    for I in range(1, L + 1):
        AP = float(I - 1) * 2.0 * PI if I <= L // 2 else -float(L - I + 1) * 2.0 * PI
        AK1[I - 1] = 2.0 * (1.0 - math.cos(AP / float(L))) * s.DXQI
    s.YND, s.YCC, s.DYFI, s.DYCI, s.WFF, s.WFB = YND, YCC, DYFI, DYCI, WFF, WFB
    s.AMPH, s.ACPH, s.APPH = AMPH, ACPH, APPH
    s.AMVR, s.ACVR, s.APVR = AMVR, ACVR, APVR
    s.Vini, s.TGAM, s.TROH, s.TALP, s.AK1, s.AK3 = Vini, TGAM, TROH, TALP, AK1, AK3
    return s


def xinout_setup(L, M, N, HX, HZ, STR2, REN) -> ChannelSetup:
    """Set-up of the main domain of a TG + main-domain run (iDomain = 3): the channel
    set-up with no bulk forcing (RHS_MOM_EXPLICIT_io applies it only to the x-periodic
    flow, src/RHS_MOM_EXPLICIT_io.f90:229) and the FISHPACK roots of BCX_io = (2, 1),
    LPEROD = 4, and the periodic z direction (FFTPACK_ROOT, src/possion3d_fishpack.f90:
    48-137), stored as the positive AK1/AK3 the Poisson y-solve subtracts from ACPH:

      AK1[m]  = -XRT(m+1) = 4 DXQI sin^2((m + 1/2) pi / (2 L)),  m = 0..L-1
      AK3[kz] = -YRT      = 4 DZQI sin^2(pi min(kz, N-kz) / N)   (the RFFTF pair of
                            wavenumber min(kz, N-kz) shares one root)
    """
    s = channel_setup(L, M, N, HX, HZ, STR2, REN, iFlowDriven=0, Cf_Given=0.0)
    PI = 2.0 * math.asin(1.0)
    DX = PI / (2.0 * float(L))
    s.AK1 = np.array([4.0 * s.DXQI * (math.sin((float(I) - 0.5) * DX) ** 2) for I in range(1, L + 1)])
    DY = PI / (2.0 * float(N))
    s.AK3 = np.array([4.0 * s.DZQI * (math.sin(float(2 * min(k, N - k)) * DY) ** 2) for k in range(N)])
    return s
