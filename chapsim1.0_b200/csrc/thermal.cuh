// Thermal solver of the main (IO) domain, run before the momentum part of
// each RK3 substep (src/SOLVE.f90:119-128):
//   k_eng_rhs    SOLVERRK3_ENG_io (src/SOLVERRK3_ENG_IO.f90:11-82) with
//                RHS_ENERGY_EXPLICIT (src/RHS_ENERGY_EXPLICIT.f90:11-155):
//                rho*h += TGAM dt RHS + TROH dt RHS0, clipped to the table's
//                [DHmin, DHmax] (search-table limiter), RHS0 = RHS; constant
//                wall heat flux on both walls
//   k_eng_props  THERM_PROP_UPDATE(IMAIND) by table search on rows 1..M; the
//                old DENSITY and Viscousity are kept as DENSITY0 and
//                Viscousity0 point by point before being overwritten (the
//                whole-field copies at the top of SOLVERRK3_ENG_io)
//   k_eng_bc     BC_WALL_Isoflux (src/BC_WALL.f90:541-619): ghost rho*h
//                extrapolated from rows 1, 2 (M, M-1), then its properties
//   k_drhodt     DENSITY_TIME_DERIVATION (src/DIVG.f90:249-317):
//                DrhoDtP = -TGAM div(G) - TROH div(G0)
// followed by k_io_props (DENSITY_Staggered, MU_Staggered from DENSITY0 and
// Viscousity0) and the momentum substep, which starts with G0 = G and
// VELOCITY_CALC_io.  Plane channel: RCCI1 = RCCI2 = RNDI1 = 1.
#pragma once
#include "common.cuh"
#include "io.cuh"
#include "thermo.cuh"

#ifndef CHS_EBIT_TABLE
#define CHS_EBIT_TABLE 4u  // a point (or its h) left the property table
#endif

struct ThermoFields {
    double *DH, *ENTH, *TEMP, *KAP, *HCP, *RHSE0, *G0, *DRHO;
};
struct ThermoParams {
    double wf_bot, wf_top;  // WALLFLUX of the bottom (+q) and top (-q) walls (src/Flow_State.f90:150-175)
    double cthecd;          // 1 / (REN PRT0)
    double dhmin, dhmax;    // LIST_DH at IMIN_DH, IMAX_DH
    // BC_Fixed_Temperature walls (0 bottom, 1 top): the wall state T, H, D, M, K held in the ghost
    // row (BC_WALL_IsoTHERMAL, src/BC_WALL.f90:484-538); 0 = constant heat flux
    int iso[2];
    double wv[2][5];
};

template <typename F>
__global__ void __launch_bounds__(IO_NT, 4) k_eng_rhs(Geo g, IoFieldsT<F> f, ThermoFields t, ThermoParams tp,
                                                   const DevState* __restrict__ st, int ns) {
    const int M = g.M, N = g.N;
    const long long tot = io_points(g);
    const double dt = st->dt;
    const double coe1n = g.tgam[ns] * dt, coe0n = g.troh[ns] * dt;
    const double XND2CL = 0.5, ZND2CL = 0.5;
    const double COE1 = g.dxi * XND2CL * 0.5;
    const double COE11 = g.dxqi * XND2CL * tp.cthecd;
    const double* Hh = t.ENTH;
    const double* T = t.TEMP;
    const double* K = t.KAP;
    const F* G1 = f.G;
    const F* G2 = f.G + g.FS;
    const F* G3 = f.G + 2 * g.FS;
    for (long long q = (long long)blockIdx.x * IO_NT + threadIdx.x; q < tot; q += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, q, i, j, k);
        const int ip = xpn(g, i), im = xmn(g, i), kp = wrapp(k, N), km = wrapm(k, N);
        const int jp = j + 1, jm = j - 1;
        const long long c = pidx(g, i, j, k);
        const long long cip = pidx(g, ip, j, k), cim = pidx(g, im, j, k);
        const long long cjp = pidx(g, i, jp, k), cjm = pidx(g, i, jm, k);
        const long long ckp = pidx(g, i, j, kp), ckm = pidx(g, i, j, km);
        const double COE2 = g.dyfi[j] * 1.0 * 0.5;
        const double COE3 = g.dzi * ZND2CL * 1.0 * 0.5;
        const double COE33 = g.dzqi * ZND2CL * 1.0 * tp.cthecd;
        const double COE22 = g.dyfi[j] * 1.0 * tp.cthecd;
        double COE221, COE222;
        if (j == 1) {  // src/RHS_ENERGY_EXPLICIT.f90:50-77: the wall face of an isothermal wall keeps DYCI
            COE221 = g.dyci[jp] / 1.0;
            COE222 = tp.iso[0] ? g.dyci[j] / 1.0 : 1.0 / 1.0;
        } else if (j == M) {
            COE222 = g.dyci[j] / 1.0;
            COE221 = tp.iso[1] ? g.dyci[jp] / 1.0 : 1.0 / 1.0;
        } else {
            COE221 = g.dyci[jp] / 1.0;
            COE222 = g.dyci[j] / 1.0;
        }
        const double hc = Hh[c], tc = T[c], kc = K[c];
        double DX_DHU = (Hh[cip] + hc) * (G1[cip] + G1[cip]) - (hc + Hh[cim]) * (G1[c] + G1[c]);
        DX_DHU = DX_DHU * COE1;
        double DY_DHV = (g.wff[jp] * Hh[cjp] + g.wfb[jp] * hc) * (G2[cjp] + G2[cjp]) -
                        (g.wff[j] * hc + g.wfb[j] * Hh[cjm]) * (G2[c] + G2[c]);
        DY_DHV = DY_DHV * COE2;
        double DZ_DHW = (Hh[ckp] + hc) * (G3[ckp] + G3[ckp]) - (hc + Hh[ckm]) * (G3[c] + G3[c]);
        DZ_DHW = DZ_DHW * COE3;
        double DX_KDT = (K[cip] + kc) * (T[cip] - tc) - (kc + K[cim]) * (tc - T[cim]);
        DX_KDT = DX_KDT * COE11;
        double KDTy1 = (g.wff[jp] * K[cjp] + g.wfb[jp] * kc) * (T[cjp] - tc) * COE221;
        double KDTy2 = (g.wff[j] * kc + g.wfb[j] * K[cjm]) * (tc - T[cjm]) * COE222;
        if (j == 1 && !tp.iso[0]) KDTy2 = -tp.wf_bot * COE222;
        else if (j == M && !tp.iso[1]) KDTy1 = -tp.wf_top * COE221;
        const double DY_KDT = (KDTy1 - KDTy2) * COE22;
        double DZ_KDT = (K[ckp] + kc) * (T[ckp] - tc) - (K[ckm] + kc) * (tc - T[ckm]);
        DZ_KDT = DZ_KDT * COE33;
        const double rhs = -DX_DHU - DY_DHV - DZ_DHW + DX_KDT + DY_KDT + DZ_KDT;
        double d = t.DH[c] + coe1n * rhs + coe0n * t.RHSE0[c];
        d = fmin(tp.dhmax - 1.0e-14, d);
        d = fmax(tp.dhmin + 1.0e-14, d);
        t.DH[c] = d;
        t.RHSE0[c] = rhs;
    }
}

// Properties of one padded point from its rho*h; the old DENSITY and
// Viscousity are kept in DENSITY0 (f.RHO) and Viscousity0 (f.MU0) first.
template <typename F>
__device__ __forceinline__ void eng_point(const PropTab& tb, const double* xdh, const double* xh, const IoFieldsT<F>& f,
                                          const ThermoFields& t, long long p, DevState* st) {
    f.RHO[p] = f.DEN[p];
    f.MU0[p] = f.MU[p];
    double o[6];
    if (!prop_point(tb, xdh, xh, t.DH[p], o)) atomicOr(&st->err, CHS_EBIT_TABLE);
    t.ENTH[p] = o[0];
    t.TEMP[p] = o[1];
    f.DEN[p] = o[2];
    f.MU[p] = o[3];
    t.KAP[p] = o[4];
    t.HCP[p] = o[5];
}

__device__ __forceinline__ void stage_keys(const PropTab& tb, double* keys, const double*& xdh, const double*& xh) {
    for (int r = threadIdx.x; r < tb.n; r += blockDim.x) {
        keys[r] = tb.xdh[r];
        keys[tb.n + r] = tb.xh[r];
    }
    __syncthreads();
    xdh = keys;
    xh = keys + tb.n;
}

template <bool SMEM, typename F>
__global__ void __launch_bounds__(PROP_NT) k_eng_props(PropTab tb, Geo g, IoFieldsT<F> f, ThermoFields t, DevState* st) {
    extern __shared__ double keys[];
    const double* xdh = tb.xdh;
    const double* xh = tb.xh;
    if (SMEM) stage_keys(tb, keys, xdh, xh);
    const long long tot = io_points(g);
    for (long long q = (long long)blockIdx.x * PROP_NT + threadIdx.x; q < tot; q += (long long)gridDim.x * PROP_NT) {
        int i, j, k;
        io_decode(g, q, i, j, k);
        eng_point(tb, xdh, xh, f, t, pidx(g, i, j, k), st);
    }
}

// ghost rows j = 0 (bottom) and j = M+1 (top), every i and k
template <bool SMEM, typename F>
__global__ void __launch_bounds__(PROP_NT) k_eng_bc(PropTab tb, Geo g, IoFieldsT<F> f, ThermoFields t, ThermoParams tp,
                                                  DevState* st) {
    extern __shared__ double keys[];
    const double* xdh = tb.xdh;
    const double* xh = tb.xh;
    if (SMEM) stage_keys(tb, keys, xdh, xh);
    const int L = g.L, M = g.M;
    const long long plane = (long long)L * g.N;
    for (long long q = (long long)blockIdx.x * PROP_NT + threadIdx.x; q < 2 * plane; q += (long long)gridDim.x * PROP_NT) {
        const bool top = q >= plane;
        const long long r = top ? q - plane : q;
        const int i = (int)(r % L), k = (int)(r / L);
        long long p;
        const int w = top ? 1 : 0;
        if (tp.iso[w]) {  // BC_WALL_IsoTHERMAL: the wall state, DH = H * D (DENSITY0, Viscousity0 keep the old row)
            p = pidx(g, i, top ? M + 1 : 0, k);
            f.RHO[p] = f.DEN[p];
            f.MU0[p] = f.MU[p];
            t.TEMP[p] = tp.wv[w][0];
            t.ENTH[p] = tp.wv[w][1];
            f.DEN[p] = tp.wv[w][2];
            f.MU[p] = tp.wv[w][3];
            t.KAP[p] = tp.wv[w][4];
            t.DH[p] = t.ENTH[p] * f.DEN[p];
            continue;
        }
        if (top) {
            p = pidx(g, i, M + 1, k);
            t.DH[p] = 2.0 * t.DH[pidx(g, i, M, k)] - g.wff[M] * t.DH[pidx(g, i, M, k)] - g.wfb[M] * t.DH[pidx(g, i, M - 1, k)];
        } else {
            p = pidx(g, i, 0, k);
            t.DH[p] = 2.0 * t.DH[pidx(g, i, 1, k)] - g.wff[2] * t.DH[pidx(g, i, 2, k)] - g.wfb[2] * t.DH[pidx(g, i, 1, k)];
        }
        eng_point(tb, xdh, xh, f, t, p, st);
    }
}

// mpart (inflow/outflow domain, else NULL): per-block sums of DrhoDtP / DYFI for the interior mass
// rate of CHK_MassConsv_io (src/processing/CHK_conservation.f90:41-53)
template <typename F>
__global__ void __launch_bounds__(IO_NT) k_drhodt(Geo g, IoFieldsT<F> f, ThermoFields t, int ns, double* __restrict__ mpart) {
    __shared__ double sred[32];
    const int N = g.N;
    const long long tot = io_points(g);
    double ms = 0.0;
    const double tgam = g.tgam[ns], troh = g.troh[ns];
    const F* G = f.G;
    const double* G0 = t.G0;
    for (long long q = (long long)blockIdx.x * IO_NT + threadIdx.x; q < tot; q += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, q, i, j, k);
        const long long c = pidx(g, i, j, k);
        const long long cip = pidx(g, xpn(g, i), j, k), ckp = pidx(g, i, j, wrapp(k, N)), cjp = pidx(g, i, j + 1, k);
        const double COE2 = g.dyfi[j] * 1.0, COE3 = g.dzi * 1.0;
        const double DIVX = ((double)G[cip] - (double)G[c]) * g.dxi;
        const double DIVX0 = (G0[cip] - G0[c]) * g.dxi;
        const double DIVY = ((double)G[cjp + g.FS] - (double)G[c + g.FS]) * COE2;
        const double DIVY0 = (G0[cjp + g.FS] - G0[c + g.FS]) * COE2;
        const double DIVZ = ((double)G[ckp + 2 * g.FS] - (double)G[c + 2 * g.FS]) * COE3;
        const double DIVZ0 = (G0[ckp + 2 * g.FS] - G0[c + 2 * g.FS]) * COE3;
        const double dr = -tgam * (DIVX + DIVY + DIVZ) - troh * (DIVX0 + DIVY0 + DIVZ0);
        t.DRHO[c] = dr;
        if (mpart) ms += dr * (1.0 / g.dyfi[j] / 1.0);
    }
    if (mpart) {
        const double b = block_sum<IO_NT>(ms, sred);
        if (threadIdx.x == 0) mpart[blockIdx.x] = b;
    }
}

// G0_io = G_io (interior; the wall values of G never change) and VELOCITY_CALC_io.
// G0 is FP64 in both precisions (a copy of the FP32 G in the mixed step).
template <typename F>
__global__ void __launch_bounds__(IO_NT) k_g0_velocity(Geo g, IoFieldsT<F> f, double* __restrict__ G0) {
    const long long tot = io_points(g);
    for (long long q = (long long)blockIdx.x * IO_NT + threadIdx.x; q < tot; q += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, q, i, j, k);
        const long long c = pidx(g, i, j, k);
        const double g1 = f.G[c], g2 = f.G[c + g.FS], g3 = f.G[c + 2 * g.FS];
        G0[c] = g1;
        G0[c + g.FS] = g2;
        G0[c + 2 * g.FS] = g3;
        if (g.xo && (i == 1 || i == g.LI)) {  // G0_io = G_io takes the inlet and outlet ghost columns too
            const long long e = i == 1 ? c - 1 : c + 1;
            for (int d = 0; d < 3; ++d) G0[e + d * g.FS] = (double)f.G[e + d * g.FS];
        }
        f.Q[c] = (F)(g1 / (double)f.DST[c]);
        f.Q[c + 2 * g.FS] = (F)(g3 / (double)f.DST[c + 2 * g.FS]);
        if (j >= 2) f.Q[c + g.FS] = (F)(g2 / (double)f.DST[c + g.FS]);
    }
}
