// Main-domain (IO, x-periodic) substep, SOLVERRK3_MOM_io
// (src/SOLVERRK3_MOM_IO.f90:11-120) with explicit (iVisScheme = 0) or
// Crank-Nicolson (iVisScheme = 1, sweeps in io_cn.cuh) viscous terms, for a
// flow whose property fields (DENSITY0, Viscousity0, Viscousity) are given
// and held fixed unless the thermal solver (thermal.cuh) updates them.
//
//   k_io_props     DENSITY_Staggered + MU_Staggered (src/MASSFLUX_CALC_IO.f90:155-329), once per upload
//   k_io_divu      DIVG_U_io (src/DIVG.f90:140-246): DivU = div(u)/3
//   k_io_rhs<CN>   CONVECTION_X/Y/Z_io, VISCOUS_ALL_EXPLT_X/Y/Z_io (or VISCOUS_PAR_EXPLT_*), RHS_MOM_EXPLICIT_io
//                  (RK combination, EXPLT0 update, pressure gradient, grid sum of the
//                  bulk-forcing integrand), one thread per point and all components
//   k_io_massflux  bulk forcing subtraction + MASSFLUX_CALC_io (G += RHS)
//   k_io_div_fftx  DIVG_io (src/DIVG.f90:54-137) + forward x transform
//   (shared)       k_fftz / k_ysolve_warp / k_fftz / k_fftx_inv of poisson.cuh: the
//                  discrete problem of FISHPACK_POIS3D_SIMPLE (same AMPH/ACPH/APPH operator
//                  and x/z eigenvalues); its singular kx = kz = 0 mode is fixed at
//                  phi_hat(y_1) = 0, which shifts DPH and PR by a constant only
//   k_io_correct   PRCALC_io (PR += DPH, minus BE*RHSLLPHI under CN), MASSFLUX_UPDATE_io
//                  (src/VELO_CORRECTION.f90:103-179), VELOCITY_CALC_io (Q = G/D_STG)
//   k_io_cfl       CFL_io (src/CFL.f90:55-107), including the viscous number
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "poisson.cuh"

#define IO_NT 256

// RHO is DENSITY0 and DEN is DENSITY (the same array while the thermal
// solver is off); MU0 is Viscousity0 and MU is Viscousity.
// PR0A/PR0B: PR0_io(:,:,:,1) and PR0_io(:,:,:,2) of iWeightedPre = 1 (NULL when
// off).  igrav/fa: iGravity and F_A of thermal_gravity (src/Flow_State.f90:95-125).
// F is the storage type of the flow fields G, Q, PR, EXPLT0, RHS, D_STG, MU_STG
// and DivU: double, or float in the mixed-precision step.  The property
// fields (DENSITY, DENSITY0, Viscousity, Viscousity0) stay FP64 (they come
// from the FP64 property update), and the kernels evaluate in FP64.
template <typename F>
struct IoFieldsT {
    F *G, *Q, *PR, *EX0, *RHS;
    double *RHO, *MU0, *MU;
    F *DST, *MST, *DIVU;
    double* DEN;
    const double *PR0A = nullptr, *PR0B = nullptr;
    double fa = 0.0;
    int igrav = 0;
};
using IoFields = IoFieldsT<double>;

// iWeightedPre: pres_epslon (src/modules.f90:483)
#define IO_PRES_EPSLON 0.001

// PGM of RHS_MOM_EXPLICIT_io (src/RHS_MOM_EXPLICIT_io.f90:103-159): the
// pressure difference between point c and its lower neighbour cm times coe,
// blended with the two PR0_io layers when iWeightedPre = 1
template <typename F>
__device__ __forceinline__ double io_pgm(const IoFieldsT<F>& f, long long c, long long cm, double pc, double pm,
                                         double coe) {
    if (f.PR0A)
        return ((f.PR0B[c] - f.PR0B[cm]) * (0.25 - IO_PRES_EPSLON) + (f.PR0A[c] - f.PR0A[cm]) * 0.5 +
                (pc - pm) * (0.25 + IO_PRES_EPSLON)) * coe;
    return (pc - pm) * coe;
}


// ---------------------------------------------------------------------------
template <typename F>
__global__ void __launch_bounds__(IO_NT) k_io_props(Geo g, IoFieldsT<F> f) {
    const int M = g.M, N = g.N;
    const long long tot = io_points(g);
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const int im = xmn(g, i), km = wrapm(k, N);
        const long long c = pidx(g, i, j, k);
        const double* R = f.RHO;
        const double* U0 = f.MU0;
        f.DST[c] = (F)((R[c] + R[pidx(g, im, j, k)]) * 0.5);
        f.DST[c + 2 * g.FS] = (F)((R[c] + R[pidx(g, i, j, km)]) * 0.5);
        f.DST[c + g.FS] = (F)(j >= 2 ? g.wff[j] * R[c] + g.wfb[j] * R[pidx(g, i, j - 1, k)] : R[pidx(g, i, 0, k)]);
        if (j >= 2) {
            f.MST[c] = (F)(((U0[c] + U0[pidx(g, im, j, k)]) * g.wff[j] + (U0[pidx(g, i, j - 1, k)] + U0[pidx(g, im, j - 1, k)]) * g.wfb[j]) * 0.5);
            f.MST[c + 2 * g.FS] = (F)(((U0[pidx(g, i, j, km)] + U0[c]) * g.wff[j] +
                                   (U0[pidx(g, i, j - 1, km)] + U0[pidx(g, i, j - 1, k)]) * g.wfb[j]) * 0.5);
        } else {
            f.MST[c] = (F)U0[pidx(g, i, 0, k)];
            f.MST[c + 2 * g.FS] = (F)U0[pidx(g, i, 0, k)];
        }
        f.MST[c + g.FS] = (F)((U0[c] + U0[pidx(g, im, j, k)] + U0[pidx(g, i, j, km)] + U0[pidx(g, im, j, km)]) * 0.5 * 0.5);
        if (j == M) {
            const long long ct = pidx(g, i, M + 1, k);
            f.DST[ct + g.FS] = (F)R[ct];
            f.MST[ct] = (F)U0[ct];
            f.MST[ct + 2 * g.FS] = (F)U0[ct];
        }
    }
}

// DIVG_U_io; also VELOCITY_CALC_io of the upload (Q = G / D_STG) when vel != 0
template <typename F>
__global__ void __launch_bounds__(IO_NT) k_io_velocity(Geo g, IoFieldsT<F> f) {
    const long long tot = io_points(g);
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const long long c = pidx(g, i, j, k);
        const double g1 = f.G[c], g3 = f.G[c + 2 * g.FS], d1 = f.DST[c], d3 = f.DST[c + 2 * g.FS];
        f.Q[c] = (F)(g1 / d1);
        f.Q[c + 2 * g.FS] = (F)(g3 / d3);
        if (j >= 2) f.Q[c + g.FS] = (F)((double)f.G[c + g.FS] / (double)f.DST[c + g.FS]);
    }
}

template <typename F>
__global__ void __launch_bounds__(IO_NT) k_io_divu(Geo g, IoFieldsT<F> f) {
    const int L = g.L, N = g.N;  // L: row stride
    const long long tot = io_points(g);
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const long long c = pidx(g, i, j, k);
        const F* Q = f.Q;
        const double u = Q[c], up = Q[pidx(g, xpn(g, i), j, k)];
        const double v = Q[c + g.FS], vp = Q[c + g.FS + L];
        const double w = Q[c + 2 * g.FS], wp = Q[pidx(g, i, j, wrapp(k, N)) + 2 * g.FS];
        const double DIVX = (up - u) * g.dxi;
        const double DIVY = (vp - v) * (g.dyfi[j] * 1.0);
        const double DIVZ = (wp - w) * (g.dzi * 1.0);
        f.DIVU[c] = (F)((DIVX + DIVY + DIVZ) / 3.0);
    }
}

// ---------------------------------------------------------------------------
// CONVECTION_X/Y/Z_io + the viscous terms + RHS_MOM_EXPLICIT_io, all three
// components per point.
//   CN = false (VisExplicit): VISCOUS_ALL_EXPLT_X/Y/Z_io, RHS = RK combination.
//   CN = true  (VisImplicit): VISCOUS_PAR_EXPLT_X/Y/Z_io
//     (src/VISCOUS_X_EXPLICIT_io.f90:131-293, VISCOUS_Y_EXPLICIT_io.f90:278-443,
//     VISCOUS_Z_EXPLICIT_io.f90:300-465): the explicit part joins the
//     convection term, the implicit part enters with alpha*dt
//     (RHS_MOM_EXPLICIT_io.f90:87-99).  The density-correction part
//     (DIVU_io, weight alpha*dt/2) is identically zero: it differentiates
//     G * DRHOI_STG, and DRHOI_STG = 1/D_STG - 1/(the same average of
//     DENSITY0) is 0 in every entry because DENSITY_IMPLICIT_add runs right
//     after DENSITY_Staggered on the same DENSITY0 (src/SOLVE.f90:123-127,
//     src/MASSFLUX_CALC_IO.f90:332-416), and 0 before that (MEMALLOCT.f90:209).
//     It is therefore not computed.  The v row j = 1 is left unwritten; the
//     Crank-Nicolson sweeps treat it as zero.
template <bool CN, typename F>
__global__ void __launch_bounds__(IO_NT, 2) k_io_rhs(Geo g, IoFieldsT<F> f, double* __restrict__ partial, DevState* __restrict__ st,
                                                  int ns) {
    __shared__ double sred[32];
    __shared__ int is_last;
    const int N = g.N;
    const long long tot = io_points(g);
    const long long FS = g.FS;
    const double dt = st->dt, tg = g.tgam[ns], tr = g.troh[ns], ta = g.talp[ns];
    const double cv = g.cvisc;
    const F* G = f.G;
    const F* Q = f.Q;
    const double* U0 = f.MU0;
    const double* U = f.MU;
    const F* MS = f.MST;
    const F* DV = f.DIVU;
    const F* PR = f.PR;
    double bulk = 0.0;
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const int ip = xpn(g, i), im = xmn(g, i), kp = wrapp(k, N), km = wrapm(k, N);
        const int jp = j + 1, jm = j - 1;
        const long long c = pidx(g, i, j, k);
        const long long cip = pidx(g, ip, j, k), cim = pidx(g, im, j, k);
        const long long cjp = pidx(g, i, jp, k), cjm = pidx(g, i, jm, k);
        const long long ckp = pidx(g, i, j, kp), ckm = pidx(g, i, j, km);
        const double wffj = g.wff[j], wfbj = g.wfb[j], wffp = g.wff[jp], wfbp = g.wfb[jp];
        const double dyfij = g.dyfi[j], dycij = g.dyci[j], dycip = g.dyci[jp];
        // -------- x momentum: CONVECTION_X_io + viscous terms --------
        double ex1, ex2 = 0.0, ex3, im1 = 0.0, im2 = 0.0, im3 = 0.0;
        {
            const double H11F = (G[cip] + G[c]) * (Q[cip] + Q[c]);
            const double H11B = (G[c] + G[cim]) * (Q[c] + Q[cim]);
            const double H11 = (H11F - H11B) * (g.dxi * 0.5 * 0.5);
            const double H12F = (G[cjp + FS] + G[pidx(g, im, jp, k) + FS]) * (wffp * Q[cjp] + wfbp * Q[c]);
            const double H12B = (G[c + FS] + G[cim + FS]) * (wffj * Q[c] + wfbj * Q[cjm]);
            const double H12 = (H12F - H12B) * (dyfij * 0.5 * 1.0);
            const double H13F = (G[ckp + 2 * FS] + G[pidx(g, im, j, kp) + 2 * FS]) * (Q[ckp] + Q[c]);
            const double H13B = (G[c + 2 * FS] + G[cim + 2 * FS]) * (Q[c] + Q[ckm]);
            const double H13 = (H13F - H13B) * ((g.dzi * 0.5 * 0.5) * 1.0);
            ex1 = -(H11 + H12 + H13);
            if constexpr (!CN) {
                double DUDX = (Q[cip] - Q[c]) * g.dxi;
                const double T11F = 0.5 * (U0[c] + U0[c]) * (DUDX - DV[c]);
                DUDX = (Q[c] - Q[cim]) * g.dxi;
                const double T11B = 0.5 * (U0[cim] + U0[cim]) * (DUDX - DV[cim]);
                const double D11 = (T11F - T11B) * (2.0 * g.dxi * cv);
                double DUDY = (Q[cjp] - Q[c]) * dycip / 1.0;
                double DVDX = (Q[cjp + FS] - Q[pidx(g, im, jp, k) + FS]) * g.dxi;
                const double T12F = MS[cjp] * (DUDY + DVDX);
                DUDY = (Q[c] - Q[cjm]) * dycij / 1.0;
                DVDX = (Q[c + FS] - Q[cim + FS]) * g.dxi;
                const double T12B = MS[c] * (DUDY + DVDX);
                const double D12 = (T12F - T12B) * (dyfij * cv * 1.0);
                double DUDZ = (Q[ckp] - Q[c]) * g.dzi;
                double DWDX = (Q[ckp + 2 * FS] - Q[pidx(g, im, j, kp) + 2 * FS]) * g.dxi;
                const double T13F = MS[ckp + FS] * (DUDZ + DWDX);
                DUDZ = (Q[c] - Q[ckm]) * g.dzi;
                DWDX = (Q[c + 2 * FS] - Q[cim + 2 * FS]) * g.dxi;
                const double T13B = MS[c + FS] * (DUDZ + DWDX);
                const double D13 = (T13F - T13B) * ((g.dzi * cv) * 1.0);
                ex1 = ex1 + D11 + D12 + D13;
            } else {
                const double coe1 = -2.0 / 3.0 * g.dxi * cv;
                double DUDX = (Q[cip] - Q[c]) * g.dxi;
                double DVDY = (Q[cjp + FS] - Q[c + FS]) * dyfij * 1.0;
                double DWDZ = (Q[ckp + 2 * FS] - Q[c + 2 * FS]) * g.dzi * 1.0;
                const double F_EX11 = U[c] * (DVDY + DWDZ), F_IM11 = U[c] * DUDX;
                DUDX = (Q[c] - Q[cim]) * g.dxi;
                DVDY = (Q[pidx(g, im, jp, k) + FS] - Q[cim + FS]) * dyfij * 1.0;
                DWDZ = (Q[pidx(g, im, j, kp) + 2 * FS] - Q[cim + 2 * FS]) * g.dzi * 1.0;
                const double B_EX11 = U[cim] * (DVDY + DWDZ), B_IM11 = U[cim] * DUDX;
                const double D11_EX = (F_EX11 - B_EX11) * coe1;
                const double D11_IM = (F_IM11 - B_IM11) * coe1 * (-2.0);
                const double coe2 = dyfij * cv * 1.0;
                double DVDX = (Q[cjp + FS] - Q[pidx(g, im, jp, k) + FS]) * g.dxi;
                double DUDY = (Q[cjp] - Q[c]) * dycip / 1.0;
                const double F_EX12 = MS[cjp] * DVDX, F_IM12 = MS[cjp] * DUDY;
                DUDY = (Q[c] - Q[cjm]) * dycij / 1.0;
                DVDX = (Q[c + FS] - Q[cim + FS]) * g.dxi;
                const double B_EX12 = MS[c] * DVDX, B_IM12 = MS[c] * DUDY;
                const double D12_EX = (F_EX12 - B_EX12) * coe2;
                const double D12_IM = (F_IM12 - B_IM12) * coe2;
                const double coe32 = (g.dzi * cv) * 1.0;
                double DUDZ = (Q[ckp] - Q[c]) * g.dzi;
                double DWDX = (Q[ckp + 2 * FS] - Q[pidx(g, im, j, kp) + 2 * FS]) * g.dxi;
                const double F_EX13 = MS[ckp + FS] * DWDX, F_IM13 = MS[ckp + FS] * DUDZ;
                DUDZ = (Q[c] - Q[ckm]) * g.dzi;
                DWDX = (Q[c + 2 * FS] - Q[cim + 2 * FS]) * g.dxi;
                const double B_EX13 = MS[c + FS] * DWDX, B_IM13 = MS[c + FS] * DUDZ;
                const double D13_EX = (F_EX13 - B_EX13) * coe32;
                const double D13_IM = (F_IM13 - B_IM13) * coe32;
                ex1 = D11_EX + D12_EX + D13_EX + ex1;
                im1 = D11_IM + D12_IM + D13_IM;
            }
        }
        // -------- y momentum (j >= 2) --------
        if (j >= 2) {
            const double H21F = (wffj * G[cip] + wfbj * G[pidx(g, ip, jm, k)]) * (Q[cip + FS] + Q[c + FS]);
            const double H21B = (wffj * G[c] + wfbj * G[cjm]) * (Q[c + FS] + Q[cim + FS]);
            const double H21 = (H21F - H21B) * (g.dxi * 0.5);
            const double H22F = (G[cjp + FS] + G[c + FS]) * (Q[cjp + FS] * 1.0 + Q[c + FS] * 1.0);
            const double H22B = (G[c + FS] + G[cjm + FS]) * (Q[c + FS] * 1.0 + Q[cjm + FS] * 1.0);
            const double H22 = (H22F - H22B) * (dycij * 0.5 * 0.5);
            const double H23F = (wffj * G[ckp + 2 * FS] * 1.0 + wfbj * G[pidx(g, i, jm, kp) + 2 * FS] * 1.0) * (Q[ckp + FS] + Q[c + FS]);
            const double H23B = (wffj * G[c + 2 * FS] * 1.0 + wfbj * G[cjm + 2 * FS] * 1.0) * (Q[c + FS] + Q[ckm + FS]);
            const double H23 = (H23F - H23B) * ((g.dzi * 0.5) * 1.0);
            ex2 = -(H21 + H22 + H23);
            if constexpr (!CN) {
                double DVDY = (Q[cjp + FS] - Q[c + FS]) * dyfij;
                const double T22F = 0.5 * (U0[c] + U0[c]) * (DVDY - DV[c]);
                DVDY = (Q[c + FS] - Q[cjm + FS]) * g.dyfi[jm];
                const double T22B = 0.5 * (U0[cjm] + U0[cjm]) * (DVDY - DV[cjm]);
                const double D22 = (T22F - T22B) * (2.0 * dycij * cv);
                double DVDX = (Q[cip + FS] - Q[c + FS]) * g.dxi;
                double DUDY = (Q[cip] - Q[pidx(g, ip, jm, k)]) * dycij;
                const double T21F = MS[cip] * (DVDX + DUDY);
                DVDX = (Q[c + FS] - Q[cim + FS]) * g.dxi;
                DUDY = (Q[c] - Q[cjm]) * dycij;
                const double T21B = MS[c] * (DVDX + DUDY);
                const double D21 = (T21F - T21B) * (g.dxi * cv);
                double DVDZ = (Q[ckp + FS] - Q[c + FS]) * g.dzi;
                double DWDY = (Q[ckp + 2 * FS] - Q[pidx(g, i, jm, kp) + 2 * FS]) * dycij;
                const double T23F = MS[ckp + 2 * FS] * (DVDZ + DWDY);
                DVDZ = (Q[c + FS] - Q[ckm + FS]) * g.dzi;
                DWDY = (Q[c + 2 * FS] - Q[cjm + 2 * FS]) * dycij;
                const double T23B = MS[c + 2 * FS] * (DVDZ + DWDY);
                const double D23 = (T23F - T23B) * (g.dzi * cv);
                ex2 = ex2 + D21 + D22 + D23;
            } else {
                const double coe2 = -2.0 / 3.0 * dycij * cv;
                double DUDX = (Q[cip] - Q[c]) * g.dxi;
                double DVDY = (Q[cjp + FS] - Q[c + FS]) * dyfij;
                double DWDZ = (Q[ckp + 2 * FS] - Q[c + 2 * FS]) * g.dzi;
                const double F_EX22 = U[c] * (DUDX + DWDZ), F_IM22 = U[c] * DVDY;
                DUDX = (Q[pidx(g, ip, jm, k)] - Q[cjm]) * g.dxi;
                DVDY = (Q[c + FS] - Q[cjm + FS]) * g.dyfi[jm];
                DWDZ = (Q[pidx(g, i, jm, kp) + 2 * FS] - Q[cjm + 2 * FS]) * g.dzi;
                const double B_EX22 = U[cjm] * (DUDX + DWDZ), B_IM22 = U[cjm] * DVDY;
                const double D22_EX = (F_EX22 - B_EX22) * coe2;
                const double D22_IM = (F_IM22 - B_IM22) * coe2 * (-2.0);
                const double coe1 = g.dxi * cv;
                double DVDX = (Q[cip + FS] - Q[c + FS]) * g.dxi;
                double DUDY = (Q[cip] - Q[pidx(g, ip, jm, k)]) * dycij;
                const double F_EX21 = MS[cip] * DUDY, F_IM21 = MS[cip] * DVDX;
                DVDX = (Q[c + FS] - Q[cim + FS]) * g.dxi;
                DUDY = (Q[c] - Q[cjm]) * dycij;
                const double B_EX21 = MS[c] * DUDY, B_IM21 = MS[c] * DVDX;
                const double D21_EX = (F_EX21 - B_EX21) * coe1;
                const double D21_IM = (F_IM21 - B_IM21) * coe1;
                const double coe3 = g.dzi * cv;
                double DVDZ = (Q[ckp + FS] - Q[c + FS]) * g.dzi;
                double DWDY = (Q[ckp + 2 * FS] - Q[pidx(g, i, jm, kp) + 2 * FS]) * dycij;
                const double F_EX23 = MS[ckp + 2 * FS] * DWDY, F_IM23 = MS[ckp + 2 * FS] * DVDZ;
                DVDZ = (Q[c + FS] - Q[ckm + FS]) * g.dzi;
                DWDY = (Q[c + 2 * FS] - Q[cjm + 2 * FS]) * dycij;
                const double B_EX23 = MS[c + 2 * FS] * DWDY, B_IM23 = MS[c + 2 * FS] * DVDZ;
                const double D23_EX = (F_EX23 - B_EX23) * coe3;
                const double D23_IM = (F_IM23 - B_IM23) * coe3;
                ex2 = D21_EX + D22_EX + D23_EX + ex2;
                im2 = D21_IM + D22_IM + D23_IM;
            }
        }
        // -------- z momentum --------
        {
            const double H31F = (G[cip] + G[pidx(g, ip, j, km)]) * (Q[cip + 2 * FS] + Q[c + 2 * FS]);
            const double H31B = (G[c] + G[ckm]) * (Q[c + 2 * FS] + Q[cim + 2 * FS]);
            const double H31 = (H31F - H31B) * (g.dxi * 0.5 * 0.5);
            const double H32F = (G[cjp + FS] + G[pidx(g, i, jp, km) + FS]) * (wffp * Q[cjp + 2 * FS] * 1.0 + wfbp * Q[c + 2 * FS] * 1.0);
            const double H32B = (G[c + FS] + G[ckm + FS]) * (wffj * Q[c + 2 * FS] * 1.0 + wfbj * Q[cjm + 2 * FS] * 1.0);
            const double H32 = (H32F - H32B) * (dyfij * 0.5);
            const double H33F = (G[ckp + 2 * FS] + G[c + 2 * FS]) * (Q[ckp + 2 * FS] + Q[c + 2 * FS]);
            const double H33B = (G[c + 2 * FS] + G[ckm + 2 * FS]) * (Q[c + 2 * FS] + Q[ckm + 2 * FS]);
            const double H33 = (H33F - H33B) * ((g.dzi * 0.5 * 0.5) * 1.0);
            ex3 = -(H31 + H32 + H33);
            if constexpr (!CN) {
                double DWDZ = (Q[ckp + 2 * FS] - Q[c + 2 * FS]) * g.dzi;
                const double T33F = 0.5 * (U0[c] + U0[c]) * (DWDZ - DV[c]);
                DWDZ = (Q[c + 2 * FS] - Q[ckm + 2 * FS]) * g.dzi;
                const double T33B = 0.5 * (U0[ckm] + U0[ckm]) * (DWDZ - DV[ckm]);
                const double D33 = (T33F - T33B) * (2.0 * g.dzi * cv);
                double DWDX = (Q[cip + 2 * FS] - Q[c + 2 * FS]) * g.dxi;
                double DUDZ = (Q[cip] - Q[pidx(g, ip, j, km)]) * g.dzi;
                const double T31F = MS[cip + FS] * (DWDX + DUDZ);
                DWDX = (Q[c + 2 * FS] - Q[cim + 2 * FS]) * g.dxi;
                DUDZ = (Q[c] - Q[ckm]) * g.dzi;
                const double T31B = MS[c + FS] * (DWDX + DUDZ);
                const double D31 = (T31F - T31B) * (g.dxi * cv);
                double DWDY = (Q[cjp + 2 * FS] - Q[c + 2 * FS]) * dycip;
                double DVDZ = (Q[cjp + FS] - Q[pidx(g, i, jp, km) + FS]) * g.dzi;
                const double T32F = MS[cjp + 2 * FS] * (DWDY + DVDZ);
                DWDY = (Q[c + 2 * FS] - Q[cjm + 2 * FS]) * dycij;
                DVDZ = (Q[c + FS] - Q[ckm + FS]) * g.dzi;
                const double T32B = MS[c + 2 * FS] * (DWDY + DVDZ);
                const double D32 = (T32F - T32B) * (dyfij * cv);
                ex3 = ex3 + D31 + D32 + D33;
            } else {
                const double coe3 = -2.0 / 3.0 * g.dzi * cv;
                double DUDX = (Q[cip] - Q[c]) * g.dxi;
                double DVDY = (Q[cjp + FS] - Q[c + FS]) * dyfij;
                double DWDZ = (Q[ckp + 2 * FS] - Q[c + 2 * FS]) * g.dzi;
                const double F_EX33 = U[c] * (DUDX + DVDY), F_IM33 = U[c] * DWDZ;
                DUDX = (Q[pidx(g, ip, j, km)] - Q[ckm]) * g.dxi;
                DVDY = (Q[pidx(g, i, jp, km) + FS] - Q[ckm + FS]) * dyfij;
                DWDZ = (Q[c + 2 * FS] - Q[ckm + 2 * FS]) * g.dzi;
                const double B_EX33 = U[ckm] * (DUDX + DVDY), B_IM33 = U[ckm] * DWDZ;
                const double D33_EX = (F_EX33 - B_EX33) * coe3;
                const double D33_IM = (F_IM33 - B_IM33) * coe3 * (-2.0);
                const double coe1 = g.dxi * cv;
                double DWDX = (Q[cip + 2 * FS] - Q[c + 2 * FS]) * g.dxi;
                double DUDZ = (Q[cip] - Q[pidx(g, ip, j, km)]) * g.dzi;
                const double F_EX31 = MS[cip + FS] * DUDZ, F_IM31 = MS[cip + FS] * DWDX;
                DWDX = (Q[c + 2 * FS] - Q[cim + 2 * FS]) * g.dxi;
                DUDZ = (Q[c] - Q[ckm]) * g.dzi;
                const double B_EX31 = MS[c + FS] * DUDZ, B_IM31 = MS[c + FS] * DWDX;
                const double D31_EX = (F_EX31 - B_EX31) * coe1;
                const double D31_IM = (F_IM31 - B_IM31) * coe1;
                const double coe2 = dyfij * cv;
                double DWDY = (Q[cjp + 2 * FS] - Q[c + 2 * FS]) * dycip;
                double DVDZ = (Q[cjp + FS] - Q[pidx(g, i, jp, km) + FS]) * g.dzi;
                const double F_EX32 = MS[cjp + 2 * FS] * DVDZ, F_IM32 = MS[cjp + 2 * FS] * DWDY;
                DWDY = (Q[c + 2 * FS] - Q[cjm + 2 * FS]) * dycij;
                DVDZ = (Q[c + FS] - Q[ckm + FS]) * g.dzi;
                const double B_EX32 = MS[c + 2 * FS] * DVDZ, B_IM32 = MS[c + 2 * FS] * DWDY;
                const double D32_EX = (F_EX32 - B_EX32) * coe2;
                const double D32_IM = (F_IM32 - B_IM32) * coe2;
                ex3 = D31_EX + D32_EX + D33_EX + ex3;
                im3 = D31_IM + D32_IM + D33_IM;
            }
        }
        // -------- RHS_MOM_EXPLICIT_io --------
        const long long ii = io_iidx(g, i, j, k);
        // with inflow the inlet face u(1) is a boundary value: its x-momentum RHS, EXPLT0 and
        // G are left alone (NXI = 2, src/RHS_MOM_EXPLICIT_io.f90:35)
        const bool ux = !(g.xo && i == 1);
        const double e01 = f.EX0[ii], e02 = f.EX0[ii + g.FI], e03 = f.EX0[ii + 2 * g.FI];
        const double pc = PR[c], pim = PR[cim], pjm = PR[cjm], pkm = PR[ckm];
        const double coa = ta * dt;
        // buoyancy (:161-226): D_STG * TALP*DT*F_A on the component |iGravity| (1/RNDI1 = 1/RCCI1 = 1)
        const int ig = f.igrav < 0 ? -f.igrav : f.igrav;
        const double cob = ta * dt * f.fa;
        double r1 = (tg * ex1 + tr * e01) * dt;
        if constexpr (CN) r1 = r1 + coa * im1;
        r1 = r1 - io_pgm(f, c, cim, pc, pim, ta * dt * g.dxi);
        if (ig == 1) r1 = r1 + f.DST[c] * cob;
        double r3 = (tg * ex3 + tr * e03) * dt;
        if constexpr (CN) r3 = r3 + coa * im3;
        r3 = r3 - io_pgm(f, c, ckm, pc, pkm, ta * dt * g.dzi);
        if (ig == 3) r3 = r3 + f.DST[c + 2 * FS] * (cob / 1.0);
        if (ux) {
            f.EX0[ii] = (F)ex1;
            f.RHS[ii] = (F)r1;
        }
        f.EX0[ii + 2 * g.FI] = (F)ex3;
        f.RHS[ii + 2 * g.FI] = (F)r3;
        if (j >= 2) {
            double r2 = (tg * ex2 + tr * e02) * dt;
            if constexpr (CN) r2 = r2 + coa * im2;
            r2 = r2 - io_pgm(f, c, cjm, pc, pjm, ta * dt * dycij / 1.0);
            if (ig == 2) r2 = r2 + f.DST[c + FS] * (cob / 1.0);
            f.EX0[ii + g.FI] = (F)ex2;
            f.RHS[ii + g.FI] = (F)r2;
        }
        if (ux) bulk += r1 / dyfij / 1.0;
    }
    double s = block_sum<IO_NT>(bulk, sred);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = s;
        __threadfence();
        const unsigned prev = atomicAdd(&st->ctr, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        double a = 0.0;
        for (int t = threadIdx.x; t < (int)gridDim.x; t += IO_NT) a += __ldcg(partial + t);
        a = block_sum<IO_NT>(a, sred);
        if (threadIdx.x == 0) {
            st->bulksum = a;
            st->ctr = 0u;
        }
    }
}

// bulk forcing (RHS_MOM_EXPLICIT_io :228-265) + MASSFLUX_CALC_io
template <typename F>
__global__ void __launch_bounds__(IO_NT) k_io_massflux(Geo g, IoFieldsT<F> f, const DevState* __restrict__ st, int ns) {
    const long long tot = io_points(g);
    double dpg = 0.0;
    if (g.iflowdriven == 1) dpg = st->bulksum / g.volm;
    else if (g.iflowdriven == 2) dpg = -0.5 * g.cf_given * (g.talp[ns] * st->dt);
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const long long c = pidx(g, i, j, k), ii = io_iidx(g, i, j, k);
        const double g1 = f.G[c], g2 = f.G[c + g.FS], g3 = f.G[c + 2 * g.FS];
        const double r1 = f.RHS[ii] - dpg, r3 = f.RHS[ii + 2 * g.FI];
        if (!(g.xo && i == 1)) f.G[c] = (F)(g1 + r1);  // NXI = 2 with inflow
        f.G[c + 2 * g.FS] = (F)(g3 + r3);
        if (j >= 2) f.G[c + g.FS] = (F)(g2 + (double)f.RHS[ii + g.FI]);
    }
}

// DIVG_io + forward x transform (same tiling as k_div_fftx)
// DRHO: DrhoDtP of the thermal solver, or NULL (zero) while it is off;
// the divergence is divided by wdiv (DIVG.f90:78-82)
template <int N1, int N2, typename F>
__global__ void __launch_bounds__(PX_NT, PX_MINB) k_io_div_fftx(Geo g, const F* __restrict__ G, double* __restrict__ RHSLL,
                                                       double2* __restrict__ SP, const DevState* __restrict__ st, int ns,
                                                       const double* __restrict__ DRHO, double wdiv) {
    extern __shared__ double2 smc[];
    const int L = g.L, M = g.M, N = g.N, LH = g.LH;
    const int LD = fft4s_ld(L);
    const int j0 = 1 + blockIdx.x * PX_TJ;
    const int k = blockIdx.y;
    const int nj = min(PX_TJ, M - j0 + 1);
    const int np = (nj + 1) >> 1;
    const int kp = wrapp(k, N);
    // wdiv: 0.25 + pres_epslon with iWeightedPre = 1, else 1 (an exact division)
    const double coe0 = 1.0 / st->dt / g.talp[ns] / wdiv;
    const double coe1 = g.dxi / 1.0;
#pragma unroll 4
    for (int p = threadIdx.x; p < 2 * np * L; p += PX_NT) {
        const int jl = p / L, i = p - jl * L;
        const int pair = jl >> 1, part = jl & 1;
        double val = 0.0;
        if (jl < nj) {
            const int j = j0 + jl;
            const long long c = pidx(g, i, j, k);
            const double u = G[c], up = G[pidx(g, wrapp(i, L), j, k)];
            const double v = G[c + g.FS], vp = G[c + g.FS + L];
            const double w = G[c + 2 * g.FS], wp = G[pidx(g, i, j, kp) + 2 * g.FS];
            const double coe2 = g.dyfi[j] / 1.0;
            const double DIVX = (up - u) * coe1, DIVY = (vp - v) * coe2, DIVZ = (wp - w) * g.dzi;
            const double DTRHO = DRHO ? DRHO[c] / 1.0 : 0.0;
            const double DQ = DIVX + DIVY + DIVZ + DTRHO;
            val = DQ * coe0;
            RHSLL[iidx(g, i, j, k)] = val;
        }
        double2* line = smc + pair * LD;
        if (part == 0) line[i].x = val; else line[i].y = val;
    }
    block_fft4s<N1, N2, -1>(smc, np, LD, g.twx);
    const double sc = 0.5 / (double)L;
    for (int p = threadIdx.x; p < np * LH; p += PX_NT) {
        const int pair = p / LH, kx = p - pair * LH;
        const double2* line = smc + pair * LD;
        const double2 z = line[kx];
        const double2 zc = line[kx == 0 ? 0 : L - kx];
        const int ja = j0 + 2 * pair;
        SP[kx + (long long)LH * ((ja - 1) + (long long)M * k)] = make_double2((z.x + zc.x) * sc, (z.y - zc.y) * sc);
        if (2 * pair + 1 < nj)
            SP[kx + (long long)LH * ((ja) + (long long)M * k)] = make_double2((z.y + zc.y) * sc, (zc.x - z.x) * sc);
    }
}

// PRCALC_io + MASSFLUX_UPDATE_io + VELOCITY_CALC_io.  RHSLL == NULL: the
// explicit scheme's PR += DPH; otherwise the Crank-Nicolson scheme's
// PR += DPH - BE * RHSLLPHI_io, BE = alpha*dt/(2 Re) (src/PRESSURE_CORRECTION.f90:113-123).
template <typename F>
__global__ void __launch_bounds__(IO_NT) k_io_correct(Geo g, IoFieldsT<F> f, const double* __restrict__ DPH,
                                                      const DevState* __restrict__ st, int ns,
                                                      const double* __restrict__ RHSLL) {
    const int M = g.M, N = g.N;
    const long long tot = io_points(g);
    const double dt = st->dt, ta = g.talp[ns];
    const double be = 0.50 * ta * dt * g.cvisc;
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const long long c = pidx(g, i, j, k);
        const double ph = DPH[c];
        const double phim = DPH[pidx(g, xmn(g, i), j, k)];
        const double phkm = DPH[pidx(g, i, j, wrapm(k, N))];
        const double phjm = j >= 2 ? DPH[pidx(g, i, j - 1, k)] : 0.0;
        const double g1 = f.G[c], g2 = f.G[c + g.FS], g3 = f.G[c + 2 * g.FS], pr = f.PR[c];
        const double d1 = f.DST[c], d2 = f.DST[c + g.FS], d3 = f.DST[c + 2 * g.FS];
        const double pn = RHSLL ? pr + ph - be * RHSLL[io_iidx(g, i, j, k)] : pr + ph;
        f.PR[c] = (F)pn;
        if (j == 1) f.PR[pidx(g, i, 0, k)] = (F)pn;
        if (j == M) f.PR[pidx(g, i, M + 1, k)] = (F)pn;
        // u faces NXI..NXE: 1..L, or 2..L+1 with inflow (MASSFLUX_UPDATE_io, src/VELO_CORRECTION.f90:121-137);
        // VELOCITY_CALC_io still divides the fixed inlet face, and leaves the outlet face's Q alone
        const double n1 = (g.xo && i == 1) ? g1 : g1 - (ph - phim) * (dt * ta * g.dxi);
        const double n3 = g3 - (ph - phkm) * (dt * ta * g.dzi);
        f.G[c] = (F)n1;
        if (g.xo && i == g.LI) {
            const double go = f.G[c + 1];
            f.G[c + 1] = (F)(go - (DPH[c + 1] - ph) * (dt * ta * g.dxi));
        }
        f.G[c + 2 * g.FS] = (F)n3;
        f.Q[c] = (F)(n1 / d1);
        f.Q[c + 2 * g.FS] = (F)(n3 / d3);
        if (j >= 2) {
            const double n2 = g2 - (ph - phjm) * (dt * ta * g.dyci[j] / 1.0);
            f.G[c + g.FS] = (F)n2;
            f.Q[c + g.FS] = (F)(n2 / d2);
        }
    }
}

template <typename F>
__global__ void __launch_bounds__(IO_NT) k_io_cfl(Geo g, IoFieldsT<F> f, double* __restrict__ partial, DevState* __restrict__ st) {
    __shared__ double sred[32];
    const int L = g.L, N = g.N;  // L: row stride
    const long long tot = io_points(g);
    double mx = 0.0;
    bool bad = false;
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const long long c = pidx(g, i, j, k);
        const F* Q = f.Q;
        double q = (fabs(((double)Q[c] + (double)Q[pidx(g, xpn(g, i), j, k)]) * g.dxi) +
                    fabs(((double)Q[c + g.FS] + (double)Q[c + g.FS + L]) * g.dyfi[j] * 1.0) +
                    fabs(((double)Q[c + 2 * g.FS] + (double)Q[pidx(g, i, j, wrapp(k, N)) + 2 * g.FS]) * g.dzi * 1.0)) * 0.5;
        const double vcf = 2.0 * g.cvisc * (g.dxqi + g.dzqi * 1.0 + g.dyfi[j] * g.dyfi[j]) * f.MU[c] / f.DEN[c];
        if (!(q == q) || !(vcf == vcf)) bad = true;
        q = fmax(q, vcf);
        mx = fmax(mx, q);
    }
    if (bad) atomicOr(&st->err, CHS_EBIT_NAN);
    if (blockIdx.x == 0 && threadIdx.x == 0) st->dtprev = st->dt;
    double r = block_max<IO_NT>(mx, sred);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

// DIVGCK_io (src/DIVGCK.f90:60-121 with DIVGCK_Comm_io :125-184), x-periodic
// main domain: max over the interior of |div G + DrhoDtP| (all three ranges of
// MAXDIVGV_io coincide).  Per-block maxima; k_maxdiv_final reduces them.  DRHO
// is NULL while the thermal solver is off (DrhoDtP = 0).
template <typename F>
__global__ void __launch_bounds__(IO_NT) k_io_divgck(Geo g, const F* __restrict__ G,
                                                     const double* __restrict__ DRHO, double* __restrict__ partial) {
    __shared__ double sred[32];
    const int L = g.L, N = g.N;  // L: row stride
    const long long tot = io_points(g);
    double mx = 0.0;
    for (long long t = (long long)blockIdx.x * IO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * IO_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const long long c = pidx(g, i, j, k);
        const double DIVX = ((double)G[pidx(g, xpn(g, i), j, k)] - (double)G[c]) * g.dxi;
        const double DIVY = ((double)G[c + g.FS + L] - (double)G[c + g.FS]) * (g.dyfi[j] * 1.0);
        const double DIVZ = ((double)G[pidx(g, i, j, wrapp(k, N)) + 2 * g.FS] - (double)G[c + 2 * g.FS]) * (g.dzi * 1.0);
        const double DTRHO = DRHO ? DRHO[c] : 0.0;
        const double DQCAP = DIVX + DIVY + DIVZ + DTRHO;
        mx = fmax(fabs(DQCAP), mx);
    }
    const double r = block_max<IO_NT>(mx, sred);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}
