// Momentum part of one RK3 substep of the periodic channel:
// SOLVERRK3_MOM_tg (src/SOLVERRK3_MOM_tg.f90:22-35) =
//   CONVECTION_X/Y/Z_tg + 3 x (RHS_CvLpGpS_tg + MOMFA_tg).
//
// Kernel split (all three velocity components per kernel):
//   k_rhs_xsweep : convection (CONVECTION_X_tg :13-64, CONVECTION_Y_tg
//                  :13-114, CONVECTION_Z_tg :13-103), RK combination,
//                  viscous and pressure-gradient terms (RHS_CvLpGpS_tg
//                  :97-161), CONVH0 update, per-block partial sums of the
//                  bulk-flux forcing (:163-181), then the cyclic x sweep
//                  (MOMFA1_X_tg, src/MOMFA_tg.f90:51-106) in shared memory.
//   k_zsweep     : cyclic z sweep (MOMFA2_Z_tg :110-169).
//   k_ysweep     : forcing subtraction, non-cyclic y sweep (MOMFA3_Y_tg
//                  :172-238) and Q += dQ (MOMFA_tg :38-44).
// The reference subtracts the forcing DPGRNS before the x sweep.  The x and
// z operators are circulant with rows summing to one, so a constant passes
// through both sweeps unchanged (to round-off) and the subtraction is
// applied before the y sweep instead, where the global sum is available.
//
// Reference quirk reproduced: for the v component (IDR = 2) the y sweep runs
// over rows j = 1..M although RHS_CvLpGpS_tg only writes rows 2..M; row 1 of
// the shared RHS array still holds the u increment of the same substep, and
// through the coupling of row 2 to row 1 it enters the v solution.  With
// Geo::fix_v_wall_row = 1 that row is zeroed instead.
#pragma once
#include "common.cuh"
#include "tdma.cuh"

#define RHS_TJ 8        // x-lines (consecutive j at fixed k) per block
#define RHS_NT 256
#define SWEEP_NT 256

// ---------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(RHS_NT) k_rhs_xsweep(Geo g, const double* __restrict__ Q, const double* __restrict__ PR,
                                                       double* __restrict__ H0, double* __restrict__ RHS,
                                                       double* __restrict__ partial, const DevState* __restrict__ st, int ns) {
    extern __shared__ double sm[];
    const int L = g.L, M = g.M, N = g.N;
    const int LS = L + 32 + 1;  // smem line stride (segment padded, odd)
    const int j0 = 1 + blockIdx.x * RHS_TJ;
    const int k = blockIdx.y;
    const int nj = min(RHS_TJ, M - j0 + 1);
    const double dt = st->dt;
    const double tg = g.tgam[ns], tr = g.troh[ns], ta = g.talp[ns];
    const double coev = ta * g.cvisc;           // COE1 of RHS_CvLpGpS_tg
    const double coep = ta * dt;                // COE2 (pressure gradient)
    const int kp = wrapp(k, N), km = wrapm(k, N);
    const double* U = Q;
    const double* V = Q + g.FS;
    const double* W = Q + 2 * g.FS;
    double* sr = sm;                              // [3][RHS_TJ][LS]
    double* sred = sm + 3 * RHS_TJ * LS;          // [32]
    double bulk = 0.0;
    const double c1x = 0.5 * 0.5 * g.dxi;         // XND2CL*XND2CL*DXI
    const double c3x = 0.5 * 0.5 * g.dzi;
    for (int p = threadIdx.x; p < nj * L; p += RHS_NT) {
        const int jl = p / L;
        const int i = p - jl * L;
        const int j = j0 + jl, jp = j + 1, jm = j - 1;
        const int ip = wrapp(i, L), im = wrapm(i, L);
        const double wffj = g.wff[j], wfbj = g.wfb[j], wffp = g.wff[jp], wfbp = g.wfb[jp];
        const long long c = pidx(g, i, j, k);
        const long long cip = pidx(g, ip, j, k), cim = pidx(g, im, j, k);
        const long long cjp = pidx(g, i, jp, k), cjm = pidx(g, i, jm, k);
        const long long ckp = pidx(g, i, j, kp), ckm = pidx(g, i, j, km);
        const double u = U[c], v = V[c], w = W[c];
        const double pc = PR[c];
        const long long ii = iidx(g, i, j, k);
        const int srow = jl * LS + seg_pos<S>(i);
        // ---------------- u (CONVECTION_X_tg) ----------------
        {
            const double uip = U[cip], uim = U[cim];
            const double H11 = ((uip + u) * (uip + u) - (uim + u) * (uim + u)) * c1x;
            const double coe2 = g.dyfi[j] * 0.5 * 1.0;
            const double H12 = ((V[cjp] + V[pidx(g, im, jp, k)]) * (wffp * U[cjp] + wfbp * u) -
                                (v + V[cim]) * (wffj * u + wfbj * U[cjm])) * coe2;
            const double coe3 = 0.5 * 0.5 * g.dzi * 1.0;
            const double H13 = ((W[ckp] + W[pidx(g, im, j, kp)]) * (U[ckp] + u) - (w + W[cim]) * (u + U[ckm])) * coe3;
            const double H = -(H11 + H12 + H13);
            const double rhsc = tg * H + tr * H0[ii];
            const double rhsl = coev * ((uip - 2.0 * u + uim) * g.dxqi + (U[ckp] - 2.0 * u + U[ckm]) * g.dzqi * 1.0 +
                                        (U[cjp] * g.apvr[j] + u * g.acvr[j] + U[cjm] * g.amvr[j]));
            H0[ii] = H;
            double r = (rhsc + rhsl) * dt;
            r = r - (pc - PR[cim]) * g.dxi * coep;
            bulk += r / g.dyfi[j] / 1.0;
            sr[0 * RHS_TJ * LS + srow] = r;
        }
        // ---------------- v (CONVECTION_Y_tg), j >= 2 ----------------
        if (j >= 2) {
            const double vip = V[cip], vim = V[cim];
            const double coe1 = g.dxi * 0.5;
            const double H21 = ((wffj * U[cip] + wfbj * U[pidx(g, ip, jm, k)]) * (vip + v) -
                                (wffj * u + wfbj * U[cjm]) * (v + vim)) * coe1;
            const double vjp = V[cjp], vjm = V[cjm];
            const double coe2 = g.dyci[j] * 0.5 * 0.5;
            const double H22 = ((vjp * 1.0 + v * 1.0) * (vjp + v) - (v * 1.0 + vjm * 1.0) * (v + vjm)) * coe2;
            const double coe31 = g.dzi * 0.5 * 1.0;
            const double vkp = V[ckp], vkm = V[ckm];
            const double H23 = ((wffj * W[ckp] * 1.0 + wfbj * W[pidx(g, i, jm, kp)] * 1.0) * (vkp + v) -
                                (wffj * w * 1.0 + wfbj * W[cjm] * 1.0) * (v + vkm)) * coe31;
            const double H = -(H21 + H22 + H23);
            const long long iv = ii + g.FI;
            const double rhsc = tg * H + tr * H0[iv];
            const double* amv = g.amvr + (M + 2);
            const double* acv = g.acvr + (M + 2);
            const double* apv = g.apvr + (M + 2);
            const double rhsl = coev * ((vip - 2.0 * v + vim) * g.dxqi + (vkp - 2.0 * v + vkm) * g.dzqi * 1.0 +
                                        (vjp * apv[j] + v * acv[j] + vjm * amv[j]));
            H0[iv] = H;
            double r = (rhsc + rhsl) * dt;
            r = r - (pc - PR[cjm]) * (g.dyci[j] / 1.0) * coep;
            sr[1 * RHS_TJ * LS + srow] = r;
        }
        // ---------------- w (CONVECTION_Z_tg) ----------------
        {
            const double wip = W[cip], wim = W[cim], wkp = W[ckp], wkm = W[ckm];
            const double H31 = ((U[cip] + U[pidx(g, ip, j, km)]) * (wip + w) - (u + U[ckm]) * (w + wim)) * c1x;
            const double coe2 = g.dyfi[j] * 0.5;
            const double H32 = ((V[cjp] + V[pidx(g, i, jp, km)]) * (wffp * W[cjp] * 1.0 + wfbp * w * 1.0) -
                                (v + V[ckm]) * (wffj * w * 1.0 + wfbj * W[cjm] * 1.0)) * coe2;
            const double H33 = ((wkp + w) * (wkp + w) - (w + wkm) * (w + wkm)) * c3x;
            const double H = -(H31 + H32 + H33);
            const long long iw = ii + 2 * g.FI;
            const double rhsc = tg * H + tr * H0[iw];
            const double* amw = g.amvr + 2 * (M + 2);
            const double* acw = g.acvr + 2 * (M + 2);
            const double* apw = g.apvr + 2 * (M + 2);
            const double rhsl = coev * ((wip - 2.0 * w + wim) * g.dxqi + (wkp - 2.0 * w + wkm) * g.dzqi * 1.0 +
                                        (W[cjp] * apw[j] + w * acw[j] + W[cjm] * amw[j]));
            H0[iw] = H;
            double r = (rhsc + rhsl) * dt;
            r = r - (pc - PR[ckm]) * g.dzi * coep;
            sr[2 * RHS_TJ * LS + srow] = r;
        }
    }
    // bulk-flux partial sum of this block (RHS of u before any sweep)
    double tot = block_sum<RHS_NT>(bulk, sred);
    if (threadIdx.x == 0) partial[blockIdx.x + gridDim.x * blockIdx.y] = tot;
    __syncthreads();
    // cyclic x sweep, one warp per line
    const double facoe = 0.5 * ta * dt * g.cvisc * 1.0 / 1.0;
    ConstCoef cf;
    cf.a = -facoe * g.dxqi;
    cf.c = cf.a;
    cf.b = 1.0 - cf.c - cf.a;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = warp; t < 3 * nj; t += RHS_NT / 32) {
        const int comp = t / nj, jl = t - comp * nj;
        if (comp == 1 && j0 + jl == 1) continue;  // MOMFA1_X_tg starts at N2I = 2 for v
        warp_tdma_smem<S, true>(sr + comp * RHS_TJ * LS + jl * LS, cf, lane);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < nj * L; p += RHS_NT) {
        const int jl = p / L;
        const int i = p - jl * L;
        const int j = j0 + jl;
        const long long ii = iidx(g, i, j, k);
        const int srow = jl * LS + seg_pos<S>(i);
        RHS[ii] = sr[srow];
        if (j >= 2) RHS[ii + g.FI] = sr[RHS_TJ * LS + srow];
        RHS[ii + 2 * g.FI] = sr[2 * RHS_TJ * LS + srow];
    }
}

// ---------------------------------------------------------------------------
// cyclic z sweep: block = 32 consecutive i at fixed j, all k, one component
template <int S>
__global__ void __launch_bounds__(SWEEP_NT) k_zsweep(Geo g, double* __restrict__ RHS, const DevState* __restrict__ st, int ns) {
    extern __shared__ double sm[];
    const int L = g.L, N = g.N;
    const int i0 = blockIdx.x * 32;
    const int j = 1 + blockIdx.y;
    const int comp = blockIdx.z;
    if (comp == 1 && j == 1) return;  // MOMFA2_Z_tg starts at N2I = 2 for v
    const int ni = min(32, L - i0);
    const int LS = N + 32 + 1;
    double* R = RHS + comp * g.FI;
    for (int p = threadIdx.x; p < 32 * N; p += SWEEP_NT) {
        const int kk = p >> 5, il = p & 31;
        if (il < ni) sm[il * LS + seg_pos<S>(kk)] = R[iidx(g, i0 + il, j, kk)];
    }
    __syncthreads();
    const double facoe = 0.5 * g.talp[ns] * st->dt * g.cvisc * 1.0 / 1.0;
    ConstCoef cf;
    cf.a = 1.0 * (-facoe * g.dzqi);
    cf.c = cf.a;
    cf.b = 1.0 - cf.c - cf.a;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int il = warp; il < ni; il += SWEEP_NT / 32) warp_tdma_smem<S, true>(sm + il * LS, cf, lane);
    __syncthreads();
    for (int p = threadIdx.x; p < 32 * N; p += SWEEP_NT) {
        const int kk = p >> 5, il = p & 31;
        if (il < ni) R[iidx(g, i0 + il, j, kk)] = sm[il * LS + seg_pos<S>(kk)];
    }
}

// ---------------------------------------------------------------------------
// y sweep + Q update: block = 32 consecutive i at fixed k, all j, u then v then w
template <int S>
__global__ void __launch_bounds__(SWEEP_NT) k_ysweep(Geo g, double* __restrict__ Q, const double* __restrict__ RHS,
                                                     const double* __restrict__ partial, int npartial,
                                                     const DevState* __restrict__ st, int ns) {
    extern __shared__ double sm[];
    const int L = g.L, M = g.M;
    const int i0 = blockIdx.x * 32;
    const int k = blockIdx.y;
    const int ni = min(32, L - i0);
    const int LS = M + 32 + 1;
    double* sl = sm;                         // [32][LS]
    double* ca = sm + 32 * LS;               // [M] a
    double* cb = ca + M;                     // [M] b
    double* cc = cb + M;                     // [M] c
    double* sdu = cc + M;                    // [32] u increment at j = 1
    double* sred = sdu + 32;                 // [32]
    const double dt = st->dt;
    const double facoe = 0.5 * g.talp[ns] * dt * g.cvisc * 1.0 / 1.0;
    // DPGRNS (RHS_CvLpGpS_tg :163-199)
    double dpg = 0.0;
    if (g.iflowdriven == 1) {
        double s = 0.0;
        for (int t = threadIdx.x; t < npartial; t += SWEEP_NT) s += partial[t];
        s = block_sum<SWEEP_NT>(s, sred);
        if (threadIdx.x == 0) sred[0] = s / g.volm;
        __syncthreads();
        dpg = sred[0];
    } else if (g.iflowdriven == 2) {
        dpg = -0.5 * g.cf_given * (g.talp[ns] * dt / 1.0);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int comp = 0; comp < 3; ++comp) {
        const double* amv = g.amvr + comp * (M + 2);
        const double* acv = g.acvr + comp * (M + 2);
        const double* apv = g.apvr + comp * (M + 2);
        __syncthreads();
        for (int j = 1 + threadIdx.x; j <= M; j += SWEEP_NT) {
            cb[j - 1] = 1.0 - facoe * acv[j];
            cc[j - 1] = -facoe * apv[j];
            ca[j - 1] = -facoe * amv[j];
        }
        const double* R = RHS + comp * g.FI;
        for (int p = threadIdx.x; p < 32 * M; p += SWEEP_NT) {
            const int jl = p >> 5, il = p & 31;  // jl = j - 1
            if (il >= ni) continue;
            double r;
            if (comp == 1 && jl == 0) r = g.fix_v_wall_row ? 0.0 : sdu[il];
            else r = R[iidx(g, i0 + il, jl + 1, k)];
            if (comp == 0) r = r - dpg;
            sl[il * LS + seg_pos<S>(jl)] = r;
        }
        __syncthreads();
        SmemCoef cf{ca, cb, cc};
        for (int il = warp; il < ni; il += SWEEP_NT / 32) warp_tdma_smem<S, false>(sl + il * LS, cf, lane);
        __syncthreads();
        double* Qc = Q + comp * g.FS;
        const int n2i = comp == 1 ? 2 : 1;
        for (int p = threadIdx.x; p < 32 * M; p += SWEEP_NT) {
            const int jl = p >> 5, il = p & 31;
            if (il >= ni) continue;
            const double x = sl[il * LS + seg_pos<S>(jl)];
            if (comp == 0 && jl == 0) sdu[il] = x;
            if (jl + 1 >= n2i) {
                const long long c = pidx(g, i0 + il, jl + 1, k);
                Qc[c] = x + Qc[c];
            }
        }
    }
}
