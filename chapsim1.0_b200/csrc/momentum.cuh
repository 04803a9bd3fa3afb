// Momentum part of one RK3 substep of the periodic channel:
// SOLVERRK3_MOM_tg (src/SOLVERRK3_MOM_tg.f90:22-35) =
//   CONVECTION_X/Y/Z_tg + 3 x (RHS_CvLpGpS_tg + MOMFA_tg).
//
// Kernel split (all three velocity components per kernel):
//   k_factors    : per substep, the line-independent factor tables of the
//                  x, z and y sweeps (warp_tdma_factor)
//   k_rhs_xsweep : convection (CONVECTION_X_tg :13-64, CONVECTION_Y_tg
//                  :13-114, CONVECTION_Z_tg :13-103), RK combination,
//                  viscous and pressure-gradient terms (RHS_CvLpGpS_tg
//                  :97-161), CONVH0 update, the grid sum of the bulk-flux
//                  forcing (:163-181), then the cyclic x sweep
//                  (MOMFA1_X_tg, src/MOMFA_tg.f90:51-106); one warp per x line
//   k_zsweep     : cyclic z sweep (MOMFA2_Z_tg :110-169)
//   k_ysweep     : forcing subtraction, non-cyclic y sweep (MOMFA3_Y_tg
//                  :172-238) and Q += dQ (MOMFA_tg :38-44)
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

#define RHS_WPB 4       // x lines (warps) per block
#ifndef RHS_MINB
#define RHS_MINB 4      // resident blocks per SM the register budget is sized for
#endif
#define SWEEP_NT 256
#define FAC_SET (TF_NF(12) * 32)   // doubles per factor table

// factor-table sets
#define FSET_X 0
#define FSET_Z 1
#define FSET_Y 2   // + component

struct YCoef {  // MOMFA3_Y_tg rows: (-F*AMVR, 1 - F*ACVR, -F*APVR), row r = j-1
    const double *am, *ac, *ap;
    double f;
    __device__ __forceinline__ double A(int r) const { return -f * am[r + 1]; }
    __device__ __forceinline__ double B(int r) const { return 1.0 - f * ac[r + 1]; }
    __device__ __forceinline__ double C(int r) const { return -f * ap[r + 1]; }
};

template <bool CYC, class C>
__device__ void factor_dispatch(int S, const C& cf, int lane, double* fac) {
    switch (S) {
        case 1: warp_tdma_factor<1, CYC>(cf, lane, fac); break;
        case 2: warp_tdma_factor<2, CYC>(cf, lane, fac); break;
        case 3: warp_tdma_factor<3, CYC>(cf, lane, fac); break;
        case 4: warp_tdma_factor<4, CYC>(cf, lane, fac); break;
        case 6: warp_tdma_factor<6, CYC>(cf, lane, fac); break;
        case 8: warp_tdma_factor<8, CYC>(cf, lane, fac); break;
        case 12: warp_tdma_factor<12, CYC>(cf, lane, fac); break;
        default: break;
    }
}

__device__ __forceinline__ void factor_set(const Geo& g, double dt, int ns, int set, double* f, int lane) {
    const double facoe = 0.5 * g.talp[ns] * dt * g.cvisc * 1.0 / 1.0;
    if (set == FSET_X) {
        ConstCoef cf;
        cf.a = -facoe * g.dxqi;  // MOMFA1_X_tg :72-78
        cf.c = cf.a;
        cf.b = 1.0 - cf.c - cf.a;
        factor_dispatch<true>(g.L / 32, cf, lane, f);
    } else if (set == FSET_Z) {
        ConstCoef cf;
        cf.a = 1.0 * (-facoe * g.dzqi);  // MOMFA2_Z_tg :133-155
        cf.c = cf.a;
        cf.b = 1.0 - cf.c - cf.a;
        factor_dispatch<true>(g.N / 32, cf, lane, f);
    } else {
        const int comp = set - FSET_Y;
        YCoef cf{g.amvr + comp * (g.M + 2), g.acvr + comp * (g.M + 2), g.apvr + comp * (g.M + 2), facoe};
        factor_dispatch<false>(g.M / 32, cf, lane, f);
    }
}

// Factor tables of one substep (block b computes set b: 0 x sweep, 1 z
// sweep, 2..4 y sweep of u, v, w) for the device-resident DT.
__global__ void __launch_bounds__(32) k_factors(Geo g, double* __restrict__ fac, const DevState* __restrict__ st, int ns) {
    factor_set(g, st->dt, ns, blockIdx.x, fac + (long long)blockIdx.x * FAC_SET, threadIdx.x);
}

// ---------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(RHS_WPB * 32, RHS_MINB) k_rhs_xsweep(Geo g, const double* __restrict__ Q, const double* __restrict__ PR,
                                                             double* __restrict__ H0, double* __restrict__ RHS,
                                                             double* __restrict__ partial, DevState* __restrict__ st,
                                                             const double* __restrict__ fac, int ns) {
    extern __shared__ double sm[];
    __shared__ double sred[32];
    __shared__ int is_last;
    const int L = g.L, M = g.M, N = g.N;
    const int LS = L + 33;  // per-line smem stride (segment padded, odd)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int line = blockIdx.x * RHS_WPB + warp;
    const int j = 1 + line % M, k = line / M;
    const int jp = j + 1, jm = j - 1;
    const double dt = st->dt;
    const double tg = g.tgam[ns], tr = g.troh[ns], ta = g.talp[ns];
    const double coev = ta * g.cvisc;  // COE1 of RHS_CvLpGpS_tg
    const double coep = ta * dt;       // COE2 (pressure gradient)
    const int kp = wrapp(k, N), km = wrapm(k, N);
    const double* U = Q;
    const double* V = Q + g.FS;
    const double* W = Q + 2 * g.FS;
    double* sl = sm + warp * 3 * LS;
    const double c1x = 0.5 * 0.5 * g.dxi;  // XND2CL*XND2CL*DXI
    const double c3x = 0.5 * 0.5 * g.dzi;
    const double wffj = g.wff[j], wfbj = g.wfb[j], wffp = g.wff[jp], wfbp = g.wfb[jp];
    const double dyfij = g.dyfi[j], dycij = g.dyci[j];
    const double dyj = 1.0 / dyfij / 1.0;  // cell height in the bulk-flux integrand
    const double amu = g.amvr[j], acu = g.acvr[j], apu = g.apvr[j];
    const double amv = g.amvr[(M + 2) + j], acv = g.acvr[(M + 2) + j], apv = g.apvr[(M + 2) + j];
    const double amw = g.amvr[2 * (M + 2) + j], acw = g.acvr[2 * (M + 2) + j], apw = g.apvr[2 * (M + 2) + j];
    const long long rowc = pidx(g, 0, j, k), rowjp = pidx(g, 0, jp, k), rowjm = pidx(g, 0, jm, k);
    const long long rowkp = pidx(g, 0, j, kp), rowkm = pidx(g, 0, j, km);
    const long long rowjpkm = pidx(g, 0, jp, km), rowjmkp = pidx(g, 0, jm, kp);
    const long long irow = iidx(g, 0, j, k);
    double bulk = 0.0;
#pragma unroll 1
    for (int kk = 0; kk < S; ++kk) {
        const int i = lane + 32 * kk;
        const int ip = wrapp(i, L), im = wrapm(i, L);
        const double u = U[rowc + i], v = V[rowc + i], w = W[rowc + i];
        const double uip = U[rowc + ip], uim = U[rowc + im];
        const double ujp = U[rowjp + i], ujm = U[rowjm + i], ukp = U[rowkp + i], ukm = U[rowkm + i];
        const double vip = V[rowc + ip], vim = V[rowc + im];
        const double vjp = V[rowjp + i], vjm = V[rowjm + i], vkp = V[rowkp + i], vkm = V[rowkm + i];
        const double wip = W[rowc + ip], wim = W[rowc + im];
        const double wjp = W[rowjp + i], wjm = W[rowjm + i], wkp = W[rowkp + i], wkm = W[rowkm + i];
        const double pc = PR[rowc + i];
        // every load of the iteration is issued before any store: H0 is read
        // and written through one pointer, which the compiler cannot reorder
        const double pim = PR[rowc + im], pjm = PR[rowjm + i], pkm = PR[rowkm + i];
        const double vjpim = V[rowjp + im], wkpim = W[rowkp + im];
        const double ujmip = U[rowjm + ip], wjmkp = W[rowjmkp + i];
        const double ukmip = U[rowkm + ip], vjpkm = V[rowjpkm + i];
        const long long ii = irow + i;
        const double h0u = H0[ii];
        const double h0v = j >= 2 ? H0[ii + g.FI] : 0.0;
        const double h0w = H0[ii + 2 * g.FI];
        const int pos = seg_pos<S>(i);
        double Hu, Hv = 0.0, Hw, ru, rv = 0.0, rw;
        // ---------------- u (CONVECTION_X_tg) ----------------
        {
            const double H11 = ((uip + u) * (uip + u) - (uim + u) * (uim + u)) * c1x;
            const double coe2 = dyfij * 0.5 * 1.0;
            const double H12 = ((vjp + vjpim) * (wffp * ujp + wfbp * u) - (v + vim) * (wffj * u + wfbj * ujm)) * coe2;
            const double coe3 = 0.5 * 0.5 * g.dzi * 1.0;
            const double H13 = ((wkp + wkpim) * (ukp + u) - (w + wim) * (u + ukm)) * coe3;
            Hu = -(H11 + H12 + H13);
            const double rhsc = tg * Hu + tr * h0u;
            const double rhsl = coev * ((uip - 2.0 * u + uim) * g.dxqi + (ukp - 2.0 * u + ukm) * g.dzqi * 1.0 +
                                        (ujp * apu + u * acu + ujm * amu));
            double r = (rhsc + rhsl) * dt;
            ru = r - (pc - pim) * g.dxi * coep;
            bulk += ru * dyj;
        }
        // ---------------- v (CONVECTION_Y_tg), j >= 2 ----------------
        if (j >= 2) {
            const double coe1 = g.dxi * 0.5;
            const double H21 = ((wffj * uip + wfbj * ujmip) * (vip + v) - (wffj * u + wfbj * ujm) * (v + vim)) * coe1;
            const double coe2 = dycij * 0.5 * 0.5;
            const double H22 = ((vjp * 1.0 + v * 1.0) * (vjp + v) - (v * 1.0 + vjm * 1.0) * (v + vjm)) * coe2;
            const double coe31 = g.dzi * 0.5 * 1.0;
            const double H23 = ((wffj * wkp * 1.0 + wfbj * wjmkp * 1.0) * (vkp + v) -
                                (wffj * w * 1.0 + wfbj * wjm * 1.0) * (v + vkm)) * coe31;
            Hv = -(H21 + H22 + H23);
            const double rhsc = tg * Hv + tr * h0v;
            const double rhsl = coev * ((vip - 2.0 * v + vim) * g.dxqi + (vkp - 2.0 * v + vkm) * g.dzqi * 1.0 +
                                        (vjp * apv + v * acv + vjm * amv));
            double r = (rhsc + rhsl) * dt;
            rv = r - (pc - pjm) * (dycij / 1.0) * coep;
        }
        // ---------------- w (CONVECTION_Z_tg) ----------------
        {
            const double H31 = ((uip + ukmip) * (wip + w) - (u + ukm) * (w + wim)) * c1x;
            const double coe2 = dyfij * 0.5;
            const double H32 = ((vjp + vjpkm) * (wffp * wjp * 1.0 + wfbp * w * 1.0) -
                                (v + vkm) * (wffj * w * 1.0 + wfbj * wjm * 1.0)) * coe2;
            const double H33 = ((wkp + w) * (wkp + w) - (w + wkm) * (w + wkm)) * c3x;
            Hw = -(H31 + H32 + H33);
            const double rhsc = tg * Hw + tr * h0w;
            const double rhsl = coev * ((wip - 2.0 * w + wim) * g.dxqi + (wkp - 2.0 * w + wkm) * g.dzqi * 1.0 +
                                        (wjp * apw + w * acw + wjm * amw));
            double r = (rhsc + rhsl) * dt;
            rw = r - (pc - pkm) * g.dzi * coep;
        }
        H0[ii] = Hu;
        if (j >= 2) H0[ii + g.FI] = Hv;
        H0[ii + 2 * g.FI] = Hw;
        sl[pos] = ru;
        if (j >= 2) sl[LS + pos] = rv;
        sl[2 * LS + pos] = rw;
    }
    __syncwarp();
    // cyclic x sweeps of this warp's three lines (MOMFA1_X_tg starts at N2I = 2 for v)
    const double* fx = fac + FSET_X * FAC_SET;
#pragma unroll 1
    for (int c = 0; c < 3; ++c)
        if (c != 1 || j >= 2) warp_tdma_apply_smem<S, true>(sl + c * LS, fx, lane);
    __syncwarp();
#pragma unroll
    for (int kk = 0; kk < S; ++kk) {
        const int i = lane + 32 * kk;
        const long long ii = irow + i;
        const int pos = seg_pos<S>(i);
        RHS[ii] = sl[pos];
        if (j >= 2) RHS[ii + g.FI] = sl[LS + pos];
        RHS[ii + 2 * g.FI] = sl[2 * LS + pos];
    }
    // grid sum of the bulk-flux integrand: block partials, then the last
    // block to finish adds them in index order (deterministic)
    for (int o = 16; o > 0; o >>= 1) bulk += __shfl_down_sync(0xffffffffu, bulk, o);
    if (lane == 0) sred[warp] = bulk;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w2 = 0; w2 < RHS_WPB; ++w2) s += sred[w2];
        partial[blockIdx.x] = s;
        __threadfence();
        const unsigned prev = atomicAdd(&st->ctr, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        double s = 0.0;
        for (int t = threadIdx.x; t < (int)gridDim.x; t += RHS_WPB * 32) s += __ldcg(partial + t);
        s = block_sum<RHS_WPB * 32>(s, sred);
        if (threadIdx.x == 0) {
            st->bulksum = s;
            st->ctr = 0u;
        }
    }
}

// ---------------------------------------------------------------------------
// cyclic z sweep: block = 32 consecutive i at fixed j, all k, one component
template <int S>
__global__ void __launch_bounds__(SWEEP_NT, (S >= 6 ? 2 : 3)) k_zsweep(Geo g, double* __restrict__ RHS, const double* __restrict__ fac) {
    extern __shared__ double sm[];
    const int N = g.N;
    const int i0 = blockIdx.x * 32;
    const int j = 1 + blockIdx.y;
    const int comp = blockIdx.z;
    if (comp == 1 && j == 1) return;  // MOMFA2_Z_tg starts at N2I = 2 for v
    const int LS = N + 33;
    double* R = RHS + comp * g.FI + iidx(g, i0, j, 0);
    const long long ks = g.PI_;
    constexpr int NIT = 4 * S;  // 32*N / SWEEP_NT
#pragma unroll 4
    for (int it = 0; it < NIT; ++it) {
        const int p = threadIdx.x + SWEEP_NT * it;
        cp_async8(sm + (p & 31) * LS + seg_pos<S>(p >> 5), R + (p & 31) + ks * (p >> 5));
    }
    cp_async_wait_all();
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* fz = fac + FSET_Z * FAC_SET;
#pragma unroll 1
    for (int il = warp; il < 32; il += SWEEP_NT / 32) warp_tdma_apply_smem<S, true>(sm + il * LS, fz, lane);
    __syncthreads();
#pragma unroll 4
    for (int it = 0; it < NIT; ++it) {
        const int p = threadIdx.x + SWEEP_NT * it;
        R[(p & 31) + ks * (p >> 5)] = sm[(p & 31) * LS + seg_pos<S>(p >> 5)];
    }
}

// ---------------------------------------------------------------------------
// y sweep + Q update: block = 32 consecutive i at fixed k, all j, u then v then w
template <int S>
__global__ void __launch_bounds__(SWEEP_NT, (S >= 6 ? 2 : 3)) k_ysweep(Geo g, double* __restrict__ Q, const double* __restrict__ RHS,
                                                     const DevState* __restrict__ st, const double* __restrict__ fac,
                                                     int ns) {
    extern __shared__ double sm[];
    __shared__ double sdu[32];  // u increment at j = 1
    const int M = g.M;
    const int i0 = blockIdx.x * 32;
    const int k = blockIdx.y;
    const int LS = M + 33;
    const double dt = st->dt;
    // DPGRNS (RHS_CvLpGpS_tg :163-199)
    double dpg = 0.0;
    if (g.iflowdriven == 1) dpg = st->bulksum / g.volm;
    else if (g.iflowdriven == 2) dpg = -0.5 * g.cf_given * (g.talp[ns] * dt / 1.0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NIT = 4 * S;  // 32*M / SWEEP_NT
    const long long js = g.L;   // stride between y rows (interior and padded fields alike)
#pragma unroll 1
    for (int comp = 0; comp < 3; ++comp) {
        const double* R = RHS + comp * g.FI + iidx(g, i0, 1, k);
#pragma unroll 4
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            cp_async8(sm + (p & 31) * LS + seg_pos<S>(p >> 5), R + (p & 31) + js * (p >> 5));
        }
        cp_async_wait_all();
        __syncthreads();
        const double* fy = fac + (FSET_Y + comp) * FAC_SET;
#pragma unroll 1
        for (int il = warp; il < 32; il += SWEEP_NT / 32) {
            double* base = sm + il * LS;
            double d[S];
#pragma unroll
            for (int q = 0; q < S; ++q) d[q] = base[lane * (S + 1) + q];
            if (comp == 0) {
#pragma unroll
                for (int q = 0; q < S; ++q) d[q] = d[q] - dpg;
            } else if (comp == 1 && lane == 0) {
                d[0] = g.fix_v_wall_row ? 0.0 : sdu[il];  // row 1 of v: see the quirk note above
            }
            warp_tdma_apply<S, false>(d, fy, lane);
#pragma unroll
            for (int q = 0; q < S; ++q) base[lane * (S + 1) + q] = d[q];
        }
        __syncthreads();
        double* Qc = Q + comp * g.FS + pidx(g, i0, 1, k);
        const int n2i = comp == 1 ? 2 : 1;
        double qv[NIT];
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            qv[it] = Qc[(p & 31) + js * (p >> 5)];
        }
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            const int jl = p >> 5, il = p & 31;
            const double x = sm[il * LS + seg_pos<S>(jl)];
            if (comp == 0 && jl == 0) sdu[il] = x;
            if (jl + 1 >= n2i) Qc[il + js * jl] = x + qv[it];
        }
        __syncthreads();
    }
}
