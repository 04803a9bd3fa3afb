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
//
// Precision: the kernels are templated on the real type R of the stored
// fields (Q, PR, CONVH0, RHS) and of their arithmetic.  R = double is the
// plain FP64 step.  R = float is the mixed-precision step: stencils and
// Crank-Nicolson sweeps in FP32 with factor tables computed in FP64 and
// stored in FP32, while the bulk-flux sum is accumulated in FP64 (per-thread
// partials, then a fixed-order block and grid tree).
#pragma once
#include "common.cuh"
#include "tdma.cuh"

#define RHS_WPB 4       // x lines (warps) per block
// Resident blocks per SM the register budget of k_rhs_xsweep is sized for:
// FP64 at 3 (about 168 registers, no spills) ran 5 % faster at 128^3 and 19 %
// at 384 x 256 x 384 than at 4 (128 registers with spills); FP32 is fastest
// at 4.
#define RHS_MINB(R) (sizeof(R) == 8 ? 3 : 4)
// The vector forms (PV adjacent points per lane) with 16-byte vectors hold two or four times the
// loaded values of the one-point form: a two-block budget in FP64 (234 registers), three in FP32
// (168, no spills).
#define RHS_MINB_P(R, PV) ((PV) * sizeof(R) > 8 ? (sizeof(R) == 4 ? 3 : 2) : RHS_MINB(R))
// points per lane of the fused right-hand side: the default form (1 in FP64, 2 in FP32) and
// the wide form, autotuned kind 3 (2 in FP64, 4 in FP32: 16-byte loads)
template <typename R> __host__ __device__ constexpr int rhs_pv(bool wide) {
    return sizeof(R) == 8 ? (wide ? 2 : 1) : (wide ? 4 : 2);
}
// PV consecutive elements through one vector access (PV * sizeof(R) = 8 or 16 bytes, aligned)
template <int PV, typename R>
__device__ __forceinline__ void ldvec(const R* p, R (&o)[PV]) {
    if constexpr (PV * sizeof(R) == 16) {
        if constexpr (sizeof(R) == 4) {
            const float4 v = *reinterpret_cast<const float4*>(p);
            o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
        } else {
            const double2 v = *reinterpret_cast<const double2*>(p);
            o[0] = v.x; o[1] = v.y;
        }
    } else {
        static_assert(PV * sizeof(R) == 8, "8- or 16-byte vectors");
        const float2 v = *reinterpret_cast<const float2*>(p);
        o[0] = v.x; o[1] = v.y;
    }
}
template <int PV, typename R>
__device__ __forceinline__ void stvec(R* p, const R (&a)[PV]) {
    if constexpr (PV * sizeof(R) == 16) {
        if constexpr (sizeof(R) == 4) *reinterpret_cast<float4*>(p) = make_float4(a[0], a[1], a[2], a[3]);
        else *reinterpret_cast<double2*>(p) = make_double2(a[0], a[1]);
    } else {
        *reinterpret_cast<float2*>(p) = make_float2(a[0], a[1]);
    }
}
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

template <bool CYC, class C, typename T>
__device__ void factor_dispatch(int S, const C& cf, int lane, T* fac) {
    switch (S) {
        case 1: warp_tdma_factor<1, CYC, C, T>(cf, lane, fac); break;
        case 2: warp_tdma_factor<2, CYC, C, T>(cf, lane, fac); break;
        case 3: warp_tdma_factor<3, CYC, C, T>(cf, lane, fac); break;
        case 4: warp_tdma_factor<4, CYC, C, T>(cf, lane, fac); break;
        case 6: warp_tdma_factor<6, CYC, C, T>(cf, lane, fac); break;
        case 8: warp_tdma_factor<8, CYC, C, T>(cf, lane, fac); break;
        case 12: warp_tdma_factor<12, CYC, C, T>(cf, lane, fac); break;
        default: break;
    }
}

template <typename T>
__device__ __forceinline__ void factor_set(const Geo& g, double dt, int ns, int set, T* f, int lane) {
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
template <typename T>
__global__ void __launch_bounds__(32) k_factors(Geo g, T* __restrict__ fac, const DevState* __restrict__ st, int ns) {
    pdl_wait();
    factor_set(g, st->dt, ns, blockIdx.x, fac + (long long)blockIdx.x * FAC_SET, threadIdx.x);
}

// ---------------------------------------------------------------------------
// The per-point arithmetic of the explicit right-hand sides, shared by the
// fused, split and bulk-staged kernels: convection (CONVECTION_X_tg :13-64,
// CONVECTION_Y_tg :13-114, CONVECTION_Z_tg :13-103), the RK combination with
// CONVH0, the viscous and pressure-gradient terms (RHS_CvLpGpS_tg :97-161),
// and the point's bulk-flux integrand.  RhsStencil holds the values a point
// reads: the three components at the point and its x, y and z neighbours,
// the cross terms, PR at the point and its -x, -y and -z neighbours, and the
// three CONVH0 values; RhsLine the coefficients of its (j, substep).
template <typename R>
struct RhsStencil {
    R u, uip, uim, ujp, ujm, ukp, ukm;
    R v, vip, vim, vjp, vjm, vkp, vkm;
    R w, wip, wim, wjp, wjm, wkp, wkm;
    R pc, pim, pjm, pkm;
    R vjpim, wkpim, ujmip, wjmkp, ukmip, vjpkm;
    R h0u, h0v, h0w;
};
template <typename R>
struct RhsLine {
    R dt, tg, tr, coev, coep, dxi, dzi, dxqi, dzqi, c1x, c3x;
    R wffj, wfbj, wffp, wfbp, dyfij, dycij;
    R amu, acu, apu, amv, acv, apv, amw, acw, apw;
    double dyj;
};
// v has no increment on row j = 1 (RHS_CvLpGpS_tg starts v at N2I = 2): vrow = j >= 2
template <typename R>
__device__ __forceinline__ void rhs_point(const RhsLine<R>& c, const RhsStencil<R>& s, bool vrow, R& Hu, R& Hv, R& Hw,
                                          R& ru, R& rv, R& rw, double& bulk) {
    const R u = s.u, uip = s.uip, uim = s.uim, ujp = s.ujp, ujm = s.ujm, ukp = s.ukp, ukm = s.ukm;
    const R v = s.v, vip = s.vip, vim = s.vim, vjp = s.vjp, vjm = s.vjm, vkp = s.vkp, vkm = s.vkm;
    const R w = s.w, wip = s.wip, wim = s.wim, wjp = s.wjp, wjm = s.wjm, wkp = s.wkp, wkm = s.wkm;
    const R pc = s.pc;
    // ---------------- u (CONVECTION_X_tg) ----------------
    {
        const R H11 = ((uip + u) * (uip + u) - (uim + u) * (uim + u)) * c.c1x;
        const R coe2 = c.dyfij * R(0.5);
        const R H12 = ((vjp + s.vjpim) * (c.wffp * ujp + c.wfbp * u) - (v + vim) * (c.wffj * u + c.wfbj * ujm)) * coe2;
        const R coe3 = c.c3x;
        const R H13 = ((wkp + s.wkpim) * (ukp + u) - (w + wim) * (u + ukm)) * coe3;
        Hu = -(H11 + H12 + H13);
        const R rhsc = c.tg * Hu + c.tr * s.h0u;
        const R rhsl = c.coev * ((uip - R(2) * u + uim) * c.dxqi + (ukp - R(2) * u + ukm) * c.dzqi +
                                 (ujp * c.apu + u * c.acu + ujm * c.amu));
        R r = (rhsc + rhsl) * c.dt;
        ru = r - (pc - s.pim) * c.dxi * c.coep;
        bulk += (double)ru * c.dyj;
    }
    // ---------------- v (CONVECTION_Y_tg), j >= 2 ----------------
    Hv = R(0);
    rv = R(0);
    if (vrow) {
        const R coe1 = c.dxi * R(0.5);
        const R H21 = ((c.wffj * uip + c.wfbj * s.ujmip) * (vip + v) - (c.wffj * u + c.wfbj * ujm) * (v + vim)) * coe1;
        const R coe2 = c.dycij * R(0.5) * R(0.5);
        const R H22 = ((vjp + v) * (vjp + v) - (v + vjm) * (v + vjm)) * coe2;
        const R coe31 = c.dzi * R(0.5);
        const R H23 = ((c.wffj * wkp + c.wfbj * s.wjmkp) * (vkp + v) - (c.wffj * w + c.wfbj * wjm) * (v + vkm)) * coe31;
        Hv = -(H21 + H22 + H23);
        const R rhsc = c.tg * Hv + c.tr * s.h0v;
        const R rhsl = c.coev * ((vip - R(2) * v + vim) * c.dxqi + (vkp - R(2) * v + vkm) * c.dzqi +
                                 (vjp * c.apv + v * c.acv + vjm * c.amv));
        R r = (rhsc + rhsl) * c.dt;
        rv = r - (pc - s.pjm) * c.dycij * c.coep;
    }
    // ---------------- w (CONVECTION_Z_tg) ----------------
    {
        const R H31 = ((uip + s.ukmip) * (wip + w) - (u + ukm) * (w + wim)) * c.c1x;
        const R coe2 = c.dyfij * R(0.5);
        const R H32 = ((vjp + s.vjpkm) * (c.wffp * wjp + c.wfbp * w) - (v + vkm) * (c.wffj * w + c.wfbj * wjm)) * coe2;
        const R H33 = ((wkp + w) * (wkp + w) - (w + wkm) * (w + wkm)) * c.c3x;
        Hw = -(H31 + H32 + H33);
        const R rhsc = c.tg * Hw + c.tr * s.h0w;
        const R rhsl = c.coev * ((wip - R(2) * w + wim) * c.dxqi + (wkp - R(2) * w + wkm) * c.dzqi +
                                 (wjp * c.apw + w * c.acw + wjm * c.amw));
        R r = (rhsc + rhsl) * c.dt;
        rw = r - (pc - s.pkm) * c.dzi * c.coep;
    }
}

// The line coefficients of (j, substep ns) in the real type R.
template <typename R>
__device__ __forceinline__ RhsLine<R> rhs_line(const Geo& g, double dt, int ns, double wffj, double wfbj, double wffp,
                                               double wfbp, double dyfi, double dyci, const double* am, const double* ac,
                                               const double* ap) {
    RhsLine<R> c;
    c.dt = (R)dt;
    c.tg = (R)g.tgam[ns];
    c.tr = (R)g.troh[ns];
    const R ta = (R)g.talp[ns];
    c.coev = ta * (R)g.cvisc;  // COE1 of RHS_CvLpGpS_tg
    c.coep = ta * c.dt;        // COE2 (pressure gradient)
    c.dxi = (R)g.dxi; c.dzi = (R)g.dzi; c.dxqi = (R)g.dxqi; c.dzqi = (R)g.dzqi;
    c.c1x = (R)(0.5 * 0.5 * g.dxi);  // XND2CL*XND2CL*DXI
    c.c3x = (R)(0.5 * 0.5 * g.dzi);
    c.wffj = (R)wffj; c.wfbj = (R)wfbj; c.wffp = (R)wffp; c.wfbp = (R)wfbp;
    c.dyfij = (R)dyfi; c.dycij = (R)dyci;
    c.amu = (R)am[0]; c.acu = (R)ac[0]; c.apu = (R)ap[0];
    c.amv = (R)am[1]; c.acv = (R)ac[1]; c.apv = (R)ap[1];
    c.amw = (R)am[2]; c.acw = (R)ac[2]; c.apw = (R)ap[2];
    c.dyj = 1.0 / dyfi / 1.0;  // cell height in the bulk-flux integrand
    return c;
}
template <typename R>
__device__ __forceinline__ RhsLine<R> rhs_line(const Geo& g, double dt, int ns, int j) {
    const int M2 = g.M + 2;
    const double am[3] = {g.amvr[j], g.amvr[M2 + j], g.amvr[2 * M2 + j]};
    const double ac[3] = {g.acvr[j], g.acvr[M2 + j], g.acvr[2 * M2 + j]};
    const double ap[3] = {g.apvr[j], g.apvr[M2 + j], g.apvr[2 * M2 + j]};
    return rhs_line<R>(g, dt, ns, g.wff[j], g.wfb[j], g.wff[j + 1], g.wfb[j + 1], g.dyfi[j], g.dyci[j], am, ac, ap);
}

// ---------------------------------------------------------------------------
template <int S, typename R, int PV>
__global__ void __launch_bounds__(RHS_WPB * 32, RHS_MINB_P(R, PV)) k_rhs_xsweep(Geo g, const R* __restrict__ Q, const R* __restrict__ PR,
                                                             R* __restrict__ H0, R* __restrict__ RHS,
                                                             double* __restrict__ partial, DevState* __restrict__ st,
                                                             const R* __restrict__ fac, int ns) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* sm = reinterpret_cast<R*>(sm_raw);
    __shared__ double sred[32];
    __shared__ int is_last;
    const int L = g.L, M = g.M, N = g.N;
    const int LS = L + 33;  // per-line smem stride (segment padded, odd)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int line = blockIdx.x * RHS_WPB + warp;
    const int j = 1 + line % M, k = line / M;
    const int jp = j + 1, jm = j - 1;
    const RhsLine<R> cl = rhs_line<R>(g, st->dt, ns, j);
    const int kp = wrapp(k, N), km = wrapm(k, N);
    const R* U = Q;
    const R* V = Q + g.FS;
    const R* W = Q + 2 * g.FS;
    R* sl = sm + warp * 3 * LS;
    const long long rowc = pidx(g, 0, j, k), rowjp = pidx(g, 0, jp, k), rowjm = pidx(g, 0, jm, k);
    const long long rowkp = pidx(g, 0, j, kp), rowkm = pidx(g, 0, j, km);
    const long long rowjpkm = pidx(g, 0, jp, km), rowjmkp = pidx(g, 0, jm, kp);
    const long long irow = iidx(g, 0, j, k);
    const bool vrow = j >= 2;
    // The line's own rows (Q, PR, CONVH0 at (j, k)) are what this kernel reads
    // from DRAM; the neighbour rows are other lines' own rows, fetched by their
    // warps at about the same time.  Requesting the later segments up front
    // keeps DRAM busy while the first segment is computed.
#pragma unroll
    for (int kk = 1; kk < S; ++kk) {
        const int i = lane + 32 * kk;
        prefetch_l2(U + rowc + i);
        prefetch_l2(V + rowc + i);
        prefetch_l2(W + rowc + i);
        prefetch_l2(PR + rowc + i);
        prefetch_l2(H0 + irow + i);
        prefetch_l2(H0 + irow + i + g.FI);
        prefetch_l2(H0 + irow + i + 2 * g.FI);
    }
    double bulk = 0.0;
    if constexpr (PV > 1 && S % PV == 0) {
        // Vector form (PV = 2 in FP32 always; PV = 2 in FP64 and 4 in FP32 as the autotuned
        // wide form): each lane takes PV adjacent points (i .. i+PV-1, one segment of the
        // x sweep's layout) per iteration with PV-element vector loads, so a warp request moves
        // PV times the bytes of the one-point form; the x neighbours outside the group are
        // single loads.  Rows start at multiples of L (a multiple of 32), so every group is
        // aligned to its vector size.
#pragma unroll 1
        for (int kk = 0; kk < S / PV; ++kk) {
            const int i = PV * lane + 32 * PV * kk;
            const int il = i == 0 ? L - 1 : i - 1, ir = i + PV == L ? 0 : i + PV;
            auto ldv = [&](const R* b, long long row, R (&o)[PV]) { ldvec<PV>(b + row + i, o); };
            R uc[PV], vc[PV], wc[PV], ujp[PV], ujm[PV], ukp[PV], ukm[PV], vjp[PV], vjm[PV], vkp[PV], vkm[PV];
            R wjp[PV], wjm[PV], wkp[PV], wkm[PV], pc[PV], pjm[PV], pkm[PV], wjmkp[PV], vjpkm[PV];
            ldv(U, rowc, uc); ldv(V, rowc, vc); ldv(W, rowc, wc);
            ldv(U, rowjp, ujp); ldv(U, rowjm, ujm); ldv(U, rowkp, ukp); ldv(U, rowkm, ukm);
            ldv(V, rowjp, vjp); ldv(V, rowjm, vjm); ldv(V, rowkp, vkp); ldv(V, rowkm, vkm);
            ldv(W, rowjp, wjp); ldv(W, rowjm, wjm); ldv(W, rowkp, wkp); ldv(W, rowkm, wkm);
            ldv(PR, rowc, pc); ldv(PR, rowjm, pjm); ldv(PR, rowkm, pkm);
            ldv(W, rowjmkp, wjmkp); ldv(V, rowjpkm, vjpkm);
            const R ul = U[rowc + il], ur = U[rowc + ir], vl = V[rowc + il], vr = V[rowc + ir];
            const R wl = W[rowc + il], wr = W[rowc + ir], pl = PR[rowc + il];
            const R vjpl = V[rowjp + il], wkpl = W[rowkp + il], ujmr = U[rowjm + ir], ukmr = U[rowkm + ir];
            // every load of the iteration is issued before any store: H0 is read
            // and written through one pointer, which the compiler cannot reorder
            const long long ii = irow + i;
            R h0u[PV], h0v[PV], h0w[PV];
            ldvec<PV>(H0 + ii, h0u);
            if (vrow) ldvec<PV>(H0 + ii + g.FI, h0v);
            else
#pragma unroll
                for (int e = 0; e < PV; ++e) h0v[e] = R(0);
            ldvec<PV>(H0 + ii + 2 * g.FI, h0w);
            R Hu[PV], Hv[PV], Hw[PV], ru[PV], rv[PV], rw[PV];
#pragma unroll
            for (int e = 0; e < PV; ++e) {
                const bool lo = e == 0, hi = e == PV - 1;
                const RhsStencil<R> sp{uc[e], hi ? ur : uc[hi ? e : e + 1], lo ? ul : uc[lo ? e : e - 1],
                                       ujp[e], ujm[e], ukp[e], ukm[e],
                                       vc[e], hi ? vr : vc[hi ? e : e + 1], lo ? vl : vc[lo ? e : e - 1],
                                       vjp[e], vjm[e], vkp[e], vkm[e],
                                       wc[e], hi ? wr : wc[hi ? e : e + 1], lo ? wl : wc[lo ? e : e - 1],
                                       wjp[e], wjm[e], wkp[e], wkm[e],
                                       pc[e], lo ? pl : pc[lo ? e : e - 1], pjm[e], pkm[e],
                                       lo ? vjpl : vjp[lo ? e : e - 1], lo ? wkpl : wkp[lo ? e : e - 1],
                                       hi ? ujmr : ujm[hi ? e : e + 1], wjmkp[e], hi ? ukmr : ukm[hi ? e : e + 1],
                                       vjpkm[e], h0u[e], h0v[e], h0w[e]};
                rhs_point(cl, sp, vrow, Hu[e], Hv[e], Hw[e], ru[e], rv[e], rw[e], bulk);
            }
            stvec<PV>(H0 + ii, Hu);
            if (vrow) stvec<PV>(H0 + ii + g.FI, Hv);
            stvec<PV>(H0 + ii + 2 * g.FI, Hw);
            const int pos = seg_pos<S>(i);  // the group's points are consecutive positions of one segment
#pragma unroll
            for (int e = 0; e < PV; ++e) {
                sl[pos + e] = ru[e];
                if (vrow) sl[LS + pos + e] = rv[e];
                sl[2 * LS + pos + e] = rw[e];
            }
        }
    } else {
#pragma unroll 1
        for (int kk = 0; kk < S; ++kk) {
            const int i = lane + 32 * kk;
            const int ip = wrapp(i, L), im = wrapm(i, L);
            RhsStencil<R> sp;
            sp.u = U[rowc + i]; sp.v = V[rowc + i]; sp.w = W[rowc + i];
            sp.uip = U[rowc + ip]; sp.uim = U[rowc + im];
            sp.ujp = U[rowjp + i]; sp.ujm = U[rowjm + i]; sp.ukp = U[rowkp + i]; sp.ukm = U[rowkm + i];
            sp.vip = V[rowc + ip]; sp.vim = V[rowc + im];
            sp.vjp = V[rowjp + i]; sp.vjm = V[rowjm + i]; sp.vkp = V[rowkp + i]; sp.vkm = V[rowkm + i];
            sp.wip = W[rowc + ip]; sp.wim = W[rowc + im];
            sp.wjp = W[rowjp + i]; sp.wjm = W[rowjm + i]; sp.wkp = W[rowkp + i]; sp.wkm = W[rowkm + i];
            sp.pc = PR[rowc + i];
            // every load of the iteration is issued before any store: H0 is read
            // and written through one pointer, which the compiler cannot reorder
            sp.pim = PR[rowc + im]; sp.pjm = PR[rowjm + i]; sp.pkm = PR[rowkm + i];
            sp.vjpim = V[rowjp + im]; sp.wkpim = W[rowkp + im];
            sp.ujmip = U[rowjm + ip]; sp.wjmkp = W[rowjmkp + i];
            sp.ukmip = U[rowkm + ip]; sp.vjpkm = V[rowjpkm + i];
            const long long ii = irow + i;
            sp.h0u = H0[ii];
            sp.h0v = vrow ? H0[ii + g.FI] : R(0);
            sp.h0w = H0[ii + 2 * g.FI];
            const int pos = seg_pos<S>(i);
            R Hu, Hv, Hw, ru, rv, rw;
            rhs_point(cl, sp, vrow, Hu, Hv, Hw, ru, rv, rw, bulk);
            H0[ii] = Hu;
            if (vrow) H0[ii + g.FI] = Hv;
            H0[ii + 2 * g.FI] = Hw;
            sl[pos] = ru;
            if (vrow) sl[LS + pos] = rv;
            sl[2 * LS + pos] = rw;
        }
    }
    __syncwarp();
    // cyclic x sweeps of this warp's three lines (MOMFA1_X_tg starts at N2I = 2 for v)
    const R* fx = fac + FSET_X * FAC_SET;
    warp_tdma_apply_smem3<S, true>(sl, LS, j >= 2, fx, lane);  // the three components together
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

// Resident blocks per SM of the persistent z sweep: 3 for FP32 lines up to
// 128 (80 registers; the two tile buffers take 41 KB), else 2 (128
// registers; longer FP32 lines would spill under the tighter budget, and
// their buffers leave room for two blocks only).
template <typename R, int S> __host__ __device__ constexpr int zsweep_blocks() { return sizeof(R) == 4 && S <= 4 ? 3 : 2; }
// Lines (consecutive i) per tile, TW: 32 or 16 (autotuned, chapsim_autotune bit 8).  16 halves the
// two tile buffers (2 x 32 x (N + 33) doubles are 213 KB at N = 384: one block per SM) and each z
// position of a tile still reads whole 32-byte sectors (64 or 128 bytes per row segment).

// ---------------------------------------------------------------------------
// cyclic z sweep.  A tile is TW (32 or 16) consecutive i at fixed j, all
// k, one component; tiles of v at j = 1 are skipped (MOMFA2_Z_tg
// starts at N2I = 2 for v).  Blocks are persistent and take tiles in a stride loop with two
// shared-memory buffers: the next tile's right-hand sides load (cp.async)
// while the current tile's 32 lines are solved and stored.
// Shared-memory layout of a tile: IL = 1 keeps each line contiguous (segment
// padded, LS = N + 33 elements per line); IL = 2 interleaves the lines in
// pairs, element z of line il at (il / 2) * 2 LS + 2 seg_pos(z) + il % 2, so
// that one cp.async of two consecutive x points (8 bytes in FP32, 16 in FP64)
// fills both lines of a pair: half the copy instructions, for 2-way bank
// conflicts in the solve's segment reads (the lane stride is 2 (S + 1)).
template <int IL> __device__ __forceinline__ int zs_line(int il, int LS) { return IL == 1 ? il * LS : (il >> 1) * 2 * LS + (il & 1); }

template <int S, typename R, int TW, int IL>
__global__ void __launch_bounds__(SWEEP_NT, (zsweep_blocks<R, S>())) k_zsweep(Geo g, R* __restrict__ RHS, const R* __restrict__ fac) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* smb = reinterpret_cast<R*>(sm_raw);
    static_assert(TW == 16 || TW == 32, "tile width");
    static_assert(IL == 1 || IL == 2, "line interleave");
    const int N = g.N, M = g.M;
    const int LS = N + 33;
    const int TS = TW * LS;
    const int nx = g.L / TW;
    const int nwork = nx * (3 * M - 1);
    const long long ks = g.PI_;
    constexpr int NIT = TW * S / 8 / IL;  // TW*N / (SWEEP_NT*IL) copies per thread
    constexpr int TP = TW / IL;           // copies per z row of a tile
    auto tile_base = [&](int t) -> R* {
        int comp, j;
        if (t < nx * M) { comp = 0; j = 1 + t / nx; }
        else if (t < nx * (2 * M - 1)) { comp = 1; j = 2 + (t - nx * M) / nx; }
        else { comp = 2; j = 1 + (t - nx * (2 * M - 1)) / nx; }
        const int i0 = TW * (t % nx);
        return RHS + comp * g.FI + iidx(g, i0, j, 0);
    };
    auto load = [&](int t, R* buf) {
        const R* Rz = tile_base(t);
#pragma unroll 4
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            const int c = p % TP, z = p / TP;
            if constexpr (IL == 1) {
                cp_async_el(buf + c * LS + seg_pos<S>(z), Rz + c + ks * z);
            } else {
                R* dst = buf + c * 2 * LS + 2 * seg_pos<S>(z);
                const R* src = Rz + 2 * c + ks * z;
                if constexpr (sizeof(R) == 8) cp_async16(dst, src);
                else cp_async8(reinterpret_cast<double*>(dst), reinterpret_cast<const double*>(src));
            }
        }
    };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const R* fz = fac + FSET_Z * FAC_SET;
    int t = blockIdx.x, b = 0;
    if (t < nwork) load(t, smb);
    cp_async_commit();
    for (; t < nwork; t += gridDim.x) {
        R* cur = smb + b * TS;
        const int tn = t + gridDim.x;
        if (tn < nwork) load(tn, smb + (b ^ 1) * TS);
        cp_async_commit();
        cp_async_wait_group<1>();
        __syncthreads();
        // lines up to 128: two per pass (il, il + 8), their chains interleaved and the factor
        // loads shared (longer lines would spill)
        constexpr int NRZ = S <= 4 ? 2 : 1;
#pragma unroll 1
        for (int il = warp; il < TW; il += NRZ * (SWEEP_NT / 32)) {
            R d[NRZ][S];
#pragma unroll
            for (int r = 0; r < NRZ; ++r)
#pragma unroll
                for (int q = 0; q < S; ++q)
                    d[r][q] = cur[zs_line<IL>(il + r * (SWEEP_NT / 32), LS) + IL * (lane * (S + 1) + q)];
            warp_tdma_apply_n<S, true, NRZ>(d, fz, lane);
#pragma unroll
            for (int r = 0; r < NRZ; ++r)
#pragma unroll
                for (int q = 0; q < S; ++q)
                    cur[zs_line<IL>(il + r * (SWEEP_NT / 32), LS) + IL * (lane * (S + 1) + q)] = d[r][q];
        }
        __syncthreads();
        R* Rz = tile_base(t);
#pragma unroll 4
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            const int c = p % TP, z = p / TP;
            if constexpr (IL == 1) {
                Rz[c + ks * z] = cur[c * LS + seg_pos<S>(z)];
            } else {
                const R* src = cur + c * 2 * LS + 2 * seg_pos<S>(z);
                R v[2] = {src[0], src[1]};
                stvec<2>(Rz + 2 * c + ks * z, v);
            }
        }
        __syncthreads();  // cur is the load target two tiles on
        b ^= 1;
    }
    cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// y sweep + Q update: block = 32 consecutive i at fixed k, all j; blocks of
// the grid's first z layer take u then v (v's row 1 reads the u increment of
// the same tile), those of the second layer w.  Splitting w off balances the
// waves: at 128^3 the 512 three-component blocks filled 444 resident slots
// and left a second wave of 68, where the two-plus-one split packs the same
// work into about four component times instead of six.
// IL: the tile layout of k_zsweep (1 lines contiguous, 2 interleaved in pairs: one copy and one
// vector access of Q per two x points).
template <int S, typename R, int IL>
__global__ void __launch_bounds__(SWEEP_NT, (S >= 6 ? 2 : (sizeof(R) == 4 ? 4 : 3))) k_ysweep(Geo g, R* __restrict__ Q, const R* __restrict__ RHS,
                                                     const DevState* __restrict__ st, const R* __restrict__ fac,
                                                     int ns) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* sm = reinterpret_cast<R*>(sm_raw);
    __shared__ R sdu[32];  // u increment at j = 1
    const int M = g.M;
    const int i0 = blockIdx.x * 32;
    const int k = blockIdx.y;
    const int LS = M + 33;
    const double dt = st->dt;
    // DPGRNS (RHS_CvLpGpS_tg :163-199)
    double dpg64 = 0.0;
    if (g.iflowdriven == 1) dpg64 = st->bulksum / g.volm;
    else if (g.iflowdriven == 2) dpg64 = -0.5 * g.cf_given * (g.talp[ns] * dt / 1.0);
    const R dpg = (R)dpg64;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NIT = 4 * S / IL;  // 32*M / (SWEEP_NT*IL) copies per thread
    constexpr int TP = 32 / IL;      // copies per y row of the tile
    const long long js = g.L;        // stride between y rows (interior and padded fields alike)
    const int comp_lo = blockIdx.z == 0 ? 0 : 2, comp_hi = blockIdx.z == 0 ? 2 : 3;
#pragma unroll 1
    for (int comp = comp_lo; comp < comp_hi; ++comp) {
        const R* Ry = RHS + comp * g.FI + iidx(g, i0, 1, k);
#pragma unroll 4
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            const int c = p % TP, jl = p / TP;
            if constexpr (IL == 1) {
                cp_async_el(sm + c * LS + seg_pos<S>(jl), Ry + c + js * jl);
            } else {
                R* dst = sm + c * 2 * LS + 2 * seg_pos<S>(jl);
                const R* src = Ry + 2 * c + js * jl;
                if constexpr (sizeof(R) == 8) cp_async16(dst, src);
                else cp_async8(reinterpret_cast<double*>(dst), reinterpret_cast<const double*>(src));
            }
        }
        cp_async_wait_all();
        __syncthreads();
        const R* fy = fac + (FSET_Y + comp) * FAC_SET;
#pragma unroll 1
        for (int il = warp; il < 32; il += SWEEP_NT / 32) {
            R* base = sm + zs_line<IL>(il, LS);
            R d[S];
#pragma unroll
            for (int q = 0; q < S; ++q) d[q] = base[IL * (lane * (S + 1) + q)];
            if (comp == 0) {
#pragma unroll
                for (int q = 0; q < S; ++q) d[q] = d[q] - dpg;
            } else if (comp == 1 && lane == 0) {
                d[0] = g.fix_v_wall_row ? R(0) : sdu[il];  // row 1 of v: see the quirk note above
            }
            warp_tdma_apply<S, false>(d, fy, lane);
#pragma unroll
            for (int q = 0; q < S; ++q) base[IL * (lane * (S + 1) + q)] = d[q];
        }
        __syncthreads();
        R* Qc = Q + comp * g.FS + pidx(g, i0, 1, k);
        const int n2i = comp == 1 ? 2 : 1;
        R qv[NIT][IL];
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            const int c = p % TP, jl = p / TP;
            if constexpr (IL == 1) qv[it][0] = Qc[c + js * jl];
            else ldvec<2>(Qc + 2 * c + js * jl, qv[it]);
        }
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const int p = threadIdx.x + SWEEP_NT * it;
            const int c = p % TP, jl = p / TP;
            if constexpr (IL == 1) {
                const R x = sm[c * LS + seg_pos<S>(jl)];
                if (comp == 0 && jl == 0) sdu[c] = x;
                if (jl + 1 >= n2i) Qc[c + js * jl] = x + qv[it][0];
            } else {
                const R* sx = sm + c * 2 * LS + 2 * seg_pos<S>(jl);
                const R x0 = sx[0], x1 = sx[1];
                if (comp == 0 && jl == 0) {
                    sdu[2 * c] = x0;
                    sdu[2 * c + 1] = x1;
                }
                if (jl + 1 >= n2i) {
                    const R o[2] = {x0 + qv[it][0], x1 + qv[it][1]};
                    stvec<2>(Qc + 2 * c + js * jl, o);
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Split form of k_rhs_xsweep: k_rhs_point computes the same right-hand sides
// point by point (one thread per point, i fastest, every load independent and
// no line-solve phase, so more warps keep loads in flight) and k_xsweep runs
// the cyclic x sweeps line by line.  It moves 6 more words per point (RHS read
// and written once more); the autotuner picks it where it is faster.
constexpr int RP_NT = 256;
constexpr int RT_I = 32, RT_J = 8;                  // tile of one block: 32 (i) x 8 (j) points per plane
constexpr int RT_HI = RT_I + 2, RT_HJ = RT_J + 2;   // with its one-point halo
constexpr int RT_PLANE = RT_HI * RT_HJ;             // values of one field in one plane
constexpr int RT_SLOT = 4 * RT_PLANE + 3 * RT_I * RT_J;  // U, V, W, PR with halo, then CONVH0 x3 (tile only)
constexpr int RT_AHEAD = 3;                         // planes in flight ahead of plane k+1
constexpr int RT_SLOTS = RT_AHEAD + 2;              // planes k-1, k, k+1 in use, k+2 .. k+RT_AHEAD+1 arriving

// 2.5D form: the block keeps planes k-1, k, k+1 of U, V, W and PR (tile +
// halo) in a shared-memory ring and marches over a chunk of k; the next
// RT_AHEAD planes are in flight (cp.async, one commit group per plane, empty
// groups past the chunk end) while plane k is computed.  Every neighbour access
// is a shared-memory hit and each Q / PR value is read from HBM about once
// per block (plus the halo and the two extra planes of a chunk).
template <typename R>
__device__ __forceinline__ void rt_load_plane(const Geo& g, const R* __restrict__ Q, const R* __restrict__ PR,
                                              const R* __restrict__ H0, R* slot, int i0, int j0, int k) {
    for (int p = threadIdx.x; p < 4 * RT_PLANE; p += RP_NT) {
        const int f = p / RT_PLANE, e = p - f * RT_PLANE;
        const int jj = e / RT_HI, ii = e - jj * RT_HI;
        int i = i0 - 1 + ii;
        i = i < 0 ? i + g.L : (i >= g.L ? i - g.L : i);
        const R* src = f == 3 ? PR : Q + (long long)f * g.FS;
        cp_async_el(slot + p, src + pidx(g, i, j0 - 1 + jj, k));
    }
    // CONVH0 of the tile (row j = 1 of the v component is never read)
    for (int p = threadIdx.x; p < 3 * RT_I * RT_J; p += RP_NT) {
        const int c = p / (RT_I * RT_J), e = p - c * (RT_I * RT_J);
        const int tj = e / RT_I, ti = e - tj * RT_I;
        cp_async_el(slot + 4 * RT_PLANE + p, H0 + c * g.FI + iidx(g, i0 + ti, j0 + tj, k));
    }
}
__device__ __forceinline__ void rt_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <typename R>
__global__ void __launch_bounds__(RP_NT, sizeof(R) == 4 ? 3 : 2) k_rhs_point(Geo g, const R* __restrict__ Q, const R* __restrict__ PR,
                                                        R* __restrict__ H0, R* __restrict__ RHS,
                                                        double* __restrict__ partial, DevState* __restrict__ st,
                                                        int ns, int kchunk) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* ring = reinterpret_cast<R*>(sm_raw);   // [slot][field][jj][ii]
    __shared__ double sred[32];
    __shared__ int is_last;
    const int L = g.L, M = g.M, N = g.N;
    const int ti = threadIdx.x % RT_I, tj = threadIdx.x / RT_I;
    const int i0 = blockIdx.x * RT_I, j0 = 1 + blockIdx.y * RT_J;
    const int k0 = blockIdx.z * kchunk, k1 = min(N, k0 + kchunk);
    const int i = i0 + ti, j = j0 + tj;
    const RhsLine<R> cl = rhs_line<R>(g, st->dt, ns, j);
    // plane kk of the march lives in slot (kk - k0 + 1) % RT_SLOTS; planes k0-1 ..
    // k0+RT_AHEAD go in first, one commit group each
    auto slot_of = [&](int kk) { return ring + ((kk - k0 + 1) % RT_SLOTS) * RT_SLOT; };
    for (int kk = k0 - 1; kk <= k0 + RT_AHEAD; ++kk) {
        if (kk <= k1) rt_load_plane<R>(g, Q, PR, H0, slot_of(kk), i0, j0, (kk % N + N) % N);
        rt_commit();
    }
    const int c = (tj + 1) * RT_HI + (ti + 1);          // this point inside a plane
    const int cim = c - 1, cip = c + 1, cjm = c - RT_HI, cjp = c + RT_HI;
    double bulk = 0.0;
    for (int k = k0; k < k1; ++k) {
        // planes up to k+1 have landed when at most RT_AHEAD - 1 groups are pending
        asm volatile("cp.async.wait_group %0;\n" ::"n"(RT_AHEAD - 1) : "memory");
        __syncthreads();
        const R* Pm = slot_of(k - 1);   // plane k-1
        const R* Pc = slot_of(k);       // plane k
        const R* Pp = slot_of(k + 1);   // plane k+1
        const R* Uc = Pc; const R* Vc = Pc + RT_PLANE; const R* Wc = Pc + 2 * RT_PLANE; const R* Rc = Pc + 3 * RT_PLANE;
        const R* Um = Pm; const R* Vm = Pm + RT_PLANE; const R* Wm = Pm + 2 * RT_PLANE; const R* Rm = Pm + 3 * RT_PLANE;
        const R* Up = Pp; const R* Vp = Pp + RT_PLANE; const R* Wp = Pp + 2 * RT_PLANE;
        RhsStencil<R> sp;
        sp.u = Uc[c]; sp.v = Vc[c]; sp.w = Wc[c];
        sp.uip = Uc[cip]; sp.uim = Uc[cim];
        sp.ujp = Uc[cjp]; sp.ujm = Uc[cjm]; sp.ukp = Up[c]; sp.ukm = Um[c];
        sp.vip = Vc[cip]; sp.vim = Vc[cim];
        sp.vjp = Vc[cjp]; sp.vjm = Vc[cjm]; sp.vkp = Vp[c]; sp.vkm = Vm[c];
        sp.wip = Wc[cip]; sp.wim = Wc[cim];
        sp.wjp = Wc[cjp]; sp.wjm = Wc[cjm]; sp.wkp = Wp[c]; sp.wkm = Wm[c];
        sp.pc = Rc[c];
        sp.pim = Rc[cim]; sp.pjm = Rc[cjm]; sp.pkm = Rm[c];
        sp.vjpim = Vc[cjp - 1]; sp.wkpim = Wp[cim];
        sp.ujmip = Uc[cjm + 1]; sp.wjmkp = Wp[cjm];
        sp.ukmip = Um[cip]; sp.vjpkm = Vm[cjp];
        const long long ii = iidx(g, i, j, k);
        const R* Hc = Pc + 4 * RT_PLANE + threadIdx.x;
        sp.h0u = Hc[0];
        sp.h0v = j >= 2 ? Hc[RT_I * RT_J] : R(0);
        sp.h0w = Hc[2 * RT_I * RT_J];
        R Hu, Hv, Hw, ru, rv, rw;
        rhs_point(cl, sp, j >= 2, Hu, Hv, Hw, ru, rv, rw, bulk);
        H0[ii] = Hu;
        H0[ii + 2 * g.FI] = Hw;
        RHS[ii] = ru;
        RHS[ii + 2 * g.FI] = rw;
        if (j >= 2) {
            H0[ii + g.FI] = Hv;
            RHS[ii + g.FI] = rv;
        }
        __syncthreads();   // plane k-1's slot is free: plane k+RT_AHEAD+1 goes there
        const int kn = k + RT_AHEAD + 1;
        if (kn <= k1) rt_load_plane<R>(g, Q, PR, H0, slot_of(kn), i0, j0, kn % N);
        rt_commit();
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    // grid sum of the bulk-flux integrand: block partials, last block in index order
    bulk = block_sum<RP_NT>(bulk, sred);
    const int nblk = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (threadIdx.x == 0) {
        partial[bid] = bulk;
        __threadfence();
        const unsigned prev = atomicAdd(&st->ctr, 1u);
        is_last = (prev == (unsigned)nblk - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        double sum = 0.0;
        for (int t = threadIdx.x; t < nblk; t += RP_NT) sum += __ldcg(partial + t);
        sum = block_sum<RP_NT>(sum, sred);
        if (threadIdx.x == 0) {
            st->bulksum = sum;
            st->ctr = 0u;
        }
    }
}

// cyclic x sweeps (MOMFA1_X_tg): one warp per (component, j, k) line, staged
// in segment-padded shared memory with coalesced loads and stores
constexpr int XS_NT = 256;
template <int S, typename R>
__global__ void __launch_bounds__(XS_NT) k_xsweep(Geo g, R* __restrict__ RHS, const R* __restrict__ fac) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* sm = reinterpret_cast<R*>(sm_raw);
    const int L = 32 * S, M = g.M;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long line = (long long)blockIdx.x * (XS_NT / 32) + warp;
    const long long nlines = 3LL * M * g.N;
    if (line >= nlines) return;
    const int comp = (int)(line / ((long long)M * g.N));
    const long long r = line - (long long)comp * M * g.N;
    const int j = 1 + (int)(r % M), k = (int)(r / M);
    if (comp == 1 && j == 1) return;  // MOMFA1_X_tg starts at N2I = 2 for v
    R* base = RHS + comp * g.FI + iidx(g, 0, j, k);
    R* sl = sm + warp * (L + 33);
    R v[S];
#pragma unroll
    for (int q = 0; q < S; ++q) v[q] = base[lane + 32 * q];
#pragma unroll
    for (int q = 0; q < S; ++q) sl[seg_pos<S>(lane + 32 * q)] = v[q];
    __syncwarp();
    warp_tdma_apply_smem<S, true>(sl, fac + FSET_X * FAC_SET, lane);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < S; ++q) base[lane + 32 * q] = sl[seg_pos<S>(lane + 32 * q)];
}
