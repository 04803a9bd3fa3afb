// Batched tridiagonal line solvers for the Crank-Nicolson sweeps.
//
// Replaces TDMAIJI_CYC (src/TDMAIJI_CYC.f90:67-157) and TDMAIJJ_nonCYC
// (src/TDMAIJJ_nonCYC.f90:67-123).  One warp solves one line of length
// n = 32*S held in shared memory, lane l owning rows l*S .. l*S+S-1:
//   1. each lane eliminates its segment's interior rows (Thomas with three
//      right-hand sides), leaving two "interface" rows per lane that couple
//      only to the neighbouring lanes' interface rows;
//   2. the interface rows are folded into one unknown per lane (the lane's
//      last row) and solved by parallel cyclic reduction over the warp with
//      register shuffles (5 steps, or 4 steps plus a 2x2 solve when cyclic);
//   3. the interior rows are back-substituted in registers.
// The systems handled here (CN factors 1 - a - c with a, c < 0, and the
// y-momentum factors) are diagonally dominant, for which both stages are
// stable.  The pressure Poisson y-solve keeps the reference's sequential
// Thomas recurrence (see poisson.cuh).
#pragma once
#include "common.cuh"

// Position of row r inside a lane-segmented shared-memory line: one pad
// word after every segment of S rows makes the per-lane stride S+1 (odd),
// so the 32 lanes of a warp hit distinct banks.
template <int S>
__device__ __forceinline__ int seg_pos(int r) { return r + r / S; }

// Coefficient functor interface: a(r), b(r), c(r) for 0-based row r.
struct ConstCoef {
    double a, b, c;
    __device__ __forceinline__ double A(int) const { return a; }
    __device__ __forceinline__ double B(int) const { return b; }
    __device__ __forceinline__ double C(int) const { return c; }
};
struct SmemCoef {  // per-row coefficients in shared memory
    const double *a, *b, *c;
    __device__ __forceinline__ double A(int r) const { return a[r]; }
    __device__ __forceinline__ double B(int r) const { return b[r]; }
    __device__ __forceinline__ double C(int r) const { return c[r]; }
};

struct Row4 { double al, be, ga, de; };

__device__ __forceinline__ Row4 shfl_row(const Row4& r, int src) {
    Row4 o;
    o.al = __shfl_sync(0xffffffffu, r.al, src);
    o.be = __shfl_sync(0xffffffffu, r.be, src);
    o.ga = __shfl_sync(0xffffffffu, r.ga, src);
    o.de = __shfl_sync(0xffffffffu, r.de, src);
    return o;
}

// Solve one line in place.  d[k] holds the right-hand side of row lane*S+k
// on entry and the solution on exit.  For CYCLIC == false the rows obey the
// zero Dirichlet condition of TDMAIJJ_nonCYC with BCJ = 0: the coupling of
// row 0 to its left and of row n-1 to its right is dropped.
template <int S, bool CYCLIC, class Coef>
__device__ __forceinline__ void warp_tdma(double (&d)[S], const Coef& cf, int lane) {
    const int r0 = lane * S;
    double A0, B0, C0, D0, A1, B1, C1, D1;
    double ap[S > 2 ? S : 1], cq[S > 2 ? S : 1];
    if constexpr (S == 1) {
        A0 = cf.A(r0); B0 = cf.B(r0); C0 = cf.C(r0); D0 = d[0];
        A1 = B1 = C1 = D1 = 0.0;
    } else if constexpr (S == 2) {
        A0 = cf.A(r0); B0 = cf.B(r0); C0 = cf.C(r0); D0 = d[0];
        A1 = cf.A(r0 + 1); B1 = cf.B(r0 + 1); C1 = cf.C(r0 + 1); D1 = d[1];
    } else {
        // forward elimination over interior rows 1..S-2:
        //   y_k + ap_k*y_0 + cq_k*y_{k+1} = d_k
        {
            double r = 1.0 / cf.B(r0 + 1);
            ap[1] = cf.A(r0 + 1) * r;
            cq[1] = cf.C(r0 + 1) * r;
            d[1] *= r;
        }
#pragma unroll
        for (int k = 2; k <= S - 2; ++k) {
            double ak = cf.A(r0 + k);
            double r = 1.0 / (cf.B(r0 + k) - ak * cq[k - 1]);
            d[k] = (d[k] - ak * d[k - 1]) * r;
            ap[k] = -ak * ap[k - 1] * r;
            cq[k] = cf.C(r0 + k) * r;
        }
        // backward: y_k = d_k - ap_k*y_0 - cq_k*y_{S-1}
#pragma unroll
        for (int k = S - 3; k >= 1; --k) {
            d[k] = d[k] - cq[k] * d[k + 1];
            ap[k] = ap[k] - cq[k] * ap[k + 1];
            cq[k] = -cq[k] * cq[k + 1];
        }
        double c0 = cf.C(r0);
        A0 = cf.A(r0);
        B0 = cf.B(r0) - c0 * ap[1];
        C0 = -c0 * cq[1];
        D0 = d[0] - c0 * d[1];
        double aL = cf.A(r0 + S - 1);
        A1 = -aL * ap[S - 2];
        B1 = cf.B(r0 + S - 1) - aL * cq[S - 2];
        C1 = cf.C(r0 + S - 1);
        D1 = d[S - 1] - aL * d[S - 2];
    }
    if constexpr (!CYCLIC) {
        if (lane == 0) A0 = 0.0;
        if (lane == 31) { if constexpr (S == 1) C0 = 0.0; else C1 = 0.0; }
    }
    // one unknown per lane: u_l = y_{S-1} of lane l
    Row4 row;
    if constexpr (S == 1) {
        row.al = A0; row.be = B0; row.ga = C0; row.de = D0;
    } else {
        const int nx = (lane + 1) & 31;
        double A0n = __shfl_sync(0xffffffffu, A0, nx);
        double B0n = __shfl_sync(0xffffffffu, B0, nx);
        double C0n = __shfl_sync(0xffffffffu, C0, nx);
        double D0n = __shfl_sync(0xffffffffu, D0, nx);
        double iB0 = 1.0 / B0, iB0n = 1.0 / B0n;
        row.al = -A1 * A0 * iB0;
        row.be = B1 - A1 * C0 * iB0 - C1 * A0n * iB0n;
        row.ga = -C1 * C0n * iB0n;
        row.de = D1 - A1 * D0 * iB0 - C1 * D0n * iB0n;
    }
    // parallel cyclic reduction over the 32 lanes
    double u;
    if constexpr (CYCLIC) {
#pragma unroll
        for (int s = 1; s <= 8; s <<= 1) {
            Row4 lo = shfl_row(row, (lane - s) & 31);
            Row4 hi = shfl_row(row, (lane + s) & 31);
            double k1 = row.al / lo.be, k2 = row.ga / hi.be;
            Row4 nr;
            nr.al = -k1 * lo.al;
            nr.ga = -k2 * hi.ga;
            nr.be = row.be - k1 * lo.ga - k2 * hi.al;
            nr.de = row.de - k1 * lo.de - k2 * hi.de;
            row = nr;
        }
        Row4 pr = shfl_row(row, lane ^ 16);
        double ci = row.al + row.ga, cm = pr.al + pr.ga;
        u = (row.de * pr.be - ci * pr.de) / (row.be * pr.be - ci * cm);
    } else {
#pragma unroll
        for (int s = 1; s <= 16; s <<= 1) {
            Row4 lo = shfl_row(row, (lane - s) & 31);
            Row4 hi = shfl_row(row, (lane + s) & 31);
            bool hasl = lane - s >= 0, hash = lane + s <= 31;
            double k1 = hasl ? row.al / lo.be : 0.0;
            double k2 = hash ? row.ga / hi.be : 0.0;
            Row4 nr;
            nr.al = hasl ? -k1 * lo.al : 0.0;
            nr.ga = hash ? -k2 * hi.ga : 0.0;
            nr.be = row.be - (hasl ? k1 * lo.ga : 0.0) - (hash ? k2 * hi.al : 0.0);
            nr.de = row.de - (hasl ? k1 * lo.de : 0.0) - (hash ? k2 * hi.de : 0.0);
            row = nr;
        }
        u = row.de / row.be;
    }
    if constexpr (S == 1) {
        d[0] = u;
    } else {
        double up = __shfl_sync(0xffffffffu, u, (lane - 1) & 31);
        double y0 = (D0 - A0 * up - C0 * u) / B0;  // A0 == 0 on lane 0 when not cyclic
        d[0] = y0;
        d[S - 1] = u;
        if constexpr (S > 2) {
#pragma unroll
            for (int k = 1; k <= S - 2; ++k) d[k] = d[k] - ap[k] * y0 - cq[k] * u;
        }
    }
}

// Solve one line stored in shared memory at base[seg_pos<S>(r)], r = 0..32*S-1.
template <int S, bool CYCLIC, class Coef>
__device__ __forceinline__ void warp_tdma_smem(double* base, const Coef& cf, int lane) {
    double d[S];
#pragma unroll
    for (int k = 0; k < S; ++k) d[k] = base[lane * (S + 1) + k];
    warp_tdma<S, CYCLIC>(d, cf, lane);
#pragma unroll
    for (int k = 0; k < S; ++k) base[lane * (S + 1) + k] = d[k];
}

// ---------------------------------------------------------------------------
// Factorised form of warp_tdma for systems whose coefficients are the same
// for every line of a batch (the constant-coefficient x and z sweeps, and
// the y sweep whose coefficients depend on the row only).  warp_tdma_factor
// runs the coefficient part of the algorithm once and stores, per lane, the
// multipliers it produces; warp_tdma_apply then performs only the
// right-hand-side part: a few FMAs per row and one shuffle per reduction
// step.  The factor table of one system is TF_NF(S) x 32 doubles, laid out
// [item][lane] so that a warp reads it with coalesced accesses.
#define TF_NF(S) (5 * (S) + 20)

// The factors are always computed in FP64; T is the type they are stored in
// (float for the FP32 sweeps of the mixed-precision step).
template <int S, bool CYCLIC, class Coef, typename T = double>
__device__ void warp_tdma_factor(const Coef& cf, int lane, T* __restrict__ fac) {
    const int r0 = lane * S;
    // item layout: [0,S) r, [S,2S) a, [2S,3S) cq(fwd), [3S,4S) ap(final), [4S,5S) cq(final),
    //   5S+0 c0, +1 aL, +2 A0, +3 C0, +4 iB0, +5 ra, +6 rb, +7..+11 k1[5], +12..+16 k2[5], +17 f1, +18 f2, +19 unused
    double rr[S > 2 ? S : 1], aa[S > 2 ? S : 1], cqf[S > 2 ? S : 1], ap[S > 2 ? S : 1], cq[S > 2 ? S : 1];
    double A0, B0, C0, A1, B1, C1, c0 = 0.0, aL = 0.0;
#pragma unroll
    for (int k = 0; k < (S > 2 ? S : 1); ++k) { rr[k] = aa[k] = cqf[k] = ap[k] = cq[k] = 0.0; }
    if constexpr (S == 1) {
        A0 = cf.A(r0); B0 = cf.B(r0); C0 = cf.C(r0);
        A1 = B1 = C1 = 0.0;
    } else if constexpr (S == 2) {
        A0 = cf.A(r0); B0 = cf.B(r0); C0 = cf.C(r0);
        A1 = cf.A(r0 + 1); B1 = cf.B(r0 + 1); C1 = cf.C(r0 + 1);
    } else {
        rr[1] = 1.0 / cf.B(r0 + 1);
        ap[1] = cf.A(r0 + 1) * rr[1];
        cq[1] = cf.C(r0 + 1) * rr[1];
#pragma unroll
        for (int k = 2; k <= S - 2; ++k) {
            aa[k] = cf.A(r0 + k);
            rr[k] = 1.0 / (cf.B(r0 + k) - aa[k] * cq[k - 1]);
            ap[k] = -aa[k] * ap[k - 1] * rr[k];
            cq[k] = cf.C(r0 + k) * rr[k];
        }
#pragma unroll
        for (int k = 0; k < S; ++k) cqf[k] = cq[k];
#pragma unroll
        for (int k = S - 3; k >= 1; --k) {
            ap[k] = ap[k] - cq[k] * ap[k + 1];
            cq[k] = -cq[k] * cq[k + 1];
        }
        c0 = cf.C(r0);
        A0 = cf.A(r0);
        B0 = cf.B(r0) - c0 * ap[1];
        C0 = -c0 * cq[1];
        aL = cf.A(r0 + S - 1);
        A1 = -aL * ap[S - 2];
        B1 = cf.B(r0 + S - 1) - aL * cq[S - 2];
        C1 = cf.C(r0 + S - 1);
    }
    if constexpr (!CYCLIC) {
        if (lane == 0) A0 = 0.0;
        if (lane == 31) { if constexpr (S == 1) C0 = 0.0; else C1 = 0.0; }
    }
    double al, be, ga, iB0 = 1.0, ra = 0.0, rb = 0.0;
    if constexpr (S == 1) {
        al = A0; be = B0; ga = C0;
    } else {
        const int nx = (lane + 1) & 31;
        double A0n = __shfl_sync(0xffffffffu, A0, nx);
        double B0n = __shfl_sync(0xffffffffu, B0, nx);
        double C0n = __shfl_sync(0xffffffffu, C0, nx);
        iB0 = 1.0 / B0;
        double iB0n = 1.0 / B0n;
        al = -A1 * A0 * iB0;
        be = B1 - A1 * C0 * iB0 - C1 * A0n * iB0n;
        ga = -C1 * C0n * iB0n;
        ra = A1 * iB0;
        rb = C1 * iB0n;
    }
    double k1s[5] = {0, 0, 0, 0, 0}, k2s[5] = {0, 0, 0, 0, 0};
    double f1, f2 = 0.0;
    const int nsteps = CYCLIC ? 4 : 5;
#pragma unroll
    for (int st = 0; st < 5; ++st) {
        if (st >= nsteps) break;
        const int s = 1 << st;
        const double lal = __shfl_sync(0xffffffffu, al, (lane - s) & 31);
        const double lbe = __shfl_sync(0xffffffffu, be, (lane - s) & 31);
        const double lga = __shfl_sync(0xffffffffu, ga, (lane - s) & 31);
        const double hal = __shfl_sync(0xffffffffu, al, (lane + s) & 31);
        const double hbe = __shfl_sync(0xffffffffu, be, (lane + s) & 31);
        const double hga = __shfl_sync(0xffffffffu, ga, (lane + s) & 31);
        bool hasl = CYCLIC || lane - s >= 0, hash = CYCLIC || lane + s <= 31;
        double k1 = hasl ? al / lbe : 0.0;
        double k2 = hash ? ga / hbe : 0.0;
        double nal = hasl ? -k1 * lal : 0.0;
        double nga = hash ? -k2 * hga : 0.0;
        double nbe = be - (hasl ? k1 * lga : 0.0) - (hash ? k2 * hal : 0.0);
        k1s[st] = k1; k2s[st] = k2;
        al = nal; be = nbe; ga = nga;
    }
    if constexpr (CYCLIC) {
        const double pal = __shfl_sync(0xffffffffu, al, lane ^ 16);
        const double pbe = __shfl_sync(0xffffffffu, be, lane ^ 16);
        const double pga = __shfl_sync(0xffffffffu, ga, lane ^ 16);
        const double ci = al + ga, cm = pal + pga;
        const double inv = 1.0 / (be * pbe - ci * cm);
        f1 = pbe * inv;
        f2 = -ci * inv;
    } else {
        f1 = 1.0 / be;
    }
    T* f = fac + lane;
#pragma unroll
    for (int k = 0; k < S; ++k) {
        if constexpr (S > 2) {
            f[(0 * S + k) * 32] = (T)rr[k];
            f[(1 * S + k) * 32] = (T)aa[k];
            f[(2 * S + k) * 32] = (T)cqf[k];
            f[(3 * S + k) * 32] = (T)ap[k];
            f[(4 * S + k) * 32] = (T)cq[k];
        } else {
            f[(0 * S + k) * 32] = T(0);
            f[(1 * S + k) * 32] = T(0);
            f[(2 * S + k) * 32] = T(0);
            f[(3 * S + k) * 32] = T(0);
            f[(4 * S + k) * 32] = T(0);
        }
    }
    const int b = 5 * S;
    f[(b + 0) * 32] = (T)c0; f[(b + 1) * 32] = (T)aL; f[(b + 2) * 32] = (T)A0; f[(b + 3) * 32] = (T)C0;
    f[(b + 4) * 32] = (T)iB0; f[(b + 5) * 32] = (T)ra; f[(b + 6) * 32] = (T)rb;
#pragma unroll
    for (int st = 0; st < 5; ++st) { f[(b + 7 + st) * 32] = (T)k1s[st]; f[(b + 12 + st) * 32] = (T)k2s[st]; }
    f[(b + 17) * 32] = (T)f1; f[(b + 18) * 32] = (T)f2;
}

// Right-hand-side part of the solve; d[k] = rhs of row lane*S+k in, solution out.
template <int S, bool CYCLIC, typename R>
__device__ __forceinline__ void warp_tdma_apply(R (&d)[S], const R* __restrict__ fac, int lane) {
    const R* f = fac + lane;
    const int b = 5 * S;
    R D0, D1;
    if constexpr (S >= 3) {
        d[1] *= f[(0 * S + 1) * 32];
#pragma unroll
        for (int k = 2; k <= S - 2; ++k) d[k] = (d[k] - f[(1 * S + k) * 32] * d[k - 1]) * f[(0 * S + k) * 32];
#pragma unroll
        for (int k = S - 3; k >= 1; --k) d[k] = d[k] - f[(2 * S + k) * 32] * d[k + 1];
        D0 = d[0] - f[(b + 0) * 32] * d[1];
        D1 = d[S - 1] - f[(b + 1) * 32] * d[S - 2];
    } else if constexpr (S == 2) {
        D0 = d[0];
        D1 = d[1];
    } else {
        D0 = d[0];
        D1 = R(0);
    }
    R de;
    if constexpr (S == 1) {
        de = D0;
    } else {
        const R D0n = __shfl_sync(0xffffffffu, D0, (lane + 1) & 31);
        de = D1 - f[(b + 5) * 32] * D0 - f[(b + 6) * 32] * D0n;
    }
    const int nsteps = CYCLIC ? 4 : 5;
#pragma unroll
    for (int st = 0; st < 5; ++st) {
        if (st >= nsteps) break;
        const int s = 1 << st;
        const R lo = __shfl_sync(0xffffffffu, de, (lane - s) & 31);
        const R hi = __shfl_sync(0xffffffffu, de, (lane + s) & 31);
        de = de - f[(b + 7 + st) * 32] * lo - f[(b + 12 + st) * 32] * hi;
    }
    R u;
    if constexpr (CYCLIC) {
        const R pd = __shfl_sync(0xffffffffu, de, lane ^ 16);
        u = de * f[(b + 17) * 32] + pd * f[(b + 18) * 32];
    } else {
        u = de * f[(b + 17) * 32];
    }
    if constexpr (S == 1) {
        d[0] = u;
    } else {
        const R up = __shfl_sync(0xffffffffu, u, (lane - 1) & 31);
        const R y0 = (D0 - f[(b + 2) * 32] * up - f[(b + 3) * 32] * u) * f[(b + 4) * 32];
        d[0] = y0;
        d[S - 1] = u;
        if constexpr (S > 2) {
#pragma unroll
            for (int k = 1; k <= S - 2; ++k) d[k] = d[k] - f[(3 * S + k) * 32] * y0 - f[(4 * S + k) * 32] * u;
        }
    }
}

// warp_tdma_apply for NR right-hand sides that share one factor table (the
// three components of an x line, or several lines of one z or y sweep): each
// factor is loaded once and the NR dependency chains interleave, which is
// what the latency-bound sweeps need.  Per right-hand side the arithmetic is
// exactly that of warp_tdma_apply.
template <int S, bool CYCLIC, int NR, typename R>
__device__ __forceinline__ void warp_tdma_apply_n(R (&d)[NR][S], const R* __restrict__ fac, int lane) {
    const R* f = fac + lane;
    const int b = 5 * S;
    R D0[NR], D1[NR];
    if constexpr (S >= 3) {
        const R f01 = f[(0 * S + 1) * 32];
#pragma unroll
        for (int r = 0; r < NR; ++r) d[r][1] *= f01;
#pragma unroll
        for (int k = 2; k <= S - 2; ++k) {
            const R fa = f[(1 * S + k) * 32], fr = f[(0 * S + k) * 32];
#pragma unroll
            for (int r = 0; r < NR; ++r) d[r][k] = (d[r][k] - fa * d[r][k - 1]) * fr;
        }
#pragma unroll
        for (int k = S - 3; k >= 1; --k) {
            const R fc = f[(2 * S + k) * 32];
#pragma unroll
            for (int r = 0; r < NR; ++r) d[r][k] = d[r][k] - fc * d[r][k + 1];
        }
        const R g0 = f[(b + 0) * 32], g1 = f[(b + 1) * 32];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            D0[r] = d[r][0] - g0 * d[r][1];
            D1[r] = d[r][S - 1] - g1 * d[r][S - 2];
        }
    } else if constexpr (S == 2) {
#pragma unroll
        for (int r = 0; r < NR; ++r) { D0[r] = d[r][0]; D1[r] = d[r][1]; }
    } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) { D0[r] = d[r][0]; D1[r] = R(0); }
    }
    R de[NR];
    if constexpr (S == 1) {
#pragma unroll
        for (int r = 0; r < NR; ++r) de[r] = D0[r];
    } else {
        const R f5 = f[(b + 5) * 32], f6 = f[(b + 6) * 32];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const R D0n = __shfl_sync(0xffffffffu, D0[r], (lane + 1) & 31);
            de[r] = D1[r] - f5 * D0[r] - f6 * D0n;
        }
    }
    const int nsteps = CYCLIC ? 4 : 5;
#pragma unroll
    for (int st = 0; st < 5; ++st) {
        if (st >= nsteps) break;
        const int s = 1 << st;
        const R k1 = f[(b + 7 + st) * 32], k2 = f[(b + 12 + st) * 32];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const R lo = __shfl_sync(0xffffffffu, de[r], (lane - s) & 31);
            const R hi = __shfl_sync(0xffffffffu, de[r], (lane + s) & 31);
            de[r] = de[r] - k1 * lo - k2 * hi;
        }
    }
    R u[NR];
    const R f17 = f[(b + 17) * 32];
    if constexpr (CYCLIC) {
        const R f18 = f[(b + 18) * 32];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const R pd = __shfl_sync(0xffffffffu, de[r], lane ^ 16);
            u[r] = de[r] * f17 + pd * f18;
        }
    } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) u[r] = de[r] * f17;
    }
    if constexpr (S == 1) {
#pragma unroll
        for (int r = 0; r < NR; ++r) d[r][0] = u[r];
    } else {
        const R f2 = f[(b + 2) * 32], f3 = f[(b + 3) * 32], f4 = f[(b + 4) * 32];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const R up = __shfl_sync(0xffffffffu, u[r], (lane - 1) & 31);
            const R y0 = (D0[r] - f2 * up - f3 * u[r]) * f4;
            d[r][0] = y0;
            d[r][S - 1] = u[r];
        }
        if constexpr (S > 2) {
#pragma unroll
            for (int k = 1; k <= S - 2; ++k) {
                const R fy0 = f[(3 * S + k) * 32], fu = f[(4 * S + k) * 32];
#pragma unroll
                for (int r = 0; r < NR; ++r) d[r][k] = d[r][k] - fy0 * d[r][0] - fu * u[r];
            }
        }
    }
}

// The three x lines of one (j, k) in segment-padded shared memory at base,
// base + ls, base + 2 ls; line 1 (v) is solved but written back only when
// keep1 (MOMFA1_X_tg starts at N2I = 2 for v).
template <int S, bool CYCLIC, typename R>
__device__ __forceinline__ void warp_tdma_apply_smem3(R* base, int ls, bool keep1, const R* __restrict__ fac, int lane) {
    R d[3][S];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < S; ++k) d[c][k] = base[c * ls + lane * (S + 1) + k];
    warp_tdma_apply_n<S, CYCLIC, 3>(d, fac, lane);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (c == 1 && !keep1) continue;
#pragma unroll
        for (int k = 0; k < S; ++k) base[c * ls + lane * (S + 1) + k] = d[c][k];
    }
}

template <int S, bool CYCLIC, typename R>
__device__ __forceinline__ void warp_tdma_apply_smem(R* base, const R* __restrict__ fac, int lane) {
    R d[S];
#pragma unroll
    for (int k = 0; k < S; ++k) d[k] = base[lane * (S + 1) + k];
    warp_tdma_apply<S, CYCLIC>(d, fac, lane);
#pragma unroll
    for (int k = 0; k < S; ++k) base[lane * (S + 1) + k] = d[k];
}

// ---------------------------------------------------------------------------
// warp_tdma (non-cyclic) with a complex right-hand side: the real and
// imaginary parts share the real coefficients, as in the per-wavenumber
// y-solves of the pressure Poisson equation.
__device__ __forceinline__ double2 c_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 c_sub_scaled(double2 a, double s, double2 b) {  // a - s*b
    return make_double2(a.x - s * b.x, a.y - s * b.y);
}

template <int S, class Coef>
__device__ __forceinline__ void warp_tdma_c(double2 (&d)[S], const Coef& cf, int lane) {
    const int r0 = lane * S;
    double A0, B0, C0, A1, B1, C1;
    double2 D0, D1;
    double ap[S > 2 ? S : 1], cq[S > 2 ? S : 1];
    if constexpr (S == 1) {
        A0 = cf.A(r0); B0 = cf.B(r0); C0 = cf.C(r0); D0 = d[0];
        A1 = B1 = C1 = 0.0; D1 = make_double2(0.0, 0.0);
    } else if constexpr (S == 2) {
        A0 = cf.A(r0); B0 = cf.B(r0); C0 = cf.C(r0); D0 = d[0];
        A1 = cf.A(r0 + 1); B1 = cf.B(r0 + 1); C1 = cf.C(r0 + 1); D1 = d[1];
    } else {
        {
            const double r = 1.0 / cf.B(r0 + 1);
            ap[1] = cf.A(r0 + 1) * r;
            cq[1] = cf.C(r0 + 1) * r;
            d[1] = c_scale(d[1], r);
        }
#pragma unroll
        for (int k = 2; k <= S - 2; ++k) {
            const double ak = cf.A(r0 + k);
            const double r = 1.0 / (cf.B(r0 + k) - ak * cq[k - 1]);
            d[k] = c_scale(c_sub_scaled(d[k], ak, d[k - 1]), r);
            ap[k] = -ak * ap[k - 1] * r;
            cq[k] = cf.C(r0 + k) * r;
        }
#pragma unroll
        for (int k = S - 3; k >= 1; --k) {
            d[k] = c_sub_scaled(d[k], cq[k], d[k + 1]);
            ap[k] = ap[k] - cq[k] * ap[k + 1];
            cq[k] = -cq[k] * cq[k + 1];
        }
        const double c0 = cf.C(r0);
        A0 = cf.A(r0);
        B0 = cf.B(r0) - c0 * ap[1];
        C0 = -c0 * cq[1];
        D0 = c_sub_scaled(d[0], c0, d[1]);
        const double aL = cf.A(r0 + S - 1);
        A1 = -aL * ap[S - 2];
        B1 = cf.B(r0 + S - 1) - aL * cq[S - 2];
        C1 = cf.C(r0 + S - 1);
        D1 = c_sub_scaled(d[S - 1], aL, d[S - 2]);
    }
    if (lane == 0) A0 = 0.0;
    if (lane == 31) { if constexpr (S == 1) C0 = 0.0; else C1 = 0.0; }
    double al, be, ga;
    double2 de;
    if constexpr (S == 1) {
        al = A0; be = B0; ga = C0; de = D0;
    } else {
        const int nx = (lane + 1) & 31;
        const double A0n = __shfl_sync(0xffffffffu, A0, nx);
        const double B0n = __shfl_sync(0xffffffffu, B0, nx);
        const double C0n = __shfl_sync(0xffffffffu, C0, nx);
        const double2 D0n = make_double2(__shfl_sync(0xffffffffu, D0.x, nx), __shfl_sync(0xffffffffu, D0.y, nx));
        const double iB0 = 1.0 / B0, iB0n = 1.0 / B0n;
        al = -A1 * A0 * iB0;
        be = B1 - A1 * C0 * iB0 - C1 * A0n * iB0n;
        ga = -C1 * C0n * iB0n;
        de = c_sub_scaled(c_sub_scaled(D1, A1 * iB0, D0), C1 * iB0n, D0n);
    }
#pragma unroll
    for (int s = 1; s <= 16; s <<= 1) {
        const int lo = (lane - s) & 31, hi = (lane + s) & 31;
        const double lal = __shfl_sync(0xffffffffu, al, lo), lbe = __shfl_sync(0xffffffffu, be, lo);
        const double lga = __shfl_sync(0xffffffffu, ga, lo);
        const double hal = __shfl_sync(0xffffffffu, al, hi), hbe = __shfl_sync(0xffffffffu, be, hi);
        const double hga = __shfl_sync(0xffffffffu, ga, hi);
        const double2 lde = make_double2(__shfl_sync(0xffffffffu, de.x, lo), __shfl_sync(0xffffffffu, de.y, lo));
        const double2 hde = make_double2(__shfl_sync(0xffffffffu, de.x, hi), __shfl_sync(0xffffffffu, de.y, hi));
        const bool hasl = lane - s >= 0, hash = lane + s <= 31;
        const double k1 = hasl ? al / lbe : 0.0;
        const double k2 = hash ? ga / hbe : 0.0;
        const double nal = hasl ? -k1 * lal : 0.0;
        const double nga = hash ? -k2 * hga : 0.0;
        be = be - (hasl ? k1 * lga : 0.0) - (hash ? k2 * hal : 0.0);
        if (hasl) de = c_sub_scaled(de, k1, lde);
        if (hash) de = c_sub_scaled(de, k2, hde);
        al = nal;
        ga = nga;
    }
    const double2 u = c_scale(de, 1.0 / be);
    if constexpr (S == 1) {
        d[0] = u;
    } else {
        const int pv = (lane - 1) & 31;
        const double2 up = make_double2(__shfl_sync(0xffffffffu, u.x, pv), __shfl_sync(0xffffffffu, u.y, pv));
        const double iB0 = 1.0 / B0;
        const double2 y0 = c_scale(c_sub_scaled(c_sub_scaled(D0, A0, up), C0, u), iB0);  // A0 == 0 on lane 0
        d[0] = y0;
        d[S - 1] = u;
        if constexpr (S > 2) {
#pragma unroll
            for (int k = 1; k <= S - 2; ++k) d[k] = c_sub_scaled(c_sub_scaled(d[k], ap[k], y0), cq[k], u);
        }
    }
}
