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
