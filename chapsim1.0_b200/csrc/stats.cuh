// On-device statistics of the periodic channel (POSTPROCESS_TG,
// src/processing/POSTPROESS.f90:11-51): the x-z plane means of
// PP_MEAN_ZX_FLOW_TG (src/processing/PP_MEAN_ZX.f90:14-307), their time
// average PP_MEAN_T_TG (src/processing/PP_MEAN_T.f90:343-392), and the
// quantities PP_MONITOR_TG prints (src/processing/PP_SCN_MONITOR.f90:147-251),
// so that an unchanged driver needs no per-step download of Q.
//
// Per y row j (plane channel: RCCI1 = RNDI1 = 1), with U_i the cell-centred
// velocity sums (two face values, the reference's U_CCT) and dU_i/dx_j the
// reference's DVDL_CCT differences:
//   U1xzL(j, 1:3) = <U_i>/2, U1xzL(j, 4) = <p>, UPxzL = <U_i p>/2,
//   U2xzL = <U_i U_j>/4 (6, upper triangle), U3xzL = <U_i U_j U_k>/8 (10),
//   DVDL1xzL = <dU>*COG1, DVDLPxzL = <p dU>*COG1, DVDL2xzL = <dU dU>*COG2 (9 x 9).
// Each thread accumulates 86 sums over its share of the row: 41 of the
// first six groups and the 45 distinct products of the 9 gradients (the 81
// entries of DVDL2xzL are symmetric, and so is COG2).  Block partials go to
// global memory; k_pp_finish adds the chunks of a row in a fixed order and
// scales (deterministic; the reference adds in its I, K loop order).
//
// Device storage of one set of means (instantaneous or time-averaged), all
// Fortran order with j fastest, M = NCL2:
//   U1xzL(M,4) | UPxzL(M,3) | U2xzL(M,6) | U3xzL(M,10) | DVDL1xzL(M,3,3) |
//   DVDLPxzL(M,3,3) | DVDL2xzL(M,9,9)   -> 122*M doubles.
#pragma once
#include "common.cuh"

#define PP_NT 128
#define PP_NACC 86
#define PP_PER_ROW 122
// offsets (in units of M) of the arrays of one set
#define PP_U1 0
#define PP_UP 4
#define PP_U2 7
#define PP_U3 13
#define PP_D1 23
#define PP_DP 32
#define PP_D2 41

// index of the product g[a]*g[b] (a <= b) among the 45 distinct ones
__host__ __device__ __forceinline__ int pp_sym(int a, int b) { return a * 9 - (a * (a - 1)) / 2 + (b - a); }

template <typename R>
__global__ void __launch_bounds__(PP_NT) k_pp_mean_zx(Geo g, const R* __restrict__ Q, const R* __restrict__ PR,
                                                      double* __restrict__ part) {
    const int L = g.L, M = g.M, N = g.N;
    const int j = 1 + blockIdx.y;
    const int jp = j + 1, jm = j - 1;
    const double dycij = g.dyci[j], dycip = g.dyci[jp], dyfij = g.dyfi[j];
    const R* U = Q;
    const R* V = Q + g.FS;
    const R* W = Q + 2 * g.FS;
    double a[PP_NACC];
#pragma unroll
    for (int q = 0; q < PP_NACC; ++q) a[q] = 0.0;
    const int plane = L * N;
    for (int t = blockIdx.x * PP_NT + threadIdx.x; t < plane; t += gridDim.x * PP_NT) {
        const int k = t / L, i = t - k * L;
        const int ip = wrapp(i, L), im = wrapm(i, L), kp = wrapp(k, N), km = wrapm(k, N);
        auto q = [&](const R* F, int ii, int jj, int kk) { return (double)F[pidx(g, ii, jj, kk)]; };
        double uc[3], ujp[3], ujm[3], ukp[3], ukm[3], uip[3], uim[3];
        uc[0] = q(U, i, j, k) + q(U, ip, j, k);
        ujp[0] = q(U, i, jp, k) + q(U, ip, jp, k);
        ujm[0] = q(U, i, jm, k) + q(U, ip, jm, k);
        ukp[0] = q(U, i, j, kp) + q(U, ip, j, kp);
        ukm[0] = q(U, i, j, km) + q(U, ip, j, km);
        uc[2] = (q(W, i, j, k) + q(W, i, j, kp)) * 1.0;
        uip[2] = (q(W, ip, j, k) + q(W, ip, j, kp)) * 1.0;
        uim[2] = (q(W, im, j, k) + q(W, im, j, kp)) * 1.0;
        ujp[2] = (q(W, i, jp, k) + q(W, i, jp, kp)) * 1.0;
        ujm[2] = (q(W, i, jm, k) + q(W, i, jm, kp)) * 1.0;
        uc[1] = (q(V, i, j, k) + q(V, i, jp, k)) * 1.0;
        uip[1] = (q(V, ip, j, k) + q(V, ip, jp, k)) * 1.0;
        uim[1] = (q(V, im, j, k) + q(V, im, jp, k)) * 1.0;
        ukp[1] = (q(V, i, j, kp) + q(V, i, jp, kp)) * 1.0;
        ukm[1] = (q(V, i, j, km) + q(V, i, jp, km)) * 1.0;
        const double p = q(PR, i, j, k);
        // MEAN U, V, W, P
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            a[m] += uc[m];
            a[4 + m] += uc[m] * p;
        }
        a[3] += p;
        // MEAN UU, UV, ... (upper triangle, storage order of U2xzL)
        a[7] += uc[0] * uc[0]; a[8] += uc[0] * uc[1]; a[9] += uc[0] * uc[2];
        a[10] += uc[1] * uc[1]; a[11] += uc[1] * uc[2]; a[12] += uc[2] * uc[2];
        // MEAN UUU, UUV, ... (storage order of U3xzL)
        a[13] += uc[0] * uc[0] * uc[0]; a[14] += uc[0] * uc[0] * uc[1]; a[15] += uc[0] * uc[0] * uc[2];
        a[16] += uc[0] * uc[1] * uc[1]; a[17] += uc[0] * uc[1] * uc[2]; a[18] += uc[0] * uc[2] * uc[2];
        a[19] += uc[1] * uc[1] * uc[1]; a[20] += uc[1] * uc[1] * uc[2]; a[21] += uc[1] * uc[2] * uc[2];
        a[22] += uc[2] * uc[2] * uc[2];
        // velocity gradients DVDL_CCT(m, n), m-major
        double d[9];
        d[0] = q(U, ip, j, k) - q(U, i, j, k);
        d[1] = (ujp[0] - uc[0]) * dycip + (uc[0] - ujm[0]) * dycij;
        d[2] = ukp[0] - ukm[0];
        d[3] = uip[1] - uim[1];
        d[4] = (q(V, i, jp, k) * 1.0 - q(V, i, j, k) * 1.0) * dyfij;
        d[5] = ukp[1] - ukm[1];
        d[6] = uip[2] - uim[2];
        d[7] = (ujp[2] - uc[2]) * dycip + (uc[2] - ujm[2]) * dycij;
        d[8] = q(W, i, j, kp) * 1.0 - q(W, i, j, k) * 1.0;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            a[23 + e] += d[e];
            a[32 + e] += d[e] * p;
        }
#pragma unroll
        for (int x = 0; x < 9; ++x)
#pragma unroll
            for (int y = x; y < 9; ++y) a[41 + pp_sym(x, y)] += d[x] * d[y];
    }
    // block reduction: warp shuffles, then the warps in index order
    __shared__ double sw[PP_NT / 32][PP_NACC];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q2 = 0; q2 < PP_NACC; ++q2) {
        double v = a[q2];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sw[warp][q2] = v;
    }
    __syncthreads();
    for (int q2 = threadIdx.x; q2 < PP_NACC; q2 += PP_NT) {
        double s = 0.0;
        for (int w = 0; w < PP_NT / 32; ++w) s += sw[w][q2];
        part[((size_t)(j - 1) * gridDim.x + blockIdx.x) * PP_NACC + q2] = s;
    }
}

// Sum of a row's chunks (in chunk order) and the scalings of PP_MEAN_ZX_FLOW_TG :257-294.
__global__ void __launch_bounds__(PP_NT) k_pp_finish(Geo g, const double* __restrict__ part, int nchunk,
                                                     double* __restrict__ out) {
    __shared__ double s[PP_NACC];
    const int M = g.M;
    const int j = 1 + blockIdx.x;
    for (int q = threadIdx.x; q < PP_NACC; q += PP_NT) {
        double v = 0.0;
        for (int c = 0; c < nchunk; ++c) v += part[((size_t)(j - 1) * nchunk + c) * PP_NACC + q];
        s[q] = v;
    }
    __syncthreads();
    const double VL = 1.0 / (double)(g.L * g.N);  // VL1313_tg (src/CONSPARA.f90:80)
    const double COE0 = VL, COE1 = VL * 0.5, COE2 = VL * (0.5 * 0.5), COE3 = VL * (0.5 * 0.5 * 0.5);
    const double cog[9] = {VL * g.dxi, VL * 0.25, VL * 0.25 * g.dzi, VL * 0.25 * g.dxi, VL,
                           VL * 0.25 * g.dzi, VL * 0.25 * g.dxi, VL * 0.25, VL * g.dzi};
    const int r = j - 1;
    if (threadIdx.x < 3) {
        const int m = threadIdx.x;
        out[(size_t)(PP_U1 + m) * M + r] = s[m] * COE1;
        out[(size_t)(PP_UP + m) * M + r] = s[4 + m] * COE1;
    }
    if (threadIdx.x == 3) out[(size_t)(PP_U1 + 3) * M + r] = s[3] * COE0;
    if (threadIdx.x < 6) out[(size_t)(PP_U2 + threadIdx.x) * M + r] = s[7 + threadIdx.x] * COE2;
    if (threadIdx.x < 10) out[(size_t)(PP_U3 + threadIdx.x) * M + r] = s[13 + threadIdx.x] * COE3;
    if (threadIdx.x < 9) {
        // DVDL1xzL(j, m, n): element (m, n) at m + 3 n (Fortran), accumulator e = 3 m + n
        const int m = threadIdx.x / 3, n = threadIdx.x % 3;
        out[(size_t)(PP_D1 + m + 3 * n) * M + r] = s[23 + 3 * m + n] * cog[3 * m + n];
        out[(size_t)(PP_DP + m + 3 * n) * M + r] = s[32 + 3 * m + n] * cog[3 * m + n];
    }
    for (int e = threadIdx.x; e < 81; e += PP_NT) {
        // DVDL2xzL(j, L1, L2), L1 = 3 M + H, L2 = 3 N + P (0-based): product of DVDL(M,H) and DVDL(N,P)
        const int l1 = e % 9, l2 = e / 9;
        const int x = l1 < l2 ? l1 : l2, y = l1 < l2 ? l2 : l1;
        out[(size_t)(PP_D2 + l1 + 9 * l2) * M + r] = s[41 + pp_sym(x, y)] * (cog[l1] * cog[l2]);
    }
}

// PP_MEAN_T_TG: avg = coe3 * avg + coe2 * inst over every entry of a set
__global__ void k_pp_time_average(double* __restrict__ avg, const double* __restrict__ inst, long long n, double coe2,
                                  double coe3) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        avg[t] = coe3 * avg[t] + coe2 * inst[t];
}

// U1mean / U1maxx of PP_MEAN_ZX_FLOW_TG (:294-305) and the PP_MONITOR_TG
// quantities (:165-226).  mon[20]: U1_XZT(1:6), UU_XZT(1:8), CF_XZT(1:4),
// U1mean_WORK_tg, U1maxx_WORK_tg.  One thread, rows in order.
__global__ void k_pp_monitor(Geo g, const double* __restrict__ inst, const double* __restrict__ avg, double ren,
                             double* __restrict__ mon) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int M = g.M;
    auto U1 = [&](const double* s, int jr, int m) { return s[(size_t)(PP_U1 + m - 1) * M + (jr - 1)]; };
    auto U2 = [&](const double* s, int jr, int l) { return s[(size_t)(PP_U2 + l - 1) * M + (jr - 1)]; };
    double mean = 0.0, mx = 0.0;
    for (int jr = 1; jr <= M; ++jr) {
        mean = mean + U1(inst, jr, 1) / g.dyfi[jr] / 1.0;
        mx = fmax(mx, fabs(U1(inst, jr, 1)));
    }
    mean = mean / g.dzi * (double)g.N / g.area_inlet;
    const int js = M / 2;
    mon[0] = U1(inst, js, 1); mon[1] = U1(avg, js, 1);
    mon[2] = U1(inst, js, 2); mon[3] = U1(avg, js, 2);
    mon[4] = U1(inst, js, 3); mon[5] = U1(avg, js, 3);
    mon[6] = U2(inst, js, 1) - U1(inst, js, 1) * U1(inst, js, 1);
    mon[7] = U2(avg, js, 1) - U1(avg, js, 1) * U1(avg, js, 1);
    mon[8] = U2(inst, js, 2) - U1(inst, js, 1) * U1(inst, js, 2);
    mon[9] = U2(avg, js, 2) - U1(avg, js, 1) * U1(avg, js, 2);
    mon[10] = U2(inst, js, 4) - U1(inst, js, 2) * U1(inst, js, 2);
    mon[11] = U2(avg, js, 4) - U1(avg, js, 2) * U1(avg, js, 2);
    mon[12] = U2(inst, js, 6) - U1(inst, js, 3) * U1(inst, js, 3);
    mon[13] = U2(avg, js, 6) - U1(avg, js, 3) * U1(avg, js, 3);
    mon[14] = (U1(inst, 1, 1) - 0.0) * g.dyfi[1] * 2.0 * 2.0 / ren;
    mon[15] = (U1(avg, 1, 1) - 0.0) * g.dyfi[1] * 2.0 * 2.0 / ren;
    mon[16] = (U1(inst, M, 1) - 0.0) * g.dyfi[M] * 2.0 * 2.0 / ren;
    mon[17] = (U1(avg, M, 1) - 0.0) * g.dyfi[M] * 2.0 * 2.0 / ren;
    mon[18] = mean;
    mon[19] = mx;
}
