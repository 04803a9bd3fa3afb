// On-device statistics of the main domain: the x-z plane means of
// PP_MEAN_ZX_FLOW_Xperiodic_io (src/processing/PP_MEAN_ZX.f90:311-796) for the
// plane channel (RCCI1 = RNDI1 = 1; the pipe-centre branch does not apply),
// so that the thermal path needs no per-step download of G, Q and the
// thermal fields.
//
// Per point (I, J, K), with the reference's cell-centred values
//   G_CCT, U_CCT (face pairs times 0.5), the gradients DVDL_CCT(m, n), and
//   with the thermal solver dHdL_CCT, dTdL_CCT (central differences),
// the sums of :431-757 are accumulated over the row's x-z plane, then scaled
// by VL1313_io (:762-805).  Every per-point product keeps the reference's
// left-to-right order; the plane sums are taken in a fixed tree order
// (per-thread partials, warps, chunks in index order) instead of the I, K
// loop, so they agree with the oracle to rounding.
//
// One set is NIO*M doubles, Fortran order with j fastest, the module arrays
// in the order the reference zeroes them (:337-381):
//   U1xzL_io(M,4) | G1xzL_io(M,3) | UPxzL_io(M,3) | U2xzL_io(M,6) | UGxzL_io(M,6) |
//   U3xzL_io(M,10) | UGUxzL_io(M,10) | DVDL1xzL_io(M,3,3) | DVDLPxzL_io(M,3,3) |
//   DVDL2xzL_io(M,9,9)                                                   (141)
// and with the thermal solver
//   T1 | D1 | H1 | M1 | T2 | D2 | H2 | DH | PH (xzL_io(M) each) | DVDL1MxzL_io(M,3,3) |
//   DVDL1MHxzL_io(M,3,3) | DVDL1MUxzL_io(M,3,3,3) | DVDL2MxzL_io(M,9,9) | UHxzL_io(M,3) |
//   GHxzL_io(M,3) | U2DHxzL_io(M,6) | DhDL1xzL_io(M,3) | DhDLPxzL_io(M,3) | DTDLKxzL_io(M,3) |
//   DTDLKUxzL_io(M,3,3) | DTDLKDVDLxzL_io(M,3,3,3) | DHDLMDVDLxzL_io(M,3,3,3)   (219 more).
// The sums are taken in seven groups of at most 60 per thread (registers),
// one launch per group: 0 the first flow moments, 1 the 45 distinct products
// of DVDL2 (symmetric), 2 the thermal moments, 3-5 the three 27-entry
// gradient correlations, 6 the 45 distinct products of DVDL2M.
#pragma once
#include "common.cuh"
#include "io.cuh"
#include "thermal.cuh"
#include "stats.cuh"

#define PPIO_FLOW 141
#define PPIO_ALL 360

__host__ __device__ constexpr int ppio_nacc(int grp) {
    return grp == 0 ? 60 : grp == 1 ? 45 : grp == 2 ? 57 : grp <= 5 ? 27 : 45;
}

template <int GRP, typename F>
__global__ void __launch_bounds__(PP_NT) k_pp_io(Geo g, IoFieldsT<F> f, ThermoFields t, double* __restrict__ part) {
    constexpr int NA = ppio_nacc(GRP);
    const int L = g.L, N = g.N;
    const int j = 1 + blockIdx.y;
    const int jp = j + 1, jm = j - 1;
    const double dycij = g.dyci[j], dycip = g.dyci[jp], dyfij = g.dyfi[j];
    const double dxi = g.dxi, dzi = g.dzi;
    const F* U = f.Q;
    const F* V = f.Q + g.FS;
    const F* W = f.Q + 2 * g.FS;
    const F* GU = f.G;
    const F* GV = f.G + g.FS;
    const F* GW = f.G + 2 * g.FS;
    double a[NA];
#pragma unroll
    for (int q = 0; q < NA; ++q) a[q] = 0.0;
    const int plane = L * N;
    for (int tt = blockIdx.x * PP_NT + threadIdx.x; tt < plane; tt += gridDim.x * PP_NT) {
        const int k = tt / L, i = tt - k * L;
        const int ip = wrapp(i, L), im = wrapm(i, L), kp = wrapp(k, N), km = wrapm(k, N);
        auto q = [&](const F* A, int ii, int jj, int kk) { return (double)A[pidx(g, ii, jj, kk)]; };
        auto d3 = [&](const double* A, int ii, int jj, int kk) { return A[pidx(g, ii, jj, kk)]; };
        double u[3], gc[3], ujp[3], ujm[3], ukp[3], ukm[3], uip[3], uim[3];
        gc[0] = (q(GU, i, j, k) + q(GU, ip, j, k)) * 0.5;
        u[0] = (q(U, i, j, k) + q(U, ip, j, k)) * 0.5;
        ujp[0] = (q(U, i, jp, k) + q(U, ip, jp, k)) * 0.5;
        ujm[0] = (q(U, i, jm, k) + q(U, ip, jm, k)) * 0.5;
        ukp[0] = (q(U, i, j, kp) + q(U, ip, j, kp)) * 0.5;
        ukm[0] = (q(U, i, j, km) + q(U, ip, j, km)) * 0.5;
        gc[2] = ((q(GW, i, j, k) + q(GW, i, j, kp)) * 1.0) * 0.5;
        u[2] = ((q(W, i, j, k) + q(W, i, j, kp)) * 1.0) * 0.5;
        uip[2] = ((q(W, ip, j, k) + q(W, ip, j, kp)) * 1.0) * 0.5;
        uim[2] = ((q(W, im, j, k) + q(W, im, j, kp)) * 1.0) * 0.5;
        ujp[2] = ((q(W, i, jp, k) + q(W, i, jp, kp)) * 1.0) * 0.5;
        ujm[2] = ((q(W, i, jm, k) + q(W, i, jm, kp)) * 1.0) * 0.5;
        gc[1] = ((q(GV, i, j, k) + q(GV, i, jp, k)) * 1.0) * 0.5;
        u[1] = ((q(V, i, j, k) + q(V, i, jp, k)) * 1.0) * 0.5;
        uip[1] = ((q(V, ip, j, k) + q(V, ip, jp, k)) * 1.0) * 0.5;
        uim[1] = ((q(V, im, j, k) + q(V, im, jp, k)) * 1.0) * 0.5;
        ukp[1] = ((q(V, i, j, kp) + q(V, i, jp, kp)) * 1.0) * 0.5;
        ukm[1] = ((q(V, i, j, km) + q(V, i, jp, km)) * 1.0) * 0.5;
        const double p = q(f.PR, i, j, k);
        // DVDL_CCT(m, n), m-major (:508-535)
        double d[9];
        d[0] = (q(U, ip, j, k) - q(U, i, j, k)) * dxi;
        d[2] = (ukp[0] - ukm[0]) * dzi * 0.5;
        d[1] = ((ujp[0] - u[0]) * dycip + (u[0] - ujm[0]) * dycij) * 0.5;
        d[3] = (uip[1] - uim[1]) * dxi * 0.5;
        d[5] = (ukp[1] - ukm[1]) * dzi * 0.5;
        d[4] = (q(V, i, jp, k) * 1.0 - q(V, i, j, k) * 1.0) * dyfij;
        d[8] = (q(W, i, j, kp) * 1.0 - q(W, i, j, k) * 1.0) * dzi;
        d[6] = (uip[2] - uim[2]) * dxi * 0.5;
        d[7] = ((ujp[2] - u[2]) * dycip + (u[2] - ujm[2]) * dycij) * 0.5;
        if constexpr (GRP == 0) {
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                a[m] += u[m];
                a[4 + m] += gc[m];
                a[7 + m] += u[m] * p;
            }
            a[3] += p;
            // U2 and UG: upper triangle in storage order L = m(7-m)/2 + n - 3
            int l = 0;
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int n = m; n < 3; ++n, ++l) {
                    a[10 + l] += u[m] * u[n];
                    a[16 + l] += u[m] * gc[n];
                }
            // U3 and UGU: storage order L = m(6-m) + n(7-n)/2 + h - 8
            l = 0;
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int n = m; n < 3; ++n)
#pragma unroll
                    for (int h = n; h < 3; ++h, ++l) {
                        a[22 + l] += u[m] * u[n] * u[h];
                        a[32 + l] += u[m] * gc[n] * u[h];
                    }
#pragma unroll
            for (int e = 0; e < 9; ++e) {
                a[42 + e] += d[e];
                a[51 + e] += d[e] * p;
            }
        } else if constexpr (GRP == 1) {
#pragma unroll
            for (int x = 0; x < 9; ++x)
#pragma unroll
                for (int y = x; y < 9; ++y) a[pp_sym(x, y)] += d[x] * d[y];
        } else {
            const double tc = d3(t.TEMP, i, j, k), dc = f.DEN[pidx(g, i, j, k)], hc = d3(t.ENTH, i, j, k);
            const double muc = f.MU[pidx(g, i, j, k)], kc = d3(t.KAP, i, j, k);
            double hdl[3], tdl[3];
            hdl[0] = (d3(t.ENTH, ip, j, k) - d3(t.ENTH, im, j, k)) * dxi * 0.5;
            hdl[2] = (d3(t.ENTH, i, j, kp) - d3(t.ENTH, i, j, km)) * dzi * 0.5;
            hdl[1] = ((d3(t.ENTH, i, jp, k) - d3(t.ENTH, i, j, k)) * dycip +
                      (d3(t.ENTH, i, j, k) - d3(t.ENTH, i, jm, k)) * dycij) * 0.5;
            tdl[0] = (d3(t.TEMP, ip, j, k) - d3(t.TEMP, im, j, k)) * dxi * 0.5;
            tdl[2] = (d3(t.TEMP, i, j, kp) - d3(t.TEMP, i, j, km)) * dzi * 0.5;
            tdl[1] = ((d3(t.TEMP, i, jp, k) - d3(t.TEMP, i, j, k)) * dycip +
                      (d3(t.TEMP, i, j, k) - d3(t.TEMP, i, jm, k)) * dycij) * 0.5;
            if constexpr (GRP == 2) {
                a[0] += tc; a[1] += dc; a[2] += hc; a[3] += muc;
                a[4] += tc * tc; a[5] += dc * dc; a[6] += hc * hc;
                a[7] += hc * dc;
                a[8] += hc * p;
#pragma unroll
                for (int e = 0; e < 9; ++e) {
                    a[9 + e] += d[e] * muc;
                    a[18 + e] += d[e] * muc * hc;
                }
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    a[27 + m] += hc * u[m];
                    a[30 + m] += hc * gc[m];
                    a[39 + m] += hdl[m];
                    a[42 + m] += hdl[m] * p;
                    a[45 + m] += tdl[m] * kc;
#pragma unroll
                    for (int n = 0; n < 3; ++n) a[48 + 3 * m + n] += tdl[m] * kc * u[n];
                }
                int l = 0;
#pragma unroll
                for (int m = 0; m < 3; ++m)
#pragma unroll
                    for (int n = m; n < 3; ++n, ++l) a[33 + l] += dc * hc * u[m] * u[n];
            } else if constexpr (GRP == 3) {
                // DVDL1MU(m, n, h) = DVDL(m, n) MU U(h): accumulator 9 h + 3 m + n
#pragma unroll
                for (int e = 0; e < 9; ++e)
#pragma unroll
                    for (int h = 0; h < 3; ++h) a[9 * h + e] += d[e] * muc * u[h];
            } else if constexpr (GRP == 4) {
                // DTDLKDVDL(m, n, h) = dTdL(m) K DVDL(n, h): accumulator 9 m + 3 n + h
#pragma unroll
                for (int m = 0; m < 3; ++m)
#pragma unroll
                    for (int e = 0; e < 9; ++e) a[9 * m + e] += tdl[m] * kc * d[e];
            } else if constexpr (GRP == 5) {
                // DHDLMDVDL(m, n, h) = dHdL(m) MU DVDL(n, h): accumulator 9 m + 3 n + h
#pragma unroll
                for (int m = 0; m < 3; ++m)
#pragma unroll
                    for (int e = 0; e < 9; ++e) a[9 * m + e] += hdl[m] * muc * d[e];
            } else {
#pragma unroll
                for (int x = 0; x < 9; ++x)
#pragma unroll
                    for (int y = x; y < 9; ++y) a[pp_sym(x, y)] += d[x] * d[y] * muc;
            }
        }
    }
    // block reduction: warp shuffles, then the warps in index order
    __shared__ double sw[PP_NT / 32][NA];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q2 = 0; q2 < NA; ++q2) {
        double v = a[q2];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sw[warp][q2] = v;
    }
    __syncthreads();
    for (int q2 = threadIdx.x; q2 < NA; q2 += PP_NT) {
        double s = 0.0;
        for (int w = 0; w < PP_NT / 32; ++w) s += sw[w][q2];
        part[((size_t)(j - 1) * gridDim.x + blockIdx.x) * NA + q2] = s;
    }
}

// The row's chunks in chunk order, scaled by VL1313_io, into the set's layout.
template <int GRP>
__global__ void __launch_bounds__(PP_NT) k_pp_io_finish(Geo g, const double* __restrict__ part, int nchunk,
                                                        double* __restrict__ out) {
    constexpr int NA = ppio_nacc(GRP);
    __shared__ double s[NA];
    const int M = g.M;
    const int j = 1 + blockIdx.x;
    const double VL = 1.0 / (double)(g.L * g.N);
    for (int q = threadIdx.x; q < NA; q += PP_NT) {
        double v = 0.0;
        for (int c = 0; c < nchunk; ++c) v += part[((size_t)(j - 1) * nchunk + c) * NA + q];
        s[q] = v * VL;
    }
    __syncthreads();
    const int r = j - 1;
    auto put = [&](int slot, double v) { out[(size_t)slot * M + r] = v; };
    const int tid = threadIdx.x;
    if constexpr (GRP == 0) {
        // U1(4) G1(3) UP(3) U2(6) UG(6) U3(10) UGU(10) at slots 0..41; accumulators in the same order
        // except U1: u (0..2), p (3); G1 at 4..6; UP at 7..9
        if (tid < 42) put(tid, s[tid]);
        if (tid < 9) {
            // DVDL1xzL(j, m, n) at slot 42 + m + 3 n, DVDLP at 51 + m + 3 n; accumulator e = 3 m + n
            const int m = tid / 3, n = tid % 3;
            put(42 + m + 3 * n, s[42 + tid]);
            put(51 + m + 3 * n, s[51 + tid]);
        }
    } else if constexpr (GRP == 1 || GRP == 6) {
        const int base = GRP == 1 ? 60 : PPIO_FLOW + 9 + 9 + 9 + 27;
        for (int e = tid; e < 81; e += PP_NT) {
            const int l1 = e % 9, l2 = e / 9;
            const int x = l1 < l2 ? l1 : l2, y = l1 < l2 ? l2 : l1;
            put(base + l1 + 9 * l2, s[pp_sym(x, y)]);
        }
    } else if constexpr (GRP == 2) {
        const int b = PPIO_FLOW;
        if (tid < 9) put(b + tid, s[tid]);  // T1 D1 H1 M1 T2 D2 H2 DH PH
        if (tid < 9) {
            const int m = tid / 3, n = tid % 3;
            put(b + 9 + m + 3 * n, s[9 + tid]);        // DVDL1M
            put(b + 18 + m + 3 * n, s[18 + tid]);      // DVDL1MH
            put(b + 135 + 21 + m + 3 * n, s[48 + tid]);  // DTDLKU(m, n), after UH GH U2DH DhDL1 DhDLP DTDLK
        }
        // after DVDL1MU (27) and DVDL2M (81): UH(3) GH(3) U2DH(6) DhDL1(3) DhDLP(3) DTDLK(3)
        const int c = b + 27 + 27 + 81;
        if (tid < 3) {
            put(c + tid, s[27 + tid]);
            put(c + 3 + tid, s[30 + tid]);
            put(c + 12 + tid, s[39 + tid]);
            put(c + 15 + tid, s[42 + tid]);
            put(c + 18 + tid, s[45 + tid]);
        }
        if (tid < 6) put(c + 6 + tid, s[33 + tid]);
    } else if constexpr (GRP == 3) {
        // DVDL1MU(m, n, h) at slot m + 3 n + 9 h; accumulator 9 h + 3 m + n
        for (int e = tid; e < 27; e += PP_NT) {
            const int h = e / 9, m = (e % 9) / 3, n = e % 3;
            put(PPIO_FLOW + 27 + m + 3 * n + 9 * h, s[e]);
        }
    } else {
        // DTDLKDVDL (GRP 4) and DHDLMDVDL (GRP 5) (m, n, h) at slot m + 3 n + 9 h; accumulator 9 m + 3 n + h
        const int base = PPIO_FLOW + 27 + 27 + 81 + 21 + 9 + (GRP == 5 ? 27 : 0);
        for (int e = tid; e < 27; e += PP_NT) {
            const int m = e / 9, n = (e % 9) / 3, h = e % 3;
            put(base + m + 3 * n + 9 * h, s[e]);
        }
    }
}
