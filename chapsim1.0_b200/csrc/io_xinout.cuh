// Main domain with inflow and outflow (iDomain = 3: TgFlowFlg and IoFlowFlg), flow
// only, explicit viscous terms: SOLVERRK3_MOM_io with TgFlowFlg
// (src/SOLVERRK3_MOM_IO.f90:11-120).  The rows of every field hold the ghost
// columns 0 and LI + 1 (NCL1S:NCL1E, Geo::xo = 1); the momentum, correction and
// CFL kernels of io.cuh run unchanged on that layout (their x neighbours are the
// ghost columns, and the inlet face u(1) is left alone).  This file holds what is
// specific to the inflow/outflow domain:
//
//   k_xio_inlet      BC_TINLET_FLOW (src/BC_INLET.f90:12-61): the inlet ghost column from
//                    the periodic TG domain's last column, the inlet face u(1) from its first
//   k_xio_outlet_a/b/c  BC_COUTLET_MOM_RK3(NS) (src/BC_COUTLET_MOM_RK3.f90:16-112): U_OUTLET of
//                    CONVCTION_OUTLET_U (:115-192), the convective update of the outlet
//                    column, and the outflow scaling of CHK_MassConsv_io
//                    (src/processing/CHK_conservation.f90:11-79)
//   k_xio_div_cosqf  DIVG_io (src/DIVG.f90:54-137) and FISHPACK's x transform COSQF through one
//                    complex FFT per row (k_xio_div_dctx: as a matrix product, for L that is no
//                    FFT length)
//   k_xio_ysolve     TRID0 (src/possion3d_fishpack.f90:309-340) per (x mode, kz)
//   k_xio_cosqb      COSQB and the 1/(SCALX SCALY) scaling -> DPH (interior; the ghost
//                    columns of DPH stay zero); k_xio_dctx_inv as a matrix product
//   k_xio_divgck     DIVGCK_io with TgFlowFlg (src/DIVGCK.f90:80-84): the three cell ranges
//   k_dt_pair        CFLMM = max(CFLMM_tg, CFLMM_io) and the dt rule (src/SOLVE.f90:79-94)
//
// FISHPACK_POIS3D_SIMPLE with BCX_io = (2, 1) is LPEROD = 4: x(0) = x(2) at the inlet,
// x(L+1) = 0 at the outlet (src/possion3d_fishpack.f90:148-152).  Its x transforms are the
// quarter-wave cosine pair, written here as the sums FFTPACK defines them by
//   COSQF  X(m) = x(1) + sum_{p=2..L} 2 x(p) cos((2m-1)(p-1) pi / (2L))
//   COSQB  x(p) = sum_{m=1..L} 4 X(m) cos((2m-1)(p-1) pi / (2L))
// (a block of rows times the L x L transform matrix, register-tiled: L^2 multiply-adds per
// row).  The z pair
// RFFTF/RFFTB is k_fftz on the real lines held as complex values.  With LPEROD = 4 no x
// root is zero, so no mode is singular and TRID0's zero-pivot branch is not taken.
#pragma once
#include "common.cuh"
#include "io.cuh"
#include "thermal.cuh"

#define XIO_NT 256
#define XD_R 32  // rows (j, k) per block of the cosine transforms
#define XD_RT 8  // rows per thread
#define XD_MT 4  // modes (or points) per thread in one pass: two adjacent pairs

// ---------------------------------------------------------------------------
// BC_TINLET_FLOW: rows j = 0..M+1 of the TG domain's last column (LT - 1) and first
// u face (column 0).  QT, PRT: the TG fields (row stride LT, field size FST).
__global__ void __launch_bounds__(XIO_NT) k_xio_inlet(Geo g, IoFields f, const double* __restrict__ QT,
                                                      const double* __restrict__ PRT, int LT, long long FST) {
    const int M = g.M;
    const long long tot = (long long)(M + 2) * g.N;
    for (long long t = (long long)blockIdx.x * XIO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * XIO_NT) {
        const int j = (int)(t % (M + 2)), k = (int)(t / (M + 2));
        const long long rt = (long long)LT * ((long long)j + (long long)(M + 2) * k);
        const long long cl = rt + LT - 1;
        const long long c0 = pidx(g, 0, j, k), c1 = c0 + 1;
        const double d0 = f.RHO[c0];
        const double u0 = QT[cl], u1 = QT[rt];
        const double v0 = QT[cl + FST], w0 = QT[cl + 2 * FST];
        f.Q[c0] = u0;
        f.Q[c1] = u1;
        f.G[c0] = u0 * d0;
        f.G[c1] = u1 * d0;
        f.Q[c0 + g.FS] = v0;
        f.G[c0 + g.FS] = v0 * d0;
        f.Q[c0 + 2 * g.FS] = w0;
        f.G[c0 + 2 * g.FS] = w0 * d0;
        f.PR[c0] = PRT[cl];
    }
}

// Velocity of the ghost columns at upload: G over the x average of DENSITY0 of the column and
// its interior neighbour (what BC_COUTLET_MOM_RK3 divides the outlet column by), all rows.
__global__ void __launch_bounds__(XIO_NT) k_xio_ghost_velocity(Geo g, IoFields f) {
    const int M = g.M, LI = g.LI;
    const long long tot = 2LL * (M + 2) * g.N;
    for (long long t = (long long)blockIdx.x * XIO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * XIO_NT) {
        const int side = (int)(t & 1);
        const long long r = t >> 1;
        const int j = (int)(r % (M + 2)), k = (int)(r / (M + 2));
        const int ig = side ? LI + 1 : 0, in = side ? LI : 1;
        const long long c = pidx(g, ig, j, k);
        const double rho = (f.RHO[pidx(g, in, j, k)] + f.RHO[c]) * 0.5;
        for (int d = 0; d < 3; ++d) f.Q[c + d * g.FS] = f.G[c + d * g.FS] / rho;
    }
}

// Fill a buffer with a constant (D_STG and MU_STG start at 1, src/MEMALLOCT.f90:200-201)
__global__ void __launch_bounds__(XIO_NT) k_fill(double* __restrict__ p, long long n, double v) {
    for (long long t = (long long)blockIdx.x * XIO_NT + threadIdx.x; t < n; t += (long long)gridDim.x * XIO_NT) p[t] = v;
}

// ---------------------------------------------------------------------------
// BC_COUTLET_MOM_RK3(NS) in three grid-wide passes over the outlet plane (each needs a value
// the previous one reduces over the whole plane); partial results per block, reduced by every
// block in block order (deterministic).  BC0: BC_CONV0(J, K, IDR) as [IDR][K][J]; state[0] =
// U_OUTLET, state[1] = CHK_Mass_CONSV0_SCALING of this substep; part: 2 doubles per block.
// The interior mass rate (sum of DrhoDtP / DYFI) comes from k_drhodt's block sums with the thermal
// solver on, and is zero without it.
//   a: extremes of UCC = (u(L) + u(L+1)) / 2 (CONVCTION_OUTLET_U, method two)
//   b: U_OUTLET = (max + min) / 2, the convective update of the outlet column (:36-58), and
//      the inlet (u face 1) and outlet (u face L+1) fluxes of CHK_MassConsv_io
//   c: the outflow scaling of u(L+1) (:62-72)
__global__ void __launch_bounds__(XIO_NT) k_xio_outlet_a(Geo g, IoFields f, double* __restrict__ part) {
    __shared__ double sred[32];
    const int M = g.M, np = M * g.N, L = g.LI;
    double mx = -1.0E20, mn = 1.0E20;
    for (int p = blockIdx.x * XIO_NT + threadIdx.x; p < np; p += gridDim.x * XIO_NT) {
        const int j = 1 + p % M, k = p / M;
        const long long c = pidx(g, L, j, k);
        const double ucc = (f.Q[c] + f.Q[c + 1]) * 0.5;
        mx = fmax(mx, ucc);
        mn = fmin(mn, ucc);
    }
    const double bmax = block_max<XIO_NT>(mx, sred);
    const double bmin = -block_max<XIO_NT>(-mn, sred);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = bmax;
        part[2 * blockIdx.x + 1] = bmin;
    }
}

__global__ void __launch_bounds__(XIO_NT) k_xio_outlet_b(Geo g, IoFields f, double* __restrict__ BC0,
                                                         const double* __restrict__ parta, double* __restrict__ partb,
                                                         double* __restrict__ state, const DevState* __restrict__ st,
                                                         int ns) {
    __shared__ double sred[32];
    __shared__ double uo;
    if (threadIdx.x == 0) {
        double mx = -1.0E20, mn = 1.0E20;
        for (int b = 0; b < (int)gridDim.x; ++b) {
            mx = fmax(mx, parta[2 * b]);
            mn = fmin(mn, parta[2 * b + 1]);
        }
        uo = 0.5 * (mx + mn);
        if (blockIdx.x == 0) state[0] = uo;
    }
    __syncthreads();
    const int M = g.M, np = M * g.N, L = g.LI;
    const double coe1 = g.dxi * uo;
    const double dt = st->dt, tg = g.tgam[ns], tr = g.troh[ns];
    double fin = 0.0, fout = 0.0;
    for (int p = blockIdx.x * XIO_NT + threadIdx.x; p < np; p += gridDim.x * XIO_NT) {
        const int j = 1 + p % M, k = p / M;
        const long long cr = pidx(g, L, j, k);
        const double rho = (f.RHO[cr] + f.RHO[cr + 1]) * 0.5;
        for (int idr = 0; idr < 3; ++idr) {
            if (idr == 1 && j < 2) continue;  // N2I = 2 for v
            const long long c = cr + idr * g.FS;
            const long long b = (long long)idr * np + (long long)(j - 1) + (long long)M * k;
            const double bc_conv = -(f.G[c + 1] - f.G[c]) * coe1;
            const double bc_rhs = tg * bc_conv + tr * BC0[b];
            BC0[b] = bc_conv;
            const double gn = f.G[c + 1] + dt * bc_rhs;
            f.G[c + 1] = gn;
            f.Q[c + 1] = gn / rho;
        }
        const double coe2 = 1.0 / g.dyfi[j] / 1.0;
        fin += f.G[pidx(g, 1, j, k)] * coe2;
        fout += f.G[cr + 1] * coe2;
    }
    const double bin = block_sum<XIO_NT>(fin, sred);
    const double bout = block_sum<XIO_NT>(fout, sred);
    if (threadIdx.x == 0) {
        partb[2 * blockIdx.x] = bin;
        partb[2 * blockIdx.x + 1] = bout;
    }
}

// mpart, nmp: the per-block sums of DrhoDtP / DYFI of k_drhodt (thermal solver on), else NULL
__global__ void __launch_bounds__(XIO_NT) k_xio_outlet_c(Geo g, IoFields f, const double* __restrict__ partb,
                                                         const double* __restrict__ mpart, int nmp,
                                                         double* __restrict__ state, DevState* __restrict__ st) {
    __shared__ double sc;
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, mr = 0.0;
        for (int q = 0; q < (int)gridDim.x; ++q) {
            a += partb[2 * q];
            b += partb[2 * q + 1];
        }
        if (mpart)
            for (int q = 0; q < nmp; ++q) mr += mpart[q];
        const double flux_in = a / g.dzi, flux_out = b / g.dzi;
        const double mass_rate = mr / g.dzi / g.dxi;
        sc = (flux_in - mass_rate) / flux_out;
        if (blockIdx.x == 0) {
            state[1] = sc;
            if (!(sc == sc) || !(state[0] == state[0])) atomicOr(&st->err, CHS_EBIT_NAN);
        }
    }
    __syncthreads();
    const double scaling = sc;
    const int M = g.M, np = M * g.N, L = g.LI;
    for (int p = blockIdx.x * XIO_NT + threadIdx.x; p < np; p += gridDim.x * XIO_NT) {
        const int j = 1 + p % M, k = p / M;
        const long long c = pidx(g, L + 1, j, k);
        const double go = f.G[c];
        const double gn = go * (scaling - 1.0) + go;
        f.G[c] = gn;
        f.Q[c] = gn / ((f.RHO[c - 1] + f.RHO[c]) * 0.5);
    }
}

// ---------------------------------------------------------------------------
// The cosine transforms are products of a block of rows with one L x L matrix, so a block
// takes XD_R rows (q = (j - 1) + M k) into shared memory and each thread accumulates
// XD_RT rows x XD_MT modes in registers, in the sum's order over p; the matrix entries
// come from global memory (L2-resident: L^2 doubles) and serve the XD_R / XD_RT thread
// groups of the block that share a mode.
//   CF[p L + m] = w_p cos((2m+1) p pi / (2L)), w_0 = 1, w_p = 2     (COSQF: sum over p)
//   CB[m L + p] = 4 cos((2m+1) p pi / (2L))                         (COSQB: sum over m)
// Both are stored summed-index-major, so C[s L + o] pairs summed index s with output index o.
#define XD_MG (XIO_NT / (XD_R / XD_RT))  // threads per row group (64): a pass covers 2 * XD_MG * 2 outputs
// output u (0..3) of thread tm in the pass starting at o0: o0 + 2 tm + (u >> 1) * 2 XD_MG + (u & 1);
// the pairs are 16-byte loads of the matrix row (L is even)
__device__ __forceinline__ int xd_out(int o0, int tm, int u) { return o0 + 2 * tm + (u >> 1) * 2 * XD_MG + (u & 1); }

__device__ __forceinline__ void xd_rows_times_matrix(const double* __restrict__ rows, const double* __restrict__ C,
                                                     int L, int nr, double (&acc)[XD_RT][XD_MT], int m0, int tm, int tr) {
#pragma unroll
    for (int r = 0; r < XD_RT; ++r)
#pragma unroll
        for (int u = 0; u < XD_MT; ++u) acc[r][u] = 0.0;
    for (int p = 0; p < L; ++p) {
        double x[XD_RT], c[XD_MT];
#pragma unroll
        for (int r = 0; r < XD_RT; ++r) {
            const int rr = tr + r * (XD_R / XD_RT);
            x[r] = rr < nr ? rows[rr * L + p] : 0.0;
        }
#pragma unroll
        for (int h = 0; h < XD_MT / 2; ++h) {
            const int m = xd_out(m0, tm, 2 * h);
            double2 cc = make_double2(0.0, 0.0);
            if (m < L) cc = __ldg(reinterpret_cast<const double2*>(C + (long long)p * L + m));
            c[2 * h] = cc.x;
            c[2 * h + 1] = cc.y;
        }
#pragma unroll
        for (int r = 0; r < XD_RT; ++r)
#pragma unroll
            for (int u = 0; u < XD_MT; ++u) acc[r][u] = acc[r][u] + x[r] * c[u];
    }
}

// DIVG_io + COSQF: the row's divergence times 1/(alpha dt) (and 1/wdiv, DIVG.f90:78-82) goes
// to shared memory, then SP[m + L ((j-1) + M k)] = (X(m), 0).
__global__ void __launch_bounds__(XIO_NT, 2) k_xio_div_dctx(Geo g, const double* __restrict__ G, const double* __restrict__ CF,
                                                         double2* __restrict__ SP, const DevState* __restrict__ st,
                                                         int ns, double wdiv, const double* __restrict__ DRHO) {
    extern __shared__ double xsm[];
    const int L = g.LI, M = g.M, N = g.N;
    double* row = xsm;  // XD_R x L
    const long long nrows = (long long)M * N;
    const long long q0 = (long long)blockIdx.x * XD_R;
    const int nr = (int)min((long long)XD_R, nrows - q0);
    const double coe0 = 1.0 / st->dt / g.talp[ns] / wdiv;
    const double coe1 = g.dxi / 1.0;
    for (int p = threadIdx.x; p < nr * L; p += XIO_NT) {
        const int r = p / L, i = 1 + (p - r * L);
        const long long q = q0 + r;
        const int j = 1 + (int)(q % M), k = (int)(q / M);
        const long long c = pidx(g, i, j, k);
        const double u = G[c], up = G[c + 1];
        const double v = G[c + g.FS], vp = G[c + g.FS + g.L];
        const double w = G[c + 2 * g.FS], wp = G[pidx(g, i, j, wrapp(k, N)) + 2 * g.FS];
        const double coe2 = g.dyfi[j] / 1.0;
        const double DIVX = (up - u) * coe1, DIVY = (vp - v) * coe2, DIVZ = (wp - w) * g.dzi;
        const double DQ = DIVX + DIVY + DIVZ + (DRHO ? DRHO[c] / 1.0 : 0.0);
        row[r * L + (i - 1)] = DQ * coe0;
    }
    __syncthreads();
    const int tm = threadIdx.x % XD_MG, tr = threadIdx.x / XD_MG;
    for (int m0 = 0; m0 < L; m0 += XD_MT * XD_MG) {  // XD_MT * XD_MG = 256 outputs per pass
        double acc[XD_RT][XD_MT];
        xd_rows_times_matrix(row, CF, L, nr, acc, m0, tm, tr);
#pragma unroll
        for (int r = 0; r < XD_RT; ++r) {
            const int rr = tr + r * (XD_R / XD_RT);
            if (rr >= nr) continue;
#pragma unroll
            for (int u = 0; u < XD_MT; ++u) {
                const int m = xd_out(m0, tm, u);
                if (m < L) SP[m + (long long)L * (q0 + rr)] = make_double2(acc[r][u], 0.0);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The same pair of transforms through one L-point complex FFT per row when L is an FFT length
// (32, 64, 96, 128, 192, 256, 384), after Makhoul's reordering:
//   COSQF: with c_p = w_p x_p and u_n = sum_p (c_p e^{i pi p / (2L)}) e^{+2 pi i p n / L},
//          X(2n) = Re u_n and X(2n+1) = Re u_{L-1-n}, n < L/2
//          (cos(pi p (4n+1) / (2L)) is the (2m+1) = 4n+1 term; 4(L-1-n)+1 = 4L - (4n+3))
//   COSQB: with v_n = X(2n), v_{L-1-n} = X(2n+1) and V_p = sum_n v_n e^{-2 pi i n p / L},
//          x(p) = 4 Re(e^{-i pi p / (2L)} V_p)
// TQ[p] = (cos, sin)(pi p / (2L)).  XF_TJ rows (j) of one k per block, one FFT line each.
#define XF_TJ 8

template <int N1, int N2>
__global__ void __launch_bounds__(PX_NT) k_xio_div_cosqf(Geo g, const double* __restrict__ G, const double2* __restrict__ TQ,
                                                         double2* __restrict__ SP, const DevState* __restrict__ st,
                                                         int ns, double wdiv, const double* __restrict__ DRHO) {
    extern __shared__ __align__(16) unsigned char xf_raw[];
    double2* smc = reinterpret_cast<double2*>(xf_raw);
    const int L = g.LI, M = g.M, N = g.N;
    const int LD = fft4s_ld(L);
    const int j0 = 1 + blockIdx.x * XF_TJ, k = blockIdx.y;
    const int nj = min(XF_TJ, M - j0 + 1);
    const double coe0 = 1.0 / st->dt / g.talp[ns] / wdiv;
    const double coe1 = g.dxi / 1.0;
    const int kp = wrapp(k, N);
    for (int p = threadIdx.x; p < nj * L; p += PX_NT) {
        const int jl = p / L, i = p - jl * L;
        const int j = j0 + jl;
        const long long c = pidx(g, i + 1, j, k);
        const double u = G[c], up = G[c + 1];
        const double v = G[c + g.FS], vp = G[c + g.FS + g.L];
        const double w = G[c + 2 * g.FS], wp = G[pidx(g, i + 1, j, kp) + 2 * g.FS];
        const double coe2 = g.dyfi[j] / 1.0;
        const double DIVX = (up - u) * coe1, DIVY = (vp - v) * coe2, DIVZ = (wp - w) * g.dzi;
        const double x = (DIVX + DIVY + DIVZ + (DRHO ? DRHO[c] / 1.0 : 0.0)) * coe0;
        const double cw = i == 0 ? x : 2.0 * x;
        const double2 t = TQ[i];
        smc[jl * LD + i] = make_double2(cw * t.x, cw * t.y);
    }
    block_fft4s<N1, N2, +1>(smc, nj, LD, g.twx);
    __syncthreads();
    for (int p = threadIdx.x; p < nj * L; p += PX_NT) {
        const int jl = p / L, m = p - jl * L;
        const int n = (m & 1) ? L - 1 - (m >> 1) : (m >> 1);
        SP[m + (long long)L * ((j0 + jl - 1) + (long long)M * k)] = make_double2(smc[jl * LD + n].x, 0.0);
    }
}

template <int N1, int N2>
__global__ void __launch_bounds__(PX_NT) k_xio_cosqb(Geo g, const double2* __restrict__ SP, const double2* __restrict__ TQ,
                                                     double* __restrict__ DPH) {
    extern __shared__ __align__(16) unsigned char xf_raw[];
    double2* smc = reinterpret_cast<double2*>(xf_raw);
    const int L = g.LI, M = g.M;
    const int LD = fft4s_ld(L);
    const int j0 = 1 + blockIdx.x * XF_TJ, k = blockIdx.y;
    const int nj = min(XF_TJ, M - j0 + 1);
    const int LHf = L / 2;
    for (int p = threadIdx.x; p < nj * L; p += PX_NT) {
        const int jl = p / L, n = p - jl * L;
        const int m = n < LHf ? 2 * n : 2 * (L - 1 - n) + 1;
        smc[jl * LD + n] = make_double2(SP[m + (long long)L * ((j0 + jl - 1) + (long long)M * k)].x, 0.0);
    }
    block_fft4s<N1, N2, -1>(smc, nj, LD, g.twx);
    __syncthreads();
    const double q4 = (double)(4 * L);
    for (int p = threadIdx.x; p < nj * L; p += PX_NT) {
        const int jl = p / L, pp = p - jl * L;
        const double2 V = smc[jl * LD + pp], t = TQ[pp];
        const double y = V.x * t.x + V.y * t.y;
        DPH[pidx(g, pp + 1, j0 + jl, k)] = 4.0 * y / q4;
    }
}

// TRID0 for every (x mode m, kz) line: BB(j) = ACPH(j) + XRT(m) + YRT(kz) with XRT = -ak1[m],
// YRT = -ak3[kz]; A = AMPH, C = APPH.  D holds the forward factors (M per line, line-major
// across threads).  Complex right-hand side: the real and imaginary lines share D.  Each
// sweep loads XY_U rows ahead of the recurrence (the loads do not wait for the previous
// row's store), so a line costs one memory latency per XY_U rows.
#define XY_U 8
__global__ void __launch_bounds__(XIO_NT) k_xio_ysolve(Geo g, double2* __restrict__ SP, double* __restrict__ D) {
    const int L = g.LI, M = g.M, N = g.N;
    const long long nl = (long long)L * N;
    const long long ln = (long long)blockIdx.x * XIO_NT + threadIdx.x;
    if (ln >= nl) return;
    const int m = (int)(ln % L), kz = (int)(ln / L);
    const double xrt = -g.ak1[m], yrt = -g.ak3[kz];
    const long long stride = L;  // element j of the line: m + L ((j - 1) + M kz)
    double2* S = SP + m + (long long)L * M * kz;
    double* Dl = D + ln;          // element j - 1 at Dl[(j - 1) * nl]
    double bb = g.acph[1] + xrt / 1.0 + yrt;
    double z = 1.0 / bb;
    double d = g.apph[1] * z;
    Dl[0] = d;
    double2 t = S[0];
    t.x = t.x * z;
    t.y = t.y * z;
    S[0] = t;
    for (int j0 = 2; j0 <= M - 1; j0 += XY_U) {
        double2 rr[XY_U];
#pragma unroll
        for (int u = 0; u < XY_U; ++u)
            if (j0 + u <= M - 1) rr[u] = S[(long long)(j0 + u - 1) * stride];
#pragma unroll
        for (int u = 0; u < XY_U; ++u) {
            const int j = j0 + u;
            if (j > M - 1) break;
            bb = g.acph[j] + xrt / 1.0 + yrt;
            z = 1.0 / (bb - g.amph[j] * d);
            d = g.apph[j] * z;
            Dl[(long long)(j - 1) * nl] = d;
            double2 r = rr[u];
            r.x = (r.x - g.amph[j] * t.x) * z;
            r.y = (r.y - g.amph[j] * t.y) * z;
            S[(long long)(j - 1) * stride] = r;
            t = r;
        }
    }
    bb = g.acph[M] + xrt / 1.0 + yrt;
    z = bb - g.amph[M] * d;
    double2 r = S[(long long)(M - 1) * stride];
    if (fabs(z) > 1.0E-14) {
        r.x = (r.x - g.amph[M] * t.x) / z;
        r.y = (r.y - g.amph[M] * t.y) / z;
    } else {
        r = make_double2(0.0, 0.0);
    }
    S[(long long)(M - 1) * stride] = r;
    for (int j0 = M - 1; j0 >= 1; j0 -= XY_U) {
        double2 ss[XY_U];
        double dd[XY_U];
#pragma unroll
        for (int u = 0; u < XY_U; ++u)
            if (j0 - u >= 1) {
                ss[u] = S[(long long)(j0 - u - 1) * stride];
                dd[u] = Dl[(long long)(j0 - u - 1) * nl];
            }
#pragma unroll
        for (int u = 0; u < XY_U; ++u) {
            const int j = j0 - u;
            if (j < 1) break;
            double2 sv = ss[u];
            sv.x = sv.x - dd[u] * r.x;
            sv.y = sv.y - dd[u] * r.y;
            S[(long long)(j - 1) * stride] = sv;
            r = sv;
        }
    }
}

// COSQB of the real parts and the scaling 1/(4 L) (the 1/N is the forward z transform's):
// DPH(p, j, k) for the interior columns p = 1..L.
__global__ void __launch_bounds__(XIO_NT, 2) k_xio_dctx_inv(Geo g, const double2* __restrict__ SP, const double* __restrict__ CB,
                                                         double* __restrict__ DPH) {
    extern __shared__ double xsm[];
    const int L = g.LI, M = g.M, N = g.N;
    double* row = xsm;  // XD_R x L
    const long long nrows = (long long)M * N;
    const long long q0 = (long long)blockIdx.x * XD_R;
    const int nr = (int)min((long long)XD_R, nrows - q0);
    for (int p = threadIdx.x; p < nr * L; p += XIO_NT) {
        const int r = p / L, m = p - r * L;
        row[r * L + m] = SP[m + (long long)L * (q0 + r)].x;
    }
    __syncthreads();
    const int tm = threadIdx.x % XD_MG, tr = threadIdx.x / XD_MG;
    const double q4 = (double)(4 * L);
    for (int p0 = 0; p0 < L; p0 += XD_MT * XD_MG) {
        double acc[XD_RT][XD_MT];
        xd_rows_times_matrix(row, CB, L, nr, acc, p0, tm, tr);
#pragma unroll
        for (int r = 0; r < XD_RT; ++r) {
            const int rr = tr + r * (XD_R / XD_RT);
            if (rr >= nr) continue;
            const long long q = q0 + rr;
            const int j = 1 + (int)(q % M), k = (int)(q / M);
#pragma unroll
            for (int u = 0; u < XD_MT; ++u) {
                const int pp = xd_out(p0, tm, u);
                if (pp < L) DPH[pidx(g, pp + 1, j, k)] = acc[r][u] / q4;
            }
        }
    }
    (void)N;
}

// DIVGCK_io with TgFlowFlg: max |div G + DrhoDtP| over the cells 2..L-1, 0..1 and L (DRHO NULL
// without the thermal solver).
// partial[3 b + r] holds block b's maximum of range r.
__global__ void __launch_bounds__(XIO_NT) k_xio_divgck(Geo g, const double* __restrict__ G, const double* __restrict__ DRHO,
                                                       double* __restrict__ partial) {
    __shared__ double sred[32];
    const int L = g.LI, M = g.M, N = g.N;
    const long long tot = (long long)(L + 1) * M * N;  // cells i = 0..L
    double mx[3] = {0.0, 0.0, 0.0};
    for (long long t = (long long)blockIdx.x * XIO_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * XIO_NT) {
        const int i = (int)(t % (L + 1));
        const long long rq = t / (L + 1);
        const int j = 1 + (int)(rq % M), k = (int)(rq / M);
        const long long c = pidx(g, i, j, k);
        const double DIVX = (G[c + 1] - G[c]) * g.dxi;
        const double DIVY = (G[c + g.FS + g.L] - G[c + g.FS]) * (g.dyfi[j] * 1.0);
        const double DIVZ = (G[pidx(g, i, j, wrapp(k, N)) + 2 * g.FS] - G[c + 2 * g.FS]) * (g.dzi * 1.0);
        const double a = fabs(DIVX + DIVY + DIVZ + (DRHO && i >= 1 ? DRHO[c] : 0.0));  // DrhoDtP of the interior
        const int r = (i >= 2 && i <= L - 1) ? 0 : (i <= 1 ? 1 : 2);
        mx[r] = fmax(mx[r], a);
    }
    for (int r = 0; r < 3; ++r) {
        const double b = block_max<XIO_NT>(mx[r], sred);
        if (threadIdx.x == 0) partial[3 * blockIdx.x + r] = b;
    }
}

// The dt of a TG + main-domain step: CFLMM = max(CFLMM_tg, CFLMM_io) (src/SOLVE.f90:79-86),
// then BCAST_COMM_STEP's rule on the main domain's DT0, DTMIN, CFLGV; DT goes to both states.
__global__ void k_dt_pair(DevState* __restrict__ tg, DevState* __restrict__ io) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double c = fmax(tg->cflmm, io->cflmm);
    double dt = fmin(fmin(io->dt0, 5.0 * io->dt), io->cflgv / c);
    dt = fmax(dt, io->dtmin);
    io->cflmm = c;
    io->dtprev = io->dt;
    tg->dtprev = tg->dt;
    io->dt = dt;
    tg->dt = dt;
    if ((dt / io->dt0) < 0.01) atomicOr(&io->err, CHS_EBIT_DT_COLLAPSE);
    if (!(dt == dt)) atomicOr(&io->err, CHS_EBIT_NAN);
}

// ---------------------------------------------------------------------------
// Thermal inflow/outflow.  The inlet state (BC_TINLET_THERML, src/BC_INLET.f90:64-84):
// v = T, H, D, M, K, CP, DH of the inlet (src/Flow_State.f90:44-50).
struct XioInlet {
    double v[7];
};

// The inlet ghost column, rows 0..M+1 (DENSITY0 and Viscousity0 keep the previous values, the
// whole-field copies at the top of SOLVERRK3_ENG_io)
__global__ void __launch_bounds__(XIO_NT) k_xio_thermal_inlet(Geo g, IoFields f, ThermoFields t, XioInlet in) {
    const long long tot = (long long)(g.M + 2) * g.N;
    for (long long q = (long long)blockIdx.x * XIO_NT + threadIdx.x; q < tot; q += (long long)gridDim.x * XIO_NT) {
        const int j = (int)(q % (g.M + 2)), k = (int)(q / (g.M + 2));
        const long long p = pidx(g, 0, j, k);
        f.RHO[p] = f.DEN[p];
        f.MU0[p] = f.MU[p];
        t.TEMP[p] = in.v[0];
        t.KAP[p] = in.v[4];
        f.DEN[p] = in.v[2];
        f.MU[p] = in.v[3];
        t.HCP[p] = in.v[5];
        t.DH[p] = in.v[6];
        t.ENTH[p] = in.v[1];
    }
}

// BC_COUTLET_ENEG_RK3(NS) (src/BC_COUTLET_ENEG_RK3.f90:11-59): U_OUTLET from the extremes of
// k_xio_outlet_a (on the current velocity), the convective RK3 update of the outlet column's
// rho*h with BC_CONV0_ENG (BC0E, [K][J]), the table limiter, THERM_PROP_UPDATE(IOULET) on rows
// 1..M of column L+1
__global__ void __launch_bounds__(PROP_NT) k_xio_energy_outlet(PropTab tb, Geo g, IoFields f, ThermoFields t,
                                                               ThermoParams tp, const double* __restrict__ parta,
                                                               int npa, double* __restrict__ BC0E, DevState* st,
                                                               int ns) {
    __shared__ double uo;
    if (threadIdx.x == 0) {
        double mx = -1.0E20, mn = 1.0E20;
        for (int b = 0; b < npa; ++b) {
            mx = fmax(mx, parta[2 * b]);
            mn = fmin(mn, parta[2 * b + 1]);
        }
        uo = 0.5 * (mx + mn);
    }
    __syncthreads();
    const int M = g.M, np = M * g.N, L = g.LI;
    const double dt = st->dt, tg = g.tgam[ns], tr = g.troh[ns];
    for (int p = blockIdx.x * PROP_NT + threadIdx.x; p < np; p += gridDim.x * PROP_NT) {
        const int j = 1 + p % M, k = p / M;
        const long long c = pidx(g, L, j, k), co = c + 1;
        const double bc_conv = -g.dxi * uo * (t.DH[co] - t.DH[c]);
        const double bc_rhs = tg * bc_conv + tr * BC0E[p];
        BC0E[p] = bc_conv;
        double d = t.DH[co] + dt * bc_rhs;
        d = fmin(tp.dhmax - 1.0e-14, d);
        d = fmax(tp.dhmin + 1.0e-14, d);
        t.DH[co] = d;
        eng_point(tb, tb.xdh, tb.xh, f, t, co, st);
    }
}

// Properties of the inlet and outlet columns (rows 1..M) from their rho*h, at the thermal start
__global__ void __launch_bounds__(PROP_NT) k_xio_ghost_props(PropTab tb, Geo g, IoFields f, ThermoFields t, DevState* st) {
    const int M = g.M, np = M * g.N;
    for (int q = blockIdx.x * PROP_NT + threadIdx.x; q < 2 * np; q += gridDim.x * PROP_NT) {
        const int side = q >= np, p = side ? q - np : q;
        const int j = 1 + p % M, k = p / M;
        eng_point(tb, tb.xdh, tb.xh, f, t, pidx(g, side ? g.LI + 1 : 0, j, k), st);
    }
}
