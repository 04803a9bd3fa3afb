// Step control and diagnostics:
//   k_cfl        CFL_tg (src/CFL.f90:13-52): per-block maxima of
//                0.5*(|(u_i+u_i+1) DXI| + |(v_j+v_j+1) DYFI| + |(w_k+w_k+1) DZI|)
//   k_dt         BCAST_COMM_STEP (src/SOLVE.f90:154-211):
//                DT = max(min(DT0, 5 DT, CFLGV/CFLMM), DTMIN); flags DT/DT0 < 0.01
//   k_divgck     DIVGCK_tg (src/DIVGCK.f90:15-55): max |div u|
//   k_bc_fields  BC_WALL_Q_tg / BC_WALL_PR_tg ghost planes (src/BC_WALL.f90:212-361)
#pragma once
#include "common.cuh"
#include "momentum.cuh"

#define DG_NT 256

// The field kernels take the stored type R of Q and PR (double, or float in
// the mixed-precision step) and evaluate in FP64.
template <typename R>
__global__ void __launch_bounds__(DG_NT) k_cfl(Geo g, const R* __restrict__ Q, double* __restrict__ partial,
                                               DevState* __restrict__ st) {
    pdl_wait();
    __shared__ double sred[32];
    const int L = g.L, M = g.M, N = g.N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nlines = M * N;
    double mx = 0.0;
    bool bad = false;
    // one warp per x line (j, k): the line's indices are decoded once; each lane
    // reads VW consecutive points of every row with 16-byte loads
    constexpr int VW = V16<R>::W;
    for (int line = blockIdx.x * (DG_NT / 32) + warp; line < nlines; line += gridDim.x * (DG_NT / 32)) {
        const int j = 1 + line % M, k = line / M;
        const long long c0 = pidx(g, 0, j, k);
        const R* U = Q + c0;
        const R* V = Q + g.FS + c0;
        const R* W = Q + 2 * g.FS + c0;
        const R* Wkp = Q + 2 * g.FS + pidx(g, 0, j, wrapp(k, N));
        const double cy = g.dyfi[j];
#pragma unroll 2
        for (int i0 = lane * VW; i0 < L; i0 += 32 * VW) {
            R u[VW], v[VW], vp[VW], w[VW], wp[VW];
            ld16(U + i0, u);
            ld16(V + i0, v);
            ld16(V + i0 + L, vp);
            ld16(W + i0, w);
            ld16(Wkp + i0, wp);
            const double un = U[i0 + VW == L ? 0 : i0 + VW];
#pragma unroll
            for (int e = 0; e < VW; ++e) {
                const double up = e + 1 < VW ? (double)u[e + 1] : un;
                const double q = (fabs(((double)u[e] + up) * g.dxi) +
                                  fabs(((double)v[e] + (double)vp[e]) * cy * 1.0) +
                                  fabs(((double)w[e] + (double)wp[e]) * g.dzi * 1.0)) * 0.5;
                if (!(q == q)) bad = true;
                mx = fmax(mx, q);
            }
        }
    }
    if (bad) atomicOr(&st->err, CHS_EBIT_NAN);
    if (blockIdx.x == 0 && threadIdx.x == 0) st->dtprev = st->dt;
    double r = block_max<DG_NT>(mx, sred);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void __launch_bounds__(DG_NT) k_dt(const double* __restrict__ partial, int np, DevState* __restrict__ st,
                                              int update_dt) {
    pdl_wait();
    __shared__ double sred[32];
    double mx = 0.0;
    for (int t = threadIdx.x; t < np; t += DG_NT) mx = fmax(mx, partial[t]);
    double c = block_max<DG_NT>(mx, sred);
    if (threadIdx.x == 0) {
        st->cflmm = c;
        if (update_dt) {
            double dt = fmin(fmin(st->dt0, 5.0 * st->dt), st->cflgv / c);
            dt = fmax(dt, st->dtmin);
            st->dt = dt;
            if ((dt / st->dt0) < 0.01) atomicOr(&st->err, CHS_EBIT_DT_COLLAPSE);
            if (!(dt == dt)) atomicOr(&st->err, CHS_EBIT_NAN);
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(DG_NT) k_divgck(Geo g, const R* __restrict__ Q, double* __restrict__ partial) {
    __shared__ double sred[32];
    const int L = g.L, M = g.M, N = g.N;
    const long long tot = (long long)L * M * N;
    double mx = 0.0;
    for (long long t = (long long)blockIdx.x * DG_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * DG_NT) {
        int i, j, k;
        io_decode(g, t, i, j, k);
        const long long c = pidx(g, i, j, k);
        const double d = ((double)Q[pidx(g, wrapp(i, L), j, k)] - (double)Q[c]) * g.dxi +
                         ((double)Q[c + g.FS + g.L] - (double)Q[c + g.FS]) * g.dyfi[j] * 1.0 +
                         ((double)Q[pidx(g, i, j, wrapp(k, N)) + 2 * g.FS] - (double)Q[c + 2 * g.FS]) * g.dzi * 1.0;
        mx = fmax(fabs(d), mx);
    }
    double r = block_max<DG_NT>(mx, sred);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void k_maxdiv_final(const double* __restrict__ partial, int np, DevState* __restrict__ st) {
    __shared__ double sred[32];
    double mx = 0.0;
    for (int t = threadIdx.x; t < np; t += DG_NT) mx = fmax(mx, partial[t]);
    double c = block_max<DG_NT>(mx, sred);
    if (threadIdx.x == 0) st->maxdiv = c;
}

// Wall ghost planes after an upload: u = w = 0 at j = 0, M+1; v = 0 at
// j = 0, 1, M+1; PR zero-gradient.
template <typename R>
__global__ void __launch_bounds__(DG_NT) k_bc_fields(Geo g, R* __restrict__ Q, R* __restrict__ PR) {
    const int L = g.L, M = g.M, N = g.N;
    const long long tot = (long long)L * N;
    for (long long t = (long long)blockIdx.x * DG_NT + threadIdx.x; t < tot; t += (long long)gridDim.x * DG_NT) {
        const int i = (int)(t % L), k = (int)(t / L);
        const long long b0 = pidx(g, i, 0, k), b1 = pidx(g, i, 1, k), bm = pidx(g, i, M, k), bt = pidx(g, i, M + 1, k);
        Q[bt] = R(0); Q[bt + 2 * g.FS] = R(0); Q[bt + g.FS] = R(0);
        Q[b0] = R(0); Q[b0 + 2 * g.FS] = R(0); Q[b1 + g.FS] = R(0); Q[b0 + g.FS] = R(0);
        PR[bt] = PR[bm];
        PR[b0] = PR[b1];
    }
}

// Step start of the captured graph: every block reduces the CFL partials
// (order-independent maximum), applies the dt rule of BCAST_COMM_STEP, and
// computes one factor table of one substep (block b: substep 1 + b / 5,
// set b % 5).  Block 0 publishes CFLMM and DT.
template <typename T>
__global__ void __launch_bounds__(32) k_dt_factors(Geo g, const double* __restrict__ partial, int np,
                                                   DevState* __restrict__ st, T* __restrict__ fac) {
    pdl_wait();
    const int lane = threadIdx.x;
    // four independent maxima, so that the partials' loads are in flight together
    double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
    int t = lane;
#pragma unroll 2
    for (; t + 96 < np; t += 128) {
        m0 = fmax(m0, partial[t]);
        m1 = fmax(m1, partial[t + 32]);
        m2 = fmax(m2, partial[t + 64]);
        m3 = fmax(m3, partial[t + 96]);
    }
    for (; t < np; t += 32) m0 = fmax(m0, partial[t]);
    double mx = fmax(fmax(m0, m1), fmax(m2, m3));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const double c = mx;
    double dt = fmin(fmin(st->dt0, 5.0 * st->dtprev), st->cflgv / c);
    dt = fmax(dt, st->dtmin);
    const int ns = 1 + blockIdx.x / 5, set = blockIdx.x % 5;
    factor_set(g, dt, ns, set, fac + (long long)(ns * 5 + set) * FAC_SET, lane);
    __syncwarp();
    if (blockIdx.x == 0 && lane == 0) {
        st->cflmm = c;
        st->dt = dt;
        if ((dt / st->dt0) < 0.01) atomicOr(&st->err, CHS_EBIT_DT_COLLAPSE);
        if (!(dt == dt)) atomicOr(&st->err, CHS_EBIT_NAN);
    }
}

// Element-wise conversion between the FP64 host-facing copies and the FP32
// fields of the mixed-precision step.
template <typename TO, typename FROM>
__global__ void __launch_bounds__(DG_NT) k_convert(TO* __restrict__ dst, const FROM* __restrict__ src, long long n) {
    for (long long t = (long long)blockIdx.x * DG_NT + threadIdx.x; t < n; t += (long long)gridDim.x * DG_NT)
        dst[t] = (TO)src[t];
}
