// Crank-Nicolson sweeps of the main-domain momentum step (iVisScheme = 1):
// MOMFA_io(NS, IDR) (src/MOMFA_io.f90:18-406) for the three components at
// once, after k_io_rhs<true> has formed the right-hand sides.
//
//   k_io_cn_xsweep<S>  MOMFA1_X_io (:79-172): cyclic in x, per-point
//                      coefficients; subtracts the bulk forcing DPGRNS from the
//                      u right-hand side on load (RHS_MOM_EXPLICIT_io.f90:228-265)
//   k_io_cn_zsweep<S>  MOMFA2_Z_io (:175-261): cyclic in z
//   k_io_cn_ysweep<S>  MOMFA3_Y_io (:264-406): non-cyclic in y with the wall
//                      rows of the u and w equations built from AMVR1 / APVRN
//                      and the half-sum of the cell and ghost viscosity; then
//                      G += RHS for j >= N2I (:38-44)
//
// The operator of component IDR is (1 - A) dG with A's rows
// (amu/rho_m, -(amu+apu)/rho_c, apu/rho_p): it acts on dG/rho.  The
// viscosities are Viscousity (cell), MU_STG (edges, from Viscousity0) and the
// densities D_STG of the component, all fixed during the substep.  Each
// coefficient is evaluated with the reference's operand order.  Two details
// of the reference are kept: the v rows divide the coupling to row j+1 by
// D_STG at row j, and the v row j = 1 (the wall face) is the identity with a
// zero right-hand side (AMVR(1,2) = APVR(1,2) = 0; its sweeps in x and z are
// skipped, N2I = 2), so its value stays 0 and the G update starts at j = 2.
//
// One warp solves one line held in shared memory (warp_tdma of tdma.cuh:
// per-lane Thomas on segments of S rows, PCR over the 32 lanes).  A block
// holds CN_LINES lines.  x lines are contiguous in memory; for z and y the
// block's lines are CN_LINES consecutive i at one (j) or (k), so each global
// row access covers CN_LINES consecutive doubles.
#pragma once
#include "common.cuh"
#include "tdma.cuh"
#include "io.cuh"

#define CN_LINES 8
#define CN_NT (CN_LINES * 32)

template <int S>
struct SegCoef {  // coefficients stored at the segment-padded positions of tdma.cuh
    const double *a, *b, *c;
    __device__ __forceinline__ double A(int r) const { return a[seg_pos<S>(r)]; }
    __device__ __forceinline__ double B(int r) const { return b[seg_pos<S>(r)]; }
    __device__ __forceinline__ double C(int r) const { return c[seg_pos<S>(r)]; }
};

// One block: CN_LINES lines x (a, b, c, d) x 32 (S+1) doubles, each line's
// region padded by 2 doubles (stride 4 SEG + 2): the z and y loads write row
// r of the block's 8 lines from consecutive threads, and an unpadded stride
// (a multiple of 32 words) put all 8 on one bank.
__host__ __device__ constexpr int cn_line_stride(int seg) { return 4 * seg + 2; }
inline size_t smem_cn(int n) { return (size_t)CN_LINES * cn_line_stride(32 * (n / 32 + 1)) * sizeof(double); }

// DPGRNS of RHS_MOM_EXPLICIT_io (:231-263)
__device__ __forceinline__ double cn_dpgrns(const Geo& g, const DevState* st, int ns) {
    if (g.iflowdriven == 1) return st->bulksum / g.volm;
    if (g.iflowdriven == 2) return -0.5 * g.cf_given * (g.talp[ns] * st->dt);
    return 0.0;
}

// x lines (j, k); component blockIdx.y (0 u, 1 v, 2 w)
template <int S, typename F>
__global__ void __launch_bounds__(CN_NT, 3) k_io_cn_xsweep(Geo g, IoFieldsT<F> f, const DevState* __restrict__ st, int ns) {
    extern __shared__ double smx[];
    constexpr int SEG = 32 * (S + 1);
    const int L = g.L, M = g.M;
    const int comp = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long line = (long long)blockIdx.x * CN_LINES + warp;
    if (line >= (long long)M * g.N) return;  // whole warp; no block barrier below
    const int j = 1 + (int)(line % M), k = (int)(line / M);
    if (comp == 1 && j == 1) return;
    double* a = smx + (size_t)warp * cn_line_stride(SEG);
    double* b = a + SEG;
    double* c = b + SEG;
    double* d = c + SEG;
    const double fac = 0.50 * g.talp[ns] * st->dt * g.cvisc;
    const double coe1 = fac * 4.0 / 3.0 * g.dxqi, coe2 = fac * g.dxqi;
    const double dpg = comp == 0 ? cn_dpgrns(g, st, ns) : 0.0;
    const F* D = f.DST + comp * g.FS;
    const F* ms = f.MST + (comp == 1 ? 0 : g.FS);
    F* R = f.RHS + comp * g.FI;
#pragma unroll 4  // several rows' coefficient loads in flight
    for (int i = lane; i < L; i += 32) {
        const int im = wrapm(i, L), ip = wrapp(i, L);
        const long long p = pidx(g, i, j, k), pm = pidx(g, im, j, k), pp = pidx(g, ip, j, k);
        double amu, apu;
        if (comp == 0) {
            amu = -coe1 * f.MU[pm];
            apu = -coe1 * f.MU[p];
        } else {
            amu = -coe2 * ms[p];
            apu = -coe2 * ms[pp];
        }
        const int s = seg_pos<S>(i);
        a[s] = amu / (double)D[pm];
        c[s] = apu / (double)D[pp];
        b[s] = 1.0 - (amu + apu) / (double)D[p];
        d[s] = comp == 0 ? (double)R[iidx(g, i, j, k)] - dpg : (double)R[iidx(g, i, j, k)];
    }
    __syncwarp();
    warp_tdma_smem<S, true>(d, SegCoef<S>{a, b, c}, lane);
    __syncwarp();
    for (int i = lane; i < L; i += 32) R[iidx(g, i, j, k)] = (F)d[seg_pos<S>(i)];
}

// z lines (i0 .. i0+CN_LINES-1, j); component blockIdx.z
template <int S, typename F>
__global__ void __launch_bounds__(CN_NT, 4) k_io_cn_zsweep(Geo g, IoFieldsT<F> f, const DevState* __restrict__ st, int ns) {
    extern __shared__ double smz[];
    constexpr int SEG = 32 * (S + 1);
    constexpr int RSTEP = CN_NT / CN_LINES;
    const int N = g.N;
    const int comp = blockIdx.z;
    const int j = 1 + blockIdx.y;
    if (comp == 1 && j == 1) return;  // uniform over the block
    const int l = threadIdx.x % CN_LINES, r0 = threadIdx.x / CN_LINES;
    const int i = blockIdx.x * CN_LINES + l;
    const double fac = 0.50 * g.talp[ns] * st->dt * g.cvisc;
    const double coe1 = fac * 4.0 / 3.0 * g.dzqi, coe2 = fac * g.dzqi;
    const F* D = f.DST + comp * g.FS;
    const F* ms = f.MST + (comp == 0 ? g.FS : 2 * g.FS);
    F* R = f.RHS + comp * g.FI;
    double* base = smz + (size_t)l * cn_line_stride(SEG);
#pragma unroll 4  // several rows' coefficient loads in flight
    for (int k = r0; k < N; k += RSTEP) {
        const int km = wrapm(k, N), kp = wrapp(k, N);
        const long long p = pidx(g, i, j, k), pm = pidx(g, i, j, km), pp = pidx(g, i, j, kp);
        double amu, apu;
        if (comp == 2) {
            amu = -coe1 * f.MU[pm] * 1.0;
            apu = -coe1 * f.MU[p] * 1.0;
        } else {
            amu = -coe2 * ms[p] * 1.0;
            apu = -coe2 * ms[pp] * 1.0;
        }
        const int s = seg_pos<S>(k);
        base[s] = amu / (double)D[pm];
        base[SEG + s] = 1.0 - (amu + apu) / (double)D[p];
        base[2 * SEG + s] = apu / (double)D[pp];
        base[3 * SEG + s] = R[iidx(g, i, j, k)];
    }
    __syncthreads();
    {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        double* bw = smz + (size_t)w * cn_line_stride(SEG);
        warp_tdma_smem<S, true>(bw + 3 * SEG, SegCoef<S>{bw, bw + SEG, bw + 2 * SEG}, lane);
    }
    __syncthreads();
    for (int k = r0; k < N; k += RSTEP) R[iidx(g, i, j, k)] = (F)base[3 * SEG + seg_pos<S>(k)];
}

// y lines (i0 .. i0+CN_LINES-1, k); component blockIdx.z; then G += solution
template <int S, typename F>
__global__ void __launch_bounds__(CN_NT) k_io_cn_ysweep(Geo g, IoFieldsT<F> f, const DevState* __restrict__ st, int ns) {
    extern __shared__ double smy[];
    constexpr int SEG = 32 * (S + 1);
    constexpr int RSTEP = CN_NT / CN_LINES;
    const int M = g.M;
    const int comp = blockIdx.z;
    const int k = blockIdx.y;
    const int l = threadIdx.x % CN_LINES, r0 = threadIdx.x / CN_LINES;
    const int i = blockIdx.x * CN_LINES + l;
    const double fac = 0.50 * g.talp[ns] * st->dt * g.cvisc;
    const double coe1 = fac * 4.0 / 3.0, coe2 = fac;
    const F* D = f.DST + comp * g.FS;
    const double* amv = g.amvr + comp * (M + 2);
    const double* apv = g.apvr + comp * (M + 2);
    const F* R = f.RHS + comp * g.FI;
    double* base = smy + (size_t)l * cn_line_stride(SEG);
#pragma unroll 3  // several rows' coefficient loads in flight
    for (int j = 1 + r0; j <= M; j += RSTEP) {
        double A, B, C, amu, apu;
        if (comp != 1) {
            const F* ms = f.MST + (comp == 0 ? 0 : 2 * g.FS);
            if (j == 1) {
                const double muqt = (f.MU[pidx(g, i, 1, k)] + f.MU[pidx(g, i, 0, k)]) * 0.5;
                amu = -coe2 * g.amvr1 * muqt;
                apu = -coe2 * apv[1] * ms[pidx(g, i, 2, k)];
                A = 0.0;
                C = apu / (double)D[pidx(g, i, 2, k)];
            } else if (j == M) {
                const double muqt = (f.MU[pidx(g, i, M, k)] + f.MU[pidx(g, i, M + 1, k)]) * 0.5;
                amu = -coe2 * amv[M] * ms[pidx(g, i, M, k)];
                apu = -coe2 * g.apvrn * muqt;
                A = amu / (double)D[pidx(g, i, M - 1, k)];
                C = 0.0;
            } else {
                amu = -coe2 * amv[j] * ms[pidx(g, i, j, k)];
                apu = -coe2 * apv[j] * ms[pidx(g, i, j + 1, k)];
                A = amu / (double)D[pidx(g, i, j - 1, k)];
                C = apu / (double)D[pidx(g, i, j + 1, k)];
            }
        } else {
            amu = -coe1 * amv[j] * f.MU[pidx(g, i, j - 1, k)];
            apu = -coe1 * apv[j] * f.MU[pidx(g, i, j, k)];
            // j = 1: the ghost D_STG(:,0,:,2) is the y-periodic halo D_STG(:,M,:,2)
            // of a run on two or more ranks; amu is zero there, so only its
            // finiteness matters.
            A = amu / (double)D[pidx(g, i, j == 1 ? M : j - 1, k)];
            C = apu / (double)D[pidx(g, i, j == 1 ? 2 : j, k)];
        }
        B = 1.0 - (amu + apu) / (double)D[pidx(g, i, j, k)];
        const int s = seg_pos<S>(j - 1);
        base[s] = A;
        base[SEG + s] = B;
        base[2 * SEG + s] = C;
        base[3 * SEG + s] = (comp == 1 && j == 1) ? 0.0 : R[iidx(g, i, j, k)];
    }
    __syncthreads();
    {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        double* bw = smy + (size_t)w * cn_line_stride(SEG);
        warp_tdma_smem<S, false>(bw + 3 * SEG, SegCoef<S>{bw, bw + SEG, bw + 2 * SEG}, lane);
    }
    __syncthreads();
    F* Gc = f.G + comp * g.FS;
    for (int j = 1 + r0; j <= M; j += RSTEP) {
        if (comp == 1 && j == 1) continue;
        const long long p = pidx(g, i, j, k);
        Gc[p] = (F)(base[3 * SEG + seg_pos<S>(j - 1)] + (double)Gc[p]);
    }
}
