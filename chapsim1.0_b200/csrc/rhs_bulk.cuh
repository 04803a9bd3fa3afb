// Fused right-hand sides + x sweep (the work of k_rhs_xsweep, momentum.cuh)
// with every row the stencil reads staged in shared memory by the bulk-copy
// (TMA) engine instead of per-thread loads.
//
// A warp owns x lines (j, k) in a stride loop over the grid.  For a line it
// needs 23 rows of length L: u, v, w at (j,k), (j+1,k), (j-1,k), (j,k+1),
// (j,k-1), v at (j+1,k-1), w at (j-1,k+1), PR at (j,k), (j-1,k), (j,k-1), and
// the three CONVH0 rows.  Lane 0 issues them as 23 cp.async.bulk copies that
// complete on the warp's mbarrier into the warp's stage; as soon as the warp
// has read a line's rows it issues the copies of its next line, which then
// arrive while it runs the x sweep and while the block's other warps compute.
// (One stage per warp and up to 8 warps per block measured faster than two
// stages and 4 warps: the arithmetic needs the extra warps to hide its
// latency, and the shared memory holds one 23-row stage per warp.)  The stencils,
// the RK combination, the viscous and pressure terms and the bulk-forcing
// partial sums are those of k_rhs_xsweep, read from shared memory; the x
// sweep runs on the line in segment-padded shared memory as there.
//
// Rows start at multiples of L elements (L >= 32), so every bulk copy is
// 16-byte aligned with a multiple-of-16 size.  The copies read Q, PR and
// CONVH0; the kernel writes CONVH0 only in the row of its own line, after
// that line's copy has completed, and writes RHS, which it does not read.
// mbarrier waits are clock-bounded (error bit, then the warp stops issuing
// and waits, bounded again, for its copies still in flight).
#pragma once
#include "common.cuh"
#include "momentum.cuh"
#include "tdma.cuh"

#define RB_ROWS 23
#define RB_WMAX 12  // warps per block at most (FP32; see rb_wmax)
// Warps per block at most: 8 for FP64 (184 registers: 8 x 32 x 184 fills the
// register file), 12 for FP32, whose stages are half the size and whose
// 153 registers leave room for 12 warps.
template <typename R> __host__ __device__ constexpr int rb_wmax() { return sizeof(R) == 8 ? 8 : RB_WMAX; }

// Shared memory of one warp: one stage of RB_ROWS rows, then the line buffer
// of the x sweep; the region is rounded up to 32 elements so that every
// warp's stage (a bulk-copy destination) starts on a 128-byte boundary.
__host__ __device__ inline int rb_warp_elems(int L) { return ((1 * RB_ROWS * L + 3 * (L + 33) + 31) / 32) * 32; }
template <typename R>
__host__ __device__ inline size_t rb_warp_bytes(int L) {
    return (size_t)rb_warp_elems(L) * sizeof(R);
}
// After the warps' regions, the block keeps the x sweep's factor table: its
// 5S+20 values per lane are read in every line's solve, and with the stages
// filling the shared memory the L1 is too small to hold them (they came from
// L2, inside the sweep's dependency chain).
template <typename R>
__host__ __device__ inline size_t rb_fac_bytes(int L) { return (size_t)TF_NF(L / 32) * 32 * sizeof(R); }
// warps per block that fit beside the factor table, given the block's
// shared-memory limit less the kernel's static shared memory
template <typename R>
inline int rb_warps(int L, long long limit) {
    const size_t per = rb_warp_bytes<R>(L);
    const long long avail = limit - (long long)rb_fac_bytes<R>(L);
    int w = avail > 0 ? (int)(avail / (long long)per) : 0;
    return w < 1 ? 0 : (w > rb_wmax<R>() ? rb_wmax<R>() : w);
}
template <typename R>
inline size_t rb_smem(int L, int nw) { return (size_t)nw * rb_warp_bytes<R>(L) + rb_fac_bytes<R>(L); }

template <typename R>
__device__ __forceinline__ void rb_issue(const Geo& g, const R* Q, const R* PR, const R* H0, int line, R* stage,
                                         uint64_t* bar) {
    const int L = g.L, M = g.M, N = g.N;
    const int j = 1 + line % M, k = line / M;
    const int jp = j + 1, jm = j - 1, kp = wrapp(k, N), km = wrapm(k, N);
    const R* U = Q;
    const R* V = Q + g.FS;
    const R* W = Q + 2 * g.FS;
    const long long c = pidx(g, 0, j, k), cjp = pidx(g, 0, jp, k), cjm = pidx(g, 0, jm, k);
    const long long ckp = pidx(g, 0, j, kp), ckm = pidx(g, 0, j, km);
    const long long ii = iidx(g, 0, j, k);
    const R* src[RB_ROWS] = {U + c, U + cjp, U + cjm, U + ckp, U + ckm,
                             V + c, V + cjp, V + cjm, V + ckp, V + ckm, V + pidx(g, 0, jp, km),
                             W + c, W + cjp, W + cjm, W + ckp, W + ckm, W + pidx(g, 0, jm, kp),
                             PR + c, PR + cjm, PR + ckm,
                             H0 + ii, H0 + ii + g.FI, H0 + ii + 2 * g.FI};
    const uint32_t rb = (uint32_t)(L * sizeof(R));
    mbar_arrive_expect_tx(bar, RB_ROWS * rb);
#pragma unroll
    for (int r = 0; r < RB_ROWS; ++r) bulk_g2s(stage + r * L, src[r], rb, bar);
}

// The y-dependent coefficients of a line (j): interpolation weights at j and
// j+1, metrics, and the viscous y coefficients of the three components.  With
// the stages and the factor table filling the shared memory the L1 is too
// small to keep them, so each line's set comes from L2: the kernel loads the
// next line's set into registers while it solves the current line.
struct RbGeo {
    double wffj, wfbj, wffp, wfbp, dyfi, dyci, am[3], ac[3], ap[3];
};
__device__ __forceinline__ RbGeo rb_geo(const Geo& g, int j) {
    RbGeo r;
    const int M2 = g.M + 2;
    r.wffj = g.wff[j]; r.wfbj = g.wfb[j]; r.wffp = g.wff[j + 1]; r.wfbp = g.wfb[j + 1];
    r.dyfi = g.dyfi[j]; r.dyci = g.dyci[j];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r.am[c] = g.amvr[c * M2 + j];
        r.ac[c] = g.acvr[c * M2 + j];
        r.ap[c] = g.apvr[c * M2 + j];
    }
    return r;
}

template <int S, typename R>
__global__ void __launch_bounds__(rb_wmax<R>() * 32, 1) k_rhs_xsweep_bulk(Geo g, const R* __restrict__ Q,
                                                                     const R* __restrict__ PR, R* __restrict__ H0,
                                                                     R* __restrict__ RHS, double* __restrict__ partial,
                                                                     DevState* __restrict__ st,
                                                                     const R* __restrict__ fac, int ns) {
    pdl_wait();
    extern __shared__ __align__(128) unsigned char rb_raw[];
    __shared__ uint64_t bars[RB_WMAX];
    __shared__ double sred[RB_WMAX];
    __shared__ int is_last;
    constexpr int L = 32 * S;
    const int M = g.M;
    const int nw = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int LS = L + 33;
    R* wbase = reinterpret_cast<R*>(rb_raw) + (size_t)warp * rb_warp_elems(L);
    R* const sg = wbase;
    R* sl = wbase + RB_ROWS * L;
    uint64_t* bar = &bars[warp];
    if (lane == 0) mbar_init(bar, 1);
    __syncwarp();
    const int nlines = M * g.N;
    const int stride = gridDim.x * nw;
    const int first = blockIdx.x * nw + warp;
    if (lane == 0) {
        if (first < nlines) rb_issue<R>(g, Q, PR, H0, first, sg, bar);
    }
    const double dts = st->dt;
    // the x sweep's factor table, staged once per block
    R* const sfx = reinterpret_cast<R*>(rb_raw) + (size_t)nw * rb_warp_elems(L);
    {
        const R* fx = fac + FSET_X * FAC_SET;
        for (int t = threadIdx.x; t < TF_NF(S) * 32; t += blockDim.x) sfx[t] = fx[t];
    }
    __syncthreads();
    double bulk = 0.0;
    uint32_t phase = 0u;
    bool pending = first < nlines;  // a copy issued and not yet consumed
    bool ok = true;
    RbGeo gn = rb_geo(g, first < nlines ? 1 + first % M : 1);
#pragma unroll 1
    for (int line = first; line < nlines; line += stride) {
        // every lane waits; the warp leaves together if any lane's budget ran out
        ok = mbar_wait_warp(bar, phase, &st->err);
        if (!ok) break;  // the copy never completed: stop issuing
        phase ^= 1u;
        pending = false;
        const int j = 1 + line % M, k = line / M;
        const RbGeo gc = gn;
        const RhsLine<R> cl = rhs_line<R>(g, dts, ns, gc.wffj, gc.wfbj, gc.wffp, gc.wfbp, gc.dyfi, gc.dyci, gc.am, gc.ac,
                                          gc.ap);
        const R* sU = sg;          // c, jp, jm, kp, km
        const R* sV = sg + 5 * L;  // c, jp, jm, kp, km, (jp, km)
        const R* sW = sg + 11 * L; // c, jp, jm, kp, km, (jm, kp)
        const R* sP = sg + 17 * L; // c, jm, km
        const R* sH = sg + 20 * L; // u, v, w
        R* H0l = H0 + iidx(g, 0, j, k);
#pragma unroll 2  // two points per lane in flight: more independent FP64 work per warp (2 % at 128^3)
        for (int kk = 0; kk < S; ++kk) {
            const int i = lane + 32 * kk;
            const int ip = i + 1 == L ? 0 : i + 1, im = i == 0 ? L - 1 : i - 1;
            RhsStencil<R> sp;
            sp.u = sU[i]; sp.uip = sU[ip]; sp.uim = sU[im];
            sp.ujp = sU[L + i]; sp.ujm = sU[2 * L + i]; sp.ukp = sU[3 * L + i]; sp.ukm = sU[4 * L + i];
            sp.v = sV[i]; sp.vip = sV[ip]; sp.vim = sV[im];
            sp.vjp = sV[L + i]; sp.vjm = sV[2 * L + i]; sp.vkp = sV[3 * L + i]; sp.vkm = sV[4 * L + i];
            sp.w = sW[i]; sp.wip = sW[ip]; sp.wim = sW[im];
            sp.wjp = sW[L + i]; sp.wjm = sW[2 * L + i]; sp.wkp = sW[3 * L + i]; sp.wkm = sW[4 * L + i];
            sp.pc = sP[i]; sp.pim = sP[im]; sp.pjm = sP[L + i]; sp.pkm = sP[2 * L + i];
            sp.vjpim = sV[L + im]; sp.wkpim = sW[3 * L + im];
            sp.ujmip = sU[2 * L + ip]; sp.wjmkp = sW[5 * L + i];
            sp.ukmip = sU[4 * L + ip]; sp.vjpkm = sV[5 * L + i];
            sp.h0u = sH[i]; sp.h0v = j >= 2 ? sH[L + i] : R(0); sp.h0w = sH[2 * L + i];
            const int pos = seg_pos<S>(i);
            R Hu, Hv, Hw, ru, rv, rw;
            rhs_point(cl, sp, j >= 2, Hu, Hv, Hw, ru, rv, rw, bulk);
            H0l[i] = Hu;
            if (j >= 2) H0l[i + g.FI] = Hv;
            H0l[i + 2 * g.FI] = Hw;
            sl[pos] = ru;
            if (j >= 2) sl[LS + pos] = rv;
            sl[2 * LS + pos] = rw;
        }
        // the stage is read: refill it with this warp's next line
        __syncwarp();
        fence_async_smem();
        if (line + stride < nlines) {
            if (lane == 0) rb_issue<R>(g, Q, PR, H0, line + stride, sg, bar);
            pending = true;
            gn = rb_geo(g, 1 + (line + stride) % M);  // arrives during this line's x sweep
        }
        // cyclic x sweeps of this line's three components (MOMFA1_X_tg starts at N2I = 2 for v)
        warp_tdma_apply_smem3<S, true>(sl, LS, j >= 2, sfx, lane);  // the three components together
        __syncwarp();
        R* Rl = RHS + iidx(g, 0, j, k);
#pragma unroll
        for (int kk = 0; kk < S; ++kk) {
            const int i = lane + 32 * kk;
            const int pos = seg_pos<S>(i);
            Rl[i] = sl[pos];
            if (j >= 2) Rl[i + g.FI] = sl[LS + pos];
            Rl[i + 2 * g.FI] = sl[2 * LS + pos];
        }
        __syncwarp();
    }
    if (!ok) {
        // the warp's copy may still be in flight: wait for it (bounded) before the block exits
        if (pending) (void)mbar_wait_warp(bar, phase, &st->err);
    }
    // grid sum of the bulk-flux integrand: warp, block (warp order), then the
    // last block adds the block partials in index order (deterministic)
    for (int o = 16; o > 0; o >>= 1) bulk += __shfl_down_sync(0xffffffffu, bulk, o);
    if (lane == 0) sred[warp] = bulk;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w2 = 0; w2 < nw; ++w2) s += sred[w2];
        partial[blockIdx.x] = s;
        __threadfence();
        const unsigned prev = atomicAdd(&st->ctr, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int t = 0; t < (int)gridDim.x; ++t) s += __ldcg(partial + t);
            st->bulksum = s;
            st->ctr = 0u;
        }
    }
}
