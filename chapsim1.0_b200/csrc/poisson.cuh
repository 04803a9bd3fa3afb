// Pressure Poisson solve and projection of one RK3 substep:
//   DIVG_tg (src/DIVG.f90:15-51), FFT99_POIS3D_periodicxz
//   (src/possion3d_FFT99.f90:271-505), VELOUPDT_tg
//   (src/VELO_CORRECTION.f90:14-100), PRCALC_tg
//   (src/PRESSURE_CORRECTION.f90:15-99) and the wall ghosts of
//   BC_WALL_PR_tg (src/BC_WALL.f90:293-361).
//
// Kernels:
//   k_div_fftx   divergence of u* / (alpha dt) -> RHSLLPHI, then the real
//                x transform of every (j, k) line (two real lines packed in
//                one complex FFT), times 1/L, into the spectral array
//   k_fftz<S>    complex z transform of every (kx, j) line; forward pass
//                multiplies by 1/N (UN3M)
//   k_ysolve_warp per (kx, kz) tridiagonal solve in y with diagonal
//                ACPH(j) - AK1(kx) - AK3(kz); zero mode pinned as in
//                TDMA_PHI_COEF (:225-231) and :341-344, :387-389
//                (phi_hat(0,y_1,0) = 0)
//   k_fftx_inv   inverse x transform -> DPH
//   k_correct    velocity correction, pressure update, PR wall ghosts
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "tdma.cuh"

#include <type_traits>

// Spectral element type of a step whose fields are stored as R: double2 in the
// FP64 step, float2 in the mixed-precision step (whose x and z transforms run
// in FP32; the y-solve converts to FP64 and back).
template <typename R> using SpecT = typename std::conditional<std::is_same<R, float>::value, float2, double2>::type;
template <typename C> __device__ __forceinline__ const C* twx_of(const Geo& g);
template <> __device__ __forceinline__ const double2* twx_of<double2>(const Geo& g) { return g.twx; }
template <> __device__ __forceinline__ const float2* twx_of<float2>(const Geo& g) { return g.twxf; }
template <typename C> __device__ __forceinline__ const C* twz_of(const Geo& g);
template <> __device__ __forceinline__ const double2* twz_of<double2>(const Geo& g) { return g.twz; }
template <> __device__ __forceinline__ const float2* twz_of<float2>(const Geo& g) { return g.twzf; }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2((double)a.x, (double)a.y); }
template <typename C> __device__ __forceinline__ C from_d2(double2 a);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }

// x-line transforms: PX_TJ x lines per block (PX_TJ / 2 packed pairs), PX_NT
// threads, PX_MINB blocks per SM in the register budget (128 registers).  The
// block loads its lines, transforms them in shared memory and stores them,
// one phase after the other; four small blocks per SM overlap those phases
// better than two blocks of twice the size.
#define PX_TJ 16
#define PX_NT 128
#define PX_MINB 4
// FP32 transforms: eight blocks per SM within 64 registers (twice the warps to
// hide the latency of the load, transform and store phases); the z transform
// likewise runs four FP32 blocks of FZ_NT threads per SM instead of two
template <typename C> __host__ __device__ constexpr int px_minb() { return sizeof(C) == 8 ? 8 : PX_MINB; }
#define FZ_TQ 16  // z-lines per block
#define FZ_NT 256
#define CR_NT 256

// ---------------------------------------------------------------------------
// R is the stored type of Q, PR, RHSLLPHI and DPH (double, or float in the
// mixed-precision step, whose x and z transforms also run in FP32); the
// divergence and the correction are evaluated in FP64.
template <typename R, int N1, int N2>
__global__ void __launch_bounds__(PX_NT, px_minb<SpecT<R>>()) k_div_fftx(Geo g, const R* __restrict__ Q, R* __restrict__ RHSLL,
                                                    SpecT<R>* __restrict__ SP, const DevState* __restrict__ st, int ns) {
    pdl_wait();
    using C = SpecT<R>;
    using T = typename CReal<C>::T;
    extern __shared__ __align__(16) unsigned char smp_raw[];
    C* smc = reinterpret_cast<C*>(smp_raw);
    const int L = g.L, M = g.M, N = g.N, LH = g.LH;
    const int LD = fft4s_ld(L);
    const int j0 = 1 + blockIdx.x * PX_TJ;
    const int k = blockIdx.y;
    const int nj = min(PX_TJ, M - j0 + 1);
    const int np = (nj + 1) >> 1;
    const int kp = wrapp(k, N);
    const double coe0 = 1.0 / (st->dt * g.talp[ns]);
    const R* U = Q;
    const R* V = Q + g.FS;
    const R* Wf = Q + 2 * g.FS;
    const double coe1 = g.dxi / 1.0;
    // one item = VW consecutive points of both rows of a packed pair, read with
    // 16-byte loads; the pair's complex values are stored to shared memory together
    constexpr int VW = V16<R>::W;
    const int LV = L / VW;
#pragma unroll 2
    for (int p = threadIdx.x; p < np * LV; p += PX_NT) {
        const int pair = p / LV, i0 = (p - pair * LV) * VW;
        T val[2][VW];
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            const int jl = 2 * pair + part;
            if (jl < nj) {
                const int j = j0 + jl;
                const long long c = pidx(g, i0, j, k);
                R u[VW], v[VW], vp[VW], w[VW], wp[VW], out[VW];
                ld16(U + c, u);
                ld16(V + c, v);
                ld16(V + c + L, vp);
                ld16(Wf + c, w);
                ld16(Wf + pidx(g, i0, j, kp), wp);
                const double un = U[pidx(g, i0 + VW == L ? 0 : i0 + VW, j, k)];  // u at i0 + VW (periodic)
                const double coe2 = g.dyfi[j] / 1.0;
#pragma unroll
                for (int e = 0; e < VW; ++e) {
                    const double uc = u[e], up = e + 1 < VW ? (double)u[e + 1] : un;
                    const double dv = (up - uc) * coe1 + ((double)vp[e] - (double)v[e]) * coe2 +
                                      ((double)wp[e] - (double)w[e]) * g.dzi;
                    const double x = dv * coe0;
                    out[e] = (R)x;
                    val[part][e] = (T)x;
                }
                st16(RHSLL + iidx(g, i0, j, k), out);
            } else {
#pragma unroll
                for (int e = 0; e < VW; ++e) val[part][e] = (T)0;
            }
        }
        C* line = smc + pair * LD + i0;
#pragma unroll
        for (int e = 0; e < VW; ++e) line[e] = mkc(val[0][e], val[1][e]);
    }
    block_fft4s<N1, N2, -1>(smc, np, LD, twx_of<C>(g));
    // unpack: A_k = (Z_k + conj Z_{L-k}) / 2, B_k = (Z_k - conj Z_{L-k}) / (2i), both times 1/L
    const T sc = (T)(0.5 / (double)L);
    for (int p = threadIdx.x; p < np * LH; p += PX_NT) {
        const int pair = p / LH, kx = p - pair * LH;
        const C* line = smc + pair * LD;
        const C z = line[kx];
        const C zc = line[kx == 0 ? 0 : L - kx];
        const C a = mkc((z.x + zc.x) * sc, (z.y - zc.y) * sc);
        const C b = mkc((z.y + zc.y) * sc, (zc.x - z.x) * sc);
        const int ja = j0 + 2 * pair;
        SP[kx + (long long)LH * ((ja - 1) + (long long)M * k)] = a;
        if (2 * pair + 1 < nj) SP[kx + (long long)LH * ((ja) + (long long)M * k)] = b;
    }
}

// ---------------------------------------------------------------------------
// complex z transform of FZ_TQ consecutive (kx, j) lines (index q = kx + LH*(j-1))
// pf_ahead > 0: the block also requests into L2 the tile of block blockIdx.x + pf_ahead (about
// one wave of resident blocks later), whose copies then find their rows there.
template <int SIGN, int N1, int N2, typename C>
__global__ void __launch_bounds__(FZ_NT, sizeof(C) == 8 ? 4 : 2) k_fftz(Geo g, C* __restrict__ SP, int pf_ahead) {
    pdl_wait();
    using T = typename CReal<C>::T;
    extern __shared__ __align__(16) unsigned char smp_raw[];
    C* smc = reinterpret_cast<C*>(smp_raw);
    const int N = g.N;
    const int LD = fft4s_ld(N);
    const long long Q = (long long)g.LH * g.M;
    const long long q0 = (long long)blockIdx.x * FZ_TQ;
    const int nq = (int)min((long long)FZ_TQ, Q - q0);
    if (pf_ahead > 0) {
        const long long qa = q0 + (long long)pf_ahead * FZ_TQ;
        if (qa + FZ_TQ <= Q) {
            constexpr int LPR = (FZ_TQ * (int)sizeof(C) + 127) / 128;  // 128-byte lines per kz row of a tile
            for (int t = threadIdx.x; t < N * LPR; t += FZ_NT) {
                const int kz = t / LPR, c = t - kz * LPR;
                prefetch_l2(reinterpret_cast<const char*>(SP + qa + Q * kz) + 128 * c);
            }
        }
    }
    for (int p = threadIdx.x; p < FZ_TQ * N; p += FZ_NT) {
        const int kz = p / FZ_TQ, ql = p - kz * FZ_TQ;
        if (ql < nq) {
            if constexpr (sizeof(C) == 16) cp_async16(smc + ql * LD + kz, SP + q0 + ql + Q * kz);
            else cp_async8(reinterpret_cast<double*>(smc + ql * LD + kz), reinterpret_cast<const double*>(SP + q0 + ql + Q * kz));
        }
    }
    cp_async_wait_all();
    block_fft4s<N1, N2, SIGN>(smc, nq, LD, twz_of<C>(g));
    const T sc = SIGN < 0 ? (T)(1.0 / (double)N) : (T)1.0;
    for (int p = threadIdx.x; p < FZ_TQ * N; p += FZ_NT) {
        const int kz = p / FZ_TQ, ql = p - kz * FZ_TQ;
        if (ql < nq) {
            C v = smc[ql * LD + kz];
            if (SIGN < 0) { v.x = v.x * sc; v.y = v.y * sc; }
            SP[q0 + ql + Q * kz] = v;
        }
    }
}

// Persistent, double-buffered form of k_fftz (autotuned alternative): a block
// owns every gridDim.x-th tile of TQ lines and issues the copies of its
// next tile (cp.async into the other buffer) before it transforms and stores
// the current one, so the loads overlap the transform and the stores, where
// the one-tile blocks of k_fftz overlap them only across blocks.  The
// arithmetic is k_fftz's: the fields are bitwise equal.
// Two blocks per SM at both precisions.  FP64: tiles of 8 lines (two 51 KB buffers at
// N = 384) and 128 threads, whose register budget holds the 384-point transform inside the
// persistent tile loop (at 256 threads and 128 registers it spilled 700 bytes); FP32: tiles
// of 16 lines and 256 threads.
template <typename C> __host__ __device__ constexpr int fzp_tq() { return sizeof(C) == 16 ? 8 : 16; }
template <typename C> __host__ __device__ constexpr int fzp_nt() { return sizeof(C) == 16 ? 128 : 256; }
template <typename C> __host__ __device__ constexpr int fzp_minb() { return 2; }

template <int SIGN, int N1, int N2, typename C>
__global__ void __launch_bounds__(fzp_nt<C>(), fzp_minb<C>()) k_fftz_pipe(Geo g, C* __restrict__ SP) {
    pdl_wait();
    constexpr int TQ = fzp_tq<C>();
    constexpr int NT = fzp_nt<C>();
    using T = typename CReal<C>::T;
    extern __shared__ __align__(16) unsigned char smp_raw[];
    const int N = g.N;
    const int LD = fft4s_ld(N);
    C* const buf0 = reinterpret_cast<C*>(smp_raw);
    const long long Q = (long long)g.LH * g.M;
    const long long ntile = (Q + TQ - 1) / TQ;
    auto issue = [&](long long tile, C* b) {
        if (tile < ntile) {
            const long long q0 = tile * TQ;
            const int nq = (int)min((long long)TQ, Q - q0);
#pragma unroll 1
            for (int p = threadIdx.x; p < TQ * N; p += NT) {
                const int kz = p / TQ, ql = p - kz * TQ;
                if (ql < nq) {
                    if constexpr (sizeof(C) == 16) cp_async16(b + ql * LD + kz, SP + q0 + ql + Q * kz);
                    else cp_async8(reinterpret_cast<double*>(b + ql * LD + kz), reinterpret_cast<const double*>(SP + q0 + ql + Q * kz));
                }
            }
        }
        cp_async_commit();  // an empty group past the end keeps the group count uniform
    };
    const T sc = SIGN < 0 ? (T)(1.0 / (double)N) : (T)1.0;
    issue(blockIdx.x, buf0);
    int cur = 0;
#pragma unroll 1
    for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x, cur ^= 1) {
        C* const bc = buf0 + cur * (TQ * LD);
        issue(tile + gridDim.x, buf0 + (cur ^ 1) * (TQ * LD));
        cp_async_wait_group<1>();  // this tile's copies (all but the newest group) have landed
        const long long q0 = tile * TQ;
        const int nq = (int)min((long long)TQ, Q - q0);
        block_fft4s<N1, N2, SIGN>(bc, nq, LD, twz_of<C>(g));  // starts and ends with a block barrier
#pragma unroll 1
        for (int p = threadIdx.x; p < TQ * N; p += NT) {
            const int kz = p / TQ, ql = p - kz * TQ;
            if (ql < nq) {
                C v = bc[ql * LD + kz];
                if (SIGN < 0) { v.x = v.x * sc; v.y = v.y * sc; }
                SP[q0 + ql + Q * kz] = v;
            }
        }
        __syncthreads();  // the buffer is the copy target of the iteration after next
    }
    cp_async_wait_group<0>();
}

// ---------------------------------------------------------------------------
// y solve of YW_L consecutive lines q = kx + LH*kz per block, one warp per
// line, by the warp Thomas/PCR hybrid with a complex right-hand side
// (warp_tdma_c).  The coefficients (AMPH, ACPH - AK1 - AK3, APPH) are formed
// on the fly, so no per-line factor arrays are read.  For kx != 0 or kz != 0
// the systems are strictly diagonally dominant (AK1 + AK3 > 0 on top of the
// weakly dominant Neumann operator), for which the reduction is stable.  The
// singular kx = kz = 0 line keeps the reference's sequential recurrence with
// its pinned first row (TDMA_PHI_COEF :225-231, :341-344, :387-389), run by
// one lane.  Lines are staged in shared memory, line l at l*LS with row r at
// seg_pos<S>(r), LS = M + 33: conflict-free both for the coalesced tile load
// (16 lines per row) and for the per-lane segment access.  Shared memory:
// two stages of YW_L such lines in the spectrum's type, plus M FP64 complex
// values for the zero mode's forward sweep when that type is float2.
#define YW_L 16
#define YW_NT 512

struct PoisCoef {
    const double *am, *ac, *ap;
    double shift;
    __device__ __forceinline__ double A(int r) const { return am[r + 1]; }
    __device__ __forceinline__ double B(int r) const { return ac[r + 1] + shift; }
    __device__ __forceinline__ double C(int r) const { return ap[r + 1]; }
};

// Factors of the zero-mode recurrence (kx = kz = 0, phi(y_1) pinned): the
// forward sweep's pivots pp[j-1] = 1/((ACPH(j) + shift) - H(j-1) AMPH(j)) and
// multipliers hz[j-1] = H(j).  They depend on the operator only (not on dt or
// the right-hand side), so they are formed once, by the expression the
// sweep itself would evaluate, and the per-substep zero-mode solve is a chain
// of multiply-adds.  zf[0..M) = pp, zf[M..2M) = hz.
__global__ void k_ysolve_zero_factors(Geo g, double* __restrict__ zf) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int M = g.M;
    const double shift = (-g.ak1[0] / 1.0 - g.ak3[0]);
    const double b = g.acph[1] + shift;
    double hp = 0.0 / b;
    zf[0] = 1.0 / b;
    zf[M] = hp;
    for (int j = 2; j <= M; ++j) {
        const double pp = 1.0 / ((g.acph[j] + shift) - hp * g.amph[j]);
        hp = j < M ? g.apph[j] * pp : 0.0;
        zf[j - 1] = pp;
        zf[M + j - 1] = hp;
    }
}

// Persistent and double-buffered: each block owns every gridDim.x-th group of
// YW_L lines.  The copies of its next group go out (cp.async into the other
// stage) before the current group is solved and written back, so the loads
// overlap the warps' solves and the stores.  One warp per line of a group.
// The stage holds the spectrum's own type (float2 in the mixed-precision
// step); a warp widens its segment to FP64 for the solve.
template <int S, typename C>
__global__ void __launch_bounds__(YW_NT, 1) k_ysolve_warp(Geo g, C* __restrict__ SP) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char yw_raw[];
    static_assert(YW_NT == 32 * YW_L, "one warp per line of a group");
    const int M = 32 * S, LH = g.LH;
    const int LS = M + 33;
    C* const stage[2] = {reinterpret_cast<C*>(yw_raw), reinterpret_cast<C*>(yw_raw) + YW_L * LS};
    const long long nl = (long long)LH * g.N;
    const long long ngr = (nl + YW_L - 1) / YW_L;
    // the staging loops: thread t moves line t % YW_L, rows t / YW_L + (YW_NT / YW_L) * it
    const int ls = threadIdx.x % YW_L, js = threadIdx.x / YW_L;
    constexpr int RS = YW_NT / YW_L;  // rows per staging step
    auto line_ptr = [&](long long q) {
        const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
        return SP + kx + (long long)LH * ((long long)M * kz);
    };
    auto issue = [&](long long gr, C* st) {
        if (gr < ngr) {
            const long long q = gr * YW_L + ls;
            if (q < nl) {
                const C* src = line_ptr(q);
                for (int j = js; j < M; j += RS) cp_async_row(st + ls * LS + seg_pos<S>(j), src + (long long)LH * j);
            }
        }
        cp_async_commit();  // an empty group past the end keeps the group count uniform
    };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    issue(blockIdx.x, stage[0]);
    int cur = 0;
#pragma unroll 1
    for (long long gr = blockIdx.x; gr < ngr; gr += gridDim.x, cur ^= 1) {
        issue(gr + gridDim.x, stage[cur ^ 1]);
        cp_async_wait_group<1>();  // this group's copies (all but the newest group) have landed
        __syncthreads();
        C* const st = stage[cur];
        const long long q = gr * YW_L + warp;
        if (q < nl) {
            const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
            C* base = st + warp * LS;
            if (q == 0) {
                // zero mode: phi(y_1) = 0 and the reference's forward/backward recurrence
                if (lane == 0) {
                    const double* pp = g.yz;
                    const double* hz = g.yz + M;
                    double2 gp = make_double2(0.0 * pp[0], 0.0 * pp[0]);
                    base[seg_pos<S>(0)] = from_d2<C>(gp);
                    // the forward intermediate g stays FP64: kept in the stage when C is
                    // double2; for a float2 stage the chain runs in a second pass below
                    if constexpr (sizeof(C) == 16) {
#pragma unroll 4
                        for (int j = 2; j <= M; ++j) {
                            const double2 rj = to_d2(base[seg_pos<S>(j - 1)]);
                            const double am = g.amph[j], p = pp[j - 1];
                            gp = make_double2((rj.x - am * gp.x) * p, (rj.y - am * gp.y) * p);
                            base[seg_pos<S>(j - 1)] = from_d2<C>(gp);
                        }
                        double2 xn = gp;
#pragma unroll 4
                        for (int j = M - 1; j >= 1; --j) {
                            const double2 gj = to_d2(base[seg_pos<S>(j - 1)]);
                            const double h = hz[j - 1];
                            xn = make_double2(gj.x - h * xn.x, gj.y - h * xn.y);
                            base[seg_pos<S>(j - 1)] = from_d2<C>(xn);
                        }
                    } else {
                        // FP32 stage: the FP64 forward values go to the FP64 scratch row of
                        // this block (after both stages), then the backward sweep
                        double2* gsc = reinterpret_cast<double2*>(reinterpret_cast<C*>(yw_raw) + 2 * YW_L * LS);
                        gsc[0] = gp;
#pragma unroll 4
                        for (int j = 2; j <= M; ++j) {
                            const double2 rj = to_d2(base[seg_pos<S>(j - 1)]);
                            const double am = g.amph[j], p = pp[j - 1];
                            gp = make_double2((rj.x - am * gp.x) * p, (rj.y - am * gp.y) * p);
                            gsc[j - 1] = gp;
                        }
                        double2 xn = gp;
                        base[seg_pos<S>(M - 1)] = from_d2<C>(xn);
#pragma unroll 4
                        for (int j = M - 1; j >= 1; --j) {
                            const double2 gj = gsc[j - 1];
                            const double h = hz[j - 1];
                            xn = make_double2(gj.x - h * xn.x, gj.y - h * xn.y);
                            base[seg_pos<S>(j - 1)] = from_d2<C>(xn);
                        }
                    }
                }
            } else {
                PoisCoef cf{g.amph, g.acph, g.apph, (-g.ak1[kx] / 1.0 - g.ak3[kz])};
                double2 d[S];
#pragma unroll
                for (int k = 0; k < S; ++k) d[k] = to_d2(base[lane * (S + 1) + k]);
                warp_tdma_c<S>(d, cf, lane);
#pragma unroll
                for (int k = 0; k < S; ++k) base[lane * (S + 1) + k] = from_d2<C>(d[k]);
            }
        }
        __syncthreads();
        {
            const long long qs = gr * YW_L + ls;
            if (qs < nl) {
                C* dst = line_ptr(qs);
                for (int j = js; j < M; j += RS) dst[(long long)LH * j] = st[ls * LS + seg_pos<S>(j)];
            }
        }
        __syncthreads();  // the stage is free for the copies issued in the next iteration but one
    }
    cp_async_wait_group<0>();
}

// ---------------------------------------------------------------------------
// Fifth y-solve variant: the sequential recurrence's factors (the same pivots
// PP and multipliers H as k_ysolve_seq_factors; k_ysolve_scan_factors stores
// the pivots line by line, F[q*M + t] = PP_t, and the kernel forms each
// H_t = APPH(t+1) PP_t, H_0 = C_0 / PP_0, H_{M-1} = 0, with the factor
// kernel's own operations, so only half the factor bytes are read) turn both sweeps
// into first-order linear recurrences,
//   forward   g_t = (r_t - A_t g_{t-1}) PP_t      (g_0 = r_0 / PP_0, r_0 = 0 on the zero mode)
//   backward  x_t = g_t - H_t x_{t+1}             (H_{M-1} = 0),
// which one warp per line evaluates as affine scans: lane l owns rows
// lS .. lS+S-1, composes its rows' maps, the 32 lane maps are combined by a
// shuffle scan (5 steps), and each lane then runs its rows' recurrence
// sequentially from its incoming value, in the reference's operation order.
// Only the spectrum is read and written (plus the factors): the forward
// intermediate stays in registers, where the sequential variant moves it
// through memory.  Lines are staged as in k_ysolve_warp (persistent,
// double-buffered groups of YW_L lines, one warp per line).  The lane maps are
// combined in tree order, so the result agrees with the sequential recurrence
// to rounding (1e-12 of the oracle on the Poisson problem).

__global__ void k_ysolve_scan_factors(Geo g, double* __restrict__ F) {
    const int M = g.M, LH = g.LH;
    const long long nl = (long long)LH * g.N;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nl; q += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
        const double shift = (-g.ak1[kx] / 1.0 - g.ak3[kz]);
        const double b = g.acph[1] + shift;
        const double c = q == 0 ? 0.0 : g.apph[1];
        double hp = c / b;
        double* f = F + q * M;
        f[0] = b;
        for (int j = 2; j <= M; ++j) {
            const double pp = 1.0 / ((g.acph[j] + shift) - hp * g.amph[j]);
            hp = j < M ? g.apph[j] * pp : 0.0;
            f[j - 1] = pp;
        }
    }
}

template <int S, typename C>
__global__ void __launch_bounds__(YW_NT, 1) k_ysolve_scan(Geo g, C* __restrict__ SP, const double* __restrict__ F) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char ysc_raw[];
    static_assert(YW_NT == 32 * YW_L, "one warp per line of a group");
    const int M = 32 * S, LH = g.LH;
    const int LS = M + 33;
    C* const stage[2] = {reinterpret_cast<C*>(ysc_raw), reinterpret_cast<C*>(ysc_raw) + YW_L * LS};
    // AMPH(t+1) at t + t / S: a lane reads rows lS .. lS+S-1, and the pad after every S rows
    // puts the lanes' rows on different banks (lane-strided reads of the unpadded rows made
    // 36 M bank conflicts per launch at 384 x 256 x 384)
    double* const sam = reinterpret_cast<double*>(reinterpret_cast<C*>(ysc_raw) + 2 * YW_L * LS);
    double* const sap = sam + (M + 32);  // APPH(t+1), the same layout
    for (int t = threadIdx.x; t < M; t += YW_NT) {
        sam[t + t / S] = g.amph[t + 1];
        sap[t + t / S] = g.apph[t + 1];
    }
    const long long nl = (long long)LH * g.N;
    const long long ngr = (nl + YW_L - 1) / YW_L;
    const int ls = threadIdx.x % YW_L, js = threadIdx.x / YW_L;
    constexpr int RS = YW_NT / YW_L;
    auto line_ptr = [&](long long q) {
        const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
        return SP + kx + (long long)LH * ((long long)M * kz);
    };
    auto issue = [&](long long gr, C* st) {
        if (gr < ngr) {
            const long long q = gr * YW_L + ls;
            if (q < nl) {
                const C* src = line_ptr(q);
                for (int j = js; j < M; j += RS) cp_async_row(st + ls * LS + seg_pos<S>(j), src + (long long)LH * j);
            }
        }
        cp_async_commit();
    };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = lane * S, s0 = lane * (S + 1);  // the lane's first row and its operator-row slot
    issue(blockIdx.x, stage[0]);
    int cur = 0;
#pragma unroll 1
    for (long long gr = blockIdx.x; gr < ngr; gr += gridDim.x, cur ^= 1) {
        issue(gr + gridDim.x, stage[cur ^ 1]);
        // this warp's line pivots (coalesced: the warp reads 32 S contiguous doubles)
        const long long q = gr * YW_L + warp;
        double pp[S], hh[S];
        if (q < nl) {
            const double* f = F + q * M + r0;
            if constexpr (S % 2 == 0) {
#pragma unroll
                for (int k = 0; k < S; k += 2) {
                    const double2 a = __ldg(reinterpret_cast<const double2*>(f + k));
                    pp[k] = a.x; pp[k + 1] = a.y;
                }
            } else {
#pragma unroll
                for (int k = 0; k < S; ++k) pp[k] = __ldg(f + k);
            }
        }
        cp_async_wait_group<1>();
        __syncthreads();  // (also the first iteration's barrier for sam and sap)
        if (q < nl) {
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int t = r0 + k;
                if (t == 0) hh[k] = (q == 0 ? 0.0 : sap[0]) / pp[0];
                else hh[k] = t < M - 1 ? sap[s0 + k] * pp[k] : 0.0;
            }
        }
        C* const st = stage[cur];
        if (q < nl) {
            C* base = st + warp * LS + lane * (S + 1);
            double2 d[S];
#pragma unroll
            for (int k = 0; k < S; ++k) d[k] = to_d2(base[k]);
            if (q == 0 && lane == 0) d[0] = make_double2(0.0, 0.0);  // the zero mode's pinned first row
            // forward: the lane's map g_out = A g_in + B over its rows (row 0 ignores g_in)
            double A = 1.0;
            double2 B = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int t = r0 + k;
                if (t == 0) {
                    A = 0.0;
                    B = make_double2(d[k].x / pp[k], d[k].y / pp[k]);
                } else {
                    const double al = -sam[s0 + k] * pp[k];
                    B = make_double2(al * B.x + d[k].x * pp[k], al * B.y + d[k].y * pp[k]);
                    A = al * A;
                }
            }
            // inclusive scan over the lanes (lane 0's map first)
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double Ap = __shfl_up_sync(0xffffffffu, A, o);
                const double Bx = __shfl_up_sync(0xffffffffu, B.x, o), By = __shfl_up_sync(0xffffffffu, B.y, o);
                if (lane >= o) {
                    B = make_double2(A * Bx + B.x, A * By + B.y);
                    A = A * Ap;
                }
            }
            double2 gp = make_double2(__shfl_up_sync(0xffffffffu, B.x, 1), __shfl_up_sync(0xffffffffu, B.y, 1));
            if (lane == 0) gp = make_double2(0.0, 0.0);
            // the lane's rows from its incoming value, in the reference's order
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int t = r0 + k;
                if (t == 0) {
                    gp = make_double2(d[k].x / pp[k], d[k].y / pp[k]);
                } else {
                    const double a = sam[s0 + k];
                    gp = make_double2((d[k].x - a * gp.x) * pp[k], (d[k].y - a * gp.y) * pp[k]);
                }
                d[k] = gp;
            }
            // backward: x_t = g_t - H_t x_{t+1}; the lane's map gives its first row's x from the next lane's
            // first row's (x_in): x = A x_in + B, composed from the lane's last row down
            A = 1.0;
            B = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = S - 1; k >= 0; --k) {
                const double ga = -hh[k];
                B = make_double2(ga * B.x + d[k].x, ga * B.y + d[k].y);
                A = ga * A;
            }
            // inclusive scan over the lanes from lane 31 down
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double Ap = __shfl_down_sync(0xffffffffu, A, o);
                const double Bx = __shfl_down_sync(0xffffffffu, B.x, o), By = __shfl_down_sync(0xffffffffu, B.y, o);
                if (lane + o < 32) {
                    B = make_double2(A * Bx + B.x, A * By + B.y);
                    A = A * Ap;
                }
            }
            double2 xn = make_double2(__shfl_down_sync(0xffffffffu, B.x, 1), __shfl_down_sync(0xffffffffu, B.y, 1));
            if (lane == 31) xn = make_double2(0.0, 0.0);  // H_{M-1} = 0: the top row is its own g
#pragma unroll
            for (int k = S - 1; k >= 0; --k) {
                xn = make_double2(d[k].x - hh[k] * xn.x, d[k].y - hh[k] * xn.y);
                base[k] = from_d2<C>(xn);
            }
        }
        __syncthreads();
        {
            const long long qs = gr * YW_L + ls;
            if (qs < nl) {
                C* dst = line_ptr(qs);
                for (int j = js; j < M; j += RS) dst[(long long)LH * j] = st[ls * LS + seg_pos<S>(j)];
            }
        }
        __syncthreads();
    }
    cp_async_wait_group<0>();
}

// ---------------------------------------------------------------------------
// The other y-solve variant: the reference's sequential Thomas recurrence
// (TDMAIJJ_nonCYC :95-121, zero mode pinned as above), one thread per
// (kx, kz) line.  The coefficient part of the recurrence (the pivots
// PP_j = 1/(B_j - H_{j-1} A_j) and multipliers H_j) depends on the operator
// only, not on dt or the right-hand side, so k_ysolve_seq_factors runs it
// once per line and keeps PP and H (2 M doubles per line, row-major over the
// lines: PP_j of line q at F[j*nl + q], H_j at F[(M+j)*nl + q]; row 1 keeps
// B_1 itself, which the first row divides by).  The per-substep solve is
// then two chains of multiply-adds.
//
// There are only LH * N lines (8320 at 128^3), so the solve is one thread per
// line, and what bounds it is the latency of its row loads.  Each thread
// keeps a ring of YS_G * YS_NG rows in shared memory, filled by cp.async in
// groups of YS_G rows (every row access is coalesced across the consecutive
// kx of a warp): while the chain consumes one group, the next YS_NG - 1 are
// in flight.  The forward chain leaves g_j in G (FP64; the spectral array
// itself when it is FP64, the FP64 array as scratch when the spectrum is
// FP32), which the backward chain streams back through the same ring.  No
// thread reads another's ring slots, so there is no block barrier.  The
// autotuner picks between this variant and the warp hybrid per grid.
#define YS_G 8
#define YS_NG 8
#define YS_NT 32
__host__ __device__ constexpr size_t smem_ysolve_seq() { return (size_t)YS_G * YS_NG * YS_NT * (sizeof(double2) + sizeof(double)); }
// With kg, the forward intermediate g of the block's lines stays in shared
// memory ([M][YS_NT] double2 after the ring) instead of making a round trip
// through global memory, and only the multipliers stream through the ring on
// the way back: 64 KB more at M = 128, chosen where two blocks still fit an SM.
// The M values of AMPH follow (the chain reads one per row; with the ring
// and g filling the shared memory the L1 is small, and the factor copies
// evicted them: every read went to L2).
inline size_t smem_ysolve_seq(int M, bool kg) {
    return smem_ysolve_seq() + (kg ? (size_t)M * YS_NT * sizeof(double2) : 0) + (size_t)M * sizeof(double);
}

__global__ void k_ysolve_seq_factors(Geo g, double* __restrict__ F) {
    const int M = g.M, LH = g.LH;
    const long long nl = (long long)LH * g.N;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nl; q += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
        const double shift = (-g.ak1[kx] / 1.0 - g.ak3[kz]);
        const double b = g.acph[1] + shift;
        const double c = q == 0 ? 0.0 : g.apph[1];
        double hp = c / b;
        F[q] = b;
        F[(long long)M * nl + q] = hp;
        for (int j = 2; j <= M; ++j) {
            const double pp = 1.0 / ((g.acph[j] + shift) - hp * g.amph[j]);
            hp = j < M ? g.apph[j] * pp : 0.0;
            F[(long long)(j - 1) * nl + q] = pp;
            F[(long long)(M + j - 1) * nl + q] = hp;
        }
    }
}

template <typename C>
__device__ __forceinline__ void cp_async_row(C* dst, const C* src) {
    if constexpr (sizeof(C) == 16) cp_async16(dst, src);
    else cp_async8(reinterpret_cast<double*>(dst), reinterpret_cast<const double*>(src));
}

template <typename C, bool KG>
__global__ void __launch_bounds__(YS_NT) k_ysolve_seq(Geo g, C* SP, double2* G, const double* __restrict__ F) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char ys_raw[];
    constexpr int NR = YS_G * YS_NG;
    double2* const ringg = reinterpret_cast<double2*>(ys_raw);  // [NR][YS_NT] rows of G (backward)
    C* const ringc = reinterpret_cast<C*>(ys_raw);              // [NR][YS_NT] rows of the spectrum (forward)
    double* const ringf = reinterpret_cast<double*>(ys_raw + (size_t)NR * YS_NT * sizeof(double2));  // factors
    double2* const gsm = reinterpret_cast<double2*>(ys_raw + smem_ysolve_seq());  // [M][YS_NT] g (KG)
    const int M = g.M, LH = g.LH, th = threadIdx.x;
    double* const sam = reinterpret_cast<double*>(ys_raw + smem_ysolve_seq() +
                                                  (KG ? (size_t)M * YS_NT * sizeof(double2) : 0));  // AMPH(t+1)
    for (int t = th; t < M; t += YS_NT) sam[t] = g.amph[t + 1];
    __syncthreads();
    const long long nl = (long long)LH * g.N;
    const long long q = (long long)blockIdx.x * YS_NT + th;
    if (q >= nl) return;  // no block barrier below
    const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
    const long long base = kx + (long long)LH * M * kz;
    C* const s = SP + base;
    double2* const gs = G + base;
    const double* const PP = F + q;
    const double* const HH = F + (long long)M * nl + q;
    const long long rs = LH;  // row stride of the spectrum
    // forward: g_1 = r_1 / B_1 (r_1 = 0 on the zero mode), g_t = (r_t - A_t g_{t-1}) PP_t
    const int nb = M / YS_G;
    auto issue_f = [&](int b) {
        if (b < nb) {
#pragma unroll
            for (int u = 0; u < YS_G; ++u) {
                const int row = b * YS_G + u, slot = (b % YS_NG) * YS_G + u;
                cp_async_row(ringc + slot * YS_NT + th, s + rs * row);
                cp_async8(ringf + slot * YS_NT + th, PP + (long long)row * nl);
            }
        }
        cp_async_commit();  // an empty group past the end keeps the group count uniform
    };
#pragma unroll 1
    for (int b = 0; b < YS_NG - 1; ++b) issue_f(b);
    double2 gp = make_double2(0.0, 0.0);
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        issue_f(b + YS_NG - 1);
        cp_async_wait_group<YS_NG - 1>();  // group b has landed
#pragma unroll
        for (int u = 0; u < YS_G; ++u) {
            const int t = b * YS_G + u, slot = (b % YS_NG) * YS_G + u;
            const double2 r = to_d2(ringc[slot * YS_NT + th]);
            const double p = ringf[slot * YS_NT + th];
            if (t == 0) {
                const double2 r0 = q == 0 ? make_double2(0.0, 0.0) : r;
                gp = make_double2(r0.x / p, r0.y / p);
            } else {
                const double a = sam[t];
                gp = make_double2((r.x - a * gp.x) * p, (r.y - a * gp.y) * p);
            }
            if (t < M - 1) {
                if constexpr (KG) gsm[t * YS_NT + th] = gp;
                else gs[rs * t] = gp;
            }
        }
    }
    cp_async_wait_group<0>();
    if constexpr (!KG) __threadfence();  // the G rows written above, before the cp.async reads below
    // backward: x_M = g_M, x_t = g_t - H_t x_{t+1}, t = M-1 .. 1 (rows t-1 = M-2 .. 0)
    double2 xn = gp;
    s[rs * (M - 1)] = from_d2<C>(xn);
    const int nbb = (M - 1 + YS_G - 1) / YS_G;
    auto issue_b = [&](int b) {
        if (b < nbb) {
#pragma unroll
            for (int u = 0; u < YS_G; ++u) {
                const int t = M - 2 - b * YS_G - u, slot = (b % YS_NG) * YS_G + u;
                if (t >= 0) {
                    if constexpr (!KG) cp_async16(ringg + slot * YS_NT + th, gs + rs * t);
                    cp_async8(ringf + slot * YS_NT + th, HH + (long long)t * nl);
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll 1
    for (int b = 0; b < YS_NG - 1; ++b) issue_b(b);
#pragma unroll 1
    for (int b = 0; b < nbb; ++b) {
        issue_b(b + YS_NG - 1);
        cp_async_wait_group<YS_NG - 1>();
#pragma unroll
        for (int u = 0; u < YS_G; ++u) {
            const int t = M - 2 - b * YS_G - u, slot = (b % YS_NG) * YS_G + u;
            if (t >= 0) {
                const double2 gt = KG ? gsm[t * YS_NT + th] : ringg[slot * YS_NT + th];
                const double h = ringf[slot * YS_NT + th];
                xn = make_double2(gt.x - h * xn.x, gt.y - h * xn.y);
                s[rs * t] = from_d2<C>(xn);
            }
        }
    }
    cp_async_wait_group<0>();
}

// ---------------------------------------------------------------------------
// Third y-solve variant: two-way elimination, two threads per mode line.
// The sequential recurrence is bound by one thread's chain of dependent
// instructions over all M rows.  Here the upper thread of a lane pair
// eliminates rows 0 .. m-1 downwards (Thomas: x_t = g_t - h_t x_{t+1}), the
// lower one rows M-1 .. m+1 upwards (x_t = g'_t - h'_t x_{t-1}), m = M/2;
// the middle row closes the system,
//   x_m = (r_m - A_m g_{m-1} - C_m g'_{m+1}) / (B_m - A_m h_{m-1} - C_m h'_{m+1}),
// and each thread substitutes back over its own half.  The result is the
// same tridiagonal solution with another rounding order: on the 128-row
// channel it agrees with the reference's one-way recurrence to 1e-14 on the
// kx, kz != 0 modes and to 1.2e-13 (relative) on the pinned zero mode, whose
// operator is the weakly dominant Neumann one.  The pivots are precomputed
// per line (k_ysolve_2w_factors): F[t*nl + q] holds 1/pivot of row t (upper
// rows, the middle row, lower rows), F[(M+t)*nl + q] the multiplier h_t or
// h'_t.  Rows move through the per-thread cp.async ring of k_ysolve_seq.
__global__ void k_ysolve_2w_factors(Geo g, double* __restrict__ F) {
    const int M = g.M, LH = g.LH, m = M / 2;
    const long long nl = (long long)LH * g.N;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nl; q += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
        const double shift = (-g.ak1[kx] / 1.0 - g.ak3[kz]);
        // upper half, rows t = 0 .. m-1 (j = t + 1); the zero mode's row 1 is decoupled (phi(y_1) = 0)
        double p = 1.0 / (g.acph[1] + shift);
        double h = (q == 0 ? 0.0 : g.apph[1]) * p;
        F[q] = p;
        F[(long long)M * nl + q] = h;
        for (int t = 1; t < m; ++t) {
            const int j = t + 1;
            p = 1.0 / ((g.acph[j] + shift) - h * g.amph[j]);
            h = g.apph[j] * p;
            F[(long long)t * nl + q] = p;
            F[(long long)(M + t) * nl + q] = h;
        }
        // lower half, rows t = M-1 .. m+1
        double pb = 1.0 / (g.acph[M] + shift);
        double hb = g.amph[M] * pb;
        F[(long long)(M - 1) * nl + q] = pb;
        F[(long long)(2 * M - 1) * nl + q] = hb;
        for (int t = M - 2; t > m; --t) {
            const int j = t + 1;
            pb = 1.0 / ((g.acph[j] + shift) - hb * g.apph[j]);
            hb = g.amph[j] * pb;
            F[(long long)t * nl + q] = pb;
            F[(long long)(M + t) * nl + q] = hb;
        }
        // middle row m
        const int jm = m + 1;
        F[(long long)m * nl + q] = 1.0 / ((g.acph[jm] + shift) - g.amph[jm] * h - g.apph[jm] * hb);
        F[(long long)(M + m) * nl + q] = 0.0;
    }
}

template <typename C>
__global__ void __launch_bounds__(YS_NT) k_ysolve_2w(Geo g, C* SP, double2* G, const double* __restrict__ F) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char ys_raw[];
    constexpr int NR = YS_G * YS_NG;
    double2* const ringg = reinterpret_cast<double2*>(ys_raw);
    C* const ringc = reinterpret_cast<C*>(ys_raw);
    double* const ringf = reinterpret_cast<double*>(ys_raw + (size_t)NR * YS_NT * sizeof(double2));
    const int M = g.M, LH = g.LH, m = M / 2, th = threadIdx.x;
    const long long nl = (long long)LH * g.N;
    const long long q = ((long long)blockIdx.x * YS_NT + th) >> 1;
    if (q >= nl) return;  // both lanes of a pair leave together; no block barrier below
    const bool lower = (th & 1) != 0;
    const unsigned pair = 3u << ((th & 31) & ~1);
    const int kz = (int)(q / LH), kx = (int)(q - (long long)kz * LH);
    const long long base = kx + (long long)LH * M * kz;
    C* const s = SP + base;
    double2* const gs = G + base;
    const double* const PP = F + q;
    const double* const HH = F + (long long)M * nl + q;
    const long long rs = LH;
    // forward: upper rows 0, 1, .., m-1; lower rows M-1, M-2, .., m+1
    const int nf = lower ? m - 1 : m;
    auto frow = [&](int i) { return lower ? M - 1 - i : i; };
    const int nbf = (nf + YS_G - 1) / YS_G;
    auto issue_f = [&](int b) {
        if (b < nbf) {
#pragma unroll
            for (int u = 0; u < YS_G; ++u) {
                const int i = b * YS_G + u, slot = (b % YS_NG) * YS_G + u;
                if (i < nf) {
                    const int row = frow(i);
                    cp_async_row(ringc + slot * YS_NT + th, s + rs * row);
                    cp_async8(ringf + slot * YS_NT + th, PP + (long long)row * nl);
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll 1
    for (int b = 0; b < YS_NG - 1; ++b) issue_f(b);
    double2 gp = make_double2(0.0, 0.0);
#pragma unroll 1
    for (int b = 0; b < nbf; ++b) {
        issue_f(b + YS_NG - 1);
        cp_async_wait_group<YS_NG - 1>();
#pragma unroll
        for (int u = 0; u < YS_G; ++u) {
            const int i = b * YS_G + u, slot = (b % YS_NG) * YS_G + u;
            if (i < nf) {
                const int t = frow(i);
                double2 r = to_d2(ringc[slot * YS_NT + th]);
                const double p = ringf[slot * YS_NT + th];
                if (i == 0) {
                    if (!lower && q == 0) r = make_double2(0.0, 0.0);
                    gp = make_double2(r.x * p, r.y * p);
                } else {
                    const double a = lower ? g.apph[t + 1] : g.amph[t + 1];
                    gp = make_double2((r.x - a * gp.x) * p, (r.y - a * gp.y) * p);
                }
                gs[rs * t] = gp;
            }
        }
    }
    cp_async_wait_group<0>();
    __threadfence();  // the G rows written above, before the cp.async reads below
    // middle row: the upper lane closes it with the lower lane's g'_{m+1}
    const double2 go = make_double2(__shfl_xor_sync(pair, gp.x, 1), __shfl_xor_sync(pair, gp.y, 1));
    double2 xm = make_double2(0.0, 0.0);
    if (!lower) {
        const double2 rm = to_d2(s[rs * m]);
        const double am = g.amph[m + 1], cm = g.apph[m + 1], pm = PP[(long long)m * nl];
        xm = make_double2((rm.x - am * gp.x - cm * go.x) * pm, (rm.y - am * gp.y - cm * go.y) * pm);
        s[rs * m] = from_d2<C>(xm);
    }
    double2 xn = make_double2(__shfl_sync(pair, xm.x, (th & 31) & ~1), __shfl_sync(pair, xm.y, (th & 31) & ~1));
    // backward: upper rows m-1 .. 0, lower rows m+1 .. M-1
    auto brow = [&](int i) { return lower ? m + 1 + i : m - 1 - i; };
    auto issue_b = [&](int b) {
        if (b < nbf) {
#pragma unroll
            for (int u = 0; u < YS_G; ++u) {
                const int i = b * YS_G + u, slot = (b % YS_NG) * YS_G + u;
                if (i < nf) {
                    const int t = brow(i);
                    cp_async16(ringg + slot * YS_NT + th, gs + rs * t);
                    cp_async8(ringf + slot * YS_NT + th, HH + (long long)t * nl);
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll 1
    for (int b = 0; b < YS_NG - 1; ++b) issue_b(b);
#pragma unroll 1
    for (int b = 0; b < nbf; ++b) {
        issue_b(b + YS_NG - 1);
        cp_async_wait_group<YS_NG - 1>();
#pragma unroll
        for (int u = 0; u < YS_G; ++u) {
            const int i = b * YS_G + u, slot = (b % YS_NG) * YS_G + u;
            if (i < nf) {
                const double2 gt = ringg[slot * YS_NT + th];
                const double h = ringf[slot * YS_NT + th];
                xn = make_double2(gt.x - h * xn.x, gt.y - h * xn.y);
                s[rs * brow(i)] = from_d2<C>(xn);
            }
        }
    }
    cp_async_wait_group<0>();
}

// ---------------------------------------------------------------------------
template <int N1, int N2, typename C>
__global__ void __launch_bounds__(PX_NT, px_minb<C>()) k_fftx_inv(Geo g, const C* __restrict__ SP,
                                                    typename CReal<C>::T* __restrict__ DPH) {
    pdl_wait();
    using T = typename CReal<C>::T;
    extern __shared__ __align__(16) unsigned char smp_raw[];
    C* smc = reinterpret_cast<C*>(smp_raw);
    const int L = g.L, M = g.M, LH = g.LH;
    const int LD = fft4s_ld(L);
    const int j0 = 1 + blockIdx.x * PX_TJ;
    const int k = blockIdx.y;
    const int nj = min(PX_TJ, M - j0 + 1);
    const int np = (nj + 1) >> 1;
    // The block's spectrum rows are requested into L2 first, 128-byte lines spread over the
    // threads, so that the loads of the item loop below (a few in flight per thread) find them
    // there: 0.657 -> 0.610 ms per 384 x 256 x 384 FP64 step.  (The same for the five field rows
    // of k_div_fftx made it slower, 1.40 -> 1.47 ms.)
    {
        const int lpr = (LH * (int)sizeof(C) + 127) / 128;
        for (int t = threadIdx.x; t < nj * lpr; t += PX_NT) {
            const int r = t / lpr, c = t - r * lpr;
            prefetch_l2(reinterpret_cast<const char*>(SP + (long long)LH * ((j0 + r - 1) + (long long)M * k)) + 128 * c);
        }
    }
    // Z_k = A_k + i B_k with A_{L-k} = conj A_k; imaginary parts of the k = 0 and
    // k = L/2 coefficients are dropped, as FFT99 does for ISIGN = +1.  Each
    // stored coefficient is read once and gives Z at k and at L - k.
#pragma unroll 2
    for (int p = threadIdx.x; p < np * LH; p += PX_NT) {
        const int pair = p / LH, ks = p - pair * LH;
        const int ja = j0 + 2 * pair;
        const bool hasb = 2 * pair + 1 < nj;
        C a = SP[ks + (long long)LH * ((ja - 1) + (long long)M * k)];
        C b = hasb ? SP[ks + (long long)LH * ((ja) + (long long)M * k)] : mkc((T)0, (T)0);
        C* line = smc + pair * LD;
        if (ks == 0 || 2 * ks == L) {
            a.y = (T)0;
            b.y = (T)0;
        } else {
            line[L - ks] = mkc(a.x - (-b.y), (-a.y) + b.x);
        }
        line[ks] = mkc(a.x - b.y, a.y + b.x);
    }
    block_fft4s<N1, N2, +1>(smc, np, LD, twx_of<C>(g));
    // DPH rows with 16-byte stores (W consecutive points per thread; L is a multiple of 4)
    constexpr int W = V16<T>::W;
    const int LV = L / W;
    for (int p = threadIdx.x; p < nj * LV; p += PX_NT) {
        const int jl = p / LV, i0 = (p - jl * LV) * W;
        const C* z = smc + (jl >> 1) * LD + i0;
        T v[W];
#pragma unroll
        for (int e = 0; e < W; ++e) v[e] = (jl & 1) ? z[e].y : z[e].x;
        st16(DPH + pidx(g, i0, j0 + jl, k), v);
    }
}

// ---------------------------------------------------------------------------
// VELOUPDT_tg + PRCALC_tg + BC_WALL_PR_tg (Q walls are never written).
// Each thread updates W = 16 / sizeof(R) consecutive points of an x line with
// 16-byte loads and stores (L is a multiple of 4); the per-point arithmetic
// is FP64, in the same order for every point.
template <typename R>
__global__ void __launch_bounds__(CR_NT) k_correct(Geo g, R* __restrict__ Q, R* __restrict__ PR,
                                                   const R* __restrict__ DPH, const R* __restrict__ RHSLL,
                                                   const DevState* __restrict__ st, int ns) {
    pdl_wait();
    constexpr int W = V16<R>::W;
    const int L = g.L, M = g.M, N = g.N;
    const unsigned LV = (unsigned)(L / W);
    const long long tot = (long long)LV * M * N;
    const long long t = (long long)blockIdx.x * CR_NT + threadIdx.x;
    if (t >= tot) return;
    const unsigned u = (unsigned)t, r = u / LV, kk = r / (unsigned)M;
    const int i0 = (int)(u - r * LV) * W, j = 1 + (int)(r - kk * (unsigned)M), k = (int)kk;
    const double dt = st->dt, ta = g.talp[ns];
    const long long c = pidx(g, i0, j, k);
    // all loads first: Q is read and written through one pointer
    R ph[W], phk[W], phj[W], uu[W], vv[W], ww[W], pr[W], ll[W];
    ld16(DPH + c, ph);
    ld16(DPH + pidx(g, i0, j, wrapm(k, N)), phk);
    if (j >= 2) ld16(DPH + c - L, phj);
    ld16(Q + c, uu);
    ld16(Q + c + g.FS, vv);
    ld16(Q + c + 2 * g.FS, ww);
    ld16(PR + c, pr);
    ld16(RHSLL + iidx(g, i0, j, k), ll);
    const double phim0 = DPH[pidx(g, wrapm(i0, L), j, k)];
    const double cx = dt * ta * g.dxi, cz = dt * ta * g.dzi, cy = dt * ta * g.dyci[j] / 1.0;
    const double be = 0.5 * ta * dt * g.cvisc * 1.0 / 1.0;
    R uo[W], vo[W], wo[W], pn[W];
#pragma unroll
    for (int e = 0; e < W; ++e) {
        const double p = ph[e], pim = e == 0 ? phim0 : (double)ph[e - 1];
        uo[e] = (R)(uu[e] - (p - pim) * cx);
        wo[e] = (R)(ww[e] - (p - (double)phk[e]) * cz);
        vo[e] = j >= 2 ? (R)(vv[e] - (p - (double)phj[e]) * cy) : vv[e];
        pn[e] = (R)(pr[e] + p - be * ll[e]);
    }
    st16(Q + c, uo);
    st16(Q + c + 2 * g.FS, wo);
    if (j >= 2) st16(Q + c + g.FS, vo);
    st16(PR + c, pn);
    if (j == 1) st16(PR + pidx(g, i0, 0, k), pn);
    if (j == M) st16(PR + pidx(g, i0, M + 1, k), pn);
}
