// Fused plane transforms of the pressure Poisson solve, for grids whose
// half-spectrum plane (L/2+1) x N fits in one block's shared memory.
//
// The periodic-channel Poisson solve (FFT99_POIS3D_periodicxz,
// src/possion3d_FFT99.f90:271-505) transforms every y row j in x (real) and
// then in z (complex) before the per-mode y solves, and back afterwards.
// The chained form (k_div_fftx, k_fftz<-1>, ..., k_fftz<+1>, k_fftx_inv)
// moves the spectrum through HBM between the x and the z transforms.  Here
// one block owns a whole row j:
//   k_div_fft2  DIVG_tg for the x-z plane of row j (RHSLLPHI written once),
//               x transform of z-line pairs (two real lines k = 2p, 2p+1
//               packed into one complex line), unpacking into z lines of the
//               half spectrum, z transform, spectrum of row j written once;
//   k_fft2_inv  the inverse: z transform of the row's half spectrum, the
//               Hermitian repacking of z-line pairs into complex x lines (the
//               imaginary parts of the kx = 0 and kx = L/2 coefficients are
//               dropped, as FFT99 does for ISIGN = +1), x transform, DPH of
//               row j.
// The transforms, their twiddles and scalings (1/L in the x unpacking, 1/N
// after the forward z transform) are those of the chained kernels; only the
// pairing of real lines differs (z pairs here, y pairs there), which changes
// round-off only.  The grid is one block per row (M blocks); the autotuner
// keeps the chained form where that is faster.
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "poisson.cuh"

#define P2_NT 512
// Threads per block: 512 in FP64 (the transforms need ~128 registers), 1024
// in FP32 (within 64 registers), twice the warps to hide the latency of the
// one block per row: the fused pressure stage 52 -> 51 us, the mixed 128^3
// step 0.489 -> 0.483-0.486 ms over two runs.  The FP32 192 x 192 plane
// keeps 512 threads: within 64 registers it would spill ~500 B.
template <typename C, int LN> __host__ __device__ constexpr int p2_nt() {
    return sizeof(C) == 8 && LN < 192 * 192 ? 1024 : P2_NT;
}

// complex words of shared memory: the packed x lines (N/2 pairs of stride
// fft4s_ld(L)) and the z lines (L/2+1 of stride fft4s_ld(N)) share one buffer
__host__ __device__ inline int plane_fft_words(int L, int N) {
    const int a = (N / 2) * fft4s_ld(L), b = (L / 2 + 1) * fft4s_ld(N);
    return a > b ? a : b;
}

template <typename R, int NX1, int NX2, int NZ1, int NZ2>
__global__ void __launch_bounds__((p2_nt<SpecT<R>, NX1 * NX2 * NZ1 * NZ2>()), 1) k_div_fft2(Geo g, const R* __restrict__ Q, R* __restrict__ RHSLL,
                                                       SpecT<R>* __restrict__ SP, const DevState* __restrict__ st,
                                                       int ns) {
    pdl_wait();
    using C = SpecT<R>;
    using T = typename CReal<C>::T;
    constexpr int NT = p2_nt<C, NX1 * NX2 * NZ1 * NZ2>();
    constexpr int L = NX1 * NX2, N = NZ1 * NZ2, LH = L / 2 + 1, NP = N / 2;
    constexpr int LDX = L + NX2 + 1, LDZ = N + NZ2 + 1;
    constexpr int NTASK = NP * LH, TPT = (NTASK + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smp_raw[];
    C* smc = reinterpret_cast<C*>(smp_raw);
    const int M = g.M;
    const int j = 1 + blockIdx.x;
    const double coe0 = 1.0 / (st->dt * g.talp[ns]);
    const double coe1 = g.dxi / 1.0;
    const double coe2 = g.dyfi[j] / 1.0;
    const R* U = Q;
    const R* V = Q + g.FS;
    const R* W = Q + 2 * g.FS;
    // 1. divergence of row j; pair p holds k = 2p (real part) and k = 2p + 1 (imaginary part)
#pragma unroll 4
    for (int p = threadIdx.x; p < N * L; p += NT) {
        const int k = p / L, i = p - k * L;
        const long long c = pidx(g, i, j, k);
        const double u = U[c], up = U[pidx(g, wrapp(i, L), j, k)];
        const double v = V[c], vp = V[c + L];
        const double w = W[c], wp = W[pidx(g, i, j, wrapp(k, N))];
        const double dv = (up - u) * coe1 + (vp - v) * coe2 + (wp - w) * g.dzi;
        const double val = dv * coe0;
        RHSLL[iidx(g, i, j, k)] = (R)val;
        C* line = smc + (k >> 1) * LDX;
        if ((k & 1) == 0) line[i].x = (T)val; else line[i].y = (T)val;
    }
    block_fft4s<NX1, NX2, -1>(smc, NP, LDX, twx_of<C>(g));
    // 2. unpack A_k = (Z_k + conj Z_{L-k}) / 2, B_k = (Z_k - conj Z_{L-k}) / (2i), times 1/L,
    //    into z line kx (at kx * LDZ), elements 2p and 2p + 1; the two layouts overlap, so
    //    every read lands in registers before the barrier and every write follows it
    const T sc = (T)(0.5 / (double)L);
    C av[TPT], bv[TPT];
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
        const int t = threadIdx.x + u * NT;
        if (t < NTASK) {
            const int pair = t / LH, kx = t - pair * LH;
            const C* line = smc + pair * LDX;
            const C z = line[kx];
            const C zc = line[kx == 0 ? 0 : L - kx];
            av[u] = mkc((z.x + zc.x) * sc, (z.y - zc.y) * sc);
            bv[u] = mkc((z.y + zc.y) * sc, (zc.x - z.x) * sc);
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
        const int t = threadIdx.x + u * NT;
        if (t < NTASK) {
            const int pair = t / LH, kx = t - pair * LH;
            smc[kx * LDZ + 2 * pair] = av[u];
            smc[kx * LDZ + 2 * pair + 1] = bv[u];
        }
    }
    block_fft4s<NZ1, NZ2, -1>(smc, LH, LDZ, twz_of<C>(g));
    // 3. spectrum of row j, scaled by 1/N: SP[kx + LH*((j-1) + M*kz)]
    const T sz = (T)(1.0 / (double)N);
    for (int p = threadIdx.x; p < LH * N; p += NT) {
        const int kz = p / LH, kx = p - kz * LH;
        C v = smc[kx * LDZ + kz];
        v.x = v.x * sz;
        v.y = v.y * sz;
        SP[kx + (long long)LH * ((j - 1) + (long long)M * kz)] = v;
    }
}

template <int NX1, int NX2, int NZ1, int NZ2, typename C>
__global__ void __launch_bounds__((p2_nt<C, NX1 * NX2 * NZ1 * NZ2>()), 1) k_fft2_inv(Geo g, const C* __restrict__ SP,
                                                       typename CReal<C>::T* __restrict__ DPH) {
    pdl_wait();
    using T = typename CReal<C>::T;
    constexpr int NT = p2_nt<C, NX1 * NX2 * NZ1 * NZ2>();
    constexpr int L = NX1 * NX2, N = NZ1 * NZ2, LH = L / 2 + 1, NP = N / 2;
    constexpr int LDX = L + NX2 + 1, LDZ = N + NZ2 + 1;
    constexpr int NTASK = NP * LH, TPT = (NTASK + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smp_raw[];
    C* smc = reinterpret_cast<C*>(smp_raw);
    const int M = g.M;
    const int j = 1 + blockIdx.x;
    // 1. row j of the spectrum into z lines (line kx at kx * LDZ)
    for (int p = threadIdx.x; p < LH * N; p += NT) {
        const int kz = p / LH, kx = p - kz * LH;
        const C* src = SP + kx + (long long)LH * ((j - 1) + (long long)M * kz);
        if constexpr (sizeof(C) == 16) cp_async16(smc + kx * LDZ + kz, src);
        else cp_async8(reinterpret_cast<double*>(smc + kx * LDZ + kz), reinterpret_cast<const double*>(src));
    }
    cp_async_wait_all();
    block_fft4s<NZ1, NZ2, +1>(smc, LH, LDZ, twz_of<C>(g));
    // 2. x line of pair p (at p * LDX): element kk = a_kk + i b_kk with a, b the spectra of
    //    z lines 2p and 2p + 1 and a_{L-k} = conj a_k; reads before the barrier, writes after
    C xa[TPT], xb[TPT];
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
        const int t = threadIdx.x + u * NT;
        if (t < NTASK) {
            const int pair = t / LH, ks = t - pair * LH;
            C a = smc[ks * LDZ + 2 * pair];
            C b = smc[ks * LDZ + 2 * pair + 1];
            if (ks == 0 || 2 * ks == L) { a.y = (T)0; b.y = (T)0; }
            xa[u] = a;
            xb[u] = b;
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
        const int t = threadIdx.x + u * NT;
        if (t < NTASK) {
            const int pair = t / LH, ks = t - pair * LH;
            const C a = xa[u], b = xb[u];
            smc[pair * LDX + ks] = mkc(a.x - b.y, a.y + b.x);
            if (ks > 0 && 2 * ks < L) smc[pair * LDX + (L - ks)] = mkc(a.x + b.y, b.x - a.y);
        }
    }
    block_fft4s<NX1, NX2, +1>(smc, NP, LDX, twx_of<C>(g));
    // 3. DPH of row j: pair p gives k = 2p (real part) and 2p + 1 (imaginary part)
    for (int p = threadIdx.x; p < N * L; p += NT) {
        const int k = p / L, i = p - k * L;
        const C z = smc[(k >> 1) * LDX + i];
        DPH[pidx(g, i, j, k)] = (k & 1) ? z.y : z.x;
    }
}

// Host dispatch over the (L, N) plane shapes the fused kernels are built for:
// defines constexpr XN1, XN2 (x split) and ZN1, ZN2 (z split) for KERNEL_CALL.
#define P2_DISPATCH_N(n_, KERNEL_CALL)                                          \
    switch (n_) {                                                               \
        case 64: { constexpr int ZN1 = 8, ZN2 = 8; KERNEL_CALL; } break;        \
        case 96: { constexpr int ZN1 = 12, ZN2 = 8; KERNEL_CALL; } break;       \
        case 128: { constexpr int ZN1 = 16, ZN2 = 8; KERNEL_CALL; } break;      \
        case 192: { constexpr int ZN1 = 16, ZN2 = 12; KERNEL_CALL; } break;     \
        default: break;                                                         \
    }
#define P2_DISPATCH(l_, n_, KERNEL_CALL)                                                  \
    switch (l_) {                                                                         \
        case 64: { constexpr int XN1 = 8, XN2 = 8; P2_DISPATCH_N(n_, KERNEL_CALL) } break;    \
        case 96: { constexpr int XN1 = 12, XN2 = 8; P2_DISPATCH_N(n_, KERNEL_CALL) } break;   \
        case 128: { constexpr int XN1 = 16, XN2 = 8; P2_DISPATCH_N(n_, KERNEL_CALL) } break;  \
        case 192: { constexpr int XN1 = 16, XN2 = 12; P2_DISPATCH_N(n_, KERNEL_CALL) } break; \
        default: break;                                                                   \
    }
// compile-time form of plane_fft_words(L, N) * sizeof(C) <= 220 KB: the
// kernels are instantiated only for the shapes whose plane fits one block
template <typename C, int XN1, int XN2, int ZN1, int ZN2>
constexpr bool plane_fft_fits() {
    constexpr int L = XN1 * XN2, N = ZN1 * ZN2;
    constexpr int a = (N / 2) * (L + XN2 + 1), b = (L / 2 + 1) * (N + ZN2 + 1);
    return (size_t)(a > b ? a : b) * sizeof(C) <= (size_t)220 * 1024;
}
template <typename R, int XN1, int XN2, int ZN1, int ZN2>
cudaError_t plane_fft_attrs(cudaError_t (*set)(const void*, size_t), size_t bytes) {
    using C = SpecT<R>;
    if constexpr (plane_fft_fits<C, XN1, XN2, ZN1, ZN2>()) {
        cudaError_t e = set((const void*)k_div_fft2<R, XN1, XN2, ZN1, ZN2>, bytes);
        if (e == cudaSuccess) e = set((const void*)k_fft2_inv<XN1, XN2, ZN1, ZN2, C>, bytes);
        return e;
    }
    return cudaErrorInvalidValue;
}
template <typename R, int XN1, int XN2, int ZN1, int ZN2>
void plane_fft_fwd(bool pdl, const Geo& g, const R* Q, R* RHSLL, SpecT<R>* SP, const DevState* st, int ns,
                   size_t smem, cudaStream_t s) {
    if constexpr (plane_fft_fits<SpecT<R>, XN1, XN2, ZN1, ZN2>())
        launch_pdl(pdl, k_div_fft2<R, XN1, XN2, ZN1, ZN2>, g.M, (p2_nt<SpecT<R>, XN1 * XN2 * ZN1 * ZN2>()), smem, s, g, Q, RHSLL, SP, st, ns);
}
template <typename C, int XN1, int XN2, int ZN1, int ZN2>
void plane_fft_inv(bool pdl, const Geo& g, const C* SP, typename CReal<C>::T* DPH, size_t smem, cudaStream_t s) {
    if constexpr (plane_fft_fits<C, XN1, XN2, ZN1, ZN2>())
        launch_pdl(pdl, k_fft2_inv<XN1, XN2, ZN1, ZN2, C>, g.M, (p2_nt<C, XN1 * XN2 * ZN1 * ZN2>()), smem, s, g, SP, DPH);
}
inline bool plane_fft_shape(int L, int N) {
    return (L == 64 || L == 96 || L == 128 || L == 192) && (N == 64 || N == 96 || N == 128 || N == 192);
}
