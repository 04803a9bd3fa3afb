// Fused plane transforms of the pressure Poisson solve for planes too large
// for one block: the x-z plane of a y row is split over a thread-block
// cluster of CS blocks, and the transpose between the x and the z transforms
// goes through distributed shared memory (the blocks of a cluster store into
// each other's shared memory) instead of through HBM.
//
// The arithmetic is that of k_div_fft2 / k_fft2_inv (plane_fft.cuh): the same
// transforms, twiddles, scalings and z-line pairing; only the division of the
// work between blocks differs.
//   k_div_fft2c  block r of the cluster of row j: DIVG_tg on the z lines
//                k in [r NK, (r+1) NK) (NK = N / CS), written to RHSLLPHI;
//                x transforms of their NK/2 packed pairs; unpacking of every
//                kx and delivery of the two z values to the block that owns
//                kx (kx in [r' KXC, (r'+1) KXC), KXC = ceil((L/2+1) / CS));
//                cluster barrier; z transforms of the owned kx lines; the
//                spectrum of row j for those kx.
//   k_fft2c_inv  the inverse: z transforms of the owned kx lines of row j;
//                Hermitian repacking of z-line pairs into complex x lines,
//                delivered to the block that owns the pair's k (the imaginary
//                parts of the kx = 0 and kx = L/2 coefficients are dropped,
//                as FFT99 does for ISIGN = +1); cluster barrier; x
//                transforms; DPH of the owned z lines.
// Remote stores start only after a cluster barrier that every block joined
// at its entry (a block's shared memory exists once it has started), and no
// block touches another's shared memory after the second barrier, so a
// block may exit as soon as it is done.  The cluster uses no TMA and no
// multicast.  Grid: CS x M blocks, cluster (CS, 1, 1), one block per SM.
#pragma once
#include <cooperative_groups.h>
#include "common.cuh"
#include "fft.cuh"
#include "poisson.cuh"

// Threads per block: 512 in FP32; 256 in FP64, whose transforms need more
// than the 128 registers a 512-thread block leaves them (a cluster block has
// at most NK/2 = 24 x lines and 25 z lines, which 256 threads still cover in
// one or two passes of each transform step).
template <typename C> __host__ __device__ constexpr int p2c_nt() { return sizeof(C) == 8 ? 512 : 256; }

__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_arrive_release() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// shared-memory layout of one block: NK/2 packed x lines of stride L + NX2 + 1,
// then KXC z lines of stride N + NZ2 + 1 (complex words)
template <int NX1, int NX2, int NZ1, int NZ2, int CS>
struct P2cShape {
    static constexpr int L = NX1 * NX2, N = NZ1 * NZ2, LH = L / 2 + 1;
    static constexpr int NK = N / CS, NPL = NK / 2;
    static constexpr int KXC = (LH + CS - 1) / CS;
    static constexpr int LDX = L + NX2 + 1, LDZ = N + NZ2 + 1;
    static constexpr int WORDS = NPL * LDX + KXC * LDZ;
    static_assert(N % (2 * CS) == 0, "each block owns whole pairs of z lines");
};

template <typename C, int NX1, int NX2, int NZ1, int NZ2, int CS>
constexpr size_t p2c_smem() {
    return (size_t)P2cShape<NX1, NX2, NZ1, NZ2, CS>::WORDS * sizeof(C);
}

template <typename R, int NX1, int NX2, int NZ1, int NZ2, int CS>
__global__ void __launch_bounds__(p2c_nt<SpecT<R>>(), 1) k_div_fft2c(Geo g, const R* __restrict__ Q, R* __restrict__ RHSLL,
                                                         SpecT<R>* __restrict__ SP, const DevState* __restrict__ st,
                                                         int ns) {
    pdl_wait();
    cluster_arrive_relaxed();  // this block has started: the others may store into its shared memory
    namespace cg = cooperative_groups;
    using C = SpecT<R>;
    using T = typename CReal<C>::T;
    using S = P2cShape<NX1, NX2, NZ1, NZ2, CS>;
    constexpr int NT = p2c_nt<C>();
    constexpr int L = S::L, N = S::N, LH = S::LH, NK = S::NK, NPL = S::NPL, KXC = S::KXC;
    constexpr int LDX = S::LDX, LDZ = S::LDZ;
    extern __shared__ __align__(16) unsigned char p2c_raw[];
    C* const xb = reinterpret_cast<C*>(p2c_raw);
    C* const zb = xb + NPL * LDX;
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const int M = g.M;
    const int j = 1 + blockIdx.y;
    const int kbase = r * NK;
    const double coe0 = 1.0 / (st->dt * g.talp[ns]);
    const double coe1 = g.dxi / 1.0;
    const double coe2 = g.dyfi[j] / 1.0;
    const R* U = Q;
    const R* V = Q + g.FS;
    const R* Wf = Q + 2 * g.FS;
    // 1. divergence of the block's z lines: pair p holds k = kbase + 2p (real part) and
    //    kbase + 2p + 1 (imaginary part); VW points of both lines per item, 16-byte loads
    constexpr int VW = V16<R>::W;
    constexpr int LV = L / VW;
#pragma unroll 2
    for (int p = threadIdx.x; p < NPL * LV; p += NT) {
        const int pair = p / LV, i0 = (p - pair * LV) * VW;
        T val[2][VW];
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            const int k = kbase + 2 * pair + part;
            const long long c = pidx(g, i0, j, k);
            R u[VW], v[VW], vp[VW], w[VW], wp[VW], out[VW];
            ld16(U + c, u);
            ld16(V + c, v);
            ld16(V + c + L, vp);
            ld16(Wf + c, w);
            ld16(Wf + pidx(g, i0, j, wrapp(k, N)), wp);
            const double un = U[pidx(g, i0 + VW == L ? 0 : i0 + VW, j, k)];
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
        }
        C* line = xb + pair * LDX + i0;
#pragma unroll
        for (int e = 0; e < VW; ++e) line[e] = mkc(val[0][e], val[1][e]);
    }
    block_fft4s<NX1, NX2, -1>(xb, NPL, LDX, twx_of<C>(g));
    // 2. A_kx = (Z_kx + conj Z_{L-kx}) / 2, B_kx = (Z_kx - conj Z_{L-kx}) / (2i), times 1/L:
    //    elements kbase + 2p and kbase + 2p + 1 of z line kx, in the block that owns kx
    cluster_wait_acquire();  // every block of the cluster has started
    const T sc = (T)(0.5 / (double)L);
    for (int t = threadIdx.x; t < NPL * LH; t += NT) {
        const int pair = t / LH, kx = t - pair * LH;
        const C* line = xb + pair * LDX;
        const C z = line[kx];
        const C zc = line[kx == 0 ? 0 : L - kx];
        const int owner = kx / KXC, lk = kx - owner * KXC;
        C* dst = cl.map_shared_rank(zb, owner) + lk * LDZ + kbase + 2 * pair;
        dst[0] = mkc((z.x + zc.x) * sc, (z.y - zc.y) * sc);
        dst[1] = mkc((z.y + zc.y) * sc, (zc.x - z.x) * sc);
    }
    cluster_arrive_release();
    cluster_wait_acquire();  // the z lines of this block are complete
    const int kx0 = r * KXC;
    const int nkx = LH - kx0 < KXC ? (LH - kx0 > 0 ? LH - kx0 : 0) : KXC;
    block_fft4s<NZ1, NZ2, -1>(zb, nkx, LDZ, twz_of<C>(g));
    // 3. spectrum of row j for the owned kx, scaled by 1/N: SP[kx + LH*((j-1) + M*kz)]
    const T sz = (T)(1.0 / (double)N);
    for (int p = threadIdx.x; p < nkx * N; p += NT) {
        const int kz = p / nkx, lk = p - kz * nkx;
        C v = zb[lk * LDZ + kz];
        v.x = v.x * sz;
        v.y = v.y * sz;
        SP[(kx0 + lk) + (long long)LH * ((j - 1) + (long long)M * kz)] = v;
    }
}

template <int NX1, int NX2, int NZ1, int NZ2, int CS, typename C>
__global__ void __launch_bounds__(p2c_nt<C>(), 1) k_fft2c_inv(Geo g, const C* __restrict__ SP,
                                                         typename CReal<C>::T* __restrict__ DPH) {
    pdl_wait();
    cluster_arrive_relaxed();
    namespace cg = cooperative_groups;
    using T = typename CReal<C>::T;
    using S = P2cShape<NX1, NX2, NZ1, NZ2, CS>;
    constexpr int NT = p2c_nt<C>();
    constexpr int L = S::L, N = S::N, LH = S::LH, NK = S::NK, NPL = S::NPL, KXC = S::KXC;
    constexpr int LDX = S::LDX, LDZ = S::LDZ;
    extern __shared__ __align__(16) unsigned char p2c_raw[];
    C* const xb = reinterpret_cast<C*>(p2c_raw);
    C* const zb = xb + NPL * LDX;
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const int M = g.M;
    const int j = 1 + blockIdx.y;
    const int kbase = r * NK;
    const int kx0 = r * KXC;
    const int nkx = LH - kx0 < KXC ? (LH - kx0 > 0 ? LH - kx0 : 0) : KXC;
    // 1. the owned kx of row j into z lines (line lk at lk * LDZ)
    for (int p = threadIdx.x; p < nkx * N; p += NT) {
        const int kz = p / nkx, lk = p - kz * nkx;
        const C* src = SP + (kx0 + lk) + (long long)LH * ((j - 1) + (long long)M * kz);
        if constexpr (sizeof(C) == 16) cp_async16(zb + lk * LDZ + kz, src);
        else cp_async8(reinterpret_cast<double*>(zb + lk * LDZ + kz), reinterpret_cast<const double*>(src));
    }
    cp_async_wait_all();
    block_fft4s<NZ1, NZ2, +1>(zb, nkx, LDZ, twz_of<C>(g));
    // 2. x line of pair p: element ks = a_ks + i b_ks with a, b the spectra of z lines 2p and
    //    2p + 1 and a_{L-ks} = conj a_ks, stored in the block that owns k = 2p
    cluster_wait_acquire();  // every block of the cluster has started
    constexpr int NP = N / 2;
    for (int t = threadIdx.x; t < nkx * NP; t += NT) {
        const int lk = t / NP, pg = t - lk * NP;
        C a = zb[lk * LDZ + 2 * pg];
        C b = zb[lk * LDZ + 2 * pg + 1];
        const int ks = kx0 + lk;
        if (ks == 0 || 2 * ks == L) { a.y = (T)0; b.y = (T)0; }
        const int owner = (2 * pg) / NK, pl = pg - owner * NPL;
        C* xl = cl.map_shared_rank(xb, owner) + pl * LDX;
        xl[ks] = mkc(a.x - b.y, a.y + b.x);
        if (ks > 0 && 2 * ks < L) xl[L - ks] = mkc(a.x + b.y, b.x - a.y);
    }
    cluster_arrive_release();
    cluster_wait_acquire();  // the x lines of this block are complete
    block_fft4s<NX1, NX2, +1>(xb, NPL, LDX, twx_of<C>(g));
    // 3. DPH of the owned z lines: pair p gives k = kbase + 2p (real part) and kbase + 2p + 1
    constexpr int VW = V16<T>::W;
    constexpr int LV = L / VW;
    for (int p = threadIdx.x; p < NPL * LV; p += NT) {
        const int pair = p / LV, i0 = (p - pair * LV) * VW;
        const C* line = xb + pair * LDX + i0;
        T o0[VW], o1[VW];
#pragma unroll
        for (int e = 0; e < VW; ++e) {
            const C z = line[e];
            o0[e] = z.x;
            o1[e] = z.y;
        }
        const int k = kbase + 2 * pair;
        st16(DPH + pidx(g, i0, j, k), o0);
        st16(DPH + pidx(g, i0, j, k + 1), o1);
    }
}

// Cluster size of the fused plane transforms for an (L, N) plane whose half
// spectrum does not fit one block: the smallest of 8 and 16 whose block
// shared memory fits 220 KB (0 when neither does, or N is not a multiple of
// 2 CS).  8 is the portable maximum; 16 needs the non-portable cluster size.
template <typename C, int NX1, int NX2, int NZ1, int NZ2>
constexpr int p2c_cluster() {
    constexpr int N = NZ1 * NZ2;
    if constexpr (N % 16 == 0 && p2c_smem<C, NX1, NX2, NZ1, NZ2, 8>() <= (size_t)220 * 1024) return 8;
    if constexpr (N % 32 == 0 && p2c_smem<C, NX1, NX2, NZ1, NZ2, 16>() <= (size_t)220 * 1024) return 16;
    return 0;
}

// launch with the cluster dimension (CS, 1, 1), and programmatic stream serialisation when pdl
template <typename... KArgs, typename... Args>
inline cudaError_t launch_cluster(bool pdl, int cs, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                  cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 2 : 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// Sets the shared-memory (and, for 16, the non-portable cluster size)
// attributes of both kernels and checks that at least one cluster of the
// shape can be resident; false when the shape has no cluster form or the
// device cannot run it.
template <typename R, int NX1, int NX2, int NZ1, int NZ2>
bool plane_fft_cluster_setup(const Geo& g) {
    using C = SpecT<R>;
    constexpr int CS = p2c_cluster<C, NX1, NX2, NZ1, NZ2>();
    if constexpr (CS == 0) {
        return false;
    } else {
        constexpr size_t sm = p2c_smem<C, NX1, NX2, NZ1, NZ2, CS>();
        auto kf = k_div_fft2c<R, NX1, NX2, NZ1, NZ2, CS>;
        auto ki = k_fft2c_inv<NX1, NX2, NZ1, NZ2, CS, C>;
        for (const void* k : {(const void*)kf, (const void*)ki}) {
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return false;
            if (CS > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
                return false;
        }
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(CS, g.M);
        cfg.blockDim = dim3(p2c_nt<C>());
        cfg.dynamicSmemBytes = sm;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CS;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nf = 0, ni = 0;
        if (cudaOccupancyMaxActiveClusters(&nf, kf, &cfg) != cudaSuccess) { cudaGetLastError(); return false; }
        if (cudaOccupancyMaxActiveClusters(&ni, ki, &cfg) != cudaSuccess) { cudaGetLastError(); return false; }
        return nf > 0 && ni > 0;
    }
}

template <typename R, int NX1, int NX2, int NZ1, int NZ2>
void plane_fft_cluster_fwd(bool pdl, const Geo& g, const R* Q, R* RHSLL, SpecT<R>* SP, const DevState* st, int ns,
                           cudaStream_t s) {
    using C = SpecT<R>;
    constexpr int CS = p2c_cluster<C, NX1, NX2, NZ1, NZ2>();
    if constexpr (CS != 0)
        launch_cluster(pdl, CS, k_div_fft2c<R, NX1, NX2, NZ1, NZ2, CS>, dim3(CS, g.M), dim3(p2c_nt<C>()),
                       p2c_smem<C, NX1, NX2, NZ1, NZ2, CS>(), s, g, Q, RHSLL, SP, st, ns);
}
template <typename C, int NX1, int NX2, int NZ1, int NZ2>
void plane_fft_cluster_inv(bool pdl, const Geo& g, const C* SP, typename CReal<C>::T* DPH, cudaStream_t s) {
    constexpr int CS = p2c_cluster<C, NX1, NX2, NZ1, NZ2>();
    if constexpr (CS != 0)
        launch_cluster(pdl, CS, k_fft2c_inv<NX1, NX2, NZ1, NZ2, CS, C>, dim3(CS, g.M), dim3(p2c_nt<C>()),
                       p2c_smem<C, NX1, NX2, NZ1, NZ2, CS>(), s, g, SP, DPH);
}

// (L, N) shapes with a cluster form: lines of 256 or 384 in both directions
#define P2C_DISPATCH_N(n_, KERNEL_CALL)                                         \
    switch (n_) {                                                               \
        case 256: { constexpr int ZN1 = 16, ZN2 = 16; KERNEL_CALL; } break;     \
        case 384: { constexpr int ZN1 = 16, ZN2 = 24; KERNEL_CALL; } break;     \
        default: break;                                                         \
    }
#define P2C_DISPATCH(l_, n_, KERNEL_CALL)                                                   \
    switch (l_) {                                                                           \
        case 256: { constexpr int XN1 = 16, XN2 = 16; P2C_DISPATCH_N(n_, KERNEL_CALL) } break; \
        case 384: { constexpr int XN1 = 16, XN2 = 24; P2C_DISPATCH_N(n_, KERNEL_CALL) } break; \
        default: break;                                                                     \
    }
inline bool plane_fft_cluster_shape(int L, int N) { return (L == 256 || L == 384) && (N == 256 || N == 384); }
