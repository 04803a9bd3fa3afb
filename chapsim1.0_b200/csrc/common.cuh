// Common definitions for the CHAPSim periodic-channel (TG) step on sm_100a.
//
// Field layout in HBM is the reference's Fortran layout, so that the C ABI
// uploads and downloads the host arrays with one contiguous copy each:
//   F(i, j, k): i = 0..L-1 (x, fastest), j = 0..M+1 (y; 0 and M+1 are the
//   wall ghost planes, 1..M interior), k = 0..N-1 (z).
//   offset = i + L * (j + (M + 2) * k)      ("padded" fields: Q, PR, DPH)
// Work arrays without ghosts (RHS, CONVH0, RHSLLPHI) use
//   offset = i + L * ((j - 1) + M * k)      ("interior" fields).
// Spectral array of the Poisson solve (kx = 0..L/2, y row j, kz):
//   offset = kx + LH * ((j - 1) + M * kz),  LH = L/2 + 1, complex double2.
#pragma once
#include <utility>
#include <cuda_runtime.h>
#include <stdint.h>

#define CHS_WARP 32

// error bits written by kernels into DevState::err
#define CHS_EBIT_NAN 1u
#define CHS_EBIT_DT_COLLAPSE 2u
#define CHS_EBIT_MMA_TIMEOUT 8u  // a bounded device wait (tensor-core commit or bulk copy) ran out

struct DevState {
    double dt;       // current DT (BCAST_COMM_STEP)
    double dt0;      // DT0
    double dtmin;    // DTMIN
    double cflgv;    // CFLGV
    double cflmm;    // last CFL maximum
    double maxdiv;   // last DIVGCK result
    double bulksum;  // sum of RHS_u / DYFI over the grid (RHS_CvLpGpS_tg :168-181)
    double dtprev;   // DT of the previous step, read by the fused dt/factor kernel
    unsigned int err;
    unsigned int ctr; // block-completion counter of the bulk-flux reduction
};

// Geometry and constant coefficients of one channel (passed by value).
struct Geo {
    int L, M, N, LH;
    // x layout: LI interior columns; xo = 0 in the x-periodic domains (L = LI), xo = 1 in the
    // main domain with inflow and outflow, whose rows hold the ghost columns 0 and LI + 1 of
    // NCL1S:NCL1E (L = LI + 2 is then the row stride and LH = LI the count of x modes)
    int LI, xo;
    long long P;    // L*(M+2): k-plane stride of padded fields
    long long FS;   // P*N: size of one padded field
    long long PI_;  // L*M: k-plane stride of interior fields
    long long FI;   // L*M*N: size of one interior field
    double dxi, dzi, dxqi, dzqi, cvisc, volm, cf_given;
    int iflowdriven;
    int fix_v_wall_row;
    // y-direction arrays, indexed by the reference's 1-based j (entry 0 unused)
    const double* dyfi;  // [M+2]
    const double* dyci;  // [M+2]
    const double* wff;   // [M+2]
    const double* wfb;   // [M+2]
    const double* amph;  // [M+2]
    const double* acph;
    const double* apph;
    const double* amvr;  // [3][M+2]
    const double* acvr;
    const double* apvr;
    const double* ak1;   // [L]  modified wavenumbers in x, 0-based kx
    const double* ak3;   // [N]  modified wavenumbers in z, 0-based kz
    double tgam[4], troh[4], talp[4];
    double amvr1, apvrn;  // wall-row factors of the Crank-Nicolson y sweep of the main domain
    double area_inlet;    // Area_inlet (src/COORDJR.f90:367-373)
    // FFT twiddles
    const double2* twx;  // [L] exp(-2 pi i e / L)
    const double2* twz;  // [N]
    const float2* twxf;  // FP32 copies (spectral stage of the mixed-precision step)
    const float2* twzf;
    const double* yz;    // [2M] factors of the zero-mode y recurrence (k_ysolve_zero_factors)
};

__device__ __forceinline__ long long pidx(const Geo& g, int i, int j, int k) {
    return (long long)i + (long long)g.L * ((long long)j + (long long)(g.M + 2) * (long long)k);
}
__device__ __forceinline__ long long iidx(const Geo& g, int i, int j, int k) {
    return (long long)i + (long long)g.L * ((long long)(j - 1) + (long long)g.M * (long long)k);
}
// Point index t = i + L*((j-1) + M*k) of the interior to (i, j, k).  Grids
// have at most 384^3 < 2^31 points, so 32-bit unsigned division is exact
// (and an order of magnitude cheaper than 64-bit division on the GPU).
// In the inflow/outflow main domain t runs over the LI interior columns and i is the
// storage column 1..LI.
__device__ __forceinline__ void io_decode(const Geo& g, long long t, int& i, int& j, int& k) {
    const unsigned u = (unsigned)t, L = (unsigned)g.LI, M = (unsigned)g.M;
    const unsigned r = u / L;
    i = (int)(u - r * L) + g.xo;
    const unsigned kk = r / M;
    j = 1 + (int)(r - kk * M);
    k = (int)kk;
}
// x neighbours of storage column i in the main-domain kernels: cyclic in the x-periodic
// domains, the ghost columns 0 and LI + 1 with inflow and outflow (IPV_io / IMV_io,
// src/INDEXSET.f90:26-52)
__device__ __forceinline__ int xpn(const Geo& g, int i) { return g.xo ? i + 1 : (i + 1 == g.L ? 0 : i + 1); }
__device__ __forceinline__ int xmn(const Geo& g, int i) { return g.xo ? i - 1 : (i == 0 ? g.L - 1 : i - 1); }
// interior-array index (RHS, EXPLT0, RHSLLPHI) of storage point (i, j, k)
__device__ __forceinline__ long long io_iidx(const Geo& g, int i, int j, int k) {
    return (long long)(i - g.xo) + (long long)g.LI * ((long long)(j - 1) + (long long)g.M * (long long)k);
}
// number of interior points
__device__ __forceinline__ long long io_points(const Geo& g) { return (long long)g.LI * g.M * g.N; }
// 16-byte vector access of W = 16 / sizeof(R) consecutive elements (float4 or
// double2); p must be 16-byte aligned
template <typename R> struct V16 { static constexpr int W = 16 / (int)sizeof(R); };
__device__ __forceinline__ void ld16(const float* p, float (&a)[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
}
__device__ __forceinline__ void ld16(const double* p, double (&a)[2]) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a[0] = v.x; a[1] = v.y;
}
__device__ __forceinline__ void st16(float* p, const float (&a)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(a[0], a[1], a[2], a[3]);
}
__device__ __forceinline__ void st16(double* p, const double (&a)[2]) {
    *reinterpret_cast<double2*>(p) = make_double2(a[0], a[1]);
}

__device__ __forceinline__ int wrapp(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__device__ __forceinline__ int wrapm(int i, int n) { return i == 0 ? n - 1 : i - 1; }

// Deterministic block reduction (fixed tree order) of one double per thread.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sbuf) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sbuf[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = (l < NT / 32) ? sbuf[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}
template <int NT>
__device__ __forceinline__ double block_max(double v, double* sbuf) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sbuf[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = (l < NT / 32) ? sbuf[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    return r;
}

// ---- shared-memory barriers and the bulk-copy (TMA) engine ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// orders this thread's generic-proxy shared-memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for phase `parity` of the mbarrier, for at most ~2^31 clocks; returns
// false (and sets the error bit) when the budget runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, unsigned int* err) {
    const long long t0 = clock64();
    uint32_t done = 0;
    while (true) {
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}" : "=r"(done) : "r"(smem_u32(mbar)), "r"(parity) : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 31)) {
            atomicOr(err, CHS_EBIT_MMA_TIMEOUT);
            return false;
        }
    }
}

// mbar_wait by every lane of a warp, with one outcome for the whole warp: the
// lanes leave the wait together, so a warp-collective instruction after it
// (tcgen05.ld, shuffles) never sees a split warp, even when a budget ran out
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* mbar, uint32_t parity, unsigned int* err) {
    return __all_sync(0xffffffffu, mbar_wait(mbar, parity, err));
}

// one arrival that also announces `bytes` of bulk-copy traffic on the mbarrier
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes) : "memory");
}

// Bulk copy (no tensor map, no multicast) of `bytes` (a multiple of 16, both
// addresses 16-byte aligned) from global to this CTA's shared memory,
// completing on the mbarrier.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(mbar)) : "memory");
}

// Programmatic dependent launch.  A kernel of the time step starts with
// pdl_wait() (griddepcontrol.wait: returns once the preceding kernel in the
// stream has completed and its writes are visible; at once when the kernel
// was launched without the attribute), so no step kernel touches global
// memory before its predecessor is done; launched with the attribute, its
// launch overlaps the end of the predecessor.  The predecessors trigger
// implicitly as their blocks exit: an explicit early trigger
// (griddepcontrol.launch_dependents at kernel entry) measured slower, 0.808
// against 0.751 ms per 128^3 step, as the waiting blocks held SM resources.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launch with programmatic stream serialisation allowed (pdl) or as a plain launch.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// Hint that a cache line is about to be read (no register or completion cost).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// 8-byte asynchronous global -> shared copy (no register staging).
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// waits until at most N committed groups of this thread are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}
// one element of a float or double array
__device__ __forceinline__ void cp_async_el(double* smem_dst, const double* gsrc) { cp_async8(smem_dst, gsrc); }
__device__ __forceinline__ void cp_async_el(float* smem_dst, const float* gsrc) { cp_async4(smem_dst, gsrc); }
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
