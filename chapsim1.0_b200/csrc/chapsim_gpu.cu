// C ABI, device context and launch sequencing of the periodic-channel step.
// Build: nvcc -gencode arch=compute_100a,code=sm_100a -O3 -shared (see Makefile).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/chapsim_gpu.h"
#include "common.cuh"
#include "diag.cuh"
#include "fft.cuh"
#include "momentum.cuh"
#include "poisson.cuh"
#include "tdma.cuh"
#include "io.cuh"
#include "io_cn.cuh"
#include "io_xinout.cuh"
#include "stats.cuh"
#include "stats_io.cuh"
#include "rhs_bulk.cuh"
#include "plane_fft.cuh"
#include "plane_fft_cluster.cuh"
#include "thermo.cuh"
#include "thermal.cuh"
#include "mlp.cuh"

#include <algorithm>

// x transform reading RHSLLPHI directly (used by chapsim_fft99_pois3d)
template <int N1, int N2>
__global__ void __launch_bounds__(PX_NT, PX_MINB) k_fftx_from_rhs(Geo g, const double* __restrict__ RHSLL, double2* __restrict__ SP) {
    extern __shared__ double2 smc[];
    const int L = g.L, M = g.M, LH = g.LH;
    const int LD = fft4s_ld(L);
    const int j0 = 1 + blockIdx.x * PX_TJ;
    const int k = blockIdx.y;
    const int nj = min(PX_TJ, M - j0 + 1);
    const int np = (nj + 1) >> 1;
    for (int p = threadIdx.x; p < 2 * np * L; p += PX_NT) {
        const int jl = p / L, i = p - jl * L;
        const int pair = jl >> 1, part = jl & 1;
        const double val = jl < nj ? RHSLL[iidx(g, i, j0 + jl, k)] : 0.0;
        double2* line = smc + pair * LD;
        if (part == 0) line[i].x = val; else line[i].y = val;
    }
    block_fft4s<N1, N2, -1>(smc, np, LD, g.twx);
    const double sc = 0.5 / (double)L;
    for (int p = threadIdx.x; p < np * LH; p += PX_NT) {
        const int pair = p / LH, kx = p - pair * LH;
        const double2* line = smc + pair * LD;
        const double2 z = line[kx];
        const double2 zc = line[kx == 0 ? 0 : L - kx];
        const int ja = j0 + 2 * pair;
        SP[kx + (long long)LH * ((ja - 1) + (long long)M * k)] = make_double2((z.x + zc.x) * sc, (z.y - zc.y) * sc);
        if (2 * pair + 1 < nj)
            SP[kx + (long long)LH * ((ja) + (long long)M * k)] = make_double2((z.y + zc.y) * sc, (zc.x - z.x) * sc);
    }
}

// ------------------------- general line solvers (ABI) ------------------------
// Coefficients per point in global memory, element e of line l at off(l) + e*es.
struct GlobalCoef {
    const double *a, *b, *c;
    long long off, es;
    __device__ __forceinline__ double A(int r) const { return a[off + r * es]; }
    __device__ __forceinline__ double B(int r) const { return b[off + r * es]; }
    __device__ __forceinline__ double C(int r) const { return c[off + r * es]; }
};

template <int S, bool CYCLIC>
__global__ void k_tdma_lines(const double* a, const double* b, const double* c, double* r, const double* bcj, int nlines,
                             long long ls, long long es, int n) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nlines) return;
    GlobalCoef cf{a, b, c, (long long)warp * ls, es};
    double d[S];
#pragma unroll
    for (int k = 0; k < S; ++k) d[k] = r[cf.off + (long long)(lane * S + k) * es];
    if (!CYCLIC && bcj) {
        if (lane == 0) d[0] -= cf.A(0) * bcj[warp];
        if (lane == 31) d[S - 1] -= cf.C(n - 1) * bcj[nlines + warp];
    }
    warp_tdma<S, CYCLIC>(d, cf, lane);
#pragma unroll
    for (int k = 0; k < S; ++k) r[cf.off + (long long)(lane * S + k) * es] = d[k];
}

// sequential reference recurrences, one thread per line, for lengths that
// are not 32*S (TDMAIJI_CYC :100-154 and TDMAIJJ_nonCYC :95-121)
__global__ void k_tdma_seq(const double* A, const double* B, const double* C, double* R, const double* bcj, double* wk,
                           int nlines, long long ls, long long es, int n, int cyclic) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const long long o = (long long)l * ls;
#define E(X, i) X[o + (long long)(i) * es]
    double* H0 = wk + (long long)l * 3 * n;
    double* G1 = H0 + n;
    double* G2 = G1 + n;
    if (cyclic) {
        H0[0] = E(C, 0) / E(B, 0); G1[0] = E(R, 0) / E(B, 0); G2[0] = -E(A, 0) / E(B, 0);
        for (int i = 1; i <= n - 3; ++i) {
            double pp = 1.0 / (E(B, i) - H0[i - 1] * E(A, i));
            double q1 = G1[i - 1] * E(A, i), q2 = G2[i - 1] * E(A, i);
            H0[i] = E(C, i) * pp; G1[i] = (E(R, i) - q1) * pp; G2[i] = -q2 * pp;
        }
        {
            int i = n - 2;
            double pp = 1.0 / (E(B, i) - H0[i - 1] * E(A, i));
            double q1 = G1[i - 1] * E(A, i), q2 = G2[i - 1] * E(A, i);
            G1[i] = (E(R, i) - q1) * pp; G2[i] = (-E(C, i) - q2) * pp;
        }
        for (int i = n - 3; i >= 0; --i) { G1[i] = -H0[i] * G1[i + 1] + G1[i]; G2[i] = -H0[i] * G2[i + 1] + G2[i]; }
        int i = n - 1;
        double pp = E(R, i) - E(C, i) * G1[0] - E(A, i) * G1[i - 1];
        double qq = E(B, i) + E(C, i) * G2[0] + E(A, i) * G2[i - 1];
        E(R, i) = pp / qq;
        for (int k = n - 2; k >= 0; --k) E(R, k) = G1[k] + G2[k] * E(R, n - 1);
    } else {
        double b1 = bcj ? bcj[l] : 0.0, b2 = bcj ? bcj[nlines + l] : 0.0;
        H0[0] = E(C, 0) / E(B, 0);
        G1[0] = (E(R, 0) - E(A, 0) * b1) / E(B, 0);
        for (int j = 1; j <= n - 2; ++j) {
            double pp = 1.0 / (E(B, j) - H0[j - 1] * E(A, j));
            H0[j] = E(C, j) * pp;
            G1[j] = (E(R, j) - E(A, j) * G1[j - 1]) * pp;
        }
        int j = n - 1;
        double pp = 1.0 / (E(B, j) - H0[j - 1] * E(A, j));
        G1[j] = (E(R, j) - E(C, j) * b2 - E(A, j) * G1[j - 1]) * pp;
        E(R, j) = G1[j];
        for (int k = n - 2; k >= 0; --k) E(R, k) = G1[k] - H0[k] * E(R, k + 1);
    }
#undef E
}


// Failure-path probe: one warp waits on an mbarrier that nothing arrives at.  The wait is the
// bounded one every tensor-core and bulk-copy stage uses (about 2^31 clocks), so the kernel gives
// up, sets the timeout bit of the error word and returns; no fault, and the context stays usable.
__global__ void k_wait_probe(unsigned int* err) {
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) mbar_init(&mbar, 1);
    __syncthreads();
    (void)mbar_wait_warp(&mbar, 0, err);
}

struct chapsim_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    Geo g{};
    double *Q = nullptr, *PR = nullptr, *H0 = nullptr, *RHS = nullptr, *RHSLL = nullptr, *DPH = nullptr;
    double* yz = nullptr;         // zero-mode factors of the warp y-solve (Geo::yz)
    double* YF = nullptr;         // factors of the sequential y-solve, 2 M doubles per line (when chosen)
    double* YF2 = nullptr;        // factors of the two-way y-solve, 2 M doubles per line (when chosen)
    double* YF3 = nullptr;        // pivots of the scan y-solve, M doubles per line, line by line (when chosen)
    int ysolve_kind = 0;          // 0: warp Thomas/PCR hybrid, 1: sequential Thomas, 2: two-way, 3: sequential with
                                  // the forward intermediate in shared memory at one block per SM, 4: warp affine
                                  // scans over the sequential factors (chapsim_autotune)
    int k1_kind = 0;              // 0: fused k_rhs_xsweep, 1: k_rhs_point + k_xsweep, 2: k_rhs_xsweep_bulk, 3: the wide
                                  // fused form, 16-byte loads (rhs_pv) (chapsim_autotune)
    int plane_kind = 0;           // 0: chained x/z transforms, 1: fused plane transforms k_div_fft2/k_fft2_inv (chapsim_autotune)
    int zs_tw = 32;               // lines per tile of the z sweep, 32 or 16 (chapsim_autotune)
    int zs_il = 1;                // z-sweep tile layout: 1 line-contiguous, 2 lines interleaved in pairs (chapsim_autotune)
    int ys_il = 1;                // the same for the y sweep (chapsim_autotune)
    bool fz_pipe = false;         // persistent double-buffered z transforms (chapsim_autotune)
    bool fz_prefetch = false;     // one-tile z transforms request the tile one wave ahead into L2 (chapsim_autotune)
    bool p2c = false;             // the fused plane transforms run as a thread-block cluster (k_div_fft2c/k_fft2c_inv)
    int rb_nw = 0;                // warps per block of k_rhs_xsweep_bulk (0: the stages do not fit)
    bool pdl = true;              // step kernels launched with programmatic dependent launch
    double2* SP = nullptr;
    float2* SPf = nullptr;       // FP32 spectral array of the mixed-precision step
    float* DPHf = nullptr;       // FP32 pressure increment of the mixed-precision step
    double* part_rhs = nullptr;  // per-block bulk-flux partial sums
    double* fac = nullptr;       // factor tables of the x, z, y sweeps, [substep][set]
    // mixed precision (CHAPSIM_PREC_MIXED): FP32 copies of the momentum-stage
    // fields; the FP64 arrays above then serve as host-transfer staging
    int prec = CHAPSIM_PREC_FP64;
    float *Qf = nullptr, *PRf = nullptr, *H0f = nullptr, *RHSf = nullptr, *RHSLLf = nullptr, *facf = nullptr;
    int npart_rhs = 0;
    double* part_red = nullptr;  // per-block CFL / divergence maxima
    int npart_red = 0;
    DevState* st = nullptr;
    DevState* st_host = nullptr;  // pinned mirror for readback
    double* ybuf = nullptr;       // device copies of y-arrays and wavenumbers
    double2* tw = nullptr;
    float2* twf = nullptr;        // FP32 copies of tw
    int domain = 1;               // 1: periodic TG channel, 2: main domain (IO), 3: main domain with inflow from
                                  // a periodic TG context and a convective outlet (iDomain = 3)
    int ivis = 0;                 // main domain: 0 explicit viscous terms, 1 Crank-Nicolson (iVisScheme)
    // statistics of the periodic channel (stats.cuh), allocated by the first call
    double *pp_inst = nullptr, *pp_avg = nullptr, *pp_part = nullptr, *pp_mon = nullptr;
    int pp_nchunk = 0;
    double *ppio_set = nullptr, *ppio_part = nullptr;  // main-domain means (PPIO_ALL per row) and chunk partials
    int nstatis = 0;              // NSTATIS_TG
    IoFields io{};                // IO-path arrays (domain 2); FP64 staging of G in the mixed-precision step
    IoFieldsT<float> iof{};       // FP32 flow fields of the mixed-precision main-domain step (Q, PR, RHS: Qf, PRf, RHSf)
    int io_grid = 0;              // blocks of the IO point-wise kernels
    cudaGraphExec_t step_exec = nullptr;
    cudaEvent_t* prof_ev = nullptr;  // when set, an event is recorded after every kernel
    int prof_n = 0;
    int kernels_per_step = 0;
    unsigned long long launches = 0;
    int nsm = 148;
    // property table for THERM_PROP_UPDATE (table search)
    void* ptab = nullptr;         // packed rows and keys, one allocation
    PropTab tab{};
    PropStatus* pstat = nullptr;
    double* pbuf = nullptr;       // staging of the host-array entry (7 doubles per point)
    long long pbuf_pts = 0;
    // thermal solver of the IO domain (chapsim_thermal_init)
    bool thermal = false;
    double* DEN = nullptr;        // DENSITY (io.RHO then holds DENSITY0)
    ThermoFields tf{};
    ThermoParams tp{};
    // learned property model
    float *mlp_par = nullptr, *mlp_grad = nullptr, *mlp_m1 = nullptr, *mlp_m2 = nullptr, *mlp_loss = nullptr;
    __nv_bfloat16 *mlp_w2 = nullptr, *mlp_w2t = nullptr, *mlp_w3 = nullptr;
    __half *mlp_w2h = nullptr, *mlp_w3h = nullptr;  // FP16 images for inference (in the same allocation)
    float *mlp_xs = nullptr, *mlp_ys = nullptr;
    double* mlp_dh = nullptr;
    int mlp_cap = 0, mlp_step = 0;
    MlpNorm mlp_norm{};
    bool mlp_ready = false, use_mlp = false;
    int mlp_act = MLP_ACT_TANH;   // hidden-layer activation (chapsim_mlp_set_activation)
    unsigned int* mlp_judge = nullptr;
    // asynchronous field dumps (chapsim_dump_begin / chapsim_dump_write)
    double* dump_dev = nullptr;   // packed interiors of the dumped fields, then dt
    double* dump_host = nullptr;  // pinned copy of dump_dev
    size_t dump_words = 0;
    int dump_nf = 0;
    bool dump_pending = false;
    cudaStream_t dump_stream = nullptr;
    cudaEvent_t dump_snap = nullptr, dump_done = nullptr;
    // pipelined host I/O (chapsim_upload_fields_async / chapsim_download_fields_async): two input and
    // two output staging slots of Q and PR, an H2D and a D2H copy stream, and per slot the events that
    // order the copies against the step stream
    double* pio_in[2] = {nullptr, nullptr};
    double* pio_out[2] = {nullptr, nullptr};
    cudaStream_t pio_h2d = nullptr, pio_d2h = nullptr;
    cudaEvent_t pio_in_ready[2] = {nullptr, nullptr}, pio_in_free[2] = {nullptr, nullptr};
    cudaEvent_t pio_out_ready[2] = {nullptr, nullptr}, pio_out_free[2] = {nullptr, nullptr};
    int pio_in_next = 0, pio_in_pending = 0, pio_in_head = 0, pio_out_next = 0;
    // inflow/outflow main domain (domain 3)
    chapsim_ctx* tg_in = nullptr;  // the periodic TG context whose fields feed the inlet
    double2* xio_tq = nullptr;     // (cos, sin)(pi p / (2L)) of the FFT form of the cosine transforms
    double* xio_cf = nullptr;      // COSQF matrix w_p cos((2m+1) p pi / (2L)), [p][m]; then the COSQB matrix
                                   // 4 cos((2m+1) p pi / (2L)), [m][p] (one allocation, 2 L^2)
    double* xio_bc0 = nullptr;     // BC_CONV0 (3 M N)
    double* xio_yd = nullptr;      // forward factors of the Poisson y-solve (L N M)
    double* xio_state = nullptr;   // U_OUTLET, CHK_Mass_CONSV0_SCALING of the last substep
    double* xio_part = nullptr;    // block maxima of the three divergence ranges
    double* xio_bc0e = nullptr;    // BC_CONV0_ENG (M N)
    double* xio_mpart = nullptr;   // block sums of the interior mass rate (io_grid)
    XioInlet xio_in{};             // inlet state of the thermal solver (chapsim_xinout_thermal_inlet)
    bool xio_in_set = false;
    cudaEvent_t xev[2] = {nullptr, nullptr};
    std::string err;
};

namespace {

thread_local std::string g_init_error;

int fail(chapsim_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_init_error = msg;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(ctx, CHAPSIM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

std::vector<double2> twiddles(int n) {
    std::vector<double2> w(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int e = 0; e < n; ++e) {
        long double a = 2.0L * pi * (long double)e / (long double)n;
        w[e].x = (double)cosl(a);
        w[e].y = (double)(-sinl(a));
    }
    return w;
}

template <typename R> size_t smem_rhs(const Geo& g) { return (size_t)(RHS_WPB * 3 * (g.L + 33)) * sizeof(R); }
template <typename R> size_t smem_z(const Geo& g, int tw) { return (size_t)(2 * tw * (g.N + 33)) * sizeof(R); }
template <typename R> size_t smem_y(const Geo& g) { return (size_t)(32 * (g.M + 33)) * sizeof(R); }
template <typename R> size_t smem_xs(const Geo& g) { return (size_t)((XS_NT / 32) * (g.L + 33)) * sizeof(R); }
template <typename R> size_t smem_rt() { return (size_t)(RT_SLOTS * RT_SLOT) * sizeof(R); }
// planes per k-chunk of the 2.5D right-hand-side kernel: enough blocks to fill
// the GPU, at least 16 planes per chunk where N allows; always divides N
int rt_chunk(const Geo& g) {
    const int tiles = (g.L / RT_I) * (g.M / RT_J);
    int chunk = g.N;
    while (chunk % 2 == 0 && chunk / 2 >= 16 && tiles * (g.N / chunk) < 4 * 148) chunk /= 2;
    return chunk;
}
template <typename C = double2>
size_t smem_px(const Geo& g) { return (size_t)((PX_TJ / 2) * fft4s_ld(g.L)) * sizeof(C); }
template <typename C = double2>
size_t smem_fz(const Geo& g) { return (size_t)(FZ_TQ * fft4s_ld(g.N)) * sizeof(C); }
template <typename C>
size_t smem_fzp(const Geo& g) { return (size_t)(2 * fzp_tq<C>() * fft4s_ld(g.N)) * sizeof(C); }
// the context's pressure increment DPH in the step's real type
template <typename R> R* dph(chapsim_ctx* c);
template <> double* dph<double>(chapsim_ctx* c) { return c->DPH; }
template <> float* dph<float>(chapsim_ctx* c) { return c->DPHf; }
// the context's spectral array of element type C
template <typename C> C* spec(chapsim_ctx* c);
template <> double2* spec<double2>(chapsim_ctx* c) { return c->SP; }
template <> float2* spec<float2>(chapsim_ctx* c) { return c->SPf; }
// fused plane transforms: built for the shape, and the plane fits one block's shared memory
template <typename C>
size_t smem_p2(const Geo& g) { return (size_t)plane_fft_words(g.L, g.N) * sizeof(C); }
template <typename C>
bool plane_fft_ok(const Geo& g) { return plane_fft_shape(g.L, g.N) && smem_p2<C>(g) <= 220 * 1024; }

// twiddles of the small DFTs inside the four-step FFT (constant memory, shared by all contexts)
cudaError_t upload_small_twiddles() {
    const long double pi = 3.141592653589793238462643383279502884L;
    double2 w[24];
    float2 wf[24];
    const int sizes[4] = {8, 12, 16, 24};
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < 4 && e == cudaSuccess; ++s) {
        const int P = sizes[s];
        for (int q = 0; q < P; ++q) {
            const long double a = 2.0L * pi * (long double)q / (long double)P;
            w[q] = make_double2((double)cosl(a), (double)(-sinl(a)));
            wf[q] = make_float2((float)cosl(a), (float)(-sinl(a)));
        }
        if (P == 8) e = cudaMemcpyToSymbol(c_w8, w, sizeof(double2) * 8);
        if (P == 12) e = cudaMemcpyToSymbol(c_w12, w, sizeof(double2) * 12);
        if (P == 16) e = cudaMemcpyToSymbol(c_w16, w, sizeof(double2) * 16);
        if (P == 24) e = cudaMemcpyToSymbol(c_w24, w, sizeof(double2) * 24);
        if (e != cudaSuccess) break;
        if (P == 8) e = cudaMemcpyToSymbol(c_w8f, wf, sizeof(float2) * 8);
        if (P == 12) e = cudaMemcpyToSymbol(c_w12f, wf, sizeof(float2) * 12);
        if (P == 16) e = cudaMemcpyToSymbol(c_w16f, wf, sizeof(float2) * 16);
        if (P == 24) e = cudaMemcpyToSymbol(c_w24f, wf, sizeof(float2) * 24);
    }
    return e;
}
template <typename C>
size_t smem_yw(const Geo& g) {
    return (size_t)(2 * YW_L * (g.M + 33)) * sizeof(C) + (sizeof(C) == 16 ? 0 : (size_t)g.M * sizeof(double2));
}

// forward declaration: DISPATCH_S is defined below
template <typename C = double2> void launch_ysolve_warp(chapsim_ctx* ctx);
template <typename C = double2> void launch_ysolve_seq(chapsim_ctx* ctx, bool kg1);
template <typename C = double2> void launch_ysolve(chapsim_ctx* ctx);

// Kernel attributes are process-wide and several contexts (of different
// grids) may share a kernel, so the dynamic shared-memory limit is raised to
// the device's opt-in maximum rather than set to one context's need, which
// could lower it below another's.  The limit does not affect occupancy.
template <typename F>
cudaError_t set_smem(F* f, size_t bytes) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa{};
    e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return e;
    const int limit = optin - (int)fa.sharedSizeBytes;  // dynamic + static must fit the opt-in size
    if ((int)bytes > limit) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
}

cudaError_t set_smem_void(const void* f, size_t bytes) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa{};
    e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return e;
    const int limit = optin - (int)fa.sharedSizeBytes;
    if ((int)bytes > limit) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
}

// a block's dynamic shared-memory limit for kernel f: the device's opt-in
// maximum less f's static shared memory (0 when it cannot be queried)
template <typename F>
long long bulk_smem_limit(F* f) {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, f) != cudaSuccess) return 0;
    return (long long)optin - (long long)fa.sharedSizeBytes;
}

#define DISPATCH_S(S_, KERNEL_CALL)                    \
    switch (S_) {                                      \
        case 1: { constexpr int S = 1; KERNEL_CALL; } break;  \
        case 2: { constexpr int S = 2; KERNEL_CALL; } break;  \
        case 3: { constexpr int S = 3; KERNEL_CALL; } break;  \
        case 4: { constexpr int S = 4; KERNEL_CALL; } break;  \
        case 6: { constexpr int S = 6; KERNEL_CALL; } break;  \
        case 8: { constexpr int S = 8; KERNEL_CALL; } break;  \
        case 12: { constexpr int S = 12; KERNEL_CALL; } break; \
        default: break;                                \
    }

bool valid_S(int s) { return s == 1 || s == 2 || s == 3 || s == 4 || s == 6 || s == 8 || s == 12; }

inline bool ysolve_seq_kg(const Geo& g) { return smem_ysolve_seq(g.M, true) <= (size_t)113 * 1024; }
// the fourth y-solve variant: the sequential recurrence with its forward
// intermediate in shared memory at one block per SM, for lines too long for two
inline bool ysolve_seq_kg1(const Geo& g) {
    return !ysolve_seq_kg(g) && smem_ysolve_seq(g.M, true) <= (size_t)227 * 1024;
}

template <typename C>
void launch_ysolve_seq(chapsim_ctx* ctx, bool kg1) {
    const Geo& g = ctx->g;
    const long long nl = (long long)g.LH * g.N;
    // the forward chain's FP64 intermediate: in shared memory where two blocks per SM still fit (or at one
    // block per SM, kg1), else in place in an FP64 spectrum, else in the FP64 array as scratch
    const int nb = (int)((nl + YS_NT - 1) / YS_NT);
    if (ysolve_seq_kg(g) || (kg1 && ysolve_seq_kg1(g)))
        launch_pdl(ctx->pdl, k_ysolve_seq<C, true>, nb, YS_NT, smem_ysolve_seq(g.M, true), ctx->stream, g, spec<C>(ctx),
                   ctx->SP, ctx->YF);
    else
        launch_pdl(ctx->pdl, k_ysolve_seq<C, false>, nb, YS_NT, smem_ysolve_seq(g.M, false), ctx->stream, g, spec<C>(ctx), ctx->SP,
                   ctx->YF);
}

template <typename C>
void launch_ysolve_2w(chapsim_ctx* ctx) {
    const Geo& g = ctx->g;
    const long long nt = 2 * (long long)g.LH * g.N;  // two threads per mode line
    launch_pdl(ctx->pdl, k_ysolve_2w<C>, (int)((nt + YS_NT - 1) / YS_NT), YS_NT, smem_ysolve_seq(), ctx->stream, g,
               spec<C>(ctx), ctx->SP, ctx->YF2);
}

template <typename C>
size_t smem_ysc(const Geo& g) {
    return (size_t)(2 * YW_L * (g.M + 33)) * sizeof(C) + (size_t)2 * (g.M + 32) * sizeof(double);
}

template <typename C>
void launch_ysolve_scan(chapsim_ctx* ctx) {
    const Geo& g = ctx->g;
    const long long nl = (long long)g.LH * g.N;
    const int nb = (int)std::min<long long>((nl + YW_L - 1) / YW_L, ctx->nsm);  // persistent: one block per SM
    DISPATCH_S(g.M / 32, (launch_pdl(ctx->pdl, k_ysolve_scan<S, C>, nb, YW_NT, smem_ysc<C>(g), ctx->stream, g,
                                     spec<C>(ctx), (const double*)ctx->YF3)));
}

template <typename C>
void launch_ysolve(chapsim_ctx* ctx) {
    if (ctx->ysolve_kind == 4 && ctx->YF3) launch_ysolve_scan<C>(ctx);
    else if (ctx->ysolve_kind == 1 && ctx->YF) launch_ysolve_seq<C>(ctx, false);
    else if (ctx->ysolve_kind == 3 && ctx->YF) launch_ysolve_seq<C>(ctx, true);
    else if (ctx->ysolve_kind == 2 && ctx->YF2) launch_ysolve_2w<C>(ctx);
    else launch_ysolve_warp<C>(ctx);
}

template <typename C>
void launch_ysolve_warp(chapsim_ctx* ctx) {
    const Geo& g = ctx->g;
    const long long nl = (long long)g.LH * g.N;
    const int nb = (int)std::min<long long>((nl + YW_L - 1) / YW_L, ctx->nsm);  // persistent: one block per SM
    DISPATCH_S(g.M / 32, (launch_pdl(ctx->pdl, k_ysolve_warp<S, C>, nb, YW_NT, smem_yw<C>(g), ctx->stream, g, spec<C>(ctx))));
}

// Momentum-stage arrays of the context in the real type R of its precision.
template <typename R>
struct StepFields {
    R *Q, *PR, *H0, *RHS, *RHSLL, *fac;
};
template <typename R> StepFields<R> step_fields(chapsim_ctx* c);
template <> StepFields<double> step_fields<double>(chapsim_ctx* c) { return {c->Q, c->PR, c->H0, c->RHS, c->RHSLL, c->fac}; }
template <> StepFields<float> step_fields<float>(chapsim_ctx* c) { return {c->Qf, c->PRf, c->H0f, c->RHSf, c->RHSLLf, c->facf}; }

template <typename R>
int configure_momentum(chapsim_ctx* ctx) {
    const Geo& g = ctx->g;
    DISPATCH_S(g.L / 32, CK(set_smem(k_rhs_xsweep<S, R, rhs_pv<R>(false)>, smem_rhs<R>(g))));
    DISPATCH_S(g.L / 32, CK(set_smem(k_rhs_xsweep<S, R, rhs_pv<R>(true)>, smem_rhs<R>(g))));
    ctx->rb_nw = 0;
    DISPATCH_S(g.L / 32, ctx->rb_nw = rb_warps<R>(g.L, bulk_smem_limit(k_rhs_xsweep_bulk<S, R>)));
    if (ctx->rb_nw > 0) DISPATCH_S(g.L / 32, CK(set_smem(k_rhs_xsweep_bulk<S, R>, rb_smem<R>(g.L, ctx->rb_nw))));
    DISPATCH_S(g.N / 32, CK(set_smem(k_zsweep<S, R, 32, 1>, smem_z<R>(g, 32))));
    DISPATCH_S(g.N / 32, CK(set_smem(k_zsweep<S, R, 16, 1>, smem_z<R>(g, 16))));
    DISPATCH_S(g.N / 32, CK(set_smem(k_zsweep<S, R, 32, 2>, smem_z<R>(g, 32))));
    DISPATCH_S(g.N / 32, CK(set_smem(k_zsweep<S, R, 16, 2>, smem_z<R>(g, 16))));
    DISPATCH_S(g.M / 32, CK(set_smem(k_ysweep<S, R, 1>, smem_y<R>(g))));
    DISPATCH_S(g.M / 32, CK(set_smem(k_ysweep<S, R, 2>, smem_y<R>(g))));
    DISPATCH_S(g.L / 32, CK(set_smem(k_xsweep<S, R>, smem_xs<R>(g))));
    CK(set_smem(k_rhs_point<R>, smem_rt<R>()));
    using C = SpecT<R>;
    DISPATCH_FFT(g.L, CK(set_smem(k_div_fftx<R, FN1, FN2>, smem_px<C>(g))));
    DISPATCH_FFT(g.L, CK(set_smem(k_fftx_inv<FN1, FN2, C>, smem_px<C>(g))));
    DISPATCH_S(g.M / 32, CK(set_smem(k_ysolve_warp<S, C>, smem_yw<C>(g))));
    DISPATCH_S(g.M / 32, CK(set_smem(k_ysolve_scan<S, C>, smem_ysc<C>(g))));
    CK(set_smem(k_ysolve_seq<C, false>, smem_ysolve_seq(g.M, false)));
    CK(set_smem(k_ysolve_seq<C, true>, smem_ysolve_seq(g.M, ysolve_seq_kg(g) || ysolve_seq_kg1(g))));
    CK(set_smem(k_ysolve_2w<C>, smem_ysolve_seq()));
    if (ctx->domain == 1 && plane_fft_ok<C>(g))
        P2_DISPATCH(g.L, g.N, CK((plane_fft_attrs<R, XN1, XN2, ZN1, ZN2>(set_smem_void, smem_p2<C>(g)))));
    // planes too large for one block: the cluster form, where the device can hold one of its clusters
    ctx->p2c = false;
    if (ctx->domain == 1 && !plane_fft_ok<C>(g) && plane_fft_cluster_shape(g.L, g.N))
        P2C_DISPATCH(g.L, g.N, (ctx->p2c = plane_fft_cluster_setup<R, XN1, XN2, ZN1, ZN2>(g)));
    DISPATCH_FFT(g.N, CK(set_smem(k_fftz<-1, FN1, FN2, C>, smem_fz<C>(g))));
    DISPATCH_FFT(g.N, CK(set_smem(k_fftz<+1, FN1, FN2, C>, smem_fz<C>(g))));
    DISPATCH_FFT(g.N, CK(set_smem(k_fftz_pipe<-1, FN1, FN2, C>, smem_fzp<C>(g))));
    DISPATCH_FFT(g.N, CK(set_smem(k_fftz_pipe<+1, FN1, FN2, C>, smem_fzp<C>(g))));
    return CHAPSIM_OK;
}

int configure_kernels(chapsim_ctx* ctx) {
    const Geo& g = ctx->g;
    // z-sweep tiles before any tuning: 16 lines where 32-line FP64 tiles leave one block per SM
    ctx->zs_tw = ctx->prec != CHAPSIM_PREC_MIXED && g.N / 32 >= 6 ? 16 : 32;
    int rc = ctx->prec == CHAPSIM_PREC_MIXED ? configure_momentum<float>(ctx) : configure_momentum<double>(ctx);
    if (rc) return rc;
    // the FP64 spectral stage serves the standalone Poisson solve and the main domain in every precision
    DISPATCH_FFT(g.L, CK(set_smem(k_fftx_inv<FN1, FN2, double2>, smem_px(g))));
    DISPATCH_FFT(g.L, CK(set_smem(k_fftx_from_rhs<FN1, FN2>, smem_px(g))));
    DISPATCH_FFT(g.L, CK(set_smem(k_io_div_fftx<FN1, FN2, double>, smem_px(g))));
    DISPATCH_FFT(g.L, CK(set_smem(k_io_div_fftx<FN1, FN2, float>, smem_px(g))));
    DISPATCH_S(g.M / 32, CK(set_smem(k_ysolve_warp<S, double2>, smem_yw<double2>(g))));
    DISPATCH_S(g.M / 32, CK(set_smem(k_ysolve_scan<S, double2>, smem_ysc<double2>(g))));
    CK(set_smem(k_ysolve_seq<double2, false>, smem_ysolve_seq(g.M, false)));
    CK(set_smem(k_ysolve_seq<double2, true>, smem_ysolve_seq(g.M, ysolve_seq_kg(g) || ysolve_seq_kg1(g))));
    CK(set_smem(k_ysolve_2w<double2>, smem_ysolve_seq()));
    DISPATCH_FFT(g.N, CK(set_smem(k_fftz<-1, FN1, FN2, double2>, smem_fz(g))));
    DISPATCH_FFT(g.N, CK(set_smem(k_fftz<+1, FN1, FN2, double2>, smem_fz(g))));
    if (ctx->domain == 2 && ctx->ivis) {
        DISPATCH_S(g.L / 32, CK(set_smem(k_io_cn_xsweep<S, double>, smem_cn(g.L))));
        DISPATCH_S(g.N / 32, CK(set_smem(k_io_cn_zsweep<S, double>, smem_cn(g.N))));
        DISPATCH_S(g.M / 32, CK(set_smem(k_io_cn_ysweep<S, double>, smem_cn(g.M))));
        DISPATCH_S(g.L / 32, CK(set_smem(k_io_cn_xsweep<S, float>, smem_cn(g.L))));
        DISPATCH_S(g.N / 32, CK(set_smem(k_io_cn_zsweep<S, float>, smem_cn(g.N))));
        DISPATCH_S(g.M / 32, CK(set_smem(k_io_cn_ysweep<S, float>, smem_cn(g.M))));
    }
    return CHAPSIM_OK;
}

// --------------------------- launch helpers ---------------------------------
inline void prof_mark(chapsim_ctx* ctx) {
    if (ctx->prof_ev) cudaEventRecord(ctx->prof_ev[ctx->prof_n++], ctx->stream);
}

// CFL partials, then the dt rule fused with the factor tables of all three substeps
template <typename R>
void launch_step_start_t(chapsim_ctx* ctx) {
    const Geo& g = ctx->g;
    StepFields<R> f = step_fields<R>(ctx);
    launch_pdl(ctx->pdl, k_cfl<R>, ctx->npart_red, DG_NT, 0, ctx->stream, g, f.Q, ctx->part_red, ctx->st);
    prof_mark(ctx);
    launch_pdl(ctx->pdl, k_dt_factors<R>, 15, 32, 0, ctx->stream, g, ctx->part_red, ctx->npart_red, ctx->st, f.fac);
    prof_mark(ctx);
    ctx->launches += 2;
}
void launch_step_start(chapsim_ctx* ctx) {
    if (ctx->prec == CHAPSIM_PREC_MIXED) launch_step_start_t<float>(ctx);
    else launch_step_start_t<double>(ctx);
}

void launch_cfl_dt(chapsim_ctx* ctx, int update_dt) {
    const Geo& g = ctx->g;
    if (ctx->prec == CHAPSIM_PREC_MIXED) launch_pdl(ctx->pdl, k_cfl<float>, ctx->npart_red, DG_NT, 0, ctx->stream, g, ctx->Qf, ctx->part_red, ctx->st);
    else launch_pdl(ctx->pdl, k_cfl<double>, ctx->npart_red, DG_NT, 0, ctx->stream, g, ctx->Q, ctx->part_red, ctx->st);
    prof_mark(ctx);
    launch_pdl(ctx->pdl, k_dt, 1, DG_NT, 0, ctx->stream, ctx->part_red, ctx->npart_red, ctx->st, update_dt);
    prof_mark(ctx);
    ctx->launches += 2;
}

// explicit right-hand sides and the x sweep, fused or split
template <typename R>
void launch_rhs_x(chapsim_ctx* ctx, const StepFields<R>& f, const R* fac, int ns) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    const int nwb = ctx->rb_nw;
    if (ctx->k1_kind == 2 && nwb > 0) {
        const int grb = std::min(ctx->nsm, (g.M * g.N + nwb - 1) / nwb);
        DISPATCH_S(g.L / 32, (launch_pdl(ctx->pdl, k_rhs_xsweep_bulk<S, R>, grb, nwb * 32, rb_smem<R>(g.L, nwb), s, 
                                 g, f.Q, f.PR, f.H0, f.RHS, ctx->part_rhs, ctx->st, fac, ns)));
    } else if (ctx->k1_kind == 1) {
        dim3 grt(g.L / RT_I, g.M / RT_J, g.N / rt_chunk(g));
        launch_pdl(ctx->pdl, k_rhs_point<R>, grt, RP_NT, smem_rt<R>(), s, g, f.Q, f.PR, f.H0, f.RHS, ctx->part_rhs, ctx->st, ns,
                                                         rt_chunk(g));
        const long long nl = 3LL * g.M * g.N;
        const int nbx = (int)((nl + XS_NT / 32 - 1) / (XS_NT / 32));
        DISPATCH_S(g.L / 32, (launch_pdl(ctx->pdl, k_xsweep<S, R>, nbx, XS_NT, smem_xs<R>(g), s, g, f.RHS, fac)));
        ctx->launches += 1;
    } else if (ctx->k1_kind == 3) {
        const int grx = g.M * g.N / RHS_WPB;
        DISPATCH_S(g.L / 32, (launch_pdl(ctx->pdl, k_rhs_xsweep<S, R, rhs_pv<R>(true)>, grx, RHS_WPB * 32, smem_rhs<R>(g), s, g,
                                         f.Q, f.PR, f.H0, f.RHS, ctx->part_rhs, ctx->st, fac, ns)));
    } else {
        const int grx = g.M * g.N / RHS_WPB;
        DISPATCH_S(g.L / 32, (launch_pdl(ctx->pdl, k_rhs_xsweep<S, R, rhs_pv<R>(false)>, grx, RHS_WPB * 32, smem_rhs<R>(g), s, g,
                                         f.Q, f.PR, f.H0, f.RHS, ctx->part_rhs, ctx->st, fac, ns)));
    }
}

// DIVG_tg + FFT99_POIS3D_periodicxz up to DPH: chained transforms, or the
// fused plane transforms (one block per y row) where chosen.  Both record the
// same profiling slots (the fused form leaves the two z-transform slots empty).
// z transforms of the periodic channel's spectrum: one tile per block (k_fftz), or the
// persistent double-buffered form (ctx->fz_pipe, chapsim_autotune bit 9)
template <int SIGN, typename C>
void launch_fftz(chapsim_ctx* ctx, C* sp) {
    const Geo& g = ctx->g;
    const long long nq = (long long)g.LH * g.M;
    if (ctx->fz_pipe) {
        const long long nt = (nq + fzp_tq<C>() - 1) / fzp_tq<C>();
        const int nb = (int)std::min<long long>(nt, (long long)fzp_minb<C>() * ctx->nsm);
        DISPATCH_FFT(g.N, (launch_pdl(ctx->pdl, k_fftz_pipe<SIGN, FN1, FN2, C>, nb, fzp_nt<C>(), smem_fzp<C>(g), ctx->stream, g, sp)));
    } else {
        const int gfz = (int)((nq + FZ_TQ - 1) / FZ_TQ);
        // prefetch distance: one wave of resident blocks (by the shared memory of a tile)
        const int bps = std::max(1, std::min(sizeof(C) == 8 ? 4 : 2, (int)((227 * 1024) / smem_fz<C>(g))));
        const int ahead = ctx->fz_prefetch ? bps * ctx->nsm : 0;
        DISPATCH_FFT(g.N, (launch_pdl(ctx->pdl, k_fftz<SIGN, FN1, FN2, C>, gfz, FZ_NT, smem_fz<C>(g), ctx->stream, g, sp, ahead)));
    }
}

template <typename R>
void launch_pressure(chapsim_ctx* ctx, const StepFields<R>& f, int ns) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    using C = SpecT<R>;
    C* sp = spec<C>(ctx);
    if (ctx->plane_kind == 1) {
        if (ctx->p2c) {
            P2C_DISPATCH(g.L, g.N, (plane_fft_cluster_fwd<R, XN1, XN2, ZN1, ZN2>(ctx->pdl, g, f.Q, f.RHSLL, sp, ctx->st, ns, s)));
        } else {
            P2_DISPATCH(g.L, g.N, (plane_fft_fwd<R, XN1, XN2, ZN1, ZN2>(ctx->pdl, g, f.Q, f.RHSLL, sp, ctx->st, ns, smem_p2<C>(g), s)));
        }
        prof_mark(ctx);
        prof_mark(ctx);
        launch_ysolve<C>(ctx);
        prof_mark(ctx);
        prof_mark(ctx);
        if (ctx->p2c) {
            P2C_DISPATCH(g.L, g.N, (plane_fft_cluster_inv<C, XN1, XN2, ZN1, ZN2>(ctx->pdl, g, sp, dph<R>(ctx), s)));
        } else {
            P2_DISPATCH(g.L, g.N, (plane_fft_inv<C, XN1, XN2, ZN1, ZN2>(ctx->pdl, g, sp, dph<R>(ctx), smem_p2<C>(g), s)));
        }
        prof_mark(ctx);
        ctx->launches += 3;
        return;
    }
    dim3 grp((g.M + PX_TJ - 1) / PX_TJ, g.N);
    DISPATCH_FFT(g.L, (launch_pdl(ctx->pdl, k_div_fftx<R, FN1, FN2>, grp, PX_NT, smem_px<C>(g), s, g, f.Q, f.RHSLL, sp, ctx->st, ns)));
    prof_mark(ctx);
    launch_fftz<-1, C>(ctx, sp);
    prof_mark(ctx);
    launch_ysolve<C>(ctx);
    prof_mark(ctx);
    launch_fftz<+1, C>(ctx, sp);
    prof_mark(ctx);
    DISPATCH_FFT(g.L, (launch_pdl(ctx->pdl, k_fftx_inv<FN1, FN2, C>, grp, PX_NT, smem_px<C>(g), s, g, sp, dph<R>(ctx))));
    prof_mark(ctx);
    ctx->launches += 5;
}

// cyclic z sweep, persistent: as many blocks as fit at once (two per SM where the two tile
// buffers allow); tiles of ctx->zs_tw lines
template <typename R>
void launch_zsweep(chapsim_ctx* ctx, const StepFields<R>& f, const R* fac) {
    const Geo& g = ctx->g;
    const int tw = ctx->zs_tw;
    const size_t sz = smem_z<R>(g, tw);
    const int zb_want = sizeof(R) == 4 && g.N / 32 <= 4 ? 3 : 2;  // zsweep_blocks<R, S>
    const int zb = sz * zb_want <= 226 * 1024 ? zb_want : (sz <= 113 * 1024 ? 2 : 1);
    const int nz = std::min((g.L / tw) * (3 * g.M - 1), zb * ctx->nsm);
    if (tw == 16 && ctx->zs_il == 2) {
        DISPATCH_S(g.N / 32, (launch_pdl(ctx->pdl, k_zsweep<S, R, 16, 2>, nz, SWEEP_NT, sz, ctx->stream, g, f.RHS, fac)));
    } else if (tw == 16) {
        DISPATCH_S(g.N / 32, (launch_pdl(ctx->pdl, k_zsweep<S, R, 16, 1>, nz, SWEEP_NT, sz, ctx->stream, g, f.RHS, fac)));
    } else if (ctx->zs_il == 2) {
        DISPATCH_S(g.N / 32, (launch_pdl(ctx->pdl, k_zsweep<S, R, 32, 2>, nz, SWEEP_NT, sz, ctx->stream, g, f.RHS, fac)));
    } else {
        DISPATCH_S(g.N / 32, (launch_pdl(ctx->pdl, k_zsweep<S, R, 32, 1>, nz, SWEEP_NT, sz, ctx->stream, g, f.RHS, fac)));
    }
}

// y sweep + update, the tile layout ctx->ys_il (chapsim_autotune bit 11)
template <typename R>
void launch_ysweep(chapsim_ctx* ctx, const StepFields<R>& f, const R* fac, int ns) {
    const Geo& g = ctx->g;
    dim3 gry(g.L / 32, g.N, 2);  // layer 0: u then v, layer 1: w
    if (ctx->ys_il == 2) {
        DISPATCH_S(g.M / 32, (launch_pdl(ctx->pdl, k_ysweep<S, R, 2>, gry, SWEEP_NT, smem_y<R>(g), ctx->stream, g, f.Q, f.RHS,
                                         ctx->st, fac, ns)));
    } else {
        DISPATCH_S(g.M / 32, (launch_pdl(ctx->pdl, k_ysweep<S, R, 1>, gry, SWEEP_NT, smem_y<R>(g), ctx->stream, g, f.Q, f.RHS,
                                         ctx->st, fac, ns)));
    }
}

template <typename R>
void launch_substep_t(chapsim_ctx* ctx, int ns, bool factors) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    StepFields<R> f = step_fields<R>(ctx);
    R* fac = f.fac + (long long)ns * 5 * FAC_SET;
    if (factors) {
        launch_pdl(ctx->pdl, k_factors<R>, 5, 32, 0, s, g, fac, ctx->st, ns);
        prof_mark(ctx);
        ctx->launches += 1;
    }
    launch_rhs_x<R>(ctx, f, fac, ns);
    prof_mark(ctx);
    launch_zsweep<R>(ctx, f, fac);
    prof_mark(ctx);
    launch_ysweep<R>(ctx, f, fac, ns);
    prof_mark(ctx);
    launch_pressure<R>(ctx, f, ns);
    const long long tot = (long long)g.L * g.M * g.N / V16<R>::W;  // one thread per 16-byte group of an x line
    launch_pdl(ctx->pdl, k_correct<R>, (int)((tot + CR_NT - 1) / CR_NT), CR_NT, 0, s, g, f.Q, f.PR, dph<R>(ctx), f.RHSLL, ctx->st, ns);
    prof_mark(ctx);
    ctx->launches += 4;
}
void launch_substep(chapsim_ctx* ctx, int ns, bool factors = true) {
    if (ctx->prec == CHAPSIM_PREC_MIXED) launch_substep_t<float>(ctx, ns, factors);
    else launch_substep_t<double>(ctx, ns, factors);
}

// FP64 staging arrays <-> FP32 fields of the mixed-precision step
int mixed_from_staging(chapsim_ctx* ctx, bool with_h0) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    const int nb = 4 * ctx->nsm;
    k_convert<float, double><<<nb, DG_NT, 0, s>>>(ctx->Qf, ctx->Q, 3 * g.FS);
    k_convert<float, double><<<nb, DG_NT, 0, s>>>(ctx->PRf, ctx->PR, g.FS);
    if (with_h0) k_convert<float, double><<<nb, DG_NT, 0, s>>>(ctx->H0f, ctx->H0, 3 * g.FI);
    ctx->launches += with_h0 ? 3 : 2;
    CK(cudaGetLastError());
    return CHAPSIM_OK;
}
int mixed_to_staging(chapsim_ctx* ctx, bool q, bool pr, bool h0) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    const int nb = 4 * ctx->nsm;
    if (q) { k_convert<double, float><<<nb, DG_NT, 0, s>>>(ctx->Q, ctx->Qf, 3 * g.FS); ctx->launches += 1; }
    if (pr) { k_convert<double, float><<<nb, DG_NT, 0, s>>>(ctx->PR, ctx->PRf, g.FS); ctx->launches += 1; }
    if (h0) { k_convert<double, float><<<nb, DG_NT, 0, s>>>(ctx->H0, ctx->H0f, 3 * g.FI); ctx->launches += 1; }
    CK(cudaGetLastError());
    return CHAPSIM_OK;
}

// ----------------------------- IO path -----------------------------------
// The main-domain fields in the storage type F of the context's precision:
// FP64 (ctx->io, Q, PR, RHS) or the FP32 flow fields of the mixed step
// (ctx->iof, Qf, PRf, RHSf); the property fields, the buoyancy and the
// weighted-pressure settings are shared.
template <typename F> IoFieldsT<F> io_fields_t(chapsim_ctx* ctx);
template <> IoFieldsT<double> io_fields_t<double>(chapsim_ctx* ctx) {
    IoFields f = ctx->io;
    f.Q = ctx->Q; f.PR = ctx->PR; f.RHS = ctx->RHS;
    f.DEN = ctx->thermal ? ctx->DEN : f.RHO;
    return f;
}
template <> IoFieldsT<float> io_fields_t<float>(chapsim_ctx* ctx) {
    IoFieldsT<float> f = ctx->iof;
    f.Q = ctx->Qf; f.PR = ctx->PRf; f.RHS = ctx->RHSf;
    f.RHO = ctx->io.RHO; f.MU0 = ctx->io.MU0; f.MU = ctx->io.MU;
    f.DEN = ctx->thermal ? ctx->DEN : f.RHO;
    f.PR0A = ctx->io.PR0A; f.PR0B = ctx->io.PR0B; f.fa = ctx->io.fa; f.igrav = ctx->io.igrav;
    return f;
}
IoFields io_fields(chapsim_ctx* ctx) { return io_fields_t<double>(ctx); }
inline bool io_mixed(const chapsim_ctx* ctx) { return ctx->prec == CHAPSIM_PREC_MIXED; }

int prop_grid(const chapsim_ctx* ctx, long long npts);
size_t prop_smem(int n);

MlpOperands mlp_ops(const chapsim_ctx* ctx) {
    return MlpOperands{ctx->mlp_w2, ctx->mlp_w3, ctx->mlp_w2t, ctx->mlp_w2h, ctx->mlp_w3h};
}

int xio_outlet_blocks(const chapsim_ctx* ctx);
// BC_TINLET_THERML and BC_COUTLET_ENEG_RK3(NS) of the inflow/outflow domain (FP64)
void xio_thermal_columns(chapsim_ctx* ctx, int ns) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    IoFields f = io_fields(ctx);
    const int gin = (int)std::min<long long>(4LL * ctx->nsm, ((long long)(g.M + 2) * g.N + XIO_NT - 1) / XIO_NT);
    k_xio_thermal_inlet<<<gin, XIO_NT, 0, s>>>(g, f, ctx->tf, ctx->xio_in);
    const int gout = xio_outlet_blocks(ctx);
    k_xio_outlet_a<<<gout, XIO_NT, 0, s>>>(g, f, ctx->xio_part);
    k_xio_energy_outlet<<<gout, PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->xio_part, gout, ctx->xio_bc0e,
                                                 ctx->st, ns);
    prof_mark(ctx);
    ctx->launches += 3;
}

// SOLVERRK3_ENG_io(NS), DENSITY_TIME_DERIVATION, DENSITY_Staggered,
// MU_Staggered, then G0 = G and VELOCITY_CALC_io of SOLVERRK3_MOM_io
template <typename F>
void launch_thermal_substep_t(chapsim_ctx* ctx, int ns) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    IoFieldsT<F> f = io_fields_t<F>(ctx);
    k_eng_rhs<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->tf, ctx->tp, ctx->st, ns);
    prof_mark(ctx);
    const size_t sm = prop_smem(ctx->tab.n);
    const long long tot = (long long)g.L * g.M * g.N, plane = 2LL * g.L * g.N;
    if (ctx->domain == 3) {
        // inflow/outflow: props of the interior, then the inlet and outlet columns, then the walls
        if (sm) k_eng_props<true, F><<<prop_grid(ctx, tot), PROP_NT, sm, s>>>(ctx->tab, g, f, ctx->tf, ctx->st);
        else k_eng_props<false, F><<<prop_grid(ctx, tot), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->st);
        prof_mark(ctx);
        xio_thermal_columns(ctx, ns);
        if (sm) k_eng_bc<true, F><<<prop_grid(ctx, plane), PROP_NT, sm, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
        else k_eng_bc<false, F><<<prop_grid(ctx, plane), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    } else if (ctx->use_mlp) {
        const long long tiles = (tot + MLP_TILE - 1) / MLP_TILE;
        MlpOut out{ctx->tf.ENTH, ctx->tf.TEMP, f.DEN, f.MU, ctx->tf.KAP, ctx->tf.HCP, f.RHO, f.MU0};
        const int gi = (int)std::min<long long>(tiles, 4LL * ctx->nsm);
        if (ctx->mlp_act == MLP_ACT_CUBIC)
            k_mlp_infer<true, MLP_ACT_CUBIC><<<gi, MLP_NT, MLP_INF_SMEM, s>>>(
                ctx->mlp_par, mlp_ops(ctx), ctx->mlp_norm, ctx->tab, g, tot, ctx->tf.DH, out, ctx->pstat, &ctx->st->err);
        else
            k_mlp_infer<true, MLP_ACT_TANH><<<gi, MLP_NT, MLP_INF_SMEM, s>>>(
                ctx->mlp_par, mlp_ops(ctx), ctx->mlp_norm, ctx->tab, g, tot, ctx->tf.DH, out, ctx->pstat, &ctx->st->err);
        prof_mark(ctx);
        if (sm) k_eng_bc<true, F><<<prop_grid(ctx, plane), PROP_NT, sm, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
        else k_eng_bc<false, F><<<prop_grid(ctx, plane), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    } else if (sm) {
        k_eng_props<true, F><<<prop_grid(ctx, tot), PROP_NT, sm, s>>>(ctx->tab, g, f, ctx->tf, ctx->st);
        prof_mark(ctx);
        k_eng_bc<true, F><<<prop_grid(ctx, plane), PROP_NT, sm, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    } else {
        k_eng_props<false, F><<<prop_grid(ctx, tot), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->st);
        prof_mark(ctx);
        k_eng_bc<false, F><<<prop_grid(ctx, plane), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    }
    prof_mark(ctx);
    k_drhodt<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->tf, ns, ctx->domain == 3 ? ctx->xio_mpart : nullptr);
    prof_mark(ctx);
    k_io_props<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f);
    prof_mark(ctx);
    k_g0_velocity<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->tf.G0);
    prof_mark(ctx);
    ctx->launches += 6;
}

void launch_io_step_start(chapsim_ctx* ctx) {
    if (io_mixed(ctx)) k_io_cfl<float><<<ctx->npart_red, IO_NT, 0, ctx->stream>>>(ctx->g, io_fields_t<float>(ctx), ctx->part_red, ctx->st);
    else k_io_cfl<double><<<ctx->npart_red, IO_NT, 0, ctx->stream>>>(ctx->g, io_fields_t<double>(ctx), ctx->part_red, ctx->st);
    prof_mark(ctx);
    k_dt<<<1, DG_NT, 0, ctx->stream>>>(ctx->part_red, ctx->npart_red, ctx->st, 1);
    prof_mark(ctx);
    ctx->launches += 2;
}

template <typename F>
void launch_io_substep_t(chapsim_ctx* ctx, int ns) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    if (ctx->thermal) launch_thermal_substep_t<F>(ctx, ns);
    IoFieldsT<F> f = io_fields_t<F>(ctx);
    if (!ctx->ivis) {
        k_io_divu<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f);
        prof_mark(ctx);
        k_io_rhs<false, F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->part_rhs, ctx->st, ns);
        prof_mark(ctx);
        k_io_massflux<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->st, ns);
        prof_mark(ctx);
    } else {
        // VISCOUS_PAR_EXPLT_* + RHS_MOM_EXPLICIT_io, then MOMFA_io's sweeps for all components
        k_io_rhs<true, F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->part_rhs, ctx->st, ns);
        prof_mark(ctx);
        dim3 gx((unsigned)((g.M * (long long)g.N + CN_LINES - 1) / CN_LINES), 3);
        DISPATCH_S(g.L / 32, (k_io_cn_xsweep<S, F><<<gx, CN_NT, smem_cn(g.L), s>>>(g, f, ctx->st, ns)));
        prof_mark(ctx);
        dim3 gz(g.L / CN_LINES, g.M, 3), gy(g.L / CN_LINES, g.N, 3);
        DISPATCH_S(g.N / 32, (k_io_cn_zsweep<S, F><<<gz, CN_NT, smem_cn(g.N), s>>>(g, f, ctx->st, ns)));
        DISPATCH_S(g.M / 32, (k_io_cn_ysweep<S, F><<<gy, CN_NT, smem_cn(g.M), s>>>(g, f, ctx->st, ns)));
        prof_mark(ctx);
        ctx->launches += 1;
    }
    // the Poisson stage is FP64 in both precisions
    dim3 grp((g.M + PX_TJ - 1) / PX_TJ, g.N);
    DISPATCH_FFT(g.L, (k_io_div_fftx<FN1, FN2, F><<<grp, PX_NT, smem_px(g), s>>>(g, f.G, ctx->RHSLL, ctx->SP,
                                                                               ctx->st, ns,
                                                                               ctx->thermal ? ctx->tf.DRHO : nullptr,
                                                                               ctx->io.PR0A ? 0.25 + IO_PRES_EPSLON : 1.0)));
    prof_mark(ctx);
    const long long nq = (long long)g.LH * g.M;
    const int gfz = (int)((nq + FZ_TQ - 1) / FZ_TQ);
    DISPATCH_FFT(g.N, (k_fftz<-1, FN1, FN2, double2><<<gfz, FZ_NT, smem_fz(g), s>>>(g, ctx->SP, 0)));
    prof_mark(ctx);
    launch_ysolve<double2>(ctx);
    prof_mark(ctx);
    DISPATCH_FFT(g.N, (k_fftz<+1, FN1, FN2, double2><<<gfz, FZ_NT, smem_fz(g), s>>>(g, ctx->SP, 0)));
    prof_mark(ctx);
    DISPATCH_FFT(g.L, (k_fftx_inv<FN1, FN2, double2><<<grp, PX_NT, smem_px(g), s>>>(g, ctx->SP, ctx->DPH)));
    prof_mark(ctx);
    k_io_correct<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->DPH, ctx->st, ns, ctx->ivis ? ctx->RHSLL : nullptr);
    prof_mark(ctx);
    ctx->launches += 9;
}
void launch_io_substep(chapsim_ctx* ctx, int ns) {
    if (io_mixed(ctx)) launch_io_substep_t<float>(ctx, ns);
    else launch_io_substep_t<double>(ctx, ns);
}

// ------------------------- inflow/outflow main domain ------------------------
size_t smem_xd(const Geo& g) { return (size_t)XD_R * g.LI * sizeof(double); }
// blocks of the outlet passes: one thread per outlet point, at most npart_red blocks (the
// partials buffer holds 3 doubles per block of npart_red: 2 for pass a, 2 for pass b fit in 4 per
// block of half as many)
int xio_outlet_blocks(const chapsim_ctx* ctx) {
    const int want = (int)(((long long)ctx->g.M * ctx->g.N + XIO_NT - 1) / XIO_NT);
    return std::max(1, std::min(want, (3 * ctx->npart_red) / 4));
}

// SOLVERRK3_MOM_io(NS) with TgFlowFlg (src/SOLVERRK3_MOM_IO.f90:11-120), explicit viscous
// terms: BC_TINLET_FLOW from the attached TG context (its substep NS must have run; the
// caller orders the two streams), BC_COUTLET_MOM_RK3, the momentum step of io.cuh (which
// leaves the inlet face u(1) alone and adds no bulk forcing), DIVG_io and FISHPACK's
// cosine/z/y solve, PRCALC_io + MASSFLUX_UPDATE_io + VELOCITY_CALC_io.
void launch_xio_substep(chapsim_ctx* ctx, int ns) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    IoFields f = io_fields(ctx);
    const chapsim_ctx* tg = ctx->tg_in;
    if (ctx->thermal) launch_thermal_substep_t<double>(ctx, ns);
    const double* drho = ctx->thermal ? ctx->tf.DRHO : nullptr;
    const int gin = (int)std::min<long long>(4LL * ctx->nsm, ((long long)(g.M + 2) * g.N + XIO_NT - 1) / XIO_NT);
    k_xio_inlet<<<gin, XIO_NT, 0, s>>>(g, f, tg->Q, tg->PR, tg->g.L, tg->g.FS);
    prof_mark(ctx);
    const int gout = xio_outlet_blocks(ctx);
    k_xio_outlet_a<<<gout, XIO_NT, 0, s>>>(g, f, ctx->xio_part);
    k_xio_outlet_b<<<gout, XIO_NT, 0, s>>>(g, f, ctx->xio_bc0, ctx->xio_part, ctx->xio_part + 2 * gout, ctx->xio_state,
                                           ctx->st, ns);
    k_xio_outlet_c<<<gout, XIO_NT, 0, s>>>(g, f, ctx->xio_part + 2 * gout, ctx->thermal ? ctx->xio_mpart : nullptr,
                                           ctx->io_grid, ctx->xio_state, ctx->st);
    prof_mark(ctx);
    k_io_divu<double><<<ctx->io_grid, IO_NT, 0, s>>>(g, f);
    prof_mark(ctx);
    k_io_rhs<false, double><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->part_rhs, ctx->st, ns);
    prof_mark(ctx);
    k_io_massflux<double><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->st, ns);
    prof_mark(ctx);
    const int nrb = (int)(((long long)g.M * g.N + XD_R - 1) / XD_R);
    int f1_, f2_;
    const bool fftx = fft4s_split(g.LI, f1_, f2_);  // an FFT length: the cosine transforms through the FFT
    dim3 gxf((g.M + XF_TJ - 1) / XF_TJ, g.N);
    const size_t smf = (size_t)XF_TJ * fft4s_ld(g.LI) * sizeof(double2);
    if (fftx) {
        DISPATCH_FFT(g.LI, (k_xio_div_cosqf<FN1, FN2><<<gxf, PX_NT, smf, s>>>(g, f.G, ctx->xio_tq, ctx->SP, ctx->st, ns, 1.0,
                                                                               drho)));
    } else {
        k_xio_div_dctx<<<nrb, XIO_NT, smem_xd(g), s>>>(g, f.G, ctx->xio_cf, ctx->SP, ctx->st, ns, 1.0, drho);
    }
    prof_mark(ctx);
    const long long nq = (long long)g.LH * g.M;  // LH = LI x modes
    const int gfz = (int)((nq + FZ_TQ - 1) / FZ_TQ);
    DISPATCH_FFT(g.N, (k_fftz<-1, FN1, FN2, double2><<<gfz, FZ_NT, smem_fz(g), s>>>(g, ctx->SP, 0)));
    prof_mark(ctx);
    k_xio_ysolve<<<(int)(((long long)g.LI * g.N + XIO_NT - 1) / XIO_NT), XIO_NT, 0, s>>>(g, ctx->SP, ctx->xio_yd);
    prof_mark(ctx);
    DISPATCH_FFT(g.N, (k_fftz<+1, FN1, FN2, double2><<<gfz, FZ_NT, smem_fz(g), s>>>(g, ctx->SP, 0)));
    prof_mark(ctx);
    if (fftx) {
        DISPATCH_FFT(g.LI, (k_xio_cosqb<FN1, FN2><<<gxf, PX_NT, smf, s>>>(g, ctx->SP, ctx->xio_tq, ctx->DPH)));
    } else {
        k_xio_dctx_inv<<<nrb, XIO_NT, smem_xd(g), s>>>(g, ctx->SP, ctx->xio_cf + (size_t)g.LI * g.LI, ctx->DPH);
    }
    prof_mark(ctx);
    k_io_correct<double><<<ctx->io_grid, IO_NT, 0, s>>>(g, f, ctx->DPH, ctx->st, ns, nullptr);
    prof_mark(ctx);
    ctx->launches += 13;
}

// CFL_tg and CFL_io of one TG + main-domain step, then CFLMM = max of the two and the dt rule
// (src/SOLVE.f90:79-94), DT in both states.  The TG stream waits for the DT.
void launch_xio_step_start(chapsim_ctx* io) {
    chapsim_ctx* tg = io->tg_in;
    launch_cfl_dt(tg, 0);
    cudaEventRecord(io->xev[0], tg->stream);
    k_io_cfl<double><<<io->npart_red, IO_NT, 0, io->stream>>>(io->g, io_fields(io), io->part_red, io->st);
    k_dt<<<1, DG_NT, 0, io->stream>>>(io->part_red, io->npart_red, io->st, 0);
    cudaStreamWaitEvent(io->stream, io->xev[0], 0);
    k_dt_pair<<<1, 32, 0, io->stream>>>(tg->st, io->st);
    cudaEventRecord(io->xev[1], io->stream);
    cudaStreamWaitEvent(tg->stream, io->xev[1], 0);
    io->launches += 3;
}

// one TG substep, then the main-domain substep that reads the TG fields; the next TG launch
// waits for that read
void launch_xio_pair_substep(chapsim_ctx* io, int ns) {
    chapsim_ctx* tg = io->tg_in;
    launch_substep(tg, ns, true);
    cudaEventRecord(io->xev[0], tg->stream);
    cudaStreamWaitEvent(io->stream, io->xev[0], 0);
    launch_xio_substep(io, ns);
    cudaEventRecord(io->xev[1], io->stream);
    cudaStreamWaitEvent(tg->stream, io->xev[1], 0);
}

int check_device_error(chapsim_ctx* ctx) {
    CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned int e = ctx->st_host->err;
    if (e) {
        unsigned int zero = 0;
        CK(cudaMemcpyAsync(&ctx->st->err, &zero, sizeof(unsigned int), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (e & CHS_EBIT_NAN) return fail(ctx, CHAPSIM_ERR_NAN, "non-finite velocity or time step on the device");
        if (e & CHS_EBIT_DT_COLLAPSE) return fail(ctx, CHAPSIM_ERR_DT_COLLAPSE, "DT/DT0 < 0.01 (time step collapse)");
        if (e & CHS_EBIT_TABLE)
            return fail(ctx, CHAPSIM_ERR_TABLE_RANGE, "rho*h (or h) left the property table during the energy update");
        if (e & CHS_EBIT_MMA_TIMEOUT)
            return fail(ctx, CHAPSIM_ERR_TIMEOUT, "a bounded device wait (tensor-core commit or bulk copy) ran out of time");
    }
    return CHAPSIM_OK;
}

int build_step_graph(chapsim_ctx* ctx) {
    if (ctx->step_exec) return CHAPSIM_OK;
    cudaGraph_t graph;
    unsigned long long before = ctx->launches;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    if (ctx->domain == 2) {
        launch_io_step_start(ctx);
        for (int ns = 1; ns <= 3; ++ns) launch_io_substep(ctx, ns);
    } else {
        launch_step_start(ctx);
        for (int ns = 1; ns <= 3; ++ns) launch_substep(ctx, ns, false);
    }
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    ctx->kernels_per_step = (int)(ctx->launches - before);
    ctx->launches = before;  // capture does not launch
    if (e != cudaSuccess) return fail(ctx, CHAPSIM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ctx->step_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, CHAPSIM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return CHAPSIM_OK;
}

}  // namespace

// ============================== C ABI ========================================
extern "C" {

int chapsim_gpu_init(const chapsim_grid_t* grid, const chapsim_coefs_t* cf, const chapsim_opts_t* opts,
                     chapsim_ctx_t** out) {
    chapsim_ctx* ctx = nullptr;
    if (!grid || !cf || !out) return fail(nullptr, CHAPSIM_ERR_BADARG, "null argument");
    *out = nullptr;
    const int L = grid->ncl1, M = grid->ncl2, N = grid->ncl3;
    if (grid->icase != 1 || grid->idomain < 1 || grid->idomain > 3)
        return fail(nullptr, CHAPSIM_ERR_BADARG,
                    "only the plane channel (iCase=1) with a periodic TG (iDomain=1), x-periodic main (2) or inflow/outflow "
                    "main (3) domain is supported");
    const bool xio = grid->idomain == 3;
    // the inflow/outflow main domain has no x FFT and no x sweep: any even NCL1_io from 4 to 768 (the
    // cosine transforms hold 32 rows of it in shared memory)
    if (xio ? (L < 4 || L > 768 || L % 2) : (L < 32 || L % 32 || !valid_S(L / 32)))
        return fail(nullptr, CHAPSIM_ERR_BADARG,
                    xio ? "NCL1_io of the inflow/outflow domain must be even, 4..768"
                        : "NCL1, NCL2, NCL3 must be 32*S with S in {1,2,3,4,6,8,12}");
    if (M < 32 || N < 32 || M % 32 || N % 32 || !valid_S(M / 32) || !valid_S(N / 32))
        return fail(nullptr, CHAPSIM_ERR_BADARG, "NCL1, NCL2, NCL3 must be 32*S with S in {1,2,3,4,6,8,12}");
    int n1_, n2_;
    if ((!xio && !fft4s_split(L, n1_, n2_)) || !fft4s_split(N, n1_, n2_))
        return fail(nullptr, CHAPSIM_ERR_BADARG, "NCL1 and NCL3 must be one of 32, 64, 96, 128, 192, 256, 384");
    if (!cf->dyfi || !cf->dyci || !cf->ycl2nd_wff || !cf->ycl2nd_wfb || !cf->amph || !cf->acph || !cf->apph ||
        !cf->amvr || !cf->acvr || !cf->apvr || !cf->ak1 || !cf->ak3)
        return fail(nullptr, CHAPSIM_ERR_BADARG, "missing coefficient array");
    if (cf->iflowdriven < 0 || cf->iflowdriven > 2) return fail(nullptr, CHAPSIM_ERR_BADARG, "iFlowDriven must be 0, 1 or 2");

    const int prec = opts ? opts->precision : CHAPSIM_PREC_FP64;
    if (prec != CHAPSIM_PREC_FP64 && prec != CHAPSIM_PREC_MIXED)
        return fail(nullptr, CHAPSIM_ERR_BADARG, "precision must be CHAPSIM_PREC_FP64 or CHAPSIM_PREC_MIXED");
    const int ivis = opts ? opts->ivisscheme : CHAPSIM_VIS_EXPLICIT;
    if (ivis != CHAPSIM_VIS_EXPLICIT && ivis != CHAPSIM_VIS_IMPLICIT)
        return fail(nullptr, CHAPSIM_ERR_BADARG, "ivisscheme must be CHAPSIM_VIS_EXPLICIT or CHAPSIM_VIS_IMPLICIT");
    if (ivis == CHAPSIM_VIS_IMPLICIT && grid->idomain == 1)
        return fail(nullptr, CHAPSIM_ERR_BADARG,
                    "ivisscheme selects the main-domain (iDomain = 2) scheme; the TG domain is always Crank-Nicolson");
    if (xio && (ivis != CHAPSIM_VIS_EXPLICIT || prec != CHAPSIM_PREC_FP64))
        return fail(nullptr, CHAPSIM_ERR_BADARG,
                    "the inflow/outflow main domain (iDomain = 3) runs the explicit viscous scheme in FP64");
    if (ivis == CHAPSIM_VIS_IMPLICIT && !(cf->amvr1 > 0.0 && cf->apvrn > 0.0 && std::isfinite(cf->amvr1) &&
                                          std::isfinite(cf->apvrn)))
        return fail(nullptr, CHAPSIM_ERR_BADARG, "the Crank-Nicolson main domain needs AMVR1 and APVRN (TDMA_COEF)");
    ctx = new chapsim_ctx();
    ctx->device = opts ? opts->device : 0;
    ctx->domain = grid->idomain;
    ctx->prec = prec;
    ctx->pdl = !(opts && opts->no_pdl);
    ctx->ivis = ivis;
    int rc;
#define INIT_CK(call)                                  \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) {                       \
            g_init_error = std::string(#call) + ": " + cudaGetErrorString(e_); \
            chapsim_gpu_finalize(ctx);                 \
            return CHAPSIM_ERR_CUDA;                   \
        }                                              \
    } while (0)
    INIT_CK(cudaSetDevice(ctx->device));
    INIT_CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    Geo& g = ctx->g;
    const int LS = xio ? L + 2 : L;  // row stride: the ghost columns 0 and L+1 with inflow/outflow
    g.L = LS; g.M = M; g.N = N; g.LH = xio ? L : L / 2 + 1;
    g.LI = L; g.xo = xio ? 1 : 0;
    g.P = (long long)LS * (M + 2);
    g.FS = g.P * N;
    g.PI_ = (long long)L * M;
    g.FI = g.PI_ * N;
    g.dxi = cf->dxi; g.dzi = cf->dzi; g.dxqi = cf->dxqi; g.dzqi = cf->dzqi;
    g.cvisc = cf->cvisc; g.volm = cf->volm; g.cf_given = cf->cf_given; g.iflowdriven = cf->iflowdriven;
    if (xio) g.iflowdriven = 0;  // no bulk forcing with inflow (src/RHS_MOM_EXPLICIT_io.f90:229)
    g.fix_v_wall_row = opts ? opts->fix_v_wall_row : 0;
    for (int s = 0; s < 4; ++s) { g.tgam[s] = cf->tgam[s]; g.troh[s] = cf->troh[s]; g.talp[s] = cf->talp[s]; }
    g.area_inlet = 0.0;  // COORDJR's loop order (RCCI1 = 1)
    for (int jc = 0; jc < M; ++jc)
        for (int kc = 0; kc < N; ++kc) g.area_inlet = g.area_inlet + 1.0 / 1.0 / cf->dyfi[jc] / cf->dzi;
    g.amvr1 = ivis == CHAPSIM_VIS_IMPLICIT ? cf->amvr1 : 0.0;
    g.apvrn = ivis == CHAPSIM_VIS_IMPLICIT ? cf->apvrn : 0.0;
    // y arrays with the reference's 1-based index (entry 0 unused)
    const int YS = M + 2;
    std::vector<double> yb((size_t)YS * 13 + L + N, 0.0);
    double* y = yb.data();
    for (int j = 1; j <= M; ++j) {
        y[0 * YS + j] = cf->dyfi[j - 1];
        y[4 * YS + j] = cf->amph[j - 1];
        y[5 * YS + j] = cf->acph[j - 1];
        y[6 * YS + j] = cf->apph[j - 1];
    }
    for (int j = 1; j <= M + 1; ++j) {
        y[1 * YS + j] = cf->dyci[j - 1];
        y[2 * YS + j] = cf->ycl2nd_wff[j - 1];
        y[3 * YS + j] = cf->ycl2nd_wfb[j - 1];
        for (int c = 0; c < 3; ++c) {
            y[(7 + c) * YS + j] = cf->amvr[(size_t)c * (M + 1) + (j - 1)];
            y[(10 + c) * YS + j] = cf->acvr[(size_t)c * (M + 1) + (j - 1)];
        }
    }
    // apvr occupies its own block after the 13 y arrays: reuse slots via a second vector
    std::vector<double> ap((size_t)3 * YS, 0.0);
    for (int j = 1; j <= M + 1; ++j)
        for (int c = 0; c < 3; ++c) ap[(size_t)c * YS + j] = cf->apvr[(size_t)c * (M + 1) + (j - 1)];
    double* ak = y + 13 * YS;
    for (int i = 0; i < L; ++i) ak[i] = cf->ak1[i];
    for (int k = 0; k < N; ++k) ak[L + k] = cf->ak3[k];
    const size_t nyb = yb.size() + ap.size();
    INIT_CK(cudaMalloc(&ctx->ybuf, nyb * sizeof(double)));
    INIT_CK(cudaMemcpy(ctx->ybuf, yb.data(), yb.size() * sizeof(double), cudaMemcpyHostToDevice));
    INIT_CK(cudaMemcpy(ctx->ybuf + yb.size(), ap.data(), ap.size() * sizeof(double), cudaMemcpyHostToDevice));
    double* yd = ctx->ybuf;
    g.dyfi = yd + 0 * YS; g.dyci = yd + 1 * YS; g.wff = yd + 2 * YS; g.wfb = yd + 3 * YS;
    g.amph = yd + 4 * YS; g.acph = yd + 5 * YS; g.apph = yd + 6 * YS;
    g.amvr = yd + 7 * YS; g.acvr = yd + 10 * YS; g.apvr = yd + yb.size();
    g.ak1 = yd + 13 * YS; g.ak3 = yd + 13 * YS + L;
    // FFT plans
    std::vector<double2> twx = twiddles(L), twz = twiddles(N);
    INIT_CK(upload_small_twiddles());
    INIT_CK(cudaMalloc(&ctx->tw, (size_t)(L + N) * sizeof(double2)));
    INIT_CK(cudaMemcpy(ctx->tw, twx.data(), L * sizeof(double2), cudaMemcpyHostToDevice));
    INIT_CK(cudaMemcpy(ctx->tw + L, twz.data(), N * sizeof(double2), cudaMemcpyHostToDevice));
    g.twx = ctx->tw; g.twz = ctx->tw + L;
    {
        std::vector<float2> twf((size_t)(L + N));
        for (int i = 0; i < L; ++i) twf[i] = make_float2((float)twx[i].x, (float)twx[i].y);
        for (int k = 0; k < N; ++k) twf[L + k] = make_float2((float)twz[k].x, (float)twz[k].y);
        INIT_CK(cudaMalloc(&ctx->twf, (size_t)(L + N) * sizeof(float2)));
        INIT_CK(cudaMemcpy(ctx->twf, twf.data(), (L + N) * sizeof(float2), cudaMemcpyHostToDevice));
        g.twxf = ctx->twf; g.twzf = ctx->twf + L;
    }
    INIT_CK(cudaMalloc(&ctx->yz, (size_t)2 * M * sizeof(double)));
    g.yz = ctx->yz;
    k_ysolve_zero_factors<<<1, 32, 0, ctx->stream>>>(g, ctx->yz);
    INIT_CK(cudaGetLastError());
    // fields
    INIT_CK(cudaMalloc(&ctx->Q, (size_t)(3 * g.FS) * sizeof(double)));
    INIT_CK(cudaMalloc(&ctx->PR, (size_t)g.FS * sizeof(double)));
    INIT_CK(cudaMalloc(&ctx->DPH, (size_t)g.FS * sizeof(double)));
    INIT_CK(cudaMemset(ctx->DPH, 0, (size_t)g.FS * sizeof(double)));  // the inflow/outflow ghost columns stay 0
    INIT_CK(cudaMalloc(&ctx->H0, (size_t)(3 * g.FI) * sizeof(double)));
    INIT_CK(cudaMalloc(&ctx->RHS, (size_t)(3 * g.FI) * sizeof(double)));
    INIT_CK(cudaMalloc(&ctx->RHSLL, (size_t)g.FI * sizeof(double)));
    INIT_CK(cudaMalloc(&ctx->SP, (size_t)g.LH * M * N * sizeof(double2)));
    ctx->npart_rhs = M * N / RHS_WPB;
    INIT_CK(cudaMalloc(&ctx->part_rhs, (size_t)ctx->npart_rhs * sizeof(double)));
    INIT_CK(cudaMalloc(&ctx->fac, (size_t)4 * 5 * FAC_SET * sizeof(double)));
    INIT_CK(cudaMemset(ctx->fac, 0, (size_t)4 * 5 * FAC_SET * sizeof(double)));

    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    ctx->nsm = nsm;
    ctx->npart_red = 4 * nsm;
    INIT_CK(cudaMalloc(&ctx->part_red, (size_t)ctx->npart_red * sizeof(double)));
    if (ctx->domain >= 2) {
        IoFields& f = ctx->io;
        INIT_CK(cudaMalloc(&f.G, (size_t)(3 * g.FS) * sizeof(double)));
        INIT_CK(cudaMalloc(&f.EX0, (size_t)(3 * g.FI) * sizeof(double)));
        INIT_CK(cudaMalloc(&f.RHO, (size_t)g.FS * sizeof(double)));
        INIT_CK(cudaMalloc(&f.MU0, (size_t)g.FS * sizeof(double)));
        INIT_CK(cudaMalloc(&f.MU, (size_t)g.FS * sizeof(double)));
        INIT_CK(cudaMalloc(&f.DST, (size_t)(3 * g.FS) * sizeof(double)));
        INIT_CK(cudaMalloc(&f.MST, (size_t)(3 * g.FS) * sizeof(double)));
        INIT_CK(cudaMalloc(&f.DIVU, (size_t)g.FS * sizeof(double)));
        INIT_CK(cudaMemset(f.G, 0, (size_t)(3 * g.FS) * sizeof(double)));
        INIT_CK(cudaMemset(f.EX0, 0, (size_t)(3 * g.FI) * sizeof(double)));
        INIT_CK(cudaMemset(f.DIVU, 0, (size_t)g.FS * sizeof(double)));
        k_fill<<<4 * nsm, XIO_NT, 0, ctx->stream>>>(f.DST, 3 * g.FS, 1.0);  // src/MEMALLOCT.f90:200-201
        k_fill<<<4 * nsm, XIO_NT, 0, ctx->stream>>>(f.MST, 3 * g.FS, 1.0);
        INIT_CK(cudaGetLastError());
        ctx->io_grid = ctx->npart_rhs < 8 * nsm ? ctx->npart_rhs : 8 * nsm;
    }
    if (xio) {
        std::vector<double> cq((size_t)4 * L), cm((size_t)2 * L * L);
        const double pi = 2.0 * std::asin(1.0);
        for (int q = 0; q < 4 * L; ++q) cq[q] = std::cos((double)q * pi / (double)(2 * L));
        for (int p = 0; p < L; ++p)
            for (int m = 0; m < L; ++m) {
                const double c = cq[(size_t)(((long long)(2 * m + 1) * p) % (4 * L))];
                cm[(size_t)p * L + m] = p == 0 ? 1.0 : 2.0 * c;       // COSQF
                cm[(size_t)L * L + (size_t)m * L + p] = 4.0 * c;      // COSQB
            }
        INIT_CK(cudaMalloc(&ctx->xio_cf, cm.size() * sizeof(double)));
        INIT_CK(cudaMemcpy(ctx->xio_cf, cm.data(), cm.size() * sizeof(double), cudaMemcpyHostToDevice));
        std::vector<double2> tq((size_t)L);
        for (int p = 0; p < L; ++p)
            tq[p] = make_double2(std::cos((double)p * pi / (double)(2 * L)), std::sin((double)p * pi / (double)(2 * L)));
        INIT_CK(cudaMalloc(&ctx->xio_tq, tq.size() * sizeof(double2)));
        INIT_CK(cudaMemcpy(ctx->xio_tq, tq.data(), tq.size() * sizeof(double2), cudaMemcpyHostToDevice));
        INIT_CK(cudaMalloc(&ctx->xio_bc0, (size_t)3 * M * N * sizeof(double)));
        INIT_CK(cudaMemset(ctx->xio_bc0, 0, (size_t)3 * M * N * sizeof(double)));
        INIT_CK(cudaMalloc(&ctx->xio_yd, (size_t)L * M * N * sizeof(double)));
        INIT_CK(cudaMalloc(&ctx->xio_state, 2 * sizeof(double)));
        INIT_CK(cudaMemset(ctx->xio_state, 0, 2 * sizeof(double)));
        INIT_CK(cudaMalloc(&ctx->xio_part, (size_t)3 * ctx->npart_red * sizeof(double)));
        INIT_CK(cudaMalloc(&ctx->xio_bc0e, (size_t)M * N * sizeof(double)));
        INIT_CK(cudaMemset(ctx->xio_bc0e, 0, (size_t)M * N * sizeof(double)));
        INIT_CK(cudaMalloc(&ctx->xio_mpart, (size_t)ctx->io_grid * sizeof(double)));
        INIT_CK(cudaEventCreateWithFlags(&ctx->xev[0], cudaEventDisableTiming));
        INIT_CK(cudaEventCreateWithFlags(&ctx->xev[1], cudaEventDisableTiming));
        if (smem_xd(g) > 48 * 1024) {
            INIT_CK(set_smem(k_xio_div_dctx, smem_xd(g)));
            INIT_CK(set_smem(k_xio_dctx_inv, smem_xd(g)));
        }
        int f1_, f2_;
        const size_t smf = (size_t)XF_TJ * fft4s_ld(L) * sizeof(double2);
        if (fft4s_split(L, f1_, f2_) && smf > 48 * 1024) {
            DISPATCH_FFT(L, INIT_CK(set_smem(k_xio_div_cosqf<FN1, FN2>, smf)));
            DISPATCH_FFT(L, INIT_CK(set_smem(k_xio_cosqb<FN1, FN2>, smf)));
        }
    }
    if (ctx->prec == CHAPSIM_PREC_MIXED) {
        INIT_CK(cudaMalloc(&ctx->Qf, (size_t)(3 * g.FS) * sizeof(float)));
        INIT_CK(cudaMalloc(&ctx->PRf, (size_t)g.FS * sizeof(float)));
        INIT_CK(cudaMalloc(&ctx->H0f, (size_t)(3 * g.FI) * sizeof(float)));
        INIT_CK(cudaMalloc(&ctx->RHSf, (size_t)(3 * g.FI) * sizeof(float)));
        INIT_CK(cudaMalloc(&ctx->RHSLLf, (size_t)g.FI * sizeof(float)));
        INIT_CK(cudaMalloc(&ctx->facf, (size_t)4 * 5 * FAC_SET * sizeof(float)));
        INIT_CK(cudaMemset(ctx->Qf, 0, (size_t)(3 * g.FS) * sizeof(float)));
        INIT_CK(cudaMemset(ctx->PRf, 0, (size_t)g.FS * sizeof(float)));
        INIT_CK(cudaMemset(ctx->H0f, 0, (size_t)(3 * g.FI) * sizeof(float)));
        INIT_CK(cudaMemset(ctx->RHSf, 0, (size_t)(3 * g.FI) * sizeof(float)));
        INIT_CK(cudaMemset(ctx->RHSLLf, 0, (size_t)g.FI * sizeof(float)));
        INIT_CK(cudaMemset(ctx->facf, 0, (size_t)4 * 5 * FAC_SET * sizeof(float)));
        INIT_CK(cudaMalloc(&ctx->SPf, (size_t)g.LH * M * N * sizeof(float2)));
        INIT_CK(cudaMalloc(&ctx->DPHf, (size_t)g.FS * sizeof(float)));
        INIT_CK(cudaMemset(ctx->DPHf, 0, (size_t)g.FS * sizeof(float)));
        if (ctx->domain == 2) {  // FP32 flow fields of the main domain (Q, PR and RHS are Qf, PRf, RHSf)
            IoFieldsT<float>& f = ctx->iof;
            INIT_CK(cudaMalloc(&f.G, (size_t)(3 * g.FS) * sizeof(float)));
            INIT_CK(cudaMalloc(&f.EX0, (size_t)(3 * g.FI) * sizeof(float)));
            INIT_CK(cudaMalloc(&f.DST, (size_t)(3 * g.FS) * sizeof(float)));
            INIT_CK(cudaMalloc(&f.MST, (size_t)(3 * g.FS) * sizeof(float)));
            INIT_CK(cudaMalloc(&f.DIVU, (size_t)g.FS * sizeof(float)));
            INIT_CK(cudaMemset(f.G, 0, (size_t)(3 * g.FS) * sizeof(float)));
            INIT_CK(cudaMemset(f.EX0, 0, (size_t)(3 * g.FI) * sizeof(float)));
            INIT_CK(cudaMemset(f.DIVU, 0, (size_t)g.FS * sizeof(float)));
        }
    }
    INIT_CK(cudaMalloc(&ctx->st, sizeof(DevState)));
    INIT_CK(cudaMallocHost(&ctx->st_host, sizeof(DevState)));
    INIT_CK(cudaMemset(ctx->Q, 0, (size_t)(3 * g.FS) * sizeof(double)));
    INIT_CK(cudaMemset(ctx->PR, 0, (size_t)g.FS * sizeof(double)));
    INIT_CK(cudaMemset(ctx->DPH, 0, (size_t)g.FS * sizeof(double)));
    INIT_CK(cudaMemset(ctx->H0, 0, (size_t)(3 * g.FI) * sizeof(double)));
    INIT_CK(cudaMemset(ctx->RHS, 0, (size_t)(3 * g.FI) * sizeof(double)));
    DevState s0{};
    s0.dt = 1e-3; s0.dt0 = 1e-3; s0.dtmin = 1e-6; s0.cflgv = 0.5;
    INIT_CK(cudaMemcpy(ctx->st, &s0, sizeof(DevState), cudaMemcpyHostToDevice));
    rc = configure_kernels(ctx);
    if (rc != CHAPSIM_OK) {
        g_init_error = ctx->err;
        chapsim_gpu_finalize(ctx);
        return rc;
    }

#undef INIT_CK
    *out = ctx;
    return CHAPSIM_OK;
}

void chapsim_gpu_finalize(chapsim_ctx_t* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->step_exec) cudaGraphExecDestroy(ctx->step_exec);
    cudaFree(ctx->Q); cudaFree(ctx->PR); cudaFree(ctx->H0); cudaFree(ctx->RHS); cudaFree(ctx->RHSLL);
    cudaFree(ctx->DPH); cudaFree(ctx->SP); cudaFree(ctx->YF); cudaFree(ctx->YF2); cudaFree(ctx->YF3); cudaFree(ctx->part_rhs); cudaFree(ctx->part_red); cudaFree(ctx->fac);
    cudaFree(ctx->st); cudaFree(ctx->ybuf); cudaFree(ctx->tw); cudaFree(ctx->twf); cudaFree(ctx->yz); cudaFree(ctx->SPf); cudaFree(ctx->DPHf);
    cudaFree(ctx->pp_inst); cudaFree(ctx->pp_avg); cudaFree(ctx->pp_part); cudaFree(ctx->pp_mon);
    cudaFree(ctx->ppio_set); cudaFree(ctx->ppio_part);
    cudaFree(ctx->io.G); cudaFree(ctx->io.EX0); cudaFree(ctx->io.RHO); cudaFree(ctx->io.MU0); cudaFree(ctx->io.MU);
    cudaFree(ctx->io.DST); cudaFree(ctx->io.MST); cudaFree(ctx->io.DIVU);
    cudaFree(ctx->iof.G); cudaFree(ctx->iof.EX0); cudaFree(ctx->iof.DST); cudaFree(ctx->iof.MST); cudaFree(ctx->iof.DIVU);
    cudaFree(const_cast<double*>(ctx->io.PR0A));
    cudaFree(ctx->ptab); cudaFree(ctx->pstat); cudaFree(ctx->pbuf);
    cudaFree(ctx->mlp_par); cudaFree(ctx->mlp_w2); cudaFree(ctx->mlp_xs); cudaFree(ctx->mlp_ys); cudaFree(ctx->mlp_dh);
    cudaFree(ctx->mlp_judge);
    cudaFree(ctx->DEN); cudaFree(ctx->tf.DH); cudaFree(ctx->tf.ENTH); cudaFree(ctx->tf.TEMP); cudaFree(ctx->tf.KAP);
    cudaFree(ctx->tf.HCP); cudaFree(ctx->tf.RHSE0); cudaFree(ctx->tf.G0); cudaFree(ctx->tf.DRHO);
    cudaFree(ctx->Qf); cudaFree(ctx->PRf); cudaFree(ctx->H0f); cudaFree(ctx->RHSf); cudaFree(ctx->RHSLLf); cudaFree(ctx->facf);
    if (ctx->st_host) cudaFreeHost(ctx->st_host);
    if (ctx->dump_stream) cudaStreamSynchronize(ctx->dump_stream);
    cudaFree(ctx->dump_dev);
    if (ctx->dump_host) cudaFreeHost(ctx->dump_host);
    if (ctx->dump_snap) cudaEventDestroy(ctx->dump_snap);
    if (ctx->dump_done) cudaEventDestroy(ctx->dump_done);
    if (ctx->dump_stream) cudaStreamDestroy(ctx->dump_stream);
    cudaFree(ctx->xio_cf); cudaFree(ctx->xio_tq); cudaFree(ctx->xio_bc0); cudaFree(ctx->xio_bc0e); cudaFree(ctx->xio_mpart); cudaFree(ctx->xio_yd); cudaFree(ctx->xio_state); cudaFree(ctx->xio_part);
    for (auto& e : ctx->xev)
        if (e) cudaEventDestroy(e);
    if (ctx->pio_h2d) cudaStreamSynchronize(ctx->pio_h2d);
    if (ctx->pio_d2h) cudaStreamSynchronize(ctx->pio_d2h);
    for (int b = 0; b < 2; ++b) {
        cudaFree(ctx->pio_in[b]); cudaFree(ctx->pio_out[b]);
        for (cudaEvent_t e : {ctx->pio_in_ready[b], ctx->pio_in_free[b], ctx->pio_out_ready[b], ctx->pio_out_free[b]})
            if (e) cudaEventDestroy(e);
    }
    if (ctx->pio_h2d) cudaStreamDestroy(ctx->pio_h2d);
    if (ctx->pio_d2h) cudaStreamDestroy(ctx->pio_d2h);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* chapsim_last_error_string(const chapsim_ctx_t* ctx) {
    return ctx ? ctx->err.c_str() : g_init_error.c_str();
}

int chapsim_upload_fields(chapsim_ctx_t* ctx, const double* q, const double* pr, const double* convh0) {
    if (!ctx || !q || !pr) return fail(ctx, CHAPSIM_ERR_BADARG, "null field");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    CK(cudaMemcpyAsync(ctx->Q, q, (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->PR, pr, (size_t)g.FS * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (convh0)
        CK(cudaMemcpyAsync(ctx->H0, convh0, (size_t)(3 * g.FI) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    else
        CK(cudaMemsetAsync(ctx->H0, 0, (size_t)(3 * g.FI) * sizeof(double), ctx->stream));
    k_bc_fields<double><<<ctx->npart_red, DG_NT, 0, ctx->stream>>>(g, ctx->Q, ctx->PR);
    ctx->launches += 1;
    CK(cudaGetLastError());
    if (ctx->prec == CHAPSIM_PREC_MIXED) {
        int rc = mixed_from_staging(ctx, true);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_download_fields(chapsim_ctx_t* ctx, double* q, double* pr, double* convh0) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    if (ctx->prec == CHAPSIM_PREC_MIXED) {
        int rc = mixed_to_staging(ctx, q != nullptr, pr != nullptr, convh0 != nullptr);
        if (rc) return rc;
    }
    if (q) CK(cudaMemcpyAsync(q, ctx->Q, (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (pr) CK(cudaMemcpyAsync(pr, ctx->PR, (size_t)g.FS * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (convh0)
        CK(cudaMemcpyAsync(convh0, ctx->H0, (size_t)(3 * g.FI) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

// ---------------------------------------------------------------------------
// Pipelined host I/O.  The fields of a run that streams them from and to host
// memory every step pass through two device staging slots in each direction,
// so that the H2D copy of the next step's input, the D2H copy of the last
// step's result and the step itself run at the same time (the copy engines of
// the two directions and the SMs).  Q and PR of a slot are one allocation
// (3 FS + FS words).
static int pio_setup(chapsim_ctx* ctx) {
    if (ctx->pio_h2d) return CHAPSIM_OK;
    const size_t bytes = (size_t)(4 * ctx->g.FS) * sizeof(double);
    for (int b = 0; b < 2; ++b) {
        CK(cudaMalloc(&ctx->pio_in[b], bytes));
        CK(cudaMalloc(&ctx->pio_out[b], bytes));
        for (cudaEvent_t* e : {&ctx->pio_in_ready[b], &ctx->pio_in_free[b], &ctx->pio_out_ready[b], &ctx->pio_out_free[b]})
            CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    CK(cudaStreamCreateWithFlags(&ctx->pio_h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ctx->pio_d2h, cudaStreamNonBlocking));
    return CHAPSIM_OK;
}

// The oldest pending upload becomes the context's fields, on the step stream:
// the staged Q and PR copied in, CONVH0 zeroed, the wall ghosts set (as
// chapsim_upload_fields), and in mixed precision the FP32 fields converted.
static int pio_commit(chapsim_ctx* ctx) {
    if (ctx->pio_in_pending == 0) return CHAPSIM_OK;
    const Geo& g = ctx->g;
    const int b = ctx->pio_in_head;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->pio_in_ready[b], 0));
    CK(cudaMemcpyAsync(ctx->Q, ctx->pio_in[b], (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->PR, ctx->pio_in[b] + 3 * g.FS, (size_t)g.FS * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    CK(cudaEventRecord(ctx->pio_in_free[b], ctx->stream));
    CK(cudaMemsetAsync(ctx->H0, 0, (size_t)(3 * g.FI) * sizeof(double), ctx->stream));
    k_bc_fields<double><<<ctx->npart_red, DG_NT, 0, ctx->stream>>>(g, ctx->Q, ctx->PR);
    ctx->launches += 1;
    CK(cudaGetLastError());
    if (ctx->prec == CHAPSIM_PREC_MIXED) {
        int rc = mixed_from_staging(ctx, true);
        if (rc) return rc;
    }
    ctx->pio_in_head ^= 1;
    ctx->pio_in_pending -= 1;
    return CHAPSIM_OK;
}

int chapsim_upload_fields_async(chapsim_ctx_t* ctx, const double* q, const double* pr) {
    if (!ctx || !q || !pr) return fail(ctx, CHAPSIM_ERR_BADARG, "null field");
    if (ctx->domain != 1) return fail(ctx, CHAPSIM_ERR_BADARG, "pipelined host I/O is for the periodic channel (TG)");
    CK(cudaSetDevice(ctx->device));
    int rc = pio_setup(ctx);
    if (rc) return rc;
    if (ctx->pio_in_pending == 2) rc = pio_commit(ctx);  // both slots hold uploads: the older one goes in first
    if (rc) return rc;
    const Geo& g = ctx->g;
    const int b = ctx->pio_in_next;
    CK(cudaStreamWaitEvent(ctx->pio_h2d, ctx->pio_in_free[b], 0));  // the slot's last commit has read it
    CK(cudaMemcpyAsync(ctx->pio_in[b], q, (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyHostToDevice, ctx->pio_h2d));
    CK(cudaMemcpyAsync(ctx->pio_in[b] + 3 * g.FS, pr, (size_t)g.FS * sizeof(double), cudaMemcpyHostToDevice, ctx->pio_h2d));
    CK(cudaEventRecord(ctx->pio_in_ready[b], ctx->pio_h2d));
    ctx->pio_in_next ^= 1;
    ctx->pio_in_pending += 1;
    return CHAPSIM_OK;
}

int chapsim_download_fields_async(chapsim_ctx_t* ctx, double* q, double* pr) {
    if (!ctx || !q || !pr) return fail(ctx, CHAPSIM_ERR_BADARG, "null field");
    if (ctx->domain != 1) return fail(ctx, CHAPSIM_ERR_BADARG, "pipelined host I/O is for the periodic channel (TG)");
    CK(cudaSetDevice(ctx->device));
    int rc = pio_setup(ctx);
    if (rc) return rc;
    const Geo& g = ctx->g;
    if (ctx->prec == CHAPSIM_PREC_MIXED) {
        rc = mixed_to_staging(ctx, true, true, false);
        if (rc) return rc;
    }
    const int b = ctx->pio_out_next;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->pio_out_free[b], 0));  // the slot's last D2H copy has read it
    CK(cudaMemcpyAsync(ctx->pio_out[b], ctx->Q, (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->pio_out[b] + 3 * g.FS, ctx->PR, (size_t)g.FS * sizeof(double), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    CK(cudaEventRecord(ctx->pio_out_ready[b], ctx->stream));
    CK(cudaStreamWaitEvent(ctx->pio_d2h, ctx->pio_out_ready[b], 0));
    CK(cudaMemcpyAsync(q, ctx->pio_out[b], (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyDeviceToHost, ctx->pio_d2h));
    CK(cudaMemcpyAsync(pr, ctx->pio_out[b] + 3 * g.FS, (size_t)g.FS * sizeof(double), cudaMemcpyDeviceToHost, ctx->pio_d2h));
    CK(cudaEventRecord(ctx->pio_out_free[b], ctx->pio_d2h));
    ctx->pio_out_next ^= 1;
    return CHAPSIM_OK;
}

int chapsim_io_wait(chapsim_ctx_t* ctx) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    if (ctx->pio_h2d) CK(cudaStreamSynchronize(ctx->pio_h2d));
    if (ctx->pio_d2h) CK(cudaStreamSynchronize(ctx->pio_d2h));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_set_dt(chapsim_ctx_t* ctx, double dt) {
    if (!ctx || !(dt > 0.0)) return fail(ctx, CHAPSIM_ERR_BADARG, "dt must be positive");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(&ctx->st->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_get_dt(chapsim_ctx_t* ctx, double* dt) {
    if (!ctx || !dt) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *dt = ctx->st_host->dt;
    return CHAPSIM_OK;
}

int chapsim_cfl_tg(chapsim_ctx_t* ctx, double* cflmm) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    if (ctx->domain != 1) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the periodic TG domain");
    CK(cudaSetDevice(ctx->device));
    launch_cfl_dt(ctx, 0);
    CK(cudaGetLastError());
    int rc = check_device_error(ctx);
    if (cflmm) *cflmm = ctx->st_host->cflmm;
    return rc;
}

static int set_step_params(chapsim_ctx_t* ctx, double dt0, double dtmin, double cflgv) {
    if (!(dt0 > 0.0) || !(dtmin > 0.0) || !(cflgv > 0.0)) return fail(ctx, CHAPSIM_ERR_BADARG, "dt0, dtmin, cflgv must be positive");
    double p[3] = {dt0, dtmin, cflgv};
    CK(cudaMemcpyAsync(&ctx->st->dt0, p, 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_step_begin(chapsim_ctx_t* ctx, double dt0, double dtmin, double cflgv, double* dt_out, double* cfl_out) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    int rc = set_step_params(ctx, dt0, dtmin, cflgv);
    if (rc) return rc;
    if (ctx->domain >= 2) launch_io_step_start(ctx);
    else launch_cfl_dt(ctx, 1);
    CK(cudaGetLastError());
    rc = check_device_error(ctx);
    if (dt_out) *dt_out = ctx->st_host->dt;
    if (cfl_out) *cfl_out = ctx->st_host->cflmm;
    return rc;
}

int chapsim_rk_substep_tg(chapsim_ctx_t* ctx, int32_t ns) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    if (ctx->domain != 1) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the periodic TG domain");
    if (ns < 0 || ns > 3) return fail(ctx, CHAPSIM_ERR_BADARG, "NS must be 0..3");
    CK(cudaSetDevice(ctx->device));
    launch_substep(ctx, ns);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_advance_tg(chapsim_ctx_t* ctx, int32_t nsteps, double dt0, double dtmin, double cflgv, double* dt_out,
                       double* cfl_out) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    if (nsteps < 0) return fail(ctx, CHAPSIM_ERR_BADARG, "nsteps < 0");
    if (ctx->domain == 3)
        return fail(ctx, CHAPSIM_ERR_BADARG, "the inflow/outflow main domain steps with its TG domain: chapsim_advance_xinout");
    CK(cudaSetDevice(ctx->device));
    int rc = pio_commit(ctx);  // the oldest fields of chapsim_upload_fields_async, if any wait
    if (rc) return rc;
    rc = set_step_params(ctx, dt0, dtmin, cflgv);
    if (rc) return rc;
    rc = build_step_graph(ctx);
    if (rc) return rc;
    for (int s = 0; s < nsteps; ++s) {
        CK(cudaGraphLaunch(ctx->step_exec, ctx->stream));
        ctx->launches += (unsigned long long)ctx->kernels_per_step;
    }
    CK(cudaGetLastError());
    rc = check_device_error(ctx);
    if (dt_out) *dt_out = ctx->st_host->dt;
    if (cfl_out) *cfl_out = ctx->st_host->cflmm;
    return rc;
}

int chapsim_divgck_tg(chapsim_ctx_t* ctx, double* maxdiv) {
    if (!ctx || !maxdiv) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    if (ctx->prec == CHAPSIM_PREC_MIXED) k_divgck<float><<<ctx->npart_red, DG_NT, 0, ctx->stream>>>(ctx->g, ctx->Qf, ctx->part_red);
    else k_divgck<double><<<ctx->npart_red, DG_NT, 0, ctx->stream>>>(ctx->g, ctx->Q, ctx->part_red);
    k_maxdiv_final<<<1, DG_NT, 0, ctx->stream>>>(ctx->part_red, ctx->npart_red, ctx->st);
    ctx->launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *maxdiv = ctx->st_host->maxdiv;
    return CHAPSIM_OK;
}

// ---- statistics of the periodic channel ----
namespace {
int pp_ensure(chapsim_ctx* ctx) {
    if (ctx->domain != 1) return fail(ctx, CHAPSIM_ERR_BADARG, "the x-z statistics cover the periodic TG domain");
    if (ctx->pp_inst) return CHAPSIM_OK;
    const Geo& g = ctx->g;
    const size_t nset = (size_t)PP_PER_ROW * g.M;
    int nchunk = (4 * ctx->nsm + g.M - 1) / g.M;
    nchunk = std::max(1, std::min(nchunk, g.L * g.N / PP_NT));
    ctx->pp_nchunk = nchunk;
    CK(cudaMalloc(&ctx->pp_inst, nset * sizeof(double)));
    CK(cudaMalloc(&ctx->pp_avg, nset * sizeof(double)));
    CK(cudaMalloc(&ctx->pp_part, (size_t)g.M * nchunk * PP_NACC * sizeof(double)));
    CK(cudaMalloc(&ctx->pp_mon, 20 * sizeof(double)));
    CK(cudaMemsetAsync(ctx->pp_inst, 0, nset * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(ctx->pp_avg, 0, nset * sizeof(double), ctx->stream));
    ctx->nstatis = 0;
    return CHAPSIM_OK;
}
// the seven arrays of one set, in storage order, with their widths
const int pp_width[7] = {4, 3, 6, 10, 9, 9, 81};
const int pp_off[7] = {PP_U1, PP_UP, PP_U2, PP_U3, PP_D1, PP_DP, PP_D2};
extern "C++" {  // a template, inside the C-linkage block of the ABI
// the seven sum groups of the main-domain means (stats_io.cuh), for the field type F
template <typename F>
void pp_io_launch(chapsim_ctx* ctx, IoFieldsT<F> f, int ngroups) {
    const Geo& g = ctx->g;
    dim3 grid(ctx->pp_nchunk, g.M);
    cudaStream_t s = ctx->stream;
    const int nc = ctx->pp_nchunk;
    k_pp_io<0, F><<<grid, PP_NT, 0, s>>>(g, f, ctx->tf, ctx->ppio_part);
    k_pp_io_finish<0><<<g.M, PP_NT, 0, s>>>(g, ctx->ppio_part, nc, ctx->ppio_set);
    k_pp_io<1, F><<<grid, PP_NT, 0, s>>>(g, f, ctx->tf, ctx->ppio_part);
    k_pp_io_finish<1><<<g.M, PP_NT, 0, s>>>(g, ctx->ppio_part, nc, ctx->ppio_set);
    if (ngroups > 2) {
        k_pp_io<2, F><<<grid, PP_NT, 0, s>>>(g, f, ctx->tf, ctx->ppio_part);
        k_pp_io_finish<2><<<g.M, PP_NT, 0, s>>>(g, ctx->ppio_part, nc, ctx->ppio_set);
        k_pp_io<3, F><<<grid, PP_NT, 0, s>>>(g, f, ctx->tf, ctx->ppio_part);
        k_pp_io_finish<3><<<g.M, PP_NT, 0, s>>>(g, ctx->ppio_part, nc, ctx->ppio_set);
        k_pp_io<4, F><<<grid, PP_NT, 0, s>>>(g, f, ctx->tf, ctx->ppio_part);
        k_pp_io_finish<4><<<g.M, PP_NT, 0, s>>>(g, ctx->ppio_part, nc, ctx->ppio_set);
        k_pp_io<5, F><<<grid, PP_NT, 0, s>>>(g, f, ctx->tf, ctx->ppio_part);
        k_pp_io_finish<5><<<g.M, PP_NT, 0, s>>>(g, ctx->ppio_part, nc, ctx->ppio_set);
        k_pp_io<6, F><<<grid, PP_NT, 0, s>>>(g, f, ctx->tf, ctx->ppio_part);
        k_pp_io_finish<6><<<g.M, PP_NT, 0, s>>>(g, ctx->ppio_part, nc, ctx->ppio_set);
    }
    ctx->launches += 2 * ngroups;
}

}  // extern "C++"
}  // namespace

int chapsim_pp_mean_zx_tg(chapsim_ctx_t* ctx) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    int rc = pp_ensure(ctx);
    if (rc) return rc;
    const Geo& g = ctx->g;
    dim3 grid(ctx->pp_nchunk, g.M);
    if (ctx->prec == CHAPSIM_PREC_MIXED)
        k_pp_mean_zx<float><<<grid, PP_NT, 0, ctx->stream>>>(g, ctx->Qf, ctx->PRf, ctx->pp_part);
    else
        k_pp_mean_zx<double><<<grid, PP_NT, 0, ctx->stream>>>(g, ctx->Q, ctx->PR, ctx->pp_part);
    k_pp_finish<<<g.M, PP_NT, 0, ctx->stream>>>(g, ctx->pp_part, ctx->pp_nchunk, ctx->pp_inst);
    ctx->launches += 2;
    CK(cudaGetLastError());
    return CHAPSIM_OK;
}

int chapsim_pp_mean_zx_io(chapsim_ctx_t* ctx) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    if (ctx->domain != 2) return fail(ctx, CHAPSIM_ERR_BADARG, "the main-domain statistics need a main-domain context");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    if (!ctx->ppio_set) {
        int nchunk = (4 * ctx->nsm + g.M - 1) / g.M;
        nchunk = std::max(1, std::min(nchunk, g.L * g.N / PP_NT));
        ctx->pp_nchunk = ctx->pp_nchunk ? ctx->pp_nchunk : nchunk;
        CK(cudaMalloc(&ctx->ppio_set, (size_t)PPIO_ALL * g.M * sizeof(double)));
        CK(cudaMalloc(&ctx->ppio_part, (size_t)g.M * ctx->pp_nchunk * 60 * sizeof(double)));
        CK(cudaMemsetAsync(ctx->ppio_set, 0, (size_t)PPIO_ALL * g.M * sizeof(double), ctx->stream));
    }
    const int ngroups = ctx->thermal ? 7 : 2;
    if (ctx->prec == CHAPSIM_PREC_MIXED) pp_io_launch<float>(ctx, io_fields_t<float>(ctx), ngroups);
    else pp_io_launch<double>(ctx, io_fields_t<double>(ctx), ngroups);
    CK(cudaGetLastError());
    return CHAPSIM_OK;
}

int chapsim_download_pp_means_io(chapsim_ctx_t* ctx, double* out, int32_t* per_row) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    if (ctx->domain != 2) return fail(ctx, CHAPSIM_ERR_BADARG, "the main-domain statistics need a main-domain context");
    if (!ctx->ppio_set) return fail(ctx, CHAPSIM_ERR_BADARG, "no main-domain means yet (call chapsim_pp_mean_zx_io)");
    CK(cudaSetDevice(ctx->device));
    const int nr = ctx->thermal ? PPIO_ALL : PPIO_FLOW;
    if (per_row) *per_row = nr;
    if (out) {
        CK(cudaMemcpyAsync(out, ctx->ppio_set, (size_t)nr * ctx->g.M * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return CHAPSIM_OK;
}

int chapsim_pp_mean_t_tg(chapsim_ctx_t* ctx, int32_t tp, int32_t pp_instn_sz) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    if (tp != 1 && tp != 2) return fail(ctx, CHAPSIM_ERR_BADARG, "TP must be T_Asymptotic_Average (1) or T_Summing_average (2)");
    if (tp == 2 && pp_instn_sz < 1) return fail(ctx, CHAPSIM_ERR_BADARG, "pp_instn_sz must be >= 1");
    CK(cudaSetDevice(ctx->device));
    int rc = pp_ensure(ctx);
    if (rc) return rc;
    ctx->nstatis += 1;
    double coe2, coe3;
    if (tp == 1) {
        coe2 = 1.0 / (double)ctx->nstatis;
        coe3 = (double)(ctx->nstatis - 1) / (double)ctx->nstatis;
    } else {
        coe2 = 1.0 / (double)pp_instn_sz;
        coe3 = 1.0;
    }
    const long long n = (long long)PP_PER_ROW * ctx->g.M;
    k_pp_time_average<<<(int)std::min<long long>((n + 255) / 256, 4LL * ctx->nsm), 256, 0, ctx->stream>>>(
        ctx->pp_avg, ctx->pp_inst, n, coe2, coe3);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return CHAPSIM_OK;
}

int chapsim_pp_monitor_tg(chapsim_ctx_t* ctx, double ren, double* mon) {
    if (!ctx || !mon || !(ren > 0.0)) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    int rc = pp_ensure(ctx);
    if (rc) return rc;
    k_pp_monitor<<<1, 32, 0, ctx->stream>>>(ctx->g, ctx->pp_inst, ctx->pp_avg, ren, ctx->pp_mon);
    ctx->launches += 1;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(mon, ctx->pp_mon, 20 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_download_pp_means_tg(chapsim_ctx_t* ctx, int32_t averaged, double* u1, double* up, double* u2,
                                 double* u3, double* dvdl1, double* dvdlp, double* dvdl2, int32_t* nstatis) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    int rc = pp_ensure(ctx);
    if (rc) return rc;
    const double* src = averaged ? ctx->pp_avg : ctx->pp_inst;
    double* dst[7] = {u1, up, u2, u3, dvdl1, dvdlp, dvdl2};
    const size_t M = (size_t)ctx->g.M;
    for (int a = 0; a < 7; ++a)
        if (dst[a])
            CK(cudaMemcpyAsync(dst[a], src + pp_off[a] * M, pp_width[a] * M * sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (nstatis) *nstatis = ctx->nstatis;
    return CHAPSIM_OK;
}

int chapsim_upload_pp_means_tg(chapsim_ctx_t* ctx, int32_t nstatis, const double* u1, const double* up,
                               const double* u2, const double* u3, const double* dvdl1, const double* dvdlp,
                               const double* dvdl2) {
    if (!ctx || nstatis < 0) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    int rc = pp_ensure(ctx);
    if (rc) return rc;
    const double* src[7] = {u1, up, u2, u3, dvdl1, dvdlp, dvdl2};
    const size_t M = (size_t)ctx->g.M;
    for (int a = 0; a < 7; ++a)
        if (src[a])
            CK(cudaMemcpyAsync(ctx->pp_avg + pp_off[a] * M, src[a], pp_width[a] * M * sizeof(double),
                               cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->nstatis = nstatis;
    return CHAPSIM_OK;
}

int chapsim_fft99_pois3d(chapsim_ctx_t* ctx, const double* rhs, double* dph) {
    if (!ctx || !rhs || !dph) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    // the divergence kernel is bypassed: RHSLLPHI is uploaded and packed by a
    // copy of the x-transform path that reads it instead of Q
    CK(cudaMemcpyAsync(ctx->RHSLL, rhs, (size_t)g.FI * sizeof(double), cudaMemcpyHostToDevice, s));
    dim3 grp((g.M + PX_TJ - 1) / PX_TJ, g.N);
    DISPATCH_FFT(g.L, (k_fftx_from_rhs<FN1, FN2><<<grp, PX_NT, smem_px(g), s>>>(g, ctx->RHSLL, ctx->SP)));
    const long long nq = (long long)g.LH * g.M;
    const int gfz = (int)((nq + FZ_TQ - 1) / FZ_TQ);
    DISPATCH_FFT(g.N, (k_fftz<-1, FN1, FN2, double2><<<gfz, FZ_NT, smem_fz(g), s>>>(g, ctx->SP, 0)));
    launch_ysolve<double2>(ctx);
    DISPATCH_FFT(g.N, (k_fftz<+1, FN1, FN2, double2><<<gfz, FZ_NT, smem_fz(g), s>>>(g, ctx->SP, 0)));
    DISPATCH_FFT(g.L, (k_fftx_inv<FN1, FN2, double2><<<grp, PX_NT, smem_px(g), s>>>(g, ctx->SP, ctx->DPH)));
    ctx->launches += 5;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dph, ctx->DPH, (size_t)g.FS * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return CHAPSIM_OK;
}

int chapsim_profile_steps(chapsim_ctx_t* ctx, int32_t nsteps, double dt0, double dtmin, double cflgv, float* ms,
                          int32_t nslots) {
    // One step = 2 + 3*9 kernel slots (2 + 3*15 with the thermal solver of the
    // main domain), launched individually with an event after each; ms[slot]
    // accumulates the duration of slot `slot` over the nsteps steps (slot 0 is
    // timed from an event recorded before it).
    if (!ctx) return CHAPSIM_ERR_BADARG;
    if (ctx->domain == 3) return fail(ctx, CHAPSIM_ERR_BADARG, "profile the inflow/outflow main domain's kernels with ncu");
    const int per = 2 + 3 * (9 + (ctx->thermal ? 6 : 0));
    if (!ms || nslots < per || nsteps < 1)
        return fail(ctx, CHAPSIM_ERR_BADARG, "ms must hold " + std::to_string(per) + " slots and nsteps >= 1");
    CK(cudaSetDevice(ctx->device));
    int rc = set_step_params(ctx, dt0, dtmin, cflgv);
    if (rc) return rc;
    std::vector<cudaEvent_t> ev(per + 1);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int i = 0; i < per; ++i) ms[i] = 0.0f;
    for (int s = 0; s < nsteps; ++s) {
        CK(cudaEventRecord(ev[0], ctx->stream));
        ctx->prof_ev = ev.data() + 1;
        ctx->prof_n = 0;
        if (ctx->domain == 2) {
            launch_io_step_start(ctx);
            for (int ns = 1; ns <= 3; ++ns) launch_io_substep(ctx, ns);
        } else {
            launch_step_start(ctx);
            for (int ns = 1; ns <= 3; ++ns) launch_substep(ctx, ns, false);
        }
        ctx->prof_ev = nullptr;
        CK(cudaGetLastError());
        CK(cudaEventSynchronize(ev[per]));
        for (int i = 0; i < per; ++i) {
            float t = 0.0f;
            CK(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
            ms[i] += t;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return check_device_error(ctx);
}

int chapsim_upload_io_fields(chapsim_ctx_t* ctx, const double* gq, const double* pr, const double* rho,
                             const double* mu0, const double* mu) {
    if (!ctx || !gq || !pr || !rho || !mu0 || !mu) return fail(ctx, CHAPSIM_ERR_BADARG, "null field");
    if (ctx->domain < 2) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the main (IO) domain");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    IoFields& f = ctx->io;
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(f.G, gq, (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->PR, pr, (size_t)g.FS * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(f.RHO, rho, (size_t)g.FS * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(f.MU0, mu0, (size_t)g.FS * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(f.MU, mu, (size_t)g.FS * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(f.EX0, 0, (size_t)(3 * g.FI) * sizeof(double), s));
    if (io_mixed(ctx)) {
        // the FP64 host fields rounded once into the FP32 flow fields
        const int nb = 4 * ctx->nsm;
        IoFieldsT<float> ff = io_fields_t<float>(ctx);
        k_convert<float, double><<<nb, DG_NT, 0, s>>>(ff.G, f.G, 3 * g.FS);
        k_convert<float, double><<<nb, DG_NT, 0, s>>>(ctx->PRf, ctx->PR, g.FS);
        CK(cudaMemsetAsync(ff.EX0, 0, (size_t)(3 * g.FI) * sizeof(float), s));
        k_bc_fields<float><<<ctx->npart_red, DG_NT, 0, s>>>(g, ff.G, ctx->PRf);
        k_io_props<float><<<ctx->io_grid, IO_NT, 0, s>>>(g, ff);
        k_io_velocity<float><<<ctx->io_grid, IO_NT, 0, s>>>(g, ff);
        k_bc_fields<float><<<ctx->npart_red, DG_NT, 0, s>>>(g, ctx->Qf, ctx->PRf);
        ctx->launches += 6;
    } else {
        k_bc_fields<double><<<ctx->npart_red, DG_NT, 0, s>>>(g, f.G, ctx->PR);  // BC_WALL_G_io, BC_WALL_PR_io
        k_io_props<double><<<ctx->io_grid, IO_NT, 0, s>>>(g, io_fields(ctx));   // DENSITY_Staggered, MU_Staggered
        k_io_velocity<double><<<ctx->io_grid, IO_NT, 0, s>>>(g, io_fields(ctx));  // VELOCITY_CALC_io
        k_bc_fields<double><<<ctx->npart_red, DG_NT, 0, s>>>(g, ctx->Q, ctx->PR);  // BC_WALL_Q_io
        ctx->launches += 4;
        if (ctx->domain == 3) {
            k_xio_ghost_velocity<<<4 * ctx->nsm, XIO_NT, 0, s>>>(g, io_fields(ctx));
            k_bc_fields<double><<<ctx->npart_red, DG_NT, 0, s>>>(g, ctx->Q, ctx->PR);
            CK(cudaMemsetAsync(ctx->xio_bc0, 0, (size_t)3 * g.M * g.N * sizeof(double), s));
            ctx->launches += 2;
        }
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return CHAPSIM_OK;
}

int chapsim_download_io_fields(chapsim_ctx_t* ctx, double* gq, double* q, double* pr) {
    if (!ctx || ctx->domain < 2) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the main (IO) domain");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    if (io_mixed(ctx)) {  // widen the FP32 flow fields into the FP64 staging arrays first
        const int nb = 4 * ctx->nsm;
        if (gq) k_convert<double, float><<<nb, DG_NT, 0, ctx->stream>>>(ctx->io.G, ctx->iof.G, 3 * g.FS);
        if (q) k_convert<double, float><<<nb, DG_NT, 0, ctx->stream>>>(ctx->Q, ctx->Qf, 3 * g.FS);
        if (pr) k_convert<double, float><<<nb, DG_NT, 0, ctx->stream>>>(ctx->PR, ctx->PRf, g.FS);
        CK(cudaGetLastError());
    }
    if (gq) CK(cudaMemcpyAsync(gq, ctx->io.G, (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (q) CK(cudaMemcpyAsync(q, ctx->Q, (size_t)(3 * g.FS) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (pr) CK(cudaMemcpyAsync(pr, ctx->PR, (size_t)g.FS * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_rk_substep_io(chapsim_ctx_t* ctx, int32_t ns) {
    if (!ctx || ctx->domain < 2) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the main (IO) domain");
    if (ns < 0 || ns > 3) return fail(ctx, CHAPSIM_ERR_BADARG, "NS must be 0..3");
    CK(cudaSetDevice(ctx->device));
    if (ctx->domain == 3) {
        if (!ctx->tg_in) return fail(ctx, CHAPSIM_ERR_BADARG, "no TG context attached (chapsim_xinout_attach)");
        if (ns < 1) return fail(ctx, CHAPSIM_ERR_BADARG, "the inflow/outflow main domain has substeps NS = 1..3");
        if (ctx->thermal && !ctx->xio_in_set)
            return fail(ctx, CHAPSIM_ERR_BADARG, "the thermal inflow needs its inlet state (chapsim_xinout_thermal_inlet)");
        CK(cudaStreamSynchronize(ctx->tg_in->stream));  // the TG substep NS feeds the inlet
        launch_xio_substep(ctx, ns);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->stream));
        return check_device_error(ctx);
    }
    launch_io_substep(ctx, ns);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

// the captured step graph holds the kernels' arguments: a new setting needs a new capture
static int drop_step_graph(chapsim_ctx* ctx) {
    if (ctx->step_exec) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaGraphExecDestroy(ctx->step_exec);
        ctx->step_exec = nullptr;
    }
    return CHAPSIM_OK;
}

int chapsim_set_buoyancy(chapsim_ctx_t* ctx, int32_t igravity, double f_a) {
    if (!ctx || ctx->domain < 2) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the main (IO) domain");
    if (igravity < -3 || igravity > 3 || !std::isfinite(f_a))
        return fail(ctx, CHAPSIM_ERR_BADARG, "iGravity must be in -3..3 and F_A finite");
    CK(cudaSetDevice(ctx->device));
    ctx->io.igrav = igravity;
    ctx->io.fa = igravity ? f_a : 0.0;
    return drop_step_graph(ctx);
}

int chapsim_upload_weighted_pressure(chapsim_ctx_t* ctx, const double* pr0_1, const double* pr0_2) {
    if (!ctx || ctx->domain != 2) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the main (IO) domain");
    if ((pr0_1 == nullptr) != (pr0_2 == nullptr))
        return fail(ctx, CHAPSIM_ERR_BADARG, "give both PR0_io layers, or neither to turn iWeightedPre off");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    const size_t fb = (size_t)g.FS * sizeof(double);
    if (!pr0_1) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(const_cast<double*>(ctx->io.PR0A));
        ctx->io.PR0A = ctx->io.PR0B = nullptr;
        return drop_step_graph(ctx);
    }
    if (!ctx->io.PR0A) {  // the two layers in one allocation
        double* p = nullptr;
        CK(cudaMalloc(&p, 2 * fb));
        ctx->io.PR0A = p;
        ctx->io.PR0B = p + g.FS;
    }
    CK(cudaMemcpyAsync(const_cast<double*>(ctx->io.PR0A), pr0_1, fb, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(const_cast<double*>(ctx->io.PR0B), pr0_2, fb, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return drop_step_graph(ctx);
}

int chapsim_cfl_io(chapsim_ctx_t* ctx, double* cflmm) {
    if (!ctx || ctx->domain < 2) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the main (IO) domain");
    CK(cudaSetDevice(ctx->device));
    if (io_mixed(ctx)) k_io_cfl<float><<<ctx->npart_red, IO_NT, 0, ctx->stream>>>(ctx->g, io_fields_t<float>(ctx), ctx->part_red, ctx->st);
    else k_io_cfl<double><<<ctx->npart_red, IO_NT, 0, ctx->stream>>>(ctx->g, io_fields(ctx), ctx->part_red, ctx->st);
    k_dt<<<1, DG_NT, 0, ctx->stream>>>(ctx->part_red, ctx->npart_red, ctx->st, 0);
    ctx->launches += 2;
    CK(cudaGetLastError());
    int rc = check_device_error(ctx);
    if (cflmm) *cflmm = ctx->st_host->cflmm;
    return rc;
}

int chapsim_probe_wait_timeout(chapsim_ctx_t* ctx) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    k_wait_probe<<<1, 32, 0, ctx->stream>>>(&ctx->st->err);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return check_device_error(ctx);
}

int chapsim_xinout_attach(chapsim_ctx_t* io, chapsim_ctx_t* tg) {
    if (!io || !tg) return fail(io, CHAPSIM_ERR_BADARG, "null context");
    if (io->domain != 3) return fail(io, CHAPSIM_ERR_BADARG, "context was not created for the inflow/outflow main domain");
    if (tg->domain != 1 || tg->prec != CHAPSIM_PREC_FP64)
        return fail(io, CHAPSIM_ERR_BADARG, "the inlet is fed by an FP64 periodic TG context");
    if (tg->device != io->device || tg->g.M != io->g.M || tg->g.N != io->g.N)
        return fail(io, CHAPSIM_ERR_BADARG, "the TG context must be on the same device with the same NCL2, NCL3");
    io->tg_in = tg;
    return CHAPSIM_OK;
}

int chapsim_advance_xinout(chapsim_ctx_t* io, int32_t nsteps, double dt0, double dtmin, double cflgv, double* dt_out,
                           double* cfl_out) {
    if (!io) return CHAPSIM_ERR_BADARG;
    if (io->domain != 3) return fail(io, CHAPSIM_ERR_BADARG, "context was not created for the inflow/outflow main domain");
    if (!io->tg_in) return fail(io, CHAPSIM_ERR_BADARG, "no TG context attached (chapsim_xinout_attach)");
    if (nsteps < 0) return fail(io, CHAPSIM_ERR_BADARG, "nsteps < 0");
    if (io->thermal && !io->xio_in_set)
        return fail(io, CHAPSIM_ERR_BADARG, "the thermal inflow needs its inlet state (chapsim_xinout_thermal_inlet)");
    chapsim_ctx* tg = io->tg_in;
    chapsim_ctx* ctx = io;  // for CK
    CK(cudaSetDevice(io->device));
    int rc = set_step_params(io, dt0, dtmin, cflgv);
    if (rc) return rc;
    rc = set_step_params(tg, dt0, dtmin, cflgv);
    if (rc) return fail(io, rc, tg->err);
    for (int s = 0; s < nsteps; ++s) {
        launch_xio_step_start(io);
        for (int ns = 1; ns <= 3; ++ns) launch_xio_pair_substep(io, ns);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(tg->stream));
    rc = check_device_error(tg);
    if (rc) return fail(io, rc, "TG domain: " + tg->err);
    rc = check_device_error(io);
    if (dt_out) *dt_out = io->st_host->dt;
    if (cfl_out) *cfl_out = io->st_host->cflmm;
    return rc;
}

int chapsim_xinout_thermal_inlet(chapsim_ctx_t* ctx, const double* state7) {
    if (!ctx || !state7) return fail(ctx, CHAPSIM_ERR_BADARG, "null argument");
    if (ctx->domain != 3 || !ctx->thermal)
        return fail(ctx, CHAPSIM_ERR_BADARG, "needs an inflow/outflow main domain with the thermal solver initialised");
    for (int a = 0; a < 7; ++a)
        if (!std::isfinite(state7[a])) return fail(ctx, CHAPSIM_ERR_BADARG, "non-finite inlet state");
    CK(cudaSetDevice(ctx->device));
    for (int a = 0; a < 7; ++a) ctx->xio_in.v[a] = state7[a];
    ctx->xio_in_set = true;
    const Geo& g = ctx->g;
    const int gin = (int)std::min<long long>(4LL * ctx->nsm, ((long long)(g.M + 2) * g.N + XIO_NT - 1) / XIO_NT);
    k_xio_thermal_inlet<<<gin, XIO_NT, 0, ctx->stream>>>(g, io_fields(ctx), ctx->tf, ctx->xio_in);
    ctx->launches += 1;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_divgck_xinout(chapsim_ctx_t* ctx, double* maxdiv3) {
    if (!ctx || !maxdiv3) return CHAPSIM_ERR_BADARG;
    if (ctx->domain != 3) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the inflow/outflow main domain");
    CK(cudaSetDevice(ctx->device));
    const int nb = ctx->npart_red;
    k_xio_divgck<<<nb, XIO_NT, 0, ctx->stream>>>(ctx->g, ctx->io.G, ctx->thermal ? ctx->tf.DRHO : nullptr, ctx->xio_part);
    ctx->launches += 1;
    CK(cudaGetLastError());
    std::vector<double> part((size_t)3 * nb);
    CK(cudaMemcpyAsync(part.data(), ctx->xio_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int r = 0; r < 3; ++r) {
        double m = 0.0;
        for (int b = 0; b < nb; ++b) m = std::max(m, part[(size_t)3 * b + r]);
        maxdiv3[r] = m;
    }
    return CHAPSIM_OK;
}

int chapsim_xinout_outlet_state(chapsim_ctx_t* ctx, double* state2) {
    if (!ctx || !state2) return CHAPSIM_ERR_BADARG;
    if (ctx->domain != 3) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the inflow/outflow main domain");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(state2, ctx->xio_state, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_divgck_io(chapsim_ctx_t* ctx, double* maxdiv) {
    if (!ctx || !maxdiv) return CHAPSIM_ERR_BADARG;
    if (ctx->domain < 2) return fail(ctx, CHAPSIM_ERR_BADARG, "context was not created for the main (IO) domain");
    CK(cudaSetDevice(ctx->device));
    if (io_mixed(ctx))
        k_io_divgck<float><<<ctx->npart_red, IO_NT, 0, ctx->stream>>>(ctx->g, ctx->iof.G,
                                                                      ctx->thermal ? ctx->tf.DRHO : nullptr, ctx->part_red);
    else
        k_io_divgck<double><<<ctx->npart_red, IO_NT, 0, ctx->stream>>>(ctx->g, ctx->io.G,
                                                                       ctx->thermal ? ctx->tf.DRHO : nullptr, ctx->part_red);
    k_maxdiv_final<<<1, DG_NT, 0, ctx->stream>>>(ctx->part_red, ctx->npart_red, ctx->st);
    ctx->launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *maxdiv = ctx->st_host->maxdiv;
    return CHAPSIM_OK;
}

int chapsim_get_stream(chapsim_ctx_t* ctx, void** stream) {
    if (!ctx || !stream) return CHAPSIM_ERR_BADARG;
    *stream = (void*)ctx->stream;
    return CHAPSIM_OK;
}

int chapsim_sync(chapsim_ctx_t* ctx) {
    if (!ctx) return CHAPSIM_ERR_BADARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

int chapsim_launch_count(const chapsim_ctx_t* ctx, uint64_t* count) {
    if (!ctx || !count) return CHAPSIM_ERR_BADARG;
    *count = ctx->launches;
    return CHAPSIM_OK;
}

int chapsim_kernels_per_step(const chapsim_ctx_t* ctx, int32_t* count) {
    if (!ctx || !count) return CHAPSIM_ERR_BADARG;
    int per = 2 + 3 * (ctx->thermal ? 15 : 9 + (ctx->k1_kind == 1 ? 1 : 0));
    *count = per;
    return CHAPSIM_OK;
}

}  // extern "C"

static int run_lines(const double* a, const double* b, const double* c, double* r, const double* bcj, int nlines,
                     long long ls, long long es, int n, bool cyclic) {
    chapsim_ctx* ctx = nullptr;
    if (!a || !b || !c || !r || nlines <= 0 || n < 3) return fail(nullptr, CHAPSIM_ERR_BADARG, "bad tridiagonal arguments");
    const size_t tot = (size_t)nlines * (size_t)n;
    double *da = nullptr, *db = nullptr, *dc = nullptr, *dr = nullptr, *dbc = nullptr, *wk = nullptr;
    auto cleanup = [&]() { cudaFree(da); cudaFree(db); cudaFree(dc); cudaFree(dr); cudaFree(dbc); cudaFree(wk); };
#define LCK(call)                                                                   \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) { cleanup(); return fail(nullptr, CHAPSIM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } \
    } while (0)
    LCK(cudaMalloc(&da, tot * 8)); LCK(cudaMalloc(&db, tot * 8)); LCK(cudaMalloc(&dc, tot * 8)); LCK(cudaMalloc(&dr, tot * 8));
    LCK(cudaMemcpy(da, a, tot * 8, cudaMemcpyHostToDevice));
    LCK(cudaMemcpy(db, b, tot * 8, cudaMemcpyHostToDevice));
    LCK(cudaMemcpy(dc, c, tot * 8, cudaMemcpyHostToDevice));
    LCK(cudaMemcpy(dr, r, tot * 8, cudaMemcpyHostToDevice));
    if (bcj) {
        LCK(cudaMalloc(&dbc, (size_t)2 * nlines * 8));
        LCK(cudaMemcpy(dbc, bcj, (size_t)2 * nlines * 8, cudaMemcpyHostToDevice));
    }
    const int S = n / 32;
    if (n % 32 == 0 && valid_S(S)) {
        const int nt = 256, nb = (int)(((long long)nlines * 32 + nt - 1) / nt);
        if (cyclic) { DISPATCH_S(S, (k_tdma_lines<S, true><<<nb, nt>>>(da, db, dc, dr, dbc, nlines, ls, es, n))); }
        else { DISPATCH_S(S, (k_tdma_lines<S, false><<<nb, nt>>>(da, db, dc, dr, dbc, nlines, ls, es, n))); }
    } else {
        LCK(cudaMalloc(&wk, (size_t)nlines * 3 * n * 8));
        k_tdma_seq<<<(nlines + 127) / 128, 128>>>(da, db, dc, dr, dbc, wk, nlines, ls, es, n, cyclic ? 1 : 0);
    }
    LCK(cudaGetLastError());
    LCK(cudaMemcpy(r, dr, tot * 8, cudaMemcpyDeviceToHost));
    cleanup();
#undef LCK
    return CHAPSIM_OK;
}

extern "C" int chapsim_tdmaiji_cyc(const double* a, const double* b, const double* c, double* r, int32_t isz, int32_t jsz) {
    // lines along I (contiguous), one per J
    return run_lines(a, b, c, r, nullptr, jsz, isz, 1, isz, true);
}

extern "C" int chapsim_tdmaijj_noncyc(const double* a, const double* b, const double* c, double* r, const double* bcj,
                                      int32_t jsz, int32_t isz) {
    // lines along J (stride ISZ), one per I
    return run_lines(a, b, c, r, bcj, isz, 1, isz, jsz, false);
}

// ----------------------- property update by table search -----------------------
namespace {
int first_min(int n, const double* a) {
    int k = 0;
    for (int i = 1; i < n; ++i) if (a[i] < a[k]) k = i;
    return k;
}
int first_max(int n, const double* a) {
    int k = 0;
    for (int i = 1; i < n; ++i) if (a[i] > a[k]) k = i;
    return k;
}
size_t prop_smem(int n) { return n <= PROP_SMEM_MAX_ROWS ? (size_t)2 * n * sizeof(double) : 0; }

int prop_grid(const chapsim_ctx* ctx, long long npts) {
    const long long want = (npts + PROP_NT - 1) / PROP_NT;
    const long long cap = 8LL * ctx->nsm;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

int prop_reset_status(chapsim_ctx* ctx) {
    CK(cudaMemsetAsync(&ctx->pstat->first_bad, 0xff, sizeof(unsigned long long), ctx->stream));
    CK(cudaMemsetAsync(&ctx->pstat->nbad, 0, 2 * sizeof(unsigned int), ctx->stream));
    return CHAPSIM_OK;
}
}  // namespace

extern "C" int chapsim_prop_table_init(chapsim_ctx_t* ctx, const chapsim_prop_table_t* t) {
    if (!ctx || !t) return fail(ctx, CHAPSIM_ERR_BADARG, "null context or table");
    const int n = t->n_list;
    if (n < 4) return fail(ctx, CHAPSIM_ERR_BADARG, "the property table needs N_LIST >= 4 rows");
    const double* need[] = {t->list_h, t->list_t, t->list_d, t->list_m, t->list_k, t->list_cp, t->list_dh,
                            t->dhh_b, t->dhh_c, t->dhh_d, t->ht_b, t->ht_c, t->ht_d, t->hd_b, t->hd_c, t->hd_d,
                            t->hm_b, t->hm_c, t->hm_d, t->hk_b, t->hk_c, t->hk_d, t->hcp_b, t->hcp_c, t->hcp_d};
    for (const double* p : need)
        if (!p) return fail(ctx, CHAPSIM_ERR_BADARG, "null property-table array");
    const double *H = t->list_h, *T = t->list_t, *DH = t->list_dh;
    // the reference's monotonicity checks (SPLINE_COEFFICIENTS_FOR_DH)
    for (int i = 1; i < n - 1; ++i) {
        if (((DH[i] - DH[i - 1]) / (T[i] - T[i - 1])) * ((DH[i + 1] - DH[i]) / (T[i + 1] - T[i])) < 0.0)
            return fail(ctx, CHAPSIM_ERR_BADARG, "the relation (rho * h) = FUNCTION (T) is not monotone");
        if (((DH[i] - DH[i - 1]) / (H[i] - H[i - 1])) * ((DH[i + 1] - DH[i]) / (H[i + 1] - H[i])) < 0.0)
            return fail(ctx, CHAPSIM_ERR_BADARG, "the relation (rho * h) = FUNCTION (h) is not monotone");
    }
    // the binary search assumes ascending abscissae
    for (int i = 1; i < n; ++i)
        if (!(H[i] > H[i - 1]) || !(DH[i] > DH[i - 1]))
            return fail(ctx, CHAPSIM_ERR_BADARG, "LIST_H and LIST_DH must increase strictly along the table");
    // pack: DH->H rows, 5 H-spline rows per table row in output order, then keys
    std::vector<SplineRow> rows((size_t)6 * n);
    const double* ys[5];
    const double* bs[5];
    const double* cs[5];
    const double* ds[5];
    auto put = [&](int s, const double* y, const double* b, const double* c, const double* d) {
        ys[s] = y; bs[s] = b; cs[s] = c; ds[s] = d;
    };
    put(0, t->list_t, t->ht_b, t->ht_c, t->ht_d);
    if (t->fix_swap) {
        put(1, t->list_d, t->hd_b, t->hd_c, t->hd_d);
        put(2, t->list_m, t->hm_b, t->hm_c, t->hm_d);
        put(3, t->list_k, t->hk_b, t->hk_c, t->hk_d);
    } else {  // THERM_PROP_UPDATE_FROM_DH: D <- HM, M <- HK, K <- HD
        put(1, t->list_m, t->hm_b, t->hm_c, t->hm_d);
        put(2, t->list_k, t->hk_b, t->hk_c, t->hk_d);
        put(3, t->list_d, t->hd_b, t->hd_c, t->hd_d);
    }
    put(4, t->list_cp, t->hcp_b, t->hcp_c, t->hcp_d);
    for (int i = 0; i < n; ++i) {
        rows[i] = SplineRow{t->list_h[i], t->dhh_b[i], t->dhh_c[i], t->dhh_d[i]};
        for (int s = 0; s < 5; ++s) rows[(size_t)n + 5 * (size_t)i + s] = SplineRow{ys[s][i], bs[s][i], cs[s][i], ds[s][i]};
    }
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->ptab);
    ctx->ptab = nullptr;
    const size_t rbytes = rows.size() * sizeof(SplineRow);
    const size_t kbytes = (size_t)2 * n * sizeof(double);
    CK(cudaMalloc(&ctx->ptab, rbytes + kbytes));
    if (!ctx->pstat) CK(cudaMalloc(&ctx->pstat, sizeof(PropStatus)));
    char* base = static_cast<char*>(ctx->ptab);
    double* keys = reinterpret_cast<double*>(base + rbytes);
    CK(cudaMemcpy(base, rows.data(), rbytes, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(keys, DH, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(keys + n, H, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    PropTab& tb = ctx->tab;
    tb.n = n;
    tb.imin_h = first_min(n, H);
    tb.imax_h = first_max(n, H);
    tb.imin_dh = first_min(n, DH);
    tb.imax_dh = first_max(n, DH);
    tb.xdh = keys;
    tb.xh = keys + n;
    tb.dhh = reinterpret_cast<const SplineRow*>(base);
    tb.hs = reinterpret_cast<const SplineRow*>(base) + n;
    const size_t sm = prop_smem(n);
    if (sm) {
        CK(set_smem(k_prop_points<true>, sm));
        CK(set_smem(k_prop_fields<true>, sm));
        CK(set_smem(k_eng_props<true, double>, sm));
        CK(set_smem(k_eng_bc<true, double>, sm));
        CK(set_smem(k_eng_props<true, float>, sm));
        CK(set_smem(k_eng_bc<true, float>, sm));
    }
    return CHAPSIM_OK;
}

extern "C" int chapsim_therm_prop_update_points(chapsim_ctx_t* ctx, int64_t npts, const double* dh, double* h,
                                                double* t, double* d, double* m, double* k, double* cp) {
    if (!ctx) return fail(nullptr, CHAPSIM_ERR_BADARG, "null context");
    if (!ctx->ptab) return fail(ctx, CHAPSIM_ERR_BADARG, "no property table (call chapsim_prop_table_init first)");
    if (npts <= 0 || !dh || !h || !t || !d || !m || !k || !cp) return fail(ctx, CHAPSIM_ERR_BADARG, "bad point arrays");
    CK(cudaSetDevice(ctx->device));
    if (npts > ctx->pbuf_pts) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->pbuf);
        ctx->pbuf = nullptr;
        ctx->pbuf_pts = 0;
        CK(cudaMalloc(&ctx->pbuf, (size_t)7 * npts * sizeof(double)));
        ctx->pbuf_pts = npts;
    }
    double* dd = ctx->pbuf;
    double* o = dd + npts;
    const size_t b = (size_t)npts * sizeof(double);
    CK(cudaMemcpyAsync(dd, dh, b, cudaMemcpyHostToDevice, ctx->stream));
    if (int rc = prop_reset_status(ctx)) return rc;
    const size_t sm = prop_smem(ctx->tab.n);
    const int grid = prop_grid(ctx, npts);
    if (sm)
        k_prop_points<true><<<grid, PROP_NT, sm, ctx->stream>>>(ctx->tab, npts, dd, o, o + npts, o + 2 * npts,
                                                                o + 3 * npts, o + 4 * npts, o + 5 * npts, ctx->pstat);
    else
        k_prop_points<false><<<grid, PROP_NT, 0, ctx->stream>>>(ctx->tab, npts, dd, o, o + npts, o + 2 * npts,
                                                                o + 3 * npts, o + 4 * npts, o + 5 * npts, ctx->pstat);
    CK(cudaGetLastError());
    ctx->launches += 1;
    double* outs[6] = {h, t, d, m, k, cp};
    for (int s = 0; s < 6; ++s) CK(cudaMemcpyAsync(outs[s], o + (size_t)s * npts, b, cudaMemcpyDeviceToHost, ctx->stream));
    PropStatus ps{};
    CK(cudaMemcpyAsync(&ps, ctx->pstat, sizeof(ps), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ps.nbad) {
        char msg[256];
        snprintf(msg, sizeof msg, "%u of %lld points outside the property table; first at index %llu (DH = %.17g)",
                 ps.nbad, (long long)npts, ps.first_bad, dh[ps.first_bad]);
        return fail(ctx, CHAPSIM_ERR_TABLE_RANGE, msg);
    }
    return CHAPSIM_OK;
}

// First properties of the thermal solver: THERM_PROP_UPDATE on the interior and
// the wall ghosts, DENSITY0 = DENSITY, Viscousity0 = Viscousity, G0_io = G_io,
// DENSITY_Staggered, MU_Staggered and VELOCITY_CALC_io
template <typename F>
void thermal_start(chapsim_ctx* ctx, size_t fb) {
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    IoFieldsT<F> f = io_fields_t<F>(ctx);
    const size_t sm = prop_smem(ctx->tab.n);
    const long long tot = (long long)g.L * g.M * g.N, plane = 2LL * g.L * g.N;
    if (sm) k_eng_props<true, F><<<prop_grid(ctx, tot), PROP_NT, sm, s>>>(ctx->tab, g, f, ctx->tf, ctx->st);
    else k_eng_props<false, F><<<prop_grid(ctx, tot), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->st);
    if constexpr (sizeof(F) == 8) {
        if (ctx->domain == 3) {  // the inlet and outlet columns from their rho*h
            k_xio_ghost_props<<<prop_grid(ctx, 2LL * g.M * g.N), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->st);
            cudaMemsetAsync(ctx->xio_bc0e, 0, (size_t)g.M * g.N * sizeof(double), s);
            ctx->launches += 1;
        }
    }
    if (sm) k_eng_bc<true, F><<<prop_grid(ctx, plane), PROP_NT, sm, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    else k_eng_bc<false, F><<<prop_grid(ctx, plane), PROP_NT, 0, s>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    cudaMemcpyAsync(ctx->io.RHO, ctx->DEN, fb, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(ctx->io.MU0, ctx->io.MU, fb, cudaMemcpyDeviceToDevice, s);
    if constexpr (sizeof(F) == 8) cudaMemcpyAsync(ctx->tf.G0, f.G, 3 * fb, cudaMemcpyDeviceToDevice, s);
    else k_convert<double, float><<<4 * ctx->nsm, DG_NT, 0, s>>>(ctx->tf.G0, f.G, 3 * g.FS);
    k_io_props<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f);
    k_io_velocity<F><<<ctx->io_grid, IO_NT, 0, s>>>(g, f);
    ctx->launches += 5;
}

// BC_WALL_THERMAL on its own (the wall rows of every column): after a change of the wall condition
template <typename F>
void thermal_walls(chapsim_ctx* ctx) {
    const Geo& g = ctx->g;
    IoFieldsT<F> f = io_fields_t<F>(ctx);
    const size_t sm = prop_smem(ctx->tab.n);
    const long long plane = 2LL * g.L * g.N;
    if (sm) k_eng_bc<true, F><<<prop_grid(ctx, plane), PROP_NT, sm, ctx->stream>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    else k_eng_bc<false, F><<<prop_grid(ctx, plane), PROP_NT, 0, ctx->stream>>>(ctx->tab, g, f, ctx->tf, ctx->tp, ctx->st);
    ctx->launches += 1;
}

extern "C" int chapsim_thermal_set_isothermal(chapsim_ctx_t* ctx, int32_t wall, const double* state5) {
    if (!ctx) return fail(nullptr, CHAPSIM_ERR_BADARG, "null context");
    if (!ctx->thermal) return fail(ctx, CHAPSIM_ERR_BADARG, "the thermal solver is not initialised (chapsim_thermal_init)");
    if (wall < 0 || wall > 1) return fail(ctx, CHAPSIM_ERR_BADARG, "wall must be 0 (bottom) or 1 (top)");
    if (state5)
        for (int a = 0; a < 5; ++a)
            if (!std::isfinite(state5[a])) return fail(ctx, CHAPSIM_ERR_BADARG, "non-finite wall state");
    CK(cudaSetDevice(ctx->device));
    ctx->tp.iso[wall] = state5 != nullptr;
    if (state5)
        for (int a = 0; a < 5; ++a) ctx->tp.wv[wall][a] = state5[a];
    if (io_mixed(ctx)) thermal_walls<float>(ctx);
    else thermal_walls<double>(ctx);
    CK(cudaGetLastError());
    if (int rc = check_device_error(ctx)) return rc;
    return drop_step_graph(ctx);
}

extern "C" int chapsim_thermal_init(chapsim_ctx_t* ctx, const double* dh, double qw_bot, double qw_top, double cthecd) {
    if (!ctx || !dh) return fail(ctx, CHAPSIM_ERR_BADARG, "null argument");
    if (ctx->domain < 2) return fail(ctx, CHAPSIM_ERR_BADARG, "the thermal solver runs in the main (IO) domain");
    if (!ctx->ptab) return fail(ctx, CHAPSIM_ERR_BADARG, "no property table (call chapsim_prop_table_init first)");
    if (!(cthecd > 0.0)) return fail(ctx, CHAPSIM_ERR_BADARG, "CTHECD must be positive");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    const size_t fb = (size_t)g.FS * sizeof(double);
    if (!ctx->thermal) {
        double** arrs[] = {&ctx->DEN, &ctx->tf.DH, &ctx->tf.ENTH, &ctx->tf.TEMP, &ctx->tf.KAP, &ctx->tf.HCP,
                           &ctx->tf.RHSE0, &ctx->tf.DRHO};
        for (double** a : arrs) {
            CK(cudaMalloc(a, fb));
            CK(cudaMemsetAsync(*a, 0, fb, s));
        }
        CK(cudaMalloc(&ctx->tf.G0, 3 * fb));
    }
    ctx->tp.wf_bot = qw_bot;
    ctx->tp.wf_top = -qw_top;
    ctx->tp.cthecd = cthecd;
    double lim[2];
    CK(cudaMemcpy(&lim[0], ctx->tab.xdh + ctx->tab.imin_dh, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&lim[1], ctx->tab.xdh + ctx->tab.imax_dh, sizeof(double), cudaMemcpyDeviceToHost));
    ctx->tp.dhmin = lim[0];
    ctx->tp.dhmax = lim[1];
    CK(cudaMemcpyAsync(ctx->tf.DH, dh, fb, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->tf.RHSE0, 0, fb, s));  // RHS_ENERGY0 = 0 (src/SOLVE.f90:40)
    CK(cudaMemcpyAsync(ctx->DEN, ctx->io.RHO, fb, cudaMemcpyDeviceToDevice, s));
    ctx->thermal = true;
    if (io_mixed(ctx)) thermal_start<float>(ctx, fb);
    else thermal_start<double>(ctx, fb);
    CK(cudaGetLastError());
    if (ctx->step_exec) {  // the captured step no longer matches
        CK(cudaStreamSynchronize(s));
        cudaGraphExecDestroy(ctx->step_exec);
        ctx->step_exec = nullptr;
    }
    return check_device_error(ctx);
}

extern "C" int chapsim_download_thermal_fields(chapsim_ctx_t* ctx, double* dh, double* h, double* t, double* d,
                                               double* m, double* k, double* cp) {
    if (!ctx || !ctx->thermal) return fail(ctx, CHAPSIM_ERR_BADARG, "the thermal solver is not active on this context");
    CK(cudaSetDevice(ctx->device));
    const size_t fb = (size_t)ctx->g.FS * sizeof(double);
    double* dst[7] = {dh, h, t, d, m, k, cp};
    const double* src[7] = {ctx->tf.DH, ctx->tf.ENTH, ctx->tf.TEMP, ctx->DEN, ctx->io.MU, ctx->tf.KAP, ctx->tf.HCP};
    for (int a = 0; a < 7; ++a)
        if (dst[a]) CK(cudaMemcpyAsync(dst[a], src[a], fb, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

// ------------------------- learned property model -------------------------
namespace {
int mlp_targets(chapsim_ctx* ctx, int n, const double* dh_host, const MlpNorm& nm) {
    CK(cudaSetDevice(ctx->device));
    if (n > ctx->mlp_cap) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->mlp_xs); cudaFree(ctx->mlp_ys); cudaFree(ctx->mlp_dh);
        ctx->mlp_xs = nullptr; ctx->mlp_ys = nullptr; ctx->mlp_dh = nullptr; ctx->mlp_cap = 0;
        CK(cudaMalloc(&ctx->mlp_xs, (size_t)n * sizeof(float)));
        CK(cudaMalloc(&ctx->mlp_ys, (size_t)n * MLP_OUT * sizeof(float)));
        CK(cudaMalloc(&ctx->mlp_dh, (size_t)n * sizeof(double)));
        ctx->mlp_cap = n;
    }
    CK(cudaMemcpyAsync(ctx->mlp_dh, dh_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (int rc = prop_reset_status(ctx)) return rc;
    k_mlp_targets<<<prop_grid(ctx, n), PROP_NT, 0, ctx->stream>>>(ctx->tab, nm, n, ctx->mlp_dh, ctx->mlp_xs, ctx->mlp_ys,
                                                                  ctx->pstat);
    ctx->launches += 1;
    CK(cudaGetLastError());
    PropStatus ps{};
    CK(cudaMemcpyAsync(&ps, ctx->pstat, sizeof(ps), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ps.nbad) return fail(ctx, CHAPSIM_ERR_TABLE_RANGE, "training sample outside the property table");
    return CHAPSIM_OK;
}

int mlp_pack(chapsim_ctx* ctx) {
    k_mlp_adam<<<1, 256, 0, ctx->stream>>>(ctx->mlp_par, ctx->mlp_grad, ctx->mlp_m1, ctx->mlp_m2, 0, 0.f, ctx->mlp_w2,
                                           ctx->mlp_w3, ctx->mlp_w2t, ctx->mlp_w2h, ctx->mlp_w3h);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return CHAPSIM_OK;
}

int mlp_check_err(chapsim_ctx* ctx) {
    CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->st_host->err & CHS_EBIT_MMA_TIMEOUT) {
        unsigned int zero = 0;
        CK(cudaMemcpy(&ctx->st->err, &zero, sizeof(zero), cudaMemcpyHostToDevice));
        return fail(ctx, CHAPSIM_ERR_TIMEOUT, "a tensor-core completion wait ran out of time");
    }
    return CHAPSIM_OK;
}

// one pass of k_mlp_train over the current training set; gradients summed into mlp_grad
int mlp_pass(chapsim_ctx* ctx, int n) {
    const int tiles = (n + MLP_TILE - 1) / MLP_TILE;
    const float inv = 1.0f / ((float)n * MLP_OUT);
    if (ctx->mlp_act == MLP_ACT_CUBIC)
        k_mlp_train<MLP_ACT_CUBIC><<<tiles, MLP_NT, MLP_TRN_SMEM, ctx->stream>>>(
            ctx->mlp_par, mlp_ops(ctx), ctx->mlp_xs, ctx->mlp_ys, n, inv, ctx->mlp_grad, ctx->mlp_loss, &ctx->st->err);
    else
        k_mlp_train<MLP_ACT_TANH><<<tiles, MLP_NT, MLP_TRN_SMEM, ctx->stream>>>(
            ctx->mlp_par, mlp_ops(ctx), ctx->mlp_xs, ctx->mlp_ys, n, inv, ctx->mlp_grad, ctx->mlp_loss, &ctx->st->err);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return CHAPSIM_OK;
}
}  // namespace

extern "C" int chapsim_mlp_init(chapsim_ctx_t* ctx, double dh_lo, double dh_hi, uint64_t seed) {
    if (!ctx) return fail(nullptr, CHAPSIM_ERR_BADARG, "null context");
    if (!ctx->ptab) return fail(ctx, CHAPSIM_ERR_BADARG, "no property table (call chapsim_prop_table_init first)");
    if (!(dh_hi > dh_lo)) return fail(ctx, CHAPSIM_ERR_BADARG, "empty trained rho*h range");
    CK(cudaSetDevice(ctx->device));
    if (!ctx->mlp_par) {
        CK(cudaMalloc(&ctx->mlp_par, 4 * MLP_NPARAM * sizeof(float) + sizeof(float)));
        ctx->mlp_grad = ctx->mlp_par + MLP_NPARAM;
        ctx->mlp_m1 = ctx->mlp_grad + MLP_NPARAM;
        ctx->mlp_m2 = ctx->mlp_m1 + MLP_NPARAM;
        ctx->mlp_loss = ctx->mlp_m2 + MLP_NPARAM;
        CK(cudaMalloc(&ctx->mlp_w2, 2 * (64 * 64 * 2 + 16 * 64) * sizeof(__nv_bfloat16)));
        ctx->mlp_w2t = ctx->mlp_w2 + 64 * 64;
        ctx->mlp_w3 = ctx->mlp_w2t + 64 * 64;
        ctx->mlp_w2h = reinterpret_cast<__half*>(ctx->mlp_w3 + 16 * 64);
        ctx->mlp_w3h = ctx->mlp_w2h + 64 * 64;
        CK(cudaFuncSetAttribute(k_mlp_train<MLP_ACT_TANH>, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_TRN_SMEM));
        CK(cudaFuncSetAttribute(k_mlp_train<MLP_ACT_CUBIC>, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_TRN_SMEM));
        CK(cudaFuncSetAttribute(k_mlp_infer<false, MLP_ACT_TANH>, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_INF_SMEM));
        CK(cudaFuncSetAttribute(k_mlp_infer<true, MLP_ACT_TANH>, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_INF_SMEM));
        CK(cudaFuncSetAttribute(k_mlp_infer<false, MLP_ACT_CUBIC>, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_INF_SMEM));
        CK(cudaFuncSetAttribute(k_mlp_infer<true, MLP_ACT_CUBIC>, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_INF_SMEM));
    }
    // output scaling from the table over the trained range
    const int ns = 4097;
    std::vector<double> dh(ns);
    for (int q = 0; q < ns; ++q) dh[q] = dh_lo + (dh_hi - dh_lo) * (double)q / (double)(ns - 1);
    MlpNorm raw{};
    raw.x_lo = (float)dh_lo;
    raw.x_hi = (float)dh_hi;
    for (int k = 0; k < MLP_OUT; ++k) { raw.off[k] = 0.f; raw.scale[k] = 1.f; }
    if (int rc = mlp_targets(ctx, ns, dh.data(), raw)) return rc;
    std::vector<float> ys((size_t)ns * MLP_OUT);
    CK(cudaMemcpy(ys.data(), ctx->mlp_ys, ys.size() * sizeof(float), cudaMemcpyDeviceToHost));
    MlpNorm nm = raw;
    for (int k = 0; k < MLP_OUT; ++k) {
        float lo = ys[k], hi = ys[k];
        for (int q = 1; q < ns; ++q) { lo = fminf(lo, ys[(size_t)q * MLP_OUT + k]); hi = fmaxf(hi, ys[(size_t)q * MLP_OUT + k]); }
        nm.off[k] = 0.5f * (lo + hi);
        nm.scale[k] = fmaxf(0.5f * (hi - lo), 1e-6f);
    }
    ctx->mlp_norm = nm;
    // Glorot-uniform weights from a SplitMix64 stream, zero biases
    std::vector<float> p(MLP_NPARAM, 0.f);
    uint64_t st = seed;
    auto next = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    const double a1 = std::sqrt(6.0 / (1 + MLP_H)), a2 = std::sqrt(6.0 / (2 * MLP_H)), a3 = std::sqrt(6.0 / (MLP_H + MLP_OUT));
    for (int q = 0; q < MLP_H; ++q) p[MLP_W1 + q] = (float)(a1 * (2 * next() - 1) * 3.0);
    for (int q = 0; q < MLP_H; ++q) p[MLP_B1 + q] = (float)((2 * next() - 1) * 2.0);
    for (int q = 0; q < MLP_H * MLP_H; ++q) p[MLP_W2 + q] = (float)(a2 * (2 * next() - 1));
    for (int q = 0; q < MLP_OUT * MLP_H; ++q) p[MLP_W3 + q] = (float)(a3 * (2 * next() - 1));
    CK(cudaMemcpy(ctx->mlp_par, p.data(), MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemset(ctx->mlp_grad, 0, (3 * MLP_NPARAM + 1) * sizeof(float)));
    CK(cudaMemset(ctx->mlp_w2, 0, (64 * 64 * 2 + 16 * 64) * sizeof(__nv_bfloat16)));
    ctx->mlp_step = 0;
    if (int rc = mlp_pack(ctx)) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->mlp_ready = true;
    return CHAPSIM_OK;
}

extern "C" int chapsim_mlp_set_activation(chapsim_ctx_t* ctx, int32_t act) {
    if (!ctx) return fail(nullptr, CHAPSIM_ERR_BADARG, "null context");
    if (act != CHAPSIM_MLP_TANH && act != CHAPSIM_MLP_CUBIC)
        return fail(ctx, CHAPSIM_ERR_BADARG, "activation must be CHAPSIM_MLP_TANH or CHAPSIM_MLP_CUBIC");
    ctx->mlp_act = act;
    return drop_step_graph(ctx);
}

extern "C" int chapsim_mlp_set_params(chapsim_ctx_t* ctx, const float* params) {
    if (!ctx || !params || !ctx->mlp_ready) return fail(ctx, CHAPSIM_ERR_BADARG, "MLP not initialised");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpy(ctx->mlp_par, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    if (int rc = mlp_pack(ctx)) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return CHAPSIM_OK;
}

extern "C" int chapsim_mlp_get_params(chapsim_ctx_t* ctx, float* params, double* norm) {
    if (!ctx || !ctx->mlp_ready) return fail(ctx, CHAPSIM_ERR_BADARG, "MLP not initialised");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    if (params) CK(cudaMemcpy(params, ctx->mlp_par, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    if (norm) {
        const MlpNorm& nm = ctx->mlp_norm;
        norm[0] = nm.x_lo; norm[1] = nm.x_hi;
        for (int k = 0; k < MLP_OUT; ++k) { norm[2 + k] = nm.off[k]; norm[2 + MLP_OUT + k] = nm.scale[k]; }
    }
    return CHAPSIM_OK;
}

extern "C" int chapsim_mlp_gradients(chapsim_ctx_t* ctx, int32_t n, const double* dh, float* grad, double* loss) {
    if (!ctx || !ctx->mlp_ready || n <= 0 || !dh || !grad) return fail(ctx, CHAPSIM_ERR_BADARG, "bad MLP gradient arguments");
    if (int rc = mlp_targets(ctx, n, dh, ctx->mlp_norm)) return rc;
    CK(cudaMemsetAsync(ctx->mlp_grad, 0, MLP_NPARAM * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->mlp_loss, 0, sizeof(float), ctx->stream));
    if (int rc = mlp_pass(ctx, n)) return rc;
    float l = 0.f;
    CK(cudaMemcpyAsync(grad, ctx->mlp_grad, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&l, ctx->mlp_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemsetAsync(ctx->mlp_grad, 0, MLP_NPARAM * sizeof(float), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (loss) *loss = l;
    return mlp_check_err(ctx);
}

extern "C" int chapsim_mlp_train(chapsim_ctx_t* ctx, int32_t n, const double* dh, int32_t iters, float lr,
                                 double* final_loss) {
    if (!ctx || !ctx->mlp_ready || n <= 0 || !dh || iters < 1 || !(lr > 0.f))
        return fail(ctx, CHAPSIM_ERR_BADARG, "bad MLP training arguments");
    if (int rc = mlp_targets(ctx, n, dh, ctx->mlp_norm)) return rc;
    CK(cudaMemsetAsync(ctx->mlp_grad, 0, MLP_NPARAM * sizeof(float), ctx->stream));
    for (int it = 0; it < iters; ++it) {
        if (it == iters - 1) CK(cudaMemsetAsync(ctx->mlp_loss, 0, sizeof(float), ctx->stream));
        if (int rc = mlp_pass(ctx, n)) return rc;
        ++ctx->mlp_step;
        k_mlp_adam<<<1, 256, 0, ctx->stream>>>(ctx->mlp_par, ctx->mlp_grad, ctx->mlp_m1, ctx->mlp_m2, ctx->mlp_step, lr,
                                               ctx->mlp_w2, ctx->mlp_w3, ctx->mlp_w2t, ctx->mlp_w2h, ctx->mlp_w3h);
        ctx->launches += 1;
    }
    CK(cudaGetLastError());
    float l = 0.f;
    CK(cudaMemcpyAsync(&l, ctx->mlp_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (final_loss) *final_loss = l;
    return mlp_check_err(ctx);
}

extern "C" int chapsim_mlp_infer_points(chapsim_ctx_t* ctx, int64_t npts, const double* dh, double* h, double* t,
                                        double* d, double* m, double* k, double* cp) {
    if (!ctx || !ctx->mlp_ready) return fail(ctx, CHAPSIM_ERR_BADARG, "MLP not initialised");
    if (npts <= 0 || !dh || !h || !t || !d || !m || !k || !cp) return fail(ctx, CHAPSIM_ERR_BADARG, "bad point arrays");
    CK(cudaSetDevice(ctx->device));
    if (npts > ctx->pbuf_pts) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->pbuf);
        ctx->pbuf = nullptr;
        ctx->pbuf_pts = 0;
        CK(cudaMalloc(&ctx->pbuf, (size_t)7 * npts * sizeof(double)));
        ctx->pbuf_pts = npts;
    }
    double* dd = ctx->pbuf;
    double* o = dd + npts;
    const size_t b = (size_t)npts * sizeof(double);
    CK(cudaMemcpyAsync(dd, dh, b, cudaMemcpyHostToDevice, ctx->stream));
    if (int rc = prop_reset_status(ctx)) return rc;
    const long long tiles = (npts + MLP_TILE - 1) / MLP_TILE;
    const int grid = (int)std::min<long long>(tiles, 4LL * ctx->nsm);
    MlpOut out{o, o + npts, o + 2 * npts, o + 3 * npts, o + 4 * npts, o + 5 * npts, nullptr, nullptr};
    if (ctx->mlp_act == MLP_ACT_CUBIC)
        k_mlp_infer<false, MLP_ACT_CUBIC><<<grid, MLP_NT, MLP_INF_SMEM, ctx->stream>>>(
            ctx->mlp_par, mlp_ops(ctx), ctx->mlp_norm, ctx->tab, ctx->g, npts, dd, out, ctx->pstat, &ctx->st->err);
    else
        k_mlp_infer<false, MLP_ACT_TANH><<<grid, MLP_NT, MLP_INF_SMEM, ctx->stream>>>(
            ctx->mlp_par, mlp_ops(ctx), ctx->mlp_norm, ctx->tab, ctx->g, npts, dd, out, ctx->pstat, &ctx->st->err);
    ctx->launches += 1;
    CK(cudaGetLastError());
    double* outs[6] = {h, t, d, m, k, cp};
    for (int s = 0; s < 6; ++s) CK(cudaMemcpyAsync(outs[s], o + (size_t)s * npts, b, cudaMemcpyDeviceToHost, ctx->stream));
    PropStatus ps{};
    CK(cudaMemcpyAsync(&ps, ctx->pstat, sizeof(ps), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (int rc = mlp_check_err(ctx)) return rc;
    if (ps.nbad) {
        char msg[160];
        snprintf(msg, sizeof msg, "%u of %lld points outside the property table; first at index %llu", ps.nbad,
                 (long long)npts, ps.first_bad);
        return fail(ctx, CHAPSIM_ERR_TABLE_RANGE, msg);
    }
    return CHAPSIM_OK;
}

extern "C" int chapsim_thermal_use_mlp(chapsim_ctx_t* ctx, int32_t enable) {
    if (!ctx || !ctx->thermal) return fail(ctx, CHAPSIM_ERR_BADARG, "the thermal solver is not active on this context");
    if (enable && !ctx->mlp_ready) return fail(ctx, CHAPSIM_ERR_BADARG, "MLP not initialised");
    if (enable && ctx->domain == 3)
        return fail(ctx, CHAPSIM_ERR_BADARG, "the inflow/outflow main domain updates its properties by table search");
    CK(cudaSetDevice(ctx->device));
    ctx->use_mlp = enable != 0;
    if (ctx->step_exec) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaGraphExecDestroy(ctx->step_exec);
        ctx->step_exec = nullptr;
    }
    return CHAPSIM_OK;
}

extern "C" int chapsim_mlp_judge(chapsim_ctx_t* ctx, double* max_rel_err) {
    if (!ctx || !ctx->thermal || !ctx->mlp_ready || !max_rel_err)
        return fail(ctx, CHAPSIM_ERR_BADARG, "the judge needs an active thermal solver and an initialised MLP");
    CK(cudaSetDevice(ctx->device));
    unsigned int* eb = reinterpret_cast<unsigned int*>(ctx->pstat);  // 6 words of scratch after the status
    if (!ctx->mlp_judge) CK(cudaMalloc(&ctx->mlp_judge, 8 * sizeof(unsigned int)));
    eb = ctx->mlp_judge;
    CK(cudaMemsetAsync(eb, 0, 8 * sizeof(unsigned int), ctx->stream));
    MlpOut cur{ctx->tf.ENTH, ctx->tf.TEMP, ctx->DEN, ctx->io.MU, ctx->tf.KAP, ctx->tf.HCP, nullptr, nullptr};
    const long long tot = (long long)ctx->g.L * ctx->g.M * ctx->g.N;
    k_mlp_judge<<<prop_grid(ctx, tot), PROP_NT, 0, ctx->stream>>>(ctx->tab, ctx->mlp_norm, ctx->g, ctx->tf.DH, cur, eb);
    ctx->launches += 1;
    CK(cudaGetLastError());
    unsigned int hb[8];
    CK(cudaMemcpyAsync(hb, eb, sizeof(hb), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int m = 0; m < MLP_OUT; ++m) {
        float f;
        memcpy(&f, &hb[m], sizeof(f));
        max_rel_err[m] = f;
    }
    return CHAPSIM_OK;
}

// ----------------------------- autotuner -----------------------------------
// Times the Poisson y-solve variants (warp Thomas/PCR hybrid, sequential
// Thomas, two-way, sequential at one block per SM, warp scans) on this
// context's grid and keeps the fastest.  The spectral array is scratch
// between substeps, so it is zeroed and solved in place.
extern "C" int chapsim_autotune(chapsim_ctx_t* ctx, int32_t force, int32_t* choice, float* ms) {
    if (!ctx) return fail(nullptr, CHAPSIM_ERR_BADARG, "null context");
    if (ctx->domain == 3) return fail(ctx, CHAPSIM_ERR_BADARG, "the inflow/outflow main domain has no tuned variants");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    cudaStream_t s = ctx->stream;
    CK(cudaStreamSynchronize(s));
    const size_t nsp = (size_t)g.LH * g.M * g.N;
    if (!ctx->YF) {
        CK(cudaMalloc(&ctx->YF, 2 * nsp * sizeof(double)));
        k_ysolve_seq_factors<<<4 * ctx->nsm, 128, 0, s>>>(g, ctx->YF);
        CK(cudaGetLastError());
    }
    if (!ctx->YF2) {
        CK(cudaMalloc(&ctx->YF2, 2 * nsp * sizeof(double)));
        k_ysolve_2w_factors<<<4 * ctx->nsm, 128, 0, s>>>(g, ctx->YF2);
        CK(cudaGetLastError());
    }
    if (!ctx->YF3) {
        CK(cudaMalloc(&ctx->YF3, nsp * sizeof(double)));
        k_ysolve_scan_factors<<<4 * ctx->nsm, 128, 0, s>>>(g, ctx->YF3);
        CK(cudaGetLastError());
    }
    // the variants are timed on the spectral array the time step uses (FP32 in the mixed-precision step)
    const bool spf = ctx->SPf != nullptr;
    if (spf) CK(cudaMemsetAsync(ctx->SPf, 0, nsp * sizeof(float2), s));
    else CK(cudaMemsetAsync(ctx->SP, 0, nsp * sizeof(double2), s));
    auto run_y = [&](int kind) {
        if (spf) {
            if (kind == 0) launch_ysolve_warp<float2>(ctx);
            else if (kind == 1) launch_ysolve_seq<float2>(ctx, false);
            else if (kind == 3) launch_ysolve_seq<float2>(ctx, true);
            else if (kind == 4) launch_ysolve_scan<float2>(ctx);
            else launch_ysolve_2w<float2>(ctx);
        } else {
            if (kind == 0) launch_ysolve_warp<double2>(ctx);
            else if (kind == 1) launch_ysolve_seq<double2>(ctx, false);
            else if (kind == 3) launch_ysolve_seq<double2>(ctx, true);
            else if (kind == 4) launch_ysolve_scan<double2>(ctx);
            else launch_ysolve_2w<double2>(ctx);
        }
    };
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const bool kg1 = ysolve_seq_kg1(g);
    float t[5] = {0.f, 0.f, 0.f, 1e30f, 0.f};
    const int reps = 5;
    for (int kind = 0; kind < 5; ++kind) {
        if (kind == 3 && !kg1) continue;
        for (int w = 0; w < 2; ++w) run_y(kind);
        CK(cudaEventRecord(e0, s));
        for (int r = 0; r < reps; ++r) run_y(kind);
        CK(cudaEventRecord(e1, s));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&t[kind], e0, e1));
        t[kind] /= reps;
    }
    ctx->launches += (kg1 ? 5 : 4) * (2 + reps);
    CK(cudaGetLastError());
    if (force >= 0) {
        ctx->ysolve_kind =
            (force & 1) ? 1 : ((force & 16) ? 2 : ((force & 32) ? (kg1 ? 3 : 1) : ((force & 64) ? 4 : 0)));
    } else {
        int best = 0;
        for (int kind = 1; kind < 5; ++kind)
            if (t[kind] < t[best]) best = kind;
        ctx->ysolve_kind = best;
    }
    CK(cudaStreamSynchronize(s));
    if (ctx->ysolve_kind != 1 && ctx->ysolve_kind != 3) {  // each factor table is read by its own variant only
        cudaFree(ctx->YF);
        ctx->YF = nullptr;
    }
    if (ctx->ysolve_kind != 2) {
        cudaFree(ctx->YF2);
        ctx->YF2 = nullptr;
    }
    if (ctx->ysolve_kind != 4) {
        cudaFree(ctx->YF3);
        ctx->YF3 = nullptr;
    }
    // explicit right-hand sides + x sweep: fused, split, or fused with bulk-copy
    // staging (periodic channel).  CONVH0 is state: kept in a temporary copy
    // and restored afterwards.
    float tk[4] = {0.f, 0.f, 0.f, 1e30f};
    if (ctx->domain == 1) {
        const bool mixed = ctx->prec == CHAPSIM_PREC_MIXED;
        const size_t hb = (size_t)3 * g.FI * (mixed ? sizeof(float) : sizeof(double));
        void* hsave = nullptr;
        CK(cudaMalloc(&hsave, hb));
        void* h0 = mixed ? (void*)ctx->H0f : (void*)ctx->H0;
        CK(cudaMemcpyAsync(hsave, h0, hb, cudaMemcpyDeviceToDevice, s));
        const int keep = ctx->k1_kind;
        const bool bulk_fits = ctx->rb_nw > 0;
        const bool pair_ok = (g.L / 32) % (mixed ? 4 : 2) == 0;  // kind 3: the wide form
        for (int kind = 0; kind < 4; ++kind) {
            if ((kind == 2 && !bulk_fits) || (kind == 3 && !pair_ok)) {
                tk[kind] = 1e30f;
                continue;
            }
            ctx->k1_kind = kind;
            auto one = [&]() {
                if (mixed) {
                    StepFields<float> f = step_fields<float>(ctx);
                    launch_rhs_x<float>(ctx, f, f.fac + 5 * FAC_SET, 1);
                } else {
                    StepFields<double> f = step_fields<double>(ctx);
                    launch_rhs_x<double>(ctx, f, f.fac + 5 * FAC_SET, 1);
                }
            };
            one();
            CK(cudaEventRecord(e0, s));
            for (int r = 0; r < reps; ++r) one();
            CK(cudaEventRecord(e1, s));
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&tk[kind], e0, e1));
            tk[kind] /= reps;
        }
        ctx->k1_kind = keep;
        CK(cudaMemcpyAsync(h0, hsave, hb, cudaMemcpyDeviceToDevice, s));
        CK(cudaStreamSynchronize(s));
        cudaFree(hsave);
        CK(cudaGetLastError());
        int best = 0;
        for (int kind = 1; kind < 4; ++kind)
            if (tk[kind] < tk[best]) best = kind;
        int fk = (force >> 1) & 3;
        if (fk == 2 && !bulk_fits) fk = 1;
        if (fk == 3 && !pair_ok) fk = 0;
        ctx->k1_kind = force >= 0 ? fk : best;
    }
    // tile shape of the z sweep: 32 or 16 lines per tile, line-contiguous or pair-interleaved
    // (v = tile16 + 2 interleaved; it rewrites RHS in place, which every substep's
    // right-hand-side kernel rewrites before reading)
    float tz[4] = {0.f, 0.f, 0.f, 0.f};
    if (ctx->domain == 1) {
        const bool mixed = ctx->prec == CHAPSIM_PREC_MIXED;
        for (int v = 0; v < 4; ++v) {
            ctx->zs_tw = (v & 1) ? 16 : 32;
            ctx->zs_il = (v & 2) ? 2 : 1;
            auto one = [&]() {
                if (mixed) {
                    StepFields<float> f = step_fields<float>(ctx);
                    launch_zsweep<float>(ctx, f, f.fac + 5 * FAC_SET);
                } else {
                    StepFields<double> f = step_fields<double>(ctx);
                    launch_zsweep<double>(ctx, f, f.fac + 5 * FAC_SET);
                }
            };
            one();
            CK(cudaEventRecord(e0, s));
            for (int r = 0; r < reps; ++r) one();
            CK(cudaEventRecord(e1, s));
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&tz[v], e0, e1));
            tz[v] /= reps;
        }
        ctx->launches += 4 * (1 + reps);
        CK(cudaGetLastError());
        int bz = 0;
        for (int v = 1; v < 4; ++v)
            if (tz[v] < tz[bz]) bz = v;
        if (force >= 0) bz = ((force & 256) ? 1 : 0) | ((force & 1024) ? 2 : 0);
        ctx->zs_tw = (bz & 1) ? 16 : 32;
        ctx->zs_il = (bz & 2) ? 2 : 1;
    }
    // tile layout of the y sweep; it adds the increments to Q, which is state: Q is kept in a
    // temporary copy and restored afterwards
    float ty[2] = {0.f, 0.f};
    if (ctx->domain == 1) {
        const bool mixed = ctx->prec == CHAPSIM_PREC_MIXED;
        const size_t qb = (size_t)3 * g.FS * (mixed ? sizeof(float) : sizeof(double));
        void* qsave = nullptr;
        CK(cudaMalloc(&qsave, qb));
        void* q0 = mixed ? (void*)ctx->Qf : (void*)ctx->Q;
        CK(cudaMemcpyAsync(qsave, q0, qb, cudaMemcpyDeviceToDevice, s));
        for (int v = 0; v < 2; ++v) {
            ctx->ys_il = v + 1;
            auto one = [&]() {
                if (mixed) {
                    StepFields<float> f = step_fields<float>(ctx);
                    launch_ysweep<float>(ctx, f, f.fac + 5 * FAC_SET, 1);
                } else {
                    StepFields<double> f = step_fields<double>(ctx);
                    launch_ysweep<double>(ctx, f, f.fac + 5 * FAC_SET, 1);
                }
            };
            one();
            CK(cudaEventRecord(e0, s));
            for (int r = 0; r < reps; ++r) one();
            CK(cudaEventRecord(e1, s));
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&ty[v], e0, e1));
            ty[v] /= reps;
        }
        ctx->launches += 2 * (1 + reps);
        CK(cudaMemcpyAsync(q0, qsave, qb, cudaMemcpyDeviceToDevice, s));
        CK(cudaStreamSynchronize(s));
        cudaFree(qsave);
        CK(cudaGetLastError());
        ctx->ys_il = force >= 0 ? ((force & 2048) ? 2 : 1) : (ty[1] < ty[0] ? 2 : 1);
    }
    // pressure stage up to DPH: chained x/z transforms or the fused plane
    // transforms (periodic channel, planes that fit one block).  It writes
    // only scratch (RHSLLPHI, the spectrum, DPH), which every substep rewrites.
    // (kind 0: chained transforms, 1: fused plane transforms, 2: chained with the persistent
    // double-buffered z transforms, 3: chained with the z transforms' wave-ahead L2 requests)
    float tp[4] = {0.f, 1e30f, 0.f, 0.f};
    if (ctx->domain == 1) {
        const bool mixed = ctx->prec == CHAPSIM_PREC_MIXED;
        bool p2 = (mixed ? plane_fft_ok<float2>(g) : plane_fft_ok<double2>(g)) || ctx->p2c;
        for (int kind = 0; kind < 4; ++kind) {
            if (kind == 1 && !p2) continue;
            ctx->plane_kind = kind == 1 ? 1 : 0;
            ctx->fz_pipe = kind == 2;
            ctx->fz_prefetch = kind == 3;
            auto one = [&]() {
                if (mixed) launch_pressure<float>(ctx, step_fields<float>(ctx), 1);
                else launch_pressure<double>(ctx, step_fields<double>(ctx), 1);
            };
            one();
            if (kind == 1 && ctx->p2c && cudaGetLastError() != cudaSuccess) {
                // the cluster launch was refused (configuration): keep the chained transforms
                ctx->p2c = false;
                p2 = false;
                tp[1] = 1e30f;
                continue;
            }
            CK(cudaEventRecord(e0, s));
            for (int r = 0; r < reps; ++r) one();
            CK(cudaEventRecord(e1, s));
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&tp[kind], e0, e1));
            tp[kind] /= reps;
        }
        CK(cudaGetLastError());
        if (force >= 0) {
            ctx->plane_kind = p2 ? (force >> 3) & 1 : 0;
            ctx->fz_pipe = (force & 512) != 0;
            ctx->fz_prefetch = (force & 4096) != 0;
        } else {
            int best = 0;
            for (int kind = 1; kind < 4; ++kind)
                if (tp[kind] < tp[best]) best = kind;
            ctx->plane_kind = best == 1 ? 1 : 0;
            ctx->fz_pipe = best == 2;
            ctx->fz_prefetch = best == 3;
        }
    }
    if (ctx->step_exec) {
        cudaGraphExecDestroy(ctx->step_exec);
        ctx->step_exec = nullptr;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (choice)
        *choice = (ctx->ysolve_kind == 1 ? 1 : 0) | (ctx->k1_kind << 1) | (ctx->plane_kind << 3) |
                  (ctx->ysolve_kind == 2 ? 16 : 0) | (ctx->ysolve_kind == 3 ? 32 : 0) | (ctx->ysolve_kind == 4 ? 64 : 0) |
                  (ctx->zs_tw == 16 ? 256 : 0) | (ctx->fz_pipe ? 512 : 0) | (ctx->zs_il == 2 ? 1024 : 0) |
                  (ctx->ys_il == 2 ? 2048 : 0) | (ctx->fz_prefetch ? 4096 : 0);
    if (ms) {
        ms[0] = t[0]; ms[1] = t[1]; ms[2] = tk[0]; ms[3] = tk[1]; ms[4] = tk[2];
        ms[5] = tp[0]; ms[6] = tp[1]; ms[7] = t[2]; ms[8] = t[3]; ms[9] = t[4];
        ms[10] = tz[0]; ms[11] = tz[1]; ms[12] = tp[2]; ms[13] = tk[3]; ms[14] = tz[2]; ms[15] = tz[3];
        ms[16] = ty[0]; ms[17] = ty[1]; ms[18] = tp[3];
    }
    return CHAPSIM_OK;
}

// ------------------------------ ensembles ----------------------------------
struct chapsim_batch {
    std::vector<chapsim_ctx*> ctx;
    int device = 0;
    cudaStream_t stream = nullptr;     // the ensemble's own stream: the graph forks from and joins to it
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t exec = nullptr;
    int kernels_per_step = 0;
    std::string err;
};

extern "C" int chapsim_batch_create(chapsim_ctx_t* const* ctxs, int32_t n, chapsim_batch_t** out) {
    if (!ctxs || n < 1 || !out) return fail(nullptr, CHAPSIM_ERR_BADARG, "bad ensemble arguments");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i]) return fail(nullptr, CHAPSIM_ERR_BADARG, "null context in ensemble");
        if (ctxs[i]->domain != 1 || ctxs[i]->device != ctxs[0]->device)
            return fail(nullptr, CHAPSIM_ERR_BADARG, "an ensemble holds periodic (TG) contexts of one device");
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) return fail(nullptr, CHAPSIM_ERR_BADARG, "a context appears twice in the ensemble");
    }
    auto* b = new chapsim_batch();
    b->ctx.assign(ctxs, ctxs + n);
    b->device = ctxs[0]->device;
    auto bail = [&](cudaError_t e, const char* what) {
        std::string m = std::string(what) + ": " + cudaGetErrorString(e);
        chapsim_batch_destroy(b);
        return fail(nullptr, CHAPSIM_ERR_CUDA, m);
    };
    cudaError_t e;
    if ((e = cudaSetDevice(b->device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
    b->join.resize(n, nullptr);
    for (int i = 0; i < n; ++i)
        if ((e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
    *out = b;
    return CHAPSIM_OK;
}

extern "C" int chapsim_batch_destroy(chapsim_batch_t* b) {
    if (!b) return CHAPSIM_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->fork) cudaEventDestroy(b->fork);
    for (cudaEvent_t ev : b->join)
        if (ev) cudaEventDestroy(ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return CHAPSIM_OK;
}

namespace {
// One RK3 step of every member, captured as one graph: the members' kernel
// chains are parallel branches forked from the ensemble stream.
int batch_capture(chapsim_batch_t* b) {
    chapsim_ctx* ctx = b->ctx[0];  // for CK's error reporting
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaEventRecord(b->fork, b->stream);
    int kernels = 0;
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        chapsim_ctx* c = b->ctx[i];
        cudaStreamWaitEvent(c->stream, b->fork, 0);
        const unsigned long long before = c->launches;
        launch_step_start(c);
        for (int ns = 1; ns <= 3; ++ns) launch_substep(c, ns, false);
        kernels += (int)(c->launches - before);
        c->launches = before;
        cudaEventRecord(b->join[i], c->stream);
        cudaStreamWaitEvent(b->stream, b->join[i], 0);
    }
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (e != cudaSuccess) return fail(ctx, CHAPSIM_ERR_CUDA, std::string("ensemble capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, CHAPSIM_ERR_CUDA, std::string("ensemble instantiate: ") + cudaGetErrorString(e));
    b->kernels_per_step = kernels;
    return CHAPSIM_OK;
}
}  // namespace

extern "C" int chapsim_batch_advance(chapsim_batch_t* b, int32_t nsteps, double dt0, double dtmin, double cflgv) {
    if (!b || nsteps < 0) return fail(nullptr, CHAPSIM_ERR_BADARG, "bad ensemble arguments");
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(nullptr, CHAPSIM_ERR_CUDA, "cudaSetDevice");
    for (chapsim_ctx* c : b->ctx) {
        int rc = set_step_params(c, dt0, dtmin, cflgv);
        if (rc) return fail(nullptr, rc, c->err);
    }
    if (!b->exec) {
        int rc = batch_capture(b);
        if (rc) return fail(nullptr, rc, b->ctx[0]->err);
    }
    for (int s = 0; s < nsteps; ++s) {
        cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
        if (e != cudaSuccess) return fail(nullptr, CHAPSIM_ERR_CUDA, std::string("ensemble launch: ") + cudaGetErrorString(e));
    }
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return fail(nullptr, CHAPSIM_ERR_CUDA, std::string("ensemble sync: ") + cudaGetErrorString(e));
    for (chapsim_ctx* c : b->ctx) {
        c->launches += (unsigned long long)nsteps * (unsigned long long)(b->kernels_per_step / (int)b->ctx.size());
        int rc = check_device_error(c);
        if (rc) return fail(nullptr, rc, c->err);
    }
    return CHAPSIM_OK;
}

extern "C" int chapsim_batch_get_stream(chapsim_batch_t* b, void** stream) {
    if (!b || !stream) return CHAPSIM_ERR_BADARG;
    *stream = (void*)b->stream;
    return CHAPSIM_OK;
}

// ------------- line solver on caller-owned device memory, no allocation -------------
// For callers that cannot let a library allocate device memory.  Examples: a host
// whose HBM is already reserved by its own caching allocator or OpenACC / CUDA Fortran
// data regions, where cudaMalloc may fail; or a time loop that must not stall, because
// cudaFree waits for the whole device.  The per-line elimination vectors of the
// sequential recurrence (k_tdma_seq) live in one fixed module-scope array instead.
//   words [0, 32)  : status block; word 0 counts lines whose solution is not finite
//   words [32, ...): 3*n doubles per line (the H, G1, G2 recurrences)
#include <mutex>

static_assert(CHAPSIM_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size must be a multiple of 256 bytes");
constexpr long long NOALLOC_STATUS_WORDS = 32;
constexpr long long NOALLOC_TOTAL_WORDS = CHAPSIM_NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_TOTAL_WORDS];

// one thread per line: counts lines with a non-finite entry
__global__ void k_count_nonfinite_lines(const double* r, int nlines, long long ls, long long es, int n,
                                        unsigned int* count) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const long long o = (long long)l * ls;
    bool bad = false;
    for (int i = 0; i < n; ++i) bad |= !isfinite(r[o + (long long)i * es]);
    if (bad) atomicAdd(count, 1u);
}

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Address of the scratch array on the current device, looked up once per device.
int noalloc_scratch(int dev, double** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(nullptr, CHAPSIM_ERR_CUDA,
                        std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CHAPSIM_OK;
}

// true when p is device (or managed) memory of device dev
bool on_device(const void* p, int dev) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == dev;
}
}  // namespace

extern "C" int chapsim_tdma_lines_noalloc(const double* a, const double* b, const double* c, double* r,
                                          const double* bcj, int32_t nlines, int64_t line_stride,
                                          int64_t elem_stride, int32_t n, int32_t cyclic, void* stream) {
    if (!a || !b || !c || !r || nlines <= 0 || n < 3 || line_stride < 1 || elem_stride < 1)
        return fail(nullptr, CHAPSIM_ERR_BADARG, "bad tridiagonal arguments (need nlines >= 1, n >= 3, strides >= 1)");
    if (cyclic && bcj) return fail(nullptr, CHAPSIM_ERR_BADARG, "cyclic systems take no Dirichlet values (bcj must be NULL)");
    const long long need = 3LL * n * nlines;
    const long long avail = NOALLOC_TOTAL_WORDS - NOALLOC_STATUS_WORDS;
    if (need > avail)
        return fail(nullptr, CHAPSIM_ERR_BADARG,
                    "chapsim_tdma_lines_noalloc: 3*n*nlines = " + std::to_string(need) +
                        " doubles of scratch exceeds the fixed limit of " + std::to_string(avail) +
                        " (CHAPSIM_NOALLOC_SCRATCH_BYTES); split the lines over several calls");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(nullptr, CHAPSIM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(nullptr, CHAPSIM_ERR_BADARG, "device ordinal out of range");
    for (const void* p : {(const void*)a, (const void*)b, (const void*)c, (const void*)r})
        if (!on_device(p, dev))
            return fail(nullptr, CHAPSIM_ERR_BADARG, "a, b, c and r must be device memory of the current device");
    if (bcj && !on_device(bcj, dev))
        return fail(nullptr, CHAPSIM_ERR_BADARG, "bcj must be device memory of the current device");
    double* scratch = nullptr;
    if (int rc = noalloc_scratch(dev, &scratch)) return rc;
    unsigned int* status = reinterpret_cast<unsigned int*>(scratch);
    double* wk = scratch + NOALLOC_STATUS_WORDS;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
#define NCK(call)                                                                                    \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return fail(nullptr, CHAPSIM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
    // the array keeps the previous call's contents: the counter must start at zero
    NCK(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    k_tdma_seq<<<(nlines + 127) / 128, 128, 0, s>>>(a, b, c, r, bcj, wk, nlines, line_stride, elem_stride, n,
                                                     cyclic ? 1 : 0);
    NCK(cudaGetLastError());
    k_count_nonfinite_lines<<<(nlines + 127) / 128, 128, 0, s>>>(r, nlines, line_stride, elem_stride, n, status);
    NCK(cudaGetLastError());
    unsigned int nbad = 0;
    NCK(cudaMemcpyAsync(&nbad, status, sizeof(nbad), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
#undef NCK
    if (nbad)
        return fail(nullptr, CHAPSIM_ERR_NAN, std::to_string(nbad) + " of " + std::to_string(nlines) +
                                                  " lines have a non-finite solution");
    return CHAPSIM_OK;
}

#include "field_dump.cuh"
