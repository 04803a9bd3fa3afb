// Learned property model: a 1 -> 64 -> 64 -> 6 MLP (tanh, or the clamped cubic
// below) from rho*h to the
// six outputs of THERM_PROP_UPDATE_FROM_DH (ENTHALPY, TEMPERATURE, DENSITY,
// Viscousity, THERMCONDT, HEATCAP), used in place of the table search inside
// its trained range; the table search stays the fallback outside it and the
// judge of its accuracy.
//
// Tensor cores: the 64 x 64 hidden layer and the output layer (6 outputs
// padded to N = 16) of 128-point tiles run as tcgen05.mma kind::f16 with
// 16-bit operands in shared memory and FP32 accumulators in tensor memory
// (TMEM), one elected thread issuing and committing to an mbarrier.  Training
// takes BF16 operands; inference takes FP16 ones (weights and activations),
// because its paired hardware tanh produces FP16 activations that go to the
// operand tile as they are.  Training uses the
// same forward pass and two more tcgen05 GEMMs for the backward pass
// (dL/dh1 = dz2 W2 and dL/dW2 = dz2^T h1); the rank-1 first layer, the small
// output-layer gradients and the optimiser run on the CUDA cores in FP32.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices; for an R x K operand the byte offset of
// element (r, k) is
//   ((((k/16)*2 + (k/8)%2) * (R/8) + r/8) * 8 + r%8) * 16 + (k%8) * 2,
// so the descriptor of K-slice s starts at s*R*32 bytes with the leading
// (K-direction) byte offset R*16 and the stride (8-row) byte offset 128.
//
// Every wait is bounded: an mbarrier wait that exceeds its clock budget sets
// an error bit and returns, and TMEM is always released before the kernel
// ends.
//
// Activations (template ACT): MLP_ACT_TANH, or MLP_ACT_CUBIC, the clamped cubic
//   c = clamp(z, -1, 1),  h = c (3 - c^2) / 2,  dh/dz = 3 (1 - c^2) / 2  (0 outside [-1, 1]),
// a C1 saturating activation that takes only min/max and multiply-adds: inference evaluates
// it on FP16 pairs on the FMA pipe, where tanh needs the special-function unit (one
// tanh.approx.f16x2 per pair) and bounds the kernel there.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "common.cuh"
#include "thermo.cuh"

#define MLP_H 64        // hidden width
#define MLP_OUT 6       // outputs: H, T, D, M, K, CP
#define MLP_NP 16       // output layer padded to the MMA N granule
#define MLP_TILE 128    // points per tile (MMA M)
#define MLP_NT 128      // threads per CTA (4 warps: one TMEM lane quarter each)
#ifndef CHS_EBIT_TABLE
#define CHS_EBIT_TABLE 4u
#endif

// parameter vector (FP32 master copy)
#define MLP_W1 0
#define MLP_B1 (MLP_W1 + MLP_H)
#define MLP_W2 (MLP_B1 + MLP_H)                 // [j][i], 64 x 64
#define MLP_B2 (MLP_W2 + MLP_H * MLP_H)
#define MLP_W3 (MLP_B2 + MLP_H)                 // [k][j], 6 x 64
#define MLP_B3 (MLP_W3 + MLP_OUT * MLP_H)
#define MLP_NPARAM (MLP_B3 + MLP_OUT)

struct MlpNorm {
    float x_lo, x_hi;           // trained rho*h range (inputs are mapped to [-1, 1])
    float off[MLP_OUT], scale[MLP_OUT];  // output k = off[k] + scale[k] * y[k]
};

// 16-bit operand images in the canonical layout, rebuilt by the optimiser:
// BF16 for training, FP16 for inference (A and B of one MMA always share the type)
struct MlpOperands {
    const __nv_bfloat16* w2;   // B of layer 2: rows j (64) x K i (64)
    const __nv_bfloat16* w3;   // B of layer 3: rows k (16, 6 used) x K j (64)
    const __nv_bfloat16* w2t;  // B of dL/dh1: rows i (64) x K j (64) = W2^T
    const __half* w2h;         // FP16 copies of w2 and w3 for inference
    const __half* w3h;
};

__host__ __device__ __forceinline__ int umma_off(int R, int r, int k) {
    return ((((k >> 4) * 2 + ((k >> 3) & 1)) * (R >> 3) + (r >> 3)) * 8 + (r & 7)) * 16 + (k & 7) * 2;
}


__device__ __forceinline__ uint64_t umma_desc(const void* base, int R, int s) {
    const uint32_t a = smem_u32(base) + (uint32_t)(s * R * 32);
    const uint64_t lbo = (uint64_t)(R * 16), sbo = 128;
    return (uint64_t)((a >> 4) & 0x3FFF) | (((lbo >> 4) & 0x3FFF) << 16) | (((sbo >> 4) & 0x3FFF) << 32) |
           (1ull << 46);
}

// kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, M x N
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// the same with FP16 A and B (formats 0)
__host__ __device__ constexpr uint32_t umma_idesc_f16(int M, int N) {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
}

__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __uint_as_float(r[c]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// The same load without its wait, into raw registers: several loads can be in flight, and
// their registers hold the data only after tmem_ld_wait().  tmem_tie16() after the wait
// passes the registers through an (empty) volatile asm, so no use of them can be
// scheduled above the wait: volatile asm statements keep their order, and every use
// depends on the tie's outputs.
__device__ __forceinline__ void tmem_ld16_raw(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_tie16(uint32_t* r) {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]));
}

// Row r of an R x 64 K-major operand from 64 floats (rounded to BF16), written
// as eight 16-byte chunks.
__device__ __forceinline__ void put_row64(unsigned char* base, int R, int r, const float* v) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        __nv_bfloat162 p0 = __floats2bfloat162_rn(v[8 * c + 0], v[8 * c + 1]);
        __nv_bfloat162 p1 = __floats2bfloat162_rn(v[8 * c + 2], v[8 * c + 3]);
        __nv_bfloat162 p2 = __floats2bfloat162_rn(v[8 * c + 4], v[8 * c + 5]);
        __nv_bfloat162 p3 = __floats2bfloat162_rn(v[8 * c + 6], v[8 * c + 7]);
        uint4 u;
        u.x = *reinterpret_cast<uint32_t*>(&p0);
        u.y = *reinterpret_cast<uint32_t*>(&p1);
        u.z = *reinterpret_cast<uint32_t*>(&p2);
        u.w = *reinterpret_cast<uint32_t*>(&p3);
        *reinterpret_cast<uint4*>(base + umma_off(R, r, 8 * c)) = u;
    }
}

__device__ __forceinline__ void copy_smem16(unsigned char* dst, const void* src, int bytes) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int q = threadIdx.x; q < bytes / 16; q += blockDim.x) d[q] = s[q];
}

__device__ __forceinline__ float mlp_x(const MlpNorm& nm, double dh) {
    return (float)(2.0 * (dh - (double)nm.x_lo) / ((double)nm.x_hi - (double)nm.x_lo) - 1.0);
}

// ---------------------------------------------------------------------------
// Inference.  Points mode: npts flat points, outputs at the same index.
// Field mode: the interior (rows 1..M) of padded fields; the old DENSITY and
// Viscousity are kept as DENSITY0 and Viscousity0 first (as k_eng_props).
// Points outside [x_lo, x_hi] take the table search, which also flags points
// outside the table (PropStatus in points mode, DevState error bit in field
// mode).
struct MlpOut {
    double *H, *T, *D, *M, *K, *CP;
    double *D0, *M0;      // field mode only
};

constexpr int MLP_INF_SMEM = 1024 + 64 * 64 * 2 + 16 * 64 * 2 + 128 * 64 * 2;

// Hardware tanh for inference, two activations per MUFU operation (PTX
// tanh.approx.f16x2): the FP32 pre-activations are rounded to FP16 (relative
// 2^-11) and the tanh is evaluated on the pair (maximum relative error about
// 2^-11).  The FP16 pair is the next layer's operand as it stands: inference
// multiplies FP16 activations by FP16 weights (a finer rounding than the BF16
// operands of training, 2^-9), so no conversion follows the activation.
// Training keeps tanhf, the activation of the CPU oracle's gradient check.
__device__ __forceinline__ uint32_t tanh2_f16(float a, float b) {
    uint32_t in, out;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(in) : "f"(b), "f"(a));  // upper half b, lower half a
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(out) : "r"(in));
    return out;
}
__device__ __forceinline__ uint32_t tanh2_f16(__half2 pre) {
    uint32_t out;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(out) : "r"(*reinterpret_cast<uint32_t*>(&pre)));
    return out;
}
// The first layer's pre-activations w1 x + b1 in FP16 pair arithmetic (on the
// FMA pipe; the packing conversion of the FP32 form shares the MUFU unit with
// the tanh): x = xh + xl split into two FP16 parts (x - xh is exact in FP32),
// then fma(w1, xh, fma(w1, xl, b1)), each fma rounded once to FP16, with w1 and
// b1 rounded to FP16.  The input's own rounding would otherwise be 2^-12 of the
// trained range, a visible shift in the steep part of the property curves.

#define MLP_ACT_TANH 0
#define MLP_ACT_CUBIC 1
// FP32 activation and its derivative (training), in an order the CPU oracle repeats exactly
template <int ACT>
__device__ __forceinline__ float act_f(float z) {
    if constexpr (ACT == MLP_ACT_TANH) {
        return tanhf(z);
    } else {
        const float c = fminf(fmaxf(z, -1.f), 1.f);
        return __fmul_rn(c, __fsub_rn(1.5f, __fmul_rn(__fmul_rn(0.5f, c), c)));
    }
}
template <int ACT>
__device__ __forceinline__ float act_d(float z, float h) {
    if constexpr (ACT == MLP_ACT_TANH) {
        return 1.f - h * h;
    } else {
        const float c = fminf(fmaxf(z, -1.f), 1.f);
        return __fmul_rn(1.5f, __fsub_rn(1.f, __fmul_rn(c, c)));
    }
}
// The clamped cubic on an FP16 pair: each product rounded to FP16, the multiply-add once
__device__ __forceinline__ uint32_t cubic2_f16(__half2 pre) {
    const __half2 c = __hmin2(__hmax2(pre, __float2half2_rn(-1.f)), __float2half2_rn(1.f));
    const __half2 s = __hfma2(__hmul2(c, c), __float2half2_rn(-0.5f), __float2half2_rn(1.5f));
    const __half2 h = __hmul2(c, s);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ uint32_t cubic2_f16(float a, float b) {
    uint32_t in;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(in) : "f"(b), "f"(a));
    return cubic2_f16(*reinterpret_cast<const __half2*>(&in));
}
template <int ACT>
__device__ __forceinline__ uint32_t act2_f16(__half2 pre) {
    if constexpr (ACT == MLP_ACT_TANH) return tanh2_f16(pre);
    else return cubic2_f16(pre);
}
template <int ACT>
__device__ __forceinline__ uint32_t act2_f16(float a, float b) {
    if constexpr (ACT == MLP_ACT_TANH) return tanh2_f16(a, b);
    else return cubic2_f16(a, b);
}

// 16-byte chunk c (k = 8c .. 8c+7) of row r of an R x 64 K-major operand
__device__ __forceinline__ void put_chunk(unsigned char* base, int R, int r, int c, uint32_t a, uint32_t b, uint32_t d,
                                          uint32_t e) {
    *reinterpret_cast<uint4*>(base + umma_off(R, r, 8 * c)) = make_uint4(a, b, d, e);
}

template <bool FIELD, int ACT>
__global__ void __launch_bounds__(MLP_NT, 4) k_mlp_infer(const float* __restrict__ par, MlpOperands ops, MlpNorm nm,
                                                         PropTab tb, Geo g, long long npts, const double* __restrict__ dh,
                                                         MlpOut out, PropStatus* ps, unsigned int* err) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    unsigned char* sW2 = sm;                  // 8 KB
    unsigned char* sW3 = sW2 + 64 * 64 * 2;   // 2 KB
    unsigned char* sA = sW3 + 16 * 64 * 2;    // 16 KB
    __shared__ uint64_t mbar;
    __shared__ uint32_t taddr_s;
    // first-layer weights and biases as FP16 pairs (w1[i], w1[i+1]) and (b1[i], b1[i+1]), four pairs
    // of each per 16-byte load; second-layer biases by fours: every thread reads the same values
    __shared__ uint4 sw1h[MLP_H / 8], sb1h[MLP_H / 8];
    __shared__ float4 sb2[MLP_H / 4];
    __shared__ float sb3[MLP_OUT];
    const int tid = threadIdx.x, warp = tid >> 5;
    copy_smem16(sW2, ops.w2h, 64 * 64 * 2);
    copy_smem16(sW3, ops.w3h, 16 * 64 * 2);
    if (tid < MLP_H / 2) {
        const __half2 w = __floats2half2_rn(par[MLP_W1 + 2 * tid], par[MLP_W1 + 2 * tid + 1]);
        const __half2 b = __floats2half2_rn(par[MLP_B1 + 2 * tid], par[MLP_B1 + 2 * tid + 1]);
        reinterpret_cast<__half2*>(sw1h)[tid] = w;
        reinterpret_cast<__half2*>(sb1h)[tid] = b;
    }
    for (int q = tid; q < MLP_H / 4; q += MLP_NT)
        sb2[q] = make_float4(par[MLP_B2 + 4 * q], par[MLP_B2 + 4 * q + 1], par[MLP_B2 + 4 * q + 2], par[MLP_B2 + 4 * q + 3]);
    if (tid < MLP_OUT) sb3[tid] = par[MLP_B3 + tid];
    if (warp == 0) tmem_alloc(&taddr_s, 128);
    if (tid == 0) mbar_init(&mbar, 1);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = taddr_s;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    uint32_t phase = 0;
    bool ok = true;
    const long long ntiles = (npts + MLP_TILE - 1) / MLP_TILE;
    // The global reads of a tile (rho*h, and in field mode the DENSITY and
    // Viscousity that become DENSITY0 and Viscousity0) are issued one tile
    // ahead, so their latency overlaps the current tile's layers.
    auto point_index = [&](long long p) -> long long {
        if (FIELD && p < npts) {
            int i, j, k;
            io_decode(g, p, i, j, k);
            return pidx(g, i, j, k);
        }
        return p;
    };
    long long p_nx = (long long)blockIdx.x * MLP_TILE + tid;
    long long idx_nx = point_index(p_nx);
    double v_nx = p_nx < npts ? dh[idx_nx] : (double)nm.x_lo;
    double d_nx = 0.0, m_nx = 0.0;
    if (FIELD && p_nx < npts) {
        d_nx = out.D[idx_nx];
        m_nx = out.M[idx_nx];
    }
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long p = p_nx, idx = idx_nx;
        const double v = v_nx, dold = d_nx, mold = m_nx;
        p_nx = (tile + gridDim.x) * MLP_TILE + tid;
        if (tile + gridDim.x < ntiles) {
            idx_nx = point_index(p_nx);
            v_nx = p_nx < npts ? dh[idx_nx] : (double)nm.x_lo;
            if (FIELD && p_nx < npts) {
                d_nx = out.D[idx_nx];
                m_nx = out.M[idx_nx];
            }
        }
        const float x = mlp_x(nm, v);
        const __half xh = __float2half_rn(x);
        const __half xl = __float2half_rn(x - __half2float(xh));
        const __half2 xh2 = __halves2half2(xh, xh), xl2 = __halves2half2(xl, xl);
        // layer 1 (rank one, CUDA cores): h1 = tanh(w1 x + b1), straight into the FP16 operand row
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const uint4 wq = sw1h[c], bq = sb1h[c];
            const uint32_t wv[4] = {wq.x, wq.y, wq.z, wq.w}, bv[4] = {bq.x, bq.y, bq.z, bq.w};
            uint32_t hv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const __half2 w = *reinterpret_cast<const __half2*>(&wv[u]);
                const __half2 b = *reinterpret_cast<const __half2*>(&bv[u]);
                hv[u] = act2_f16<ACT>(__hfma2(w, xh2, __hfma2(w, xl2, b)));
            }
            put_chunk(sA, MLP_TILE, tid, c, hv[0], hv[1], hv[2], hv[3]);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < 4; ++s)
                umma_bf16(tmem, umma_desc(sA, 128, s), umma_desc(sW2, 64, s), umma_idesc_f16(128, 64), s > 0);
            umma_commit(&mbar);
        }
        ok = mbar_wait_warp(&mbar, phase, err) && ok;
        phase ^= 1;
        tc_fence_after();
        // layer 2 epilogue: the row's 64 accumulators in four loads and one wait, + b2, tanh, FP16 row
        uint32_t acc[64];
#pragma unroll
        for (int q = 0; q < 4; ++q) tmem_ld16_raw(tmem + lane_base + 16 * q, acc + 16 * q);
        tmem_ld_wait();
#pragma unroll
        for (int q = 0; q < 4; ++q) tmem_tie16(acc + 16 * q);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float4 b0 = sb2[2 * c], b1 = sb2[2 * c + 1];
            const uint32_t* a = acc + 8 * c;
            auto f = [&](int e) { return __uint_as_float(a[e]); };
            put_chunk(sA, MLP_TILE, tid, c, act2_f16<ACT>(f(0) + b0.x, f(1) + b0.y),
                      act2_f16<ACT>(f(2) + b0.z, f(3) + b0.w), act2_f16<ACT>(f(4) + b1.x, f(5) + b1.y),
                      act2_f16<ACT>(f(6) + b1.z, f(7) + b1.w));
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < 4; ++s)
                umma_bf16(tmem + 64, umma_desc(sA, 128, s), umma_desc(sW3, 16, s), umma_idesc_f16(128, 16), s > 0);
            umma_commit(&mbar);
        }
        ok = mbar_wait_warp(&mbar, phase, err) && ok;
        phase ^= 1;
        tc_fence_after();
        tmem_ld16_raw(tmem + lane_base + 64, acc);
        tmem_ld_wait();
        tmem_tie16(acc);
        if (p < npts) {
            double o[6];
            if (v < (double)nm.x_lo || v > (double)nm.x_hi) {
                if (!prop_point(tb, tb.xdh, tb.xh, v, o)) {
                    if (FIELD) {
                        atomicOr(err, CHS_EBIT_TABLE);
                    } else {
                        atomicAdd(&ps->nbad, 1u);
                        atomicMin(&ps->first_bad, (unsigned long long)p);
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < MLP_OUT; ++k)
                    o[k] = (double)(nm.off[k] + nm.scale[k] * (__uint_as_float(acc[k]) + sb3[k]));
            }
            if (FIELD) {
                out.D0[idx] = dold;
                out.M0[idx] = mold;
            }
            out.H[idx] = o[0]; out.T[idx] = o[1]; out.D[idx] = o[2];
            out.M[idx] = o[3]; out.K[idx] = o[4]; out.CP[idx] = o[5];
        }
        tc_fence_before();
        if (!__syncthreads_and(ok)) break;   // an MMA wait ran out: leave together
    }
    tc_fence_after();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 128);
}

// ---------------------------------------------------------------------------
// One training pass over ntr samples (x in [-1, 1], targets y normalised):
// forward, MSE loss, backward; gradients (and the loss) are added to grad[]
// (FP32 atomics).  Tile t of the grid covers samples t*128 .. t*128+127.
constexpr int MLP_TRN_SMEM = 1024 + 3 * 64 * 64 * 2 + 16 * 64 * 2 + 3 * 128 * 64 * 2 + 128 * 128 * 2 + 64 * 128 * 2 +
                             128 * 64 * 4;

template <int ACT>
__global__ void __launch_bounds__(MLP_NT) k_mlp_train(const float* __restrict__ par, MlpOperands ops,
                                                      const float* __restrict__ xs, const float* __restrict__ ys,
                                                      int ntr, float inv_count, float* __restrict__ grad,
                                                      float* __restrict__ loss, unsigned int* err) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    unsigned char* sW2 = sm;                    // B: W2  (64 x 64)
    unsigned char* sW2T = sW2 + 8192;           // B: W2^T (64 x 64)
    unsigned char* sW3 = sW2T + 8192;           // B: W3  (16 x 64)
    unsigned char* sH1 = sW3 + 2048 + 8192;     // A: h1  (128 x 64)     [after a spare 8 KB]
    unsigned char* sH2 = sH1 + 16384;           // A: h2  (128 x 64)
    unsigned char* sDZ = sH2 + 16384;           // A: dz2 (128 x 64)
    unsigned char* sDZT = sDZ + 16384;          // A: dz2^T (128 rows, 64 used, x K = 128 samples)
    unsigned char* sH1T = sDZT + 32768;         // B: h1^T  (64 x K = 128 samples)
    float* sRed = reinterpret_cast<float*>(sH1T + 16384);  // [128 samples][64]: per-sample terms of the small gradients
    __shared__ uint64_t mbar;
    __shared__ uint32_t taddr_s;
    __shared__ float sw1[MLP_H], sb1[MLP_H], sb2[MLP_H], sW3f[MLP_OUT * MLP_H], sb3[MLP_OUT];
    __shared__ float sDy[MLP_TILE][MLP_OUT + 1], sX[MLP_TILE], sLoss[MLP_TILE];
    const int tid = threadIdx.x, warp = tid >> 5;
    copy_smem16(sW2, ops.w2, 8192);
    copy_smem16(sW2T, ops.w2t, 8192);
    copy_smem16(sW3, ops.w3, 2048);
    // rows 64..127 of dz2^T stay zero
    for (int q = tid; q < 32768 / 16; q += MLP_NT) reinterpret_cast<uint4*>(sDZT)[q] = make_uint4(0, 0, 0, 0);
    for (int q = tid; q < MLP_H; q += MLP_NT) {
        sw1[q] = par[MLP_W1 + q];
        sb1[q] = par[MLP_B1 + q];
        sb2[q] = par[MLP_B2 + q];
    }
    for (int q = tid; q < MLP_OUT * MLP_H; q += MLP_NT) sW3f[q] = par[MLP_W3 + q];
    if (tid < MLP_OUT) sb3[tid] = par[MLP_B3 + tid];
    if (warp == 0) tmem_alloc(&taddr_s, 256);
    if (tid == 0) mbar_init(&mbar, 1);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = taddr_s;   // cols [0,64) layer 2, [64,80) layer 3, [128,192) dL/dh1, [192,256) dL/dW2
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    uint32_t phase = 0;
    const int p = blockIdx.x * MLP_TILE + tid;
    const bool live = p < ntr;
    const float x = live ? xs[p] : 0.f;
    // ---- forward ----
    float h1[MLP_H], h2[MLP_H], acc[16];
    float dz2[MLP_H];  // holds the second layer's activation derivative until the backward pass scales it
#pragma unroll
    for (int i = 0; i < MLP_H; ++i) h1[i] = act_f<ACT>(fmaf(sw1[i], x, sb1[i]));
    put_row64(sH1, 128, tid, h1);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < 4; ++s) umma_bf16(tmem, umma_desc(sH1, 128, s), umma_desc(sW2, 64, s), umma_idesc(128, 64), s > 0);
        umma_commit(&mbar);
    }
    mbar_wait_warp(&mbar, phase, err);
    phase ^= 1;
    tc_fence_after();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        tmem_ld16(tmem + lane_base + 16 * q, acc);
        tmem_ld_wait();
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            const float z = acc[c] + sb2[16 * q + c];
            h2[16 * q + c] = act_f<ACT>(z);
            dz2[16 * q + c] = act_d<ACT>(z, h2[16 * q + c]);
        }
    }
    put_row64(sH2, 128, tid, h2);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < 4; ++s)
            umma_bf16(tmem + 64, umma_desc(sH2, 128, s), umma_desc(sW3, 16, s), umma_idesc(128, 16), s > 0);
        umma_commit(&mbar);
    }
    mbar_wait_warp(&mbar, phase, err);
    phase ^= 1;
    tc_fence_after();
    tmem_ld16(tmem + lane_base + 64, acc);
    tmem_ld_wait();
    // ---- loss and output layer ----
    float dy[MLP_OUT];
    float lsum = 0.f;
#pragma unroll
    for (int k = 0; k < MLP_OUT; ++k) {
        const float e = live ? (acc[k] + sb3[k]) - ys[(long long)p * MLP_OUT + k] : 0.f;
        lsum += e * e;
        dy[k] = 2.f * e * inv_count;
        sDy[tid][k] = dy[k];
    }
    sLoss[tid] = lsum * inv_count;
    sX[tid] = live ? x : 0.f;
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) sRed[tid * MLP_H + j] = h2[j];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < MLP_OUT; ++k) s = fmaf(dy[k], sW3f[k * MLP_H + j], s);
        dz2[j] = s * dz2[j];
    }
    __syncthreads();
    // dW3[k][j] = sum_p dy[p][k] h2[p][j], db3, loss: column sums over the tile
    for (int q = tid; q < MLP_OUT * MLP_H; q += MLP_NT) {
        const int k = q / MLP_H, j = q % MLP_H;
        float a = 0.f;
        for (int r = 0; r < MLP_TILE; ++r) a = fmaf(sDy[r][k], sRed[r * MLP_H + j], a);
        atomicAdd(&grad[MLP_W3 + q], a);
    }
    if (tid < MLP_OUT) {
        float a = 0.f;
        for (int r = 0; r < MLP_TILE; ++r) a += sDy[r][tid];
        atomicAdd(&grad[MLP_B3 + tid], a);
    }
    if (tid == MLP_OUT) {
        float a = 0.f;
        for (int r = 0; r < MLP_TILE; ++r) a += sLoss[r];
        atomicAdd(loss, a);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) sRed[tid * MLP_H + j] = dz2[j];
    __syncthreads();
    if (tid < MLP_H) {  // db2
        float a = 0.f;
        for (int r = 0; r < MLP_TILE; ++r) a += sRed[r * MLP_H + tid];
        atomicAdd(&grad[MLP_B2 + tid], a);
    }
    // dz2 as A (rows = samples) and transposed (rows = hidden units, K = samples); h1 transposed
    put_row64(sDZ, 128, tid, dz2);
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
        const __nv_bfloat16 b = __float2bfloat16_rn(dz2[j]);
        *reinterpret_cast<__nv_bfloat16*>(sDZT + umma_off(128, j, tid)) = b;
        *reinterpret_cast<__nv_bfloat16*>(sH1T + umma_off(64, j, tid)) = __float2bfloat16_rn(h1[j]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < 4; ++s)
            umma_bf16(tmem + 128, umma_desc(sDZ, 128, s), umma_desc(sW2T, 64, s), umma_idesc(128, 64), s > 0);
#pragma unroll
        for (int s = 0; s < 8; ++s)
            umma_bf16(tmem + 192, umma_desc(sDZT, 128, s), umma_desc(sH1T, 64, s), umma_idesc(128, 64), s > 0);
        umma_commit(&mbar);
    }
    mbar_wait_warp(&mbar, phase, err);
    phase ^= 1;
    tc_fence_after();
    // dL/dh1 -> first layer (per-sample dz1 staged, then column sums)
    __syncthreads();   // the db2 sums above are done with sRed
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        tmem_ld16(tmem + lane_base + 128 + 16 * q, acc);
        tmem_ld_wait();
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            const int i = 16 * q + c;
            sRed[tid * MLP_H + i] = live ? acc[c] * act_d<ACT>(fmaf(sw1[i], x, sb1[i]), h1[i]) : 0.f;
        }
    }
    // dL/dW2: TMEM lane j (threads 0..63) holds row j
    if (tid < MLP_H) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tmem + lane_base + 192 + 16 * q, acc);
            tmem_ld_wait();
#pragma unroll
            for (int c = 0; c < 16; ++c) atomicAdd(&grad[MLP_W2 + tid * MLP_H + 16 * q + c], acc[c]);
        }
    } else {
        // the other lanes still take part in the warp-collective loads
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tmem + lane_base + 192 + 16 * q, acc);
            tmem_ld_wait();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (tid < MLP_H) {  // dw1, db1
        float a = 0.f, b = 0.f;
        for (int r = 0; r < MLP_TILE; ++r) {
            const float d = sRed[r * MLP_H + tid];
            a = fmaf(d, sX[r], a);
            b += d;
        }
        atomicAdd(&grad[MLP_W1 + tid], a);
        atomicAdd(&grad[MLP_B1 + tid], b);
    }
    tc_fence_after();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 256);
}

// Adam step on the FP32 master parameters, then the 16-bit operand images
// (BF16 for training, FP16 for inference).  grad is cleared for the next
// pass.  One block of 256 threads.  With step == 0 only the images are
// rebuilt (after new parameters).
__global__ void __launch_bounds__(256) k_mlp_adam(float* __restrict__ par, float* __restrict__ grad,
                                                  float* __restrict__ m1, float* __restrict__ m2, int step, float lr,
                                                  __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w3,
                                                  __nv_bfloat16* __restrict__ w2t, __half* __restrict__ w2h,
                                                  __half* __restrict__ w3h) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    for (int q = threadIdx.x; step > 0 && q < MLP_NPARAM; q += blockDim.x) {
        const float gq = grad[q];
        const float a = b1 * m1[q] + (1.f - b1) * gq;
        const float b = b2 * m2[q] + (1.f - b2) * gq * gq;
        m1[q] = a;
        m2[q] = b;
        par[q] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
        grad[q] = 0.f;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < MLP_H * MLP_H; q += blockDim.x) {
        const int j = q / MLP_H, i = q % MLP_H;
        const __nv_bfloat16 v = __float2bfloat16_rn(par[MLP_W2 + q]);
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(w2) + umma_off(64, j, i)) = v;
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(w2t) + umma_off(64, i, j)) = v;
        *reinterpret_cast<__half*>(reinterpret_cast<unsigned char*>(w2h) + umma_off(64, j, i)) =
            __float2half_rn(par[MLP_W2 + q]);
    }
    for (int q = threadIdx.x; q < MLP_NP * MLP_H; q += blockDim.x) {
        const int k = q / MLP_H, j = q % MLP_H;
        const float v = k < MLP_OUT ? par[MLP_W3 + k * MLP_H + j] : 0.f;
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(w3) + umma_off(16, k, j)) =
            __float2bfloat16_rn(v);
        *reinterpret_cast<__half*>(reinterpret_cast<unsigned char*>(w3h) + umma_off(16, k, j)) = __float2half_rn(v);
    }
}

// Training set: normalised inputs and table-search targets for n rho*h values.
__global__ void __launch_bounds__(PROP_NT) k_mlp_targets(PropTab tb, MlpNorm nm, int n, const double* __restrict__ dh,
                                                         float* __restrict__ xs, float* __restrict__ ys,
                                                         PropStatus* ps) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        double o[6];
        if (!prop_point(tb, tb.xdh, tb.xh, dh[p], o)) atomicAdd(&ps->nbad, 1u);
        xs[p] = mlp_x(nm, dh[p]);
#pragma unroll
        for (int k = 0; k < MLP_OUT; ++k) ys[(long long)p * MLP_OUT + k] = (float)((o[k] - nm.off[k]) / nm.scale[k]);
    }
}

// Judge: per output, the largest |model - table| / max(|table|, scale) over
// the interior of the fields the model produced (non-negative floats compare
// as integers, so atomicMax on their bits is the float maximum).
__global__ void __launch_bounds__(PROP_NT) k_mlp_judge(PropTab tb, MlpNorm nm, Geo g, const double* __restrict__ DH,
                                                       MlpOut cur, unsigned int* __restrict__ errbits) {
    const long long tot = (long long)g.L * g.M * g.N;
    float e[MLP_OUT] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        io_decode(g, q, i, j, k);
        const long long idx = pidx(g, i, j, k);
        double o[6];
        prop_point(tb, tb.xdh, tb.xh, DH[idx], o);
        const double c[6] = {cur.H[idx], cur.T[idx], cur.D[idx], cur.M[idx], cur.K[idx], cur.CP[idx]};
#pragma unroll
        for (int m = 0; m < MLP_OUT; ++m)
            e[m] = fmaxf(e[m], (float)(fabs(c[m] - o[m]) / fmax(fabs(o[m]), (double)nm.scale[m])));
    }
#pragma unroll
    for (int m = 0; m < MLP_OUT; ++m) {
        float v = e[m];
        for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
        if ((threadIdx.x & 31) == 0) atomicMax(errbits + m, __float_as_uint(v));
    }
}
