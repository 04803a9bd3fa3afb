// Batched complex FFT in shared memory (four-step, registers per thread).
//
// Stands in for the vendored Temperton FFT99 / CFFT99 (lib/fft99) used by
// FFT99_POIS3D_periodicxz (src/possion3d_FFT99.f90:271-505).  Only the
// discrete transform has to be reproduced, not Temperton's factorisation:
//   forward (SIGN = -1): X[k] = sum_j x[j] exp(-2 pi i j k / n)
//   inverse (SIGN = +1): x[j] = sum_k X[k] exp(+2 pi i j k / n)
// (unnormalised; callers apply the reference's 1/L and 1/N factors).
// Twiddles come from tables computed on the host in extended precision: the
// per-length table tw[e] = exp(-2 pi i e / n) and the constant-memory tables
// of the small DFTs.
#pragma once
#include "common.cuh"

// The transforms are templated on the complex element type C: double2
// (FP64 throughout) or float2 (the spectral stage of the mixed-precision
// step).  CReal<C>::T is the matching real type.
template <typename C> struct CReal;
template <> struct CReal<double2> { using T = double; };
template <> struct CReal<float2> { using T = float; };
__device__ __forceinline__ double2 mkc(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mkc(float x, float y) { return make_float2(x, y); }

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return mkc(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return mkc(a.x - b.x, a.y - b.y); }

// ---------------------------------------------------------------------------
// Four-step FFT in shared memory: n = n1 * n2 with n1, n2 in {4, 8, 12, 16, 24}
// (n1 + 1 odd).
//   x[j1 + n1 j2] -> (A) for every j1 an n2-point DFT over j2 in registers,
//   times W_n^(j1 k2) -> Y(j1, k2) stored at k2 (n1 + 1) + j1 (odd stride, so
//   the column reads of step C are bank-conflict free) -> (C) for every k2 an
//   n1-point DFT over j1 -> X[k2 + n2 k1] in natural order, in place.
// Input and output are in natural order (no digit reversal); each line needs
// n + n2 + 1 complex words of shared memory.  The small DFTs are mixed-radix
// (4, 2, 3) Cooley-Tukey recursions unrolled at compile time, with their
// twiddles in constant memory (FP64 and FP32 copies).
__constant__ double2 c_w8[8], c_w12[12], c_w16[16], c_w24[24];
__constant__ float2 c_w8f[8], c_w12f[12], c_w16f[16], c_w24f[24];

template <int P, typename C> struct CwTab;
template <> struct CwTab<8, double2> { __device__ static double2 at(int e) { return c_w8[e]; } };
template <> struct CwTab<12, double2> { __device__ static double2 at(int e) { return c_w12[e]; } };
template <> struct CwTab<16, double2> { __device__ static double2 at(int e) { return c_w16[e]; } };
template <> struct CwTab<24, double2> { __device__ static double2 at(int e) { return c_w24[e]; } };
template <> struct CwTab<6, double2> { __device__ static double2 at(int e) { return c_w24[4 * e]; } };
template <> struct CwTab<8, float2> { __device__ static float2 at(int e) { return c_w8f[e]; } };
template <> struct CwTab<12, float2> { __device__ static float2 at(int e) { return c_w12f[e]; } };
template <> struct CwTab<16, float2> { __device__ static float2 at(int e) { return c_w16f[e]; } };
template <> struct CwTab<24, float2> { __device__ static float2 at(int e) { return c_w24f[e]; } };
template <> struct CwTab<6, float2> { __device__ static float2 at(int e) { return c_w24f[4 * e]; } };

// W_P^e = exp(SIGN 2 pi i e / P)
template <int P, int SIGN, typename C>
__device__ __forceinline__ C cw(int e) {
    C w = CwTab<P, C>::at(e % P);
    if (SIGN > 0) w.y = -w.y;
    return w;
}

template <int P, int SIGN, typename C> struct SmallDft;

template <int SIGN, typename C> struct SmallDft<2, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};
template <int SIGN, typename C> struct SmallDft<3, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        using T = typename CReal<C>::T;
        const T h = (T)0.86602540378443864676;  // sin(2 pi / 3)
        const C s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        const C c = mkc(v[0].x - (T)0.5 * s.x, v[0].y - (T)0.5 * s.y);
        const C t = mkc(-SIGN * h * d.y, SIGN * h * d.x);
        v[0] = cadd(v[0], s);
        v[1] = cadd(c, t);
        v[2] = csub(c, t);
    }
};
template <int SIGN, typename C> struct SmallDft<4, SIGN, C> {
    __device__ __forceinline__ static void run(C* v) {
        const C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const C s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        const C wd = mkc(-SIGN * d13.y, SIGN * d13.x);
        v[0] = cadd(s02, s13);
        v[1] = cadd(d02, wd);
        v[2] = csub(s02, s13);
        v[3] = csub(d02, wd);
    }
};
// P = A * B: A sub-DFTs of length B over v[a + A b], twiddle W_P^(a kb), then
// B DFTs of length A; output X[kb + B ka].
template <int P> struct Split { static constexpr int A = (P % 4 == 0 && P != 4) ? 4 : ((P % 2 == 0 && P != 2) ? 2 : 3); };
template <int P, int SIGN, typename C> struct SmallDft {
    __device__ __forceinline__ static void run(C* v) {
        constexpr int A = Split<P>::A, B = P / A;
        C u[A][B];
#pragma unroll
        for (int a = 0; a < A; ++a) {
#pragma unroll
            for (int b = 0; b < B; ++b) u[a][b] = v[a + A * b];
            SmallDft<B, SIGN, C>::run(u[a]);
#pragma unroll
            for (int kb = 1; kb < B; ++kb)
                if (a > 0) u[a][kb] = cmul(u[a][kb], cw<P, SIGN, C>(a * kb));
        }
#pragma unroll
        for (int kb = 0; kb < B; ++kb) {
            C t[A];
#pragma unroll
            for (int a = 0; a < A; ++a) t[a] = u[a][kb];
            SmallDft<A, SIGN, C>::run(t);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) v[kb + B * ka] = t[ka];
        }
    }
};

template <int N1, int N2, int SIGN, typename C>
__device__ void block_fft4s(C* buf, int nl, int ld, const C* __restrict__ tw) {
    // Each pass is in place (all reads of a line, barrier, all writes), so one
    // iteration of a pass always holds whole lines.
    __syncthreads();
    {  // step A: tasks (line, j1)
        const int lpi = blockDim.x / N1;  // lines per iteration
        for (int l0 = 0; l0 < nl; l0 += lpi) {
            const int line = l0 + threadIdx.x / N1, j1 = threadIdx.x % N1;
            const bool on = threadIdx.x < lpi * N1 && line < nl;
            C v[N2];
            C* x = buf + (long long)(on ? line : 0) * ld;
            if (on) {
#pragma unroll
                for (int j2 = 0; j2 < N2; ++j2) v[j2] = x[j1 + N1 * j2];
            }
            __syncthreads();
            if (on) {
                SmallDft<N2, SIGN, C>::run(v);
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) {
                    C w = tw[j1 * k2];
                    if (SIGN > 0) w.y = -w.y;
                    x[k2 * (N1 + 1) + j1] = (j1 == 0 || k2 == 0) ? v[k2] : cmul(v[k2], w);
                }
            }
            __syncthreads();
        }
    }
    {  // step C: tasks (line, k2)
        const int lpi = blockDim.x / N2;
        for (int l0 = 0; l0 < nl; l0 += lpi) {
            const int line = l0 + threadIdx.x / N2, k2 = threadIdx.x % N2;
            const bool on = threadIdx.x < lpi * N2 && line < nl;
            C v[N1];
            C* x = buf + (long long)(on ? line : 0) * ld;
            if (on) {
#pragma unroll
                for (int j1 = 0; j1 < N1; ++j1) v[j1] = x[k2 * (N1 + 1) + j1];
            }
            __syncthreads();
            if (on) {
                SmallDft<N1, SIGN, C>::run(v);
#pragma unroll
                for (int k1 = 0; k1 < N1; ++k1) x[k2 + N2 * k1] = v[k1];
            }
            __syncthreads();
        }
    }
}

// n1 x n2 split of the supported lengths (chosen for register use: no or
// small spills under the two-blocks-per-SM register budget)
__host__ __device__ inline bool fft4s_split(int n, int& n1, int& n2) {
    switch (n) {
        case 32: n1 = 4; n2 = 8; return true;
        case 64: n1 = 8; n2 = 8; return true;
        case 96: n1 = 12; n2 = 8; return true;
        case 128: n1 = 16; n2 = 8; return true;
        case 192: n1 = 16; n2 = 12; return true;
        case 256: n1 = 16; n2 = 16; return true;
        case 384: n1 = 16; n2 = 24; return true;
        default: return false;
    }
}
__host__ __device__ inline int fft4s_ld(int n) {
    int n1 = 0, n2 = 0;
    fft4s_split(n, n1, n2);
    return n + n2 + 1;
}

// Host dispatch of a kernel templated on the split of the line length n:
// defines constexpr FN1, FN2 for KERNEL_CALL.
#define DISPATCH_FFT(n_, KERNEL_CALL)                                               \
    switch (n_) {                                                                  \
        case 32: { constexpr int FN1 = 4, FN2 = 8; KERNEL_CALL; } break;           \
        case 64: { constexpr int FN1 = 8, FN2 = 8; KERNEL_CALL; } break;           \
        case 96: { constexpr int FN1 = 12, FN2 = 8; KERNEL_CALL; } break;          \
        case 128: { constexpr int FN1 = 16, FN2 = 8; KERNEL_CALL; } break;         \
        case 192: { constexpr int FN1 = 16, FN2 = 12; KERNEL_CALL; } break;        \
        case 256: { constexpr int FN1 = 16, FN2 = 16; KERNEL_CALL; } break;        \
        case 384: { constexpr int FN1 = 16, FN2 = 24; KERNEL_CALL; } break;        \
        default: break;                                                            \
    }
