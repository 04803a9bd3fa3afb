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

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

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
// twiddles in constant memory.
__constant__ double2 c_w8[8], c_w12[12], c_w16[16], c_w24[24];

template <int P> __device__ __forceinline__ double2 cwtab(int e);
template <> __device__ __forceinline__ double2 cwtab<8>(int e) { return c_w8[e]; }
template <> __device__ __forceinline__ double2 cwtab<12>(int e) { return c_w12[e]; }
template <> __device__ __forceinline__ double2 cwtab<16>(int e) { return c_w16[e]; }
template <> __device__ __forceinline__ double2 cwtab<24>(int e) { return c_w24[e]; }
template <> __device__ __forceinline__ double2 cwtab<6>(int e) { return c_w24[4 * e]; }

// W_P^e = exp(SIGN 2 pi i e / P)
template <int P, int SIGN>
__device__ __forceinline__ double2 cw(int e) {
    double2 w = cwtab<P>(e % P);
    if (SIGN > 0) w.y = -w.y;
    return w;
}

template <int P, int SIGN> struct SmallDft;

template <int SIGN> struct SmallDft<2, SIGN> {
    __device__ __forceinline__ static void run(double2* v) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};
template <int SIGN> struct SmallDft<3, SIGN> {
    __device__ __forceinline__ static void run(double2* v) {
        const double h = 0.86602540378443864676;  // sin(2 pi / 3)
        const double2 s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        const double2 c = make_double2(v[0].x - 0.5 * s.x, v[0].y - 0.5 * s.y);
        const double2 t = make_double2(-SIGN * h * d.y, SIGN * h * d.x);
        v[0] = cadd(v[0], s);
        v[1] = cadd(c, t);
        v[2] = csub(c, t);
    }
};
template <int SIGN> struct SmallDft<4, SIGN> {
    __device__ __forceinline__ static void run(double2* v) {
        const double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const double2 s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        const double2 wd = make_double2(-SIGN * d13.y, SIGN * d13.x);
        v[0] = cadd(s02, s13);
        v[1] = cadd(d02, wd);
        v[2] = csub(s02, s13);
        v[3] = csub(d02, wd);
    }
};
// P = A * B: A sub-DFTs of length B over v[a + A b], twiddle W_P^(a kb), then
// B DFTs of length A; output X[kb + B ka].
template <int P> struct Split { static constexpr int A = (P % 4 == 0 && P != 4) ? 4 : ((P % 2 == 0 && P != 2) ? 2 : 3); };
template <int P, int SIGN> struct SmallDft {
    __device__ __forceinline__ static void run(double2* v) {
        constexpr int A = Split<P>::A, B = P / A;
        double2 u[A][B];
#pragma unroll
        for (int a = 0; a < A; ++a) {
#pragma unroll
            for (int b = 0; b < B; ++b) u[a][b] = v[a + A * b];
            SmallDft<B, SIGN>::run(u[a]);
#pragma unroll
            for (int kb = 1; kb < B; ++kb)
                if (a > 0) u[a][kb] = cmul(u[a][kb], cw<P, SIGN>(a * kb));
        }
#pragma unroll
        for (int kb = 0; kb < B; ++kb) {
            double2 t[A];
#pragma unroll
            for (int a = 0; a < A; ++a) t[a] = u[a][kb];
            SmallDft<A, SIGN>::run(t);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) v[kb + B * ka] = t[ka];
        }
    }
};

template <int N1, int N2, int SIGN>
__device__ void block_fft4s(double2* buf, int nl, int ld, const double2* __restrict__ tw) {
    // Each pass is in place (all reads of a line, barrier, all writes), so one
    // iteration of a pass always holds whole lines.
    __syncthreads();
    {  // step A: tasks (line, j1)
        const int lpi = blockDim.x / N1;  // lines per iteration
        for (int l0 = 0; l0 < nl; l0 += lpi) {
            const int line = l0 + threadIdx.x / N1, j1 = threadIdx.x % N1;
            const bool on = threadIdx.x < lpi * N1 && line < nl;
            double2 v[N2];
            double2* x = buf + (long long)(on ? line : 0) * ld;
            if (on) {
#pragma unroll
                for (int j2 = 0; j2 < N2; ++j2) v[j2] = x[j1 + N1 * j2];
            }
            __syncthreads();
            if (on) {
                SmallDft<N2, SIGN>::run(v);
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) {
                    double2 w = tw[j1 * k2];
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
            double2 v[N1];
            double2* x = buf + (long long)(on ? line : 0) * ld;
            if (on) {
#pragma unroll
                for (int j1 = 0; j1 < N1; ++j1) v[j1] = x[k2 * (N1 + 1) + j1];
            }
            __syncthreads();
            if (on) {
                SmallDft<N1, SIGN>::run(v);
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
