// Batched in-place complex FFT in shared memory, mixed radix 2/3/4.
//
// Stands in for the vendored Temperton FFT99 / CFFT99 (lib/fft99) used by
// FFT99_POIS3D_periodicxz (src/possion3d_FFT99.f90:271-505).  Only the
// discrete transform has to be reproduced, not Temperton's factorisation:
//   forward (SIGN = -1): X[k] = sum_j x[j] exp(-2 pi i j k / n)
//   inverse (SIGN = +1): x[j] = sum_k X[k] exp(+2 pi i j k / n)
// (unnormalised; callers apply the reference's 1/L and 1/N factors).
//
// Algorithm: iterative decimation in time.  The caller stores input element
// j at position perm[j] (mixed-radix digit reversal for the pass order
// rad[0], rad[1], ...); pass p with radix r and span m combines, for every
// group of m*r positions, the elements g*m*r + k + t*m (t = 0..r-1), after
// multiplying element t by W_{m r}^{t k}.  Output is in natural order.
// Twiddles come from a table tw[e] = exp(-2 pi i e / n) computed on the
// host in extended precision.
#pragma once
#include "common.cuh"

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// FFT of nl lines of length n, line l at buf + l*ld, executed by all
// threads of the block.  Contains __syncthreads(); every thread must call.
template <int SIGN>
__device__ void block_fft(double2* buf, int n, int nl, int ld, const double2* __restrict__ tw,
                          const int* rad, int nrad) {
    int m = 1;
    for (int p = 0; p < nrad; ++p) {
        const int r = rad[p];
        const int nb = n / r;        // butterflies per line
        const int tstride = n / (m * r);
        const int total = nb * nl;
        __syncthreads();
        for (int b = threadIdx.x; b < total; b += blockDim.x) {
            const int line = b / nb;
            const int jb = b - line * nb;
            const int g = jb / m;
            const int k = jb - g * m;
            double2* base = buf + (long long)line * ld + g * m * r + k;
            if (r == 4) {
                double2 v0 = base[0], v1 = base[m], v2 = base[2 * m], v3 = base[3 * m];
                if (k) {
                    double2 w1 = tw[k * tstride], w2 = tw[2 * k * tstride], w3 = tw[3 * k * tstride];
                    if (SIGN > 0) { w1.y = -w1.y; w2.y = -w2.y; w3.y = -w3.y; }
                    v1 = cmul(v1, w1); v2 = cmul(v2, w2); v3 = cmul(v3, w3);
                }
                double2 s02 = cadd(v0, v2), d02 = csub(v0, v2);
                double2 s13 = cadd(v1, v3), d13 = csub(v1, v3);
                // W_4 = exp(SIGN * i pi / 2) = SIGN * i ;  W*d13 = SIGN*(-d13.y, d13.x)
                double2 wd = make_double2(-SIGN * d13.y, SIGN * d13.x);
                base[0] = cadd(s02, s13);
                base[m] = cadd(d02, wd);
                base[2 * m] = csub(s02, s13);
                base[3 * m] = csub(d02, wd);
            } else if (r == 2) {
                double2 v0 = base[0], v1 = base[m];
                if (k) {
                    double2 w1 = tw[k * tstride];
                    if (SIGN > 0) w1.y = -w1.y;
                    v1 = cmul(v1, w1);
                }
                base[0] = cadd(v0, v1);
                base[m] = csub(v0, v1);
            } else {  // r == 3
                double2 v0 = base[0], v1 = base[m], v2 = base[2 * m];
                if (k) {
                    double2 w1 = tw[k * tstride], w2 = tw[2 * k * tstride];
                    if (SIGN > 0) { w1.y = -w1.y; w2.y = -w2.y; }
                    v1 = cmul(v1, w1); v2 = cmul(v2, w2);
                }
                const double h = 0.86602540378443864676;  // sin(2 pi / 3)
                double2 s = cadd(v1, v2), df = csub(v1, v2);
                double2 c = make_double2(v0.x - 0.5 * s.x, v0.y - 0.5 * s.y);
                // W_3 = (-1/2, SIGN*h):  X1 = c + SIGN*i*h*df,  X2 = c - SIGN*i*h*df
                double2 t = make_double2(-SIGN * h * df.y, SIGN * h * df.x);
                base[0] = cadd(v0, s);
                base[m] = cadd(c, t);
                base[2 * m] = csub(c, t);
            }
        }
        m *= r;
    }
    __syncthreads();
}
