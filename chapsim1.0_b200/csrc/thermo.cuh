// Thermophysical property update by table search (THERM_PROP_UPDATE,
// src/THERM_PROP_UPDATE.f90:124-168, table arm of THERM_PROP_UPDATE_FROM_DH
// :14-67, spline_interpolation_* src/thermo_properties_table_searching.f90:382-724).
//
// Per point: h from rho*h by the DH->H spline, then T, rho, mu, kappa, cp from
// the H-splines.  The reference runs one binary search per spline call (seven
// per point); all H-splines share LIST_H as abscissae, so one search for h
// serves the five that are evaluated (the beta spline's result is discarded by
// the reference and is not computed).  The search and the cubic are the
// reference's: I = 1, J = N+1 bisection, then y + dx (b + dx (c + dx d)),
// evaluated with explicitly rounded operations so the result is bitwise the
// CPU's (no fused multiply-add contraction).
#pragma once
#include "common.cuh"

constexpr int PROP_NT = 256;
constexpr int PROP_SMEM_MAX_ROWS = 6144;  // both key lists staged in shared memory up to this size (96 KB)

// One spline row {y, b, c, d}, 32-byte aligned.
struct __align__(32) SplineRow {
    double y, b, c, d;
};

// Device copy of the table.  hs holds 5 rows per table row, in output order
// (T, DENSITY, Viscousity, THERMCONDT, HEATCAP); the reference's swapped
// assignment (or the physical one) is applied when the table is packed.
struct PropTab {
    int n;
    int imin_h, imax_h, imin_dh, imax_dh;  // 0-based MINLOC/MAXLOC of LIST_H and LIST_DH
    const double* xdh;                     // LIST_DH
    const double* xh;                      // LIST_H
    const SplineRow* dhh;                  // n rows of the DH->H spline
    const SplineRow* hs;                   // 5n rows of the H-splines
};

struct PropStatus {
    unsigned long long first_bad;  // smallest flat index of a point outside the table (~0 if none)
    unsigned int nbad;             // number of such points
    unsigned int pad;
};

__device__ __forceinline__ int prop_search(const double* __restrict__ key, int n, double u) {
    int i = 0, j = n;
    while (j > i + 1) {
        const int k = (i + j) >> 1;
        if (u < key[k]) j = k; else i = k;
    }
    return i;
}

__device__ __forceinline__ double prop_cubic(const SplineRow& r, double dx) {
    double t = __dmul_rn(dx, r.d);
    t = __dadd_rn(r.c, t);
    t = __dmul_rn(dx, t);
    t = __dadd_rn(r.b, t);
    t = __dmul_rn(dx, t);
    return __dadd_rn(r.y, t);
}

__device__ __forceinline__ SplineRow load_row(const SplineRow* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return SplineRow{a.x, a.y, b.x, b.y};
}

__device__ __forceinline__ bool prop_out_of_range(const double* key, int imin, int imax, double u) {
    return __dsub_rn(u, key[imin]) < -1.0e-8 || __dsub_rn(u, key[imax]) > 1.0e-8;
}

// Point q: reads dh, writes the six fields.  Returns false when the point (or
// its h) lies outside the table, where the reference stops.
__device__ __forceinline__ bool prop_point(const PropTab& tb, const double* xdh, const double* xh, double dh,
                                           double out[6]) {
    bool ok = !prop_out_of_range(xdh, tb.imin_dh, tb.imax_dh, dh);
    const int i = prop_search(xdh, tb.n, dh);
    const double h = prop_cubic(load_row(tb.dhh + i), __dsub_rn(dh, xdh[i]));
    ok = ok && !prop_out_of_range(xh, tb.imin_h, tb.imax_h, h);
    const int m = prop_search(xh, tb.n, h);
    const double dx = __dsub_rn(h, xh[m]);
    out[0] = h;
    const SplineRow* r = tb.hs + 5 * (long long)m;
#pragma unroll
    for (int s = 0; s < 5; ++s) out[1 + s] = prop_cubic(load_row(r + s), dx);
    return ok;
}

__device__ __forceinline__ void prop_flag(PropStatus* st, unsigned long long q) {
    atomicAdd(&st->nbad, 1u);
    atomicMin(&st->first_bad, q);
}

// Flat arrays of npts points.  Grid-stride, so the staged keys serve many points.
template <bool SMEM>
__global__ void __launch_bounds__(PROP_NT) k_prop_points(PropTab tb, long long npts, const double* __restrict__ dh,
                                                         double* __restrict__ H, double* __restrict__ T,
                                                         double* __restrict__ D, double* __restrict__ M,
                                                         double* __restrict__ K, double* __restrict__ CP,
                                                         PropStatus* st) {
    extern __shared__ double keys[];
    const double* xdh = tb.xdh;
    const double* xh = tb.xh;
    if (SMEM) {
        for (int r = threadIdx.x; r < tb.n; r += blockDim.x) {
            keys[r] = tb.xdh[r];
            keys[tb.n + r] = tb.xh[r];
        }
        __syncthreads();
        xdh = keys;
        xh = keys + tb.n;
    }
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npts; q += (long long)gridDim.x * blockDim.x) {
        double o[6];
        if (!prop_point(tb, xdh, xh, __ldg(dh + q), o)) prop_flag(st, (unsigned long long)q);
        H[q] = o[0]; T[q] = o[1]; D[q] = o[2]; M[q] = o[3]; K[q] = o[4]; CP[q] = o[5];
    }
}

// Padded (L, 0:M+1, N) fields, rows j = 1..M (THERM_PROP_UPDATE(IMAIND) of
// the periodic domain, i = 1..NCL1).  The flagged index is the padded offset.
template <bool SMEM>
__global__ void __launch_bounds__(PROP_NT) k_prop_fields(PropTab tb, Geo g, const double* __restrict__ dh,
                                                         double* __restrict__ H, double* __restrict__ T,
                                                         double* __restrict__ D, double* __restrict__ M,
                                                         double* __restrict__ K, double* __restrict__ CP,
                                                         PropStatus* st) {
    extern __shared__ double keys[];
    const double* xdh = tb.xdh;
    const double* xh = tb.xh;
    if (SMEM) {
        for (int r = threadIdx.x; r < tb.n; r += blockDim.x) {
            keys[r] = tb.xdh[r];
            keys[tb.n + r] = tb.xh[r];
        }
        __syncthreads();
        xdh = keys;
        xh = keys + tb.n;
    }
    const long long tot = (long long)g.L * g.M * g.N;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        io_decode(g, q, i, j, k);
        const long long p = pidx(g, i, j, k);
        double o[6];
        if (!prop_point(tb, xdh, xh, __ldg(dh + p), o)) prop_flag(st, (unsigned long long)p);
        H[p] = o[0]; T[p] = o[1]; D[p] = o[2]; M[p] = o[3]; K[p] = o[4]; CP[p] = o[5];
    }
}
