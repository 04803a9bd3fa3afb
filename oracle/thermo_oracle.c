/*
 * thermo_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of CHAPSim's property update from rho*h by table
 * search (iThermoProperty = search_table), used by tests/ and the CPU
 * baseline as the checker of the CUDA property kernel.  Nothing in the
 * product library links or calls it.
 *
 * Follows, statement by statement and in the same floating-point order
 * (compiled with -ffp-contract=off):
 *   Property_Table_Nondimensionalization  src/thermo_properties_table_searching.f90:1226-1346
 *   BiSection_LIST_T                      src/thermo_properties_table_searching.f90:808-839
 *   CUBIC_SPLINE (Forsythe-Malcolm-Moler) src/thermo_properties_table_searching.f90:842-936
 *   SPLINE_COEFFICIENTS_FOR_DH / _FOR_H   src/thermo_properties_table_searching.f90:972-1128
 *   spline_interpolation_DHH/HT/HD/HM/HK/HCp/HB
 *                                         src/thermo_properties_table_searching.f90:382-724
 *   THERM_PROP_UPDATE_FROM_DH (table arm) src/THERM_PROP_UPDATE.f90:14-67
 * Arrays are 0-based here; indices reported to callers are the reference's
 * 1-based ones.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* CUBIC_SPLINE(N, X, Y, B, C, D): natural-order FMM spline with end
 * conditions from third divided differences. */
void orc_cubic_spline(int n, const double* x, const double* y, double* b, double* c, double* d) {
    if (n < 2) return;
    if (n < 3) {
        b[0] = (y[1] - y[0]) / (x[1] - x[0]);
        c[0] = 0.0; d[0] = 0.0;
        b[1] = b[0]; c[1] = 0.0; d[1] = 0.0;
        return;
    }
    const int nm1 = n - 1; /* NM1, 1-based count */
    /* step 1: tridiagonal system; 1-based I maps to i = I-1 */
    d[0] = x[1] - x[0];
    c[1] = (y[1] - y[0]) / d[0];
    for (int I = 2; I <= nm1; ++I) {
        const int i = I - 1;
        d[i] = x[i + 1] - x[i];
        b[i] = 2.0 * (d[i - 1] + d[i]);
        c[i + 1] = (y[i + 1] - y[i]) / d[i];
        c[i] = c[i + 1] - c[i];
    }
    /* step 2: end conditions */
    b[0] = -d[0];
    b[n - 1] = -d[n - 2];
    c[0] = 0.0;
    c[n - 1] = 0.0;
    if (n != 3) {
        c[0] = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0]);
        c[n - 1] = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4]);
        c[0] = c[0] * d[0] * d[0] / (x[3] - x[0]);
        c[n - 1] = -c[n - 1] * (d[n - 2] * d[n - 2]) / (x[n - 1] - x[n - 4]);
    }
    /* step 3: forward elimination */
    for (int I = 2; I <= n; ++I) {
        const int i = I - 1;
        const double t = d[i - 1] / b[i - 1];
        b[i] = b[i] - t * d[i - 1];
        c[i] = c[i] - t * c[i - 1];
    }
    /* step 4: back substitution */
    c[n - 1] = c[n - 1] / b[n - 1];
    for (int L = 1; L <= nm1; ++L) {
        const int i = n - L - 1;
        c[i] = (c[i] - d[i] * c[i + 1]) / b[i];
    }
    /* step 5: polynomial coefficients */
    b[n - 1] = (y[n - 1] - y[nm1 - 1]) / d[nm1 - 1] + d[nm1 - 1] * (c[nm1 - 1] + 2.0 * c[n - 1]);
    for (int I = 1; I <= nm1; ++I) {
        const int i = I - 1;
        b[i] = (y[i + 1] - y[i]) / d[i] - d[i] * (c[i + 1] + 2.0 * c[i]);
        d[i] = (c[i + 1] - c[i]) / d[i];
        c[i] = 3.0 * c[i];
    }
    c[n - 1] = 3.0 * c[n - 1];
    d[n - 1] = d[nm1 - 1];
}

/* Binary search of spline_interpolation_*: I = 1, J = N+1 (0-based: 0, n),
 * x(I) <= u < x(I+1); u at or above the last knot gives I = N. */
int orc_spline_index(int n, const double* xl, double u) {
    int i = 0, j = n;
    while (j > i + 1) {
        const int k = (i + j) / 2;
        if (u < xl[k]) j = k; else i = k;
    }
    return i;
}

/* One spline_interpolation_* call.  Returns 0, or 1 / 2 when u lies more
 * than 1e-8 below xl[imin] / above xl[imax] (the reference STOPs there). */
int orc_spline_eval(int n, const double* xl, const double* yl, const double* b, const double* c, const double* d,
                    int imin, int imax, double u, double* out) {
    if ((u - xl[imin]) < -1.0e-8) return 1;
    if ((u - xl[imax]) > 1.0e-8) return 2;
    const int i = orc_spline_index(n, xl, u);
    const double dx = u - xl[i];
    *out = yl[i] + dx * (b[i] + dx * (c[i] + dx * d[i]));
    return 0;
}

static int minloc(int n, const double* a) {
    int k = 0;
    for (int i = 1; i < n; ++i) if (a[i] < a[k]) k = i;
    return k;
}
static int maxloc(int n, const double* a) {
    int k = 0;
    for (int i = 1; i < n; ++i) if (a[i] > a[k]) k = i;
    return k;
}

/* Property_Table_Nondimensionalization.  raw: n rows of the table file's 8
 * columns (P, H, T, D, M, K, CP, B), row-major.  lists (8*n): H, T, D, M, K,
 * CP, B, DH, sorted by T and scaled by the reference state at T0; ref (6):
 * H0, D0, K0, M0, CP0, B0 (dimensional). */
void orc_table_nondim(int n, const double* raw, double T0, double* lists, double* ref) {
    double* H = lists;
    double* T = lists + n;
    double* D = lists + 2 * n;
    double* M = lists + 3 * n;
    double* K = lists + 4 * n;
    double* CP = lists + 5 * n;
    double* B = lists + 6 * n;
    double* DH = lists + 7 * n;
    for (int i = 0; i < n; ++i) {
        H[i] = raw[8 * i + 1]; T[i] = raw[8 * i + 2]; D[i] = raw[8 * i + 3]; M[i] = raw[8 * i + 4];
        K[i] = raw[8 * i + 5]; CP[i] = raw[8 * i + 6]; B[i] = raw[8 * i + 7]; DH[i] = 0.0;
    }
    /* selection sort on T (MINLOC: first minimum of T(I:N)) */
    for (int i = 0; i < n; ++i) {
        const int k = minloc(n - i, T + i) + i;
        double* cols[7] = {T, D, H, M, K, B, CP};
        for (int c = 0; c < 7; ++c) {
            const double buf = cols[c][i];
            cols[c][i] = cols[c][k];
            cols[c][k] = buf;
        }
    }
    /* BiSection_LIST_T(T0, IE, IS), 1-based IS = 1, IE = N */
    int is = 1, ie = n;
    while ((ie - is) > 1) {
        const int im = is + (ie - is) / 2;
        const double vs = T[is - 1] - T0;
        const double vm = T[im - 1] - T0;
        if (vs * vm > 0.0) is = im; else ie = im;
    }
    const double sfs = (T[ie - 1] - T0) / (T[ie - 1] - T[is - 1]);
    const double sfe = 1.0 - sfs;
    const double H0 = sfe * H[ie - 1] + sfs * H[is - 1];
    const double D0 = sfe * D[ie - 1] + sfs * D[is - 1];
    const double K0 = sfe * K[ie - 1] + sfs * K[is - 1];
    const double M0 = sfe * M[ie - 1] + sfs * M[is - 1];
    const double CP0 = sfe * CP[ie - 1] + sfs * CP[is - 1];
    const double B0 = sfe * B[ie - 1] + sfs * B[is - 1];
    for (int i = 0; i < n; ++i) {
        H[i] = (H[i] - H0) / T0 / CP0;
        T[i] = T[i] / T0;
        D[i] = D[i] / D0;
        M[i] = M[i] / M0;
        K[i] = K[i] / K0;
        CP[i] = CP[i] / CP0;
        B[i] = B[i] / B0;
        DH[i] = D[i] * H[i];
    }
    ref[0] = H0; ref[1] = D0; ref[2] = K0; ref[3] = M0; ref[4] = CP0; ref[5] = B0;
}

/* Table with spline coefficients, as built by SPLINE_COEFFICIENTS_FOR_DH
 * (DH->H) and SPLINE_COEFFICIENTS_FOR_H (H->T, D, M, K, CP, B). */
typedef struct {
    int n, fix_swap;
    int imin_h, imax_h, imin_dh, imax_dh; /* 0-based */
    double* lists;                        /* 8*n: H, T, D, M, K, CP, B, DH */
    double* coef;                         /* 7 splines x 3 x n: DHH, HT, HD, HM, HK, HCP, HB; each B, C, D */
} orc_table;

enum { SP_DHH = 0, SP_HT, SP_HD, SP_HM, SP_HK, SP_HCP, SP_HB, SP_COUNT };

static double* spl(orc_table* t, int s, int which) { return t->coef + ((size_t)s * 3 + which) * t->n; }

void* orc_table_create(int n, const double* lists, int fix_swap) {
    if (n < 4) return NULL;
    orc_table* t = (orc_table*)calloc(1, sizeof(orc_table));
    t->n = n;
    t->fix_swap = fix_swap;
    t->lists = (double*)malloc(sizeof(double) * 8 * n);
    memcpy(t->lists, lists, sizeof(double) * 8 * n);
    t->coef = (double*)calloc((size_t)SP_COUNT * 3 * n, sizeof(double));
    const double* H = t->lists;
    const double* DH = t->lists + 7 * n;
    t->imax_h = maxloc(n, H);
    t->imin_h = minloc(n, H);
    t->imax_dh = maxloc(n, DH);
    t->imin_dh = minloc(n, DH);
    orc_cubic_spline(n, DH, H, spl(t, SP_DHH, 0), spl(t, SP_DHH, 1), spl(t, SP_DHH, 2));
    for (int s = SP_HT; s <= SP_HB; ++s) {
        /* LIST_T, D, M, K, CP, B are lists[1..6] */
        const double* y = t->lists + (size_t)(s - SP_HT + 1) * n;
        orc_cubic_spline(n, H, y, spl(t, s, 0), spl(t, s, 1), spl(t, s, 2));
    }
    return t;
}

void orc_table_destroy(void* p) {
    orc_table* t = (orc_table*)p;
    if (!t) return;
    free(t->lists);
    free(t->coef);
    free(t);
}

/* coefficient block of spline s: out (3*n) */
void orc_table_coefs(void* p, int s, double* out) {
    orc_table* t = (orc_table*)p;
    memcpy(out, spl(t, s, 0), sizeof(double) * 3 * t->n);
}

/* 0-based IMIN_H, IMAX_H, IMIN_DH, IMAX_DH */
void orc_table_extrema(void* p, int* out) {
    orc_table* t = (orc_table*)p;
    out[0] = t->imin_h; out[1] = t->imax_h; out[2] = t->imin_dh; out[3] = t->imax_dh;
}

static int eval_s(orc_table* t, int s, const double* xl, int imin, int imax, double u, double* out) {
    const double* y = (s == SP_DHH) ? t->lists : t->lists + (size_t)(s - SP_HT + 1) * t->n;
    return orc_spline_eval(t->n, xl, y, spl(t, s, 0), spl(t, s, 1), spl(t, s, 2), imin, imax, u, out);
}

/* THERM_PROP_UPDATE_FROM_DH, table arm, over npts points.  out: 6*npts
 * (ENTHALPY, TEMPERATURE, DENSITY, Viscousity, THERMCONDT, HEATCAP).  With
 * fix_swap = 0 the reference's assignment is kept: DENSITY <- HM spline,
 * Viscousity <- HK spline, THERMCONDT <- HD spline.  Returns the number of
 * points outside the table (the reference STOPs on the first); *first_bad
 * gets the smallest such index, or -1. */
long orc_prop_update(void* p, long npts, const double* dh, double* out, long* first_bad) {
    orc_table* t = (orc_table*)p;
    const double* H = t->lists;
    const double* DH = t->lists + 7 * t->n;
    long nbad = 0, fb = -1;
#pragma omp parallel for reduction(+ : nbad) schedule(static)
    for (long q = 0; q < npts; ++q) {
        double h = 0, T = 0, vd = 0, vm = 0, vk = 0, cp = 0, b = 0;
        int rc = eval_s(t, SP_DHH, DH, t->imin_dh, t->imax_dh, dh[q], &h);
        if (!rc) rc |= eval_s(t, SP_HT, H, t->imin_h, t->imax_h, h, &T);
        if (!rc) {
            if (t->fix_swap) {
                rc |= eval_s(t, SP_HD, H, t->imin_h, t->imax_h, h, &vd);
                rc |= eval_s(t, SP_HM, H, t->imin_h, t->imax_h, h, &vm);
                rc |= eval_s(t, SP_HK, H, t->imin_h, t->imax_h, h, &vk);
            } else {
                rc |= eval_s(t, SP_HM, H, t->imin_h, t->imax_h, h, &vd);
                rc |= eval_s(t, SP_HK, H, t->imin_h, t->imax_h, h, &vm);
                rc |= eval_s(t, SP_HD, H, t->imin_h, t->imax_h, h, &vk);
            }
            rc |= eval_s(t, SP_HCP, H, t->imin_h, t->imax_h, h, &cp);
            rc |= eval_s(t, SP_HB, H, t->imin_h, t->imax_h, h, &b);
        }
        out[q] = h; out[npts + q] = T; out[2 * npts + q] = vd;
        out[3 * npts + q] = vm; out[4 * npts + q] = vk; out[5 * npts + q] = cp;
        if (rc) {
            ++nbad;
#pragma omp critical
            if (fb < 0 || q < fb) fb = q;
        }
    }
    if (first_bad) *first_bad = fb;
    return nbad;
}

/* One point of THERM_PROP_UPDATE_FROM_DH (table arm): out = H, T, DENSITY,
 * Viscousity, THERMCONDT, HEATCAP.  Returns nonzero when the point (or its
 * h) is outside the table, where the reference STOPs. */
int orc_prop_point(void* p, double dh, double* out) {
    orc_table* t = (orc_table*)p;
    const double* H = t->lists;
    const double* DH = t->lists + 7 * t->n;
    double h = 0, T = 0, vd = 0, vm = 0, vk = 0, cp = 0, b = 0;
    int rc = eval_s(t, SP_DHH, DH, t->imin_dh, t->imax_dh, dh, &h);
    if (!rc) rc |= eval_s(t, SP_HT, H, t->imin_h, t->imax_h, h, &T);
    if (!rc) {
        if (t->fix_swap) {
            rc |= eval_s(t, SP_HD, H, t->imin_h, t->imax_h, h, &vd);
            rc |= eval_s(t, SP_HM, H, t->imin_h, t->imax_h, h, &vm);
            rc |= eval_s(t, SP_HK, H, t->imin_h, t->imax_h, h, &vk);
        } else {
            rc |= eval_s(t, SP_HM, H, t->imin_h, t->imax_h, h, &vd);
            rc |= eval_s(t, SP_HK, H, t->imin_h, t->imax_h, h, &vm);
            rc |= eval_s(t, SP_HD, H, t->imin_h, t->imax_h, h, &vk);
        }
        rc |= eval_s(t, SP_HCP, H, t->imin_h, t->imax_h, h, &cp);
        rc |= eval_s(t, SP_HB, H, t->imin_h, t->imax_h, h, &b);
    }
    out[0] = h; out[1] = T; out[2] = vd; out[3] = vm; out[4] = vk; out[5] = cp;
    return rc;
}

/* DHmin, DHmax of SPLINE_COEFFICIENTS_FOR_H (:1115-1118): LIST_DH at IMIN_DH, IMAX_DH */
void orc_table_dh_limits(void* p, double* out) {
    orc_table* t = (orc_table*)p;
    const double* DH = t->lists + 7 * t->n;
    out[0] = DH[t->imin_dh];
    out[1] = DH[t->imax_dh];
}
