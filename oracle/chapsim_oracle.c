/*
 * chapsim_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of CHAPSim's fractional-step time step for the
 * periodic ("TG", iDomain=1) plane channel (iCase=1).  It exists to check
 * the CUDA path and to provide the timed CPU baseline; nothing in the product
 * library links, loads or calls it.  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may use it.
 *
 * Every routine follows the Fortran subroutine named in its comment,
 * statement by statement and in the same floating-point operation order,
 * so that results agree with the reference to round-off.  Pinning: the
 * setup stage (mesh, metrics, TDMA/Poisson coefficients, Poiseuille
 * profile) is checked against the reference's own CHK_*.dat dumps of
 * test_cases_template/TC8_Channel_IO_thermal_LiquidWater/0_log_monitors.
 *
 * Layout (identical to the reference and to the CUDA path):
 *   field F(i, j, k), i = 1..L, j = 0..M+1 (ghosts at 0 and M+1), k = 1..N,
 *   column-major, x fastest:  off = (i-1) + L*(j + (M+2)*(k-1)).
 *   Q holds u, v, w as three consecutive such fields.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int L, M, N, NND2;
    int xo, LS;  /* x offset and x stride: 0, L (x-periodic); 1, L+2 (inflow/outflow main domain, ghost
                    columns i = 0 and L+1, NCL1S:NCL1E of src/READINI.f90:597-605) */
    double HX, HZ, STR2, REN, CVISC;
    int iFlowDriven;
    double Cf_Given;
    double DT, DT0, DTMIN, CFLGV, CFLMM;
    /* CONSPARA */
    double DX, DZ, DXI, DZI, DXQI, DZQI;
    /* COORDJR (1-based, index 0 unused) */
    double *YND, *YCC, *DYFI, *DYCI, *WFF, *WFB;
    double Area_inlet, VOLM;
    /* TDMA_COEF */
    double *AMPH, *ACPH, *APPH;
    double *AMVR[4], *ACVR[4], *APVR[4];
    double AMVR1, APVRN;
    /* LAMPOISLPROF */
    double *Vini;
    /* CONS_RKCOEF */
    double TGAM[4], TROH[4], TALP[4];
    /* FFT99_ROOT */
    double *AK1, *AK3;
    /* fields */
    double *Q, *PR, *CONVH0;
    double *QTMP, *DPH, *RHSLLPHI, *RHS;
    /* Poisson spectral work (LH, M, N) */
    double *SRe, *SIm;
    int nthreads;
    int fix_v_wall_row; /* 0: reproduce the reference (default) */
    /* IO (main-domain) path, allocated by orc_io_enable */
    int io;
    double *G, *EXPLT0, *RHO, *MU0, *MU, *DSTG, *MUSTG, *DIVU, *DRHODT;
    double* DEN; /* DENSITY; RHO holds DENSITY0 (equal while the thermal solver is off) */
    int ivis;       /* iVisScheme: 0 explicit (VisExplicit), 1 Crank-Nicolson (VisImplicit) */
    double* DRHOI;  /* DRHOI_STG(:,:,:,1:3) of DENSITY_IMPLICIT_add */
    double CFLMM_IO;
    /* thermal solver (orc_thermal_enable): SOLVERRK3_ENG_io with the table-search properties */
    int thermal;
    void* tab;
    double *DH, *ENTH, *TEMP, *KAPPA, *HCP, *RHSE, *RHSE0, *G0;
    double QW_BOT, QW_TOP, CTHECD, DHMIN, DHMAX;
    /* BC_Fixed_Temperature walls (0 bottom, 1 top): the wall state T, H, D, M, K of T_WAL_GV ...
       (src/Flow_State.f90:186-230), held in the ghost rows (BC_WALL_IsoTHERMAL) */
    int iso[2];
    double WV[2][5];
    int prop_err;
    /* buoyancy (thermal_gravity, src/Flow_State.f90:95-125): iGravity and F_A */
    int igrav;
    double F_A;
    /* iWeightedPre = 1: PR0_io(:,:,:,1:2) (src/FLOWSTART.f90:83-85), NULL when off */
    double *PR0A, *PR0B;
    /* inflow/outflow main domain (iDomain = 3): BC_CONV0 (src/MEMALLOCT.f90:172), the
       FISHPACK x roots -XRT (LPEROD = 4), U_OUTLET and CHK_Mass_CONSV0_SCALING of the last step */
    double *BCCONV0, *AKX;
    double U_OUTLET, MASS_SCALING;
    /* thermal inflow/outflow: BC_CONV0_ENG (src/MEMALLOCT.f90:173) and the inlet state T, H, D, M, K,
       CP, DH of BC_TINLET_THERML (src/Flow_State.f90:44-50) */
    double* BCCONV0E;
    double XIN[7];
    int xin_set;
} orc_t;

#define FOFF(o, i, j, k) ((size_t)((i) - 1 + (o)->xo) + (size_t)(o)->LS * ((size_t)(j) + (size_t)((o)->M + 2) * (size_t)((k) - 1)))
#define FSZ(o) ((size_t)(o)->LS * (size_t)((o)->M + 2) * (size_t)(o)->N)
#define QV(o, i, j, k, c) ((o)->Q[FOFF(o, i, j, k) + (size_t)((c) - 1) * FSZ(o)])
#define F3(a, o, i, j, k) ((a)[FOFF(o, i, j, k)])
#define H0V(o, i, j, k, c) ((o)->CONVH0[FOFF(o, i, j, k) + (size_t)((c) - 1) * FSZ(o)])
#define GV(o, i, j, k, c) ((o)->G[FOFF(o, i, j, k) + (size_t)((c) - 1) * FSZ(o)])
#define E0V(o, i, j, k, c) ((o)->EXPLT0[FOFF(o, i, j, k) + (size_t)((c) - 1) * FSZ(o)])
#define DSV(o, i, j, k, c) ((o)->DSTG[FOFF(o, i, j, k) + (size_t)((c) - 1) * FSZ(o)])
#define MSV(o, i, j, k, c) ((o)->MUSTG[FOFF(o, i, j, k) + (size_t)((c) - 1) * FSZ(o)])

/* IPV_io / IMV_io (src/INDEXSET.f90:26-52): cyclic in x-periodic domains, the ghost columns */
/* 0 and L+1 in the inflow/outflow main domain                                              */
static inline int IPV(const orc_t* o, int i) { return (i == o->L && !o->xo) ? 1 : i + 1; }
static inline int IMV(const orc_t* o, int i) { return (i == 1 && !o->xo) ? o->L : i - 1; }
static inline int KPV(const orc_t* o, int k) { return k == o->N ? 1 : k + 1; }
static inline int KMV(const orc_t* o, int k) { return k == 1 ? o->N : k - 1; }

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

/* ------------------------------------------------------------------ */
/* Complex FFT (mixed radix, recursive).  Unnormalised:                  */
/*   X[k] = sum_j x[j] exp(sign * 2*pi*i*j*k/n).                        */
/* Only the discrete transform has to be reproduced to round-off; the   */
/* Temperton FFT99/CFFT99 factorisation itself is not restated.         */
/* ------------------------------------------------------------------ */
typedef struct { double re, im; } cplx;

static void fft_rec(int n, const cplx* in, int stride, cplx* out, int sign, const cplx* wtab, int wstride) {
    if (n == 1) { out[0] = in[0]; return; }
    int p;
    if (n % 4 == 0 && n > 4) p = 4;
    else if (n % 2 == 0) p = 2;
    else if (n % 3 == 0) p = 3;
    else if (n % 5 == 0) p = 5;
    else p = n;
    int m = n / p;
    if (p == n) {
        /* direct DFT */
        for (int k = 0; k < n; ++k) {
            double sr = 0, si = 0;
            for (int j = 0; j < n; ++j) {
                int e = (int)(((long)j * k) % n);
                cplx w = wtab[(size_t)e * wstride];
                double xr = in[(size_t)j * stride].re, xi = in[(size_t)j * stride].im;
                sr += xr * w.re - xi * w.im;
                si += xr * w.im + xi * w.re;
            }
            out[k].re = sr; out[k].im = si;
        }
        return;
    }
    for (int q = 0; q < p; ++q)
        fft_rec(m, in + (size_t)q * stride, stride * p, out + (size_t)q * m, sign, wtab, wstride * p);
    cplx tmp[8];
    for (int k = 0; k < m; ++k) {
        cplx t[8];
        for (int q = 0; q < p; ++q) {
            cplx a = out[(size_t)q * m + k];
            cplx w = wtab[(size_t)((q * k) % n) * wstride];
            t[q].re = a.re * w.re - a.im * w.im;
            t[q].im = a.re * w.im + a.im * w.re;
        }
        for (int r = 0; r < p; ++r) {
            double sr = 0, si = 0;
            for (int q = 0; q < p; ++q) {
                cplx w = wtab[(size_t)(((q * r * m) % n)) * wstride];
                sr += t[q].re * w.re - t[q].im * w.im;
                si += t[q].re * w.im + t[q].im * w.re;
            }
            tmp[r].re = sr; tmp[r].im = si;
        }
        for (int r = 0; r < p; ++r) out[(size_t)r * m + k] = tmp[r];
    }
}

static cplx* fft_table(int n, int sign) {
    cplx* w = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < n; ++k) {
        long double a = 2.0L * pi * (long double)k / (long double)n;
        w[k].re = (double)cosl(a);
        w[k].im = (double)(sign * sinl(a));
    }
    return w;
}

/* Exported for tests: in-place complex FFT of one line. */
void orc_fft_complex(int n, double* re, double* im, int sign) {
    cplx* in = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    cplx* out = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    cplx* w = fft_table(n, sign);
    for (int j = 0; j < n; ++j) { in[j].re = re[j]; in[j].im = im[j]; }
    fft_rec(n, in, 1, out, sign, w, 1);
    for (int j = 0; j < n; ++j) { re[j] = out[j].re; im[j] = out[j].im; }
    free(in); free(out); free(w);
}

/* ------------------------------------------------------------------ */
/* Setup: CONSPARA (src/CONSPARA.f90:54-73), COORDJR (src/COORDJR.f90:  */
/* 38-145), AREA_INOUTLET (:345-395), MESH_YWEIGHT_FACTORS (:416-442), */
/* TDMA_COEF (src/TDMA_COEF.f90:44-110), LAMPOISLPROF                   */
/* (src/LAMPOISLPROF.f90:17-60), CONS_RKCOEF (src/CONS_RKCOEF.f90:     */
/* 25-51), FFT99_ROOT (src/possion3d_FFT99.f90:140-202).                */
/* ------------------------------------------------------------------ */
static void setup(orc_t* o) {
    int L = o->L, M = o->M, N = o->N, NND2 = M + 1;
    const double PI = 2.0 * asin(1.0);
    /* CONSPARA */
    o->DX = o->HX / (double)L;
    o->DXI = 1.0 / o->DX;
    o->DXQI = o->DXI * o->DXI;
    o->DZ = o->HZ / (double)N;
    o->DZI = 1.0 / o->DZ;
    o->DZQI = o->DZI * o->DZI;
    o->CVISC = 1.0 / o->REN;
    /* COORDJR, channel */
    double COE1 = 0.5;
    for (int J = 1; J <= NND2; ++J) {
        double X2 = (double)(J - 1) / (double)(NND2 - 1);
        o->YND[J] = tanh(o->STR2 * (X2 - COE1)) / tanh(o->STR2 * COE1);
    }
    for (int J = 1; J <= M; ++J) o->YCC[J] = (o->YND[J] + o->YND[J + 1]) * 0.5;
    for (int J = 1; J <= M; ++J) o->DYFI[J] = 1.0 / (o->YND[J + 1] - o->YND[J]);
    for (int J = 2; J <= NND2 - 1; ++J) o->DYCI[J] = 1.0 / ((o->YND[J + 1] - o->YND[J - 1]) * 0.5);
    o->DYCI[1] = 2.0 / (o->YND[2] - o->YND[1]);
    o->DYCI[NND2] = 2.0 / (o->YND[NND2] - o->YND[M]);
    /* AREA_INOUTLET (RCCI1 = 1 for the channel) */
    o->Area_inlet = 0.0;
    for (int JC = 1; JC <= M; ++JC)
        for (int KC = 1; KC <= N; ++KC) o->Area_inlet = o->Area_inlet + 1.0 / 1.0 / o->DYFI[JC] / o->DZI;
    o->VOLM = 0.0;
    for (int KC = 1; KC <= N; ++KC)
        for (int JC = 1; JC <= M; ++JC)
            for (int IC = 1; IC <= L; ++IC) o->VOLM = o->VOLM + 1.0 / 1.0 / o->DYFI[JC];
    /* MESH_YWEIGHT_FACTORS */
    for (int JC = 2; JC <= M; ++JC) {
        int JM = JC - 1;
        o->WFF[JC] = (o->YND[JC] - o->YCC[JM]) / (o->YCC[JC] - o->YCC[JM]);
        o->WFB[JC] = (o->YCC[JC] - o->YND[JC]) / (o->YCC[JC] - o->YCC[JM]);
    }
    o->WFB[1] = 1.0; o->WFF[1] = 0.0;
    o->WFB[NND2] = 0.0; o->WFF[NND2] = 1.0;
    /* TDMA_COEF, channel */
    for (int JC = 1; JC <= M; ++JC) {
        int JP = JC + 1;
        o->AMPH[JC] = o->DYFI[JC] * o->DYCI[JC];
        o->APPH[JC] = o->DYFI[JC] * o->DYCI[JP];
        if (JC == 1) o->AMPH[JC] = o->DYFI[JC] * o->DYCI[JC] * 0.5;
        if (JP == NND2) o->APPH[JC] = o->DYFI[JC] * o->DYCI[JP] * 0.5;
    }
    for (int JC = 1; JC <= M; ++JC) o->ACPH[JC] = -(o->AMPH[JC] + o->APPH[JC]);
    o->ACPH[1] = o->AMPH[1] + o->ACPH[1];
    o->AMPH[1] = 0.0;
    o->ACPH[M] = o->APPH[M] + o->ACPH[M];
    o->APPH[M] = 0.0;
    for (int IDR = 1; IDR <= 3; ++IDR) {
        double *AM = o->AMVR[IDR], *AC = o->ACVR[IDR], *AP = o->APVR[IDR];
        if (IDR == 1 || IDR == 3) {
            for (int JC = 2; JC <= M - 1; ++JC) {
                int JP = JC + 1;
                AM[JC] = o->DYFI[JC] * o->DYCI[JC];
                AP[JC] = o->DYFI[JC] * o->DYCI[JP];
                AC[JC] = -(AM[JC] + AP[JC]);
            }
            double UCAJ = 4.0 / (2.0 / o->DYCI[2] + 1.0 / o->DYFI[1]);
            AM[1] = 0.0;
            AP[1] = UCAJ * o->DYCI[2];
            AC[1] = -UCAJ * (o->DYCI[2] + 2.0 * o->DYFI[1]);
            o->AMVR1 = UCAJ * (2.0 * o->DYFI[1]);
            UCAJ = 4.0 / (2.0 / o->DYCI[M] + 1.0 / o->DYFI[M]);
            AM[M] = UCAJ * o->DYCI[M];
            AP[M] = 0.0;
            AC[M] = -UCAJ * (2.0 * o->DYFI[M] + o->DYCI[M]);
            o->APVRN = UCAJ * (2.0 * o->DYFI[M]);
        } else {
            for (int JC = 2; JC <= M; ++JC) {
                int JM = JC - 1;
                AM[JC] = o->DYFI[JM] * o->DYCI[JC];
                AP[JC] = o->DYFI[JC] * o->DYCI[JC];
                AC[JC] = -(AM[JC] + AP[JC]);
            }
            AM[1] = 0.0; AP[1] = 0.0; AC[1] = 1.0;
            AM[NND2] = 0.0; AP[NND2] = 0.0; AC[NND2] = 1.0;
        }
    }
    /* LAMPOISLPROF, channel: a = 1, b = 0, PCOE = 3/2 */
    {
        double Y1 = -1.0, Y2 = 1.0, a = (1.0 - (-1.0)) / 2.0, b = 0.0, PCOE = 3.0 / 2.0;
        for (int J = 1; J <= M; ++J) {
            if (o->YCC[J] < Y2 && o->YCC[J] > Y1)
                o->Vini[J] = (1.0 - ((o->YCC[J] - b) * (o->YCC[J] - b)) / a / a) * PCOE;
            else
                o->Vini[J] = 0.0;
        }
    }
    /* CONS_RKCOEF */
    o->TGAM[0] = 1.0; o->TGAM[1] = 8.0 / 15.0; o->TGAM[2] = 5.0 / 12.0; o->TGAM[3] = 3.0 / 4.0;
    o->TROH[0] = 0.0; o->TROH[1] = 0.0; o->TROH[2] = -17.0 / 60.0; o->TROH[3] = -5.0 / 12.0;
    for (int s = 0; s < 4; ++s) o->TALP[s] = o->TGAM[s] + o->TROH[s];
    /* FFT99_ROOT modified wavenumbers */
    {
        int N1MH = L / 2, N3MH = N / 2, N1MP = N1MH + 1, N3MP = N3MH + 1;
        for (int K = 1; K <= N; ++K) {
            double AN = (K <= N3MH) ? (double)(K - 1) * 2.0 * PI : -(double)(N - K + 1) * 2.0 * PI;
            (void)N3MP;
            o->AK3[K] = 2.0 * (1.0 - cos(AN / (double)N)) * o->DZQI;
        }
        for (int I = 1; I <= L; ++I) {
            double AP = (I <= N1MH) ? (double)(I - 1) * 2.0 * PI : -(double)(L - I + 1) * 2.0 * PI;
            (void)N1MP;
            o->AK1[I] = 2.0 * (1.0 - cos(AP / (double)L)) * o->DXQI;
        }
    }
}

static orc_t* create_impl(int L, int M, int N, double HX, double HZ, double STR2, double REN, int iFlowDriven,
                          double Cf_Given, double DT0, double DTMIN, double CFLGV, int xo) {
    if (L < 4 || M < 4 || N < 4 || (L % 2) || (N % 2)) return NULL;
    orc_t* o = (orc_t*)calloc(1, sizeof(orc_t));
    o->L = L; o->M = M; o->N = N; o->NND2 = M + 1;
    o->xo = xo; o->LS = L + 2 * xo;
    o->HX = HX; o->HZ = HZ; o->STR2 = STR2; o->REN = REN;
    o->iFlowDriven = iFlowDriven; o->Cf_Given = Cf_Given;
    o->DT0 = DT0; o->DT = DT0; o->DTMIN = DTMIN; o->CFLGV = CFLGV;
    o->nthreads = 1;
    size_t ny = (size_t)M + 3;
    o->YND = dalloc(ny); o->YCC = dalloc(ny); o->DYFI = dalloc(ny); o->DYCI = dalloc(ny);
    o->WFF = dalloc(ny); o->WFB = dalloc(ny);
    o->AMPH = dalloc(ny); o->ACPH = dalloc(ny); o->APPH = dalloc(ny);
    for (int c = 1; c <= 3; ++c) { o->AMVR[c] = dalloc(ny); o->ACVR[c] = dalloc(ny); o->APVR[c] = dalloc(ny); }
    o->Vini = dalloc(ny);
    o->AK1 = dalloc((size_t)L + 1); o->AK3 = dalloc((size_t)N + 1);
    size_t fs = FSZ(o);
    o->Q = dalloc(3 * fs); o->PR = dalloc(fs); o->CONVH0 = dalloc(3 * fs);
    o->QTMP = dalloc(fs); o->DPH = dalloc(fs); o->RHSLLPHI = dalloc(fs); o->RHS = dalloc(fs);
    size_t LH = xo ? (size_t)L : (size_t)L / 2 + 1;  /* the cosine transform keeps L x modes */
    o->SRe = dalloc(LH * (size_t)M * (size_t)N); o->SIm = dalloc(LH * (size_t)M * (size_t)N);
    setup(o);
    if (xo) {
        /* FFTPACK_ROOT with LP = 5 (src/possion3d_fishpack.f90:65-111): XRT(I) =                  */
        /* -4 DXQI sin^2((I - 1/2) pi / (2 L)); AKX holds -XRT (the AK1 of the cosine modes)      */
        double PI = 2.0 * asin(1.0), DX = PI / (2.0 * (double)L);
        o->AKX = dalloc((size_t)L + 1);
        for (int I = 1; I <= L; ++I) {
            double sn = sin(((double)I - 0.5) * DX);
            o->AKX[I] = 4.0 * o->DXQI * (sn * sn);
        }
        o->BCCONV0 = dalloc(3 * (size_t)M * (size_t)N);
        o->BCCONV0E = dalloc((size_t)M * (size_t)N);
    }
    return o;
}

orc_t* orc_create(int L, int M, int N, double HX, double HZ, double STR2, double REN, int iFlowDriven,
                  double Cf_Given, double DT0, double DTMIN, double CFLGV) {
    return create_impl(L, M, N, HX, HZ, STR2, REN, iFlowDriven, Cf_Given, DT0, DTMIN, CFLGV, 0);
}

/* The main domain of iDomain = 3 (TgFlowFlg and IoFlowFlg): x runs over NCL1S:NCL1E = 0:L+1 with */
/* the inlet ghost column 0 fed by a periodic TG domain and the convective outlet column L+1.     */
orc_t* orc_create_xinout(int L, int M, int N, double HX, double HZ, double STR2, double REN, double DT0,
                         double DTMIN, double CFLGV) {
    return create_impl(L, M, N, HX, HZ, STR2, REN, 0, 0.0, DT0, DTMIN, CFLGV, 1);
}

void orc_destroy(orc_t* o) {
    if (!o) return;
    free(o->YND); free(o->YCC); free(o->DYFI); free(o->DYCI); free(o->WFF); free(o->WFB);
    free(o->AMPH); free(o->ACPH); free(o->APPH);
    for (int c = 1; c <= 3; ++c) { free(o->AMVR[c]); free(o->ACVR[c]); free(o->APVR[c]); }
    free(o->Vini); free(o->AK1); free(o->AK3);
    free(o->Q); free(o->PR); free(o->CONVH0); free(o->QTMP); free(o->DPH); free(o->RHSLLPHI); free(o->RHS);
    free(o->SRe); free(o->SIm);
    free(o->PR0A); free(o->PR0B);
    free(o->G); free(o->EXPLT0); free(o->RHO); free(o->MU0); free(o->MU); free(o->DSTG); free(o->MUSTG);
    free(o->DIVU); free(o->DRHODT); free(o->DEN); free(o->DRHOI);
    free(o->DH); free(o->ENTH); free(o->TEMP); free(o->KAPPA); free(o->HCP); free(o->RHSE); free(o->RHSE0); free(o->G0);
    free(o->BCCONV0); free(o->AKX); free(o->BCCONV0E);
    free(o);
}

void orc_set_threads(orc_t* o, int n) {
    o->nthreads = n < 1 ? 1 : n;
#ifdef _OPENMP
    omp_set_num_threads(o->nthreads);
#endif
}
void orc_set_fix_v_wall_row(orc_t* o, int f) { o->fix_v_wall_row = f; }

/* Setup export.  y-arrays are written 1-based into out[0..]: out[j-1] = A(j). */
void orc_get_y(const orc_t* o, int which, int idr, double* out) {
    int M = o->M, n = (which == 0 || which == 3 || which == 4 || which == 5) ? M + 1 : M;
    const double* a = NULL;
    switch (which) {
        case 0: a = o->YND; break;
        case 1: a = o->YCC; break;
        case 2: a = o->DYFI; break;
        case 3: a = o->DYCI; break;
        case 4: a = o->WFF; break;
        case 5: a = o->WFB; break;
        case 6: a = o->AMPH; break;
        case 7: a = o->ACPH; break;
        case 8: a = o->APPH; break;
        case 9: a = o->AMVR[idr]; n = M + 1; break;
        case 10: a = o->ACVR[idr]; n = M + 1; break;
        case 11: a = o->APVR[idr]; n = M + 1; break;
        case 12: a = o->Vini; break;
        default: return;
    }
    for (int j = 1; j <= n; ++j) out[j - 1] = a[j];
}
/* scalars: DX, DZ, DXI, DZI, DXQI, DZQI, VOLM, Area_inlet, AMVR1, APVRN, CVISC, DT */
void orc_get_scalars(const orc_t* o, double* s) {
    s[0] = o->DX; s[1] = o->DZ; s[2] = o->DXI; s[3] = o->DZI; s[4] = o->DXQI; s[5] = o->DZQI;
    s[6] = o->VOLM; s[7] = o->Area_inlet; s[8] = o->AMVR1; s[9] = o->APVRN; s[10] = o->CVISC; s[11] = o->DT;
}

void orc_set_fields(orc_t* o, const double* Q, const double* PR, const double* H0) {
    size_t fs = FSZ(o);
    if (Q) memcpy(o->Q, Q, 3 * fs * sizeof(double));
    if (PR) memcpy(o->PR, PR, fs * sizeof(double));
    if (H0) memcpy(o->CONVH0, H0, 3 * fs * sizeof(double));
    else memset(o->CONVH0, 0, 3 * fs * sizeof(double));
}
void orc_get_fields(const orc_t* o, double* Q, double* PR, double* H0) {
    size_t fs = FSZ(o);
    if (Q) memcpy(Q, o->Q, 3 * fs * sizeof(double));
    if (PR) memcpy(PR, o->PR, fs * sizeof(double));
    if (H0) memcpy(H0, o->CONVH0, 3 * fs * sizeof(double));
}
void orc_get_work(const orc_t* o, int which, double* out) {
    size_t fs = FSZ(o);
    const double* a = which == 0 ? o->DPH : which == 1 ? o->RHSLLPHI : which == 2 ? o->RHS : o->QTMP;
    memcpy(out, a, fs * sizeof(double));
}
void orc_set_dt(orc_t* o, double dt) { o->DT = dt; }
double orc_get_dt(const orc_t* o) { return o->DT; }

/* ------------------------------------------------------------------ */
/* Line solvers                                                         */
/* ------------------------------------------------------------------ */
/* TDMAIJI_CYC (src/TDMAIJI_CYC.f90:67-157), one line of length n with  */
/* coefficient arrays a, b, c and rhs r (0-based); w is scratch 3*n.    */
static void tdma_cyc_line(int n, const double* A, const double* B, const double* C, double* R, double* w) {
    double *H0 = w, *G1 = w + n, *G2 = w + 2 * n;
    int IS = 0, IEND = n - 1;
    H0[IS] = C[IS] / B[IS];
    G1[IS] = R[IS] / B[IS];
    G2[IS] = -A[IS] / B[IS];
    for (int I = IS + 1; I <= IEND - 2; ++I) {
        double PP = 1.0 / (B[I] - H0[I - 1] * A[I]);
        double QQ1 = G1[I - 1] * A[I];
        double QQ2 = G2[I - 1] * A[I];
        H0[I] = C[I] * PP;
        G1[I] = (R[I] - QQ1) * PP;
        G2[I] = -QQ2 * PP;
    }
    {
        int I = IEND - 1;
        double PP = 1.0 / (B[I] - H0[I - 1] * A[I]);
        double QQ1 = G1[I - 1] * A[I];
        double QQ2 = G2[I - 1] * A[I];
        G1[I] = (R[I] - QQ1) * PP;
        G2[I] = (-C[I] - QQ2) * PP;
    }
    for (int I = IEND - 2; I >= IS; --I) {
        G1[I] = -H0[I] * G1[I + 1] + G1[I];
        G2[I] = -H0[I] * G2[I + 1] + G2[I];
    }
    {
        int I = IEND;
        double PP = R[I] - C[I] * G1[IS] - A[I] * G1[I - 1];
        double QQ1 = B[I] + C[I] * G2[IS] + A[I] * G2[I - 1];
        R[I] = PP / QQ1;
    }
    for (int I = IEND - 1; I >= IS; --I) R[I] = G1[I] + G2[I] * R[IEND];
}

/* TDMAIJJ_nonCYC (src/TDMAIJJ_nonCYC.f90:67-123), zero Dirichlet BC.  */
static void tdma_noncyc_line(int n, const double* A, const double* B, const double* C, double* R, double* w) {
    double *H = w, *G = w + n;
    const double BC1 = 0.0, BC2 = 0.0;
    H[0] = C[0] / B[0];
    G[0] = (R[0] - A[0] * BC1) / B[0];
    for (int J = 1; J <= n - 2; ++J) {
        double PP = 1.0 / (B[J] - H[J - 1] * A[J]);
        H[J] = C[J] * PP;
        G[J] = (R[J] - A[J] * G[J - 1]) * PP;
    }
    {
        int J = n - 1;
        double PP = 1.0 / (B[J] - H[J - 1] * A[J]);
        G[J] = (R[J] - C[J] * BC2 - A[J] * G[J - 1]) * PP;
        R[J] = G[J];
    }
    for (int J = n - 2; J >= 0; --J) R[J] = G[J] - H[J] * R[J + 1];
}

/* Exported single-line solvers for unit tests. */
void orc_tdma_cyc(int n, const double* A, const double* B, const double* C, double* R) {
    double* w = dalloc(3 * (size_t)n);
    tdma_cyc_line(n, A, B, C, R, w);
    free(w);
}
void orc_tdma_noncyc(int n, const double* A, const double* B, const double* C, double* R) {
    double* w = dalloc(2 * (size_t)n);
    tdma_noncyc_line(n, A, B, C, R, w);
    free(w);
}

/* ------------------------------------------------------------------ */
/* CONVECTION_X_tg (src/CONVECTION_X.f90:13-64)                        */
/* ------------------------------------------------------------------ */
static void convection_x(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    const double XND2CL = 0.5, ZND2CL = 0.5;
    memset(o->QTMP, 0, FSZ(o) * sizeof(double));
    double COE1 = XND2CL * XND2CL * o->DXI;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * XND2CL * 1.0;
        double COE3 = XND2CL * ZND2CL * o->DZI * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double H11 = ((QV(o, IP, JC, KC, 1) + QV(o, IC, JC, KC, 1)) * (QV(o, IP, JC, KC, 1) + QV(o, IC, JC, KC, 1)) -
                              (QV(o, IM, JC, KC, 1) + QV(o, IC, JC, KC, 1)) * (QV(o, IM, JC, KC, 1) + QV(o, IC, JC, KC, 1))) * COE1;
                double H12 = ((QV(o, IC, JP, KC, 2) + QV(o, IM, JP, KC, 2)) *
                                  (o->WFF[JJP] * QV(o, IC, JP, KC, 1) + o->WFB[JJP] * QV(o, IC, JC, KC, 1)) -
                              (QV(o, IC, JC, KC, 2) + QV(o, IM, JC, KC, 2)) *
                                  (o->WFF[JJ] * QV(o, IC, JC, KC, 1) + o->WFB[JJ] * QV(o, IC, JM, KC, 1))) * COE2;
                double H13 = ((QV(o, IC, JC, KP, 3) + QV(o, IM, JC, KP, 3)) * (QV(o, IC, JC, KP, 1) + QV(o, IC, JC, KC, 1)) -
                              (QV(o, IC, JC, KC, 3) + QV(o, IM, JC, KC, 3)) * (QV(o, IC, JC, KC, 1) + QV(o, IC, JC, KM, 1))) * COE3;
                F3(o->QTMP, o, IC, JC, KC) = -(H11 + H12 + H13);
            }
        }
    }
}

/* CONVECTION_Y_tg (src/CONVECTION_Y.f90:13-114), channel branch.  The  */
/* v-equation skips the wall face j = 1 (NYI = 2).                      */
static void convection_y(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    const double XND2CL = 0.5, YND2CL = 0.5, ZND2CL = 0.5;
    memset(o->DPH, 0, FSZ(o) * sizeof(double));
    double COE1 = o->DXI * XND2CL;
    double COE30 = o->DZI * ZND2CL;
#pragma omp parallel for schedule(static)
    for (int JC = 2; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC;
        double COE2 = o->DYCI[JJ] * YND2CL * YND2CL;
        double COE31 = COE30 * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double H21 = ((o->WFF[JJ] * QV(o, IP, JC, KC, 1) + o->WFB[JJ] * QV(o, IP, JM, KC, 1)) *
                                  (QV(o, IP, JC, KC, 2) + QV(o, IC, JC, KC, 2)) -
                              (o->WFF[JJ] * QV(o, IC, JC, KC, 1) + o->WFB[JJ] * QV(o, IC, JM, KC, 1)) *
                                  (QV(o, IC, JC, KC, 2) + QV(o, IM, JC, KC, 2))) * COE1;
                double H22 = ((QV(o, IC, JP, KC, 2) * 1.0 + QV(o, IC, JC, KC, 2) * 1.0) * (QV(o, IC, JP, KC, 2) + QV(o, IC, JC, KC, 2)) -
                              (QV(o, IC, JC, KC, 2) * 1.0 + QV(o, IC, JM, KC, 2) * 1.0) * (QV(o, IC, JC, KC, 2) + QV(o, IC, JM, KC, 2))) * COE2;
                double H23 = ((o->WFF[JJ] * QV(o, IC, JC, KP, 3) * 1.0 + o->WFB[JJ] * QV(o, IC, JM, KP, 3) * 1.0) *
                                  (QV(o, IC, JC, KP, 2) + QV(o, IC, JC, KC, 2)) -
                              (o->WFF[JJ] * QV(o, IC, JC, KC, 3) * 1.0 + o->WFB[JJ] * QV(o, IC, JM, KC, 3) * 1.0) *
                                  (QV(o, IC, JC, KC, 2) + QV(o, IC, JC, KM, 2))) * COE31;
                F3(o->DPH, o, IC, JC, KC) = -(H21 + H22 + H23);
            }
        }
    }
}

/* CONVECTION_Z_tg (src/CONVECTION_Z.f90:13-103), channel branch.       */
static void convection_z(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    const double XND2CL = 0.5, ZND2CL = 0.5;
    memset(o->RHSLLPHI, 0, FSZ(o) * sizeof(double));
    double COE1 = XND2CL * ZND2CL * o->DXI;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * ZND2CL;
        double COE3 = ZND2CL * ZND2CL * o->DZI * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double H31 = ((QV(o, IP, JC, KC, 1) + QV(o, IP, JC, KM, 1)) * (QV(o, IP, JC, KC, 3) + QV(o, IC, JC, KC, 3)) -
                              (QV(o, IC, JC, KC, 1) + QV(o, IC, JC, KM, 1)) * (QV(o, IC, JC, KC, 3) + QV(o, IM, JC, KC, 3))) * COE1;
                double H32 = ((QV(o, IC, JP, KC, 2) + QV(o, IC, JP, KM, 2)) *
                                  (o->WFF[JJP] * QV(o, IC, JP, KC, 3) * 1.0 + o->WFB[JJP] * QV(o, IC, JC, KC, 3) * 1.0) -
                              (QV(o, IC, JC, KC, 2) + QV(o, IC, JC, KM, 2)) *
                                  (o->WFF[JJ] * QV(o, IC, JC, KC, 3) * 1.0 + o->WFB[JJ] * QV(o, IC, JM, KC, 3) * 1.0)) * COE2;
                double H33 = ((QV(o, IC, JC, KP, 3) + QV(o, IC, JC, KC, 3)) * (QV(o, IC, JC, KP, 3) + QV(o, IC, JC, KC, 3)) -
                              (QV(o, IC, JC, KC, 3) + QV(o, IC, JC, KM, 3)) * (QV(o, IC, JC, KC, 3) + QV(o, IC, JC, KM, 3))) * COE3;
                F3(o->RHSLLPHI, o, IC, JC, KC) = -(H31 + H32 + H33);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* RHS_CvLpGpS_tg (src/RHS_CvLpGpS_tg.f90:12-204).  RHS rows j < NII     */
/* are left untouched, exactly as in the reference (the module array    */
/* keeps its previous contents there).                                  */
/* ------------------------------------------------------------------ */
static void rhs_cvlpgps(orc_t* o, int NS, int IDR) {
    int L = o->L, M = o->M, N = o->N;
    int NII = (IDR == 2) ? 2 : 1;
    const double* CONVH = IDR == 1 ? o->QTMP : IDR == 2 ? o->DPH : o->RHSLLPHI;
    const double RMC2 = 1.0; /* RCCI2 / RNDI2 = 1 in the channel */
    double COE1 = o->TALP[NS] * o->CVISC * 1.0 / 1.0;
    double DT = o->DT;
    const double *APVR = o->APVR[IDR], *ACVR = o->ACVR[IDR], *AMVR = o->AMVR[IDR];
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC) {
        int KM = KMV(o, KC), KP = KPV(o, KC);
        for (int JC = NII; JC <= M; ++JC) {
            int JM = JC - 1, JP = JC + 1, JJ = JC;
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double CV = F3(CONVH, o, IC, JC, KC);
                double RHSC = o->TGAM[NS] * CV + o->TROH[NS] * H0V(o, IC, JC, KC, IDR);
                double RHSL = COE1 * ((QV(o, IP, JC, KC, IDR) - 2.0 * QV(o, IC, JC, KC, IDR) + QV(o, IM, JC, KC, IDR)) * o->DXQI +
                                      (QV(o, IC, JC, KP, IDR) - 2.0 * QV(o, IC, JC, KC, IDR) + QV(o, IC, JC, KM, IDR)) * o->DZQI * RMC2 +
                                      (QV(o, IC, JP, KC, IDR) * APVR[JJ] + QV(o, IC, JC, KC, IDR) * ACVR[JJ] +
                                       QV(o, IC, JM, KC, IDR) * AMVR[JJ]));
                H0V(o, IC, JC, KC, IDR) = CV;
                F3(o->RHS, o, IC, JC, KC) = (RHSC + RHSL) * DT;
            }
        }
    }
    double COE2 = o->TALP[NS] * DT / 1.0;
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC) {
        int KM = KMV(o, KC);
        for (int JC = NII; JC <= M; ++JC) {
            int JM = JC - 1, JJ = JC;
            double SUCACJ = o->DYCI[JJ] / 1.0;
            for (int IC = 1; IC <= L; ++IC) {
                int IM = IMV(o, IC);
                double PGM;
                if (IDR == 1) PGM = (F3(o->PR, o, IC, JC, KC) - F3(o->PR, o, IM, JC, KC)) * o->DXI * COE2;
                else if (IDR == 2) PGM = (F3(o->PR, o, IC, JC, KC) - F3(o->PR, o, IC, JM, KC)) * SUCACJ * COE2;
                else PGM = (F3(o->PR, o, IC, JC, KC) - F3(o->PR, o, IC, JC, KM)) * o->DZI * COE2;
                F3(o->RHS, o, IC, JC, KC) = F3(o->RHS, o, IC, JC, KC) - PGM;
            }
        }
    }
    if (IDR == 1) {
        double DPGRNS = 0.0;
        if (o->iFlowDriven == 1) {
            /* naive sum in the reference's loop order: IC, JC, KC */
            double INTGRHSY = 0.0;
            for (int IC = 1; IC <= L; ++IC)
                for (int JC = 1; JC <= M; ++JC)
                    for (int KC = 1; KC <= N; ++KC)
                        INTGRHSY = INTGRHSY + F3(o->RHS, o, IC, JC, KC) / o->DYFI[JC] / 1.0;
            DPGRNS = INTGRHSY / o->VOLM;
        } else if (o->iFlowDriven == 2) {
            DPGRNS = -0.5 * o->Cf_Given * COE2;
        }
#pragma omp parallel for schedule(static)
        for (int K = 1; K <= N; ++K)
            for (int J = NII; J <= M; ++J)
                for (int I = 1; I <= L; ++I) F3(o->RHS, o, I, J, K) = F3(o->RHS, o, I, J, K) - DPGRNS;
    }
}

/* MOMFA_tg + MOMFA1_X_tg + MOMFA2_Z_tg + MOMFA3_Y_tg                   */
/* (src/MOMFA_tg.f90:15-238).                                           */
static void momfa(orc_t* o, int NS, int IDR) {
    int L = o->L, M = o->M, N = o->N;
    double FACOE = 0.5 * o->TALP[NS] * o->DT * o->CVISC * 1.0 / 1.0;
    int N2I = (IDR == 2) ? 2 : 1;
    /* x sweep: cyclic, constant coefficients */
    {
        double COE = -FACOE * o->DXQI;
#pragma omp parallel
        {
            double* A = dalloc((size_t)L); double* B = dalloc((size_t)L); double* C = dalloc((size_t)L);
            double* R = dalloc((size_t)L); double* w = dalloc(3 * (size_t)L);
#pragma omp for schedule(static)
            for (int K = 1; K <= N; ++K)
                for (int J = N2I; J <= M; ++J) {
                    for (int I = 1; I <= L; ++I) {
                        C[I - 1] = COE; A[I - 1] = COE; B[I - 1] = 1.0 - C[I - 1] - A[I - 1];
                        R[I - 1] = F3(o->RHS, o, I, J, K);
                    }
                    tdma_cyc_line(L, A, B, C, R, w);
                    for (int I = 1; I <= L; ++I) F3(o->RHS, o, I, J, K) = R[I - 1];
                }
            free(A); free(B); free(C); free(R); free(w);
        }
    }
    /* z sweep: cyclic, constant coefficients */
    {
        double RMC2 = 1.0 * (-FACOE * o->DZQI);
#pragma omp parallel
        {
            double* A = dalloc((size_t)N); double* B = dalloc((size_t)N); double* C = dalloc((size_t)N);
            double* R = dalloc((size_t)N); double* w = dalloc(3 * (size_t)N);
#pragma omp for schedule(static)
            for (int I = 1; I <= L; ++I)
                for (int J = N2I; J <= M; ++J) {
                    for (int K = 1; K <= N; ++K) {
                        C[K - 1] = RMC2; A[K - 1] = RMC2; B[K - 1] = 1.0 - C[K - 1] - A[K - 1];
                        R[K - 1] = F3(o->RHS, o, I, J, K);
                    }
                    tdma_cyc_line(N, A, B, C, R, w);
                    for (int K = 1; K <= N; ++K) F3(o->RHS, o, I, J, K) = R[K - 1];
                }
            free(A); free(B); free(C); free(R); free(w);
        }
    }
    /* y sweep: non-cyclic over J = 1..M for every component */
    {
        const double *AMVR = o->AMVR[IDR], *ACVR = o->ACVR[IDR], *APVR = o->APVR[IDR];
#pragma omp parallel
        {
            double* A = dalloc((size_t)M); double* B = dalloc((size_t)M); double* C = dalloc((size_t)M);
            double* R = dalloc((size_t)M); double* w = dalloc(2 * (size_t)M);
#pragma omp for schedule(static)
            for (int K = 1; K <= N; ++K)
                for (int I = 1; I <= L; ++I) {
                    for (int J = 1; J <= M; ++J) {
                        R[J - 1] = F3(o->RHS, o, I, J, K);
                        B[J - 1] = 1.0 - FACOE * ACVR[J];
                        C[J - 1] = -FACOE * APVR[J];
                        A[J - 1] = -FACOE * AMVR[J];
                    }
                    if (IDR == 2 && o->fix_v_wall_row) R[0] = 0.0;
                    tdma_noncyc_line(M, A, B, C, R, w);
                    for (int J = 1; J <= M; ++J) F3(o->RHS, o, I, J, K) = R[J - 1];
                }
            free(A); free(B); free(C); free(R); free(w);
        }
    }
#pragma omp parallel for schedule(static)
    for (int K = 1; K <= N; ++K)
        for (int J = N2I; J <= M; ++J)
            for (int I = 1; I <= L; ++I) QV(o, I, J, K, IDR) = F3(o->RHS, o, I, J, K) + QV(o, I, J, K, IDR);
}

/* BC_WALL_Q_tg / BC_WALL_PR_tg / BC_WALL_DPH_tg (src/BC_WALL.f90:212-432) */
static void bc_wall_q(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    for (int K = 1; K <= N; ++K)
        for (int I = 1 - o->xo; I <= L + o->xo; ++I) {
            QV(o, I, M + 1, K, 1) = 0.0; QV(o, I, M + 1, K, 3) = 0.0; QV(o, I, M + 1, K, 2) = 0.0;
            QV(o, I, 0, K, 1) = 0.0; QV(o, I, 0, K, 3) = 0.0; QV(o, I, 1, K, 2) = 0.0; QV(o, I, 0, K, 2) = 0.0;
        }
}
static void bc_wall_scalar(orc_t* o, double* F) {
    int L = o->L, M = o->M, N = o->N;
    for (int K = 1; K <= N; ++K)
        for (int I = 1 - o->xo; I <= L + o->xo; ++I) {
            F3(F, o, I, M + 1, K) = F3(F, o, I, M, K);
            F3(F, o, I, 0, K) = F3(F, o, I, 1, K);
        }
}

/* DIVG_tg (src/DIVG.f90:15-51) */
static void divg(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
    double COE0 = 1.0 / (o->DT * o->TALP[NS]);
    memset(o->RHSLLPHI, 0, FSZ(o) * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JP = JC + 1, JJ = JC;
        double COE1 = o->DXI / 1.0;
        double COE2 = o->DYFI[JJ] / 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC);
                double DV = (QV(o, IP, JC, KC, 1) - QV(o, IC, JC, KC, 1)) * COE1 + (QV(o, IC, JP, KC, 2) - QV(o, IC, JC, KC, 2)) * COE2 +
                            (QV(o, IC, JC, KP, 3) - QV(o, IC, JC, KC, 3)) * o->DZI;
                F3(o->RHSLLPHI, o, IC, JC, KC) = DV * COE0;
            }
        }
    }
}

/* FFT99_POIS3D_periodicxz (src/possion3d_FFT99.f90:271-505) with the    */
/* coefficients of TDMA_PHI_COEF (:204-239).  Forward: x transform with */
/* 1/L (FFT99, ISIGN=-1), z transform (CFFT99, ISIGN=-1) times 1/N.     */
/* Zero mode: RHS(1,1,1) = 0 and row 1 decoupled (phi(y_1) = 0).        */
/* src: (L, 0:M+1, N) field; dst: (L, 0:M+1, N) field (rows 1..M).       */
static void poisson(orc_t* o, const double* src, double* dst) {
    int L = o->L, M = o->M, N = o->N, LH = L / 2 + 1;
    double UN3M = 1.0 / (double)N;
    cplx* wfx = fft_table(L, -1);
    cplx* wbx = fft_table(L, +1);
    cplx* wfz = fft_table(N, -1);
    cplx* wbz = fft_table(N, +1);
    double* SRe = o->SRe;
    double* SIm = o->SIm;
#define SIX(I, J, K) ((size_t)((I) - 1) + (size_t)LH * ((size_t)((J) - 1) + (size_t)M * (size_t)((K) - 1)))
#pragma omp parallel
    {
        int nmax = L > N ? L : N;
        cplx* a = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
        cplx* b = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for schedule(static)
        for (int J = 1; J <= M; ++J) {
            for (int K = 1; K <= N; ++K) {
                for (int I = 1; I <= L; ++I) { a[I - 1].re = F3(src, o, I, J, K); a[I - 1].im = 0.0; }
                fft_rec(L, a, 1, b, -1, wfx, 1);
                for (int I = 1; I <= LH; ++I) {
                    SRe[SIX(I, J, K)] = b[I - 1].re / (double)L;
                    SIm[SIX(I, J, K)] = b[I - 1].im / (double)L;
                }
            }
            for (int I = 1; I <= LH; ++I) {
                for (int K = 1; K <= N; ++K) { a[K - 1].re = SRe[SIX(I, J, K)]; a[K - 1].im = SIm[SIX(I, J, K)]; }
                fft_rec(N, a, 1, b, -1, wfz, 1);
                for (int K = 1; K <= N; ++K) {
                    SRe[SIX(I, J, K)] = b[K - 1].re * UN3M;
                    SIm[SIX(I, J, K)] = b[K - 1].im * UN3M;
                }
            }
        }
        free(a); free(b);
    }
    SRe[SIX(1, 1, 1)] = 0.0;
    SIm[SIX(1, 1, 1)] = 0.0;
#pragma omp parallel
    {
        double* A = dalloc((size_t)M); double* B = dalloc((size_t)M); double* C = dalloc((size_t)M);
        double* R = dalloc((size_t)M); double* w = dalloc(2 * (size_t)M);
#pragma omp for schedule(static)
        for (int K = 1; K <= N; ++K)
            for (int I = 1; I <= LH; ++I) {
                for (int J = 1; J <= M; ++J) {
                    C[J - 1] = o->APPH[J];
                    A[J - 1] = o->AMPH[J];
                    B[J - 1] = o->ACPH[J] + (-o->AK1[I] / 1.0 - o->AK3[K]);
                }
                if (I == 1 && K == 1) {
                    B[0] = o->ACPH[1] + (-o->AK1[1] / 1.0 - o->AK3[1]);
                    C[0] = 0.0;
                    A[0] = 0.0;
                }
                for (int part = 0; part < 2; ++part) {
                    double* S = part ? SIm : SRe;
                    for (int J = 1; J <= M; ++J) R[J - 1] = S[SIX(I, J, K)];
                    if (K == 1 && I == 1) R[0] = 0.0;
                    tdma_noncyc_line(M, A, B, C, R, w);
                    for (int J = 1; J <= M; ++J) S[SIX(I, J, K)] = R[J - 1];
                }
            }
        free(A); free(B); free(C); free(R); free(w);
    }
#pragma omp parallel
    {
        int nmax = L > N ? L : N;
        cplx* a = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
        cplx* b = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for schedule(static)
        for (int J = 1; J <= M; ++J) {
            for (int I = 1; I <= LH; ++I) {
                for (int K = 1; K <= N; ++K) { a[K - 1].re = SRe[SIX(I, J, K)]; a[K - 1].im = SIm[SIX(I, J, K)]; }
                fft_rec(N, a, 1, b, +1, wbz, 1);
                for (int K = 1; K <= N; ++K) { SRe[SIX(I, J, K)] = b[K - 1].re; SIm[SIX(I, J, K)] = b[K - 1].im; }
            }
            for (int K = 1; K <= N; ++K) {
                /* FFT99 ISIGN=+1: x(j) = sum_k c(k) exp(+2 pi i j k / L), c(L-k) = conj(c(k));
                   the imaginary parts of the k = 0 and k = L/2 coefficients do not enter. */
                for (int I = 1; I <= LH; ++I) { a[I - 1].re = SRe[SIX(I, J, K)]; a[I - 1].im = SIm[SIX(I, J, K)]; }
                a[0].im = 0.0;
                a[L / 2].im = 0.0;
                for (int I = LH + 1; I <= L; ++I) { a[I - 1].re = a[L - I + 1].re; a[I - 1].im = -a[L - I + 1].im; }
                fft_rec(L, a, 1, b, +1, wbx, 1);
                for (int I = 1; I <= L; ++I) F3(dst, o, I, J, K) = b[I - 1].re;
            }
        }
        free(a); free(b);
    }
#undef SIX
    free(wfx); free(wbx); free(wfz); free(wbz);
}

/* Exported Poisson solve on caller arrays in the (L, 0:M+1, N) layout. */
void orc_poisson(orc_t* o, const double* rhs, double* dph) { poisson(o, rhs, dph); }

/* VELOUPDT_tg (src/VELO_CORRECTION.f90:14-100) */
static void veloupdt(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
    double COE1 = o->DT * o->TALP[NS] * o->DXI;
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC)
        for (int JC = 1; JC <= M; ++JC)
            for (int IC = 1; IC <= L; ++IC) {
                int IM = IMV(o, IC);
                double DFX11 = F3(o->DPH, o, IC, JC, KC) - F3(o->DPH, o, IM, JC, KC);
                QV(o, IC, JC, KC, 1) = QV(o, IC, JC, KC, 1) - DFX11 * COE1;
            }
    COE1 = o->DT * o->TALP[NS] * o->DZI;
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC) {
        int KM = KMV(o, KC);
        for (int JC = 1; JC <= M; ++JC)
            for (int IC = 1; IC <= L; ++IC) {
                double DFX33 = F3(o->DPH, o, IC, JC, KC) - F3(o->DPH, o, IC, JC, KM);
                QV(o, IC, JC, KC, 3) = QV(o, IC, JC, KC, 3) - DFX33 * COE1;
            }
    }
#pragma omp parallel for schedule(static)
    for (int JC = 2; JC <= M; ++JC) {
        int JJ = JC, JM = JC - 1;
        double C1 = o->DT * o->TALP[NS] * o->DYCI[JJ] / 1.0;
        for (int KC = 1; KC <= N; ++KC)
            for (int IC = 1; IC <= L; ++IC) {
                double DFX22 = F3(o->DPH, o, IC, JC, KC) - F3(o->DPH, o, IC, JM, KC);
                QV(o, IC, JC, KC, 2) = QV(o, IC, JC, KC, 2) - DFX22 * C1;
            }
    }
}

/* PRCALC_tg (src/PRESSURE_CORRECTION.f90:15-99) */
static void prcalc(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
    double BE = 0.5 * o->TALP[NS] * o->DT * o->CVISC * 1.0 / 1.0;
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC)
        for (int JC = 1; JC <= M; ++JC)
            for (int IC = 1; IC <= L; ++IC) {
                double LLPHI = F3(o->RHSLLPHI, o, IC, JC, KC);
                F3(o->PR, o, IC, JC, KC) = F3(o->PR, o, IC, JC, KC) + F3(o->DPH, o, IC, JC, KC) - BE * LLPHI;
            }
}

/* SOLVERRK3_MOM_tg(NS) (src/SOLVERRK3_MOM_tg.f90:13-56) */
int orc_substep(orc_t* o, int NS) {
    if (NS < 0 || NS > 3) return -1;
    convection_x(o);
    convection_y(o);
    convection_z(o);
    for (int IDR = 1; IDR <= 3; ++IDR) {
        rhs_cvlpgps(o, NS, IDR);
        momfa(o, NS, IDR);
    }
    bc_wall_q(o);
    divg(o, NS);
    memset(o->DPH, 0, FSZ(o) * sizeof(double));
    poisson(o, o->RHSLLPHI, o->DPH);
    bc_wall_scalar(o, o->DPH);
    veloupdt(o, NS);
    bc_wall_q(o);
    prcalc(o, NS);
    bc_wall_scalar(o, o->PR);
    return 0;
}

/* CFL_tg (src/CFL.f90:13-52) */
double orc_cfl(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    double CFLMA = 0.0;
    for (int K = 1; K <= N; ++K) {
        int KP = KPV(o, K);
        for (int J = 1; J <= M; ++J) {
            int JP = J + 1, JC = J;
            for (int I = 1; I <= L; ++I) {
                int IP = IPV(o, I);
                double QCF = (fabs((QV(o, I, J, K, 1) + QV(o, IP, J, K, 1)) * o->DXI) +
                              fabs((QV(o, I, J, K, 2) + QV(o, I, JP, K, 2)) * o->DYFI[JC] * 1.0) +
                              fabs((QV(o, I, J, K, 3) + QV(o, I, J, KP, 3)) * o->DZI * 1.0)) * 0.5;
                CFLMA = fmax(CFLMA, QCF);
            }
        }
    }
    o->CFLMM = CFLMA;
    return CFLMA;
}

/* dt rule of BCAST_COMM_STEP (src/SOLVE.f90:177-178); returns 1 when   */
/* DT/DT0 < 0.01 (the reference dumps and STOPs, :199-207).             */
int orc_step_dt(orc_t* o, double* dt_out) {
    double c = orc_cfl(o);
    double dt = fmin(fmin(o->DT0, 5.0 * o->DT), o->CFLGV / c);
    dt = fmax(dt, o->DTMIN);
    o->DT = dt;
    if (dt_out) *dt_out = dt;
    return (dt / o->DT0) < 0.01 ? 1 : 0;
}

/* One time step of SOLVE (src/SOLVE.f90:75-134): CFL/dt + 3 substeps. */
int orc_run_steps(orc_t* o, int nsteps, double* dts) {
    for (int s = 0; s < nsteps; ++s) {
        double dt;
        if (orc_step_dt(o, &dt)) return 1;
        if (dts) dts[s] = dt;
        for (int NS = 1; NS <= 3; ++NS) orc_substep(o, NS);
    }
    return 0;
}

/* DIVGCK_tg (src/DIVGCK.f90:15-55) */
double orc_divgck(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    double DIVX = 0.0;
    for (int K = 1; K <= N; ++K) {
        int KP = KPV(o, K);
        for (int J = 1; J <= M; ++J) {
            int JP = J + 1, JJ = J;
            for (int I = 1; I <= L; ++I) {
                int IP = IPV(o, I);
                double DQCAP = (QV(o, IP, J, K, 1) - QV(o, I, J, K, 1)) * o->DXI +
                               (QV(o, I, JP, K, 2) - QV(o, I, J, K, 2)) * o->DYFI[JJ] * 1.0 +
                               (QV(o, I, J, KP, 3) - QV(o, I, J, K, 3)) * o->DZI * 1.0;
                DIVX = fmax(fabs(DQCAP), DIVX);
            }
        }
    }
    return DIVX;
}


/* ====================================================================== */
/* IO (main-domain, x-periodic) path with explicit viscous terms:         */
/* SOLVERRK3_MOM_io (src/SOLVERRK3_MOM_IO.f90:11-120, iVisScheme = 0)      */
/* for a flow whose thermodynamics is not yet active (the property fields */
/* DENSITY0 / Viscousity0 are given and fixed; DrhoDtP = 0).               */
/* ====================================================================== */

void orc_io_enable(orc_t* o) {
    if (o->io) return;
    size_t fs = FSZ(o);
    o->G = dalloc(3 * fs); o->EXPLT0 = dalloc(3 * fs); o->RHO = dalloc(fs); o->MU0 = dalloc(fs); o->MU = dalloc(fs);
    o->DSTG = dalloc(3 * fs); o->MUSTG = dalloc(3 * fs); o->DIVU = dalloc(fs); o->DRHODT = dalloc(fs);
    o->DEN = dalloc(fs);
    o->DRHOI = dalloc(3 * fs);
    /* D_STG and MU_STG start at 1 (src/MEMALLOCT.f90:200-201); DENSITY_Staggered and MU_Staggered */
    /* fill the interior, the ghost columns of the inflow/outflow domain keep it                  */
    for (size_t e = 0; e < 3 * fs; ++e) { o->DSTG[e] = 1.0; o->MUSTG[e] = 1.0; }
    o->io = 1;
}

/* DENSITY_Staggered (src/MASSFLUX_CALC_IO.f90:262-329) and MU_Staggered   */
/* (:155-259) from the cell-centred DENSITY0 (RHO) and Viscousity0 (MU0). */
static void io_staggered_props(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    for (int K = 1; K <= N; ++K) {
        int KM = KMV(o, K);
        for (int J = 1; J <= M; ++J)
            for (int I = 1; I <= L; ++I) {
                int IM = IMV(o, I);
                DSV(o, I, J, K, 1) = (F3(o->RHO, o, I, J, K) + F3(o->RHO, o, IM, J, K)) * 0.5;
                DSV(o, I, J, K, 3) = (F3(o->RHO, o, I, J, K) + F3(o->RHO, o, I, J, KM)) * 0.5;
                if (J >= 2) DSV(o, I, J, K, 2) = o->WFF[J] * F3(o->RHO, o, I, J, K) + o->WFB[J] * F3(o->RHO, o, I, J - 1, K);
                if (J >= 2)
                    MSV(o, I, J, K, 1) = ((F3(o->MU0, o, I, J, K) + F3(o->MU0, o, IM, J, K)) * o->WFF[J] +
                                          (F3(o->MU0, o, I, J - 1, K) + F3(o->MU0, o, IM, J - 1, K)) * o->WFB[J]) * 0.5;
                MSV(o, I, J, K, 2) = (F3(o->MU0, o, I, J, K) + F3(o->MU0, o, IM, J, K) + F3(o->MU0, o, I, J, KM) +
                                      F3(o->MU0, o, IM, J, KM)) * 0.5 * 0.5;
                if (J >= 2)
                    MSV(o, I, J, K, 3) = ((F3(o->MU0, o, I, J, KM) + F3(o->MU0, o, I, J, K)) * o->WFF[J] +
                                          (F3(o->MU0, o, I, J - 1, KM) + F3(o->MU0, o, I, J - 1, K)) * o->WFB[J]) * 0.5;
            }
        for (int I = 1; I <= L; ++I) {
            DSV(o, I, 1, K, 2) = F3(o->RHO, o, I, 0, K);
            DSV(o, I, M + 1, K, 2) = F3(o->RHO, o, I, M + 1, K);
            MSV(o, I, 1, K, 1) = F3(o->MU0, o, I, 0, K);
            MSV(o, I, 1, K, 3) = F3(o->MU0, o, I, 0, K);
            MSV(o, I, M + 1, K, 1) = F3(o->MU0, o, I, M + 1, K);
            MSV(o, I, M + 1, K, 3) = F3(o->MU0, o, I, M + 1, K);
        }
    }
}

/* BC_WALL_G_io (src/BC_WALL.f90:435-481) */
static void io_bc_wall_g(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    for (int K = 1; K <= N; ++K)
        for (int I = 1 - o->xo; I <= L + o->xo; ++I) {
            GV(o, I, 0, K, 1) = 0.0; GV(o, I, 0, K, 3) = 0.0; GV(o, I, 1, K, 2) = 0.0; GV(o, I, 0, K, 2) = 0.0;
            GV(o, I, M + 1, K, 1) = 0.0; GV(o, I, M + 1, K, 3) = 0.0; GV(o, I, M + 1, K, 2) = 0.0;
        }
}

/* VELOCITY_CALC_io (src/MASSFLUX_CALC_IO.f90:96-152) + BC_WALL_Q_io */
static void io_velocity_calc(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
#pragma omp parallel for schedule(static)
    for (int K = 1; K <= N; ++K)
        for (int J = 1; J <= M; ++J)
            for (int I = 1; I <= L; ++I) {
                QV(o, I, J, K, 1) = GV(o, I, J, K, 1) / DSV(o, I, J, K, 1);
                QV(o, I, J, K, 3) = GV(o, I, J, K, 3) / DSV(o, I, J, K, 3);
                if (J >= 2) QV(o, I, J, K, 2) = GV(o, I, J, K, 2) / DSV(o, I, J, K, 2);
            }
    bc_wall_q(o);
}

/* Field set-up of ReStart_INSTANT_VARS_io (src/processing/RESTART_io.f90:
 * 16-200) for a restart with the thermal solver not yet active: G, PR and the
 * property fields are given (padded layout); ghosts, D_STG, MU_STG, Q follow. */
void orc_io_set_fields(orc_t* o, const double* G, const double* PR, const double* RHO, const double* MU0,
                       const double* MU) {
    orc_io_enable(o);
    size_t fs = FSZ(o);
    memcpy(o->G, G, 3 * fs * sizeof(double));
    memcpy(o->PR, PR, fs * sizeof(double));
    memcpy(o->RHO, RHO, fs * sizeof(double));
    memcpy(o->DEN, RHO, fs * sizeof(double));
    memcpy(o->MU0, MU0, fs * sizeof(double));
    memcpy(o->MU, MU, fs * sizeof(double));
    memset(o->EXPLT0, 0, 3 * fs * sizeof(double));
    memset(o->DRHODT, 0, fs * sizeof(double));
    io_bc_wall_g(o);
    bc_wall_scalar(o, o->PR);
    io_staggered_props(o);
    io_velocity_calc(o);
    if (o->xo) {
        /* the ghost columns' velocity: G over the x average of DENSITY0 of the column and its */
        /* interior neighbour (the division BC_COUTLET_MOM_RK3 applies to the outlet column)    */
        int L = o->L, M = o->M, N = o->N;
        for (int K = 1; K <= N; ++K)
            for (int J = 0; J <= M + 1; ++J)
                for (int side = 0; side < 2; ++side) {
                    int IG = side ? L + 1 : 0, IN = side ? L : 1;
                    double RHO = (F3(o->RHO, o, IN, J, K) + F3(o->RHO, o, IG, J, K)) * 0.5;
                    for (int c = 1; c <= 3; ++c) QV(o, IG, J, K, c) = GV(o, IG, J, K, c) / RHO;
                }
        memset(o->BCCONV0, 0, 3 * (size_t)M * (size_t)N * sizeof(double));
    }
}

void orc_io_get_fields(const orc_t* o, double* G, double* Q, double* PR) {
    size_t fs = FSZ(o);
    if (G) memcpy(G, o->G, 3 * fs * sizeof(double));
    if (Q) memcpy(Q, o->Q, 3 * fs * sizeof(double));
    if (PR) memcpy(PR, o->PR, fs * sizeof(double));
}

/* CONVECTION_X_io (src/CONVECTION_X.f90:67-156) */
static void io_convection_x(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    memset(o->QTMP, 0, FSZ(o) * sizeof(double));
    double COE1 = o->DXI * 0.5 * 0.5, COE3 = o->DZI * 0.5 * 0.5;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * 0.5 * 1.0, COE32 = COE3 * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1 + o->xo; IC <= L; ++IC) {  /* NXI = 2 with TgFlowFlg (:92) */
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double H11F = (GV(o, IP, JC, KC, 1) + GV(o, IC, JC, KC, 1)) * (QV(o, IP, JC, KC, 1) + QV(o, IC, JC, KC, 1));
                double H11B = (GV(o, IC, JC, KC, 1) + GV(o, IM, JC, KC, 1)) * (QV(o, IC, JC, KC, 1) + QV(o, IM, JC, KC, 1));
                double H11 = (H11F - H11B) * COE1;
                double H12F = (GV(o, IC, JP, KC, 2) + GV(o, IM, JP, KC, 2)) *
                              (o->WFF[JJP] * QV(o, IC, JP, KC, 1) + o->WFB[JJP] * QV(o, IC, JC, KC, 1));
                double H12B = (GV(o, IC, JC, KC, 2) + GV(o, IM, JC, KC, 2)) *
                              (o->WFF[JJ] * QV(o, IC, JC, KC, 1) + o->WFB[JJ] * QV(o, IC, JM, KC, 1));
                double H12 = (H12F - H12B) * COE2;
                double H13F = (GV(o, IC, JC, KP, 3) + GV(o, IM, JC, KP, 3)) * (QV(o, IC, JC, KP, 1) + QV(o, IC, JC, KC, 1));
                double H13B = (GV(o, IC, JC, KC, 3) + GV(o, IM, JC, KC, 3)) * (QV(o, IC, JC, KC, 1) + QV(o, IC, JC, KM, 1));
                double H13 = (H13F - H13B) * COE32;
                F3(o->QTMP, o, IC, JC, KC) = -(H11 + H12 + H13);
            }
        }
    }
}

/* CONVECTION_Y_io (src/CONVECTION_Y.f90:117-272), channel */
static void io_convection_y(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    memset(o->DPH, 0, FSZ(o) * sizeof(double));
    double COE1 = o->DXI * 0.5, COE30 = o->DZI * 0.5;
#pragma omp parallel for schedule(static)
    for (int JC = 2; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC;
        double COE2 = o->DYCI[JJ] * 0.5 * 0.5, COE31 = COE30 * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double H21F = (o->WFF[JJ] * GV(o, IP, JC, KC, 1) + o->WFB[JJ] * GV(o, IP, JM, KC, 1)) *
                              (QV(o, IP, JC, KC, 2) + QV(o, IC, JC, KC, 2));
                double H21B = (o->WFF[JJ] * GV(o, IC, JC, KC, 1) + o->WFB[JJ] * GV(o, IC, JM, KC, 1)) *
                              (QV(o, IC, JC, KC, 2) + QV(o, IM, JC, KC, 2));
                double H21 = (H21F - H21B) * COE1;
                double H22F = (GV(o, IC, JP, KC, 2) + GV(o, IC, JC, KC, 2)) * (QV(o, IC, JP, KC, 2) * 1.0 + QV(o, IC, JC, KC, 2) * 1.0);
                double H22B = (GV(o, IC, JC, KC, 2) + GV(o, IC, JM, KC, 2)) * (QV(o, IC, JC, KC, 2) * 1.0 + QV(o, IC, JM, KC, 2) * 1.0);
                double H22 = (H22F - H22B) * COE2;
                double H23F = (o->WFF[JJ] * GV(o, IC, JC, KP, 3) * 1.0 + o->WFB[JJ] * GV(o, IC, JM, KP, 3) * 1.0) *
                              (QV(o, IC, JC, KP, 2) + QV(o, IC, JC, KC, 2));
                double H23B = (o->WFF[JJ] * GV(o, IC, JC, KC, 3) * 1.0 + o->WFB[JJ] * GV(o, IC, JM, KC, 3) * 1.0) *
                              (QV(o, IC, JC, KC, 2) + QV(o, IC, JC, KM, 2));
                double H23 = (H23F - H23B) * COE31;
                F3(o->DPH, o, IC, JC, KC) = -(H21 + H22 + H23);
            }
        }
    }
}

/* CONVECTION_Z_io (src/CONVECTION_Z.f90:106-303), channel */
static void io_convection_z(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    memset(o->RHSLLPHI, 0, FSZ(o) * sizeof(double));
    double COE1 = o->DXI * 0.5 * 0.5, COE30 = o->DZI * 0.5 * 0.5;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * 0.5, COE31 = COE30 * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double H31F = (GV(o, IP, JC, KC, 1) + GV(o, IP, JC, KM, 1)) * (QV(o, IP, JC, KC, 3) + QV(o, IC, JC, KC, 3));
                double H31B = (GV(o, IC, JC, KC, 1) + GV(o, IC, JC, KM, 1)) * (QV(o, IC, JC, KC, 3) + QV(o, IM, JC, KC, 3));
                double H31 = (H31F - H31B) * COE1;
                double H32F = (GV(o, IC, JP, KC, 2) + GV(o, IC, JP, KM, 2)) *
                              (o->WFF[JJP] * QV(o, IC, JP, KC, 3) * 1.0 + o->WFB[JJP] * QV(o, IC, JC, KC, 3) * 1.0);
                double H32B = (GV(o, IC, JC, KC, 2) + GV(o, IC, JC, KM, 2)) *
                              (o->WFF[JJ] * QV(o, IC, JC, KC, 3) * 1.0 + o->WFB[JJ] * QV(o, IC, JM, KC, 3) * 1.0);
                double H32 = (H32F - H32B) * COE2;
                double H33F = (GV(o, IC, JC, KP, 3) + GV(o, IC, JC, KC, 3)) * (QV(o, IC, JC, KP, 3) + QV(o, IC, JC, KC, 3));
                double H33B = (GV(o, IC, JC, KC, 3) + GV(o, IC, JC, KM, 3)) * (QV(o, IC, JC, KC, 3) + QV(o, IC, JC, KM, 3));
                double H33 = (H33F - H33B) * COE31;
                F3(o->RHSLLPHI, o, IC, JC, KC) = -(H31 + H32 + H33);
            }
        }
    }
}

/* DIVG_U_io (src/DIVG.f90:140-246): DivU = div(u) / 3 */
static void io_divg_u(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    memset(o->DIVU, 0, FSZ(o) * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JP = JC + 1, JJ = JC;
        double COE2 = o->DYFI[JJ] * 1.0, COE3 = o->DZI * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC);
                double DIVX = (QV(o, IP, JC, KC, 1) - QV(o, IC, JC, KC, 1)) * o->DXI;
                double DIVY = (QV(o, IC, JP, KC, 2) - QV(o, IC, JC, KC, 2)) * COE2;
                double DIVZ = (QV(o, IC, JC, KP, 3) - QV(o, IC, JC, KC, 3)) * COE3;
                F3(o->DIVU, o, IC, JC, KC) = (DIVX + DIVY + DIVZ) / 3.0;
            }
        }
    }
}

/* VISCOUS_ALL_EXPLT_X_io (src/VISCOUS_X_EXPLICIT_io.f90:13-128) */
static void io_viscous_x(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    double COE1 = 2.0 * o->DXI * o->CVISC, COE3 = o->DZI * o->CVISC;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * o->CVISC * 1.0, COE32 = COE3 * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double DUDX = (QV(o, IP, JC, KC, 1) - QV(o, IC, JC, KC, 1)) * o->DXI;
                double TAU11F = 0.5 * (F3(o->MU0, o, IC, JC, KC) + F3(o->MU0, o, IC, JC, KC)) * (DUDX - F3(o->DIVU, o, IC, JC, KC));
                DUDX = (QV(o, IC, JC, KC, 1) - QV(o, IM, JC, KC, 1)) * o->DXI;
                double TAU11B = 0.5 * (F3(o->MU0, o, IM, JC, KC) + F3(o->MU0, o, IM, JC, KC)) * (DUDX - F3(o->DIVU, o, IM, JC, KC));
                double DTAU11DX = (TAU11F - TAU11B) * COE1;
                double VIS12P = MSV(o, IC, JP, KC, 1);
                double DUDY = (QV(o, IC, JP, KC, 1) - QV(o, IC, JC, KC, 1)) * o->DYCI[JJP] / 1.0;
                double DVDX = (QV(o, IC, JP, KC, 2) - QV(o, IM, JP, KC, 2)) * o->DXI;
                double TAU12F = VIS12P * (DUDY + DVDX);
                double VIS12C = MSV(o, IC, JC, KC, 1);
                DUDY = (QV(o, IC, JC, KC, 1) - QV(o, IC, JM, KC, 1)) * o->DYCI[JJ] / 1.0;
                DVDX = (QV(o, IC, JC, KC, 2) - QV(o, IM, JC, KC, 2)) * o->DXI;
                double TAU12B = VIS12C * (DUDY + DVDX);
                double DTAU12DY = (TAU12F - TAU12B) * COE2;
                double VIS13P = MSV(o, IC, JC, KP, 2);
                double DUDZ = (QV(o, IC, JC, KP, 1) - QV(o, IC, JC, KC, 1)) * o->DZI;
                double DWDX = (QV(o, IC, JC, KP, 3) - QV(o, IM, JC, KP, 3)) * o->DXI;
                double TAU13F = VIS13P * (DUDZ + DWDX);
                double VIS13C = MSV(o, IC, JC, KC, 2);
                DUDZ = (QV(o, IC, JC, KC, 1) - QV(o, IC, JC, KM, 1)) * o->DZI;
                DWDX = (QV(o, IC, JC, KC, 3) - QV(o, IM, JC, KC, 3)) * o->DXI;
                double TAU13B = VIS13C * (DUDZ + DWDX);
                double DTAU13DZ = (TAU13F - TAU13B) * COE32;
                F3(o->QTMP, o, IC, JC, KC) = F3(o->QTMP, o, IC, JC, KC) + DTAU11DX + DTAU12DY + DTAU13DZ;
            }
        }
    }
}

/* VISCOUS_ALL_EXPLT_Y_io (src/VISCOUS_Y_EXPLICIT_io.f90:14-120), channel */
static void io_viscous_y(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    double COE1 = o->DXI * o->CVISC, COE3 = o->DZI * o->CVISC;
#pragma omp parallel for schedule(static)
    for (int JC = 2; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJM = JJ - 1;
        double COE2 = 2.0 * o->DYCI[JJ] * o->CVISC;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double DVDY = (QV(o, IC, JP, KC, 2) - QV(o, IC, JC, KC, 2)) * o->DYFI[JJ];
                double TAU22F = 0.5 * (F3(o->MU0, o, IC, JC, KC) + F3(o->MU0, o, IC, JC, KC)) * (DVDY - F3(o->DIVU, o, IC, JC, KC));
                DVDY = (QV(o, IC, JC, KC, 2) - QV(o, IC, JM, KC, 2)) * o->DYFI[JJM];
                double TAU22B = 0.5 * (F3(o->MU0, o, IC, JM, KC) + F3(o->MU0, o, IC, JM, KC)) * (DVDY - F3(o->DIVU, o, IC, JM, KC));
                double DTAU22DY = (TAU22F - TAU22B) * COE2;
                double VIS21P = MSV(o, IP, JC, KC, 1);
                double DVDX = (QV(o, IP, JC, KC, 2) - QV(o, IC, JC, KC, 2)) * o->DXI;
                double DUDY = (QV(o, IP, JC, KC, 1) - QV(o, IP, JM, KC, 1)) * o->DYCI[JJ];
                double TAU21F = VIS21P * (DVDX + DUDY);
                double VIS21C = MSV(o, IC, JC, KC, 1);
                DVDX = (QV(o, IC, JC, KC, 2) - QV(o, IM, JC, KC, 2)) * o->DXI;
                DUDY = (QV(o, IC, JC, KC, 1) - QV(o, IC, JM, KC, 1)) * o->DYCI[JJ];
                double TAU21B = VIS21C * (DVDX + DUDY);
                double DTAU21DX = (TAU21F - TAU21B) * COE1;
                double VIS23P = MSV(o, IC, JC, KP, 3);
                double DVDZ = (QV(o, IC, JC, KP, 2) - QV(o, IC, JC, KC, 2)) * o->DZI;
                double DWDY = (QV(o, IC, JC, KP, 3) - QV(o, IC, JM, KP, 3)) * o->DYCI[JJ];
                double TAU23F = VIS23P * (DVDZ + DWDY);
                double VIS23C = MSV(o, IC, JC, KC, 3);
                DVDZ = (QV(o, IC, JC, KC, 2) - QV(o, IC, JC, KM, 2)) * o->DZI;
                DWDY = (QV(o, IC, JC, KC, 3) - QV(o, IC, JM, KC, 3)) * o->DYCI[JJ];
                double TAU23B = VIS23C * (DVDZ + DWDY);
                double DTAU23DZ = (TAU23F - TAU23B) * COE3;
                F3(o->DPH, o, IC, JC, KC) = F3(o->DPH, o, IC, JC, KC) + DTAU21DX + DTAU22DY + DTAU23DZ;
            }
        }
    }
}

/* VISCOUS_ALL_EXPLT_Z_io (src/VISCOUS_Z_EXPLICIT_io.f90:13-100), channel */
static void io_viscous_z(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    double COE1 = o->DXI * o->CVISC, COE3 = 2.0 * o->DZI * o->CVISC;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * o->CVISC;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double DWDZ = (QV(o, IC, JC, KP, 3) - QV(o, IC, JC, KC, 3)) * o->DZI;
                double TAU33F = 0.5 * (F3(o->MU0, o, IC, JC, KC) + F3(o->MU0, o, IC, JC, KC)) * (DWDZ - F3(o->DIVU, o, IC, JC, KC));
                DWDZ = (QV(o, IC, JC, KC, 3) - QV(o, IC, JC, KM, 3)) * o->DZI;
                double TAU33B = 0.5 * (F3(o->MU0, o, IC, JC, KM) + F3(o->MU0, o, IC, JC, KM)) * (DWDZ - F3(o->DIVU, o, IC, JC, KM));
                double DTAU33DZ = (TAU33F - TAU33B) * COE3;
                double VIS31P = MSV(o, IP, JC, KC, 2);
                double DWDX = (QV(o, IP, JC, KC, 3) - QV(o, IC, JC, KC, 3)) * o->DXI;
                double DUDZ = (QV(o, IP, JC, KC, 1) - QV(o, IP, JC, KM, 1)) * o->DZI;
                double TAU31F = VIS31P * (DWDX + DUDZ);
                double VIS31C = MSV(o, IC, JC, KC, 2);
                DWDX = (QV(o, IC, JC, KC, 3) - QV(o, IM, JC, KC, 3)) * o->DXI;
                DUDZ = (QV(o, IC, JC, KC, 1) - QV(o, IC, JC, KM, 1)) * o->DZI;
                double TAU31B = VIS31C * (DWDX + DUDZ);
                double DTAU31DX = (TAU31F - TAU31B) * COE1;
                double VIS32P = MSV(o, IC, JP, KC, 3);
                double DWDY = (QV(o, IC, JP, KC, 3) - QV(o, IC, JC, KC, 3)) * o->DYCI[JJP];
                double DVDZ = (QV(o, IC, JP, KC, 2) - QV(o, IC, JP, KM, 2)) * o->DZI;
                double TAU32F = VIS32P * (DWDY + DVDZ);
                double VIS32C = MSV(o, IC, JC, KC, 3);
                DWDY = (QV(o, IC, JC, KC, 3) - QV(o, IC, JM, KC, 3)) * o->DYCI[JJ];
                DVDZ = (QV(o, IC, JC, KC, 2) - QV(o, IC, JC, KM, 2)) * o->DZI;
                double TAU32B = VIS32C * (DWDY + DVDZ);
                double DTAU32DY = (TAU32F - TAU32B) * COE2;
                F3(o->RHSLLPHI, o, IC, JC, KC) = F3(o->RHSLLPHI, o, IC, JC, KC) + DTAU31DX + DTAU32DY + DTAU33DZ;
            }
        }
    }
}

/* iWeightedPre: pres_epslon (src/modules.f90:483) */
#define PRES_EPSLON 0.001

/* Pressure-gradient term PGM of RHS_MOM_EXPLICIT_io (:103-159) between the */
/* points a and b (b the lower neighbour), with the weighted-pressure blend  */
/* of PR0_io(:,:,:,2), PR0_io(:,:,:,1) and PR_io when iWeightedPre = 1.      */
static inline double io_pgm(const orc_t* o, size_t a, size_t b, double COE2) {
    if (o->PR0A)
        return ((o->PR0B[a] - o->PR0B[b]) * (0.25 - PRES_EPSLON) + (o->PR0A[a] - o->PR0A[b]) * 0.5 +
                (o->PR[a] - o->PR[b]) * (0.25 + PRES_EPSLON)) * COE2;
    return (o->PR[a] - o->PR[b]) * COE2;
}

/* RHS_MOM_EXPLICIT_io(NS, IDR) (src/RHS_MOM_EXPLICIT_io.f90:11-304), plane */
/* channel (RNDI1 = RCCI1 = 1): RK combination, pressure gradient (weighted  */
/* or not), buoyancy, bulk forcing, save-back.                               */
static void io_rhs_mom_explicit(orc_t* o, int NS, int IDR) {
    int L = o->L, M = o->M, N = o->N;
    int NYI = (IDR == 2) ? 2 : 1;
    int NXI = (o->xo && IDR == 1) ? 2 : 1;  /* TgFlowFlg: the inlet face u(1) is a boundary value (:35) */
    double* EX = IDR == 1 ? o->QTMP : IDR == 2 ? o->DPH : o->RHSLLPHI;
    double DT = o->DT;
    if (!o->ivis) {
        memset(o->RHS, 0, FSZ(o) * sizeof(double));
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC)
            for (int JC = NYI; JC <= M; ++JC)
                for (int IC = NXI; IC <= L; ++IC) {
                    double RHSC = F3(EX, o, IC, JC, KC);
                    double RHSL = E0V(o, IC, JC, KC, IDR);
                    F3(o->RHS, o, IC, JC, KC) = (o->TGAM[NS] * RHSC + o->TROH[NS] * RHSL) * DT;
                    E0V(o, IC, JC, KC, IDR) = RHSC;
                }
    } else {
        /* VisImplicit (:87-99): RHS holds the implicit viscous part, DIVU the density correction */
        double COE2 = o->TALP[NS] * DT;
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC)
            for (int JC = NYI; JC <= M; ++JC)
                for (int IC = NXI; IC <= L; ++IC) {
                    double RHSC = F3(EX, o, IC, JC, KC);
                    double RHSL = E0V(o, IC, JC, KC, IDR);
                    F3(o->RHS, o, IC, JC, KC) = (o->TGAM[NS] * RHSC + o->TROH[NS] * RHSL) * DT +
                                                COE2 * F3(o->RHS, o, IC, JC, KC) + 0.5 * COE2 * F3(o->DIVU, o, IC, JC, KC);
                    E0V(o, IC, JC, KC, IDR) = RHSC;
                }
    }
    if (IDR == 1) {
        double COE2 = o->TALP[NS] * DT * o->DXI;
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC)
            for (int JC = 1; JC <= M; ++JC)
                for (int IC = NXI; IC <= L; ++IC) {
                    double PGM = io_pgm(o, FOFF(o, IC, JC, KC), FOFF(o, IMV(o, IC), JC, KC), COE2);
                    F3(o->RHS, o, IC, JC, KC) = F3(o->RHS, o, IC, JC, KC) - PGM;
                }
    } else if (IDR == 2) {
#pragma omp parallel for schedule(static)
        for (int JC = 2; JC <= M; ++JC) {
            double COE2 = o->TALP[NS] * DT * o->DYCI[JC] / 1.0;
            for (int KC = 1; KC <= N; ++KC)
                for (int IC = NXI; IC <= L; ++IC) {
                    double PGM = io_pgm(o, FOFF(o, IC, JC, KC), FOFF(o, IC, JC - 1, KC), COE2);
                    F3(o->RHS, o, IC, JC, KC) = F3(o->RHS, o, IC, JC, KC) - PGM;
                }
        }
    } else {
        double COE2 = o->TALP[NS] * DT * o->DZI;
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC);
            for (int JC = 1; JC <= M; ++JC)
                for (int IC = NXI; IC <= L; ++IC) {
                    double PGM = io_pgm(o, FOFF(o, IC, JC, KC), FOFF(o, IC, JC, KM), COE2);
                    F3(o->RHS, o, IC, JC, KC) = F3(o->RHS, o, IC, JC, KC) - PGM;
                }
        }
    }
    /* buoyancy (:161-226): D_STG(:,:,:,IDR) * TALP*DT*F_A on the component |iGravity| */
    /* (the 1/RNDI1, 1/RCCI1 factors of the y and z directions are 1 in the channel)   */
    if (abs(o->igrav) == IDR) {
        double COE2 = o->TALP[NS] * DT * o->F_A;
        int JS = IDR == 2 ? 2 : 1;
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC)
            for (int JC = JS; JC <= M; ++JC) {
                double C2 = IDR == 1 ? COE2 : COE2 / 1.0;
                for (int IC = NXI; IC <= L; ++IC)
                    F3(o->RHS, o, IC, JC, KC) = F3(o->RHS, o, IC, JC, KC) + DSV(o, IC, JC, KC, IDR) * C2;
            }
    }
    if (IDR == 1 && !o->xo) {  /* bulk forcing of the streamwise-periodic flow only (:229) */
        double DPGRNS = 0.0;
        if (o->iFlowDriven == 1) {
            double INTGRHSY = 0.0;  /* loop order JC, IC, KC */
            for (int JC = 1; JC <= M; ++JC)
                for (int IC = NXI; IC <= L; ++IC)
                    for (int KC = 1; KC <= N; ++KC) INTGRHSY = INTGRHSY + F3(o->RHS, o, IC, JC, KC) / o->DYFI[JC] / 1.0;
            DPGRNS = INTGRHSY / o->VOLM;
        } else if (o->iFlowDriven == 2) {
            DPGRNS = -0.5 * o->Cf_Given * (o->TALP[NS] * DT);
        }
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC)
            for (int JC = 1; JC <= M; ++JC)
                for (int IC = NXI; IC <= L; ++IC) F3(o->RHS, o, IC, JC, KC) = F3(o->RHS, o, IC, JC, KC) - DPGRNS;
    }
    if (o->ivis) return;  /* the save-back (:267-301) is the explicit scheme's */
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC)
        for (int JC = NYI; JC <= M; ++JC)
            for (int IC = NXI; IC <= L; ++IC) F3(EX, o, IC, JC, KC) = F3(o->RHS, o, IC, JC, KC);
}

/* MASSFLUX_CALC_io (src/MASSFLUX_CALC_IO.f90:15-93): G += explicit RHS */
static void io_massflux_calc(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC)
        for (int JC = 1; JC <= M; ++JC)
            for (int IC = 1; IC <= L; ++IC) {
                if (IC > o->xo) GV(o, IC, JC, KC, 1) = GV(o, IC, JC, KC, 1) + F3(o->QTMP, o, IC, JC, KC);  /* NXI */
                GV(o, IC, JC, KC, 3) = GV(o, IC, JC, KC, 3) + F3(o->RHSLLPHI, o, IC, JC, KC);
                if (JC >= 2) GV(o, IC, JC, KC, 2) = GV(o, IC, JC, KC, 2) + F3(o->DPH, o, IC, JC, KC);
            }
}

/* DIVG_io (src/DIVG.f90:54-137) */
static void io_divg(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
    double COE0 = o->PR0A ? 1.0 / o->DT / o->TALP[NS] / (0.25 + PRES_EPSLON) : 1.0 / o->DT / o->TALP[NS];
    memset(o->RHSLLPHI, 0, FSZ(o) * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JP = JC + 1, JJ = JC;
        double COE1 = o->DXI / 1.0, COE2 = o->DYFI[JJ] / 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC);
                double DIVX = (GV(o, IP, JC, KC, 1) - GV(o, IC, JC, KC, 1)) * COE1;
                double DIVY = (GV(o, IC, JP, KC, 2) - GV(o, IC, JC, KC, 2)) * COE2;
                double DIVZ = (GV(o, IC, JC, KP, 3) - GV(o, IC, JC, KC, 3)) * o->DZI;
                double DTRHO = F3(o->DRHODT, o, IC, JC, KC) / 1.0;
                double DQCAP = DIVX + DIVY + DIVZ + DTRHO;
                F3(o->RHSLLPHI, o, IC, JC, KC) = DQCAP * COE0;
            }
        }
    }
}

/* PRCALC_io explicit (src/PRESSURE_CORRECTION.f90:102-170) and           */
/* MASSFLUX_UPDATE_io (src/VELO_CORRECTION.f90:103-179)                   */
static void io_prcalc_massflux_update(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
    if (o->ivis) {
        double BE = 0.50 * o->TALP[NS] * o->DT * o->CVISC;  /* VisImplicit (:113-123) */
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC)
            for (int JC = 1; JC <= M; ++JC)
                for (int IC = 1; IC <= L; ++IC) {
                    double LLphi = F3(o->RHSLLPHI, o, IC, JC, KC);
                    F3(o->PR, o, IC, JC, KC) = F3(o->PR, o, IC, JC, KC) + F3(o->DPH, o, IC, JC, KC) - BE * LLphi;
                }
    } else {
#pragma omp parallel for schedule(static)
        for (int KC = 1; KC <= N; ++KC)
            for (int JC = 1; JC <= M; ++JC)
                for (int IC = 1; IC <= L; ++IC) F3(o->PR, o, IC, JC, KC) = F3(o->PR, o, IC, JC, KC) + F3(o->DPH, o, IC, JC, KC);
    }
    bc_wall_scalar(o, o->PR);
    double COE1 = o->DT * o->TALP[NS] * o->DXI;
    /* u faces NXI..NXE: 1..L, or 2..L+1 with TgFlowFlg (the outlet face included, :121-127) */
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC)
        for (int JC = 1; JC <= M; ++JC)
            for (int IC = 1 + o->xo; IC <= L + o->xo; ++IC) {
                double DFX11 = F3(o->DPH, o, IC, JC, KC) - F3(o->DPH, o, IMV(o, IC), JC, KC);
                GV(o, IC, JC, KC, 1) = GV(o, IC, JC, KC, 1) - DFX11 * COE1;
            }
    COE1 = o->DT * o->TALP[NS] * o->DZI;
#pragma omp parallel for schedule(static)
    for (int KC = 1; KC <= N; ++KC) {
        int KM = KMV(o, KC);
        for (int JC = 1; JC <= M; ++JC)
            for (int IC = 1; IC <= L; ++IC) {
                double DFX33 = F3(o->DPH, o, IC, JC, KC) - F3(o->DPH, o, IC, JC, KM);
                GV(o, IC, JC, KC, 3) = GV(o, IC, JC, KC, 3) - DFX33 * COE1;
            }
    }
#pragma omp parallel for schedule(static)
    for (int JC = 2; JC <= M; ++JC) {
        double C1 = o->DT * o->TALP[NS] * o->DYCI[JC] / 1.0;
        for (int KC = 1; KC <= N; ++KC)
            for (int IC = 1; IC <= L; ++IC) {
                double DFX22 = F3(o->DPH, o, IC, JC, KC) - F3(o->DPH, o, IC, JC - 1, KC);
                GV(o, IC, JC, KC, 2) = GV(o, IC, JC, KC, 2) - DFX22 * C1;
            }
    }
    io_bc_wall_g(o);
}

/* ---------------------------------------------------------------------- */
/* Crank-Nicolson form of the main-domain momentum step (iVisScheme = 1,  */
/* VisImplicit): the viscous split after Nicoud (2000) into an explicit   */
/* part (added to the convection term), an implicit part (RK weight       */
/* alpha*dt) and a density-correction part, then MOMFA_io's approximate   */
/* factorisation with per-point coefficients from Viscousity, MU_STG and  */
/* D_STG.  Plane channel: RCCI1 = RCCI2 = RNDI1 = RNDI2 = 1 (kept as the  */
/* factors 1.0 where the reference multiplies or divides by them).        */
/* ---------------------------------------------------------------------- */
#define DRV(o, i, j, k, c) ((o)->DRHOI[FOFF(o, i, j, k) + (size_t)((c) - 1) * FSZ(o)])

void orc_io_set_vis_scheme(orc_t* o, int ivis) { o->ivis = ivis ? 1 : 0; }

/* thermal_gravity (src/Flow_State.f90:95-125): iGravity selects the momentum */
/* component that takes the buoyancy term, F_A its coefficient.              */
void orc_io_set_buoyancy(orc_t* o, int igravity, double f_a) {
    o->igrav = igravity;
    o->F_A = f_a;
}

/* iWeightedPre = 1 with PR0_io(:,:,:,1) = pr0_1 and PR0_io(:,:,:,2) = pr0_2  */
/* (padded layout); NULL turns it off.                                       */
void orc_io_set_weighted_pressure(orc_t* o, const double* pr0_1, const double* pr0_2) {
    free(o->PR0A);
    free(o->PR0B);
    o->PR0A = o->PR0B = NULL;
    if (!pr0_1 || !pr0_2) return;
    o->PR0A = dalloc(FSZ(o));
    o->PR0B = dalloc(FSZ(o));
    memcpy(o->PR0A, pr0_1, FSZ(o) * sizeof(double));
    memcpy(o->PR0B, pr0_2, FSZ(o) * sizeof(double));
}

/* max |DRHOI_STG| over the interior and the v wall rows (0 by construction) */
double orc_io_drhoi_maxabs(const orc_t* o) {
    double m = 0.0;
    size_t n = 3 * FSZ(o);
    for (size_t q = 0; q < n; ++q) m = fmax(m, fabs(o->DRHOI[q]));
    return m;
}

/* DENSITY_IMPLICIT_add (src/MASSFLUX_CALC_IO.f90:332-416): 1/D_STG minus */
/* 1/(the same average of DENSITY0); SOLVE.f90:123-127 calls it right     */
/* after DENSITY_Staggered, so every entry is 1/x - 1/x = 0.              */
static void io_density_implicit_add(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    for (int I = 1; I <= L; ++I) {
        int IM = IMV(o, I);
        for (int J = 1; J <= M; ++J)
            for (int K = 1; K <= N; ++K) {
                double DEN_STG = (F3(o->RHO, o, I, J, K) + F3(o->RHO, o, IM, J, K)) * 0.5;
                DRV(o, I, J, K, 1) = 1.0 / DSV(o, I, J, K, 1) - 1.0 / DEN_STG;
            }
    }
    for (int K = 1; K <= N; ++K) {
        int KM = KMV(o, K);
        for (int J = 1; J <= M; ++J)
            for (int I = 1; I <= L; ++I) {
                double DEN_STG = (F3(o->RHO, o, I, J, K) + F3(o->RHO, o, I, J, KM)) * 0.5;
                DRV(o, I, J, K, 3) = 1.0 / DSV(o, I, J, K, 3) - 1.0 / DEN_STG;
            }
    }
    for (int J = 2; J <= M; ++J)
        for (int K = 1; K <= N; ++K)
            for (int I = 1; I <= L; ++I) {
                double DEN_STG = o->WFF[J] * F3(o->RHO, o, I, J, K) + o->WFB[J] * F3(o->RHO, o, I, J - 1, K);
                DRV(o, I, J, K, 2) = 1.0 / DSV(o, I, J, K, 2) - 1.0 / DEN_STG;
            }
    for (int K = 1; K <= N; ++K)
        for (int I = 1; I <= L; ++I) {
            DRV(o, I, 1, K, 2) = 0.0;
            DRV(o, I, M + 1, K, 2) = 0.0;
        }
}

/* VISCOUS_PAR_EXPLT_X_io (src/VISCOUS_X_EXPLICIT_io.f90:131-293):          */
/* QTMP += explicit part, RHS = implicit part, DIVU = density correction.  */
/* The tau13 correction takes Q_io (not G_io) times DRHOI_STG, as there.  */
static void io_viscous_par_x(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    memset(o->RHS, 0, FSZ(o) * sizeof(double));
    double COE1 = -2.0 / 3.0 * o->DXI * o->CVISC, COE3 = o->DZI * o->CVISC;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * o->CVISC * 1.0, COE32 = COE3 * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double DUDX = (QV(o, IP, JC, KC, 1) - QV(o, IC, JC, KC, 1)) * o->DXI;
                double DVDY = (QV(o, IC, JP, KC, 2) - QV(o, IC, JC, KC, 2)) * o->DYFI[JJ] * 1.0;
                double DWDZ = (QV(o, IC, JC, KP, 3) - QV(o, IC, JC, KC, 3)) * o->DZI * 1.0;
                double T11F_EX = F3(o->MU, o, IC, JC, KC) * (DVDY + DWDZ);
                double T11F_IM = F3(o->MU, o, IC, JC, KC) * DUDX;
                DUDX = (GV(o, IP, JC, KC, 1) * DRV(o, IP, JC, KC, 1) - GV(o, IC, JC, KC, 1) * DRV(o, IC, JC, KC, 1)) * o->DXI;
                double T11F_AD = F3(o->MU, o, IC, JC, KC) * DUDX;
                DUDX = (QV(o, IC, JC, KC, 1) - QV(o, IM, JC, KC, 1)) * o->DXI;
                DVDY = (QV(o, IM, JP, KC, 2) - QV(o, IM, JC, KC, 2)) * o->DYFI[JJ] * 1.0;
                DWDZ = (QV(o, IM, JC, KP, 3) - QV(o, IM, JC, KC, 3)) * o->DZI * 1.0;
                double T11B_EX = F3(o->MU, o, IM, JC, KC) * (DVDY + DWDZ);
                double T11B_IM = F3(o->MU, o, IM, JC, KC) * DUDX;
                DUDX = (GV(o, IC, JC, KC, 1) * DRV(o, IC, JC, KC, 1) - GV(o, IM, JC, KC, 1) * DRV(o, IM, JC, KC, 1)) * o->DXI;
                double T11B_AD = F3(o->MU, o, IM, JC, KC) * DUDX;
                double D11_EX = (T11F_EX - T11B_EX) * COE1;
                double D11_IM = (T11F_IM - T11B_IM) * COE1 * (-2.0);
                double D11_AD = (T11F_AD - T11B_AD) * COE1 * (-2.0);

                double VIS12P = MSV(o, IC, JP, KC, 1);
                double DVDX = (QV(o, IC, JP, KC, 2) - QV(o, IM, JP, KC, 2)) * o->DXI;
                double DUDY = (QV(o, IC, JP, KC, 1) - QV(o, IC, JC, KC, 1)) * o->DYCI[JJP] / 1.0;
                double T12F_EX = VIS12P * DVDX, T12F_IM = VIS12P * DUDY;
                DUDY = (GV(o, IC, JP, KC, 1) * DRV(o, IC, JP, KC, 1) - GV(o, IC, JC, KC, 1) * DRV(o, IC, JC, KC, 1)) * o->DYCI[JJP] / 1.0;
                double T12F_AD = VIS12P * DUDY;
                double VIS12C = MSV(o, IC, JC, KC, 1);
                DUDY = (QV(o, IC, JC, KC, 1) - QV(o, IC, JM, KC, 1)) * o->DYCI[JJ] / 1.0;
                DVDX = (QV(o, IC, JC, KC, 2) - QV(o, IM, JC, KC, 2)) * o->DXI;
                double T12B_EX = VIS12C * DVDX, T12B_IM = VIS12C * DUDY;
                DUDY = (GV(o, IC, JC, KC, 1) * DRV(o, IC, JC, KC, 1) - GV(o, IC, JM, KC, 1) * DRV(o, IC, JM, KC, 1)) * o->DYCI[JJ] / 1.0;
                double T12B_AD = VIS12C * DUDY;
                double D12_EX = (T12F_EX - T12B_EX) * COE2;
                double D12_IM = (T12F_IM - T12B_IM) * COE2;
                double D12_AD = (T12F_AD - T12B_AD) * COE2;

                double VIS13P = MSV(o, IC, JC, KP, 2);
                double DUDZ = (QV(o, IC, JC, KP, 1) - QV(o, IC, JC, KC, 1)) * o->DZI;
                double DWDX = (QV(o, IC, JC, KP, 3) - QV(o, IM, JC, KP, 3)) * o->DXI;
                double T13F_EX = VIS13P * DWDX, T13F_IM = VIS13P * DUDZ;
                DUDZ = (QV(o, IC, JC, KP, 1) * DRV(o, IC, JC, KP, 1) - QV(o, IC, JC, KC, 1) * DRV(o, IC, JC, KC, 1)) * o->DZI;
                double T13F_AD = VIS13P * DUDZ;
                double VIS13C = MSV(o, IC, JC, KC, 2);
                DUDZ = (QV(o, IC, JC, KC, 1) - QV(o, IC, JC, KM, 1)) * o->DZI;
                DWDX = (QV(o, IC, JC, KC, 3) - QV(o, IM, JC, KC, 3)) * o->DXI;
                double T13B_EX = VIS13C * DWDX, T13B_IM = VIS13C * DUDZ;
                DUDZ = (QV(o, IC, JC, KC, 1) * DRV(o, IC, JC, KC, 1) - QV(o, IC, JC, KM, 1) * DRV(o, IC, JC, KM, 1)) * o->DZI;
                double T13B_AD = VIS13C * DUDZ;
                double D13_EX = (T13F_EX - T13B_EX) * COE32;
                double D13_IM = (T13F_IM - T13B_IM) * COE32;
                double D13_AD = (T13F_AD - T13B_AD) * COE32;

                F3(o->QTMP, o, IC, JC, KC) = D11_EX + D12_EX + D13_EX + F3(o->QTMP, o, IC, JC, KC);
                F3(o->RHS, o, IC, JC, KC) = D11_IM + D12_IM + D13_IM;
                F3(o->DIVU, o, IC, JC, KC) = D11_AD + D12_AD + D13_AD;
            }
        }
    }
}

/* VISCOUS_PAR_EXPLT_Y_io (src/VISCOUS_Y_EXPLICIT_io.f90:278-443), channel: */
/* rows 2..M (the wall face j = 1 keeps RHS = 0).                          */
static void io_viscous_par_y(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    memset(o->RHS, 0, FSZ(o) * sizeof(double));
    double COE1 = o->DXI * o->CVISC, COE3 = o->DZI * o->CVISC;
#pragma omp parallel for schedule(static)
    for (int JC = 2; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJM = JJ - 1;
        double COE2 = -2.0 / 3.0 * o->DYCI[JJ] * o->CVISC;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double DUDX = (QV(o, IP, JC, KC, 1) - QV(o, IC, JC, KC, 1)) * o->DXI;
                double DVDY = (QV(o, IC, JP, KC, 2) - QV(o, IC, JC, KC, 2)) * o->DYFI[JJ];
                double DWDZ = (QV(o, IC, JC, KP, 3) - QV(o, IC, JC, KC, 3)) * o->DZI;
                double T22F_EX = F3(o->MU, o, IC, JC, KC) * (DUDX + DWDZ);
                double T22F_IM = F3(o->MU, o, IC, JC, KC) * DVDY;
                DVDY = (GV(o, IC, JP, KC, 2) * DRV(o, IC, JP, KC, 2) - GV(o, IC, JC, KC, 2) * DRV(o, IC, JC, KC, 2)) * o->DYFI[JJ];
                double T22F_AD = F3(o->MU, o, IC, JC, KC) * DVDY;
                DUDX = (QV(o, IP, JM, KC, 1) - QV(o, IC, JM, KC, 1)) * o->DXI;
                DVDY = (QV(o, IC, JC, KC, 2) - QV(o, IC, JM, KC, 2)) * o->DYFI[JJM];
                DWDZ = (QV(o, IC, JM, KP, 3) - QV(o, IC, JM, KC, 3)) * o->DZI;
                double T22B_EX = F3(o->MU, o, IC, JM, KC) * (DUDX + DWDZ);
                double T22B_IM = F3(o->MU, o, IC, JM, KC) * DVDY;
                DVDY = (GV(o, IC, JC, KC, 2) * DRV(o, IC, JC, KC, 2) - GV(o, IC, JM, KC, 2) * DRV(o, IC, JM, KC, 2)) * o->DYFI[JJM];
                double T22B_AD = F3(o->MU, o, IC, JM, KC) * DVDY;
                double D22_EX = (T22F_EX - T22B_EX) * COE2;
                double D22_IM = (T22F_IM - T22B_IM) * COE2 * (-2.0);
                double D22_AD = (T22F_AD - T22B_AD) * COE2 * (-2.0);

                double VIS21P = MSV(o, IP, JC, KC, 1);
                double DVDX = (QV(o, IP, JC, KC, 2) - QV(o, IC, JC, KC, 2)) * o->DXI;
                double DUDY = (QV(o, IP, JC, KC, 1) - QV(o, IP, JM, KC, 1)) * o->DYCI[JJ];
                double T21F_EX = VIS21P * DUDY, T21F_IM = VIS21P * DVDX;
                DVDX = (GV(o, IP, JC, KC, 2) * DRV(o, IP, JC, KC, 2) - GV(o, IC, JC, KC, 2) * DRV(o, IC, JC, KC, 2)) * o->DXI;
                double T21F_AD = VIS21P * DVDX;
                double VIS21C = MSV(o, IC, JC, KC, 1);
                DVDX = (QV(o, IC, JC, KC, 2) - QV(o, IM, JC, KC, 2)) * o->DXI;
                DUDY = (QV(o, IC, JC, KC, 1) - QV(o, IC, JM, KC, 1)) * o->DYCI[JJ];
                double T21B_EX = VIS21C * DUDY, T21B_IM = VIS21C * DVDX;
                DVDX = (GV(o, IC, JC, KC, 2) * DRV(o, IC, JC, KC, 2) - GV(o, IM, JC, KC, 2) * DRV(o, IM, JC, KC, 2)) * o->DXI;
                double T21B_AD = VIS21C * DVDX;
                double D21_EX = (T21F_EX - T21B_EX) * COE1;
                double D21_IM = (T21F_IM - T21B_IM) * COE1;
                double D21_AD = (T21F_AD - T21B_AD) * COE1;

                double VIS23P = MSV(o, IC, JC, KP, 3);
                double DVDZ = (QV(o, IC, JC, KP, 2) - QV(o, IC, JC, KC, 2)) * o->DZI;
                double DWDY = (QV(o, IC, JC, KP, 3) - QV(o, IC, JM, KP, 3)) * o->DYCI[JJ];
                double T23F_EX = VIS23P * DWDY, T23F_IM = VIS23P * DVDZ;
                DVDZ = (GV(o, IC, JC, KP, 2) * DRV(o, IC, JC, KP, 2) - GV(o, IC, JC, KC, 2) * DRV(o, IC, JC, KC, 2)) * o->DZI;
                double T23F_AD = VIS23P * DVDZ;
                double VIS23C = MSV(o, IC, JC, KC, 3);
                DVDZ = (QV(o, IC, JC, KC, 2) - QV(o, IC, JC, KM, 2)) * o->DZI;
                DWDY = (QV(o, IC, JC, KC, 3) - QV(o, IC, JM, KC, 3)) * o->DYCI[JJ];
                double T23B_EX = VIS23C * DWDY, T23B_IM = VIS23C * DVDZ;
                DVDZ = (GV(o, IC, JC, KC, 2) * DRV(o, IC, JC, KC, 2) - GV(o, IC, JC, KM, 2) * DRV(o, IC, JC, KM, 2)) * o->DZI;
                double T23B_AD = VIS23C * DVDZ;
                double D23_EX = (T23F_EX - T23B_EX) * COE3;
                double D23_IM = (T23F_IM - T23B_IM) * COE3;
                double D23_AD = (T23F_AD - T23B_AD) * COE3;

                F3(o->DPH, o, IC, JC, KC) = D21_EX + D22_EX + D23_EX + F3(o->DPH, o, IC, JC, KC);
                F3(o->RHS, o, IC, JC, KC) = D21_IM + D22_IM + D23_IM;
                F3(o->DIVU, o, IC, JC, KC) = D21_AD + D22_AD + D23_AD;
            }
        }
    }
}

/* VISCOUS_PAR_EXPLT_Z_io (src/VISCOUS_Z_EXPLICIT_io.f90:300-465), channel */
static void io_viscous_par_z(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    memset(o->RHS, 0, FSZ(o) * sizeof(double));
    double COE1 = o->DXI * o->CVISC, COE3 = -2.0 / 3.0 * o->DZI * o->CVISC;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JM = JC - 1, JP = JC + 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * o->CVISC;
        for (int KC = 1; KC <= N; ++KC) {
            int KM = KMV(o, KC), KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC), IM = IMV(o, IC);
                double DUDX = (QV(o, IP, JC, KC, 1) - QV(o, IC, JC, KC, 1)) * o->DXI;
                double DVDY = (QV(o, IC, JP, KC, 2) - QV(o, IC, JC, KC, 2)) * o->DYFI[JJ];
                double DWDZ = (QV(o, IC, JC, KP, 3) - QV(o, IC, JC, KC, 3)) * o->DZI;
                double T33F_EX = F3(o->MU, o, IC, JC, KC) * (DUDX + DVDY);
                double T33F_IM = F3(o->MU, o, IC, JC, KC) * DWDZ;
                DWDZ = (GV(o, IC, JC, KP, 3) * DRV(o, IC, JC, KP, 3) - GV(o, IC, JC, KC, 3) * DRV(o, IC, JC, KC, 3)) * o->DZI;
                double T33F_AD = F3(o->MU, o, IC, JC, KC) * DWDZ;
                DUDX = (QV(o, IP, JC, KM, 1) - QV(o, IC, JC, KM, 1)) * o->DXI;
                DVDY = (QV(o, IC, JP, KM, 2) - QV(o, IC, JC, KM, 2)) * o->DYFI[JJ];
                DWDZ = (QV(o, IC, JC, KC, 3) - QV(o, IC, JC, KM, 3)) * o->DZI;
                double T33B_EX = F3(o->MU, o, IC, JC, KM) * (DUDX + DVDY);
                double T33B_IM = F3(o->MU, o, IC, JC, KM) * DWDZ;
                DWDZ = (GV(o, IC, JC, KC, 3) * DRV(o, IC, JC, KC, 3) - GV(o, IC, JC, KM, 3) * DRV(o, IC, JC, KM, 3)) * o->DZI;
                double T33B_AD = F3(o->MU, o, IC, JC, KM) * DWDZ;
                double D33_EX = (T33F_EX - T33B_EX) * COE3;
                double D33_IM = (T33F_IM - T33B_IM) * COE3 * (-2.0);
                double D33_AD = (T33F_AD - T33B_AD) * COE3 * (-2.0);

                double VIS31P = MSV(o, IP, JC, KC, 2);
                double DWDX = (QV(o, IP, JC, KC, 3) - QV(o, IC, JC, KC, 3)) * o->DXI;
                double DUDZ = (QV(o, IP, JC, KC, 1) - QV(o, IP, JC, KM, 1)) * o->DZI;
                double T31F_EX = VIS31P * DUDZ, T31F_IM = VIS31P * DWDX;
                DWDX = (GV(o, IP, JC, KC, 3) * DRV(o, IP, JC, KC, 3) - GV(o, IC, JC, KC, 3) * DRV(o, IC, JC, KC, 3)) * o->DXI;
                double T31F_AD = VIS31P * DWDX;
                double VIS31C = MSV(o, IC, JC, KC, 2);
                DWDX = (QV(o, IC, JC, KC, 3) - QV(o, IM, JC, KC, 3)) * o->DXI;
                DUDZ = (QV(o, IC, JC, KC, 1) - QV(o, IC, JC, KM, 1)) * o->DZI;
                double T31B_EX = VIS31C * DUDZ, T31B_IM = VIS31C * DWDX;
                DWDX = (GV(o, IC, JC, KC, 3) * DRV(o, IC, JC, KC, 3) - GV(o, IM, JC, KC, 3) * DRV(o, IM, JC, KC, 3)) * o->DXI;
                double T31B_AD = VIS31C * DWDX;
                double D31_EX = (T31F_EX - T31B_EX) * COE1;
                double D31_IM = (T31F_IM - T31B_IM) * COE1;
                double D31_AD = (T31F_AD - T31B_AD) * COE1;

                double VIS32P = MSV(o, IC, JP, KC, 3);
                double DWDY = (QV(o, IC, JP, KC, 3) - QV(o, IC, JC, KC, 3)) * o->DYCI[JJP];
                double DVDZ = (QV(o, IC, JP, KC, 2) - QV(o, IC, JP, KM, 2)) * o->DZI;
                double T32F_EX = VIS32P * DVDZ, T32F_IM = VIS32P * DWDY;
                DWDY = (GV(o, IC, JP, KC, 3) * DRV(o, IC, JP, KC, 3) - GV(o, IC, JC, KC, 3) * DRV(o, IC, JC, KC, 3)) * o->DYCI[JJP];
                double T32F_AD = VIS32P * DWDY;
                double VIS32C = MSV(o, IC, JC, KC, 3);
                DWDY = (QV(o, IC, JC, KC, 3) - QV(o, IC, JM, KC, 3)) * o->DYCI[JJ];
                DVDZ = (QV(o, IC, JC, KC, 2) - QV(o, IC, JC, KM, 2)) * o->DZI;
                double T32B_EX = VIS32C * DVDZ, T32B_IM = VIS32C * DWDY;
                DWDY = (GV(o, IC, JC, KC, 3) * DRV(o, IC, JC, KC, 3) - GV(o, IC, JM, KC, 3) * DRV(o, IC, JM, KC, 3)) * o->DYCI[JJ];
                double T32B_AD = VIS32C * DWDY;
                double D32_EX = (T32F_EX - T32B_EX) * COE2;
                double D32_IM = (T32F_IM - T32B_IM) * COE2;
                double D32_AD = (T32F_AD - T32B_AD) * COE2;

                F3(o->RHSLLPHI, o, IC, JC, KC) = D31_EX + D32_EX + D33_EX + F3(o->RHSLLPHI, o, IC, JC, KC);
                F3(o->RHS, o, IC, JC, KC) = D31_IM + D32_IM + D33_IM;
                F3(o->DIVU, o, IC, JC, KC) = D31_AD + D32_AD + D33_AD;
            }
        }
    }
}

/* MOMFA_io(NS, IDR) (src/MOMFA_io.f90:18-76): x sweep MOMFA1_X_io (:79-172,  */
/* cyclic), z sweep MOMFA2_Z_io (:175-261, cyclic), y sweep MOMFA3_Y_io       */
/* (:264-406, TDMAIJJ_nonCYC with BCJ = 0), then G += RHS for j >= N2I.       */
/* The y-sweep row 1 of the v equation has AMVR(1,2) = APVR(1,2) = 0, so its */
/* coefficients are (0, 1, 0) whatever the densities it divides by; the     */
/* ghost D_STG(:,0,:,2) it reads is taken as the y-periodic halo value      */
/* D_STG(:,M,:,2) that INTFC_VARS3 leaves there in a run of two or more     */
/* ranks.  The v rows use D_STG(j) for the j+1 coupling, as the reference.  */
static void io_momfa(orc_t* o, int NS, int IDR) {
    int L = o->L, M = o->M, N = o->N;
    double FACOE = 0.50 * o->TALP[NS] * o->DT * o->CVISC;
    int N2I = (IDR == 2) ? 2 : 1;
    /* ---- x ---- */
    {
        double COE1 = FACOE * 4.0 / 3.0 * o->DXQI, COE2 = FACOE * o->DXQI;
#pragma omp parallel
        {
            double *A = dalloc(L), *B = dalloc(L), *C = dalloc(L), *R = dalloc(L), *w = dalloc(3 * (size_t)L);
#pragma omp for schedule(static) collapse(2)
            for (int KC = 1; KC <= N; ++KC)
                for (int JC = N2I; JC <= M; ++JC) {
                    for (int IC = 1; IC <= L; ++IC) {
                        int IM = IMV(o, IC), IP = IPV(o, IC);
                        double AMU, APU;
                        if (IDR == 1) {
                            AMU = -COE1 * F3(o->MU, o, IM, JC, KC);
                            APU = -COE1 * F3(o->MU, o, IC, JC, KC);
                        } else if (IDR == 2) {
                            AMU = -COE2 * MSV(o, IC, JC, KC, 1);
                            APU = -COE2 * MSV(o, IP, JC, KC, 1);
                        } else {
                            AMU = -COE2 * MSV(o, IC, JC, KC, 2);
                            APU = -COE2 * MSV(o, IP, JC, KC, 2);
                        }
                        A[IC - 1] = AMU / DSV(o, IM, JC, KC, IDR);
                        C[IC - 1] = APU / DSV(o, IP, JC, KC, IDR);
                        B[IC - 1] = 1.0 - (AMU + APU) / DSV(o, IC, JC, KC, IDR);
                        R[IC - 1] = F3(o->RHS, o, IC, JC, KC);
                    }
                    tdma_cyc_line(L, A, B, C, R, w);
                    for (int IC = 1; IC <= L; ++IC) F3(o->RHS, o, IC, JC, KC) = R[IC - 1];
                }
            free(A); free(B); free(C); free(R); free(w);
        }
    }
    /* ---- z ---- */
    {
        double COE1 = FACOE * 4.0 / 3.0 * o->DZQI, COE2 = FACOE * o->DZQI;
#pragma omp parallel
        {
            double *A = dalloc(N), *B = dalloc(N), *C = dalloc(N), *R = dalloc(N), *w = dalloc(3 * (size_t)N);
#pragma omp for schedule(static) collapse(2)
            for (int JC = N2I; JC <= M; ++JC)
                for (int IC = 1; IC <= L; ++IC) {
                    for (int KC = 1; KC <= N; ++KC) {
                        int KM = KMV(o, KC), KP = KPV(o, KC);
                        double AMU, APU;
                        if (IDR == 1) {
                            AMU = -COE2 * MSV(o, IC, JC, KC, 2) * 1.0;
                            APU = -COE2 * MSV(o, IC, JC, KP, 2) * 1.0;
                        } else if (IDR == 2) {
                            AMU = -COE2 * MSV(o, IC, JC, KC, 3) * 1.0;
                            APU = -COE2 * MSV(o, IC, JC, KP, 3) * 1.0;
                        } else {
                            AMU = -COE1 * F3(o->MU, o, IC, JC, KM) * 1.0;
                            APU = -COE1 * F3(o->MU, o, IC, JC, KC) * 1.0;
                        }
                        A[KC - 1] = AMU / DSV(o, IC, JC, KM, IDR);
                        C[KC - 1] = APU / DSV(o, IC, JC, KP, IDR);
                        B[KC - 1] = 1.0 - (AMU + APU) / DSV(o, IC, JC, KC, IDR);
                        R[KC - 1] = F3(o->RHS, o, IC, JC, KC);
                    }
                    tdma_cyc_line(N, A, B, C, R, w);
                    for (int KC = 1; KC <= N; ++KC) F3(o->RHS, o, IC, JC, KC) = R[KC - 1];
                }
            free(A); free(B); free(C); free(R); free(w);
        }
    }
    /* ---- y ---- */
    {
        double COE1 = FACOE * 4.0 / 3.0, COE2 = FACOE;
        const double* AMV = o->AMVR[IDR];
        const double* APV = o->APVR[IDR];
#pragma omp parallel
        {
            double *A = dalloc(M), *B = dalloc(M), *C = dalloc(M), *R = dalloc(M), *w = dalloc(2 * (size_t)M);
#pragma omp for schedule(static) collapse(2)
            for (int KC = 1; KC <= N; ++KC)
                for (int IC = 1; IC <= L; ++IC) {
                    for (int JC = 1; JC <= M; ++JC) {
                        int JM = JC - 1, JP = JC + 1;
                        double AMU, APU, AJ, CJ, BJ;
                        if (IDR == 1 || IDR == 3) {
                            if (JC == 1) {
                                double MUQT = (F3(o->MU, o, IC, JC, KC) + F3(o->MU, o, IC, JM, KC)) * 0.5;
                                AMU = -COE2 * o->AMVR1 * MUQT;
                                APU = -COE2 * APV[JC] * MSV(o, IC, JP, KC, IDR);
                                AJ = 0.0;
                                CJ = APU / DSV(o, IC, JP, KC, IDR);
                            } else if (JC == M) {
                                double MUQT = (F3(o->MU, o, IC, M, KC) + F3(o->MU, o, IC, M + 1, KC)) * 0.5;
                                AMU = -COE2 * AMV[JC] * MSV(o, IC, JC, KC, IDR);
                                APU = -COE2 * o->APVRN * MUQT;
                                AJ = AMU / DSV(o, IC, JM, KC, IDR);
                                CJ = 0.0;
                            } else {
                                AMU = -COE2 * AMV[JC] * MSV(o, IC, JC, KC, IDR);
                                APU = -COE2 * APV[JC] * MSV(o, IC, JP, KC, IDR);
                                AJ = AMU / DSV(o, IC, JM, KC, IDR);
                                CJ = APU / DSV(o, IC, JP, KC, IDR);
                            }
                            BJ = 1.0 - (AMU + APU) / DSV(o, IC, JC, KC, IDR);
                        } else {
                            if (JC == 1) {
                                AMU = -COE1 * AMV[JC] * F3(o->MU, o, IC, JM, KC);
                                APU = -COE1 * APV[JC] * F3(o->MU, o, IC, JC, KC);
                                AJ = AMU / DSV(o, IC, M, KC, 2);  /* D_STG(:,0,:,2): y-periodic halo */
                                CJ = APU / DSV(o, IC, JP, KC, 2);
                                BJ = 1.0 - (AMU + APU) / DSV(o, IC, JC, KC, 2);
                            } else {
                                AMU = -COE1 * AMV[JC] * F3(o->MU, o, IC, JM, KC);
                                APU = -COE1 * APV[JC] * F3(o->MU, o, IC, JC, KC);
                                AJ = AMU / DSV(o, IC, JM, KC, 2);
                                CJ = APU / DSV(o, IC, JC, KC, 2);
                                BJ = 1.0 - (AMU + APU) / DSV(o, IC, JC, KC, 2);
                            }
                        }
                        A[JC - 1] = AJ; B[JC - 1] = BJ; C[JC - 1] = CJ;
                        R[JC - 1] = F3(o->RHS, o, IC, JC, KC);
                    }
                    tdma_noncyc_line(M, A, B, C, R, w);
                    for (int JC = 1; JC <= M; ++JC) F3(o->RHS, o, IC, JC, KC) = R[JC - 1];
                }
            free(A); free(B); free(C); free(R); free(w);
        }
    }
#pragma omp parallel for schedule(static)
    for (int K = 1; K <= N; ++K)
        for (int J = N2I; J <= M; ++J)
            for (int I = 1; I <= L; ++I) GV(o, I, J, K, IDR) = F3(o->RHS, o, I, J, K) + GV(o, I, J, K, IDR);
}

/* SOLVERRK3_MOM_io(NS) (src/SOLVERRK3_MOM_IO.f90:11-120), explicit or      */
/* Crank-Nicolson viscous scheme (orc_io_set_vis_scheme).                  */
/* The pressure Poisson equation is the one FISHPACK_POIS3D_SIMPLE solves */
/* (same AMPH/ACPH/APPH operator and x/z eigenvalues); its singular       */
/* kx = kz = 0 mode is fixed here as in FFT99 (phi_hat(y_1) = 0), which    */
/* changes DPH and PR by an x-z-y constant only.                           */
int orc_io_substep(orc_t* o, int NS) {
    if (!o->io || NS < 0 || NS > 3) return -1;
    if (o->thermal) memcpy(o->G0, o->G, 3 * FSZ(o) * sizeof(double));  /* G0_io = G_io (:25) */
    io_velocity_calc(o);
    io_convection_x(o);
    io_convection_y(o);
    io_convection_z(o);
    if (!o->ivis) {
        io_divg_u(o);
        io_viscous_x(o);
        io_rhs_mom_explicit(o, NS, 1);
        io_viscous_y(o);
        io_rhs_mom_explicit(o, NS, 2);
        io_viscous_z(o);
        io_rhs_mom_explicit(o, NS, 3);
        io_massflux_calc(o);
    } else {
        io_viscous_par_x(o);
        io_rhs_mom_explicit(o, NS, 1);
        io_momfa(o, NS, 1);
        io_viscous_par_y(o);
        io_rhs_mom_explicit(o, NS, 2);
        io_momfa(o, NS, 2);
        io_viscous_par_z(o);
        io_rhs_mom_explicit(o, NS, 3);
        io_momfa(o, NS, 3);
    }
    io_bc_wall_g(o);
    io_divg(o, NS);
    memset(o->DPH, 0, FSZ(o) * sizeof(double));
    poisson(o, o->RHSLLPHI, o->DPH);
    bc_wall_scalar(o, o->DPH);
    io_prcalc_massflux_update(o, NS);
    io_velocity_calc(o);
    return 0;
}


/* ====================================================================== */
/* Thermal solver of the IO domain (SOLVE.f90:119-128): SOLVERRK3_ENG_io    */
/* (src/SOLVERRK3_ENG_IO.f90:11-82) with RHS_ENERGY_EXPLICIT               */
/* (src/RHS_ENERGY_EXPLICIT.f90:11-155), THERM_PROP_UPDATE(IMAIND) by table */
/* search, BC_WALL_THERMAL with constant wall heat flux on both walls       */
/* (BC_WALL_Isoflux, src/BC_WALL.f90:541-619), then DENSITY_TIME_DERIVATION */
/* (src/DIVG.f90:249-317), DENSITY_Staggered and MU_Staggered.  Plane      */
/* channel: RCCI1 = RCCI2 = RNDI1 = 1.                                     */
/* ====================================================================== */
int orc_prop_point(void* tab, double dh, double* out);
void orc_table_dh_limits(void* tab, double* out);

static void thermal_point(orc_t* o, int I, int J, int K) {
    double v[6];
    if (orc_prop_point(o->tab, F3(o->DH, o, I, J, K), v)) o->prop_err = 1;
    F3(o->ENTH, o, I, J, K) = v[0];
    F3(o->TEMP, o, I, J, K) = v[1];
    F3(o->DEN, o, I, J, K) = v[2];
    F3(o->MU, o, I, J, K) = v[3];
    F3(o->KAPPA, o, I, J, K) = v[4];
    F3(o->HCP, o, I, J, K) = v[5];
}

/* THERM_PROP_UPDATE(IMAIND): rows 1..M */
static void thermal_props_interior(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    for (int J = 1; J <= M; ++J)
        for (int I = 1; I <= L; ++I)
            for (int K = 1; K <= N; ++K) thermal_point(o, I, J, K);
}

/* BC_WALL_IsoTHERMAL (src/BC_WALL.f90:484-538): the ghost row holds the wall state; DH = H * D */
static void thermal_wall_state(orc_t* o, int w, int I, int J, int K) {
    F3(o->TEMP, o, I, J, K) = o->WV[w][0];
    F3(o->ENTH, o, I, J, K) = o->WV[w][1];
    F3(o->DEN, o, I, J, K) = o->WV[w][2];
    F3(o->MU, o, I, J, K) = o->WV[w][3];
    F3(o->KAPPA, o, I, J, K) = o->WV[w][4];
    F3(o->DH, o, I, J, K) = F3(o->ENTH, o, I, J, K) * F3(o->DEN, o, I, J, K);
}

/* BC_WALL_THERMAL (src/BC_WALL.f90:622-643): per wall BC_WALL_Isoflux (:541-619, ghost rho*h
 * extrapolated, then its properties) or BC_WALL_IsoTHERMAL; columns NCL1S..NCL1E */
static void thermal_bc(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    for (int I = 1 - o->xo; I <= L + o->xo; ++I)
        for (int K = 1; K <= N; ++K) {
            if (o->iso[1]) {
                thermal_wall_state(o, 1, I, M + 1, K);
                continue;
            }
            F3(o->DH, o, I, M + 1, K) = 2.0 * F3(o->DH, o, I, M, K) - o->WFF[M] * F3(o->DH, o, I, M, K) -
                                        o->WFB[M] * F3(o->DH, o, I, M - 1, K);
            thermal_point(o, I, M + 1, K);
        }
    for (int I = 1 - o->xo; I <= L + o->xo; ++I)
        for (int K = 1; K <= N; ++K) {
            if (o->iso[0]) {
                thermal_wall_state(o, 0, I, 0, K);
                continue;
            }
            F3(o->DH, o, I, 0, K) = 2.0 * F3(o->DH, o, I, 1, K) - o->WFF[2] * F3(o->DH, o, I, 2, K) -
                                    o->WFB[2] * F3(o->DH, o, I, 1, K);
            thermal_point(o, I, 0, K);
        }
}

/* RHS_ENERGY_EXPLICIT, constant heat flux on both walls */
static void rhs_energy_explicit(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    const double XND2CL = 0.5, ZND2CL = 0.5, CTHECD = o->CTHECD;
    const double COE1 = o->DXI * XND2CL * 0.5;
    const double COE11 = o->DXQI * XND2CL * CTHECD;
    const double WF_BOT = o->QW_BOT, WF_TOP = -o->QW_TOP; /* WALLFLUX (src/Flow_State.f90:150-175) */
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JP = JC + 1, JM = JC - 1, JJ = JC, JJP = JJ + 1;
        double COE2 = o->DYFI[JJ] * 1.0 * 0.5;
        double COE3 = o->DZI * ZND2CL * 1.0 * 0.5;
        double COE33 = o->DZQI * ZND2CL * 1.0 * CTHECD;
        double COE22 = o->DYFI[JJ] * 1.0 * CTHECD;
        double COE221, COE222;
        if (JJ == 1) {  /* src/RHS_ENERGY_EXPLICIT.f90:50-66 */
            COE221 = o->DYCI[JJP] / 1.0;
            COE222 = o->iso[0] ? o->DYCI[JJ] / 1.0 : 1.0 / 1.0;
        } else if (JJ == M) {  /* :68-77 */
            COE222 = o->DYCI[JJ] / 1.0;
            COE221 = o->iso[1] ? o->DYCI[JJP] / 1.0 : 1.0 / 1.0;
        } else {
            COE221 = o->DYCI[JJP] / 1.0;
            COE222 = o->DYCI[JJ] / 1.0;
        }
        for (int IC = 1; IC <= L; ++IC) {
            int IP = IPV(o, IC), IM = IMV(o, IC);
            for (int KC = 1; KC <= N; ++KC) {
                int KP = KPV(o, KC), KM = KMV(o, KC);
#define HH(i, j, k) F3(o->ENTH, o, i, j, k)
#define TT(i, j, k) F3(o->TEMP, o, i, j, k)
#define KK(i, j, k) F3(o->KAPPA, o, i, j, k)
                double DX_DHU = (HH(IP, JC, KC) + HH(IC, JC, KC)) * (GV(o, IP, JC, KC, 1) + GV(o, IP, JC, KC, 1)) -
                                (HH(IC, JC, KC) + HH(IM, JC, KC)) * (GV(o, IC, JC, KC, 1) + GV(o, IC, JC, KC, 1));
                DX_DHU = DX_DHU * COE1;
                double DY_DHV = (o->WFF[JJP] * HH(IC, JP, KC) + o->WFB[JJP] * HH(IC, JC, KC)) *
                                    (GV(o, IC, JP, KC, 2) + GV(o, IC, JP, KC, 2)) -
                                (o->WFF[JJ] * HH(IC, JC, KC) + o->WFB[JJ] * HH(IC, JM, KC)) *
                                    (GV(o, IC, JC, KC, 2) + GV(o, IC, JC, KC, 2));
                DY_DHV = DY_DHV * COE2;
                double DZ_DHW = (HH(IC, JC, KP) + HH(IC, JC, KC)) * (GV(o, IC, JC, KP, 3) + GV(o, IC, JC, KP, 3)) -
                                (HH(IC, JC, KC) + HH(IC, JC, KM)) * (GV(o, IC, JC, KC, 3) + GV(o, IC, JC, KC, 3));
                DZ_DHW = DZ_DHW * COE3;
                double DX_KDT = (KK(IP, JC, KC) + KK(IC, JC, KC)) * (TT(IP, JC, KC) - TT(IC, JC, KC)) -
                                (KK(IC, JC, KC) + KK(IM, JC, KC)) * (TT(IC, JC, KC) - TT(IM, JC, KC));
                DX_KDT = DX_KDT * COE11;
                double KDTy1 = (o->WFF[JJP] * KK(IC, JP, KC) + o->WFB[JJP] * KK(IC, JC, KC)) *
                               (TT(IC, JP, KC) - TT(IC, JC, KC)) * COE221;
                double KDTy2 = (o->WFF[JJ] * KK(IC, JC, KC) + o->WFB[JJ] * KK(IC, JM, KC)) *
                               (TT(IC, JC, KC) - TT(IC, JM, KC)) * COE222;
                if (JJ == 1 && !o->iso[0]) KDTy2 = -WF_BOT * COE222;
                else if (JJ == M && !o->iso[1]) KDTy1 = -WF_TOP * COE221;
                double DY_KDT = (KDTy1 - KDTy2) * COE22;
                double DZ_KDT = (KK(IC, JC, KP) + KK(IC, JC, KC)) * (TT(IC, JC, KP) - TT(IC, JC, KC)) -
                                (KK(IC, JC, KM) + KK(IC, JC, KC)) * (TT(IC, JC, KC) - TT(IC, JC, KM));
                DZ_KDT = DZ_KDT * COE33;
                F3(o->RHSE, o, IC, JC, KC) = -DX_DHU - DY_DHV - DZ_DHW + DX_KDT + DY_KDT + DZ_KDT;
#undef HH
#undef TT
#undef KK
            }
        }
    }
}

/* DENSITY_TIME_DERIVATION(NS) */
static void density_time_derivation(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
#pragma omp parallel for schedule(static)
    for (int JC = 1; JC <= M; ++JC) {
        int JP = JC + 1, JJ = JC;
        double COE2 = o->DYFI[JJ] * 1.0, COE3 = o->DZI * 1.0;
        for (int IC = 1; IC <= L; ++IC) {
            int IP = IPV(o, IC);
            for (int KC = 1; KC <= N; ++KC) {
                int KP = KPV(o, KC);
                size_t fs = FSZ(o);
#define G0V(i, j, k, c) (o->G0[FOFF(o, i, j, k) + (size_t)((c) - 1) * fs])
                double DIVX = (GV(o, IP, JC, KC, 1) - GV(o, IC, JC, KC, 1)) * o->DXI;
                double DIVX0 = (G0V(IP, JC, KC, 1) - G0V(IC, JC, KC, 1)) * o->DXI;
                double DIVY = (GV(o, IC, JP, KC, 2) - GV(o, IC, JC, KC, 2)) * COE2;
                double DIVY0 = (G0V(IC, JP, KC, 2) - G0V(IC, JC, KC, 2)) * COE2;
                double DIVZ = (GV(o, IC, JC, KP, 3) - GV(o, IC, JC, KC, 3)) * COE3;
                double DIVZ0 = (G0V(IC, JC, KP, 3) - G0V(IC, JC, KC, 3)) * COE3;
#undef G0V
                F3(o->DRHODT, o, IC, JC, KC) = -o->TGAM[NS] * (DIVX + DIVY + DIVZ) - o->TROH[NS] * (DIVX0 + DIVY0 + DIVZ0);
            }
        }
    }
}

/* BC_TINLET_THERML (src/BC_INLET.f90:64-84): the inlet ghost column holds the inlet state */
static void xio_thermal_inlet(orc_t* o) {
    int M = o->M, N = o->N;
    for (int J = 0; J <= M + 1; ++J)
        for (int K = 1; K <= N; ++K) {
            F3(o->TEMP, o, 0, J, K) = o->XIN[0];
            F3(o->KAPPA, o, 0, J, K) = o->XIN[4];
            F3(o->DEN, o, 0, J, K) = o->XIN[2];
            F3(o->MU, o, 0, J, K) = o->XIN[3];
            F3(o->HCP, o, 0, J, K) = o->XIN[5];
            F3(o->DH, o, 0, J, K) = o->XIN[6];
            F3(o->ENTH, o, 0, J, K) = o->XIN[1];
        }
}

/* BC_COUTLET_ENEG_RK3(NS) (src/BC_COUTLET_ENEG_RK3.f90:11-59): U_OUTLET of CONVCTION_OUTLET_U on  */
/* the current velocity, the convective RK3 update of the outlet column's rho*h with BC_CONV0_ENG, */
/* the table limiter, then THERM_PROP_UPDATE(IOULET) (rows 1..M of column L+1)                    */
static void xio_energy_outlet(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
    double UxMax = -1.0E20, UxMin = 1.0E20;
    for (int K = 1; K <= N; ++K)
        for (int J = 1; J <= M; ++J) {
            double UCC = (QV(o, L, J, K, 1) + QV(o, L + 1, J, K, 1)) * 0.5;
            if (UCC > UxMax) UxMax = UCC;
            if (UCC < UxMin) UxMin = UCC;
        }
    double U_OUTLET = 0.5 * (UxMax + UxMin);
    const double REALMIN = 1.0e-14;
    for (int K = 1; K <= N; ++K)
        for (int J = 1; J <= M; ++J) {
            double BC_CONV = -o->DXI * U_OUTLET * (F3(o->DH, o, L + 1, J, K) - F3(o->DH, o, L, J, K));
            double* b0 = o->BCCONV0E + (size_t)(J - 1) + (size_t)M * (size_t)(K - 1);
            double BC_RHS = o->TGAM[NS] * BC_CONV + o->TROH[NS] * (*b0);
            *b0 = BC_CONV;
            F3(o->DH, o, L + 1, J, K) = F3(o->DH, o, L + 1, J, K) + o->DT * BC_RHS;
        }
    for (int K = 1; K <= N; ++K)
        for (int J = 1; J <= M; ++J) {
            double d = F3(o->DH, o, L + 1, J, K);
            d = fmin(o->DHMAX - REALMIN, d);
            d = fmax(o->DHMIN + REALMIN, d);
            F3(o->DH, o, L + 1, J, K) = d;
        }
    for (int J = 1; J <= M; ++J)
        for (int K = 1; K <= N; ++K) thermal_point(o, L + 1, J, K);
}

/* The inlet state of a thermal TG + main-domain run: v = T, H, D, M, K, CP, DH (applied at once) */
int orc_xio_thermal_inlet(orc_t* o, const double* v) {
    if (!o->xo || !o->thermal) return -1;
    for (int a = 0; a < 7; ++a) o->XIN[a] = v[a];
    o->xin_set = 1;
    xio_thermal_inlet(o);
    return 0;
}

/* Energy part of RK substep NS and the property / density coupling that
 * precedes SOLVERRK3_MOM_io(NS).  Returns nonzero when a point fell outside
 * the property table (the reference STOPs there). */
int orc_thermal_substep(orc_t* o, int NS) {
    if (!o->thermal || NS < 1 || NS > 3) return -1;
    int L = o->L, M = o->M, N = o->N;
    size_t fs = FSZ(o);
    memcpy(o->MU0, o->MU, fs * sizeof(double));   /* Viscousity0 = Viscousity */
    memcpy(o->RHO, o->DEN, fs * sizeof(double));  /* DENSITY0 = DENSITY */
    double COE1 = o->TGAM[NS] * o->DT, COE0 = o->TROH[NS] * o->DT;
    rhs_energy_explicit(o);
    const double REALMIN = 1.0e-14;
    for (int J = 1; J <= M; ++J)
        for (int I = 1; I <= L; ++I)
            for (int K = 1; K <= N; ++K) {
                double d = F3(o->DH, o, I, J, K) + COE1 * F3(o->RHSE, o, I, J, K) + COE0 * F3(o->RHSE0, o, I, J, K);
                d = fmin(o->DHMAX - REALMIN, d);
                d = fmax(o->DHMIN + REALMIN, d);
                F3(o->DH, o, I, J, K) = d;
                F3(o->RHSE0, o, I, J, K) = F3(o->RHSE, o, I, J, K);
            }
    o->prop_err = 0;
    thermal_props_interior(o);
    if (o->xo) {
        xio_thermal_inlet(o);
        xio_energy_outlet(o, NS);
    }
    thermal_bc(o);
    density_time_derivation(o, NS);
    io_staggered_props(o);
    if (o->ivis) io_density_implicit_add(o);
    return o->prop_err;
}

/* Starts the thermal solver on an IO state set by orc_io_set_fields: DH
 * (padded field, rows 1..M used) with the table-search properties, constant
 * nondimensional wall heat fluxes qw_bot, qw_top (WALLFLUX = +qw_bot at the
 * bottom, -qw_top at the top) and CTHECD = 1 / (REN PRT0).  Properties of
 * the interior and, through BC_WALL_Isoflux, of the wall ghosts follow from
 * DH; DENSITY0 = DENSITY, Viscousity0 = Viscousity, RHS_ENERGY0 = 0 (SOLVE.f90:40),
 * G0_io = G_io; D_STG, MU_STG and the velocity are recomputed. */
int orc_thermal_enable(orc_t* o, void* tab, const double* DH, double qw_bot, double qw_top, double cthecd) {
    if (!o->io || !tab) return -1;
    size_t fs = FSZ(o);
    if (!o->thermal) {
        o->DH = dalloc(fs); o->ENTH = dalloc(fs); o->TEMP = dalloc(fs); o->KAPPA = dalloc(fs); o->HCP = dalloc(fs);
        o->RHSE = dalloc(fs); o->RHSE0 = dalloc(fs); o->G0 = dalloc(3 * fs);
    }
    o->thermal = 1;
    o->tab = tab;
    o->QW_BOT = qw_bot; o->QW_TOP = qw_top; o->CTHECD = cthecd;
    double lim[2];
    orc_table_dh_limits(tab, lim);
    o->DHMIN = lim[0]; o->DHMAX = lim[1];
    memcpy(o->DH, DH, fs * sizeof(double));
    memset(o->RHSE0, 0, fs * sizeof(double));
    o->prop_err = 0;
    thermal_props_interior(o);
    if (o->xo) { /* the inlet and outlet columns from their given rho*h */
        for (int J = 1; J <= o->M; ++J)
            for (int K = 1; K <= o->N; ++K) {
                thermal_point(o, 0, J, K);
                thermal_point(o, o->L + 1, J, K);
            }
        memset(o->BCCONV0E, 0, (size_t)o->M * (size_t)o->N * sizeof(double));
    }
    thermal_bc(o);
    memcpy(o->MU0, o->MU, fs * sizeof(double));
    memcpy(o->RHO, o->DEN, fs * sizeof(double));
    memcpy(o->G0, o->G, 3 * fs * sizeof(double));
    io_staggered_props(o);
    io_velocity_calc(o);
    return o->prop_err;
}

/* BC_Fixed_Temperature on wall w (0 bottom, 1 top) with the wall state v = T, H, D, M, K, or the
 * constant heat flux of orc_thermal_enable again (v NULL); the wall's ghost row is set at once */
int orc_thermal_set_isothermal(orc_t* o, int w, const double* v) {
    if (!o->thermal || w < 0 || w > 1) return -1;
    o->iso[w] = v != NULL;
    if (v)
        for (int a = 0; a < 5; ++a) o->WV[w][a] = v[a];
    o->prop_err = 0;
    thermal_bc(o);
    return o->prop_err;
}

/* thermal fields: out = DH, ENTHALPY, TEMPERATURE, DENSITY, Viscousity, THERMCONDT, HEATCAP (7 padded fields) */
void orc_thermal_get(const orc_t* o, double* out) {
    size_t fs = FSZ(o);
    const double* src[7] = {o->DH, o->ENTH, o->TEMP, o->DEN, o->MU, o->KAPPA, o->HCP};
    for (int a = 0; a < 7; ++a) memcpy(out + a * fs, src[a], fs * sizeof(double));
}

/* DIVGCK_io (src/DIVGCK.f90:60-121) via DIVGCK_Comm_io (:125-184), x-periodic:
 * max |div G + DrhoDtP|, loop order JC, KC, IC. */
double orc_io_divgck(const orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    double DIVMAX = 0.0;
    for (int JC = 1; JC <= M; ++JC) {
        int JP = JC + 1, JJ = JC;
        double COE2 = o->DYFI[JJ] * 1.0, COE3 = o->DZI * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KP = KPV(o, KC);
            for (int IC = 1; IC <= L; ++IC) {
                int IP = IPV(o, IC);
                double DIVX = (GV(o, IP, JC, KC, 1) - GV(o, IC, JC, KC, 1)) * o->DXI;
                double DIVY = (GV(o, IC, JP, KC, 2) - GV(o, IC, JC, KC, 2)) * COE2;
                double DIVZ = (GV(o, IC, JC, KP, 3) - GV(o, IC, JC, KC, 3)) * COE3;
                double DTRHO = F3(o->DRHODT, o, IC, JC, KC);
                double DQCAP = DIVX + DIVY + DIVZ + DTRHO;
                DIVMAX = fmax(fabs(DQCAP), DIVMAX);
            }
        }
    }
    return DIVMAX;
}

/* CFL_io (src/CFL.f90:55-107), including the viscous number */
double orc_io_cfl(orc_t* o) {
    int L = o->L, M = o->M, N = o->N;
    double CFLMA = 0.0;
    for (int K = 1; K <= N; ++K) {
        int KP = KPV(o, K);
        for (int J = 1; J <= M; ++J) {
            int JP = J + 1, JJ = J;
            for (int I = 1; I <= L; ++I) {
                int IP = IPV(o, I);
                double QCF = (fabs((QV(o, I, J, K, 1) + QV(o, IP, J, K, 1)) * o->DXI) +
                              fabs((QV(o, I, J, K, 2) + QV(o, I, JP, K, 2)) * o->DYFI[JJ] * 1.0) +
                              fabs((QV(o, I, J, K, 3) + QV(o, I, J, KP, 3)) * o->DZI * 1.0)) * 0.5;
                double VCF = 2.0 * o->CVISC * (o->DXQI + o->DZQI * 1.0 + o->DYFI[JJ] * o->DYFI[JJ]) * F3(o->MU, o, I, J, K) /
                             F3(o->DEN, o, I, J, K);
                QCF = fmax(QCF, VCF);
                CFLMA = fmax(CFLMA, QCF);
            }
        }
    }
    o->CFLMM_IO = CFLMA;
    return CFLMA;
}

/* One step of SOLVE for the IO domain: CFL_io, dt rule, three substeps. */
int orc_io_run_steps(orc_t* o, int nsteps, double* cfl_dt) {
    for (int s = 0; s < nsteps; ++s) {
        double c = orc_io_cfl(o);
        double dt = fmin(fmin(o->DT0, 5.0 * o->DT), o->CFLGV / c);
        dt = fmax(dt, o->DTMIN);
        o->DT = dt;
        if (cfl_dt) cfl_dt[s] = c * dt;
        if ((dt / o->DT0) < 0.01) return 1;
        for (int NS = 1; NS <= 3; ++NS) {
            if (o->thermal && orc_thermal_substep(o, NS)) return 2;
            orc_io_substep(o, NS);
        }
    }
    return 0;
}

/* ====================================================================== */
/* Main domain with inflow and outflow (iDomain = 3: TgFlowFlg and        */
/* IoFlowFlg), flow and (orc_xio_thermal_inlet) the thermal solver,       */
/* explicit viscous terms.  x runs over 0..L+1: the inlet ghost column 0   */
/* and the inlet face u(1) come from the periodic TG domain each substep  */
/* (BC_TINLET_FLOW), the outlet column L+1 takes a convective update      */
/* (BC_COUTLET_MOM_RK3), and the pressure Poisson equation is FISHPACK's  */
/* with BCX_io = (2, 1).                                                    */
/* ====================================================================== */

/* BC_TINLET_FLOW (src/BC_INLET.f90:12-61), rows J = 0..M+1 */
static void xio_inlet(orc_t* o, const orc_t* tg) {
    int M = o->M, N = o->N, LT = tg->L;
    for (int J = 0; J <= M + 1; ++J)
        for (int K = 1; K <= N; ++K) {
            double D0 = F3(o->RHO, o, 0, J, K);
            QV(o, 0, J, K, 1) = QV(tg, LT, J, K, 1);
            QV(o, 1, J, K, 1) = QV(tg, 1, J, K, 1);
            GV(o, 0, J, K, 1) = QV(o, 0, J, K, 1) * D0;
            GV(o, 1, J, K, 1) = QV(o, 1, J, K, 1) * D0;
            QV(o, 0, J, K, 2) = QV(tg, LT, J, K, 2);
            GV(o, 0, J, K, 2) = QV(o, 0, J, K, 2) * D0;
            QV(o, 0, J, K, 3) = QV(tg, LT, J, K, 3);
            GV(o, 0, J, K, 3) = QV(o, 0, J, K, 3) * D0;
            F3(o->PR, o, 0, J, K) = F3(tg->PR, tg, LT, J, K);
        }
    for (int J = 0; J <= M + 1; ++J)
        for (int K = 1; K <= N; ++K) F3(o->DPH, o, 0, J, K) = 0.0;
}

#define BCV(o, j, k, c) ((o)->BCCONV0[(size_t)((j) - 1) + (size_t)(o)->M * ((size_t)((k) - 1) + (size_t)(o)->N * (size_t)((c) - 1))])

/* BC_COUTLET_MOM_RK3(NS) (src/BC_COUTLET_MOM_RK3.f90:16-112) with U_OUTLET of CONVCTION_OUTLET_U  */
/* (:115-192, method two: the mean of the largest and smallest outlet u) and the outflow scaling */
/* of CHK_MassConsv_io (src/processing/CHK_conservation.f90:11-79, method 1).                   */
static void xio_outlet(orc_t* o, int NS) {
    int L = o->L, M = o->M, N = o->N;
    double UxMax = -1.0E20, UxMin = 1.0E20;
    for (int K = 1; K <= N; ++K)
        for (int J = 1; J <= M; ++J) {
            double UCC = (QV(o, L, J, K, 1) + QV(o, L + 1, J, K, 1)) * 0.5;
            if (UCC > UxMax) UxMax = UCC;
            if (UCC < UxMin) UxMin = UCC;
        }
    o->U_OUTLET = 0.5 * (UxMax + UxMin);
    double COE1 = o->DXI * o->U_OUTLET;
    for (int IDR = 1; IDR <= 3; ++IDR) {
        int N2I = IDR == 2 ? 2 : 1;
        for (int K = 1; K <= N; ++K)
            for (int J = N2I; J <= M; ++J) {
                double BC_CONV = -(GV(o, L + 1, J, K, IDR) - GV(o, L, J, K, IDR)) * COE1;
                double BC_RHS = o->TGAM[NS] * BC_CONV + o->TROH[NS] * BCV(o, J, K, IDR);
                BCV(o, J, K, IDR) = BC_CONV;
                GV(o, L + 1, J, K, IDR) = GV(o, L + 1, J, K, IDR) + o->DT * BC_RHS;
                double RHO = (F3(o->RHO, o, L, J, K) + F3(o->RHO, o, L + 1, J, K)) * 0.5;
                QV(o, L + 1, J, K, IDR) = GV(o, L + 1, J, K, IDR) / RHO;
            }
    }
    /* CHK_MassConsv_io: inlet and outlet (NCL1E = L+1) fluxes, and the mass rate of the interior */
    double FluxIntg_INL = 0.0, FluxIntg_OUT = 0.0, MASS_RATE_INTG = 0.0;
    for (int JC = 1; JC <= M; ++JC) {
        double COE2 = 1.0 / o->DYFI[JC] / 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            FluxIntg_INL = FluxIntg_INL + GV(o, 1, JC, KC, 1) * COE2;
            FluxIntg_OUT = FluxIntg_OUT + GV(o, L + 1, JC, KC, 1) * COE2;
        }
    }
    FluxIntg_INL = FluxIntg_INL / o->DZI;
    FluxIntg_OUT = FluxIntg_OUT / o->DZI;
    for (int JC = 1; JC <= M; ++JC) {
        double COE2 = 1.0 / o->DYFI[JC] / 1.0;
        for (int KC = 1; KC <= N; ++KC)
            for (int IC = 1; IC <= L; ++IC) MASS_RATE_INTG = F3(o->DRHODT, o, IC, JC, KC) * COE2 + MASS_RATE_INTG;
    }
    MASS_RATE_INTG = MASS_RATE_INTG / o->DZI / o->DXI;
    o->MASS_SCALING = (FluxIntg_INL - MASS_RATE_INTG) / FluxIntg_OUT;
    for (int J = 1; J <= M; ++J)
        for (int K = 1; K <= N; ++K) {
            GV(o, L + 1, J, K, 1) = GV(o, L + 1, J, K, 1) * (o->MASS_SCALING - 1.0) + GV(o, L + 1, J, K, 1);
            double RHO = (F3(o->RHO, o, L, J, K) + F3(o->RHO, o, L + 1, J, K)) * 0.5;
            QV(o, L + 1, J, K, 1) = GV(o, L + 1, J, K, 1) / RHO;
        }
    io_bc_wall_g(o);
    bc_wall_q(o);
}

/* The x and z eigenvalues of the FISHPACK solve as positive numbers: AKX(I) = -XRT(I) (LP = 5),   */
/* and -YRT of the periodic z direction (MP = 1): 4 DZQI sin^2(pi kz / N) for the complex mode kz */
/* (the RFFTF half-complex pair of wavenumber min(kz, N-kz) shares one root, :118-124).            */
static double xio_akz(const orc_t* o, int kz) {
    int kk = kz <= o->N - kz ? kz : o->N - kz;
    double PI = 2.0 * asin(1.0), DY = PI / (2.0 * (double)o->N);
    double sn = sin((double)(2 * kk) * DY);
    return 4.0 * o->DZQI * (sn * sn);
}
double orc_xio_akz(const orc_t* o, int kz) { return xio_akz(o, kz); }
double orc_xio_akx(const orc_t* o, int I) { return o->AKX ? o->AKX[I] : 0.0; }

/* FISHPACK_POIS3D_SIMPLE (src/possion3d_fishpack.f90:344-460) with LPEROD = 4 (BCX_io = (2, 1):  */
/* x(0) = x(2), x(L+1) = 0) and MPEROD = 0 (periodic z).  The transforms are written as the sums  */
/* FFTPACK defines them by:                                                                       */
/*   COSQF  X(m) = x(1) + sum_{p=2..L} 2 x(p) cos((2m-1)(p-1) pi / (2L))                          */
/*   COSQB  x(p) = sum_{m=1..L} 4 X(m) cos((2m-1)(p-1) pi / (2L))                                 */
/* and the z pair RFFTF/RFFTB as the complex DFT of the real line (its half-complex half).  TRID0 */
/* (:309-340) solves each (m, kz) line with BB = ACPH + XRT(m)/RCCI2 + YRT(kz); no x mode is       */
/* singular (XRT < 0), so its zero-pivot branch is not taken.  The result is scaled by            */
/* 1/(SCALX*SCALY) = 1/(4 L N) (1/N applied after the forward z transform).                        */
static void poisson_xinout(orc_t* o, const double* src, double* dst) {
    int L = o->L, M = o->M, N = o->N;
    double UN3M = 1.0 / (double)N;
    double PI = 2.0 * asin(1.0);
    int Q4 = 4 * L;
    double* cq = dalloc((size_t)Q4);
    for (int q = 0; q < Q4; ++q) cq[q] = cos((double)q * PI / (double)(2 * L));
    cplx* wfz = fft_table(N, -1);
    cplx* wbz = fft_table(N, +1);
    double* SRe = o->SRe;
    double* SIm = o->SIm;
#define SXM(I, J, K) ((size_t)((I) - 1) + (size_t)L * ((size_t)((J) - 1) + (size_t)M * (size_t)((K) - 1)))
#pragma omp parallel
    {
        int nmax = L > N ? L : N;
        cplx* a = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
        cplx* b = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for schedule(static)
        for (int J = 1; J <= M; ++J) {
            for (int K = 1; K <= N; ++K)
                for (int m = 1; m <= L; ++m) {
                    double X = F3(src, o, 1, J, K);
                    for (int p = 2; p <= L; ++p) X = X + 2.0 * F3(src, o, p, J, K) * cq[((2 * m - 1) * (p - 1)) % Q4];
                    SRe[SXM(m, J, K)] = X;
                }
            for (int m = 1; m <= L; ++m) {
                for (int K = 1; K <= N; ++K) { a[K - 1].re = SRe[SXM(m, J, K)]; a[K - 1].im = 0.0; }
                fft_rec(N, a, 1, b, -1, wfz, 1);
                for (int K = 1; K <= N; ++K) {
                    SRe[SXM(m, J, K)] = b[K - 1].re * UN3M;
                    SIm[SXM(m, J, K)] = b[K - 1].im * UN3M;
                }
            }
        }
        free(a); free(b);
    }
#pragma omp parallel
    {
        double* D = dalloc((size_t)M);
        double* T = dalloc((size_t)M);
        double* BB = dalloc((size_t)M);
#pragma omp for schedule(static)
        for (int K = 1; K <= N; ++K) {
            double YRT = -xio_akz(o, K - 1);
            for (int m = 1; m <= L; ++m) {
                double XRT = -o->AKX[m];
                for (int J = 1; J <= M; ++J) BB[J - 1] = o->ACPH[J] + XRT / 1.0 + YRT;
                for (int part = 0; part < 2; ++part) {
                    double* S = part ? SIm : SRe;
                    for (int J = 1; J <= M; ++J) T[J - 1] = S[SXM(m, J, K)];
                    /* TRID0 */
                    int NR = M, MM1 = NR - 1;
                    double Z = 1.0 / BB[0];
                    D[0] = o->APPH[1] * Z;
                    T[0] = T[0] * Z;
                    for (int I = 2; I <= MM1; ++I) {
                        Z = 1.0 / (BB[I - 1] - o->AMPH[I] * D[I - 2]);
                        D[I - 1] = o->APPH[I] * Z;
                        T[I - 1] = (T[I - 1] - o->AMPH[I] * T[I - 2]) * Z;
                    }
                    Z = BB[NR - 1] - o->AMPH[NR] * D[MM1 - 1];
                    if (fabs(Z) > 1.0E-14) T[NR - 1] = (T[NR - 1] - o->AMPH[NR] * T[MM1 - 1]) / Z;
                    else T[NR - 1] = 0.0;
                    for (int IP = 1; IP <= MM1; ++IP) {
                        int I = NR - IP;
                        T[I - 1] = T[I - 1] - D[I - 1] * T[I];
                    }
                    for (int J = 1; J <= M; ++J) S[SXM(m, J, K)] = T[J - 1];
                }
            }
        }
        free(D); free(T); free(BB);
    }
#pragma omp parallel
    {
        int nmax = L > N ? L : N;
        cplx* a = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
        cplx* b = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for schedule(static)
        for (int J = 1; J <= M; ++J) {
            for (int m = 1; m <= L; ++m) {
                for (int K = 1; K <= N; ++K) { a[K - 1].re = SRe[SXM(m, J, K)]; a[K - 1].im = SIm[SXM(m, J, K)]; }
                fft_rec(N, a, 1, b, +1, wbz, 1);
                for (int K = 1; K <= N; ++K) SRe[SXM(m, J, K)] = b[K - 1].re;
            }
            for (int K = 1; K <= N; ++K)
                for (int p = 1; p <= L; ++p) {
                    double x = 0.0;
                    for (int m = 1; m <= L; ++m) x = x + 4.0 * SRe[SXM(m, J, K)] * cq[((2 * m - 1) * (p - 1)) % Q4];
                    F3(dst, o, p, J, K) = x / (double)Q4;
                }
        }
        free(a); free(b);
    }
#undef SXM
    free(cq); free(wfz); free(wbz);
}

/* SOLVERRK3_MOM_io(NS) with TgFlowFlg (src/SOLVERRK3_MOM_IO.f90:11-120), iVisScheme = 0 */
int orc_xio_substep(orc_t* o, const orc_t* tg, int NS) {
    if (!o->io || !o->xo || tg->xo || tg->M != o->M || tg->N != o->N || NS < 1 || NS > 3 || o->ivis)
        return -1;
    if (o->thermal) memcpy(o->G0, o->G, 3 * FSZ(o) * sizeof(double));  /* G0_io = G_io (:25) */
    io_velocity_calc(o);
    xio_inlet(o, tg);
    xio_outlet(o, NS);
    io_convection_x(o);
    io_convection_y(o);
    io_convection_z(o);
    io_divg_u(o);
    io_viscous_x(o);
    io_rhs_mom_explicit(o, NS, 1);
    io_viscous_y(o);
    io_rhs_mom_explicit(o, NS, 2);
    io_viscous_z(o);
    io_rhs_mom_explicit(o, NS, 3);
    io_massflux_calc(o);
    io_bc_wall_g(o);
    io_divg(o, NS);
    memset(o->DPH, 0, FSZ(o) * sizeof(double));
    poisson_xinout(o, o->RHSLLPHI, o->DPH);
    bc_wall_scalar(o, o->DPH);
    io_prcalc_massflux_update(o, NS);
    io_velocity_calc(o);
    return 0;
}

/* The SOLVE loop of a TG + main-domain run (src/SOLVE.f90:75-134): CFL_tg and CFL_io, DT from  */
/* CFLMM = max of the two (the dt rule of BCAST_COMM_STEP, :154-211), then per NS the TG substep */
/* and the main-domain substep.  cfl_dt[s] = CFLMM * DT of step s.                               */
int orc_xio_run_steps(orc_t* o, orc_t* tg, int nsteps, double* cfl_dt) {
    for (int s = 0; s < nsteps; ++s) {
        double ctg = orc_cfl(tg), cio = orc_io_cfl(o);
        double c = fmax(ctg, cio);
        double dt = fmin(fmin(o->DT0, 5.0 * o->DT), o->CFLGV / c);
        dt = fmax(dt, o->DTMIN);
        o->DT = dt;
        tg->DT = dt;
        if (cfl_dt) cfl_dt[s] = c * dt;
        if ((dt / o->DT0) < 0.01) return 1;
        for (int NS = 1; NS <= 3; ++NS) {
            orc_substep(tg, NS);
            if (o->thermal) {
                if (!o->xin_set) return 3;
                if (orc_thermal_substep(o, NS)) return 4;
            }
            if (orc_xio_substep(o, tg, NS)) return 2;
        }
    }
    return 0;
}

/* DIVGCK_io with TgFlowFlg (src/DIVGCK.f90:60-100): MAXDIVGV_io(1:3) over the cells 2..L-1, */
/* 0..1 and L of DIVGCK_Comm_io (|div G + DrhoDtP|).                                         */
static double xio_divmax(const orc_t* o, int I0, int I1) {
    int M = o->M, N = o->N;
    double DIVMAX = 0.0;
    for (int JC = 1; JC <= M; ++JC) {
        double COE2 = o->DYFI[JC] * 1.0;
        for (int KC = 1; KC <= N; ++KC) {
            int KP = KPV(o, KC);
            for (int IC = I0; IC <= I1; ++IC) {
                int IP = IC + 1;
                double DIVX = (GV(o, IP, JC, KC, 1) - GV(o, IC, JC, KC, 1)) * o->DXI;
                double DIVY = (GV(o, IC, JC + 1, KC, 2) - GV(o, IC, JC, KC, 2)) * COE2;
                double DIVZ = (GV(o, IC, JC, KP, 3) - GV(o, IC, JC, KC, 3)) * o->DZI;
                double DQCAP = DIVX + DIVY + DIVZ + F3(o->DRHODT, o, IC, JC, KC);
                DIVMAX = fmax(fabs(DQCAP), DIVMAX);
            }
        }
    }
    return DIVMAX;
}
void orc_xio_divgck(const orc_t* o, double* out) {
    out[0] = xio_divmax(o, 2, o->L - 1);
    out[1] = xio_divmax(o, 0, 1);
    out[2] = xio_divmax(o, o->L, o->L);
}
void orc_xio_outlet_state(const orc_t* o, double* out) {
    out[0] = o->U_OUTLET;
    out[1] = o->MASS_SCALING;
}
/* Poisson solve alone (tests): rhs and dph are (0:L+1, 0:M+1, N) fields, interior rows used. */
void orc_xio_poisson(orc_t* o, const double* rhs, double* dph) {
    memset(dph, 0, FSZ(o) * sizeof(double));
    poisson_xinout(o, rhs, dph);
}

/* Monitor quantities of PP_MONITOR_Xperiodic_io (src/processing/
 * PP_SCN_MONITOR.f90:255-625) that follow from the instantaneous x-z means
 * of PP_MEAN_ZX_FLOW_Xperiodic_io (src/processing/PP_MEAN_ZX.f90:311-883):
 * out[0] Uc = <G1>/<D> at j = M/2, out[1] u'u'_c, out[2] u'v'_c,
 * out[3] Gmaxx = max_j |<G1>|, out[4] bulk G (G1BULK). Cell-centred values:
 * G_CCT(1) = (G1(i) + G1(i+1))/2, G_CCT(2) = (G2(j) + G2(j+1))/2, likewise U. */
void orc_io_monitor(orc_t* o, double* out) {
    int L = o->L, M = o->M, N = o->N;
    double VL1313 = 1.0 / (double)(L * N);
    double gmax = 0.0, uc = 0, uu = 0, uv = 0, g1c = 0, dc = 0;
    double rate = 0.0;
    for (int J = 1; J <= M; ++J) {
        double G1 = 0, G2 = 0, UG1 = 0, UG2 = 0, D1 = 0;
        for (int I = 1; I <= L; ++I) {
            int IP = IPV(o, I);
            for (int K = 1; K <= N; ++K) {
                double gc1 = (GV(o, I, J, K, 1) + GV(o, IP, J, K, 1)) * 0.5;
                double uc1 = (QV(o, I, J, K, 1) + QV(o, IP, J, K, 1)) * 0.5;
                double gc2 = ((GV(o, I, J, K, 2) + GV(o, I, J + 1, K, 2)) * 1.0) * 0.5;
                G1 += gc1;
                G2 += gc2;
                UG1 += uc1 * gc1;
                UG2 += uc1 * gc2;
                D1 += F3(o->DEN, o, I, J, K);
            }
        }
        G1 *= VL1313; G2 *= VL1313; UG1 *= VL1313; UG2 *= VL1313; D1 *= VL1313;
        gmax = fmax(gmax, fabs(G1));
        rate += G1 / o->DYFI[J];
        if (J == M / 2) {
            g1c = G1; dc = D1;
            uc = G1 / D1;
            uu = UG1 - G1 * G1 / D1;
            uv = UG2 - G1 * G2 / D1;
        }
    }
    (void)g1c; (void)dc;
    out[0] = uc; out[1] = uu; out[2] = uv; out[3] = gmax; out[4] = rate / 2.0;
}


/* ====================================================================== */
/* Statistics of the periodic channel (POSTPROCESS_TG).  The means of one  */
/* set are stored as out[122*M]: U1xzL(M,4) | UPxzL(M,3) | U2xzL(M,6) |    */
/* U3xzL(M,10) | DVDL1xzL(M,3,3) | DVDLPxzL(M,3,3) | DVDL2xzL(M,9,9),      */
/* Fortran order (j fastest).  Plane channel: RCCI1 = RNDI1 = 1.           */
/* ====================================================================== */
#define PPA(arr, off, J, c) (arr)[(size_t)((off) + (c)) * M + (size_t)((J) - 1)]

/* PP_MEAN_ZX_FLOW_TG (src/processing/PP_MEAN_ZX.f90:14-307), loop order J, I, K */
void orc_pp_mean_zx_tg(const orc_t* o, double* out) {
    const int L = o->L, M = o->M, N = o->N;
    const double VL = 1.0 / (double)(L * N);
    const double COE0 = VL, COE1 = VL * 0.5, COE2 = VL * (0.5 * 0.5), COE3 = VL * (0.5 * 0.5 * 0.5);
    double COG1[3][3] = {{VL * o->DXI, VL * 0.25, VL * 0.25 * o->DZI},
                         {VL * 0.25 * o->DXI, VL, VL * 0.25 * o->DZI},
                         {VL * 0.25 * o->DXI, VL * 0.25, VL * o->DZI}};
#pragma omp parallel for schedule(static)
    for (int J = 1; J <= M; ++J) {
        const int JP = J + 1, JM = J - 1, JJ = J, JJP = J + 1;
        double U1[4] = {0}, UP[3] = {0}, U2[6] = {0}, U3[10] = {0}, D1[3][3] = {{0}}, DP[3][3] = {{0}};
        double D2[9][9];
        memset(D2, 0, sizeof(D2));
        for (int I = 1; I <= L; ++I) {
            const int IP = IPV(o, I), IM = IMV(o, I);
            for (int K = 1; K <= N; ++K) {
                const int KP = KPV(o, K), KM = KMV(o, K);
                double U[3], UJP[3], UJM[3], UKP[3], UKM[3], UIP[3], UIM[3];
                U[0] = QV(o, I, J, K, 1) + QV(o, IP, J, K, 1);
                UJP[0] = QV(o, I, JP, K, 1) + QV(o, IP, JP, K, 1);
                UJM[0] = QV(o, I, JM, K, 1) + QV(o, IP, JM, K, 1);
                UKP[0] = QV(o, I, J, KP, 1) + QV(o, IP, J, KP, 1);
                UKM[0] = QV(o, I, J, KM, 1) + QV(o, IP, J, KM, 1);
                U[2] = (QV(o, I, J, K, 3) + QV(o, I, J, KP, 3)) * 1.0;
                UIP[2] = (QV(o, IP, J, K, 3) + QV(o, IP, J, KP, 3)) * 1.0;
                UIM[2] = (QV(o, IM, J, K, 3) + QV(o, IM, J, KP, 3)) * 1.0;
                UJP[2] = (QV(o, I, JP, K, 3) + QV(o, I, JP, KP, 3)) * 1.0;
                UJM[2] = (QV(o, I, JM, K, 3) + QV(o, I, JM, KP, 3)) * 1.0;
                U[1] = (QV(o, I, J, K, 2) + QV(o, I, JP, K, 2)) * 1.0;
                UIP[1] = (QV(o, IP, J, K, 2) + QV(o, IP, JP, K, 2)) * 1.0;
                UIM[1] = (QV(o, IM, J, K, 2) + QV(o, IM, JP, K, 2)) * 1.0;
                UKP[1] = (QV(o, I, J, KP, 2) + QV(o, I, JP, KP, 2)) * 1.0;
                UKM[1] = (QV(o, I, J, KM, 2) + QV(o, I, JP, KM, 2)) * 1.0;
                const double P = F3(o->PR, o, I, J, K);
                for (int m = 0; m < 3; ++m) {
                    U1[m] = U1[m] + U[m];
                    UP[m] = UP[m] + U[m] * P;
                }
                U1[3] = U1[3] + P;
                for (int m = 1; m <= 3; ++m)
                    for (int n = m; n <= 3; ++n) {
                        int l = (m * (7 - m)) / 2 + n - 3;
                        U2[l - 1] = U2[l - 1] + U[m - 1] * U[n - 1];
                    }
                for (int m = 1; m <= 3; ++m)
                    for (int n = m; n <= 3; ++n)
                        for (int h = n; h <= 3; ++h) {
                            int l = m * (6 - m) + (n * (7 - n)) / 2 + h - 8;
                            U3[l - 1] = U3[l - 1] + U[m - 1] * U[n - 1] * U[h - 1];
                        }
                double D[3][3];
                D[0][0] = QV(o, IP, J, K, 1) - QV(o, I, J, K, 1);
                D[0][1] = (UJP[0] - U[0]) * o->DYCI[JJP] + (U[0] - UJM[0]) * o->DYCI[JJ];
                D[0][2] = UKP[0] - UKM[0];
                D[1][0] = UIP[1] - UIM[1];
                D[1][1] = (QV(o, I, JP, K, 2) * 1.0 - QV(o, I, J, K, 2) * 1.0) * o->DYFI[JJ];
                D[1][2] = UKP[1] - UKM[1];
                D[2][0] = UIP[2] - UIM[2];
                D[2][1] = (UJP[2] - U[2]) * o->DYCI[JJP] + (U[2] - UJM[2]) * o->DYCI[JJ];
                D[2][2] = QV(o, I, J, KP, 3) * 1.0 - QV(o, I, J, K, 3) * 1.0;
                for (int m = 0; m < 3; ++m)
                    for (int n = 0; n < 3; ++n) {
                        D1[m][n] = D1[m][n] + D[m][n];
                        DP[m][n] = DP[m][n] + D[m][n] * P;
                    }
                for (int m = 0; m < 3; ++m)
                    for (int h = 0; h < 3; ++h)
                        for (int n = 0; n < 3; ++n)
                            for (int p = 0; p < 3; ++p) D2[m * 3 + h][n * 3 + p] = D2[m * 3 + h][n * 3 + p] + D[m][h] * D[n][p];
            }
        }
        PPA(out, 0, J, 3) = U1[3] * COE0;
        for (int m = 0; m < 3; ++m) PPA(out, 0, J, m) = U1[m] * COE1;
        for (int m = 0; m < 3; ++m) PPA(out, 4, J, m) = UP[m] * COE1;
        for (int l = 0; l < 6; ++l) PPA(out, 7, J, l) = U2[l] * COE2;
        for (int l = 0; l < 10; ++l) PPA(out, 13, J, l) = U3[l] * COE3;
        for (int m = 0; m < 3; ++m)
            for (int n = 0; n < 3; ++n) {
                PPA(out, 23, J, m + 3 * n) = D1[m][n] * COG1[m][n];
                PPA(out, 32, J, m + 3 * n) = DP[m][n] * COG1[m][n];
            }
        for (int l1 = 0; l1 < 9; ++l1)
            for (int l2 = 0; l2 < 9; ++l2)
                PPA(out, 41, J, l1 + 9 * l2) = D2[l1][l2] * (COG1[l1 / 3][l1 % 3] * COG1[l2 / 3][l2 % 3]);
    }
}

/* ====================================================================== */
/* Statistics of the main domain: PP_MEAN_ZX_FLOW_Xperiodic_io           */
/* (src/processing/PP_MEAN_ZX.f90:311-796), plane channel (RCCI1 = RNDI1 */
/* = 1, no pipe-centre branch).  One set is out[NIO*M], Fortran order     */
/* with j fastest, the module arrays in the order the reference zeroes    */
/* them: U1xzL_io(M,4) | G1xzL_io(M,3) | UPxzL_io(M,3) | U2xzL_io(M,6) |   */
/* UGxzL_io(M,6) | U3xzL_io(M,10) | UGUxzL_io(M,10) | DVDL1xzL_io(M,3,3) | */
/* DVDLPxzL_io(M,3,3) | DVDL2xzL_io(M,9,9)  (141 per row), then with the  */
/* thermal solver: T1 | D1 | H1 | M1 | T2 | D2 | H2 | DH | PH (M each) |  */
/* DVDL1MxzL_io(M,3,3) | DVDL1MHxzL_io(M,3,3) | DVDL1MUxzL_io(M,3,3,3) |   */
/* DVDL2MxzL_io(M,9,9) | UHxzL_io(M,3) | GHxzL_io(M,3) | U2DHxzL_io(M,6) | */
/* DhDL1xzL_io(M,3) | DhDLPxzL_io(M,3) | DTDLKxzL_io(M,3) |               */
/* DTDLKUxzL_io(M,3,3) | DTDLKDVDLxzL_io(M,3,3,3) | DHDLMDVDLxzL_io(M,3,3,3) */
/* (219 more).  Loop order J, I, K as the reference; every product in its */
/* left-to-right order.                                                   */
/* ====================================================================== */
int orc_pp_io_per_row(const orc_t* o) { return o->thermal ? 360 : 141; }

void orc_pp_mean_zx_io(const orc_t* o, double* out) {
    const int L = o->L, M = o->M, N = o->N;
    const double VL = 1.0 / (double)(L * N);  /* VL1313_io */
    const int th = o->thermal;
#pragma omp parallel for schedule(static)
    for (int J = 1; J <= M; ++J) {
        const int JP = J + 1, JM = J - 1, JJ = J, JJP = J + 1;
        double U1[4] = {0}, G1[3] = {0}, UP[3] = {0}, U2[6] = {0}, UG[6] = {0}, U3[10] = {0}, UGU[10] = {0};
        double D1[3][3] = {{0}}, DP[3][3] = {{0}}, D2[9][9];
        double T1 = 0, Dn1 = 0, H1 = 0, M1 = 0, T2 = 0, Dn2 = 0, H2 = 0, DHs = 0, PHs = 0;
        double D1M[3][3] = {{0}}, D1MH[3][3] = {{0}}, D1MU[3][3][3], D2M[9][9];
        double UH[3] = {0}, GH[3] = {0}, U2DH[6] = {0}, HD1[3] = {0}, HDP[3] = {0}, TK[3] = {0}, TKU[3][3] = {{0}};
        double TKD[3][3][3], HMD[3][3][3];
        memset(D2, 0, sizeof(D2)); memset(D2M, 0, sizeof(D2M)); memset(D1MU, 0, sizeof(D1MU));
        memset(TKD, 0, sizeof(TKD)); memset(HMD, 0, sizeof(HMD));
        for (int I = 1; I <= L; ++I) {
            const int IP = IPV(o, I), IM = IMV(o, I);
            for (int K = 1; K <= N; ++K) {
                const int KP = KPV(o, K), KM = KMV(o, K);
                double G[3], U[3], UJP[3], UJM[3], UKP[3], UKM[3], UIP[3], UIM[3];
                G[0] = (GV(o, I, J, K, 1) + GV(o, IP, J, K, 1)) * 0.5;
                U[0] = (QV(o, I, J, K, 1) + QV(o, IP, J, K, 1)) * 0.5;
                UJP[0] = (QV(o, I, JP, K, 1) + QV(o, IP, JP, K, 1)) * 0.5;
                UJM[0] = (QV(o, I, JM, K, 1) + QV(o, IP, JM, K, 1)) * 0.5;
                UKP[0] = (QV(o, I, J, KP, 1) + QV(o, IP, J, KP, 1)) * 0.5;
                UKM[0] = (QV(o, I, J, KM, 1) + QV(o, IP, J, KM, 1)) * 0.5;
                G[2] = ((GV(o, I, J, K, 3) + GV(o, I, J, KP, 3)) * 1.0) * 0.5;
                U[2] = ((QV(o, I, J, K, 3) + QV(o, I, J, KP, 3)) * 1.0) * 0.5;
                UIP[2] = ((QV(o, IP, J, K, 3) + QV(o, IP, J, KP, 3)) * 1.0) * 0.5;
                UIM[2] = ((QV(o, IM, J, K, 3) + QV(o, IM, J, KP, 3)) * 1.0) * 0.5;
                UJP[2] = ((QV(o, I, JP, K, 3) + QV(o, I, JP, KP, 3)) * 1.0) * 0.5;
                UJM[2] = ((QV(o, I, JM, K, 3) + QV(o, I, JM, KP, 3)) * 1.0) * 0.5;
                G[1] = ((GV(o, I, J, K, 2) + GV(o, I, JP, K, 2)) * 1.0) * 0.5;
                U[1] = ((QV(o, I, J, K, 2) + QV(o, I, JP, K, 2)) * 1.0) * 0.5;
                UIP[1] = ((QV(o, IP, J, K, 2) + QV(o, IP, JP, K, 2)) * 1.0) * 0.5;
                UIM[1] = ((QV(o, IM, J, K, 2) + QV(o, IM, JP, K, 2)) * 1.0) * 0.5;
                UKP[1] = ((QV(o, I, J, KP, 2) + QV(o, I, JP, KP, 2)) * 1.0) * 0.5;
                UKM[1] = ((QV(o, I, J, KM, 2) + QV(o, I, JP, KM, 2)) * 1.0) * 0.5;
                const double P = F3(o->PR, o, I, J, K);
                for (int m = 0; m < 3; ++m) {
                    U1[m] = U1[m] + U[m];
                    G1[m] = G1[m] + G[m];
                    UP[m] = UP[m] + U[m] * P;
                }
                U1[3] = U1[3] + P;
                for (int m = 1; m <= 3; ++m)
                    for (int n = m; n <= 3; ++n) {
                        const int l = (m * (7 - m)) / 2 + n - 3;
                        UG[l - 1] = UG[l - 1] + U[m - 1] * G[n - 1];
                        U2[l - 1] = U2[l - 1] + U[m - 1] * U[n - 1];
                    }
                for (int m = 1; m <= 3; ++m)
                    for (int n = m; n <= 3; ++n)
                        for (int h = n; h <= 3; ++h) {
                            const int l = m * (6 - m) + (n * (7 - n)) / 2 + h - 8;
                            UGU[l - 1] = UGU[l - 1] + U[m - 1] * G[n - 1] * U[h - 1];
                        }
                for (int m = 1; m <= 3; ++m)
                    for (int n = m; n <= 3; ++n)
                        for (int h = n; h <= 3; ++h) {
                            const int l = m * (6 - m) + (n * (7 - n)) / 2 + h - 8;
                            U3[l - 1] = U3[l - 1] + U[m - 1] * U[n - 1] * U[h - 1];
                        }
                double D[3][3];
                D[0][0] = (QV(o, IP, J, K, 1) - QV(o, I, J, K, 1)) * o->DXI;
                D[0][2] = (UKP[0] - UKM[0]) * o->DZI * 0.5;
                D[0][1] = ((UJP[0] - U[0]) * o->DYCI[JJP] + (U[0] - UJM[0]) * o->DYCI[JJ]) * 0.5;
                D[1][0] = (UIP[1] - UIM[1]) * o->DXI * 0.5;
                D[1][2] = (UKP[1] - UKM[1]) * o->DZI * 0.5;
                D[1][1] = (QV(o, I, JP, K, 2) * 1.0 - QV(o, I, J, K, 2) * 1.0) * o->DYFI[JJ];
                D[2][2] = (QV(o, I, J, KP, 3) * 1.0 - QV(o, I, J, K, 3) * 1.0) * o->DZI;
                D[2][0] = (UIP[2] - UIM[2]) * o->DXI * 0.5;
                D[2][1] = ((UJP[2] - U[2]) * o->DYCI[JJP] + (U[2] - UJM[2]) * o->DYCI[JJ]) * 0.5;
                for (int m = 0; m < 3; ++m)
                    for (int n = 0; n < 3; ++n) {
                        D1[m][n] = D1[m][n] + D[m][n];
                        DP[m][n] = DP[m][n] + D[m][n] * P;
                    }
                for (int m = 0; m < 3; ++m)
                    for (int h = 0; h < 3; ++h)
                        for (int n = 0; n < 3; ++n)
                            for (int p = 0; p < 3; ++p) D2[m * 3 + h][n * 3 + p] = D2[m * 3 + h][n * 3 + p] + D[m][h] * D[n][p];
                if (!th) continue;
                const double Tc = F3(o->TEMP, o, I, J, K), Dc = F3(o->DEN, o, I, J, K);
                const double Hc = F3(o->ENTH, o, I, J, K), MUc = F3(o->MU, o, I, J, K);
                const double Kc = F3(o->KAPPA, o, I, J, K);
                T1 = T1 + Tc; Dn1 = Dn1 + Dc; H1 = H1 + Hc; M1 = M1 + MUc;
                T2 = T2 + Tc * Tc; Dn2 = Dn2 + Dc * Dc; H2 = H2 + Hc * Hc;
                DHs = DHs + Hc * Dc;
                PHs = PHs + Hc * P;
                double HDL[3], TDL[3];
                HDL[0] = (F3(o->ENTH, o, IP, J, K) - F3(o->ENTH, o, IM, J, K)) * o->DXI * 0.5;
                HDL[2] = (F3(o->ENTH, o, I, J, KP) - F3(o->ENTH, o, I, J, KM)) * o->DZI * 0.5;
                HDL[1] = ((F3(o->ENTH, o, I, JP, K) - F3(o->ENTH, o, I, J, K)) * o->DYCI[JJP] +
                          (F3(o->ENTH, o, I, J, K) - F3(o->ENTH, o, I, JM, K)) * o->DYCI[JJ]) * 0.5;
                TDL[0] = (F3(o->TEMP, o, IP, J, K) - F3(o->TEMP, o, IM, J, K)) * o->DXI * 0.5;
                TDL[2] = (F3(o->TEMP, o, I, J, KP) - F3(o->TEMP, o, I, J, KM)) * o->DZI * 0.5;
                TDL[1] = ((F3(o->TEMP, o, I, JP, K) - F3(o->TEMP, o, I, J, K)) * o->DYCI[JJP] +
                          (F3(o->TEMP, o, I, J, K) - F3(o->TEMP, o, I, JM, K)) * o->DYCI[JJ]) * 0.5;
                for (int m = 0; m < 3; ++m)
                    for (int n = 0; n < 3; ++n) {
                        D1M[m][n] = D1M[m][n] + D[m][n] * MUc;
                        D1MH[m][n] = D1MH[m][n] + D[m][n] * MUc * Hc;
                        for (int h = 0; h < 3; ++h) D1MU[m][n][h] = D1MU[m][n][h] + D[m][n] * MUc * U[h];
                    }
                for (int m = 0; m < 3; ++m)
                    for (int h = 0; h < 3; ++h)
                        for (int n = 0; n < 3; ++n)
                            for (int p = 0; p < 3; ++p)
                                D2M[m * 3 + h][n * 3 + p] = D2M[m * 3 + h][n * 3 + p] + D[m][h] * D[n][p] * MUc;
                for (int m = 0; m < 3; ++m) {
                    UH[m] = UH[m] + Hc * U[m];
                    GH[m] = GH[m] + Hc * G[m];
                    HD1[m] = HD1[m] + HDL[m];
                    HDP[m] = HDP[m] + HDL[m] * P;
                    TK[m] = TK[m] + TDL[m] * Kc;
                    for (int n = 0; n < 3; ++n) {
                        TKU[m][n] = TKU[m][n] + TDL[m] * Kc * U[n];
                        for (int h = 0; h < 3; ++h) {
                            TKD[m][n][h] = TKD[m][n][h] + TDL[m] * Kc * D[n][h];
                            HMD[m][n][h] = HMD[m][n][h] + HDL[m] * MUc * D[n][h];
                        }
                    }
                }
                for (int m = 1; m <= 3; ++m)
                    for (int n = m; n <= 3; ++n) {
                        const int l = (m * (7 - m)) / 2 + n - 3;
                        U2DH[l - 1] = U2DH[l - 1] + Dc * Hc * U[m - 1] * U[n - 1];
                    }
            }
        }
        int off = 0;
#define PUT(v) (out[(size_t)(off++) * M + (size_t)(J - 1)] = (v) * VL)
        for (int m = 0; m < 4; ++m) PUT(U1[m]);
        for (int m = 0; m < 3; ++m) PUT(G1[m]);
        for (int m = 0; m < 3; ++m) PUT(UP[m]);
        for (int l = 0; l < 6; ++l) PUT(U2[l]);
        for (int l = 0; l < 6; ++l) PUT(UG[l]);
        for (int l = 0; l < 10; ++l) PUT(U3[l]);
        for (int l = 0; l < 10; ++l) PUT(UGU[l]);
        for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(D1[m][n]);
        for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(DP[m][n]);
        for (int l2 = 0; l2 < 9; ++l2) for (int l1 = 0; l1 < 9; ++l1) PUT(D2[l1][l2]);
        if (th) {
            PUT(T1); PUT(Dn1); PUT(H1); PUT(M1); PUT(T2); PUT(Dn2); PUT(H2); PUT(DHs); PUT(PHs);
            for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(D1M[m][n]);
            for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(D1MH[m][n]);
            for (int h = 0; h < 3; ++h) for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(D1MU[m][n][h]);
            for (int l2 = 0; l2 < 9; ++l2) for (int l1 = 0; l1 < 9; ++l1) PUT(D2M[l1][l2]);
            for (int m = 0; m < 3; ++m) PUT(UH[m]);
            for (int m = 0; m < 3; ++m) PUT(GH[m]);
            for (int l = 0; l < 6; ++l) PUT(U2DH[l]);
            for (int m = 0; m < 3; ++m) PUT(HD1[m]);
            for (int m = 0; m < 3; ++m) PUT(HDP[m]);
            for (int m = 0; m < 3; ++m) PUT(TK[m]);
            for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(TKU[m][n]);
            for (int h = 0; h < 3; ++h) for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(TKD[m][n][h]);
            for (int h = 0; h < 3; ++h) for (int n = 0; n < 3; ++n) for (int m = 0; m < 3; ++m) PUT(HMD[m][n][h]);
        }
#undef PUT
    }
}

/* PP_MEAN_T_TG(TP) (src/processing/PP_MEAN_T.f90:343-392) on a set of means */
void orc_pp_mean_t_tg(int M, int tp, int pp_instn_sz, const double* inst, double* avg, int* nstatis) {
    *nstatis = *nstatis + 1;
    double COE2, COE3;
    if (tp == 1) {
        COE2 = 1.0 / (double)(*nstatis);
        COE3 = (double)(*nstatis - 1) / (double)(*nstatis);
    } else {
        COE2 = 1.0 / (double)pp_instn_sz;
        COE3 = 1.0;
    }
    for (size_t q = 0; q < (size_t)122 * M; ++q) avg[q] = COE3 * avg[q] + COE2 * inst[q];
}

/* PP_MONITOR_TG quantities (src/processing/PP_SCN_MONITOR.f90:165-226) and
 * U1mean_WORK_tg, U1maxx_WORK_tg (PP_MEAN_ZX.f90:294-305); mon[20] */
void orc_pp_monitor_tg(const orc_t* o, const double* inst, const double* avg, double REN, double* mon) {
    const int M = o->M;
    double mean = 0.0, mx = 0.0;
    for (int J = 1; J <= M; ++J) {
        mean = mean + PPA(inst, 0, J, 0) / o->DYFI[J] / 1.0;
        mx = fmax(mx, fabs(PPA(inst, 0, J, 0)));
    }
    mean = mean / o->DZI * (double)o->N / o->Area_inlet;
    const int JS = M / 2;
    mon[0] = PPA(inst, 0, JS, 0); mon[1] = PPA(avg, 0, JS, 0);
    mon[2] = PPA(inst, 0, JS, 1); mon[3] = PPA(avg, 0, JS, 1);
    mon[4] = PPA(inst, 0, JS, 2); mon[5] = PPA(avg, 0, JS, 2);
    mon[6] = PPA(inst, 7, JS, 0) - PPA(inst, 0, JS, 0) * PPA(inst, 0, JS, 0);
    mon[7] = PPA(avg, 7, JS, 0) - PPA(avg, 0, JS, 0) * PPA(avg, 0, JS, 0);
    mon[8] = PPA(inst, 7, JS, 1) - PPA(inst, 0, JS, 0) * PPA(inst, 0, JS, 1);
    mon[9] = PPA(avg, 7, JS, 1) - PPA(avg, 0, JS, 0) * PPA(avg, 0, JS, 1);
    mon[10] = PPA(inst, 7, JS, 3) - PPA(inst, 0, JS, 1) * PPA(inst, 0, JS, 1);
    mon[11] = PPA(avg, 7, JS, 3) - PPA(avg, 0, JS, 1) * PPA(avg, 0, JS, 1);
    mon[12] = PPA(inst, 7, JS, 5) - PPA(inst, 0, JS, 2) * PPA(inst, 0, JS, 2);
    mon[13] = PPA(avg, 7, JS, 5) - PPA(avg, 0, JS, 2) * PPA(avg, 0, JS, 2);
    double DUDY = (PPA(inst, 0, 1, 0) - 0.0) * o->DYFI[1] * 2.0;
    mon[14] = DUDY * 2.0 / REN;
    DUDY = (PPA(avg, 0, 1, 0) - 0.0) * o->DYFI[1] * 2.0;
    mon[15] = DUDY * 2.0 / REN;
    DUDY = (PPA(inst, 0, M, 0) - 0.0) * o->DYFI[M] * 2.0;
    mon[16] = DUDY * 2.0 / REN;
    DUDY = (PPA(avg, 0, M, 0) - 0.0) * o->DYFI[M] * 2.0;
    mon[17] = DUDY * 2.0 / REN;
    mon[18] = mean;
    mon[19] = mx;
}
#undef PPA
