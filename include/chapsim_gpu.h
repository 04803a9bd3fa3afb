/*
 * chapsim_gpu.h -- C ABI of the B200 implementation of CHAPSim's
 * fractional-step time step for the periodic plane channel (TG domain).
 *
 * The Fortran host (CHAPSim's driver, readdata.ini parser and file I/O)
 * stays unchanged; its subroutine bodies call these entry points through an
 * ISO_C_BINDING shim module.  All arguments are plain C types:
 * array arguments are host pointers to Fortran-ordered FP64 arrays with the
 * reference's shapes, copied with one contiguous transfer each.
 *
 * Every entry point returns CHAPSIM_OK (0) or a negative error code; the
 * shim maps a nonzero code to CALL ERRHDL(msg, MYID) (src/WRTHDL.f90:48-63),
 * which keeps the reference's "log + STOP" behaviour.
 */
#ifndef CHAPSIM_GPU_H
#define CHAPSIM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHAPSIM_OK 0
#define CHAPSIM_ERR_CUDA (-1)        /* a CUDA call failed */
#define CHAPSIM_ERR_NAN (-2)         /* non-finite velocity or dt */
#define CHAPSIM_ERR_DT_COLLAPSE (-3) /* DT/DT0 < 0.01: src/SOLVE.f90:199-207 dumps and STOPs */
#define CHAPSIM_ERR_TABLE_RANGE (-4) /* property table out of range: spline_interpolation_* STOP */
#define CHAPSIM_ERR_TIMEOUT (-5)     /* a bounded device wait expired */
#define CHAPSIM_ERR_BADARG (-6)      /* invalid argument or unsupported grid */
#define CHAPSIM_ERR_NOMEM (-7)       /* device allocation failed */

typedef struct chapsim_ctx chapsim_ctx_t;

/* Grid: NCL1 (NCL1_tg or NCL1_io), NCL2, NCL3 of src/modules.f90 (mesh_info).
 * Only the plane channel (iCase = 1) is accepted, in the periodic TG domain
 * (iDomain = 1), the x-periodic main domain (iDomain = 2), or the main domain of
 * a TG + main-domain run with inflow and outflow (idomain = 3; the TG domain is a
 * separate idomain = 1 context, see chapsim_xinout_attach).
 * L and N must factor into 2s and 3s (FFT lengths), L, M, N must be
 * multiples of 32 between 32 and 384; with idomain = 3, L = NCL1_io is any even
 * number from 4 to 768. */
typedef struct {
    int32_t ncl1;   /* L */
    int32_t ncl2;   /* M */
    int32_t ncl3;   /* N */
    int32_t icase;  /* must be 1 (ICHANL) */
    int32_t idomain;/* 1 (ITG), 2 (IIO, x-periodic main domain) or 3 (main domain with inflow
                       from a TG context and a convective outlet, TgFlowFlg)               */
} chapsim_grid_t;

/* Coefficients computed by the host's set-up routines, passed unchanged.
 * y-arrays are 1-based in Fortran; here element [j-1] holds A(j). */
typedef struct {
    double dxi, dzi, dxqi, dzqi; /* CONSPARA (src/CONSPARA.f90:54-73)            */
    double cvisc;                /* CVISC = 1/REN (src/SOLVE.f90:168)            */
    double volm;                 /* VOLM_tg (src/COORDJR.f90:372-381)            */
    double cf_given;             /* Cf_Given (readdata.ini [fluid])              */
    int32_t iflowdriven;         /* 1 constant mass flux, 2 constant Cf          */
    int32_t pad0;
    const double* dyfi;          /* DYFI(1:NCL2)                                 */
    const double* dyci;          /* DYCI(1:NND2)                                 */
    const double* ycl2nd_wff;    /* YCL2ND_WFF(1:NND2)                           */
    const double* ycl2nd_wfb;    /* YCL2ND_WFB(1:NND2)                           */
    const double* amph;          /* AMPH(1:NCL2) (src/TDMA_COEF.f90:44-65)       */
    const double* acph;          /* ACPH(1:NCL2)                                 */
    const double* apph;          /* APPH(1:NCL2)                                 */
    const double* amvr;          /* AMVR(1:NND2, 1:3), Fortran order             */
    const double* acvr;          /* ACVR(1:NND2, 1:3)                            */
    const double* apvr;          /* APVR(1:NND2, 1:3)                            */
    const double* ak1;           /* AK1(1:NCL1) (src/possion3d_FFT99.f90:180-198);
                                    idomain 3: -XRT(1:NCL1) of FFTPACK_ROOT with
                                    LP = 5 (src/possion3d_fishpack.f90:65-111),
                                    4 DXQI sin^2((I-1/2) pi/(2 NCL1))           */
    const double* ak3;           /* AK3(1:NCL3); idomain 3: -YRT, 4 DZQI
                                    sin^2(pi min(k, NCL3-k)/NCL3), k = 0..NCL3-1 */
    double tgam[4], troh[4], talp[4]; /* CONS_RKCOEF (src/CONS_RKCOEF.f90:25-51) */
    double amvr1, apvrn;         /* AMVR1, APVRN wall-row factors of TDMA_COEF
                                    (src/TDMA_COEF.f90:79-87); read only when
                                    ivisscheme = CHAPSIM_VIS_IMPLICIT          */
} chapsim_coefs_t;

#define CHAPSIM_PREC_FP64 0  /* every field and operation in FP64 (the reference's precision) */
#define CHAPSIM_PREC_MIXED 1 /* FP32 velocity, pressure, CONVH0 and RHS storage; FP32 stencils and
                                Crank-Nicolson sweeps; FP64 Poisson spectrum, y-solve (with the
                                kx = kz = 0 mode), DPH, divergence, projection and bulk-flux sums */

typedef struct {
    int32_t device;          /* CUDA device ordinal                                            */
    int32_t fix_v_wall_row;  /* 0: keep the reference's v-sweep row-1 input (the u increment of
                                the same substep, MOMFA3_Y_tg); 1: zero it                      */
    int32_t precision;       /* CHAPSIM_PREC_FP64 (default) or CHAPSIM_PREC_MIXED (TG domain)  */
    int32_t ivisscheme;      /* iVisScheme of the main domain (iDomain = 2):
                                CHAPSIM_VIS_EXPLICIT (default) or CHAPSIM_VIS_IMPLICIT          */
    int32_t no_pdl;          /* 0 (default): the step's kernels are launched with programmatic
                                dependent launch (each kernel's blocks are scheduled while its
                                predecessor drains); 1: plain launches                         */
    int32_t reserved[3];
} chapsim_opts_t;

#define CHAPSIM_VIS_EXPLICIT 0 /* VisExplicit: VISCOUS_ALL_EXPLT_* + MASSFLUX_CALC_io */
#define CHAPSIM_VIS_IMPLICIT 1 /* VisImplicit: VISCOUS_PAR_EXPLT_* + MOMFA_io (Crank-Nicolson
                                  sweeps with per-point coefficients) + PRCALC_io's CN form */

/* Allocates the device fields and uploads coefficients.  Hooks in after
 * FFT99_POIS3D_INIT (src/DNS_THERMAL.f90:118-130). */
int chapsim_gpu_init(const chapsim_grid_t* grid, const chapsim_coefs_t* coefs, const chapsim_opts_t* opts,
                     chapsim_ctx_t** out);
void chapsim_gpu_finalize(chapsim_ctx_t* ctx);
const char* chapsim_last_error_string(const chapsim_ctx_t* ctx);

/* Field transfer.  q: Q_tg(NCL1, 0:NCL2+1, NCL3, 3); pr: PR_tg(NCL1, 0:NCL2+1, NCL3);
 * convh0: CONVH0_tg(NCL1, NCL2, NCL3, 3) or NULL (upload: zero; download: skipped).
 * Upload also applies BC_WALL_Q_tg / BC_WALL_PR_tg to the ghost planes
 * (src/BC_WALL.f90:212-361).  Called after the host writes a restart or
 * initial field, and before any host consumer of the fields. */
int chapsim_upload_fields(chapsim_ctx_t* ctx, const double* q, const double* pr, const double* convh0);
int chapsim_download_fields(chapsim_ctx_t* ctx, double* q, double* pr, double* convh0);

/* Pipelined field transfer of the periodic channel, for a driver that streams Q and PR from and to host
 * memory every step (the same transfer points as chapsim_upload_fields / chapsim_download_fields,
 * src/SOLVE.f90:75-134; the reference's fields stay in host memory, so it has no copy).  Neither call waits:
 * - chapsim_upload_fields_async starts the H2D copy of q and pr (layouts as above) into one of two device
 *   staging slots.  The next chapsim_advance_tg makes the oldest staged upload the context's fields first
 *   (CONVH0 zero, wall ghosts applied: as chapsim_upload_fields).  With both slots full, a third upload
 *   commits the older one at once.
 * - chapsim_download_fields_async copies the current Q and PR into one of two staging slots on the step
 *   stream and starts their D2H copy into q and pr.
 * - chapsim_io_wait returns when every copy and step issued so far has finished.
 * The host buffers must stay valid and unchanged (upload) or unread (download) until chapsim_io_wait;
 * they should be pinned (cudaHostAlloc / cudaHostRegister), or the copies do not overlap.  The staging
 * slots (4 (3 + 1) FS words of device memory) are allocated by the first call. */
int chapsim_upload_fields_async(chapsim_ctx_t* ctx, const double* q, const double* pr);
int chapsim_download_fields_async(chapsim_ctx_t* ctx, double* q, double* pr);
int chapsim_io_wait(chapsim_ctx_t* ctx);

/* The module variable DT (src/modules.f90 init_info) as seen by the device. */
int chapsim_set_dt(chapsim_ctx_t* ctx, double dt);
int chapsim_get_dt(chapsim_ctx_t* ctx, double* dt);

/* CFL_tg (src/CFL.f90:13-52): CFLMM_tg of the resident velocity. */
int chapsim_cfl_tg(chapsim_ctx_t* ctx, double* cflmm);

/* CFL_tg + the dt rule of BCAST_COMM_STEP (src/SOLVE.f90:79-94,154-211):
 * DT = max(min(DT0, 5*DT, CFLGV/CFLMM), DTMIN) on the device; returns
 * CHAPSIM_ERR_DT_COLLAPSE when DT/DT0 < 0.01. */
int chapsim_step_begin(chapsim_ctx_t* ctx, double dt0, double dtmin, double cflgv, double* dt_out,
                       double* cfl_out);

/* SOLVERRK3_MOM_tg(NS) (src/SOLVERRK3_MOM_tg.f90:13-56), NS = 0..3, with
 * the device-resident DT.  NS = 0 is the initial projection step of
 * CALC_INITIALIZATION_tg (src/INITIAL_FL_FLD_TG.f90:109-139). */
int chapsim_rk_substep_tg(chapsim_ctx_t* ctx, int32_t ns);

/* nsteps iterations of the SOLVE loop body (src/SOLVE.f90:75-134) without
 * post-processing: CFL, dt rule and the three RK substeps, replayed as one
 * captured CUDA graph per step with dt kept on the device.  dt_out and
 * cfl_out (may be NULL) receive the values of the last step. */
int chapsim_advance_tg(chapsim_ctx_t* ctx, int32_t nsteps, double dt0, double dtmin, double cflgv, double* dt_out,
                       double* cfl_out);

/* DIVGCK_tg (src/DIVGCK.f90:15-55): max |div u| of the resident velocity. */
int chapsim_divgck_tg(chapsim_ctx_t* ctx, double* maxdiv);

/* FFT99_POIS3D_periodicxz(ITG) (src/possion3d_FFT99.f90:271-505) on host
 * arrays: rhs = RHSLLPHI_tg(NCL1, NCL2, NCL3), dph = DPH_tg(NCL1, 0:NCL2+1,
 * NCL3) (rows 1..NCL2 written). */
int chapsim_fft99_pois3d(chapsim_ctx_t* ctx, const double* rhs, double* dph);

/* TDMAIJI_CYC(A,B,C,R,1,ISZ,1,JSZ) (src/TDMAIJI_CYC.f90:67): cyclic
 * tridiagonal systems along the first index of (ISZ, JSZ) arrays; R is
 * overwritten with the solution.  Host arrays. */
int chapsim_tdmaiji_cyc(const double* a, const double* b, const double* c, double* r, int32_t isz, int32_t jsz);

/* TDMAIJJ_nonCYC(A,B,C,R,BCJ,1,JSZ,1,ISZ) (src/TDMAIJJ_nonCYC.f90:67):
 * systems along the second index of (ISZ, JSZ) arrays with Dirichlet values
 * BCJ(ISZ, 2) (may be NULL for zero).  Host arrays. */
int chapsim_tdmaijj_noncyc(const double* a, const double* b, const double* c, double* r, const double* bcj,
                           int32_t jsz, int32_t isz);

/* Fixed size of the device scratch array used by chapsim_tdma_lines_noalloc
 * (16 MiB per device: a 256-byte status block, then 2,097,120 doubles). */
#define CHAPSIM_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)

/* No counterpart in the reference.  The same tridiagonal line solves as
 * chapsim_tdmaiji_cyc (cyclic != 0) and chapsim_tdmaijj_noncyc (cyclic == 0),
 * for a caller that keeps its arrays on the device and cannot let the library
 * allocate: a host whose HBM is already held by its own pool or data regions,
 * or a time loop that must not stall on the device-wide wait of cudaFree.
 * The call allocates nothing: its work vectors live in one module-scope
 * device array of CHAPSIM_NOALLOC_SCRATCH_BYTES.
 *   a, b, c, r: device memory of the current device; element e of line l is
 *     at l*line_stride + e*elem_stride, e < n; r is overwritten.
 *   bcj: NULL (zero) or 2*nlines device doubles, the Dirichlet values before
 *     the first and after the last row of each line (non-cyclic only).
 *   stream: cudaStream_t as void* (NULL = default stream); the call waits for
 *     it before returning.
 * Limits and errors: n >= 3; 3*n*nlines must not exceed 2,097,120, else
 * CHAPSIM_ERR_BADARG with the sizes in chapsim_last_error_string(NULL);
 * host pointers give CHAPSIM_ERR_BADARG; a non-finite solution on any line
 * gives CHAPSIM_ERR_NAN.
 * Set-up: the first call on each device (the one current in the calling
 * thread) looks up the array's address with cudaGetSymbolAddress and keeps
 * it; make that first call before any stream capture begins.  The address is
 * kept for the life of the process: a cudaDeviceReset of that device after
 * its first call is not supported (later calls would use a stale address).
 * Sharing: all calls on a device use the same array, which keeps the last
 * call's contents (the call clears its status counter itself).  Calls that
 * overlap in time on one device, e.g. from two host threads, race on it and
 * must be serialised by the caller. */
int chapsim_tdma_lines_noalloc(const double* a, const double* b, const double* c, double* r, const double* bcj,
                               int32_t nlines, int64_t line_stride, int64_t elem_stride, int32_t n, int32_t cyclic,
                               void* stream);

/* ---- Main (IO) domain, explicit viscous terms (context created with
 * grid.idomain = 2).  SOLVERRK3_MOM_io(NS) (src/SOLVERRK3_MOM_IO.f90:11-120,
 * iVisScheme = 0) for a flow whose property fields are fixed (thermal solver
 * not yet active).  chapsim_advance_tg runs the IO step (CFL_io, dt rule, three
 * substeps) for such a context. */

/* ReStart_INSTANT_VARS_io (src/processing/RESTART_io.f90:16-200) field set-up:
 * g = G_io(NCL1, 0:NCL2+1, NCL3, 3) (rho*u), pr = PR_io, rho = DENSITY0,
 * mu0 = Viscousity0, mu = Viscousity (each (NCL1, 0:NCL2+1, NCL3)).  Applies
 * BC_WALL_G_io/BC_WALL_PR_io, DENSITY_Staggered, MU_Staggered and
 * VELOCITY_CALC_io; EXPLT0_io is zeroed. */
int chapsim_upload_io_fields(chapsim_ctx_t* ctx, const double* g, const double* pr, const double* rho,
                             const double* mu0, const double* mu);
/* g = G_io, q = Q_io (velocity), pr = PR_io; any may be NULL. */
int chapsim_download_io_fields(chapsim_ctx_t* ctx, double* g, double* q, double* pr);
/* SOLVERRK3_MOM_io(NS) with the device-resident DT, in the viscous scheme
 * chosen by chapsim_opts_t.ivisscheme (src/SOLVERRK3_MOM_IO.f90:43-79). */
int chapsim_rk_substep_io(chapsim_ctx_t* ctx, int32_t ns);
/* CFL_io (src/CFL.f90:55-107): CFLMM_io including the viscous number. */
int chapsim_cfl_io(chapsim_ctx_t* ctx, double* cflmm);
/* Buoyancy of RHS_MOM_EXPLICIT_io (src/RHS_MOM_EXPLICIT_io.f90:161-226), set up
 * as thermal_gravity does (src/Flow_State.f90:95-125): component |igravity| of
 * the momentum right-hand side (1 x, 2 y, 3 z; 0 none) takes
 * D_STG * TALP(NS)*DT*F_A, before the bulk-forcing sum.  f_a is the host's
 * F_A (+-L0/U0^2 * 9.80665 for iGravity = +-1, -2, 3; 0 otherwise).  Main
 * domain only; CHAPSIM_ERR_BADARG for |igravity| > 3 or a non-finite f_a. */
int chapsim_set_buoyancy(chapsim_ctx_t* ctx, int32_t igravity, double f_a);
/* iWeightedPre = 1 (src/RHS_MOM_EXPLICIT_io.f90:103-159, src/DIVG.f90:78-82):
 * pr0_1 = PR0_io(:,:,:,1), pr0_2 = PR0_io(:,:,:,2), each (NCL1, 0:NCL2+1,
 * NCL3) host arrays (the reference sets both to PR_io at the start,
 * src/FLOWSTART.f90:83-85, and keeps them).  The pressure gradient becomes
 * ((PR0_2 diff)(1/4 - eps) + (PR0_1 diff)/2 + (PR diff)(1/4 + eps)) and DIVG_io
 * divides by (1/4 + eps), eps = pres_epslon = 0.001.  Both NULL turns it off;
 * one NULL is CHAPSIM_ERR_BADARG.  Main domain only. */
int chapsim_upload_weighted_pressure(chapsim_ctx_t* ctx, const double* pr0_1, const double* pr0_2);
/* DIVGCK_io (src/DIVGCK.f90:60-184), x-periodic main domain: MAXDIVGV_io, the
 * max over the interior of |div G + DrhoDtP| (the three ranges coincide). */
int chapsim_divgck_io(chapsim_ctx_t* ctx, double* maxdiv);

/* No counterpart in the reference: the failure path of the bounded device waits.  One warp
 * waits on an mbarrier that nothing arrives at, with the clock budget (about 2^31 clocks)
 * of every tensor-core completion and bulk-copy wait; the call returns CHAPSIM_ERR_TIMEOUT
 * after about a second, and the context stays usable (the error word is cleared). */
int chapsim_probe_wait_timeout(chapsim_ctx_t* ctx);

/* ---- Main domain with inflow and outflow (grid.idomain = 3): the IO part of a
 * TG + main-domain run (iDomain = 3, TgFlowFlg and IoFlowFlg), explicit viscous terms, FP64,
 * flow only or with the thermal solver (chapsim_xinout_thermal_inlet).
 * Fields carry the x ghost columns NCL1S:NCL1E = 0:NCL1+1: chapsim_upload_io_fields /
 * chapsim_download_io_fields take (0:NCL1+1, 0:NCL2+1, NCL3) arrays (and G_io(..., 3));
 * the upload also sets the ghost columns' velocity to G over the x average of DENSITY0
 * of the column and its interior neighbour, and zeroes BC_CONV0.  No bulk forcing
 * (src/RHS_MOM_EXPLICIT_io.f90:229); chapsim_set_buoyancy, chapsim_cfl_io,
 * chapsim_divgck_io (max over the cells 1..NCL1) and the thermal solver (table search; see
 * chapsim_xinout_thermal_inlet) apply; iWeightedPre, the learned property model, the
 * main-domain statistics, chapsim_advance_tg, chapsim_autotune and chapsim_profile_steps do
 * not (CHAPSIM_ERR_BADARG). */

/* The periodic TG context whose fields feed BC_TINLET_FLOW (src/BC_INLET.f90:12-61):
 * FP64, same device, same NCL2, NCL3 and y mesh (the x spacing must match, as
 * CONSPARA checks, src/CONSPARA.f90:44-52).  The TG context must outlive its use. */
int chapsim_xinout_attach(chapsim_ctx_t* io, chapsim_ctx_t* tg);
/* chapsim_rk_substep_io(io, NS), NS = 1..3, on an idomain 3 context runs
 * SOLVERRK3_MOM_io(NS) with TgFlowFlg (src/SOLVERRK3_MOM_IO.f90:11-120): BC_TINLET_FLOW
 * from the attached TG context's resident fields (run its substep NS first),
 * BC_COUTLET_MOM_RK3(NS) (src/BC_COUTLET_MOM_RK3.f90:16-192 with CHK_MassConsv_io,
 * src/processing/CHK_conservation.f90:11-79), the momentum step with the inlet face u(1)
 * fixed, DIVG_io, FISHPACK_POIS3D_SIMPLE with BCX_io = (2, 1) (LPEROD = 4,
 * src/possion3d_fishpack.f90:344-460), PRCALC_io and MASSFLUX_UPDATE_io over the u faces
 * 2..NCL1+1 (src/VELO_CORRECTION.f90:121-137). */

/* nsteps iterations of the SOLVE loop of a TG + main-domain run (src/SOLVE.f90:75-134):
 * CFL_tg and CFL_io, DT from CFLMM = max(CFLMM_tg, CFLMM_io) by the dt rule, then per NS
 * SOLVERRK3_MOM_tg(NS) on the attached TG context and SOLVERRK3_MOM_io(NS) here.  Both
 * contexts' DT follow; dt_out / cfl_out (may be NULL) receive DT and CFLMM of the last step.
 * CHAPSIM_ERR_DT_COLLAPSE as chapsim_advance_tg. */
int chapsim_advance_xinout(chapsim_ctx_t* io, int32_t nsteps, double dt0, double dtmin, double cflgv, double* dt_out,
                           double* cfl_out);
/* Thermal inflow/outflow (iThermoDynamics = 1 with TgFlowFlg): after chapsim_thermal_init on the
 * idomain = 3 context (DH over 0:NCL1+1; the inlet and outlet columns' properties follow from it),
 * state7 = T_inlet, H_inlet, D_inlet, M_inlet, K_inlet, CP_inlet, DH_inlet (src/Flow_State.f90:
 * 44-50).  Each substep then runs SOLVERRK3_ENG_io with BC_TINLET_THERML (src/BC_INLET.f90:64-84:
 * the inlet column holds that state) and BC_COUTLET_ENEG_RK3 (src/BC_COUTLET_ENEG_RK3.f90:11-59:
 * convective outflow of rho*h with the table limiter, THERM_PROP_UPDATE(IOULET)), and the outflow
 * scaling of BC_COUTLET_MOM_RK3 takes the interior mass rate of DrhoDtP.  Table search only
 * (chapsim_thermal_use_mlp is CHAPSIM_ERR_BADARG here). */
int chapsim_xinout_thermal_inlet(chapsim_ctx_t* ctx, const double* state7);
/* DIVGCK_io with TgFlowFlg (src/DIVGCK.f90:80-84): MAXDIVGV_io(1:3), the max |div G| over
 * the cells 2..NCL1-1, 0..1 and NCL1 (DrhoDtP = 0). */
int chapsim_divgck_xinout(chapsim_ctx_t* ctx, double* maxdiv3);
/* U_OUTLET (CONVCTION_OUTLET_U) and CHK_Mass_CONSV0_SCALING of the last substep. */
int chapsim_xinout_outlet_state(chapsim_ctx_t* ctx, double* state2);

/* ---- Thermophysical properties by table search ----
 * The nondimensional table and spline coefficients of the thermal_info module
 * after Property_Table_Nondimensionalization
 * (src/thermo_properties_table_searching.f90:1226-1346) and
 * SPLINE_COEFFICIENTS_FOR_DH / _FOR_H (:972-1128): LIST_H, LIST_T, LIST_D,
 * LIST_M, LIST_K, LIST_CP, LIST_DH and SplineCoeff_{DHH,HT,HD,HM,HK,HCp}_{B,C,D},
 * each N_LIST doubles.  LIST_B and the HB spline are not needed: the
 * reference discards the beta it interpolates. */
typedef struct {
    int32_t n_list;   /* N_LIST (>= 4) */
    int32_t fix_swap; /* 0: the reference's assignment in THERM_PROP_UPDATE_FROM_DH
                         (DENSITY <- HM spline, Viscousity <- HK, THERMCONDT <- HD);
                         1: DENSITY <- HD, Viscousity <- HM, THERMCONDT <- HK */
    const double *list_h, *list_t, *list_d, *list_m, *list_k, *list_cp, *list_dh;
    const double *dhh_b, *dhh_c, *dhh_d;
    const double *ht_b, *ht_c, *ht_d;
    const double *hd_b, *hd_c, *hd_d;
    const double *hm_b, *hm_c, *hm_d;
    const double *hk_b, *hk_c, *hk_d;
    const double *hcp_b, *hcp_c, *hcp_d;
} chapsim_prop_table_t;

/* Copies the table to the device (replacing any earlier one).  Applies the
 * reference's monotonicity checks of rho*h against T and h
 * (SPLINE_COEFFICIENTS_FOR_DH, :1016-1023) and, because the binary search
 * needs it, requires LIST_H and LIST_DH to increase strictly:
 * CHAPSIM_ERR_BADARG otherwise. */
int chapsim_prop_table_init(chapsim_ctx_t* ctx, const chapsim_prop_table_t* table);

/* THERM_PROP_UPDATE_FROM_DH, table arm (src/THERM_PROP_UPDATE.f90:14-67), on
 * npts host points: dh = DH in, h, t, d, m, k, cp = ENTHALPY, TEMPERATURE,
 * DENSITY, Viscousity, THERMCONDT, HEATCAP out.  Bitwise the reference's
 * spline evaluation.  A point (or its h) more than 1e-8 outside the table
 * gives CHAPSIM_ERR_TABLE_RANGE, where the reference STOPs
 * (spline_interpolation_*, :404-417); the message names the first such
 * point.  The other points are still written. */
int chapsim_therm_prop_update_points(chapsim_ctx_t* ctx, int64_t npts, const double* dh, double* h, double* t,
                                     double* d, double* m, double* k, double* cp);

/* ---- Thermal solver of the main (IO) domain (iThermoDynamics = 1, table search) ----
 * Starts SOLVERRK3_ENG_io (src/SOLVERRK3_ENG_IO.f90:11-82) on a context
 * created with grid.idomain = 2 whose flow fields are uploaded and whose
 * property table is set.  dh = DH(NCL1, 0:NCL2+1, NCL3) (rows 1..NCL2 used);
 * ENTHALPY, TEMPERATURE, DENSITY, Viscousity, THERMCONDT and HEATCAP follow
 * from it by THERM_PROP_UPDATE and, on the wall ghosts, BC_WALL_Isoflux
 * (src/BC_WALL.f90:541-619).  Both walls carry a constant heat flux:
 * WALLFLUX = +qw_bot at the bottom and -qw_top at the top (nondimensional
 * thermalWall_nondim, src/Flow_State.f90:140-175); cthecd = CTHECD =
 * 1/(REN PRT0) (src/SOLVE.f90:168).  DENSITY0 = DENSITY, Viscousity0 =
 * Viscousity, RHS_ENERGY0 = 0 and G0_io = G_io at start.  From then on every
 * IO substep (chapsim_rk_substep_io, chapsim_advance_tg) runs
 * SOLVERRK3_ENG_io(NS), DENSITY_TIME_DERIVATION(NS), DENSITY_Staggered and
 * MU_Staggered before SOLVERRK3_MOM_io(NS), as SOLVE does
 * (src/SOLVE.f90:119-133); a point leaving the table gives
 * CHAPSIM_ERR_TABLE_RANGE. */
int chapsim_thermal_init(chapsim_ctx_t* ctx, const double* dh, double qw_bot, double qw_top, double cthecd);
/* BC_Fixed_Temperature (iThermalWallType = 2) on wall 0 (bottom, iBotWall) or 1 (top):
 * state5 = the wall state T, H, D, M, K of T_WAL_GV, H_WAL_GV, D_WAL_GV, M_WAL_GV,
 * K_WAL_GV (src/Flow_State.f90:186-230, nondimensional), held in the wall's ghost row
 * (BC_WALL_IsoTHERMAL, src/BC_WALL.f90:484-538, with DH = H * D), and the wall face of
 * RHS_ENERGY_EXPLICIT keeps its DYCI conduction term (src/RHS_ENERGY_EXPLICIT.f90:50-77).
 * NULL returns the wall to the constant heat flux of chapsim_thermal_init.  Call after
 * chapsim_thermal_init; the ghost row is set at once. */
int chapsim_thermal_set_isothermal(chapsim_ctx_t* ctx, int32_t wall, const double* state5);

/* The thermal fields, each (NCL1, 0:NCL2+1, NCL3); any pointer may be NULL:
 * DH, ENTHALPY, TEMPERATURE, DENSITY, Viscousity, THERMCONDT, HEATCAP. */
int chapsim_download_thermal_fields(chapsim_ctx_t* ctx, double* dh, double* h, double* t, double* d, double* m,
                                    double* k, double* cp);

/* ---- Learned property model (no counterpart in the reference) ----
 * A 1 -> 64 -> 64 -> 6 tanh MLP from rho*h to the six outputs of
 * THERM_PROP_UPDATE_FROM_DH (ENTHALPY, TEMPERATURE, DENSITY, Viscousity,
 * THERMCONDT, HEATCAP), with tensor-core (tcgen05) layers on 16-bit operands
 * (BF16 in training, FP16 in inference) and FP32 accumulation, trained on the
 * GPU against the table search, which stays the
 * fallback outside the trained rho*h range and the judge of its accuracy.
 * Parameters (4678 floats): w1[64], b1[64], W2[64][64] (out, in), b2[64],
 * W3[6][64], b3[6]; inputs map [dh_lo, dh_hi] to [-1, 1]; output k is
 * off[k] + scale[k] * y[k] with off/scale from the table over that range.
 * The property table must be set first (chapsim_prop_table_init). */
int chapsim_mlp_init(chapsim_ctx_t* ctx, double dh_lo, double dh_hi, uint64_t seed);
int chapsim_mlp_set_params(chapsim_ctx_t* ctx, const float* params);
/* Hidden-layer activation of training and inference (default CHAPSIM_MLP_TANH).
 * CHAPSIM_MLP_CUBIC is the clamped cubic c = clamp(z, -1, 1), h = c (3 - c^2) / 2:
 * inference evaluates it with multiply-adds on FP16 pairs instead of the
 * special-function unit's tanh.  Set it before training; parameters trained
 * with one activation do not carry over to the other. */
#define CHAPSIM_MLP_TANH 0
#define CHAPSIM_MLP_CUBIC 1
int chapsim_mlp_set_activation(chapsim_ctx_t* ctx, int32_t act);
/* params (4678) and/or norm (14: dh_lo, dh_hi, off[6], scale[6]); either may be NULL */
int chapsim_mlp_get_params(chapsim_ctx_t* ctx, float* params, double* norm);
/* Gradient of the mean squared error of the normalised outputs against the
 * table search over n host samples (one forward/backward pass, no update). */
int chapsim_mlp_gradients(chapsim_ctx_t* ctx, int32_t n, const double* dh, float* grad, double* loss);
/* iters full-batch Adam steps (learning rate lr) on n host samples; final_loss
 * receives the loss of the last pass. */
int chapsim_mlp_train(chapsim_ctx_t* ctx, int32_t n, const double* dh, int32_t iters, float lr, double* final_loss);
/* Model evaluation of npts host points (table search outside the trained range). */
int chapsim_mlp_infer_points(chapsim_ctx_t* ctx, int64_t npts, const double* dh, double* h, double* t, double* d,
                             double* m, double* k, double* cp);
/* Thermal step: 1 = the interior property update of every substep uses the
 * model (wall ghosts and points outside the trained range keep the table
 * search), 0 = table search everywhere. */
int chapsim_thermal_use_mlp(chapsim_ctx_t* ctx, int32_t enable);
/* Judge: max over the interior of |field - table(DH)| / max(|table(DH)|, scale)
 * for each of the six outputs (max_rel_err[6]); the caller runs it every N
 * steps and switches back to the table when it exceeds its bound. */
int chapsim_mlp_judge(chapsim_ctx_t* ctx, double* max_rel_err);

/* ---- Statistics of the periodic channel (POSTPROCESS_TG, src/processing/POSTPROESS.f90:11-51) ----
 * Computed on the device from the resident fields, so the driver needs no
 * per-step download of Q.  Arrays are the postprocess_info module arrays in
 * Fortran order, M = NCL2: U1xzL_tg(M, 4), UPxzL_tg(M, 3), U2xzL_tg(M, 6),
 * U3xzL_tg(M, 10), DVDL1xzL_tg(M, 3, 3), DVDLPxzL_tg(M, 3, 3), DVDL2xzL_tg(M, 9, 9);
 * the time averages (U1xztL_tg ...) have the same shapes.  Sums over the x-z
 * plane are taken in a fixed tree order instead of the reference's I, K loop. */
/* PP_MEAN_ZX_FLOW_TG (src/processing/PP_MEAN_ZX.f90:14-307): instantaneous means. */
int chapsim_pp_mean_zx_tg(chapsim_ctx_t* ctx);
/* PP_MEAN_T_TG(TP) (src/processing/PP_MEAN_T.f90:343-392): NSTATIS_TG += 1 and
 * avg = COE3 avg + COE2 inst; tp = 1 (T_Asymptotic_Average) or 2
 * (T_Summing_average, with pp_instn_sz). */
int chapsim_pp_mean_t_tg(chapsim_ctx_t* ctx, int32_t tp, int32_t pp_instn_sz);
/* PP_MONITOR_TG (src/processing/PP_SCN_MONITOR.f90:147-251) quantities from the
 * current instantaneous and averaged means: mon[20] = U1_XZT(1:6), UU_XZT(1:8),
 * CF_XZT(1:4), U1mean_WORK_tg, U1maxx_WORK_tg (the last two of
 * PP_MEAN_ZX_FLOW_TG :294-305).  ren = REN. */
int chapsim_pp_monitor_tg(chapsim_ctx_t* ctx, double ren, double* mon);
/* Downloads the instantaneous (averaged = 0) or time-averaged (1) means; any
 * pointer may be NULL; nstatis receives NSTATIS_TG. */
int chapsim_download_pp_means_tg(chapsim_ctx_t* ctx, int32_t averaged, double* u1, double* up, double* u2,
                                 double* u3, double* dvdl1, double* dvdlp, double* dvdl2, int32_t* nstatis);
/* ---- Statistics of the main domain (POSTPROCESS_io's PP_MEAN_ZX_FLOW_Xperiodic_io,
 * src/processing/PP_MEAN_ZX.f90:311-796; plane channel) ----
 * chapsim_pp_mean_zx_io computes the instantaneous x-z means of a main-domain
 * context on the device from its resident fields (G, Q, PR and, with the
 * thermal solver, TEMPERATURE, DENSITY, ENTHALPY, Viscousity, THERMCONDT).
 * One set holds per_row * M doubles, per_row = 141 (flow) or 360 (with the
 * thermal solver), the module arrays in the order the reference zeroes them
 * (Fortran order, j fastest): U1xzL_io(M,4), G1xzL_io(M,3), UPxzL_io(M,3),
 * U2xzL_io(M,6), UGxzL_io(M,6), U3xzL_io(M,10), UGUxzL_io(M,10),
 * DVDL1xzL_io(M,3,3), DVDLPxzL_io(M,3,3), DVDL2xzL_io(M,9,9), then T1, D1, H1,
 * M1, T2, D2, H2, DH, PHxzL_io(M), DVDL1MxzL_io(M,3,3), DVDL1MHxzL_io(M,3,3),
 * DVDL1MUxzL_io(M,3,3,3), DVDL2MxzL_io(M,9,9), UHxzL_io(M,3), GHxzL_io(M,3),
 * U2DHxzL_io(M,6), DhDL1xzL_io(M,3), DhDLPxzL_io(M,3), DTDLKxzL_io(M,3),
 * DTDLKUxzL_io(M,3,3), DTDLKDVDLxzL_io(M,3,3,3), DHDLMDVDLxzL_io(M,3,3,3).
 * Plane sums are taken in a fixed tree order.  A periodic-domain context
 * gives CHAPSIM_ERR_BADARG. */
int chapsim_pp_mean_zx_io(chapsim_ctx_t* ctx);
/* Downloads the last set (out may be NULL); per_row (may be NULL) receives 141 or 360. */
int chapsim_download_pp_means_io(chapsim_ctx_t* ctx, double* out, int32_t* per_row);
/* Restart of the time averages (the reader of the averaged-statistics file). */
int chapsim_upload_pp_means_tg(chapsim_ctx_t* ctx, int32_t nstatis, const double* u1, const double* up,
                               const double* u2, const double* u3, const double* dvdl1, const double* dvdlp,
                               const double* dvdl2);

/* ---- Field files (.D) and asynchronous dumps ----
 * Replace WRT_INSTANT_VARS_TG (src/processing/WRT_VARS_TG.f90:13-100),
 * WRT_INSTANT_VARS_FLOW_IO / _THERMAL_IO (src/processing/WRT_VARS_IO.f90:24-227)
 * and the readers of ReStart_INSTANT_VARS_TG (src/processing/RESTART_tg.f90:11-56).
 * A .D file: int32[4] {NCL1, NCL2, NCL3, ITERG}, float64[3] {PhyTIME, REN, DT},
 * then float64 (NCL1, NCL2, NCL3) in Fortran order, no ghost planes. */
int chapsim_write_dfile(const char* path, int32_t L, int32_t M, int32_t N, int32_t iterg, double time, double ren,
                        double dt, const double* field);
/* dims4 = {L, M, N, ITERG}, reals3 = {PhyTIME, REN, DT}; field (capacity in
 * doubles) may be NULL to read the header only.  A payload whose size does not
 * match the header is CHAPSIM_ERR_BADARG. */
int chapsim_read_dfile(const char* path, int32_t* dims4, double* reals3, double* field, int64_t capacity);
/* Snapshot U, V, W, P (and T, D, H, M, K with the thermal solver) and the
 * device dt in stream order, then copy the snapshot to pinned host memory on
 * a stream of the context's own, overlapping the steps launched next. */
int chapsim_dump_begin(chapsim_ctx_t* ctx);
/* Waits for the dump's copy and writes <path_prefix><PhyTIME as ES15.9>_U.D,
 * _V.D, _W.D, _P.D (and _T.D, _D.D, _H.D, _M.D, _K.D); the DT in the headers
 * is the device dt at the snapshot, returned in dt_out (may be NULL).  The
 * reference's prefix is <FilePath1>DNS_perixz_INSTANT_T. */
int chapsim_dump_write(chapsim_ctx_t* ctx, const char* path_prefix, int32_t iterg, double time, double ren,
                       double* dt_out);

/* ---- Autotuner and ensembles (no counterpart in the reference) ---- */

/* Times the alternative kernels of the step on this context's grid and keeps
 * the fastest of each group (force = -1), or the ones forced (force = 0..8191):
 *   bits 0, 4, 5 and 6: Poisson y-solve, all 0 = warp Thomas/PCR hybrid,
 *          bit 0 = the reference's sequential Thomas recurrence, one thread
 *          per mode, bit 4 = two-way elimination, two threads per mode,
 *          bit 5 = the sequential recurrence with its forward intermediate in
 *          shared memory at one block per SM (lines longer than two blocks
 *          per SM allow; elsewhere it means bit 0), bit 6 = one warp per mode
 *          line evaluating the sequential recurrence's two sweeps as affine
 *          scans over its precomputed factors; the lowest set bit wins;
 *   bits 1-2: explicit right-hand sides + x sweep (periodic channel only),
 *          0 = fused (one warp per x line, per-thread loads; two adjacent
 *          points per lane in FP32), 1 = split into a point-wise kernel and
 *          a line-sweep kernel, 2 = fused with the stencil rows staged in
 *          shared memory by bulk copies, 3 = the wide fused form, 16-byte
 *          loads of two adjacent points per lane in FP64 or four in FP32
 *          (L / 32 a multiple of 2 or 4; elsewhere it means 0);
 *   bit 3: pressure stage (periodic channel only), 0 = chained x and z
 *          transforms, 1 = fused plane transforms: one block per y row where
 *          the row's half spectrum fits one block's shared memory, one
 *          thread-block cluster per row (the x-z transpose in distributed
 *          shared memory) for 256- and 384-point planes; otherwise 0 is kept
 *          whatever is forced;
 *   bit 8: tile shape of the z sweep (periodic channel only), 0 = 32
 *          consecutive x lines per tile, 1 = 16;
 *   bit 9: with the chained transforms, the z transforms as persistent
 *          blocks that load their next tile while transforming the current
 *          one (periodic channel only; timed as a third pressure-stage form);
 *   bit 10: z-sweep tile layout (periodic channel only), 0 = each x line
 *          contiguous in shared memory, 1 = lines interleaved in pairs (one
 *          copy instruction per two points);
 *   bit 11: the same for the y sweep (Q is restored after its trials);
 *   bit 12: with the chained transforms, each z-transform block also
 *          requests into L2 the tile of the block one wave later (timed as a
 *          fourth pressure-stage form).
 * choice receives the kept setting in the same bit form; ms[19] (may be NULL)
 * the mean durations of y-solve (hybrid, sequential), right-hand sides
 * (fused, split, bulk-staged), pressure stage up to DPH (chained, fused;
 * 1e30 where a variant does not apply), the two-way y-solve, the
 * sequential y-solve at one block per SM (1e30 where it does not apply) and
 * the scan y-solve, the z sweep with 32- and with 16-line tiles (0 where it
 * does not apply), the pressure stage with the double-buffered z
 * transforms, the wide right-hand side (1e30 where it does not apply), and
 * the z sweep with pair-interleaved 32- and 16-line tiles, the y sweep with
 * line-contiguous and pair-interleaved tiles, and the pressure stage with
 * the z transforms' wave-ahead requests.
 * CONVH0 is restored after the trial launches. */
int chapsim_autotune(chapsim_ctx_t* ctx, int32_t force, int32_t* choice, float* ms);

/* An ensemble of independent periodic channels (any grids and precisions, one
 * device) advanced together: one CUDA graph per step holds every member's
 * kernels as parallel branches, so small members fill the GPU together.
 * Members keep their own dt; each step of chapsim_batch_advance is the
 * members' chapsim_advance_tg step. */
typedef struct chapsim_batch chapsim_batch_t;
int chapsim_batch_create(chapsim_ctx_t* const* ctxs, int32_t n, chapsim_batch_t** out);
int chapsim_batch_advance(chapsim_batch_t* batch, int32_t nsteps, double dt0, double dtmin, double cflgv);
int chapsim_batch_get_stream(chapsim_batch_t* batch, void** stream);
int chapsim_batch_destroy(chapsim_batch_t* batch);

/* Profiling: runs nsteps steps (as chapsim_advance_tg, without the graph)
 * with a CUDA event after every kernel slot; ms[slot] receives the summed
 * duration of slot `slot` of a step.  Periodic channel: k_cfl, k_dt_factors,
 * then for each substep k_rhs_xsweep, k_zsweep, k_ysweep, k_div_fftx,
 * k_fftz_fwd, k_ysolve, k_fftz_inv, k_fftx_inv, k_correct (29 slots).
 * Main domain: k_io_cfl, k_dt, then for each substep (with the thermal
 * solver) k_eng_rhs, the property update (table search or model), k_eng_bc,
 * k_drhodt, k_io_props, k_g0_velocity, then the momentum step's three
 * slots (explicit: k_io_divu, k_io_rhs, k_io_massflux; Crank-Nicolson:
 * k_io_rhs, the x sweep, the z and y sweeps) and k_io_div_fftx, k_fftz_fwd,
 * k_ysolve, k_fftz_inv, k_fftx_inv, k_io_correct (29 slots, 47 with the
 * thermal solver). */
int chapsim_profile_steps(chapsim_ctx_t* ctx, int32_t nsteps, double dt0, double dtmin, double cflgv, float* ms,
                          int32_t nslots);

/* The cudaStream_t (as void*) all of the context's work is queued on. */
int chapsim_get_stream(chapsim_ctx_t* ctx, void** stream);

/* Waits for all work queued on the context's stream. */
int chapsim_sync(chapsim_ctx_t* ctx);

/* Number of kernels this context has launched so far (graph replays count
 * each kernel node). */
int chapsim_launch_count(const chapsim_ctx_t* ctx, uint64_t* count);

/* Kernels launched per call of chapsim_advance_tg per step (for accounting). */
int chapsim_kernels_per_step(const chapsim_ctx_t* ctx, int32_t* count);

#ifdef __cplusplus
}
#endif
#endif /* CHAPSIM_GPU_H */
