/*
 * kmm.h -- C ABI of the B200 Kim-Moin-Moser channel timestep.
 *
 * This is the drop-in boundary between the reference's Fortran host program
 * (FFTW_DNS/code/src/dns/main_dns.f90, which keeps its time loop, its
 * subroutine names and dns.config) and the GPU implementation of the hot path:
 * solvers.f90 (Chebyshev-tau solvers, influence matrix, vcw3dp), derivatives.f90
 * (Chebyshev / Fourier derivatives), helpers.f90 (norm, xyzfft, polymer coupling)
 * and part_track.f90 (tracer and inertial-particle integrators).
 *
 * Conventions
 *  - Every entry point returns an int status (KMM_OK == 0).  The reference
 *    `stop`s on the same conditions (CFL > 1, solvers.f90:3510-3514; particle
 *    interpolation index < 1, part_track.f90:580-590; grid mismatch,
 *    main_dns.f90:961-970); the Fortran shim calls `stop` on nonzero.
 *  - Arrays cross the boundary as plain host pointers in the reference's own
 *    Fortran layout (column major, y fastest):
 *        spectral field   complex(8) (nyp,nz,nxh)   -> interleaved re/im doubles
 *        3/2 physical     real(8)    (nyp,mz,mx)
 *        wall rows        complex(8) (nz,nxh)
 *        mean modes       real(8)    (nyp)
 *        particles        real(8)    (npart)
 *        initial fields   real(8)    (nyp,nz,nx)
 *        imatrix          integer(4) (nyp,mz,mx)
 *    The context owns one device mirror per field; kmm_upload / kmm_download move
 *    a whole field between the host array and its mirror.  Routines operate on
 *    the mirrors named by kmm_field ids, so the state stays resident in HBM and
 *    the host syncs only at restart / output cadence.
 *  - One host thread per context.  Calls are asynchronous on the context's
 *    stream except kmm_download, kmm_sync and status reads.
 *  - Grid sizes are run-time values (the reference has them as compile-time
 *    parameters in grid_size.f90:1-47).
 */
#ifndef KMM_H
#define KMM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KMM_ABI_VERSION 1

/* ---- status codes -------------------------------------------------------- */
enum kmm_status {
    KMM_OK = 0,
    KMM_ERR_ARG = 1,          /* bad argument, unknown field, size mismatch        */
    KMM_ERR_CUDA = 2,         /* CUDA runtime error (message in kmm_last_error)     */
    KMM_ERR_CFL = 3,          /* max CFL > 1        (solvers.f90:3510-3514)         */
    KMM_ERR_NAN = 4,          /* non-finite value in the state                      */
    KMM_ERR_INTERP = 5,       /* particle cell index out of range (part_track.f90:580-590) */
    KMM_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up                 */
    KMM_ERR_NOMEM = 7,        /* device allocation failed                           */
    KMM_ERR_UNSUPPORTED = 8,  /* option not available in this build                 */
    KMM_ERR_PCFL = 9          /* inertial-particle CFL umax1 dt/ap >= 10 (part_track.f90:215-222) */
};

/* ---- run parameters -------------------------------------------------------
 * One member per value `setstuff` reads from dns.config (main_dns.f90:934-1068),
 * in file order, plus the module switches the reference selects at compile time
 * (-DSCALAR / -DPOLYMER, Makefile:9-10) and a few variants that have no
 * counterpart in the reference (each defaults to the reference behaviour).    */
typedef struct kmm_params {
    int    nsteps, iprnfrq;
    double dt, gain, ugain, theta;
    int    ny, nz, nx;              /* NY1, NZ1, NX1 (grid_size.f90:2)               */
    int    bftail;
    double yl, zl, xl, re, xstart, uinf;
    int    kwall, perturbtime;
    double r_tau, gravity;
    int    irstrt, crstrt, print3d, geomtype, particle_flag, flow_select;
    int    itarget, ipeter, ipolyflag, scl_flag;
    int    npart, new_part;
    double ratio, ap, c_mu;
    int    cd_switch;
    double zlmax, tpoly, alpha_poly, diffpoly, c11z, c22z, c33z, qbeta;
    double diff, deltat, sigmax, sigmay, sigmaz;
    int    src_start, src_stop, scltarg;
    int    cadence;
    double spts;
    /* modules (-DSCALAR, -DPOLYMER) */
    int    scalar_on, polymer_on;
    /* variants (0 = reference behaviour) */
    int    scalar_bc;      /* 0: zero-flux walls (main_dns.f90:350-353); 1: scalar = 0 at both walls */
    double scalar_q;       /* uniform volumetric scalar source added to -u.grad(c); 0: none           */
    int    tracer_scheme;  /* 0: explicit Euler (part_track.f90:416-421); 1: Williamson RK3           */
    int    precision;      /* 0: FP64 drop-in; 1: mixed (FP32 transforms / products, FP64 solves)     */
    int    ib_spread_all;  /* 0: immersed-boundary drag is spread only in the y-planes i <= kmaxsurf, the
                              reference's test (solvers.f90:3069; kmaxsurf is the largest solid x index,
                              main_dns.f90:1526-1535); 1: in every y-plane, so each solid cell's drag is
                              spread in its own plane (geometries whose solid y-planes lie above kmaxsurf,
                              such as a cylinder in mid-channel, otherwise receive no force)             */
    double flow_rate;      /* 0: constant mean pressure gradient dPdx (init_flow.f90:117); > 0: constant
                              flow rate -- after each mean-mode solve a uniform pressure-gradient
                              correction holds the trapezoid bulk velocity of helpers.f90:1355-1359 at
                              this value (the correction of the last step is kmm_stats.dpdx - dPdx)     */
} kmm_params;

/* ---- field ids -------------------------------------------------------------
 * Names follow the reference's variable names in main_dns.f90:23-100.       */
enum kmm_field {
    /* spectral complex(8) (nyp,nz,nxh) */
    KMM_U = 0, KMM_V, KMM_W, KMM_OMX, KMM_OMY, KMM_OMZ,
    KMM_FN, KMM_FNM1, KMM_GN, KMM_GNM1,
    KMM_U11, KMM_U12, KMM_U13, KMM_U21, KMM_U22, KMM_U23, KMM_U31, KMM_U32, KMM_U33,
    KMM_LU, KMM_LV, KMM_LW,
    KMM_GF1, KMM_GF2,
    KMM_WRKC, KMM_WRK1,
    KMM_SCALAR, KMM_SCLX, KMM_SCLY, KMM_SCLZ, KMM_SCN, KMM_SCNM1,
    KMM_C11, KMM_C12, KMM_C13, KMM_C21, KMM_C22, KMM_C23, KMM_C31, KMM_C32, KMM_C33,
    KMM_C11N, KMM_C12N, KMM_C13N, KMM_C22N, KMM_C23N, KMM_C33N,
    KMM_C11NM1, KMM_C12NM1, KMM_C13NM1, KMM_C22NM1, KMM_C23NM1, KMM_C33NM1,
    KMM_STR11N, KMM_STR12N, KMM_STR13N, KMM_STR22N, KMM_STR23N, KMM_STR33N,
    KMM_STR11NM1, KMM_STR12NM1, KMM_STR13NM1, KMM_STR22NM1, KMM_STR23NM1, KMM_STR33NM1,
    KMM_QP11, KMM_QP12, KMM_QP13, KMM_QP22, KMM_QP23, KMM_QP33,
    KMM_T1, KMM_T2, KMM_T3,
    /* dcIJK = d(c_IJ)/dx_K, derivatives.f90:148-254 */
    KMM_DC111, KMM_DC112, KMM_DC113, KMM_DC121, KMM_DC122, KMM_DC123, KMM_DC131, KMM_DC132, KMM_DC133,
    KMM_DC211, KMM_DC212, KMM_DC213, KMM_DC221, KMM_DC222, KMM_DC223, KMM_DC231, KMM_DC232, KMM_DC233,
    KMM_DC311, KMM_DC312, KMM_DC313, KMM_DC321, KMM_DC322, KMM_DC323, KMM_DC331, KMM_DC332, KMM_DC333,
    KMM_CSOURCE,
    KMM_NSPECTRAL,

    /* real(8) (nyp) */
    KMM_U0 = 200, KMM_W0, KMM_H1N, KMM_H1NM1, KMM_H3N, KMM_H3NM1, KMM_UXMEAN,
    KMM_NMEAN_END,

    /* complex(8) (nz,nxh) */
    KMM_BCTOP = 300, KMM_BCBOT, KMM_DNV1B, KMM_DNV1T, KMM_DNV2B, KMM_DNV2T, KMM_DENOM, KMM_C1, KMM_C2,
    KMM_NWALL_END,

    /* real(8) (nyp,mz,mx), 3/2-rule physical grid */
    KMM_FXINTG = 400, KMM_FYINTG, KMM_FZINTG, KMM_UP3D, KMM_VP3D, KMM_WP3D, KMM_SWIRL3D,
    /* the physical fields of the inertial-particle path (particle_flag > 0): vorticity, velocity
     * gradient, Laplacian, and the previous step's velocity and Laplacian (solvers.f90:1824-1829,
     * 3464-3476) */
    KMM_WX3D, KMM_WY3D, KMM_WZ3D,
    KMM_U11P3D, KMM_U12P3D, KMM_U13P3D, KMM_U21P3D, KMM_U22P3D, KMM_U23P3D, KMM_U31P3D, KMM_U32P3D, KMM_U33P3D,
    KMM_LUP3D, KMM_LVP3D, KMM_LWP3D, KMM_UOLD, KMM_VOLD, KMM_WOLD, KMM_LUNM1, KMM_LVNM1, KMM_LWNM1,
    /* the scalar source vcw3dp adds (scsource, solvers.f90:2076-2210): the particle Gaussians of
     * scl_flag = 2 or the targeted source of scl_flag = 4, 5; written by every vcw3dp with
     * scl_flag >= 2 */
    KMM_SCSOURCE,
    KMM_NPHYS_END,

    /* integer(4) (nyp,mz,mx) */
    KMM_IMATRIX = 500,

    /* real(8) (npart) */
    KMM_XPART = 600, KMM_YPART, KMM_ZPART, KMM_UPART, KMM_VPART, KMM_WPART, KMM_SWIRLPART,
    KMM_NPART_END,

    /* real(8) (nyp,nz,nx): initial physical fields (COMMON /init/, main_dns.f90:98) */
    KMM_INITU = 700, KMM_INITV, KMM_INITW, KMM_INITSCL,
    KMM_NINIT_END
};

/* run diagnostics gathered by the last vcw3dp / step (host copy after kmm_stats) */
typedef struct kmm_stats {
    double cflmax;       /* max over the 3/2 grid of (|u|/dx+|v|/dy+|w|/dz) dt (solvers.f90:2985-2986) */
    double umax;         /* max |u| on the 3/2 grid                                                  */
    int    it;           /* COMMON /itime/ it after the call                                         */
    int    status;       /* last nonzero status raised on the device (0 if none)                     */
    double pumax;        /* inertial particles: running max |u_fluid - u_particle| (umax1, part_track.f90:736-742) */
    double pcfl;         /* inertial particles: umax1 dt / ap of the last update (part_track.f90:215-216) */
    double dpdx;         /* mean pressure gradient that drove the last step: dPdx, plus the flow-rate
                            correction when kmm_params.flow_rate > 0                                    */
} kmm_stats;

typedef struct kmm_ctx kmm_ctx;

/* ---- context ------------------------------------------------------------- */
/* Replaces setstuff + setbcs (main_dns.f90:829-1418): wavenumbers, Chebyshev
 * weights c(i), ycoord/seght, dy/deta, BC coefficients by flow_select, the
 * mean pressure gradient of init_flow.f90:117 and the force-spreading matrix of
 * forcepre (main_dns.f90:1551-1558).  `device` is the CUDA ordinal.          */
int  kmm_ctx_create(const kmm_params *params, int device, kmm_ctx **out);
int  kmm_ctx_destroy(kmm_ctx *ctx);
const char *kmm_last_error(const kmm_ctx *ctx);
int  kmm_abi_version(void);

/* element count and element size (bytes) of a field, 0 elements if unknown */
int  kmm_field_size(const kmm_ctx *ctx, int field, size_t *nelem, int *elem_bytes);
/* whole-field copies between a host array in reference layout and its mirror */
int  kmm_upload(kmm_ctx *ctx, int field, const void *host, size_t bytes);
int  kmm_download(kmm_ctx *ctx, int field, void *host, size_t bytes);
/* copy one mirror into another (the reference's n -> n-1 history copies) */
int  kmm_copy(kmm_ctx *ctx, int dst, int src);
int  kmm_zero(kmm_ctx *ctx, int field);
/* COMMON /itime/ it */
int  kmm_set_it(kmm_ctx *ctx, int it);
int  kmm_sync(kmm_ctx *ctx);
int  kmm_get_stats(kmm_ctx *ctx, kmm_stats *out);

/* ---- derivatives (derivatives.f90) --------------------------------------- */
/* cderiv(f,df), derivatives.f90:258-314 */
int  kmm_cderiv(kmm_ctx *ctx, int f, int df);
/* c{0,1,2}der{b,t}w(wrkc,wrk1,iy), derivatives.f90:318-653:
 * order 0/1/2, wall 0 = bottom (y=-1, "b"), 1 = top (y=+1, "t"); writes row iy (1-based) of `out` */
int  kmm_wallderiv(kmm_ctx *ctx, int f, int order, int wall, int out, int iy);
/* gradv, derivatives.f90:6-86 (u,v,w -> u11..u33, Lu, Lv, Lw) */
int  kmm_gradv(kmm_ctx *ctx);
/* gradscl, derivatives.f90:90-144 */
int  kmm_gradscl(kmm_ctx *ctx);
/* derivscji, derivatives.f90:148-254 */
int  kmm_derivscji(kmm_ctx *ctx);

/* ---- solvers (solvers.f90) ----------------------------------------------- */
/* gfcn twice + common denominator: solvers.f90:5-172, main_dns.f90:151-161 */
int  kmm_gfcn(kmm_ctx *ctx);
/* phirhs(v,wrkc,wrk1,fn,fnm1,bcbot,bctop,var), solvers.f90:555-676; zeroes KMM_BCTOP/KMM_BCBOT */
int  kmm_phirhs(kmm_ctx *ctx, int v, int fn, int fnm1, double var);
/* the kx loop around solve(u,x,g,dyde,bctop,bcbot,ib,a,wrkc), solvers.f90:174-553,
 * main_dns.f90:393-407; BC rows from KMM_BCTOP / KMM_BCBOT                  */
int  kmm_solve(kmm_ctx *ctx, int u, double g, int ib);
/* the kx loop around penta(u,x,g,dyde,ib,at,bt,gtop,ab,bb,gbot,a,wrkc), solvers.f90:680-1061,
 * main_dns.f90:479-484; gtop/gbot from KMM_BCTOP / KMM_BCBOT               */
int  kmm_penta(kmm_ctx *ctx, int u, double g, int ib, double at, double bt, double ab, double bb);
/* uzero(u0,h1,h1l,uflag), solvers.f90:1065-1493 (uflag 1: u0,h1n,h1nm1; 3: w0,h3n,h3nm1) */
int  kmm_uzero(kmm_ctx *ctx, int uflag);
/* phi = d2v/dy2 - k^2 v in place, main_dns.f90:363-375 */
int  kmm_phi_from_v(kmm_ctx *ctx);
/* influence-matrix combination v += c1 gf1 + c2 gf2, main_dns.f90:426-466 */
int  kmm_influence(kmm_ctx *ctx);
/* veloc(u,v,w,u0,w0,omy,wrkc), solvers.f90:1576-1659 */
int  kmm_veloc(kmm_ctx *ctx);
/* vort(u,v,w,omx,omz), solvers.f90:1663-1722 */
int  kmm_vort(kmm_ctx *ctx);
/* nonlin(fn,omz,gn,wrkc,wrk1), solvers.f90:1497-1572 */
int  kmm_nonlin(kmm_ctx *ctx);
/* vcw3dp(...), solvers.f90:1726-3538: dealiased u x omega (+ scalar, polymer,
 * immersed-boundary, mean-pressure-gradient terms) into fn, gn, omz (+ scn,
 * c_n, str_n, qp); CFL check; tracer update when npart > 0.  Returns
 * KMM_ERR_CFL when max CFL > 1, as the reference stops.                     */
int  kmm_vcw3dp(kmm_ctx *ctx);

/* ---- helpers (helpers.f90) ----------------------------------------------- */
/* norm(a), helpers.f90:91-158 */
int  kmm_norm(kmm_ctx *ctx, int f);
/* xyzfft(a,b,-1), helpers.f90:6-87: physical (nyp,nz,nx) field `src` (KMM_INIT*) -> spectral `dst` */
int  kmm_xyzfft(kmm_ctx *ctx, int dst, int src);
/* polyNL, helpers.f90:610-674 (into KMM_T1.. scratch named by the reference's cNL arrays) */
int  kmm_polynl(kmm_ctx *ctx);
/* polyforce(qp..,t1,t2,t3), helpers.f90:498-560 */
int  kmm_polyforce(kmm_ctx *ctx);
/* subforce(gn,fn,omz,t1,t2,t3), helpers.f90:564-606 */
int  kmm_subforce(kmm_ctx *ctx);

/* ---- main-program blocks (main_dns.f90) --------------------------------- */
/* spectral smoothing of the nonlinear terms, main_dns.f90:710-745 */
int  kmm_filter(kmm_ctx *ctx);
/* initial(...), main_dns.f90:1602-2231.  irstrt = 0: initial fields from KMM_INITU/V/W (and
 * KMM_INITSCL).  irstrt >= 1: the host has uploaded the records of setup/restart (KMM_V, KMM_FN,
 * KMM_FNM1, KMM_OMY, KMM_GN, KMM_GNM1, KMM_U0, KMM_H1N, KMM_H1NM1, KMM_W0, KMM_H3N, KMM_H3NM1;
 * KMM_FXINTG/FYINTG/FZINTG) -- and of setup/c-restart with scalar + polymer and crstrt = 1 --
 * which are used as they are (main_dns.f90:1742-1917); the step counter restarts at 0. */
int  kmm_initial(kmm_ctx *ctx);
/* one iteration of the time loop body, main_dns.f90:198-811, fused */
int  kmm_step(kmm_ctx *ctx);
/* `n` iterations (stops early with the status of a failing step) */
int  kmm_run(kmm_ctx *ctx, int n);

/* ---- state held in host arrays ---------------------------------------------
 * The reference's time loop works on host arrays (main_dns.f90:198-811).  kmm_bind_host makes
 * `host` (bytes = the field's size, reference layout) the home of a spectral, mean-mode, wall or
 * particle field; host = NULL unbinds it, and field < 0 with host = NULL unbinds all.  Page-locked
 * memory (cudaHostAlloc / cudaHostRegister) lets the copies run asynchronously; pageable memory
 * works but serialises them.
 * kmm_run_host runs `n` iterations as a host loop around the solver would: before every step each
 * bound field is copied host -> device, after every step device -> host, so the host arrays hold
 * each step's result (also that of a step that returns a stop status such as KMM_ERR_CFL, after
 * which it returns).  A step's downloads and the next step's uploads run together on two copy
 * streams, chunk by chunk; the history fields' downloads (FNM1, GNM1, SCNM1, the polymer n-1
 * records) run during the step.  The host arrays must not be touched during the call.  Without
 * bindings it is kmm_run.                                                                      */
int  kmm_bind_host(kmm_ctx *ctx, int field, void *host, size_t bytes);
int  kmm_run_host(kmm_ctx *ctx, int n);

/* ---- particles (part_track.f90) ----------------------------------------- */
/* tracer_update(u,v,w), part_track.f90:360-433, from KMM_UP3D/VP3D/WP3D */
int  kmm_tracer_update(kmm_ctx *ctx);
/* init_part's velocity interpolation, part_track.f90:229-292 */
int  kmm_init_part(kmm_ctx *ctx);
/* The interpolation cell of every particle at its current position, as fluid_interp looks it up
 * (part_track.f90:560-577): cells[p] = imin (x, 1..mx), cells[npart + p] = jmin (z, 1..mz),
 * cells[2 npart + p] = kmax (y, the upper Chebyshev node; kmin = kmax + 1), 1-based.  `n` is
 * the number of ints in `cells` (>= 3 npart).  Returns KMM_ERR_INTERP if any particle's index is
 * out of range (the reference stops there); its entries are then 0.                           */
int  kmm_tracer_cells(kmm_ctx *ctx, int *cells, size_t n);
/* calcswirl (helpers.f90:197-404, solvers.f90:3421 and 3480): swirl strength from the spectral
 * velocity gradients U11..U33 (kmm_gradv; after kmm_step run kmm_veloc first, the fused step
 * keeps only the prognostic fields) into SWIRL3D, and at each particle into SWIRLPART.  The
 * reference evaluates it inside every vcw3dp; here it is called at output cadence.      */
int  kmm_calcswirl(kmm_ctx *ctx);
/* The targets of the last scl_flag = 4 source (findmaxQ, helpers.f90:678-953, placed at
 * solvers.f90:2170-2203): 1-based (x, y, z) grid indices of the 3/2 grid, 3 ints each, in
 * placement order, into ijk (n ints available).  Returns their number (0 .. 1023), or a negative
 * status (KMM_ERR_ARG) for bad arguments.  Replaces reading the reference's Qx/Qy/Qz after the
 * loop; not in the reference's interface.                                                       */
int  kmm_target_list(kmm_ctx *ctx, int *ijk, int n);
/* Flow statistics of writeoutputs (helpers.f90:1227-1438) from the current state (runs
 * kmm_veloc first).  prof: 7 * (ny+1) doubles (host) = mean u profile (solvers.f90:3486-3494),
 * u'_rms, v_rms, w_rms, R12 = <u'v>, T12 = <du/dy>/re, and (not in the reference) the kinetic
 * energy profile 0.5 <u^2 + v^2 + w^2>; scal: 4 doubles = bulk velocity (trapezoid of
 * helpers.f90:1355-1359), top and bottom wall shear <du/dy>/re, bulk kinetic energy (same
 * trapezoid).  The x-z means come from Parseval sums over the modes, which equal the
 * reference's 3/2-grid means exactly for the dealiased fields.                          */
int  kmm_flowstats(kmm_ctx *ctx, double *prof, double *scal);

/* ---- ensemble (no counterpart in the reference, whose multi-run driver starts independent
 * processes, LO_multi_run/setup.py:93-101) ----------------------------------------------
 * Advance n independent contexts (any grids, any devices) by one step each.  Every member's
 * step is enqueued on its own stream before any is waited on, so the members overlap on the
 * GPU; members that need the routine path (polymer, IB) step synchronously.  When every member
 * is on one device, takes the fused step with graph replay and KMM_OPT_ENSEMBLE_GRAPH = 1, the
 * whole ensemble step is one CUDA graph whose child graphs are the members' captured steps
 * (cached per member set; one launch per ensemble step).  status[m] receives
 * each member's kmm_step status; the return value is the first nonzero one (KMM_OK if none).
 * The members must be distinct contexts; a context must not be used from another host thread
 * during the call.                                                                          */
#define KMM_MAX_ENSEMBLE 256
int  kmm_ensemble_step(kmm_ctx **ctxs, int n, int *status);
int  kmm_ensemble_run(kmm_ctx **ctxs, int n, int nsteps, int *status);

/* ---- options --------------------------------------------------------------- */
enum kmm_option {
    KMM_OPT_FUSED = 1,  /* 1 (default): kmm_step runs the fused kernels when the run has no polymer and no
                           immersed boundary; 0: kmm_step runs the routine-by-routine kernels   */
    KMM_OPT_COLUMN_BLOCKED = 2, /* 1 (default): the fused step's column kernels hold a column on 16
                           lanes in blocks of ny/16 coefficients (ny = 32, 64, 96, 128);
                           0: one warp per column, coefficient i on lane i mod 32           */
    KMM_OPT_GRAPH = 3,         /* 1 (default): once the tracers are initialised, the fused step is
                           captured into two CUDA graphs (the history buffers alternate between
                           two arrangements) and replayed; 0: launched kernel by kernel.  Steps
                           with stage timing on (kmm_set_timing) always run kernel by kernel. */
    KMM_OPT_ZTMA = 4,          /* 1 (default): the fused step's z transforms (FP64 and mixed) move their
                           tiles with TMA (tensor-map bulk copies, mz = 48, 96, 144, 192); 0:
                           plain loads and stores                                            */
    KMM_OPT_WAIT_LIMIT_MS = 5, /* limit of every device-side wait on an mbarrier (bulk / TMA copies), in
                           milliseconds, 100 .. 60000 (default 2000).  A wait that runs out records
                           KMM_ERR_TIMEOUT in the step status.  The limit is per device and
                           process-wide (every context on the device shares it).            */
    KMM_OPT_XBIG = 6,          /* 0 (default): the routine path's FP64 x stage keeps a row of every input
                           field in shared memory, and passes through an HBM buffer of the physical
                           inputs only where that does not fit (long 3/2 grids with polymer); 1:
                           always the two-pass form (same transforms and pointwise terms)    */
    KMM_OPT_TC_DCT = 7,        /* the routine path's mixed form (precision = 1): 1 runs its y (Chebyshev)
                           transforms as 3xTF32 GEMMs of the cosine matrix on the tcgen05 tensor
                           cores (ny = 32, 64, 96, 128); 0 (default) as FP32 FFTs of the even
                           extension                                                          */
    KMM_OPT_DERIVED_INPUTS = 8, /* 1 (default): inside the routine step, vcw3dp forms the x and z derivatives
                           of its inputs (i kx, i kz times the y-transformed field, in the z
                           inverse) instead of transforming them as separate spectral fields,
                           and the step computes only the y derivatives; 0: every input
                           materialised (gradv, gradscl, derivscji) as in the reference.  Off
                           with inertial particles, which read the gradient on the 3/2 grid.
                           The U11 .. DC333 mirrors then hold only their y-derivative members
                           after a step (kmm_gradv / kmm_derivscji recompute them)          */
    KMM_OPT_ENSEMBLE_GRAPH = 9 /* 1 (default): kmm_ensemble_step replays the members' step graphs as
                           one parent graph where it can (see above); 0: one graph launch per
                           member on its own stream.  Read from every member (all must be 1). */
};
int  kmm_set_option(kmm_ctx *ctx, int option, int value);

/* ---- bounded-wait check (no counterpart in the reference) ---------------------------
 * Runs the library's bounded mbarrier wait, with a limit of `limit_ms` (0 < limit_ms <= 10000),
 * on a barrier that nothing arrives on and no copy targets, so the wait must run out; the kernel
 * then records KMM_ERR_TIMEOUT and returns, as the step kernels do.  Returns KMM_ERR_TIMEOUT when
 * the wait gave up (the expected outcome), KMM_OK if it did not, another status on a CUDA error.
 * The context stays usable afterwards.                                                    */
int  kmm_wait_selftest(kmm_ctx *ctx, double limit_ms);

/* ---- transform without device allocation --------------------------------------
 * kmm_xyzfft_noalloc has no counterpart in the reference.  It is kmm_xyzfft (the physical ->
 * spectral transform of an initial field, helpers.f90:6-87) for callers that cannot allocate
 * device memory: a host whose device memory belongs to another allocator or a fixed budget, or a
 * time-critical loop that cannot afford cudaMalloc's implicit device synchronisation, and that
 * therefore has no kmm context (creating one allocates).  The caller passes device pointers:
 * `phys` real(8) (ny+1, nz, nx) and `spec` complex(8) (ny+1, nz, nx/2), both in the reference's
 * Fortran layout, and a cudaStream_t (NULL for the legacy default stream).  Nothing is allocated:
 * the working copy of the physical field lives in a file-scope device array of
 * KMM_XYZFFT_NOALLOC_MAX doubles (32 MiB) that every GPU loading the library holds until the
 * process exits; (ny+1)*nz*nx above that limit is rejected with KMM_ERR_ARG before any work, as are
 * transform lengths 2*ny, nx, nz that are not 2^a 3^b 5^c or exceed 4096.  Each call looks up the
 * array's device address on the current device (cudaGetSymbolAddress, which allocates nothing).
 * A call whose transform lengths differ from the previous call's on that device first sends new
 * twiddle tables from pageable host memory, so it returns only when the stream has reached that
 * copy.  Every call on a device shares the array and overwrites it completely; calls that overlap
 * on the GPU (other streams) race on it, and calls from two host threads at once also race on the
 * library's host-side cache of addresses and twiddle lengths, so serialise all calls.   */
#define KMM_XYZFFT_NOALLOC_MAX (4 * 1024 * 1024)
int  kmm_xyzfft_noalloc(const double *phys, double *spec, int nx, int ny, int nz, void *stream);

/* ---- instrumentation (no counterpart in the reference, whose only profiling is the
 * cadence timer of main_dns.f90:797-809) --------------------------------------- */
enum kmm_stage {
    KMM_STAGE_COLUMN = 0,   /* linear stage of the step before vcw3dp (main_dns.f90:203-606)   */
    KMM_STAGE_DCT_FWD,      /* vcw3dp: Chebyshev -> physical y                                  */
    KMM_STAGE_ZFFT_BWD,     /* vcw3dp: zero-pad + inverse z transform                           */
    KMM_STAGE_XPHYS,        /* vcw3dp: inverse x transform + pointwise terms                    */
    KMM_STAGE_XFWD,         /* vcw3dp: forward x transform                                      */
    KMM_STAGE_ZFFT_FWD,     /* vcw3dp: forward z transform + truncation                         */
    KMM_STAGE_DCT_BWD,      /* vcw3dp: physical -> Chebyshev y                                  */
    KMM_STAGE_POST,         /* after vcw3dp: norms, polymer force, filter, nonlin (607-771)     */
    KMM_NSTAGES
};
/* record CUDA events around each stage (on = 1) until the next kmm_get_stage_times */
int  kmm_set_timing(kmm_ctx *ctx, int on);
/* summed milliseconds and record counts per kmm_stage since the last call */
int  kmm_get_stage_times(kmm_ctx *ctx, double *ms, int *count, int nstages);
/* number of kernel launches the context has issued so far */
long long kmm_launch_count(const kmm_ctx *ctx);
/* CUDA events on the context's stream: record into slot (0..15), elapsed ms between two slots */
int  kmm_event_record(kmm_ctx *ctx, int slot);
int  kmm_event_elapsed(kmm_ctx *ctx, int slot_a, int slot_b, double *ms);

#ifdef __cplusplus
}
#endif
#endif /* KMM_H */
