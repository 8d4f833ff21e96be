// kmm_internal.cuh -- shared definitions of the B200 KMM library (context, helpers, device FFT).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/kmm.h"

#define KMM_MAXF 800
#define KMM_MAX_FFT_FACTORS 16
#define KMM_MAX_NYP 1025
#define KMM_TIMER_RECORDS 4096

// ---------------------------------------------------------------------------
// error handling: every CUDA call goes through CK, which records the message
// in the context and returns KMM_ERR_CUDA from the enclosing function.
// ---------------------------------------------------------------------------
#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e__ = (call);                                                             \
        if (e__ != cudaSuccess) {                                                             \
            kmm_set_error(ctx, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e__)); \
            return KMM_ERR_CUDA;                                                              \
        }                                                                                     \
    } while (0)

#define CKL()                                \
    do {                                     \
        CK(cudaGetLastError());              \
        ctx->launches++;                     \
    } while (0)
#define RET(x) do { int r__ = (x); if (r__) return r__; } while (0)

// FFT plan: n = product of fac[] (radices 4, 2, 3, 5); tw[m] = exp(-2 pi i m / n) in FP64
struct DevPlan {
    int n, nf;
    int fac[KMM_MAX_FFT_FACTORS];
    const double2 *tw;
};

struct kmm_ctx {
    kmm_params p;
    int device;
    cudaStream_t stream;
    cudaStream_t side;           // fused step: the tracers run here, overlapping the z-forward and back stages
    cudaStream_t side2;          // fused step: with `side`, the scalar and omega_y column kernels beside v's
    cudaEvent_t fork_ev, join_ev, cfork_ev, cjoin_ev[2];
    // grid (grid_size.f90:1-47, run-time here)
    int nx, ny, nz, nyp, nym, nxh, nyh, nzh, nyhp, nyhm, mx, mz;
    size_t nspec;   // nyp*nz*nxh
    size_t nphys;   // nyp*mz*mx
    // COMMON /solver/, /flow/, /domain/ values (main_dns.f90:934-1165)
    double re, dt, theta, gain, ugain, dyde, alpha, beta, dPdx, xl, yl, zl, uinf, pi;
    double atu, btu, gtu, abu, bbu, gbu, atw, btw, gtw, abw, bbw, gbw;
    int nt, nb;
    double p1t, p1b, p2t, p2b;
    int substep;
    int it;
    int in_step;                 // inside kmm_step (intermediate copies only kept when needed)
    int kmaxsurf;
    int ib_ylo, ib_yhi;          // 1-based y-planes holding the solid cells (0, 0: none)
    // host and device copies of wavenumbers, Chebyshev weights, grid
    double *h_wavx, *h_wavz, *h_c, *h_ycoord, *h_seght;
    double *d_wavx, *d_wavz, *d_c, *d_ycoord, *d_seght;
    double h_fspread[10][10];
    double *d_fspread;
    // field mirrors
    void *f[KMM_MAXF];
    // scratch
    double2 *wrk[6];            // spectral-size scratch
    double2 *pl_in, *pl_out;     // y-physical spectral-xz planes (fields x nyp x nxh x nz)
    double2 *q_in, *q_out;       // after the z transform (fields x nyp x mz x nxh)
    size_t pl_in_fields, pl_out_fields;
    double *d_cfl;               // nyp
    int *d_status;               // device-raised status
    double *d_pumax;             // inertial particles: part_track's running max relative speed (umax1)
    double *d_umax;              // scratch for |u| max (per plane)
    double *d_scratch;           // 9*KMM_MAX_NYP doubles for the (0,0)-mode solver
    double *h_pin;               // pinned host: cfl[KMM_MAX_NYP], umax[KMM_MAX_NYP], status (step read-backs)
    double *scsource;            // the KMM_SCSOURCE field's storage (scl_flag = 2, 4, 5)
    // targeted sources (scl_flag = 4, 5): -Q on the 3/2 grid, the candidate list and its count,
    // the placed targets' centres, reduction scratch; the host copy of the last targets
    double *d_tgtq, *d_tgtc, *d_tgtred;
    void *d_tgtlist, *h_tgtlist;
    unsigned *d_tgtcnt;
    size_t tgt_cap;
    int ntarg;
    int *h_targ;                 // 3 * 1023 ints: x, y, z grid indices (1-based) of the targets
    DevPlan py2, pmz, pmx, pnx, pnz;
    DevPlan wy2, wmz, wmx;        // same lengths, radix-8-first factorisation for the warp FFT
    double2 *tw_store[5];
    kmm_stats stats;
    char err[512];
    // instrumentation: kernel launches issued, and CUDA-event stage timers (bench / profiling)
    long long launches;
    int timing_on;
    int tm_n;
    int tm_stage[KMM_TIMER_RECORDS];
    cudaEvent_t tm_ev[2 * KMM_TIMER_RECORDS];
    int tm_ev_ready;
    cudaEvent_t user_ev[16];
    // fused-path state (tau tables, stage buffers) and the general path's physical scratch
    struct KmmFused *fused;
    double *po, *drag;
    size_t po_n, drag_n;
    double *xbig;     // physical inputs of the two-pass x stage (3/2 grids past the shared-memory rows)
    size_t xbig_n;
    int force_xbig;   // KMM_OPT_XBIG
    int use_tcdct;    // KMM_OPT_TC_DCT: the mixed routine path's y transforms on the tensor cores
    int use_derived;  // KMM_OPT_DERIVED_INPUTS: vcw3dp forms the x / z derivative inputs itself
    int *d_tcstat;    // device status word of the tensor-core transforms (KMM_ERR_TIMEOUT)
    int use_fused;
    int use_colblk;   // fused step: blocked-layout column kernels where compiled (default 1)
    // fused step replayed from CUDA graphs (one per parity of the swapped history buffers)
    int use_graph, graph_ready;
    cudaGraphExec_t gexec[2];
    long long gkernels[2];   // kernels in each graph (added to the launch count per replay)
    cudaGraph_t ggraph[2];   // the captured graphs (child graphs of an ensemble step)
    unsigned long long ggen;  // incremented whenever the graphs are captured or released
    int use_ens_graph;        // KMM_OPT_ENSEMBLE_GRAPH
    cudaEvent_t ens_ev;       // an ensemble graph's completion, waited on by this member's stream
    void *g_fn0;      // the FN buffer of parity 0
    int use_ztma;     // FP64 inverse z transform through TMA tile copies (default 1)
    void *ztma;       // its cached tensor maps (kmm_ztma.cu)
    void *tauc;       // tau tables of the routine solves' (g, boundary-condition) configurations (kmm_fused.cu)
    float2 *rtw32[3]; // FP32 twiddles of 2 ny, mz, mx for the routine path's mixed form (kmm_fused.cu)
    double *d_frate;  // constant flow rate: W, G, the last correction, scratch (kmm_column.cu)
    int frate_ready;
    void *hoststate;  // host arrays bound by kmm_bind_host, their copy streams and events (kmm_hoststate.cu)
};

void kmm_hoststate_release(kmm_ctx *ctx);
void kmm_fused_release(kmm_ctx *ctx);
int kmm_fused_step(kmm_ctx *ctx);
// the fused step in two halves: enqueue every kernel and the read-back of CFL / status, then wait
// and evaluate (kmm_fused_step = launch + finish; the ensemble launches all members first)
int kmm_fused_launch(kmm_ctx *ctx);
int kmm_fused_finish(kmm_ctx *ctx);
int kmm_fused_graph_for_step(kmm_ctx *ctx, int *parity);
unsigned long long kmm_graph_generation();   // a process-wide counter: every capture / release gets a new value
void kmm_ensemble_forget(kmm_ctx *ctx);      // drop the cached ensemble graphs that hold ctx
void kmm_fused_replayed(kmm_ctx *ctx, int parity);
// one fused step enqueued on ctx->stream: through the captured graphs when enabled and ready
// (captured on first use), else kernel by kernel
int kmm_fused_enqueue(kmm_ctx *ctx);
void kmm_graph_release(kmm_ctx *ctx);
bool kmm_fused_applicable(const kmm_ctx *ctx);
// TMA forms of the z transforms, FP64 and FP32 (kmm_ztma.cu)
bool kmm_ztma_supported(const kmm_ctx *ctx);
int kmm_zb_tma(kmm_ctx *ctx, const double2 *yp, double2 *q, int nbase, int nq, const double2 *tw);
int kmm_zf_tma(kmm_ctx *ctx, const double2 *r, double2 *yo, int nout, const double2 *tw);
int kmm_zb_tma32(kmm_ctx *ctx, const float2 *yp, float2 *q, int nbase, int nq, const float2 *tw);
int kmm_zf_tma32(kmm_ctx *ctx, const float2 *r, float2 *yo, int nout, const float2 *tw);
void kmm_ztma_release(kmm_ctx *ctx);
// bounded-wait limits of the units with mbarrier waits (on the current device; nonzero on failure)
int kmm_ztma_set_wait_limit(unsigned long long ns);
int kmm_plane_set_wait_limit(unsigned long long ns);
void kmm_tic(kmm_ctx *ctx);
void kmm_toc(kmm_ctx *ctx, int stage);

void kmm_set_error(kmm_ctx *ctx, const char *fmt, ...);

// field helpers (kmm_ctx.cu)
int kmm_field_info(const kmm_ctx *ctx, int field, size_t *nelem, int *eb);
void *kmm_field_ptr(kmm_ctx *ctx, int field);   // allocates (zeroed) on first use, NULL on failure
static inline double2 *SPEC(kmm_ctx *ctx, int f) { return (double2 *)kmm_field_ptr(ctx, f); }
static inline double *REAL(kmm_ctx *ctx, int f) { return (double *)kmm_field_ptr(ctx, f); }
// the pinned status word after the cfl and umax rows of h_pin, and the flow-rate correction after it
static inline int *kmm_h_pin_status(kmm_ctx *ctx) { return (int *)(ctx->h_pin + 2 * KMM_MAX_NYP); }
static inline double *kmm_h_pin_delta(kmm_ctx *ctx) { return ctx->h_pin + 2 * KMM_MAX_NYP + 1; }
static inline int *kmm_h_pin_tcstat(kmm_ctx *ctx) { return (int *)(ctx->h_pin + 2 * KMM_MAX_NYP + 2); }
#define KMM_H_PIN_DOUBLES (2 * KMM_MAX_NYP + 3)

// internal entry points shared between translation units
int kmm_internal_cderiv(kmm_ctx *ctx, const double2 *f, double2 *df);
// cderiv of n independent (input, output) pairs, KMM_CDERIV_BATCH to a launch (no output may be
// another pair's input; an output may be its own pair's input)
#define KMM_CDERIV_BATCH 16
int kmm_internal_cderiv_many(kmm_ctx *ctx, const double2 *const *f, double2 *const *df, int n);
int kmm_internal_norm(kmm_ctx *ctx, double2 *a);
// norm of nf distinct fields, KMM_NORM_BATCH to a launch (the same values as one call per field)
#define KMM_NORM_BATCH 32
int kmm_internal_norm_many(kmm_ctx *ctx, double2 *const *a, int nf);
int kmm_internal_wallderiv(kmm_ctx *ctx, const double2 *f, int order, int wall, double2 *out, int iy);
int kmm_internal_solve(kmm_ctx *ctx, double2 *u, double g, int ib, const double2 *bct, const double2 *bcb);
// uzero for u0 (uflag 1) or w0 (3) on stream st (one block, the (0,0) mode)
int kmm_internal_uzero(kmm_ctx *ctx, int uflag, cudaStream_t st);
// the routine solve / penta with the blocked column kernels (ny = 32, 64, 96, 128; ib = 0);
// KMM_ERR_UNSUPPORTED where they do not apply (kmm_colblk.cu)
int kmm_colblk_solve(kmm_ctx *ctx, double2 *u, double g, int robin, double at, double bt, double ab, double bb,
                     const double2 *gt, const double2 *gb);
// the same over nf distinct fields of one configuration (same g, boundary coefficients and
// boundary values), KMM_SOLVE_BATCH to a launch
#define KMM_SOLVE_BATCH 8
int kmm_colblk_solve_many(kmm_ctx *ctx, double2 *const *u, int nf, double g, int robin, double at, double bt,
                          double ab, double bb, const double2 *gt, const double2 *gb);
// the routine step's phirhs followed by one or two tau solves with zero boundary values, fused per
// column pair (blocked kernels, ny = 32 .. 128 and 256): x[m] <- solve(phirhs([phi of] x[m]; fn[m], fnm1[m],
// var)), fnm1[m] = NULL taking 2 fn[m]; KMM_ERR_UNSUPPORTED where the blocked kernels do not apply
struct KmmSolveSpec {
    double g;
    int robin;   // 1: penta (Robin coefficients at, bt, ab, bb), 0: solve (Dirichlet)
    double at, bt, ab, bb;
};
int kmm_colblk_phirhs_solve(kmm_ctx *ctx, double2 *const *x, const double2 *const *fn, const double2 *const *fnm1,
                            int nf, double var, int phi, int nsolve, const KmmSolveSpec *spec);
// penta (ib = 0) of nf distinct fields of one configuration
int kmm_internal_penta_many(kmm_ctx *ctx, double2 *const *u, int nf, double g, double at, double bt, double ab,
                            double bb, const double2 *gt, const double2 *gb);
// phirhs of nf independent fields (at most KMM_PHI_BATCH), each with its own two scratch fields;
// FM[m] = NULL takes 2 F[m] as the n-1 term (the polymer components' call)
#define KMM_PHI_BATCH 8
int kmm_internal_phirhs_many(kmm_ctx *ctx, double2 *const *V, const double2 *const *F, const double2 *const *FM,
                             int nf, double var, double2 *const *wrkc, double2 *const *wrk1);
// the cached tau tables of one configuration and the tau-row reciprocals (kmm_fused.cu)
int kmm_tau_tabset(kmm_ctx *ctx, double g, int robin, double at, double bt, double ab, double bb, const double **tabs,
                   const double **rj);
void kmm_tau_release(kmm_ctx *ctx);
// FP32 twiddle tables (2 ny, mz, mx) of the routine path's mixed form, built on first use (kmm_fused.cu)
int kmm_routine_tw32(kmm_ctx *ctx, const float2 **y2, const float2 **mz, const float2 **mx);
int kmm_internal_penta(kmm_ctx *ctx, double2 *u, double g, int ib, double at, double bt, double ab, double bb,
                       const double2 *gt, const double2 *gb);
int kmm_internal_set_constant_mode(kmm_ctx *ctx, double2 *a, double value);
int kmm_plan_init(kmm_ctx *ctx, DevPlan *p, int n, int slot);
void kmm_plan_r8(const DevPlan *src, DevPlan *dst);
int kmm_smem_attr(kmm_ctx *ctx, const void *func, size_t bytes);
int kmm_ensure_plane_buffers(kmm_ctx *ctx, int nin, int nout);
// (nyp,mz,mx) host array <-> internal [y][z][x] device array (one of host_src / host_dst is NULL)
int kmm_phys_layout(kmm_ctx *ctx, int field, void *dev, const void *host_src, void *host_dst);
int kmm_internal_polynl(kmm_ctx *ctx, double2 *const *nl);
int kmm_internal_phirhs(kmm_ctx *ctx, double2 *V, const double2 *F, const double2 *FM, double var);
// the y transforms of nf fields (dir 0: FP64 columns -> FP32 planes; 1: FP32 planes -> FP64
// columns) as 3xTF32 tcgen05 GEMMs (kmm_tcdct.cu); KMM_ERR_UNSUPPORTED where they do not apply
#define KMM_TC_MAXF 64
int kmm_tc_dct(kmm_ctx *ctx, int dir, const void *const *in, void *const *out, int nf);
bool kmm_derived_inputs(const kmm_ctx *ctx);
// constant flow rate (kmm_params.flow_rate > 0): tables built once by kmm_initial, the correction
// after every u0 solve (kmm_column.cu)
int kmm_flowrate_setup(kmm_ctx *ctx);
int kmm_flowrate_apply(kmm_ctx *ctx, cudaStream_t st);

// ---------------------------------------------------------------------------
// complex helpers on double2
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cdivr(double2 a, double s) { return make_double2(a.x / s, a.y / s); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// i*s*a for real s
__host__ __device__ __forceinline__ double2 cimul(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }
// complex division as C99 does for finite operands (a/b)
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    double den = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / den, (a.y * b.x - a.x * b.y) / den);
}

// ---------------------------------------------------------------------------
// shared-memory Stockham FFT over a batch of sequences.
//   a, b: two smem buffers; sequence s occupies [s*ld, s*ld + n).
//   sign -1: exp(-2 pi i jk/n) (FFTW_FORWARD), +1: exp(+...) (FFTW_BACKWARD).
//   All threads of the block must call it; returns the buffer holding the result.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void radix_dft(int R, double2 *v, int sign) {
    if (R == 2) {
        double2 a0 = v[0], a1 = v[1];
        v[0] = cadd(a0, a1);
        v[1] = csub(a0, a1);
    } else if (R == 4) {
        double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        double2 b0 = cadd(v[1], v[3]);
        double2 d = csub(v[1], v[3]);
        double2 b1 = sign < 0 ? make_double2(d.y, -d.x) : make_double2(-d.y, d.x);  // sign*i*d
        v[0] = cadd(a0, b0);
        v[1] = cadd(a1, b1);
        v[2] = csub(a0, b0);
        v[3] = csub(a1, b1);
    } else if (R == 3) {
        const double s3 = 0.86602540378443864676 * (double)sign;
        double2 t1 = cadd(v[1], v[2]);
        double2 t2 = csub(v[0], cscale(t1, 0.5));
        double2 d = csub(v[1], v[2]);
        double2 t3 = make_double2(s3 * d.x, s3 * d.y);
        double2 o0 = cadd(v[0], t1);
        v[1] = make_double2(t2.x - t3.y, t2.y + t3.x);   // t2 + i t3
        v[2] = make_double2(t2.x + t3.y, t2.y - t3.x);   // t2 - i t3
        v[0] = o0;
    } else {  // R == 5
        const double c5a = 0.30901699437494742410, c5b = -0.80901699437494742410;
        const double s5a = 0.95105651629515357212 * (double)sign, s5b = 0.58778525229247312917 * (double)sign;
        double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        double2 o0 = cadd(v[0], cadd(t1, t2));
        double2 r1 = cadd(v[0], cadd(cscale(t1, c5a), cscale(t2, c5b)));
        double2 r2 = cadd(v[0], cadd(cscale(t1, c5b), cscale(t2, c5a)));
        double2 m1 = cadd(cscale(t3, s5a), cscale(t4, s5b));
        double2 m2 = csub(cscale(t3, s5b), cscale(t4, s5a));
        double2 i1 = make_double2(-m1.y, m1.x), i2 = make_double2(-m2.y, m2.x);
        v[0] = o0;
        v[1] = cadd(r1, i1);
        v[4] = csub(r1, i1);
        v[2] = cadd(r2, i2);
        v[3] = csub(r2, i2);
    }
}

__device__ __forceinline__ double2 *fft_smem(const DevPlan &P, double2 *a, double2 *b, int nseq, int ld, int sign) {
    const int n = P.n;
    double2 *src = a, *dst = b;
    int Ns = 1;
    for (int f = 0; f < P.nf; ++f) {
        const int R = P.fac[f];
        const int nR = n / R;
        const int tstep = n / (Ns * R);
        const int total = nseq * nR;
        for (int t = threadIdx.x; t < total; t += blockDim.x) {
            const int s = t / nR, j = t - s * nR;
            const int k = j % Ns;
            const double2 *sp = src + (size_t)s * ld;
            double2 *dp = dst + (size_t)s * ld;
            double2 v[5];
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                if (r < R) {
                    double2 x = sp[j + r * nR];
                    if (r && k) {
                        double2 w = __ldg(&P.tw[(r * k * tstep) % n]);
                        if (sign > 0) w.y = -w.y;
                        x = cmul(x, w);
                    }
                    v[r] = x;
                }
            }
            radix_dft(R, v, sign);
            const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int q = 0; q < 5; ++q)
                if (q < R) dp[idxD + q * Ns] = v[q];
        }
        __syncthreads();
        double2 *tmp = src;
        src = dst;
        dst = tmp;
        Ns *= R;
    }
    return src;
}

// radix-8 DFT (two radix-4 halves + the W8 twiddles), same sign convention as radix_dft
__device__ __forceinline__ void radix8_dft(double2 *v, int sign) {
    double2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    radix_dft(4, e, sign);
    radix_dft(4, o, sign);
    const double h = 0.70710678118654752440;
    // W8^q o[q], W8 = exp(sign 2 pi i / 8)
    double2 t1 = make_double2(h * (o[1].x - sign * o[1].y), h * (o[1].y + sign * o[1].x));
    double2 t2 = sign < 0 ? make_double2(o[2].y, -o[2].x) : make_double2(-o[2].y, o[2].x);
    double2 t3 = make_double2(h * (-o[3].x - sign * o[3].y), h * (-o[3].y + sign * o[3].x));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);
    v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);
    v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);
    v[7] = csub(e[3], t3);
}

// ---------------------------------------------------------------------------
// warp-private Stockham FFT: one sequence of length P.n in the warp's own shared buffers a, b;
// only __syncwarp between stages.  Radices 8, 4, 2, 3, 5 (plan from kmm_plan_r8).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 *fft_warp(const DevPlan &P, double2 *a, double2 *b, int sign) {
    const int n = P.n;
    const int lane = threadIdx.x & 31;
    double2 *src = a, *dst = b;
    int Ns = 1;
    for (int f = 0; f < P.nf; ++f) {
        const int R = P.fac[f];
        const int nR = n / R;
        const int tstep = n / (Ns * R);
        for (int j = lane; j < nR; j += 32) {
            const int k = j % Ns;
            double2 v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                if (r < R) {
                    double2 x = src[j + r * nR];
                    if (r && k) {
                        double2 w = __ldg(&P.tw[(r * k * tstep) % n]);
                        if (sign > 0) w.y = -w.y;
                        x = cmul(x, w);
                    }
                    v[r] = x;
                }
            }
            if (R == 8) radix8_dft(v, sign);
            else radix_dft(R, v, sign);
            const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (q < R) dst[idxD + q * Ns] = v[q];
        }
        __syncwarp();
        double2 *tmp = src;
        src = dst;
        dst = tmp;
        Ns *= R;
    }
    return src;
}

static inline int kmm_blocks(size_t n, int threads) {
    size_t b = (n + threads - 1) / threads;
    if (b > 148 * 32) b = 148 * 32;
    if (b < 1) b = 1;
    return (int)b;
}
