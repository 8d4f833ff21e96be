// kmm_ctx.cu -- context lifetime, field mirrors, FFT plans (setstuff / setbcs / forcepre equivalents).
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>

#include "kmm_internal.cuh"

void kmm_set_error(kmm_ctx *ctx, const char *fmt, ...) {
    if (!ctx) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
    va_end(ap);
}

extern "C" const char *kmm_last_error(const kmm_ctx *ctx) { return ctx ? ctx->err : "null context"; }
extern "C" int kmm_abi_version(void) { return KMM_ABI_VERSION; }

int kmm_field_info(const kmm_ctx *c, int f, size_t *nelem, int *eb) {
    size_t n = 0;
    int b = 0;
    if (f >= 0 && f < KMM_NSPECTRAL) { n = c->nspec; b = 16; }
    else if (f >= KMM_U0 && f < KMM_NMEAN_END) { n = (size_t)c->nyp; b = 8; }
    else if (f >= KMM_BCTOP && f < KMM_NWALL_END) { n = (size_t)c->nz * c->nxh; b = 16; }
    else if (f >= KMM_FXINTG && f < KMM_NPHYS_END) { n = c->nphys; b = 8; }
    else if (f == KMM_IMATRIX) { n = c->nphys; b = 4; }
    else if (f >= KMM_XPART && f < KMM_NPART_END) { n = (size_t)(c->p.npart > 0 ? c->p.npart : 0); b = 8; }
    else if (f >= KMM_INITU && f < KMM_NINIT_END) { n = (size_t)c->nyp * c->nz * c->nx; b = 8; }
    if (nelem) *nelem = n;
    if (eb) *eb = b;
    return b ? KMM_OK : KMM_ERR_ARG;
}

void *kmm_field_ptr(kmm_ctx *ctx, int f) {
    if (f < 0 || f >= KMM_MAXF) return NULL;
    if (ctx->f[f]) return ctx->f[f];
    size_t n;
    int b;
    if (kmm_field_info(ctx, f, &n, &b)) return NULL;
    size_t bytes = n * (size_t)b;
    if (bytes == 0) bytes = 16;
    void *p = NULL;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        kmm_set_error(ctx, "cudaMalloc(%zu) failed for field %d", bytes, f);
        return NULL;
    }
    if (cudaMemsetAsync(p, 0, bytes, ctx->stream) != cudaSuccess) {
        cudaFree(p);
        return NULL;
    }
    ctx->f[f] = p;
    return p;
}

extern "C" int kmm_field_size(const kmm_ctx *ctx, int field, size_t *nelem, int *elem_bytes) {
    if (!ctx) return KMM_ERR_ARG;
    return kmm_field_info(ctx, field, nelem, elem_bytes);
}

extern "C" int kmm_upload(kmm_ctx *ctx, int field, const void *host, size_t bytes) {
    if (!ctx || !host) return KMM_ERR_ARG;
    size_t n;
    int b;
    if (kmm_field_info(ctx, field, &n, &b) || bytes != n * (size_t)b) {
        kmm_set_error(ctx, "kmm_upload: field %d expects %zu bytes, got %zu", field, n * (size_t)b, bytes);
        return KMM_ERR_ARG;
    }
    void *d = kmm_field_ptr(ctx, field);
    if (!d) return KMM_ERR_NOMEM;
    if (field == KMM_IMATRIX) ctx->kmaxsurf = -1;  // recomputed on the next vcw3dp
    if (field == KMM_IMATRIX || (field >= KMM_FXINTG && field < KMM_NPHYS_END))
        return kmm_phys_layout(ctx, field, d, host, NULL);
    CK(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return KMM_OK;
}

extern "C" int kmm_download(kmm_ctx *ctx, int field, void *host, size_t bytes) {
    if (!ctx || !host) return KMM_ERR_ARG;
    size_t n;
    int b;
    if (kmm_field_info(ctx, field, &n, &b) || bytes != n * (size_t)b) {
        kmm_set_error(ctx, "kmm_download: field %d expects %zu bytes, got %zu", field, n * (size_t)b, bytes);
        return KMM_ERR_ARG;
    }
    void *d = kmm_field_ptr(ctx, field);
    if (!d) return KMM_ERR_NOMEM;
    if (field == KMM_IMATRIX || (field >= KMM_FXINTG && field < KMM_NPHYS_END))
        return kmm_phys_layout(ctx, field, d, NULL, host);
    CK(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return KMM_OK;
}

extern "C" int kmm_copy(kmm_ctx *ctx, int dst, int src) {
    if (!ctx) return KMM_ERR_ARG;
    size_t n1, n2;
    int b1, b2;
    if (kmm_field_info(ctx, dst, &n1, &b1) || kmm_field_info(ctx, src, &n2, &b2) || n1 != n2 || b1 != b2)
        return KMM_ERR_ARG;
    void *d = kmm_field_ptr(ctx, dst), *s = kmm_field_ptr(ctx, src);
    if (!d || !s) return KMM_ERR_NOMEM;
    CK(cudaMemcpyAsync(d, s, n1 * (size_t)b1, cudaMemcpyDeviceToDevice, ctx->stream));
    return KMM_OK;
}

extern "C" int kmm_zero(kmm_ctx *ctx, int field) {
    if (!ctx) return KMM_ERR_ARG;
    size_t n;
    int b;
    if (kmm_field_info(ctx, field, &n, &b)) return KMM_ERR_ARG;
    void *d = kmm_field_ptr(ctx, field);
    if (!d) return KMM_ERR_NOMEM;
    CK(cudaMemsetAsync(d, 0, n * (size_t)b, ctx->stream));
    return KMM_OK;
}

extern "C" int kmm_set_it(kmm_ctx *ctx, int it) {
    if (!ctx) return KMM_ERR_ARG;
    ctx->it = it;
    kmm_graph_release(ctx);   // the captured steps assume the tracer phase of the current it
    return KMM_OK;
}

extern "C" int kmm_sync(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return KMM_OK;
}

extern "C" int kmm_get_stats(kmm_ctx *ctx, kmm_stats *out) {
    if (!ctx || !out) return KMM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->stats.it = ctx->it;
    ctx->stats.dpdx = ctx->dPdx - (ctx->p.flow_rate > 0.0 ? *kmm_h_pin_delta(ctx) : 0.0);
    *out = ctx->stats;
    return KMM_OK;
}

// FFT plan with FP64 twiddles computed on the host in long double
int kmm_plan_init(kmm_ctx *ctx, DevPlan *p, int n, int slot) {
    int m = n, nf = 0;
    static const int rads[4] = {4, 2, 3, 5};
    for (int r = 0; r < 4; ++r)
        while (m % rads[r] == 0 && nf < KMM_MAX_FFT_FACTORS) {
            p->fac[nf++] = rads[r];
            m /= rads[r];
        }
    if (m != 1) {
        kmm_set_error(ctx, "transform length %d is not of the form 2^a 3^b 5^c", n);
        return KMM_ERR_ARG;
    }
    p->n = n;
    p->nf = nf;
    double2 *h = (double2 *)malloc(sizeof(double2) * (size_t)n);
    for (int k = 0; k < n; ++k) {
        long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
        h[k] = make_double2((double)cosl(a), -(double)sinl(a));
    }
    double2 *d = NULL;
    cudaError_t e = cudaMalloc(&d, sizeof(double2) * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(d, h, sizeof(double2) * (size_t)n, cudaMemcpyHostToDevice);
    free(h);
    if (e != cudaSuccess) {
        kmm_set_error(ctx, "plan %d: %s", n, cudaGetErrorString(e));
        return KMM_ERR_CUDA;
    }
    ctx->tw_store[slot] = d;
    p->tw = d;
    return KMM_OK;
}

// same transform length and twiddle table, factors ordered 8, 4, 2, 3, 5 (fewer warp-FFT stages)
void kmm_plan_r8(const DevPlan *src, DevPlan *dst) {
    *dst = *src;
    int m = src->n, nf = 0;
    static const int rads[5] = {8, 4, 2, 3, 5};
    for (int r = 0; r < 5; ++r)
        while (m % rads[r] == 0 && nf < KMM_MAX_FFT_FACTORS) {
            dst->fac[nf++] = rads[r];
            m /= rads[r];
        }
    dst->nf = nf;
}

// setbcs, main_dns.f90:1175-1418
static void setbcs(kmm_ctx *c) {
    switch (c->p.flow_select) {
    case 1: case 11:
        c->atu = 1; c->btu = 0; c->gtu = 0; c->atw = 1; c->btw = 0; c->gtw = 0;
        c->abu = 1; c->bbu = 0; c->gbu = 0; c->abw = 1; c->bbw = 0; c->gbw = 0;
        c->nt = 1; c->nb = 1; break;
    case 2: case 12:
        c->atu = 1; c->btu = 0; c->gtu = c->uinf; c->atw = 1; c->btw = 0; c->gtw = 0;
        c->abu = 1; c->bbu = 0; c->gbu = 0; c->abw = 1; c->bbw = 0; c->gbw = 0;
        c->nt = 1; c->nb = 1; break;
    case 3:
        c->atu = 1; c->btu = 0; c->gtu = c->uinf; c->atw = 1; c->btw = 0; c->gtw = c->uinf;
        c->abu = 1; c->bbu = 0; c->gbu = 0; c->abw = 1; c->bbw = 0; c->gbw = 0;
        c->nt = 1; c->nb = 1; break;
    case 4:
        c->atu = 0; c->btu = 1; c->gtu = 0; c->atw = 0; c->btw = 1; c->gtw = 0;
        c->abu = 1; c->bbu = 0; c->gbu = 0; c->abw = 1; c->bbw = 0; c->gbw = 0;
        c->nt = 2; c->nb = 1; break;
    default:
        c->atu = 0; c->btu = 1; c->gtu = 0; c->atw = 0; c->btw = 1; c->gtw = 0;
        c->abu = 0; c->bbu = 1; c->gbu = 0; c->abw = 0; c->bbw = 1; c->gbw = 0;
        c->nt = 2; c->nb = 2; break;
    }
    c->p1b = 1.0; c->p1t = -1.0; c->p2b = -1.0; c->p2t = 0.5;
}

extern "C" int kmm_ctx_destroy(kmm_ctx *ctx);

extern "C" int kmm_ctx_create(const kmm_params *p, int device, kmm_ctx **out) {
    if (!p || !out) return KMM_ERR_ARG;
    *out = NULL;
    if (p->nx < 4 || p->ny < 8 || p->nz < 4 || p->nx % 2 || p->ny % 2 || p->nz % 4 || p->ny + 1 > KMM_MAX_NYP)
        return KMM_ERR_ARG;
    if (p->npart < 0 || p->dt <= 0 || p->re <= 0 || p->theta <= 0) return KMM_ERR_ARG;
    kmm_ctx *ctx = (kmm_ctx *)calloc(1, sizeof(kmm_ctx));
    ctx->p = *p;
    ctx->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ctx->side2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ctx->cfork_ev, cudaEventDisableTiming));
    for (int e = 0; e < 2; ++e) CK(cudaEventCreateWithFlags(&ctx->cjoin_ev[e], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming));
    kmm_ctx *c = ctx;
    c->nx = p->nx; c->ny = p->ny; c->nz = p->nz;
    c->nyp = c->ny + 1; c->nym = c->ny - 1; c->nxh = c->nx / 2; c->nyh = c->ny / 2; c->nzh = c->nz / 2;
    c->nyhp = c->nyh + 1; c->nyhm = c->nyh - 1; c->mx = 3 * c->nx / 2; c->mz = 3 * c->nz / 2;
    c->nspec = (size_t)c->nyp * c->nz * c->nxh;
    c->nphys = (size_t)c->nyp * c->mz * c->mx;
    c->re = p->re; c->dt = p->dt; c->theta = p->theta; c->gain = p->gain; c->ugain = p->ugain;
    c->xl = p->xl; c->yl = p->yl; c->zl = p->zl; c->uinf = p->uinf;
    c->pi = 2.0 * acos(0.0);
    // setstuff, main_dns.f90:1112-1165
    c->h_ycoord = (double *)calloc((size_t)c->nyp, sizeof(double));
    c->h_seght = (double *)calloc((size_t)c->nyp, sizeof(double));
    c->h_ycoord[0] = c->yl / 2.0;
    for (int k = 2; k <= c->nyp; ++k) {
        c->h_ycoord[k - 1] = cos((double)(k - 1) * c->pi / (double)c->ny) * (c->yl / 2.0);
        c->h_seght[k - 1] = fabs(c->h_ycoord[k - 1] - c->h_ycoord[k - 2]);
    }
    c->h_seght[0] = c->h_seght[c->nyp - 1];
    c->alpha = 2.0 * c->pi / c->xl;
    c->beta = 2.0 * c->pi / c->zl;
    c->h_wavx = (double *)calloc((size_t)c->nxh, sizeof(double));
    c->h_wavz = (double *)calloc((size_t)c->nz, sizeof(double));
    for (int k = 1; k <= c->nxh; ++k) c->h_wavx[k - 1] = (double)(k - 1) * c->alpha;
    for (int j = 1; j <= c->nzh; ++j) c->h_wavz[j - 1] = (double)(j - 1) * c->beta;
    for (int j = c->nzh + 1; j <= c->nz; ++j) c->h_wavz[j - 1] = (double)(j - c->nz - 1) * c->beta;
    c->h_c = (double *)calloc((size_t)c->nyp, sizeof(double));
    for (int i = 0; i < c->nyp; ++i) c->h_c[i] = 1.0;
    c->h_c[0] = 2.0;
    c->h_c[c->nyp - 1] = 2.0;
    c->dyde = 2.0 / c->yl;
    setbcs(c);
    c->dPdx = -2.0 / c->yl * pow(2.0 * p->r_tau / (c->yl * c->re), 2);  // init_flow.f90:117
    for (int i = 1; i <= 10; ++i)
        for (int j = 1; j <= 10; ++j) {
            double dsq = (double)((i - 1) * (i - 1)) + (double)((j - 1) * (j - 1));
            c->h_fspread[i - 1][j - 1] = dsq < 13 ? exp(-2.0 * dsq) : 0.0;   // main_dns.f90:1551-1558
        }
    {   // substep_check, part_track.f90:296-356
        double Pi_f = 1.0 / (p->ratio + 0.5), tau;
        if (p->cd_switch == 0) tau = 1.0;
        else if (p->cd_switch == 1) tau = c->re * p->ap * p->ap / (6.0 * Pi_f);
        else tau = 2.0 * c->re * p->ap * p->ap / (9.0 * Pi_f);
        double s = 2.0 * c->dt / tau;
        c->substep = (int)ceil(s > 1.0 ? s : 1.0);
    }
    c->kmaxsurf = -1;
    c->use_fused = 1;
    c->use_colblk = 1;
    c->use_graph = 1;
    c->use_ztma = 1;
    c->use_derived = 1;
    c->use_ens_graph = 1;
#define DUP(dst, src, n)                                                        \
    do {                                                                        \
        CK(cudaMalloc(&(dst), sizeof(double) * (size_t)(n)));                   \
        CK(cudaMemcpy((dst), (src), sizeof(double) * (size_t)(n), cudaMemcpyHostToDevice)); \
    } while (0)
    DUP(c->d_wavx, c->h_wavx, c->nxh);
    DUP(c->d_wavz, c->h_wavz, c->nz);
    DUP(c->d_c, c->h_c, c->nyp);
    DUP(c->d_ycoord, c->h_ycoord, c->nyp);
    DUP(c->d_seght, c->h_seght, c->nyp);
    DUP(c->d_fspread, &c->h_fspread[0][0], 100);
#undef DUP
    CK(cudaMalloc(&c->d_cfl, sizeof(double) * (size_t)c->nyp));
    CK(cudaMalloc(&c->d_umax, sizeof(double) * (size_t)c->nyp));
    CK(cudaMalloc(&c->d_status, sizeof(int)));
    CK(cudaMalloc(&c->d_tcstat, sizeof(int)));
    CK(cudaMemset(c->d_tcstat, 0, sizeof(int)));
    CK(cudaMalloc(&c->d_pumax, sizeof(double)));
    CK(cudaMemset(c->d_pumax, 0, sizeof(double)));
    CK(cudaMalloc(&c->d_scratch, sizeof(double) * 9 * KMM_MAX_NYP));
    CK(cudaMallocHost(&c->h_pin, sizeof(double) * KMM_H_PIN_DOUBLES));
    memset(c->h_pin, 0, sizeof(double) * KMM_H_PIN_DOUBLES);
    CK(cudaMemset(c->d_status, 0, sizeof(int)));
    for (int w = 0; w < 6; ++w) {
        CK(cudaMalloc(&c->wrk[w], sizeof(double2) * c->nspec));
        CK(cudaMemset(c->wrk[w], 0, sizeof(double2) * c->nspec));
    }
    int st = kmm_plan_init(c, &c->py2, 2 * c->ny, 0);
    if (!st) st = kmm_plan_init(c, &c->pmz, c->mz, 1);
    if (!st) st = kmm_plan_init(c, &c->pmx, c->mx, 2);
    if (!st) st = kmm_plan_init(c, &c->pnx, c->nx, 3);
    if (!st) st = kmm_plan_init(c, &c->pnz, c->nz, 4);
    if (!st) {
        kmm_plan_r8(&c->py2, &c->wy2);
        kmm_plan_r8(&c->pmz, &c->wmz);
        kmm_plan_r8(&c->pmx, &c->wmx);
    }
    if (st) {
        kmm_ctx_destroy(c);
        return st;
    }
    *out = c;
    return KMM_OK;
}

extern "C" int kmm_ctx_destroy(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->tm_ev_ready)
        for (int e = 0; e < 2 * KMM_TIMER_RECORDS; ++e) cudaEventDestroy(ctx->tm_ev[e]);
    for (int e = 0; e < 16; ++e)
        if (ctx->user_ev[e]) cudaEventDestroy(ctx->user_ev[e]);
    kmm_ensemble_forget(ctx);   // cached ensemble graphs replay this context's buffers
    kmm_hoststate_release(ctx);
    kmm_graph_release(ctx);
    kmm_fused_release(ctx);
    kmm_ztma_release(ctx);
    kmm_tau_release(ctx);
    if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
    if (ctx->po) cudaFree(ctx->po);
    if (ctx->drag) cudaFree(ctx->drag);
    if (ctx->d_frate) cudaFree(ctx->d_frate);
    if (ctx->xbig) cudaFree(ctx->xbig);
    for (int f = 0; f < KMM_MAXF; ++f)
        if (ctx->f[f]) cudaFree(ctx->f[f]);
    for (int w = 0; w < 6; ++w)
        if (ctx->wrk[w]) cudaFree(ctx->wrk[w]);
    void *ptrs[] = {ctx->d_wavx, ctx->d_wavz, ctx->d_c, ctx->d_ycoord, ctx->d_seght, ctx->d_fspread, ctx->d_cfl,
                    ctx->d_umax, ctx->d_status, ctx->d_tcstat, ctx->d_pumax, ctx->d_scratch, ctx->pl_in, ctx->pl_out, ctx->q_in, ctx->q_out,
                    ctx->d_tgtq, ctx->d_tgtc, ctx->d_tgtred, ctx->d_tgtlist, ctx->d_tgtcnt};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i)
        if (ptrs[i]) cudaFree(ptrs[i]);
    for (int s = 0; s < 5; ++s)
        if (ctx->tw_store[s]) cudaFree(ctx->tw_store[s]);
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->ens_ev) cudaEventDestroy(ctx->ens_ev);
    if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
    if (ctx->cfork_ev) cudaEventDestroy(ctx->cfork_ev);
    for (int e = 0; e < 2; ++e)
        if (ctx->cjoin_ev[e]) cudaEventDestroy(ctx->cjoin_ev[e]);
    if (ctx->side2) cudaStreamDestroy(ctx->side2);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    free(ctx->h_wavx); free(ctx->h_wavz); free(ctx->h_c); free(ctx->h_ycoord); free(ctx->h_seght);
    if (ctx->h_tgtlist) cudaFreeHost(ctx->h_tgtlist);
    free(ctx->h_targ);
    free(ctx);
    return KMM_OK;
}

// y-physical plane buffers for vcw3dp (sized on first use / growth)
int kmm_ensure_plane_buffers(kmm_ctx *ctx, int nin, int nout) {
    if ((size_t)nin > ctx->pl_in_fields) {
        if (ctx->pl_in) cudaFree(ctx->pl_in);
        if (ctx->q_in) cudaFree(ctx->q_in);
        ctx->pl_in = NULL; ctx->q_in = NULL;
        CK(cudaMalloc(&ctx->pl_in, sizeof(double2) * ctx->nspec * (size_t)nin));
        CK(cudaMalloc(&ctx->q_in, sizeof(double2) * (size_t)ctx->nyp * ctx->mz * ctx->nxh * (size_t)nin));
        ctx->pl_in_fields = (size_t)nin;
    }
    if ((size_t)nout > ctx->pl_out_fields) {
        if (ctx->pl_out) cudaFree(ctx->pl_out);
        if (ctx->q_out) cudaFree(ctx->q_out);
        ctx->pl_out = NULL; ctx->q_out = NULL;
        CK(cudaMalloc(&ctx->pl_out, sizeof(double2) * ctx->nspec * (size_t)nout));
        CK(cudaMalloc(&ctx->q_out, sizeof(double2) * (size_t)ctx->nyp * ctx->mz * ctx->nxh * (size_t)nout));
        ctx->pl_out_fields = (size_t)nout;
    }
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// instrumentation
// ---------------------------------------------------------------------------
void kmm_tic(kmm_ctx *ctx) {
    if (!ctx->timing_on || ctx->tm_n >= KMM_TIMER_RECORDS) return;
    cudaEventRecord(ctx->tm_ev[2 * ctx->tm_n], ctx->stream);
}

void kmm_toc(kmm_ctx *ctx, int stage) {
    if (!ctx->timing_on || ctx->tm_n >= KMM_TIMER_RECORDS) return;
    cudaEventRecord(ctx->tm_ev[2 * ctx->tm_n + 1], ctx->stream);
    ctx->tm_stage[ctx->tm_n++] = stage;
}

extern "C" int kmm_set_timing(kmm_ctx *ctx, int on) {
    if (!ctx) return KMM_ERR_ARG;
    if (on && !ctx->tm_ev_ready) {
        for (int e = 0; e < 2 * KMM_TIMER_RECORDS; ++e) CK(cudaEventCreate(&ctx->tm_ev[e]));
        ctx->tm_ev_ready = 1;
    }
    ctx->timing_on = on;
    ctx->tm_n = 0;
    return KMM_OK;   // steps run kernel by kernel while timing is on (kmm_fused_enqueue)
}

extern "C" int kmm_get_stage_times(kmm_ctx *ctx, double *ms, int *count, int nstages) {
    if (!ctx || !ms || !count || nstages <= 0) return KMM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    for (int s = 0; s < nstages; ++s) { ms[s] = 0.0; count[s] = 0; }
    for (int r = 0; r < ctx->tm_n; ++r) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, ctx->tm_ev[2 * r], ctx->tm_ev[2 * r + 1]));
        const int s = ctx->tm_stage[r];
        if (s >= 0 && s < nstages) { ms[s] += t; count[s] += 1; }
    }
    ctx->tm_n = 0;
    return KMM_OK;
}

extern "C" long long kmm_launch_count(const kmm_ctx *ctx) { return ctx ? ctx->launches : -1; }

extern "C" int kmm_event_record(kmm_ctx *ctx, int slot) {
    if (!ctx || slot < 0 || slot >= 16) return KMM_ERR_ARG;
    if (!ctx->user_ev[slot]) CK(cudaEventCreate(&ctx->user_ev[slot]));
    CK(cudaEventRecord(ctx->user_ev[slot], ctx->stream));
    return KMM_OK;
}

extern "C" int kmm_event_elapsed(kmm_ctx *ctx, int a, int b, double *ms) {
    if (!ctx || !ms || a < 0 || a >= 16 || b < 0 || b >= 16 || !ctx->user_ev[a] || !ctx->user_ev[b]) return KMM_ERR_ARG;
    CK(cudaEventSynchronize(ctx->user_ev[b]));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ctx->user_ev[a], ctx->user_ev[b]));
    *ms = (double)t;
    return KMM_OK;
}

// raise a kernel's dynamic shared-memory limit to `bytes` (static + dynamic above 48 KB needs the
// opt-in; max 227 KB)
int kmm_smem_attr(kmm_ctx *ctx, const void *func, size_t bytes) {
    if (bytes <= 16 * 1024) return KMM_OK;   // the kernels here keep < 32 KB static shared memory
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, func));
    const size_t total = bytes + fa.sharedSizeBytes;
    if (total <= 48 * 1024) return KMM_OK;
    if (total > 227 * 1024) {
        kmm_set_error(ctx, "kernel needs %zu bytes of shared memory (> 227 KB)", total);
        return KMM_ERR_UNSUPPORTED;
    }
    // while a step is being captured into a graph the attribute is already set by the uncaptured
    // step that precedes every capture
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return KMM_OK;
    CK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return KMM_OK;
}

extern "C" int kmm_set_option(kmm_ctx *ctx, int option, int value) {
    if (!ctx) return KMM_ERR_ARG;
    switch (option) {
    case KMM_OPT_FUSED: ctx->use_fused = value ? 1 : 0; kmm_graph_release(ctx); return KMM_OK;
    case KMM_OPT_COLUMN_BLOCKED: ctx->use_colblk = value ? 1 : 0; kmm_graph_release(ctx); return KMM_OK;
    case KMM_OPT_GRAPH: ctx->use_graph = value ? 1 : 0; kmm_graph_release(ctx); return KMM_OK;
    case KMM_OPT_ZTMA: ctx->use_ztma = value ? 1 : 0; kmm_graph_release(ctx); return KMM_OK;
    case KMM_OPT_XBIG: ctx->force_xbig = value ? 1 : 0; return KMM_OK;
    case KMM_OPT_TC_DCT: ctx->use_tcdct = value ? 1 : 0; return KMM_OK;
    case KMM_OPT_DERIVED_INPUTS: ctx->use_derived = value ? 1 : 0; return KMM_OK;
    case KMM_OPT_ENSEMBLE_GRAPH: ctx->use_ens_graph = value ? 1 : 0; return KMM_OK;
    case KMM_OPT_WAIT_LIMIT_MS: {
        if (value < 100 || value > 60000) {
            kmm_set_error(ctx, "wait limit %d ms outside 100 .. 60000", value);
            return KMM_ERR_ARG;
        }
        const unsigned long long ns = (unsigned long long)value * 1000000ull;
        CK(cudaSetDevice(ctx->device));
        CK(cudaStreamSynchronize(ctx->stream));
        if (kmm_plane_set_wait_limit(ns) || kmm_ztma_set_wait_limit(ns)) {
            kmm_set_error(ctx, "setting the wait limit failed");
            return KMM_ERR_CUDA;
        }
        return KMM_OK;
    }
    default: return KMM_ERR_ARG;
    }
}
