// kmm_step.cu -- host-side orchestration of the main program's blocks (main_dns.f90):
// Green's functions (gfcn, solvers.f90:5-172), initial (main_dns.f90:1602-2231) and the body
// of the time loop (main_dns.f90:198-811).  Every device call goes through the routine entry
// points of the other translation units, in the reference's order.
#include <atomic>
#include <mutex>

#include <math.h>

#include "kmm_internal.cuh"

// ---------------------------------------------------------------------------
// gfcn: two Green's functions + wall derivatives + common denominator
// ---------------------------------------------------------------------------
__global__ void k_gfcn_bc(double2 *bct, double2 *bcb, int nz, int nxh, double pt, double pb) {
    const int n = nz * nxh;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int j = e % nz, k = e / nz;
        double2 t = make_double2(pt, pt), b = make_double2(pb, pb);
        if (k == 0 && j >= nz / 2) { t.y = -t.y; b.y = -b.y; }   // conjg for j = nz/2+1..nz, kx = 0
        if (e == 0) { t = make_double2(pt, 0.0); b = make_double2(pb, 0.0); }
        bct[e] = t;
        bcb[e] = b;
    }
}

// (0,0) mode real + Hermitian symmetrisation of the kx = 0 plane (solvers.f90:118-139)
__global__ void k_gfcn_sym(double2 *g, int nyp, int nz) {
    const int n = nyp * (nz / 2);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int i = e % nyp, j = e / nyp;
        if (j == 0) {
            g[i].y = 0.0;
        } else {
            const int jp = nz - j;
            double2 x = g[(size_t)j * nyp + i], y = g[(size_t)jp * nyp + i];
            double2 m = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
            g[(size_t)j * nyp + i] = m;
            g[(size_t)jp * nyp + i] = make_double2(m.x, -m.y);
        }
    }
}

__global__ void k_gather_row(const double2 *w, double2 *dnvb, double2 *dnvt, int ncols, int nyp) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += gridDim.x * blockDim.x) {
        dnvb[c] = w[(size_t)c * nyp + 0];
        dnvt[c] = w[(size_t)c * nyp + 1];
    }
}

__global__ void k_denom(double2 *den, const double2 *d1t, const double2 *d2b, const double2 *d2t, const double2 *d1b,
                        int n) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        den[e] = csub(cmul(d1t[e], d2b[e]), cmul(d2t[e], d1b[e]));
}

static int gfcn1(kmm_ctx *ctx, int gf, int dnvbf, int dnvtf, double pb, double pt) {
    double2 *g = SPEC(ctx, gf), *bct = SPEC(ctx, KMM_BCTOP), *bcb = SPEC(ctx, KMM_BCBOT);
    double2 *dnvb = SPEC(ctx, dnvbf), *dnvt = SPEC(ctx, dnvtf);
    if (!g || !bct || !bcb || !dnvb || !dnvt) return KMM_ERR_NOMEM;
    const int nw = ctx->nz * ctx->nxh;
    k_gfcn_bc<<<kmm_blocks(nw, 256), 256, 0, ctx->stream>>>(bct, bcb, ctx->nz, ctx->nxh, pt, pb);
    CKL();
    CK(cudaMemsetAsync(g, 0, sizeof(double2) * ctx->nspec, ctx->stream));
    RET(kmm_internal_solve(ctx, g, ctx->re / (ctx->theta * ctx->dt), 0, bct, bcb));
    CK(cudaMemsetAsync(bct, 0, sizeof(double2) * nw, ctx->stream));
    CK(cudaMemsetAsync(bcb, 0, sizeof(double2) * nw, ctx->stream));
    RET(kmm_internal_solve(ctx, g, 0.0, 0, bct, bcb));
    k_gfcn_sym<<<kmm_blocks((size_t)ctx->nyp * ctx->nz / 2, 256), 256, 0, ctx->stream>>>(g, ctx->nyp, ctx->nz);
    CKL();
    double2 *wrkc = ctx->wrk[2], *wrk1 = ctx->wrk[3];
    if (ctx->nb == 1) { RET(kmm_internal_wallderiv(ctx, g, 1, 0, wrkc, 1)); }
    else { RET(kmm_internal_cderiv(ctx, g, wrk1)); RET(kmm_internal_wallderiv(ctx, wrk1, 1, 0, wrkc, 1)); }
    if (ctx->nt == 1) { RET(kmm_internal_wallderiv(ctx, g, 1, 1, wrkc, 2)); }
    else { RET(kmm_internal_cderiv(ctx, g, wrk1)); RET(kmm_internal_wallderiv(ctx, wrk1, 1, 1, wrkc, 2)); }
    k_gather_row<<<kmm_blocks(nw, 256), 256, 0, ctx->stream>>>(wrkc, dnvb, dnvt, nw, ctx->nyp);
    CKL();
    return KMM_OK;
}

extern "C" int kmm_gfcn(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    RET(gfcn1(ctx, KMM_GF1, KMM_DNV1B, KMM_DNV1T, ctx->p1b, ctx->p1t));
    RET(gfcn1(ctx, KMM_GF2, KMM_DNV2B, KMM_DNV2T, ctx->p2b, ctx->p2t));
    const int nw = ctx->nz * ctx->nxh;
    k_denom<<<kmm_blocks(nw, 256), 256, 0, ctx->stream>>>(SPEC(ctx, KMM_DENOM), SPEC(ctx, KMM_DNV1T),
                                                          SPEC(ctx, KMM_DNV2B), SPEC(ctx, KMM_DNV2T),
                                                          SPEC(ctx, KMM_DNV1B), nw);
    CKL();
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// small spectral helpers used by initial / step
// ---------------------------------------------------------------------------
// omy = i kz u - i kx w; (0,0) mode zero (main_dns.f90:1954-1968)
__global__ void k_init_omy(const double2 *u, const double2 *w, double2 *omy, const double *wavx, const double *wavz,
                           size_t n, int nyp, int nz) {
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const size_t jk = idx / nyp;
        const int j = (int)(jk % nz), k = (int)(jk / nz);
        double2 a = cimul(u[idx], wavz[j]), b = cimul(w[idx], wavx[k]);
        omy[idx] = (j == 0 && k == 0) ? make_double2(0.0, 0.0) : csub(a, b);
    }
}

// u0 = Re u(:,1,1), w0 = Re w(:,1,1); u(:,1,1) = u0, v(:,1,1) = 0, w(:,1,1) = w0 (main_dns.f90:1994-2005)
__global__ void k_init_mean(double2 *u, double2 *v, double2 *w, double *u0, double *w0, int nyp) {
    for (int i = threadIdx.x; i < nyp; i += blockDim.x) {
        u0[i] = u[i].x;
        w0[i] = w[i].x;
        u[i] = make_double2(u0[i], 0.0);
        v[i] = make_double2(0.0, 0.0);
        w[i] = make_double2(w0[i], 0.0);
    }
}

// h1n = Re gn(:,1,1), h3n = Re omz(:,1,1) (main_dns.f90:748-751)
__global__ void k_hmean(const double2 *gn, const double2 *omz, double *h1n, double *h3n, int nyp) {
    for (int i = threadIdx.x; i < nyp; i += blockDim.x) {
        h1n[i] = gn[i].x;
        h3n[i] = omz[i].x;
    }
}

// omy(:,1,1) = 0 (main_dns.f90:494-502)
__global__ void k_zero_mean(double2 *a, int nyp) {
    for (int i = threadIdx.x; i < nyp; i += blockDim.x) a[i] = make_double2(0.0, 0.0);
}

__global__ void k_add(double2 *y, const double2 *x, size_t n) {
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x)
        y[idx] = cadd(y[idx], x[idx]);
}

// norm of a list of distinct fields in one launch per KMM_NORM_BATCH of them
static int norm_ids(kmm_ctx *ctx, const int *ids, int n) {
    double2 *a[KMM_NORM_BATCH];
    for (int m0 = 0; m0 < n; m0 += KMM_NORM_BATCH) {
        const int nb = n - m0 < KMM_NORM_BATCH ? n - m0 : KMM_NORM_BATCH;
        for (int m = 0; m < nb; ++m) {
            a[m] = SPEC(ctx, ids[m0 + m]);
            if (!a[m]) return KMM_ERR_NOMEM;
        }
        RET(kmm_internal_norm_many(ctx, a, nb));
    }
    return KMM_OK;
}

static int norm_range(kmm_ctx *ctx, int first, int n) {
    int ids[KMM_NORM_BATCH];
    for (int m0 = 0; m0 < n; m0 += KMM_NORM_BATCH) {
        const int nb = n - m0 < KMM_NORM_BATCH ? n - m0 : KMM_NORM_BATCH;
        for (int m = 0; m < nb; ++m) ids[m] = first + m0 + m;
        RET(norm_ids(ctx, ids, nb));
    }
    return KMM_OK;
}

static const int kPolyComp[6] = {KMM_C11, KMM_C12, KMM_C13, KMM_C22, KMM_C23, KMM_C33};
static const int kQp[6] = {KMM_QP11, KMM_QP12, KMM_QP13, KMM_QP22, KMM_QP23, KMM_QP33};

static int poly_norm_c(kmm_ctx *ctx) { return norm_range(ctx, KMM_C11, 9); }

static int poly_norm_dc(kmm_ctx *ctx) { return norm_range(ctx, KMM_DC111, 27); }

static int poly_norm_out(kmm_ctx *ctx) {
    RET(poly_norm_c(ctx));
    RET(norm_range(ctx, KMM_C11N, 6));
    RET(norm_range(ctx, KMM_STR11N, 6));
    return norm_ids(ctx, kQp, 6);
}

// constant conformation tensor: xyzfft of a constant keeps only Chebyshev mode 0 of the (0,0) mode
static int poly_set_constant(kmm_ctx *ctx) {
    const double cz[9] = {ctx->p.c11z, 0, 0, 0, ctx->p.c22z, 0, 0, 0, ctx->p.c33z};
    for (int m = 0; m < 9; ++m) RET(kmm_internal_set_constant_mode(ctx, SPEC(ctx, KMM_C11 + m), cz[m]));
    return KMM_OK;
}

static double2 *poly_scratch(kmm_ctx *ctx, int m) {
    const int id = KMM_NSPECTRAL + m;   // private ids past the public spectral range
    if (!ctx->f[id]) {
        if (cudaMalloc(&ctx->f[id], sizeof(double2) * ctx->nspec) != cudaSuccess) return NULL;
        cudaMemsetAsync(ctx->f[id], 0, sizeof(double2) * ctx->nspec, ctx->stream);
    }
    return (double2 *)ctx->f[id];
}

// ---------------------------------------------------------------------------
// initial with irstrt >= 1 (main_dns.f90:1742-1917).  The host has uploaded the two records of
// setup/restart (v, fn, fnm1, omy, gn, gnm1, u0, h1n, h1nm1, w0, h3n, h3nm1; fxintg, fyintg,
// fzintg) and, with scalar + polymer and crstrt = 1, the five records of setup/c-restart; none of
// them is normalised or recomputed.  Only the scalar / polymer start values are set:
//   scalar only      : scalar and csource from setscl, not normalised (main_dns.f90:1810-1815)
//   scalar + polymer : crstrt = 0: setpoly, scalar gradient and conformation-tensor derivatives
//                      (normalised), scn, cIJn, strIJn, qpIJ zeroed (main_dns.f90:1817-1908);
//                      crstrt = 1: everything from c-restart (main_dns.f90:1909-1916)
// csource is zero at the start of the reference program and the crstrt = 1 branch leaves it so.
// ---------------------------------------------------------------------------
static int initial_restart(kmm_ctx *ctx) {
    if (!ctx->p.scalar_on) return KMM_OK;
    RET(kmm_zero(ctx, KMM_CSOURCE));
    if (ctx->p.polymer_on && ctx->p.crstrt != 0) return KMM_OK;
    RET(kmm_xyzfft(ctx, KMM_SCALAR, KMM_INITSCL));
    if (!ctx->p.polymer_on) return KMM_OK;
    RET(poly_set_constant(ctx));
    RET(kmm_gradscl(ctx));
    { static const int l[3] = {KMM_SCLX, KMM_SCLY, KMM_SCLZ}; RET(norm_ids(ctx, l, 3)); }
    RET(kmm_derivscji(ctx));
    RET(poly_norm_c(ctx));
    RET(poly_norm_dc(ctx));
    RET(kmm_zero(ctx, KMM_SCN));
    for (int m = 0; m < 6; ++m) {
        RET(kmm_zero(ctx, KMM_C11N + m));
        RET(kmm_zero(ctx, KMM_STR11N + m));
        RET(kmm_zero(ctx, kQp[m]));
    }
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// initial, after the setup's gfcn (main_dns.f90:151-161, 1602-2231)
// ---------------------------------------------------------------------------
extern "C" int kmm_initial(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    kmm_graph_release(ctx);
    const size_t n = ctx->nspec;
    RET(kmm_gfcn(ctx));
    RET(kmm_flowrate_setup(ctx));
    ctx->it = 0;
    if (ctx->p.irstrt >= 1) {
        RET(initial_restart(ctx));
        CK(cudaStreamSynchronize(ctx->stream));
        return KMM_OK;
    }
    RET(kmm_xyzfft(ctx, KMM_U, KMM_INITU));
    RET(kmm_xyzfft(ctx, KMM_V, KMM_INITV));
    RET(kmm_xyzfft(ctx, KMM_W, KMM_INITW));
    if (ctx->p.scalar_on) {
        RET(kmm_xyzfft(ctx, KMM_SCALAR, KMM_INITSCL));
        RET(kmm_zero(ctx, KMM_CSOURCE));
    }
    if (ctx->p.polymer_on) RET(poly_set_constant(ctx));
    k_init_omy<<<kmm_blocks(n, 256), 256, 0, ctx->stream>>>(SPEC(ctx, KMM_U), SPEC(ctx, KMM_W), SPEC(ctx, KMM_OMY),
                                                            ctx->d_wavx, ctx->d_wavz, n, ctx->nyp, ctx->nz);
    CKL();
    static const int l1[4] = {KMM_U, KMM_V, KMM_W, KMM_OMY};
    RET(norm_ids(ctx, l1, 4));
    if (ctx->p.scalar_on) { static const int l[2] = {KMM_SCALAR, KMM_CSOURCE}; RET(norm_ids(ctx, l, 2)); }
    if (ctx->p.polymer_on) RET(poly_norm_c(ctx));
    k_init_mean<<<1, 256, 0, ctx->stream>>>(SPEC(ctx, KMM_U), SPEC(ctx, KMM_V), SPEC(ctx, KMM_W), REAL(ctx, KMM_U0),
                                           REAL(ctx, KMM_W0), ctx->nyp);
    CKL();
    RET(norm_ids(ctx, l1, 4));
    RET(kmm_vort(ctx));
    { static const int l[2] = {KMM_OMX, KMM_OMZ}; RET(norm_ids(ctx, l, 2)); }
    if (ctx->p.scalar_on) {
        RET(kmm_gradscl(ctx));
        static const int l[3] = {KMM_SCLX, KMM_SCLY, KMM_SCLZ};
        RET(norm_ids(ctx, l, 3));
    }
    RET(kmm_gradv(ctx));
    { static const int l[12] = {KMM_U11, KMM_U12, KMM_U13, KMM_U21, KMM_U22, KMM_U23, KMM_U31, KMM_U32, KMM_U33,
                                KMM_LU, KMM_LV, KMM_LW};
      RET(norm_ids(ctx, l, 12)); }
    if (ctx->p.polymer_on) {
        RET(kmm_derivscji(ctx));
        RET(poly_norm_c(ctx));
        RET(poly_norm_dc(ctx));
    }
    int st = kmm_vcw3dp(ctx);
    if (st != KMM_OK && st != KMM_ERR_CFL && st != KMM_ERR_INTERP && st != KMM_ERR_NAN && st != KMM_ERR_PCFL) return st;
    { static const int l[5] = {KMM_V, KMM_OMY, KMM_FN, KMM_GN, KMM_OMZ}; RET(norm_ids(ctx, l, 5)); }
    if (ctx->p.polymer_on) {
        RET(poly_norm_out(ctx));
        if (ctx->it >= ctx->p.src_start) {
            RET(kmm_polyforce(ctx));
            static const int l[3] = {KMM_T1, KMM_T2, KMM_T3};
            RET(norm_ids(ctx, l, 3));
            RET(kmm_subforce(ctx));
        }
    }
    if (ctx->p.scalar_on && ctx->p.src_start == 0) {
        k_add<<<kmm_blocks(n, 256), 256, 0, ctx->stream>>>(SPEC(ctx, KMM_SCN), SPEC(ctx, KMM_CSOURCE), n);
        CKL();
    }
    k_hmean<<<1, 256, 0, ctx->stream>>>(SPEC(ctx, KMM_GN), SPEC(ctx, KMM_OMZ), REAL(ctx, KMM_H1N), REAL(ctx, KMM_H3N),
                                       ctx->nyp);
    CKL();
    RET(kmm_nonlin(ctx));
    { static const int l[2] = {KMM_FN, KMM_GN}; RET(norm_ids(ctx, l, 2)); }
    if (ctx->p.scalar_on) RET(kmm_norm(ctx, KMM_SCN));
    RET(kmm_copy(ctx, KMM_FNM1, KMM_FN));
    RET(kmm_copy(ctx, KMM_GNM1, KMM_GN));
    if (ctx->p.scalar_on) RET(kmm_copy(ctx, KMM_SCNM1, KMM_SCN));
    if (ctx->p.polymer_on)
        for (int m = 0; m < 6; ++m) {
            RET(kmm_copy(ctx, KMM_C11NM1 + m, KMM_C11N + m));
            RET(kmm_copy(ctx, KMM_STR11NM1 + m, KMM_STR11N + m));
        }
    RET(kmm_copy(ctx, KMM_H1NM1, KMM_H1N));
    RET(kmm_copy(ctx, KMM_H3NM1, KMM_H3N));
    CK(cudaStreamSynchronize(ctx->stream));
    return st;
}

// vcw3dp inside the routine step forms the x and z derivatives among its inputs in its z inverse
// (KMM_OPT_DERIVED_INPUTS, default 1), except where inertial particles need the materialised
// velocity gradient and Laplacian on the 3/2 grid, or the targeted scalar sources the spectral
// velocity gradient U11..U33
bool kmm_derived_inputs(const kmm_ctx *ctx) {
    return ctx->use_derived && !(ctx->p.particle_flag > 0 && ctx->p.npart > 0) &&
           !(ctx->p.scalar_on && (ctx->p.scl_flag == 4 || ctx->p.scl_flag == 5));
}

// the routine step's history copies (c11nm1 = c11n ..., scnm1 = scn, fnm1 = fn, gnm1 = gn;
// main_dns.f90:268-275, 335, 386, 418)
// as an exchange of the two fields' buffers: the n field is next written whole by vcw3dp, and
// nothing reads it in between, so after the exchange both fields hold what the copy would leave
static int swap_fields(kmm_ctx *ctx, int nm1, int n) {
    if (!kmm_field_ptr(ctx, nm1) || !kmm_field_ptr(ctx, n)) return KMM_ERR_NOMEM;
    void *t = ctx->f[nm1];
    ctx->f[nm1] = ctx->f[n];
    ctx->f[n] = t;
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// one iteration of the time loop, main_dns.f90:198-811
// ---------------------------------------------------------------------------
extern "C" int kmm_step(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    if (ctx->use_fused && kmm_fused_applicable(ctx)) return kmm_fused_step(ctx);
    if (ctx->p.precision == 1) {
        // the routine path's mixed form runs its transforms at the compiled lengths only; never fall
        // back silently to FP64
        const int ly = 2 * ctx->ny, mz = ctx->mz, mx = ctx->mx;
        const bool ok_y = ly == 64 || ly == 128 || ly == 192 || ly == 256 || ly == 512;
        const bool ok_z = mz == 48 || mz == 96 || mz == 144 || mz == 192 || mz == 576;
        const bool ok_x = mx == 48 || mx == 96 || mx == 144 || mx == 192 || mx == 576;
        if (!(ok_y && ok_z && ok_x)) {
            kmm_set_error(ctx, "mixed precision needs nx, nz in {32, 64, 96, 128, 384} and ny in {32, 64, 96, 128, 256}");
            return KMM_ERR_UNSUPPORTED;
        }
    }
    const double re = ctx->re, dt = ctx->dt, th = ctx->theta;
    ctx->it += 1;
    const int it = ctx->it;
    kmm_tic(ctx);
    if (ctx->p.polymer_on) {
        if (it == ctx->p.src_start - 1 || (it == ctx->p.irstrt && ctx->p.crstrt == 0)) RET(poly_set_constant(ctx));
        if (it >= ctx->p.src_start) {
            double2 *nl[6];
            for (int m = 0; m < 6; ++m) {
                nl[m] = poly_scratch(ctx, m);
                if (!nl[m]) return KMM_ERR_NOMEM;
            }
            RET(kmm_internal_polynl(ctx, nl));
            // the six components' phirhs and penta: its n-1 term 2 nl is formed in the kernel (NULL)
            double2 *cm[6];
            const double2 *nlc[6], *nl2c[6];
            for (int m = 0; m < 6; ++m) {
                cm[m] = SPEC(ctx, kPolyComp[m]);
                if (!cm[m]) return KMM_ERR_NOMEM;
                nlc[m] = nl[m];
                nl2c[m] = NULL;
            }
            const double g = (re * ctx->p.diffpoly) / (dt * th);
            const KmmSolveSpec sp = {g, 1, 0.0, 1.0, 0.0, 1.0};
            RET(kmm_zero(ctx, KMM_BCTOP));
            RET(kmm_zero(ctx, KMM_BCBOT));
            int pst = kmm_colblk_phirhs_solve(ctx, cm, nlc, nl2c, 6, ctx->p.diffpoly, 0, 1, &sp);
            if (pst == KMM_ERR_UNSUPPORTED) {
                // batched launches, each component with its own wrkc and wrk1 (scratch ids 12 .. 23)
                double2 *wc[6], *w1[6];
                for (int m = 0; m < 6; ++m) {
                    wc[m] = poly_scratch(ctx, 12 + m);
                    w1[m] = poly_scratch(ctx, 18 + m);
                    if (!wc[m] || !w1[m]) return KMM_ERR_NOMEM;
                }
                RET(kmm_internal_phirhs_many(ctx, cm, nlc, nl2c, 6, ctx->p.diffpoly, wc, w1));
                pst = kmm_internal_penta_many(ctx, cm, 6, g, 0.0, 1.0, 0.0, 1.0, SPEC(ctx, KMM_BCTOP),
                                              SPEC(ctx, KMM_BCBOT));
            }
            RET(pst);
            for (int m = 0; m < 6; ++m) {
                RET(swap_fields(ctx, KMM_C11NM1 + m, KMM_C11N + m));
                RET(swap_fields(ctx, KMM_STR11NM1 + m, KMM_STR11N + m));
            }
            RET(norm_ids(ctx, kPolyComp, 6));
            RET(kmm_copy(ctx, KMM_C21, KMM_C12));
            RET(kmm_copy(ctx, KMM_C31, KMM_C13));
            RET(kmm_copy(ctx, KMM_C32, KMM_C23));
        }
    }
    // phirhs and its solves in one blocked kernel per field where compiled (every boundary value
    // is zero: phirhs zeroes bctop / bcbot, main_dns.f90:39, solvers.f90:670-671), else routine by
    // routine
    auto phi_solve = [&](int x, int fn, int fnm1, double var, int phi, int nsolve, const KmmSolveSpec *sp) -> int {
        double2 *xp = SPEC(ctx, x);
        const double2 *fp = SPEC(ctx, fn), *fmp = SPEC(ctx, fnm1);
        if (!xp || !fp || !fmp) return KMM_ERR_NOMEM;
        return kmm_colblk_phirhs_solve(ctx, &xp, &fp, &fmp, 1, var, phi, nsolve, sp);
    };
    if (ctx->p.scalar_on) {
        const double g = (re * ctx->p.diff) / (dt * th);
        const KmmSolveSpec sp = ctx->p.scalar_bc == 1 ? KmmSolveSpec{g, 1, 1.0, 0.0, 1.0, 0.0}
                                                      : KmmSolveSpec{g, 1, 0.0, 1.0, 0.0, 1.0};
        RET(kmm_zero(ctx, KMM_BCTOP));   // bcscltop = bcsclbot = 0 (main_dns.f90:39)
        RET(kmm_zero(ctx, KMM_BCBOT));
        int st = phi_solve(KMM_SCALAR, KMM_SCN, KMM_SCNM1, ctx->p.diff, 0, 1, &sp);
        if (st == KMM_ERR_UNSUPPORTED) {
            RET(kmm_phirhs(ctx, KMM_SCALAR, KMM_SCN, KMM_SCNM1, ctx->p.diff));
            st = kmm_penta(ctx, KMM_SCALAR, g, 0, sp.at, sp.bt, sp.ab, sp.bb);
        }
        RET(st);
        RET(swap_fields(ctx, KMM_SCNM1, KMM_SCN));
    }
    {
        const KmmSolveSpec sv[2] = {{re / (dt * th), 0, 0.0, 0.0, 0.0, 0.0}, {0.0, 0, 0.0, 0.0, 0.0, 0.0}};
        int st = phi_solve(KMM_V, KMM_FN, KMM_FNM1, 1.0, 1, 2, sv);
        if (st == KMM_ERR_UNSUPPORTED) {
            RET(kmm_phi_from_v(ctx));
            RET(kmm_phirhs(ctx, KMM_V, KMM_FN, KMM_FNM1, 1.0));
            RET(kmm_solve(ctx, KMM_V, sv[0].g, 0));
            st = kmm_solve(ctx, KMM_V, sv[1].g, 0);
        }
        RET(st);
        RET(swap_fields(ctx, KMM_FNM1, KMM_FN));
    }
    {
        const KmmSolveSpec so = {re / (dt * th), 1, ctx->atu, ctx->btu, ctx->abu, ctx->bbu};
        int st = phi_solve(KMM_OMY, KMM_GN, KMM_GNM1, 1.0, 0, 1, &so);
        if (st == KMM_ERR_UNSUPPORTED) {
            RET(kmm_phirhs(ctx, KMM_OMY, KMM_GN, KMM_GNM1, 1.0));
            RET(kmm_influence(ctx));
            st = kmm_penta(ctx, KMM_OMY, so.g, 0, so.at, so.bt, so.ab, so.bb);
        } else if (st == KMM_OK) {
            st = kmm_influence(ctx);   // v only: omega_y's solve does not depend on it
        }
        RET(st);
        RET(swap_fields(ctx, KMM_GNM1, KMM_GN));
    }
    RET(kmm_zero(ctx, KMM_BCTOP));   // as phirhs leaves them
    RET(kmm_zero(ctx, KMM_BCBOT));
    // the u0 and w0 solves (each one block) side by side: w0's on the side stream
    CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
    RET(kmm_internal_uzero(ctx, 3, ctx->side));
    RET(kmm_internal_uzero(ctx, 1, ctx->stream));
    RET(kmm_flowrate_apply(ctx, ctx->stream));
    CK(cudaEventRecord(ctx->join_ev, ctx->side));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0));
    k_zero_mean<<<1, 256, 0, ctx->stream>>>(SPEC(ctx, KMM_OMY), ctx->nyp);
    CKL();
    RET(kmm_copy(ctx, KMM_H1NM1, KMM_H1N));
    RET(kmm_copy(ctx, KMM_H3NM1, KMM_H3N));
    { static const int l[2] = {KMM_V, KMM_OMY}; RET(norm_ids(ctx, l, 2)); }
    RET(kmm_veloc(ctx));
    { static const int l[2] = {KMM_U, KMM_W}; RET(norm_ids(ctx, l, 2)); }
    RET(kmm_vort(ctx));
    { static const int l[2] = {KMM_OMX, KMM_OMZ}; RET(norm_ids(ctx, l, 2)); }
    // with derived inputs vcw3dp forms the x and z derivatives itself (in its z inverse): only the
    // y derivatives are computed here, in one batched cderiv launch
    const bool derived = kmm_derived_inputs(ctx);
    const double2 *dsrc[KMM_CDERIV_BATCH];
    double2 *ddst[KMM_CDERIV_BATCH];
    int nd = 0;
    int dnorm[KMM_CDERIV_BATCH];
    auto want_dy = [&](int f, int df) -> int {
        dsrc[nd] = SPEC(ctx, f);
        ddst[nd] = SPEC(ctx, df);
        if (!dsrc[nd] || !ddst[nd]) return KMM_ERR_NOMEM;
        dnorm[nd++] = df;
        return KMM_OK;
    };
    if (ctx->p.scalar_on) {
        RET(kmm_norm(ctx, KMM_SCALAR));
        if (derived) {
            RET(want_dy(KMM_SCALAR, KMM_SCLY));
        } else {
            RET(kmm_gradscl(ctx));
            static const int l[3] = {KMM_SCLX, KMM_SCLY, KMM_SCLZ};
            RET(norm_ids(ctx, l, 3));
        }
    }
    const bool targeted = ctx->p.scalar_on && (ctx->p.scl_flag == 4 || ctx->p.scl_flag == 5);
    if (ctx->p.polymer_on || ctx->p.particle_flag > 0 || targeted) {
        // the velocity gradient / Laplacian feed only the polymer terms, inertial particles and the
        // targeted scalar sources (the reference computes them every step, main_dns.f90:544)
        if (derived) {
            RET(want_dy(KMM_U, KMM_U12));
            RET(want_dy(KMM_V, KMM_U22));
            RET(want_dy(KMM_W, KMM_U32));
        } else {
            RET(kmm_gradv(ctx));
            static const int l[12] = {KMM_U11, KMM_U12, KMM_U13, KMM_U21, KMM_U22, KMM_U23, KMM_U31, KMM_U32,
                                      KMM_U33, KMM_LU, KMM_LV, KMM_LW};
            RET(norm_ids(ctx, l, 12));
        }
    }
    if (ctx->p.polymer_on) {
        if (derived) {
            RET(poly_norm_c(ctx));
            static const int uq[6] = {0, 1, 2, 4, 5, 8};   // c11 c12 c13 c22 c23 c33
            for (int m = 0; m < 6; ++m) RET(want_dy(KMM_C11 + uq[m], KMM_DC111 + 3 * uq[m] + 1));
        } else {
            RET(kmm_derivscji(ctx));
            RET(poly_norm_c(ctx));
            RET(poly_norm_dc(ctx));
        }
    }
    if (nd) {
        RET(kmm_internal_cderiv_many(ctx, dsrc, ddst, nd));
        RET(norm_ids(ctx, dnorm, nd));
    }
    kmm_toc(ctx, KMM_STAGE_COLUMN);
    ctx->in_step = 1;
    int st = kmm_vcw3dp(ctx);
    ctx->in_step = 0;
    if (st != KMM_OK) return st;
    kmm_tic(ctx);
    { static const int l[5] = {KMM_V, KMM_OMY, KMM_FN, KMM_GN, KMM_OMZ}; RET(norm_ids(ctx, l, 5)); }
    if (ctx->p.scalar_on) { static const int l[2] = {KMM_SCALAR, KMM_SCN}; RET(norm_ids(ctx, l, 2)); }
    if (ctx->p.polymer_on) {
        if (it >= ctx->p.src_start - 1) RET(poly_norm_out(ctx));
        if (it >= ctx->p.src_start) {
            RET(kmm_polyforce(ctx));
            static const int l[3] = {KMM_T1, KMM_T2, KMM_T3};
            RET(norm_ids(ctx, l, 3));
            RET(kmm_subforce(ctx));
        }
    }
    RET(kmm_filter(ctx));
    k_hmean<<<1, 256, 0, ctx->stream>>>(SPEC(ctx, KMM_GN), SPEC(ctx, KMM_OMZ), REAL(ctx, KMM_H1N), REAL(ctx, KMM_H3N),
                                       ctx->nyp);
    CKL();
    { static const int l[3] = {KMM_FN, KMM_GN, KMM_OMZ}; RET(norm_ids(ctx, l, 3)); }
    RET(kmm_nonlin(ctx));
    { static const int l[2] = {KMM_FN, KMM_GN}; RET(norm_ids(ctx, l, 2)); }
    if (ctx->p.scalar_on) RET(kmm_norm(ctx, KMM_SCN));
    kmm_toc(ctx, KMM_STAGE_POST);
    return KMM_OK;
}

extern "C" int kmm_run(kmm_ctx *ctx, int n) {
    if (!ctx || n < 0) return KMM_ERR_ARG;
    for (int s = 0; s < n; ++s) RET(kmm_step(ctx));
    CK(cudaStreamSynchronize(ctx->stream));
    return KMM_OK;
}

extern "C" int kmm_polynl(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *nl[6];
    for (int m = 0; m < 6; ++m) {
        nl[m] = poly_scratch(ctx, m);
        if (!nl[m]) return KMM_ERR_NOMEM;
    }
    return kmm_internal_polynl(ctx, nl);
}

// ---------------------------------------------------------------------------
// ensemble of independent runs (the reference's multi-run driver launches them as separate
// processes, LO_multi_run/setup.py:93-101): every member's step is enqueued on its own stream
// before any member is waited on, so the members' kernels overlap on the GPU
// ---------------------------------------------------------------------------
static int ensemble_step_all(kmm_ctx **ctxs, int n, int *status);
static int ensemble_step_graph(kmm_ctx **ctxs, int n, int *status);

// the caller's current device is restored before returning
extern "C" int kmm_ensemble_step(kmm_ctx **ctxs, int n, int *status) {
    if (!ctxs || n <= 0 || n > KMM_MAX_ENSEMBLE || !status) return KMM_ERR_ARG;
    int dev0 = 0;
    if (cudaGetDevice(&dev0) != cudaSuccess) return KMM_ERR_CUDA;
    int st = ensemble_step_graph(ctxs, n, status);
    if (st == KMM_ERR_UNSUPPORTED) st = ensemble_step_all(ctxs, n, status);
    cudaSetDevice(dev0);
    return st;
}

// ---- the whole ensemble step as one CUDA graph -----------------------------------------
// A parent graph holds every member's captured step (the graph of its current history
// arrangement) as an independent child graph.  Parent graphs are cached per member set, the
// members' arrangements and their graphs' generations; the generations come from one
// process-wide counter, so a graph captured anew (or a context created at a freed one's
// address) never matches a cached entry, and destroying a context drops the entries holding it.
#define ENS_CACHE 4
struct EnsGraph {
    int n;
    kmm_ctx *m[KMM_MAX_ENSEMBLE];
    unsigned long long gen[KMM_MAX_ENSEMBLE];
    unsigned char par[KMM_MAX_ENSEMBLE];
    cudaGraphExec_t exec;
    int device;
};
static EnsGraph g_ens[ENS_CACHE];
static int g_ens_next = 0;
static std::mutex g_ens_mu;
static std::atomic<unsigned long long> g_graph_gen{0};

unsigned long long kmm_graph_generation() { return ++g_graph_gen; }

static void ens_drop(EnsGraph &e) {
    if (e.exec) {
        int d0 = 0;
        cudaGetDevice(&d0);
        cudaSetDevice(e.device);
        cudaGraphExecDestroy(e.exec);
        cudaSetDevice(d0);
    }
    e.exec = NULL;
    e.n = 0;
}

void kmm_ensemble_forget(kmm_ctx *ctx) {
    std::lock_guard<std::mutex> lk(g_ens_mu);
    for (int c = 0; c < ENS_CACHE; ++c)
        for (int i = 0; i < g_ens[c].n; ++i)
            if (g_ens[c].m[i] == ctx) {
                ens_drop(g_ens[c]);
                break;
            }
}

// KMM_ERR_UNSUPPORTED: the members cannot run as one graph this step (the caller falls back)
static int ensemble_step_graph(kmm_ctx **ctxs, int n, int *status) {
    if (n < 2) return KMM_ERR_UNSUPPORTED;
    const int dev = ctxs[0] ? ctxs[0]->device : -1;
    for (int m = 0; m < n; ++m) {
        kmm_ctx *c = ctxs[m];
        if (!c || c->device != dev || !c->use_ens_graph) return KMM_ERR_UNSUPPORTED;
        for (int q = 0; q < m; ++q)
            if (ctxs[q] == c) return KMM_ERR_UNSUPPORTED;
    }
    if (cudaSetDevice(dev) != cudaSuccess) return KMM_ERR_UNSUPPORTED;
    unsigned char par[KMM_MAX_ENSEMBLE];
    for (int m = 0; m < n; ++m) {
        int p = 0;
        const int st = kmm_fused_graph_for_step(ctxs[m], &p);
        if (st != KMM_OK) return st < 0 ? KMM_ERR_UNSUPPORTED : st;
        par[m] = (unsigned char)p;
    }
    std::lock_guard<std::mutex> lk(g_ens_mu);
    EnsGraph *hit = NULL;
    for (int c = 0; c < ENS_CACHE && !hit; ++c) {
        EnsGraph &e = g_ens[c];
        if (e.n != n || !e.exec || e.device != dev) continue;
        bool same = true;
        for (int m = 0; m < n && same; ++m)
            same = e.m[m] == ctxs[m] && e.gen[m] == ctxs[m]->ggen && e.par[m] == par[m];
        if (same) hit = &e;
    }
    if (!hit) {
        EnsGraph &e = g_ens[g_ens_next];
        g_ens_next = (g_ens_next + 1) % ENS_CACHE;
        ens_drop(e);
        cudaGraph_t parent = NULL;
        cudaError_t err = cudaGraphCreate(&parent, 0);
        for (int m = 0; m < n && err == cudaSuccess; ++m) {
            cudaGraphNode_t node;
            err = cudaGraphAddChildGraphNode(&node, parent, NULL, 0, ctxs[m]->ggraph[par[m]]);
        }
        if (err == cudaSuccess) err = cudaGraphInstantiate(&e.exec, parent, 0);
        if (parent) cudaGraphDestroy(parent);
        if (err != cudaSuccess) {
            cudaGetLastError();
            e.exec = NULL;
            return KMM_ERR_UNSUPPORTED;
        }
        e.n = n;
        e.device = dev;
        for (int m = 0; m < n; ++m) {
            e.m[m] = ctxs[m];
            e.gen[m] = ctxs[m]->ggen;
            e.par[m] = par[m];
        }
        hit = &e;
    }
    // order the graph after every member's earlier work and every member's later work after it
    // (CUDA errors are reported on member 0)
    kmm_ctx *ctx = ctxs[0];
    cudaStream_t s0 = ctx->stream;
    for (int m = 0; m < n; ++m) {
        kmm_ctx *c = ctxs[m];
        if (!c->ens_ev) CK(cudaEventCreateWithFlags(&c->ens_ev, cudaEventDisableTiming));
        if (m > 0) {
            CK(cudaEventRecord(c->ens_ev, c->stream));
            CK(cudaStreamWaitEvent(s0, c->ens_ev, 0));
        }
    }
    CK(cudaGraphLaunch(hit->exec, s0));
    CK(cudaEventRecord(ctxs[0]->ens_ev, s0));
    for (int m = 1; m < n; ++m) CK(cudaStreamWaitEvent(ctxs[m]->stream, ctxs[0]->ens_ev, 0));
    int first = KMM_OK;
    for (int m = 0; m < n; ++m) {
        kmm_fused_replayed(ctxs[m], par[m]);
        status[m] = kmm_fused_finish(ctxs[m]);
        if (first == KMM_OK && status[m] != KMM_OK) first = status[m];
    }
    return first;
}

static int ensemble_step_all(kmm_ctx **ctxs, int n, int *status) {
    bool launched[KMM_MAX_ENSEMBLE];
    for (int m = 0; m < n; ++m) {
        kmm_ctx *c = ctxs[m];
        launched[m] = false;
        if (!c) {
            status[m] = KMM_ERR_ARG;
            continue;
        }
        if (cudaSetDevice(c->device) != cudaSuccess) {
            status[m] = KMM_ERR_CUDA;
            continue;
        }
        if (c->use_fused && kmm_fused_applicable(c)) {
            status[m] = kmm_fused_enqueue(c);
            launched[m] = status[m] == KMM_OK;
        } else {
            status[m] = kmm_step(c);   // routine path: runs to completion on its own stream
        }
    }
    int first = KMM_OK;
    for (int m = 0; m < n; ++m) {
        if (launched[m]) {
            cudaSetDevice(ctxs[m]->device);
            status[m] = kmm_fused_finish(ctxs[m]);
        }
        if (first == KMM_OK && status[m] != KMM_OK) first = status[m];
    }
    return first;
}

extern "C" int kmm_ensemble_run(kmm_ctx **ctxs, int n, int nsteps, int *status) {
    if (nsteps < 0) return KMM_ERR_ARG;
    for (int s = 0; s < nsteps; ++s) {
        const int st = kmm_ensemble_step(ctxs, n, status);
        if (st != KMM_OK) return st;
    }
    return KMM_OK;
}
