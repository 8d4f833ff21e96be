// kmm_fused.cu -- the time-loop body (main_dns.f90:198-811) as five fused kernels, for the fluid
// and passive-scalar equations (no polymer, no immersed boundary):
//
//   k_col_fwd : per (kx,kz) column pair, one warp per column: scalar CN/AB2 + Robin tau solve,
//               phi = v'' - k^2 v, phirhs, Helmholtz + Poisson tau solves, omega_y phirhs,
//               influence-matrix correction, omega_y Robin solve, mean modes (uzero), norm,
//               veloc, y-derivatives, and the Chebyshev -> physical DCT-I of the eight fields the
//               nonlinear stage needs (u, v, w, omega_y, du/dy, dw/dy, c, dc/dy) written in column
//               layout (main_dns.f90:325-544, solvers.f90:555-1722).
//   k_zb      : (kx, y) tiles: derive omega_x, omega_z, dc/dx, dc/dz, zero-pad to mz and inverse
//               z transform (solvers.f90:2578-2803).
//   k_fx      : (kmm_fast.cu) x transforms + pointwise products, warp per (y,z) row.
//   k_zf      : forward z transform, truncation, /(mx mz) (solvers.f90:3180-3273).
//   k_col_bwd : per column pair: DCT-I back (/ny, halved ends), norm, spectral filter, mean
//               nonlinear profiles h1n/h3n, nonlin (solvers.f90:3279-3416, main_dns.f90:606-771).
//
// The state keeps the reference's layout; the n -> n-1 history copies are pointer swaps.  The
// tau pivots and border weights are built once per run by k_tau_tables with the reference's own
// recurrences (eqsolve, pntsolve).
#include <math.h>

#include "kmm_fft.cuh"
#include "kmm_fused.cuh"

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------

struct TabCfg {
    double g;
    int robin;
    double at, bt, ab, bb;
    double bsign;   // +1: penta's mixedbc (ab + dyde bb n^2); -1: psolve1d's mixedbc1d (ab - dyde bb n^2)
};

__device__ __forceinline__ void tab_row(int i, int par, double wn, double dyde, int nyh, int nyhm, double &a1, double &a2,
                                        double &a3) {
    const int j = par == 0 ? 2 * i : 2 * i + 1;
    const double rj1 = 1.0 / (double)(4 * j * (j - 1));
    const double rj2 = 1.0 / (double)(2 * (j * j - 1));
    const double rj3 = 1.0 / (double)(4 * j * (j + 1));
    a1 = wn * rj1;
    a2 = -1.0 * dyde * dyde - wn * rj2;
    a3 = wn * rj3;
    if (par == 0) {
        if (i == 1) a1 = 2.0 * a1;
        if (i == nyhm) a3 = 0.0;
        if (i == nyh) { a2 = -1.0 * dyde * dyde; a3 = 0.0; }
    } else {
        if (i == nyhm - 1) a3 = 0.0;
        if (i == nyhm) { a2 = -1.0 * dyde * dyde; a3 = 0.0; }
    }
}

// one thread per column: d(i) chain (eqsolve / pntsolve), forward multipliers, border weights and
// final f values for one configuration
__global__ void k_tau_tables(double *td, double *te, double *tb1, double *tb2, double *tf, TabCfg C,
                             const double *wavx, const double *wavz, int ncols, int nz, int nyp, double dyde) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncols) return;
    const int ny = nyp - 1, nyh = ny / 2, nyhm = nyh - 1, nyhp = nyh + 1;
    const int j = col % nz, k = col / nz;
    const double wn = wavz[j] * wavz[j] + wavx[k] * wavx[k] + C.g;
    double *D = td + (size_t)col * nyp, *Te = te + (size_t)col * nyp;
    double *B1 = tb1 + (size_t)col * nyp, *B2 = tb2 ? tb2 + (size_t)col * nyp : NULL;
    for (int P = 0; P < nyp; ++P) { D[P] = 1.0; Te[P] = 0.0; B1[P] = 0.0; if (B2) B2[P] = 0.0; }
    for (int par = 0; par < 2; ++par) {
        const int n = par == 0 ? nyhp : nyh, m = n - 1;
        // pivots
        double a1, a2, a3, b1, b2, b3;
        tab_row(m, par, wn, dyde, nyh, nyhm, a1, a2, a3);
        D[2 * m + par] = a2;
        for (int i = m - 1; i >= 1; --i) {
            tab_row(i, par, wn, dyde, nyh, nyhm, a1, a2, a3);
            tab_row(i + 1, par, wn, dyde, nyh, nyhm, b1, b2, b3);
            D[2 * i + par] = a2 - a3 * b1 / D[2 * (i + 1) + par];
            Te[2 * i + par] = a3 / D[2 * (i + 1) + par];
        }
        // border rows
        for (int pass = 0; pass < (C.robin ? 2 : 1); ++pass) {
            // Dirichlet: t = 1; Robin pass 0 = top row (tt), pass 1 = bottom row (tb) (mixedbc, fillt)
            double *B = pass == 0 ? B1 : B2;
#define TVAL(q) (!C.robin ? 1.0 : [&](int qq) -> double {                       \
                int jj = par == 0 ? 2 * qq - 1 : 2 * qq;                             \
                int j1 = jj - 1;                                                     \
                if (pass == 0) return C.at + dyde * C.bt * (double)(j1 * j1);        \
                double v = C.ab + C.bsign * dyde * C.bb * (double)(j1 * j1);         \
                return (jj % 2 == 0) ? -v : v;                                       \
            }(q))
            tab_row(m, par, wn, dyde, nyh, nyhm, a1, a2, a3);
            double f = TVAL(m) - TVAL(n) * a1 / D[2 * m + par];
            B[2 * m + par] = TVAL(n) / D[2 * m + par];
            for (int i = m - 1; i >= 1; --i) {
                tab_row(i, par, wn, dyde, nyh, nyhm, a1, a2, a3);
                B[2 * i + par] = f / D[2 * i + par];
                f = TVAL(i) - f * a1 / D[2 * i + par];
            }
#undef TVAL
            tf[(size_t)col * 4 + (C.robin ? 2 * pass + par : par)] = f;
        }
    }
}



// lane-blocked copy of per-column tables for the blocked column kernels (kmm_colblk.cuh, K = ny / 16):
// coefficient P = t K + m (m < K) of a column at m * 16 + t, P = 16 K in place; recip stores 1 / v
__global__ void k_tab_block(const double *__restrict__ src, double *__restrict__ dst, int ncols, int nyp, int K,
                            int recip) {
    const size_t n = (size_t)ncols * nyp;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const size_t col = e / nyp;
        const int P = (int)(e - col * nyp);
        const int d = P < 16 * K ? (P % K) * 16 + P / K : P;
        const double v = src[e];
        dst[col * nyp + d] = recip ? 1.0 / v : v;
    }
}

// the blocked copies of one configuration's td (as 1 / d), te, tb1, tb2 (tf is per column, unchanged)
static int block_tables(kmm_ctx *ctx, const double *const src[4], double *dst[4], int ncols) {
    const int K = ctx->ny / 16;
    const size_t n = (size_t)ncols * ctx->nyp;
    const int nb = (int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184);
    for (int a = 0; a < 4; ++a) {
        CK(cudaMalloc(&dst[a], sizeof(double) * n));
        k_tab_block<<<nb, 256, 0, ctx->stream>>>(src[a], dst[a], ncols, ctx->nyp, K, a == 0);
        CKL();
    }
    return KMM_OK;
}

// the three rj rows (1/(4j(j-1)), 1/(2(j^2-1)), 1/(4j(j+1))) on the host, in natural or lane-blocked order
static void rj_rows(double *h, int nyp, bool blocked) {
    const int ny = nyp - 1, K = ny / 16;
    for (int j = 0; j < 3 * nyp; ++j) h[j] = 0.0;
    for (int j = 2; j < nyp; ++j) {
        const int d = (blocked && j < 16 * K) ? (j % K) * 16 + j / K : j;
        h[d] = 1.0 / (double)(4 * j * (j - 1));
        h[nyp + d] = 1.0 / (double)(2 * (j * j - 1));
        h[2 * nyp + d] = 1.0 / (double)(4 * j * (j + 1));
    }
}

static int upload_rj(kmm_ctx *ctx, double **out, bool blocked) {
    const int nyp = ctx->nyp;
    double *h = (double *)calloc(3 * (size_t)nyp, sizeof(double));
    if (!h) return KMM_ERR_NOMEM;
    rj_rows(h, nyp, blocked);
    cudaError_t e = cudaMalloc(out, sizeof(double) * 3 * nyp);
    if (e == cudaSuccess) e = cudaMemcpy(*out, h, sizeof(double) * 3 * nyp, cudaMemcpyHostToDevice);
    free(h);
    CK(e);
    return KMM_OK;
}

// FP32 twiddles exp(-2 pi i m/n), rounded from long double, for the mixed-precision transforms
static int make_twf(kmm_ctx *ctx, int n, float2 **out) {
    float2 *h = (float2 *)malloc(sizeof(float2) * (size_t)n);
    for (int k = 0; k < n; ++k) {
        const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
        h[k] = make_float2((float)cosl(a), -(float)sinl(a));
    }
    cudaError_t e = cudaMalloc(out, sizeof(float2) * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(*out, h, sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice);
    free(h);
    CK(e);
    return KMM_OK;
}

static int build_tables(kmm_ctx *ctx) {
    if (ctx->fused) return KMM_OK;
    KmmFused *F = (KmmFused *)calloc(1, sizeof(KmmFused));
    ctx->fused = F;
    const int ncols = ctx->nz * ctx->nxh;
    const double g1 = ctx->re / (ctx->dt * ctx->theta);
    const double gs = ctx->re * ctx->p.diff / (ctx->dt * ctx->theta);
    TabCfg cfg[TB_N];
    cfg[TB_PHI] = {g1, 0, 0, 0, 0, 0, 1.0};
    cfg[TB_V] = {0.0, 0, 0, 0, 0, 0, 1.0};
    cfg[TB_OMY] = {g1, 1, ctx->atu, ctx->btu, ctx->abu, ctx->bbu, 1.0};
    if (ctx->p.scalar_bc == 1) cfg[TB_SCL] = {gs, 1, 1.0, 0.0, 1.0, 0.0, 1.0};
    else cfg[TB_SCL] = {gs, 1, 0.0, 1.0, 0.0, 1.0, 1.0};
    // mean modes (uzero -> psolve1d, solvers.f90:1065-1245): only the (0,0) column; w0 passes btu
    cfg[TB_U0] = {g1, 1, ctx->atu, ctx->btu, ctx->abu, ctx->bbu, -1.0};
    cfg[TB_W0] = {g1, 1, ctx->atw, ctx->btu, ctx->abw, ctx->bbw, -1.0};
    FusedTabs &T = F->tabs;
    for (int c = 0; c < TB_N; ++c) {
        const int nc = (c == TB_U0 || c == TB_W0) ? 1 : ncols;   // the mean modes use column (0,0) only
        const size_t n = (size_t)nc * ctx->nyp;
        CK(cudaMalloc(&T.td[c], sizeof(double) * n));
        CK(cudaMalloc(&T.te[c], sizeof(double) * n));
        CK(cudaMalloc(&T.tb1[c], sizeof(double) * n));
        CK(cudaMalloc(&T.tb2[c], sizeof(double) * n));
        CK(cudaMalloc(&T.tf[c], sizeof(double) * 4 * nc));
        T.g[c] = cfg[c].g;
        k_tau_tables<<<(nc + 127) / 128, 128, 0, ctx->stream>>>(T.td[c], T.te[c], T.tb1[c], T.tb2[c], T.tf[c], cfg[c],
                                                               ctx->d_wavx, ctx->d_wavz, nc, ctx->nz, ctx->nyp,
                                                               ctx->dyde);
        CKL();
    }
    // reciprocals of the tau row coefficients (the same divisions as the device's tau_rhs)
    RET(upload_rj(ctx, &F->rj, false));
    if (ctx->ny % 16 == 0) {   // the blocked column kernels' copies
        for (int c = 0; c < TB_N; ++c) {
            const int nc = (c == TB_U0 || c == TB_W0) ? 1 : ncols;
            const double *src[4] = {T.td[c], T.te[c], T.tb1[c], T.tb2[c]};
            double *dst[4];
            RET(block_tables(ctx, src, dst, nc));
            F->btabs.td[c] = dst[0]; F->btabs.te[c] = dst[1]; F->btabs.tb1[c] = dst[2]; F->btabs.tb2[c] = dst[3];
            F->btabs.tf[c] = T.tf[c];
            F->btabs.g[c] = T.g[c];
        }
        RET(upload_rj(ctx, &F->brj, true));
    }
    RET(make_twf(ctx, 2 * ctx->ny, &F->twf_y2));
    RET(make_twf(ctx, ctx->mz, &F->twf_mz));
    RET(make_twf(ctx, ctx->mx, &F->twf_mx));
    const size_t ncp = (size_t)ncols * ctx->nyp, nq = (size_t)ctx->nyp * ctx->mz * ctx->nxh;
    CK(cudaMalloc(&F->yp, sizeof(double2) * ncp * 8));
    CK(cudaMalloc(&F->q, sizeof(double2) * nq * 10));
    CK(cudaMalloc(&F->r, sizeof(double2) * nq * 4));
    CK(cudaMalloc(&F->yo, sizeof(double2) * ncp * 4));
    return KMM_OK;
}

// tau tables of the routine path's solve / penta calls: one set per (g, boundary-condition)
// configuration met, built on first use with the same recurrences as the fused step's and kept
// for the context's lifetime (a run meets a handful: v's two solves, omega_y, the scalar and the
// polymer components)
#define KMM_TAU_SETS 12
struct TauCache {
    int n;
    TabCfg cfg[KMM_TAU_SETS];
    double *tabs[KMM_TAU_SETS][5];   // td (as 1 / d), te, tb1, tb2 in the lane-blocked order; tf
    double *rj;                      // lane-blocked rj rows
};

int kmm_tau_tabset(kmm_ctx *ctx, double g, int robin, double at, double bt, double ab, double bb, const double **tabs,
                   const double **rj) {
    TauCache *C = (TauCache *)ctx->tauc;
    if (!C) {
        C = (TauCache *)calloc(1, sizeof(TauCache));
        if (!C) return KMM_ERR_NOMEM;
        ctx->tauc = C;
        RET(upload_rj(ctx, &C->rj, true));
    }
    const TabCfg want = {g, robin, robin ? at : 0.0, robin ? bt : 0.0, robin ? ab : 0.0, robin ? bb : 0.0, 1.0};
    int s = -1;
    for (int i = 0; i < C->n && s < 0; ++i) {
        const TabCfg &c = C->cfg[i];
        if (c.g == want.g && c.robin == want.robin && c.at == want.at && c.bt == want.bt && c.ab == want.ab &&
            c.bb == want.bb)
            s = i;
    }
    if (s < 0) {
        if (C->n == KMM_TAU_SETS) return KMM_ERR_UNSUPPORTED;   // the caller keeps the table-free kernels
        s = C->n;
        const int ncols = ctx->nz * ctx->nxh;
        const size_t n = (size_t)ncols * ctx->nyp;
        double *canon[4] = {NULL, NULL, NULL, NULL};
        for (int a = 0; a < 4; ++a) CK(cudaMalloc(&canon[a], sizeof(double) * n));
        CK(cudaMalloc(&C->tabs[s][4], sizeof(double) * 4 * ncols));
        k_tau_tables<<<(ncols + 127) / 128, 128, 0, ctx->stream>>>(canon[0], canon[1], canon[2], canon[3],
                                                                  C->tabs[s][4], want, ctx->d_wavx, ctx->d_wavz,
                                                                  ncols, ctx->nz, ctx->nyp, ctx->dyde);
        CKL();
        const double *src[4] = {canon[0], canon[1], canon[2], canon[3]};
        const int bst = block_tables(ctx, src, C->tabs[s], ncols);
        CK(cudaStreamSynchronize(ctx->stream));   // once per configuration, before the canonical copies go
        for (int a = 0; a < 4; ++a) cudaFree(canon[a]);
        RET(bst);
        C->cfg[s] = want;
        C->n = s + 1;
    }
    for (int a = 0; a < 5; ++a) tabs[a] = C->tabs[s][a];
    *rj = C->rj;
    return KMM_OK;
}

int kmm_routine_tw32(kmm_ctx *ctx, const float2 **y2, const float2 **mz, const float2 **mx) {
    const int n[3] = {2 * ctx->ny, ctx->mz, ctx->mx};
    for (int t = 0; t < 3; ++t)
        if (!ctx->rtw32[t]) RET(make_twf(ctx, n[t], &ctx->rtw32[t]));
    *y2 = ctx->rtw32[0];
    *mz = ctx->rtw32[1];
    *mx = ctx->rtw32[2];
    return KMM_OK;
}

void kmm_tau_release(kmm_ctx *ctx) {
    for (int t = 0; t < 3; ++t) {
        if (ctx->rtw32[t]) cudaFree(ctx->rtw32[t]);
        ctx->rtw32[t] = NULL;
    }
    TauCache *C = (TauCache *)ctx->tauc;
    if (!C) return;
    for (int i = 0; i < C->n; ++i)
        for (int a = 0; a < 5; ++a) cudaFree(C->tabs[i][a]);
    cudaFree(C->rj);
    free(C);
    ctx->tauc = NULL;
}

void kmm_fused_release(kmm_ctx *ctx) {
    KmmFused *F = ctx->fused;
    if (!F) return;
    for (int c = 0; c < TB_N; ++c) {
        cudaFree(F->tabs.td[c]); cudaFree(F->tabs.te[c]); cudaFree(F->tabs.tb1[c]); cudaFree(F->tabs.tb2[c]);
        cudaFree(F->tabs.tf[c]);
        cudaFree(F->btabs.td[c]); cudaFree(F->btabs.te[c]); cudaFree(F->btabs.tb1[c]); cudaFree(F->btabs.tb2[c]);
    }
    cudaFree(F->yp); cudaFree(F->q); cudaFree(F->r); cudaFree(F->yo); cudaFree(F->rj); cudaFree(F->brj);
    cudaFree(F->twf_y2); cudaFree(F->twf_mz); cudaFree(F->twf_mx);
    free(F);
    ctx->fused = NULL;
}


// ---------------------------------------------------------------------------
// column helpers
// ---------------------------------------------------------------------------
// phirhs on one column (solvers.f90:633-675): x <- RHS of the CN/AB2 Helmholtz problem
template <int E>
__device__ __forceinline__ void col_phirhs(Col<E> &x, const Col<E> &fn, const Col<E> &fnm1, double re, double var,
                                           double dt, double th, double w2, int nyp, double dyde) {
    const double a = -re * var / (dt * th), b = re * var / (2.0 * th);
    const double c = (1.0 - th) * w2;
    Col<E> w;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        double2 r;
        r.x = a * x.v[e].x - b * (3.0 * fn.v[e].x - fnm1.v[e].x);
        r.y = a * x.v[e].y - b * (3.0 * fn.v[e].y - fnm1.v[e].y);
        if (th > 0.99) x.v[e] = r;
        r.x = r.x + c * x.v[e].x / th;
        r.y = r.y + c * x.v[e].y / th;
        w.v[e] = r;
    }
    Col<E> d1, d2;
    col_cderiv<E>(d1, x, nyp, dyde);
    col_cderiv<E>(d2, d1, nyp, dyde);
#pragma unroll
    for (int e = 0; e < E; ++e)
        x.v[e] = make_double2(w.v[e].x - (1.0 - th) * d2.v[e].x / th, w.v[e].y - (1.0 - th) * d2.v[e].y / th);
}

// norm (helpers.f90:91-158) on a column pair held by the two warps of the block.  The exchange
// buffer holds one column per warp; kx = 0 pairs (j, nz-j) average, (0,0) becomes real, the
// kz Nyquist column is zeroed.
template <int E>
__device__ __forceinline__ void col_norm(Col<E> &x, double2 *xbuf, int kx, int j, int nzh) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (kx == 0) {
#pragma unroll
        for (int e = 0; e < E; ++e) xbuf[warp * 32 * E + lane + 32 * e] = x.v[e];
        __syncthreads();
        if (j != 0 && j != nzh) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const double2 mine = x.v[e], oth = xbuf[(1 - warp) * 32 * E + lane + 32 * e];
                // both warps form m = 0.5 (a_j + conj(a_jp)) from the same operands
                const double2 aj = warp == 0 ? mine : oth, ajp = warp == 0 ? oth : mine;
                const double2 m = make_double2(0.5 * (aj.x + ajp.x), 0.5 * (aj.y - ajp.y));
                x.v[e] = warp == 0 ? m : make_double2(m.x, -m.y);
            }
        }
        __syncthreads();
    }
    if (j == nzh) {
#pragma unroll
        for (int e = 0; e < E; ++e) x.v[e] = make_double2(0.0, 0.0);
    } else if (kx == 0 && j == 0) {
#pragma unroll
        for (int e = 0; e < E; ++e) x.v[e].y = 0.0;
    }
}

// DCT-I of one column through the warp FFT (even extension of length 2 ny):
//   to_phys: scale by c(i)/2 first (solvers.f90:2241-2546);  !to_phys: /ny, halve the ends (3279-3416)
template <int E, int L0>
__device__ __forceinline__ void col_dct(Col<E> &x, double2 *a, double2 *b, const DevPlan &P, int nyp, bool to_phys) {
    const int lane = threadIdx.x & 31;
    const int ny = nyp - 1, L = 2 * ny;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane + 32 * e;
        if (i < nyp) {
            double2 v = x.v[e];
            if (to_phys && i > 0 && i < ny) v = make_double2(v.x * 0.5, v.y * 0.5);
            a[i] = v;
            if (i > 0 && i < ny) a[L - i] = v;
        }
    }
    __syncwarp();
    const double2 *r;
    if constexpr (L0 > 0) r = fft_warp_ct<double2, L0, -1>(a, b, P.tw);
    else r = fft_warp(P, a, b, -1);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane + 32 * e;
        double2 v = i < nyp ? r[i] : make_double2(0.0, 0.0);
        if (!to_phys) {
            v = make_double2(v.x / (double)ny, v.y / (double)ny);
            if (i == 0 || i == ny) v = make_double2(v.x / 2.0, v.y / 2.0);
        }
        x.v[e] = v;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// forward column kernel
// ---------------------------------------------------------------------------

// L0 > 0: 2 ny is the compile-time constant L0 (specialised DCT); L0 = 0: runtime plan
template <int E, int L0>
__global__ void __launch_bounds__(64) k_col_fwd(ColFwdArgs A, FusedTabs T, const __grid_constant__ DevPlan P) {
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nyp = A.nyp, ny = nyp - 1, L = 2 * ny;
    double2 *xbuf = sm;                                   // 2 * 32 * E
    double2 *fa = sm + 64 * E + (size_t)warp * 2 * L, *fb = fa + L;
    const int npair = A.nz / 2;
    const int q = blockIdx.x % npair, kx = blockIdx.x / npair;
    const int j = warp == 0 ? q : (q == 0 ? A.nzh : A.nz - q);
    const int col = kx * A.nz + j;
    const size_t off = (size_t)col * nyp;
    const double kxv = A.wavx[kx], kzv = A.wavz[j];
    const double w2 = kzv * kzv + kxv * kxv;
    const double g1 = A.re / (A.dt * A.th);
    const bool mean = (kx == 0 && j == 0);
    const size_t ncols = (size_t)A.nz * A.nxh;

    // ---- passive scalar (main_dns.f90:325-359)
    Col<E> s;
    if (A.scalar) {
        col_load<E>(s, A.scal + off, nyp);
        Col<E> n1, n0;
        col_load<E>(n1, A.scn + off, nyp);
        col_load<E>(n0, A.scnm1 + off, nyp);
        col_phirhs<E>(s, n1, n0, A.re, A.diff, A.dt, A.th, w2, nyp, A.dyde);
        const TauTab ts = tab_at(T, TB_SCL, col, nyp);
        col_solve_robin<E>(s, ts, make_double2(0.0, 0.0), make_double2(0.0, 0.0), w2 + T.g[TB_SCL], nyp, A.c0);
    }
    // ---- wall-normal velocity: phi, phirhs, Helmholtz + Poisson (main_dns.f90:363-407)
    Col<E> v, d1, d2;
    col_load<E>(v, A.v + off, nyp);
    col_cderiv<E>(d1, v, nyp, A.dyde);
    col_cderiv<E>(d2, d1, nyp, A.dyde);
#pragma unroll
    for (int e = 0; e < E; ++e) v.v[e] = make_double2(d2.v[e].x - w2 * v.v[e].x, d2.v[e].y - w2 * v.v[e].y);
    {
        Col<E> f1, f0;
        col_load<E>(f1, A.fn + off, nyp);
        col_load<E>(f0, A.fnm1 + off, nyp);
        col_phirhs<E>(v, f1, f0, A.re, 1.0, A.dt, A.th, w2, nyp, A.dyde);
    }
    {
        const TauTab tp = tab_at(T, TB_PHI, col, nyp);
        col_solve_dirichlet<E>(v, tp, make_double2(0.0, 0.0), make_double2(0.0, 0.0), w2 + g1, nyp, A.c0);
        const TauTab tv = tab_at(T, TB_V, col, nyp);
        col_solve_dirichlet<E>(v, tv, make_double2(0.0, 0.0), make_double2(0.0, 0.0), w2, nyp, A.c0);
    }
    // ---- normal vorticity phirhs (main_dns.f90:411-422)
    Col<E> om;
    col_load<E>(om, A.omy + off, nyp);
    {
        Col<E> g1c, g0c;
        col_load<E>(g1c, A.gn + off, nyp);
        col_load<E>(g0c, A.gnm1 + off, nyp);
        col_phirhs<E>(om, g1c, g0c, A.re, 1.0, A.dt, A.th, w2, nyp, A.dyde);
    }
    // ---- influence matrix (main_dns.f90:426-466)
    {
        double2 wb, wt, tmp;
        if (A.nb == 1 && A.nt == 1) {
            col_wall1<E>(v, nyp, A.dyde, wb, wt);
        } else {
            Col<E> dv;
            col_cderiv<E>(dv, v, nyp, A.dyde);
            double2 b2, t2;
            col_wall1<E>(dv, nyp, A.dyde, b2, t2);
            col_wall1<E>(v, nyp, A.dyde, wb, wt);
            if (A.nb == 2) wb = b2;
            if (A.nt == 2) wt = t2;
            (void)tmp;
        }
        const double2 c1 = cdiv(csub(cmul(wb, A.dnv2t[col]), cmul(wt, A.dnv2b[col])), A.denom[col]);
        const double2 c2 = cdiv(csub(cmul(wt, A.dnv1b[col]), cmul(wb, A.dnv1t[col])), A.denom[col]);
        Col<E> gfa;
        col_load<E>(gfa, A.gf1 + off, nyp);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double2 a = cmul(c1, gfa.v[e]);
            v.v[e] = make_double2(v.v[e].x + a.x, v.v[e].y + a.y);
        }
        col_load<E>(gfa, A.gf2 + off, nyp);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double2 b = cmul(c2, gfa.v[e]);
            v.v[e] = make_double2(v.v[e].x + b.x, v.v[e].y + b.y);
        }
    }
    // ---- normal vorticity Robin solve (main_dns.f90:479-484)
    {
        const TauTab to = tab_at(T, TB_OMY, col, nyp);
        col_solve_robin<E>(om, to, make_double2(0.0, 0.0), make_double2(0.0, 0.0), w2 + g1, nyp, A.c0);
    }
    // ---- mean modes (main_dns.f90:489-502): uzero for u0 and w0 with the warp Robin solver
    if (mean) {
        const double th = A.th;
        for (int which = 0; which < 2; ++which) {
            double *U = which == 0 ? A.u0 : A.w0;
            const double *H = which == 0 ? A.h1n : A.h3n, *HL = which == 0 ? A.h1nm1 : A.h3nm1;
            Col<E> uc, dd1, dd2;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int i = lane + 32 * e;
                uc.v[e] = make_double2(i < nyp ? U[i] : 0.0, 0.0);
            }
            // wrk1 = -re u0/(dt th) - re (3 h1 - h1l)/(2 th); u0 <- wrk1 - (1-th) u0''/th (solvers.f90:1127-1143)
            col_cderiv<E>(dd1, uc, nyp, A.dyde);
            col_cderiv<E>(dd2, dd1, nyp, A.dyde);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int i = lane + 32 * e;
                double r = 0.0;
                if (i < nyp) {
                    const double w1 = -A.re * uc.v[e].x / (A.dt * th) - A.re * (3.0 * H[i] - HL[i]) / (2.0 * th);
                    r = (th > 0.99) ? w1 : w1 - (1.0 - th) * dd2.v[e].x / th;
                }
                uc.v[e] = make_double2(r, 0.0);
            }
            const TauTab tm = tab_at(T, which == 0 ? TB_U0 : TB_W0, 0, nyp);
            const double gt = which == 0 ? A.gtu : A.gtw, gb = which == 0 ? A.gbu : A.gbw;
            col_solve_robin<E>(uc, tm, make_double2(gt, 0.0), make_double2(gb, 0.0), g1, nyp, A.c0);
            __syncwarp();
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int i = lane + 32 * e;
                if (i < nyp) U[i] = uc.v[e].x;
            }
        }
        __syncwarp();
        for (int i = lane; i < nyp; i += 32) {
            A.h1nm1[i] = A.h1n[i];
            A.h3nm1[i] = A.h3n[i];
        }
#pragma unroll
        for (int e = 0; e < E; ++e) om.v[e] = make_double2(0.0, 0.0);
    }
    // ---- norm(v), norm(omy); veloc (main_dns.f90:520-526, solvers.f90:1576-1659)
    col_norm<E>(v, xbuf, kx, j, A.nzh);
    col_norm<E>(om, xbuf, kx, j, A.nzh);
    Col<E> u, w;
    {
        Col<E> dv;
        col_cderiv<E>(dv, v, nyp, A.dyde);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double2 d = dv.v[e], o = om.v[e];
            if (kx > 0) {
                const double2 sa = cadd(cimul(d, -kxv), cimul(o, kzv));
                u.v[e] = make_double2(-sa.x / w2, -sa.y / w2);
                const double2 sb = csub(cimul(d, -kzv), cimul(o, kxv));
                w.v[e] = make_double2(-sb.x / w2, -sb.y / w2);
            } else if (j > 0) {
                const double kz2 = kzv * kzv;
                const double2 sa = cimul(o, kzv);
                u.v[e] = make_double2(-sa.x / kz2, -sa.y / kz2);
                const double2 sb = cimul(d, -kzv);
                w.v[e] = make_double2(-sb.x / kz2, -sb.y / kz2);
            }
        }
        if (mean) {
            __syncwarp();
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int i = lane + 32 * e;
                u.v[e] = make_double2(i < nyp ? A.u0[i] : 0.0, 0.0);
                w.v[e] = make_double2(i < nyp ? A.w0[i] : 0.0, 0.0);
                v.v[e] = make_double2(0.0, 0.0);
            }
        }
        // norm(u), norm(w): the pair is conjugate-symmetric already; zero the kz Nyquist column
        if (j == A.nzh) {
#pragma unroll
            for (int e = 0; e < E; ++e) { u.v[e] = make_double2(0.0, 0.0); w.v[e] = make_double2(0.0, 0.0); }
        }
    }
    col_store<E>(A.v + off, v, nyp);
    col_store<E>(A.omy + off, om, nyp);
    // ---- y-physical outputs: u, v, w, omega_y, du/dy, dw/dy [, c, dc/dy]
    double2 *yp = A.yp;
    col_dct<E, L0>(v, fa, fb, P, nyp, true);
    col_store<E>(yp + 1 * ncols * nyp + off, v, nyp);
    col_dct<E, L0>(om, fa, fb, P, nyp, true);
    col_store<E>(yp + 3 * ncols * nyp + off, om, nyp);
    col_cderiv<E>(d1, u, nyp, A.dyde);
    col_dct<E, L0>(u, fa, fb, P, nyp, true);
    col_store<E>(yp + 0 * ncols * nyp + off, u, nyp);
    col_dct<E, L0>(d1, fa, fb, P, nyp, true);
    col_store<E>(yp + 4 * ncols * nyp + off, d1, nyp);
    col_cderiv<E>(d1, w, nyp, A.dyde);
    col_dct<E, L0>(w, fa, fb, P, nyp, true);
    col_store<E>(yp + 2 * ncols * nyp + off, w, nyp);
    col_dct<E, L0>(d1, fa, fb, P, nyp, true);
    col_store<E>(yp + 5 * ncols * nyp + off, d1, nyp);
    if (A.scalar) {
        col_norm<E>(s, xbuf, kx, j, A.nzh);
        col_store<E>(A.scal + off, s, nyp);
        col_cderiv<E>(d1, s, nyp, A.dyde);
        col_dct<E, L0>(s, fa, fb, P, nyp, true);
        col_store<E>(yp + 6 * ncols * nyp + off, s, nyp);
        col_dct<E, L0>(d1, fa, fb, P, nyp, true);
        col_store<E>(yp + 7 * ncols * nyp + off, d1, nyp);
    }
}

// ---------------------------------------------------------------------------
// z transforms on (kx, y) tiles
// ---------------------------------------------------------------------------
#define ZT_KX 4
#define ZT_Y 4
#define ZT_WARPS (ZT_KX * ZT_Y)

// Q[g][y][z][kx], g = u v w wx wy wz [cx cy cz], from the y-physical base fields
// MZ > 0: compile-time z length (specialised FFT); MZ = 0: runtime plan
template <int MZ>
__global__ void __launch_bounds__(ZT_WARPS * 32) k_zb(const double2 *__restrict__ yp, double2 *__restrict__ q,
                                                      const double *__restrict__ wavx, const double *__restrict__ wavz,
                                                      const __grid_constant__ DevPlan P, int nout, int nyp, int nz, int nxh, int mz_rt) {
    const int mz = MZ > 0 ? MZ : mz_rt;
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kl = warp % ZT_KX, yl = warp / ZT_KX;
    const int kx = blockIdx.x * ZT_KX + kl, y = blockIdx.y * ZT_Y + yl;
    const bool act = kx < nxh && y < nyp;
    const size_t ncols = (size_t)nz * nxh;
    const int nzh = nz / 2;
    double2 *a = sm + (size_t)warp * 2 * mz, *b = a + mz;
    double2 *stage = sm + (size_t)ZT_WARPS * 2 * mz;   // [y][z][kx] tile for the store
    const double kxv = act ? wavx[kx] : 0.0;
    auto SW = [](int x) { return MZ > 0 ? swz<double2>(x) : x; };
    for (int g = 0; g < nout; ++g) {
        if (act) {
            for (int z = lane; z < mz; z += 32) a[SW(z)] = make_double2(0.0, 0.0);
            __syncwarp();
            for (int kz = lane; kz < nz; kz += 32) {
                const size_t o = ((size_t)kx * nz + kz) * nyp + y;
                const double kzv = wavz[kz];
                double2 val;
                switch (g < 6 ? g : g + 1) {   // q fields: u v w wx wy wz [cx cy cz]
                case 3: {   // wx = dw/dy - i kz v
                    const double2 dw = __ldg(yp + 5 * ncols * nyp + o), vv = __ldg(yp + 1 * ncols * nyp + o);
                    val = csub(dw, cimul(vv, kzv));
                } break;
                case 4: val = __ldg(yp + 3 * ncols * nyp + o); break;
                case 5: {   // wz = i kx v - du/dy
                    const double2 vv = __ldg(yp + 1 * ncols * nyp + o), du = __ldg(yp + 4 * ncols * nyp + o);
                    val = csub(cimul(vv, kxv), du);
                } break;
                case 6: val = __ldg(yp + 6 * ncols * nyp + o); break;
                case 7: val = cimul(__ldg(yp + 6 * ncols * nyp + o), kxv); break;
                case 8: val = __ldg(yp + 7 * ncols * nyp + o); break;
                case 9: val = cimul(__ldg(yp + 6 * ncols * nyp + o), kzv); break;
                default: val = __ldg(yp + (size_t)g * ncols * nyp + o); break;   // u v w
                }
                const int jj = kz < nzh ? kz : (mz - nz) + kz;
                a[SW(jj)] = val;
            }
            __syncwarp();
            const double2 *r;
            if constexpr (MZ > 0) r = fft_warp_ct<double2, MZ, +1, 1, true>(a, b, P.tw);
            else r = fft_warp(P, a, b, +1);
            for (int z = lane; z < mz; z += 32) stage[((size_t)yl * mz + z) * ZT_KX + kl] = r[SW(z)];
        }
        __syncthreads();
        // store rows of ZT_KX consecutive kx
        const int kx0 = blockIdx.x * ZT_KX;
        for (int t = threadIdx.x; t < ZT_Y * mz * ZT_KX; t += blockDim.x) {
            const int kk = t % ZT_KX, zz = (t / ZT_KX) % mz, yy = t / (ZT_KX * mz);
            const int ky = blockIdx.y * ZT_Y + yy;
            if (ky < nyp && kx0 + kk < nxh)
                q[(((size_t)g * nyp + ky) * mz + zz) * nxh + kx0 + kk] = stage[t];
        }
        __syncthreads();
    }
}

// y-physical outputs [o][ncols][nyp] from R[o][y][z][kx]
template <int MZ>
__global__ void __launch_bounds__(ZT_WARPS * 32) k_zf(const double2 *__restrict__ r, double2 *__restrict__ yo, const __grid_constant__ DevPlan P,
                                                      int nout, int nyp, int nz, int nxh, int mz_rt, double scale) {
    const int mz = MZ > 0 ? MZ : mz_rt;
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kl = warp % ZT_KX, yl = warp / ZT_KX;
    const int kx = blockIdx.x * ZT_KX + kl, y = blockIdx.y * ZT_Y + yl;
    const bool act = kx < nxh && y < nyp;
    const size_t ncols = (size_t)nz * nxh;
    const int nzh = nz / 2;
    double2 *a = sm + (size_t)warp * 2 * mz, *b = a + mz;
    double2 *stage = sm + (size_t)ZT_WARPS * 2 * mz;   // [kx][kz][y] tile for the store
    auto SW = [](int x) { return MZ > 0 ? swz<double2>(x) : x; };
    for (int o = 0; o < nout; ++o) {
        if (act) {
            for (int z = lane; z < mz; z += 32) a[SW(z)] = __ldg(r + (((size_t)o * nyp + y) * mz + z) * nxh + kx);
            __syncwarp();
            const double2 *res;
            if constexpr (MZ > 0) res = fft_warp_ct<double2, MZ, -1, 1, true>(a, b, P.tw);
            else res = fft_warp(P, a, b, -1);
            for (int kz = lane; kz < nz; kz += 32) {
                const int jj = kz < nzh ? kz : (mz - nz) + kz;
                const double2 v = res[SW(jj)];
                stage[((size_t)kl * nz + kz) * ZT_Y + yl] = make_double2(v.x / scale, v.y / scale);
            }
        }
        __syncthreads();
        const int kx0 = blockIdx.x * ZT_KX, y0 = blockIdx.y * ZT_Y;
        for (int t = threadIdx.x; t < ZT_KX * nz * ZT_Y; t += blockDim.x) {
            const int yy = t % ZT_Y, kz = (t / ZT_Y) % nz, kk = t / (ZT_Y * nz);
            if (kx0 + kk < nxh && y0 + yy < nyp)
                yo[(size_t)o * ncols * nyp + ((size_t)(kx0 + kk) * nz + kz) * nyp + y0 + yy] = stage[t];
        }
        __syncthreads();
    }
}

// Specialised z kernels for the compiled lengths MZ (nz = 2 MZ / 3), C = double2 (FP64) or
// float2 (mixed precision), with the next field's column values fetched into registers while the
// current field's FFT runs.
template <int MZ, typename C>
__global__ void __launch_bounds__(ZT_WARPS * 32) k_zb2(const C *__restrict__ yp, C *__restrict__ q,
                                                       const double *__restrict__ wavx, const double *__restrict__ wavz,
                                                       const C *__restrict__ tw, int nout, int nyp, int nxh) {
    typedef typename kct::Real<C>::T T;
    constexpr int NZ = 2 * MZ / 3, NZH = NZ / 2, NE = (NZ + 31) / 32;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kl = warp % ZT_KX, yl = warp / ZT_KX;
    const int kx = blockIdx.x * ZT_KX + kl, y = blockIdx.y * ZT_Y + yl;
    const bool act = kx < nxh && y < nyp;
    const int ldc = col_ld<C>(nyp);
    const size_t fs = (size_t)NZ * nxh * ldc;   // field stride of the column layout
    C *a = sm + (size_t)warp * 2 * MZ, *b = a + MZ;
    C *stage = sm + (size_t)ZT_WARPS * 2 * MZ;   // [y][z][kx] tile for the store
    const T kxv = act ? (T)wavx[kx] : (T)0;
    const C zc = kct::mk<C>((T)0, (T)0);
    C pf[NE];
    // value of q field g at (kx, kz, y) from the y-physical base fields u v w omega_y du/dy dw/dy [c dc/dy]
    auto fetch = [&](int g) {
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int kz = lane + 32 * e;
            C val = zc;
            if (act && kz < NZ) {
                const size_t o = ((size_t)kx * NZ + kz) * ldc + y;
                const T kzv = (T)wavz[kz];
                switch (g < 6 ? g : g + 1) {   // q fields: u v w wx wy wz [cx cy cz]
                case 3: {                      // wx = dw/dy - i kz v
                    const C dw = __ldg(yp + 5 * fs + o), vv = __ldg(yp + 1 * fs + o);
                    val = kct::mk<C>(dw.x + kzv * vv.y, dw.y - kzv * vv.x);
                } break;
                case 4: val = __ldg(yp + 3 * fs + o); break;
                case 5: {   // wz = i kx v - du/dy
                    const C vv = __ldg(yp + 1 * fs + o), du = __ldg(yp + 4 * fs + o);
                    val = kct::mk<C>(-kxv * vv.y - du.x, kxv * vv.x - du.y);
                } break;
                case 7: {
                    const C cc = __ldg(yp + 6 * fs + o);
                    val = kct::mk<C>(-kxv * cc.y, kxv * cc.x);
                } break;
                case 8: val = __ldg(yp + 7 * fs + o); break;
                case 9: {
                    const C cc = __ldg(yp + 6 * fs + o);
                    val = kct::mk<C>(-kzv * cc.y, kzv * cc.x);
                } break;
                default: val = __ldg(yp + (size_t)g * fs + o); break;   // u v w
                }
            }
            pf[e] = val;
        }
    };
    fetch(0);
    for (int g = 0; g < nout; ++g) {
        if (act) {
            for (int z = NZH + lane; z < MZ - NZH; z += 32) a[swz<C>(z)] = zc;   // padding modes
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                const int kz = lane + 32 * e;
                if (kz < NZ) a[swz<C>(kz < NZH ? kz : (MZ - NZ) + kz)] = pf[e];
            }
            __syncwarp();
        }
        if (g + 1 < nout) fetch(g + 1);
        if (act) {
            const C *r = fft_warp_ct<C, MZ, +1, 1, true>(a, b, tw);
            for (int z = lane; z < MZ; z += 32) stage[((size_t)yl * MZ + z) * ZT_KX + kl] = r[swz<C>(z)];
        }
        __syncthreads();
        // store rows of ZT_KX consecutive kx
        const int kx0 = blockIdx.x * ZT_KX;
        for (int t = threadIdx.x; t < ZT_Y * MZ * ZT_KX; t += blockDim.x) {
            const int kk = t % ZT_KX, zz = (t / ZT_KX) % MZ, yy = t / (ZT_KX * MZ);
            const int ky = blockIdx.y * ZT_Y + yy;
            if (ky < nyp && kx0 + kk < nxh) q[(((size_t)g * nyp + ky) * MZ + zz) * nxh + kx0 + kk] = stage[t];
        }
        __syncthreads();
    }
}

template <int MZ, typename C>
__global__ void __launch_bounds__(ZT_WARPS * 32) k_zf2(const C *__restrict__ r, C *__restrict__ yo,
                                                       const C *__restrict__ tw, int nout, int nyp, int nxh,
                                                       double scale) {
    typedef typename kct::Real<C>::T T;
    constexpr int NZ = 2 * MZ / 3, NZH = NZ / 2, NE = (MZ + 31) / 32;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kl = warp % ZT_KX, yl = warp / ZT_KX;
    const int kx = blockIdx.x * ZT_KX + kl, y = blockIdx.y * ZT_Y + yl;
    const bool act = kx < nxh && y < nyp;
    const size_t ncols = (size_t)NZ * nxh;
    C *a = sm + (size_t)warp * 2 * MZ, *b = a + MZ;
    C *stage = sm + (size_t)ZT_WARPS * 2 * MZ;   // [kx][kz][y] tile for the store
    const T rs = (T)(1.0 / scale);
    C pf[NE];
    auto fetch = [&](int o) {
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int z = lane + 32 * e;
            if (act && z < MZ) pf[e] = __ldg(r + (((size_t)o * nyp + y) * MZ + z) * nxh + kx);
        }
    };
    fetch(0);
    for (int o = 0; o < nout; ++o) {
        if (act) {
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                const int z = lane + 32 * e;
                if (z < MZ) a[swz<C>(z)] = pf[e];
            }
            __syncwarp();
        }
        if (o + 1 < nout) fetch(o + 1);
        if (act) {
            const C *res = fft_warp_ct<C, MZ, -1, 1, true>(a, b, tw);
            for (int kz = lane; kz < NZ; kz += 32) {
                const C v = res[swz<C>(kz < NZH ? kz : (MZ - NZ) + kz)];
                // FP64 divides by mx mz as the reference normalises; FP32 multiplies by the reciprocal
                stage[((size_t)kl * NZ + kz) * ZT_Y + yl] =
                    sizeof(T) == 8 ? kct::mk<C>((T)(v.x / scale), (T)(v.y / scale)) : kct::mk<C>(v.x * rs, v.y * rs);
            }
        }
        __syncthreads();
        const int kx0 = blockIdx.x * ZT_KX, y0 = blockIdx.y * ZT_Y;
        for (int t = threadIdx.x; t < ZT_KX * NZ * ZT_Y; t += blockDim.x) {
            const int yy = t % ZT_Y, kz = (t / ZT_Y) % NZ, kk = t / (ZT_Y * NZ);
            if (kx0 + kk < nxh && y0 + yy < nyp)
                yo[((size_t)o * ncols + (size_t)(kx0 + kk) * NZ + kz) * col_ld<C>(nyp) + y0 + yy] = stage[t];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// backward column kernel
// ---------------------------------------------------------------------------

template <int E, int L0>
__global__ void __launch_bounds__(64) k_col_bwd(ColBwdArgs A, const __grid_constant__ DevPlan P) {
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nyp = A.nyp, ny = nyp - 1, L = 2 * ny;
    double2 *xbuf = sm;
    double2 *fa = sm + 64 * E + (size_t)warp * 2 * L, *fb = fa + L;
    const int npair = A.nz / 2;
    const int q = blockIdx.x % npair, kx = blockIdx.x / npair;
    const int j = warp == 0 ? q : (q == 0 ? A.nzh : A.nz - q);
    const int col = kx * A.nz + j;
    const size_t off = (size_t)col * nyp;
    const size_t ncols = (size_t)A.nz * A.nxh;
    const double kxv = A.wavx[kx], kzv = A.wavz[j];
    Col<E> h1, h2, h3;
    col_load<E>(h1, A.yo + 0 * ncols * nyp + off, nyp);
    col_dct<E, L0>(h1, fa, fb, P, nyp, false);
    col_load<E>(h2, A.yo + 1 * ncols * nyp + off, nyp);
    col_dct<E, L0>(h2, fa, fb, P, nyp, false);
    col_load<E>(h3, A.yo + 2 * ncols * nyp + off, nyp);
    col_dct<E, L0>(h3, fa, fb, P, nyp, false);
    // norm(fn), norm(gn), norm(omz) after vcw3dp (main_dns.f90:620-624)
    col_norm<E>(h2, xbuf, kx, j, A.nzh);
    col_norm<E>(h1, xbuf, kx, j, A.nzh);
    col_norm<E>(h3, xbuf, kx, j, A.nzh);
    // spectral filter (main_dns.f90:710-745)
    const int j1 = j + 1;
    const int jjf = (j1 > A.nzh) ? A.nz - j1 + 1 : j1 - 1;
    const double zr = (double)jjf / (double)A.nzh;
    double z2 = zr * zr, z4 = z2 * z2, z8 = z4 * z4;
    const double zs = exp(-3.0 * (z8 * z2));
    Col<E> sc;
    if (A.scalar) {
        col_load<E>(sc, A.yo + 3 * ncols * nyp + off, nyp);
        col_dct<E, L0>(sc, fa, fb, P, nyp, false);
        col_norm<E>(sc, xbuf, kx, j, A.nzh);
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane + 32 * e;
        const double yr = (double)i / (double)ny;
        const double y2 = yr * yr, y4 = y2 * y2, y8 = y4 * y4;
        const double ys = exp(-3.0 * (y8 * y2));
        h3.v[e] = make_double2(h3.v[e].x * zs * ys, h3.v[e].y * zs * ys);
        h1.v[e] = make_double2(h1.v[e].x * zs * ys, h1.v[e].y * zs * ys);
        h2.v[e] = make_double2(h2.v[e].x * zs * ys, h2.v[e].y * zs * ys);
        if (A.scalar) sc.v[e] = make_double2(sc.v[e].x * zs * ys, sc.v[e].y * zs * ys);
    }
    // h1n = Re gn(:,1,1), h3n = Re omz(:,1,1) (main_dns.f90:748-751)
    if (kx == 0 && j == 0) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int i = lane + 32 * e;
            if (i < nyp) { A.h1n[i] = h1.v[e].x; A.h3n[i] = h3.v[e].x; }
        }
    }
    // nonlin (solvers.f90:1497-1572): fn = -k^2 h2 - d/dy(i(kz h3 + kx h1)); gn = i(kz h1 - kx h3)
    Col<E> t, d;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const double2 s = make_double2(kzv * h3.v[e].x + kxv * h1.v[e].x, kzv * h3.v[e].y + kxv * h1.v[e].y);
        t.v[e] = make_double2(-s.y, s.x);
    }
    col_cderiv<E>(d, t, nyp, A.dyde);
    const double w2 = -kxv * kxv - kzv * kzv;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        h2.v[e] = make_double2(w2 * h2.v[e].x - d.v[e].x, w2 * h2.v[e].y - d.v[e].y);
        const double2 s = make_double2(kzv * h1.v[e].x - kxv * h3.v[e].x, kzv * h1.v[e].y - kxv * h3.v[e].y);
        h1.v[e] = make_double2(-s.y, s.x);
    }
    col_store<E>(A.fn + off, h2, nyp);
    col_store<E>(A.gn + off, h1, nyp);
    col_store<E>(A.omz + off, h3, nyp);
    if (A.scalar) col_store<E>(A.scn + off, sc, nyp);
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
int kmm_fast_x(kmm_ctx *ctx, const double2 *q, double2 *r, int ic, int nout, bool save_uvw, double *up3,
               double *vp3, double *wp3);
int kmm_fast_x2(kmm_ctx *ctx, const void *q, void *r, const void *tw, bool fp32, int ic, int nout, bool save_uvw,
                double *up3, double *vp3, double *wp3);
int kmm_tracers(kmm_ctx *ctx);

// the fused path applies when: no polymer, no immersed boundary, Dirichlet-type velocity walls
// (nb = nt = 1 or 2), nyp in the compiled register layouts, and the x transform instance exists
bool kmm_fused_applicable(const kmm_ctx *ctx) {
    if (ctx->p.polymer_on || ctx->f[KMM_IMATRIX] != NULL) return false;
    // the flow-rate correction sits between the v and the u, w column kernels, which only the
    // blocked kernels (ny = 32, 64, 96, 128) launch separately
    const bool blocked = ctx->use_colblk && (ctx->ny == 32 || ctx->ny == 64 || ctx->ny == 96 || ctx->ny == 128);
    if (ctx->p.flow_rate > 0.0 && !blocked) return false;
    if (ctx->p.scalar_on && ctx->p.scl_flag >= 2) return false;
    if (ctx->p.particle_flag > 0 && ctx->p.npart > 0) return false;   // inertial particles: routine vcw3dp
    const int E = (ctx->nyp + 31) / 32;
    if (!(E == 2 || E == 3 || E == 4 || E == 5 || E == 9)) return false;
    const int Ex = (ctx->mx + 31) / 32;
    if (!(Ex == 1 || Ex == 2 || Ex == 3 || Ex == 5 || Ex == 6 || Ex == 9 || Ex == 12)) return false;
    return true;
}


int kmm_tracers_enqueue(kmm_ctx *ctx, cudaStream_t st);

int kmm_fused_step(kmm_ctx *ctx) {
    RET(kmm_fused_enqueue(ctx));
    return kmm_fused_finish(ctx);
}

// ---------------------------------------------------------------------------
// CUDA-graph replay of the fused step.  kmm_fused_launch swaps the history buffers (FN/FNM1,
// GN/GNM1, SCN/SCNM1) on the host after enqueueing a step, so consecutive steps use one of two
// pointer arrangements; one graph is captured per arrangement.  Capturing runs the host code of
// a step without executing it on the device, so the step counter is restored after each capture
// and two captures leave the arrangement where it started.
// ---------------------------------------------------------------------------
void kmm_graph_release(kmm_ctx *ctx) {
    if (!ctx->graph_ready) return;
    cudaStreamSynchronize(ctx->stream);
    for (int p = 0; p < 2; ++p) {
        if (ctx->gexec[p]) cudaGraphExecDestroy(ctx->gexec[p]);
        if (ctx->ggraph[p]) cudaGraphDestroy(ctx->ggraph[p]);
        ctx->gexec[p] = NULL;
        ctx->ggraph[p] = NULL;
    }
    ctx->graph_ready = 0;
    ctx->ggen = kmm_graph_generation();
}

static void swap_history(kmm_ctx *ctx) {
    void *t;
    t = ctx->f[KMM_FN]; ctx->f[KMM_FN] = ctx->f[KMM_FNM1]; ctx->f[KMM_FNM1] = t;
    t = ctx->f[KMM_GN]; ctx->f[KMM_GN] = ctx->f[KMM_GNM1]; ctx->f[KMM_GNM1] = t;
    if (ctx->p.scalar_on) { t = ctx->f[KMM_SCN]; ctx->f[KMM_SCN] = ctx->f[KMM_SCNM1]; ctx->f[KMM_SCNM1] = t; }
}

static int capture_graphs(kmm_ctx *ctx) {
    static const int hist[6] = {KMM_FN, KMM_FNM1, KMM_GN, KMM_GNM1, KMM_SCN, KMM_SCNM1};
    void *saved[6];
    for (int h = 0; h < 6; ++h) saved[h] = ctx->f[hist[h]];
    const int it0 = ctx->it;
    ctx->g_fn0 = ctx->f[KMM_FN];
    for (int p = 0; p < 2; ++p) {
        cudaGraph_t g = NULL;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        int st = KMM_OK;
        const long long l0 = ctx->launches;
        if (e == cudaSuccess) {
            st = kmm_fused_launch(ctx);
            e = cudaStreamEndCapture(ctx->stream, &g);
        }
        ctx->gkernels[p] = ctx->launches - l0;
        ctx->launches = l0;
        if (e == cudaSuccess && st == KMM_OK) e = cudaGraphInstantiate(&ctx->gexec[p], g, 0);
        ctx->ggraph[p] = g;   // kept: an ensemble step adds it to its parent graph as a child
        if (e != cudaSuccess || st != KMM_OK) {
            for (int h = 0; h < 6; ++h) ctx->f[hist[h]] = saved[h];
            ctx->it = it0;
            for (int q = 0; q < 2; ++q) {
                if (ctx->gexec[q]) { cudaGraphExecDestroy(ctx->gexec[q]); ctx->gexec[q] = NULL; }
                if (ctx->ggraph[q]) { cudaGraphDestroy(ctx->ggraph[q]); ctx->ggraph[q] = NULL; }
            }
            cudaGetLastError();
            kmm_set_error(ctx, "graph capture of the fused step failed (%s)", cudaGetErrorString(e));
            return st != KMM_OK ? st : KMM_ERR_CUDA;
        }
    }
    ctx->it = it0;          // captured, not executed
    ctx->graph_ready = 1;   // the two captured swaps restored arrangement 0
    ctx->ggen = kmm_graph_generation();
    return KMM_OK;
}

// the graph a replayed fused step of this context would launch now (capturing it first), or -1
// when the step is not replayed from a graph; *parity receives the arrangement
int kmm_fused_graph_for_step(kmm_ctx *ctx, int *parity) {
    const bool graphable = ctx->use_fused && kmm_fused_applicable(ctx) && ctx->use_graph && !ctx->timing_on &&
                           ctx->fused != NULL && ctx->it >= ctx->p.irstrt;
    if (!graphable) return -1;
    if (!ctx->graph_ready) RET(capture_graphs(ctx));
    *parity = ctx->f[KMM_FN] == ctx->g_fn0 ? 0 : 1;
    return KMM_OK;
}

// after an ensemble graph replayed this member's step: the host side of kmm_fused_enqueue
void kmm_fused_replayed(kmm_ctx *ctx, int parity) {
    ctx->launches += ctx->gkernels[parity];
    swap_history(ctx);
    ctx->it += 1;
}

int kmm_fused_enqueue(kmm_ctx *ctx) {
    // graphs only after the step that initialises the tracers (it == irstrt) and the tau tables
    const bool graphable = ctx->use_graph && !ctx->timing_on && ctx->fused != NULL && ctx->it >= ctx->p.irstrt;
    if (!graphable) return kmm_fused_launch(ctx);
    if (!ctx->graph_ready) RET(capture_graphs(ctx));
    const int parity = ctx->f[KMM_FN] == ctx->g_fn0 ? 0 : 1;
    CK(cudaGraphLaunch(ctx->gexec[parity], ctx->stream));
    ctx->launches += ctx->gkernels[parity];
    swap_history(ctx);
    ctx->it += 1;
    return KMM_OK;
}

int kmm_fused_launch(kmm_ctx *ctx) {
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mz = ctx->mz;
    const size_t ncols = (size_t)nz * nxh;
    const int scalar = ctx->p.scalar_on ? 1 : 0;
    const int nbase = scalar ? 8 : 6, nq = scalar ? 9 : 6, nout = scalar ? 4 : 3;
    RET(build_tables(ctx));
    KmmFused *FU = ctx->fused;
    double2 *g_yp = FU->yp, *g_q = FU->q, *g_r = FU->r, *g_yo = FU->yo;
    (void)nbase;
    // the mixed-precision form (FP32 transforms and products, FP64 solves) has compiled kernels
    // for ny, nx, nz in {32, 64, 96, 128} (nx, nz: the 3/2 lengths 48 .. 192)
    const bool f32 = ctx->p.precision == 1;
    const bool ct_mz = (mz == 48 || mz == 96 || mz == 144 || mz == 192);
    const bool ct_mx = (ctx->mx == 48 || ctx->mx == 96 || ctx->mx == 144 || ctx->mx == 192);
    const bool ct_y = (ctx->ny == 32 || ctx->ny == 64 || ctx->ny == 96 || ctx->ny == 128);
    if (f32 && !(ct_mz && ct_mx && ct_y && ctx->use_colblk)) {
        kmm_set_error(ctx, "mixed precision needs nx, ny, nz in {32, 64, 96, 128} and the blocked column kernels");
        return KMM_ERR_UNSUPPORTED;
    }
    ctx->it += 1;

    // history copies fnm1 = fn, gnm1 = gn, scnm1 = scn become pointer swaps: the kernels read the
    // old n / n-1 fields and the new n fields are written into the swapped-out buffers
    void *fn_old = kmm_field_ptr(ctx, KMM_FN), *fnm1_old = kmm_field_ptr(ctx, KMM_FNM1);
    void *gn_old = kmm_field_ptr(ctx, KMM_GN), *gnm1_old = kmm_field_ptr(ctx, KMM_GNM1);
    void *sn_old = scalar ? kmm_field_ptr(ctx, KMM_SCN) : NULL, *snm1_old = scalar ? kmm_field_ptr(ctx, KMM_SCNM1) : NULL;
    ColFwdArgs F;
    memset(&F, 0, sizeof(F));
    F.v = SPEC(ctx, KMM_V); F.omy = SPEC(ctx, KMM_OMY);
    F.fn = (double2 *)fn_old; F.fnm1 = (double2 *)fnm1_old; F.gn = (double2 *)gn_old; F.gnm1 = (double2 *)gnm1_old;
    F.scal = scalar ? SPEC(ctx, KMM_SCALAR) : NULL; F.scn = (double2 *)sn_old; F.scnm1 = (double2 *)snm1_old;
    F.gf1 = SPEC(ctx, KMM_GF1); F.gf2 = SPEC(ctx, KMM_GF2);
    F.dnv1b = SPEC(ctx, KMM_DNV1B); F.dnv1t = SPEC(ctx, KMM_DNV1T); F.dnv2b = SPEC(ctx, KMM_DNV2B);
    F.dnv2t = SPEC(ctx, KMM_DNV2T); F.denom = SPEC(ctx, KMM_DENOM);
    F.u0 = REAL(ctx, KMM_U0); F.w0 = REAL(ctx, KMM_W0); F.h1n = REAL(ctx, KMM_H1N); F.h1nm1 = REAL(ctx, KMM_H1NM1);
    F.h3n = REAL(ctx, KMM_H3N); F.h3nm1 = REAL(ctx, KMM_H3NM1); F.scratch = ctx->d_scratch;
    F.yp = g_yp; F.wavx = ctx->d_wavx; F.wavz = ctx->d_wavz;
    F.nz = nz; F.nxh = nxh; F.nyp = nyp; F.nzh = ctx->nzh; F.scalar = scalar; F.nb = ctx->nb; F.nt = ctx->nt;
    F.re = ctx->re; F.dt = ctx->dt; F.th = ctx->theta; F.dyde = ctx->dyde; F.diff = ctx->p.diff; F.c0 = ctx->h_c[0];
    F.atu = ctx->atu; F.btu = ctx->btu; F.gtu = ctx->gtu; F.abu = ctx->abu; F.bbu = ctx->bbu; F.gbu = ctx->gbu;
    F.atw = ctx->atw; F.gtw = ctx->gtw; F.abw = ctx->abw; F.bbw = ctx->bbw; F.gbw = ctx->gbw;
    const int E = (nyp + 31) / 32;
    const size_t smc = sizeof(double2) * (64 * (size_t)E + 2 * 2 * 2 * (size_t)ctx->ny);
    const int nblk = (int)(ncols / 2);
    kmm_tic(ctx);
    int cst = ctx->use_colblk ? kmm_colblk_fwd(ctx, F, FU->btabs, FU->brj, f32 ? (const void *)FU->twf_y2 : (const void *)ctx->wy2.tw, f32)
                              : KMM_ERR_UNSUPPORTED;
    if (cst != KMM_OK && cst != KMM_ERR_UNSUPPORTED) return cst;
    if (cst == KMM_ERR_UNSUPPORTED) {
#define COLF(EE, LL)                                                                                  \
    do {                                                                                              \
        RET(kmm_smem_attr(ctx, (const void *)k_col_fwd<EE, LL>, smc));                                \
        k_col_fwd<EE, LL><<<nblk, 64, smc, ctx->stream>>>(F, FU->tabs, ctx->wy2);                       \
    } while (0)
    switch (2 * ctx->ny) {   // specialised lengths: ny = 32, 64, 96, 128
    case 64: COLF(2, 64); break;
    case 128: COLF(3, 128); break;
    case 192: COLF(4, 192); break;
    case 256: COLF(5, 256); break;
    default:
        switch (E) {
        case 2: COLF(2, 0); break;
        case 3: COLF(3, 0); break;
        case 4: COLF(4, 0); break;
        case 5: COLF(5, 0); break;
        case 9: COLF(9, 0); break;
        default: return KMM_ERR_UNSUPPORTED;
        }
    }
#undef COLF
    CKL();
    }
    kmm_toc(ctx, KMM_STAGE_COLUMN);
    // swap the history buffers: FNM1 <- old FN (read above), FN will receive the new terms
    ctx->f[KMM_FNM1] = fn_old; ctx->f[KMM_FN] = fnm1_old;
    ctx->f[KMM_GNM1] = gn_old; ctx->f[KMM_GN] = gnm1_old;
    if (scalar) { ctx->f[KMM_SCNM1] = sn_old; ctx->f[KMM_SCN] = snm1_old; }

    // z inverse transforms
    CK(cudaMemsetAsync(ctx->d_cfl, 0, sizeof(double) * nyp, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_umax, 0, sizeof(double) * nyp, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    const size_t smz = sizeof(double2) * ((size_t)ZT_WARPS * 2 * mz + (size_t)ZT_Y * mz * ZT_KX);
    const size_t smzf = sizeof(double2) * ((size_t)ZT_WARPS * 2 * mz + (size_t)ZT_KX * nz * ZT_Y);
    const dim3 gz((nxh + ZT_KX - 1) / ZT_KX, (nyp + ZT_Y - 1) / ZT_Y);
    kmm_tic(ctx);
#define ZB2(MM, CC)                                                                                   \
    do {                                                                                              \
        RET(kmm_smem_attr(ctx, (const void *)k_zb2<MM, CC>, smz));                                    \
        k_zb2<MM, CC><<<gz, ZT_WARPS * 32, smz, ctx->stream>>>((const CC *)g_yp, (CC *)g_q, ctx->d_wavx, \
                                                             ctx->d_wavz, (const CC *)twz, nq, nyp, nxh); \
    } while (0)
    const void *twz = f32 ? (const void *)FU->twf_mz : (const void *)ctx->wmz.tw;
    if (!f32 && kmm_ztma_supported(ctx)) {
        RET(kmm_zb_tma(ctx, g_yp, g_q, scalar ? 8 : 6, nq, (const double2 *)twz));
    } else if (f32 && kmm_ztma_supported(ctx)) {
        RET(kmm_zb_tma32(ctx, (const float2 *)g_yp, (float2 *)g_q, scalar ? 8 : 6, nq, (const float2 *)twz));
    } else if (f32) {
        switch (mz) {
        case 48: ZB2(48, float2); break;
        case 96: ZB2(96, float2); break;
        case 144: ZB2(144, float2); break;
        default: ZB2(192, float2); break;
        }
    } else {
        switch (mz) {   // specialised lengths: nz = 32, 64, 96, 128
        case 48: ZB2(48, double2); break;
        case 96: ZB2(96, double2); break;
        case 144: ZB2(144, double2); break;
        case 192: ZB2(192, double2); break;
        default:
            RET(kmm_smem_attr(ctx, (const void *)k_zb<0>, smz));
            k_zb<0><<<gz, ZT_WARPS * 32, smz, ctx->stream>>>(g_yp, g_q, ctx->d_wavx, ctx->d_wavz, ctx->wmz, nq, nyp, nz,
                                                           nxh, mz);
            break;
        }
    }
#undef ZB2
    CKL();
    kmm_toc(ctx, KMM_STAGE_ZFFT_BWD);
    // x transforms + products
    double *up3 = NULL, *vp3 = NULL, *wp3 = NULL;
    if (ctx->p.npart > 0) { up3 = REAL(ctx, KMM_UP3D); vp3 = REAL(ctx, KMM_VP3D); wp3 = REAL(ctx, KMM_WP3D); }
    kmm_tic(ctx);
    {
        const int xst = kmm_fast_x2(ctx, g_q, g_r, f32 ? (const void *)FU->twf_mx : (const void *)ctx->wmx.tw, f32,
                                    scalar ? 6 : -1, nout, ctx->p.npart > 0, up3, vp3, wp3);
        if (xst == KMM_ERR_UNSUPPORTED) RET(kmm_fast_x(ctx, g_q, g_r, scalar ? 6 : -1, nout, ctx->p.npart > 0, up3, vp3, wp3));
        else RET(xst);
    }
    kmm_toc(ctx, KMM_STAGE_XPHYS);
    // tracers (solvers.f90:3463-3476) on the side stream: they read only the particles and the
    // 3/2-grid u, v, w just written, so they overlap the z-forward and back stages (kept in line
    // while the stages are being timed)
    const bool tracers_forked = ctx->p.npart > 0 && !ctx->timing_on;
    if (tracers_forked) {
        CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
        CK(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
        RET(kmm_tracers_enqueue(ctx, ctx->side));
    }
    // z forward transforms
    kmm_tic(ctx);
#define ZF2(MM, CC)                                                                                   \
    do {                                                                                              \
        RET(kmm_smem_attr(ctx, (const void *)k_zf2<MM, CC>, smzf));                                   \
        k_zf2<MM, CC><<<gz, ZT_WARPS * 32, smzf, ctx->stream>>>((const CC *)g_r, (CC *)g_yo, (const CC *)twz, \
                                                              nout, nyp, nxh, (double)ctx->mx * (double)mz); \
    } while (0)
    if (!f32 && kmm_ztma_supported(ctx)) {
        RET(kmm_zf_tma(ctx, g_r, g_yo, nout, (const double2 *)twz));
    } else if (f32 && kmm_ztma_supported(ctx)) {
        RET(kmm_zf_tma32(ctx, (const float2 *)g_r, (float2 *)g_yo, nout, (const float2 *)twz));
    } else if (f32) {
        switch (mz) {
        case 48: ZF2(48, float2); break;
        case 96: ZF2(96, float2); break;
        case 144: ZF2(144, float2); break;
        default: ZF2(192, float2); break;
        }
    } else {
        switch (mz) {
        case 48: ZF2(48, double2); break;
        case 96: ZF2(96, double2); break;
        case 144: ZF2(144, double2); break;
        case 192: ZF2(192, double2); break;
        default:
            RET(kmm_smem_attr(ctx, (const void *)k_zf<0>, smzf));
            k_zf<0><<<gz, ZT_WARPS * 32, smzf, ctx->stream>>>(g_r, g_yo, ctx->wmz, nout, nyp, nz, nxh, mz,
                                                            (double)ctx->mx * (double)mz);
            break;
        }
    }
#undef ZF2
    CKL();
    kmm_toc(ctx, KMM_STAGE_ZFFT_FWD);
    // back to Chebyshev space, norm, filter, nonlin
    ColBwdArgs B;
    B.yo = g_yo; B.fn = SPEC(ctx, KMM_FN); B.gn = SPEC(ctx, KMM_GN); B.omz = SPEC(ctx, KMM_OMZ);
    B.scn = scalar ? SPEC(ctx, KMM_SCN) : NULL; B.h1n = REAL(ctx, KMM_H1N); B.h3n = REAL(ctx, KMM_H3N);
    B.wavx = ctx->d_wavx; B.wavz = ctx->d_wavz; B.nz = nz; B.nxh = nxh; B.nyp = nyp; B.nzh = ctx->nzh;
    B.scalar = scalar; B.dyde = ctx->dyde;
    kmm_tic(ctx);
    cst = ctx->use_colblk ? kmm_colblk_bwd(ctx, B, f32 ? (const void *)FU->twf_y2 : (const void *)ctx->wy2.tw, f32)
                          : KMM_ERR_UNSUPPORTED;
    if (cst != KMM_OK && cst != KMM_ERR_UNSUPPORTED) return cst;
    if (cst == KMM_ERR_UNSUPPORTED) {
#define COLB(EE, LL)                                                                                  \
    do {                                                                                              \
        RET(kmm_smem_attr(ctx, (const void *)k_col_bwd<EE, LL>, smc));                                \
        k_col_bwd<EE, LL><<<nblk, 64, smc, ctx->stream>>>(B, ctx->wy2);                                \
    } while (0)
    switch (2 * ctx->ny) {
    case 64: COLB(2, 64); break;
    case 128: COLB(3, 128); break;
    case 192: COLB(4, 192); break;
    case 256: COLB(5, 256); break;
    default:
        switch (E) {
        case 2: COLB(2, 0); break;
        case 3: COLB(3, 0); break;
        case 4: COLB(4, 0); break;
        case 5: COLB(5, 0); break;
        case 9: COLB(9, 0); break;
        default: return KMM_ERR_UNSUPPORTED;
        }
    }
#undef COLB
    CKL();
    }
    kmm_toc(ctx, KMM_STAGE_POST);
    if (tracers_forked) {
        CK(cudaEventRecord(ctx->join_ev, ctx->side));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0));
    } else {
        RET(kmm_tracers_enqueue(ctx, ctx->stream));
    }
    // the CFL maxima and the tracer status go to pinned host memory for kmm_fused_finish
    // (solvers.f90:3497-3514)
    double *h_cfl = ctx->h_pin, *h_um = ctx->h_pin + KMM_MAX_NYP;
    CK(cudaMemcpyAsync(h_cfl, ctx->d_cfl, sizeof(double) * nyp, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(h_um, ctx->d_umax, sizeof(double) * nyp, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(kmm_h_pin_status(ctx), ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    return KMM_OK;
}

int kmm_fused_finish(kmm_ctx *ctx) {
    const int nyp = ctx->nyp;
    CK(cudaStreamSynchronize(ctx->stream));
    const double *h_cfl = ctx->h_pin, *h_um = ctx->h_pin + KMM_MAX_NYP;
    int st = KMM_OK;
    if (ctx->p.npart > 0 && *kmm_h_pin_status(ctx)) {
        kmm_set_error(ctx, "particle interpolation cell index out of range (part_track.f90:580-590)");
        st = KMM_ERR_INTERP;
    }
    double cflmax = 0.0, umax = 0.0;
    bool nan = false;
    for (int i = 0; i < nyp; ++i) {
        if (h_cfl[i] != h_cfl[i]) nan = true;
        else if (h_cfl[i] > cflmax) cflmax = h_cfl[i];
        if (h_um[i] > umax) umax = h_um[i];
    }
    ctx->stats.cflmax = nan ? NAN : cflmax;
    ctx->stats.umax = umax;
    if (st == KMM_OK && nan) st = KMM_ERR_NAN;
    if (st == KMM_OK && cflmax > 1.0) st = KMM_ERR_CFL;
    ctx->stats.status = st;
    return st;
}
