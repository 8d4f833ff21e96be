/*
 * kmm_oracle.c -- CPU restatement of the reference KMM timestep (TEST INFRASTRUCTURE ONLY).
 *
 * Loaded only by tests/, the smoke check and bench.py's CPU legs; never by the
 * product.  See kmm_oracle.h for scope and parity status ("parity unpinned"
 * against the Fortran binary, pinned by mathematical known answers).
 *
 * Reference paths below are relative to FFTW_DNS/code/src/dns/ of
 * ryankellybp11/Polymer_DNS.  Arrays keep the reference's Fortran layout
 * (column major, y fastest); indices in comments are the reference's 1-based
 * ones, code is 0-based.
 */
#include "kmm_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------------- */
/* FFT: mixed-radix Stockham, FFTW sign conventions (sign -1 forward).      */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n, nf, fac[40];
    cplx *tw; /* tw[m] = exp(-2 pi i m / n) */
} fftplan;

static int fft_factor(int n, int *fac)
{
    int nf = 0;
    static const int rads[4] = {4, 2, 3, 5};
    for (int r = 0; r < 4; ++r)
        while (n % rads[r] == 0) { fac[nf++] = rads[r]; n /= rads[r]; }
    return n == 1 ? nf : -1;
}

static int plan_init(fftplan *p, int n)
{
    p->n = n;
    p->nf = fft_factor(n, p->fac);
    if (p->nf < 0 && n != 1) return -1;
    if (n == 1) p->nf = 0;
    p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    for (int m = 0; m < n; ++m) {
        long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        p->tw[m] = (double)cosl(a) - I * (double)sinl(a);
    }
    return 0;
}

static void plan_free(fftplan *p) { free(p->tw); p->tw = NULL; }

/* in-place on x, scratch y (length n); sign -1: exp(-2 pi i jk/n), +1: exp(+...) */
static void fft_exec(const fftplan *p, cplx *x, cplx *y, int sign)
{
    const int n = p->n;
    cplx *src = x, *dst = y;
    int Ns = 1;
    const double s3 = 0.86602540378443864676 * (double)sign;
    const double c5a = 0.30901699437494742410, c5b = -0.80901699437494742410;
    const double s5a = 0.95105651629515357212 * (double)sign, s5b = 0.58778525229247312917 * (double)sign;
    for (int f = 0; f < p->nf; ++f) {
        const int R = p->fac[f];
        const int nR = n / R;
        const int tstep = n / (Ns * R);
        for (int j = 0; j < nR; ++j) {
            const int k = j % Ns;
            cplx v[5];
            for (int r = 0; r < R; ++r) {
                cplx a = src[j + r * nR];
                if (r && k) {
                    cplx w = p->tw[(size_t)((long)r * k * tstep % n)];
                    if (sign > 0) w = conj(w);
                    a *= w;
                }
                v[r] = a;
            }
            cplx o[5];
            if (R == 2) {
                o[0] = v[0] + v[1];
                o[1] = v[0] - v[1];
            } else if (R == 3) {
                cplx t1 = v[1] + v[2];
                cplx t2 = v[0] - 0.5 * t1;
                cplx t3 = s3 * (v[1] - v[2]);
                o[0] = v[0] + t1;
                o[1] = t2 + I * t3;
                o[2] = t2 - I * t3;
            } else if (R == 4) {
                cplx a0 = v[0] + v[2], a1 = v[0] - v[2];
                cplx b0 = v[1] + v[3], b1 = (double)sign * I * (v[1] - v[3]);
                o[0] = a0 + b0;
                o[1] = a1 + b1;
                o[2] = a0 - b0;
                o[3] = a1 - b1;
            } else { /* R == 5 */
                cplx t1 = v[1] + v[4], t2 = v[2] + v[3];
                cplx t3 = v[1] - v[4], t4 = v[2] - v[3];
                o[0] = v[0] + t1 + t2;
                cplx r1 = v[0] + c5a * t1 + c5b * t2;
                cplx r2 = v[0] + c5b * t1 + c5a * t2;
                cplx i1 = I * (s5a * t3 + s5b * t4);
                cplx i2 = I * (s5b * t3 - s5a * t4);
                o[1] = r1 + i1;
                o[4] = r1 - i1;
                o[2] = r2 + i2;
                o[3] = r2 - i2;
            }
            const int idxD = (j / Ns) * Ns * R + k;
            for (int q = 0; q < R; ++q) dst[idxD + q * Ns] = o[q];
        }
        cplx *t = src; src = dst; dst = t;
        Ns *= R;
    }
    if (src != x) memcpy(x, src, sizeof(cplx) * (size_t)n);
}

/* REDFT00 (DCT-I) of a complex column of length nn = N+1, via the even extension of length 2N */
static void dct1_c(const fftplan *p2, const cplx *x, cplx *out, cplx *w1, cplx *w2)
{
    const int N = p2->n / 2;
    for (int i = 0; i <= N; ++i) w1[i] = x[i];
    for (int i = 1; i < N; ++i) w1[2 * N - i] = x[i];
    fft_exec(p2, w1, w2, -1);
    for (int k = 0; k <= N; ++k) out[k] = w1[k];
}

/* c2r of two Hermitian rows at once: a, b have n/2+1 entries; outputs length n.
 * FFTW's c2r ignores the imaginary parts of the k=0 and k=n/2 entries. */
static void c2r_pair(const fftplan *p, const cplx *a, const cplx *b, double *ra, double *rb, cplx *w1, cplx *w2)
{
    const int n = p->n, h = n / 2;
    for (int k = 0; k <= h; ++k) {
        cplx A = a[k], B = b ? b[k] : 0.0;
        if (k == 0 || k == h) { A = creal(A); B = creal(B); }
        w1[k] = A + I * B;
        if (k > 0 && k < h) w1[n - k] = conj(A) + I * conj(B);
    }
    fft_exec(p, w1, w2, +1);
    for (int m = 0; m < n; ++m) {
        ra[m] = creal(w1[m]);
        if (rb) rb[m] = cimag(w1[m]);
    }
}

/* r2c of two real rows at once; outputs n/2+1 entries each */
static void r2c_pair(const fftplan *p, const double *ra, const double *rb, cplx *a, cplx *b, cplx *w1, cplx *w2)
{
    const int n = p->n, h = n / 2;
    for (int m = 0; m < n; ++m) w1[m] = ra[m] + I * (rb ? rb[m] : 0.0);
    fft_exec(p, w1, w2, -1);
    for (int k = 0; k <= h; ++k) {
        cplx Z = w1[k], Zc = conj(w1[(n - k) % n]);
        a[k] = 0.5 * (Z + Zc);
        if (b) b[k] = -0.5 * I * (Z - Zc);
    }
}

/* ------------------------------------------------------------------------- */
/* context                                                                    */
/* ------------------------------------------------------------------------- */
#define MAXF 800

struct orc_ctx {
    kmm_params p;
    int nx, ny, nz, nyp, nym, nxh, nyh, nzh, nyhp, nyhm, mx, mz;
    double re, dt, theta, gain, ugain, dyde, alpha, beta, dPdx, xl, yl, zl, uinf, pi;
    double atu, btu, gtu, abu, bbu, gbu, atw, btw, gtw, abw, bbw, gbw;
    int nt, nb;
    double p1t, p1b, p2t, p2b;
    double *wavx, *wavz, *c, *ycoord, *seght;
    double fspread[10][10]; /* fspread(j,i) -> fspread[i-1][j-1] */
    int kmaxsurf;
    int it;
    int substep;
    double umax1; /* part_track's saved running max of the particle relative velocity */
    void *fld[MAXF];
    kmm_stats stats;
    fftplan py2, pmz, pmx, pnx, pnz; /* 2*ny (DCT), mz, mx, nx, nz */
    double *cfl;
    double *scsource; /* the KMM_SCSOURCE field's storage */
    int frate_ready;                    /* constant flow rate: W and G built */
    double frate_w[1025], frate_g[1025];
    int ntarg;                          /* scl_flag = 4: the targets of the last source, 3 ints each */
    int targ[3 * 1023];
};

#define SIDX(C, i, j, k) ((((size_t)(k)) * (size_t)(C)->nz + (size_t)(j)) * (size_t)(C)->nyp + (size_t)(i))
#define PIDX(C, i, j, k) ((((size_t)(k)) * (size_t)(C)->mz + (size_t)(j)) * (size_t)(C)->nyp + (size_t)(i))
#define WIDX(C, j, k) (((size_t)(k)) * (size_t)(C)->nz + (size_t)(j))

int orc_field_size(orc_ctx *c, int f, size_t *nelem, int *eb)
{
    size_t n = 0;
    int b = 0;
    if (f >= 0 && f < KMM_U0) { n = (size_t)c->nyp * c->nz * c->nxh; b = 16; } /* ids past KMM_NSPECTRAL: private scratch */
    else if (f >= KMM_U0 && f < KMM_NMEAN_END) { n = (size_t)c->nyp; b = 8; }
    else if (f >= KMM_BCTOP && f < KMM_NWALL_END) { n = (size_t)c->nz * c->nxh; b = 16; }
    else if (f >= KMM_FXINTG && f < KMM_NPHYS_END) { n = (size_t)c->nyp * c->mz * c->mx; b = 8; }
    else if (f == KMM_IMATRIX) { n = (size_t)c->nyp * c->mz * c->mx; b = 4; }
    else if (f >= KMM_XPART && f < KMM_NPART_END) { n = (size_t)(c->p.npart > 0 ? c->p.npart : 0); b = 8; }
    else if (f >= KMM_INITU && f < KMM_NINIT_END) { n = (size_t)c->nyp * c->nz * c->nx; b = 8; }
    if (nelem) *nelem = n;
    if (eb) *eb = b;
    return b ? KMM_OK : KMM_ERR_ARG;
}

void *orc_field(orc_ctx *c, int f)
{
    size_t n;
    int b;
    if (f < 0 || f >= MAXF || orc_field_size(c, f, &n, &b) != KMM_OK) return NULL;
    if (!c->fld[f]) c->fld[f] = calloc(n ? n : 1, (size_t)b);
    return c->fld[f];
}

static cplx *SF(orc_ctx *c, int f) { return (cplx *)orc_field(c, f); }
static double *RF(orc_ctx *c, int f) { return (double *)orc_field(c, f); }

int orc_copy(orc_ctx *c, int dst, int src)
{
    size_t n1, n2;
    int b1, b2;
    if (orc_field_size(c, dst, &n1, &b1) || orc_field_size(c, src, &n2, &b2) || n1 != n2 || b1 != b2) return KMM_ERR_ARG;
    memcpy(orc_field(c, dst), orc_field(c, src), n1 * (size_t)b1);
    return KMM_OK;
}

int orc_zero(orc_ctx *c, int f)
{
    size_t n;
    int b;
    if (orc_field_size(c, f, &n, &b)) return KMM_ERR_ARG;
    memset(orc_field(c, f), 0, n * (size_t)b);
    return KMM_OK;
}

int orc_set_it(orc_ctx *c, int it) { c->it = it; return KMM_OK; }
int orc_get_stats(orc_ctx *c, kmm_stats *s) { c->stats.it = c->it; *s = c->stats; return KMM_OK; }
double orc_dpdx(orc_ctx *c) { return c->dPdx; }

/* OpenMP threads of the parallel loops (n <= 0: all host cores); returns the count in effect */
int orc_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* setbcs, main_dns.f90:1175-1418 */
static void setbcs(orc_ctx *c)
{
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
    default: /* 0, 5, 10: shear-free */
        c->atu = 0; c->btu = 1; c->gtu = 0; c->atw = 0; c->btw = 1; c->gtw = 0;
        c->abu = 0; c->bbu = 1; c->gbu = 0; c->abw = 0; c->bbw = 1; c->gbw = 0;
        c->nt = 2; c->nb = 2; break;
    }
    c->p1b = 1.0; c->p1t = -1.0; c->p2b = -1.0; c->p2t = 0.5;
}

int orc_ctx_create(const kmm_params *p, orc_ctx **out)
{
    if (!p || !out) return KMM_ERR_ARG;
    if (p->nx < 4 || p->ny < 8 || p->nz < 4 || p->nx % 2 || p->ny % 2 || p->nz % 4 != 0) return KMM_ERR_ARG;
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    c->p = *p;
    c->nx = p->nx; c->ny = p->ny; c->nz = p->nz;
    c->nyp = c->ny + 1; c->nym = c->ny - 1; c->nxh = c->nx / 2; c->nyh = c->ny / 2; c->nzh = c->nz / 2;
    c->nyhp = c->nyh + 1; c->nyhm = c->nyh - 1; c->mx = 3 * c->nx / 2; c->mz = 3 * c->nz / 2;
    c->re = p->re; c->dt = p->dt; c->theta = p->theta; c->gain = p->gain; c->ugain = p->ugain;
    c->xl = p->xl; c->yl = p->yl; c->zl = p->zl; c->uinf = p->uinf;
    c->pi = 2.0 * acos(0.0);
    /* setstuff, main_dns.f90:1112-1165 */
    c->ycoord = (double *)calloc((size_t)c->nyp, sizeof(double));
    c->seght = (double *)calloc((size_t)c->nyp, sizeof(double));
    c->ycoord[0] = c->yl / 2.0;
    for (int k = 2; k <= c->nyp; ++k) {
        c->ycoord[k - 1] = cos((double)(k - 1) * c->pi / (double)c->ny) * (c->yl / 2.0);
        c->seght[k - 1] = fabs(c->ycoord[k - 1] - c->ycoord[k - 2]);
    }
    c->seght[0] = c->seght[c->nyp - 1];
    c->alpha = 2.0 * c->pi / c->xl;
    c->beta = 2.0 * c->pi / c->zl;
    c->wavx = (double *)calloc((size_t)c->nxh, sizeof(double));
    c->wavz = (double *)calloc((size_t)c->nz, sizeof(double));
    for (int k = 1; k <= c->nxh; ++k) c->wavx[k - 1] = (double)(k - 1) * c->alpha;
    for (int j = 1; j <= c->nzh; ++j) c->wavz[j - 1] = (double)(j - 1) * c->beta;
    for (int j = c->nzh + 1; j <= c->nz; ++j) c->wavz[j - 1] = (double)(j - c->nz - 1) * c->beta;
    c->c = (double *)calloc((size_t)c->nyp, sizeof(double));
    for (int i = 0; i < c->nyp; ++i) c->c[i] = 1.0;
    c->c[0] = 2.0; c->c[c->nyp - 1] = 2.0;
    c->dyde = 2.0 / c->yl;
    setbcs(c);
    /* init_flow.f90:117 (channel): dPdx = -2/yl (2 R_tau/(yl re))^2 */
    c->dPdx = -2.0 / c->yl * pow(2.0 * p->r_tau / (c->yl * c->re), 2);
    c->stats.dpdx = c->dPdx;
    /* forcepre: force-spreading matrix, main_dns.f90:1551-1558 */
    for (int i = 1; i <= 10; ++i)
        for (int j = 1; j <= 10; ++j) {
            double dsq = (double)((i - 1) * (i - 1)) + (double)((j - 1) * (j - 1));
            c->fspread[i - 1][j - 1] = dsq < 13 ? exp(-2.0 * dsq) : 0.0;
        }
    c->kmaxsurf = 0;
    /* substep_check, part_track.f90:296-356 */
    {
        double Pi_f = 1.0 / (p->ratio + 0.5), tau;
        if (p->cd_switch == 0) tau = 1.0;
        else if (p->cd_switch == 1) tau = c->re * p->ap * p->ap / (6.0 * Pi_f);
        else tau = 2.0 * c->re * p->ap * p->ap / (9.0 * Pi_f);
        double s = 2.0 * c->dt / tau;
        c->substep = (int)ceil(s > 1.0 ? s : 1.0);
    }
    if (plan_init(&c->py2, 2 * c->ny) || plan_init(&c->pmz, c->mz) || plan_init(&c->pmx, c->mx) ||
        plan_init(&c->pnx, c->nx) || plan_init(&c->pnz, c->nz)) {
        orc_ctx_destroy(c);
        return KMM_ERR_ARG;
    }
    c->cfl = (double *)calloc((size_t)c->nyp, sizeof(double));
    *out = c;
    return KMM_OK;
}

void orc_ctx_destroy(orc_ctx *c)
{
    if (!c) return;
    for (int f = 0; f < MAXF; ++f) free(c->fld[f]);
    free(c->wavx); free(c->wavz); free(c->c); free(c->ycoord); free(c->seght); free(c->cfl);
    plan_free(&c->py2); plan_free(&c->pmz); plan_free(&c->pmx); plan_free(&c->pnx); plan_free(&c->pnz);
    free(c);
}

/* kmaxsurf from imatrix, forcepre main_dns.f90:1524-1535 */
static void update_kmaxsurf(orc_ctx *c)
{
    int *im = (int *)orc_field(c, KMM_IMATRIX);
    int km = 0;
    for (int k = 1; k <= c->mx; ++k)
        for (int j = 1; j <= c->mz; ++j)
            for (int i = 1; i <= c->nyp; ++i) {
                int t = im[PIDX(c, i - 1, j - 1, k - 1)];
                if (t == 1 || t == 3 || t == 4)
                    if (k >= km) km = k;
            }
    c->kmaxsurf = km;
}

/* ------------------------------------------------------------------------- */
/* standalone transforms                                                      */
/* ------------------------------------------------------------------------- */
int orc_dct1(int n, const double *in, double *out)
{
    fftplan p;
    if (n < 2 || plan_init(&p, 2 * (n - 1))) return KMM_ERR_ARG;
    cplx *x = malloc(sizeof(cplx) * n), *o = malloc(sizeof(cplx) * n);
    cplx *w1 = malloc(sizeof(cplx) * 2 * (n - 1)), *w2 = malloc(sizeof(cplx) * 2 * (n - 1));
    for (int i = 0; i < n; ++i) x[i] = in[i];
    dct1_c(&p, x, o, w1, w2);
    for (int i = 0; i < n; ++i) out[i] = creal(o[i]);
    free(x); free(o); free(w1); free(w2); plan_free(&p);
    return KMM_OK;
}

int orc_fft(int n, const double *in, double *out, int sign)
{
    fftplan p;
    if (plan_init(&p, n)) return KMM_ERR_ARG;
    cplx *x = malloc(sizeof(cplx) * n), *w = malloc(sizeof(cplx) * n);
    memcpy(x, in, sizeof(cplx) * n);
    fft_exec(&p, x, w, sign < 0 ? -1 : 1);
    memcpy(out, x, sizeof(cplx) * n);
    free(x); free(w); plan_free(&p);
    return KMM_OK;
}

int orc_rfft(int n, const double *in, double *out)
{
    fftplan p;
    if (n % 2 || plan_init(&p, n)) return KMM_ERR_ARG;
    cplx *w1 = malloc(sizeof(cplx) * n), *w2 = malloc(sizeof(cplx) * n);
    r2c_pair(&p, in, NULL, (cplx *)out, NULL, w1, w2);
    free(w1); free(w2); plan_free(&p);
    return KMM_OK;
}

int orc_irfft(int n, const double *in, double *out)
{
    fftplan p;
    if (n % 2 || plan_init(&p, n)) return KMM_ERR_ARG;
    cplx *w1 = malloc(sizeof(cplx) * n), *w2 = malloc(sizeof(cplx) * n);
    c2r_pair(&p, (const cplx *)in, NULL, out, NULL, w1, w2);
    free(w1); free(w2); plan_free(&p);
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* derivatives.f90                                                            */
/* ------------------------------------------------------------------------- */
/* cderiv(f,df), derivatives.f90:258-314 */
static void cderiv_arr(const orc_ctx *c, const cplx *f, cplx *df)
{
    const int nyp = c->nyp, ny = c->ny, nym = c->nym;
    const double dyde = c->dyde;
#pragma omp parallel for schedule(static)
    for (int col = 0; col < c->nz * c->nxh; ++col) {
        const cplx *fc = f + (size_t)col * nyp;
        cplx *d = df + (size_t)col * nyp;
        d[nyp - 1] = 0.0;                                    /* df(nyp) = 0                 */
        d[ny - 1] = 2.0 * (double)ny * fc[nyp - 1] * dyde;   /* df(ny) = 2 ny f(nyp) dyde   */
        for (int i = nym; i >= 1; --i)                       /* df(i) = df(i+2) + 2 i f(i+1) dyde */
            d[i - 1] = d[i + 1] + 2.0 * (double)i * fc[i] * dyde;
        d[0] = 0.5 * d[0];
    }
}

int orc_cderiv(orc_ctx *c, int f, int df)
{
    if (f == df) return KMM_ERR_ARG;
    cderiv_arr(c, SF(c, f), SF(c, df));
    return KMM_OK;
}

/* cderiv1d(f,df), derivatives.f90:657-704 */
static void cderiv1d(const orc_ctx *c, const double *f, double *df)
{
    const int nyp = c->nyp, ny = c->ny;
    df[nyp - 1] = 0.0;
    df[ny - 1] = 2.0 * (double)ny * f[nyp - 1] * c->dyde;
    for (int i = c->nym; i >= 1; --i) df[i - 1] = df[i + 1] + 2.0 * (double)i * f[i] * c->dyde;
    df[0] = 0.5 * df[0];
}

/* c{0,1,2}der{b,t}w(wrkc,wrk1,iy), derivatives.f90:318-653 */
static void wallderiv_arr(const orc_ctx *c, const cplx *f, int order, int wall, cplx *out, int iy)
{
    const int nyp = c->nyp;
    const double dyde = c->dyde;
    for (int col = 0; col < c->nz * c->nxh; ++col) {
        const cplx *fc = f + (size_t)col * nyp;
        cplx acc = 0.0;
        double sgn = (wall == 0) ? (order == 0 ? -1.0 : 1.0) : 1.0;
        for (int i = 1; i <= nyp; ++i) {
            double rp = (double)(i - 1);
            if (wall == 0) sgn = -sgn;
            if (order == 0) acc = acc + sgn * fc[i - 1];
            else if (order == 1) acc = acc + rp * rp * sgn * fc[i - 1] * dyde;
            else {
                double rp2 = rp * rp;
                acc = acc + (rp2 - 1.0) * rp2 * sgn * fc[i - 1] * dyde * dyde / 3.0;
            }
        }
        out[(size_t)col * nyp + (iy - 1)] = acc;
    }
}

int orc_wallderiv(orc_ctx *c, int f, int order, int wall, int out, int iy)
{
    if (order < 0 || order > 2 || wall < 0 || wall > 1 || iy < 1 || iy > c->nyp) return KMM_ERR_ARG;
    wallderiv_arr(c, SF(c, f), order, wall, SF(c, out), iy);
    return KMM_OK;
}

/* gradv, derivatives.f90:6-86 */
int orc_gradv(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->nz * c->nxh;
    cplx *u = SF(c, KMM_U), *v = SF(c, KMM_V), *w = SF(c, KMM_W);
    cplx *w1 = malloc(sizeof(cplx) * n), *w2 = malloc(sizeof(cplx) * n), *w3 = malloc(sizeof(cplx) * n);
    cplx *u11 = SF(c, KMM_U11), *u12 = SF(c, KMM_U12), *u13 = SF(c, KMM_U13);
    cplx *u21 = SF(c, KMM_U21), *u22 = SF(c, KMM_U22), *u23 = SF(c, KMM_U23);
    cplx *u31 = SF(c, KMM_U31), *u32 = SF(c, KMM_U32), *u33 = SF(c, KMM_U33);
    cplx *Lu = SF(c, KMM_LU), *Lv = SF(c, KMM_LV), *Lw = SF(c, KMM_LW);
    cderiv_arr(c, u, u12); cderiv_arr(c, v, u22); cderiv_arr(c, w, u32);
    cderiv_arr(c, u12, w1); cderiv_arr(c, u22, w2); cderiv_arr(c, u32, w3);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j) {
            double wn2 = c->wavx[k] * c->wavx[k] + c->wavz[j] * c->wavz[j];
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                u11[x] = I * c->wavx[k] * u[x];
                u21[x] = I * c->wavx[k] * v[x];
                u31[x] = I * c->wavx[k] * w[x];
                u13[x] = I * c->wavz[j] * u[x];
                u23[x] = I * c->wavz[j] * v[x];
                u33[x] = I * c->wavz[j] * w[x];
                Lu[x] = w1[x] - wn2 * u[x];
                Lv[x] = w2[x] - wn2 * v[x];
                Lw[x] = w3[x] - wn2 * w[x];
            }
        }
    free(w1); free(w2); free(w3);
    return KMM_OK;
}

/* gradscl, derivatives.f90:90-144 */
int orc_gradscl(orc_ctx *c)
{
    cplx *s = SF(c, KMM_SCALAR), *sx = SF(c, KMM_SCLX), *sy = SF(c, KMM_SCLY), *sz = SF(c, KMM_SCLZ);
    cderiv_arr(c, s, sy);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j)
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                sx[x] = I * c->wavx[k] * s[x];
                sz[x] = I * c->wavz[j] * s[x];
            }
    return KMM_OK;
}

/* derivscji, derivatives.f90:148-254: dcIJK = d c_IJ / d x_K */
int orc_derivscji(orc_ctx *c)
{
    for (int ij = 0; ij < 9; ++ij) {
        cplx *cf = SF(c, KMM_C11 + ij);
        cplx *dx = SF(c, KMM_DC111 + 3 * ij), *dy = SF(c, KMM_DC111 + 3 * ij + 1), *dz = SF(c, KMM_DC111 + 3 * ij + 2);
        cderiv_arr(c, cf, dy);
#pragma omp parallel for collapse(2)
        for (int k = 0; k < c->nxh; ++k)
            for (int j = 0; j < c->nz; ++j)
                for (int i = 0; i < c->nyp; ++i) {
                    size_t x = SIDX(c, i, j, k);
                    dx[x] = I * c->wavx[k] * cf[x];
                    dz[x] = I * c->wavz[j] * cf[x];
                }
    }
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* solvers.f90: Dirichlet / Neumann tau solver `solve`                        */
/* ------------------------------------------------------------------------- */
/* a(nyhp,nz,3) -> A[(l)*(nyhp*nz) + k*nyhp + i], 0-based i,k, l = 0..2 */
#define AIDX(C, i, k, l) ((size_t)(l) * (size_t)(C)->nyhp * (size_t)(C)->nz + (size_t)(k) * (size_t)(C)->nyhp + (size_t)(i))

/* evnc, solvers.f90:324-352 */
static void evnc(const orc_ctx *c, double *a, const double *wn, double dyde)
{
    for (int i = 1; i <= c->nyh; ++i) {
        int j = 2 * i;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        double rj2 = 1.0 / (double)(2 * (j * j - 1));
        double rj3 = 1.0 / (double)(4 * j * (j + 1));
        for (int k = 0; k < c->nz; ++k) {
            a[AIDX(c, i - 1, k, 0)] = wn[k] * rj1;
            a[AIDX(c, i - 1, k, 1)] = -1.0 * dyde * dyde - wn[k] * rj2;
            a[AIDX(c, i - 1, k, 2)] = wn[k] * rj3;
        }
    }
    for (int k = 0; k < c->nz; ++k) {
        a[AIDX(c, 0, k, 0)] = 2.0 * a[AIDX(c, 0, k, 0)];
        a[AIDX(c, c->nyhm - 1, k, 2)] = 0.0;
        a[AIDX(c, c->nyh - 1, k, 1)] = -1.0 * dyde * dyde;
        a[AIDX(c, c->nyh - 1, k, 2)] = 0.0;
    }
}

/* oddc, solvers.f90:354-383 */
static void oddc(const orc_ctx *c, double *a, const double *wn, double dyde)
{
    for (int i = 1; i <= c->nyhm; ++i) {
        int j = 2 * i + 1;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        double rj2 = 1.0 / (double)(2 * (j * j - 1));
        double rj3 = 1.0 / (double)(4 * j * (j + 1));
        for (int k = 0; k < c->nz; ++k) {
            a[AIDX(c, i - 1, k, 0)] = wn[k] * rj1;
            a[AIDX(c, i - 1, k, 1)] = -1.0 * dyde * dyde - wn[k] * rj2;
            a[AIDX(c, i - 1, k, 2)] = wn[k] * rj3;
        }
    }
    for (int k = 0; k < c->nz; ++k) {
        a[AIDX(c, c->nyhm - 2, k, 2)] = 0.0;
        a[AIDX(c, c->nyhm - 1, k, 1)] = -1.0 * dyde * dyde;
        a[AIDX(c, c->nyhm - 1, k, 2)] = 0.0;
    }
}

/* s(0:ny,nz) view of a slab u(nyp,nz): s(j,k) = u[k*nyp + j] */
#define S0(u, j, k) (u)[(size_t)(k) * nyp + (size_t)(j)]
/* wrk(nyp,nz) 1-based view */
#define W1(w, i, k) (w)[(size_t)(k) * nyp + (size_t)((i) - 1)]

/* evns / pntevns RHS rows 2..nyhp (solvers.f90:387-448, 807-850) */
static void evns_rows(const orc_ctx *c, const cplx *s, cplx *wrk)
{
    const int nyp = c->nyp, ny = c->ny;
    for (int i = 2; i <= c->nyhm; ++i) {
        int j = 2 * i - 2, jp2 = j + 2, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        double rj2 = 1.0 / (double)(2 * (j * j - 1));
        double rj3 = 1.0 / (double)(4 * j * (j + 1));
        for (int k = 0; k < c->nz; ++k)
            W1(wrk, i, k) = -c->c[jm2] * S0(s, jm2, k) * rj1 + S0(s, j, k) * rj2 - S0(s, jp2, k) * rj3;
    }
    {
        int j = ny - 2, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        double rj2 = 1.0 / (double)(2 * (j * j - 1));
        for (int k = 0; k < c->nz; ++k) W1(wrk, c->nyh, k) = -S0(s, jm2, k) * rj1 + S0(s, j, k) * rj2;
    }
    {
        int j = ny, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        for (int k = 0; k < c->nz; ++k) W1(wrk, c->nyhp, k) = -S0(s, jm2, k) * rj1;
    }
}

/* odds / pntodds RHS rows 2..nyh (solvers.f90:450-496, 852-902) */
static void odds_rows(const orc_ctx *c, const cplx *s, cplx *wrk)
{
    const int nyp = c->nyp, ny = c->ny;
    for (int i = 2; i <= c->nyhm - 1; ++i) {
        int j = 2 * i - 1, jp2 = j + 2, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        double rj2 = 1.0 / (double)(2 * (j * j - 1));
        double rj3 = 1.0 / (double)(4 * j * (j + 1));
        for (int k = 0; k < c->nz; ++k)
            W1(wrk, i, k) = -S0(s, jm2, k) * rj1 + S0(s, j, k) * rj2 - S0(s, jp2, k) * rj3;
    }
    {
        int i = c->nyhm, j = ny - 3, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        double rj2 = 1.0 / (double)(2 * (j * j - 1));
        for (int k = 0; k < c->nz; ++k) W1(wrk, i, k) = -S0(s, jm2, k) * rj1 + S0(s, j, k) * rj2;
    }
    {
        int i = c->nyh, j = ny - 1, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1));
        for (int k = 0; k < c->nz; ++k) W1(wrk, i, k) = -S0(s, jm2, k) * rj1;
    }
}

/* eqsolve(a,t,wrk,nrank), solvers.f90:500-553 */
static void eqsolve(const orc_ctx *c, const double *a, const double *t, cplx *wrk, int nrank, double *d, double *f)
{
    const int nyp = c->nyp, nz = c->nz;
    const int m = nrank - 1, mm1 = m - 1;
#define A(i, k, l) a[AIDX(c, (i) - 1, k, (l) - 1)]
#define D(i, k) d[(size_t)(k) * nyp + (size_t)((i) - 1)]
    for (int k = 0; k < nz; ++k) D(m, k) = A(m, k, 2);
    for (int i = mm1; i >= 1; --i)
        for (int k = 0; k < nz; ++k) {
            D(i, k) = A(i, k, 2) - A(i, k, 3) * A(i + 1, k, 1) / D(i + 1, k);
            W1(wrk, i + 1, k) = W1(wrk, i + 1, k) - A(i, k, 3) * W1(wrk, i + 2, k) / D(i + 1, k);
        }
    for (int k = 0; k < nz; ++k) {
        f[k] = t[m - 1] - t[nrank - 1] * A(m, k, 1) / D(m, k);
        W1(wrk, 1, k) = W1(wrk, 1, k) - t[nrank - 1] * W1(wrk, nrank, k) / D(m, k);
    }
    for (int i = mm1; i >= 1; --i)
        for (int k = 0; k < nz; ++k) {
            W1(wrk, 1, k) = W1(wrk, 1, k) - f[k] * W1(wrk, i + 1, k) / D(i, k);
            f[k] = t[i - 1] - f[k] * A(i, k, 1) / D(i, k);
        }
    for (int k = 0; k < nz; ++k) W1(wrk, 1, k) = W1(wrk, 1, k) / f[k];
    for (int i = 2; i <= nrank; ++i)
        for (int k = 0; k < nz; ++k) W1(wrk, i, k) = (W1(wrk, i, k) - A(i - 1, k, 1) * W1(wrk, i - 1, k)) / D(i - 1, k);
#undef A
#undef D
}

/* solve(u,x,g,dyde,bctop,bcbot,ib,a,wrkc) on one kx slab, solvers.f90:174-283 */
static void solve_slab(const orc_ctx *c, cplx *u, double x, double g, const cplx *bctop, const cplx *bcbot, int ib)
{
    const int nyp = c->nyp, nz = c->nz;
    double *t = calloc((size_t)nyp, sizeof(double)), *wn = calloc((size_t)nz, sizeof(double));
    double *a = calloc((size_t)3 * c->nyhp * nz, sizeof(double));
    double *d = calloc((size_t)nyp * nz, sizeof(double)), *f = calloc((size_t)nz, sizeof(double));
    cplx *wrk = calloc((size_t)nyp * nz, sizeof(cplx));
    if (ib == 0)
        for (int j = 0; j < nyp; ++j) t[j] = 1.0; /* dircbc */
    for (int k = 0; k < nz; ++k) wn[k] = c->wavz[k] * c->wavz[k] + x + g;
    int kzero = -1;
    if (ib != 0)
        for (int k = 0; k < nz; ++k)
            if (wn[k] <= 1.0e-20) { kzero = k; wn[k] = 1.0; }
    /* even problem */
    int nrank = c->nyhp;
    evnc(c, a, wn, c->dyde);
    evns_rows(c, u, wrk);
    for (int k = 0; k < nz; ++k) W1(wrk, 1, k) = (ib == 0) ? 0.5 * (bctop[k] + bcbot[k]) : 0.5 * (bctop[k] - bcbot[k]);
    if (ib != 0)
        for (int j = 1; j <= nrank; ++j) t[j - 1] = c->dyde * (double)((2 * (j - 1)) * (2 * (j - 1))); /* neumbc ip=0 */
    eqsolve(c, a, t, wrk, nrank, d, f);
    for (int j = 1; j <= nyp; j += 2) {
        int i = (j + 1) / 2;
        for (int k = 0; k < nz; ++k) u[(size_t)k * nyp + (j - 1)] = W1(wrk, i, k);
    }
    /* odd problem */
    nrank = c->nyh;
    oddc(c, a, wn, c->dyde);
    odds_rows(c, u, wrk);
    for (int k = 0; k < nz; ++k) W1(wrk, 1, k) = (ib == 0) ? 0.5 * (bctop[k] - bcbot[k]) : 0.5 * (bctop[k] + bcbot[k]);
    if (ib != 0)
        for (int j = 1; j <= nrank; ++j) t[j - 1] = c->dyde * (double)((2 * (j - 1) + 1) * (2 * (j - 1) + 1)); /* neumbc ip=1 */
    eqsolve(c, a, t, wrk, nrank, d, f);
    for (int j = 2; j <= c->ny; j += 2) {
        int i = j / 2;
        for (int k = 0; k < nz; ++k) u[(size_t)k * nyp + (j - 1)] = W1(wrk, i, k);
    }
    if (ib != 0 && kzero >= 0)
        for (int j = 0; j < nyp; ++j) u[(size_t)kzero * nyp + j] = 0.0;
    free(t); free(wn); free(a); free(d); free(f); free(wrk);
}

int orc_solve(orc_ctx *c, int uf, double g, int ib)
{
    cplx *u = SF(c, uf), *bt = SF(c, KMM_BCTOP), *bb = SF(c, KMM_BCBOT);
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < c->nxh; ++k)
        solve_slab(c, u + (size_t)k * c->nz * c->nyp, c->wavx[k] * c->wavx[k], g, bt + (size_t)k * c->nz,
                   bb + (size_t)k * c->nz, ib);
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* solvers.f90: Robin tau solver `penta`                                      */
/* ------------------------------------------------------------------------- */
typedef struct { /* the `save`d state of pntsolve, solvers.f90:915-918 */
    cplx *gs;   /* (nyhp,nz,2) */
    double *cs, *ds; /* (nyhp,nz,2) */
    cplx *s;    /* (2,nz) */
    double *f;  /* (2,nz,2) */
} pnt_state;

#define GS(st, i, k, ip) (st)->gs[((size_t)((ip) - 1) * nz + (size_t)(k)) * nyhp + (size_t)((i) - 1)]
#define CS(st, i, k, ip) (st)->cs[((size_t)((ip) - 1) * nz + (size_t)(k)) * nyhp + (size_t)((i) - 1)]
#define DS(st, i, k, ip) (st)->ds[((size_t)((ip) - 1) * nz + (size_t)(k)) * nyhp + (size_t)((i) - 1)]
#define SS(st, js, k) (st)->s[(size_t)(k) * 2 + (size_t)((js) - 1)]
#define FF(st, js, k, ip) (st)->f[((size_t)((ip) - 1) * nz + (size_t)(k)) * 2 + (size_t)((js) - 1)]

/* fillt(nrank,ip,ipass,t), solvers.f90:1021-1061 */
static void fillt(int nrank, int ip, int ipass, const double *tt, const double *tb, double *t)
{
    for (int j = 1; j <= nrank; ++j) {
        int k = (ip == 1) ? 2 * j - 1 : 2 * j;
        t[j - 1] = (ipass == 1) ? tb[k - 1] : tt[k - 1];
    }
}

/* pntsolve(a,t,wrk,gtop,gbot,ip,nrank), solvers.f90:906-1017 */
static void pntsolve(const orc_ctx *c, const double *a, double *t, cplx *wrk, const cplx *gtop, const cplx *gbot,
                     int ip, int nrank, const double *tt, const double *tb, pnt_state *st)
{
    const int nyp = c->nyp, nz = c->nz, nyhp = c->nyhp;
#define A(i, k, l) a[AIDX(c, (i) - 1, k, (l) - 1)]
    int ipass = 1;
    if (ip == 1)
        for (int k = 0; k < nz; ++k) { SS(st, 1, k) = gtop[k]; SS(st, 2, k) = gbot[k]; }
    int js = 2;
    const int n = nrank, m = n - 1, mm1 = m - 1;
    for (int i = 1; i <= m; ++i)
        for (int k = 0; k < nz; ++k) { GS(st, i, k, ip) = W1(wrk, i, k); CS(st, i, k, ip) = A(i, k, 1); }
    for (int k = 0; k < nz; ++k) { DS(st, m, k, ip) = A(m, k, 2); GS(st, n, k, ip) = W1(wrk, n, k); }
    for (int i = mm1; i >= 1; --i)
        for (int k = 0; k < nz; ++k) {
            DS(st, i, k, ip) = A(i, k, 2) - A(i, k, 3) * CS(st, i + 1, k, ip) / DS(st, i + 1, k, ip);
            GS(st, i + 1, k, ip) = GS(st, i + 1, k, ip) - A(i, k, 3) * GS(st, i + 2, k, ip) / DS(st, i + 1, k, ip);
        }
    for (;;) {
        fillt(n, ip, ipass, tt, tb, t);
        for (int k = 0; k < nz; ++k) {
            FF(st, js, k, ip) = t[m - 1] - t[n - 1] * CS(st, m, k, ip) / DS(st, m, k, ip);
            SS(st, js, k) = SS(st, js, k) - t[n - 1] * GS(st, n, k, ip) / DS(st, m, k, ip);
        }
        for (int i = mm1; i >= 1; --i)
            for (int k = 0; k < nz; ++k) {
                SS(st, js, k) = SS(st, js, k) - FF(st, js, k, ip) * GS(st, i + 1, k, ip) / DS(st, i, k, ip);
                FF(st, js, k, ip) = t[i - 1] - FF(st, js, k, ip) * CS(st, i, k, ip) / DS(st, i, k, ip);
            }
        if (ipass == 1) { ipass = 2; js = 1; continue; }
        break;
    }
    if (ip == 2 && ipass == 2) {
        for (int k = 0; k < nz; ++k) {
            double det = FF(st, 1, k, 1) * FF(st, 2, k, 2) - FF(st, 2, k, 1) * FF(st, 1, k, 2);
            W1(wrk, 1, k) = (SS(st, 1, k) * FF(st, 2, k, 2) - SS(st, 2, k) * FF(st, 1, k, 2)) / det;
            W1(wrk, 2, k) = (SS(st, 2, k) * FF(st, 1, k, 1) - SS(st, 1, k) * FF(st, 2, k, 1)) / det;
            for (int i = 2; i <= n + 1; ++i) {
                int ii = 2 * i - 1;
                W1(wrk, ii, k) = (GS(st, i, k, 1) - CS(st, i - 1, k, 1) * W1(wrk, ii - 2, k)) / DS(st, i - 1, k, 1);
            }
            for (int i = 2; i <= n; ++i) {
                int ii = 2 * i;
                W1(wrk, ii, k) = (GS(st, i, k, 2) - CS(st, i - 1, k, 2) * W1(wrk, ii - 2, k)) / DS(st, i - 1, k, 2);
            }
        }
    }
#undef A
}

/* penta(u,x,g,dyde,ib,at,bt,gtop,ab,bb,gbot,a,wrkc) on one kx slab, solvers.f90:680-773 */
static void penta_slab(const orc_ctx *c, cplx *u, double x, double g, int ib, double at, double bt,
                       const cplx *gtop, double ab, double bb, const cplx *gbot)
{
    const int nyp = c->nyp, nz = c->nz, nyhp = c->nyhp;
    double *tt = calloc((size_t)nyp, sizeof(double)), *tb = calloc((size_t)nyp, sizeof(double));
    /* mixedbc, solvers.f90:777-803 */
    for (int j = 1; j <= nyp; ++j) {
        int j1 = j - 1;
        tt[j - 1] = at + c->dyde * bt * (double)(j1 * j1);
        tb[j - 1] = ab + c->dyde * bb * (double)(j1 * j1);
    }
    for (int j = 2; j <= nyp; j += 2) tb[j - 1] = -tb[j - 1];
    double *wn = calloc((size_t)nz, sizeof(double)), *t = calloc((size_t)nyp, sizeof(double));
    double *a = calloc((size_t)3 * nyhp * nz, sizeof(double));
    cplx *wrk = calloc((size_t)nyp * nz, sizeof(cplx));
    pnt_state st;
    st.gs = calloc((size_t)nyhp * nz * 2, sizeof(cplx));
    st.cs = calloc((size_t)nyhp * nz * 2, sizeof(double));
    st.ds = calloc((size_t)nyhp * nz * 2, sizeof(double));
    st.s = calloc((size_t)2 * nz, sizeof(cplx));
    st.f = calloc((size_t)4 * nz, sizeof(double));
    for (int k = 0; k < nz; ++k) wn[k] = c->wavz[k] * c->wavz[k] + x + g;
    int kzero = -1;
    if (ib != 0)
        for (int k = 0; k < nz; ++k)
            if (wn[k] <= 1.0e-20) { kzero = k; wn[k] = 1.0; }
    evnc(c, a, wn, c->dyde);
    evns_rows(c, u, wrk); /* pntevns */
    pntsolve(c, a, t, wrk, gtop, gbot, 1, c->nyhp, tt, tb, &st);
    oddc(c, a, wn, c->dyde);
    odds_rows(c, u, wrk); /* pntodds */
    pntsolve(c, a, t, wrk, gtop, gbot, 2, c->nyh, tt, tb, &st);
    for (int k = 0; k < nz; ++k)
        for (int j = 1; j <= nyp; ++j) u[(size_t)k * nyp + (j - 1)] = W1(wrk, j, k);
    if (ib != 0 && kzero >= 0)
        for (int j = 0; j < nyp; ++j) u[(size_t)kzero * nyp + j] = 0.0;
    free(tt); free(tb); free(wn); free(t); free(a); free(wrk);
    free(st.gs); free(st.cs); free(st.ds); free(st.s); free(st.f);
}

int orc_penta(orc_ctx *c, int uf, double g, int ib, double at, double bt, double ab, double bb)
{
    cplx *u = SF(c, uf), *gt = SF(c, KMM_BCTOP), *gb = SF(c, KMM_BCBOT);
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < c->nxh; ++k)
        penta_slab(c, u + (size_t)k * c->nz * c->nyp, c->wavx[k] * c->wavx[k], g, ib, at, bt, gt + (size_t)k * c->nz, ab,
                   bb, gb + (size_t)k * c->nz);
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* solvers.f90: mean modes `uzero` / psolve1d                                 */
/* ------------------------------------------------------------------------- */
/* p1dsolve(a,t,wrk,gamt,gamb,ip,nrank), solvers.f90:1400-1493 (state saved across the two calls) */
typedef struct { double cs[2][1024], ds[2][1024], gs[2][1024], f[2][2], s[2]; } p1d_state;

static void p1dsolve(const double a[][3], double *t, double *wrk, double gamt, double gamb, int ip, int nrank,
                     const double *tt, const double *tb, p1d_state *st)
{
#define PCS(i, ipp) st->cs[(ipp) - 1][(i) - 1]
#define PDS(i, ipp) st->ds[(ipp) - 1][(i) - 1]
#define PGS(i, ipp) st->gs[(ipp) - 1][(i) - 1]
#define PA(i, l) a[(i) - 1][(l) - 1]
    int ipass = 1;
    if (ip == 1) { st->s[0] = gamt; st->s[1] = gamb; }
    int js = 2;
    int n = nrank, m = n - 1, mm1 = m - 1;
    for (int i = 1; i <= m; ++i) { PGS(i, ip) = wrk[i - 1]; PCS(i, ip) = PA(i, 1); }
    PDS(m, ip) = PA(m, 2);
    PGS(n, ip) = wrk[n - 1];
    for (int i = mm1; i >= 1; --i) {
        PDS(i, ip) = PA(i, 2) - PA(i, 3) * PCS(i + 1, ip) / PDS(i + 1, ip);
        PGS(i + 1, ip) = PGS(i + 1, ip) - PA(i, 3) * PGS(i + 2, ip) / PDS(i + 1, ip);
    }
    for (;;) {
        fillt(n, ip, ipass, tt, tb, t);
        st->f[js - 1][ip - 1] = t[m - 1] - t[n - 1] * PCS(m, ip) / PDS(m, ip);
        st->s[js - 1] = st->s[js - 1] - t[n - 1] * PGS(n, ip) / PDS(m, ip);
        for (int i = mm1; i >= 1; --i) {
            st->s[js - 1] = st->s[js - 1] - st->f[js - 1][ip - 1] * PGS(i + 1, ip) / PDS(i, ip);
            st->f[js - 1][ip - 1] = t[i - 1] - st->f[js - 1][ip - 1] * PCS(i, ip) / PDS(i, ip);
        }
        if (ipass == 1) { ipass = 2; js = 1; continue; }
        break;
    }
    if (ip == 2 && ipass == 2) {
        double (*f)[2] = st->f;
        double det = f[0][0] * f[1][1] - f[1][0] * f[0][1];
        wrk[0] = (st->s[0] * f[1][1] - st->s[1] * f[0][1]) / det;
        wrk[1] = (st->s[1] * f[0][0] - st->s[0] * f[1][0]) / det;
        n = n + 1;
        for (int i = 2; i <= n; ++i) {
            int ii = 2 * i - 1;
            wrk[ii - 1] = (PGS(i, 1) - PCS(i - 1, 1) * wrk[ii - 3]) / PDS(i - 1, 1);
        }
        n = n - 1;
        for (int i = 2; i <= n; ++i) {
            int ii = 2 * i;
            wrk[ii - 1] = (PGS(i, 2) - PCS(i - 1, 2) * wrk[ii - 3]) / PDS(i - 1, 2);
        }
    }
#undef PCS
#undef PDS
#undef PGS
#undef PA
}

/* psolve1d(u,g,dyde,at,bt,gtop,ab,bb,gbot,t), solvers.f90:1180-1245 */
static void psolve1d(const orc_ctx *c, double *u, double g, double dyde, double at, double bt, double gtop, double ab,
                     double bb, double gbot)
{
    const int nyp = c->nyp, ny = c->ny;
    double tt[1025], tb[1025], t[1025], wrk[1025], a[1025][3];
    double x = 0.0;
    /* mixedbc1d, solvers.f90:1249-1269 (note the minus sign in tb) */
    for (int j = 1; j <= nyp; ++j) {
        int j1 = j - 1;
        tt[j - 1] = at + dyde * bt * (double)(j1 * j1);
        tb[j - 1] = ab - dyde * bb * (double)(j1 * j1);
    }
    for (int j = 2; j <= nyp; j += 2) tb[j - 1] = -tb[j - 1];
    p1d_state st;
    memset(&st, 0, sizeof(st));
    double wn = c->wavz[0] * c->wavz[0] + x + g;
    /* p1devnc, solvers.f90:1273-1297 */
    for (int i = 1; i <= c->nyh; ++i) {
        int j = 2 * i;
        double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1)), rj3 = 1.0 / (double)(4 * j * (j + 1));
        a[i - 1][0] = wn * rj1;
        a[i - 1][1] = -1.0 * dyde * dyde - wn * rj2;
        a[i - 1][2] = wn * rj3;
    }
    a[0][0] = 2.0 * a[0][0];
    a[c->nyhm - 1][2] = 0.0;
    a[c->nyh - 1][1] = -1.0 * dyde * dyde;
    a[c->nyh - 1][2] = 0.0;
    /* p1devns, solvers.f90:1327-1358 */
    for (int i = 2; i <= c->nyhm; ++i) {
        int j = 2 * i - 2, jp2 = j + 2, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1)), rj3 = 1.0 / (double)(4 * j * (j + 1));
        wrk[i - 1] = -c->c[jm2] * u[jm2] * rj1 + u[j] * rj2 - u[jp2] * rj3;
    }
    {
        int j = ny - 2, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1));
        wrk[c->nyh - 1] = -u[jm2] * rj1 + u[j] * rj2;
        j = ny; jm2 = j - 2;
        rj1 = 1.0 / (double)(4 * j * (j - 1));
        wrk[c->nyhp - 1] = -u[jm2] * rj1;
    }
    p1dsolve((const double(*)[3])a, t, wrk, gtop, gbot, 1, c->nyhp, tt, tb, &st);
    /* p1doddc, solvers.f90:1300-1323 */
    for (int i = 1; i <= c->nyhm; ++i) {
        int j = 2 * i + 1;
        double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1)), rj3 = 1.0 / (double)(4 * j * (j + 1));
        a[i - 1][0] = wn * rj1;
        a[i - 1][1] = -1.0 * dyde * dyde - wn * rj2;
        a[i - 1][2] = wn * rj3;
    }
    a[c->nyhm - 2][2] = 0.0;
    a[c->nyhm - 1][1] = -1.0 * dyde * dyde;
    a[c->nyhm - 1][2] = 0.0;
    /* p1dodds, solvers.f90:1361-1397 */
    for (int i = 2; i <= c->nyhm - 1; ++i) {
        int j = 2 * i - 1, jp2 = j + 2, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1)), rj3 = 1.0 / (double)(4 * j * (j + 1));
        wrk[i - 1] = -u[jm2] * rj1 + u[j] * rj2 - u[jp2] * rj3;
    }
    {
        int i = c->nyhm, j = ny - 3, jm2 = j - 2;
        double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1));
        wrk[i - 1] = -u[jm2] * rj1 + u[j] * rj2;
        i = c->nyh; j = ny - 1; jm2 = j - 2;
        rj1 = 1.0 / (double)(4 * j * (j - 1));
        wrk[i - 1] = -u[jm2] * rj1;
    }
    p1dsolve((const double(*)[3])a, t, wrk, gtop, gbot, 2, c->nyh, tt, tb, &st);
    for (int j = 0; j < nyp; ++j) u[j] = wrk[j];
}

/* uzero(u0,h1,h1l,uflag), solvers.f90:1065-1176 */
/* uzero on explicit arrays (u0 in / out, h1 = h_n, h1l = h_(n-1)) */
static void uzero_arrays(orc_ctx *c, int uflag, double *u0, const double *h1, const double *h1l)
{
    double wrk1[1025], t[1025];
    const double re = c->re, dt = c->dt, th = c->theta;
    for (int i = 0; i < c->nyp; ++i) wrk1[i] = -re * u0[i] / (dt * th) - re * (3.0 * h1[i] - h1l[i]) / (2.0 * th);
    if (th > 0.99) {
        for (int i = 0; i < c->nyp; ++i) u0[i] = wrk1[i];
    } else {
        cderiv1d(c, u0, t);
        cderiv1d(c, t, u0);
        for (int i = 0; i < c->nyp; ++i) u0[i] = wrk1[i] - (1.0 - th) * u0[i] / th;
    }
    double g = re / (th * dt);
    if (uflag == 1) psolve1d(c, u0, g, c->dyde, c->atu, c->btu, c->gtu, c->abu, c->bbu, c->gbu);
    else psolve1d(c, u0, g, c->dyde, c->atw, c->btu, c->gtw, c->abw, c->bbw, c->gbw); /* btu: as the reference passes */
}

int orc_uzero(orc_ctx *c, int uflag)
{
    if (c->nyp > 1024) return KMM_ERR_ARG;
    uzero_arrays(c, uflag, RF(c, uflag == 1 ? KMM_U0 : KMM_W0), RF(c, uflag == 1 ? KMM_H1N : KMM_H3N),
                 RF(c, uflag == 1 ? KMM_H1NM1 : KMM_H3NM1));
    return KMM_OK;
}

/* Constant flow rate (kmm_params.flow_rate > 0; no counterpart in the reference, which holds dPdx
 * constant, init_flow.f90:117, solvers.f90:3044-3045).  The bulk velocity is the trapezoid of
 * writeoutputs (helpers.f90:1355-1359) over the Gauss-Lobatto points of the mean profile
 * u(y_i) = sum_n u0_n cos(n pi i / ny), i.e. Q = sum_n W_n u0_n with
 * W_n = (1/yl) sum_i (cos(n pi i/ny) + cos(n pi (i+1)/ny)) / 2 |y_(i+1) - y_i|.  G is the response of
 * the u0 step (uzero) to a unit uniform acceleration over one step with homogeneous walls: the
 * solve with h_n = h_(n-1) = T_0 from u0 = 0, less the solve with zero forcing (which carries the
 * wall values).  After each u0 solve, delta = (flow_rate - Q) / (W . G) and u0 += delta G: the step
 * was driven by the mean pressure gradient dPdx - delta. */
static void frate_setup(orc_ctx *c)
{
    const int nyp = c->nyp, ny = c->ny;
    for (int n = 0; n < nyp; ++n) {
        double w = 0.0;
        for (int i = 0; i < ny; ++i)
            w += 1.0 / c->yl * 0.5 * (cos((double)n * c->pi * (double)(i + 1) / (double)ny) +
                                      cos((double)n * c->pi * (double)i / (double)ny)) *
                 fabs(c->ycoord[i + 1] - c->ycoord[i]);
        c->frate_w[n] = w;
    }
    double ua[1025] = {0.0}, ub[1025] = {0.0}, ha[1025] = {0.0}, hb[1025] = {0.0};
    ha[0] = 1.0;
    uzero_arrays(c, 1, ua, ha, ha);
    uzero_arrays(c, 1, ub, hb, hb);
    for (int i = 0; i < nyp; ++i) c->frate_g[i] = ua[i] - ub[i];
    c->frate_ready = 1;
}

static void frate_apply(orc_ctx *c)
{
    if (!(c->p.flow_rate > 0.0)) { c->stats.dpdx = c->dPdx; return; }
    if (!c->frate_ready) frate_setup(c);
    double *u0 = RF(c, KMM_U0);
    double q = 0.0, wg = 0.0;
    for (int i = 0; i < c->nyp; ++i) { q += c->frate_w[i] * u0[i]; wg += c->frate_w[i] * c->frate_g[i]; }
    const double d = (c->p.flow_rate - q) / wg;
    for (int i = 0; i < c->nyp; ++i) u0[i] += d * c->frate_g[i];
    c->stats.dpdx = c->dPdx - d;
}

/* ------------------------------------------------------------------------- */
/* solvers.f90: gfcn, phirhs, nonlin, veloc, vort                             */
/* ------------------------------------------------------------------------- */
/* gfcn(gfns,a,wrkc,wrk1,bct,bcb,dnvb,dnvt,nb,nt,pb,pt), solvers.f90:5-172 */
static void gfcn1(orc_ctx *c, int gf, int dnvbf, int dnvtf, double pb, double pt)
{
    cplx *gfns = SF(c, gf), *bct = SF(c, KMM_BCTOP), *bcb = SF(c, KMM_BCBOT);
    const size_t nw = (size_t)c->nz * c->nxh;
    double g = c->re / (c->theta * c->dt);
    for (size_t x = 0; x < nw; ++x) { bct[x] = pt + I * pt; bcb[x] = pb + I * pb; }
    for (int j = c->nz / 2; j < c->nz; ++j) { bct[j] = conj(bct[j]); bcb[j] = conj(bcb[j]); }
    memset(gfns, 0, sizeof(cplx) * (size_t)c->nyp * nw);
    bct[0] = pt; bcb[0] = pb;
    orc_solve(c, gf, g, 0);
    for (size_t x = 0; x < nw; ++x) { bct[x] = 0.0; bcb[x] = 0.0; }
    orc_solve(c, gf, 0.0, 0);
    for (int i = 0; i < c->nyp; ++i) gfns[SIDX(c, i, 0, 0)] = creal(gfns[SIDX(c, i, 0, 0)]);
    for (int j = 2; j <= c->nz / 2; ++j) {
        int jp = c->nz + 2 - j;
        for (int i = 0; i < c->nyp; ++i)
            gfns[SIDX(c, i, j - 1, 0)] = 0.5 * (gfns[SIDX(c, i, j - 1, 0)] + conj(gfns[SIDX(c, i, jp - 1, 0)]));
    }
    for (int j = 2; j <= c->nz / 2; ++j) {
        int jp = c->nz + 2 - j;
        for (int i = 0; i < c->nyp; ++i) gfns[SIDX(c, i, jp - 1, 0)] = conj(gfns[SIDX(c, i, j - 1, 0)]);
    }
    const size_t n = (size_t)c->nyp * nw;
    cplx *wrkc = calloc(n, sizeof(cplx)), *wrk1 = calloc(n, sizeof(cplx));
    if (c->nb == 1) wallderiv_arr(c, gfns, 1, 0, wrkc, 1);
    else { cderiv_arr(c, gfns, wrk1); wallderiv_arr(c, wrk1, 1, 0, wrkc, 1); }
    if (c->nt == 1) wallderiv_arr(c, gfns, 1, 1, wrkc, 2);
    else { cderiv_arr(c, gfns, wrk1); wallderiv_arr(c, wrk1, 1, 1, wrkc, 2); }
    cplx *dnvt = SF(c, dnvtf), *dnvb = SF(c, dnvbf);
    for (size_t x = 0; x < nw; ++x) { dnvt[x] = wrkc[x * c->nyp + 1]; dnvb[x] = wrkc[x * c->nyp + 0]; }
    free(wrkc); free(wrk1);
}

int orc_gfcn(orc_ctx *c)
{
    gfcn1(c, KMM_GF1, KMM_DNV1B, KMM_DNV1T, c->p1b, c->p1t);
    gfcn1(c, KMM_GF2, KMM_DNV2B, KMM_DNV2T, c->p2b, c->p2t);
    cplx *d = SF(c, KMM_DENOM), *d1t = SF(c, KMM_DNV1T), *d2b = SF(c, KMM_DNV2B), *d2t = SF(c, KMM_DNV2T), *d1b = SF(c, KMM_DNV1B);
    for (size_t x = 0; x < (size_t)c->nz * c->nxh; ++x) d[x] = d1t[x] * d2b[x] - d2t[x] * d1b[x]; /* main_dns.f90:155-161 */
    return KMM_OK;
}

/* phirhs(v,wrkc,wrk1,fn,fnm1,bcbot,bctop,var), solvers.f90:555-676 */
int orc_phirhs(orc_ctx *c, int vf, int fnf, int fnm1f, double var)
{
    const size_t nw = (size_t)c->nz * c->nxh, n = (size_t)c->nyp * nw;
    cplx *bct = SF(c, KMM_BCTOP), *bcb = SF(c, KMM_BCBOT);
    for (size_t x = 0; x < nw; ++x) { bct[x] = 0.0; bcb[x] = 0.0; }
    cplx *v = SF(c, vf), *fn = SF(c, fnf), *fnm1 = SF(c, fnm1f);
    cplx *wrkc = malloc(sizeof(cplx) * n), *wrk1 = malloc(sizeof(cplx) * n);
    const double re = c->re, dt = c->dt, th = c->theta;
#pragma omp parallel for
    for (size_t x = 0; x < n; ++x)
        wrkc[x] = -re * var / (dt * th) * v[x] - re * var / (2.0 * th) * (3.0 * fn[x] - fnm1[x]);
    if (th > 0.99) memcpy(v, wrkc, sizeof(cplx) * n);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j) {
            double w2 = c->wavz[j] * c->wavz[j] + c->wavx[k] * c->wavx[k];
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                wrkc[x] = wrkc[x] + (1.0 - th) * w2 * v[x] / th;
            }
        }
    cderiv_arr(c, v, wrk1);
    cderiv_arr(c, wrk1, v);
#pragma omp parallel for
    for (size_t x = 0; x < n; ++x) v[x] = wrkc[x] - (1.0 - th) * v[x] / th;
    free(wrkc); free(wrk1);
    return KMM_OK;
}

/* main_dns.f90:363-375: v <- d2v/dy2 - (kx^2+kz^2) v */
int orc_phi_from_v(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->nz * c->nxh;
    cplx *v = SF(c, KMM_V), *wrk1 = malloc(sizeof(cplx) * n), *wrkc = malloc(sizeof(cplx) * n);
    cderiv_arr(c, v, wrk1);
    cderiv_arr(c, wrk1, wrkc);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j) {
            double wn2 = c->wavx[k] * c->wavx[k] + c->wavz[j] * c->wavz[j];
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                v[x] = wrkc[x] - wn2 * v[x];
            }
        }
    free(wrk1); free(wrkc);
    return KMM_OK;
}

/* influence-matrix composite solution, main_dns.f90:426-466 */
int orc_influence(orc_ctx *c)
{
    const size_t nw = (size_t)c->nz * c->nxh, n = (size_t)c->nyp * nw;
    cplx *v = SF(c, KMM_V), *wrkc = calloc(n, sizeof(cplx)), *wrk1 = calloc(n, sizeof(cplx));
    const int iyb = 2, iyt = 4;
    if (c->nb == 1) {
        wallderiv_arr(c, v, 1, 0, wrkc, iyb);
        if (c->nt == 1) wallderiv_arr(c, v, 1, 1, wrkc, iyt);
        else { cderiv_arr(c, v, wrk1); wallderiv_arr(c, wrk1, 1, 1, wrkc, iyt); }
    } else {
        cderiv_arr(c, v, wrk1);
        wallderiv_arr(c, wrk1, 1, 0, wrkc, iyb);
        if (c->nt == 1) wallderiv_arr(c, v, 1, 1, wrkc, iyt);
        else { cderiv_arr(c, v, wrk1); wallderiv_arr(c, wrk1, 1, 1, wrkc, iyt); }
    }
    cplx *c1 = SF(c, KMM_C1), *c2 = SF(c, KMM_C2), *gf1 = SF(c, KMM_GF1), *gf2 = SF(c, KMM_GF2);
    cplx *d2t = SF(c, KMM_DNV2T), *d2b = SF(c, KMM_DNV2B), *d1b = SF(c, KMM_DNV1B), *d1t = SF(c, KMM_DNV1T), *den = SF(c, KMM_DENOM);
#pragma omp parallel for
    for (size_t x = 0; x < nw; ++x) {
        cplx wb = wrkc[x * c->nyp + (iyb - 1)], wt = wrkc[x * c->nyp + (iyt - 1)];
        c1[x] = (wb * d2t[x] - wt * d2b[x]) / den[x];
        c2[x] = (wt * d1b[x] - wb * d1t[x]) / den[x];
        for (int i = 0; i < c->nyp; ++i) {
            size_t y = x * c->nyp + i;
            v[y] = v[y] + c1[x] * gf1[y] + c2[x] * gf2[y];
        }
    }
    free(wrkc); free(wrk1);
    return KMM_OK;
}

/* nonlin(fn,omz,gn,wrkc,wrk1), solvers.f90:1497-1572 */
int orc_nonlin(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->nz * c->nxh;
    cplx *fn = SF(c, KMM_FN), *gn = SF(c, KMM_GN), *omz = SF(c, KMM_OMZ);
    cplx *wrkc = malloc(sizeof(cplx) * n), *wrk1 = malloc(sizeof(cplx) * n);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j)
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                wrkc[x] = I * (c->wavz[j] * omz[x] + c->wavx[k] * gn[x]);
            }
    cderiv_arr(c, wrkc, wrk1);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j) {
            double w2 = -c->wavx[k] * c->wavx[k] - c->wavz[j] * c->wavz[j];
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                fn[x] = w2 * fn[x] - wrk1[x];
                gn[x] = I * (c->wavz[j] * gn[x] - c->wavx[k] * omz[x]);
            }
        }
    free(wrkc); free(wrk1);
    return KMM_OK;
}

/* veloc(u,v,w,u0,w0,omy,wrkc), solvers.f90:1576-1659 */
int orc_veloc(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->nz * c->nxh;
    cplx *u = SF(c, KMM_U), *v = SF(c, KMM_V), *w = SF(c, KMM_W), *omy = SF(c, KMM_OMY);
    double *u0 = RF(c, KMM_U0), *w0 = RF(c, KMM_W0);
    cplx *wrkc = malloc(sizeof(cplx) * n);
    cderiv_arr(c, v, wrkc);
#pragma omp parallel for collapse(2)
    for (int k = 1; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j) {
            double w2 = c->wavx[k] * c->wavx[k] + c->wavz[j] * c->wavz[j];
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                u[x] = -(-I * c->wavx[k] * wrkc[x] + I * c->wavz[j] * omy[x]) / w2;
                w[x] = -(-I * c->wavz[j] * wrkc[x] - I * c->wavx[k] * omy[x]) / w2;
            }
        }
    for (int j = 1; j < c->nz; ++j) {
        double w2 = c->wavz[j] * c->wavz[j];
        for (int i = 0; i < c->nyp; ++i) {
            size_t x = SIDX(c, i, j, 0);
            u[x] = -(I * c->wavz[j] * omy[x]) / w2;
            w[x] = -(-I * c->wavz[j] * wrkc[x]) / w2;
        }
    }
    for (int i = 0; i < c->nyp; ++i) {
        u[SIDX(c, i, 0, 0)] = u0[i];
        v[SIDX(c, i, 0, 0)] = 0.0;
        w[SIDX(c, i, 0, 0)] = w0[i];
    }
    free(wrkc);
    return KMM_OK;
}

/* vort(u,v,w,omx,omz), solvers.f90:1663-1722 */
int orc_vort(orc_ctx *c)
{
    cplx *u = SF(c, KMM_U), *v = SF(c, KMM_V), *w = SF(c, KMM_W), *omx = SF(c, KMM_OMX), *omz = SF(c, KMM_OMZ);
    cderiv_arr(c, u, omz);
    cderiv_arr(c, w, omx);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j)
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                omz[x] = I * c->wavx[k] * v[x] - omz[x];
                omx[x] = omx[x] - I * c->wavz[j] * v[x];
            }
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* helpers.f90                                                                */
/* ------------------------------------------------------------------------- */
/* norm(a), helpers.f90:91-158 */
static void norm_arr(const orc_ctx *c, cplx *a)
{
    for (int i = 0; i < c->nyp; ++i) a[SIDX(c, i, 0, 0)] = creal(a[SIDX(c, i, 0, 0)]);
    for (int j = 2; j <= c->nz / 2; ++j) {
        int jp = c->nz + 2 - j;
        for (int i = 0; i < c->nyp; ++i)
            a[SIDX(c, i, j - 1, 0)] = 0.5 * (a[SIDX(c, i, j - 1, 0)] + conj(a[SIDX(c, i, jp - 1, 0)]));
    }
    for (int j = 2; j <= c->nz / 2; ++j) {
        int jp = c->nz + 2 - j;
        for (int i = 0; i < c->nyp; ++i) a[SIDX(c, i, jp - 1, 0)] = conj(a[SIDX(c, i, j - 1, 0)]);
    }
    for (int k = 0; k < c->nxh; ++k)
        for (int i = 0; i < c->nyp; ++i) a[SIDX(c, i, c->nzh, k)] = 0.0; /* a(i,nzhp,k) = 0 */
}

int orc_norm(orc_ctx *c, int f)
{
    if (f < 0 || f >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    norm_arr(c, SF(c, f));
    return KMM_OK;
}

/* xyzfft(a,b,-1), helpers.f90:6-87 */
int orc_xyzfft(orc_ctx *c, int dstf, int srcf)
{
    const int nyp = c->nyp, nz = c->nz, nx = c->nx, ny = c->ny, nxh = c->nxh;
    const double *b0 = RF(c, srcf);
    cplx *a = SF(c, dstf);
    if (!b0 || !a || dstf >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    double *b = malloc(sizeof(double) * (size_t)nyp * nz * nx);
    memcpy(b, b0, sizeof(double) * (size_t)nyp * nz * nx);
    cplx *ap = malloc(sizeof(cplx) * (size_t)nyp * nz * (nx / 2 + 1));
    /* y-transform */
#pragma omp parallel
    {
        cplx *x = malloc(sizeof(cplx) * nyp), *o = malloc(sizeof(cplx) * nyp);
        cplx *w1 = malloc(sizeof(cplx) * 2 * ny), *w2 = malloc(sizeof(cplx) * 2 * ny);
#pragma omp for collapse(2)
        for (int k = 0; k < nx; ++k)
            for (int j = 0; j < nz; ++j) {
                double *col = b + ((size_t)k * nz + j) * nyp;
                for (int i = 0; i < nyp; ++i) x[i] = col[i];
                dct1_c(&c->py2, x, o, w1, w2);
                for (int i = 0; i < nyp; ++i) col[i] = creal(o[i]) / (double)ny;
                col[0] = col[0] / 2.0;
                col[nyp - 1] = col[nyp - 1] / 2.0;
            }
        free(x); free(o); free(w1); free(w2);
    }
    /* x-transform (r2c over nx, /nx) */
#pragma omp parallel
    {
        double *row = malloc(sizeof(double) * nx);
        cplx *out = malloc(sizeof(cplx) * (nx / 2 + 1));
        cplx *w1 = malloc(sizeof(cplx) * nx), *w2 = malloc(sizeof(cplx) * nx);
#pragma omp for collapse(2)
        for (int j = 0; j < nz; ++j)
            for (int i = 0; i < nyp; ++i) {
                for (int k = 0; k < nx; ++k) row[k] = b[((size_t)k * nz + j) * nyp + i];
                r2c_pair(&c->pnx, row, NULL, out, NULL, w1, w2);
                for (int k = 0; k <= nx / 2; ++k) ap[((size_t)k * nz + j) * nyp + i] = out[k] / (double)nx;
            }
        free(row); free(out); free(w1); free(w2);
    }
    /* z-transform (forward c2c over nz, /nz) */
#pragma omp parallel
    {
        cplx *col = malloc(sizeof(cplx) * nz), *w = malloc(sizeof(cplx) * nz);
#pragma omp for collapse(2)
        for (int k = 0; k < nxh; ++k)
            for (int i = 0; i < nyp; ++i) {
                for (int j = 0; j < nz; ++j) col[j] = ap[((size_t)k * nz + j) * nyp + i];
                fft_exec(&c->pnz, col, w, -1);
                for (int j = 0; j < nz; ++j) a[SIDX(c, i, j, k)] = col[j] / (double)nz;
            }
        free(col); free(w);
    }
    free(b); free(ap);
    return KMM_OK;
}

/* polyNL, helpers.f90:610-674; results in the C_NM1-independent scratch (T fields are reused by polyforce,
 * so the six NL fields live in KMM_C11..-shaped temporaries owned here) */
static cplx *g_polynl_scratch(orc_ctx *c, int comp)
{
    /* six scratch spectral arrays appended after the public ids */
    int id = KMM_NSPECTRAL + comp;
    if (!c->fld[id]) c->fld[id] = calloc((size_t)c->nyp * c->nz * c->nxh, sizeof(cplx));
    return (cplx *)c->fld[id];
}

static const int poly_comp[6] = {KMM_C11, KMM_C12, KMM_C13, KMM_C22, KMM_C23, KMM_C33};

int orc_polynl(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->nz * c->nxh;
    const double tpolyinv = 1.0 / c->p.tpoly;
    for (int m = 0; m < 6; ++m) {
        cplx *nl = g_polynl_scratch(c, m);
        cplx *cn = SF(c, KMM_C11N + m), *cnm1 = SF(c, KMM_C11NM1 + m);
        cplx *sn = SF(c, KMM_STR11N + m), *snm1 = SF(c, KMM_STR11NM1 + m);
#pragma omp parallel for
        for (size_t x = 0; x < n; ++x)
            nl[x] = 3.0 * (cn[x] - tpolyinv * sn[x]) - (cnm1[x] - tpolyinv * snm1[x]);
    }
    return KMM_OK;
}

/* polyforce(qp11..qp33,t1,t2,t3), helpers.f90:498-560 */
int orc_polyforce(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->nz * c->nxh;
    cplx *s11 = SF(c, KMM_QP11), *s12 = SF(c, KMM_QP12), *s13 = SF(c, KMM_QP13);
    cplx *s22 = SF(c, KMM_QP22), *s23 = SF(c, KMM_QP23), *s33 = SF(c, KMM_QP33);
    cplx *t1 = SF(c, KMM_T1), *t2 = SF(c, KMM_T2), *t3 = SF(c, KMM_T3);
    cplx *w1 = malloc(sizeof(cplx) * n), *w2 = malloc(sizeof(cplx) * n), *w3 = malloc(sizeof(cplx) * n);
    cderiv_arr(c, s12, w1);
    cderiv_arr(c, s22, w2);
    cderiv_arr(c, s23, w3);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j)
            for (int i = 0; i < c->nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                t1[x] = I * (c->wavx[k] * s11[x] + c->wavz[j] * s13[x]) + w1[x];
                t2[x] = I * (c->wavx[k] * s12[x] + c->wavz[j] * s23[x]) + w2[x];
                t3[x] = I * (c->wavx[k] * s13[x] + c->wavz[j] * s33[x]) + w3[x];
            }
    free(w1); free(w2); free(w3);
    return KMM_OK;
}

/* subforce(gn,fn,omz,t1,t2,t3), helpers.f90:564-606 */
int orc_subforce(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->nz * c->nxh;
    cplx *gn = SF(c, KMM_GN), *fn = SF(c, KMM_FN), *omz = SF(c, KMM_OMZ);
    cplx *t1 = SF(c, KMM_T1), *t2 = SF(c, KMM_T2), *t3 = SF(c, KMM_T3);
    for (size_t x = 0; x < n; ++x) { gn[x] += t1[x]; fn[x] += t2[x]; omz[x] += t3[x]; }
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* main_dns.f90: spectral filter                                              */
/* ------------------------------------------------------------------------- */
int orc_filter(orc_ctx *c)
{
    cplx *omz = SF(c, KMM_OMZ), *gn = SF(c, KMM_GN), *fn = SF(c, KMM_FN);
    cplx *scn = c->p.scalar_on ? SF(c, KMM_SCN) : NULL;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 1; j <= c->nz; ++j) {
            int jj = j - 1;
            if (j > c->nzh) jj = c->nz - j + 1;
            double zs = exp(-3.0 * pow((double)jj / (double)c->nzh, 10));
            for (int i = 1; i <= c->nyp; ++i) {
                double ys = exp(-3.0 * pow((double)(i - 1) / (double)c->ny, 10));
                size_t x = SIDX(c, i - 1, j - 1, k);
                omz[x] = omz[x] * zs * ys;
                gn[x] = gn[x] * zs * ys;
                fn[x] = fn[x] * zs * ys;
                if (scn) scn[x] = scn[x] * zs * ys;
                if (c->p.polymer_on) {
                    for (int m = 0; m < 6; ++m) {
                        cplx *a = (cplx *)c->fld[KMM_C11N + m], *s = (cplx *)c->fld[KMM_STR11N + m];
                        if (a) a[x] = a[x] * zs * ys;
                        if (s) s[x] = s[x] * zs * ys;
                    }
                }
            }
        }
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* part_track.f90: tracer path                                                */
/* ------------------------------------------------------------------------- */
/* interpolate3, part_track.f90:1184-1221 */
static double interpolate3(double x, double y, double z, double x0, double x1, double y0, double y1, double z0, double z1,
                           double c000, double c100, double c001, double c101, double c010, double c110, double c011,
                           double c111)
{
    double xd = (x1 > x0) ? (x - x0) / (x1 - x0) : 0.0;
    double yd = (y1 > y0) ? (y - y0) / (y1 - y0) : 0.0;
    double zd = (z1 > z0) ? (z - z0) / (z1 - z0) : 0.0;
    double c00 = c000 * (1.0 - xd) + c100 * xd;
    double c01 = c001 * (1.0 - xd) + c101 * xd;
    double c10 = c010 * (1.0 - xd) + c110 * xd;
    double c11 = c011 * (1.0 - xd) + c111 * xd;
    double c0 = c00 * (1.0 - yd) + c10 * yd;
    double c1 = c01 * (1.0 - yd) + c11 * yd;
    return c0 * (1.0 - zd) + c1 * zd;
}

/* fluid_interp(xp,yp,zp,u,v,w,uf,vf,wf), part_track.f90:518-613; returns nonzero where the reference stops */
static int fluid_interp(const orc_ctx *c, double xp, double yp, double zp, const double *u, const double *v,
                        const double *w, double *uf, double *vf, double *wf)
{
    const int mx = c->mx, mz = c->mz;
    double delxm = c->xl / (double)mx, delzm = c->zl / (double)mz;
    int imin = ((int)floor(xp / delxm) + mx) % mx + 1;
    int imax = imin % mx + 1;
    int jmin = ((int)floor(zp / delzm) + mz) % mz + 1;
    int jmax = jmin % mz + 1;
    int kmax = (int)floor(1.0 + (double)c->ny / c->pi * acos(2.0 * yp / c->yl));
    int kmin = kmax + 1;
    if (imin < 1 || jmin < 1 || kmin < 1 || kmin > c->nyp || kmax < 1) return KMM_ERR_INTERP;
    double xmin = (double)(imin - 1) * delxm, xmax = (double)(imax - 1) * delxm;
    double ymin = c->ycoord[kmin - 1], ymax = c->ycoord[kmax - 1];
    double zmin = (double)(jmin - 1) * delzm, zmax = (double)(jmax - 1) * delzm;
#define P3(f, i, j, k) (f)[PIDX(c, (i) - 1, (j) - 1, (k) - 1)]
#define INTERP(f) interpolate3(xp, yp, zp, xmin, xmax, ymin, ymax, zmin, zmax, P3(f, kmin, jmin, imin), \
        P3(f, kmin, jmin, imax), P3(f, kmin, jmax, imin), P3(f, kmin, jmax, imax), P3(f, kmax, jmin, imin), \
        P3(f, kmax, jmin, imax), P3(f, kmax, jmax, imin), P3(f, kmax, jmax, imax))
    *uf = INTERP(u);
    *vf = INTERP(v);
    *wf = INTERP(w);
#undef INTERP
#undef P3
    return KMM_OK;
}

/* the interpolation cell fluid_interp looks up for every particle (part_track.f90:560-577):
 * cells[p] = imin, cells[np + p] = jmin, cells[2 np + p] = kmax, 1-based; 0 and KMM_ERR_INTERP
 * where the reference stops (part_track.f90:580-590) */
int orc_tracer_cells(orc_ctx *c, int *cells, size_t n)
{
    const int np = c->p.npart, mx = c->mx, mz = c->mz;
    if (np <= 0) return KMM_OK;
    if (n < 3 * (size_t)np) return KMM_ERR_ARG;
    const double *xpa = RF(c, KMM_XPART), *ypa = RF(c, KMM_YPART), *zpa = RF(c, KMM_ZPART);
    const double delxm = c->xl / (double)mx, delzm = c->zl / (double)mz;
    int st = KMM_OK;
    for (int p = 0; p < np; ++p) {
        int imin = ((int)floor(xpa[p] / delxm) + mx) % mx + 1;
        int jmin = ((int)floor(zpa[p] / delzm) + mz) % mz + 1;
        int kmax = (int)floor(1.0 + (double)c->ny / c->pi * acos(2.0 * ypa[p] / c->yl));
        int kmin = kmax + 1;
        int ok = !(imin < 1 || jmin < 1 || kmin < 1 || kmin > c->nyp || kmax < 1);
        cells[p] = ok ? imin : 0;
        cells[np + p] = ok ? jmin : 0;
        cells[2 * np + p] = ok ? kmax : 0;
        if (!ok) st = KMM_ERR_INTERP;
    }
    return st;
}

/* init_part, part_track.f90:229-292: particle velocity forced to the fluid's */
int orc_init_part(orc_ctx *c)
{
    int np = c->p.npart, st = KMM_OK;
    double *xp = RF(c, KMM_XPART), *yp = RF(c, KMM_YPART), *zp = RF(c, KMM_ZPART);
    double *up = RF(c, KMM_UPART), *vp = RF(c, KMM_VPART), *wp = RF(c, KMM_WPART);
    const double *u = RF(c, KMM_UP3D), *v = RF(c, KMM_VP3D), *w = RF(c, KMM_WP3D);
    for (int j = 0; j < np; ++j)
        if (fluid_interp(c, xp[j], yp[j], zp[j], u, v, w, &up[j], &vp[j], &wp[j])) st = KMM_ERR_INTERP;
    return st;
}

/* tracer_update(u,v,w), part_track.f90:360-433 (Euler, with the substep-reduced dt of part_track.f90:128) */
int orc_tracer_update(orc_ctx *c)
{
    int np = c->p.npart, st = KMM_OK;
    double *xpa = RF(c, KMM_XPART), *ypa = RF(c, KMM_YPART), *zpa = RF(c, KMM_ZPART);
    double *upa = RF(c, KMM_UPART), *vpa = RF(c, KMM_VPART), *wpa = RF(c, KMM_WPART);
    const double *u = RF(c, KMM_UP3D), *v = RF(c, KMM_VP3D), *w = RF(c, KMM_WP3D);
    const double dt = c->dt / (double)c->substep;
    const double Height = c->ycoord[0] - c->p.ap, ybot = c->p.ap + c->ycoord[c->nyp - 1];
    const double xl = c->xl, zl = c->zl;
#pragma omp parallel for reduction(max : st)
    for (int j = 0; j < np; ++j) {
        double xp = xpa[j], yp = ypa[j], zp = zpa[j], up = upa[j], vp = vpa[j], wp = wpa[j];
        if (c->p.tracer_scheme == 1) {
            /* variant: Williamson low-storage RK3 on dx/dt = u(x) with the frozen 3/2-grid field */
            static const double ak[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
            static const double bk[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
            double qx = 0, qy = 0, qz = 0, uu = up, vv = vp, ww = wp;
            for (int s = 0; s < 3; ++s) {
                if (fluid_interp(c, xp, yp, zp, u, v, w, &uu, &vv, &ww)) st = KMM_ERR_INTERP;
                qx = ak[s] * qx + dt * uu;
                qy = ak[s] * qy + dt * vv;
                qz = ak[s] * qz + dt * ww;
                xp = fmod(xl + xp + bk[s] * qx, xl);
                yp = fmax(fmin(yp + bk[s] * qy, Height), ybot);
                zp = fmod(zl + zp + bk[s] * qz, zl);
            }
        } else {
            xp = fmod(xl + xp + up * dt, xl);
            yp = fmax(fmin(yp + vp * dt, Height), ybot);
            zp = fmod(zl + zp + wp * dt, zl);
        }
        if (fluid_interp(c, xp, yp, zp, u, v, w, &up, &vp, &wp)) st = KMM_ERR_INTERP;
        xpa[j] = xp; ypa[j] = yp; zpa[j] = zp; upa[j] = up; vpa[j] = vp; wpa[j] = wp;
    }
    return st;
}

/* ------------------------------------------------------------------------- */
/* part_track.f90: inertial particles (particle_flag > 0), Maxey-Riley with RK4 */
/* ------------------------------------------------------------------------- */
typedef struct {
    const double *u, *v, *w, *uo, *vo, *wo, *wx, *wy, *wz, *g[9], *L[3], *Lo[3];
} mr_fields;

/* SubDerivative, part_track.f90:896-1075: the fluid's material derivative and the time
 * derivative of its Laplacian at the particle.  The time derivatives are taken at the eight
 * cell corners first ((f - f_old)/dt with the substep dt) and then interpolated. */
static void mr_subderivative(const orc_ctx *c, const mr_fields *F, double dt, double uf, double vf, double wf,
                             double xp0, double yp0, double zp0, double *sDu, double *sDv, double *sDw, double *dLu,
                             double *dLv, double *dLw)
{
    const int mx = c->mx, mz = c->mz;
    const double delxm = c->xl / (double)mx, delzm = c->zl / (double)mz;
    const int imin = ((int)floor(xp0 / delxm) + mx) % mx + 1, imax = imin % mx + 1;
    const int jmin = ((int)floor(zp0 / delzm) + mz) % mz + 1, jmax = jmin % mz + 1;
    const int kmax = (int)floor(1.0 + (double)c->ny / c->pi * acos(2.0 * yp0 / c->yl)), kmin = kmax + 1;
    const double xmin = (double)(imin - 1) * delxm, xmax = (double)(imax - 1) * delxm;
    const double ymin = c->ycoord[kmin - 1], ymax = c->ycoord[kmax - 1];
    const double zmin = (double)(jmin - 1) * delzm, zmax = (double)(jmax - 1) * delzm;
    const int gk[8] = {kmin, kmin, kmin, kmin, kmax, kmax, kmax, kmax};
    const int gj[8] = {jmin, jmin, jmax, jmax, jmin, jmin, jmax, jmax};
    const int gi[8] = {imin, imax, imin, imax, imin, imax, imin, imax};
    double dudt[3][8], dLudt[3][8], gv[9][8];
    for (int n = 0; n < 8; ++n) {
        const size_t x = PIDX(c, gk[n] - 1, gj[n] - 1, gi[n] - 1);
        dudt[0][n] = (F->u[x] - F->uo[x]) / dt;
        dudt[1][n] = (F->v[x] - F->vo[x]) / dt;
        dudt[2][n] = (F->w[x] - F->wo[x]) / dt;
        for (int m = 0; m < 3; ++m) dLudt[m][n] = (F->L[m][x] - F->Lo[m][x]) / dt;
        for (int m = 0; m < 9; ++m) gv[m][n] = F->g[m][x];
    }
#define I3(a) interpolate3(xp0, yp0, zp0, xmin, xmax, ymin, ymax, zmin, zmax, (a)[0], (a)[1], (a)[2], (a)[3], (a)[4], \
                           (a)[5], (a)[6], (a)[7])
    double gr[9];
    for (int m = 0; m < 9; ++m) gr[m] = I3(gv[m]);   /* dufdx, dufdy, dufdz, dvfdx, ..., dwfdz */
    const double dudt_p = I3(dudt[0]), dvdt_p = I3(dudt[1]), dwdt_p = I3(dudt[2]);
    *dLu = I3(dLudt[0]);
    *dLv = I3(dLudt[1]);
    *dLw = I3(dLudt[2]);
#undef I3
    *sDu = dudt_p + uf * gr[0] + vf * gr[1] + wf * gr[2];
    *sDv = dvdt_p + uf * gr[3] + vf * gr[4] + wf * gr[5];
    *sDw = dwdt_p + uf * gr[6] + vf * gr[7] + wf * gr[8];
}

/* RKstage, part_track.f90:759-892: forces at the stage point, then the stage update from the
 * start-of-step state (h = dt for stage 3, dt/2 otherwise) */
static int mr_stage(const orc_ctx *c, const mr_fields *F, int sn, double dt, double *un, double *vn, double *wn,
                    double *xp, double *yp, double *zp, double *Ku, double *Kv, double *Kw, double xp_old,
                    double yp_old, double zp_old, double up_old, double vp_old, double wp_old)
{
    const double ratio = c->p.ratio, ap = c->p.ap, re = c->re;
    const double Pi_f = 1.0 / (ratio + 0.5), Pi_p = ratio / (ratio + 0.5), C_L = 0.5;
    const double Height = c->ycoord[0] - ap;
    double uf, vf, wf, wxf, wyf, wzf, Luf, Lvf, Lwf;
    int st = fluid_interp(c, *xp, *yp, *zp, F->u, F->v, F->w, &uf, &vf, &wf);
    st |= fluid_interp(c, *xp, *yp, *zp, F->wx, F->wy, F->wz, &wxf, &wyf, &wzf);
    st |= fluid_interp(c, *xp, *yp, *zp, F->L[0], F->L[1], F->L[2], &Luf, &Lvf, &Lwf);
    if (st) return KMM_ERR_INTERP;
    double sDu, sDv, sDw, dLu, dLv, dLw;
    mr_subderivative(c, F, dt, uf, vf, wf, *xp, *yp, *zp, &sDu, &sDv, &sDw, &dLu, &dLv, &dLw);
    const double Re_p = 2 * ap * re * sqrt((uf - *un) * (uf - *un) + (vf - *vn) * (vf - *vn) + (wf - *wn) * (wf - *wn));
    double C_D = 0.0;
    if (c->p.cd_switch == 1) C_D = 16 / (2 * ap * re) * c->p.c_mu;
    else if (c->p.cd_switch == 2) C_D = 24 / (2 * ap * re) * (1 + 0.15 * pow(Re_p, 0.687));
    else if (c->p.cd_switch == 3) C_D = Re_p > 1.0 ? 16.31 * pow(Re_p, -0.8331) : 17.28 * pow(Re_p, -0.9711);
    const double a6 = ap * ap / 6.0;
    const double ru = uf - *un + a6 * Luf, rv = vf - *vn + a6 * Lvf, rw = wf - *wn + a6 * Lwf;
    const double PGX = 1.5 * sDu, DX = C_D * 3 / (8 * ap) * ru, LX = C_L * (rv * wzf - rw * wyf);
    const double FX = 3.0 / 20.0 * (ap * ap) * dLu;
    const double PGY = 1.5 * sDv, DY = C_D * 3 / (8 * ap) * rv, LY = C_L * (rw * wxf - ru * wzf);
    const double FY = 3.0 / 20.0 * (ap * ap) * dLv;
    const double PGZ = 1.5 * sDw, DZ = C_D * 3 / (8 * ap) * rw, LZ = C_L * (ru * wyf - rv * wxf);
    const double FZ = 3.0 / 20.0 * (ap * ap) * dLw;
    *Ku = Pi_f * (PGX + DX + LX + FX);
    *Kv = Pi_f * (PGY + DY + LY + FY) - c->p.gravity * (Pi_f - Pi_p);
    *Kw = Pi_f * (PGZ + DZ + LZ + FZ);
    const double h = sn == 3 ? dt : dt / 2.0;
    *un = up_old + h * *Ku;
    *vn = vp_old + h * *Kv;
    *wn = wp_old + h * *Kw;
    *xp = fmod(c->xl + xp_old + h * *un, c->xl);
    *yp = fmax(fmin(yp_old + h * *vn, Height), ap + c->ycoord[c->nyp - 1]);
    *zp = fmod(c->zl + zp_old + h * *wn, c->zl);
    return KMM_OK;
}

/* RK4, part_track.f90:617-755: one substep of one particle; *umax1 = max(*umax1, relative speed) */
static int mr_rk4(const orc_ctx *c, const mr_fields *F, double dt, double *xp0, double *yp0, double *zp0, double *up,
                  double *vp, double *wp, double *umax1)
{
    const double ap = c->p.ap, Height = c->ycoord[0] - ap, ybot = ap + c->ycoord[c->nyp - 1];
    double xp = *xp0, yp = *yp0, zp = *zp0, un = *up, vn = *vp, wn = *wp;
    double K[4][3], s2[3], s3[3], s4[3];
    int st = KMM_OK;
    for (int sn = 1; sn <= 4; ++sn) {
        st |= mr_stage(c, F, sn, dt, &un, &vn, &wn, &xp, &yp, &zp, &K[sn - 1][0], &K[sn - 1][1], &K[sn - 1][2], *xp0,
                       *yp0, *zp0, *up, *vp, *wp);
        if (st) return KMM_ERR_INTERP;
        double *d = sn == 1 ? s2 : sn == 2 ? s3 : sn == 3 ? s4 : NULL;
        if (d) { d[0] = un; d[1] = vn; d[2] = wn; }
    }
    *xp0 = fmod(c->xl + *xp0 + dt * (*up / 6 + s2[0] / 3 + s3[0] / 3 + s4[0] / 6), c->xl);
    *yp0 = fmax(fmin(*yp0 + dt * (*vp / 6 + s2[1] / 3 + s3[1] / 3 + s4[1] / 6), Height), ybot);
    *zp0 = fmod(c->zl + *zp0 + dt * (*wp / 6 + s2[2] / 3 + s3[2] / 3 + s4[2] / 6), c->zl);
    *up = *up + dt * (K[0][0] / 6 + K[1][0] / 3 + K[2][0] / 3 + K[3][0] / 6);
    const double vp_new = *vp + dt * (K[0][1] / 6 + K[1][1] / 3 + K[2][1] / 3 + K[3][1] / 6);
    *wp = *wp + dt * (K[0][2] / 6 + K[1][2] / 3 + K[2][2] / 3 + K[3][2] / 6);
    /* elastic bounce off a wall the particle was clamped to */
    if ((*yp0 == Height && vp_new > 0.0) || (*yp0 == ybot && vp_new < 0.0)) *vp = -vp_new;
    else *vp = vp_new;
    double uf, vf, wf;
    if (fluid_interp(c, *xp0, *yp0, *zp0, F->u, F->v, F->w, &uf, &vf, &wf)) return KMM_ERR_INTERP;
    const double um = sqrt((uf - *up) * (uf - *up) + (vf - *vp) * (vf - *vp) + (wf - *wp) * (wf - *wp));
    if (um > *umax1) *umax1 = um;
    return KMM_OK;
}

/* the particle_flag > 0 branch of part_track, part_track.f90:125-176: `substep` RK4 substeps
 * of dt/substep per particle */
int orc_inertial_update(orc_ctx *c)
{
    mr_fields F;
    F.u = RF(c, KMM_UP3D); F.v = RF(c, KMM_VP3D); F.w = RF(c, KMM_WP3D);
    F.uo = RF(c, KMM_UOLD); F.vo = RF(c, KMM_VOLD); F.wo = RF(c, KMM_WOLD);
    F.wx = RF(c, KMM_WX3D); F.wy = RF(c, KMM_WY3D); F.wz = RF(c, KMM_WZ3D);
    for (int m = 0; m < 9; ++m) F.g[m] = RF(c, KMM_U11P3D + m);
    for (int m = 0; m < 3; ++m) { F.L[m] = RF(c, KMM_LUP3D + m); F.Lo[m] = RF(c, KMM_LUNM1 + m); }
    double *xpa = RF(c, KMM_XPART), *ypa = RF(c, KMM_YPART), *zpa = RF(c, KMM_ZPART);
    double *upa = RF(c, KMM_UPART), *vpa = RF(c, KMM_VPART), *wpa = RF(c, KMM_WPART);
    const double dt = c->dt / (double)c->substep;
    const int np = c->p.npart, nsub = c->substep;
    double umax1 = c->umax1;
    int st = KMM_OK;
#pragma omp parallel for reduction(max : umax1, st)
    for (int j = 0; j < np; ++j)
        for (int s = 0; s < nsub; ++s) {
            double xp = xpa[j], yp = ypa[j], zp = zpa[j], up = upa[j], vp = vpa[j], wp = wpa[j];
            int e = mr_rk4(c, &F, dt, &xp, &yp, &zp, &up, &vp, &wp, &umax1);
            if (e > st) st = e;
            xpa[j] = xp; ypa[j] = yp; zpa[j] = zp; upa[j] = up; vpa[j] = vp; wpa[j] = wp;
        }
    c->umax1 = umax1;
    return st;
}

/* ------------------------------------------------------------------------- */
/* solvers.f90: vcw3dp                                                        */
/* ------------------------------------------------------------------------- */
/* physical-plane field slots */
enum {
    P_U, P_V, P_W, P_WX, P_WY, P_WZ, P_U11, P_U12, P_U13, P_U21, P_U22, P_U23, P_U31, P_U32, P_U33, P_LU, P_LV, P_LW,
    P_SC, P_CX, P_CY, P_CZ,
    P_C11, P_C12, P_C13, P_C21, P_C22, P_C23, P_C31, P_C32, P_C33,
    P_DC111, /* 27 slots */
    P_NIN = P_DC111 + 27
};
enum { O_GN, O_FN, O_OMZ, O_SCN, O_C11N, O_STR11N = O_C11N + 6, O_QP11 = O_STR11N + 6, O_NOUT = O_QP11 + 6 };

static double swirl_point(double r11, double r12, double r13, double r21, double r22, double r23, double r31,
                          double r32, double r33);
static void to_phys3d(orc_ctx *c, const cplx *src, double *phys);

/* ------------------------------------------------------------------------- */
/* targeted scalar sources (solvers.f90:2164-2206)                            */
/* ------------------------------------------------------------------------- */
#define ORC_QN 32768    /* grid_size.f90:2, the length of findmaxQ's candidate list */
#define ORC_NTARG 1023  /* solvers.f90:2172: targets are added while cnt < 1024 */

/* calcQ (helpers.f90:1519-1552): Q = (rotation - strain) / 2 */
static double q_point(double u11, double u12, double u13, double u21, double u22, double u23, double u31,
                      double u32, double u33)
{
    const double strain = u11 * u11 + u22 * u22 + u33 * u33;
    const double rot = -2.0 * (u12 * u21 + u13 * u31 + u23 * u32);
    return 0.5 * (rot - strain);
}

/* Shell_Sort (helpers.f90:1557-1594), 1-based as written: increments n/2, then *5/11 (2 -> 1);
 * b, c, d follow a's moves */
static void shell_sort(double *a, int *b, int *c, int *d, int n)
{
    int inc = n / 2;
    while (inc > 0) {
        for (int i = inc + 1; i <= n; ++i) {
            int j = i;
            const double t1 = a[i - 1];
            const int t2 = b[i - 1], t3 = c[i - 1], t4 = d[i - 1];
            while (j >= inc + 1 && a[j - inc - 1] > t1) {
                a[j - 1] = a[j - inc - 1];
                b[j - 1] = b[j - inc - 1];
                c[j - 1] = c[j - inc - 1];
                d[j - 1] = d[j - inc - 1];
                j -= inc;
            }
            a[j - 1] = t1;
            b[j - 1] = t2;
            c[j - 1] = t3;
            d[j - 1] = t4;
        }
        inc = inc == 2 ? 1 : inc * 5 / 11;
    }
}

/* scl_flag = 4 (solvers.f90:2164-2204 with findmaxQ, helpers.f90:678-953): the nine gradients and
 * the scalar on the 3/2 grid, beta = exp(-alpha_poly |c|), Q (calcQ) negated; the interior grid
 * minima of -Q that are negative, in the reference's loop order (x outer, then z, y inner) and at
 * most qn of them; Shell_Sort of the qn-long list; then, walking the sorted list, a Gaussian of
 * widths sigma around every point with beta > 0.8 until 1023 have been placed.  Where the
 * reference is undefined the restatement chooses:
 *   - the scalar enters with its real and imaginary parts (findmaxQ assigns the imaginary part to
 *     scr, helpers.f90:774, and never sets sci);
 *   - the list starts from zeros on every call (the reference's Qmin keeps the previous call's
 *     entries, solvers.f90:1938, whose indices have been reset to 0);
 *   - the walk stops at the end of the found minima (the reference reads on past them). */
static void target_findmaxq(orc_ctx *c)
{
    const int nyp = c->nyp, mz = c->mz, mx = c->mx, ny = c->ny;
    const size_t nphys = (size_t)nyp * mz * mx;
    double *g[9], *sc = malloc(sizeof(double) * nphys), *qc = malloc(sizeof(double) * nphys);
    for (int m = 0; m < 9; ++m) {
        g[m] = malloc(sizeof(double) * nphys);
        to_phys3d(c, SF(c, KMM_U11 + m), g[m]);
    }
    to_phys3d(c, SF(c, KMM_SCALAR), sc);
#pragma omp parallel for
    for (size_t q = 0; q < nphys; ++q) {
        qc[q] = -q_point(g[0][q], g[1][q], g[2][q], g[3][q], g[4][q], g[5][q], g[6][q], g[7][q], g[8][q]);
        sc[q] = exp(-c->p.alpha_poly * fabs(sc[q]));   /* beta */
    }
    double *qmin = calloc(ORC_QN, sizeof(double));
    int *qx = calloc(ORC_QN, sizeof(int)), *qy = calloc(ORC_QN, sizeof(int)), *qz = calloc(ORC_QN, sizeof(int));
    int cnt = 1;
#define QC(i, j, k) qc[PIDX(c, (i) - 1, (j) - 1, (k) - 1)]
    for (int k = 2; k <= mx - 1; ++k)
        for (int j = 2; j <= mz - 1; ++j)
            for (int i = 2; i <= ny; ++i) {
                const double v = QC(i, j, k);
                if (v < 0 && cnt <= ORC_QN && v < QC(i + 1, j, k) && v < QC(i - 1, j, k) && v < QC(i, j + 1, k) &&
                    v < QC(i, j - 1, k) && v < QC(i, j, k + 1) && v < QC(i, j, k - 1)) {
                    qmin[cnt - 1] = v;
                    qx[cnt - 1] = k;
                    qy[cnt - 1] = i;
                    qz[cnt - 1] = j;
                    ++cnt;
                }
            }
#undef QC
    shell_sort(qmin, qx, qy, qz, ORC_QN);
    double *out = c->scsource;
    memset(out, 0, sizeof(double) * nphys);
    const double delxm = c->xl / (double)mx, delzm = c->zl / (double)mz;
    const double sx = c->p.sigmax, sy = c->p.sigmay, sz = c->p.sigmaz, dT = c->p.deltat;
    c->ntarg = 0;
    for (int n = 1, placed = 1; placed < ORC_NTARG + 1 && n <= ORC_QN; ++n) {
        const int kk = qx[n - 1], ii = qy[n - 1], jj = qz[n - 1];
        if (kk == 0) break;   /* the end of the found minima */
        if (!(sc[PIDX(c, ii - 1, jj - 1, kk - 1)] > 0.8)) continue;
        const double xc1 = delxm * (double)(kk - 1), yc1 = c->ycoord[ii - 1], zc1 = delzm * (double)(jj - 1);
#pragma omp parallel for
        for (int k = 1; k <= mx; ++k) {
            const double xsq = pow((double)(k - 1) * delxm - xc1, 2), betax = xsq / (2.0 * sx * sx);
            if (betax < 18.0)
                for (int j = 1; j <= mz; ++j) {
                    const double zsq = pow((double)(j - 1) * delzm - zc1, 2), betaz = zsq / (2.0 * sz * sz);
                    if (betax + betaz < 18.0)
                        for (int i = 1; i <= nyp; ++i) {
                            const double ysq = pow(c->ycoord[i - 1] - yc1, 2), betay = ysq / (2.0 * sy * sy);
                            if (betax + betay + betaz < 18.0)
                                out[PIDX(c, i - 1, j - 1, k - 1)] += dT * exp(-(betax + betay + betaz));
                        }
                }
        }
        c->targ[3 * c->ntarg] = kk;
        c->targ[3 * c->ntarg + 1] = ii;
        c->targ[3 * c->ntarg + 2] = jj;
        ++c->ntarg;
        ++placed;
    }
    for (int m = 0; m < 9; ++m) free(g[m]);
    free(sc); free(qc); free(qmin); free(qx); free(qy); free(qz);
}

/* scl_flag = 5 (solvers.f90:2205-2206 with newtarget, helpers.f90:957-1222): the swirl strength of
 * the 3/2-grid gradients (calcswirl) scaled to [0, 1] by its maximum, then by spts over its volume
 * integral with the cells' widths Lx, Lz and the half-spacings Ly of the Chebyshev nodes, summed in
 * the reference's loop order (x outer, z, y inner; the reference leaves scsum unset, 0 here). */
static void target_newtarget(orc_ctx *c)
{
    const int nyp = c->nyp, mz = c->mz, mx = c->mx, ny = c->ny;
    const size_t nphys = (size_t)nyp * mz * mx;
    double *g[9];
    for (int m = 0; m < 9; ++m) {
        g[m] = malloc(sizeof(double) * nphys);
        to_phys3d(c, SF(c, KMM_U11 + m), g[m]);
    }
    double *out = c->scsource;
#pragma omp parallel for schedule(dynamic, 4096)
    for (size_t q = 0; q < nphys; ++q)
        out[q] = swirl_point(g[0][q], g[1][q], g[2][q], g[3][q], g[4][q], g[5][q], g[6][q], g[7][q], g[8][q]);
    double qmax = out[0];
    for (size_t q = 1; q < nphys; ++q)
        if (out[q] > qmax) qmax = out[q];
    const double lx = c->xl / (double)mx, lz = c->zl / (double)mz;
    const double *yc = c->ycoord;
    double scsum = 0.0;
    for (int k = 0; k < mx; ++k)
        for (int j = 0; j < mz; ++j)
            for (int i = 0; i < nyp; ++i) {
                double ly;
                if (i == 0) ly = fabs(yc[1] - yc[0]) / 2.0;
                else if (i == nyp - 1) ly = fabs(yc[nyp - 1] - yc[ny - 1]) / 2.0;
                else ly = fabs(yc[i + 1] - yc[i]) / 2.0 + fabs(yc[i] - yc[i - 1]) / 2.0;
                const size_t q = PIDX(c, i, j, k);
                out[q] = out[q] / qmax;
                scsum = scsum + out[q] * lx * ly * lz;
            }
    const double var1 = c->p.spts / scsum;
    for (size_t q = 0; q < nphys; ++q) out[q] = out[q] * var1;
    for (int m = 0; m < 9; ++m) free(g[m]);
}

int orc_target_list(orc_ctx *c, int *ijk, int n)
{
    if (!c || (n > 0 && !ijk)) return -1;
    for (int m = 0; m < 3 * c->ntarg && m < n; ++m) ijk[m] = c->targ[m];
    return c->ntarg;
}

/* scalar source scl_flag == 2, solvers.f90:2079-2118 */
static void scalar_source_particles(orc_ctx *c)
{
    const size_t n = (size_t)c->nyp * c->mz * c->mx;
    c->scsource = RF(c, KMM_SCSOURCE);
    double *sc = c->scsource;
    memset(sc, 0, n * sizeof(double));
    const double delxm = c->xl / (double)c->mx, delzm = c->zl / (double)c->mz;
    const double sx = c->p.sigmax, sy = c->p.sigmay, sz = c->p.sigmaz, dT = c->p.deltat;
    const double *xp = RF(c, KMM_XPART), *yp = RF(c, KMM_YPART), *zp = RF(c, KMM_ZPART);
    for (int np = 0; np < c->p.npart; ++np) {
        double xc1 = xp[np], yc1 = yp[np], zc1 = zp[np];
#pragma omp parallel for
        for (int k = 1; k <= c->mx; ++k) {
            double xsq = pow((double)(k - 1) * delxm - xc1, 2), betax = xsq / (2.0 * sx * sx);
            if (betax < 20.0)
                for (int j = 1; j <= c->mz; ++j) {
                    double zsq = pow((double)(j - 1) * delzm - zc1, 2), betaz = zsq / (2.0 * sz * sz);
                    if (betax + betaz < 20.0)
                        for (int i = 1; i <= c->nyp; ++i) {
                            double ysq = pow(c->ycoord[i - 1] - yc1, 2), betay = ysq / (2.0 * sy * sy);
                            if (betax + betay + betaz < 18.0)
                                sc[PIDX(c, i - 1, j - 1, k - 1)] += dT * exp(-(betax + betay + betaz));
                        }
                }
        }
    }
}

int orc_vcw3dp(orc_ctx *c)
{
    const int nyp = c->nyp, nz = c->nz, nxh = c->nxh, mx = c->mx, mz = c->mz, ny = c->ny, nzh = c->nzh;
    const size_t nspec = (size_t)nyp * nz * nxh;
    const int scal = c->p.scalar_on, poly = c->p.polymer_on;
    const int it = c->it;
    const int poly_act = poly && (it >= c->p.src_start - 1);
    const double re = c->re, dt = c->dt;
    const double delxm = c->xl / (double)mx, delzm = c->zl / (double)mz;
    int *imatrix = (int *)orc_field(c, KMM_IMATRIX);
    double *fxi = RF(c, KMM_FXINTG), *fyi = RF(c, KMM_FYINTG), *fzi = RF(c, KMM_FZINTG);
    update_kmaxsurf(c);
    for (size_t x = 0; x < (size_t)nyp * mz * mx; ++x) {
        int t = imatrix[x];
        if (!(t == 0 || t == 1 || t == 3 || t == 4 || t == 11)) return KMM_ERR_UNSUPPORTED;
    }

    /* scalar source, solvers.f90:2076-2210: particle Gaussians (2), targeted (4, 5), else zero */
    const int in_window = it >= c->p.src_start && it <= c->p.src_stop;
    if (scal && c->p.scl_flag >= 2) c->scsource = RF(c, KMM_SCSOURCE);   /* the field's storage */
    if (scal && c->p.scl_flag == 2 && in_window) scalar_source_particles(c);
    else if (scal && c->p.scl_flag == 4 && in_window) target_findmaxq(c);
    else if (scal && c->p.scl_flag == 5 && in_window) target_newtarget(c);
    else if (scal && c->p.scl_flag >= 2) {
        memset(c->scsource, 0, sizeof(double) * (size_t)nyp * mz * mx);
    }

    /* inputs in the reference's order, solvers.f90:2241-2399 */
    int in_ids[P_NIN], in_slot[P_NIN], nin = 0;
    static const int fl[18] = {KMM_U, KMM_V, KMM_W, KMM_OMX, KMM_OMY, KMM_OMZ, KMM_U11, KMM_U12, KMM_U13, KMM_U21,
                               KMM_U22, KMM_U23, KMM_U31, KMM_U32, KMM_U33, KMM_LU, KMM_LV, KMM_LW};
    for (int m = 0; m < 18; ++m) { in_ids[nin] = fl[m]; in_slot[nin++] = P_U + m; }
    if (scal) {
        int sl[4] = {KMM_SCALAR, KMM_SCLX, KMM_SCLY, KMM_SCLZ};
        for (int m = 0; m < 4; ++m) { in_ids[nin] = sl[m]; in_slot[nin++] = P_SC + m; }
    }
    if (poly_act) {
        for (int m = 0; m < 9; ++m) { in_ids[nin] = KMM_C11 + m; in_slot[nin++] = P_C11 + m; }
        for (int m = 0; m < 27; ++m) { in_ids[nin] = KMM_DC111 + m; in_slot[nin++] = P_DC111 + m; }
    }
    int out_ids[O_NOUT], out_slot[O_NOUT], nout = 0;
    out_ids[nout] = KMM_GN; out_slot[nout++] = O_GN;
    out_ids[nout] = KMM_FN; out_slot[nout++] = O_FN;
    out_ids[nout] = KMM_OMZ; out_slot[nout++] = O_OMZ;
    if (scal) { out_ids[nout] = KMM_SCN; out_slot[nout++] = O_SCN; }
    if (poly_act) {
        for (int m = 0; m < 6; ++m) { out_ids[nout] = KMM_C11N + m; out_slot[nout++] = O_C11N + m; }
        for (int m = 0; m < 6; ++m) { out_ids[nout] = KMM_STR11N + m; out_slot[nout++] = O_STR11N + m; }
        static const int q[6] = {KMM_QP11, KMM_QP12, KMM_QP13, KMM_QP22, KMM_QP23, KMM_QP33};
        for (int m = 0; m < 6; ++m) { out_ids[nout] = q[m]; out_slot[nout++] = O_QP11 + m; }
    }

    /* resolve (and allocate) every field before the parallel regions */
    cplx *inp[P_NIN], *outp[O_NOUT];
    for (int f = 0; f < nin; ++f) inp[f] = SF(c, in_ids[f]);
    for (int f = 0; f < nout; ++f) outp[f] = SF(c, out_ids[f]);
    (void)RF(c, KMM_UXMEAN);
    for (int f = KMM_XPART; f < KMM_NPART_END; ++f) (void)orc_field(c, f);
    /* scale by c(i)/2 and DCT-I along y (REDFT00), solvers.f90:2241-2546 */
    cplx **yin = calloc((size_t)nin, sizeof(cplx *));
    for (int f = 0; f < nin; ++f) yin[f] = malloc(sizeof(cplx) * nspec);
    cplx **yout = calloc((size_t)nout, sizeof(cplx *));
    for (int f = 0; f < nout; ++f) yout[f] = calloc(nspec, sizeof(cplx));
#pragma omp parallel
    {
        cplx *x = malloc(sizeof(cplx) * nyp), *o = malloc(sizeof(cplx) * nyp);
        cplx *w1 = malloc(sizeof(cplx) * 2 * ny), *w2 = malloc(sizeof(cplx) * 2 * ny);
#pragma omp for collapse(2)
        for (int f = 0; f < nin; ++f)
            for (int col = 0; col < nz * nxh; ++col) {
                const cplx *src = inp[f] + (size_t)col * nyp;
                for (int i = 0; i < nyp; ++i) {
                    double fac = c->c[i] / 2.0;
                    x[i] = creal(src[i]) * fac + I * (cimag(src[i]) * fac);
                }
                dct1_c(&c->py2, x, o, w1, w2);
                memcpy(yin[f] + (size_t)col * nyp, o, sizeof(cplx) * nyp);
            }
        free(x); free(o); free(w1); free(w2);
    }

    for (int i = 0; i < nyp; ++i) c->cfl[i] = 0.0;
    double *up3d = RF(c, KMM_UP3D), *vp3d = RF(c, KMM_VP3D), *wp3d = RF(c, KMM_WP3D);
    /* inertial particles read the vorticity, velocity gradient and Laplacian on the 3/2 grid
       (wx3d .. wz3d, u11p3d .. u33p3d, Lup3d .. Lwp3d; solvers.f90:3464-3466) */
    const int inertial = c->p.particle_flag > 0 && c->p.npart > 0;
    double *p3d[15];
    for (int m = 0; m < 15; ++m) p3d[m] = inertial ? RF(c, KMM_WX3D + m) : NULL;
    if (inertial)
        for (int m = 0; m < 6; ++m) (void)RF(c, KMM_UOLD + m);
    const double zl2 = c->p.zlmax * c->p.zlmax;
    const int kmaxsurf = c->kmaxsurf;

    /* loop over y-planes, solvers.f90:2550-3276 */
#pragma omp parallel
    {
        const int hx = mx / 2 + 1;
        cplx *spec[P_NIN];
        double *phys[P_NIN];
        for (int s = 0; s < P_NIN; ++s) { spec[s] = NULL; phys[s] = NULL; }
        for (int f = 0; f < nin; ++f) {
            spec[in_slot[f]] = malloc(sizeof(cplx) * (size_t)mz * hx);
            phys[in_slot[f]] = malloc(sizeof(double) * (size_t)mz * mx);
        }
        double *op[O_NOUT];
        cplx *os[O_NOUT];
        for (int s = 0; s < O_NOUT; ++s) {
            op[s] = malloc(sizeof(double) * (size_t)mz * mx);
            os[s] = malloc(sizeof(cplx) * (size_t)mz * hx);
        }
        double *dragx = malloc(sizeof(double) * (size_t)mz * mx), *dragy = malloc(sizeof(double) * (size_t)mz * mx),
               *dragz = malloc(sizeof(double) * (size_t)mz * mx);
        int wl = mx > mz ? mx : mz;
        cplx *w1 = malloc(sizeof(cplx) * wl), *w2 = malloc(sizeof(cplx) * wl);
        cplx *ra = malloc(sizeof(cplx) * hx), *rb = malloc(sizeof(cplx) * hx);
        double *rowa = malloc(sizeof(double) * mx), *rowb = malloc(sizeof(double) * mx);

#pragma omp for schedule(dynamic)
        for (int i = 0; i < nyp; ++i) {
            /* pack with z zero-padding, z c2c backward, x c2r: solvers.f90:2578-2879 */
            for (int f = 0; f < nin; ++f) {
                cplx *s = spec[in_slot[f]];
                memset(s, 0, sizeof(cplx) * (size_t)mz * hx);
                for (int k = 0; k < nxh; ++k) {
                    /* zero-padded column: modes j <= nzh stay, j > nzh move to (mz-nz)+j */
                    cplx *zc = w1;
                    for (int j = 0; j < mz; ++j) zc[j] = 0.0;
                    for (int j = 1; j <= nz; ++j) {
                        int jj = (j <= nzh) ? j : (mz - nz) + j;
                        zc[jj - 1] = yin[f][SIDX(c, i, j - 1, k)];
                    }
                    fft_exec(&c->pmz, zc, w2, +1);
                    for (int j = 0; j < mz; ++j) s[(size_t)j * hx + k] = zc[j];
                }
            }
            for (int f = 0; f < nin; f += 2) {
                int sa = in_slot[f], sb = (f + 1 < nin) ? in_slot[f + 1] : -1;
                for (int j = 0; j < mz; ++j) {
                    c2r_pair(&c->pmx, spec[sa] + (size_t)j * hx, sb >= 0 ? spec[sb] + (size_t)j * hx : NULL, rowa,
                             sb >= 0 ? rowb : NULL, w1, w2);
                    for (int k = 0; k < mx; ++k) {
                        phys[sa][(size_t)k * mz + j] = rowa[k];
                        if (sb >= 0) phys[sb][(size_t)k * mz + j] = rowb[k];
                    }
                }
            }
            double *up = phys[P_U], *vp = phys[P_V], *wp = phys[P_W];
            double *wxp = phys[P_WX], *wyp = phys[P_WY], *wzp = phys[P_WZ];
            double *vwx = op[O_GN], *vwy = op[O_FN], *vwz = op[O_OMZ], *vc = op[O_SCN];
            for (size_t x = 0; x < (size_t)mz * mx; ++x) { dragx[x] = 0.0; dragy[x] = 0.0; dragz[x] = 0.0; }
            double cfli = 0.0;
            /* pointwise terms, solvers.f90:2885-3110 (k outer, j inner, as the reference) */
            for (int k = 1; k <= mx; ++k)
                for (int j = 1; j <= mz; ++j) {
                    const size_t q = (size_t)(k - 1) * mz + (j - 1);
                    vwx[q] = vp[q] * wzp[q] - wp[q] * wyp[q];
                    vwy[q] = -up[q] * wzp[q] + wp[q] * wxp[q];
                    vwz[q] = up[q] * wyp[q] - vp[q] * wxp[q];
                    if (scal) vc[q] = -(up[q] * phys[P_CX][q] + vp[q] * phys[P_CY][q] + wp[q] * phys[P_CZ][q]);
                    if (poly_act) {
                        double c11 = phys[P_C11][q], c12 = phys[P_C12][q], c13 = phys[P_C13][q];
                        double c21 = phys[P_C21][q], c22 = phys[P_C22][q], c23 = phys[P_C23][q];
                        double c31 = phys[P_C31][q], c32 = phys[P_C32][q], c33 = phys[P_C33][q];
                        double u11 = phys[P_U11][q], u12 = phys[P_U12][q], u13 = phys[P_U13][q];
                        double u21 = phys[P_U21][q], u22 = phys[P_U22][q], u23 = phys[P_U23][q];
                        double u31 = phys[P_U31][q], u32 = phys[P_U32][q], u33 = phys[P_U33][q];
#define DC(ij, kk) phys[P_DC111 + 3 * (ij) + (kk)][q]
                        op[O_C11N + 0][q] = c11 * u11 + c12 * u12 + c13 * u13 + c11 * u11 + c21 * u12 + c31 * u13 -
                                            (up[q] * DC(0, 0) + vp[q] * DC(0, 1) + wp[q] * DC(0, 2));
                        op[O_C11N + 1][q] = c11 * u21 + c12 * u22 + c13 * u23 + c12 * u11 + c22 * u12 + c32 * u13 -
                                            (up[q] * DC(1, 0) + vp[q] * DC(1, 1) + wp[q] * DC(1, 2));
                        op[O_C11N + 2][q] = c11 * u31 + c12 * u32 + c13 * u33 + c13 * u11 + c23 * u12 + c33 * u13 -
                                            (up[q] * DC(2, 0) + vp[q] * DC(2, 1) + wp[q] * DC(2, 2));
                        op[O_C11N + 3][q] = c21 * u21 + c22 * u22 + c23 * u23 + c12 * u21 + c22 * u22 + c32 * u23 -
                                            (up[q] * DC(4, 0) + vp[q] * DC(4, 1) + wp[q] * DC(4, 2));
                        op[O_C11N + 4][q] = c21 * u31 + c22 * u32 + c23 * u33 + c13 * u21 + c23 * u22 + c33 * u23 -
                                            (up[q] * DC(5, 0) + vp[q] * DC(5, 1) + wp[q] * DC(5, 2));
                        op[O_C11N + 5][q] = c31 * u31 + c32 * u32 + c33 * u33 + c13 * u31 + c23 * u32 + c33 * u33 -
                                            (up[q] * DC(8, 0) + vp[q] * DC(8, 1) + wp[q] * DC(8, 2));
#undef DC
                        double trp = c11 + c22 + c33;
                        double s6[6] = {c11, c12, c13, c22, c23, c33};
                        for (int m = 0; m < 6; ++m)
                            op[O_STR11N + m][q] = (c->p.ipeter == 0) ? s6[m] : ((zl2 - 3.0) / (zl2 - trp)) * s6[m];
                        op[O_STR11N + 0][q] -= 1.0;
                        op[O_STR11N + 3][q] -= 1.0;
                        op[O_STR11N + 5][q] -= 1.0;
                        double beta_poly = c->p.qbeta;
                        if (c->p.itarget == 1) {
                            double sc = fabs(phys[P_SC] ? phys[P_SC][q] : 0.0);
                            if (c->p.alpha_poly * sc < 18.0) beta_poly = exp(-c->p.alpha_poly * sc);
                        } else if (c->p.itarget == 2) {
                            double sc = fabs(phys[P_SC] ? phys[P_SC][q] : 0.0);
                            beta_poly = 1.0 / (c->p.alpha_poly * sc + 1.0);
                        }
                        double zbeta1 = (1.0 - beta_poly) / (re * beta_poly * c->p.tpoly);
                        for (int m = 0; m < 6; ++m) op[O_QP11 + m][q] = zbeta1 * op[O_STR11N + m][q];
                    }
                    double cflcheck = (fabs(up[q]) / delxm + fabs(vp[q]) / c->seght[i] + fabs(wp[q]) / delzm) * dt;
                    if (cflcheck > cfli) cfli = cflcheck;
                    /* immersed boundary, solvers.f90:2996-3059 */
                    const size_t g3 = PIDX(c, i, j - 1, k - 1);
                    const int t = imatrix[g3];
                    if (t == 1 || (t == 4 && it <= c->p.perturbtime)) {
                        fxi[g3] = fxi[g3] + up[q];
                        fyi[g3] = fyi[g3] + vp[q];
                        fzi[g3] = fzi[g3] + wp[q];
                        dragx[q] = (-c->ugain * up[q]) - c->gain * fxi[g3];
                        dragy[q] = (-c->ugain * vp[q]) - c->gain * fyi[g3];
                        dragz[q] = (-c->ugain * wp[q]) - c->gain * fzi[g3];
                    } else if (t == 3) {
                        fzi[g3] = fzi[g3] + wp[q];
                        dragz[q] = -c->ugain * wp[q] - c->gain * fzi[g3];
                    } else if (t == 11) {
                        dragx[q] = 1.0;
                    } else if (t == 0 && c->p.flow_select == 1) {
                        vwx[q] = vwx[q] - c->dPdx;
                    }
                    if (scal) {
                        if (c->p.scl_flag >= 2) vc[q] = vc[q] + c->scsource[g3] / dt;
                        if (c->p.scalar_q != 0.0) vc[q] = vc[q] + c->p.scalar_q;
                    }
                    /* 5x5 force spreading, solvers.f90:3069-3108.  The j-range test of the reference
                     * (j >= 3 .or. j <= mz-2) is always true, so targets j+jj fall outside 1..mz and
                     * land in the neighbouring x column of the column-major plane; targets outside the
                     * plane array itself are dropped here.  With ib_spread_all (no counterpart in the
                     * reference) every plane spreads once any solid cell exists. */
                    if ((c->p.ib_spread_all && kmaxsurf > 0) || i + 1 <= kmaxsurf) {
                        for (int ii = -2; ii <= 2; ++ii) {
                            int ipii = k + ii;
                            int idif = 1 + abs(ii);
                            if (ipii < 1) ipii += mx;
                            if (ipii > mx) ipii -= mx;
                            for (int jj = -2; jj <= 2; ++jj) {
                                int jdif = 1 + abs(jj);
                                double segdrag = c->fspread[idif - 1][jdif - 1];
                                long jpjj = j + jj;
                                long flat = (jpjj - 1) + (long)(ipii - 1) * mz;
                                if (flat < 0 || flat >= (long)mz * mx) continue;
                                vwx[flat] += segdrag * dragx[q];
                                vwy[flat] += segdrag * dragy[q];
                                vwz[flat] += segdrag * dragz[q];
                            }
                        }
                    }
                }
            c->cfl[i] = cfli;
            for (int k = 0; k < mx; ++k)
                for (int j = 0; j < mz; ++j) {
                    size_t g = PIDX(c, i, j, k), q = (size_t)k * mz + j;
                    up3d[g] = up[q]; vp3d[g] = vp[q]; wp3d[g] = wp[q];
                    if (inertial)
                        for (int m = 0; m < 15; ++m) p3d[m][g] = phys[P_WX + m][q];
                }
            /* x r2c, z c2c forward, truncate and scale: solvers.f90:3147-3273 */
            for (int o = 0; o < nout; o += 2) {
                int sa = out_slot[o], sb = (o + 1 < nout) ? out_slot[o + 1] : -1;
                for (int j = 0; j < mz; ++j) {
                    for (int k = 0; k < mx; ++k) {
                        rowa[k] = op[sa][(size_t)k * mz + j];
                        if (sb >= 0) rowb[k] = op[sb][(size_t)k * mz + j];
                    }
                    r2c_pair(&c->pmx, rowa, sb >= 0 ? rowb : NULL, ra, sb >= 0 ? rb : NULL, w1, w2);
                    for (int k = 0; k < hx; ++k) {
                        os[sa][(size_t)j * hx + k] = ra[k];
                        if (sb >= 0) os[sb][(size_t)j * hx + k] = rb[k];
                    }
                }
            }
            for (int o = 0; o < nout; ++o) {
                int s = out_slot[o];
                for (int k = 0; k < nxh; ++k) {
                    for (int j = 0; j < mz; ++j) w1[j] = os[s][(size_t)j * hx + k];
                    fft_exec(&c->pmz, w1, w2, -1);
                    for (int j = 1; j <= nz; ++j) {
                        int jj = (j <= nzh) ? j : (mz - nz) + j;
                        yout[o][SIDX(c, i, j - 1, k)] =
                            creal(w1[jj - 1]) / (double)(mx * mz) + I * (cimag(w1[jj - 1]) / (double)(mx * mz));
                    }
                }
            }
        }
        for (int f = 0; f < nin; ++f) { free(spec[in_slot[f]]); free(phys[in_slot[f]]); }
        for (int s = 0; s < O_NOUT; ++s) { free(op[s]); free(os[s]); }
        free(dragx); free(dragy); free(dragz); free(w1); free(w2); free(ra); free(rb); free(rowa); free(rowb);
    }

    /* DCT-I back, /ny, halve first and last: solvers.f90:3279-3416 */
#pragma omp parallel
    {
        cplx *o = malloc(sizeof(cplx) * nyp), *w1 = malloc(sizeof(cplx) * 2 * ny), *w2 = malloc(sizeof(cplx) * 2 * ny);
#pragma omp for collapse(2)
        for (int f = 0; f < nout; ++f)
            for (int col = 0; col < nz * nxh; ++col) {
                dct1_c(&c->py2, yout[f] + (size_t)col * nyp, o, w1, w2);
                cplx *dst = outp[f] + (size_t)col * nyp;
                for (int i = 0; i < nyp; ++i) dst[i] = (creal(o[i]) + I * cimag(o[i])) / (double)ny;
                dst[0] = dst[0] / 2.0;
                dst[nyp - 1] = dst[nyp - 1] / 2.0;
            }
        free(o); free(w1); free(w2);
    }
    for (int f = 0; f < nin; ++f) free(yin[f]);
    for (int f = 0; f < nout; ++f) free(yout[f]);
    free(yin); free(yout);

    /* tracers, solvers.f90:3463-3476 */
    int st = KMM_OK;
    if (c->p.npart > 0) {
        if (it == c->p.irstrt) st = orc_init_part(c);
        else if (inertial) st = orc_inertial_update(c);
        else st = orc_tracer_update(c);
        if (inertial) {
            /* u_old = up3d, ..., Lwnm1 = Lwp3d after part_track (solvers.f90:3469-3476) */
            static const int cur[6] = {KMM_UP3D, KMM_VP3D, KMM_WP3D, KMM_LUP3D, KMM_LVP3D, KMM_LWP3D};
            for (int m = 0; m < 6; ++m) orc_copy(c, KMM_UOLD + m, cur[m]);
            /* particle CFL, part_track.f90:213-222 (umax1 keeps its value between calls) */
            c->stats.pumax = c->umax1;
            c->stats.pcfl = c->umax1 * c->dt / c->p.ap;
            if (st == KMM_OK && c->stats.pcfl >= 10.0) st = KMM_ERR_PCFL;
        }
    }
    /* mean u profile, solvers.f90:3487-3495 */
    if (c->p.flow_select == 1 || c->p.flow_select == 4) {
        double *uxm = RF(c, KMM_UXMEAN);
        for (int i = 0; i < nyp; ++i) {
            double s = 0.0;
            for (int k = 0; k < mx; ++k) {
                double sz = 0.0;
                for (int j = 0; j < mz; ++j) sz += up3d[PIDX(c, i, j, k)];
                s += sz / (double)mz;
            }
            uxm[i] = s / (double)mx;
        }
    }
    /* CFL check, solvers.f90:3497-3514 */
    double cflmax = 0.0, umax = 0.0;
    for (int i = 0; i < nyp; ++i)
        if (c->cfl[i] > cflmax) cflmax = c->cfl[i];
    for (size_t x = 0; x < (size_t)nyp * mz * mx; ++x)
        if (fabs(up3d[x]) > umax) umax = fabs(up3d[x]);
    c->stats.cflmax = cflmax;
    c->stats.umax = umax;
    if (st == KMM_OK && cflmax > 1.0) st = KMM_ERR_CFL;
    if (st == KMM_OK && !(cflmax == cflmax)) st = KMM_ERR_NAN;
    c->stats.status = st;
    return st;
}

/* ------------------------------------------------------------------------- */
/* main_dns.f90: initial + time loop body                                     */
/* ------------------------------------------------------------------------- */
static void norm_list(orc_ctx *c, const int *ids, int n)
{
    for (int m = 0; m < n; ++m) norm_arr(c, SF(c, ids[m]));
}

static void poly_norm_c(orc_ctx *c)
{
    for (int m = 0; m < 9; ++m) norm_arr(c, SF(c, KMM_C11 + m));
}

static void poly_norm_dc(orc_ctx *c)
{
    for (int m = 0; m < 27; ++m) norm_arr(c, SF(c, KMM_DC111 + m));
}

static void poly_norm_out(orc_ctx *c)
{
    poly_norm_c(c);
    for (int m = 0; m < 6; ++m) norm_arr(c, SF(c, KMM_C11N + m));
    for (int m = 0; m < 6; ++m) norm_arr(c, SF(c, KMM_STR11N + m));
    static const int q[6] = {KMM_QP11, KMM_QP12, KMM_QP13, KMM_QP22, KMM_QP23, KMM_QP33};
    norm_list(c, q, 6);
}

/* constant conformation tensor, main_dns.f90:206-235 (xyzfft of a constant keeps only the (0,0) mode 0) */
static void poly_set_constant(orc_ctx *c)
{
    double cz[9] = {c->p.c11z, 0, 0, 0, c->p.c22z, 0, 0, 0, c->p.c33z};
    double *b = RF(c, KMM_INITSCL); /* scratch physical array reused through a private copy */
    const size_t np = (size_t)c->nyp * c->nz * c->nx;
    double *save = malloc(sizeof(double) * np);
    memcpy(save, b, sizeof(double) * np);
    for (int m = 0; m < 9; ++m) {
        for (size_t x = 0; x < np; ++x) b[x] = cz[m];
        orc_xyzfft(c, KMM_C11 + m, KMM_INITSCL);
    }
    memcpy(b, save, sizeof(double) * np);
    free(save);
}

/* gfcn + denominator (main_dns.f90:151-161), then initial(...), main_dns.f90:1602-2231, irstrt = 0 branch */
/* `initial` with irstrt >= 1 (main_dns.f90:1742-1917).  The host has already placed the two
 * records of setup/restart (v, fn, fnm1, omy, gn, gnm1, u0, h1n, h1nm1, w0, h3n, h3nm1;
 * fxintg, fyintg, fzintg) and, with the scalar and polymer modules and crstrt = 1, the five
 * records of setup/c-restart.  None of those is normalised or recomputed; only the scalar and
 * polymer start values are set as the reference sets them:
 *   scalar only      : scalar and csource from setscl, NOT normalised (main_dns.f90:1810-1815)
 *   scalar + polymer : crstrt = 0: setpoly, the scalar gradient and the conformation-tensor
 *                      derivatives (normalised), and zero scn, cIJn, strIJn, qpIJ
 *                      (main_dns.f90:1817-1908); crstrt = 1: all from c-restart (1909-1916).
 * csource is zero at the start of the reference program and the crstrt = 1 branch leaves it so. */
static int orc_initial_restart(orc_ctx *c)
{
    if (!c->p.scalar_on) return 0;
    orc_zero(c, KMM_CSOURCE);
    if (c->p.polymer_on && c->p.crstrt != 0) return 0;   /* everything from c-restart */
    orc_xyzfft(c, KMM_SCALAR, KMM_INITSCL);
    if (!c->p.polymer_on) return 0;
    poly_set_constant(c);
    orc_gradscl(c);
    { int l[3] = {KMM_SCLX, KMM_SCLY, KMM_SCLZ}; norm_list(c, l, 3); }
    orc_derivscji(c);
    poly_norm_c(c);
    poly_norm_dc(c);
    orc_zero(c, KMM_SCN);
    for (int m = 0; m < 6; ++m) {
        orc_zero(c, KMM_C11N + m);
        orc_zero(c, KMM_STR11N + m);
        orc_zero(c, KMM_QP11 + m);
    }
    return 0;
}

int orc_initial(orc_ctx *c)
{
    const int nyp = c->nyp;
    const size_t n = (size_t)nyp * c->nz * c->nxh;
    /* setup part of the main program: Green's functions before initial, main_dns.f90:151-161 */
    orc_gfcn(c);
    c->it = 0;
    if (c->p.irstrt >= 1) return orc_initial_restart(c);
    orc_xyzfft(c, KMM_U, KMM_INITU);
    orc_xyzfft(c, KMM_V, KMM_INITV);
    orc_xyzfft(c, KMM_W, KMM_INITW);
    if (c->p.scalar_on) {
        orc_xyzfft(c, KMM_SCALAR, KMM_INITSCL);
        orc_zero(c, KMM_CSOURCE);
    }
    if (c->p.polymer_on) poly_set_constant(c);
    cplx *u = SF(c, KMM_U), *v = SF(c, KMM_V), *w = SF(c, KMM_W), *omy = SF(c, KMM_OMY);
    for (int k = 0; k < c->nxh; ++k)
        for (int j = 0; j < c->nz; ++j)
            for (int i = 0; i < nyp; ++i) {
                size_t x = SIDX(c, i, j, k);
                omy[x] = I * c->wavz[j] * u[x] - I * c->wavx[k] * w[x];
            }
    for (int i = 0; i < nyp; ++i) omy[SIDX(c, i, 0, 0)] = 0.0;
    int l1[4] = {KMM_U, KMM_V, KMM_W, KMM_OMY};
    norm_list(c, l1, 4);
    if (c->p.scalar_on) { int l[2] = {KMM_SCALAR, KMM_CSOURCE}; norm_list(c, l, 2); }
    if (c->p.polymer_on) poly_norm_c(c);
    double *u0 = RF(c, KMM_U0), *w0 = RF(c, KMM_W0);
    for (int i = 0; i < nyp; ++i) { u0[i] = creal(u[SIDX(c, i, 0, 0)]); w0[i] = creal(w[SIDX(c, i, 0, 0)]); }
    for (int i = 0; i < nyp; ++i) {
        u[SIDX(c, i, 0, 0)] = u0[i];
        v[SIDX(c, i, 0, 0)] = 0.0;
        w[SIDX(c, i, 0, 0)] = w0[i];
    }
    norm_list(c, l1, 4);
    orc_vort(c);
    { int l[2] = {KMM_OMX, KMM_OMZ}; norm_list(c, l, 2); }
    if (c->p.scalar_on) {
        orc_gradscl(c);
        int l[3] = {KMM_SCLX, KMM_SCLY, KMM_SCLZ};
        norm_list(c, l, 3);
    }
    orc_gradv(c);
    { int l[12] = {KMM_U11, KMM_U12, KMM_U13, KMM_U21, KMM_U22, KMM_U23, KMM_U31, KMM_U32, KMM_U33, KMM_LU, KMM_LV, KMM_LW};
      norm_list(c, l, 12); }
    if (c->p.polymer_on) {
        orc_derivscji(c);
        poly_norm_c(c);
        poly_norm_dc(c);
    }
    int st = orc_vcw3dp(c);
    { int l[5] = {KMM_V, KMM_OMY, KMM_FN, KMM_GN, KMM_OMZ}; norm_list(c, l, 5); }
    if (c->p.polymer_on) {
        poly_norm_out(c);
        if (c->it >= c->p.src_start) {
            orc_polyforce(c);
            int l[3] = {KMM_T1, KMM_T2, KMM_T3};
            norm_list(c, l, 3);
            orc_subforce(c);
        }
    }
    if (c->p.scalar_on && c->p.src_start == 0) {
        cplx *scn = SF(c, KMM_SCN), *cs = SF(c, KMM_CSOURCE);
        for (size_t x = 0; x < n; ++x) scn[x] = scn[x] + cs[x];
    }
    double *h1n = RF(c, KMM_H1N), *h3n = RF(c, KMM_H3N);
    cplx *gn = SF(c, KMM_GN), *omz = SF(c, KMM_OMZ);
    for (int i = 0; i < nyp; ++i) { h1n[i] = creal(gn[SIDX(c, i, 0, 0)]); h3n[i] = creal(omz[SIDX(c, i, 0, 0)]); }
    orc_nonlin(c);
    { int l[2] = {KMM_FN, KMM_GN}; norm_list(c, l, 2); }
    if (c->p.scalar_on) norm_arr(c, SF(c, KMM_SCN));
    orc_copy(c, KMM_FNM1, KMM_FN);
    orc_copy(c, KMM_GNM1, KMM_GN);
    if (c->p.scalar_on) orc_copy(c, KMM_SCNM1, KMM_SCN);
    if (c->p.polymer_on) {
        for (int m = 0; m < 6; ++m) { orc_copy(c, KMM_C11NM1 + m, KMM_C11N + m); orc_copy(c, KMM_STR11NM1 + m, KMM_STR11N + m); }
    }
    orc_copy(c, KMM_H1NM1, KMM_H1N);
    orc_copy(c, KMM_H3NM1, KMM_H3N);
    return st;
}

/* one iteration of `do it = 1,nsteps`, main_dns.f90:198-811 */
int orc_step(orc_ctx *c)
{
    const int nyp = c->nyp;
    const double re = c->re, dt = c->dt, th = c->theta;
    c->it += 1;
    const int it = c->it;
    if (c->p.polymer_on) {
        if (it == c->p.src_start - 1 || (it == c->p.irstrt && c->p.crstrt == 0)) poly_set_constant(c);
        if (it >= c->p.src_start) {
            orc_polynl(c);
            for (int m = 0; m < 6; ++m) {
                /* phirhs(cIJ, ..., cIJNL, 2.0*cIJNL, ..., diffpoly), main_dns.f90:248-261 */
                int tmp = KMM_NSPECTRAL + 6 + m;
                const size_t n = (size_t)nyp * c->nz * c->nxh;
                if (!c->fld[tmp]) c->fld[tmp] = calloc(n, sizeof(cplx));
                cplx *nl = g_polynl_scratch(c, m), *nl2 = (cplx *)c->fld[tmp];
                for (size_t x = 0; x < n; ++x) nl2[x] = 2.0 * nl[x];
                /* phirhs reads fn / fnm1 by field id: point the scratch ids at them */
                orc_phirhs(c, poly_comp[m], KMM_NSPECTRAL + m, tmp, c->p.diffpoly);
            }
            for (int m = 0; m < 6; ++m) { orc_copy(c, KMM_C11NM1 + m, KMM_C11N + m); orc_copy(c, KMM_STR11NM1 + m, KMM_STR11N + m); }
            double g = (re * c->p.diffpoly) / (dt * th);
            orc_zero(c, KMM_BCTOP);
            orc_zero(c, KMM_BCBOT);
            for (int m = 0; m < 6; ++m) orc_penta(c, poly_comp[m], g, 0, 0.0, 1.0, 0.0, 1.0);
            for (int m = 0; m < 6; ++m) norm_arr(c, SF(c, poly_comp[m]));
            orc_copy(c, KMM_C21, KMM_C12);
            orc_copy(c, KMM_C31, KMM_C13);
            orc_copy(c, KMM_C32, KMM_C23);
        }
    }
    if (c->p.scalar_on) {
        orc_phirhs(c, KMM_SCALAR, KMM_SCN, KMM_SCNM1, c->p.diff);
        orc_copy(c, KMM_SCNM1, KMM_SCN);
        double g = (re * c->p.diff) / (dt * th);
        /* bcscltop = bcsclbot = 0 (main_dns.f90:39) */
        orc_zero(c, KMM_BCTOP);
        orc_zero(c, KMM_BCBOT);
        if (c->p.scalar_bc == 1) orc_penta(c, KMM_SCALAR, g, 0, 1.0, 0.0, 1.0, 0.0);
        else orc_penta(c, KMM_SCALAR, g, 0, 0.0, 1.0, 0.0, 1.0);
    }
    orc_phi_from_v(c);
    orc_phirhs(c, KMM_V, KMM_FN, KMM_FNM1, 1.0);
    orc_copy(c, KMM_FNM1, KMM_FN);
    orc_solve(c, KMM_V, re / (dt * th), 0);
    orc_solve(c, KMM_V, 0.0, 0);
    orc_phirhs(c, KMM_OMY, KMM_GN, KMM_GNM1, 1.0);
    orc_copy(c, KMM_GNM1, KMM_GN);
    orc_influence(c);
    orc_penta(c, KMM_OMY, re / (dt * th), 0, c->atu, c->btu, c->abu, c->bbu);
    orc_uzero(c, 1);
    frate_apply(c);
    orc_uzero(c, 3);
    cplx *omy = SF(c, KMM_OMY);
    for (int i = 0; i < nyp; ++i) omy[SIDX(c, i, 0, 0)] = 0.0;
    orc_copy(c, KMM_H1NM1, KMM_H1N);
    orc_copy(c, KMM_H3NM1, KMM_H3N);
    { int l[2] = {KMM_V, KMM_OMY}; norm_list(c, l, 2); }
    orc_veloc(c);
    { int l[2] = {KMM_U, KMM_W}; norm_list(c, l, 2); }
    orc_vort(c);
    { int l[2] = {KMM_OMX, KMM_OMZ}; norm_list(c, l, 2); }
    if (c->p.scalar_on) {
        norm_arr(c, SF(c, KMM_SCALAR));
        orc_gradscl(c);
        int l[3] = {KMM_SCLX, KMM_SCLY, KMM_SCLZ};
        norm_list(c, l, 3);
    }
    orc_gradv(c);
    { int l[12] = {KMM_U11, KMM_U12, KMM_U13, KMM_U21, KMM_U22, KMM_U23, KMM_U31, KMM_U32, KMM_U33, KMM_LU, KMM_LV, KMM_LW};
      norm_list(c, l, 12); }
    if (c->p.polymer_on) {
        orc_derivscji(c);
        poly_norm_c(c);
        poly_norm_dc(c);
    }
    int st = orc_vcw3dp(c);
    { int l[5] = {KMM_V, KMM_OMY, KMM_FN, KMM_GN, KMM_OMZ}; norm_list(c, l, 5); }
    if (c->p.scalar_on) { int l[2] = {KMM_SCALAR, KMM_SCN}; norm_list(c, l, 2); }
    if (c->p.polymer_on) {
        if (it >= c->p.src_start - 1) poly_norm_out(c);
        if (it >= c->p.src_start) {
            orc_polyforce(c);
            int l[3] = {KMM_T1, KMM_T2, KMM_T3};
            norm_list(c, l, 3);
            orc_subforce(c);
        }
    }
    orc_filter(c);
    double *h1n = RF(c, KMM_H1N), *h3n = RF(c, KMM_H3N);
    cplx *gn = SF(c, KMM_GN), *omz = SF(c, KMM_OMZ);
    for (int i = 0; i < nyp; ++i) { h1n[i] = creal(gn[SIDX(c, i, 0, 0)]); h3n[i] = creal(omz[SIDX(c, i, 0, 0)]); }
    { int l[3] = {KMM_FN, KMM_GN, KMM_OMZ}; norm_list(c, l, 3); }
    orc_nonlin(c);
    { int l[2] = {KMM_FN, KMM_GN}; norm_list(c, l, 2); }
    if (c->p.scalar_on) norm_arr(c, SF(c, KMM_SCN));
    return st;
}

int orc_run(orc_ctx *c, int n)
{
    for (int s = 0; s < n; ++s) {
        int st = orc_step(c);
        if (st) return st;
    }
    return KMM_OK;
}

/* ------------------------------------------------------------------------- */
/* swirl strength (diagnostic), helpers.f90:197-404                           */
/* ------------------------------------------------------------------------- */
/* eig (helpers.f90:197-275): Cardano's closed form of the eigenvalues of the 3x3 velocity-gradient
 * matrix in complex arithmetic, restated term by term: tr = trace, P = (tr^2 - 3 M2)/9 with M2 the
 * sum of the principal 2x2 minors, Q = tr^3/27 - tr M2/6 + det/2, S = (Q + (Q^2 - P^3)^(1/2))^(1/3)
 * (principal powers, as the Fortran complex ** real), then
 *   l1 = tr/3 + P/S + S,  l2,3 = tr/3 -+ sqrt(3)(P/S - S) i/2 - P/(2S) - S/2.
 * calcswirl (helpers.f90:339-404): swirl = sqrt(Im l1^2 + Im l2^2 + Im l3^2), and 0 where that is
 * not a finite positive number (the reference's floor(swirl/swirl) /= 1 test). */
static double swirl_point(double r11, double r12, double r13, double r21, double r22, double r23, double r31,
                          double r32, double r33)
{
    const cplx u11 = r11, u12 = r12, u13 = r13, u21 = r21, u22 = r22, u23 = r23, u31 = r31, u32 = r32, u33 = r33;
    const cplx tr = u11 + u22 + u33;
    const cplx P = tr * tr / 9.0 - (u11 * u22) / 3.0 + (u12 * u21) / 3.0 - (u11 * u33) / 3.0 + (u13 * u31) / 3.0 -
                   (u22 * u33) / 3.0 + (u23 * u32) / 3.0;
    const cplx M2 = u11 * u22 - u12 * u21 + u11 * u33 - u13 * u31 + u22 * u33 - u23 * u32;
    const cplx Q = tr * tr * tr / 27.0 - (tr * M2) / 6.0 + (u11 * u22 * u33) / 2.0 - (u11 * u23 * u32) / 2.0 -
                   (u12 * u21 * u33) / 2.0 + (u12 * u23 * u31) / 2.0 + (u13 * u21 * u32) / 2.0 -
                   (u13 * u22 * u31) / 2.0;
    const cplx S = cpow(Q + cpow(Q * Q - P * P * P, 0.5), 1.0 / 3.0);
    const cplx PS = P / S;
    const cplx l1 = tr / 3.0 + PS + S;
    const cplx rot = (sqrt(3.0) * (PS - S) * I) / 2.0;
    const cplx l2 = tr / 3.0 - rot - PS / 2.0 - S / 2.0;
    const cplx l3 = tr / 3.0 + rot - PS / 2.0 - S / 2.0;
    const double a = cimag(l1), b = cimag(l2), d = cimag(l3);
    double sw = sqrt(a * a + b * b + d * d);
    if (!(sw > 0.0 && sw <= DBL_MAX)) sw = 0.0;
    return sw;
}

/* calcswirl: the nine velocity gradients u11..u33 (spectral, from gradv) to physical space on the
 * 3/2 grid with the transforms of vcw3dp (solvers.f90:2241-2879), swirl at every point into
 * SWIRL3D (nyp,mz,mx) (solvers.f90:3421), and its value at each particle into SWIRLPART
 * (fluid_interp1, solvers.f90:3480). */
/* one spectral field (nyp,nz,nxh) to physical values on the 3/2 grid (nyp,mz,mx), with the
 * transforms of vcw3dp: c(i)/2 scaling and DCT-I along y (solvers.f90:2241-2546), zero-padded
 * inverse c2c along z and c2r along x (solvers.f90:2578-2879) */
static void to_phys3d(orc_ctx *c, const cplx *src, double *phys)
{
    const int nyp = c->nyp, nz = c->nz, nxh = c->nxh, mx = c->mx, mz = c->mz, ny = c->ny, nzh = c->nzh;
    const size_t nspec = (size_t)nyp * nz * nxh;
    const int hx = mx / 2 + 1;
    cplx *yin = malloc(sizeof(cplx) * nspec);
#pragma omp parallel
    {
        cplx *x = malloc(sizeof(cplx) * nyp), *o = malloc(sizeof(cplx) * nyp);
        cplx *w1 = malloc(sizeof(cplx) * 2 * ny), *w2 = malloc(sizeof(cplx) * 2 * ny);
#pragma omp for
        for (int col = 0; col < nz * nxh; ++col) {
            const cplx *sp = src + (size_t)col * nyp;
            for (int i = 0; i < nyp; ++i) {
                double fac = c->c[i] / 2.0;
                x[i] = creal(sp[i]) * fac + I * (cimag(sp[i]) * fac);
            }
            dct1_c(&c->py2, x, o, w1, w2);
            memcpy(yin + (size_t)col * nyp, o, sizeof(cplx) * nyp);
        }
        free(x); free(o); free(w1); free(w2);
    }
#pragma omp parallel
    {
        int wl = mx > mz ? mx : mz;
        cplx *w1 = malloc(sizeof(cplx) * wl), *w2 = malloc(sizeof(cplx) * wl);
        cplx *s = malloc(sizeof(cplx) * (size_t)mz * hx);
        double *row = malloc(sizeof(double) * mx);
#pragma omp for
        for (int i = 0; i < nyp; ++i) {
            memset(s, 0, sizeof(cplx) * (size_t)mz * hx);
            for (int k = 0; k < nxh; ++k) {
                for (int j = 0; j < mz; ++j) w1[j] = 0.0;
                for (int j = 1; j <= nz; ++j) {
                    int jj = (j <= nzh) ? j : (mz - nz) + j;
                    w1[jj - 1] = yin[SIDX(c, i, j - 1, k)];
                }
                fft_exec(&c->pmz, w1, w2, +1);
                for (int j = 0; j < mz; ++j) s[(size_t)j * hx + k] = w1[j];
            }
            for (int j = 0; j < mz; ++j) {
                c2r_pair(&c->pmx, s + (size_t)j * hx, NULL, row, NULL, w1, w2);
                for (int k = 0; k < mx; ++k) phys[PIDX(c, i, j, k)] = row[k];
            }
        }
        free(w1); free(w2); free(s); free(row);
    }
    free(yin);
}

int orc_calcswirl(orc_ctx *c)
{
    const size_t nphys = (size_t)c->nyp * c->mz * c->mx;
    double *phys[9];
    for (int m = 0; m < 9; ++m) {
        phys[m] = malloc(sizeof(double) * nphys);
        to_phys3d(c, SF(c, KMM_U11 + m), phys[m]);
    }
    double *sw = RF(c, KMM_SWIRL3D);
#pragma omp parallel for schedule(dynamic, 4096)
    for (size_t q = 0; q < nphys; ++q)
        sw[q] = swirl_point(phys[0][q], phys[1][q], phys[2][q], phys[3][q], phys[4][q], phys[5][q], phys[6][q],
                            phys[7][q], phys[8][q]);
    int st = KMM_OK;
    if (c->p.npart > 0) {
        const double *xp = RF(c, KMM_XPART), *yp = RF(c, KMM_YPART), *zp = RF(c, KMM_ZPART);
        double *spart = RF(c, KMM_SWIRLPART);
        for (int n = 0; n < c->p.npart; ++n) {
            double a, b;
            if (fluid_interp(c, xp[n], yp[n], zp[n], sw, sw, sw, &spart[n], &a, &b)) st = KMM_ERR_INTERP;
        }
    }
    for (int m = 0; m < 9; ++m) free(phys[m]);
    return st;
}

/* Flow statistics of writeoutputs (helpers.f90:1227-1438) from the current state: veloc, then
 * u, v, w and u12 = du/dy on the 3/2 grid, and the reference's loops: the mean profile (the
 * uxmean of solvers.f90:3486-3494), u'_rms, v_rms, w_rms, R12 = <u'v>, T12 = <u12>/re, the bulk
 * velocity by the trapezoid of helpers.f90:1355-1359, the top / bottom wall shear <u12>/re at
 * y index 1 / nyp.  Added (not in the reference): the kinetic-energy profile 0.5 <u^2+v^2+w^2>
 * and its bulk value by the same trapezoid.
 *   prof[7][nyp] = umean, urms, vrms, wrms, R12, T12, ke;  scal[4] = massflux, tau_top, tau_bot, ke_bulk */
int orc_flowstats(orc_ctx *c, double *prof, double *scal)
{
    const int nyp = c->nyp, mz = c->mz, mx = c->mx;
    const size_t nphys = (size_t)nyp * mz * mx, nspec = (size_t)nyp * c->nz * c->nxh;
    int st = orc_veloc(c);
    if (st) return st;
    cplx *du = malloc(sizeof(cplx) * nspec);
    cderiv_arr(c, SF(c, KMM_U), du);
    double *u = malloc(sizeof(double) * nphys), *v = malloc(sizeof(double) * nphys);
    double *w = malloc(sizeof(double) * nphys), *u12 = malloc(sizeof(double) * nphys);
    to_phys3d(c, SF(c, KMM_U), u);
    to_phys3d(c, SF(c, KMM_V), v);
    to_phys3d(c, SF(c, KMM_W), w);
    to_phys3d(c, du, u12);
    free(du);
    double *umean = prof, *urms = prof + nyp, *vrms = prof + 2 * nyp, *wrms = prof + 3 * nyp;
    double *R12 = prof + 4 * nyp, *T12 = prof + 5 * nyp, *ke = prof + 6 * nyp;
    const double re = c->re, nm = (double)mx * (double)mz;
    for (int i = 0; i < nyp; ++i) {
        double s = 0.0;
        for (int k = 0; k < mx; ++k) {
            double sz = 0.0;
            for (int j = 0; j < mz; ++j) sz += u[PIDX(c, i, j, k)];
            s += sz / mz;
        }
        umean[i] = s / mx;
    }
    for (int i = 0; i < nyp; ++i) {
        double a = 0.0, b = 0.0, d = 0.0, r = 0.0, t = 0.0, e = 0.0;
        for (int k = 0; k < mx; ++k)
            for (int j = 0; j < mz; ++j) {
                const size_t q = PIDX(c, i, j, k);
                const double up = u[q] - umean[i];
                a += up * up;
                b += v[q] * v[q];
                d += w[q] * w[q];
                r += up * v[q];
                t += u12[q] / re;
                e += 0.5 * (u[q] * u[q] + v[q] * v[q] + w[q] * w[q]);
            }
        urms[i] = sqrt(a / nm);
        vrms[i] = sqrt(b / nm);
        wrms[i] = sqrt(d / nm);
        R12[i] = r / nm;
        T12[i] = t / nm;
        ke[i] = e / nm;
    }
    double mf = 0.0, kb = 0.0;
    for (int i = 0; i < nyp - 1; ++i) {
        const double dy = fabs(c->ycoord[i + 1] - c->ycoord[i]);
        mf += 1.0 / c->yl * 0.5 * (umean[i + 1] + umean[i]) * dy;
        kb += 1.0 / c->yl * 0.5 * (ke[i + 1] + ke[i]) * dy;
    }
    scal[0] = mf;
    scal[1] = T12[0];
    scal[2] = T12[nyp - 1];
    scal[3] = kb;
    free(u); free(v); free(w); free(u12);
    return KMM_OK;
}
