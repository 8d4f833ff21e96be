// kmm_column.cu -- per-(kx,kz)-column routines of solvers.f90 / derivatives.f90 / helpers.f90.
//
// Spectral fields are complex(8) (nyp,nz,nxh), y fastest: column col = k*nz + j holds the nyp
// Chebyshev coefficients of wavenumber pair (kx = wavx(k), kz = wavz(j)) contiguously, so a tile
// of TILE consecutive columns is one contiguous block of TILE*nyp double2 -> fully coalesced
// loads and stores.  The y recurrences (Chebyshev derivative, tau eliminations) run with one
// thread per column on the tile in shared memory, in the reference's own operation order.
// This file is compiled with -fmad=false so those recurrences round like the reference's
// separate multiply / add sequence.
#include <math.h>

#include "kmm_internal.cuh"

#define TILE 16
#define TPB 128

static inline size_t tile_smem(int nyp, int nbuf) { return sizeof(double2) * (size_t)TILE * nyp * nbuf; }

__device__ __forceinline__ void tile_load(double2 *s, const double2 *__restrict__ g, int col0, int ncol, int nyp) {
    const size_t n = (size_t)ncol * nyp;
    const double2 *src = g + (size_t)col0 * nyp;
    for (size_t e = threadIdx.x; e < n; e += blockDim.x) s[e] = src[e];
}

__device__ __forceinline__ void tile_store(double2 *__restrict__ g, const double2 *s, int col0, int ncol, int nyp) {
    const size_t n = (size_t)ncol * nyp;
    double2 *dst = g + (size_t)col0 * nyp;
    for (size_t e = threadIdx.x; e < n; e += blockDim.x) dst[e] = s[e];
}

// ---------------------------------------------------------------------------
// cderiv(f,df), derivatives.f90:258-314: two independent parity chains per column
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TPB) k_cderiv(const double2 *__restrict__ f, double2 *__restrict__ df, int ncols,
                                                int nyp, double dyde) {
    extern __shared__ double2 sm[];
    double2 *sf = sm, *sd = sm + (size_t)TILE * nyp;
    const int col0 = blockIdx.x * TILE;
    const int ncol = min(TILE, ncols - col0);
    tile_load(sf, f, col0, ncol, nyp);
    __syncthreads();
    const int t = threadIdx.x;
    if (t < 2 * ncol) {
        const int cl = t >> 1, par = t & 1;
        const double2 *F = sf + (size_t)cl * nyp;
        double2 *D = sd + (size_t)cl * nyp;
        const int ny = nyp - 1;
        double2 acc;
        int idx;
        if (par == (ny & 1)) {          // chain through index ny: D[ny] = 0
            acc = make_double2(0.0, 0.0);
            D[ny] = acc;
            idx = ny - 2;
        } else {                        // chain through ny-1: D[ny-1] = 2 ny F[ny] dyde
            double s = 2.0 * (double)ny;
            acc = make_double2(s * F[ny].x * dyde, s * F[ny].y * dyde);
            D[ny - 1] = acc;
            idx = ny - 3;
        }
        for (; idx >= 0; idx -= 2) {    // D[idx] = D[idx+2] + 2 (idx+1) F[idx+1] dyde
            double s = 2.0 * (double)(idx + 1);
            double2 fv = F[idx + 1];
            acc = make_double2(acc.x + s * fv.x * dyde, acc.y + s * fv.y * dyde);
            D[idx] = acc;
        }
        if (par == 0) D[0] = make_double2(0.5 * D[0].x, 0.5 * D[0].y);
    }
    __syncthreads();
    tile_store(df, sd, col0, ncol, nyp);
}

// The same two chains with a half-warp per column for ny = 16 K: lane t holds the K consecutive
// coefficients t K .. t K + K - 1 in registers and the chains run lane by lane from the top, the
// carries D[(t+1) K] and D[(t+1) K + 1] handed down by shuffles, so every D[i] is the same sum in
// the same order as above (bitwise equal) while the columns keep the whole SM busy.  The block's
// 8 columns (one contiguous run in global memory) pass through shared memory with coalesced loads
// and stores; coefficient i sits at i + i / K there, so a lane's K values start K + 1 slots after
// its neighbour's and the 16 lanes' accesses spread over the banks.
// up to KMM_CDERIV_BATCH independent (input, output) pairs per launch, blockIdx.y picking the pair
struct CderivList {
    const double2 *f[KMM_CDERIV_BATCH];
    double2 *df[KMM_CDERIV_BATCH];
};

template <int K>
__global__ void __launch_bounds__(128) k_cderiv_hw(CderivList list, int ncols, double dyde) {
    constexpr int NY = 16 * K, NYP = NY + 1, SK = K + 1, CS = 16 * SK + 1;
    __shared__ double2 s[8 * CS];
    const double2 *f = list.f[blockIdx.y];
    double2 *df = list.df[blockIdx.y];
    const int col0 = blockIdx.x * 8;
    const int ncb = min(8, ncols - col0);
    const double2 *src = f + (size_t)col0 * NYP;
    {   // every load of the block's columns in flight at once, then into shared memory
        constexpr int NLD = (8 * NYP + 127) / 128;
        double2 tmp[NLD];
#pragma unroll
        for (int u = 0; u < NLD; ++u) {
            const int e = threadIdx.x + 128 * u;
            if (e < ncb * NYP) tmp[u] = src[e];
        }
#pragma unroll
        for (int u = 0; u < NLD; ++u) {
            const int e = threadIdx.x + 128 * u;
            if (e < ncb * NYP) {
                const int c = e / NYP, i = e - c * NYP;
                s[c * CS + i + i / K] = tmp[u];
            }
        }
    }
    __syncthreads();
    const int c = threadIdx.x >> 4, t = threadIdx.x & 15;
    if (c < ncb) {
        // both columns of the warp present -> the full mask; else the present half alone
        const unsigned mask = (c | 1) < ncb ? 0xffffffffu : ((threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu);
        double2 *S = s + c * CS;
        double2 v[K];
#pragma unroll
        for (int m = 0; m < K; ++m) v[m] = S[t * SK + m];
        const double2 ftop = S[16 * SK];
        double2 fnext;   // F[(t+1) K]
        fnext.x = __shfl_down_sync(mask, v[0].x, 1, 16);
        fnext.y = __shfl_down_sync(mask, v[0].y, 1, 16);
        if (t == 15) fnext = ftop;
        // terms of D[j] = D[j+2] + 2 (j+1) F[j+1] dyde, j = t K + m
        double2 w[K];
#pragma unroll
        for (int m = 0; m < K; ++m) {
            const double sc = 2.0 * (double)(t * K + m + 1);
            const double2 fv = m + 1 < K ? v[m + 1] : fnext;
            w[m] = make_double2(sc * fv.x * dyde, sc * fv.y * dyde);
        }
        // carries from above lane 15: D[NY] = 0, and D[NY-1] = 2 NY F[NY] dyde is lane 15's top term
        double2 clo = make_double2(0.0, 0.0), chi = make_double2(0.0, 0.0);
        double2 d[K];
#pragma unroll
        for (int m = 0; m < K; ++m) d[m] = make_double2(0.0, 0.0);
        for (int r = 15; r >= 0; --r) {
            if (t == r) {
                // top two slots from the carries (lane 15: D[NY-1] is its term alone, D[NY-2] = D[NY] + term)
                d[K - 1] = t == 15 ? w[K - 1] : make_double2(chi.x + w[K - 1].x, chi.y + w[K - 1].y);
                d[K - 2] = make_double2(clo.x + w[K - 2].x, clo.y + w[K - 2].y);
#pragma unroll
                for (int m = K - 3; m >= 0; --m) d[m] = make_double2(d[m + 2].x + w[m].x, d[m + 2].y + w[m].y);
            }
            if (r > 0) {
                chi.x = __shfl_sync(mask, d[1].x, r, 16);
                chi.y = __shfl_sync(mask, d[1].y, r, 16);
                clo.x = __shfl_sync(mask, d[0].x, r, 16);
                clo.y = __shfl_sync(mask, d[0].y, r, 16);
            }
        }
        if (t == 0) d[0] = make_double2(0.5 * d[0].x, 0.5 * d[0].y);
        __syncwarp(mask);   // every lane of the column has read its values before they are overwritten
#pragma unroll
        for (int m = 0; m < K; ++m) S[t * SK + m] = d[m];
        if (t == 15) S[16 * SK] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2 *dst = df + (size_t)col0 * NYP;
    for (int e = threadIdx.x; e < ncb * NYP; e += blockDim.x) {
        const int c2 = e / NYP, i = e - c2 * NYP;
        dst[e] = s[c2 * CS + i + i / K];
    }
}

int kmm_internal_cderiv_many(kmm_ctx *ctx, const double2 *const *f, double2 *const *df, int n) {
    const int ncols = ctx->nz * ctx->nxh;
    const int ny = ctx->nyp - 1;
    if (ctx->use_colblk && ny % 16 == 0 && ny >= 32 && (ny <= 128 || ny == 256)) {
        const int nblk = (ncols + 7) / 8;
        for (int p0 = 0; p0 < n; p0 += KMM_CDERIV_BATCH) {
            const int nb = n - p0 < KMM_CDERIV_BATCH ? n - p0 : KMM_CDERIV_BATCH;
            CderivList list;
            for (int m = 0; m < nb; ++m) {
                list.f[m] = f[p0 + m];
                list.df[m] = df[p0 + m];
            }
            const dim3 grid(nblk, nb);
            switch (ny / 16) {
            case 2: k_cderiv_hw<2><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            case 3: k_cderiv_hw<3><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            case 4: k_cderiv_hw<4><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            case 5: k_cderiv_hw<5><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            case 6: k_cderiv_hw<6><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            case 7: k_cderiv_hw<7><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            case 8: k_cderiv_hw<8><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            case 16: k_cderiv_hw<16><<<grid, 128, 0, ctx->stream>>>(list, ncols, ctx->dyde); break;
            }
            CKL();
        }
        return KMM_OK;
    }
    const size_t sm = tile_smem(ctx->nyp, 2);
    RET(kmm_smem_attr(ctx, (const void *)k_cderiv, sm));
    for (int m = 0; m < n; ++m) {
        k_cderiv<<<(ncols + TILE - 1) / TILE, TPB, sm, ctx->stream>>>(f[m], df[m], ncols, ctx->nyp, ctx->dyde);
        CKL();
    }
    return KMM_OK;
}

int kmm_internal_cderiv(kmm_ctx *ctx, const double2 *f, double2 *df) { return kmm_internal_cderiv_many(ctx, &f, &df, 1); }

extern "C" int kmm_cderiv(kmm_ctx *ctx, int f, int df) {
    if (!ctx || f == df) return KMM_ERR_ARG;
    double2 *a = SPEC(ctx, f), *b = SPEC(ctx, df);
    if (!a || !b || f >= KMM_NSPECTRAL || df >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    return kmm_internal_cderiv(ctx, a, b);
}

// ---------------------------------------------------------------------------
// c{0,1,2}der{b,t}w, derivatives.f90:318-653: one warp per column, then the
// partial sums are folded in the reference's index order by lane 0.
// ---------------------------------------------------------------------------
__global__ void k_wallderiv(const double2 *__restrict__ f, double2 *__restrict__ out, int ncols, int nyp, int order,
                            int wall, int iy, double dyde) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= ncols) return;
    const double2 *F = f + (size_t)warp * nyp;
    // each lane accumulates a contiguous chunk in ascending order; chunks are then added in order
    const int chunk = (nyp + 31) / 32;
    const int i0 = lane * chunk, i1 = min(nyp, i0 + chunk);
    double2 acc = make_double2(0.0, 0.0);
    for (int i = i0; i < i1; ++i) {
        double rp = (double)i;
        double sgn = 1.0;
        if (wall == 0) sgn = (order == 0) ? ((i & 1) ? -1.0 : 1.0) : ((i & 1) ? 1.0 : -1.0);
        double2 v = F[i];
        double wgt;
        if (order == 0) {
            acc = make_double2(acc.x + sgn * v.x, acc.y + sgn * v.y);
            continue;
        } else if (order == 1) {
            wgt = rp * rp * sgn;
            acc = make_double2(acc.x + wgt * v.x * dyde, acc.y + wgt * v.y * dyde);
        } else {
            double rp2 = rp * rp;
            wgt = (rp2 - 1.0) * rp2 * sgn;
            acc = make_double2(acc.x + wgt * v.x * dyde * dyde / 3.0, acc.y + wgt * v.y * dyde * dyde / 3.0);
        }
    }
    for (int off = 1; off < 32; off <<= 1) {
        double ax = __shfl_down_sync(0xffffffffu, acc.x, off);
        double ay = __shfl_down_sync(0xffffffffu, acc.y, off);
        if ((lane & (2 * off - 1)) == 0) { acc.x += ax; acc.y += ay; }
    }
    if (lane == 0) out[(size_t)warp * nyp + (iy - 1)] = acc;
}

int kmm_internal_wallderiv(kmm_ctx *ctx, const double2 *f, int order, int wall, double2 *out, int iy) {
    const int ncols = ctx->nz * ctx->nxh;
    const int threads = 256;
    const int blocks = (ncols * 32 + threads - 1) / threads;
    k_wallderiv<<<blocks, threads, 0, ctx->stream>>>(f, out, ncols, ctx->nyp, order, wall, iy, ctx->dyde);
    CKL();
    return KMM_OK;
}

extern "C" int kmm_wallderiv(kmm_ctx *ctx, int f, int order, int wall, int out, int iy) {
    if (!ctx || order < 0 || order > 2 || wall < 0 || wall > 1 || iy < 1 || iy > ctx->nyp) return KMM_ERR_ARG;
    if (f >= KMM_NSPECTRAL || out >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    double2 *a = SPEC(ctx, f), *b = SPEC(ctx, out);
    if (!a || !b) return KMM_ERR_NOMEM;
    return kmm_internal_wallderiv(ctx, a, order, wall, b, iy);
}

// ---------------------------------------------------------------------------
// norm(a), helpers.f90:91-158
// ---------------------------------------------------------------------------
// one launch norms up to KMM_NORM_BATCH distinct fields, blockIdx.y picking the field
struct NormList {
    double2 *p[KMM_NORM_BATCH];
};

__global__ void k_norm(NormList list, int nyp, int nz, int nxh, int nzh) {
    double2 *a = list.p[blockIdx.y];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int npair = nyp * (nz / 2);      // j = 1..nz/2 (0-based j = 0 handles the (0,0) mode)
    if (t < npair) {
        const int i = t % nyp, j = t / nyp;  // 0-based j in [0, nz/2)
        if (j == 0) {
            double2 v = a[i];
            a[i] = make_double2(v.x, 0.0);
        } else {
            const int jp = nz - j;           // 0-based partner of j (1-based nz+2-j)
            double2 x = a[(size_t)j * nyp + i], y = a[(size_t)jp * nyp + i];
            double2 m = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
            a[(size_t)j * nyp + i] = m;
            a[(size_t)jp * nyp + i] = make_double2(m.x, -m.y);
        }
    } else {
        const int u = t - npair;
        if (u < nyp * nxh) {
            const int i = u % nyp, k = u / nyp;
            a[((size_t)k * nz + nzh) * nyp + i] = make_double2(0.0, 0.0);
        }
    }
}

int kmm_internal_norm_many(kmm_ctx *ctx, double2 *const *a, int nf) {
    const int n = ctx->nyp * (ctx->nz / 2) + ctx->nyp * ctx->nxh;
    for (int f0 = 0; f0 < nf; f0 += KMM_NORM_BATCH) {
        NormList list;
        const int nb = nf - f0 < KMM_NORM_BATCH ? nf - f0 : KMM_NORM_BATCH;
        for (int m = 0; m < nb; ++m) {
            if (!a[f0 + m]) return KMM_ERR_NOMEM;
            list.p[m] = a[f0 + m];
        }
        k_norm<<<dim3((n + 255) / 256, nb), 256, 0, ctx->stream>>>(list, ctx->nyp, ctx->nz, ctx->nxh, ctx->nzh);
        CKL();
    }
    return KMM_OK;
}

int kmm_internal_norm(kmm_ctx *ctx, double2 *a) { return kmm_internal_norm_many(ctx, &a, 1); }

extern "C" int kmm_norm(kmm_ctx *ctx, int f) {
    if (!ctx || f < 0 || f >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    double2 *a = SPEC(ctx, f);
    if (!a) return KMM_ERR_NOMEM;
    return kmm_internal_norm(ctx, a);
}

// ---------------------------------------------------------------------------
// tau solvers.  Matrix rows of evnc / oddc (solvers.f90:324-383), recomputed on the fly:
//   even (ip=0) row i, j = 2i;  odd (ip=1) row i, j = 2i+1:
//   a1 = wn rj1, a2 = -dyde^2 - wn rj2, a3 = wn rj3 with the end-row overrides.
// ---------------------------------------------------------------------------
struct TauRow { double a1, a2, a3; };

__device__ __forceinline__ TauRow tau_row(int i, int par, double wn, double dyde, int nyh, int nyhm) {
    TauRow r;
    const int j = par == 0 ? 2 * i : 2 * i + 1;
    const double rj1 = 1.0 / (double)(4 * j * (j - 1));
    const double rj2 = 1.0 / (double)(2 * (j * j - 1));
    const double rj3 = 1.0 / (double)(4 * j * (j + 1));
    r.a1 = wn * rj1;
    r.a2 = -1.0 * dyde * dyde - wn * rj2;
    r.a3 = wn * rj3;
    if (par == 0) {
        if (i == 1) r.a1 = 2.0 * r.a1;
        if (i == nyhm) r.a3 = 0.0;
        if (i == nyh) { r.a2 = -1.0 * dyde * dyde; r.a3 = 0.0; }
    } else {
        if (i == nyhm - 1) r.a3 = 0.0;
        if (i == nyhm) { r.a2 = -1.0 * dyde * dyde; r.a3 = 0.0; }
    }
    return r;
}

// RHS rows 2..nrank of evns/pntevns (par 0) or odds/pntodds (par 1), written in place at the
// parity positions W(i) = col[2(i-1)+par]; c0 = c(0) Chebyshev weight (2).
__device__ __forceinline__ void tau_rhs_inplace(double2 *col, int par, int ny, int nyh, int nyhm, double c0) {
#define POS(i) (2 * ((i) - 1) + par)
    if (par == 0) {
        // rows i = 2..nyhm use s(j-2), s(j), s(j+2), j = 2i-2 (solvers.f90:387-448)
        double2 sm2 = col[0], s0 = col[2];
        for (int i = 2; i <= nyhm; ++i) {
            const int j = 2 * i - 2;
            double2 sp2 = col[j + 2];
            const double rj1 = 1.0 / (double)(4 * j * (j - 1));
            const double rj2 = 1.0 / (double)(2 * (j * j - 1));
            const double rj3 = 1.0 / (double)(4 * j * (j + 1));
            const double cm = (j - 2 == 0) ? c0 : 1.0;
            double2 w;
            w.x = -cm * sm2.x * rj1 + s0.x * rj2 - sp2.x * rj3;
            w.y = -cm * sm2.y * rj1 + s0.y * rj2 - sp2.y * rj3;
            col[POS(i)] = w;
            sm2 = s0;
            s0 = sp2;
        }
        {   // row nyh: j = ny-2
            const int j = ny - 2;
            const double rj1 = 1.0 / (double)(4 * j * (j - 1));
            const double rj2 = 1.0 / (double)(2 * (j * j - 1));
            double2 w;
            w.x = -sm2.x * rj1 + s0.x * rj2;
            w.y = -sm2.y * rj1 + s0.y * rj2;
            col[POS(nyh)] = w;
        }
        {   // row nyhp: j = ny, s(ny-2) is the current s0
            const int j = ny;
            const double rj1 = 1.0 / (double)(4 * j * (j - 1));
            col[POS(nyh + 1)] = make_double2(-s0.x * rj1, -s0.y * rj1);
        }
    } else {
        // rows i = 2..nyhm-1, j = 2i-1 (solvers.f90:450-496)
        double2 sm2 = col[1], s0 = col[3];
        for (int i = 2; i <= nyhm - 1; ++i) {
            const int j = 2 * i - 1;
            double2 sp2 = col[j + 2];
            const double rj1 = 1.0 / (double)(4 * j * (j - 1));
            const double rj2 = 1.0 / (double)(2 * (j * j - 1));
            const double rj3 = 1.0 / (double)(4 * j * (j + 1));
            double2 w;
            w.x = -sm2.x * rj1 + s0.x * rj2 - sp2.x * rj3;
            w.y = -sm2.y * rj1 + s0.y * rj2 - sp2.y * rj3;
            col[POS(i)] = w;
            sm2 = s0;
            s0 = sp2;
        }
        {   // row nyhm: j = ny-3
            const int j = ny - 3;
            const double rj1 = 1.0 / (double)(4 * j * (j - 1));
            const double rj2 = 1.0 / (double)(2 * (j * j - 1));
            double2 w;
            w.x = -sm2.x * rj1 + s0.x * rj2;
            w.y = -sm2.y * rj1 + s0.y * rj2;
            col[POS(nyhm)] = w;
        }
        {   // row nyh: j = ny-1, s(ny-3) is the current s0
            const int j = ny - 1;
            const double rj1 = 1.0 / (double)(4 * j * (j - 1));
            col[POS(nyh)] = make_double2(-s0.x * rj1, -s0.y * rj1);
        }
    }
#undef POS
}

// eqsolve(a,t,wrk,nrank), solvers.f90:500-553, in place at parity positions; d: local scratch
__device__ __forceinline__ double tau_t(int q, int par, int ib, double dyde) {
    if (ib == 0) return 1.0;                               // dircbc
    const int m2 = par == 0 ? 2 * (q - 1) : 2 * (q - 1) + 1; // neumbc
    return dyde * (double)(m2 * m2);
}

__device__ void eqsolve_inplace(double2 *col, int par, int nrank, double wn, double dyde, int nyh, int nyhm, int ib,
                                double *d) {
#define W(i) col[2 * ((i) - 1) + par]
    const int m = nrank - 1, mm1 = m - 1;
    d[m] = tau_row(m, par, wn, dyde, nyh, nyhm).a2;
    for (int i = mm1; i >= 1; --i) {
        TauRow ri = tau_row(i, par, wn, dyde, nyh, nyhm);
        TauRow rn = tau_row(i + 1, par, wn, dyde, nyh, nyhm);
        d[i] = ri.a2 - ri.a3 * rn.a1 / d[i + 1];
        double2 w1 = W(i + 1), w2 = W(i + 2);
        W(i + 1) = make_double2(w1.x - ri.a3 * w2.x / d[i + 1], w1.y - ri.a3 * w2.y / d[i + 1]);
    }
    TauRow rm = tau_row(m, par, wn, dyde, nyh, nyhm);
    const double tn = tau_t(nrank, par, ib, dyde);
    double f = tau_t(m, par, ib, dyde) - tn * rm.a1 / d[m];
    double2 w1 = W(1), wn_ = W(nrank);
    w1 = make_double2(w1.x - tn * wn_.x / d[m], w1.y - tn * wn_.y / d[m]);
    for (int i = mm1; i >= 1; --i) {
        TauRow ri = tau_row(i, par, wn, dyde, nyh, nyhm);
        double2 wi = W(i + 1);
        w1 = make_double2(w1.x - f * wi.x / d[i], w1.y - f * wi.y / d[i]);
        f = tau_t(i, par, ib, dyde) - f * ri.a1 / d[i];
    }
    w1 = make_double2(w1.x / f, w1.y / f);
    W(1) = w1;
    double2 prev = w1;
    for (int i = 2; i <= nrank; ++i) {
        TauRow rp = tau_row(i - 1, par, wn, dyde, nyh, nyhm);
        double2 wi = W(i);
        prev = make_double2((wi.x - rp.a1 * prev.x) / d[i - 1], (wi.y - rp.a1 * prev.y) / d[i - 1]);
        W(i) = prev;
    }
#undef W
}

// solve(u,x,g,dyde,bctop,bcbot,ib,a,wrkc), solvers.f90:174-283 for every (kx,kz) column
__global__ void __launch_bounds__(TPB) k_solve(double2 *__restrict__ u, const double2 *__restrict__ bct,
                                               const double2 *__restrict__ bcb, const double *__restrict__ wavx,
                                               const double *__restrict__ wavz, int ncols, int nz, int nyp, double g,
                                               int ib, double dyde, double c0) {
    extern __shared__ double2 sm[];
    const int col0 = blockIdx.x * TILE;
    const int ncol = min(TILE, ncols - col0);
    tile_load(sm, u, col0, ncol, nyp);
    __syncthreads();
    const int t = threadIdx.x;
    if (t < ncol) {
        const int ny = nyp - 1, nyh = ny / 2, nyhm = nyh - 1, nyhp = nyh + 1;
        const int colg = col0 + t;
        const int j = colg % nz, k = colg / nz;
        double2 *col = sm + (size_t)t * nyp;
        double wn = wavz[j] * wavz[j] + wavx[k] * wavx[k] + g;
        bool kzero = false;
        if (ib != 0 && wn <= 1.0e-20) { kzero = true; wn = 1.0; }
        double *d = (double *)(sm + (size_t)TILE * nyp) + (size_t)t * (nyhp + 1);
        const double2 bt = bct[colg], bb = bcb[colg];
        for (int par = 0; par < 2; ++par) {
            const int nrank = par == 0 ? nyhp : nyh;
            tau_rhs_inplace(col, par, ny, nyh, nyhm, c0);
            // BC row: evns / odds
            double2 w1;
            if ((ib == 0) == (par == 0)) w1 = make_double2(0.5 * (bt.x + bb.x), 0.5 * (bt.y + bb.y));
            else w1 = make_double2(0.5 * (bt.x - bb.x), 0.5 * (bt.y - bb.y));
            col[par] = w1;
            eqsolve_inplace(col, par, nrank, wn, dyde, nyh, nyhm, ib, d);
        }
        if (kzero)
            for (int i = 0; i < nyp; ++i) col[i] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    tile_store(u, sm, col0, ncol, nyp);
}

int kmm_internal_solve(kmm_ctx *ctx, double2 *u, double g, int ib, const double2 *bct, const double2 *bcb) {
    if (ib == 0) {   // blocked column kernels with cached tables where they are compiled
        const int st = kmm_colblk_solve(ctx, u, g, 0, 0.0, 0.0, 0.0, 0.0, bct, bcb);
        if (st != KMM_ERR_UNSUPPORTED) return st;
    }
    const int ncols = ctx->nz * ctx->nxh;
    const size_t smem = tile_smem(ctx->nyp, 1) + sizeof(double) * TILE * (size_t)(ctx->nyhp + 1);
    RET(kmm_smem_attr(ctx, (const void *)k_solve, smem));
    k_solve<<<(ncols + TILE - 1) / TILE, TPB, smem, ctx->stream>>>(
        u, bct, bcb, ctx->d_wavx, ctx->d_wavz, ncols, ctx->nz, ctx->nyp, g, ib, ctx->dyde, ctx->h_c[0]);
    CKL();
    return KMM_OK;
}

extern "C" int kmm_solve(kmm_ctx *ctx, int u, double g, int ib) {
    if (!ctx || u < 0 || u >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    double2 *a = SPEC(ctx, u), *bt = SPEC(ctx, KMM_BCTOP), *bb = SPEC(ctx, KMM_BCBOT);
    if (!a || !bt || !bb) return KMM_ERR_NOMEM;
    return kmm_internal_solve(ctx, a, g, ib, bt, bb);
}

// penta: mixedbc + pntevns/pntodds + pntsolve + fillt, solvers.f90:680-1061
__global__ void __launch_bounds__(TPB) k_penta(double2 *__restrict__ u, const double2 *__restrict__ gtop,
                                               const double2 *__restrict__ gbot, const double *__restrict__ wavx,
                                               const double *__restrict__ wavz, int ncols, int nz, int nyp, double g,
                                               int ib, double at, double bt, double ab, double bb, double dyde,
                                               double c0) {
    extern __shared__ double2 sm[];
    const int col0 = blockIdx.x * TILE;
    const int ncol = min(TILE, ncols - col0);
    tile_load(sm, u, col0, ncol, nyp);
    __syncthreads();
    const int t = threadIdx.x;
    if (t < ncol) {
        const int ny = nyp - 1, nyh = ny / 2, nyhm = nyh - 1, nyhp = nyh + 1;
        const int colg = col0 + t;
        const int j = colg % nz, k = colg / nz;
        double2 *col = sm + (size_t)t * nyp;   // gs(i,ip) lives at the parity positions of the column
        double wn = wavz[j] * wavz[j] + wavx[k] * wavx[k] + g;
        bool kzero = false;
        if (ib != 0 && wn <= 1.0e-20) { kzero = true; wn = 1.0; }
        double *dsb = (double *)(sm + (size_t)TILE * nyp) + (size_t)t * 2 * (nyhp + 1);
        double *ds[2] = {dsb, dsb + (nyhp + 1)};
        double f[2][2];
        double2 s[2];
        s[0] = gtop[colg];
        s[1] = gbot[colg];
        for (int par = 0; par < 2; ++par) {
            const int ip = par + 1;
            const int n = par == 0 ? nyhp : nyh, m = n - 1, mm1 = m - 1;
            tau_rhs_inplace(col, par, ny, nyh, nyhm, c0);
#define GS(i) col[2 * ((i) - 1) + par]
            double *D = ds[par];
            D[m] = tau_row(m, par, wn, dyde, nyh, nyhm).a2;
            for (int i = mm1; i >= 1; --i) {
                TauRow ri = tau_row(i, par, wn, dyde, nyh, nyhm);
                TauRow rn = tau_row(i + 1, par, wn, dyde, nyh, nyhm);
                D[i] = ri.a2 - ri.a3 * rn.a1 / D[i + 1];
                double2 g1 = GS(i + 1), g2 = GS(i + 2);
                GS(i + 1) = make_double2(g1.x - ri.a3 * g2.x / D[i + 1], g1.y - ri.a3 * g2.y / D[i + 1]);
            }
            // ipass 1 eliminates into the bottom row (js = 2, tb), ipass 2 into the top row (js = 1, tt)
            for (int ipass = 1; ipass <= 2; ++ipass) {
                const int js = ipass == 1 ? 2 : 1;
                // fillt: t(q) = t{b,t}(2q-1) (even) or t{b,t}(2q) (odd); mixedbc: tt(jj) = at + dyde bt (jj-1)^2,
                // tb(jj) = (ab + dyde bb (jj-1)^2) (-1)^(jj-1)
#define TVAL(q) ([&](int qq) -> double {                                         \
                    int jj = par == 0 ? 2 * qq - 1 : 2 * qq;                    \
                    int j1 = jj - 1;                                            \
                    if (ipass == 2) return at + dyde * bt * (double)(j1 * j1);   \
                    double v = ab + dyde * bb * (double)(j1 * j1);               \
                    return (jj % 2 == 0) ? -v : v;                              \
                }(q))
                TauRow rm = tau_row(m, par, wn, dyde, nyh, nyhm);
                double ff = TVAL(m) - TVAL(n) * rm.a1 / D[m];
                double2 gn = GS(n);
                double tn = TVAL(n);
                double2 ss = s[js - 1];
                ss = make_double2(ss.x - tn * gn.x / D[m], ss.y - tn * gn.y / D[m]);
                for (int i = mm1; i >= 1; --i) {
                    TauRow ri = tau_row(i, par, wn, dyde, nyh, nyhm);
                    double2 gi = GS(i + 1);
                    ss = make_double2(ss.x - ff * gi.x / D[i], ss.y - ff * gi.y / D[i]);
                    ff = TVAL(i) - ff * ri.a1 / D[i];
                }
                s[js - 1] = ss;
                f[js - 1][par] = ff;
#undef TVAL
            }
#undef GS
        }
        // 2x2 system for the first even / odd unknowns, then both back substitutions
        const double det = f[0][0] * f[1][1] - f[1][0] * f[0][1];
        double2 x0 = make_double2((s[0].x * f[1][1] - s[1].x * f[0][1]) / det, (s[0].y * f[1][1] - s[1].y * f[0][1]) / det);
        double2 x1 = make_double2((s[1].x * f[0][0] - s[0].x * f[1][0]) / det, (s[1].y * f[0][0] - s[0].y * f[1][0]) / det);
        col[0] = x0;
        col[1] = x1;
        {
            double2 prev = x0;
            for (int i = 2; i <= nyhp; ++i) {   // even: wrk(2i-1)
                TauRow rp = tau_row(i - 1, 0, wn, dyde, nyh, nyhm);
                double2 gi = col[2 * (i - 1)];
                prev = make_double2((gi.x - rp.a1 * prev.x) / ds[0][i - 1], (gi.y - rp.a1 * prev.y) / ds[0][i - 1]);
                col[2 * (i - 1)] = prev;
            }
            prev = x1;
            for (int i = 2; i <= nyh; ++i) {    // odd: wrk(2i)
                TauRow rp = tau_row(i - 1, 1, wn, dyde, nyh, nyhm);
                double2 gi = col[2 * (i - 1) + 1];
                prev = make_double2((gi.x - rp.a1 * prev.x) / ds[1][i - 1], (gi.y - rp.a1 * prev.y) / ds[1][i - 1]);
                col[2 * (i - 1) + 1] = prev;
            }
        }
        if (kzero)
            for (int i = 0; i < nyp; ++i) col[i] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    tile_store(u, sm, col0, ncol, nyp);
}

int kmm_internal_penta_many(kmm_ctx *ctx, double2 *const *u, int nf, double g, double at, double bt, double ab,
                            double bb, const double2 *gt, const double2 *gb) {
    const int st = kmm_colblk_solve_many(ctx, u, nf, g, 1, at, bt, ab, bb, gt, gb);
    if (st != KMM_ERR_UNSUPPORTED) return st;
    for (int m = 0; m < nf; ++m) RET(kmm_internal_penta(ctx, u[m], g, 0, at, bt, ab, bb, gt, gb));
    return KMM_OK;
}

int kmm_internal_penta(kmm_ctx *ctx, double2 *u, double g, int ib, double at, double bt, double ab, double bb,
                       const double2 *gt, const double2 *gb) {
    if (ib == 0) {   // blocked column kernels with cached tables where they are compiled
        const int st = kmm_colblk_solve(ctx, u, g, 1, at, bt, ab, bb, gt, gb);
        if (st != KMM_ERR_UNSUPPORTED) return st;
    }
    const int ncols = ctx->nz * ctx->nxh;
    const size_t smem = tile_smem(ctx->nyp, 1) + sizeof(double) * TILE * 2 * (size_t)(ctx->nyhp + 1);
    RET(kmm_smem_attr(ctx, (const void *)k_penta, smem));
    k_penta<<<(ncols + TILE - 1) / TILE, TPB, smem, ctx->stream>>>(
        u, gt, gb, ctx->d_wavx, ctx->d_wavz, ncols, ctx->nz, ctx->nyp, g, ib, at, bt, ab, bb, ctx->dyde, ctx->h_c[0]);
    CKL();
    return KMM_OK;
}

extern "C" int kmm_penta(kmm_ctx *ctx, int u, double g, int ib, double at, double bt, double ab, double bb) {
    if (!ctx || u < 0 || u >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    double2 *a = SPEC(ctx, u), *gt = SPEC(ctx, KMM_BCTOP), *gb = SPEC(ctx, KMM_BCBOT);
    if (!a || !gt || !gb) return KMM_ERR_NOMEM;
    return kmm_internal_penta(ctx, a, g, ib, at, bt, ab, bb, gt, gb);
}

// ---------------------------------------------------------------------------
// uzero / psolve1d / p1d*, solvers.f90:1065-1493 (one thread: the (0,0) mode only)
// ---------------------------------------------------------------------------
__device__ void cderiv1d_dev(const double *f, double *df, int nyp, double dyde) {
    const int ny = nyp - 1;
    df[nyp - 1] = 0.0;
    df[ny - 1] = 2.0 * (double)ny * f[nyp - 1] * dyde;
    for (int i = ny - 1; i >= 1; --i) df[i - 1] = df[i + 1] + 2.0 * (double)i * f[i] * dyde;
    df[0] = 0.5 * df[0];
}

// The (0,0)-mode solve on one block, over shared-memory copies of the profile and every scratch
// row.  What the serial reference does row by row with no dependence between rows (the right-hand
// sides, the tau rows, the boundary rows t) is spread over the block's threads; the recurrences
// (the elimination of each parity, the two boundary-row eliminations of each parity, the sum
// into s, the back substitution of each parity) run on one thread each, the independent ones at
// the same time.  Each value is formed by the same expression in the same order as the serial
// loop (solvers.f90:1065-1493), so the result is the same to the bit.
#define UZ_ROWS 26
static inline size_t uzero_smem(int nyp) { return sizeof(double) * UZ_ROWS * (size_t)nyp; }

__global__ void __launch_bounds__(128) k_uzero(double *u0g, const double *h1g, const double *h1lg, int nyp, double re,
                                               double dt, double th, double dyde, double at, double bt, double gtop,
                                               double ab, double bb, double gbot, double c0, double wz0) {
    extern __shared__ double su[];
    __shared__ double fq[2][2][2];   // [par][pass]: the final ff, the first term taken from s
    const int L = nyp;
    double *u0 = su, *h1 = su + L, *h1l = su + 2 * L, *wrk1 = su + 3 * L, *tmp = su + 4 * L, *out = su + 5 * L;
    // per-parity rows (pointer arithmetic, not arrays of pointers, so nothing goes to local memory)
#define UZ_ROW(r, par) (su + (size_t)((r) + (par)) * L)
#define CS(par) UZ_ROW(6, par)     // sub-diagonal c
#define DS(par) UZ_ROW(8, par)     // eliminated diagonal d
#define GS(par) UZ_ROW(10, par)    // right-hand side g
#define WRK(par) UZ_ROW(12, par)   // p1devns / p1dodds rows
#define A2(par) UZ_ROW(14, par)    // tau-row diagonal
#define A3(par) UZ_ROW(16, par)    // tau-row super-diagonal
    // rows 18 .. 25: t and the ss terms q of (par, pass)
    const int ny = nyp - 1, nyh = ny / 2, nyhm = nyh - 1, nyhp = nyh + 1;
    const int tid = threadIdx.x, nth = blockDim.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < nyp; i += nth) {
        u0[i] = u0g[i];
        h1[i] = h1g[i];
        h1l[i] = h1lg[i];
    }
    __syncthreads();
    for (int i = tid; i < nyp; i += nth) wrk1[i] = -re * u0[i] / (dt * th) - re * (3.0 * h1[i] - h1l[i]) / (2.0 * th);
    __syncthreads();
    if (th > 0.99) {
        for (int i = tid; i < nyp; i += nth) u0[i] = wrk1[i];
    } else {
        if (tid == 0) {
            cderiv1d_dev(u0, tmp, nyp, dyde);
            cderiv1d_dev(tmp, u0, nyp, dyde);
        }
        __syncthreads();
        for (int i = tid; i < nyp; i += nth) u0[i] = wrk1[i] - (1.0 - th) * u0[i] / th;
    }
    const double g = re / (th * dt);
    // psolve1d, solvers.f90:1180-1245 with mixedbc1d (minus sign in tb, solvers.f90:1249-1269)
    const double wn = wz0 * wz0 + 0.0 + g;
    for (int q = tid; q < 2 * nyp; q += nth) WRK(q / nyp)[q % nyp] = 0.0;
    __syncthreads();
    // right-hand-side rows (p1devns / p1dodds) and the tau rows of both parities, row by row
    for (int e = tid; e < 2 * nyp; e += nth) {
        const int par = e / nyp, i = e % nyp;
        const int n = par == 0 ? nyhp : nyh, m = n - 1;
        if (par == 0) {
            if (i >= 2 && i <= nyhm) {
                int j = 2 * i - 2;
                double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1)), rj3 = 1.0 / (double)(4 * j * (j + 1));
                double cm = (j - 2 == 0) ? c0 : 1.0;
                WRK(0)[i - 1] = -cm * u0[j - 2] * rj1 + u0[j] * rj2 - u0[j + 2] * rj3;
            } else if (i == nyh) {
                int j = ny - 2;
                double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1));
                WRK(0)[nyh - 1] = -u0[j - 2] * rj1 + u0[j] * rj2;
            } else if (i == nyhp) {
                int j = ny;
                double rj1 = 1.0 / (double)(4 * j * (j - 1));
                WRK(0)[nyhp - 1] = -u0[j - 2] * rj1;
            }
        } else {
            if (i >= 2 && i <= nyhm - 1) {
                int j = 2 * i - 1;
                double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1)), rj3 = 1.0 / (double)(4 * j * (j + 1));
                WRK(1)[i - 1] = -u0[j - 2] * rj1 + u0[j] * rj2 - u0[j + 2] * rj3;
            } else if (i == nyhm) {
                int j = ny - 3;
                double rj1 = 1.0 / (double)(4 * j * (j - 1)), rj2 = 1.0 / (double)(2 * (j * j - 1));
                WRK(1)[nyhm - 1] = -u0[j - 2] * rj1 + u0[j] * rj2;
            } else if (i == nyh) {
                int j = ny - 1;
                double rj1 = 1.0 / (double)(4 * j * (j - 1));
                WRK(1)[nyh - 1] = -u0[j - 2] * rj1;
            }
        }
        if (i >= 1 && i <= m) {
            const TauRow r = tau_row(i, par, wn, dyde, nyh, nyhm);
            CS(par)[i] = r.a1;
            A2(par)[i] = r.a2;
            A3(par)[i] = r.a3;
        }
    }
    __syncthreads();
    // p1dsolve elimination: one thread per parity
    if (lane == 0 && warp < 2) {
        const int par = warp;
        const int n = par == 0 ? nyhp : nyh, m = n - 1, mm1 = m - 1;
        for (int i = 1; i <= m; ++i) GS(par)[i] = WRK(par)[i - 1];
        DS(par)[m] = A2(par)[m];
        GS(par)[n] = WRK(par)[n - 1];
        for (int i = mm1; i >= 1; --i) {
            DS(par)[i] = A2(par)[i] - A3(par)[i] * CS(par)[i + 1] / DS(par)[i + 1];
            GS(par)[i + 1] = GS(par)[i + 1] - A3(par)[i] * GS(par)[i + 2] / DS(par)[i + 1];
        }
    }
    // the boundary rows t of (par, pass)
    for (int e = tid; e < 4 * nyp; e += nth) {
        const int k = e / nyp, q = e % nyp + 1;
        const int par = k >> 1, ipass = (k & 1) + 1;
        const int n = par == 0 ? nyhp : nyh;
        if (q <= n) {
            int jj = par == 0 ? 2 * q - 1 : 2 * q, j1 = jj - 1;
            double v = ipass == 2 ? at + dyde * bt * (double)(j1 * j1) : ab - dyde * bb * (double)(j1 * j1);
            if (ipass == 1 && jj % 2 == 0) v = -v;
            su[(size_t)(18 + k) * L + q - 1] = v;
        }
    }
    __syncthreads();
    // the boundary-row eliminations: one thread per (par, pass); the terms leaving s are kept
    if (lane == 0) {
        const int k = warp, par = k >> 1, ipass = (k & 1) + 1;
        const int n = par == 0 ? nyhp : nyh, m = n - 1, mm1 = m - 1;
        const double *t = su + (size_t)(18 + k) * L;
        double *q = su + (size_t)(22 + k) * L;
        double ff = t[m - 1] - t[n - 1] * CS(par)[m] / DS(par)[m];
        fq[par][ipass - 1][1] = t[n - 1] * GS(par)[n] / DS(par)[m];
        for (int i = mm1; i >= 1; --i) {
            q[i] = ff * GS(par)[i + 1] / DS(par)[i];
            ff = t[i - 1] - ff * CS(par)[i] / DS(par)[i];
        }
        fq[par][ipass - 1][0] = ff;
    }
    __syncthreads();
    // s in the reference's order (parity 0 then 1, pass 1 then 2), the 2x2 system for out(1:2)
    if (tid == 0) {
        double f[2][2], s[2];
        s[0] = gtop;
        s[1] = gbot;
        for (int par = 0; par < 2; ++par) {
            const int n = par == 0 ? nyhp : nyh, m = n - 1, mm1 = m - 1;
            for (int ipass = 1; ipass <= 2; ++ipass) {
                const int js = ipass == 1 ? 2 : 1;
                const double *q = su + (size_t)(22 + 2 * par + ipass - 1) * L;
                double ss = s[js - 1] - fq[par][ipass - 1][1];
                for (int i = mm1; i >= 1; --i) ss = ss - q[i];
                s[js - 1] = ss;
                f[js - 1][par] = fq[par][ipass - 1][0];
            }
        }
        const double det = f[0][0] * f[1][1] - f[1][0] * f[0][1];
        out[0] = (s[0] * f[1][1] - s[1] * f[0][1]) / det;
        out[1] = (s[1] * f[0][0] - s[0] * f[1][0]) / det;
    }
    __syncthreads();
    // back substitution: one thread per parity
    if (lane == 0 && warp == 0) {
        for (int i = 2; i <= nyhp; ++i) {
            int ii = 2 * i - 1;
            out[ii - 1] = (GS(0)[i] - CS(0)[i - 1] * out[ii - 3]) / DS(0)[i - 1];
        }
    } else if (lane == 0 && warp == 1) {
        for (int i = 2; i <= nyh; ++i) {
            int ii = 2 * i;
            out[ii - 1] = (GS(1)[i] - CS(1)[i - 1] * out[ii - 3]) / DS(1)[i - 1];
        }
    }
    __syncthreads();
    for (int i = tid; i < nyp; i += nth) u0g[i] = out[i];
#undef CS
#undef DS
#undef GS
#undef WRK
#undef A2
#undef A3
#undef UZ_ROW
}

int kmm_internal_uzero(kmm_ctx *ctx, int uflag, cudaStream_t st) {
    double *u0 = REAL(ctx, uflag == 1 ? KMM_U0 : KMM_W0);
    double *h1 = REAL(ctx, uflag == 1 ? KMM_H1N : KMM_H3N);
    double *h1l = REAL(ctx, uflag == 1 ? KMM_H1NM1 : KMM_H3NM1);
    if (!u0 || !h1 || !h1l) return KMM_ERR_NOMEM;
    const size_t sm = uzero_smem(ctx->nyp);
    RET(kmm_smem_attr(ctx, (const void *)k_uzero, sm));
    // uflag 3 passes btu, as the reference does (solvers.f90:1173)
    if (uflag == 1)
        k_uzero<<<1, 128, sm, st>>>(u0, h1, h1l, ctx->nyp, ctx->re, ctx->dt, ctx->theta, ctx->dyde, ctx->atu,
                                    ctx->btu, ctx->gtu, ctx->abu, ctx->bbu, ctx->gbu, ctx->h_c[0], ctx->h_wavz[0]);
    else
        k_uzero<<<1, 128, sm, st>>>(u0, h1, h1l, ctx->nyp, ctx->re, ctx->dt, ctx->theta, ctx->dyde, ctx->atw,
                                    ctx->btu, ctx->gtw, ctx->abw, ctx->bbw, ctx->gbw, ctx->h_c[0], ctx->h_wavz[0]);
    CKL();
    return KMM_OK;
}

extern "C" int kmm_uzero(kmm_ctx *ctx, int uflag) {
    if (!ctx || (uflag != 1 && uflag != 3)) return KMM_ERR_ARG;
    return kmm_internal_uzero(ctx, uflag, ctx->stream);
}

// ---------------------------------------------------------------------------
// Constant flow rate (kmm_params.flow_rate > 0; no counterpart in the reference, which holds the
// mean pressure gradient dPdx of init_flow.f90:117 constant).  The bulk velocity is the trapezoid
// of writeoutputs (helpers.f90:1355-1359) over the Gauss-Lobatto points of the mean profile
// u(y_i) = sum_n u0_n cos(n pi i / ny): Q = W . u0 with
// W_n = (1/yl) sum_i (cos(n pi i/ny) + cos(n pi (i+1)/ny)) / 2 |y_(i+1) - y_i| (FP64, host).  G is the
// response of the u0 step to a unit uniform acceleration over one step with homogeneous walls: the
// uzero solve with h_n = h_(n-1) = T_0 from u0 = 0, less the same solve with zero forcing.  After
// each u0 solve one warp sets delta = (flow_rate - W . u0) / (W . G) and u0 += delta G; the step was
// then driven by dPdx - delta (kmm_stats.dpdx).
// d_frate layout: W [nyp] | G [nyp] | delta [1] | scratch 4 nyp (ua, ha, ub, hb)
// ---------------------------------------------------------------------------
__global__ void k_frate_fill(double *s, int nyp) {
    for (int i = threadIdx.x; i < 4 * nyp; i += blockDim.x) s[i] = (i == nyp) ? 1.0 : 0.0;   // ha[0] = 1
}

__global__ void k_frate_g(double *G, const double *ua, const double *ub, int nyp) {
    for (int i = threadIdx.x; i < nyp; i += blockDim.x) G[i] = ua[i] - ub[i];
}

__global__ void k_flowrate(double *__restrict__ u0, const double *__restrict__ W, const double *__restrict__ G, int nyp,
                           double target, double *__restrict__ delta) {
    const int lane = threadIdx.x & 31;
    double q = 0.0, wg = 0.0;
    for (int i = lane; i < nyp; i += 32) {
        q += W[i] * u0[i];
        wg += W[i] * G[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        q += __shfl_xor_sync(0xffffffffu, q, o);
        wg += __shfl_xor_sync(0xffffffffu, wg, o);
    }
    const double d = (target - q) / wg;
    for (int i = lane; i < nyp; i += 32) u0[i] += d * G[i];
    if (lane == 0) *delta = d;
}

int kmm_flowrate_setup(kmm_ctx *ctx) {
    if (!(ctx->p.flow_rate > 0.0) || ctx->frate_ready) return KMM_OK;
    const int nyp = ctx->nyp, ny = ctx->ny;
    if (!ctx->d_frate) CK(cudaMalloc(&ctx->d_frate, sizeof(double) * (6 * (size_t)nyp + 1)));
    double *W = ctx->d_frate, *G = W + nyp, *sc = W + 2 * nyp + 1;
    double *hw = (double *)malloc(sizeof(double) * (size_t)nyp);
    for (int n = 0; n < nyp; ++n) {
        double w = 0.0;
        for (int i = 0; i < ny; ++i)
            w += 1.0 / ctx->yl * 0.5 * (cos((double)n * ctx->pi * (double)(i + 1) / (double)ny) +
                                        cos((double)n * ctx->pi * (double)i / (double)ny)) *
                 fabs(ctx->h_ycoord[i + 1] - ctx->h_ycoord[i]);
        hw[n] = w;
    }
    cudaError_t e = cudaMemcpyAsync(W, hw, sizeof(double) * (size_t)nyp, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    free(hw);
    CK(e);
    k_frate_fill<<<1, 256, 0, ctx->stream>>>(sc, nyp);
    CKL();
    double *ua = sc, *ha = sc + nyp, *ub = sc + 2 * nyp, *hb = sc + 3 * nyp;
    const size_t sm = uzero_smem(nyp);
    RET(kmm_smem_attr(ctx, (const void *)k_uzero, sm));
    k_uzero<<<1, 128, sm, ctx->stream>>>(ua, ha, ha, nyp, ctx->re, ctx->dt, ctx->theta, ctx->dyde, ctx->atu, ctx->btu,
                                         ctx->gtu, ctx->abu, ctx->bbu, ctx->gbu, ctx->h_c[0], ctx->h_wavz[0]);
    CKL();
    k_uzero<<<1, 128, sm, ctx->stream>>>(ub, hb, hb, nyp, ctx->re, ctx->dt, ctx->theta, ctx->dyde, ctx->atu, ctx->btu,
                                         ctx->gtu, ctx->abu, ctx->bbu, ctx->gbu, ctx->h_c[0], ctx->h_wavz[0]);
    CKL();
    k_frate_g<<<1, 256, 0, ctx->stream>>>(G, ua, ub, nyp);
    CKL();
    CK(cudaMemsetAsync(W + 2 * nyp, 0, sizeof(double), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->frate_ready = 1;
    return KMM_OK;
}

// after the u0 solve (main_dns.f90:489-492), on stream st; the correction goes to the pinned slot
// read by kmm_get_stats
int kmm_flowrate_apply(kmm_ctx *ctx, cudaStream_t st) {
    if (!(ctx->p.flow_rate > 0.0)) return KMM_OK;
    if (!ctx->frate_ready) {
        kmm_set_error(ctx, "constant flow rate: kmm_initial has not run");
        return KMM_ERR_ARG;
    }
    const int nyp = ctx->nyp;
    double *W = ctx->d_frate, *G = W + nyp, *delta = W + 2 * nyp;
    k_flowrate<<<1, 32, 0, st>>>(REAL(ctx, KMM_U0), W, G, nyp, ctx->p.flow_rate, delta);
    CKL();
    CK(cudaMemcpyAsync(kmm_h_pin_delta(ctx), delta, sizeof(double), cudaMemcpyDeviceToHost, st));
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// pointwise spectral kernels
// ---------------------------------------------------------------------------
#define GRID_LOOP(n) for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (n); idx += (size_t)gridDim.x * blockDim.x)
#define DECOMP()                              \
    const int i = (int)(idx % nyp);           \
    const size_t jk = idx / nyp;              \
    const int j = (int)(jk % nz);             \
    const int k = (int)(jk / nz);             \
    (void)i; (void)j; (void)k;

// phirhs first part, solvers.f90:633-664: wrkc = -re var/(dt th) v - re var/(2 th)(3 fn - fnm1) [+ (1-th) w2 v/th]
// up to KMM_PHI_BATCH independent fields per launch (blockIdx.y picks the field)
struct PhiList {
    double2 *v[KMM_PHI_BATCH];
    const double2 *fn[KMM_PHI_BATCH];
    const double2 *fnm1[KMM_PHI_BATCH];
    double2 *wrkc[KMM_PHI_BATCH];
};

__global__ void k_phirhs_a(PhiList L, const double *__restrict__ wavx, const double *__restrict__ wavz, size_t n,
                           int nyp, int nz, double re, double var, double dt, double th) {
    double2 *__restrict__ v = L.v[blockIdx.y];
    const double2 *__restrict__ fn = L.fn[blockIdx.y];
    const double2 *__restrict__ fnm1 = L.fnm1[blockIdx.y];
    double2 *__restrict__ wrkc = L.wrkc[blockIdx.y];
    const double a = -re * var / (dt * th), b = re * var / (2.0 * th);
    GRID_LOOP(n) {
        DECOMP();
        double2 vv = v[idx], f = fn[idx];
        // fnm1 = NULL: the n-1 term is 2 fn (the polymer components' call, main_dns.f90:250-260),
        // formed here exactly instead of read
        const double2 fm = fnm1 ? fnm1[idx] : make_double2(2.0 * f.x, 2.0 * f.y);
        double2 w;
        w.x = a * vv.x - b * (3.0 * f.x - fm.x);
        w.y = a * vv.y - b * (3.0 * f.y - fm.y);
        if (th > 0.99) { vv = w; v[idx] = w; }
        const double w2 = wavz[j] * wavz[j] + wavx[k] * wavx[k];
        const double c = (1.0 - th) * w2;
        w.x = w.x + c * vv.x / th;
        w.y = w.y + c * vv.y / th;
        wrkc[idx] = w;
    }
}

// phirhs last part, solvers.f90:668-675: v = wrkc - (1-th) v''/th
__global__ void k_phirhs_b(PhiList L, size_t n, double th) {
    double2 *__restrict__ v = L.v[blockIdx.y];
    const double2 *__restrict__ wrkc = L.wrkc[blockIdx.y];
    GRID_LOOP(n) {
        double2 w = wrkc[idx], d = v[idx];
        v[idx] = make_double2(w.x - (1.0 - th) * d.x / th, w.y - (1.0 - th) * d.y / th);
    }
}

__global__ void k_zero_wall(double2 *a, double2 *b, size_t n) {
    GRID_LOOP(n) { a[idx] = make_double2(0.0, 0.0); b[idx] = make_double2(0.0, 0.0); }
}

extern "C" int kmm_phirhs(kmm_ctx *ctx, int v, int fn, int fnm1, double var) {
    if (!ctx || v >= KMM_NSPECTRAL || fn >= KMM_NSPECTRAL || fnm1 >= KMM_NSPECTRAL) return KMM_ERR_ARG;
    double2 *V = SPEC(ctx, v), *F = SPEC(ctx, fn), *FM = SPEC(ctx, fnm1);
    if (!V || !F || !FM) return KMM_ERR_NOMEM;
    return kmm_internal_phirhs(ctx, V, F, FM, var);
}

int kmm_internal_phirhs_many(kmm_ctx *ctx, double2 *const *V, const double2 *const *F, const double2 *const *FM,
                             int nf, double var, double2 *const *wrkc, double2 *const *wrk1) {
    double2 *bt = SPEC(ctx, KMM_BCTOP), *bb = SPEC(ctx, KMM_BCBOT);
    if (!bt || !bb) return KMM_ERR_NOMEM;
    if (nf < 1 || nf > KMM_PHI_BATCH) return KMM_ERR_ARG;
    const size_t nw = (size_t)ctx->nz * ctx->nxh, n = ctx->nspec;
    k_zero_wall<<<kmm_blocks(nw, 256), 256, 0, ctx->stream>>>(bt, bb, nw);
    CKL();
    PhiList L;
    for (int m = 0; m < nf; ++m) {
        L.v[m] = V[m];
        L.fn[m] = F[m];
        L.fnm1[m] = FM[m];
        L.wrkc[m] = wrkc[m];
    }
    const dim3 grid(kmm_blocks(n, 256), nf);
    k_phirhs_a<<<grid, 256, 0, ctx->stream>>>(L, ctx->d_wavx, ctx->d_wavz, n, ctx->nyp, ctx->nz, ctx->re, var, ctx->dt,
                                              ctx->theta);
    CKL();
    RET(kmm_internal_cderiv_many(ctx, V, wrk1, nf));
    RET(kmm_internal_cderiv_many(ctx, wrk1, V, nf));
    k_phirhs_b<<<grid, 256, 0, ctx->stream>>>(L, n, ctx->theta);
    CKL();
    return KMM_OK;
}

int kmm_internal_phirhs(kmm_ctx *ctx, double2 *V, const double2 *F, const double2 *FM, double var) {
    return kmm_internal_phirhs_many(ctx, &V, &F, &FM, 1, var, &ctx->wrk[0], &ctx->wrk[1]);
}

// main_dns.f90:363-375
__global__ void k_phi(double2 *__restrict__ v, const double2 *__restrict__ d2, const double *__restrict__ wavx,
                      const double *__restrict__ wavz, size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double wn2 = wavx[k] * wavx[k] + wavz[j] * wavz[j];
        double2 a = d2[idx], b = v[idx];
        v[idx] = make_double2(a.x - wn2 * b.x, a.y - wn2 * b.y);
    }
}

extern "C" int kmm_phi_from_v(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *v = SPEC(ctx, KMM_V);
    if (!v) return KMM_ERR_NOMEM;
    RET(kmm_internal_cderiv(ctx, v, ctx->wrk[1]));
    RET(kmm_internal_cderiv(ctx, ctx->wrk[1], ctx->wrk[0]));
    k_phi<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(v, ctx->wrk[0], ctx->d_wavx, ctx->d_wavz, ctx->nspec,
                                                                ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

// influence-matrix combination, main_dns.f90:456-466
__global__ void k_influence(double2 *__restrict__ v, const double2 *__restrict__ wrkc, const double2 *__restrict__ gf1,
                            const double2 *__restrict__ gf2, const double2 *__restrict__ d1b,
                            const double2 *__restrict__ d1t, const double2 *__restrict__ d2b,
                            const double2 *__restrict__ d2t, const double2 *__restrict__ den, double2 *c1o,
                            double2 *c2o, int ncols, int nyp, int iyb, int iyt) {
    const int col = blockIdx.x;
    if (col >= ncols) return;
    const double2 wb = wrkc[(size_t)col * nyp + iyb - 1], wt = wrkc[(size_t)col * nyp + iyt - 1];
    const double2 c1 = cdiv(csub(cmul(wb, d2t[col]), cmul(wt, d2b[col])), den[col]);
    const double2 c2 = cdiv(csub(cmul(wt, d1b[col]), cmul(wb, d1t[col])), den[col]);
    if (threadIdx.x == 0) { c1o[col] = c1; c2o[col] = c2; }
    for (int i = threadIdx.x; i < nyp; i += blockDim.x) {
        size_t x = (size_t)col * nyp + i;
        double2 a = cmul(c1, gf1[x]), b = cmul(c2, gf2[x]);
        double2 vv = v[x];
        v[x] = make_double2(vv.x + a.x + b.x, vv.y + a.y + b.y);
    }
}

extern "C" int kmm_influence(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *v = SPEC(ctx, KMM_V), *wrkc = ctx->wrk[2], *wrk1 = ctx->wrk[3];
    const int iyb = 2, iyt = 4;
    if (ctx->nb == 1) {
        RET(kmm_internal_wallderiv(ctx, v, 1, 0, wrkc, iyb));
        if (ctx->nt == 1) { RET(kmm_internal_wallderiv(ctx, v, 1, 1, wrkc, iyt)); }
        else { RET(kmm_internal_cderiv(ctx, v, wrk1)); RET(kmm_internal_wallderiv(ctx, wrk1, 1, 1, wrkc, iyt)); }
    } else {
        RET(kmm_internal_cderiv(ctx, v, wrk1));
        RET(kmm_internal_wallderiv(ctx, wrk1, 1, 0, wrkc, iyb));
        if (ctx->nt == 1) { RET(kmm_internal_wallderiv(ctx, v, 1, 1, wrkc, iyt)); }
        else { RET(kmm_internal_cderiv(ctx, v, wrk1)); RET(kmm_internal_wallderiv(ctx, wrk1, 1, 1, wrkc, iyt)); }
    }
    const int ncols = ctx->nz * ctx->nxh;
    k_influence<<<ncols, 128, 0, ctx->stream>>>(v, wrkc, SPEC(ctx, KMM_GF1), SPEC(ctx, KMM_GF2), SPEC(ctx, KMM_DNV1B),
                                               SPEC(ctx, KMM_DNV1T), SPEC(ctx, KMM_DNV2B), SPEC(ctx, KMM_DNV2T),
                                               SPEC(ctx, KMM_DENOM), SPEC(ctx, KMM_C1), SPEC(ctx, KMM_C2), ncols,
                                               ctx->nyp, iyb, iyt);
    CKL();
    return KMM_OK;
}

// veloc, solvers.f90:1576-1659 (wrkc = dv/dy)
__global__ void k_veloc(double2 *__restrict__ u, double2 *__restrict__ v, double2 *__restrict__ w,
                        const double2 *__restrict__ dv, const double2 *__restrict__ omy, const double *__restrict__ u0,
                        const double *__restrict__ w0, const double *__restrict__ wavx, const double *__restrict__ wavz,
                        size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double2 d = dv[idx], o = omy[idx];
        if (k > 0) {
            const double w2 = wavx[k] * wavx[k] + wavz[j] * wavz[j];
            // u = -(-i kx dv + i kz om)/w2 ; w = -(-i kz dv - i kx om)/w2
            double2 a = cimul(d, -wavx[k]), b = cimul(o, wavz[j]);
            double2 s = cadd(a, b);
            u[idx] = make_double2(-s.x / w2, -s.y / w2);
            double2 c = cimul(d, -wavz[j]), e = cimul(o, wavx[k]);
            double2 t = csub(c, e);
            w[idx] = make_double2(-t.x / w2, -t.y / w2);
        } else if (j > 0) {
            const double w2 = wavz[j] * wavz[j];
            double2 b = cimul(o, wavz[j]);
            u[idx] = make_double2(-b.x / w2, -b.y / w2);
            double2 c = cimul(d, -wavz[j]);
            w[idx] = make_double2(-c.x / w2, -c.y / w2);
        } else {
            u[idx] = make_double2(u0[i], 0.0);
            v[idx] = make_double2(0.0, 0.0);
            w[idx] = make_double2(w0[i], 0.0);
        }
    }
}

extern "C" int kmm_veloc(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *u = SPEC(ctx, KMM_U), *v = SPEC(ctx, KMM_V), *w = SPEC(ctx, KMM_W), *omy = SPEC(ctx, KMM_OMY);
    double *u0 = REAL(ctx, KMM_U0), *w0 = REAL(ctx, KMM_W0);
    if (!u || !v || !w || !omy || !u0 || !w0) return KMM_ERR_NOMEM;
    RET(kmm_internal_cderiv(ctx, v, ctx->wrk[0]));
    k_veloc<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(u, v, w, ctx->wrk[0], omy, u0, w0, ctx->d_wavx,
                                                                  ctx->d_wavz, ctx->nspec, ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

// vort, solvers.f90:1663-1722: omz = i kx v - du/dy; omx = dw/dy - i kz v
__global__ void k_vort(const double2 *__restrict__ v, double2 *__restrict__ omx, double2 *__restrict__ omz,
                       const double *__restrict__ wavx, const double *__restrict__ wavz, size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double2 vv = v[idx];
        omz[idx] = csub(cimul(vv, wavx[k]), omz[idx]);
        omx[idx] = csub(omx[idx], cimul(vv, wavz[j]));
    }
}

extern "C" int kmm_vort(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *u = SPEC(ctx, KMM_U), *v = SPEC(ctx, KMM_V), *w = SPEC(ctx, KMM_W);
    double2 *omx = SPEC(ctx, KMM_OMX), *omz = SPEC(ctx, KMM_OMZ);
    if (!u || !v || !w || !omx || !omz) return KMM_ERR_NOMEM;
    {
        const double2 *in[2] = {u, w};
        double2 *out[2] = {omz, omx};
        RET(kmm_internal_cderiv_many(ctx, in, out, 2));
    }
    k_vort<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(v, omx, omz, ctx->d_wavx, ctx->d_wavz, ctx->nspec,
                                                                 ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

// gradv, derivatives.f90:6-86
__global__ void k_gradv(const double2 *__restrict__ u, const double2 *__restrict__ v, const double2 *__restrict__ w,
                        double2 *u11, double2 *u21, double2 *u31, double2 *u13, double2 *u23, double2 *u33,
                        double2 *Lu, double2 *Lv, double2 *Lw, const double2 *__restrict__ d2u,
                        const double2 *__restrict__ d2v, const double2 *__restrict__ d2w,
                        const double *__restrict__ wavx, const double *__restrict__ wavz, size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double kx = wavx[k], kz = wavz[j];
        const double wn2 = kx * kx + kz * kz;
        const double2 a = u[idx], b = v[idx], c = w[idx];
        u11[idx] = cimul(a, kx);
        u21[idx] = cimul(b, kx);
        u31[idx] = cimul(c, kx);
        u13[idx] = cimul(a, kz);
        u23[idx] = cimul(b, kz);
        u33[idx] = cimul(c, kz);
        double2 p = d2u[idx], q = d2v[idx], r = d2w[idx];
        Lu[idx] = make_double2(p.x - wn2 * a.x, p.y - wn2 * a.y);
        Lv[idx] = make_double2(q.x - wn2 * b.x, q.y - wn2 * b.y);
        Lw[idx] = make_double2(r.x - wn2 * c.x, r.y - wn2 * c.y);
    }
}

extern "C" int kmm_gradv(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *u = SPEC(ctx, KMM_U), *v = SPEC(ctx, KMM_V), *w = SPEC(ctx, KMM_W);
    double2 *u12 = SPEC(ctx, KMM_U12), *u22 = SPEC(ctx, KMM_U22), *u32 = SPEC(ctx, KMM_U32);
    {
        const double2 *in1[3] = {u, v, w}, *in2[3] = {u12, u22, u32};
        double2 *out1[3] = {u12, u22, u32}, *out2[3] = {ctx->wrk[0], ctx->wrk[1], ctx->wrk[2]};
        RET(kmm_internal_cderiv_many(ctx, in1, out1, 3));
        RET(kmm_internal_cderiv_many(ctx, in2, out2, 3));
    }
    k_gradv<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(
        u, v, w, SPEC(ctx, KMM_U11), SPEC(ctx, KMM_U21), SPEC(ctx, KMM_U31), SPEC(ctx, KMM_U13), SPEC(ctx, KMM_U23),
        SPEC(ctx, KMM_U33), SPEC(ctx, KMM_LU), SPEC(ctx, KMM_LV), SPEC(ctx, KMM_LW), ctx->wrk[0], ctx->wrk[1],
        ctx->wrk[2], ctx->d_wavx, ctx->d_wavz, ctx->nspec, ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

// i kx a -> dx, i kz a -> dz (gradscl / derivscji x,z parts)
__global__ void k_dxdz(const double2 *__restrict__ a, double2 *__restrict__ dx, double2 *__restrict__ dz,
                       const double *__restrict__ wavx, const double *__restrict__ wavz, size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double2 v = a[idx];
        dx[idx] = cimul(v, wavx[k]);
        dz[idx] = cimul(v, wavz[j]);
    }
}

// k_dxdz over up to 9 fields (blockIdx.y picks the field)
struct DxdzList {
    const double2 *a[9];
    double2 *dx[9], *dz[9];
};

__global__ void k_dxdz_many(DxdzList L, const double *__restrict__ wavx, const double *__restrict__ wavz, size_t n,
                            int nyp, int nz) {
    const double2 *__restrict__ a = L.a[blockIdx.y];
    double2 *__restrict__ dx = L.dx[blockIdx.y];
    double2 *__restrict__ dz = L.dz[blockIdx.y];
    GRID_LOOP(n) {
        DECOMP();
        const double2 v = a[idx];
        dx[idx] = cimul(v, wavx[k]);
        dz[idx] = cimul(v, wavz[j]);
    }
}

extern "C" int kmm_gradscl(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *s = SPEC(ctx, KMM_SCALAR);
    RET(kmm_internal_cderiv(ctx, s, SPEC(ctx, KMM_SCLY)));
    k_dxdz<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(s, SPEC(ctx, KMM_SCLX), SPEC(ctx, KMM_SCLZ),
                                                                 ctx->d_wavx, ctx->d_wavz, ctx->nspec, ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

extern "C" int kmm_derivscji(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    {   // the nine y derivatives in one launch, then the x / z ones
        const double2 *in[9];
        double2 *out[9];
        for (int ij = 0; ij < 9; ++ij) {
            in[ij] = SPEC(ctx, KMM_C11 + ij);
            out[ij] = SPEC(ctx, KMM_DC111 + 3 * ij + 1);
            if (!in[ij] || !out[ij]) return KMM_ERR_NOMEM;
        }
        RET(kmm_internal_cderiv_many(ctx, in, out, 9));
    }
    DxdzList L;
    for (int ij = 0; ij < 9; ++ij) {
        L.a[ij] = SPEC(ctx, KMM_C11 + ij);
        L.dx[ij] = SPEC(ctx, KMM_DC111 + 3 * ij);
        L.dz[ij] = SPEC(ctx, KMM_DC111 + 3 * ij + 2);
        if (!L.dx[ij] || !L.dz[ij]) return KMM_ERR_NOMEM;
    }
    k_dxdz_many<<<dim3(kmm_blocks(ctx->nspec, 256), 9), 256, 0, ctx->stream>>>(L, ctx->d_wavx, ctx->d_wavz, ctx->nspec,
                                                                              ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

// nonlin, solvers.f90:1497-1572
__global__ void k_nonlin_a(const double2 *__restrict__ omz, const double2 *__restrict__ gn, double2 *__restrict__ wrkc,
                           const double *__restrict__ wavx, const double *__restrict__ wavz, size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double2 o = omz[idx], g = gn[idx];
        double2 s = make_double2(wavz[j] * o.x + wavx[k] * g.x, wavz[j] * o.y + wavx[k] * g.y);
        wrkc[idx] = make_double2(-s.y, s.x);
    }
}

__global__ void k_nonlin_b(double2 *__restrict__ fn, double2 *__restrict__ gn, const double2 *__restrict__ omz,
                           const double2 *__restrict__ d, const double *__restrict__ wavx,
                           const double *__restrict__ wavz, size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double w2 = -wavx[k] * wavx[k] - wavz[j] * wavz[j];
        double2 f = fn[idx], dd = d[idx];
        fn[idx] = make_double2(w2 * f.x - dd.x, w2 * f.y - dd.y);
        const double2 g = gn[idx], o = omz[idx];
        double2 s = make_double2(wavz[j] * g.x - wavx[k] * o.x, wavz[j] * g.y - wavx[k] * o.y);
        gn[idx] = make_double2(-s.y, s.x);
    }
}

extern "C" int kmm_nonlin(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *fn = SPEC(ctx, KMM_FN), *gn = SPEC(ctx, KMM_GN), *omz = SPEC(ctx, KMM_OMZ);
    k_nonlin_a<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(omz, gn, ctx->wrk[0], ctx->d_wavx, ctx->d_wavz,
                                                                     ctx->nspec, ctx->nyp, ctx->nz);
    CKL();
    RET(kmm_internal_cderiv(ctx, ctx->wrk[0], ctx->wrk[1]));
    k_nonlin_b<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(fn, gn, omz, ctx->wrk[1], ctx->d_wavx,
                                                                     ctx->d_wavz, ctx->nspec, ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

// spectral smoothing, main_dns.f90:710-745 (factors precomputed per column / per y with the
// reference's formulas; exp of an argument evaluated identically on every call)
struct PtrList16 { double2 *p[16]; };

__global__ void k_filter(const __grid_constant__ PtrList16 ptrs, int nptr, size_t n, int nyp, int nz, int nzh, int ny) {
    GRID_LOOP(n) {
        DECOMP();
        const int j1 = j + 1;
        const int jj = (j1 > nzh) ? nz - j1 + 1 : j1 - 1;
        const double zr = (double)jj / (double)nzh, yr = (double)i / (double)ny;
        double z2 = zr * zr, z4 = z2 * z2, z8 = z4 * z4;
        double y2 = yr * yr, y4 = y2 * y2, y8 = y4 * y4;
        const double zs = exp(-3.0 * (z8 * z2));
        const double ys = exp(-3.0 * (y8 * y2));
        for (int p = 0; p < nptr; ++p) {
            double2 a = ptrs.p[p][idx];
            a = make_double2(a.x * zs * ys, a.y * zs * ys);
            ptrs.p[p][idx] = a;
        }
    }
}

extern "C" int kmm_filter(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    PtrList16 h;
    int np = 0;
    h.p[np++] = SPEC(ctx, KMM_OMZ);
    h.p[np++] = SPEC(ctx, KMM_GN);
    h.p[np++] = SPEC(ctx, KMM_FN);
    if (ctx->p.scalar_on) h.p[np++] = SPEC(ctx, KMM_SCN);
    if (ctx->p.polymer_on) {
        for (int m = 0; m < 6; ++m) h.p[np++] = SPEC(ctx, KMM_C11N + m);
        for (int m = 0; m < 6; ++m) h.p[np++] = SPEC(ctx, KMM_STR11N + m);
    }
    for (int q = 0; q < np; ++q)
        if (!h.p[q]) return KMM_ERR_NOMEM;
    k_filter<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(h, np, ctx->nspec, ctx->nyp, ctx->nz, ctx->nzh,
                                                                   ctx->ny);
    CKL();
    return KMM_OK;
}

// polyNL, helpers.f90:610-674 -> scratch NL fields in ctx->wrk? (six fields: use T1..T3 + WRKC/WRK1 is not enough)
// the six components in one launch (blockIdx.y picks the component)
struct PolyNlList {
    double2 *nl[6];
    const double2 *cn[6], *cnm1[6], *sn[6], *snm1[6];
};

__global__ void k_polynl(PolyNlList L, size_t n, double tinv) {
    double2 *__restrict__ nl = L.nl[blockIdx.y];
    const double2 *__restrict__ cn = L.cn[blockIdx.y];
    const double2 *__restrict__ cnm1 = L.cnm1[blockIdx.y];
    const double2 *__restrict__ sn = L.sn[blockIdx.y];
    const double2 *__restrict__ snm1 = L.snm1[blockIdx.y];
    GRID_LOOP(n) {
        double2 a = cn[idx], b = sn[idx], c = cnm1[idx], d = snm1[idx];
        nl[idx] = make_double2(3.0 * (a.x - tinv * b.x) - (c.x - tinv * d.x), 3.0 * (a.y - tinv * b.y) - (c.y - tinv * d.y));
    }
}

__global__ void k_polyforce(const double2 *s11, const double2 *s12, const double2 *s13, const double2 *s22,
                            const double2 *s23, const double2 *s33, const double2 *w1, const double2 *w2,
                            const double2 *w3, double2 *t1, double2 *t2, double2 *t3, const double *wavx,
                            const double *wavz, size_t n, int nyp, int nz) {
    GRID_LOOP(n) {
        DECOMP();
        const double kx = wavx[k], kz = wavz[j];
        double2 a = cimul(make_double2(kx * s11[idx].x + kz * s13[idx].x, kx * s11[idx].y + kz * s13[idx].y), 1.0);
        double2 b = cimul(make_double2(kx * s12[idx].x + kz * s23[idx].x, kx * s12[idx].y + kz * s23[idx].y), 1.0);
        double2 c = cimul(make_double2(kx * s13[idx].x + kz * s33[idx].x, kx * s13[idx].y + kz * s33[idx].y), 1.0);
        t1[idx] = cadd(a, w1[idx]);
        t2[idx] = cadd(b, w2[idx]);
        t3[idx] = cadd(c, w3[idx]);
    }
}

extern "C" int kmm_polyforce(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    double2 *s11 = SPEC(ctx, KMM_QP11), *s12 = SPEC(ctx, KMM_QP12), *s13 = SPEC(ctx, KMM_QP13);
    double2 *s22 = SPEC(ctx, KMM_QP22), *s23 = SPEC(ctx, KMM_QP23), *s33 = SPEC(ctx, KMM_QP33);
    {
        const double2 *in[3] = {s12, s22, s23};
        double2 *out[3] = {ctx->wrk[0], ctx->wrk[1], ctx->wrk[2]};
        RET(kmm_internal_cderiv_many(ctx, in, out, 3));
    }
    k_polyforce<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(
        s11, s12, s13, s22, s23, s33, ctx->wrk[0], ctx->wrk[1], ctx->wrk[2], SPEC(ctx, KMM_T1), SPEC(ctx, KMM_T2),
        SPEC(ctx, KMM_T3), ctx->d_wavx, ctx->d_wavz, ctx->nspec, ctx->nyp, ctx->nz);
    CKL();
    return KMM_OK;
}

__global__ void k_subforce(double2 *gn, double2 *fn, double2 *omz, const double2 *t1, const double2 *t2,
                           const double2 *t3, size_t n) {
    GRID_LOOP(n) {
        gn[idx] = cadd(gn[idx], t1[idx]);
        fn[idx] = cadd(fn[idx], t2[idx]);
        omz[idx] = cadd(omz[idx], t3[idx]);
    }
}

extern "C" int kmm_subforce(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    k_subforce<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(SPEC(ctx, KMM_GN), SPEC(ctx, KMM_FN),
                                                                     SPEC(ctx, KMM_OMZ), SPEC(ctx, KMM_T1),
                                                                     SPEC(ctx, KMM_T2), SPEC(ctx, KMM_T3), ctx->nspec);
    CKL();
    return KMM_OK;
}

// polyNL into six caller-provided buffers
int kmm_internal_polynl(kmm_ctx *ctx, double2 *const *nl) {
    const double tinv = 1.0 / ctx->p.tpoly;
    PolyNlList L;
    for (int m = 0; m < 6; ++m) {
        L.nl[m] = nl[m];
        L.cn[m] = SPEC(ctx, KMM_C11N + m);
        L.cnm1[m] = SPEC(ctx, KMM_C11NM1 + m);
        L.sn[m] = SPEC(ctx, KMM_STR11N + m);
        L.snm1[m] = SPEC(ctx, KMM_STR11NM1 + m);
        if (!L.cn[m] || !L.cnm1[m] || !L.sn[m] || !L.snm1[m]) return KMM_ERR_NOMEM;
    }
    k_polynl<<<dim3(kmm_blocks(ctx->nspec, 256), 6), 256, 0, ctx->stream>>>(L, ctx->nspec, tinv);
    CKL();
    return KMM_OK;
}

// a(0,0 mode, Chebyshev 0) = value, everything else 0 (xyzfft of a constant field)
__global__ void k_constant_mode(double2 *a, size_t n, double value) {
    GRID_LOOP(n) { a[idx] = make_double2(idx == 0 ? value : 0.0, 0.0); }
}

int kmm_internal_set_constant_mode(kmm_ctx *ctx, double2 *a, double value) {
    k_constant_mode<<<kmm_blocks(ctx->nspec, 256), 256, 0, ctx->stream>>>(a, ctx->nspec, value);
    CKL();
    return KMM_OK;
}
