// kmm_fused.cuh -- definitions shared by the fused-step kernels (kmm_fused.cu, kmm_colblk.cu).
#pragma once

#include "kmm_warpcol.cuh"

// tau-solver configurations with tables
enum { TB_PHI = 0, TB_V = 1, TB_OMY = 2, TB_SCL = 3, TB_U0 = 4, TB_W0 = 5, TB_N = 6 };

// per-column tables of one configuration, indexed by coefficient position P = 2 i + parity:
//   td = pivots d(i), te = forward multipliers a3(i)/d(i+1), tb1/tb2 = border weights of the
//   top / bottom boundary row, tf[4] = final border values
struct FusedTabs {
    double *td[TB_N], *te[TB_N], *tb1[TB_N], *tb2[TB_N], *tf[TB_N];
    double g[TB_N];
};

// leading dimension of the column-layout intermediates Y[f][kx][kz][y] and Yo: FP32 columns are
// padded to an even length so that every column starts on a 16-byte boundary (a TMA row); FP64
// columns (16 nyp bytes) need no padding
template <typename C>
__host__ __device__ __forceinline__ int col_ld(int nyp) { return sizeof(C) == 8 ? ((nyp + 1) & ~1) : nyp; }

struct KmmFused {
    FusedTabs tabs;
    // the same tables and rj rows in the lane-blocked order of the blocked column kernels
    // (kmm_colblk.cuh), td there holding 1 / d; built where ny is a multiple of 16
    FusedTabs btabs;
    double2 *yp, *q, *r, *yo;
    double *rj;   // 1/(4j(j-1)), 1/(2(j^2-1)), 1/(4j(j+1)) for j = 0..ny, three rows of nyp
    double *brj;
    float2 *twf_y2, *twf_mz, *twf_mx;   // FP32 twiddles (mixed precision) of lengths 2 ny, mz, mx
};

static __device__ __forceinline__ TauTab tab_at(const FusedTabs &T, int c, int col, int nyp) {
    TauTab t;
    t.td = T.td[c] + (size_t)col * nyp;
    t.te = T.te[c] + (size_t)col * nyp;
    t.tb1 = T.tb1[c] + (size_t)col * nyp;
    t.tb2 = T.tb2[c] + (size_t)col * nyp;
    t.tf = T.tf[c] + (size_t)col * 4;
    return t;
}

struct ColFwdArgs {
    double2 *v, *omy, *fn, *fnm1, *gn, *gnm1, *scal, *scn, *scnm1;
    const double2 *gf1, *gf2, *dnv1b, *dnv1t, *dnv2b, *dnv2t, *denom;
    double *u0, *w0, *h1n, *h1nm1, *h3n, *h3nm1, *scratch;
    double2 *yp;      // y-physical outputs [8][ncols][nyp]
    const double *wavx, *wavz;
    int nz, nxh, nyp, nzh, scalar, nb, nt;
    double re, dt, th, dyde, diff, c0;
    double atu, btu, gtu, abu, bbu, gbu, atw, gtw, abw, bbw, gbw;
};

struct ColBwdArgs {
    const double2 *yo;    // [nout][ncols][nyp]: h1, h2, h3 [, sc]
    double2 *fn, *gn, *omz, *scn;
    double *h1n, *h3n;
    const double *wavx, *wavz;
    int nz, nxh, nyp, nzh, scalar;
    double dyde;
};

// blocked-layout column kernels (kmm_colblk.cu) for ny = 32, 64, 96, 128; KMM_ERR_UNSUPPORTED
// for other ny.  tw: twiddles of length 2 ny in the plane precision (float2 when fp32).
int kmm_colblk_fwd(kmm_ctx *ctx, const ColFwdArgs &A, const FusedTabs &T, const double *rj, const void *tw,
                   bool fp32);
int kmm_colblk_bwd(kmm_ctx *ctx, const ColBwdArgs &B, const void *tw, bool fp32);
