// kmm_colblk.cu -- the column stages of the fused step (kmm_fused.cu) in the blocked layout of
// kmm_colblk.cuh: one warp per (kz, -kz) column pair, 16 lanes per column.  The sequence of
// operations is that of k_col_fwd / k_col_bwd (main_dns.f90:325-544 and 606-771 with
// solvers.f90:555-1722, 3279-3416); only the data layout and the scan structure differ.
#include <math.h>

#include "kmm_fft.cuh"
#include "kmm_colblk.cuh"

#define CB_WARPS 4   // column pairs per block
#ifndef KMM_CB_MINB
#define KMM_CB_MINB 3
#endif
#define CB_MINB KMM_CB_MINB   // blocks per SM the register budget is sized for
// blocks per SM for the FP64 kernels that spill at CB_MINB's register budget: the scalar and u/w
// kernels and the back kernel run faster with two blocks and no (or little) spilling
#ifndef KMM_CB_MINB_FWD
#define KMM_CB_MINB_FWD 2
#endif
#ifndef KMM_CB_MINB_BWD
#define KMM_CB_MINB_BWD 2
#endif
// blocks per SM each kernel's register budget is sized for, as measured per kernel: FP64 scalar,
// u/w and back kernels two, v three, omega_y four; in FP32 the scalar, u/w and omega_y kernels
// four, v and the back kernel three
template <typename C> struct CbMinB {
    static constexpr bool f64 = sizeof(C) == 16;
    static constexpr int fwd = f64 ? KMM_CB_MINB_FWD : 4;   // k_bcol_scl, k_bcol_uw
    static constexpr int omy = 4;   // with bphirhs_g (its histories staged in shared memory)
    static constexpr int v = CB_MINB;
    static constexpr int bwd = f64 ? KMM_CB_MINB_BWD : 3;
};

// shared memory of one warp: region A holds the bload_s / bstore_s scratch (2 (NY + 8) double2)
// and bdct_store / bload_dct's natural-order column pair (2 (NY + 8) elements of C, within the
// swizzled rows); region B the DCT passes' transpose buffer (2 N = 4 NY elements of C).  A's size
// is a multiple of 128 bytes, so B's swizzled rows keep their bank alignment.  bphirhs_g's two
// staged columns (4 (NY + 8) double2) span both regions, which the FP32 forms widen to hold.
template <int K, typename C>
struct CbSmem {
    static constexpr size_t a_bytes = 2 * (16 * K + 8) * sizeof(double2);
    static constexpr size_t b_bytes = 4 * 16 * K * sizeof(C);
    static constexpr size_t stage_bytes = 4 * (16 * K + 8) * sizeof(double2);
    static constexpr size_t warp_bytes = a_bytes + b_bytes > stage_bytes ? a_bytes + b_bytes : stage_bytes;
    static_assert(a_bytes % 128 == 0, "region B starts on a 128-byte boundary");
};

// phirhs on one column pair (solvers.f90:633-675), the n and n-1 terms in registers
template <int K>
__device__ __forceinline__ void bphirhs(BCol<K> &x, const BCol<K> &fn, const BCol<K> &fnm1, double re, double var,
                                        double dt, double th, double w2, double dyde, unsigned mask) {
    const double a = -re * var / (dt * th), b = re * var / (2.0 * th);
    const double c = (1.0 - th) * w2;
    BCol<K> w;
#pragma unroll
    for (int m = 0; m <= K; ++m) {
        double2 r;
        r.x = a * x.v[m].x - b * (3.0 * fn.v[m].x - fnm1.v[m].x);
        r.y = a * x.v[m].y - b * (3.0 * fn.v[m].y - fnm1.v[m].y);
        if (th > 0.99) x.v[m] = r;
        r.x = r.x + c * x.v[m].x / th;
        r.y = r.y + c * x.v[m].y / th;
        w.v[m] = r;
    }
    BCol<K> d1, d2;
    bcderiv<K>(d1, x, dyde, mask);
    bcderiv<K>(d2, d1, dyde, mask);
#pragma unroll
    for (int m = 0; m <= K; ++m)
        x.v[m] = make_double2(w.v[m].x - (1.0 - th) * d2.v[m].x / th, w.v[m].y - (1.0 - th) * d2.v[m].y / th);
}

// The same with the n and n-1 terms read from global memory
// (fn, fnm1 at the pair's columns) through the warp's scratch buf (4 (16 K + 8) double2): both are
// staged with coalesced loads and read slot by slot, and for th <= 0.99 the derivatives are formed
// first, so that at most three column variables are live; per coefficient the arithmetic is
// w = a x - b (3 fn - fnm1) + (1 - th) k^2 x / th, x <- w - (1 - th) x'' / th.
template <int K>
__device__ __forceinline__ void bphirhs_g(BCol<K> &x, const double2 *__restrict__ fn, const double2 *__restrict__ fnm1,
                                          double2 *buf, double re, double var, double dt, double th, double w2,
                                          double dyde, unsigned mask) {
    const double a = -re * var / (dt * th), b = re * var / (2.0 * th);
    const double c = (1.0 - th) * w2;
    const int t = bl_t(), h = (threadIdx.x >> 4) & 1;
    double2 *b0 = buf + h * (16 * K + 8), *b1 = buf + 2 * (16 * K + 8) + h * (16 * K + 8);
    {
        double2 r0[K], r1[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            r0[j] = fn[t + 16 * j];
            r1[j] = fnm1[t + 16 * j];
        }
        const double2 top0 = fn[16 * K], top1 = fnm1[16 * K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            b0[swz<double2>(t + 16 * j)] = r0[j];
            b1[swz<double2>(t + 16 * j)] = r1[j];
        }
        if (t == 15) {
            b0[swz<double2>(16 * K)] = top0;
            b1[swz<double2>(16 * K)] = top1;
        }
    }
    __syncwarp();
    if (th > 0.99) {   // x takes the right-hand side before its derivatives are formed
        BCol<K> w;
#pragma unroll
        for (int m = 0; m <= K; ++m) {
            const int i = bidx<K>(m);
            const double2 f = b0[swz<double2>(i)], fm = b1[swz<double2>(i)];
            double2 r;
            r.x = a * x.v[m].x - b * (3.0 * f.x - fm.x);
            r.y = a * x.v[m].y - b * (3.0 * f.y - fm.y);
            x.v[m] = r;
            r.x = r.x + c * x.v[m].x / th;
            r.y = r.y + c * x.v[m].y / th;
            w.v[m] = r;
        }
        __syncwarp();
        BCol<K> d1, d2;
        bcderiv<K>(d1, x, dyde, mask);
        bcderiv<K>(d2, d1, dyde, mask);
#pragma unroll
        for (int m = 0; m <= K; ++m)
            x.v[m] = make_double2(w.v[m].x - (1.0 - th) * d2.v[m].x / th, w.v[m].y - (1.0 - th) * d2.v[m].y / th);
        return;
    }
    BCol<K> d2;
    {
        BCol<K> d1;
        bcderiv<K>(d1, x, dyde, mask);
        bcderiv<K>(d2, d1, dyde, mask);
    }
#pragma unroll
    for (int m = 0; m <= K; ++m) {
        const int i = bidx<K>(m);
        const double2 f = b0[swz<double2>(i)], fm = b1[swz<double2>(i)];
        double2 r;
        r.x = a * x.v[m].x - b * (3.0 * f.x - fm.x);
        r.y = a * x.v[m].y - b * (3.0 * f.y - fm.y);
        r.x = r.x + c * x.v[m].x / th;
        r.y = r.y + c * x.v[m].y / th;
        x.v[m] = make_double2(r.x - (1.0 - th) * d2.v[m].x / th, r.y - (1.0 - th) * d2.v[m].y / th);
    }
    __syncwarp();
}

// the column pair of the calling warp
struct BPair {
    int kx, q, j, col;
    int tcol;   // column whose tau tables serve this one: kz and -kz share k^2, so half 1 reads half 0's
    size_t off;
    double kxv, kzv, w2;
    bool mean;
};

template <int K>
__device__ __forceinline__ bool bpair(BPair &P, int nz, int nzh, int nxh, const double *wavx, const double *wavz) {
    const int warp = threadIdx.x >> 5, h = (threadIdx.x >> 4) & 1;
    const int npair = nz / 2;
    const int pr = blockIdx.x * CB_WARPS + warp;
    if (pr >= nxh * npair) return false;
    P.q = pr % npair;
    P.kx = pr / npair;
    P.j = h == 0 ? P.q : (P.q == 0 ? nzh : nz - P.q);
    P.col = P.kx * nz + P.j;
    P.tcol = P.q == 0 ? P.col : P.kx * nz + P.q;   // q = 0 pairs kz = 0 with the Nyquist kz: not shared
    P.off = (size_t)P.col * (16 * K + 1);
    P.kxv = wavx[P.kx];
    P.kzv = wavz[P.j];
    P.w2 = P.kzv * P.kzv + P.kxv * P.kxv;
    P.mean = (P.kx == 0 && P.j == 0);
    return true;
}

// The forward column stage as four kernels, in this order (each reads only what the previous
// ones have finished): scalar; omega_y; v (with the mean modes); u, w and the y-physical
// outputs of the velocity.  Splitting keeps each kernel's registers and code small; the price
// is one extra read of v and omega_y.

// passive scalar (main_dns.f90:325-359): CN/AB2 right-hand side, Robin solve, norm, store; y-physical c, dc/dy
template <int K, typename C>
__global__ void __launch_bounds__(CB_WARPS * 32, CbMinB<C>::fwd) k_bcol_scl(ColFwdArgs A, FusedTabs T, const double *__restrict__ rj,
                                                            const C *__restrict__ tw) {
    constexpr int NY = 16 * K, NYP = NY + 1;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ double2 sm[];
    char *wreg = reinterpret_cast<char *>(sm) + (size_t)(threadIdx.x >> 5) * CbSmem<K, C>::warp_bytes;
    C *fa = reinterpret_cast<C *>(wreg), *fb = reinterpret_cast<C *>(wreg + CbSmem<K, C>::a_bytes);
    double2 *wsm = reinterpret_cast<double2 *>(wreg);   // bload_s / bstore_s scratch (fa's space)
    BPair P;
    if (!bpair<K>(P, A.nz, A.nzh, A.nxh, A.wavx, A.wavz)) return;   // whole warps: no block barrier below
    const size_t fstride = (size_t)A.nz * A.nxh * col_ld<C>(NYP), yoff = (size_t)P.col * col_ld<C>(NYP);
    const double2 zero = make_double2(0.0, 0.0);
    BCol<K> s, d1;
    bload_s<K>(s, A.scal + P.off, wsm);
    {
        BCol<K> n1, n0;
        bload_s<K>(n1, A.scn + P.off, wsm);
        bload_s<K>(n0, A.scnm1 + P.off, wsm);
        bphirhs<K>(s, n1, n0, A.re, A.diff, A.dt, A.th, P.w2, A.dyde, FULL);
    }
    const TauTab ts = tab_at(T, TB_SCL, P.tcol, NYP);
    bsolve_robin<K>(s, ts, zero, zero, P.w2 + T.g[TB_SCL], A.c0, rj, FULL);
    bnorm<K>(s, P.kx, P.j, A.nzh);
    bstore_s<K>(A.scal + P.off, s, wsm);
    // one column variable live through each transform (the register-resident FFT needs the rest)
    bdct_store<K, C>(s, fa, fb, tw, (C *)A.yp + 6 * fstride + yoff);
    bcderiv<K>(d1, s, A.dyde, FULL);
    bdct_store<K, C>(d1, fa, fb, tw, (C *)A.yp + 7 * fstride + yoff);
}

// normal vorticity (main_dns.f90:411-422, 479-484, 500-502, 520-526): phirhs, Robin solve, zero
// on the mean column, norm, store; y-physical omega_y
template <int K, typename C>
__global__ void __launch_bounds__(CB_WARPS * 32, CbMinB<C>::omy) k_bcol_omy(ColFwdArgs A, FusedTabs T, const double *__restrict__ rj,
                                                            const C *__restrict__ tw) {
    constexpr int NY = 16 * K, NYP = NY + 1;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ double2 sm[];
    char *wreg = reinterpret_cast<char *>(sm) + (size_t)(threadIdx.x >> 5) * CbSmem<K, C>::warp_bytes;
    C *fa = reinterpret_cast<C *>(wreg), *fb = reinterpret_cast<C *>(wreg + CbSmem<K, C>::a_bytes);
    double2 *wsm = reinterpret_cast<double2 *>(wreg);   // bload_s / bstore_s scratch (fa's space)
    BPair P;
    if (!bpair<K>(P, A.nz, A.nzh, A.nxh, A.wavx, A.wavz)) return;
    const size_t fstride = (size_t)A.nz * A.nxh * col_ld<C>(NYP), yoff = (size_t)P.col * col_ld<C>(NYP);
    const double g1 = A.re / (A.dt * A.th);
    const double2 zero = make_double2(0.0, 0.0);
    BCol<K> om;
    bload_s<K>(om, A.omy + P.off, wsm);
    bphirhs_g<K>(om, A.gn + P.off, A.gnm1 + P.off, wsm, A.re, 1.0, A.dt, A.th, P.w2, A.dyde, FULL);
    const TauTab to = tab_at(T, TB_OMY, P.tcol, NYP);
    bsolve_robin<K>(om, to, zero, zero, P.w2 + g1, A.c0, rj, FULL);
    if (P.mean) {
#pragma unroll
        for (int m = 0; m <= K; ++m) om.v[m] = zero;
    }
    bnorm<K>(om, P.kx, P.j, A.nzh);
    bstore_s<K>(A.omy + P.off, om, wsm);
    bdct_store<K, C>(om, fa, fb, tw, (C *)A.yp + 3 * fstride + yoff);
}

// wall-normal velocity (main_dns.f90:363-407, 426-466, 489-502, 520): phi, phirhs, Helmholtz and
// Poisson solves, influence-matrix correction, uzero for the mean modes, norm, store; y-physical v
template <int K, typename C>
__global__ void __launch_bounds__(CB_WARPS * 32, CbMinB<C>::v) k_bcol_v(ColFwdArgs A, FusedTabs T, const double *__restrict__ rj,
                                                          const C *__restrict__ tw) {
    constexpr int NY = 16 * K, NYP = NY + 1;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ double2 sm[];
    char *wreg = reinterpret_cast<char *>(sm) + (size_t)(threadIdx.x >> 5) * CbSmem<K, C>::warp_bytes;
    C *fa = reinterpret_cast<C *>(wreg), *fb = reinterpret_cast<C *>(wreg + CbSmem<K, C>::a_bytes);
    double2 *wsm = reinterpret_cast<double2 *>(wreg);   // bload_s / bstore_s scratch (fa's space)
    const int lane = threadIdx.x & 31, h = lane >> 4;
    BPair P;
    if (!bpair<K>(P, A.nz, A.nzh, A.nxh, A.wavx, A.wavz)) return;
    const size_t fstride = (size_t)A.nz * A.nxh * col_ld<C>(NYP), yoff = (size_t)P.col * col_ld<C>(NYP);
    const double g1 = A.re / (A.dt * A.th);
    const double2 zero = make_double2(0.0, 0.0);
    const double w2 = P.w2;
    BCol<K> v;
    {
        BCol<K> d1, d2;
        bload_s<K>(v, A.v + P.off, wsm);
        bcderiv<K>(d1, v, A.dyde, FULL);
        bcderiv<K>(d2, d1, A.dyde, FULL);
#pragma unroll
        for (int m = 0; m <= K; ++m) v.v[m] = make_double2(d2.v[m].x - w2 * v.v[m].x, d2.v[m].y - w2 * v.v[m].y);
    }
    if constexpr (sizeof(C) == 16) {   // FP64: the register form (measured faster at this budget)
        BCol<K> f1, f0;
        bload_s<K>(f1, A.fn + P.off, wsm);
        bload_s<K>(f0, A.fnm1 + P.off, wsm);
        bphirhs<K>(v, f1, f0, A.re, 1.0, A.dt, A.th, w2, A.dyde, FULL);
    } else {
        bphirhs_g<K>(v, A.fn + P.off, A.fnm1 + P.off, wsm, A.re, 1.0, A.dt, A.th, w2, A.dyde, FULL);
    }
    {
        const TauTab tp = tab_at(T, TB_PHI, P.tcol, NYP);
        bsolve_dirichlet<K>(v, tp, zero, zero, w2 + g1, A.c0, rj, FULL);
        const TauTab tv = tab_at(T, TB_V, P.tcol, NYP);
        bsolve_dirichlet<K>(v, tv, zero, zero, w2, A.c0, rj, FULL);
    }
    // influence matrix
    {
        double2 wb, wt;
        if (A.nb == 1 && A.nt == 1) {
            bwall1<K>(v, A.dyde, wb, wt, FULL);
        } else {
            BCol<K> dv;
            bcderiv<K>(dv, v, A.dyde, FULL);
            double2 b2, t2;
            bwall1<K>(dv, A.dyde, b2, t2, FULL);
            bwall1<K>(v, A.dyde, wb, wt, FULL);
            if (A.nb == 2) wb = b2;
            if (A.nt == 2) wt = t2;
        }
        const double2 c1 = cdiv(csub(cmul(wb, A.dnv2t[P.col]), cmul(wt, A.dnv2b[P.col])), A.denom[P.col]);
        const double2 c2 = cdiv(csub(cmul(wt, A.dnv1b[P.col]), cmul(wb, A.dnv1t[P.col])), A.denom[P.col]);
        BCol<K> gfa;
        bload_s<K>(gfa, A.gf1 + P.off, wsm);
#pragma unroll
        for (int m = 0; m <= K; ++m) {
            const double2 a = cmul(c1, gfa.v[m]);
            v.v[m] = make_double2(v.v[m].x + a.x, v.v[m].y + a.y);
        }
        bload_s<K>(gfa, A.gf2 + P.off, wsm);
#pragma unroll
        for (int m = 0; m <= K; ++m) {
            const double2 b = cmul(c2, gfa.v[m]);
            v.v[m] = make_double2(v.v[m].x + b.x, v.v[m].y + b.y);
        }
    }
    // mean modes: uzero for u0 and w0 on the (0,0) column's half-warp
    if (P.kx == 0 && P.q == 0) {
        if (h == 0) {
            constexpr unsigned HM = 0x0000ffffu;
            const double th = A.th;
            const int t = lane & 15;
            for (int which = 0; which < 2; ++which) {
                double *U = which == 0 ? A.u0 : A.w0;
                const double *H = which == 0 ? A.h1n : A.h3n, *HL = which == 0 ? A.h1nm1 : A.h3nm1;
                BCol<K> uc, dd1, dd2;
#pragma unroll
                for (int m = 0; m <= K; ++m) uc.v[m] = make_double2(U[bidx<K>(m)], 0.0);
                // wrk1 = -re u0/(dt th) - re (3 h1 - h1l)/(2 th); u0 <- wrk1 - (1-th) u0''/th (solvers.f90:1127-1143)
                bcderiv<K>(dd1, uc, A.dyde, HM);
                bcderiv<K>(dd2, dd1, A.dyde, HM);
#pragma unroll
                for (int m = 0; m <= K; ++m) {
                    const int i = bidx<K>(m);
                    const double w1 = -A.re * uc.v[m].x / (A.dt * th) - A.re * (3.0 * H[i] - HL[i]) / (2.0 * th);
                    const double r = (th > 0.99) ? w1 : w1 - (1.0 - th) * dd2.v[m].x / th;
                    uc.v[m] = make_double2(r, 0.0);
                }
                const TauTab tm = tab_at(T, which == 0 ? TB_U0 : TB_W0, 0, NYP);
                const double gt = which == 0 ? A.gtu : A.gtw, gb = which == 0 ? A.gbu : A.gbw;
                bsolve_robin<K>(uc, tm, make_double2(gt, 0.0), make_double2(gb, 0.0), g1, A.c0, rj, HM);
                __syncwarp(HM);
#pragma unroll
                for (int m = 0; m < K; ++m) U[t * K + m] = uc.v[m].x;
                if (t == 15) U[NY] = uc.v[K].x;
                __syncwarp(HM);
            }
        }
        __syncwarp();
        for (int i = lane; i < NYP; i += 32) {
            A.h1nm1[i] = A.h1n[i];
            A.h3nm1[i] = A.h3n[i];
        }
    }
    bnorm<K>(v, P.kx, P.j, A.nzh);
    if (P.mean) {
#pragma unroll
        for (int m = 0; m <= K; ++m) v.v[m] = zero;
    }
    bstore_s<K>(A.v + P.off, v, wsm);
    bdct_store<K, C>(v, fa, fb, tw, (C *)A.yp + 1 * fstride + yoff);
}

// veloc (solvers.f90:1576-1659) from the new v and omega_y; y-physical u, du/dy, w, dw/dy
template <int K, typename C>
__global__ void __launch_bounds__(CB_WARPS * 32, CbMinB<C>::fwd) k_bcol_uw(ColFwdArgs A, const C *__restrict__ tw) {
    constexpr int NY = 16 * K, NYP = NY + 1;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ double2 sm[];
    char *wreg = reinterpret_cast<char *>(sm) + (size_t)(threadIdx.x >> 5) * CbSmem<K, C>::warp_bytes;
    C *fa = reinterpret_cast<C *>(wreg), *fb = reinterpret_cast<C *>(wreg + CbSmem<K, C>::a_bytes);
    double2 *wsm = reinterpret_cast<double2 *>(wreg);   // bload_s / bstore_s scratch (fa's space)
    BPair P;
    if (!bpair<K>(P, A.nz, A.nzh, A.nxh, A.wavx, A.wavz)) return;
    const size_t fstride = (size_t)A.nz * A.nxh * col_ld<C>(NYP), yoff = (size_t)P.col * col_ld<C>(NYP);
    const double2 zero = make_double2(0.0, 0.0);
    const double kxv = P.kxv, kzv = P.kzv, w2 = P.w2;
    BCol<K> u, w;
    {
        BCol<K> v, om, dv;
        bload_s<K>(v, A.v + P.off, wsm);
        bload_s<K>(om, A.omy + P.off, wsm);
        bcderiv<K>(dv, v, A.dyde, FULL);
#pragma unroll
        for (int m = 0; m <= K; ++m) {
            const double2 d = dv.v[m], o = om.v[m];
            if (P.kx > 0) {
                const double2 sa = cadd(cimul(d, -kxv), cimul(o, kzv));
                u.v[m] = make_double2(-sa.x / w2, -sa.y / w2);
                const double2 sb = csub(cimul(d, -kzv), cimul(o, kxv));
                w.v[m] = make_double2(-sb.x / w2, -sb.y / w2);
            } else if (P.j > 0) {
                const double kz2 = kzv * kzv;
                const double2 sa = cimul(o, kzv);
                u.v[m] = make_double2(-sa.x / kz2, -sa.y / kz2);
                const double2 sb = cimul(d, -kzv);
                w.v[m] = make_double2(-sb.x / kz2, -sb.y / kz2);
            } else {
                u.v[m] = zero;
                w.v[m] = zero;
            }
        }
    }
    if (P.mean) {
#pragma unroll
        for (int m = 0; m <= K; ++m) {
            const int i = bidx<K>(m);
            u.v[m] = make_double2(A.u0[i], 0.0);
            w.v[m] = make_double2(A.w0[i], 0.0);
        }
    }
    // norm(u), norm(w): the pair is conjugate-symmetric already; zero the kz Nyquist column
    if (P.j == A.nzh) {
#pragma unroll
        for (int m = 0; m <= K; ++m) {
            u.v[m] = zero;
            w.v[m] = zero;
        }
    }
    BCol<K> d1;
    bcderiv<K>(d1, u, A.dyde, FULL);
    bdct_store<K, C>(u, fa, fb, tw, (C *)A.yp + 0 * fstride + yoff);
    bdct_store<K, C>(d1, fa, fb, tw, (C *)A.yp + 4 * fstride + yoff);
    bcderiv<K>(d1, w, A.dyde, FULL);
    bdct_store<K, C>(w, fa, fb, tw, (C *)A.yp + 2 * fstride + yoff);
    bdct_store<K, C>(d1, fa, fb, tw, (C *)A.yp + 5 * fstride + yoff);
}

template <int K, typename C>
__global__ void __launch_bounds__(CB_WARPS * 32, CbMinB<C>::bwd) k_bcol_bwd(ColBwdArgs A, const C *__restrict__ tw) {
    constexpr int NY = 16 * K, NYP = NY + 1;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, h = lane >> 4;
    char *wreg = reinterpret_cast<char *>(sm) + (size_t)warp * CbSmem<K, C>::warp_bytes;
    C *fa = reinterpret_cast<C *>(wreg), *fb = reinterpret_cast<C *>(wreg + CbSmem<K, C>::a_bytes);
    double2 *wsm = reinterpret_cast<double2 *>(wreg);   // bload_s / bstore_s scratch (fa's space)
    const int npair = A.nz / 2;
    const int pr = blockIdx.x * CB_WARPS + warp;
    if (pr >= A.nxh * npair) return;
    const int q = pr % npair, kx = pr / npair;
    const int j = h == 0 ? q : (q == 0 ? A.nzh : A.nz - q);
    const int col = kx * A.nz + j;
    const size_t off = (size_t)col * NYP;
    const size_t ncols = (size_t)A.nz * A.nxh;
    const double kxv = A.wavx[kx], kzv = A.wavz[j];
    // spectral filter (main_dns.f90:710-745): exp(-3 (|kz|/nzh)^10) exp(-3 (i/ny)^10)
    const int j1 = j + 1;
    const int jjf = (j1 > A.nzh) ? A.nz - j1 + 1 : j1 - 1;
    const double zr = (double)jjf / (double)A.nzh;
    const double z2 = zr * zr, z4 = z2 * z2, z8 = z4 * z4;
    const double zs = exp(-3.0 * (z8 * z2));
    double ys[K + 1];
#pragma unroll
    for (int m = 0; m <= K; ++m) {
        const double yr = (double)bidx<K>(m) / (double)NY;
        const double y2 = yr * yr, y4 = y2 * y2, y8 = y4 * y4;
        ys[m] = exp(-3.0 * (y8 * y2));
    }
    auto filt = [&](BCol<K> &x) {
#pragma unroll
        for (int m = 0; m <= K; ++m) x.v[m] = make_double2(x.v[m].x * zs * ys[m], x.v[m].y * zs * ys[m]);
    };
    // each term: DCT back (/ny, halved ends), norm after vcw3dp (main_dns.f90:620-624), filter.
    // The scalar term first, then h1 and h3 (gn, omz and the y-derivative fn needs), then h2.
    if (A.scalar) {
        BCol<K> sc;
        bload_dct<K, C>(sc, (const C *)A.yo + (3 * ncols + col) * col_ld<C>(NYP), fa, fb, tw);
        bnorm<K>(sc, kx, j, A.nzh);
        filt(sc);
        bstore_s<K>(A.scn + off, sc, wsm);
    }
    if constexpr (sizeof(C) == 16) {
        // one column variable live through each transform: h3 is stored as omz and re-read (from L2)
        // once h1 has been transformed, and -d waits in fn's output column while h2 is transformed
        {
            BCol<K> h3;
            bload_dct<K, C>(h3, (const C *)A.yo + (2 * ncols + col) * col_ld<C>(NYP), fa, fb, tw);
            bnorm<K>(h3, kx, j, A.nzh);
            filt(h3);
            bstore_s<K>(A.omz + off, h3, wsm);
        }
        BCol<K> d;
        {
            BCol<K> h1, h3;
            bload_dct<K, C>(h1, (const C *)A.yo + (0 * ncols + col) * col_ld<C>(NYP), fa, fb, tw);
            bnorm<K>(h1, kx, j, A.nzh);
            filt(h1);
            __syncwarp();
            bload_s<K>(h3, A.omz + off, wsm);
            // h1n = Re gn(:,1,1), h3n = Re omz(:,1,1) (main_dns.f90:748-751)
            if (kx == 0 && j == 0) {
                const int t = lane & 15;
    #pragma unroll
                for (int m = 0; m < K; ++m) {
                    A.h1n[t * K + m] = h1.v[m].x;
                    A.h3n[t * K + m] = h3.v[m].x;
                }
                if (t == 15) {
                    A.h1n[NY] = h1.v[K].x;
                    A.h3n[NY] = h3.v[K].x;
                }
            }
            // nonlin (solvers.f90:1497-1572): fn = -k^2 h2 - d/dy(i(kz h3 + kx h1)); gn = i(kz h1 - kx h3)
            BCol<K> tt;
    #pragma unroll
            for (int m = 0; m <= K; ++m) {
                const double2 s = make_double2(kzv * h3.v[m].x + kxv * h1.v[m].x, kzv * h3.v[m].y + kxv * h1.v[m].y);
                tt.v[m] = make_double2(-s.y, s.x);
            }
    #pragma unroll
            for (int m = 0; m <= K; ++m) {
                const double2 s = make_double2(kzv * h1.v[m].x - kxv * h3.v[m].x, kzv * h1.v[m].y - kxv * h3.v[m].y);
                h1.v[m] = make_double2(-s.y, s.x);
            }
            bstore_s<K>(A.gn + off, h1, wsm);
            bcderiv<K>(d, tt, A.dyde, FULL);
        }
    #pragma unroll
        for (int m = 0; m <= K; ++m) d.v[m] = make_double2(-d.v[m].x, -d.v[m].y);
        bstore_s<K>(A.fn + off, d, wsm);
        BCol<K> h2;
        bload_dct<K, C>(h2, (const C *)A.yo + (1 * ncols + col) * col_ld<C>(NYP), fa, fb, tw);
        bnorm<K>(h2, kx, j, A.nzh);
        filt(h2);
        __syncwarp();
        bload_s<K>(d, A.fn + off, wsm);
        const double w2 = -kxv * kxv - kzv * kzv;
    #pragma unroll
        for (int m = 0; m <= K; ++m) h2.v[m] = make_double2(w2 * h2.v[m].x + d.v[m].x, w2 * h2.v[m].y + d.v[m].y);
        bstore_s<K>(A.fn + off, h2, wsm);
    } else {   // FP32 transforms: the register budget holds h1, h3 and d at once
        BCol<K> h1, h3, d;
        bload_dct<K, C>(h1, (const C *)A.yo + (0 * ncols + col) * col_ld<C>(NYP), fa, fb, tw);
        bload_dct<K, C>(h3, (const C *)A.yo + (2 * ncols + col) * col_ld<C>(NYP), fa, fb, tw);
        bnorm<K>(h1, kx, j, A.nzh);
        bnorm<K>(h3, kx, j, A.nzh);
        filt(h3);
        filt(h1);
        // h1n = Re gn(:,1,1), h3n = Re omz(:,1,1) (main_dns.f90:748-751)
        if (kx == 0 && j == 0) {
            const int t = lane & 15;
    #pragma unroll
            for (int m = 0; m < K; ++m) {
                A.h1n[t * K + m] = h1.v[m].x;
                A.h3n[t * K + m] = h3.v[m].x;
            }
            if (t == 15) {
                A.h1n[NY] = h1.v[K].x;
                A.h3n[NY] = h3.v[K].x;
            }
        }
        // nonlin (solvers.f90:1497-1572): fn = -k^2 h2 - d/dy(i(kz h3 + kx h1)); gn = i(kz h1 - kx h3)
        {
            BCol<K> tt;
    #pragma unroll
            for (int m = 0; m <= K; ++m) {
                const double2 s = make_double2(kzv * h3.v[m].x + kxv * h1.v[m].x, kzv * h3.v[m].y + kxv * h1.v[m].y);
                tt.v[m] = make_double2(-s.y, s.x);
            }
            bcderiv<K>(d, tt, A.dyde, FULL);
        }
    #pragma unroll
        for (int m = 0; m <= K; ++m) {
            const double2 s = make_double2(kzv * h1.v[m].x - kxv * h3.v[m].x, kzv * h1.v[m].y - kxv * h3.v[m].y);
            h1.v[m] = make_double2(-s.y, s.x);
        }
        bstore_s<K>(A.gn + off, h1, wsm);
        bstore_s<K>(A.omz + off, h3, wsm);
        BCol<K> h2;
        bload_dct<K, C>(h2, (const C *)A.yo + (1 * ncols + col) * col_ld<C>(NYP), fa, fb, tw);
        bnorm<K>(h2, kx, j, A.nzh);
        filt(h2);
        const double w2 = -kxv * kxv - kzv * kzv;
    #pragma unroll
        for (int m = 0; m <= K; ++m) h2.v[m] = make_double2(w2 * h2.v[m].x - d.v[m].x, w2 * h2.v[m].y - d.v[m].y);
        bstore_s<K>(A.fn + off, h2, wsm);
    }
    (void)h;
}

// K = ny / 16 where blocked kernels are compiled: the fused column kernels for ny = 32 .. 128 (K <=
// 8), the routine path's solver also for ny = 256
static int colblk_k(const kmm_ctx *ctx) {
    const int ny = ctx->ny;
    if (ny != 32 && ny != 64 && ny != 96 && ny != 128 && ny != 256) return 0;
    return ny / 16;
}

int kmm_colblk_fwd(kmm_ctx *ctx, const ColFwdArgs &A, const FusedTabs &T, const double *rj, const void *tw,
                   bool fp32) {
    const int K = colblk_k(ctx);
    if (!K) return KMM_ERR_UNSUPPORTED;
    const int npairs = ctx->nxh * (ctx->nz / 2);
    const int nblk = (npairs + CB_WARPS - 1) / CB_WARPS;
    // scalar and omega_y (independent of v and of each other) on the two side streams, v on the
    // main stream, so each kernel's last partial wave overlaps the others; u, w after all three
    cudaStream_t s_scl = ctx->side, s_omy = ctx->side2;
    CK(cudaEventRecord(ctx->cfork_ev, ctx->stream));
    CK(cudaStreamWaitEvent(s_omy, ctx->cfork_ev, 0));
    if (A.scalar) CK(cudaStreamWaitEvent(s_scl, ctx->cfork_ev, 0));
#define BF(KK, CC)                                                                                    \
    do {                                                                                              \
        const CC *twc = (const CC *)tw;                                                               \
        const size_t smem = (size_t)CB_WARPS * CbSmem<KK, CC>::warp_bytes;                            \
        if (A.scalar) {                                                                               \
            RET(kmm_smem_attr(ctx, (const void *)k_bcol_scl<KK, CC>, smem));                          \
            k_bcol_scl<KK, CC><<<nblk, CB_WARPS * 32, smem, s_scl>>>(A, T, rj, twc);                   \
            CKL();                                                                                    \
            CK(cudaEventRecord(ctx->cjoin_ev[0], s_scl));                                             \
        }                                                                                             \
        RET(kmm_smem_attr(ctx, (const void *)k_bcol_omy<KK, CC>, smem));                              \
        k_bcol_omy<KK, CC><<<nblk, CB_WARPS * 32, smem, s_omy>>>(A, T, rj, twc);                       \
        CKL();                                                                                        \
        CK(cudaEventRecord(ctx->cjoin_ev[1], s_omy));                                                 \
        RET(kmm_smem_attr(ctx, (const void *)k_bcol_v<KK, CC>, smem));                                \
        k_bcol_v<KK, CC><<<nblk, CB_WARPS * 32, smem, ctx->stream>>>(A, T, rj, twc);                   \
        CKL();                                                                                        \
        RET(kmm_flowrate_apply(ctx, ctx->stream));                                                    \
        if (A.scalar) CK(cudaStreamWaitEvent(ctx->stream, ctx->cjoin_ev[0], 0));                      \
        CK(cudaStreamWaitEvent(ctx->stream, ctx->cjoin_ev[1], 0));                                    \
        RET(kmm_smem_attr(ctx, (const void *)k_bcol_uw<KK, CC>, smem));                               \
        k_bcol_uw<KK, CC><<<nblk, CB_WARPS * 32, smem, ctx->stream>>>(A, twc);                         \
        CKL();                                                                                        \
        return KMM_OK;                                                                                \
    } while (0)
    if (fp32) {
        switch (K) {
        case 2: BF(2, float2);
        case 4: BF(4, float2);
        case 6: BF(6, float2);
        case 8: BF(8, float2);
        default: return KMM_ERR_UNSUPPORTED;
        }
    }
    switch (K) {
    case 2: BF(2, double2);
    case 4: BF(4, double2);
    case 6: BF(6, double2);
    case 8: BF(8, double2);
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef BF
}

// ---------------------------------------------------------------------------
// The routine path's solve (Dirichlet, solvers.f90:174-553) and penta (Robin, 680-1061) with
// ib = 0 over a whole field in the blocked layout: one warp per (kz, -kz) pair, the boundary
// values from bctop / bcbot, the configuration's tables from the per-context cache.
// ---------------------------------------------------------------------------
struct SolveList {
    double2 *u[KMM_SOLVE_BATCH];
};

template <int K>
__global__ void __launch_bounds__(CB_WARPS * 32, CB_MINB) k_bsolve(SolveList ul, const double2 *__restrict__ gtop,
                                                                  const double2 *__restrict__ gbot, const double *td,
                                                                  const double *te, const double *tb1,
                                                                  const double *tb2, const double *tf,
                                                                  const double *__restrict__ rj,
                                                                  const double *__restrict__ wavx,
                                                                  const double *__restrict__ wavz, int nz, int nzh,
                                                                  int nxh, double g, int robin, double c0) {
    constexpr int NYP = 16 * K + 1;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ double2 sbuf[CB_WARPS][2 * (16 * K + 8)];
    double2 *wsm = sbuf[threadIdx.x >> 5];   // bload_s / bstore_s scratch
    double2 *u = ul.u[blockIdx.y];
    BPair P;
    if (!bpair<K>(P, nz, nzh, nxh, wavx, wavz)) return;
    TauTab T;
    T.td = td + (size_t)P.tcol * NYP;
    T.te = te + (size_t)P.tcol * NYP;
    T.tb1 = tb1 + (size_t)P.tcol * NYP;
    T.tb2 = tb2 + (size_t)P.tcol * NYP;
    T.tf = tf + (size_t)P.tcol * 4;
    BCol<K> s;
    bload_s<K>(s, u + P.off, wsm);
    const double2 gt = gtop[P.col], gb = gbot[P.col];
    if (robin) bsolve_robin<K>(s, T, gt, gb, P.w2 + g, c0, rj, FULL);
    else bsolve_dirichlet<K>(s, T, gt, gb, P.w2 + g, c0, rj, FULL);
    bstore_s<K>(u + P.off, s, wsm);
}

int kmm_colblk_solve_many(kmm_ctx *ctx, double2 *const *u, int nf, double g, int robin, double at, double bt,
                          double ab, double bb, const double2 *gt, const double2 *gb) {
    const int K = colblk_k(ctx);
    if (!K || !ctx->use_colblk) return KMM_ERR_UNSUPPORTED;
    const double *tb[5], *rj = NULL;
    const int st = kmm_tau_tabset(ctx, g, robin, at, bt, ab, bb, tb, &rj);
    if (st != KMM_OK) return st;
    const int npairs = ctx->nxh * (ctx->nz / 2);
    const int nblk = (npairs + CB_WARPS - 1) / CB_WARPS;
    for (int f0 = 0; f0 < nf; f0 += KMM_SOLVE_BATCH) {
        const int nb = nf - f0 < KMM_SOLVE_BATCH ? nf - f0 : KMM_SOLVE_BATCH;
        SolveList ul;
        for (int m = 0; m < nb; ++m) ul.u[m] = u[f0 + m];
        const dim3 grid(nblk, nb);
#define BS(KK)                                                                                                      \
    k_bsolve<KK><<<grid, CB_WARPS * 32, 0, ctx->stream>>>(ul, gt, gb, tb[0], tb[1], tb[2], tb[3], tb[4], rj,         \
                                                          ctx->d_wavx, ctx->d_wavz, ctx->nz, ctx->nzh, ctx->nxh, g, \
                                                          robin, ctx->h_c[0])
        switch (K) {
        case 2: BS(2); break;
        case 4: BS(4); break;
        case 6: BS(6); break;
        case 8: BS(8); break;
        case 16: BS(16); break;
        default: return KMM_ERR_UNSUPPORTED;
        }
#undef BS
        CKL();
    }
    return KMM_OK;
}

int kmm_colblk_solve(kmm_ctx *ctx, double2 *u, double g, int robin, double at, double bt, double ab, double bb,
                     const double2 *gt, const double2 *gb) {
    return kmm_colblk_solve_many(ctx, &u, 1, g, robin, at, bt, ab, bb, gt, gb);
}

// ---------------------------------------------------------------------------
// The routine step's phirhs followed by its solve(s), in one pass over each column pair: [phi =
// v'' - k^2 v (main_dns.f90:363-375),] phirhs (solvers.f90:555-676) with the nonlinear terms fn,
// fnm1 (fnm1 = NULL: the n-1 term is 2 fn), then one or two tau solves with zero boundary values
// (solve, solvers.f90:174-553, or penta, 680-1061; ib = 0).  The same arithmetic as k_phirhs_a /
// cderiv / k_phirhs_b followed by k_bsolve, without the intermediate fields.
// ---------------------------------------------------------------------------
struct PhiSolveJobs {
    double2 *x[KMM_SOLVE_BATCH];
    const double2 *fn[KMM_SOLVE_BATCH];
    const double2 *fnm1[KMM_SOLVE_BATCH];
};

struct PhiSolveCfg {   // the cached tables of one solve's configuration, its g, Robin (1) or Dirichlet (0)
    const double *tab[5];
    double g;
    int robin;
};

template <int K>
__device__ __forceinline__ void bsolve_cfg(BCol<K> &x, const PhiSolveCfg &S, const BPair &P, double c0,
                                           const double *rj) {
    constexpr int NYP = 16 * K + 1;
    constexpr unsigned FULL = 0xffffffffu;
    const double2 zero = make_double2(0.0, 0.0);
    TauTab T;
    T.td = S.tab[0] + (size_t)P.tcol * NYP;
    T.te = S.tab[1] + (size_t)P.tcol * NYP;
    T.tb1 = S.tab[2] + (size_t)P.tcol * NYP;
    T.tb2 = S.tab[3] + (size_t)P.tcol * NYP;
    T.tf = S.tab[4] + (size_t)P.tcol * 4;
    if (S.robin) bsolve_robin<K>(x, T, zero, zero, P.w2 + S.g, c0, rj, FULL);
    else bsolve_dirichlet<K>(x, T, zero, zero, P.w2 + S.g, c0, rj, FULL);
}

// (ny = 256: the 17 coefficients per lane of each column need the 2-block register budget)
template <int K>
__global__ void __launch_bounds__(CB_WARPS * 32, K > 8 ? 2 : CB_MINB)
    k_bphirhs_solve(PhiSolveJobs J, PhiSolveCfg S0, PhiSolveCfg S1, int nsolve, int phi,
                    const double *__restrict__ rj, const double *__restrict__ wavx, const double *__restrict__ wavz,
                    int nz, int nzh, int nxh, double re, double var, double dt, double th, double dyde, double c0) {
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ double2 sbuf[CB_WARPS][2 * (16 * K + 8)];
    double2 *wsm = sbuf[threadIdx.x >> 5];   // bload_s / bstore_s scratch
    double2 *X = J.x[blockIdx.y];
    const double2 *F = J.fn[blockIdx.y], *FM = J.fnm1[blockIdx.y];
    BPair P;
    if (!bpair<K>(P, nz, nzh, nxh, wavx, wavz)) return;
    BCol<K> x;
    bload_s<K>(x, X + P.off, wsm);
    if (phi) {
        BCol<K> d1, d2;
        bcderiv<K>(d1, x, dyde, FULL);
        bcderiv<K>(d2, d1, dyde, FULL);
#pragma unroll
        for (int m = 0; m <= K; ++m)
            x.v[m] = make_double2(d2.v[m].x - P.w2 * x.v[m].x, d2.v[m].y - P.w2 * x.v[m].y);
    }
    {
        BCol<K> f1, f0;
        bload_s<K>(f1, F + P.off, wsm);
        if (FM) {
            bload_s<K>(f0, FM + P.off, wsm);
        } else {
#pragma unroll
            for (int m = 0; m <= K; ++m) f0.v[m] = make_double2(2.0 * f1.v[m].x, 2.0 * f1.v[m].y);
        }
        bphirhs<K>(x, f1, f0, re, var, dt, th, P.w2, dyde, FULL);
    }
    bsolve_cfg<K>(x, S0, P, c0, rj);
    if (nsolve > 1) bsolve_cfg<K>(x, S1, P, c0, rj);
    bstore_s<K>(X + P.off, x, wsm);
}

int kmm_colblk_phirhs_solve(kmm_ctx *ctx, double2 *const *x, const double2 *const *fn, const double2 *const *fnm1,
                            int nf, double var, int phi, int nsolve, const KmmSolveSpec *spec) {
    const int K = colblk_k(ctx);
    if (!K || !ctx->use_colblk) return KMM_ERR_UNSUPPORTED;
    if (nf < 1 || nf > KMM_SOLVE_BATCH || nsolve < 1 || nsolve > 2) return KMM_ERR_ARG;
    PhiSolveCfg S[2];
    const double *rj = NULL;
    for (int k = 0; k < 2; ++k) {
        const KmmSolveSpec &q = spec[k < nsolve ? k : 0];
        const int st = kmm_tau_tabset(ctx, q.g, q.robin, q.at, q.bt, q.ab, q.bb, S[k].tab, &rj);
        if (st != KMM_OK) return st;
        S[k].g = q.g;
        S[k].robin = q.robin;
    }
    PhiSolveJobs J;
    for (int m = 0; m < nf; ++m) {
        J.x[m] = x[m];
        J.fn[m] = fn[m];
        J.fnm1[m] = fnm1[m];
    }
    const int npairs = ctx->nxh * (ctx->nz / 2);
    const dim3 grid((npairs + CB_WARPS - 1) / CB_WARPS, nf);
#define PS(KK)                                                                                                    \
    k_bphirhs_solve<KK><<<grid, CB_WARPS * 32, 0, ctx->stream>>>(J, S[0], S[1], nsolve, phi, rj, ctx->d_wavx,   \
                                                                ctx->d_wavz, ctx->nz, ctx->nzh, ctx->nxh, ctx->re, \
                                                                var, ctx->dt, ctx->theta, ctx->dyde, ctx->h_c[0])
    switch (K) {
    case 2: PS(2); break;
    case 4: PS(4); break;
    case 6: PS(6); break;
    case 8: PS(8); break;
    case 16: PS(16); break;
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef PS
    CKL();
    return KMM_OK;
}

int kmm_colblk_bwd(kmm_ctx *ctx, const ColBwdArgs &B, const void *tw, bool fp32) {
    const int K = colblk_k(ctx);
    if (!K) return KMM_ERR_UNSUPPORTED;
    const int npairs = ctx->nxh * (ctx->nz / 2);
    const int nblk = (npairs + CB_WARPS - 1) / CB_WARPS;
#define BB(KK, CC)                                                                                    \
    do {                                                                                              \
        const size_t smem = (size_t)CB_WARPS * CbSmem<KK, CC>::warp_bytes;                            \
        RET(kmm_smem_attr(ctx, (const void *)k_bcol_bwd<KK, CC>, smem));                              \
        k_bcol_bwd<KK, CC><<<nblk, CB_WARPS * 32, smem, ctx->stream>>>(B, (const CC *)tw);             \
        CKL();                                                                                        \
        return KMM_OK;                                                                                \
    } while (0)
    if (fp32) {
        switch (K) {
        case 2: BB(2, float2);
        case 4: BB(4, float2);
        case 6: BB(6, float2);
        case 8: BB(8, float2);
        default: return KMM_ERR_UNSUPPORTED;
        }
    }
    switch (K) {
    case 2: BB(2, double2);
    case 4: BB(4, double2);
    case 6: BB(6, double2);
    case 8: BB(8, double2);
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef BB
}
