// kmm_colblk.cuh -- column primitives with a blocked coefficient layout: a column of nyp = 16 K + 1
// Chebyshev coefficients lives on the 16 lanes of a half-warp, lane t holding the K consecutive
// coefficients i = t K + m (m < K) in v[m] and every lane holding the last coefficient i = 16 K
// in v[K].  A warp carries two columns, the (kz, -kz) pair that norm couples.
//
// Against the strided warp-per-column layout (kmm_warpcol.cuh) a recurrence over the column is a
// short serial pass inside the lane plus a 4-level shuffle scan over the lanes, for both parities
// at once, instead of a 4-level scan per register slot; neighbours i +- 2 cost four shuffles.
//   - cderiv (derivatives.f90:258-314): D_i = sum over m > i, m = i+1 (mod 2) of 2 m f_m dyde,
//     D_0 halved: per-parity suffix sums.
//   - tau right-hand sides (evns/odds, pntevns/pntodds, solvers.f90:387-496, 807-902).
//   - eliminations (eqsolve, pntsolve): forward elimination = affine suffix scan per parity,
//     border row = dot product, back substitution = affine prefix scan, with the per-column
//     pivot / multiplier / border tables the reference's recurrences give (k_tau_tables).
// Every primitive takes the shuffle mask of the lanes that execute it: the full warp, or one
// half-warp (the mean-mode column).
//
// The tau tables and the tau row reciprocals rj are read in the lane-blocked order (bpos): a
// column's table holds coefficient P = t K + m (m < K) at m * 16 + t and P = 16 K at 16 K, so the
// 16 lanes' reads of one slot m are 128 contiguous bytes; the pivot table holds 1 / d(P), the
// pivots being used only as divisors (the same correctly rounded quotient, formed once when the
// tables are built).
#pragma once

#include "kmm_fft.cuh"
#include "kmm_fused.cuh"

template <int K>
struct BCol {
    double2 v[K + 1];
};

__device__ __forceinline__ int bl_t() { return threadIdx.x & 15; }

__device__ __forceinline__ double sh16_down(unsigned m, double v, int off) { return __shfl_down_sync(m, v, off, 16); }
__device__ __forceinline__ double sh16_up(unsigned m, double v, int off) { return __shfl_up_sync(m, v, off, 16); }
__device__ __forceinline__ double sh16_xor(unsigned m, double v, int x) { return __shfl_xor_sync(m, v, x, 16); }
__device__ __forceinline__ double sh16_idx(unsigned m, double v, int src) { return __shfl_sync(m, v, src, 16); }
__device__ __forceinline__ double2 sh16_down(unsigned m, double2 v, int off) {
    return make_double2(sh16_down(m, v.x, off), sh16_down(m, v.y, off));
}
__device__ __forceinline__ double2 sh16_up(unsigned m, double2 v, int off) {
    return make_double2(sh16_up(m, v.x, off), sh16_up(m, v.y, off));
}
__device__ __forceinline__ double2 sh16_xor(unsigned m, double2 v, int x) {
    return make_double2(sh16_xor(m, v.x, x), sh16_xor(m, v.y, x));
}
__device__ __forceinline__ double2 sh16_idx(unsigned m, double2 v, int src) {
    return make_double2(sh16_idx(m, v.x, src), sh16_idx(m, v.y, src));
}

// coefficient index of slot m
template <int K>
__device__ __forceinline__ int bidx(int m) {
    return m < K ? bl_t() * K + m : 16 * K;
}

// position of slot m's coefficient in a lane-blocked table
template <int K>
__device__ __forceinline__ int bpos(int m) {
    return m < K ? m * 16 + bl_t() : 16 * K;
}

template <int K>
__device__ __forceinline__ void bload(BCol<K> &c, const double2 *__restrict__ p) {
    const int t = bl_t();
#pragma unroll
    for (int m = 0; m < K; ++m) c.v[m] = p[t * K + m];
    c.v[K] = p[16 * K];
}

template <int K>
__device__ __forceinline__ void bstore(double2 *__restrict__ p, const BCol<K> &c) {
    const int t = bl_t();
#pragma unroll
    for (int m = 0; m < K; ++m) p[t * K + m] = c.v[m];
    if (t == 15) p[16 * K] = c.v[K];
}

// bload / bstore through the warp's shared scratch buf (2 (16 K + 8) double2): the 16 lanes of a
// column move 16 consecutive coefficients per access (256 contiguous bytes) instead of lane-blocked
// runs 128 B apart, and the blocked layout is formed in shared memory (swizzled rows: both the
// contiguous and the blocked accesses take the minimum number of wavefronts).  Every lane of the
// warp takes part; buf is free again on return.
template <int K>
__device__ __forceinline__ void bload_s(BCol<K> &c, const double2 *__restrict__ p, double2 *buf) {
    const int t = bl_t();
    double2 *b = buf + ((threadIdx.x >> 4) & 1) * (16 * K + 8);
    double2 r[K];
#pragma unroll
    for (int j = 0; j < K; ++j) r[j] = p[t + 16 * j];
    c.v[K] = p[16 * K];
#pragma unroll
    for (int j = 0; j < K; ++j) b[swz<double2>(t + 16 * j)] = r[j];
    __syncwarp();
#pragma unroll
    for (int m = 0; m < K; ++m) c.v[m] = b[swz<double2>(t * K + m)];
    __syncwarp();
}

template <int K>
__device__ __forceinline__ void bstore_s(double2 *__restrict__ p, const BCol<K> &c, double2 *buf) {
    const int t = bl_t();
    double2 *b = buf + ((threadIdx.x >> 4) & 1) * (16 * K + 8);
#pragma unroll
    for (int m = 0; m < K; ++m) b[swz<double2>(t * K + m)] = c.v[m];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < K; ++j) p[t + 16 * j] = b[swz<double2>(t + 16 * j)];
    if (t == 15) p[16 * K] = c.v[K];
    __syncwarp();
}

// sum over the 16 lanes (every lane gets the total)
__device__ __forceinline__ double2 bsum16(unsigned mask, double2 v) {
#pragma unroll
    for (int x = 1; x < 16; x <<= 1) v = cadd(v, sh16_xor(mask, v, x));
    return v;
}

// d = cderiv(f)
template <int K>
__device__ __forceinline__ void bcderiv(BCol<K> &d, const BCol<K> &f, double dyde, unsigned mask) {
    const int t = bl_t();
    double2 w[K];
    double2 te = make_double2(0.0, 0.0), to = make_double2(0.0, 0.0);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const double fi = 2.0 * (double)(t * K + m);
        w[m] = make_double2(fi * f.v[m].x * dyde, fi * f.v[m].y * dyde);
        if (m & 1) to = cadd(to, w[m]);
        else te = cadd(te, w[m]);
    }
    // inclusive suffix sums of the lane totals, then the next lane's value
#pragma unroll
    for (int off = 1; off < 16; off <<= 1) {
        const double2 ue = sh16_down(mask, te, off), uo = sh16_down(mask, to, off);
        if (t + off < 16) {
            te = cadd(te, ue);
            to = cadd(to, uo);
        }
    }
    double2 re = sh16_down(mask, te, 1), ro = sh16_down(mask, to, 1);
    if (t == 15) {
        re = make_double2(0.0, 0.0);
        ro = make_double2(0.0, 0.0);
    }
    const double ft = 2.0 * (double)(16 * K);
    re = cadd(re, make_double2(ft * f.v[K].x * dyde, ft * f.v[K].y * dyde));   // the last (even) coefficient
#pragma unroll
    for (int m = K - 1; m >= 0; --m) {
        if (m & 1) {
            d.v[m] = re;
            ro = cadd(ro, w[m]);
        } else {
            d.v[m] = ro;
            re = cadd(re, w[m]);
        }
    }
    if (t == 0) d.v[0] = make_double2(0.5 * d.v[0].x, 0.5 * d.v[0].y);
    d.v[K] = make_double2(0.0, 0.0);
}

// tau right-hand-side rows of both parities in place; rows i < 2 (the boundary rows) are left as
// they are.  rj: three rows of nyp reciprocals 1/(4j(j-1)), 1/(2(j^2-1)), 1/(4j(j+1)).
template <int K>
__device__ __forceinline__ void btau_rhs(BCol<K> &s, double c0, const double *__restrict__ rj, unsigned mask) {
    constexpr int NY = 16 * K, NYP = NY + 1;
    const int t = bl_t();
    const double2 lo0 = sh16_up(mask, s.v[K - 2], 1), lo1 = sh16_up(mask, s.v[K - 1], 1);
    double2 hi0 = sh16_down(mask, s.v[0], 1), hi1 = sh16_down(mask, s.v[1], 1);
    if (t == 15) {
        hi0 = s.v[K];
        hi1 = make_double2(0.0, 0.0);
    }
    const double2 topm2 = sh16_idx(mask, s.v[K - 2], 15);
    double2 out[K + 1];
#pragma unroll
    for (int m = 0; m <= K; ++m) {
        const int j = bidx<K>(m);
        if (j < 2) {
            out[m] = s.v[m];
            continue;
        }
        const double2 a = m == K ? topm2 : (m >= 2 ? s.v[m - 2] : (m == 0 ? lo0 : lo1));
        const double2 b = s.v[m];
        const double2 c = m == K ? make_double2(0.0, 0.0) : (m + 2 < K ? s.v[m + 2] : (m + 2 == K ? hi0 : hi1));
        const int q = bpos<K>(m);
        const double rj1 = rj[q], rj2 = rj[NYP + q], rj3 = rj[2 * NYP + q];
        double2 w;
        if ((j & 1) == 0) {
            if (j <= NY - 4) {
                const double cm = (j == 2) ? c0 : 1.0;
                w.x = -cm * a.x * rj1 + b.x * rj2 - c.x * rj3;
                w.y = -cm * a.y * rj1 + b.y * rj2 - c.y * rj3;
            } else if (j == NY - 2) {
                w.x = -a.x * rj1 + b.x * rj2;
                w.y = -a.y * rj1 + b.y * rj2;
            } else {   // j == NY
                w.x = -a.x * rj1;
                w.y = -a.y * rj1;
            }
        } else {
            if (j <= NY - 5) {
                w.x = -a.x * rj1 + b.x * rj2 - c.x * rj3;
                w.y = -a.y * rj1 + b.y * rj2 - c.y * rj3;
            } else if (j == NY - 3) {
                w.x = -a.x * rj1 + b.x * rj2;
                w.y = -a.y * rj1 + b.y * rj2;
            } else {   // j == NY - 1
                w.x = -a.x * rj1;
                w.y = -a.y * rj1;
            }
        }
        out[m] = w;
    }
#pragma unroll
    for (int m = 0; m <= K; ++m) s.v[m] = out[m];
}

// forward elimination, per parity p, positions P = 2+p .. top_p descending (top_0 = NY, the last
// coefficient; top_1 = NY-1):  y_P = W_P - te[P] y_{P+2},  y_top = W_top.  Rows P < 2 unchanged.
// Pass 1 composes each lane's affine map from its carry-in to its lowest slot, a shuffle scan
// gives every lane its carry-in, pass 2 runs the recurrence serially from that carry.
template <int K>
__device__ __forceinline__ void bforward(BCol<K> &w, const double *__restrict__ te, unsigned mask) {
    constexpr int NY = 16 * K;
    const int t = bl_t();
    double A0 = 1.0, A1 = 1.0;
    double2 B0 = make_double2(0.0, 0.0), B1 = make_double2(0.0, 0.0);
#pragma unroll
    for (int m = K - 1; m >= 0; --m) {
        const int P = t * K + m;
        const double a = (P < 2 + (m & 1) || P == NY - 1) ? 0.0 : -te[m * 16 + t];
        const double2 W = w.v[m];
        if ((m & 1) == 0) {
            B0 = make_double2(a * B0.x + W.x, a * B0.y + W.y);
            A0 = a * A0;
        } else {
            B1 = make_double2(a * B1.x + W.x, a * B1.y + W.y);
            A1 = a * A1;
        }
    }
    // suffix composition of the lane maps y_low(t) = A_t y_low(t+1) + B_t
#pragma unroll
    for (int off = 1; off < 16; off <<= 1) {
        const double a0 = sh16_down(mask, A0, off), a1 = sh16_down(mask, A1, off);
        const double2 b0 = sh16_down(mask, B0, off), b1 = sh16_down(mask, B1, off);
        if (t + off < 16) {
            B0 = make_double2(A0 * b0.x + B0.x, A0 * b0.y + B0.y);
            B1 = make_double2(A1 * b1.x + B1.x, A1 * b1.y + B1.y);
            A0 = A0 * a0;
            A1 = A1 * a1;
        }
    }
    // carry into lane 15: the last coefficient for the even chain, nothing for the odd one
    const double2 c15 = w.v[K];
    const double2 Y0 = make_double2(A0 * c15.x + B0.x, A0 * c15.y + B0.y);
    double2 c0 = sh16_down(mask, Y0, 1), c1 = sh16_down(mask, B1, 1);
    if (t == 15) {
        c0 = c15;
        c1 = make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int m = K - 1; m >= 0; --m) {
        const int P = t * K + m;
        const double a = (P < 2 + (m & 1) || P == NY - 1) ? 0.0 : -te[m * 16 + t];
        double2 &c = (m & 1) ? c1 : c0;
        c = make_double2(a * c.x + w.v[m].x, a * c.y + w.v[m].y);
        w.v[m] = c;
    }
}

// border rows: sum over P = 2+p .. top_p of tb[P] y_P, for p = 0 (se) and 1 (so)
template <int K>
__device__ __forceinline__ void bborder(const BCol<K> &y, const double *__restrict__ tb, double2 &se, double2 &so,
                                        unsigned mask) {
    const int t = bl_t();
    double2 ae = make_double2(0.0, 0.0), ao = make_double2(0.0, 0.0);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const int P = t * K + m;
        if (P >= 2 + (m & 1)) {
            const double tv = tb[m * 16 + t];
            if (m & 1) {
                ao.x += tv * y.v[m].x;
                ao.y += tv * y.v[m].y;
            } else {
                ae.x += tv * y.v[m].x;
                ae.y += tv * y.v[m].y;
            }
        }
    }
    if (t == 15) {
        const double tv = tb[16 * K];
        ae.x += tv * y.v[K].x;
        ae.y += tv * y.v[K].y;
    }
    se = bsum16(mask, ae);
    so = bsum16(mask, ao);
}

// back substitution, per parity ascending: x_p = x1_p (boundary row), x_P = (y_P - a1(P) x_{P-2}) / d[P]
// with a1(P) = wn / (4P(P-1)) (doubled for P = 2); the same two passes as bforward
template <int K>
__device__ __forceinline__ void bbacksub(BCol<K> &y, double2 x1e, double2 x1o, const double *__restrict__ td, double wn,
                                         const double *__restrict__ rj, unsigned mask) {
    constexpr int NY = 16 * K;
    const int t = bl_t();
    double rd[K], am[K];
    double A0 = 1.0, A1 = 1.0;
    double2 B0 = make_double2(0.0, 0.0), B1 = make_double2(0.0, 0.0);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const int p = m & 1;
        const int P = t * K + m;
        double2 b;
        if (P == p) {
            rd[m] = 0.0;
            am[m] = 0.0;
            b = p ? x1o : x1e;
        } else {
            const double r = td[m * 16 + t];   // 1 / d(P)
            double a1 = wn * rj[m * 16 + t];
            if (P == 2) a1 = 2.0 * a1;
            rd[m] = r;
            am[m] = -a1 * r;
            b = make_double2(y.v[m].x * r, y.v[m].y * r);
        }
        const double a = am[m];
        if (p == 0) {
            B0 = make_double2(a * B0.x + b.x, a * B0.y + b.y);
            A0 = a * A0;
        } else {
            B1 = make_double2(a * B1.x + b.x, a * B1.y + b.y);
            A1 = a * A1;
        }
    }
    // prefix composition of the lane maps x_high(t) = A_t x_high(t-1) + B_t
#pragma unroll
    for (int off = 1; off < 16; off <<= 1) {
        const double a0 = sh16_up(mask, A0, off), a1 = sh16_up(mask, A1, off);
        const double2 b0 = sh16_up(mask, B0, off), b1 = sh16_up(mask, B1, off);
        if (t >= off) {
            B0 = make_double2(A0 * b0.x + B0.x, A0 * b0.y + B0.y);
            B1 = make_double2(A1 * b1.x + B1.x, A1 * b1.y + B1.y);
            A0 = A0 * a0;
            A1 = A1 * a1;
        }
    }
    double2 c0 = sh16_up(mask, B0, 1), c1 = sh16_up(mask, B1, 1);
    if (t == 0) {
        c0 = make_double2(0.0, 0.0);
        c1 = make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const int p = m & 1;
        const int P = t * K + m;
        double2 &c = p ? c1 : c0;
        if (P == p) c = p ? x1o : x1e;
        else c = make_double2(am[m] * c.x + y.v[m].x * rd[m], am[m] * c.y + y.v[m].y * rd[m]);
        y.v[m] = c;
    }
    // the last coefficient (row n of the even system)
    const double2 xm2 = sh16_idx(mask, y.v[K - 2], 15);
    const double r = td[NY];
    const double a = -(wn * rj[NY]) * r;
    y.v[K] = make_double2(a * xm2.x + y.v[K].x * r, a * xm2.y + y.v[K].y * r);
}

// solve(...) with ib = 0 (Dirichlet), solvers.f90:174-283
template <int K>
__device__ __forceinline__ void bsolve_dirichlet(BCol<K> &s, const TauTab &T, double2 bct, double2 bcb, double wn,
                                                 double c0, const double *__restrict__ rj, unsigned mask) {
    btau_rhs<K>(s, c0, rj, mask);
    bforward<K>(s, T.te, mask);
    double2 se, so;
    bborder<K>(s, T.tb1, se, so, mask);
    const double2 w1e = make_double2(0.5 * (bct.x + bcb.x), 0.5 * (bct.y + bcb.y));
    const double2 w1o = make_double2(0.5 * (bct.x - bcb.x), 0.5 * (bct.y - bcb.y));
    const double fe = T.tf[0], fo = T.tf[1];
    const double2 x1e = make_double2((w1e.x - se.x) / fe, (w1e.y - se.y) / fe);
    const double2 x1o = make_double2((w1o.x - so.x) / fo, (w1o.y - so.y) / fo);
    bbacksub<K>(s, x1e, x1o, T.td, wn, rj, mask);
}

// penta(...) Robin BCs, solvers.f90:680-1061
template <int K>
__device__ __forceinline__ void bsolve_robin(BCol<K> &s, const TauTab &T, double2 gtop, double2 gbot, double wn,
                                             double c0, const double *__restrict__ rj, unsigned mask) {
    btau_rhs<K>(s, c0, rj, mask);
    bforward<K>(s, T.te, mask);
    double2 ste, sto, sbe, sbo;
    bborder<K>(s, T.tb1, ste, sto, mask);
    bborder<K>(s, T.tb2, sbe, sbo, mask);
    // s(js) = g(js) - even part - odd part (the reference subtracts the even pass first)
    const double2 s1 = csub(csub(gtop, ste), sto);
    const double2 s2 = csub(csub(gbot, sbe), sbo);
    const double f11 = T.tf[0], f12 = T.tf[1], f21 = T.tf[2], f22 = T.tf[3];
    const double det = f11 * f22 - f21 * f12;
    const double2 x1e = make_double2((s1.x * f22 - s2.x * f12) / det, (s1.y * f22 - s2.y * f12) / det);
    const double2 x1o = make_double2((s2.x * f11 - s1.x * f21) / det, (s2.y * f11 - s1.y * f21) / det);
    bbacksub<K>(s, x1e, x1o, T.td, wn, rj, mask);
}

// wall functionals c1derbw / c1dertw (derivatives.f90:362-401, 522-560)
template <int K>
__device__ __forceinline__ void bwall1(const BCol<K> &f, double dyde, double2 &bot, double2 &top, unsigned mask) {
    const int t = bl_t();
    double2 b = make_double2(0.0, 0.0), tp = make_double2(0.0, 0.0);
#pragma unroll
    for (int m = 0; m <= K; ++m) {
        if (m == K && t != 15) continue;   // the last coefficient counted once
        const int i = bidx<K>(m);
        const double rp = (double)i;
        const double sgn = (i & 1) ? 1.0 : -1.0;
        const double wb = rp * rp * sgn, wt = rp * rp;
        b.x += wb * f.v[m].x * dyde;
        b.y += wb * f.v[m].y * dyde;
        tp.x += wt * f.v[m].x * dyde;
        tp.y += wt * f.v[m].y * dyde;
    }
    bot = bsum16(mask, b);
    top = bsum16(mask, tp);
}

// norm (helpers.f90:91-158) on the column pair of a warp: half 0 holds kz = j, half 1 its
// partner (nz - j, or nzh for j = 0).  On kx = 0 the pair (j, nz-j) averages to a conjugate
// pair, (0,0) becomes real; the kz Nyquist column is zeroed.  Called by the full warp.
template <int K>
__device__ __forceinline__ void bnorm(BCol<K> &x, int kx, int j, int nzh) {
    const int h = (threadIdx.x >> 4) & 1;
    if (kx == 0) {
#pragma unroll
        for (int m = 0; m <= K; ++m) {
            const double2 mine = x.v[m];
            const double2 oth = make_double2(__shfl_xor_sync(0xffffffffu, mine.x, 16), __shfl_xor_sync(0xffffffffu, mine.y, 16));
            if (j != 0 && j != nzh) {
                const double2 aj = h == 0 ? mine : oth, ajp = h == 0 ? oth : mine;
                const double2 mm = make_double2(0.5 * (aj.x + ajp.x), 0.5 * (aj.y - ajp.y));
                x.v[m] = h == 0 ? mm : make_double2(mm.x, -mm.y);
            }
        }
    }
    if (j == nzh) {
#pragma unroll
        for (int m = 0; m <= K; ++m) x.v[m] = make_double2(0.0, 0.0);
    } else if (kx == 0 && j == 0) {
#pragma unroll
        for (int m = 0; m <= K; ++m) x.v[m].y = 0.0;
    }
}

// park a column pair in the warp's shared buffer (swizzled like the DCT buffers) and fetch it back
template <int K>
__device__ __forceinline__ void bstash(const BCol<K> &x, double2 *buf) {
    const int t = bl_t(), h = (threadIdx.x >> 4) & 1;
#pragma unroll
    for (int m = 0; m < K; ++m) buf[swz<double2>(h * 32 * K + t * K + m)] = x.v[m];
    if (t == 15) buf[swz<double2>(h * 32 * K + 16 * K)] = x.v[K];
}
template <int K>
__device__ __forceinline__ void bunstash(BCol<K> &x, const double2 *buf) {
    const int t = bl_t(), h = (threadIdx.x >> 4) & 1;
#pragma unroll
    for (int m = 0; m < K; ++m) x.v[m] = buf[swz<double2>(h * 32 * K + t * K + m)];
    x.v[K] = buf[swz<double2>(h * 32 * K + 16 * K)];
}

// ---- DCT-I by a two-pass FFT with the data in registers -------------------------------------
// The DCT-I of a column (nyp = NY + 1 values) is the DFT of its even extension of length
// N = 2 NY = 16 M.  With n = 16 n1 + n2 and k = k1 + M k2:
//   X[k1 + M k2] = sum_n2 W16^(n2 k2) W_N^(n2 k1) sum_n1 x[16 n1 + n2] W_M^(n1 k1)
// Pass 1: lane n2 of the column's 16 lanes holds x[16 n1 + n2] (n1 < M), takes the M-point DFT
// in registers and applies the twiddle W_N^(n2 k1); one shared-memory transpose; pass 2: lane
// k1 < M takes the 16-point DFT over n2 in registers and holds X[k1 + M k2].  Two shared-memory
// round trips per transform instead of one per Stockham stage.

// The two passes on the warp's two columns.  In: xin[n1] = x[16 n1 + n2] on lane (h, n2).  Out, on
// lane (h, k1 < M): xout[k2] = X[k1 + M k2] for k2 <= 8 (the indices up to N/2 = NY).  tw: the
// N-point twiddles exp(-2 pi i m/N); s: the warp's shared buffer (2 N elements).
template <int K, typename C>
__device__ __forceinline__ void bdct_passes(const C (&xin)[2 * K], C (&xout)[9], C *s, const C *__restrict__ tw) {
    constexpr int M = 2 * K, N = 16 * M;
    const int t = bl_t(), h = (threadIdx.x >> 4) & 1;
    C v[M];
#pragma unroll
    for (int n1 = 0; n1 < M; ++n1) v[n1] = xin[n1];
    RegDft<C, M>::run(v, tw, 16);   // W_M^j = W_N^(16 j)
    // twiddle W_N^(n2 k1); transpose through s[h N + 16 k1 + n2]
#pragma unroll
    for (int k1 = 0; k1 < M; ++k1) {
        const C w = (t * k1) ? kct::mul(v[k1], __ldg(tw + t * k1)) : v[k1];
        s[swz<C>(h * N + 16 * k1 + t)] = w;
    }
    __syncwarp();
    if (t < M) {
        C u[16];
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) u[n2] = s[swz<C>(h * N + 16 * t + n2)];
        RegDft<C, 16>::run(u, tw, M);   // W_16^j = W_N^(M j)
#pragma unroll
        for (int k2 = 0; k2 <= 8; ++k2) xout[k2] = u[k2];
    }
    __syncwarp();
}

// y-physical values of the warp's two columns (DCT-I of c(i)/2-scaled coefficients,
// solvers.f90:2241-2546) written to dst in precision C: the coefficients are rounded to C
// before the transform, which then runs in C.
template <int K, typename C>
__device__ __forceinline__ void bdct_store(const BCol<K> &x, C *a, C *b, const C *tw, C *__restrict__ dst) {
    typedef typename kct::Real<C>::T T;
    constexpr int NY = 16 * K, N = 2 * NY, M = 2 * K;
    const int t = bl_t(), h = (threadIdx.x >> 4) & 1;
    const int base = h * (NY + 8);
    // the scaled column into shared memory in natural order; each lane then gathers its
    // stride-16 subsequence of the even extension
#pragma unroll
    for (int m = 0; m <= K; ++m) {
        if (m == K && t != 15) continue;
        const int i = bidx<K>(m);
        double2 v = x.v[m];
        if (i > 0 && i < NY) v = make_double2(v.x * 0.5, v.y * 0.5);
        a[swz<C>(base + i)] = kct::mk<C>((T)v.x, (T)v.y);
    }
    __syncwarp();
    C xin[M], xout[9];
#pragma unroll
    for (int n1 = 0; n1 < M; ++n1) {
        const int n = 16 * n1 + t;
        xin[n1] = a[swz<C>(base + (n <= NY ? n : N - n))];
    }
    __syncwarp();
    bdct_passes<K, C>(xin, xout, b, tw);
    if (t < M) {
#pragma unroll
        for (int k2 = 0; k2 <= 8; ++k2) {
            const int k = t + M * k2;
            if (k <= NY) dst[k] = xout[k2];
        }
    }
}

// Chebyshev coefficients of the warp's two columns from y-physical values in precision C
// (DCT-I, /ny, first and last halved, solvers.f90:3279-3416); the transform runs in C and the
// result is widened to FP64.
template <int K, typename C>
__device__ __forceinline__ void bload_dct(BCol<K> &x, const C *__restrict__ src, C *a, C *b, const C *tw) {
    constexpr int NY = 16 * K, N = 2 * NY, M = 2 * K;
    const int t = bl_t(), h = (threadIdx.x >> 4) & 1;
    const int base = h * (NY + 8);
    C xin[M], xout[9];
#pragma unroll
    for (int n1 = 0; n1 < M; ++n1) {
        const int n = 16 * n1 + t;
        xin[n1] = src[n <= NY ? n : N - n];
    }
    bdct_passes<K, C>(xin, xout, b, tw);
    // X[k1 + M k2] on lane k1 -> the blocked layout through shared memory
    if (t < M) {
#pragma unroll
        for (int k2 = 0; k2 <= 8; ++k2) {
            const int k = t + M * k2;
            if (k <= NY) a[swz<C>(base + k)] = xout[k2];
        }
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m <= K; ++m) {
        const int i = bidx<K>(m);
        const C c = a[swz<C>(base + i)];
        double2 v = make_double2((double)c.x / (double)NY, (double)c.y / (double)NY);
        if (i == 0 || i == NY) v = make_double2(v.x / 2.0, v.y / 2.0);
        x.v[m] = v;
    }
    __syncwarp();
}

