// kmm_warpcol.cuh -- warp-per-column primitives for the fused column stage.
//
// A warp owns one (kx,kz) column of nyp Chebyshev coefficients in registers with a strided
// layout: lane l, slot e holds coefficient i = l + 32 e.  Coefficient parity equals lane parity,
// so the even and odd tau systems (solvers.f90:174-553, 680-1061) live in the even and odd
// half-warps and every recurrence becomes a shuffle scan with even offsets.
//   - cderiv (derivatives.f90:258-314): per-parity suffix sums of 2 i f_i dyde, shifted by one.
//   - tau right-hand sides (evns/odds, pntevns/pntodds): neighbours i +- 2 by shuffles.
//   - eliminations (eqsolve, pntsolve): forward elimination = affine suffix scan, border row =
//     dot product, back substitution = affine prefix scan; the pivots d(i), the forward
//     multipliers a3(i)/d(i+1) and the border weights depend only on (kx, kz, g, BCs) and come
//     from tables built once per run with the reference's own recurrences.
#pragma once

#include "kmm_internal.cuh"

#define FULLMASK 0xffffffffu

__device__ __forceinline__ double2 shfl_d2(double2 v, int src) {
    return make_double2(__shfl_sync(FULLMASK, v.x, src), __shfl_sync(FULLMASK, v.y, src));
}
__device__ __forceinline__ double2 shfl_down_d2(double2 v, int off) {
    return make_double2(__shfl_down_sync(FULLMASK, v.x, off), __shfl_down_sync(FULLMASK, v.y, off));
}
__device__ __forceinline__ double2 shfl_up_d2(double2 v, int off) {
    return make_double2(__shfl_up_sync(FULLMASK, v.x, off), __shfl_up_sync(FULLMASK, v.y, off));
}
__device__ __forceinline__ double2 shfl_xor_d2(double2 v, int m) {
    return make_double2(__shfl_xor_sync(FULLMASK, v.x, m), __shfl_xor_sync(FULLMASK, v.y, m));
}

template <int E>
struct Col {
    double2 v[E];
};

template <int E>
__device__ __forceinline__ void col_load(Col<E> &c, const double2 *__restrict__ p, int nyp) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane + 32 * e;
        c.v[e] = i < nyp ? p[i] : make_double2(0.0, 0.0);
    }
}

template <int E>
__device__ __forceinline__ void col_store(double2 *__restrict__ p, const Col<E> &c, int nyp) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane + 32 * e;
        if (i < nyp) p[i] = c.v[e];
    }
}

// per-parity warp sum (result at every lane of the same parity)
__device__ __forceinline__ double2 parity_sum(double2 v) {
#pragma unroll
    for (int m = 2; m < 32; m <<= 1) v = cadd(v, shfl_xor_d2(v, m));
    return v;
}
__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int m = 1; m < 32; m <<= 1) v = cadd(v, shfl_xor_d2(v, m));
    return v;
}

// cderiv: D_i = sum_{m > i, m = i+1 mod 2} 2 m f_m dyde, D_0 halved
template <int E>
__device__ __forceinline__ void col_cderiv(Col<E> &d, const Col<E> &f, int nyp, double dyde) {
    const int lane = threadIdx.x & 31;
    double2 S[E];
    double2 carry_e = make_double2(0.0, 0.0), carry_o = make_double2(0.0, 0.0);
#pragma unroll
    for (int e = E - 1; e >= 0; --e) {
        const int i = lane + 32 * e;
        double2 v = (i >= 1 && i < nyp) ? make_double2(2.0 * (double)i * f.v[e].x * dyde, 2.0 * (double)i * f.v[e].y * dyde)
                                        : make_double2(0.0, 0.0);
#pragma unroll
        for (int off = 2; off < 32; off <<= 1) {
            const double2 t = shfl_down_d2(v, off);
            if (lane + off < 32) v = cadd(v, t);
        }
        const double2 te = shfl_d2(v, 0), to = shfl_d2(v, 1);
        S[e] = cadd(v, (lane & 1) ? carry_o : carry_e);
        carry_e = cadd(carry_e, te);
        carry_o = cadd(carry_o, to);
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const double2 nxt = shfl_down_d2(S[e], 1);
        const double2 nb = (e + 1 < E) ? shfl_d2(S[e + 1], 0) : make_double2(0.0, 0.0);
        const int i = lane + 32 * e;
        double2 r = lane < 31 ? nxt : nb;
        if (i >= nyp) r = make_double2(0.0, 0.0);
        if (i == 0) r = make_double2(0.5 * r.x, 0.5 * r.y);
        d.v[e] = r;
    }
}

// neighbours i + 2 and i - 2 (0 outside 0..nyp-1)
template <int E>
__device__ __forceinline__ void col_nbr2(const Col<E> &s, Col<E> &sp2, Col<E> &sm2, int nyp) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const double2 dn = shfl_down_d2(s.v[e], 2);
        const double2 nx = (e + 1 < E) ? shfl_d2(s.v[e + 1], (lane - 30) & 31) : make_double2(0.0, 0.0);
        const double2 up = shfl_up_d2(s.v[e], 2);
        const double2 pv = (e > 0) ? shfl_d2(s.v[e - 1], (lane + 30) & 31) : make_double2(0.0, 0.0);
        const int i = lane + 32 * e;
        sp2.v[e] = (i + 2 < nyp) ? (lane <= 29 ? dn : nx) : make_double2(0.0, 0.0);
        sm2.v[e] = (i - 2 >= 0) ? (lane >= 2 ? up : pv) : make_double2(0.0, 0.0);
    }
}

// tau right-hand-side rows for both parities in place (evns/odds without the BC row,
// solvers.f90:387-496 / pntevns/pntodds 807-902); position i = p (row 1) is left as is
template <int E>
__device__ __forceinline__ void col_tau_rhs(Col<E> &s, int nyp, double c0) {
    const int ny = nyp - 1;
    const int lane = threadIdx.x & 31;
    Col<E> sp2, sm2;
    col_nbr2<E>(s, sp2, sm2, nyp);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int j = lane + 32 * e;
        if (j < 2 || j >= nyp) continue;
        const double rj1 = 1.0 / (double)(4 * j * (j - 1));
        const double rj2 = 1.0 / (double)(2 * (j * j - 1));
        const double rj3 = 1.0 / (double)(4 * j * (j + 1));
        const double2 a = sm2.v[e], b = s.v[e], c = sp2.v[e];
        double2 w;
        if ((j & 1) == 0) {
            if (j <= ny - 4) {
                const double cm = (j == 2) ? c0 : 1.0;
                w.x = -cm * a.x * rj1 + b.x * rj2 - c.x * rj3;
                w.y = -cm * a.y * rj1 + b.y * rj2 - c.y * rj3;
            } else if (j == ny - 2) {
                w.x = -a.x * rj1 + b.x * rj2;
                w.y = -a.y * rj1 + b.y * rj2;
            } else {   // j == ny
                w.x = -a.x * rj1;
                w.y = -a.y * rj1;
            }
        } else {
            if (j <= ny - 5) {
                w.x = -a.x * rj1 + b.x * rj2 - c.x * rj3;
                w.y = -a.y * rj1 + b.y * rj2 - c.y * rj3;
            } else if (j == ny - 3) {
                w.x = -a.x * rj1 + b.x * rj2;
                w.y = -a.y * rj1 + b.y * rj2;
            } else {   // j == ny - 1
                w.x = -a.x * rj1;
                w.y = -a.y * rj1;
            }
        }
        s.v[e] = w;
    }
}

// tau matrix row coefficient a1(i) of evnc / oddc (solvers.f90:324-383), i = 1..m
__device__ __forceinline__ double tau_a1(int i, int par, double wn) {
    const int j = par == 0 ? 2 * i : 2 * i + 1;
    double a1 = wn * (1.0 / (double)(4 * j * (j - 1)));
    if (par == 0 && i == 1) a1 = 2.0 * a1;
    return a1;
}

// Tables per column and configuration, indexed by coefficient position P = 2i + parity:
//   td[P] = d(i) (i >= 1), te[P] = a3(i)/d(i+1) (forward multiplier), tb1/tb2[P] = border weights
//   of rows 2..n (for Dirichlet tb1 only), tf[0..3] = final f values:
//   Dirichlet: tf[par] ; Robin: tf[2*(js-1) + par] = f(js, par)  (js 1 = top / tt, 2 = bottom / tb)
struct TauTab {
    const double *td, *te, *tb1, *tb2, *tf;
};

// forward elimination (affine suffix scan); y at every valid position, BC position untouched
template <int E>
__device__ __forceinline__ void col_forward(Col<E> &w, const double *__restrict__ te, int nyp) {
    const int lane = threadIdx.x & 31, par = lane & 1;
    const int ny = nyp - 1;
    const int n = par == 0 ? ny / 2 + 1 : ny / 2;     // rows
    const int top = 2 * (n - 1) + par;                 // position of row n
    double2 carry = make_double2(0.0, 0.0);
#pragma unroll
    for (int e = E - 1; e >= 0; --e) {
        const int P = lane + 32 * e;
        double a, b0, b1;
        if (P < 2 + par || P > top) {             // BC row or beyond the system: y = W, no coupling
            a = 0.0;
        } else {
            a = (P == top) ? 0.0 : -te[P];
        }
        b0 = (P <= top) ? w.v[e].x : 0.0;
        b1 = (P <= top) ? w.v[e].y : 0.0;
        // inclusive suffix composition within the block: (a,b) <- (a,b) o (a',b')
#pragma unroll
        for (int off = 2; off < 32; off <<= 1) {
            const double a2 = __shfl_down_sync(FULLMASK, a, off);
            const double c0 = __shfl_down_sync(FULLMASK, b0, off);
            const double c1 = __shfl_down_sync(FULLMASK, b1, off);
            if (lane + off < 32) {
                b0 = a * c0 + b0;
                b1 = a * c1 + b1;
                a = a * a2;
            }
        }
        // apply to the carry (y at the lowest position of the next block of this parity)
        double2 y = make_double2(a * carry.x + b0, a * carry.y + b1);
        if (P >= 2 + par && P <= top) w.v[e] = y;
        const double2 ye = shfl_d2(y, 0), yo = shfl_d2(y, 1);
        carry = par ? yo : ye;
    }
}

// border-row dot products sum_{P in rows 2..n} t[P] y_P for this lane's parity
template <int E>
__device__ __forceinline__ double2 col_border(const Col<E> &y, const double *__restrict__ tb, int nyp) {
    const int lane = threadIdx.x & 31, par = lane & 1;
    const int ny = nyp - 1;
    const int n = par == 0 ? ny / 2 + 1 : ny / 2;
    const int top = 2 * (n - 1) + par;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int P = lane + 32 * e;
        if (P >= 2 + par && P <= top) {
            const double t = tb[P];
            acc.x += t * y.v[e].x;
            acc.y += t * y.v[e].y;
        }
    }
    return parity_sum(acc);
}

// back substitution (affine prefix scan) from x at the BC position (row 1)
template <int E>
__device__ __forceinline__ void col_backsub(Col<E> &y, double2 x1, const double *__restrict__ td, double wn, int nyp) {
    const int lane = threadIdx.x & 31, par = lane & 1;
    const int ny = nyp - 1;
    const int n = par == 0 ? ny / 2 + 1 : ny / 2;
    const int top = 2 * (n - 1) + par;
    double2 carry = make_double2(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int P = lane + 32 * e;
        double a = 0.0, b0 = 0.0, b1 = 0.0;
        if (P == par) {
            b0 = x1.x;
            b1 = x1.y;
        } else if (P >= 2 + par && P <= top) {
            const int i = (P - par) / 2;
            const double d = td[P];
            a = -tau_a1(i, par, wn) / d;
            b0 = y.v[e].x / d;
            b1 = y.v[e].y / d;
        }
        // inclusive prefix composition: (a,b) <- (a,b) o (a',b') with (a',b') from lane - off
#pragma unroll
        for (int off = 2; off < 32; off <<= 1) {
            const double a2 = __shfl_up_sync(FULLMASK, a, off);
            const double c0 = __shfl_up_sync(FULLMASK, b0, off);
            const double c1 = __shfl_up_sync(FULLMASK, b1, off);
            if (lane >= off) {
                b0 = a * c0 + b0;
                b1 = a * c1 + b1;
                a = a * a2;
            }
        }
        double2 x = make_double2(a * carry.x + b0, a * carry.y + b1);
        y.v[e] = (P <= top) ? x : make_double2(0.0, 0.0);
        const double2 xe = shfl_d2(x, 30), xo = shfl_d2(x, 31);
        carry = par ? xo : xe;
    }
}

// solve(...) with ib = 0 (Dirichlet), solvers.f90:174-283; s holds the right-hand side column
template <int E>
__device__ __forceinline__ void col_solve_dirichlet(Col<E> &s, const TauTab &T, double2 bct, double2 bcb, double wn,
                                                    int nyp, double c0) {
    const int lane = threadIdx.x & 31, par = lane & 1;
    col_tau_rhs<E>(s, nyp, c0);
    col_forward<E>(s, T.te, nyp);
    const double2 sig = col_border<E>(s, T.tb1, nyp);
    // BC row: even 0.5(top + bot), odd 0.5(top - bot)
    const double2 w1 = par == 0 ? make_double2(0.5 * (bct.x + bcb.x), 0.5 * (bct.y + bcb.y))
                                : make_double2(0.5 * (bct.x - bcb.x), 0.5 * (bct.y - bcb.y));
    const double f = T.tf[par];
    const double2 x1 = make_double2((w1.x - sig.x) / f, (w1.y - sig.y) / f);
    col_backsub<E>(s, x1, T.td, wn, nyp);
}

// penta(...) Robin BCs, solvers.f90:680-1061
template <int E>
__device__ __forceinline__ void col_solve_robin(Col<E> &s, const TauTab &T, double2 gtop, double2 gbot, double wn,
                                                int nyp, double c0) {
    const int lane = threadIdx.x & 31, par = lane & 1;
    col_tau_rhs<E>(s, nyp, c0);
    col_forward<E>(s, T.te, nyp);
    const double2 st = col_border<E>(s, T.tb1, nyp);   // top row (tt) contributions of this parity
    const double2 sb = col_border<E>(s, T.tb2, nyp);   // bottom row (tb)
    const double2 st_o = shfl_xor_d2(st, 1), sb_o = shfl_xor_d2(sb, 1);
    const double2 st_e = par ? st_o : st, st_od = par ? st : st_o;
    const double2 sb_e = par ? sb_o : sb, sb_od = par ? sb : sb_o;
    // s(js) = g(js) - even part - odd part (the reference subtracts the even pass first)
    const double2 s1 = csub(csub(gtop, st_e), st_od);
    const double2 s2 = csub(csub(gbot, sb_e), sb_od);
    const double f11 = T.tf[0], f12 = T.tf[1], f21 = T.tf[2], f22 = T.tf[3];
    const double det = f11 * f22 - f21 * f12;
    double2 x1;
    if (par == 0) x1 = make_double2((s1.x * f22 - s2.x * f12) / det, (s1.y * f22 - s2.y * f12) / det);
    else x1 = make_double2((s2.x * f11 - s1.x * f21) / det, (s2.y * f11 - s1.y * f21) / det);
    col_backsub<E>(s, x1, T.td, wn, nyp);
}

// wall functionals c1derbw / c1dertw (derivatives.f90:362-401, 522-560)
template <int E>
__device__ __forceinline__ void col_wall1(const Col<E> &f, int nyp, double dyde, double2 &bot, double2 &top) {
    const int lane = threadIdx.x & 31;
    double2 b = make_double2(0.0, 0.0), t = make_double2(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int i = lane + 32 * e;
        if (i < nyp) {
            const double rp = (double)i;
            const double sgn = (i & 1) ? 1.0 : -1.0;
            const double wb = rp * rp * sgn, wt = rp * rp;
            b.x += wb * f.v[e].x * dyde;
            b.y += wb * f.v[e].y * dyde;
            t.x += wt * f.v[e].x * dyde;
            t.y += wt * f.v[e].y * dyde;
        }
    }
    bot = warp_sum(b);
    top = warp_sum(t);
}
