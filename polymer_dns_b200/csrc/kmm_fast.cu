// kmm_fast.cu -- the x stage of vcw3dp as one warp-per-row kernel (fluid and scalar terms).
//
// One warp owns one (y, z) row of the 3/2 grid: Hermitian c2r of two fields per complex FFT
// (warp-private Stockham in shared memory, __syncwarp only), the physical values of every field
// held in registers (lane l owns x = l + 32 e), the pointwise terms of solvers.f90:2885-3063
// (u x omega, -u.grad(c), the uniform scalar source, dPdx where imatrix = 0 for flow_select 1,
// CFL and |u|), the tracer copies of u, v, w, then r2c of two outputs per FFT, truncated to kx <
// nxh.  This replaces the k_xphys + k_xfwd pair (and their HBM round trip of the physical
// outputs) whenever there is no polymer and no immersed boundary.
#include <math.h>

#include "kmm_fft.cuh"

#define FX_WARPS 4
// blocks per SM the specialised x stage is register-sized for: three in FP64 (four spill and run no
// faster), four for the FP32 form of the mixed precision (no spills; 7 % faster than three)
template <typename C> struct Fx2MinB { static constexpr int v = sizeof(C) == 16 ? 3 : 4; };

struct FxArgs {
    int nout, ic, flow_select, save_uvw;   // ic: index in q of dc/dx (dc/dy, dc/dz follow), -1 without scalar
    double delxm, delzm, dt, dPdx, scalar_q;
};

// MX > 0: the x length is the compile-time constant MX (specialised FFT); MX = 0: runtime plan.
// q holds u v w wx wy wz at indices 0..5.  The fields are brought to physical space in pairs and
// consumed as soon as the products that need them are formed, so at most seven physical fields
// are live per lane.
template <int E, int MX>
__global__ void __launch_bounds__(FX_WARPS * 32, 3) k_fx(const double2 *__restrict__ q, double2 *__restrict__ r,
                                                      double *__restrict__ up3, double *__restrict__ vp3,
                                                      double *__restrict__ wp3, const double *__restrict__ seght,
                                                      double *__restrict__ cfl, double *__restrict__ umax, const __grid_constant__ DevPlan P,
                                                      FxArgs A, int nyp, int mz, int mx_rt, int nxh) {
    extern __shared__ double2 sm[];
    const int mx = MX > 0 ? MX : mx_rt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = blockIdx.y;
    const int z = blockIdx.x * FX_WARPS + warp;
    double2 *a = sm + (size_t)warp * 2 * mx, *b = a + mx;
    const int hx = mx / 2;
    auto SW = [](int x) { return MX > 0 ? swz<double2>(x) : x; };
    double cmax = 0.0, umx = 0.0;
    // Hermitian c2r of fields f and g (g < 0: none) in one complex FFT: ra = field f, rb = field g
    auto inv_pair = [&](int f, int g, double *ra, double *rb) {
        const double2 *qa = q + (((size_t)f * nyp + y) * mz + z) * nxh;
        const double2 *qb = q + (((size_t)(g < 0 ? f : g) * nyp + y) * mz + z) * nxh;
        for (int k = lane; k < mx; k += 32) {
            const int kk = k <= hx ? k : mx - k;
            double2 Av = make_double2(0.0, 0.0), Bv = make_double2(0.0, 0.0);
            if (kk < nxh) {
                Av = qa[kk];
                if (g >= 0) Bv = qb[kk];
            }
            if (k == 0 || k == hx) { Av.y = 0.0; Bv.y = 0.0; }   // c2r ignores Im of DC / Nyquist
            a[SW(k)] = k <= hx ? make_double2(Av.x - Bv.y, Av.y + Bv.x) : make_double2(Av.x + Bv.y, -Av.y + Bv.x);
        }
        __syncwarp();
        const double2 *res;
        if constexpr (MX > 0) res = fft_warp_ct<double2, MX, +1, 1, true>(a, b, P.tw);
        else res = fft_warp(P, a, b, +1);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = lane + 32 * e;
            if (x < mx) {
                const double2 v = res[SW(x)];
                ra[e] = v.x;
                rb[e] = v.y;
            }
        }
        __syncwarp();
    };
    // r2c of two physical outputs in one complex FFT, kept for kx < nxh: ra -> output o, rb -> o + 1
    auto fwd_pair = [&](int o, bool has_g, const double *ra, const double *rb) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = lane + 32 * e;
            if (x < mx) a[SW(x)] = make_double2(ra[e], has_g ? rb[e] : 0.0);
        }
        __syncwarp();
        const double2 *res;
        if constexpr (MX > 0) res = fft_warp_ct<double2, MX, -1, 1, true>(a, b, P.tw);
        else res = fft_warp(P, a, b, -1);
        double2 *oa = r + (((size_t)o * nyp + y) * mz + z) * nxh;
        double2 *ob = r + (((size_t)(o + 1) * nyp + y) * mz + z) * nxh;
        for (int k = lane; k < nxh; k += 32) {
            const double2 Z = res[SW(k)];
            const double2 Zc = cconj(res[SW(k == 0 ? 0 : mx - k)]);
            oa[k] = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y + Zc.y));
            if (has_g) {
                const double2 d = csub(Z, Zc);
                ob[k] = make_double2(0.5 * d.y, -0.5 * d.x);
            }
        }
        __syncwarp();
    };
    if (z < mz) {
        double u[E], v[E], w[E], t0[E], t1[E], t2[E];
        inv_pair(0, 1, u, v);
        inv_pair(2, 3, w, t0);    // t0 = wx
        inv_pair(4, 5, t1, t2);   // t1 = wy, t2 = wz
        // ---- pointwise terms (solvers.f90:2891-3063)
        const double sg = seght[y];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = lane + 32 * e;
            if (x < mx) {
                const double up = u[e], vp = v[e], wp = w[e];
                const double wxp = t0[e], wyp = t1[e], wzp = t2[e];
                double h1 = vp * wzp - wp * wyp;
                const double h2 = -up * wzp + wp * wxp;
                const double h3 = up * wyp - vp * wxp;
                if (A.flow_select == 1) h1 = h1 - A.dPdx;
                t0[e] = h1;
                t1[e] = h2;
                t2[e] = h3;
                const double cc = (fabs(up) / A.delxm + fabs(vp) / sg + fabs(wp) / A.delzm) * A.dt;
                cmax = (cc != cc) ? cc : fmax(cmax, cc);
                umx = fmax(umx, fabs(up));
                if (A.save_uvw) {
                    const size_t g3 = ((size_t)y * mz + z) * mx + x;
                    up3[g3] = up;
                    vp3[g3] = vp;
                    wp3[g3] = wp;
                }
            }
        }
        fwd_pair(0, true, t0, t1);   // h1, h2
        if (A.ic >= 0) {
            // -u.grad(c) [+ uniform source]: (u cx + v cy) first, then + w cz, as the reference sums
            double sacc[E];
            inv_pair(A.ic, A.ic + 1, t0, t1);
#pragma unroll
            for (int e = 0; e < E; ++e) sacc[e] = u[e] * t0[e] + v[e] * t1[e];
            inv_pair(A.ic + 2, -1, t0, t1);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                double vc = -(sacc[e] + w[e] * t0[e]);
                if (A.scalar_q != 0.0) vc = vc + A.scalar_q;
                t1[e] = vc;
            }
            fwd_pair(2, A.nout > 3, t2, t1);   // h3, scalar term
        } else {
            fwd_pair(2, false, t2, t1);
        }
    }
    // ---- per-plane CFL / |u| maxima
    for (int off = 16; off; off >>= 1) {
        const double c2 = __shfl_down_sync(0xffffffffu, cmax, off);
        const double u2 = __shfl_down_sync(0xffffffffu, umx, off);
        cmax = (c2 != c2) ? c2 : fmax(cmax, c2);
        umx = fmax(umx, u2);
    }
    if (lane == 0 && z < mz) {
        atomicMax((unsigned long long *)&cfl[y], (unsigned long long)__double_as_longlong(cmax));
        atomicMax((unsigned long long *)&umax[y], (unsigned long long)__double_as_longlong(umx));
    }
}

// returns KMM_ERR_UNSUPPORTED when mx has no compiled instance (caller falls back to the general path)
// Specialised x stage for the compiled lengths MX (nxh = MX/3): as k_fx, plus
//   - each field pair is read once (its nxh coefficients per row) and the Hermitian extension is
//     built in shared memory;
//   - the next pair's coefficients are fetched into registers while the current FFT runs;
//   - C = double2 (FP64) or float2 (FP32 transforms and products of the mixed-precision form;
//     the CFL numbers and the tracer copies of u, v, w are widened to FP64).
template <int MX, typename C>
__global__ void __launch_bounds__(FX_WARPS * 32, Fx2MinB<C>::v) k_fx2(const C *__restrict__ q, C *__restrict__ r,
                                                          double *__restrict__ up3, double *__restrict__ vp3,
                                                          double *__restrict__ wp3, const double *__restrict__ seght,
                                                          double *__restrict__ cfl, double *__restrict__ umax,
                                                          const C *__restrict__ tw, FxArgs A, int nyp, int mz) {
    typedef typename kct::Real<C>::T T;
    constexpr int E = (MX + 31) / 32;
    constexpr int NXH = MX / 3;
    constexpr int NE = (NXH + 31) / 32;   // coefficients per lane of one field row
    constexpr int HX = MX / 2;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = blockIdx.y;
    const int z = blockIdx.x * FX_WARPS + warp;
    C *a = sm + (size_t)warp * 2 * MX, *b = a + MX;
    double cmax = 0.0, umx = 0.0;
    const C zc = kct::mk<C>((T)0, (T)0);
    C pa[NE], pb[NE];   // coefficients of the pair in flight
    auto fetch = [&](int f, int g) {
        const C *qa = q + (((size_t)f * nyp + y) * mz + z) * NXH;
        const C *qb = q + (((size_t)(g < 0 ? f : g) * nyp + y) * mz + z) * NXH;
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int k = lane + 32 * e;
            pa[e] = (k < NXH) ? __ldg(qa + k) : zc;
            pb[e] = (g >= 0 && k < NXH) ? __ldg(qb + k) : zc;
        }
    };
    // Hermitian c2r of the fetched pair: Z_k = A_k + i B_k (k <= HX), conj(A) + i conj(B) mirrored
    auto inv = [&](T *ra, T *rb) {
        for (int k = lane; k <= MX - NXH; k += 32)
            if (k >= NXH) a[swz<C>(k)] = zc;   // modes nxh .. mx-nxh are not carried
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int k = lane + 32 * e;
            if (k < NXH) {
                C Av = pa[e], Bv = pb[e];
                if (k == 0) { Av.y = (T)0; Bv.y = (T)0; }   // c2r ignores Im of DC
                a[swz<C>(k)] = kct::mk<C>(Av.x - Bv.y, Av.y + Bv.x);
                if (k > 0) a[swz<C>(MX - k)] = kct::mk<C>(Av.x + Bv.y, -Av.y + Bv.x);
            }
        }
        __syncwarp();
    };
    // the last FFT stage of MX = 96, 192, 576 leaves output x = lane + 32 e in lane `lane` (its
    // stride is a multiple of 32): it writes the lane's registers directly
    constexpr bool REG_OUT = kct::stride(MX, kct::nfac(MX) - 1) % 32 == 0;
    auto run_inv = [&](T *ra, T *rb) {
        if constexpr (REG_OUT) {
            auto ld = [&](int x) { return a[swz<C>(x)]; };
            auto st = [&](int x, C v) {
                ra[x >> 5] = v.x;
                rb[x >> 5] = v.y;
            };
            auto pre = [] {};
            fft_warp_ct_io<C, MX, +1>(ld, st, pre, b, a, tw);
        } else {
            const C *res = fft_warp_ct<C, MX, +1, 1, true>(a, b, tw);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int x = lane + 32 * e;
                if (x < MX) {
                    const C v = res[swz<C>(x)];
                    ra[e] = v.x;
                    rb[e] = v.y;
                }
            }
        }
        __syncwarp();
    };
    auto fwd_pair = [&](int o, bool has_g, const T *ra, const T *rb) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = lane + 32 * e;
            if (x < MX) a[swz<C>(x)] = kct::mk<C>(ra[e], has_g ? rb[e] : (T)0);
        }
        __syncwarp();
        const C *res = fft_warp_ct<C, MX, -1, 1, true>(a, b, tw);
        C *oa = r + (((size_t)o * nyp + y) * mz + z) * NXH;
        C *ob = r + (((size_t)(o + 1) * nyp + y) * mz + z) * NXH;
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int k = lane + 32 * e;
            if (k < NXH) {
                const C Z = res[swz<C>(k)];
                C Zc = res[swz<C>(k == 0 ? 0 : MX - k)];
                Zc.y = -Zc.y;
                oa[k] = kct::mk<C>((T)0.5 * (Z.x + Zc.x), (T)0.5 * (Z.y + Zc.y));
                if (has_g) ob[k] = kct::mk<C>((T)0.5 * (Z.y - Zc.y), (T)-0.5 * (Z.x - Zc.x));
            }
        }
        __syncwarp();
    };
    (void)HX;
    if (z < mz) {
        T u[E], v[E], w[E], t0[E], t1[E], t2[E];
        fetch(0, 1);
        inv(u, v);
        fetch(2, 3);
        run_inv(u, v);
        inv(w, t0);
        fetch(4, 5);
        run_inv(w, t0);   // t0 = wx
        inv(t1, t2);
        if (A.ic >= 0) fetch(A.ic, A.ic + 1);
        run_inv(t1, t2);   // t1 = wy, t2 = wz
        // ---- pointwise terms (solvers.f90:2891-3063)
        const T sg = (T)seght[y];
        const T dxm = (T)A.delxm, dzm = (T)A.delzm, dtt = (T)A.dt, dp = (T)A.dPdx;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = lane + 32 * e;
            if (x < MX) {
                const T up = u[e], vp = v[e], wp = w[e];
                const T wxp = t0[e], wyp = t1[e], wzp = t2[e];
                T h1 = vp * wzp - wp * wyp;
                const T h2 = -up * wzp + wp * wxp;
                const T h3 = up * wyp - vp * wxp;
                if (A.flow_select == 1) h1 = h1 - dp;
                t0[e] = h1;
                t1[e] = h2;
                t2[e] = h3;
                const double cc = (double)((fabs(up) / dxm + fabs(vp) / sg + fabs(wp) / dzm) * dtt);
                cmax = (cc != cc) ? cc : fmax(cmax, cc);
                umx = fmax(umx, (double)fabs(up));
                if (A.save_uvw) {
                    const size_t g3 = ((size_t)y * mz + z) * MX + x;
                    up3[g3] = (double)up;
                    vp3[g3] = (double)vp;
                    wp3[g3] = (double)wp;
                }
            }
        }
        fwd_pair(0, true, t0, t1);   // h1, h2
        if (A.ic >= 0) {
            // -u.grad(c) [+ uniform source]: (u cx + v cy) first, then + w cz, as the reference sums
            T sacc[E];
            inv(t0, t1);
            fetch(A.ic + 2, -1);
            run_inv(t0, t1);
#pragma unroll
            for (int e = 0; e < E; ++e) sacc[e] = u[e] * t0[e] + v[e] * t1[e];
            inv(t0, t1);
            run_inv(t0, t1);
            const T sq = (T)A.scalar_q;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                T vc = -(sacc[e] + w[e] * t0[e]);
                if (A.scalar_q != 0.0) vc = vc + sq;
                t1[e] = vc;
            }
            fwd_pair(2, A.nout > 3, t2, t1);   // h3, scalar term
        } else {
            fwd_pair(2, false, t2, t1);
        }
    }
    // ---- per-plane CFL / |u| maxima
    for (int off = 16; off; off >>= 1) {
        const double c2 = __shfl_down_sync(0xffffffffu, cmax, off);
        const double u2 = __shfl_down_sync(0xffffffffu, umx, off);
        cmax = (c2 != c2) ? c2 : fmax(cmax, c2);
        umx = fmax(umx, u2);
    }
    if (lane == 0 && z < mz) {
        atomicMax((unsigned long long *)&cfl[y], (unsigned long long)__double_as_longlong(cmax));
        atomicMax((unsigned long long *)&umax[y], (unsigned long long)__double_as_longlong(umx));
    }
}

static FxArgs fx_args(const kmm_ctx *ctx, int ic, int nout, bool save_uvw) {
    FxArgs A;
    A.ic = ic;
    A.nout = nout;
    A.flow_select = ctx->p.flow_select;
    A.save_uvw = save_uvw ? 1 : 0;
    A.delxm = ctx->xl / (double)ctx->mx;
    A.delzm = ctx->zl / (double)ctx->mz;
    A.dt = ctx->dt;
    A.dPdx = ctx->dPdx;
    A.scalar_q = ctx->p.scalar_q;
    return A;
}

// specialised x stage (k_fx2) for mx = 48, 96, 144, 192; fp32: q, r and tw are float2.
// KMM_ERR_UNSUPPORTED for other mx.
int kmm_fast_x2(kmm_ctx *ctx, const void *q, void *r, const void *tw, bool fp32, int ic, int nout, bool save_uvw,
                double *up3, double *vp3, double *wp3) {
    if (nout < 3 || nout > 4 || (nout == 4) != (ic >= 0)) return KMM_ERR_UNSUPPORTED;
    const FxArgs A = fx_args(ctx, ic, nout, save_uvw);
    const int mx = ctx->mx, mz = ctx->mz;
    const size_t smem = (fp32 ? sizeof(float2) : sizeof(double2)) * 2 * (size_t)mx * FX_WARPS;
    const dim3 grid((mz + FX_WARPS - 1) / FX_WARPS, ctx->nyp);
#define FX2(MM, CC)                                                                                     \
    do {                                                                                                \
        RET(kmm_smem_attr(ctx, (const void *)k_fx2<MM, CC>, smem));                                     \
        k_fx2<MM, CC><<<grid, FX_WARPS * 32, smem, ctx->stream>>>((const CC *)q, (CC *)r, up3, vp3, wp3, \
                                                                ctx->d_seght, ctx->d_cfl, ctx->d_umax,  \
                                                                (const CC *)tw, A, ctx->nyp, mz);       \
        CKL();                                                                                          \
        return KMM_OK;                                                                                  \
    } while (0)
    if (fp32) {
        switch (mx) {
        case 48: FX2(48, float2);
        case 96: FX2(96, float2);
        case 144: FX2(144, float2);
        case 192: FX2(192, float2);
        default: return KMM_ERR_UNSUPPORTED;
        }
    }
    switch (mx) {
    case 48: FX2(48, double2);
    case 96: FX2(96, double2);
    case 144: FX2(144, double2);
    case 192: FX2(192, double2);
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef FX2
}

// ic: index in q of dc/dx (-1: no scalar terms); nout 3 (h1 h2 h3) or 4 (+ scalar term)
int kmm_fast_x(kmm_ctx *ctx, const double2 *q, double2 *r, int ic, int nout, bool save_uvw, double *up3,
               double *vp3, double *wp3) {
    if (nout < 3 || nout > 4 || (nout == 4) != (ic >= 0)) return KMM_ERR_UNSUPPORTED;
    const int st2 = kmm_fast_x2(ctx, q, r, ctx->wmx.tw, false, ic, nout, save_uvw, up3, vp3, wp3);
    if (st2 != KMM_ERR_UNSUPPORTED) return st2;
    const FxArgs A = fx_args(ctx, ic, nout, save_uvw);
    const int mx = ctx->mx, mz = ctx->mz;
    const size_t smem = sizeof(double2) * 2 * (size_t)mx * FX_WARPS;
    const dim3 grid((mz + FX_WARPS - 1) / FX_WARPS, ctx->nyp);
    const int E = (mx + 31) / 32;
#define FX_LAUNCH(EE, MM)                                                                               \
    do {                                                                                                \
        RET(kmm_smem_attr(ctx, (const void *)k_fx<EE, MM>, smem));                                      \
        k_fx<EE, MM><<<grid, FX_WARPS * 32, smem, ctx->stream>>>(q, r, up3, vp3, wp3, ctx->d_seght, ctx->d_cfl, \
                                                            ctx->d_umax, ctx->wmx, A, ctx->nyp, mz, mx,   \
                                                            ctx->nxh);                                  \
        CKL();                                                                                          \
        return KMM_OK;                                                                                  \
    } while (0)
    switch (E) {
    case 1: FX_LAUNCH(1, 0);
    case 2: FX_LAUNCH(2, 0);
    case 3: FX_LAUNCH(3, 0);
    case 5: FX_LAUNCH(5, 0);
    case 6: FX_LAUNCH(6, 0);
    case 9: FX_LAUNCH(9, 0);
    case 12: FX_LAUNCH(12, 0);
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef FX_LAUNCH
}
