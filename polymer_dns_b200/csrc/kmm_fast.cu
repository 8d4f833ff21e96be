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
#define FX_MAXF 10   // u v w wx wy wz [c cx cy cz]
#define FX_MAXO 4    // h1 h2 h3 [sc]

struct FxArgs {
    int nin, nout, scalar, flow_select, save_uvw;
    double delxm, delzm, dt, dPdx, scalar_q;
};

// MX > 0: the x length is the compile-time constant MX (specialised FFT); MX = 0: runtime plan
template <int E, int MX>
__global__ void __launch_bounds__(FX_WARPS * 32, 1) k_fx(const double2 *__restrict__ q, double2 *__restrict__ r,
                                                      double *__restrict__ up3, double *__restrict__ vp3,
                                                      double *__restrict__ wp3, const double *__restrict__ seght,
                                                      double *__restrict__ cfl, double *__restrict__ umax, DevPlan P,
                                                      FxArgs A, int nyp, int mz, int mx_rt, int nxh) {
    extern __shared__ double2 sm[];
    const int mx = MX > 0 ? MX : mx_rt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = blockIdx.y;
    const int z = blockIdx.x * FX_WARPS + warp;
    double2 *a = sm + (size_t)warp * 2 * mx, *b = a + mx;
    const bool active = z < mz;
    const int hx = mx / 2;
    double ph[FX_MAXF][E];
    double cmax = 0.0, umx = 0.0;
    if (active) {
        // ---- inverse x transforms, two fields per complex FFT
#pragma unroll
        for (int f = 0; f < FX_MAXF; f += 2) {
            if (f < A.nin) {
                const int g = f + 1;
                const bool has_g = g < A.nin;
                const double2 *qa = q + (((size_t)f * nyp + y) * mz + z) * nxh;
                const double2 *qb = q + (((size_t)g * nyp + y) * mz + z) * nxh;
                for (int k = lane; k < mx; k += 32) {
                    const int kk = k <= hx ? k : mx - k;
                    double2 Av = make_double2(0.0, 0.0), Bv = make_double2(0.0, 0.0);
                    if (kk < nxh) {
                        Av = qa[kk];
                        if (has_g) Bv = qb[kk];
                    }
                    if (k == 0 || k == hx) { Av.y = 0.0; Bv.y = 0.0; }   // c2r ignores Im of DC / Nyquist
                    a[k] = k <= hx ? make_double2(Av.x - Bv.y, Av.y + Bv.x) : make_double2(Av.x + Bv.y, -Av.y + Bv.x);
                }
                __syncwarp();
                const double2 *res;
                if constexpr (MX > 0) res = fft_warp_ct<double2, MX, +1>(a, b, P.tw);
                else res = fft_warp(P, a, b, +1);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int x = lane + 32 * e;
                    if (x < mx) {
                        const double2 v = res[x];
                        ph[f][e] = v.x;
                        if (g < FX_MAXF) ph[g][e] = v.y;
                    }
                }
                __syncwarp();
            }
        }
        // ---- pointwise terms (solvers.f90:2891-3063)
        const double sg = seght[y];
        double out[FX_MAXO][E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int x = lane + 32 * e;
            if (x < mx) {
                const double up = ph[0][e], vp = ph[1][e], wp = ph[2][e];
                const double wxp = ph[3][e], wyp = ph[4][e], wzp = ph[5][e];
                double h1 = vp * wzp - wp * wyp;
                const double h2 = -up * wzp + wp * wxp;
                const double h3 = up * wyp - vp * wxp;
                if (A.flow_select == 1) h1 = h1 - A.dPdx;
                out[0][e] = h1;
                out[1][e] = h2;
                out[2][e] = h3;
                if (A.scalar) {
                    double vc = -(up * ph[7][e] + vp * ph[8][e] + wp * ph[9][e]);
                    if (A.scalar_q != 0.0) vc = vc + A.scalar_q;
                    out[3][e] = vc;
                }
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
        // ---- forward x transforms, two outputs per complex FFT, keep kx < nxh
#pragma unroll
        for (int o = 0; o < FX_MAXO; o += 2) {
            if (o < A.nout) {
                const int g = o + 1;
                const bool has_g = g < A.nout;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int x = lane + 32 * e;
                    if (x < mx) a[x] = make_double2(out[o][e], has_g && g < FX_MAXO ? out[g][e] : 0.0);
                }
                __syncwarp();
                const double2 *res;
                if constexpr (MX > 0) res = fft_warp_ct<double2, MX, -1>(a, b, P.tw);
                else res = fft_warp(P, a, b, -1);
                double2 *ra = r + (((size_t)o * nyp + y) * mz + z) * nxh;
                double2 *rb = r + (((size_t)g * nyp + y) * mz + z) * nxh;
                for (int k = lane; k < nxh; k += 32) {
                    const double2 Z = res[k];
                    const double2 Zc = cconj(res[k == 0 ? 0 : mx - k]);
                    ra[k] = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y + Zc.y));
                    if (has_g) {
                        const double2 d = csub(Z, Zc);
                        rb[k] = make_double2(0.5 * d.y, -0.5 * d.x);
                    }
                }
                __syncwarp();
            }
        }
    }
    // ---- per-plane CFL / |u| maxima
    for (int off = 16; off; off >>= 1) {
        const double c2 = __shfl_down_sync(0xffffffffu, cmax, off);
        const double u2 = __shfl_down_sync(0xffffffffu, umx, off);
        cmax = (c2 != c2) ? c2 : fmax(cmax, c2);
        umx = fmax(umx, u2);
    }
    if (lane == 0 && active) {
        atomicMax((unsigned long long *)&cfl[y], (unsigned long long)__double_as_longlong(cmax));
        atomicMax((unsigned long long *)&umax[y], (unsigned long long)__double_as_longlong(umx));
    }
}

// returns KMM_ERR_UNSUPPORTED when mx has no compiled instance (caller falls back to the general path)
int kmm_fast_x(kmm_ctx *ctx, const double2 *q, double2 *r, int nin, int nout, bool save_uvw, double *up3,
               double *vp3, double *wp3) {
    if (nin > FX_MAXF || nout > FX_MAXO) return KMM_ERR_UNSUPPORTED;
    FxArgs A;
    A.nin = nin;
    A.nout = nout;
    A.scalar = ctx->p.scalar_on ? 1 : 0;
    A.flow_select = ctx->p.flow_select;
    A.save_uvw = save_uvw ? 1 : 0;
    A.delxm = ctx->xl / (double)ctx->mx;
    A.delzm = ctx->zl / (double)ctx->mz;
    A.dt = ctx->dt;
    A.dPdx = ctx->dPdx;
    A.scalar_q = ctx->p.scalar_q;
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
    switch (mx) {   // specialised lengths: nx = 32, 64, 96, 128
    case 48: FX_LAUNCH(2, 48);
    case 96: FX_LAUNCH(3, 96);
    case 144: FX_LAUNCH(5, 144);
    case 192: FX_LAUNCH(6, 192);
    default: break;
    }
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
