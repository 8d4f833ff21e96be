// kmm_tracer.cu -- tracer integrator (part_track.f90), xyzfft (helpers.f90:6-87) and the
// 3/2-grid layout conversion between the reference's (nyp,mz,mx) arrays and the internal
// [y][z][x] layout.
#include <math.h>

#include "kmm_internal.cuh"

// ---------------------------------------------------------------------------
// layout conversion: Fortran (nyp,mz,mx) <-> internal [y][z][x]
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_f2p(const T *__restrict__ src, T *__restrict__ dst, int nyp, int mz, int mx) {
    const size_t n = (size_t)nyp * mz * mx;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        // e enumerates the Fortran array: e = i + nyp*(j + mz*k)
        const int i = (int)(e % nyp);
        const size_t jk = e / nyp;
        const int j = (int)(jk % mz), k = (int)(jk / mz);
        dst[((size_t)i * mz + j) * mx + k] = src[e];
    }
}

template <typename T>
__global__ void k_p2f(const T *__restrict__ src, T *__restrict__ dst, int nyp, int mz, int mx) {
    const size_t n = (size_t)nyp * mz * mx;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % nyp);
        const size_t jk = e / nyp;
        const int j = (int)(jk % mz), k = (int)(jk / mz);
        dst[e] = src[((size_t)i * mz + j) * mx + k];
    }
}

int kmm_phys_layout(kmm_ctx *ctx, int field, void *dev, const void *host_src, void *host_dst) {
    const size_t n = ctx->nphys;
    const size_t eb = field == KMM_IMATRIX ? 4 : 8;
    void *tmp = NULL;
    CK(cudaMallocAsync(&tmp, n * eb, ctx->stream));
    if (host_src) {
        CK(cudaMemcpyAsync(tmp, host_src, n * eb, cudaMemcpyHostToDevice, ctx->stream));
        if (eb == 4) k_f2p<int><<<kmm_blocks(n, 256), 256, 0, ctx->stream>>>((const int *)tmp, (int *)dev, ctx->nyp, ctx->mz, ctx->mx);
        else k_f2p<double><<<kmm_blocks(n, 256), 256, 0, ctx->stream>>>((const double *)tmp, (double *)dev, ctx->nyp, ctx->mz, ctx->mx);
        CKL();
    } else {
        if (eb == 4) k_p2f<int><<<kmm_blocks(n, 256), 256, 0, ctx->stream>>>((const int *)dev, (int *)tmp, ctx->nyp, ctx->mz, ctx->mx);
        else k_p2f<double><<<kmm_blocks(n, 256), 256, 0, ctx->stream>>>((const double *)dev, (double *)tmp, ctx->nyp, ctx->mz, ctx->mx);
        CKL();
        CK(cudaMemcpyAsync(host_dst, tmp, n * eb, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaFreeAsync(tmp, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// fluid_interp / interpolate3, part_track.f90:518-613, 1184-1221 (internal [y][z][x] layout)
// ---------------------------------------------------------------------------
struct TracerArgs {
    int nyp, ny, mz, mx, npart, scheme;
    double xl, yl, zl, delxm, delzm, pi, dt, height, ybot;
};

__device__ __forceinline__ double interpolate3(double x, double y, double z, double x0, double x1, double y0, double y1,
                                               double z0, double z1, double c000, double c100, double c001,
                                               double c101, double c010, double c110, double c011, double c111) {
    const double xd = (x1 > x0) ? (x - x0) / (x1 - x0) : 0.0;
    const double yd = (y1 > y0) ? (y - y0) / (y1 - y0) : 0.0;
    const double zd = (z1 > z0) ? (z - z0) / (z1 - z0) : 0.0;
    const double c00 = c000 * (1.0 - xd) + c100 * xd;
    const double c01 = c001 * (1.0 - xd) + c101 * xd;
    const double c10 = c010 * (1.0 - xd) + c110 * xd;
    const double c11 = c011 * (1.0 - xd) + c111 * xd;
    const double c0 = c00 * (1.0 - yd) + c10 * yd;
    const double c1 = c01 * (1.0 - yd) + c11 * yd;
    return c0 * (1.0 - zd) + c1 * zd;
}

__device__ __forceinline__ int fluid_interp(const TracerArgs &T, const double *__restrict__ ycoord, double xp, double yp,
                                            double zp, const double *__restrict__ u, const double *__restrict__ v,
                                            const double *__restrict__ w, double *uf, double *vf, double *wf) {
    const int mx = T.mx, mz = T.mz;
    const int imin = ((int)floor(xp / T.delxm) + mx) % mx + 1;
    const int imax = imin % mx + 1;
    const int jmin = ((int)floor(zp / T.delzm) + mz) % mz + 1;
    const int jmax = jmin % mz + 1;
    const int kmax = (int)floor(1.0 + (double)T.ny / T.pi * acos(2.0 * yp / T.yl));
    const int kmin = kmax + 1;
    if (imin < 1 || jmin < 1 || kmin < 1 || kmin > T.nyp || kmax < 1) return 1;
    const double xmin = (double)(imin - 1) * T.delxm, xmax = (double)(imax - 1) * T.delxm;
    const double ymin = ycoord[kmin - 1], ymax = ycoord[kmax - 1];
    const double zmin = (double)(jmin - 1) * T.delzm, zmax = (double)(jmax - 1) * T.delzm;
#define G(f, ky, jz, ix) __ldg(&(f)[((size_t)((ky) - 1) * mz + ((jz) - 1)) * mx + ((ix) - 1)])
#define INTERP(f) interpolate3(xp, yp, zp, xmin, xmax, ymin, ymax, zmin, zmax, G(f, kmin, jmin, imin), \
        G(f, kmin, jmin, imax), G(f, kmin, jmax, imin), G(f, kmin, jmax, imax), G(f, kmax, jmin, imin), \
        G(f, kmax, jmin, imax), G(f, kmax, jmax, imin), G(f, kmax, jmax, imax))
    *uf = INTERP(u);
    *vf = INTERP(v);
    *wf = INTERP(w);
#undef INTERP
#undef G
    return 0;
}

__global__ void k_init_part(TracerArgs T, const double *__restrict__ ycoord, const double *__restrict__ xpa,
                            const double *__restrict__ ypa, const double *__restrict__ zpa, double *upa, double *vpa,
                            double *wpa, const double *__restrict__ u, const double *__restrict__ v,
                            const double *__restrict__ w, int *status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= T.npart) return;
    double uf, vf, wf;
    if (fluid_interp(T, ycoord, xpa[j], ypa[j], zpa[j], u, v, w, &uf, &vf, &wf)) {
        atomicMax(status, KMM_ERR_INTERP);
        return;
    }
    upa[j] = uf; vpa[j] = vf; wpa[j] = wf;
}

// tracer_update, part_track.f90:360-433 (+ the RK3 variant)
__global__ void k_tracer_update(TracerArgs T, const double *__restrict__ ycoord, double *xpa, double *ypa, double *zpa,
                                double *upa, double *vpa, double *wpa, const double *__restrict__ u,
                                const double *__restrict__ v, const double *__restrict__ w, int *status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= T.npart) return;
    double xp = xpa[j], yp = ypa[j], zp = zpa[j], up = upa[j], vp = vpa[j], wp = wpa[j];
    const double dt = T.dt;
    int bad = 0;
    if (T.scheme == 1) {
        const double ak[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
        const double bk[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
        double qx = 0.0, qy = 0.0, qz = 0.0, uu, vv, ww;
        for (int s = 0; s < 3; ++s) {
            bad |= fluid_interp(T, ycoord, xp, yp, zp, u, v, w, &uu, &vv, &ww);
            qx = ak[s] * qx + dt * uu;
            qy = ak[s] * qy + dt * vv;
            qz = ak[s] * qz + dt * ww;
            xp = fmod(T.xl + xp + bk[s] * qx, T.xl);
            yp = fmax(fmin(yp + bk[s] * qy, T.height), T.ybot);
            zp = fmod(T.zl + zp + bk[s] * qz, T.zl);
        }
    } else {
        xp = fmod(T.xl + xp + up * dt, T.xl);
        yp = fmax(fmin(yp + vp * dt, T.height), T.ybot);
        zp = fmod(T.zl + zp + wp * dt, T.zl);
    }
    bad |= fluid_interp(T, ycoord, xp, yp, zp, u, v, w, &up, &vp, &wp);
    if (bad) atomicMax(status, KMM_ERR_INTERP);
    xpa[j] = xp; ypa[j] = yp; zpa[j] = zp; upa[j] = up; vpa[j] = vp; wpa[j] = wp;
}

static TracerArgs tracer_args(const kmm_ctx *ctx) {
    TracerArgs T;
    T.nyp = ctx->nyp; T.ny = ctx->ny; T.mz = ctx->mz; T.mx = ctx->mx; T.npart = ctx->p.npart;
    T.scheme = ctx->p.tracer_scheme;
    T.xl = ctx->xl; T.yl = ctx->yl; T.zl = ctx->zl;
    T.delxm = ctx->xl / (double)ctx->mx;
    T.delzm = ctx->zl / (double)ctx->mz;
    T.pi = ctx->pi;
    T.dt = ctx->dt / (double)ctx->substep;
    T.height = ctx->h_ycoord[0] - ctx->p.ap;
    T.ybot = ctx->p.ap + ctx->h_ycoord[ctx->nyp - 1];
    return T;
}

static int tracer_launch(kmm_ctx *ctx, bool init) {
    if (ctx->p.npart <= 0) return KMM_OK;
    TracerArgs T = tracer_args(ctx);
    double *x = REAL(ctx, KMM_XPART), *y = REAL(ctx, KMM_YPART), *z = REAL(ctx, KMM_ZPART);
    double *u = REAL(ctx, KMM_UPART), *v = REAL(ctx, KMM_VPART), *w = REAL(ctx, KMM_WPART);
    double *f1 = REAL(ctx, KMM_UP3D), *f2 = REAL(ctx, KMM_VP3D), *f3 = REAL(ctx, KMM_WP3D);
    if (!x || !y || !z || !u || !v || !w || !f1 || !f2 || !f3) return KMM_ERR_NOMEM;
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    const int nb = (T.npart + 255) / 256;
    if (init) k_init_part<<<nb, 256, 0, ctx->stream>>>(T, ctx->d_ycoord, x, y, z, u, v, w, f1, f2, f3, ctx->d_status);
    else k_tracer_update<<<nb, 256, 0, ctx->stream>>>(T, ctx->d_ycoord, x, y, z, u, v, w, f1, f2, f3, ctx->d_status);
    CKL();
    int h = 0;
    CK(cudaMemcpyAsync(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h) kmm_set_error(ctx, "particle interpolation cell index out of range (part_track.f90:580-590)");
    return h ? KMM_ERR_INTERP : KMM_OK;
}

// called from vcw3dp: init at it == irstrt (part_track.f90:132-134), Euler/RK3 update otherwise
int kmm_tracers(kmm_ctx *ctx) { return tracer_launch(ctx, ctx->it == ctx->p.irstrt); }

// the same without waiting, on stream `st`: the cell-index status stays in d_status for the
// caller to read back
int kmm_tracers_enqueue(kmm_ctx *ctx, cudaStream_t st) {
    if (ctx->p.npart <= 0) return KMM_OK;
    const bool init = ctx->it == ctx->p.irstrt;
    TracerArgs T = tracer_args(ctx);
    double *x = REAL(ctx, KMM_XPART), *y = REAL(ctx, KMM_YPART), *z = REAL(ctx, KMM_ZPART);
    double *u = REAL(ctx, KMM_UPART), *v = REAL(ctx, KMM_VPART), *w = REAL(ctx, KMM_WPART);
    double *f1 = REAL(ctx, KMM_UP3D), *f2 = REAL(ctx, KMM_VP3D), *f3 = REAL(ctx, KMM_WP3D);
    if (!x || !y || !z || !u || !v || !w || !f1 || !f2 || !f3) return KMM_ERR_NOMEM;
    const int nb = (T.npart + 255) / 256;
    if (init) k_init_part<<<nb, 256, 0, st>>>(T, ctx->d_ycoord, x, y, z, u, v, w, f1, f2, f3, ctx->d_status);
    else k_tracer_update<<<nb, 256, 0, st>>>(T, ctx->d_ycoord, x, y, z, u, v, w, f1, f2, f3, ctx->d_status);
    CKL();
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// inertial particles (particle_flag > 0): Maxey-Riley equations with RK4, part_track.f90:617-1075
// One thread per particle; its `substep` RK4 substeps of dt/substep run back to back.
// ---------------------------------------------------------------------------
struct MRFields {
    const double *u, *v, *w, *uo, *vo, *wo, *wx, *wy, *wz, *g[9], *L[3], *Lo[3];
};
struct MRArgs {
    double ratio, ap, re, c_mu, gravity;
    int cd_switch, nsub;
};

// SubDerivative, part_track.f90:896-1075: corner time derivatives ((f - f_old)/dt with the
// substep dt) interpolated to the particle, and the material derivative of the fluid velocity
__device__ void mr_subderivative(const TracerArgs &T, const MRFields &F, const double *__restrict__ ycoord, double uf,
                                 double vf, double wf, double xp0, double yp0, double zp0, double *sD, double *dL) {
    const int mx = T.mx, mz = T.mz;
    const int imin = ((int)floor(xp0 / T.delxm) + mx) % mx + 1, imax = imin % mx + 1;
    const int jmin = ((int)floor(zp0 / T.delzm) + mz) % mz + 1, jmax = jmin % mz + 1;
    const int kmax = (int)floor(1.0 + (double)T.ny / T.pi * acos(2.0 * yp0 / T.yl)), kmin = kmax + 1;
    const double xmin = (double)(imin - 1) * T.delxm, xmax = (double)(imax - 1) * T.delxm;
    const double ymin = ycoord[kmin - 1], ymax = ycoord[kmax - 1];
    const double zmin = (double)(jmin - 1) * T.delzm, zmax = (double)(jmax - 1) * T.delzm;
    // corner n: (gk, gj, gi) = ({kmin x4, kmax x4}, {jmin, jmin, jmax, jmax} x2, {imin, imax} x4)
    size_t gx[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const int k = n < 4 ? kmin : kmax, j = (n & 2) ? jmax : jmin, i = (n & 1) ? imax : imin;
        gx[n] = ((size_t)(k - 1) * mz + (j - 1)) * mx + (i - 1);
    }
#define I3(a) interpolate3(xp0, yp0, zp0, xmin, xmax, ymin, ymax, zmin, zmax, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7])
    double gr[9];
#pragma unroll 1
    for (int m = 0; m < 9; ++m) {
        double c[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) c[n] = __ldg(&F.g[m][gx[n]]);
        gr[m] = I3(c);
    }
    const double *cur[6] = {F.u, F.v, F.w, F.L[0], F.L[1], F.L[2]};
    const double *old[6] = {F.uo, F.vo, F.wo, F.Lo[0], F.Lo[1], F.Lo[2]};
    double tdv[6];
#pragma unroll 1
    for (int m = 0; m < 6; ++m) {
        double c[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) c[n] = (__ldg(&cur[m][gx[n]]) - __ldg(&old[m][gx[n]])) / T.dt;
        tdv[m] = I3(c);
    }
#undef I3
    sD[0] = tdv[0] + uf * gr[0] + vf * gr[1] + wf * gr[2];
    sD[1] = tdv[1] + uf * gr[3] + vf * gr[4] + wf * gr[5];
    sD[2] = tdv[2] + uf * gr[6] + vf * gr[7] + wf * gr[8];
    dL[0] = tdv[3];
    dL[1] = tdv[4];
    dL[2] = tdv[5];
}

// RKstage, part_track.f90:759-892: forces at the stage point, then the stage update from the
// substep's start (h = dt at stage 3, dt/2 otherwise); returns nonzero on a bad cell index
__device__ int mr_stage(const TracerArgs &T, const MRArgs &M, const MRFields &F, const double *__restrict__ ycoord,
                        int sn, double *un, double *xp, double *K, const double *x0, const double *u0) {
    const double ap = M.ap, re = M.re;
    const double Pi_f = 1.0 / (M.ratio + 0.5), Pi_p = M.ratio / (M.ratio + 0.5), C_L = 0.5;
    double uf, vf, wf, wxf, wyf, wzf, Luf, Lvf, Lwf;
    int bad = fluid_interp(T, ycoord, xp[0], xp[1], xp[2], F.u, F.v, F.w, &uf, &vf, &wf);
    bad |= fluid_interp(T, ycoord, xp[0], xp[1], xp[2], F.wx, F.wy, F.wz, &wxf, &wyf, &wzf);
    bad |= fluid_interp(T, ycoord, xp[0], xp[1], xp[2], F.L[0], F.L[1], F.L[2], &Luf, &Lvf, &Lwf);
    if (bad) return 1;
    double sD[3], dL[3];
    mr_subderivative(T, F, ycoord, uf, vf, wf, xp[0], xp[1], xp[2], sD, dL);
    const double Re_p = 2 * ap * re * sqrt((uf - un[0]) * (uf - un[0]) + (vf - un[1]) * (vf - un[1]) +
                                           (wf - un[2]) * (wf - un[2]));
    double C_D = 0.0;
    if (M.cd_switch == 1) C_D = 16 / (2 * ap * re) * M.c_mu;
    else if (M.cd_switch == 2) C_D = 24 / (2 * ap * re) * (1 + 0.15 * pow(Re_p, 0.687));
    else if (M.cd_switch == 3) C_D = Re_p > 1.0 ? 16.31 * pow(Re_p, -0.8331) : 17.28 * pow(Re_p, -0.9711);
    const double a6 = ap * ap / 6.0;
    const double ru = uf - un[0] + a6 * Luf, rv = vf - un[1] + a6 * Lvf, rw = wf - un[2] + a6 * Lwf;
    const double cd = C_D * 3 / (8 * ap), fx = 3.0 / 20.0 * (ap * ap);
    K[0] = Pi_f * (1.5 * sD[0] + cd * ru + C_L * (rv * wzf - rw * wyf) + fx * dL[0]);
    K[1] = Pi_f * (1.5 * sD[1] + cd * rv + C_L * (rw * wxf - ru * wzf) + fx * dL[1]) - M.gravity * (Pi_f - Pi_p);
    K[2] = Pi_f * (1.5 * sD[2] + cd * rw + C_L * (ru * wyf - rv * wxf) + fx * dL[2]);
    const double h = sn == 3 ? T.dt : T.dt / 2.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) un[c] = u0[c] + h * K[c];
    xp[0] = fmod(T.xl + x0[0] + h * un[0], T.xl);
    xp[1] = fmax(fmin(x0[1] + h * un[1], T.height), T.ybot);
    xp[2] = fmod(T.zl + x0[2] + h * un[2], T.zl);
    return 0;
}

__global__ void __launch_bounds__(128) k_inertial(TracerArgs T, MRArgs M, MRFields F, const double *__restrict__ ycoord,
                                                  double *xpa, double *ypa, double *zpa, double *upa, double *vpa,
                                                  double *wpa, double *pumax, int *status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= T.npart) return;
    double x0[3] = {xpa[j], ypa[j], zpa[j]}, u0[3] = {upa[j], vpa[j], wpa[j]};
    double um1 = 0.0;
    int bad = 0;
    for (int s = 0; s < M.nsub && !bad; ++s) {
        // RK4, part_track.f90:617-755
        double xp[3] = {x0[0], x0[1], x0[2]}, un[3] = {u0[0], u0[1], u0[2]};
        double K[4][3], us[3][3];
        for (int sn = 1; sn <= 4 && !bad; ++sn) {
            bad |= mr_stage(T, M, F, ycoord, sn, un, xp, K[sn - 1], x0, u0);
            if (sn < 4)
                for (int c = 0; c < 3; ++c) us[sn - 1][c] = un[c];
        }
        if (bad) break;
        const double dt = T.dt;
        x0[0] = fmod(T.xl + x0[0] + dt * (u0[0] / 6 + us[0][0] / 3 + us[1][0] / 3 + us[2][0] / 6), T.xl);
        x0[1] = fmax(fmin(x0[1] + dt * (u0[1] / 6 + us[0][1] / 3 + us[1][1] / 3 + us[2][1] / 6), T.height), T.ybot);
        x0[2] = fmod(T.zl + x0[2] + dt * (u0[2] / 6 + us[0][2] / 3 + us[1][2] / 3 + us[2][2] / 6), T.zl);
        u0[0] = u0[0] + dt * (K[0][0] / 6 + K[1][0] / 3 + K[2][0] / 3 + K[3][0] / 6);
        const double vp_new = u0[1] + dt * (K[0][1] / 6 + K[1][1] / 3 + K[2][1] / 3 + K[3][1] / 6);
        u0[2] = u0[2] + dt * (K[0][2] / 6 + K[1][2] / 3 + K[2][2] / 3 + K[3][2] / 6);
        // elastic bounce off a wall the particle was clamped to
        u0[1] = ((x0[1] == T.height && vp_new > 0.0) || (x0[1] == T.ybot && vp_new < 0.0)) ? -vp_new : vp_new;
        double uf, vf, wf;
        bad |= fluid_interp(T, ycoord, x0[0], x0[1], x0[2], F.u, F.v, F.w, &uf, &vf, &wf);
        if (bad) break;
        um1 = fmax(um1, sqrt((uf - u0[0]) * (uf - u0[0]) + (vf - u0[1]) * (vf - u0[1]) + (wf - u0[2]) * (wf - u0[2])));
    }
    if (bad) atomicMax(status, KMM_ERR_INTERP);
    // running max of non-negative doubles through their bit patterns (NaN compares larger)
    atomicMax((unsigned long long *)pumax, (unsigned long long)__double_as_longlong(um1));
    xpa[j] = x0[0]; ypa[j] = x0[1]; zpa[j] = x0[2];
    upa[j] = u0[0]; vpa[j] = u0[1]; wpa[j] = u0[2];
}

// the particle_flag > 0 branch of part_track (part_track.f90:125-176, 213-222) and the copies of
// the velocity and Laplacian kept for the next step's time derivatives (solvers.f90:3469-3476)
int kmm_inertial(kmm_ctx *ctx) {
    if (ctx->p.npart <= 0) return KMM_OK;
    const bool init = ctx->it == ctx->p.irstrt;
    TracerArgs T = tracer_args(ctx);
    double *x = REAL(ctx, KMM_XPART), *y = REAL(ctx, KMM_YPART), *z = REAL(ctx, KMM_ZPART);
    double *u = REAL(ctx, KMM_UPART), *v = REAL(ctx, KMM_VPART), *w = REAL(ctx, KMM_WPART);
    MRFields F;
    F.u = REAL(ctx, KMM_UP3D); F.v = REAL(ctx, KMM_VP3D); F.w = REAL(ctx, KMM_WP3D);
    F.uo = REAL(ctx, KMM_UOLD); F.vo = REAL(ctx, KMM_VOLD); F.wo = REAL(ctx, KMM_WOLD);
    F.wx = REAL(ctx, KMM_WX3D); F.wy = REAL(ctx, KMM_WY3D); F.wz = REAL(ctx, KMM_WZ3D);
    for (int m = 0; m < 9; ++m) F.g[m] = REAL(ctx, KMM_U11P3D + m);
    for (int m = 0; m < 3; ++m) { F.L[m] = REAL(ctx, KMM_LUP3D + m); F.Lo[m] = REAL(ctx, KMM_LUNM1 + m); }
    if (!x || !y || !z || !u || !v || !w || !F.u || !F.v || !F.w || !F.uo || !F.vo || !F.wo || !F.wx || !F.wy || !F.wz)
        return KMM_ERR_NOMEM;
    for (int m = 0; m < 9; ++m) if (!F.g[m]) return KMM_ERR_NOMEM;
    for (int m = 0; m < 3; ++m) if (!F.L[m] || !F.Lo[m]) return KMM_ERR_NOMEM;
    MRArgs M;
    M.ratio = ctx->p.ratio; M.ap = ctx->p.ap; M.re = ctx->re; M.c_mu = ctx->p.c_mu; M.gravity = ctx->p.gravity;
    M.cd_switch = ctx->p.cd_switch; M.nsub = ctx->substep;
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    if (init) {
        k_init_part<<<(T.npart + 255) / 256, 256, 0, ctx->stream>>>(T, ctx->d_ycoord, x, y, z, u, v, w, F.u, F.v, F.w,
                                                                     ctx->d_status);
    } else {
        k_inertial<<<(T.npart + 127) / 128, 128, 0, ctx->stream>>>(T, M, F, ctx->d_ycoord, x, y, z, u, v, w,
                                                                   ctx->d_pumax, ctx->d_status);
    }
    CKL();
    static const int cur[6] = {KMM_UP3D, KMM_VP3D, KMM_WP3D, KMM_LUP3D, KMM_LVP3D, KMM_LWP3D};
    for (int m = 0; m < 6; ++m)
        CK(cudaMemcpyAsync(REAL(ctx, KMM_UOLD + m), REAL(ctx, cur[m]), sizeof(double) * ctx->nphys,
                           cudaMemcpyDeviceToDevice, ctx->stream));
    int h = 0;
    double um1 = 0.0;
    CK(cudaMemcpyAsync(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&um1, ctx->d_pumax, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->stats.pumax = um1;
    ctx->stats.pcfl = um1 * ctx->dt / ctx->p.ap;   // with the full dt (part_track.f90:215)
    if (h) {
        kmm_set_error(ctx, "particle interpolation cell index out of range (part_track.f90:580-590)");
        return KMM_ERR_INTERP;
    }
    if (ctx->stats.pcfl >= 10.0) {
        kmm_set_error(ctx, "particle CFL %.3g >= 10 (part_track.f90:217-221)", ctx->stats.pcfl);
        return KMM_ERR_PCFL;
    }
    return KMM_OK;
}

// swirl at each particle (fluid_interp1 on swirl_3d, solvers.f90:3480)
__global__ void k_swirl_part(TracerArgs T, const double *__restrict__ ycoord, const double *__restrict__ xp,
                             const double *__restrict__ yp, const double *__restrict__ zp,
                             const double *__restrict__ sw, double *__restrict__ sp, int *status) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= T.npart) return;
    double a, b, c;
    if (fluid_interp(T, ycoord, xp[n], yp[n], zp[n], sw, sw, sw, &a, &b, &c)) {
        atomicOr(status, 1);
        return;
    }
    sp[n] = a;
}

int kmm_swirl_particles(kmm_ctx *ctx) {
    if (ctx->p.npart <= 0) return KMM_OK;
    TracerArgs T = tracer_args(ctx);
    double *x = REAL(ctx, KMM_XPART), *y = REAL(ctx, KMM_YPART), *z = REAL(ctx, KMM_ZPART);
    double *sw = REAL(ctx, KMM_SWIRL3D), *sp = REAL(ctx, KMM_SWIRLPART);
    if (!x || !y || !z || !sw || !sp) return KMM_ERR_NOMEM;
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    k_swirl_part<<<(T.npart + 255) / 256, 256, 0, ctx->stream>>>(T, ctx->d_ycoord, x, y, z, sw, sp, ctx->d_status);
    CKL();
    int h = 0;
    CK(cudaMemcpyAsync(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h) kmm_set_error(ctx, "particle interpolation cell index out of range (part_track.f90:580-590)");
    return h ? KMM_ERR_INTERP : KMM_OK;
}

extern "C" int kmm_tracer_update(kmm_ctx *ctx) { return ctx ? tracer_launch(ctx, false) : KMM_ERR_ARG; }
extern "C" int kmm_init_part(kmm_ctx *ctx) { return ctx ? tracer_launch(ctx, true) : KMM_ERR_ARG; }

// the interpolation cell of each particle, the lookup of fluid_interp (part_track.f90:560-577)
// with the same expressions as fluid_interp above; out-of-range entries are 0 and raise *bad
__global__ void k_tracer_cells(TracerArgs T, const double *__restrict__ xpa, const double *__restrict__ ypa,
                               const double *__restrict__ zpa, int *__restrict__ cells, int *bad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= T.npart) return;
    const double xp = xpa[p], yp = ypa[p], zp = zpa[p];
    const int imin = ((int)floor(xp / T.delxm) + T.mx) % T.mx + 1;
    const int jmin = ((int)floor(zp / T.delzm) + T.mz) % T.mz + 1;
    const int kmax = (int)floor(1.0 + (double)T.ny / T.pi * acos(2.0 * yp / T.yl));
    const int kmin = kmax + 1;
    const bool ok = !(imin < 1 || jmin < 1 || kmin < 1 || kmin > T.nyp || kmax < 1);
    cells[p] = ok ? imin : 0;
    cells[T.npart + p] = ok ? jmin : 0;
    cells[2 * T.npart + p] = ok ? kmax : 0;
    if (!ok) atomicExch(bad, 1);
}

extern "C" int kmm_tracer_cells(kmm_ctx *ctx, int *cells, size_t n) {
    if (!ctx || !cells) return KMM_ERR_ARG;
    const int np = ctx->p.npart;
    if (np <= 0) return KMM_OK;
    if (n < 3 * (size_t)np) {
        kmm_set_error(ctx, "kmm_tracer_cells: %zu ints given, 3 npart = %zu needed", n, 3 * (size_t)np);
        return KMM_ERR_ARG;
    }
    const double *xp = REAL(ctx, KMM_XPART), *yp = REAL(ctx, KMM_YPART), *zp = REAL(ctx, KMM_ZPART);
    if (!xp || !yp || !zp) return KMM_ERR_NOMEM;
    int *d = NULL;
    CK(cudaMallocAsync(&d, sizeof(int) * (3 * (size_t)np + 1), ctx->stream));
    CK(cudaMemsetAsync(d + 3 * (size_t)np, 0, sizeof(int), ctx->stream));
    k_tracer_cells<<<(np + 255) / 256, 256, 0, ctx->stream>>>(tracer_args(ctx), xp, yp, zp, d, d + 3 * (size_t)np);
    CKL();
    int bad = 0;
    CK(cudaMemcpyAsync(cells, d, sizeof(int) * 3 * (size_t)np, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&bad, d + 3 * (size_t)np, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaFreeAsync(d, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (bad) {
        kmm_set_error(ctx, "particle interpolation cell index out of range (part_track.f90:580-590)");
        return KMM_ERR_INTERP;
    }
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// xyzfft(a,b,-1), helpers.f90:6-87: physical (nyp,nz,nx) -> spectral (nyp,nz,nxh)
// ---------------------------------------------------------------------------
// y: DCT-I of each real column, /ny, halve the end values (in place on a real copy)
__global__ void k_xyz_y(double *__restrict__ b, const __grid_constant__ DevPlan P, int nyp, int ncols) {
    extern __shared__ double2 sm[];
    const int ny = nyp - 1, L = 2 * ny;
    const int col = blockIdx.x;
    if (col >= ncols) return;
    double2 *a = sm, *c = sm + L;
    double *src = b + (size_t)col * nyp;
    for (int i = threadIdx.x; i < nyp; i += blockDim.x) {
        const double v = src[i];
        a[i] = make_double2(v, 0.0);
        if (i > 0 && i < ny) a[L - i] = make_double2(v, 0.0);
    }
    __syncthreads();
    double2 *r = fft_smem(P, a, c, 1, L, -1);
    for (int i = threadIdx.x; i < nyp; i += blockDim.x) {
        double v = r[i].x / (double)ny;
        if (i == 0 || i == ny) v = v / 2.0;
        src[i] = v;
    }
}

// x: r2c over nx for each (i,j) line (stride nz*nyp), /nx, keep k < nxh -> complex work (nyp,nz,nxh)
__global__ void k_xyz_x(const double *__restrict__ b, double2 *__restrict__ a, const __grid_constant__ DevPlan P, int nyp, int nz, int nx) {
    extern __shared__ double2 sm[];
    const int line = blockIdx.x;   // i + nyp*j
    const int i = line % nyp, j = line / nyp;
    double2 *s = sm, *t = sm + nx;
    for (int k = threadIdx.x; k < nx; k += blockDim.x) s[k] = make_double2(b[((size_t)k * nz + j) * nyp + i], 0.0);
    __syncthreads();
    double2 *r = fft_smem(P, s, t, 1, nx, -1);
    const int nxh = nx / 2;
    for (int k = threadIdx.x; k < nxh; k += blockDim.x) {
        double2 v = r[k];
        a[((size_t)k * nz + j) * nyp + i] = make_double2(v.x / (double)nx, v.y / (double)nx);
    }
}

// z: forward c2c over nz for each (i,k) line, /nz
__global__ void k_xyz_z(double2 *__restrict__ a, const __grid_constant__ DevPlan P, int nyp, int nz) {
    extern __shared__ double2 sm[];
    const int line = blockIdx.x;   // i + nyp*k
    const int i = line % nyp, k = line / nyp;
    double2 *s = sm, *t = sm + nz;
    for (int j = threadIdx.x; j < nz; j += blockDim.x) s[j] = a[((size_t)k * nz + j) * nyp + i];
    __syncthreads();
    double2 *r = fft_smem(P, s, t, 1, nz, -1);
    for (int j = threadIdx.x; j < nz; j += blockDim.x) {
        double2 v = r[j];
        a[((size_t)k * nz + j) * nyp + i] = make_double2(v.x / (double)nz, v.y / (double)nz);
    }
}

extern "C" int kmm_xyzfft(kmm_ctx *ctx, int dst, int src) {
    if (!ctx || dst < 0 || dst >= KMM_NSPECTRAL || src < KMM_INITU || src >= KMM_NINIT_END) return KMM_ERR_ARG;
    double *b0 = REAL(ctx, src);
    double2 *a = SPEC(ctx, dst);
    if (!b0 || !a) return KMM_ERR_NOMEM;
    const size_t np = (size_t)ctx->nyp * ctx->nz * ctx->nx;
    double *b = NULL;
    CK(cudaMallocAsync((void **)&b, sizeof(double) * np, ctx->stream));
    CK(cudaMemcpyAsync(b, b0, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    k_xyz_y<<<ctx->nz * ctx->nx, 128, sizeof(double2) * 4 * ctx->ny, ctx->stream>>>(b, ctx->py2, ctx->nyp, ctx->nz * ctx->nx);
    CKL();
    k_xyz_x<<<ctx->nyp * ctx->nz, 128, sizeof(double2) * 2 * ctx->nx, ctx->stream>>>(b, a, ctx->pnx, ctx->nyp, ctx->nz, ctx->nx);
    CKL();
    k_xyz_z<<<ctx->nyp * ctx->nxh, 128, sizeof(double2) * 2 * ctx->nz, ctx->stream>>>(a, ctx->pnz, ctx->nyp, ctx->nz);
    CKL();
    CK(cudaFreeAsync(b, ctx->stream));
    return KMM_OK;
}
