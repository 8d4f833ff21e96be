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

// the same without waiting: the cell-index status stays in d_status for the caller to read back
int kmm_tracers_enqueue(kmm_ctx *ctx) {
    if (ctx->p.npart <= 0) return KMM_OK;
    const bool init = ctx->it == ctx->p.irstrt;
    TracerArgs T = tracer_args(ctx);
    double *x = REAL(ctx, KMM_XPART), *y = REAL(ctx, KMM_YPART), *z = REAL(ctx, KMM_ZPART);
    double *u = REAL(ctx, KMM_UPART), *v = REAL(ctx, KMM_VPART), *w = REAL(ctx, KMM_WPART);
    double *f1 = REAL(ctx, KMM_UP3D), *f2 = REAL(ctx, KMM_VP3D), *f3 = REAL(ctx, KMM_WP3D);
    if (!x || !y || !z || !u || !v || !w || !f1 || !f2 || !f3) return KMM_ERR_NOMEM;
    const int nb = (T.npart + 255) / 256;
    if (init) k_init_part<<<nb, 256, 0, ctx->stream>>>(T, ctx->d_ycoord, x, y, z, u, v, w, f1, f2, f3, ctx->d_status);
    else k_tracer_update<<<nb, 256, 0, ctx->stream>>>(T, ctx->d_ycoord, x, y, z, u, v, w, f1, f2, f3, ctx->d_status);
    CKL();
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

// ---------------------------------------------------------------------------
// xyzfft(a,b,-1), helpers.f90:6-87: physical (nyp,nz,nx) -> spectral (nyp,nz,nxh)
// ---------------------------------------------------------------------------
// y: DCT-I of each real column, /ny, halve the end values (in place on a real copy)
__global__ void k_xyz_y(double *__restrict__ b, DevPlan P, int nyp, int ncols) {
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
__global__ void k_xyz_x(const double *__restrict__ b, double2 *__restrict__ a, DevPlan P, int nyp, int nz, int nx) {
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
__global__ void k_xyz_z(double2 *__restrict__ a, DevPlan P, int nyp, int nz) {
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
