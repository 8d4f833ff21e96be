// kmm_noalloc.cu -- kmm_xyzfft_noalloc: the physical -> spectral transform of initial fields
// (the same kernels as kmm_xyzfft) for callers that cannot allocate device memory.
//
// Who needs it: a host whose device memory is owned by another allocator (a framework's memory
// pool, a fixed per-process budget) or a time-critical loop that cannot afford cudaMalloc's
// implicit device synchronisation, and that has no kmm context (creating one allocates).  The
// caller passes the input and output device arrays; the only scratch the transform needs (a
// working copy of the physical field, plus the FFT twiddle tables) lives in file-scope device
// arrays of fixed size that every GPU loading this library holds until the process exits.
#include <math.h>
#include <stdlib.h>

#include "kmm_internal.cuh"

__global__ void k_xyz_y(double *__restrict__ b, DevPlan P, int nyp, int ncols);
__global__ void k_xyz_x(const double *__restrict__ b, double2 *__restrict__ a, DevPlan P, int nyp, int nz, int nx);
__global__ void k_xyz_z(double2 *__restrict__ a, DevPlan P, int nyp, int nz);

#define NOALLOC_TW_MAX 4096   // longest transform: 2 ny, nx and nz each at most this

// working copy of the physical field: KMM_XYZFFT_NOALLOC_MAX doubles (32 MiB)
static __device__ __align__(256) double g_noalloc_scratch[KMM_XYZFFT_NOALLOC_MAX];
// twiddles of the three transforms (2 ny, nx, nz)
static __device__ __align__(256) double2 g_noalloc_tw[3 * NOALLOC_TW_MAX];

#define NOALLOC_MAX_DEVICES 64
static double *s_scratch[NOALLOC_MAX_DEVICES];
static double2 *s_tw[NOALLOC_MAX_DEVICES];
static double2 s_tw_host[NOALLOC_MAX_DEVICES][3 * NOALLOC_TW_MAX];   // staging kept alive for async copies
static int s_tw_len[NOALLOC_MAX_DEVICES][3];

static bool noalloc_plan(int n, DevPlan *p) {
    int m = n, nf = 0;
    static const int rads[4] = {4, 2, 3, 5};
    for (int r = 0; r < 4; ++r)
        while (m % rads[r] == 0 && nf < KMM_MAX_FFT_FACTORS) {
            p->fac[nf++] = rads[r];
            m /= rads[r];
        }
    p->n = n;
    p->nf = nf;
    return m == 1 && n <= NOALLOC_TW_MAX;
}

extern "C" int kmm_xyzfft_noalloc(const double *phys, double *spec, int nx, int ny, int nz, void *stream) {
    if (!phys || !spec) return KMM_ERR_ARG;
    if (nx < 4 || ny < 8 || nz < 4 || nx % 2 || ny % 2) return KMM_ERR_ARG;
    const size_t nyp = (size_t)ny + 1;
    if (nyp * (size_t)nz * (size_t)nx > (size_t)KMM_XYZFFT_NOALLOC_MAX) return KMM_ERR_ARG;   // beyond the scratch
    DevPlan py2, pnx, pnz;
    if (!noalloc_plan(2 * ny, &py2) || !noalloc_plan(nx, &pnx) || !noalloc_plan(nz, &pnz)) return KMM_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return KMM_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    // the arrays' device addresses on the current device, resolved on every call (a lookup that
    // allocates nothing); if they moved (the device was reset and the module reloaded), the
    // twiddles cached there are gone and are sent again
    {
        void *a = NULL, *b = NULL;
        if (cudaGetSymbolAddress(&a, g_noalloc_scratch) != cudaSuccess) return KMM_ERR_CUDA;
        if (cudaGetSymbolAddress(&b, g_noalloc_tw) != cudaSuccess) return KMM_ERR_CUDA;
        if ((double *)a != s_scratch[dev] || (double2 *)b != s_tw[dev])
            for (int t = 0; t < 3; ++t) s_tw_len[dev][t] = 0;
        s_scratch[dev] = (double *)a;
        s_tw[dev] = (double2 *)b;
    }
    // twiddles exp(-2 pi i m/n), computed in long double as the context plans are; re-sent only
    // when a transform length changes.  The staging buffer is ordinary (pageable) host memory, so
    // such a call returns only once the stream has reached the copy.
    const int lens[3] = {2 * ny, nx, nz};
    DevPlan *plans[3] = {&py2, &pnx, &pnz};
    for (int t = 0; t < 3; ++t) {
        const int n = lens[t];
        double2 *h = s_tw_host[dev] + t * NOALLOC_TW_MAX;
        if (s_tw_len[dev][t] != n) {
            for (int k = 0; k < n; ++k) {
                long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
                h[k] = make_double2((double)cosl(ang), -(double)sinl(ang));
            }
            if (cudaMemcpyAsync(s_tw[dev] + t * NOALLOC_TW_MAX, h, sizeof(double2) * (size_t)n, cudaMemcpyHostToDevice,
                                st) != cudaSuccess)
                return KMM_ERR_CUDA;
            s_tw_len[dev][t] = n;
        }
        plans[t]->tw = s_tw[dev] + t * NOALLOC_TW_MAX;
    }
    // shared memory of each kernel (at most 128 KiB at the 4096 limit): lengths past the 48 KiB
    // default opt in once; setting a function attribute allocates nothing
    const size_t sy = sizeof(double2) * 4 * (size_t)ny, sx = sizeof(double2) * 2 * (size_t)nx,
                 sz = sizeof(double2) * 2 * (size_t)nz;
    const void *kern[3] = {(const void *)k_xyz_y, (const void *)k_xyz_x, (const void *)k_xyz_z};
    const size_t need[3] = {sy, sx, sz};
    for (int t = 0; t < 3; ++t)
        if (need[t] > 48 * 1024 &&
            cudaFuncSetAttribute(kern[t], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need[t]) != cudaSuccess)
            return KMM_ERR_CUDA;
    // same sequence as kmm_xyzfft: copy, y DCT-I (/ny, halved ends), x r2c (/nx), z c2c (/nz)
    double *b = s_scratch[dev];
    if (cudaMemcpyAsync(b, phys, sizeof(double) * nyp * (size_t)nz * (size_t)nx, cudaMemcpyDeviceToDevice, st) !=
        cudaSuccess)
        return KMM_ERR_CUDA;
    k_xyz_y<<<nz * nx, 128, sy, st>>>(b, py2, (int)nyp, nz * nx);
    if (cudaGetLastError() != cudaSuccess) return KMM_ERR_CUDA;
    k_xyz_x<<<(int)nyp * nz, 128, sx, st>>>(b, (double2 *)spec, pnx, (int)nyp, nz, nx);
    if (cudaGetLastError() != cudaSuccess) return KMM_ERR_CUDA;
    k_xyz_z<<<(int)nyp * (nx / 2), 128, sz, st>>>((double2 *)spec, pnz, (int)nyp, nz);
    if (cudaGetLastError() != cudaSuccess) return KMM_ERR_CUDA;
    return KMM_OK;
}
