// kmm_plane.cu -- vcw3dp (solvers.f90:1726-3538): dealiased nonlinear terms on the 3/2 grid.
//
// Data flow per call (all FP64):
//   1. k_dct_fwd : spectral columns (nyp,nz,nxh) * c(i)/2 -> DCT-I along y (REDFT00)
//                  -> plane layout PL[f][y][kx][kz]                        (solvers.f90:2241-2546)
//   2. k_zfft_bwd: zero-pad kz nz -> mz (modes j > nzh move to (mz-nz)+j), inverse c2c along z
//                  -> Q[f][y][z][kx]                                        (solvers.f90:2578-2803)
//   3. k_xphys   : per (y,z) row: Hermitian c2r along x (two fields per complex FFT),
//                  pointwise u x omega, -u.grad(c), polymer source/stress, CFL, immersed
//                  boundary forces and dPdx; physical outputs -> PO[o][y][z][x],
//                  u,v,w -> 3/2-grid copies for the tracers                 (solvers.f90:2806-3139)
//   4. k_spread  : 5x5 force spreading for the planes i <= kmaxsurf (or all, ib_spread_all) (solvers.f90:3069-3108)
//   5. k_xfwd    : r2c along x, keep kx < nxh                              (solvers.f90:3147-3177)
//   6. k_zfft_fwd: c2c along z, truncate to nz, /(mx*mz) -> PL[o][y][kx][kz] (solvers.f90:3180-3273)
//   7. k_dct_bwd : DCT-I along y, /ny, halve first and last coefficient    (solvers.f90:3279-3416)
// The internal 3/2-grid layout is [y][z][x] (x fastest); kmm_upload / kmm_download convert the
// reference's (nyp,mz,mx) arrays.
#include <math.h>

#include <algorithm>
#include <vector>

#include "kmm_internal.cuh"
#include "kmm_fft.cuh"
#include "kmm_async.cuh"

#define MAXIO 64

struct FieldPtrs { const double2 *p[MAXIO]; };
struct FieldPtrsW { double2 *p[MAXIO]; };

// Block FFT buffers.  At the compiled lengths each of the 8 warps owns NQ = NB / 8 consecutive
// sequences, stored swizzled (swz<C>, kmm_fft.cuh) within the warp's region, and the warps'
// regions lie FB_PAD elements further apart than NQ n: the radix stages then run free of bank
// conflicts, and so do the transposing loads and stores around the transform, whose 8 (or 16)
// concurrent sequences would otherwise sit n apart on the same banks.  The runtime FFT of the
// other lengths keeps the plain layout (sequence c at c n).
#define FB_PAD 1

// elements of one buffer (a or b) of NB sequences of length n
__host__ __device__ constexpr int fb_len(int nb, int n) { return nb * n + 8 * FB_PAD; }

__device__ __forceinline__ bool fb_compiled(int n) {
    return n == 48 || n == 64 || n == 96 || n == 128 || n == 144 || n == 192 || n == 256 || n == 576;
}

// position of element i of sequence c (ct: n is a compiled length)
template <typename C, int NB>
__device__ __forceinline__ int fb_at(int c, int i, int n, bool ct) {
    constexpr int NQ = NB / 8;
    if (!ct) return c * n + i;
    const int wq = c / NQ, q = c - wq * NQ;
    return wq * (NQ * n + FB_PAD) + swz<C>(q * n + i);
}

// batched FFT of NB sequences of length N (layout of fb_at) by the block's 8 warps, NB / 8
// sequences each, with the compile-time warp FFT; returns the buffer holding the result, visible
// to the whole block
template <typename C, int N, int S, int NB>
__device__ __forceinline__ C *fft_block_ct(C *a, C *b, const C *tw) {
    constexpr int NQ = NB / 8;
    static_assert(NB % 8 == 0, "8 warps share the sequences");
    static_assert(N % (sizeof(C) == 16 ? 8 : 16) == 0, "swizzle rows of 128 bytes");
    const size_t w = (size_t)(threadIdx.x >> 5) * (NQ * N + FB_PAD);
    C *r = fft_warp_ct<C, N, S, NQ, true>(a + w, b + w, tw);
    __syncthreads();
    return r - w;
}

// the same for the compiled lengths (the 3/2 grids of 32 .. 128 and 384, 2 ny for ny = 32 .. 128), the
// runtime block FFT for any other (FP64 only: the FP32 forms of the mixed precision run at the
// compiled lengths, which the host checks); blockDim = 256; tw: the table of length n in C
template <typename C, int S, int NB>
__device__ C *fft_block(const DevPlan &P, C *a, C *b, const C *tw, int n) {
    switch (n) {
    case 48: return fft_block_ct<C, 48, S, NB>(a, b, tw);
    case 64: return fft_block_ct<C, 64, S, NB>(a, b, tw);
    case 96: return fft_block_ct<C, 96, S, NB>(a, b, tw);
    case 128: return fft_block_ct<C, 128, S, NB>(a, b, tw);
    case 144: return fft_block_ct<C, 144, S, NB>(a, b, tw);
    case 192: return fft_block_ct<C, 192, S, NB>(a, b, tw);
    case 256: return fft_block_ct<C, 256, S, NB>(a, b, tw);
    case 576: return fft_block_ct<C, 576, S, NB>(a, b, tw);
    default:
        if constexpr (sizeof(C) == sizeof(double2)) return fft_smem(P, a, b, NB, n, S);
        else return a;
    }
}

// ---------------------------------------------------------------------------
// 1. forward Chebyshev -> physical y (scaled by c(i)/2), columns -> plane layout
// ---------------------------------------------------------------------------
#define DCT_CB 8
#define LDG 4   // global loads per thread issued together in the transforms' staging loops
template <typename C>
__global__ void __launch_bounds__(256) k_dct_fwd(const __grid_constant__ FieldPtrs in, C *__restrict__ pl, const __grid_constant__ DevPlan P, const C *__restrict__ tw,
                                                 int nyp, int nz, int nxh, int ncols) {
    typedef typename kct::Real<C>::T T;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int ny = nyp - 1, L = 2 * ny;
    const int f = blockIdx.y;
    const int col0 = blockIdx.x * DCT_CB;
    const int ncb = min(DCT_CB, ncols - col0);
    C *a = sm, *b = sm + fb_len(DCT_CB, L);
    const bool ct = fb_compiled(L);
    const double2 *src = in.p[f] + (size_t)col0 * nyp;
    // loads in groups of LDG per thread, all in flight before their shared-memory stores
    for (int e0 = threadIdx.x; e0 < ncb * nyp; e0 += LDG * 256) {
        double2 wv[LDG];
#pragma unroll
        for (int u = 0; u < LDG; ++u)
            if (e0 + 256 * u < ncb * nyp) wv[u] = src[e0 + 256 * u];
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            if (e >= ncb * nyp) break;
            const int c = e / nyp, i = e - c * nyp;
            const double2 w = wv[u];
            const double fac = (i == 0 || i == ny) ? 1.0 : 0.5;   // c(i)/2.0
            const C v = kct::mk<C>((T)(w.x * fac), (T)(w.y * fac));
            a[fb_at<C, DCT_CB>(c, i, L, ct)] = v;
            if (i > 0 && i < ny) a[fb_at<C, DCT_CB>(c, L - i, L, ct)] = v;
        }
    }
    for (int e = threadIdx.x; e < (DCT_CB - ncb) * L; e += blockDim.x)
        a[fb_at<C, DCT_CB>(ncb + e / L, e % L, L, ct)] = kct::mk<C>((T)0, (T)0);
    __syncthreads();
    C *r = fft_block<C, -1, DCT_CB>(P, a, b, tw, L);
    // PL[f][y][kx][kz]: col = kx*nz + kz
    for (int e = threadIdx.x; e < ncb * nyp; e += blockDim.x) {
        const int y = e / ncb, c = e - y * ncb;
        const int col = col0 + c;
        const int kx = col / nz, kz = col - kx * nz;
        pl[(((size_t)f * nyp + y) * nxh + kx) * nz + kz] = r[fb_at<C, DCT_CB>(c, y, L, ct)];
    }
}

// DCT-I of one column by an N-point FFT (N = ny, a compiled length), on one warp:
//   X_k = x_0 + (-1)^k x_N + 2 sum_{n=1}^{N-1} x_n cos(pi n k / N),  k = 0 .. N,
// the DFT of the even extension of length 2N that k_dct_fwd / k_dct_bwd transform otherwise.
// With y_j = (x_j + x_{N-j}) / 2 + sin(pi j / N) (x_j - x_{N-j}) (j < N) and Y = FFT_N(y):
//   X_{2m} = Y_m + Y_{N-m} (Y_N = Y_0),  X_{2m+1} = X_{2m-1} - i (Y_m - Y_{N-m}),
//   X_1 = x_0 - x_N + 2 sum_{n=1}^{N-1} x_n cos(pi n / N)
// (the half-length form of the DCT-I; the real and imaginary parts of the column are two real
// sequences, carried together).  x: the column's N + 1 values in shared memory, overwritten by X;
// a, b: the warp's FFT buffers (N elements, swizzled); tw: the 2N-point twiddles exp(-i pi m / N).
template <typename C, int N>
__device__ __forceinline__ void dct1_half(C *x, C *a, C *b, const C *__restrict__ tw) {
    typedef typename kct::Real<C>::T T;
    constexpr int H = N / 2, Q = (H + 31) / 32;
    const int lane = threadIdx.x & 31;
    C seed = kct::mk<C>((T)0, (T)0);
    for (int j = lane; j < N; j += 32) {
        const C xj = x[j], xr = x[N - j];
        const C w = tw[j];   // (cos, -sin) of pi j / N
        const C sm = kct::add(xj, xr), df = kct::sub(xj, xr);
        const T sn = -w.y;
        a[swz<C>(j)] = kct::mk<C>((T)0.5 * sm.x + sn * df.x, (T)0.5 * sm.y + sn * df.y);
        seed = j == 0 ? kct::add(seed, df) : kct::add(seed, kct::scl(xj, (T)2 * w.x));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1)
        seed = kct::add(seed, kct::mk<C>(__shfl_xor_sync(0xffffffffu, seed.x, o), __shfl_xor_sync(0xffffffffu, seed.y, o)));
    __syncwarp();
    // N = 256: the FFT in place in a (one buffer per warp: three blocks per SM instead of two)
    const C *Y;
    if constexpr (N == 256) {
        fft_warp_ct_inplace<C, N, -1, 2>(a, tw);
        Y = a;
    } else {
        Y = fft_warp_ct<C, N, -1, 1, true, 2>(a, b, tw);
    }
    // odd outputs: X_{2m+1} = seed + sum_{t=1}^{m} d_t, d_t = -i (Y_t - Y_{N-t}); lane holds m = lane Q .. lane Q + Q - 1
    C d[Q];
    C tot = kct::mk<C>((T)0, (T)0);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int m = lane * Q + q;
        C v = kct::mk<C>((T)0, (T)0);
        if (m >= 1 && m < H) {
            const C df = kct::sub(Y[swz<C>(m)], Y[swz<C>(N - m)]);
            v = kct::mk<C>(df.y, -df.x);
        }
        tot = kct::add(tot, v);
        d[q] = tot;   // inclusive prefix within the lane
    }
    C excl = tot;   // inclusive scan of the lane totals, then shifted to exclusive
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const C u = kct::mk<C>(__shfl_up_sync(0xffffffffu, excl.x, o), __shfl_up_sync(0xffffffffu, excl.y, o));
        if (lane >= o) excl = kct::add(excl, u);
    }
    excl = kct::sub(excl, tot);
    // even outputs (all lanes read Y before anyone writes x)
    C ev[(H + 1 + 31) / 32];
#pragma unroll
    for (int e = 0; e < (H + 1 + 31) / 32; ++e) {
        const int m = lane + 32 * e;
        if (m <= H) ev[e] = kct::add(Y[swz<C>(m)], Y[swz<C>(m == 0 ? 0 : N - m)]);
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < (H + 1 + 31) / 32; ++e) {
        const int m = lane + 32 * e;
        if (m <= H) x[2 * m] = ev[e];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int m = lane * Q + q;
        if (m < H) x[2 * m + 1] = kct::add(seed, kct::add(excl, d[q]));
    }
    __syncwarp();
}

// k_dct_fwd for ny in {48, 64, 96, 128, 256} with the half-length DCT-I: a warp per column, the
// block's 8 columns staged in shared memory (column stride N + 1, odd: the transposing store
// reads 8 columns at one y without bank conflicts)
template <typename C, int N>
__global__ void __launch_bounds__(256) k_dct_fwd_h(const __grid_constant__ FieldPtrs in, C *__restrict__ pl, const C *__restrict__ tw, int nz,
                                                   int nxh, int ncols) {
    typedef typename kct::Real<C>::T T;
    constexpr int NYP = N + 1;
    extern __shared__ double2 smd[];
    C *xs = reinterpret_cast<C *>(smd);
    C *a = xs + DCT_CB * NYP, *b = a + fb_len(DCT_CB, N);
    const int f = blockIdx.y;
    const int col0 = blockIdx.x * DCT_CB;
    const int ncb = min(DCT_CB, ncols - col0);
    const double2 *src = in.p[f] + (size_t)col0 * NYP;
    for (int e0 = threadIdx.x; e0 < ncb * NYP; e0 += LDG * 256) {
        double2 wv[LDG];
#pragma unroll
        for (int u = 0; u < LDG; ++u)
            if (e0 + 256 * u < ncb * NYP) wv[u] = src[e0 + 256 * u];
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            if (e >= ncb * NYP) break;
            const int i = e % NYP;
            const double fac = (i == 0 || i == N) ? 1.0 : 0.5;   // c(i)/2.0
            xs[e] = kct::mk<C>((T)(wv[u].x * fac), (T)(wv[u].y * fac));
        }
    }
    __syncthreads();
    const int c = threadIdx.x >> 5;
    if (c < ncb) dct1_half<C, N>(xs + c * NYP, a + c * (N + FB_PAD), b + c * (N + FB_PAD), tw);
    __syncthreads();
    // PL[f][y][kx][kz]: col = kx*nz + kz
    for (int e = threadIdx.x; e < ncb * NYP; e += blockDim.x) {
        const int y = e / ncb, cc = e - y * ncb;
        const int col = col0 + cc;
        const int kx = col / nz, kz = col - kx * nz;
        pl[(((size_t)f * NYP + y) * nxh + kx) * nz + kz] = xs[cc * NYP + y];
    }
}

// ---------------------------------------------------------------------------
// 2. z: zero-pad + inverse c2c (FFTW_BACKWARD)
// ---------------------------------------------------------------------------
#define ZKB 8   // kx columns per block of the z transforms (one sequence per warp; 4 blocks per SM)
// where each output field of the z inverse comes from: plane base[f] of the y-transformed inputs,
// multiplied by 1 (mult 0), i kx (1) or i kz (2) -- the x and z derivatives of a field formed here
// instead of as separate spectral fields with their own y transforms
struct ZRecipe {
    unsigned char base[MAXIO], mult[MAXIO];
};

// the rows the x stage reads for each pair of inputs (2 p, 2 p + 1): the z-inverse outputs qa and
// qb, or (xd = 1) the one row qa, the pair's second input being i kx times the first, formed in
// the x stage (qb = 255: the pair has one input)
struct XRecipe {
    unsigned char qa[MAXIO / 2], qb[MAXIO / 2], xd[MAXIO / 2];
};

// the z inverse at a compiled length N: warp c transforms column c of the block, its FFT's first
// stage reading the column's nz modes straight from global memory (zero-padded to N, times i kx or
// i kz where the recipe asks), its last stage writing the block buffer in the fb_at layout;
// returns that buffer, visible to the whole block
template <typename C, int N>
__device__ __forceinline__ C *zbwd_io(const C *__restrict__ src, C *a, C *b, const C *__restrict__ tw, int nk, int nz,
                                      int kx0, int mult, const double *__restrict__ wavx,
                                      const double *__restrict__ wavz) {
    typedef typename kct::Real<C>::T T;
    static_assert(ZKB == 8, "one column per warp");
    C *res = kct::nfac(N) % 2 == 1 ? a : b;
    const int c = threadIdx.x >> 5;
    if (c < nk) {
        const size_t w = (size_t)c * (N + FB_PAD);
        const C *col = src + (size_t)c * nz;
        const int nzh = nz / 2, hi = N - nz + nzh;
        auto ld = [&](int z) {
            C v = kct::mk<C>((T)0, (T)0);
            if (z < nzh || z >= hi) {
                const int j = z < nzh ? z : z - (N - nz);
                v = col[j];
                if (mult) {   // i k v
                    const T k = (T)(mult == 1 ? wavx[kx0 + c] : wavz[j]);
                    v = kct::mk<C>(-k * v.y, k * v.x);
                }
            }
            return v;
        };
        auto st = [&](int x, C v) { res[w + swz<C>(x)] = v; };
        auto pre = [] {};
        fft_warp_ct_io<C, N, +1>(ld, st, pre, a + w, b + w, tw);
    }
    __syncthreads();
    return res;
}

// BIG (mz = 576 only): one buffer per block, each warp's FFT in place (fft_warp_ct_inplace), so two
// blocks share an SM where the two 74 KB buffers held it to one
template <typename C, bool BIG = false>
__global__ void __launch_bounds__(256, BIG ? 2 : 4) k_zfft_bwd(const C *__restrict__ pl, C *__restrict__ q, const __grid_constant__ DevPlan P,
                                                  const C *__restrict__ tw, int nyp, int nz, int nxh, int mz,
                                                  const __grid_constant__ ZRecipe R, const double *__restrict__ wavx,
                                                  const double *__restrict__ wavz) {
    typedef typename kct::Real<C>::T T;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int y = blockIdx.y, f = blockIdx.z, fb = R.base[f], mult = R.mult[f];
    const int kx0 = blockIdx.x * ZKB;
    const int nk = min(ZKB, nxh - kx0);
    const int nzh = nz / 2;
    C *a = sm, *b = sm + fb_len(ZKB, mz);
    const bool ct = fb_compiled(mz);
    const C *src = pl + (((size_t)fb * nyp + y) * nxh + kx0) * nz;
    C *r = NULL;
    if constexpr (!BIG) switch (mz) {
    case 48: r = zbwd_io<C, 48>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    case 64: r = zbwd_io<C, 64>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    case 96: r = zbwd_io<C, 96>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    case 128: r = zbwd_io<C, 128>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    case 144: r = zbwd_io<C, 144>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    case 192: r = zbwd_io<C, 192>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    case 256: r = zbwd_io<C, 256>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    case 576: r = zbwd_io<C, 576>(src, a, b, tw, nk, nz, kx0, mult, wavx, wavz); break;
    default: break;
    }
    if (!r) {   // the runtime block FFT: stage the zero-padded columns, then transform
        for (int e = threadIdx.x; e < fb_len(ZKB, mz); e += blockDim.x) a[e] = kct::mk<C>((T)0, (T)0);
        __syncthreads();
        for (int e0 = threadIdx.x; e0 < nk * nz; e0 += LDG * 256) {
            C wv[LDG];
#pragma unroll
            for (int u = 0; u < LDG; ++u)
                if (e0 + 256 * u < nk * nz) wv[u] = src[e0 + 256 * u];
#pragma unroll
            for (int u = 0; u < LDG; ++u) {
                const int e = e0 + 256 * u;
                if (e >= nk * nz) break;
                const int c = e / nz, j = e - c * nz;
                const int jj = (j < nzh) ? j : (mz - nz) + j;
                C v = wv[u];
                if (mult) {   // i k v
                    const T k = (T)(mult == 1 ? wavx[kx0 + c] : wavz[j]);
                    v = kct::mk<C>(-k * v.y, k * v.x);
                }
                a[fb_at<C, ZKB>(c, jj, mz, ct)] = v;
            }
        }
        __syncthreads();
        if constexpr (BIG) {
            const int w = threadIdx.x >> 5;
            if (w < nk) fft_warp_ct_inplace<C, 576, +1>(a + (size_t)w * (576 + FB_PAD), tw);
            __syncthreads();
            r = a;
        } else {
            r = fft_block<C, +1, ZKB>(P, a, b, tw, mz);
        }
    }
    C *dst = q + (((size_t)f * nyp + y) * mz) * nxh;
    for (int e = threadIdx.x; e < nk * mz; e += blockDim.x) {
        const int z = e / nk, c = e - z * nk;
        dst[(size_t)z * nxh + kx0 + c] = r[fb_at<C, ZKB>(c, z, mz, ct)];
    }
}

// ---------------------------------------------------------------------------
// 3. x: c2r + pointwise physics
// ---------------------------------------------------------------------------
// input slots (order of the physical arrays used below)
enum { S_U, S_V, S_W, S_WX, S_WY, S_WZ, S_U11, S_U12, S_U13, S_U21, S_U22, S_U23, S_U31, S_U32, S_U33,
       S_SC, S_CX, S_CY, S_CZ, S_C11, S_DC111 = S_C11 + 9, S_LU = S_DC111 + 27, S_LV, S_LW, S_NSLOT };
enum { O_H1, O_H2, O_H3, O_SC, O_C11N, O_STR11N = O_C11N + 6, O_QP11 = O_STR11N + 6, O_NSLOT = O_QP11 + 6 };

// 3/2-grid copies kept for the inertial-particle path: wx, wy, wz, u11 .. u33 (slots S_WX .. S_U33),
// then Lu, Lv, Lw; p[0] == NULL when the path is off
struct Save3D { double *p[15]; };

struct PhysArgs {
    int slot_of_in[S_NSLOT];    // index into the input list, -1 if not transformed
    int slot_of_out[O_NSLOT];   // index into the output list, -1 if not produced
    int nin, nout;
    int scalar, polymer, ipeter, itarget, scl_flag, flow_select, it, perturbtime, save_uvw, ib_any;
    double delxm, delzm, dt, dPdx, gain, ugain, zl2, qbeta, alpha_poly, re, tpoly, scalar_q;
};

__device__ __forceinline__ void atomic_max_pos(double *addr, double v) {
    // max of non-negative doubles (NaN bit patterns compare larger and propagate)
    atomicMax((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

// the pointwise terms of one 3/2-grid point (solvers.f90:2885-3063): u x omega, -u.grad(c) and
// its sources, the polymer source / stress / qp terms, CFL, immersed-boundary forces and dPdx,
// the tracer / inertial-particle copies; `in(slot)` is the physical value of an input slot here
template <typename IN_T, typename PO_T>
__device__ __forceinline__ void xphys_point(const IN_T &in, const PhysArgs &A, const Save3D &sv, int y, int z, int k,
                                            int nyp, int mz, int mx, double sg, PO_T *__restrict__ po,
                                            double *__restrict__ drag, double *__restrict__ up3,
                                            double *__restrict__ vp3, double *__restrict__ wp3,
                                            const int *__restrict__ imatrix, double *__restrict__ fxi,
                                            double *__restrict__ fyi, double *__restrict__ fzi,
                                            const double *__restrict__ scsource, double &cmax, double &umx) {
#define IN(s) in(s)
    const double up = IN(S_U), vp = IN(S_V), wp = IN(S_W);
    const double wxp = IN(S_WX), wyp = IN(S_WY), wzp = IN(S_WZ);
    double out[O_NSLOT];
    out[O_H1] = vp * wzp - wp * wyp;
    out[O_H2] = -up * wzp + wp * wxp;
    out[O_H3] = up * wyp - vp * wxp;
    if (A.scalar) out[O_SC] = -(up * IN(S_CX) + vp * IN(S_CY) + wp * IN(S_CZ));
    if (A.polymer) {
        double c[9], gu[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) { c[m] = IN(S_C11 + m); gu[m] = IN(S_U11 + m); }
        const double c11 = c[0], c12 = c[1], c13 = c[2], c21 = c[3], c22 = c[4], c23 = c[5], c31 = c[6], c32 = c[7], c33 = c[8];
        const double u11 = gu[0], u12 = gu[1], u13 = gu[2], u21 = gu[3], u22 = gu[4], u23 = gu[5], u31 = gu[6], u32 = gu[7], u33 = gu[8];
#define DC(ij, kk) IN(S_DC111 + 3 * (ij) + (kk))
        out[O_C11N + 0] = c11 * u11 + c12 * u12 + c13 * u13 + c11 * u11 + c21 * u12 + c31 * u13 - (up * DC(0, 0) + vp * DC(0, 1) + wp * DC(0, 2));
        out[O_C11N + 1] = c11 * u21 + c12 * u22 + c13 * u23 + c12 * u11 + c22 * u12 + c32 * u13 - (up * DC(1, 0) + vp * DC(1, 1) + wp * DC(1, 2));
        out[O_C11N + 2] = c11 * u31 + c12 * u32 + c13 * u33 + c13 * u11 + c23 * u12 + c33 * u13 - (up * DC(2, 0) + vp * DC(2, 1) + wp * DC(2, 2));
        out[O_C11N + 3] = c21 * u21 + c22 * u22 + c23 * u23 + c12 * u21 + c22 * u22 + c32 * u23 - (up * DC(4, 0) + vp * DC(4, 1) + wp * DC(4, 2));
        out[O_C11N + 4] = c21 * u31 + c22 * u32 + c23 * u33 + c13 * u21 + c23 * u22 + c33 * u23 - (up * DC(5, 0) + vp * DC(5, 1) + wp * DC(5, 2));
        out[O_C11N + 5] = c31 * u31 + c32 * u32 + c33 * u33 + c13 * u31 + c23 * u32 + c33 * u33 - (up * DC(8, 0) + vp * DC(8, 1) + wp * DC(8, 2));
#undef DC
        const double trp = c11 + c22 + c33;
        const double s6[6] = {c11, c12, c13, c22, c23, c33};
        const double pf = (A.zl2 - 3.0) / (A.zl2 - trp);
#pragma unroll
        for (int m = 0; m < 6; ++m) out[O_STR11N + m] = A.ipeter == 0 ? s6[m] : pf * s6[m];
        out[O_STR11N + 0] -= 1.0;
        out[O_STR11N + 3] -= 1.0;
        out[O_STR11N + 5] -= 1.0;
        double beta_poly = A.qbeta;
        if (A.itarget == 1) {
            const double sc = fabs(A.scalar ? IN(S_SC) : 0.0);
            if (A.alpha_poly * sc < 18.0) beta_poly = exp(-A.alpha_poly * sc);
        } else if (A.itarget == 2) {
            const double sc = fabs(A.scalar ? IN(S_SC) : 0.0);
            beta_poly = 1.0 / (A.alpha_poly * sc + 1.0);
        }
        const double zbeta1 = (1.0 - beta_poly) / (A.re * beta_poly * A.tpoly);
#pragma unroll
        for (int m = 0; m < 6; ++m) out[O_QP11 + m] = zbeta1 * out[O_STR11N + m];
    }
    const double cflcheck = (fabs(up) / A.delxm + fabs(vp) / sg + fabs(wp) / A.delzm) * A.dt;
    cmax = fmax(cmax, cflcheck);
    if (cflcheck != cflcheck) cmax = cflcheck;
    umx = fmax(umx, fabs(up));
    // immersed boundary (solvers.f90:2996-3059); fxintg etc. in [y][z][x] layout
    const size_t g3 = ((size_t)y * mz + z) * mx + k;
    double dx = 0.0, dy = 0.0, dz = 0.0;
    if (A.ib_any) {
        const int t = imatrix[g3];
        if (t == 1 || (t == 4 && A.it <= A.perturbtime)) {
            const double fx = fxi[g3] + up, fy = fyi[g3] + vp, fz = fzi[g3] + wp;
            fxi[g3] = fx; fyi[g3] = fy; fzi[g3] = fz;
            dx = (-A.ugain * up) - A.gain * fx;
            dy = (-A.ugain * vp) - A.gain * fy;
            dz = (-A.ugain * wp) - A.gain * fz;
        } else if (t == 3) {
            const double fz = fzi[g3] + wp;
            fzi[g3] = fz;
            dz = -A.ugain * wp - A.gain * fz;
        } else if (t == 11) {
            dx = 1.0;
        } else if (t == 0 && A.flow_select == 1) {
            out[O_H1] = out[O_H1] - A.dPdx;
        }
        drag[0 * (size_t)nyp * mz * mx + g3] = dx;
        drag[1 * (size_t)nyp * mz * mx + g3] = dy;
        drag[2 * (size_t)nyp * mz * mx + g3] = dz;
    } else if (A.flow_select == 1) {
        out[O_H1] = out[O_H1] - A.dPdx;
    }
    if (A.scalar) {
        if (A.scl_flag >= 2) out[O_SC] = out[O_SC] + scsource[g3] / A.dt;
        if (A.scalar_q != 0.0) out[O_SC] = out[O_SC] + A.scalar_q;
    }
    for (int o = 0; o < O_NSLOT; ++o) {
        const int s = A.slot_of_out[o];
        if (s >= 0) po[(size_t)s * nyp * mz * mx + g3] = (PO_T)out[o];
    }
    if (A.save_uvw) { up3[g3] = up; vp3[g3] = vp; wp3[g3] = wp; }
    if (sv.p[0]) {
#pragma unroll
        for (int m = 0; m < 12; ++m) sv.p[m][g3] = IN(S_WX + m);
#pragma unroll
        for (int m = 0; m < 3; ++m) sv.p[12 + m][g3] = IN(S_LU + m);
    }
#undef IN
}

#define XZB 2
__global__ void __launch_bounds__(256) k_xphys(const double2 *__restrict__ q, double *__restrict__ po,
                                               double *__restrict__ drag, double *__restrict__ up3,
                                               double *__restrict__ vp3, double *__restrict__ wp3,
                                               const int *__restrict__ imatrix, double *__restrict__ fxi,
                                               double *__restrict__ fyi, double *__restrict__ fzi,
                                               const double *__restrict__ scsource, const double *__restrict__ seght,
                                               double *__restrict__ cfl, double *__restrict__ umax, const __grid_constant__ DevPlan P,
                                               PhysArgs A, Save3D sv, int nyp, int mz, int mx, int nxh) {
    extern __shared__ double2 sm[];
    const int y = blockIdx.y;
    const int z0 = blockIdx.x * XZB;
    const int nzr = min(XZB, mz - z0);
    const int hx = mx / 2;
    // smem: phys[nin][XZB][mx] doubles, then FFT scratch a,b [XZB][mx] double2
    double *phys = (double *)sm;
    double2 *fa = (double2 *)(phys + (size_t)A.nin * XZB * mx);
    double2 *fb = fa + (size_t)XZB * mx;
    for (int f = 0; f < A.nin; f += 2) {
        const int g = f + 1 < A.nin ? f + 1 : -1;
        // Hermitian extension of A + iB for each row
        for (int e = threadIdx.x; e < XZB * mx; e += blockDim.x) {
            const int r = e / mx, k = e - r * mx;
            double2 v = make_double2(0.0, 0.0);
            if (r < nzr) {
                const int z = z0 + r;
                int kk = k <= hx ? k : mx - k;      // source mode
                double2 A_ = make_double2(0.0, 0.0), B_ = make_double2(0.0, 0.0);
                if (kk < nxh) {
                    A_ = q[(((size_t)f * nyp + y) * mz + z) * nxh + kk];
                    if (g >= 0) B_ = q[(((size_t)g * nyp + y) * mz + z) * nxh + kk];
                }
                if (k == 0 || k == hx) { A_.y = 0.0; B_.y = 0.0; }   // c2r ignores Im of DC / Nyquist
                if (k <= hx) v = make_double2(A_.x - B_.y, A_.y + B_.x);          // A + iB
                else v = make_double2(A_.x + B_.y, -A_.y + B_.x);                 // conj(A) + i conj(B)
            }
            fa[e] = v;
        }
        __syncthreads();
        double2 *r = fft_smem(P, fa, fb, XZB, mx, +1);
        for (int e = threadIdx.x; e < XZB * mx; e += blockDim.x) {
            const int rr = e / mx, k = e - rr * mx;
            phys[((size_t)f * XZB + rr) * mx + k] = r[e].x;
            if (g >= 0) phys[((size_t)g * XZB + rr) * mx + k] = r[e].y;
        }
        __syncthreads();
    }
    // pointwise terms, solvers.f90:2885-3063
    double cmax = 0.0, umx = 0.0;
    const double sg = seght[y];
    for (int e = threadIdx.x; e < nzr * mx; e += blockDim.x) {
        const int rr = e / mx, k = e - rr * mx;
        auto in = [&](int sl) { return phys[((size_t)A.slot_of_in[sl] * XZB + rr) * mx + k]; };
        xphys_point(in, A, sv, y, z0 + rr, k, nyp, mz, mx, sg, po, drag, up3, vp3, wp3, imatrix, fxi, fyi, fzi, scsource,
                    cmax, umx);
    }
    // block reductions of the CFL number and |u| for this plane
    __shared__ double red[2][32];
    for (int off = 16; off; off >>= 1) {
        double c2 = __shfl_down_sync(0xffffffffu, cmax, off);
        double u2 = __shfl_down_sync(0xffffffffu, umx, off);
        cmax = (c2 != c2) ? c2 : fmax(cmax, c2);
        umx = fmax(umx, u2);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = cmax; red[1][w] = umx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q2 = 1; q2 < (int)(blockDim.x >> 5); ++q2) {
            cmax = (red[0][q2] != red[0][q2]) ? red[0][q2] : fmax(cmax, red[0][q2]);
            umx = fmax(umx, red[1][q2]);
        }
        atomic_max_pos(&cfl[y], cmax);
        atomic_max_pos(&umax[y], umx);
    }
}

// 3''. the x stage for 3/2 grids too long for a row of every input field to fit in shared memory
// (k_xphys needs nin x 2 rows x mx doubles: 507 KB for the 55 polymer inputs at mx = 576).  Two
// passes through HBM: k_xinv_big takes the Hermitian c2r of one field pair for XZB rows with the
// runtime block FFT (the same transform as k_xphys) into a physical buffer [f][y][z][x]; k_xpoint
// evaluates the same pointwise terms (xphys_point) with one thread per 3/2-grid point, every block
// inside one y-plane for the CFL / |u| reductions.
__global__ void __launch_bounds__(256) k_xinv_big(const double2 *__restrict__ q, double *__restrict__ pb, const __grid_constant__ DevPlan P,
                                                  int nin, int nyp, int mz, int mx, int nxh) {
    extern __shared__ double2 sm[];
    const int y = blockIdx.y, f = 2 * blockIdx.z, g = f + 1 < nin ? f + 1 : -1;
    const int z0 = blockIdx.x * XZB, nzr = min(XZB, mz - z0), hx = mx / 2;
    double2 *fa = sm, *fb = sm + (size_t)XZB * mx;
    const size_t nphys = (size_t)nyp * mz * mx;
    for (int e = threadIdx.x; e < XZB * mx; e += blockDim.x) {
        const int r = e / mx, k = e - r * mx;
        double2 v = make_double2(0.0, 0.0);
        if (r < nzr) {
            const int z = z0 + r;
            const int kk = k <= hx ? k : mx - k;
            double2 A_ = make_double2(0.0, 0.0), B_ = make_double2(0.0, 0.0);
            if (kk < nxh) {
                A_ = q[(((size_t)f * nyp + y) * mz + z) * nxh + kk];
                if (g >= 0) B_ = q[(((size_t)g * nyp + y) * mz + z) * nxh + kk];
            }
            if (k == 0 || k == hx) { A_.y = 0.0; B_.y = 0.0; }
            if (k <= hx) v = make_double2(A_.x - B_.y, A_.y + B_.x);
            else v = make_double2(A_.x + B_.y, -A_.y + B_.x);
        }
        fa[e] = v;
    }
    __syncthreads();
    double2 *r = fft_smem(P, fa, fb, XZB, mx, +1);
    for (int e = threadIdx.x; e < nzr * mx; e += blockDim.x) {
        const int rr = e / mx, k = e - rr * mx;
        const size_t g3 = ((size_t)y * mz + z0 + rr) * mx + k;
        pb[(size_t)f * nphys + g3] = r[e].x;
        if (g >= 0) pb[(size_t)g * nphys + g3] = r[e].y;
    }
}

// pass 1 at the compiled lengths (MX = 576: nx = 384), in either precision: one warp per (y, z)
// row and field pair, the Hermitian extension of A + iB (as in k_xphys2) through the compile-time
// warp FFT (FP64: run in place in one buffer, fft_warp_ct_ip, so four blocks of four warps share an
// SM instead of three), the two real rows stored to the physical buffer in precision C by its last
// stage
#define XBW 4   // rows (warps) per block of k_xinv_big2
template <int MX, typename C>
__global__ void __launch_bounds__(XBW * 32, sizeof(C) == 16 ? 4 : 6) k_xinv_big2(const C *__restrict__ q, typename kct::Real<C>::T *__restrict__ pb,
                                                        const C *__restrict__ tw, int nin, int nyp, int mz,
                                                        const __grid_constant__ XRecipe X,
                                                        const double *__restrict__ wavx) {
    typedef typename kct::Real<C>::T T;
    constexpr int NXH = MX / 3;
    extern __shared__ double2 smd[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.x * XBW + warp, y = blockIdx.y, f = 2 * blockIdx.z, g = f + 1 < nin ? f + 1 : -1;
    if (z >= mz) return;   // whole warps: no block barrier below
    // FP64: one buffer per warp, the FFT in place; FP32: two (its registers allow six blocks per SM)
    constexpr int NBUF = sizeof(C) == 16 ? 1 : 2;
    C *a = reinterpret_cast<C *>(smd) + (size_t)warp * NBUF * MX;
    const int pr = blockIdx.z;
    const bool xd = X.xd[pr];
    const C *qa = q + (((size_t)X.qa[pr] * nyp + y) * mz + z) * NXH;
    const C *qb = q + (((size_t)((g >= 0 && !xd) ? X.qb[pr] : X.qa[pr]) * nyp + y) * mz + z) * NXH;
    const C zc = kct::mk<C>((T)0, (T)0);
    for (int k = NXH + lane; k <= MX - NXH; k += 32) a[swz<C>(k)] = zc;
    for (int kk = lane; kk < NXH; kk += 32) {
        C A_ = qa[kk], B_ = g >= 0 ? qb[kk] : zc;
        if (xd) {   // the pair's second input is i kx times the first
            const T kx = (T)wavx[kk];
            B_ = kct::mk<C>(-kx * A_.y, kx * A_.x);
        }
        if (kk == 0) { A_.y = (T)0; B_.y = (T)0; }   // c2r ignores Im of the mean mode
        a[swz<C>(kk)] = kct::mk<C>(A_.x - B_.y, A_.y + B_.x);
        if (kk > 0) a[swz<C>(MX - kk)] = kct::mk<C>(A_.x + B_.y, -A_.y + B_.x);
    }
    __syncwarp();
    const size_t nphys = (size_t)nyp * mz * MX, g3 = ((size_t)y * mz + z) * MX;
    // the FFT's last stage stores the two real rows straight to the physical buffer (consecutive
    // lanes, consecutive x)
    T *pf = pb + (size_t)f * nphys + g3, *pg = pb + (size_t)(g >= 0 ? g : f) * nphys + g3;
    auto st = [&](int x, C v) {
        pf[x] = v.x;
        if (g >= 0) pg[x] = v.y;
    };
    if constexpr (NBUF == 1) {
        fft_warp_ct_ip<C, MX, +1>(a, st, tw);
    } else {
        auto ld = [&](int x) { return a[swz<C>(x)]; };
        auto pre = [] {};
        fft_warp_ct_io<C, MX, +1>(ld, st, pre, a + MX, a, tw);
    }
}

// pass 2: the pointwise terms from the physical buffer (precision T) into po (precision T)
template <typename T>
__global__ void __launch_bounds__(256) k_xpoint(const T *__restrict__ pb, T *__restrict__ po,
                                                double *__restrict__ drag, double *__restrict__ up3,
                                                double *__restrict__ vp3, double *__restrict__ wp3,
                                                const int *__restrict__ imatrix, double *__restrict__ fxi,
                                                double *__restrict__ fyi, double *__restrict__ fzi,
                                                const double *__restrict__ scsource, const double *__restrict__ seght,
                                                double *__restrict__ cfl, double *__restrict__ umax, PhysArgs A,
                                                Save3D sv, int nyp, int mz, int mx) {
    const int y = blockIdx.y;
    const size_t nplane = (size_t)mz * mx, nphys = (size_t)nyp * nplane;
    double cmax = 0.0, umx = 0.0;
    const double sg = seght[y];
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nplane; e += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(e / mx), k = (int)(e - (size_t)z * mx);
        const size_t g3 = (size_t)y * nplane + e;
        auto in = [&](int sl) { return (double)pb[(size_t)A.slot_of_in[sl] * nphys + g3]; };
        xphys_point(in, A, sv, y, z, k, nyp, mz, mx, sg, po, drag, up3, vp3, wp3, imatrix, fxi, fyi, fzi, scsource, cmax,
                    umx);
    }
    __shared__ double red[2][32];
    for (int off = 16; off; off >>= 1) {
        double c2 = __shfl_down_sync(0xffffffffu, cmax, off);
        double u2 = __shfl_down_sync(0xffffffffu, umx, off);
        cmax = (c2 != c2) ? c2 : fmax(cmax, c2);
        umx = fmax(umx, u2);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = cmax; red[1][w] = umx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q2 = 1; q2 < (int)(blockDim.x >> 5); ++q2) {
            cmax = (red[0][q2] != red[0][q2]) ? red[0][q2] : fmax(cmax, red[0][q2]);
            umx = fmax(umx, red[1][q2]);
        }
        atomic_max_pos(&cfl[y], cmax);
        atomic_max_pos(&umax[y], umx);
    }
}

// 3'. the same x stage for the compiled lengths MX = 48, 96, 144, 192 (nx = 32 .. 128): one block
// per (y, z) row, XPW warps.  Each warp takes field pairs in turn: the Hermitian extension of
// A + iB (modes nxh .. mx - nxh not carried; c2r ignores Im of the DC mode) through the
// compile-time warp FFT into the row's physical table in shared memory; then the block evaluates
// the pointwise terms.  The two physical rows of a pair are one buffer of MX complex values, which
// serves as the FFT's second (ping-pong) buffer once the pair's input has been read out of it, so
// a warp needs only one private buffer and two 7-warp blocks fit on an SM even with 55 fields.
// The generic k_xphys tiles two rows per block and transforms them with the runtime block FFT.
#define XW 4    // warps of k_xfwd2
// warps of k_xphys2: 7 in FP64 (two blocks per SM, held by shared memory and registers; the 28
// field pairs of the polymer + scalar inputs then take four full rounds, where 8 warps left half
// of them idle in the last round before the block barrier: 3.8 % faster at 128^3); 4 in FP32,
// whose halved row buffer already lets four blocks share an SM, where 8-warp blocks would be held
// to two by registers with more idle threads in the pointwise pass
template <typename C>
struct XpW {
    static constexpr int n = sizeof(C) == 16 ? 7 : 4;
};
template <int MX, typename C>
__global__ void __launch_bounds__(XpW<C>::n * 32) k_xphys2(const C *__restrict__ q, typename kct::Real<C>::T *__restrict__ po,
                                                    double *__restrict__ drag, double *__restrict__ up3,
                                                    double *__restrict__ vp3, double *__restrict__ wp3,
                                                    const int *__restrict__ imatrix, double *__restrict__ fxi,
                                                    double *__restrict__ fyi, double *__restrict__ fzi,
                                                    const double *__restrict__ scsource,
                                                    const double *__restrict__ seght, double *__restrict__ cfl,
                                                    double *__restrict__ umax, const C *__restrict__ tw,
                                                    PhysArgs A, Save3D sv, int nyp, int mz, int *status,
                                                    const __grid_constant__ XRecipe X, const double *__restrict__ wavx) {
    typedef typename kct::Real<C>::T T;
    constexpr int XPW = XpW<C>::n;
    constexpr int NXH = MX / 3;
    constexpr unsigned ROWB = NXH * sizeof(C);   // one field's row of kx modes
    static_assert(ROWB % 16 == 0 && (MX * sizeof(T)) % 16 == 0, "16-byte bulk copies");
    extern __shared__ double2 smd[];
    C *fab = reinterpret_cast<C *>(smd);                                  // per warp: a [MX]
    T *phys = reinterpret_cast<T *>(fab + (size_t)XPW * MX);              // [nin rounded up to even][MX]
    __shared__ uint64_t xbar[MAXIO / 2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.x, y = blockIdx.y;
    C *a = fab + (size_t)warp * MX;
    const int npairs = (A.nin + 1) / 2;
    // every input row of this (y, z) goes into the first 2 MX / 3 reals of its field's phys row by
    // one bulk copy, issued up front (one barrier per field pair), so the whole row set is in
    // flight at once; each pair's transform later overwrites its own rows only
    if (threadIdx.x == 0) {
        for (int pr = 0; pr < npairs; ++pr) kasync::mbar_init(&xbar[pr], 1);
        kasync::mbar_init_fence();
        for (int pr = 0; pr < npairs; ++pr) {
            const int f = 2 * pr, g = f + 1 < A.nin ? f + 1 : -1;
            const bool two = g >= 0 && !X.xd[pr];
            kasync::mbar_expect_tx(&xbar[pr], two ? 2 * ROWB : ROWB);
            kasync::bulk_g2s(phys + (size_t)f * MX, q + (((size_t)X.qa[pr] * nyp + y) * mz + z) * NXH, ROWB,
                             &xbar[pr]);
            if (two)
                kasync::bulk_g2s(phys + (size_t)g * MX, q + (((size_t)X.qb[pr] * nyp + y) * mz + z) * NXH, ROWB,
                                 &xbar[pr]);
        }
    }
    __syncthreads();
    bool ok = true;
    for (int pr = warp; pr < npairs; pr += XPW) {
        const int f = 2 * pr, g = f + 1 < A.nin ? f + 1 : -1;
        C *b = reinterpret_cast<C *>(phys + (size_t)f * MX);   // the pair's rows f, f + 1
        // every lane waits (its own acquire of the copied rows); the warp goes on only if all saw them
        if (!__all_sync(0xffffffffu, kasync::mbar_wait(&xbar[pr], 0))) {
            ok = false;
            continue;
        }
        const bool xd = X.xd[pr];
        const C *qa = reinterpret_cast<const C *>(phys + (size_t)f * MX);
        const C *qb = (g >= 0 && !xd) ? reinterpret_cast<const C *>(phys + (size_t)g * MX) : qa;
        // Hermitian extension: Z_k = A_k + i B_k for k < nxh, conj(A) + i conj(B) at mx - k, and the
        // modes nxh .. mx - nxh (the Nyquist mode mx / 2 among them) not carried; B = i kx A for an
        // x-derivative pair
        const C zc = kct::mk<C>((T)0, (T)0);
        for (int k = NXH + lane; k <= MX - NXH; k += 32) a[swz<C>(k)] = zc;
        for (int kk = lane; kk < NXH; kk += 32) {
            C A_ = qa[kk], B_ = g >= 0 ? qb[kk] : zc;
            if (xd) {
                const T kx = (T)wavx[kk];
                B_ = kct::mk<C>(-kx * A_.y, kx * A_.x);
            }
            if (kk == 0) { A_.y = (T)0; B_.y = (T)0; }   // c2r ignores Im of the mean mode
            a[swz<C>(kk)] = kct::mk<C>(A_.x - B_.y, A_.y + B_.x);
            if (kk > 0) a[swz<C>(MX - kk)] = kct::mk<C>(A_.x + B_.y, -A_.y + B_.x);
        }
        __syncwarp();
        if constexpr (kct::nfac(MX) % 2 == 1) {
            // an odd number of FFT stages: the first writes the pair's rows (as one complex
            // buffer), the second reads them back into a, and the last reads a and writes the
            // two real rows straight into the rows it no longer needs
            T *pf = phys + (size_t)f * MX, *pg = phys + (size_t)(g >= 0 ? g : f) * MX;
            auto ld = [&](int x) { return a[swz<C>(x)]; };
            auto st = [&](int x, C v) {
                pf[x] = v.x;
                if (g >= 0) pg[x] = v.y;
            };
            auto pre = [] {};
            fft_warp_ct_io<C, MX, +1>(ld, st, pre, b, a, tw);
        } else {
            const C *r = fft_warp_ct<C, MX, +1, 1, true>(a, b, tw);
            // the result may sit in the pair's own rows: read it all before writing the real rows
            constexpr int E = (MX + 31) / 32;
            C rv[E];
#pragma unroll
            for (int e = 0; e < E; ++e)
                if (lane + 32 * e < MX) rv[e] = r[swz<C>(lane + 32 * e)];
            __syncwarp();
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int x = lane + 32 * e;
                if (x < MX) {
                    phys[(size_t)f * MX + x] = rv[e].x;
                    if (g >= 0) phys[(size_t)g * MX + x] = rv[e].y;
                }
            }
        }
        __syncwarp();
    }
    if (!__all_sync(0xffffffffu, ok)) {
        // a copy that never completed: record it, give the copies in flight a second bounded wait
        // (shared memory must outlive them) and leave this row
        if (lane == 0) atomicMax(status, KMM_ERR_TIMEOUT);
        for (int pr = warp; pr < npairs; pr += XPW) kasync::mbar_wait(&xbar[pr], 0);
    }
    __syncthreads();
    double cmax = 0.0, umx = 0.0;
    const double sg = seght[y];
    for (int k = threadIdx.x; k < MX; k += blockDim.x) {
        auto in = [&](int sl) { return (double)phys[(size_t)A.slot_of_in[sl] * MX + k]; };
        xphys_point(in, A, sv, y, z, k, nyp, mz, MX, sg, po, drag, up3, vp3, wp3, imatrix, fxi, fyi, fzi, scsource, cmax,
                    umx);
    }
    __shared__ double red[2][XPW];
    for (int off = 16; off; off >>= 1) {
        const double c2 = __shfl_down_sync(0xffffffffu, cmax, off);
        const double u2 = __shfl_down_sync(0xffffffffu, umx, off);
        cmax = (c2 != c2) ? c2 : fmax(cmax, c2);
        umx = fmax(umx, u2);
    }
    if (lane == 0) { red[0][warp] = cmax; red[1][warp] = umx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < XPW; ++w) {
            cmax = (red[0][w] != red[0][w]) ? red[0][w] : fmax(cmax, red[0][w]);
            umx = fmax(umx, red[1][w]);
        }
        atomic_max_pos(&cfl[y], cmax);
        atomic_max_pos(&umax[y], umx);
    }
}

// 5'. r2c along x for the compiled lengths: one block per (y, z) row, warps over output pairs
// (two real rows packed as one complex FFT, split by Hermitian symmetry, modes kx < nxh kept)
template <int MX, typename C>
__global__ void __launch_bounds__(XW * 32) k_xfwd2(const typename kct::Real<C>::T *__restrict__ po, C *__restrict__ q,
                                                   const C *__restrict__ tw, int nout, int nyp, int mz) {
    typedef typename kct::Real<C>::T T;
    constexpr int NXH = MX / 3;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.x, y = blockIdx.y;
    C *a = sm + (size_t)warp * 2 * MX, *b = a + MX;
    const size_t n3 = (size_t)nyp * mz * MX, g3 = ((size_t)y * mz + z) * MX;
    for (int pr = warp; pr < (nout + 1) / 2; pr += XW) {
        const int o = 2 * pr, g = o + 1 < nout ? o + 1 : -1;
        // the FFT's first stage reads the two real rows straight from global memory, its last
        // writes the scratch buffer the stage does not read
        const T *ro = po + (size_t)o * n3 + g3, *rg = po + (size_t)(g >= 0 ? g : o) * n3 + g3;
        auto ld = [&](int x) { return kct::mk<C>(ro[x], g >= 0 ? rg[x] : (T)0); };
        C *r = kct::nfac(MX) % 2 == 0 ? b : a;
        auto st = [&](int x, C v) { r[swz<C>(x)] = v; };
        auto pre = [] {};
        fft_warp_ct_io<C, MX, -1>(ld, st, pre, a, b, tw);
        __syncwarp();
        for (int k = lane; k < NXH; k += 32) {
            const C Z = r[swz<C>(k)];
            C Zc = r[swz<C>(k == 0 ? 0 : MX - k)];
            Zc.y = -Zc.y;
            q[(((size_t)o * nyp + y) * mz + z) * NXH + k] = kct::mk<C>((T)0.5 * (Z.x + Zc.x), (T)0.5 * (Z.y + Zc.y));
            if (g >= 0)   // -i/2 (Z - Zc)
                q[(((size_t)g * nyp + y) * mz + z) * NXH + k] = kct::mk<C>((T)0.5 * (Z.y - Zc.y), (T)-0.5 * (Z.x - Zc.x));
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// 4. 5x5 force spreading with the reference's sequential-loop semantics (solvers.f90:3069-3108):
//    the plane loop runs k (x) outer, j (z) inner and assigns vwx(j,k) before adding its own and
//    its neighbours' spread; a contribution from source q to target t survives only if t was
//    assigned no later than q, i.e. flat(t) <= flat(q) with flat = (j-1) + (k-1)*mz.  Targets
//    are computed in the column-major plane without a j-range check (the reference's test
//    `j .ge. 3 .or. j .le. mz-2` is always true), so j+jj outside 1..mz lands in the next or
//    previous x column; targets outside the plane array are dropped.
// ---------------------------------------------------------------------------
template <typename PO_T>
__global__ void k_spread(PO_T *__restrict__ po, const double *__restrict__ drag, const double *__restrict__ fspread,
                         int nyp, int mz, int mx, int kmaxsurf, int y0, int o1, int o2, int o3) {
    const size_t nplane = (size_t)mz * mx;
    const int y = y0 + blockIdx.y;
    if (y + 1 > kmaxsurf) return;
    const size_t n3 = (size_t)nyp * nplane;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nplane; e += (size_t)gridDim.x * blockDim.x) {
        // target t in reference flat order: t = jt + kt*mz (0-based); consecutive threads take
        // consecutive kt, the contiguous x index of po and drag
        const int jt = (int)(e / mx), kt = (int)(e % mx);
        const long t = (long)jt + (long)kt * mz;
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int ii = -2; ii <= 2; ++ii)
            for (int jj = -2; jj <= 2; ++jj) {
                const long s = t - jj;                 // = jq + X*mz with X = wrap(kq+ii) - 1
                if (s < 0 || s >= (long)nplane) continue;
                const int jq = (int)(s % mz);
                const int X = (int)(s / mz);
                int kq = X - ii;                        // 0-based source column before wrap
                if (kq < 0) kq += mx;
                if (kq >= mx) kq -= mx;
                const long qflat = (long)jq + (long)kq * mz;
                if (qflat < t) continue;                // overwritten by the later assignment of t
                const double sw = fspread[(abs(ii)) * 10 + abs(jj)];
                const size_t gq = ((size_t)y * mz + jq) * mx + kq;
                ax += sw * drag[gq];
                ay += sw * drag[n3 + gq];
                az += sw * drag[2 * n3 + gq];
            }
        const size_t gt = ((size_t)y * mz + jt) * mx + kt;
        if (o1 >= 0) po[(size_t)o1 * n3 + gt] = (PO_T)((double)po[(size_t)o1 * n3 + gt] + ax);
        if (o2 >= 0) po[(size_t)o2 * n3 + gt] = (PO_T)((double)po[(size_t)o2 * n3 + gt] + ay);
        if (o3 >= 0) po[(size_t)o3 * n3 + gt] = (PO_T)((double)po[(size_t)o3 * n3 + gt] + az);
    }
}

// ---------------------------------------------------------------------------
// 5. x: r2c (two real rows per complex FFT), keep kx < nxh
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_xfwd(const double *__restrict__ po, double2 *__restrict__ q, const __grid_constant__ DevPlan P,
                                              int nout, int nyp, int mz, int mx, int nxh) {
    extern __shared__ double2 sm[];
    const int y = blockIdx.y;
    const int z0 = blockIdx.x * XZB;
    const int nzr = min(XZB, mz - z0);
    double2 *fa = sm, *fb = sm + (size_t)XZB * mx;
    const size_t n3 = (size_t)nyp * mz * mx;
    for (int o = 0; o < nout; o += 2) {
        const int g = o + 1 < nout ? o + 1 : -1;
        for (int e = threadIdx.x; e < XZB * mx; e += blockDim.x) {
            const int r = e / mx, k = e - r * mx;
            double2 v = make_double2(0.0, 0.0);
            if (r < nzr) {
                const size_t g3 = ((size_t)y * mz + z0 + r) * mx + k;
                v.x = po[(size_t)o * n3 + g3];
                if (g >= 0) v.y = po[(size_t)g * n3 + g3];
            }
            fa[e] = v;
        }
        __syncthreads();
        double2 *r = fft_smem(P, fa, fb, XZB, mx, -1);
        for (int e = threadIdx.x; e < nzr * nxh; e += blockDim.x) {
            const int rr = e / nxh, k = e - rr * nxh;
            const double2 Z = r[rr * mx + k];
            const double2 Zc = cconj(r[rr * mx + ((mx - k) % mx)]);
            const double2 a = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y + Zc.y));
            const size_t d = (((size_t)o * nyp + y) * mz + z0 + rr) * nxh + k;
            q[d] = a;
            if (g >= 0) {
                const double2 dd = csub(Z, Zc);                 // -i/2 (Z - Zc)
                q[(((size_t)g * nyp + y) * mz + z0 + rr) * nxh + k] = make_double2(0.5 * dd.y, -0.5 * dd.x);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// 6. z: forward c2c, truncate to nz, /(mx*mz)
// ---------------------------------------------------------------------------
// BIG (mz = 576 only): one buffer, each warp's FFT in place, as in k_zfft_bwd
template <typename C, bool BIG = false>
__global__ void __launch_bounds__(256, BIG ? 2 : 4) k_zfft_fwd(const C *__restrict__ q, C *__restrict__ pl, const __grid_constant__ DevPlan P,
                                                  const C *__restrict__ tw, int nyp, int nz, int nxh, int mz,
                                                  double scale) {
    typedef typename kct::Real<C>::T T;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int y = blockIdx.y, f = blockIdx.z;
    const int kx0 = blockIdx.x * ZKB;
    const int nk = min(ZKB, nxh - kx0);
    const int nzh = nz / 2;
    C *a = sm, *b = sm + fb_len(ZKB, mz);
    const bool ct = fb_compiled(mz);
    const C *src = q + (((size_t)f * nyp + y) * mz) * nxh;
    for (int e0 = threadIdx.x; e0 < ZKB * mz; e0 += LDG * 256) {
        C wv[LDG];
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            const int z = e / ZKB, c = e - z * ZKB;
            wv[u] = (e < ZKB * mz && c < nk) ? src[(size_t)z * nxh + kx0 + c] : kct::mk<C>((T)0, (T)0);
        }
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            if (e >= ZKB * mz) break;
            const int z = e / ZKB, c = e - z * ZKB;
            a[fb_at<C, ZKB>(c, z, mz, ct)] = wv[u];
        }
    }
    __syncthreads();
    C *r;
    if constexpr (BIG) {
        const int w = threadIdx.x >> 5;
        if (w < nk) fft_warp_ct_inplace<C, 576, -1>(a + (size_t)w * (576 + FB_PAD), tw);
        __syncthreads();
        r = a;
    } else {
        r = fft_block<C, -1, ZKB>(P, a, b, tw, mz);
    }
    C *dst = pl + (((size_t)f * nyp + y) * nxh + kx0) * nz;
    for (int e = threadIdx.x; e < nk * nz; e += blockDim.x) {
        const int c = e / nz, j = e - c * nz;
        const int jj = (j < nzh) ? j : (mz - nz) + j;
        const C v = r[fb_at<C, ZKB>(c, jj, mz, ct)];
        dst[e] = kct::mk<C>((T)(v.x / scale), (T)(v.y / scale));
    }
}

// ---------------------------------------------------------------------------
// 7. y: DCT-I back to Chebyshev coefficients, /ny, halve the end coefficients
// ---------------------------------------------------------------------------
template <typename C>
__global__ void __launch_bounds__(256) k_dct_bwd(const C *__restrict__ pl, const __grid_constant__ FieldPtrsW out, const __grid_constant__ DevPlan P,
                                                 const C *__restrict__ tw, int nyp, int nz, int nxh, int ncols) {
    typedef typename kct::Real<C>::T T;
    extern __shared__ double2 smd[];
    C *sm = reinterpret_cast<C *>(smd);
    const int ny = nyp - 1, L = 2 * ny;
    const int f = blockIdx.y;
    const int col0 = blockIdx.x * DCT_CB;
    const int ncb = min(DCT_CB, ncols - col0);
    C *a = sm, *b = sm + fb_len(DCT_CB, L);
    const bool ct = fb_compiled(L);
    for (int e = threadIdx.x; e < fb_len(DCT_CB, L); e += blockDim.x) a[e] = kct::mk<C>((T)0, (T)0);
    __syncthreads();
    for (int e0 = threadIdx.x; e0 < ncb * nyp; e0 += LDG * 256) {
        C wv[LDG];
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            if (e < ncb * nyp) {
                const int y = e / ncb, c = e - y * ncb;
                const int col = col0 + c;
                const int kx = col / nz, kz = col - kx * nz;
                wv[u] = pl[(((size_t)f * nyp + y) * nxh + kx) * nz + kz];
            }
        }
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            if (e >= ncb * nyp) break;
            const int y = e / ncb, c = e - y * ncb;
            a[fb_at<C, DCT_CB>(c, y, L, ct)] = wv[u];
            if (y > 0 && y < ny) a[fb_at<C, DCT_CB>(c, L - y, L, ct)] = wv[u];
        }
    }
    __syncthreads();
    C *r = fft_block<C, -1, DCT_CB>(P, a, b, tw, L);
    double2 *dst = out.p[f] + (size_t)col0 * nyp;
    for (int e = threadIdx.x; e < ncb * nyp; e += blockDim.x) {
        const int c = e / nyp, i = e - c * nyp;
        const C rv = r[fb_at<C, DCT_CB>(c, i, L, ct)];
        double2 v = make_double2((double)rv.x / (double)ny, (double)rv.y / (double)ny);
        if (i == 0 || i == ny) v = make_double2(v.x / 2.0, v.y / 2.0);
        dst[e] = v;
    }
}

// k_dct_bwd for ny in {48, 64, 96, 128, 256} with the half-length DCT-I (layout as k_dct_fwd_h)
template <typename C, int N>
__global__ void __launch_bounds__(256) k_dct_bwd_h(const C *__restrict__ pl, const __grid_constant__ FieldPtrsW out, const C *__restrict__ tw,
                                                   int nz, int nxh, int ncols) {
    constexpr int NYP = N + 1;
    extern __shared__ double2 smd[];
    C *xs = reinterpret_cast<C *>(smd);
    C *a = xs + DCT_CB * NYP, *b = a + fb_len(DCT_CB, N);
    const int f = blockIdx.y;
    const int col0 = blockIdx.x * DCT_CB;
    const int ncb = min(DCT_CB, ncols - col0);
    for (int e0 = threadIdx.x; e0 < ncb * NYP; e0 += LDG * 256) {
        C wv[LDG];
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            if (e < ncb * NYP) {
                const int y = e / ncb, cc = e - y * ncb;
                const int col = col0 + cc;
                const int kx = col / nz, kz = col - kx * nz;
                wv[u] = pl[(((size_t)f * NYP + y) * nxh + kx) * nz + kz];
            }
        }
#pragma unroll
        for (int u = 0; u < LDG; ++u) {
            const int e = e0 + 256 * u;
            if (e >= ncb * NYP) break;
            const int y = e / ncb, cc = e - y * ncb;
            xs[cc * NYP + y] = wv[u];
        }
    }
    __syncthreads();
    const int c = threadIdx.x >> 5;
    if (c < ncb) dct1_half<C, N>(xs + c * NYP, a + c * (N + FB_PAD), b + c * (N + FB_PAD), tw);
    __syncthreads();
    double2 *dst = out.p[f] + (size_t)col0 * NYP;
    for (int e = threadIdx.x; e < ncb * NYP; e += blockDim.x) {
        const C rv = xs[e];
        const int i = e % NYP;
        double2 v = make_double2((double)rv.x / (double)N, (double)rv.y / (double)N);
        if (i == 0 || i == N) v = make_double2(v.x / 2.0, v.y / 2.0);
        dst[e] = v;
    }
}

// launch the half-length DCT-I kernels where ny is one of their lengths: KMM_ERR_UNSUPPORTED
// otherwise (the caller then runs k_dct_fwd / k_dct_bwd)
template <typename C>
static int dct_h_fwd(kmm_ctx *ctx, int nf, const FieldPtrs &in, C *pl, const C *tw, int nz, int nxh, int ncols) {
    const int ny = ctx->nyp - 1;
    const size_t nbuf = ny == 256 ? 1 : 2;   // dct1_half's FFT runs in place at ny = 256
    const size_t sm = sizeof(C) * ((size_t)DCT_CB * (ny + 1) + nbuf * (size_t)fb_len(DCT_CB, ny));
    const dim3 grid((ncols + DCT_CB - 1) / DCT_CB, nf);
#define DH(NN)                                                                                            \
    do {                                                                                                  \
        RET(kmm_smem_attr(ctx, (const void *)k_dct_fwd_h<C, NN>, sm));                                    \
        k_dct_fwd_h<C, NN><<<grid, 256, sm, ctx->stream>>>(in, pl, tw, nz, nxh, ncols);                     \
        CKL();                                                                                            \
        return KMM_OK;                                                                                    \
    } while (0)
    switch (ny) {
    case 48: DH(48);
    case 64: DH(64);
    case 96: DH(96);
    case 128: DH(128);
    case 256: DH(256);
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef DH
}

template <typename C>
static int dct_h_bwd(kmm_ctx *ctx, int nf, const C *pl, const FieldPtrsW &out, const C *tw, int nz, int nxh, int ncols) {
    const int ny = ctx->nyp - 1;
    const size_t nbuf = ny == 256 ? 1 : 2;   // dct1_half's FFT runs in place at ny = 256
    const size_t sm = sizeof(C) * ((size_t)DCT_CB * (ny + 1) + nbuf * (size_t)fb_len(DCT_CB, ny));
    const dim3 grid((ncols + DCT_CB - 1) / DCT_CB, nf);
#define DH(NN)                                                                                            \
    do {                                                                                                  \
        RET(kmm_smem_attr(ctx, (const void *)k_dct_bwd_h<C, NN>, sm));                                    \
        k_dct_bwd_h<C, NN><<<grid, 256, sm, ctx->stream>>>(pl, out, tw, nz, nxh, ncols);                    \
        CKL();                                                                                            \
        return KMM_OK;                                                                                    \
    } while (0)
    switch (ny) {
    case 48: DH(48);
    case 64: DH(64);
    case 96: DH(96);
    case 128: DH(128);
    case 256: DH(256);
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef DH
}

// ---------------------------------------------------------------------------
// physical scratch (outputs, drag) sized on demand
// ---------------------------------------------------------------------------
static int ensure_phys(kmm_ctx *ctx, int nout, bool need_drag) {
    size_t n = ctx->nphys * (size_t)nout;
    if (n > ctx->po_n) {
        if (ctx->po) { CK(cudaStreamSynchronize(ctx->stream)); cudaFree(ctx->po); }
        ctx->po = NULL;
        CK(cudaMalloc(&ctx->po, sizeof(double) * n));
        ctx->po_n = n;
    }
    if (need_drag && 3 * ctx->nphys > ctx->drag_n) {
        if (ctx->drag) { CK(cudaStreamSynchronize(ctx->stream)); cudaFree(ctx->drag); }
        ctx->drag = NULL;
        CK(cudaMalloc(&ctx->drag, sizeof(double) * 3 * ctx->nphys));
        ctx->drag_n = 3 * ctx->nphys;
    }
    return KMM_OK;
}

// physical input buffer of the two-pass x stage: nin fields of (nyp, mz, mx) doubles
static int ensure_xbig(kmm_ctx *ctx, int nin) {
    const size_t n = ctx->nphys * (size_t)nin;
    if (n > ctx->xbig_n) {
        if (ctx->xbig) { CK(cudaStreamSynchronize(ctx->stream)); cudaFree(ctx->xbig); }
        ctx->xbig = NULL;
        ctx->xbig_n = 0;
        if (cudaMalloc(&ctx->xbig, sizeof(double) * n) != cudaSuccess) {
            cudaGetLastError();
            kmm_set_error(ctx, "two-pass x stage: cudaMalloc(%zu) failed", sizeof(double) * n);
            return KMM_ERR_NOMEM;
        }
        ctx->xbig_n = n;
    }
    return KMM_OK;
}

__global__ void k_kmaxsurf(const int *__restrict__ im, int *out, int nyp, int mz, int mx) {
    const size_t n = (size_t)nyp * mz * mx;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int t = im[e];
        if (t == 1 || t == 3 || t == 4) atomicMax(out, (int)(e % mx) + 1);   // 1-based x index k
        if (!(t == 0 || t == 1 || t == 3 || t == 4 || t == 11)) atomicOr(out + 1, 1);
        if (t == 1 || t == 3 || t == 4 || t == 11) {   // y-planes that can hold a nonzero drag
            const int y1 = (int)(e / ((size_t)mz * mx)) + 1;
            atomicMin(out + 2, y1);
            atomicMax(out + 3, y1);
        }
    }
}

int kmm_update_kmaxsurf(kmm_ctx *ctx) {
    if (ctx->kmaxsurf >= 0) return KMM_OK;
    int *im = (int *)kmm_field_ptr(ctx, KMM_IMATRIX);
    if (!im) return KMM_ERR_NOMEM;
    int h[4] = {0, 0, 1 << 30, 0};
    int *tmp = NULL;
    CK(cudaMallocAsync((void **)&tmp, 4 * sizeof(int), ctx->stream));
    CK(cudaMemcpyAsync(tmp, h, 4 * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    k_kmaxsurf<<<kmm_blocks(ctx->nphys, 256), 256, 0, ctx->stream>>>(im, tmp, ctx->nyp, ctx->mz, ctx->mx);
    CKL();
    CK(cudaMemcpyAsync(h, tmp, 4 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaFreeAsync(tmp, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h[1]) {
        kmm_set_error(ctx, "imatrix holds a cell type other than 0, 1, 3, 4, 11 (buffer/suction/moving-wall types are not built)");
        return KMM_ERR_UNSUPPORTED;
    }
    ctx->kmaxsurf = h[0];
    ctx->ib_ylo = h[3] > 0 ? h[2] : 0;
    ctx->ib_yhi = h[3];
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// scalar source of the particles (scl_flag = 2, solvers.f90:2079-2118): a Gaussian of widths
// sigmax, sigmay, sigmaz and weight deltaT around every particle, with the reference's cut-offs
// (betax < 20, betax + betaz < 20, betax + betay + betaz < 18) and no periodic images.  One warp
// per particle walks the x and z points that can pass the cut-offs (the range widened by one point
// each side; the reference's tests decide), lanes over y; contributions are added with FP64
// atomics (the reference sums its OpenMP threads' private copies, so its order is not fixed
// either).  Layout [y][z][x].
// ---------------------------------------------------------------------------
__global__ void k_scsource(const double *__restrict__ xp, const double *__restrict__ yp, const double *__restrict__ zp,
                           int npart, const double *__restrict__ ycoord, double *sc, int nyp, int mz, int mx,
                           double delxm, double delzm, double sx, double sy, double sz, double dT) {
    const int n = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (n >= npart) return;
    const int lane = threadIdx.x & 31;
    const double xc = xp[n], yc = yp[n], zc = zp[n];
    const double ax = 2.0 * (sx * sx), ay = 2.0 * (sy * sy), az = 2.0 * (sz * sz);
    const double rx = sqrt(20.0 * ax), rz = sqrt(20.0 * az);
    const int k0 = max(0, (int)floor((xc - rx) / delxm) - 1), k1 = min(mx - 1, (int)ceil((xc + rx) / delxm) + 1);
    const int j0 = max(0, (int)floor((zc - rz) / delzm) - 1), j1 = min(mz - 1, (int)ceil((zc + rz) / delzm) + 1);
    for (int k = k0; k <= k1; ++k) {
        const double dx = (double)k * delxm - xc;
        const double bx = (dx * dx) / ax;
        if (!(bx < 20.0)) continue;
        for (int j = j0; j <= j1; ++j) {
            const double dz = (double)j * delzm - zc;
            const double bz = (dz * dz) / az;
            if (!(bx + bz < 20.0)) continue;
            for (int i = lane; i < nyp; i += 32) {
                const double dy = ycoord[i] - yc;
                const double by = (dy * dy) / ay;
                const double b = bx + by + bz;
                if (b < 18.0) atomicAdd(&sc[((size_t)i * mz + j) * mx + k], dT * exp(-b));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
int kmm_tracers(kmm_ctx *ctx);   // kmm_tracer.cu
int kmm_inertial(kmm_ctx *ctx);  // kmm_tracer.cu
int kmm_fast_x(kmm_ctx *ctx, const double2 *q, double2 *r, int ic, int nout, bool save_uvw, double *up3,
               double *vp3, double *wp3);   // kmm_fast.cu


int kmm_target_source(kmm_ctx *ctx);

extern "C" int kmm_vcw3dp(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mx = ctx->mx, mz = ctx->mz;
    const int ncols = nz * nxh;
    const int it = ctx->it;
    const bool scal = ctx->p.scalar_on != 0;
    const bool poly = ctx->p.polymer_on && (it >= ctx->p.src_start - 1);
    // the immersed-boundary branches run only when an imatrix was uploaded (all-fluid otherwise)
    const bool ib_any = ctx->f[KMM_IMATRIX] != NULL;
    if (ib_any) RET(kmm_update_kmaxsurf(ctx));
    // inertial particles (particle_flag > 0) read the vorticity, gradient and Laplacian on the 3/2 grid
    const bool inertial = ctx->p.particle_flag > 0 && ctx->p.npart > 0;

    // inputs actually consumed by the physics (the reference also transforms u_ij and the
    // Laplacian every step; those only feed output, swirl and the inertial-particle path)
    PhysArgs A;
    memset(&A, 0, sizeof(A));
    for (int s = 0; s < S_NSLOT; ++s) A.slot_of_in[s] = -1;
    for (int o = 0; o < O_NSLOT; ++o) A.slot_of_out[o] = -1;
    FieldPtrs in;       // the fields that are y-transformed (the planes the z inverse reads)
    FieldPtrsW outp;
    ZRecipe zr;         // for each input slot's z-inverse output: its plane and multiplier
    int nin = 0, nout = 0, nbase = 0;
    // Inside a routine step without inertial particles the x and z derivatives among the inputs
    // (the velocity gradient's i kx / i kz columns, the scalar's, the conformation tensor's) are
    // formed in the z inverse from their field's plane, and the symmetric tensor's duplicate
    // components share one plane: 23 y transforms instead of 55 with polymer and scalar.  The
    // step computes only the y derivatives for it (kmm_step).
    const bool derived = kmm_derived_inputs(ctx) && ctx->in_step;
    auto add_base = [&](int fid) -> int {
        const double2 *p = SPEC(ctx, fid);
        if (!p) return -1;
        for (int b = 0; b < nbase; ++b)
            if (in.p[b] == p) return b;
        if (nbase >= MAXIO) return -1;
        in.p[nbase] = p;
        return nbase++;
    };
    auto add_in_from = [&](int slot, int base_fid, int mult) -> int {
        const int b = add_base(base_fid);
        if (b < 0) return KMM_ERR_NOMEM;
        if (nin >= MAXIO) return KMM_ERR_UNSUPPORTED;
        A.slot_of_in[slot] = nin;
        zr.base[nin] = (unsigned char)b;
        zr.mult[nin] = (unsigned char)mult;
        ++nin;
        return KMM_OK;
    };
    auto add_in = [&](int slot, int fid) -> int { return add_in_from(slot, fid, 0); };
    auto add_out = [&](int slot, int fid) -> int {
        double2 *p = SPEC(ctx, fid);
        if (!p) return KMM_ERR_NOMEM;
        if (nout >= MAXIO) return KMM_ERR_UNSUPPORTED;
        A.slot_of_out[slot] = nout;
        outp.p[nout++] = p;
        return KMM_OK;
    };
    static const int fl[6] = {KMM_U, KMM_V, KMM_W, KMM_OMX, KMM_OMY, KMM_OMZ};
    for (int m = 0; m < 6; ++m) RET(add_in(S_U + m, fl[m]));
    if (scal) {
        RET(add_in(S_SC, KMM_SCALAR));
        if (derived) {
            RET(add_in_from(S_CX, KMM_SCALAR, 1));
            RET(add_in(S_CY, KMM_SCLY));
            RET(add_in_from(S_CZ, KMM_SCALAR, 2));
        } else {
            RET(add_in(S_CX, KMM_SCLX));
            RET(add_in(S_CY, KMM_SCLY));
            RET(add_in(S_CZ, KMM_SCLZ));
        }
    }
    static const int gu[9] = {KMM_U11, KMM_U12, KMM_U13, KMM_U21, KMM_U22, KMM_U23, KMM_U31, KMM_U32, KMM_U33};
    if (poly || inertial)
        for (int m = 0; m < 9; ++m) {
            // u_ij = d u_i / d x_j: j = x, z from u_i itself, j = y the cderiv field
            const int comp = m / 3, dir = m % 3;
            if (derived && dir != 1) RET(add_in_from(S_U11 + m, KMM_U + comp, dir == 0 ? 1 : 2));
            else RET(add_in(S_U11 + m, gu[m]));
        }
    if (inertial)
        for (int m = 0; m < 3; ++m) RET(add_in(S_LU + m, KMM_LU + m));
    if (poly) {
        // c_ij and dc_ijk = d c_ij / d x_k; c21 = c12, c31 = c13, c32 = c23 (copied by the step)
        static const int uniq[9] = {0, 1, 2, 1, 4, 5, 2, 5, 8};
        for (int m = 0; m < 9; ++m) RET(add_in(S_C11 + m, KMM_C11 + (derived ? uniq[m] : m)));
        for (int m = 0; m < 27; ++m) {
            const int ij = m / 3, k = m % 3;
            if (!derived) RET(add_in(S_DC111 + m, KMM_DC111 + m));
            else if (k == 1) RET(add_in(S_DC111 + m, KMM_DC111 + 3 * uniq[ij] + 1));
            else RET(add_in_from(S_DC111 + m, KMM_C11 + uniq[ij], k == 0 ? 1 : 2));
        }
    }
    RET(add_out(O_H1, KMM_GN));
    RET(add_out(O_H2, KMM_FN));
    // h3 is written into omz, an input: stage it in the output plane buffer and write it last
    RET(add_out(O_H3, KMM_OMZ));
    if (scal) RET(add_out(O_SC, KMM_SCN));
    if (poly) {
        for (int m = 0; m < 6; ++m) RET(add_out(O_C11N + m, KMM_C11N + m));
        for (int m = 0; m < 6; ++m) RET(add_out(O_STR11N + m, KMM_STR11N + m));
        static const int qq[6] = {KMM_QP11, KMM_QP12, KMM_QP13, KMM_QP22, KMM_QP23, KMM_QP33};
        for (int m = 0; m < 6; ++m) RET(add_out(O_QP11 + m, qq[m]));
    }
    // x derivatives formed in the x stage (with polymer, derived inputs and a compiled x stage:
    // k_xphys2 or the two-pass k_xinv_big2): every input i kx f whose f is also an input moves
    // right after it, an odd place, and the x stage builds their pair from the one row of f; the
    // z inverse produces the other nq inputs only
    bool xform[MAXIO];
    for (int i = 0; i < MAXIO; ++i) xform[i] = false;
    const bool x_compiled = ((mx == 48 || mx == 96 || mx == 144 || mx == 192) &&
                             !(ctx->force_xbig && ctx->p.precision == 0)) ||
                            mx == 576;
    if (derived && poly && x_compiled) {
        int slot_at[MAXIO];
        for (int i = 0; i < nin; ++i) slot_at[i] = -1;
        for (int sl = 0; sl < S_NSLOT; ++sl)
            if (A.slot_of_in[sl] >= 0) slot_at[A.slot_of_in[sl]] = sl;
        int order[MAXIO], no = 0;
        bool used[MAXIO], odd_x[MAXIO];
        for (int i = 0; i < nin; ++i) used[i] = odd_x[i] = false;
        for (int d = 0; d < nin; ++d) {
            if (zr.mult[d] != 1) continue;
            int f = -1;
            for (int c = 0; c < nin && f < 0; ++c)
                if (!used[c] && zr.mult[c] == 0 && zr.base[c] == zr.base[d]) f = c;
            if (f < 0) continue;
            used[f] = used[d] = true;
            order[no++] = f;
            odd_x[no] = true;
            order[no++] = d;
        }
        for (int c = 0; c < nin; ++c)
            if (!used[c]) order[no++] = c;
        ZRecipe z2;
        for (int pos = 0; pos < nin; ++pos) {
            const int old = order[pos];
            z2.base[pos] = zr.base[old];
            z2.mult[pos] = zr.mult[old];
            if (slot_at[old] >= 0) A.slot_of_in[slot_at[old]] = pos;
            xform[pos] = odd_x[pos];
        }
        zr = z2;
    }
    // the z inverse's outputs (the inputs not formed in the x stage, compacted) and the x stage's rows
    int nq = 0;
    unsigned char qidx[MAXIO];
    ZRecipe zq;
    for (int i = 0; i < nin; ++i) {
        if (xform[i]) continue;
        qidx[i] = (unsigned char)nq;
        zq.base[nq] = zr.base[i];
        zq.mult[nq] = zr.mult[i];
        ++nq;
    }
    XRecipe xr;
    for (int pr = 0; pr < (nin + 1) / 2; ++pr) {
        const int f = 2 * pr, g = f + 1;
        xr.qa[pr] = qidx[f];
        xr.xd[pr] = (unsigned char)(g < nin && xform[g]);
        xr.qb[pr] = g >= nin ? (unsigned char)255 : (xform[g] ? qidx[f] : qidx[g]);
    }
    A.nin = nin;
    A.nout = nout;
    A.scalar = scal;
    A.polymer = poly;
    A.ipeter = ctx->p.ipeter;
    A.itarget = ctx->p.itarget;
    A.scl_flag = ctx->p.scl_flag;
    A.flow_select = ctx->p.flow_select;
    A.it = it;
    A.perturbtime = ctx->p.perturbtime;
    A.save_uvw = 1;
    A.ib_any = ib_any;
    A.delxm = ctx->xl / (double)mx;
    A.delzm = ctx->zl / (double)mz;
    A.dt = ctx->dt;
    A.dPdx = ctx->dPdx;
    A.gain = ctx->gain;
    A.ugain = ctx->ugain;
    A.zl2 = ctx->p.zlmax * ctx->p.zlmax;
    A.qbeta = ctx->p.qbeta;
    A.alpha_poly = ctx->p.alpha_poly;
    A.re = ctx->re;
    A.tpoly = ctx->p.tpoly;
    A.scalar_q = ctx->p.scalar_q;

    RET(kmm_ensure_plane_buffers(ctx, nin, nout));
    RET(ensure_phys(ctx, nout, ib_any));
    double *up3 = REAL(ctx, KMM_UP3D), *vp3 = REAL(ctx, KMM_VP3D), *wp3 = REAL(ctx, KMM_WP3D);
    Save3D sv;
    for (int m = 0; m < 15; ++m) {
        sv.p[m] = inertial ? REAL(ctx, KMM_WX3D + m) : NULL;
        if (inertial && !sv.p[m]) return KMM_ERR_NOMEM;
    }
    double *fxi = NULL, *fyi = NULL, *fzi = NULL;
    int *im = NULL;
    if (ib_any) {
        fxi = REAL(ctx, KMM_FXINTG); fyi = REAL(ctx, KMM_FYINTG); fzi = REAL(ctx, KMM_FZINTG);
        im = (int *)kmm_field_ptr(ctx, KMM_IMATRIX);
    }
    if (scal && ctx->p.scl_flag >= 2) {
        // the source array holds only this call's source: the particle Gaussians (scl_flag = 2) or
        // the targeted source (4, 5) inside src_start..src_stop, zero otherwise (solvers.f90:2076-2210)
        ctx->scsource = REAL(ctx, KMM_SCSOURCE);   // the field's storage (freed with the fields)
        if (!ctx->scsource) return KMM_ERR_NOMEM;
        CK(cudaMemsetAsync(ctx->scsource, 0, sizeof(double) * ctx->nphys, ctx->stream));
        const int np = ctx->p.npart;
        const bool window = it >= ctx->p.src_start && it <= ctx->p.src_stop;
        if ((ctx->p.scl_flag == 4 || ctx->p.scl_flag == 5) && window) RET(kmm_target_source(ctx));
        if (ctx->p.scl_flag == 2 && np > 0 && window) {
            const double *xp = REAL(ctx, KMM_XPART), *yp = REAL(ctx, KMM_YPART), *zp = REAL(ctx, KMM_ZPART);
            if (!xp || !yp || !zp) return KMM_ERR_NOMEM;
            k_scsource<<<(np + 7) / 8, 256, 0, ctx->stream>>>(xp, yp, zp, np, ctx->d_ycoord, ctx->scsource, nyp, mz,
                                                              mx, ctx->xl / (double)mx, ctx->zl / (double)mz,
                                                              ctx->p.sigmax, ctx->p.sigmay, ctx->p.sigmaz,
                                                              ctx->p.deltat);
            CKL();
        }
    }

    const size_t sm_dct = sizeof(double2) * 2 * (size_t)fb_len(DCT_CB, 2 * ctx->ny);
    const size_t sm_z = sizeof(double2) * 2 * (size_t)fb_len(ZKB, mz);
    const size_t sm_x = sizeof(double) * (size_t)nin * XZB * mx + sizeof(double2) * 2 * XZB * mx;
    const size_t sm_xf = sizeof(double2) * 2 * XZB * mx;
    RET(kmm_smem_attr(ctx, (const void *)k_dct_fwd<double2>, sm_dct));
    RET(kmm_smem_attr(ctx, (const void *)k_dct_bwd<double2>, sm_dct));
    RET(kmm_smem_attr(ctx, (const void *)k_zfft_bwd<double2>, sm_z));
    RET(kmm_smem_attr(ctx, (const void *)k_zfft_fwd<double2>, sm_z));
    RET(kmm_smem_attr(ctx, (const void *)k_dct_fwd<float2>, sm_dct));
    RET(kmm_smem_attr(ctx, (const void *)k_dct_bwd<float2>, sm_dct));
    RET(kmm_smem_attr(ctx, (const void *)k_zfft_bwd<float2>, sm_z));
    RET(kmm_smem_attr(ctx, (const void *)k_zfft_fwd<float2>, sm_z));
    // mz = 576: the one-buffer forms (in-place warp FFTs, two blocks per SM)
    const bool zbig = mz == 576;
    const size_t sm_zb = sizeof(double2) * (size_t)fb_len(ZKB, mz);
    if (zbig) {
        RET(kmm_smem_attr(ctx, (const void *)k_zfft_bwd<double2, true>, sm_zb));
        RET(kmm_smem_attr(ctx, (const void *)k_zfft_fwd<double2, true>, sm_zb));
        RET(kmm_smem_attr(ctx, (const void *)k_zfft_bwd<float2, true>, sm_zb));
        RET(kmm_smem_attr(ctx, (const void *)k_zfft_fwd<float2, true>, sm_zb));
    }
    // rows of every input field in shared memory (k_xphys) unless that exceeds the 227 KB limit:
    // then the two-pass x stage through an HBM buffer of the physical inputs (k_xinv_big, k_xpoint)
    // (always at mx = 576, whose compiled transforms serve the two-pass form in both precisions)
    const bool mx_compiled = mx == 48 || mx == 96 || mx == 144 || mx == 192;
    const bool xbig = (!mx_compiled && (sm_x + 1024 > 227 * 1024 || mx == 576)) ||
                      (ctx->force_xbig && ctx->p.precision == 0);
    if (xbig) {
        RET(ensure_xbig(ctx, nin));
        RET(kmm_smem_attr(ctx, (const void *)k_xinv_big, sm_xf));
    } else {
        RET(kmm_smem_attr(ctx, (const void *)k_xphys, sm_x));
    }
    RET(kmm_smem_attr(ctx, (const void *)k_xfwd, sm_xf));
    CK(cudaMemsetAsync(ctx->d_cfl, 0, sizeof(double) * nyp, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_umax, 0, sizeof(double) * nyp, ctx->stream));

    // the mixed form (FP32 transforms and plane intermediates, pointwise terms evaluated in FP64 from
    // the FP32 values, FP64 state) inside kmm_step; FP64 elsewhere (initial, diagnostics)
    const bool f32 = ctx->p.precision == 1 && ctx->in_step;
    const float2 *tw_y2 = NULL, *tw_mz = NULL, *tw_mx = NULL;
    if (f32) RET(kmm_routine_tw32(ctx, &tw_y2, &tw_mz, &tw_mx));
    float2 *pl_in32 = (float2 *)ctx->pl_in, *q_in32 = (float2 *)ctx->q_in;
    float2 *pl_out32 = (float2 *)ctx->pl_out, *q_out32 = (float2 *)ctx->q_out;
    float *po32 = (float *)ctx->po;
    kmm_tic(ctx);
    // the tensor-core y transforms of the mixed form (KMM_OPT_TC_DCT); their status word is read
    // back with the CFL numbers
    const bool tcd = f32 && ctx->use_tcdct;
    if (tcd) CK(cudaMemsetAsync(ctx->d_tcstat, 0, sizeof(int), ctx->stream));
    int tcf = KMM_ERR_UNSUPPORTED;
    if (tcd) {
        const void *pin[MAXIO];
        void *pout[MAXIO];
        for (int m = 0; m < nbase; ++m) {
            pin[m] = in.p[m];
            pout[m] = pl_in32 + (size_t)m * ctx->nspec;
        }
        tcf = kmm_tc_dct(ctx, 0, pin, pout, nbase);
        if (tcf != KMM_OK && tcf != KMM_ERR_UNSUPPORTED) return tcf;
    }
    if (tcf != KMM_OK) {
        const int dst = f32 ? dct_h_fwd<float2>(ctx, nbase, in, pl_in32, tw_y2, nz, nxh, ncols)
                            : dct_h_fwd<double2>(ctx, nbase, in, ctx->pl_in, ctx->py2.tw, nz, nxh, ncols);
        if (dst != KMM_ERR_UNSUPPORTED) {
            RET(dst);
        } else {
            if (f32)
                k_dct_fwd<float2><<<dim3((ncols + DCT_CB - 1) / DCT_CB, nbase), 256, sm_dct, ctx->stream>>>(
                    in, pl_in32, ctx->py2, tw_y2, nyp, nz, nxh, ncols);
            else
                k_dct_fwd<double2><<<dim3((ncols + DCT_CB - 1) / DCT_CB, nbase), 256, sm_dct, ctx->stream>>>(
                    in, ctx->pl_in, ctx->py2, ctx->py2.tw, nyp, nz, nxh, ncols);
            CKL();
        }
    }
    kmm_toc(ctx, KMM_STAGE_DCT_FWD);
    kmm_tic(ctx);
    {
        const dim3 gz((nxh + ZKB - 1) / ZKB, nyp, nq);
        if (f32 && zbig)
            k_zfft_bwd<float2, true><<<gz, 256, sm_zb, ctx->stream>>>(pl_in32, q_in32, ctx->pmz, tw_mz, nyp, nz, nxh, mz,
                                                                      zq, ctx->d_wavx, ctx->d_wavz);
        else if (f32)
            k_zfft_bwd<float2><<<gz, 256, sm_z, ctx->stream>>>(pl_in32, q_in32, ctx->pmz, tw_mz, nyp, nz, nxh, mz, zq,
                                                              ctx->d_wavx, ctx->d_wavz);
        else if (zbig)
            k_zfft_bwd<double2, true><<<gz, 256, sm_zb, ctx->stream>>>(ctx->pl_in, ctx->q_in, ctx->pmz, ctx->pmz.tw, nyp,
                                                                       nz, nxh, mz, zq, ctx->d_wavx, ctx->d_wavz);
        else
            k_zfft_bwd<double2><<<gz, 256, sm_z, ctx->stream>>>(ctx->pl_in, ctx->q_in, ctx->pmz, ctx->pmz.tw, nyp, nz,
                                                               nxh, mz, zq, ctx->d_wavx, ctx->d_wavz);
    }
    CKL();
    kmm_toc(ctx, KMM_STAGE_ZFFT_BWD);
    bool fast_done = false, xstat = false;
    const bool sc_source = scal && ctx->p.scl_flag >= 2;
    if (!poly && !ib_any && !inertial && !sc_source && !f32) {
        // fused warp-per-row x stage (no polymer, no immersed boundary, no inertial particles, no
        // particle scalar source)
        kmm_tic(ctx);
        const bool save = ctx->p.npart > 0 || !ctx->in_step;
        const int fst = kmm_fast_x(ctx, ctx->q_in, ctx->q_out, scal ? A.slot_of_in[S_CX] : -1, nout, save, up3, vp3, wp3);
        if (fst == KMM_OK) fast_done = true;
        else if (fst != KMM_ERR_UNSUPPORTED) return fst;
        kmm_toc(ctx, KMM_STAGE_XPHYS);
    }
    if (!fast_done) {
        kmm_tic(ctx);
        // status of the x stage's bulk copies (KMM_ERR_TIMEOUT), read back with the CFL numbers
        CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
        const size_t eb = f32 ? sizeof(float) : sizeof(double);   // bytes per real of the intermediates
        const size_t xpw = f32 ? XpW<float2>::n : XpW<double2>::n;
        const size_t sm_x2 = eb * (size_t)(nin + (nin & 1)) * mx + 2 * eb * xpw * (size_t)mx;
#define XP2(MM, CC, QQ, PO, TW)                                                                                  \
    do {                                                                                                         \
        RET(kmm_smem_attr(ctx, (const void *)k_xphys2<MM, CC>, sm_x2));                                          \
        k_xphys2<MM, CC><<<dim3(mz, nyp), XpW<CC>::n * 32, sm_x2, ctx->stream>>>(                                         \
            QQ, PO, ctx->drag, up3, vp3, wp3, im, fxi, fyi, fzi, ctx->scsource, ctx->d_seght, ctx->d_cfl,          \
            ctx->d_umax, TW, A, sv, nyp, mz, ctx->d_status, xr, ctx->d_wavx);                                   \
    } while (0)
#define XP2S(MM)                                                                                                 \
    do {                                                                                                         \
        if (f32) XP2(MM, float2, q_in32, po32, tw_mx);                                                           \
        else XP2(MM, double2, ctx->q_in, ctx->po, ctx->wmx.tw);                                                  \
    } while (0)
        switch (xbig ? 0 : mx) {
        case 48: XP2S(48); break;
        case 96: XP2S(96); break;
        case 144: XP2S(144); break;
        case 192: XP2S(192); break;
        default:
            if (!xbig) {
                k_xphys<<<dim3((mz + XZB - 1) / XZB, nyp), 256, sm_x, ctx->stream>>>(
                    ctx->q_in, ctx->po, ctx->drag, up3, vp3, wp3, im, fxi, fyi, fzi, ctx->scsource, ctx->d_seght,
                    ctx->d_cfl, ctx->d_umax, ctx->pmx, A, sv, nyp, mz, mx, nxh);
            } else {
                const dim3 g1((mz + XBW - 1) / XBW, nyp, (nin + 1) / 2);
                const size_t sm_b2 = 2 * eb * (f32 ? 2 : 1) * XBW * (size_t)mx;   // complex rows per warp
                if (mx == 576 && f32) {
                    RET(kmm_smem_attr(ctx, (const void *)k_xinv_big2<576, float2>, sm_b2));
                    k_xinv_big2<576, float2><<<g1, XBW * 32, sm_b2, ctx->stream>>>(q_in32, (float *)ctx->xbig, tw_mx,
                                                                                    nin, nyp, mz, xr, ctx->d_wavx);
                } else if (mx == 576) {
                    RET(kmm_smem_attr(ctx, (const void *)k_xinv_big2<576, double2>, sm_b2));
                    k_xinv_big2<576, double2><<<g1, XBW * 32, sm_b2, ctx->stream>>>(ctx->q_in, ctx->xbig, ctx->wmx.tw,
                                                                                     nin, nyp, mz, xr, ctx->d_wavx);
                } else {
                    k_xinv_big<<<dim3((mz + XZB - 1) / XZB, nyp, (nin + 1) / 2), 256, sm_xf, ctx->stream>>>(
                        ctx->q_in, ctx->xbig, ctx->pmx, nin, nyp, mz, mx, nxh);
                }
                CKL();
                const int bpp = (int)(((size_t)mz * mx + 255) / 256);
                if (f32)
                    k_xpoint<float><<<dim3(bpp < 64 ? bpp : 64, nyp), 256, 0, ctx->stream>>>(
                        (const float *)ctx->xbig, po32, ctx->drag, up3, vp3, wp3, im, fxi, fyi, fzi, ctx->scsource,
                        ctx->d_seght, ctx->d_cfl, ctx->d_umax, A, sv, nyp, mz, mx);
                else
                    k_xpoint<double><<<dim3(bpp < 64 ? bpp : 64, nyp), 256, 0, ctx->stream>>>(
                        ctx->xbig, ctx->po, ctx->drag, up3, vp3, wp3, im, fxi, fyi, fzi, ctx->scsource, ctx->d_seght,
                        ctx->d_cfl, ctx->d_umax, A, sv, nyp, mz, mx);
            }
            break;
        }
#undef XP2S
#undef XP2
        CKL();
        CK(cudaMemcpyAsync(kmm_h_pin_status(ctx), ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        xstat = true;
        if (ib_any && ctx->kmaxsurf > 0) {
            // the reference spreads in the planes i <= kmaxsurf (an x extent, main_dns.f90:1526-1535);
            // ib_spread_all (no counterpart in the reference) spreads in every plane
            const int ksp = (ctx->p.ib_spread_all || ctx->kmaxsurf >= nyp) ? nyp : ctx->kmaxsurf;
            // planes without a solid cell carry zero drag and add nothing: only the planes
            // ib_ylo .. min(ib_yhi, ksp) (1-based) are swept
            const int y0 = ctx->ib_ylo > 0 ? ctx->ib_ylo - 1 : 0, y1 = ctx->ib_yhi < ksp ? ctx->ib_yhi : ksp;
            if (ctx->ib_ylo > 0 && y1 > y0) {
                const dim3 gs(kmm_blocks((size_t)mz * mx, 256) > 64 ? 64 : kmm_blocks((size_t)mz * mx, 256), y1 - y0);
                if (f32)
                    k_spread<float><<<gs, 256, 0, ctx->stream>>>(po32, ctx->drag, ctx->d_fspread, nyp, mz, mx, ksp, y0,
                                                                 A.slot_of_out[O_H1], A.slot_of_out[O_H2],
                                                                 A.slot_of_out[O_H3]);
                else
                    k_spread<double><<<gs, 256, 0, ctx->stream>>>(ctx->po, ctx->drag, ctx->d_fspread, nyp, mz, mx,
                                                                  ksp, y0, A.slot_of_out[O_H1], A.slot_of_out[O_H2],
                                                                  A.slot_of_out[O_H3]);
                CKL();
            }
        }
        kmm_toc(ctx, KMM_STAGE_XPHYS);   // the spreading counts with the pointwise stage
        kmm_tic(ctx);
        const size_t sm_xf2 = 2 * eb * 2 * XW * (size_t)mx;
#define XF2(MM, CC, PO, QQ, TW)                                                                                 \
    do {                                                                                                        \
        RET(kmm_smem_attr(ctx, (const void *)k_xfwd2<MM, CC>, sm_xf2));                                         \
        k_xfwd2<MM, CC><<<dim3(mz, nyp), XW * 32, sm_xf2, ctx->stream>>>(PO, QQ, TW, nout, nyp, mz);             \
    } while (0)
#define XF2S(MM)                                                                                                \
    do {                                                                                                        \
        if (f32) XF2(MM, float2, po32, q_out32, tw_mx);                                                         \
        else XF2(MM, double2, ctx->po, ctx->q_out, ctx->wmx.tw);                                                \
    } while (0)
        switch (mx) {
        case 48: XF2S(48); break;
        case 96: XF2S(96); break;
        case 144: XF2S(144); break;
        case 192: XF2S(192); break;
        case 576: XF2S(576); break;
        default:
            k_xfwd<<<dim3((mz + XZB - 1) / XZB, nyp), 256, sm_xf, ctx->stream>>>(ctx->po, ctx->q_out, ctx->pmx, nout, nyp,
                                                                                 mz, mx, nxh);
            break;
        }
#undef XF2S
#undef XF2
        CKL();
        kmm_toc(ctx, KMM_STAGE_XFWD);
    }
    kmm_tic(ctx);
    {
        const dim3 gz((nxh + ZKB - 1) / ZKB, nyp, nout);
        const double zs = (double)mx * (double)mz;
        if (f32 && zbig)
            k_zfft_fwd<float2, true><<<gz, 256, sm_zb, ctx->stream>>>(q_out32, pl_out32, ctx->pmz, tw_mz, nyp, nz, nxh,
                                                                      mz, zs);
        else if (f32)
            k_zfft_fwd<float2><<<gz, 256, sm_z, ctx->stream>>>(q_out32, pl_out32, ctx->pmz, tw_mz, nyp, nz, nxh, mz, zs);
        else if (zbig)
            k_zfft_fwd<double2, true><<<gz, 256, sm_zb, ctx->stream>>>(ctx->q_out, ctx->pl_out, ctx->pmz, ctx->pmz.tw,
                                                                       nyp, nz, nxh, mz, zs);
        else
            k_zfft_fwd<double2><<<gz, 256, sm_z, ctx->stream>>>(ctx->q_out, ctx->pl_out, ctx->pmz, ctx->pmz.tw, nyp, nz,
                                                               nxh, mz, zs);
    }
    CKL();
    kmm_toc(ctx, KMM_STAGE_ZFFT_FWD);
    kmm_tic(ctx);
    int tcb = KMM_ERR_UNSUPPORTED;
    if (tcd) {
        const void *pin[MAXIO];
        void *pout[MAXIO];
        for (int m = 0; m < nout; ++m) {
            pin[m] = pl_out32 + (size_t)m * ctx->nspec;
            pout[m] = outp.p[m];
        }
        tcb = kmm_tc_dct(ctx, 1, pin, pout, nout);
        if (tcb != KMM_OK && tcb != KMM_ERR_UNSUPPORTED) return tcb;
        CK(cudaMemcpyAsync(kmm_h_pin_tcstat(ctx), ctx->d_tcstat, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (tcb != KMM_OK) {
        const int dst = f32 ? dct_h_bwd<float2>(ctx, nout, pl_out32, outp, tw_y2, nz, nxh, ncols)
                            : dct_h_bwd<double2>(ctx, nout, ctx->pl_out, outp, ctx->py2.tw, nz, nxh, ncols);
        if (dst != KMM_ERR_UNSUPPORTED) {
            RET(dst);
        } else {
            if (f32)
                k_dct_bwd<float2><<<dim3((ncols + DCT_CB - 1) / DCT_CB, nout), 256, sm_dct, ctx->stream>>>(
                    pl_out32, outp, ctx->py2, tw_y2, nyp, nz, nxh, ncols);
            else
                k_dct_bwd<double2><<<dim3((ncols + DCT_CB - 1) / DCT_CB, nout), 256, sm_dct, ctx->stream>>>(
                    ctx->pl_out, outp, ctx->py2, ctx->py2.tw, nyp, nz, nxh, ncols);
            CKL();
        }
    }
    kmm_toc(ctx, KMM_STAGE_DCT_BWD);

    // tracers (solvers.f90:3463-3476)
    int st = KMM_OK;
    if (ctx->p.npart > 0) {
        st = inertial ? kmm_inertial(ctx) : kmm_tracers(ctx);
        if (st != KMM_OK && st != KMM_ERR_INTERP && st != KMM_ERR_PCFL) return st;
    }
    // CFL check (solvers.f90:3497-3514)
    double h_cfl[KMM_MAX_NYP], h_um[KMM_MAX_NYP];
    CK(cudaMemcpyAsync(h_cfl, ctx->d_cfl, sizeof(double) * nyp, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(h_um, ctx->d_umax, sizeof(double) * nyp, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double cflmax = 0.0, umax = 0.0;
    bool nan = false;
    for (int i = 0; i < nyp; ++i) {
        if (h_cfl[i] != h_cfl[i]) nan = true;
        else if (h_cfl[i] > cflmax) cflmax = h_cfl[i];
        if (h_um[i] > umax) umax = h_um[i];
    }
    ctx->stats.cflmax = nan ? NAN : cflmax;
    ctx->stats.umax = umax;
    if (xstat && *kmm_h_pin_status(ctx) == KMM_ERR_TIMEOUT) {
        kmm_set_error(ctx, "x stage: a bulk copy of the input rows did not complete");
        st = KMM_ERR_TIMEOUT;
    }
    if (tcd && *kmm_h_pin_tcstat(ctx) == KMM_ERR_TIMEOUT) {
        kmm_set_error(ctx, "tensor-core y transform: an MMA completion wait ran out");
        st = KMM_ERR_TIMEOUT;
    }
    if (st == KMM_OK && nan) st = KMM_ERR_NAN;
    if (st == KMM_OK && cflmax > 1.0) st = KMM_ERR_CFL;
    ctx->stats.status = st;
    return st;
}

// ---------------------------------------------------------------------------
// calcswirl (helpers.f90:197-404, called at solvers.f90:3421): swirl strength on the 3/2 grid
// from the nine velocity gradients
// ---------------------------------------------------------------------------
// principal powers z^(1/2), z^(1/3) as exp(p log z) = |z|^p e^(i p arg z), with CUDA's sqrt, cbrt,
// hypot, atan2 and sincos
__device__ __forceinline__ double2 cpow_half(double2 z) {
    const double r = hypot(z.x, z.y), th = atan2(z.y, z.x);
    double s, c;
    sincos(0.5 * th, &s, &c);
    const double m = sqrt(r);
    return make_double2(m * c, m * s);
}
__device__ __forceinline__ double2 cpow_third(double2 z) {
    const double r = hypot(z.x, z.y), th = atan2(z.y, z.x);
    double s, c;
    sincos(th / 3.0, &s, &c);
    const double m = cbrt(r);
    return make_double2(m * c, m * s);
}

// eig (helpers.f90:197-275) in Cardano's closed form for real gradients: tr = trace,
// P = (tr^2 - 3 M2)/9 (M2: sum of principal 2x2 minors), Q = tr^3/27 - tr M2/6 + det/2,
// S = (Q + (Q^2 - P^3)^(1/2))^(1/3); l1 = tr/3 + P/S + S, l2,3 = tr/3 -+ sqrt(3)(P/S - S) i/2 -
// P/(2S) - S/2.  P, Q and Q^2 - P^3 are real for real gradients, so only the powers and the
// divisions by S are complex.  swirl = sqrt(sum Im(l)^2), 0 where not finite and positive.
__device__ __forceinline__ double swirl_point(double u11, double u12, double u13, double u21, double u22, double u23,
                                              double u31, double u32, double u33) {
    const double tr = u11 + u22 + u33;
    const double P = tr * tr / 9.0 - (u11 * u22) / 3.0 + (u12 * u21) / 3.0 - (u11 * u33) / 3.0 + (u13 * u31) / 3.0 -
                     (u22 * u33) / 3.0 + (u23 * u32) / 3.0;
    const double M2 = u11 * u22 - u12 * u21 + u11 * u33 - u13 * u31 + u22 * u33 - u23 * u32;
    const double Q = tr * tr * tr / 27.0 - (tr * M2) / 6.0 + (u11 * u22 * u33) / 2.0 - (u11 * u23 * u32) / 2.0 -
                     (u12 * u21 * u33) / 2.0 + (u12 * u23 * u31) / 2.0 + (u13 * u21 * u32) / 2.0 -
                     (u13 * u22 * u31) / 2.0;
    const double2 sq = cpow_half(make_double2(Q * Q - P * P * P, 0.0));
    const double2 S = cpow_third(make_double2(Q + sq.x, sq.y));
    const double2 PS = cdiv(make_double2(P, 0.0), S);
    const double2 D = csub(PS, S);
    // Im of each eigenvalue: l1 = tr/3 + P/S + S; l2,3 = tr/3 -+ (sqrt(3)/2) i D - P/(2S) - S/2
    const double im1 = PS.y + S.y;
    const double rot_im = sqrt(3.0) * D.x / 2.0;   // Im(sqrt(3) D i / 2)
    const double im2 = -rot_im - PS.y / 2.0 - S.y / 2.0;
    const double im3 = rot_im - PS.y / 2.0 - S.y / 2.0;
    double sw = sqrt(im1 * im1 + im2 * im2 + im3 * im3);
    if (!(sw > 0.0 && sw <= 1.7976931348623157e308)) sw = 0.0;
    return sw;
}

#define SW_WARPS 4
// one warp per (y, z) row: Hermitian c2r of the nine gradients (two per complex FFT) into shared
// rows, then the swirl of every x into SWIRL3D [y][z][x]
__global__ void __launch_bounds__(SW_WARPS * 32) k_swirl_x(const double2 *__restrict__ q, double *__restrict__ sw,
                                                           const __grid_constant__ DevPlan P, int nyp, int mz, int mx, int nxh) {
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = blockIdx.y, z = blockIdx.x * SW_WARPS + warp;
    if (z >= mz) return;
    double2 *a = sm + (size_t)warp * (2 * mx + 5 * mx), *b = a + mx;
    double *ph = (double *)(b + mx);   // [9][mx]
    const int hx = mx / 2;
    for (int f = 0; f < 9; f += 2) {
        const int g = f + 1;
        const double2 *qa = q + (((size_t)f * nyp + y) * mz + z) * nxh;
        const double2 *qb = q + (((size_t)(g < 9 ? g : f) * nyp + y) * mz + z) * nxh;
        for (int k = lane; k < mx; k += 32) {
            const int kk = k <= hx ? k : mx - k;
            double2 Av = make_double2(0.0, 0.0), Bv = make_double2(0.0, 0.0);
            if (kk < nxh) {
                Av = qa[kk];
                if (g < 9) Bv = qb[kk];
            }
            if (k == 0 || k == hx) { Av.y = 0.0; Bv.y = 0.0; }
            a[k] = k <= hx ? make_double2(Av.x - Bv.y, Av.y + Bv.x) : make_double2(Av.x + Bv.y, -Av.y + Bv.x);
        }
        __syncwarp();
        const double2 *res = fft_warp(P, a, b, +1);
        for (int x = lane; x < mx; x += 32) {
            const double2 v = res[x];
            ph[(size_t)f * mx + x] = v.x;
            if (g < 9) ph[(size_t)g * mx + x] = v.y;
        }
        __syncwarp();
    }
    for (int x = lane; x < mx; x += 32) {
#define PH(m) ph[(size_t)(m) * mx + x]
        sw[((size_t)y * mz + z) * mx + x] = swirl_point(PH(0), PH(1), PH(2), PH(3), PH(4), PH(5), PH(6), PH(7), PH(8));
#undef PH
    }
}

int kmm_swirl_particles(kmm_ctx *ctx);

extern "C" int kmm_calcswirl(kmm_ctx *ctx) {
    if (!ctx) return KMM_ERR_ARG;
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mz = ctx->mz, mx = ctx->mx;
    const int ncols = nz * nxh;
    FieldPtrs in;
    for (int m = 0; m < 9; ++m) {
        in.p[m] = SPEC(ctx, KMM_U11 + m);
        if (!in.p[m]) return KMM_ERR_NOMEM;
    }
    double *sw = REAL(ctx, KMM_SWIRL3D);
    if (!sw) return KMM_ERR_NOMEM;
    RET(kmm_ensure_plane_buffers(ctx, 9, 0));
    const size_t sm_dct = sizeof(double2) * 2 * (size_t)fb_len(DCT_CB, 2 * ctx->ny);
    const size_t sm_z = sizeof(double2) * 2 * (size_t)fb_len(ZKB, mz);
    const size_t sm_s = sizeof(double2) * (size_t)SW_WARPS * 7 * mx;
    RET(kmm_smem_attr(ctx, (const void *)k_dct_fwd<double2>, sm_dct));
    RET(kmm_smem_attr(ctx, (const void *)k_zfft_bwd<double2>, sm_z));
    RET(kmm_smem_attr(ctx, (const void *)k_swirl_x, sm_s));
    k_dct_fwd<double2><<<dim3((ncols + DCT_CB - 1) / DCT_CB, 9), 256, sm_dct, ctx->stream>>>(in, ctx->pl_in, ctx->py2,
                                                                                               ctx->py2.tw, nyp, nz,
                                                                                               nxh, ncols);
    CKL();
    ZRecipe zr;
    for (int m = 0; m < 9; ++m) {
        zr.base[m] = (unsigned char)m;
        zr.mult[m] = 0;
    }
    k_zfft_bwd<double2><<<dim3((nxh + ZKB - 1) / ZKB, nyp, 9), 256, sm_z, ctx->stream>>>(
        ctx->pl_in, ctx->q_in, ctx->pmz, ctx->pmz.tw, nyp, nz, nxh, mz, zr, ctx->d_wavx, ctx->d_wavz);
    CKL();
    k_swirl_x<<<dim3((mz + SW_WARPS - 1) / SW_WARPS, nyp), SW_WARPS * 32, sm_s, ctx->stream>>>(ctx->q_in, sw, ctx->wmx,
                                                                                            nyp, mz, mx, nxh);
    CKL();
    return ctx->p.npart > 0 ? kmm_swirl_particles(ctx) : KMM_OK;
}

// ---------------------------------------------------------------------------
// targeted scalar sources of vcw3dp (solvers.f90:2164-2206)
//   scl_flag = 4 (findmaxQ, helpers.f90:678-953): Gaussians of widths sigma at the strongest local
//     maxima of the Q criterion (calcQ, helpers.f90:1519-1552) where the polymer factor
//     beta = exp(-alpha_poly |c|) exceeds 0.8, at most 1023 of them;
//   scl_flag = 5 (newtarget, helpers.f90:957-1222): the swirl strength scaled to [0, 1] by its
//     maximum and then to a volume integral of spts.
// Where the reference is undefined: the scalar enters findmaxQ with its real and imaginary parts
// (the reference assigns the imaginary part to scr and never sets sci, helpers.f90:774); the
// candidate list starts from zeros on every call (the reference's saved Qmin keeps the previous
// call's values, with indices reset to 0, solvers.f90:1938); the walk over the sorted list stops at
// the end of the found minima; newtarget's sum starts from 0 (scsum is left unset).
// ---------------------------------------------------------------------------
#define TG_QN 32768     // findmaxQ's list length (grid_size.f90:2)
#define TG_NTARG 1023   // targets placed while cnt < 1024 (solvers.f90:2172)

__device__ __forceinline__ double q_point(double u11, double u12, double u13, double u21, double u22, double u23,
                                          double u31, double u32, double u33) {
    const double strain = u11 * u11 + u22 * u22 + u33 * u33;
    const double rot = -2.0 * (u12 * u21 + u13 * u31 + u23 * u32);
    return 0.5 * (rot - strain);
}

// one warp per (y, z) row: Hermitian c2r of the nf inputs in pairs (the nine gradients, and for
// MODE 4 the scalar), then per x: MODE 5 the swirl into o0; MODE 4 -Q into o0 and beta into o1
template <int MODE>
__global__ void __launch_bounds__(SW_WARPS * 32) k_target_x(const double2 *__restrict__ q, double *__restrict__ o0,
                                                            double *__restrict__ o1, const __grid_constant__ DevPlan P,
                                                            double alpha_poly, int nyp, int mz, int mx, int nxh) {
    constexpr int NF = MODE == 4 ? 10 : 9;
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = blockIdx.y, z = blockIdx.x * SW_WARPS + warp;
    if (z >= mz) return;
    double2 *a = sm + (size_t)warp * (2 * mx + 5 * mx), *b = a + mx;
    double *ph = (double *)(b + mx);   // [NF][mx]
    const int hx = mx / 2;
    for (int f = 0; f < NF; f += 2) {
        const int g = f + 1;
        const double2 *qa = q + (((size_t)f * nyp + y) * mz + z) * nxh;
        const double2 *qb = q + (((size_t)(g < NF ? g : f) * nyp + y) * mz + z) * nxh;
        for (int k = lane; k < mx; k += 32) {
            const int kk = k <= hx ? k : mx - k;
            double2 Av = make_double2(0.0, 0.0), Bv = make_double2(0.0, 0.0);
            if (kk < nxh) {
                Av = qa[kk];
                if (g < NF) Bv = qb[kk];
            }
            if (k == 0 || k == hx) { Av.y = 0.0; Bv.y = 0.0; }
            a[k] = k <= hx ? make_double2(Av.x - Bv.y, Av.y + Bv.x) : make_double2(Av.x + Bv.y, -Av.y + Bv.x);
        }
        __syncwarp();
        const double2 *res = fft_warp(P, a, b, +1);
        for (int x = lane; x < mx; x += 32) {
            const double2 v = res[x];
            ph[(size_t)f * mx + x] = v.x;
            if (g < NF) ph[(size_t)g * mx + x] = v.y;
        }
        __syncwarp();
    }
    for (int x = lane; x < mx; x += 32) {
        const size_t g3 = ((size_t)y * mz + z) * mx + x;
#define PH(m) ph[(size_t)(m) * mx + x]
        if (MODE == 5) {
            o0[g3] = swirl_point(PH(0), PH(1), PH(2), PH(3), PH(4), PH(5), PH(6), PH(7), PH(8));
        } else {
            o0[g3] = -q_point(PH(0), PH(1), PH(2), PH(3), PH(4), PH(5), PH(6), PH(7), PH(8));
            o1[g3] = exp(-alpha_poly * fabs(PH(9)));
        }
#undef PH
    }
}

// the largest value of a non-negative field (its bit pattern orders like the value): red[0]
__global__ void k_target_max(const double *__restrict__ f, size_t n, unsigned long long *red) {
    double m = 0.0;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, f[e]);
    for (int off = 16; off; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) atomicMax(red, (unsigned long long)__double_as_longlong(m));
}

// f <- f / fmax in place, and per block the partial volume integral of f Lx Ly Lz (Ly the Chebyshev
// node's half-spacings, helpers.f90:1198-1210) into part[blockIdx.x]; blocks span whole y-planes
// in turn so the sum of the partials in block order is deterministic
#define TG_SUM_THREADS 256
__global__ void __launch_bounds__(TG_SUM_THREADS) k_target_norm(double *__restrict__ f, const double *__restrict__ red,
                                                                const double *__restrict__ yc, double *__restrict__ part,
                                                                int nyp, size_t nplane, double lxlz) {
    __shared__ double sh[TG_SUM_THREADS / 32];
    const double fmax_ = red[0];
    const int ny = nyp - 1;
    double acc = 0.0;
    const size_t n = (size_t)nyp * nplane;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / nplane);
        double ly;
        if (i == 0) ly = fabs(yc[1] - yc[0]) / 2.0;
        else if (i == nyp - 1) ly = fabs(yc[nyp - 1] - yc[ny - 1]) / 2.0;
        else ly = fabs(yc[i + 1] - yc[i]) / 2.0 + fabs(yc[i] - yc[i - 1]) / 2.0;
        const double v = f[e] / fmax_;
        f[e] = v;
        acc += v * (lxlz * ly);
    }
    for (int off = 16; off; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < TG_SUM_THREADS / 32; ++w) t += sh[w];
        part[blockIdx.x] = t;
    }
}

// f <- f * spts / sum(part) (var1, helpers.f90:1213-1220)
__global__ void k_target_scale(double *__restrict__ f, const double *__restrict__ part, int nparts, size_t n,
                               double spts) {
    __shared__ double var1;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < nparts; ++b) t += part[b];
        var1 = spts / t;
    }
    __syncthreads();
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        f[e] = f[e] * var1;
}

// a candidate of findmaxQ: its place in the reference's loop order (x outer, z, y inner over the
// interior points), -Q and beta there
struct TgCand {
    long long order;
    double q, beta;
};

// interior grid points (1-based y 2..ny, z 2..mz-1, x 2..mx-1) whose -Q is negative and below all
// six neighbours: appended to the list (capacity cap; *cnt counts them all)
__global__ void k_target_minima(const double *__restrict__ nq, const double *__restrict__ beta, TgCand *__restrict__ list,
                                unsigned *__restrict__ cnt, size_t cap, int nyp, int mz, int mx) {
    const size_t nplane = (size_t)mz * mx, n = (size_t)nyp * nplane;
    const int ny = nyp - 1;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / nplane), r = (int)(e - (size_t)i * nplane), j = r / mx, k = r - j * mx;   // 0-based
        if (i < 1 || i > ny - 1 || j < 1 || j > mz - 2 || k < 1 || k > mx - 2) continue;
        const double v = nq[e];
        if (!(v < 0.0)) continue;
        if (v < nq[e + nplane] && v < nq[e - nplane] && v < nq[e + mx] && v < nq[e - mx] && v < nq[e + 1] &&
            v < nq[e - 1]) {
            const unsigned s = atomicAdd(cnt, 1u);
            if (s < cap) {
                TgCand c;
                c.order = ((long long)(k - 1) * (mz - 2) + (j - 1)) * (long long)(ny - 1) + (i - 1);
                c.q = v;
                c.beta = beta[e];
                list[s] = c;
            }
        }
    }
}

// the source of the placed targets: per point, every target's Gaussian in placement order with the
// reference's cut-offs (solvers.f90:2177-2200), so each point's sum has the reference's order
__global__ void k_target_deposit(double *__restrict__ sc, const double *__restrict__ tc, int nt,
                                 const double *__restrict__ ycoord, int nyp, int mz, int mx, double delxm, double delzm,
                                 double sx, double sy, double sz, double dT) {
    const size_t nplane = (size_t)mz * mx, n = (size_t)nyp * nplane;
    const double ax = 2.0 * sx * sx, ay = 2.0 * sy * sy, az = 2.0 * sz * sz;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / nplane), r = (int)(e - (size_t)i * nplane), j = r / mx, k = r - j * mx;
        const double xk = (double)k * delxm, zj = (double)j * delzm, yi = ycoord[i];
        double acc = 0.0;
        for (int t = 0; t < nt; ++t) {
            const double dx = xk - tc[3 * t], betax = dx * dx / ax;
            if (!(betax < 18.0)) continue;
            const double dz = zj - tc[3 * t + 2], betaz = dz * dz / az;
            if (!(betax + betaz < 18.0)) continue;
            const double dy = yi - tc[3 * t + 1], betay = dy * dy / ay;
            if (betax + betay + betaz < 18.0) acc += dT * exp(-(betax + betay + betaz));
        }
        sc[e] = acc;
    }
}

// Shell_Sort of findmaxQ's list (helpers.f90:1557-1594): the reference's increments (n / 2, then
// * 5 / 11, 2 -> 1), which decide the order of equal values; b, c, d, e follow a's moves
static void tg_shell_sort(double *a, int *b, int *c, int *d, double *e, int n) {
    int inc = n / 2;
    while (inc > 0) {
        for (int i = inc; i < n; ++i) {
            int j = i;
            const double t1 = a[i], t5 = e[i];
            const int t2 = b[i], t3 = c[i], t4 = d[i];
            while (j >= inc && a[j - inc] > t1) {
                a[j] = a[j - inc]; b[j] = b[j - inc]; c[j] = c[j - inc]; d[j] = d[j - inc]; e[j] = e[j - inc];
                j -= inc;
            }
            a[j] = t1; b[j] = t2; c[j] = t3; d[j] = t4; e[j] = t5;
        }
        inc = inc == 2 ? 1 : inc * 5 / 11;
    }
}

// the scalar source of scl_flag 4 or 5 into ctx->scsource (the caller zeroes it outside the
// source window); the nine gradients U11..U33 are current
int kmm_target_source(kmm_ctx *ctx) {
    const int flag = ctx->p.scl_flag;
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mz = ctx->mz, mx = ctx->mx;
    const int ncols = nz * nxh, nf = flag == 4 ? 10 : 9;
    const size_t nphys = ctx->nphys, nplane = (size_t)mz * mx;
    FieldPtrs in;
    for (int m = 0; m < 9; ++m) {
        in.p[m] = SPEC(ctx, KMM_U11 + m);
        if (!in.p[m]) return KMM_ERR_NOMEM;
    }
    if (flag == 4) {
        in.p[9] = SPEC(ctx, KMM_SCALAR);
        if (!in.p[9]) return KMM_ERR_NOMEM;
    }
    RET(kmm_ensure_plane_buffers(ctx, nf, 0));
    if (!ctx->d_tgtred) CK(cudaMalloc(&ctx->d_tgtred, sizeof(double) * 2048));
    const size_t sm_dct = sizeof(double2) * 2 * (size_t)fb_len(DCT_CB, 2 * ctx->ny);
    const size_t sm_z = sizeof(double2) * 2 * (size_t)fb_len(ZKB, mz);
    const size_t sm_s = sizeof(double2) * (size_t)SW_WARPS * 7 * mx;
    RET(kmm_smem_attr(ctx, (const void *)k_dct_fwd<double2>, sm_dct));
    RET(kmm_smem_attr(ctx, (const void *)k_zfft_bwd<double2>, sm_z));
    k_dct_fwd<double2><<<dim3((ncols + DCT_CB - 1) / DCT_CB, nf), 256, sm_dct, ctx->stream>>>(in, ctx->pl_in, ctx->py2,
                                                                                                ctx->py2.tw, nyp, nz,
                                                                                                nxh, ncols);
    CKL();
    ZRecipe zr;
    for (int m = 0; m < nf; ++m) {
        zr.base[m] = (unsigned char)m;
        zr.mult[m] = 0;
    }
    k_zfft_bwd<double2><<<dim3((nxh + ZKB - 1) / ZKB, nyp, nf), 256, sm_z, ctx->stream>>>(
        ctx->pl_in, ctx->q_in, ctx->pmz, ctx->pmz.tw, nyp, nz, nxh, mz, zr, ctx->d_wavx, ctx->d_wavz);
    CKL();
    const dim3 gx((mz + SW_WARPS - 1) / SW_WARPS, nyp);
    const int nb = (int)((nphys + 255) / 256 < 2048 ? (nphys + 255) / 256 : 2048);
    if (flag == 5) {
        RET(kmm_smem_attr(ctx, (const void *)k_target_x<5>, sm_s));
        k_target_x<5><<<gx, SW_WARPS * 32, sm_s, ctx->stream>>>(ctx->q_in, ctx->scsource, NULL, ctx->wmx, 0.0, nyp, mz,
                                                               mx, nxh);
        CKL();
        CK(cudaMemsetAsync(ctx->d_tgtred, 0, sizeof(double), ctx->stream));
        k_target_max<<<nb, 256, 0, ctx->stream>>>(ctx->scsource, nphys, (unsigned long long *)ctx->d_tgtred);
        CKL();
        const int npart = nb < 2047 ? nb : 2047;
        k_target_norm<<<npart, TG_SUM_THREADS, 0, ctx->stream>>>(ctx->scsource, ctx->d_tgtred, ctx->d_ycoord,
                                                                 ctx->d_tgtred + 1, nyp, nplane,
                                                                 (ctx->xl / (double)mx) * (ctx->zl / (double)mz));
        CKL();
        k_target_scale<<<nb, 256, 0, ctx->stream>>>(ctx->scsource, ctx->d_tgtred + 1, npart, nphys, ctx->p.spts);
        CKL();
        return KMM_OK;
    }
    // scl_flag = 4: -Q into d_tgtq, beta into the source array (overwritten by the deposit below)
    if (!ctx->d_tgtq) CK(cudaMalloc(&ctx->d_tgtq, sizeof(double) * nphys));
    if (!ctx->d_tgtcnt) CK(cudaMalloc(&ctx->d_tgtcnt, sizeof(unsigned)));
    if (!ctx->d_tgtc) CK(cudaMalloc(&ctx->d_tgtc, sizeof(double) * 3 * TG_NTARG));
    if (!ctx->h_targ) {
        ctx->h_targ = (int *)calloc(3 * TG_NTARG, sizeof(int));
        if (!ctx->h_targ) return KMM_ERR_NOMEM;
    }
    if (!ctx->d_tgtlist) {
        const size_t cap = nphys < ((size_t)1 << 22) ? nphys : ((size_t)1 << 22);
        CK(cudaMalloc(&ctx->d_tgtlist, sizeof(TgCand) * cap));
        CK(cudaMallocHost(&ctx->h_tgtlist, sizeof(TgCand) * cap));
        ctx->tgt_cap = cap;
    }
    RET(kmm_smem_attr(ctx, (const void *)k_target_x<4>, sm_s));
    k_target_x<4><<<gx, SW_WARPS * 32, sm_s, ctx->stream>>>(ctx->q_in, ctx->d_tgtq, ctx->scsource, ctx->wmx,
                                                           ctx->p.alpha_poly, nyp, mz, mx, nxh);
    CKL();
    CK(cudaMemsetAsync(ctx->d_tgtcnt, 0, sizeof(unsigned), ctx->stream));
    k_target_minima<<<nb, 256, 0, ctx->stream>>>(ctx->d_tgtq, ctx->scsource, (TgCand *)ctx->d_tgtlist, ctx->d_tgtcnt,
                                                 ctx->tgt_cap, nyp, mz, mx);
    CKL();
    unsigned *hcnt = (unsigned *)kmm_h_pin_status(ctx);   // the pinned status word, free until the x stage
    CK(cudaMemcpyAsync(hcnt, ctx->d_tgtcnt, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const size_t found = *hcnt;
    if (found > ctx->tgt_cap) {
        kmm_set_error(ctx, "scl_flag = 4: %zu candidate minima exceed the list capacity %zu", found, ctx->tgt_cap);
        return KMM_ERR_UNSUPPORTED;
    }
    TgCand *hl = (TgCand *)ctx->h_tgtlist;
    if (found) {
        CK(cudaMemcpyAsync(hl, ctx->d_tgtlist, sizeof(TgCand) * found, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    // the first qn minima in the reference's loop order, then its sort of the qn-long list
    std::sort(hl, hl + found, [](const TgCand &a, const TgCand &b) { return a.order < b.order; });
    const int nkeep = found < TG_QN ? (int)found : TG_QN;
    std::vector<double> qv(TG_QN, 0.0), bv(TG_QN, 0.0);
    std::vector<int> qx(TG_QN, 0), qy(TG_QN, 0), qz(TG_QN, 0);
    const int ny = ctx->ny;
    for (int c = 0; c < nkeep; ++c) {
        const long long o = hl[c].order;
        const int i = (int)(o % (ny - 1)), jk = (int)(o / (ny - 1)), j = jk % (mz - 2), k = jk / (mz - 2);
        qv[c] = hl[c].q;
        bv[c] = hl[c].beta;
        qx[c] = k + 2;   // 1-based x, y, z indices (the reference's Qx, Qy, Qz)
        qy[c] = i + 2;
        qz[c] = j + 2;
    }
    tg_shell_sort(qv.data(), qx.data(), qy.data(), qz.data(), bv.data(), TG_QN);
    double *hc = (double *)malloc(sizeof(double) * 3 * TG_NTARG);
    if (!hc) return KMM_ERR_NOMEM;
    const double delxm = ctx->xl / (double)mx, delzm = ctx->zl / (double)mz;
    int nt = 0;
    for (int n = 0; n < TG_QN && nt < TG_NTARG; ++n) {
        if (qx[n] == 0) break;   // the end of the found minima
        if (!(bv[n] > 0.8)) continue;
        hc[3 * nt] = delxm * (double)(qx[n] - 1);
        hc[3 * nt + 1] = ctx->h_ycoord[qy[n] - 1];
        hc[3 * nt + 2] = delzm * (double)(qz[n] - 1);
        ctx->h_targ[3 * nt] = qx[n];
        ctx->h_targ[3 * nt + 1] = qy[n];
        ctx->h_targ[3 * nt + 2] = qz[n];
        ++nt;
    }
    ctx->ntarg = nt;
    cudaError_t e = nt ? cudaMemcpyAsync(ctx->d_tgtc, hc, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, ctx->stream)
                       : cudaSuccess;
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);   // hc is pageable and freed next
    free(hc);
    CK(e);
    k_target_deposit<<<nb, 256, 0, ctx->stream>>>(ctx->scsource, ctx->d_tgtc, nt, ctx->d_ycoord, nyp, mz, mx, delxm,
                                                  delzm, ctx->p.sigmax, ctx->p.sigmay, ctx->p.sigmaz, ctx->p.deltat);
    CKL();
    return KMM_OK;
}

extern "C" int kmm_target_list(kmm_ctx *ctx, int *ijk, int n) {
    if (!ctx || n < 0 || (n > 0 && !ijk)) return -KMM_ERR_ARG;
    for (int m = 0; m < 3 * ctx->ntarg && m < n; ++m) ijk[m] = ctx->h_targ[m];
    return ctx->ntarg;
}

// ---------------------------------------------------------------------------
// flow statistics of writeoutputs (helpers.f90:1227-1438) by Parseval over the 3/2 grid: the
// x-z mean of a product of two band-limited fields is the weighted sum of mode products
// (weight 1 for kx = 0, 2 for kx > 0, the conjugate half); the mean profile is the (0,0) mode.
// ---------------------------------------------------------------------------
#define FS_THREADS 256
// one block per y: PL[f][y][kx][kz] holds y-physical u, v, w, du/dy (f = 0..3) ->
// acc[y][6] = umean, <u'^2>, <v^2>, <w^2>, <u'v>, <du/dy>
__global__ void __launch_bounds__(FS_THREADS) k_flowstats(const double2 *__restrict__ pl, double *__restrict__ acc,
                                                          int nyp, int nz, int nxh) {
    __shared__ double red[4][FS_THREADS / 32];
    const int y = blockIdx.x;
    const size_t fs = (size_t)nyp * nxh * nz;
    const double2 *pu = pl + (size_t)y * nxh * nz, *pv = pu + fs, *pw = pv + fs;
    double su = 0.0, sv = 0.0, sw = 0.0, suv = 0.0;
    for (int e = threadIdx.x; e < nxh * nz; e += FS_THREADS) {
        const int kx = e / nz;
        const double wt = kx == 0 ? 1.0 : 2.0;
        const double2 u = pu[e], v = pv[e], w = pw[e];
        sv += wt * (v.x * v.x + v.y * v.y);
        sw += wt * (w.x * w.x + w.y * w.y);
        if (e != 0) {   // u' = u - umean drops the (0,0) mode
            su += wt * (u.x * u.x + u.y * u.y);
            suv += wt * (u.x * v.x + u.y * v.y);
        }
    }
    double vals[4] = {su, sv, sw, suv};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        double x = vals[m];
        for (int off = 16; off; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) red[m][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double out[4];
        for (int m = 0; m < 4; ++m) {
            double x = 0.0;
            for (int w = 0; w < FS_THREADS / 32; ++w) x += red[m][w];
            out[m] = x;
        }
        acc[(size_t)y * 6 + 0] = pu[0].x;
        acc[(size_t)y * 6 + 1] = out[0];
        acc[(size_t)y * 6 + 2] = out[1];
        acc[(size_t)y * 6 + 3] = out[2];
        acc[(size_t)y * 6 + 4] = out[3];
        acc[(size_t)y * 6 + 5] = pl[3 * fs + (size_t)y * nxh * nz].x;
    }
}

extern "C" int kmm_flowstats(kmm_ctx *ctx, double *prof, double *scal) {
    if (!ctx || !prof || !scal) return KMM_ERR_ARG;
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh;
    const int ncols = nz * nxh;
    RET(kmm_veloc(ctx));
    double2 *du = ctx->wrk[0];
    RET(kmm_internal_cderiv(ctx, SPEC(ctx, KMM_U), du));
    FieldPtrs in;
    in.p[0] = SPEC(ctx, KMM_U);
    in.p[1] = SPEC(ctx, KMM_V);
    in.p[2] = SPEC(ctx, KMM_W);
    in.p[3] = du;
    RET(kmm_ensure_plane_buffers(ctx, 4, 0));
    const size_t sm_dct = sizeof(double2) * 2 * (size_t)fb_len(DCT_CB, 2 * ctx->ny);
    RET(kmm_smem_attr(ctx, (const void *)k_dct_fwd<double2>, sm_dct));
    k_dct_fwd<double2><<<dim3((ncols + DCT_CB - 1) / DCT_CB, 4), 256, sm_dct, ctx->stream>>>(in, ctx->pl_in, ctx->py2,
                                                                                               ctx->py2.tw, nyp, nz,
                                                                                               nxh, ncols);
    CKL();
    double *acc = ctx->d_scratch;   // 9 KMM_MAX_NYP doubles: 6 nyp used here
    k_flowstats<<<nyp, FS_THREADS, 0, ctx->stream>>>(ctx->pl_in, acc, nyp, nz, nxh);
    CKL();
    double h[6 * KMM_MAX_NYP];
    CK(cudaMemcpyAsync(h, acc, sizeof(double) * 6 * nyp, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double *umean = prof, *urms = prof + nyp, *vrms = prof + 2 * nyp, *wrms = prof + 3 * nyp;
    double *R12 = prof + 4 * nyp, *T12 = prof + 5 * nyp, *ke = prof + 6 * nyp;
    for (int i = 0; i < nyp; ++i) {
        const double *a = h + (size_t)i * 6;
        umean[i] = a[0];
        urms[i] = sqrt(a[1]);
        vrms[i] = sqrt(a[2]);
        wrms[i] = sqrt(a[3]);
        R12[i] = a[4];
        T12[i] = a[5] / ctx->re;
        ke[i] = 0.5 * (a[0] * a[0] + a[1] + a[2] + a[3]);
    }
    double mf = 0.0, kb = 0.0;
    for (int i = 0; i < nyp - 1; ++i) {
        const double dy = fabs(ctx->h_ycoord[i + 1] - ctx->h_ycoord[i]);
        mf += 1.0 / ctx->yl * 0.5 * (umean[i + 1] + umean[i]) * dy;
        kb += 1.0 / ctx->yl * 0.5 * (ke[i + 1] + ke[i]) * dy;
    }
    scal[0] = mf;
    scal[1] = T12[0];
    scal[2] = T12[nyp - 1];
    scal[3] = kb;
    return KMM_OK;
}

// ---------------------------------------------------------------------------
// bounded-wait check: one mbarrier that nothing arrives on and no copy targets, waited on with the
// same bounded wait the bulk-copy kernels use; when the limit runs out the CTA records
// KMM_ERR_TIMEOUT and returns, exactly as k_xphys2 and the TMA z kernels do.  No copy is in
// flight, so giving up leaves nothing behind.
// ---------------------------------------------------------------------------
__global__ void k_wait_selftest(int *status, unsigned long long limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        kasync::mbar_init(&bar, 1);
        kasync::mbar_init_fence();
    }
    __syncthreads();
    const bool ok = kasync::mbar_wait_for(&bar, 0, limit_ns);
    if (!__all_sync(0xffffffffu, ok) && (threadIdx.x & 31) == 0) atomicMax(status, KMM_ERR_TIMEOUT);
}

// this unit's bounded-wait limit on the current device (KMM_OPT_WAIT_LIMIT_MS)
int kmm_plane_set_wait_limit(unsigned long long ns) { return kasync::kasync_set_wait_limit(ns) == cudaSuccess ? 0 : 1; }

extern "C" int kmm_wait_selftest(kmm_ctx *ctx, double limit_ms) {
    if (!ctx || !(limit_ms > 0.0) || limit_ms > 10000.0) return KMM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    k_wait_selftest<<<1, 32, 0, ctx->stream>>>(ctx->d_status, (unsigned long long)(limit_ms * 1e6));
    CKL();
    int st = 0;
    CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (st == KMM_ERR_TIMEOUT) kmm_set_error(ctx, "bounded wait ran out after %.3f ms (expected)", limit_ms);
    return st;
}
