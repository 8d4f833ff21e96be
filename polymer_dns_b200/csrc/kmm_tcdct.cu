// kmm_tcdct.cu -- the y (Chebyshev) transforms of the routine path's mixed form as split-precision
// GEMMs on the fifth-generation tensor cores (tcgen05, TMEM accumulators).
//
// Work (solvers.f90:2402-2546 forward, 3279-3416 backward; FFTW REDFT00 in the reference):
//   forward  X_y = sum_n a_n cos(pi n y / ny)                        (Chebyshev -> Gauss-Lobatto values)
//            = the c(n)/2 pre-scale + REDFT00 of the reference, exactly;
//   backward a_n = s_n sum_y w_y p_y cos(pi n y / ny),  w_y = 1 (y = 0, ny) else 2,
//            s_n = 1/ny, halved at n = 0, ny                          (REDFT00, /ny, halved ends).
// Both are D = T x P with the fixed (ny+1) x (ny+1) cosine matrix T, over the 2 nz nxh real
// sequences (real and imaginary parts of every column) of each field.
//
// GEMM shape per tile: M = 128 output indices (y, or n) held by T (the A operand, resident in
// shared memory), N = 64 real sequences = 32 complex columns (the B operand, re parts in rows
// 0..31, im parts in rows 32..63), K = ny + 1 padded to a multiple of 8.  For ny = 128 the 129th
// output (index 128) is a signed sum formed on the CUDA cores in FP64 while the tile is
// converted.  Precision: 3xTF32 -- each operand is split into a TF32 head and a TF32 tail
// (x = hi + lo to ~22 bits) and D = T_lo P_hi + T_hi P_lo + T_hi P_hi with FP32 accumulation in
// TMEM, the FP32-class accuracy the mixed form's FFTs have.
//
// Kernel: persistent, one CTA of 8 warps per SM (A hi / lo 139 KB + B hi / lo 70 KB of shared
// memory at ny = 128).  Per tile: all warps load the 32 columns (FP64 spectral columns forward,
// FP32 planes backward) into registers; warps 0-3 drain the previous tile's accumulator from TMEM
// (tcgen05.ld) and store it while those loads are in flight; the tile is split and written into
// the canonical no-swizzle K-major operand layout (8-row x 16-byte core matrices); one thread
// issues the 3 x K/8 tcgen05.mma (kind::tf32, 128 x 64 x 8 each) into one of two TMEM
// accumulators and commits them to an mbarrier.  Every wait is bounded (the unit's wait limit);
// a wait that runs out records KMM_ERR_TIMEOUT, waits (bounded) for the MMAs still in flight,
// frees TMEM and ends the CTA.
#include "kmm_internal.cuh"
#include "kmm_async.cuh"

namespace {

constexpr int TC_THREADS = 256;
constexpr int TC_CT = 32;          // complex columns per tile
constexpr int TC_N = 2 * TC_CT;    // real sequences per tile (GEMM N)
constexpr int TC_M = 128;          // GEMM M (one TMEM lane per output index)
constexpr int TC_TMEM_COLS = 128;  // two 64-column FP32 accumulators

struct TcFields {
    const void *p[KMM_TC_MAXF];
};
struct TcFieldsW {
    void *p[KMM_TC_MAXF];
};

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// x = hi + lo: hi the TF32 rounding of x, lo the TF32 rounding of the remainder
__device__ __forceinline__ void split_tf32(double x, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32((float)x);
    lo = to_tf32((float)(x - (double)__uint_as_float(hi)));
}

// shared-memory matrix descriptor, canonical K-major layout without swizzle: core matrices of
// 8 rows x 16 bytes stored contiguously (128 B), `sbo` bytes between core matrices adjacent in M / N,
// `lbo` bytes between core matrices adjacent in K; bits 46-47 = 1 (the sm_100 descriptor version)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2),
// both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t tc_idesc(int m, int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 accumulator columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld16(uint32_t ta, uint32_t *r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(ta));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// byte offset of element (row, k) in a K-major no-swizzle operand with `rows` rows
__device__ __forceinline__ uint32_t kmaj_off(int row, int k, int rows) {
    return (uint32_t)((k >> 2) * (rows / 8) * 128 + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// register type of a loaded input element: FP64 spectral coefficients forward, FP32 plane values
// backward
template <int DIR>
struct InT {
    typedef double2 T;
    static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
};
template <>
struct InT<1> {
    typedef float2 T;
    static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
};

template <int NY>
struct TcShape {
    static constexpr int NYP = NY + 1;
    static constexpr int K = (NYP + 7) / 8 * 8;          // GEMM K: ny + 1 padded to the MMA's K step
    static constexpr int KG = K / 4;                      // 16-byte core-matrix columns along K
    static constexpr int G = (KG + 7) / 8;               // of those, per warp
    static constexpr int A_BYTES = TC_M * K * 4, B_BYTES = TC_N * K * 4;
    static constexpr int LBO_A = (TC_M / 8) * 128, LBO_B = (TC_N / 8) * 128;
    static constexpr int XN_DOUBLES = 2 * 8 * 32 * 2;     // [buffer][warp][lane][re, im]
    static constexpr size_t SMEM = 2 * (size_t)A_BYTES + 2 * (size_t)B_BYTES + XN_DOUBLES * 8 + 64;
};

// One bounded wait on an MMA commit barrier; on a timeout records the status
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t &phase, int *status) {
    const bool ok = kasync::mbar_wait(bar, phase);
    phase ^= 1u;
    if (!ok && (threadIdx.x & 31) == 0) atomicMax(status, KMM_ERR_TIMEOUT);
    return ok;
}

// DIR 0 (forward): in = FP64 spectral columns [f][col][n], out = FP32 planes [f][y][col].
// DIR 1 (backward): in = FP32 planes [f][y][col], out = FP64 spectral columns [f][col][n].
// tw2: the 2 ny-point FP64 twiddles exp(-i pi m / ny).
template <int NY, int DIR>
__global__ void __launch_bounds__(TC_THREADS, 1) k_tcdct(TcFields in, TcFieldsW out, const double2 *__restrict__ tw2,
                                                         int nf, int ncols, int *status) {
    using S = TcShape<NY>;
    constexpr int NYP = S::NYP, K = S::K, KG = S::KG, G = S::G;
    constexpr uint32_t IDESC = tc_idesc(TC_M, TC_N);
    extern __shared__ __align__(1024) uint8_t tsm[];
    uint8_t *Ahi = tsm, *Alo = tsm + S::A_BYTES, *Bhi = Alo + S::A_BYTES, *Blo = Bhi + S::B_BYTES;
    double *xn = reinterpret_cast<double *>(Blo + S::B_BYTES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(xn + S::XN_DOUBLES);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        kasync::mbar_init(&bar[0], 1);
        kasync::mbar_init(&bar[1], 1);
        kasync::mbar_init_fence();
    }
    // A = the cosine matrix with the direction's weights, rows m = output index, columns k = input
    for (int e = tid; e < TC_M * K; e += TC_THREADS) {
        const int m = e / K, k = e - m * K;
        double v = 0.0;
        if (m <= NY && k <= NY) {
            v = tw2[(m * k) % (2 * NY)].x;   // cos(pi m k / ny)
            if (DIR == 1) {
                const double sm = (m == 0 || m == NY) ? 0.5 / (double)NY : 1.0 / (double)NY;
                const double wk = (k == 0 || k == NY) ? 1.0 : 2.0;
                v = v * wk * sm;
            }
        }
        uint32_t h, l;
        split_tf32(v, h, l);
        const uint32_t off = kmaj_off(m, k, TC_M);
        *reinterpret_cast<uint32_t *>(Ahi + off) = h;
        *reinterpret_cast<uint32_t *>(Alo + off) = l;
    }
    // B rows beyond ny (k >= NYP) stay zero for every tile: clear once
    for (int e = tid; e < S::B_BYTES / 4; e += TC_THREADS) {
        reinterpret_cast<uint32_t *>(Bhi)[e] = 0u;
        reinterpret_cast<uint32_t *>(Blo)[e] = 0u;
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const int tpf = ncols / TC_CT;   // tiles per field
    const int ntiles = nf * tpf;
    uint32_t ph[2] = {0u, 0u};
    bool ok = true;
    int pf = 0, pc0 = 0;
    for (int it = 0, t = blockIdx.x;; ++it, t += gridDim.x) {
        const bool have = t < ntiles && ok;
        const int buf = it & 1;
        // (a) the previous tile's MMAs are done: B may be overwritten, its accumulator is ready
        if (it > 0) {
            ok = tc_wait(&bar[buf ^ 1], ph[buf ^ 1], status) && ok;
            tc_fence_after();
        }
        // (b) this tile's inputs into registers: lane = column, warp w takes K groups w, w + 8, ...
        int f = 0, c0 = 0;
        typename InT<DIR>::T v[G][4];
        if (have) {
            f = t / tpf;
            c0 = (t - f * tpf) * TC_CT;
#pragma unroll
            for (int gi = 0; gi < G; ++gi) {
                const int g = warp + 8 * gi;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int n = 4 * g + q;
                    typename InT<DIR>::T x = InT<DIR>::zero();
                    if (g < KG && n < NYP) {
                        if (DIR == 0)   // FP64 spectral column (c0 + lane), coefficient n
                            x = reinterpret_cast<const typename InT<DIR>::T *>(in.p[f])[(size_t)(c0 + lane) * NYP + n];
                        else            // FP32 plane y = n, column c0 + lane
                            x = reinterpret_cast<const typename InT<DIR>::T *>(in.p[f])[(size_t)n * ncols + c0 + lane];
                    }
                    v[gi][q] = x;
                }
            }
        }
        // (c) drain the previous tile's accumulator
        if (it > 0 && ok) {
            if (warp < 4) {
                const uint32_t ta = tmem + (uint32_t)(64 * (buf ^ 1)) + ((uint32_t)(32 * warp) << 16);
                const int m = 32 * warp + lane;   // output index of this lane
#pragma unroll 1
                for (int cb = 0; cb < TC_CT; cb += 16) {   // 16 columns: re at cb.., im at 32 + cb..
                    uint32_t r[32];
                    tmem_ld16(ta + (uint32_t)cb, r);
                    tmem_ld16(ta + (uint32_t)(32 + cb), r + 16);
                    tmem_wait_ld();
                    if (m <= NY) {
                        if (DIR == 0) {
                            float4 *dst = reinterpret_cast<float4 *>(
                                reinterpret_cast<float2 *>(out.p[pf]) + (size_t)m * ncols + pc0 + cb);
#pragma unroll
                            for (int c = 0; c < 16; c += 2)
                                dst[c / 2] = make_float4(__uint_as_float(r[c]), __uint_as_float(r[16 + c]),
                                                         __uint_as_float(r[c + 1]), __uint_as_float(r[17 + c]));
                        } else {
                            double2 *dst = reinterpret_cast<double2 *>(out.p[pf]) + (size_t)(pc0 + cb) * NYP + m;
#pragma unroll
                            for (int c = 0; c < 16; ++c)
                                dst[(size_t)c * NYP] =
                                    make_double2((double)__uint_as_float(r[c]), (double)__uint_as_float(r[16 + c]));
                        }
                    }
                }
            }
            if (NY == 128 && warp == 4) {   // the output index ny: the FP64 signed sums of the tile
                double sre = 0.0, sim = 0.0;
#pragma unroll
                for (int w = 0; w < 8; ++w) {
                    sre += xn[(((buf ^ 1) * 8 + w) * 32 + lane) * 2];
                    sim += xn[(((buf ^ 1) * 8 + w) * 32 + lane) * 2 + 1];
                }
                if (DIR == 0) {
                    reinterpret_cast<float2 *>(out.p[pf])[(size_t)NY * ncols + pc0 + lane] =
                        make_float2((float)sre, (float)sim);
                } else {
                    const double s = 0.5 / (double)NY;
                    reinterpret_cast<double2 *>(out.p[pf])[(size_t)(pc0 + lane) * NYP + NY] = make_double2(s * sre, s * sim);
                }
            }
            tc_fence_before();
        }
        if (!have) break;
        // (d) split into the B operand: re of column c in row c, im in row 32 + c
        double sre = 0.0, sim = 0.0;
#pragma unroll
        for (int gi = 0; gi < G; ++gi) {
            const int g = warp + 8 * gi;
            if (g < KG) {
                uint32_t phr[4], plr[4], phi[4], pli[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int n = 4 * g + q;
                    split_tf32((double)v[gi][q].x, phr[q], plr[q]);
                    split_tf32((double)v[gi][q].y, phi[q], pli[q]);
                    if (NY == 128 && n <= NY) {
                        const double wgt = (DIR == 0) ? ((n & 1) ? -1.0 : 1.0)
                                                      : ((n & 1) ? -1.0 : 1.0) * ((n == 0 || n == NY) ? 1.0 : 2.0);
                        sre += wgt * (double)v[gi][q].x;
                        sim += wgt * (double)v[gi][q].y;
                    }
                }
                const uint32_t ore = kmaj_off(lane, 4 * g, TC_N), oim = kmaj_off(32 + lane, 4 * g, TC_N);
                *reinterpret_cast<uint4 *>(Bhi + ore) = make_uint4(phr[0], phr[1], phr[2], phr[3]);
                *reinterpret_cast<uint4 *>(Blo + ore) = make_uint4(plr[0], plr[1], plr[2], plr[3]);
                *reinterpret_cast<uint4 *>(Bhi + oim) = make_uint4(phi[0], phi[1], phi[2], phi[3]);
                *reinterpret_cast<uint4 *>(Blo + oim) = make_uint4(pli[0], pli[1], pli[2], pli[3]);
            }
        }
        if (NY == 128) {
            xn[((buf * 8 + warp) * 32 + lane) * 2] = sre;
            xn[((buf * 8 + warp) * 32 + lane) * 2 + 1] = sim;
        }
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        // (f) one thread issues the tile's MMAs: the two tail products first, then hi x hi
        if (tid == 0) {
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(64 * buf);
            const uint32_t ah = su32(Ahi), al = su32(Alo), bh = su32(Bhi), bl = su32(Blo);
            uint32_t acc = 0u;
#pragma unroll 1
            for (int pass = 0; pass < 3; ++pass) {
                const uint32_t a0 = pass == 0 ? al : ah, b0 = pass == 1 ? bl : bh;
#pragma unroll 1
                for (int s = 0; s < K / 8; ++s) {
                    mma_tf32(d, sdesc(a0 + (uint32_t)(2 * s * S::LBO_A), S::LBO_A, 128),
                             sdesc(b0 + (uint32_t)(2 * s * S::LBO_B), S::LBO_B, 128), IDESC, acc);
                    acc = 1u;
                }
            }
            mma_commit(&bar[buf]);
        }
        pf = f;
        pc0 = c0;
    }
    // after a timeout: wait (bounded) for whatever MMA may still be in flight before freeing TMEM
    if (!ok) {
        kasync::mbar_wait(&bar[0], ph[0]);
        kasync::mbar_wait(&bar[1], ph[1]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
    }
}

__device__ __forceinline__ void mma_tf32_ts(uint32_t d, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d),
        "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc));
}

// 8 consecutive 32-bit TMEM columns of this warp's 32 lanes from registers
__device__ __forceinline__ void tmem_st8(uint32_t ta, const uint32_t *r) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(ta), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// The forward transform with the cosine matrix in TMEM and the input tiles staged by bulk copies.
// TMEM (512 columns): T_hi in columns [0, K), T_lo in [K, 2K) (one row per lane), accumulators at
// 384 and 448.  Shared memory: two staging buffers holding one tile's 32 raw FP64 columns each
// (a contiguous 32 (ny+1) x 16-byte range, one cp.async.bulk), the B operand (hi / lo), the signed
// sums of the ny row.  While tile i is converted and multiplied, tile i + 1 is in flight; the copy
// of tile i + 2 is issued as soon as tile i's staging buffer has been read.
template <int NY>
struct TcFwd2 {
    static constexpr int NYP = NY + 1, K = TcShape<NY>::K, KG = K / 4, G = (KG + 7) / 8;
    static constexpr int STG_BYTES = TC_CT * NYP * 16;
    static constexpr int B_BYTES = TC_N * K * 4, LBO_B = (TC_N / 8) * 128;
    static constexpr int XN_DOUBLES = 2 * 8 * 32 * 2;
    static constexpr size_t SMEM = 2 * (size_t)STG_BYTES + 2 * (size_t)B_BYTES + XN_DOUBLES * 8 + 128;
    static constexpr uint32_t D0 = 384;   // TMEM column of the first accumulator
};

template <int NY>
__global__ void __launch_bounds__(TC_THREADS, 1) k_tcdct_fwd2(TcFields in, TcFieldsW out, const double2 *__restrict__ tw2,
                                                              int nf, int ncols, int *status) {
    using S = TcFwd2<NY>;
    constexpr int NYP = S::NYP, K = S::K, KG = S::KG, G = S::G;
    constexpr uint32_t IDESC = tc_idesc(TC_M, TC_N);
    extern __shared__ __align__(1024) uint8_t tsm[];
    uint8_t *stg0 = tsm, *stg1 = tsm + S::STG_BYTES;
    uint8_t *Bhi = tsm + 2 * S::STG_BYTES, *Blo = Bhi + S::B_BYTES;
    double *xn = reinterpret_cast<double *>(Blo + S::B_BYTES);
    uint64_t *tbar = reinterpret_cast<uint64_t *>(xn + S::XN_DOUBLES);   // [2] staging copies
    uint64_t *mbar = tbar + 2;                                             // [2] MMA commits
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tpf = ncols / TC_CT, ntiles = nf * tpf;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)), "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    auto tile_src = [&](int t) -> const void * {
        const int f = t / tpf, c0 = (t - f * tpf) * TC_CT;
        return reinterpret_cast<const double2 *>(in.p[f]) + (size_t)c0 * NYP;
    };
    bool pend[2] = {false, false};
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            kasync::mbar_init(&tbar[b], 1);
            kasync::mbar_init(&mbar[b], 1);
        }
        kasync::mbar_init_fence();
        for (int b = 0; b < 2; ++b) {
            const int t = blockIdx.x + b * gridDim.x;
            if (t < ntiles) {
                kasync::mbar_expect_tx(&tbar[b], S::STG_BYTES);
                kasync::bulk_g2s(b ? stg1 : stg0, tile_src(t), S::STG_BYTES, &tbar[b]);
                pend[b] = true;
            }
        }
    }
    for (int e = tid; e < S::B_BYTES / 4; e += TC_THREADS) {
        reinterpret_cast<uint32_t *>(Bhi)[e] = 0u;
        reinterpret_cast<uint32_t *>(Blo)[e] = 0u;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    // the cosine matrix into TMEM: warp w writes rows (lanes) 32 w .. 32 w + 31
    if (warp < 4) {
        const int m = 32 * warp + lane;
        const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll 1
        for (int k0 = 0; k0 < K; k0 += 8) {
            uint32_t h[8], l[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = k0 + q;
                const double v = (m <= NY && k <= NY) ? tw2[(m * k) % (2 * NY)].x : 0.0;
                split_tf32(v, h[q], l[q]);
            }
            tmem_st8(trow + (uint32_t)k0, h);
            tmem_st8(trow + (uint32_t)(K + k0), l);
        }
        tmem_wait_st();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    uint32_t tph[2] = {0u, 0u}, mph[2] = {0u, 0u};
    bool ok = true;
    int pf = 0, pc0 = 0;
    for (int it = 0, t = blockIdx.x;; ++it, t += gridDim.x) {
        const int s = it & 1;
        const bool have = t < ntiles && ok;
        if (it > 0) {   // the previous tile's MMAs: B free, accumulator s ^ 1 ready
            ok = tc_wait(&mbar[s ^ 1], mph[s ^ 1], status) && ok;
            tc_fence_after();
        }
        if (have) {     // this tile's staging copy
            const bool got = kasync::mbar_wait(&tbar[s], tph[s]);
            tph[s] ^= 1u;
            if (tid == 0) pend[s] = false;
            if (!got) {
                if (lane == 0) atomicMax(status, KMM_ERR_TIMEOUT);
                ok = false;
            }
        }
        if (it > 0 && ok) {   // drain the previous tile's accumulator
            if (warp < 4) {
                const uint32_t ta = tmem + S::D0 + (uint32_t)(64 * (s ^ 1)) + ((uint32_t)(32 * warp) << 16);
                const int m = 32 * warp + lane;
#pragma unroll 1
                for (int cb = 0; cb < TC_CT; cb += 16) {
                    uint32_t r[32];
                    tmem_ld16(ta + (uint32_t)cb, r);
                    tmem_ld16(ta + (uint32_t)(32 + cb), r + 16);
                    tmem_wait_ld();
                    if (m <= NY) {
                        float4 *dst = reinterpret_cast<float4 *>(reinterpret_cast<float2 *>(out.p[pf]) +
                                                                 (size_t)m * ncols + pc0 + cb);
#pragma unroll
                        for (int c = 0; c < 16; c += 2)
                            dst[c / 2] = make_float4(__uint_as_float(r[c]), __uint_as_float(r[16 + c]),
                                                     __uint_as_float(r[c + 1]), __uint_as_float(r[17 + c]));
                    }
                }
            }
            if (NY == 128 && warp == 4) {
                double sre = 0.0, sim = 0.0;
#pragma unroll
                for (int w = 0; w < 8; ++w) {
                    sre += xn[(((s ^ 1) * 8 + w) * 32 + lane) * 2];
                    sim += xn[(((s ^ 1) * 8 + w) * 32 + lane) * 2 + 1];
                }
                reinterpret_cast<float2 *>(out.p[pf])[(size_t)NY * ncols + pc0 + lane] =
                    make_float2((float)sre, (float)sim);
            }
            tc_fence_before();
        }
        if (!have || !ok) break;
        const int f = t / tpf, c0 = (t - f * tpf) * TC_CT;
        // split the staged tile into B: lane = column, re in row lane, im in row 32 + lane
        const double2 *st = reinterpret_cast<const double2 *>(s ? stg1 : stg0) + (size_t)lane * NYP;
        double sre = 0.0, sim = 0.0;
#pragma unroll
        for (int gi = 0; gi < G; ++gi) {
            const int g = warp + 8 * gi;
            if (g < KG) {
                uint32_t phr[4], plr[4], phi[4], pli[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int n = 4 * g + q;
                    const double2 x = n < NYP ? st[n] : make_double2(0.0, 0.0);
                    split_tf32(x.x, phr[q], plr[q]);
                    split_tf32(x.y, phi[q], pli[q]);
                    if (NY == 128 && n <= NY) {
                        const double wgt = (n & 1) ? -1.0 : 1.0;
                        sre += wgt * x.x;
                        sim += wgt * x.y;
                    }
                }
                const uint32_t ore = kmaj_off(lane, 4 * g, TC_N), oim = kmaj_off(32 + lane, 4 * g, TC_N);
                *reinterpret_cast<uint4 *>(Bhi + ore) = make_uint4(phr[0], phr[1], phr[2], phr[3]);
                *reinterpret_cast<uint4 *>(Blo + ore) = make_uint4(plr[0], plr[1], plr[2], plr[3]);
                *reinterpret_cast<uint4 *>(Bhi + oim) = make_uint4(phi[0], phi[1], phi[2], phi[3]);
                *reinterpret_cast<uint4 *>(Blo + oim) = make_uint4(pli[0], pli[1], pli[2], pli[3]);
            }
        }
        if (NY == 128) {
            xn[((s * 8 + warp) * 32 + lane) * 2] = sre;
            xn[((s * 8 + warp) * 32 + lane) * 2 + 1] = sim;
        }
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            // staging buffer s has been read: the copy of the tile two ahead goes into it
            const int tn = t + 2 * gridDim.x;
            if (tn < ntiles) {
                kasync::mbar_expect_tx(&tbar[s], S::STG_BYTES);
                kasync::bulk_g2s(s ? stg1 : stg0, tile_src(tn), S::STG_BYTES, &tbar[s]);
                pend[s] = true;
            }
            const uint32_t d = tmem + S::D0 + (uint32_t)(64 * s);
            const uint32_t bh = su32(Bhi), bl = su32(Blo);
            uint32_t acc = 0u;
#pragma unroll 1
            for (int pass = 0; pass < 3; ++pass) {   // T_lo P_hi, T_hi P_lo, T_hi P_hi
                const uint32_t acol = pass == 0 ? (uint32_t)K : 0u, b0 = pass == 1 ? bl : bh;
#pragma unroll 1
                for (int ks = 0; ks < K / 8; ++ks) {
                    mma_tf32_ts(d, tmem + acol + (uint32_t)(8 * ks), sdesc(b0 + (uint32_t)(2 * ks * S::LBO_B), S::LBO_B, 128),
                                IDESC, acc);
                    acc = 1u;
                }
            }
            mma_commit(&mbar[s]);
        }
        pf = f;
        pc0 = c0;
    }
    // after a timeout: wait (bounded) for the MMAs and copies that may still be in flight
    if (!ok && tid == 0) {
        kasync::mbar_wait(&mbar[0], mph[0]);
        kasync::mbar_wait(&mbar[1], mph[1]);
        for (int b = 0; b < 2; ++b)
            if (pend[b]) kasync::mbar_wait(&tbar[b], tph[b]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

}  // namespace

// the y transforms of nf fields as tcgen05 GEMMs; KMM_ERR_UNSUPPORTED where they do not apply
// (ny not 32, 64, 96, 128; nz nxh not a multiple of 32; more than KMM_TC_MAXF fields)
int kmm_tc_dct(kmm_ctx *ctx, int dir, const void *const *in, void *const *out, int nf) {
    const int ny = ctx->ny, ncols = ctx->nz * ctx->nxh;
    if (!(ny == 32 || ny == 64 || ny == 96 || ny == 128) || ncols % TC_CT != 0 || nf <= 0 || nf > KMM_TC_MAXF)
        return KMM_ERR_UNSUPPORTED;
    TcFields fi;
    TcFieldsW fo;
    for (int m = 0; m < nf; ++m) {
        fi.p[m] = in[m];
        fo.p[m] = out[m];
    }
    int dev = 0, nsm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int ntiles = nf * (ncols / TC_CT);
    const int grid = ntiles < nsm ? ntiles : nsm;
    const double2 *tw = ctx->py2.tw;
#define TC(NN, DD)                                                                                           \
    do {                                                                                                     \
        const size_t sm = TcShape<NN>::SMEM;                                                                 \
        RET(kmm_smem_attr(ctx, (const void *)k_tcdct<NN, DD>, sm));                                         \
        k_tcdct<NN, DD><<<grid, TC_THREADS, sm, ctx->stream>>>(fi, fo, tw, nf, ncols, ctx->d_tcstat);       \
        CKL();                                                                                               \
        return KMM_OK;                                                                                       \
    } while (0)
#define TF(NN)                                                                                               \
    do {                                                                                                     \
        const size_t sm = TcFwd2<NN>::SMEM;                                                                  \
        RET(kmm_smem_attr(ctx, (const void *)k_tcdct_fwd2<NN>, sm));                                        \
        k_tcdct_fwd2<NN><<<grid, TC_THREADS, sm, ctx->stream>>>(fi, fo, tw, nf, ncols, ctx->d_tcstat);      \
        CKL();                                                                                               \
        return KMM_OK;                                                                                       \
    } while (0)
    if (dir == 0) {
        switch (ny) {
        case 32: TF(32);
        case 64: TF(64);
        case 96: TF(96);
        default: TF(128);
        }
    }
#undef TF
    switch (ny) {
    case 32: TC(32, 1);
    case 64: TC(64, 1);
    case 96: TC(96, 1);
    default: TC(128, 1);
    }
#undef TC
}
