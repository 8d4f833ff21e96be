// kmm_ztma.cu -- the fused step's z transforms (FP64 and the FP32 of the mixed form) with TMA
// tile copies.
//
// Work of the stage (solvers.f90:2578-2803 for the velocity, vorticity and scalar-gradient
// fields): from the y-physical base fields u, v, w, omega_y, du/dy, dw/dy [, c, dc/dy] in column
// layout [f][kx][kz][y], form the nine z-spectral inputs of the x stage (u v w wx wy wz [cx cy
// cz]; wx = dw/dy - i kz v, wz = i kx v - du/dy, cx = i kx c, cz = i kz c), zero-pad kz from nz to
// mz (modes j > nz/2 move to mz - nz + j), inverse c2c along z, and store Q[g][y][z][kx].
//
// Data movement: one CTA per (kx, 4 consecutive y).  Its thread 0 issues one tiled TMA load per
// base field (box: 4 y x all nz kz of one kx, 64 B rows, 64-byte swizzle), each on its own
// mbarrier, into a ring of three tile slots (below).  Four warps each form one y column per output
// field from the tiles and transform it (the warp-private compile-time FFT of kmm_fft.cuh); the
// results go to a [y][z] staging tile, which a tiled TMA store (box: 1 kx x mz z x 4 y) writes out
// while the next field is transformed.  62.5 KB of shared memory per CTA at mz = 192, so three
// CTAs share an SM.  (Forming the inputs inside the FFT's first stage and writing the staging tile
// from its last, as the FP32 form and the forward transforms do, made this kernel 11 % slower: the
// staging tile's barrier then falls between two FFT stages.  Keeping the FFT's output in registers
// across the barrier, as the forward transforms do, made it 8 % slower, and so did one FFT buffer
// per warp (the transform in place) with four CTAs per SM.)
//
// Every wait on an mbarrier is bounded (KMM_OPT_WAIT_LIMIT_MS, default 2 s of %globaltimer); a wait
// that runs out records KMM_ERR_TIMEOUT in the step's status word and the CTA finishes without the
// data.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "kmm_internal.cuh"
#include "kmm_async.cuh"
#include "kmm_fft.cuh"
#include "kmm_fused.cuh"

#define ZTM_YT 4       // y columns per CTA (= warps)
#define ZTM_WARPS ZTM_YT

namespace {

__device__ __forceinline__ uint32_t sm_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(bar)), "r"(bytes) : "memory");
}

// wait for phase `phase` of a barrier, at most the unit's limit (kasync_wait_ns, default 2 s)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase) { return kasync::mbar_wait(bar, phase); }

__device__ __forceinline__ void tma_load4(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                          uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(sm_addr(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(sm_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_store4(const CUtensorMap *tm, int c0, int c1, int c2, int c3, const void *src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(tm),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(sm_addr(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// the staging tile may be overwritten once every committed store has read it
__device__ __forceinline__ void tma_store_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// generic-proxy writes to shared memory -> visible to the TMA (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace

// tile element (kz, y) of one base field: 64-byte rows (4 y values of 16 B), 64-byte swizzle
// (16-byte chunk index XOR bits 7-8 of the byte offset)
__device__ __forceinline__ int ztile_idx(int kz, int y) { return kz * ZTM_YT + (y ^ ((kz >> 1) & 3)); }

// the z lengths whose FFT's last stage leaves output z = lane + 32 e in lane `lane` (its stride is
// a multiple of 32), so that the stage can write the lane's registers
template <int MZ>
constexpr bool ZREG = MZ % 32 == 0 && kct::stride(MZ, kct::nfac(MZ) - 1) % 32 == 0;

// The base-field tiles pass through a ring of ZB_SLOTS shared-memory slots: the q fields are formed
// in the order ZB_ORDER (each needs at most two base fields live), every base field is loaded into
// slot ZB_SLOT[f] -- fields 0, 2, 3 at the start, then ZB_AFTER[k] once step k has read the slot's
// previous tile -- so a CTA holds 3 tiles instead of 8 and three CTAs share an SM.
#define ZB_SLOTS 3
__device__ __forceinline__ int zb_order(int k) { return k == 1 ? 2 : k == 2 ? 4 : k == 3 ? 1 : k == 4 ? 3 : k == 7 ? 8 : k == 8 ? 7 : k; }
__device__ __forceinline__ int zb_slot(int f) { return (f == 0 || f == 1 || f == 7) ? 0 : (f == 2 || f == 5 || f == 6) ? 1 : 2; }
__device__ __forceinline__ int zb_after(int k) { return k == 0 ? 1 : k == 1 ? 5 : k == 2 ? 4 : k == 4 ? 6 : k == 5 ? 7 : -1; }

template <int MZ>
__global__ void __launch_bounds__(ZTM_WARPS * 32, 3)
    k_zb_tma(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
             const double *__restrict__ wavx, const double *__restrict__ wavz, const double2 *__restrict__ tw,
             int nbase, int nq, int *status) {
    constexpr int NZ = 2 * MZ / 3, NZH = NZ / 2, TILE = NZ * ZTM_YT;
    extern __shared__ unsigned char zsm_raw[];
    // 1024-byte aligned base: tiles [ZB_SLOTS][NZ][YT], FFT scratch [warps][2][MZ], stage [YT][MZ], barriers
    double2 *tiles = reinterpret_cast<double2 *>((reinterpret_cast<uintptr_t>(zsm_raw) + 1023) & ~(uintptr_t)1023);
    double2 *scr = tiles + (size_t)ZB_SLOTS * TILE;
    double2 *stage = scr + (size_t)ZTM_WARPS * 2 * MZ;
    uint64_t *bar = reinterpret_cast<uint64_t *>(stage + (size_t)ZTM_YT * MZ);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kx = blockIdx.x, y0 = blockIdx.y * ZTM_YT;
    if (threadIdx.x == 0) {
        for (int f = 0; f < nbase; ++f) mbar_init(&bar[f], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned issued = 0;   // base fields whose tile load has been issued (thread 0)
    auto load = [&](int f) {
        if (f < 0 || f >= nbase) return;
        mbar_expect_tx(&bar[f], (unsigned)(TILE * sizeof(double2)));
        tma_load4(tiles + (size_t)zb_slot(f) * TILE, &tin, 2 * y0, 0, kx, f, &bar[f]);
        issued |= 1u << f;
    };
    if (threadIdx.x == 0) {
        load(0);
        load(2);
        load(3);
    }
    const double kxv = wavx[kx];
    const int y = warp;
    double2 *a = scr + (size_t)warp * 2 * MZ, *b = a + MZ;
    unsigned ready = 0;
    bool ok = true;
    auto need = [&](int f) {
        if (!((ready >> f) & 1u)) {
            ok = mbar_wait(&bar[f], 0) && ok;
            ready |= 1u << f;
        }
    };
    for (int k = 0; k < nq; ++k) {
        const int g = zb_order(k);
        // base fields of q field g (u v w wx wy wz cx cy cz)
        int f0, f1 = -1;
        switch (g) {
        case 3: f0 = 5; f1 = 1; break;
        case 4: f0 = 3; break;
        case 5: f0 = 1; f1 = 4; break;
        case 6: case 8: f0 = 6; break;
        case 7: f0 = 7; break;
        default: f0 = g; break;
        }
        need(f0);
        if (f1 >= 0) need(f1);
        const double2 *t0 = tiles + (size_t)zb_slot(f0) * TILE, *t1 = f1 >= 0 ? tiles + (size_t)zb_slot(f1) * TILE : t0;
        for (int z = lane; z < MZ; z += 32) {
            double2 val = make_double2(0.0, 0.0);
            if (z < NZH || z >= MZ - NZH) {
                const int kz = z < NZH ? z : z - (MZ - NZ);
                const int ti = ztile_idx(kz, y);
                const double2 p = ok ? t0[ti] : val;
                switch (g) {
                case 3: {   // wx = dw/dy - i kz v
                    const double kzv = wavz[kz];
                    const double2 vv = ok ? t1[ti] : val;
                    val = make_double2(p.x + kzv * vv.y, p.y - kzv * vv.x);
                } break;
                case 5: {   // wz = i kx v - du/dy  (p = v, t1 = du/dy)
                    const double2 du = ok ? t1[ti] : val;
                    val = make_double2(-kxv * p.y - du.x, kxv * p.x - du.y);
                } break;
                case 6: val = make_double2(-kxv * p.y, kxv * p.x); break;   // i kx c
                case 8: {
                    const double kzv = wavz[kz];
                    val = make_double2(-kzv * p.y, kzv * p.x);   // i kz c
                } break;
                default: val = p; break;
                }
            }
            a[swz<double2>(z)] = val;
        }
        __syncwarp();
        const double2 *r = fft_warp_ct<double2, MZ, +1, 1, true>(a, b, tw);
        if (threadIdx.x == 0) tma_store_wait_read();   // the previous field's store has read the stage
        __syncthreads();
        for (int z = lane; z < MZ; z += 32) stage[(size_t)y * MZ + z] = r[swz<double2>(z)];
        fence_async_smem();   // also orders this step's tile reads before the next load into the slot
        __syncthreads();
        if (threadIdx.x == 0) {
            tma_store4(&tout, 2 * kx, 0, y0, g, stage);
            load(zb_after(k));
        }
    }
    if (threadIdx.x == 0) {
        tma_store_wait_read();   // shared memory must outlive the last store's read
        // after a timeout, wait (bounded) for any tile load still in flight before the CTA exits
        if (!ok)
            for (int f = 0; f < nbase; ++f)
                if (((issued >> f) & 1u) && !((ready >> f) & 1u)) mbar_wait(&bar[f], 0);
    }
    if (!ok && lane == 0) atomicMax(status, KMM_ERR_TIMEOUT);
}

// Forward z transform of the x stage's outputs (solvers.f90:3180-3273): R[o][y][z][kx] -> c2c
// along z, truncate to nz (mode j > nz/2 from mz - nz + j), divide by mx mz, store in column
// layout Yo[o][kx][kz][y].  One CTA per (kx, 4 consecutive y): one TMA load per field (box 1 kx x
// mz z x 4 y, rows of 16 B), one warp per y column, and a TMA store per field of the [kz][4 y]
// result tile (64 B rows, 64-byte swizzle: the layout of the inverse transform's input tiles).
// The input tiles pass through two shared-memory slots: fields 0 and 1 are loaded at the start,
// field o + 2 into slot o mod 2 once field o has been read, so three CTAs share an SM.  The first
// FFT stage reads its column straight from the tile.
#define ZF_SLOTS 2
template <int MZ>
__global__ void __launch_bounds__(ZTM_WARPS * 32, 3)
    k_zf_tma(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
             const double2 *__restrict__ tw, int nout, double scale, int *status) {
    constexpr int NZ = 2 * MZ / 3, NZH = NZ / 2, TIN = MZ * ZTM_YT, TOUT = NZ * ZTM_YT;
    extern __shared__ unsigned char zsm_raw[];
    // 1024-byte aligned: out stage [NZ][YT] (swizzled), in tiles [ZF_SLOTS][YT][MZ], scratch, barriers
    double2 *stage = reinterpret_cast<double2 *>((reinterpret_cast<uintptr_t>(zsm_raw) + 1023) & ~(uintptr_t)1023);
    double2 *tiles = stage + TOUT;
    double2 *scr = tiles + (size_t)ZF_SLOTS * TIN;
    uint64_t *bar = reinterpret_cast<uint64_t *>(scr + (size_t)ZTM_WARPS * 2 * MZ);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kx = blockIdx.x, y0 = blockIdx.y * ZTM_YT;
    if (threadIdx.x == 0) {
        for (int o = 0; o < nout; ++o) mbar_init(&bar[o], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned issued = 0, ready = 0;
    auto load = [&](int o) {
        if (o >= nout) return;
        mbar_expect_tx(&bar[o], (unsigned)(TIN * sizeof(double2)));
        tma_load4(tiles + (size_t)(o % ZF_SLOTS) * TIN, &tin, 2 * kx, 0, y0, o, &bar[o]);
        issued |= 1u << o;
    };
    if (threadIdx.x == 0) {
        load(0);
        load(1);
    }
    const int y = warp;
    double2 *a = scr + (size_t)warp * 2 * MZ, *b = a + MZ;
    bool ok = true;
    for (int o = 0; o < nout; ++o) {
        ok = mbar_wait(&bar[o], 0) && ok;
        ready |= 1u << o;
        const double2 *t = tiles + (size_t)(o % ZF_SLOTS) * TIN + (size_t)y * MZ;
        // the first FFT stage reads the tile row, the last writes the scratch buffer it does not read
        auto ld = [&](int z) { return ok ? t[z] : make_double2(0.0, 0.0); };
        auto pre = [] {};
        if constexpr (ZREG<MZ>) {
            // the last stage leaves output z = lane + 32 e in lane `lane`: registers, truncated
            // into the staging tile once the previous field's store has read it
            double2 rv[MZ / 32];
            auto st = [&](int z, double2 v) { rv[z >> 5] = v; };
            fft_warp_ct_io<double2, MZ, -1>(ld, st, pre, a, b, tw);
            if (threadIdx.x == 0) tma_store_wait_read();   // the previous field's store has read the stage
            __syncthreads();
#pragma unroll
            for (int e = 0; e < MZ / 32; ++e) {
                const int z = lane + 32 * e;
                if (z < NZH || z >= MZ - NZH) {
                    const int kz = z < NZH ? z : z - (MZ - NZ);
                    stage[ztile_idx(kz, y)] = make_double2(rv[e].x / scale, rv[e].y / scale);   // the reference's /(mx mz)
                }
            }
        } else {
            double2 *r = kct::nfac(MZ) % 2 == 0 ? b : a;
            auto st = [&](int z, double2 v) { r[swz<double2>(z)] = v; };
            fft_warp_ct_io<double2, MZ, -1>(ld, st, pre, a, b, tw);
            __syncwarp();
            if (threadIdx.x == 0) tma_store_wait_read();   // the previous field's store has read the stage
            __syncthreads();
            for (int kz = lane; kz < NZ; kz += 32) {
                const double2 v = r[swz<double2>(kz < NZH ? kz : (MZ - NZ) + kz)];
                stage[ztile_idx(kz, y)] = make_double2(v.x / scale, v.y / scale);   // the reference's /(mx mz)
            }
        }
        fence_async_smem();   // also orders this field's tile reads before the next load into the slot
        __syncthreads();
        if (threadIdx.x == 0) {
            tma_store4(&tout, 2 * y0, 0, kx, o, stage);
            load(o + ZF_SLOTS);
        }
    }
    if (threadIdx.x == 0) {
        tma_store_wait_read();
        if (!ok)
            for (int o = 0; o < nout; ++o)
                if (((issued >> o) & 1u) && !((ready >> o) & 1u)) mbar_wait(&bar[o], 0);
    }
    if (!ok && lane == 0) atomicMax(status, KMM_ERR_TIMEOUT);
}

// ---------------------------------------------------------------------------
// FP32 forms (mixed precision: float2 intermediates).  A TMA row must hold at least 16 bytes, so a
// CTA covers two kx (one 16-byte row of the [y][z][kx] planes) and 4 y: 8 columns, one warp each.
// Column tiles [kx][kz][4 y] have 32-byte rows with the 32-byte swizzle (16-byte chunk index XOR
// bit 7 of the byte offset); FP32 columns are padded to an even length (col_ld) so that each
// starts on a 16-byte boundary.  Same work and operation order as k_zb2 / k_zf2 with float2.
// ---------------------------------------------------------------------------
#define ZT32_KX 2
#define ZT32_WARPS (ZT32_KX * ZTM_YT)

// float2 element (kz, y) of a [kz][4 y] tile with 32-byte rows, 32-byte swizzle
__device__ __forceinline__ int ztile32_idx(int kz, int y) {
    return kz * ZTM_YT + ((((y >> 1) ^ ((kz >> 2) & 1)) << 1) | (y & 1));
}

template <int MZ>
__global__ void __launch_bounds__(ZT32_WARPS * 32, 2)
    k_zb_tma32(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
               const double *__restrict__ wavx, const double *__restrict__ wavz, const float2 *__restrict__ tw,
               int nbase, int nq, int *status) {
    constexpr int NZ = 2 * MZ / 3, NZH = NZ / 2, TILE = NZ * ZTM_YT;   // float2 per (field, kx) tile
    extern __shared__ unsigned char zsm_raw[];
    // tiles [nbase][KX][NZ][YT], scratch [warps][2][MZ], stage [YT][MZ][KX], barriers
    float2 *tiles = reinterpret_cast<float2 *>((reinterpret_cast<uintptr_t>(zsm_raw) + 1023) & ~(uintptr_t)1023);
    float2 *scr = tiles + (size_t)nbase * ZT32_KX * TILE;
    float2 *stage = scr + (size_t)ZT32_WARPS * 2 * MZ;
    uint64_t *bar = reinterpret_cast<uint64_t *>(stage + (size_t)ZTM_YT * MZ * ZT32_KX);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kx0 = blockIdx.x * ZT32_KX, y0 = blockIdx.y * ZTM_YT;
    const int kl = warp / ZTM_YT, y = warp % ZTM_YT, kx = kx0 + kl;
    if (threadIdx.x == 0) {
        for (int f = 0; f < nbase; ++f) mbar_init(&bar[f], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int f = 0; f < nbase; ++f) {
            mbar_expect_tx(&bar[f], (unsigned)(ZT32_KX * TILE * sizeof(float2)));
            tma_load4(tiles + (size_t)f * ZT32_KX * TILE, &tin, 2 * y0, 0, kx0, f, &bar[f]);
        }
    }
    const float kxv = (float)wavx[kx];
    float2 *a = scr + (size_t)warp * 2 * MZ, *b = a + MZ;
    unsigned ready = 0;
    bool ok = true;
    auto need = [&](int f) {
        if (!((ready >> f) & 1u)) {
            ok = mbar_wait(&bar[f], 0) && ok;
            ready |= 1u << f;
        }
    };
    for (int g = 0; g < nq; ++g) {
        int f0, f1 = -1;
        switch (g) {
        case 3: f0 = 5; f1 = 1; break;
        case 4: f0 = 3; break;
        case 5: f0 = 1; f1 = 4; break;
        case 6: case 8: f0 = 6; break;
        case 7: f0 = 7; break;
        default: f0 = g; break;
        }
        need(f0);
        if (f1 >= 0) need(f1);
        const float2 *t0 = tiles + ((size_t)f0 * ZT32_KX + kl) * TILE;
        const float2 *t1 = f1 >= 0 ? tiles + ((size_t)f1 * ZT32_KX + kl) * TILE : t0;
        auto ld = [&](int z) {
            float2 val = make_float2(0.f, 0.f);
            if (z < NZH || z >= MZ - NZH) {
                const int kz = z < NZH ? z : z - (MZ - NZ);
                const int ti = ztile32_idx(kz, y);
                const float2 p = ok ? t0[ti] : val;
                switch (g) {
                case 3: {   // wx = dw/dy - i kz v
                    const float kzv = (float)wavz[kz];
                    const float2 vv = ok ? t1[ti] : val;
                    val = make_float2(p.x + kzv * vv.y, p.y - kzv * vv.x);
                } break;
                case 5: {   // wz = i kx v - du/dy
                    const float2 du = ok ? t1[ti] : val;
                    val = make_float2(-kxv * p.y - du.x, kxv * p.x - du.y);
                } break;
                case 6: val = make_float2(-kxv * p.y, kxv * p.x); break;
                case 8: {
                    const float kzv = (float)wavz[kz];
                    val = make_float2(-kzv * p.y, kzv * p.x);
                } break;
                default: val = p; break;
                }
            }
            return val;
        };
        auto pre = [&]() {
            if (threadIdx.x == 0) tma_store_wait_read();
            __syncthreads();
        };
        auto st = [&](int z, float2 v) { stage[((size_t)y * MZ + z) * ZT32_KX + kl] = v; };
        fft_warp_ct_io<float2, MZ, +1>(ld, st, pre, a, b, tw);
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) tma_store4(&tout, 2 * kx0, 0, y0, g, stage);
    }
    if (threadIdx.x == 0) tma_store_wait_read();
    if (!ok && lane == 0) atomicMax(status, KMM_ERR_TIMEOUT);
}

template <int MZ>
__global__ void __launch_bounds__(ZT32_WARPS * 32, 2)
    k_zf_tma32(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout,
               const float2 *__restrict__ tw, int nout, float rscale, int *status) {
    constexpr int NZ = 2 * MZ / 3, NZH = NZ / 2, TIN = MZ * ZTM_YT * ZT32_KX, TOUT = NZ * ZTM_YT;
    extern __shared__ unsigned char zsm_raw[];
    // out stage [KX][NZ][YT] (swizzled), in tiles [nout][YT][MZ][KX], scratch, barriers
    float2 *stage = reinterpret_cast<float2 *>((reinterpret_cast<uintptr_t>(zsm_raw) + 1023) & ~(uintptr_t)1023);
    float2 *tiles = stage + (size_t)ZT32_KX * TOUT;
    float2 *scr = tiles + (size_t)nout * TIN;
    uint64_t *bar = reinterpret_cast<uint64_t *>(scr + (size_t)ZT32_WARPS * 2 * MZ);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kx0 = blockIdx.x * ZT32_KX, y0 = blockIdx.y * ZTM_YT;
    const int kl = warp / ZTM_YT, y = warp % ZTM_YT;
    if (threadIdx.x == 0) {
        for (int o = 0; o < nout; ++o) mbar_init(&bar[o], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int o = 0; o < nout; ++o) {
            mbar_expect_tx(&bar[o], (unsigned)(TIN * sizeof(float2)));
            tma_load4(tiles + (size_t)o * TIN, &tin, 2 * kx0, 0, y0, o, &bar[o]);
        }
    }
    float2 *a = scr + (size_t)warp * 2 * MZ, *b = a + MZ;
    bool ok = true;
    for (int o = 0; o < nout; ++o) {
        ok = mbar_wait(&bar[o], 0) && ok;
        const float2 *t = tiles + (size_t)o * TIN;
        auto ld = [&](int z) { return ok ? t[((size_t)y * MZ + z) * ZT32_KX + kl] : make_float2(0.f, 0.f); };
        auto pre = [] {};
        if constexpr (ZREG<MZ>) {
            float2 rv[MZ / 32];
            auto st = [&](int z, float2 v) { rv[z >> 5] = v; };
            fft_warp_ct_io<float2, MZ, -1>(ld, st, pre, a, b, tw);
            if (threadIdx.x == 0) tma_store_wait_read();
            __syncthreads();
#pragma unroll
            for (int e = 0; e < MZ / 32; ++e) {
                const int z = lane + 32 * e;
                if (z < NZH || z >= MZ - NZH) {
                    const int kz = z < NZH ? z : z - (MZ - NZ);
                    stage[(size_t)kl * TOUT + ztile32_idx(kz, y)] = make_float2(rv[e].x * rscale, rv[e].y * rscale);
                }
            }
        } else {
            float2 *r = kct::nfac(MZ) % 2 == 0 ? b : a;
            auto st = [&](int z, float2 v) { r[swz<float2>(z)] = v; };
            fft_warp_ct_io<float2, MZ, -1>(ld, st, pre, a, b, tw);
            __syncwarp();
            if (threadIdx.x == 0) tma_store_wait_read();
            __syncthreads();
            for (int kz = lane; kz < NZ; kz += 32) {
                const float2 v = r[swz<float2>(kz < NZH ? kz : (MZ - NZ) + kz)];
                stage[(size_t)kl * TOUT + ztile32_idx(kz, y)] = make_float2(v.x * rscale, v.y * rscale);
            }
        }
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) tma_store4(&tout, 2 * y0, 0, kx0, o, stage);
    }
    if (threadIdx.x == 0) tma_store_wait_read();
    if (!ok && lane == 0) atomicMax(status, KMM_ERR_TIMEOUT);
}

// ---------------------------------------------------------------------------
// host side: tensor maps (cached per context, re-encoded when a buffer or size changes) and the
// launches
// ---------------------------------------------------------------------------
struct ZtmaPair {
    CUtensorMap in, out;
    const void *src, *dst;
    int nyp, nz, nxh, mz, nsrc, ndst, f32;
};
struct ZtmaMaps {
    ZtmaPair inv, fwd;   // inverse: Y (base fields) -> Q; forward: R -> Yo
};

static PFN_cuTensorMapEncodeTiled_v12000 ztma_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = NULL;
    if (!fn) {
        void *p = NULL;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// this unit's bounded-wait limit on the current device (KMM_OPT_WAIT_LIMIT_MS)
int kmm_ztma_set_wait_limit(unsigned long long ns) { return kasync::kasync_set_wait_limit(ns) == cudaSuccess ? 0 : 1; }

void kmm_ztma_release(kmm_ctx *ctx) {
    free(ctx->ztma);
    ctx->ztma = NULL;
}

bool kmm_ztma_supported(const kmm_ctx *ctx) {
    const int mz = ctx->mz;
    return ctx->use_ztma && (mz == 48 || mz == 96 || mz == 144 || mz == 192);
}

static ZtmaMaps *ztma_maps(kmm_ctx *ctx) {
    if (!ctx->ztma) {
        void *m = NULL;
        if (posix_memalign(&m, 64, sizeof(ZtmaMaps))) return NULL;   // CUtensorMap: 64-byte alignment
        memset(m, 0, sizeof(ZtmaMaps));
        ctx->ztma = m;
    }
    return (ZtmaMaps *)ctx->ztma;
}

static bool pair_current(const ZtmaPair &P, const void *src, const void *dst, const kmm_ctx *ctx, int nsrc, int ndst,
                         int f32) {
    return P.src == src && P.dst == dst && P.nyp == ctx->nyp && P.nz == ctx->nz && P.nxh == ctx->nxh &&
           P.mz == ctx->mz && P.nsrc == nsrc && P.ndst == ndst && P.f32 == f32;
}

// column layout [f][kx][kz][y] as reals (a complex value is 2 reals; FP32 columns padded to an
// even length): (2 nyp, nz, nxh, nf); FP64 box (2 YT, nz, 1, 1) with 64-byte rows and swizzle,
// FP32 box (2 YT, nz, 2, 1) with 32-byte rows and swizzle
static CUresult map_columns(PFN_cuTensorMapEncodeTiled_v12000 enc, CUtensorMap *m, const void *base,
                            const kmm_ctx *ctx, int nf, CUtensorMapL2promotion l2, bool f32) {
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh;
    const cuuint64_t cb = f32 ? (cuuint64_t)8 * col_ld<float2>(nyp) : (cuuint64_t)16 * nyp;   // column bytes
    cuuint64_t d[4] = {(cuuint64_t)2 * nyp, (cuuint64_t)nz, (cuuint64_t)nxh, (cuuint64_t)nf};
    cuuint64_t st[3] = {cb, (cuuint64_t)nz * cb, (cuuint64_t)nz * nxh * cb};
    cuuint32_t box[4] = {2 * ZTM_YT, (cuuint32_t)nz, f32 ? (cuuint32_t)ZT32_KX : 1u, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)base, d, st, box,
               es, CU_TENSOR_MAP_INTERLEAVE_NONE, f32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B, l2,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

// plane layout [f][y][z][kx] as reals: (2 nxh, mz, nyp, nf), box (16 bytes of kx, mz, YT, 1): one
// kx in FP64, two in FP32; no swizzle
static CUresult map_planes(PFN_cuTensorMapEncodeTiled_v12000 enc, CUtensorMap *m, const void *base,
                           const kmm_ctx *ctx, int nf, CUtensorMapL2promotion l2, bool f32) {
    const int nyp = ctx->nyp, nxh = ctx->nxh, mz = ctx->mz;
    const cuuint64_t eb = f32 ? 8 : 16;   // bytes per complex value
    cuuint64_t d[4] = {(cuuint64_t)2 * nxh, (cuuint64_t)mz, (cuuint64_t)nyp, (cuuint64_t)nf};
    cuuint64_t st[3] = {(cuuint64_t)nxh * eb, (cuuint64_t)mz * nxh * eb, (cuuint64_t)nyp * mz * nxh * eb};
    cuuint32_t box[4] = {f32 ? 4u : 2u, (cuuint32_t)mz, ZTM_YT, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)base, d, st, box,
               es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, l2, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

static int pair_encode(kmm_ctx *ctx, ZtmaPair &P, bool inverse, const void *src, const void *dst, int nsrc, int ndst,
                       bool f32) {
    if (pair_current(P, src, dst, ctx, nsrc, ndst, f32 ? 1 : 0)) return KMM_OK;
    PFN_cuTensorMapEncodeTiled_v12000 enc = ztma_encoder();
    if (!enc) {
        kmm_set_error(ctx, "cuTensorMapEncodeTiled is not available from the driver");
        return KMM_ERR_CUDA;
    }
    CUresult r1, r2;
    if (inverse) {
        r1 = map_columns(enc, &P.in, src, ctx, nsrc, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, f32);
        r2 = map_planes(enc, &P.out, dst, ctx, ndst, CU_TENSOR_MAP_L2_PROMOTION_NONE, f32);
    } else {
        r1 = map_planes(enc, &P.in, src, ctx, nsrc, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, f32);
        r2 = map_columns(enc, &P.out, dst, ctx, ndst, CU_TENSOR_MAP_L2_PROMOTION_NONE, f32);
    }
    if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS) {
        kmm_set_error(ctx, "tensor map encoding failed (%d, %d)", (int)r1, (int)r2);
        P.src = NULL;
        return KMM_ERR_CUDA;
    }
    P.src = src; P.dst = dst; P.nsrc = nsrc; P.ndst = ndst; P.f32 = f32 ? 1 : 0;
    P.nyp = ctx->nyp; P.nz = ctx->nz; P.nxh = ctx->nxh; P.mz = ctx->mz;
    return KMM_OK;
}

int kmm_zb_tma(kmm_ctx *ctx, const double2 *yp, double2 *q, int nbase, int nq, const double2 *tw) {
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mz = ctx->mz;
    ZtmaMaps *M = ztma_maps(ctx);
    if (!M) return KMM_ERR_NOMEM;
    RET(pair_encode(ctx, M->inv, true, yp, q, nbase, nq, false));
    const size_t smem = 1024 + sizeof(double2) * ((size_t)ZB_SLOTS * nz * ZTM_YT + (size_t)ZTM_WARPS * 2 * mz +
                                                  (size_t)ZTM_YT * mz) + 8 * sizeof(uint64_t);
    const dim3 grid(nxh, (nyp + ZTM_YT - 1) / ZTM_YT);
#define ZTM_LAUNCH(MM)                                                                                           \
    do {                                                                                                         \
        RET(kmm_smem_attr(ctx, (const void *)k_zb_tma<MM>, smem));                                               \
        k_zb_tma<MM><<<grid, ZTM_WARPS * 32, smem, ctx->stream>>>(M->inv.in, M->inv.out, ctx->d_wavx, ctx->d_wavz, \
                                                                  tw, nbase, nq, ctx->d_status);                 \
    } while (0)
    switch (mz) {
    case 48: ZTM_LAUNCH(48); break;
    case 96: ZTM_LAUNCH(96); break;
    case 144: ZTM_LAUNCH(144); break;
    case 192: ZTM_LAUNCH(192); break;
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef ZTM_LAUNCH
    return KMM_OK;   // the caller checks the launch and counts it
}

int kmm_zf_tma(kmm_ctx *ctx, const double2 *r, double2 *yo, int nout, const double2 *tw) {
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mz = ctx->mz;
    ZtmaMaps *M = ztma_maps(ctx);
    if (!M) return KMM_ERR_NOMEM;
    RET(pair_encode(ctx, M->fwd, false, r, yo, nout, nout, false));
    const size_t smem = 1024 + sizeof(double2) * ((size_t)nz * ZTM_YT + (size_t)ZF_SLOTS * mz * ZTM_YT +
                                                  (size_t)ZTM_WARPS * 2 * mz) + 8 * sizeof(uint64_t);
    const dim3 grid(nxh, (nyp + ZTM_YT - 1) / ZTM_YT);
    const double scale = (double)ctx->mx * (double)mz;
#define ZTF_LAUNCH(MM)                                                                                      \
    do {                                                                                                    \
        RET(kmm_smem_attr(ctx, (const void *)k_zf_tma<MM>, smem));                                          \
        k_zf_tma<MM><<<grid, ZTM_WARPS * 32, smem, ctx->stream>>>(M->fwd.in, M->fwd.out, tw, nout, scale,   \
                                                                  ctx->d_status);                          \
    } while (0)
    switch (mz) {
    case 48: ZTF_LAUNCH(48); break;
    case 96: ZTF_LAUNCH(96); break;
    case 144: ZTF_LAUNCH(144); break;
    case 192: ZTF_LAUNCH(192); break;
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef ZTF_LAUNCH
    return KMM_OK;   // the caller checks the launch and counts it
}

// FP32 forms (mixed precision)
int kmm_zb_tma32(kmm_ctx *ctx, const float2 *yp, float2 *q, int nbase, int nq, const float2 *tw) {
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mz = ctx->mz;
    if (nxh % ZT32_KX) return KMM_ERR_UNSUPPORTED;
    ZtmaMaps *M = ztma_maps(ctx);
    if (!M) return KMM_ERR_NOMEM;
    RET(pair_encode(ctx, M->inv, true, yp, q, nbase, nq, true));
    const size_t smem = 1024 + sizeof(float2) * ((size_t)nbase * ZT32_KX * nz * ZTM_YT + (size_t)ZT32_WARPS * 2 * mz +
                                                 (size_t)ZTM_YT * mz * ZT32_KX) + 8 * sizeof(uint64_t);
    const dim3 grid(nxh / ZT32_KX, (nyp + ZTM_YT - 1) / ZTM_YT);
#define ZTM32_LAUNCH(MM)                                                                                      \
    do {                                                                                                      \
        RET(kmm_smem_attr(ctx, (const void *)k_zb_tma32<MM>, smem));                                          \
        k_zb_tma32<MM><<<grid, ZT32_WARPS * 32, smem, ctx->stream>>>(M->inv.in, M->inv.out, ctx->d_wavx,      \
                                                                     ctx->d_wavz, tw, nbase, nq, ctx->d_status); \
    } while (0)
    switch (mz) {
    case 48: ZTM32_LAUNCH(48); break;
    case 96: ZTM32_LAUNCH(96); break;
    case 144: ZTM32_LAUNCH(144); break;
    case 192: ZTM32_LAUNCH(192); break;
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef ZTM32_LAUNCH
    return KMM_OK;   // the caller checks the launch and counts it
}

int kmm_zf_tma32(kmm_ctx *ctx, const float2 *r, float2 *yo, int nout, const float2 *tw) {
    const int nyp = ctx->nyp, nz = ctx->nz, nxh = ctx->nxh, mz = ctx->mz;
    if (nxh % ZT32_KX) return KMM_ERR_UNSUPPORTED;
    ZtmaMaps *M = ztma_maps(ctx);
    if (!M) return KMM_ERR_NOMEM;
    RET(pair_encode(ctx, M->fwd, false, r, yo, nout, nout, true));
    const size_t smem = 1024 + sizeof(float2) * ((size_t)ZT32_KX * nz * ZTM_YT + (size_t)nout * mz * ZTM_YT * ZT32_KX +
                                                 (size_t)ZT32_WARPS * 2 * mz) + 8 * sizeof(uint64_t);
    const dim3 grid(nxh / ZT32_KX, (nyp + ZTM_YT - 1) / ZTM_YT);
    const float rscale = (float)(1.0 / ((double)ctx->mx * (double)mz));
#define ZTF32_LAUNCH(MM)                                                                                    \
    do {                                                                                                    \
        RET(kmm_smem_attr(ctx, (const void *)k_zf_tma32<MM>, smem));                                        \
        k_zf_tma32<MM><<<grid, ZT32_WARPS * 32, smem, ctx->stream>>>(M->fwd.in, M->fwd.out, tw, nout, rscale, \
                                                                     ctx->d_status);                        \
    } while (0)
    switch (mz) {
    case 48: ZTF32_LAUNCH(48); break;
    case 96: ZTF32_LAUNCH(96); break;
    case 144: ZTF32_LAUNCH(144); break;
    case 192: ZTF32_LAUNCH(192); break;
    default: return KMM_ERR_UNSUPPORTED;
    }
#undef ZTF32_LAUNCH
    return KMM_OK;
}
