// kmm_fft.cuh -- warp-private Stockham FFTs specialised at compile time for one transform length.
//
// The runtime-plan FFT (fft_warp) spends most of its instructions on integer division, modulo and
// radix dispatch.  Here the length N is a template argument: the radix sequence (8, 4, 2, 3, 5,
// the order of kmm_plan_r8) and every stride are constants, the butterfly loop over j = lane +
// 32 it has a fixed trip count, j % Ns and j / Ns become shifts for the power-of-two strides,
// and the twiddle index r k tstep never reaches N, so it needs no modulo.  The arithmetic per
// butterfly is the same as fft_warp's: twiddle multiply of inputs r >= 1, then the radix-R DFT.
//
// C is double2 or float2; the twiddle table holds exp(-2 pi i m / N), m = 0..N-1, in the same type.
#pragma once

#include "kmm_internal.cuh"

namespace kct {

__host__ __device__ constexpr int radix_at(int r) { return r == 0 ? 8 : r == 1 ? 4 : r == 2 ? 2 : r == 3 ? 3 : 5; }

// number of factors of n over radices 8, 4, 2, 3, 5 (-1 when n has another prime factor)
__host__ __device__ constexpr int nfac(int n) {
    int c = 0;
    for (int r = 0; r < 5; ++r)
        while (n % radix_at(r) == 0) {
            n /= radix_at(r);
            ++c;
        }
    return n == 1 ? c : -1;
}

// f-th factor
__host__ __device__ constexpr int fac(int n, int f) {
    int c = 0;
    for (int r = 0; r < 5; ++r)
        while (n % radix_at(r) == 0) {
            if (c == f) return radix_at(r);
            n /= radix_at(r);
            ++c;
        }
    return 1;
}

// product of the first f factors (the Stockham stride Ns of stage f)
__host__ __device__ constexpr int stride(int n, int f) {
    int p = 1;
    for (int i = 0; i < f; ++i) p *= fac(n, i);
    return p;
}

// ---- complex arithmetic on double2 / float2
template <typename C>
struct Real;
template <>
struct Real<double2> {
    typedef double T;
};
template <>
struct Real<float2> {
    typedef float T;
};

template <typename C>
__device__ __forceinline__ C mk(typename Real<C>::T x, typename Real<C>::T y) {
    C c;
    c.x = x;
    c.y = y;
    return c;
}
template <typename C>
__device__ __forceinline__ C add(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C sub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C>
__device__ __forceinline__ C mul(C a, C b) { return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C>
__device__ __forceinline__ C scl(C a, typename Real<C>::T s) { return mk<C>(a.x * s, a.y * s); }

}   // namespace kct

// Shared-memory swizzle of the FFT buffers: element x of a 128-byte row r = x / E (E = 8 double2
// or 16 float2 per row) is stored at column (x mod E) xor (r mod E).  Unit-stride runs, the
// stride-R writes of a radix-R stage and the blocked K-per-lane column accesses then spread over
// all banks.  Callers that pass SWZ = true to fft_warp_ct write the input and read the output
// through swz<C>().
template <typename C>
__device__ __forceinline__ int swz(int x) {
    constexpr int RB = sizeof(C) == 16 ? 3 : 4;
    constexpr int RM = (1 << RB) - 1;
    return x ^ ((x >> RB) & RM);
}

namespace kct {

// radix-R DFTs, X_q = sum_r v_r exp(S 2 pi i r q / R); the same operation sequence as radix_dft /
// radix8_dft of the runtime FFT
template <typename C, int R, int S>
struct Dft;

template <typename C, int S>
struct Dft<C, 2, S> {
    static __device__ __forceinline__ void run(C *v) {
        const C a0 = v[0], a1 = v[1];
        v[0] = add(a0, a1);
        v[1] = sub(a0, a1);
    }
};

template <typename C, int S>
struct Dft<C, 4, S> {
    static __device__ __forceinline__ void run(C *v) {
        const C a0 = add(v[0], v[2]), a1 = sub(v[0], v[2]);
        const C b0 = add(v[1], v[3]);
        const C d = sub(v[1], v[3]);
        const C b1 = S < 0 ? mk<C>(d.y, -d.x) : mk<C>(-d.y, d.x);   // S i d
        v[0] = add(a0, b0);
        v[1] = add(a1, b1);
        v[2] = sub(a0, b0);
        v[3] = sub(a1, b1);
    }
};

template <typename C, int S>
struct Dft<C, 3, S> {
    static __device__ __forceinline__ void run(C *v) {
        typedef typename Real<C>::T T;
        const T s3 = (T)0.86602540378443864676 * (T)S;
        const C t1 = add(v[1], v[2]);
        const C t2 = sub(v[0], scl(t1, (T)0.5));
        const C d = sub(v[1], v[2]);
        const C t3 = mk<C>(s3 * d.x, s3 * d.y);
        const C o0 = add(v[0], t1);
        v[1] = mk<C>(t2.x - t3.y, t2.y + t3.x);
        v[2] = mk<C>(t2.x + t3.y, t2.y - t3.x);
        v[0] = o0;
    }
};

template <typename C, int S>
struct Dft<C, 5, S> {
    static __device__ __forceinline__ void run(C *v) {
        typedef typename Real<C>::T T;
        const T c5a = (T)0.30901699437494742410, c5b = (T)-0.80901699437494742410;
        const T s5a = (T)0.95105651629515357212 * (T)S, s5b = (T)0.58778525229247312917 * (T)S;
        const C t1 = add(v[1], v[4]), t2 = add(v[2], v[3]);
        const C t3 = sub(v[1], v[4]), t4 = sub(v[2], v[3]);
        const C o0 = add(v[0], add(t1, t2));
        const C r1 = add(v[0], add(scl(t1, c5a), scl(t2, c5b)));
        const C r2 = add(v[0], add(scl(t1, c5b), scl(t2, c5a)));
        const C m1 = add(scl(t3, s5a), scl(t4, s5b));
        const C m2 = sub(scl(t3, s5b), scl(t4, s5a));
        const C i1 = mk<C>(-m1.y, m1.x), i2 = mk<C>(-m2.y, m2.x);
        v[0] = o0;
        v[1] = add(r1, i1);
        v[4] = sub(r1, i1);
        v[2] = add(r2, i2);
        v[3] = sub(r2, i2);
    }
};

template <typename C, int S>
struct Dft<C, 8, S> {
    static __device__ __forceinline__ void run(C *v) {
        typedef typename Real<C>::T T;
        C e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        Dft<C, 4, S>::run(e);
        Dft<C, 4, S>::run(o);
        const T h = (T)0.70710678118654752440;
        const C t1 = mk<C>(h * (o[1].x - (T)S * o[1].y), h * (o[1].y + (T)S * o[1].x));
        const C t2 = S < 0 ? mk<C>(o[2].y, -o[2].x) : mk<C>(-o[2].y, o[2].x);
        const C t3 = mk<C>(h * (-o[3].x - (T)S * o[3].y), h * (-o[3].y + (T)S * o[3].x));
        v[0] = add(e[0], o[0]);
        v[4] = sub(e[0], o[0]);
        v[1] = add(e[1], t1);
        v[5] = sub(e[1], t1);
        v[2] = add(e[2], t2);
        v[6] = sub(e[2], t2);
        v[3] = add(e[3], t3);
        v[7] = sub(e[3], t3);
    }
};

// one Stockham stage: butterflies j = 0..N/R-1 of each of the NQ sequences (stored N apart)
// spread over the 32 lanes
template <typename C, int N, int F, int S, int NQ, bool SWZ, int TWS>
__device__ __forceinline__ void stage(const C *__restrict__ src, C *__restrict__ dst, const C *__restrict__ tw,
                                      int lane) {
    constexpr int R = fac(N, F);
    constexpr int NS = stride(N, F);
    constexpr int NR = N / R;
    constexpr int TSTEP = N / (NS * R);
    constexpr int IT = (NQ * NR + 31) / 32;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int u = lane + 32 * it;
        if ((NQ * NR) % 32 == 0 || u < NQ * NR) {
            const int sq = NQ > 1 ? u / NR : 0;
            const int j = NQ > 1 ? u - sq * NR : u;
            const int base = sq * N;
            const int k = j % NS;
            C v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int xi = base + j + r * NR;
                C x = src[SWZ ? swz<C>(xi) : xi];
                if (NS > 1 && r > 0 && k) {
                    C w = __ldg(&tw[r * k * TSTEP * TWS]);
                    if (S > 0) w.y = -w.y;
                    x = mul(x, w);
                }
                v[r] = x;
            }
            Dft<C, R, S>::run(v);
            const int idxD = base + (j - k) * R + k;
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int xo = idxD + q * NS;
                dst[SWZ ? swz<C>(xo) : xo] = v[q];
            }
        }
    }
}

template <typename C, int N, int F, int S, int NQ, bool SWZ, int TWS, bool END>
struct Step;
template <typename C, int N, int F, int S, int NQ, bool SWZ, int TWS>
struct Step<C, N, F, S, NQ, SWZ, TWS, true> {
    static __device__ __forceinline__ C *go(C *src, C *, const C *, int) { return src; }
};
template <typename C, int N, int F, int S, int NQ, bool SWZ, int TWS>
struct Step<C, N, F, S, NQ, SWZ, TWS, false> {
    static __device__ __forceinline__ C *go(C *src, C *dst, const C *tw, int lane) {
        stage<C, N, F, S, NQ, SWZ, TWS>(src, dst, tw, lane);
        __syncwarp();
        return Step<C, N, F + 1, S, NQ, SWZ, TWS, (F + 1 >= nfac(N))>::go(dst, src, tw, lane);
    }
};

// stage F of one sequence with its inputs from ld(x) and its outputs to st(x, value): the same
// butterflies, twiddles and operation order as stage()
template <typename C, int N, int F, int S, int TWS, typename LD, typename ST>
__device__ __forceinline__ void stage_io(LD &ld, ST &st, const C *__restrict__ tw, int lane) {
    constexpr int R = fac(N, F);
    constexpr int NS = stride(N, F);
    constexpr int NR = N / R;
    constexpr int TSTEP = N / (NS * R);
    constexpr int IT = (NR + 31) / 32;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int j = lane + 32 * it;
        if (NR % 32 == 0 || j < NR) {
            const int k = j % NS;
            C v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                C x = ld(j + r * NR);
                if (NS > 1 && r > 0 && k) {
                    C w = __ldg(&tw[r * k * TSTEP * TWS]);
                    if (S > 0) w.y = -w.y;
                    x = mul(x, w);
                }
                v[r] = x;
            }
            Dft<C, R, S>::run(v);
            const int idxD = (j - k) * R + k;
#pragma unroll
            for (int q = 0; q < R; ++q) st(idxD + q * NS, v[q]);
        }
    }
}

// stage F of one sequence in place in the swizzled buffer x: every lane reads and transforms all
// its butterflies' inputs before the warp writes any output (the same arithmetic as stage())
template <typename C, int N, int F, int S, int TWS>
__device__ __forceinline__ void stage_ip(C *x, const C *__restrict__ tw, int lane) {
    constexpr int R = fac(N, F);
    constexpr int NS = stride(N, F);
    constexpr int NR = N / R;
    constexpr int TSTEP = N / (NS * R);
    constexpr int IT = (NR + 31) / 32;
    C v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int j = lane + 32 * it;
        if (NR % 32 == 0 || j < NR) {
            const int k = j % NS;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                C u = x[swz<C>(j + r * NR)];
                if (NS > 1 && r > 0 && k) {
                    C w = __ldg(&tw[r * k * TSTEP * TWS]);
                    if (S > 0) w.y = -w.y;
                    u = mul(u, w);
                }
                v[it][r] = u;
            }
            Dft<C, R, S>::run(v[it]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int j = lane + 32 * it;
        if (NR % 32 == 0 || j < NR) {
            const int k = j % NS;
            const int idxD = (j - k) * R + k;
#pragma unroll
            for (int q = 0; q < R; ++q) x[swz<C>(idxD + q * NS)] = v[it][q];
        }
    }
    __syncwarp();
}

template <typename C, int N, int F, int S, int TWS, bool END>
struct IpSteps;
template <typename C, int N, int F, int S, int TWS>
struct IpSteps<C, N, F, S, TWS, true> {
    static __device__ __forceinline__ void go(C *, const C *, int) {}
};
template <typename C, int N, int F, int S, int TWS>
struct IpSteps<C, N, F, S, TWS, false> {
    static __device__ __forceinline__ void go(C *x, const C *tw, int lane) {
        stage_ip<C, N, F, S, TWS>(x, tw, lane);
        IpSteps<C, N, F + 1, S, TWS, (F + 2 >= nfac(N))>::go(x, tw, lane);
    }
};

// the stages between the first and the last, ping-ponging between two swizzled buffers; returns
// the buffer holding the output of the last of them
template <typename C, int N, int F, int S, int TWS, bool END>
struct MidSteps;
template <typename C, int N, int F, int S, int TWS>
struct MidSteps<C, N, F, S, TWS, true> {
    static __device__ __forceinline__ C *go(C *src, C *, const C *, int) { return src; }
};
template <typename C, int N, int F, int S, int TWS>
struct MidSteps<C, N, F, S, TWS, false> {
    static __device__ __forceinline__ C *go(C *src, C *dst, const C *tw, int lane) {
        stage<C, N, F, S, 1, true, TWS>(src, dst, tw, lane);
        __syncwarp();
        return MidSteps<C, N, F + 1, S, TWS, (F + 2 >= nfac(N))>::go(dst, src, tw, lane);
    }
};
}   // namespace kct

// S = -1: exp(-2 pi i jk/N) (FFTW_FORWARD), +1: exp(+...) (FFTW_BACKWARD).  NQ sequences of
// length N lie N apart in a; b is a scratch buffer of the same size (both private to the calling
// warp); the input must be visible to the whole warp (__syncwarp after writing it).  Returns the
// buffer holding the result.  SWZ: the buffers are swizzled (element x at swz<C>(x)).  TWS: the
// table holds the twiddles of length TWS N (exp(-2 pi i m/N) is entry TWS m).
template <typename C, int N, int S, int NQ = 1, bool SWZ = false, int TWS = 1>
__device__ __forceinline__ C *fft_warp_ct(C *a, C *b, const C *tw) {
    static_assert(kct::nfac(N) > 0, "transform length must be 2^a 3^b 5^c");
    return kct::Step<C, N, 0, S, NQ, SWZ, TWS, false>::go(a, b, tw, threadIdx.x & 31);
}

// fft_warp_ct of one sequence whose first stage reads its input through ld(x) (element x of the
// sequence) and whose last stage writes its output through st(x, value), natural order, so that
// neither needs a copy pass through shared memory; the stages in between use the swizzled
// buffers a and b (private to the warp).  pre() runs between the second-last and the last stage
// in every thread of the warp (a block-wide barrier there must be reached by every warp).  Same
// arithmetic as fft_warp_ct.  The last stage reads buffer a when nfac(N) is even, else b; st may
// write the other one.
template <typename C, int N, int S, int TWS = 1, typename LD, typename ST, typename PRE>
__device__ __forceinline__ void fft_warp_ct_io(LD ld, ST st, PRE pre, C *a, C *b, const C *tw) {
    constexpr int L = kct::nfac(N);
    static_assert(L >= 2, "fft_warp_ct_io needs at least two stages");
    const int lane = threadIdx.x & 31;
    auto to_a = [&](int x, C v) { a[swz<C>(x)] = v; };
    kct::stage_io<C, N, 0, S, TWS>(ld, to_a, tw, lane);
    __syncwarp();
    const C *src = kct::MidSteps<C, N, 1, S, TWS, (2 >= L)>::go(a, b, tw, lane);
    pre();
    auto from_src = [&](int x) { return src[swz<C>(x)]; };
    kct::stage_io<C, N, L - 1, S, TWS>(from_src, st, tw, lane);
}

// fft_warp_ct of one sequence held in one swizzled buffer a (the input visible to the whole warp):
// every stage but the last runs in place (stage_ip), and the last reads a and writes its output
// through st(x, value), so a warp needs one buffer of N elements instead of two.  Same arithmetic
// as fft_warp_ct.
template <typename C, int N, int S, int TWS = 1, typename ST>
__device__ __forceinline__ void fft_warp_ct_ip(C *a, ST st, const C *tw) {
    constexpr int L = kct::nfac(N);
    static_assert(L >= 1, "transform length must be 2^a 3^b 5^c");
    const int lane = threadIdx.x & 31;
    kct::IpSteps<C, N, 0, S, TWS, (1 >= L)>::go(a, tw, lane);
    auto from_a = [&](int x) { return a[swz<C>(x)]; };
    kct::stage_io<C, N, L - 1, S, TWS>(from_a, st, tw, lane);
}

// the same with every stage in place: the result is left in a (natural order, swizzled)
template <typename C, int N, int S, int TWS = 1>
__device__ __forceinline__ void fft_warp_ct_inplace(C *a, const C *tw) {
    constexpr int L = kct::nfac(N);
    const int lane = threadIdx.x & 31;
    kct::IpSteps<C, N, 0, S, TWS, (1 >= L)>::go(a, tw, lane);
    kct::stage_ip<C, N, L - 1, S, TWS>(a, tw, lane);
}

// the transform lengths with compiled instances (3/2-rule grids of nx, nz = 32, 64, 96, 128, 384
// and the Chebyshev extensions 2 ny = 64, 128, 192, 256, 512)
#define KMM_CT_LEN_LIST(X) X(48) X(64) X(96) X(128) X(144) X(192) X(256) X(512) X(576)

// ---------------------------------------------------------------------------
// In-register DFTs of small lengths (two-pass transforms): X_k = sum_j v_j exp(-2 pi i j k / M),
// natural order in and out.  Lengths that are not a single radix split as M = A B with
// j = B a + b, k = c + A d:  X[c + A d] = sum_b W_M^(bc) W_B^(bd) sum_a v[B a + b] W_A^(ac);
// W_M^j is entry `step` j of the twiddle table tw (a table of length step M).
// ---------------------------------------------------------------------------
template <typename C, int A, int B>
__device__ __forceinline__ void regdft_ab(C *v, const C *__restrict__ tw, int step) {
    constexpr int M = A * B;
    C Q[B][A];
#pragma unroll
    for (int b = 0; b < B; ++b) {
        C u[A];
#pragma unroll
        for (int a = 0; a < A; ++a) u[a] = v[B * a + b];
        kct::Dft<C, A, -1>::run(u);
#pragma unroll
        for (int c = 0; c < A; ++c) Q[b][c] = (b * c) ? kct::mul(u[c], __ldg(tw + step * ((b * c) % M))) : u[c];
    }
#pragma unroll
    for (int c = 0; c < A; ++c) {
        C u[B];
#pragma unroll
        for (int b = 0; b < B; ++b) u[b] = Q[b][c];
        kct::Dft<C, B, -1>::run(u);
#pragma unroll
        for (int d = 0; d < B; ++d) v[c + A * d] = u[d];
    }
}

template <typename C, int M>
struct RegDft;
template <typename C>
struct RegDft<C, 3> {
    static __device__ __forceinline__ void run(C *v, const C *, int) { kct::Dft<C, 3, -1>::run(v); }
};
template <typename C>
struct RegDft<C, 4> {
    static __device__ __forceinline__ void run(C *v, const C *, int) { kct::Dft<C, 4, -1>::run(v); }
};
template <typename C>
struct RegDft<C, 8> {
    static __device__ __forceinline__ void run(C *v, const C *, int) { kct::Dft<C, 8, -1>::run(v); }
};
template <typename C>
struct RegDft<C, 6> {
    static __device__ __forceinline__ void run(C *v, const C *tw, int step) { regdft_ab<C, 2, 3>(v, tw, step); }
};
template <typename C>
struct RegDft<C, 9> {
    static __device__ __forceinline__ void run(C *v, const C *tw, int step) { regdft_ab<C, 3, 3>(v, tw, step); }
};
template <typename C>
struct RegDft<C, 12> {
    static __device__ __forceinline__ void run(C *v, const C *tw, int step) { regdft_ab<C, 4, 3>(v, tw, step); }
};
template <typename C>
struct RegDft<C, 16> {
    static __device__ __forceinline__ void run(C *v, const C *tw, int step) { regdft_ab<C, 4, 4>(v, tw, step); }
};
