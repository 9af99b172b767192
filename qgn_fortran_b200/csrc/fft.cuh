// fft.cuh -- FP64 shared-memory FFT building blocks for sm_100a.
//
// A transform of length N (power of two, 16..2048) is carried out by G = N/T threads
// (T = TP elements per thread, TP = 16 or 32, fewer for N < TP) as a sequence of Stockham
// decimation-in-time radix passes: radix TP for every pass except the last, which
// takes the remaining factor.  Each pass reads T values from shared memory into
// registers, applies the inter-pass twiddles, performs register-resident radix-R
// DFTs and writes the results back in place (the load and store halves of a pass
// are separated by a barrier).  Indices are padded by one element per TP
// (p -> p + p/TP) so that both the strided stores of the first pass and the
// contiguous accesses of later passes are free of bank-group conflicts.
// TP = 32 halves the shared-memory round trips of a 512- or 1024-point transform (two
// passes instead of three) at twice the registers; the FP32 transforms use it.
//
// Twiddles come from a per-length table tw[m] = exp(-2*pi*i*m/N) computed on the
// host in long double; DIR=-1 is the forward (exp(-i...)) transform of MKL's
// DftiComputeForward, DIR=+1 the unnormalised backward transform.
#pragma once
#include <cuda_runtime.h>

namespace qgn {

// complex arithmetic on double2 (FP64 path) and float2 (FP32 path of the mixed mode)
template <class CT> struct CTraits;
template <> struct CTraits<double2> {
    using R = double;
    __host__ __device__ static double2 make(double a, double b) { return make_double2(a, b); }
};
template <> struct CTraits<float2> {
    using R = float;
    __host__ __device__ static float2 make(float a, float b) { return make_float2(a, b); }
};
template <class CT>
__device__ __forceinline__ CT cmk(typename CTraits<CT>::R a, typename CTraits<CT>::R b) {
    return CTraits<CT>::make(a, b);
}
template <class CT> __device__ __forceinline__ CT cadd(CT a, CT b) { return cmk<CT>(a.x + b.x, a.y + b.y); }
template <class CT> __device__ __forceinline__ CT csub(CT a, CT b) { return cmk<CT>(a.x - b.x, a.y - b.y); }
template <class CT> __device__ __forceinline__ CT cmul(CT a, CT b) {
    return cmk<CT>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class CT> __device__ __forceinline__ CT cconj(CT a) { return cmk<CT>(a.x, -a.y); }
template <class CT> __device__ __forceinline__ CT czero() { return cmk<CT>(0, 0); }

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

// padded shared-memory index of element p of a transform whose radix passes take TP elements
// per thread: one pad element per TP, so that the first pass's stores (stride TP) and the later
// passes' contiguous accesses hit distinct bank groups
template <int TP = 16>
__device__ __forceinline__ int fpad(int p) { return p + p / TP; }
// padded length of one transform of length N
template <int TP = 16>
__host__ __device__ constexpr int fpadlen(int N) { return N + N / TP; }

// Multiply by exp(DIR * 2*pi*i * m/16); m is a compile-time constant after unrolling.
template <int DIR, class CT>
__device__ __forceinline__ CT rot16(CT a, int m) {
    using R = typename CTraits<CT>::R;
    constexpr R C1 = (R)0.92387953251128675613;  // cos(pi/8)
    constexpr R S1 = (R)0.38268343236508977173;  // sin(pi/8)
    constexpr R HH = (R)0.70710678118654752440;  // sqrt(2)/2
    switch (m & 15) {
        case 0: return a;
        case 4: return DIR > 0 ? cmk<CT>(-a.y, a.x) : cmk<CT>(a.y, -a.x);
        case 8: return cmk<CT>(-a.x, -a.y);
        case 12: return DIR > 0 ? cmk<CT>(a.y, -a.x) : cmk<CT>(-a.y, a.x);
        case 2: { R s = DIR * HH; return cmk<CT>(HH * a.x - s * a.y, s * a.x + HH * a.y); }
        case 6: { R s = DIR * HH; return cmk<CT>(-HH * a.x - s * a.y, s * a.x - HH * a.y); }
        case 10: { R s = -DIR * HH; return cmk<CT>(-HH * a.x - s * a.y, s * a.x - HH * a.y); }
        case 14: { R s = -DIR * HH; return cmk<CT>(HH * a.x - s * a.y, s * a.x + HH * a.y); }
        default: break;
    }
    R c, s;
    switch (m & 15) {
        case 1: c = C1; s = S1; break;
        case 3: c = S1; s = C1; break;
        case 5: c = -S1; s = C1; break;
        case 7: c = -C1; s = S1; break;
        case 9: c = -C1; s = -S1; break;
        case 11: c = -S1; s = -C1; break;
        case 13: c = S1; s = -C1; break;
        default: c = C1; s = -S1; break;  // 15
    }
    s = DIR * s;
    return cmk<CT>(a.x * c - a.y * s, a.x * s + a.y * c);
}

// Multiply by exp(DIR * 2*pi*i * m/32) for 0 <= m < 16; m is a compile-time constant after
// unrolling.  Even m reduce to rot16; odd m use cos and sin of pi/16 and 3*pi/16.
template <int DIR, class CT>
__device__ __forceinline__ CT rot32(CT a, int m) {
    using R = typename CTraits<CT>::R;
    if ((m & 1) == 0) return rot16<DIR>(a, m >> 1);
    constexpr R A = (R)0.98078528040323044913;  // cos(pi/16)
    constexpr R B = (R)0.19509032201612826785;  // sin(pi/16)
    constexpr R E = (R)0.83146961230254523708;  // cos(3 pi/16)
    constexpr R F = (R)0.55557023301960222474;  // sin(3 pi/16)
    R c, s;
    switch (m & 15) {
        case 1: c = A; s = B; break;
        case 3: c = E; s = F; break;
        case 5: c = F; s = E; break;
        case 7: c = B; s = A; break;
        case 9: c = -B; s = A; break;
        case 11: c = -F; s = E; break;
        case 13: c = -E; s = F; break;
        default: c = -A; s = B; break;  // 15
    }
    s = DIR * s;
    return cmk<CT>(a.x * c - a.y * s, a.x * s + a.y * c);
}

// Multiply by exp(DIR * 2*pi*i * k/R), 0 <= k < R/2.
template <int R, int DIR, class CT>
__device__ __forceinline__ CT rot_root(CT a, int k) {
    if constexpr (R == 32) return rot32<DIR>(a, k);
    else return rot16<DIR>(a, k * (16 / R));
}

// cos and sin of 2 pi k / R for the non-trivial roots of the radix-2 butterflies
// (R = 8, 16, 32; 0 < k < R/2, k != R/4), from the first-octant constants
__host__ __device__ constexpr double root_cos(int R, int k) {
    const int m = k * (32 / R);   // angle in units of pi/16, 0 < m < 16, m != 8
    constexpr double c[9] = {1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
                             0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
                             0.19509032201612826785, 0.0};
    return m <= 8 ? c[m] : -c[16 - m];
}
__host__ __device__ constexpr double root_sin(int R, int k) {
    const int m = k * (32 / R);
    constexpr double c[9] = {1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
                             0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
                             0.19509032201612826785, 0.0};
    return m <= 8 ? c[8 - m] : c[m - 8];
}

// Radix-2 butterfly (e + w o, e - w o), w = exp(DIR 2 pi i k / R), k a compile-time constant
// after unrolling.  Trivial roots (k = 0: w = 1; k = R/4: w = DIR i) are additions; the others
// use the tangent form: with |c| >= |s|, w o = c (o.x - t o.y, o.y + t o.x), t = s/c, and with
// |s| > |c|, w o = s (r o.x - o.y, o.x + r o.y), r = c/s -- two FMAs for the scaled product and
// one per output component, six in all against eight for product then sum and difference, and
// at most two roundings per output (|t|, |r| <= 1).
template <int R, int DIR, class CT>
__device__ __forceinline__ void bfly(CT& a, CT& b, int k) {
    using T = typename CTraits<CT>::R;
    const CT e = a, o = b;
    if (k == 0) {
        a = cadd(e, o);
        b = csub(e, o);
        return;
    }
    if (4 * k == R) {   // w o = DIR i o
        const CT t = DIR > 0 ? cmk<CT>(-o.y, o.x) : cmk<CT>(o.y, -o.x);
        a = cadd(e, t);
        b = csub(e, t);
        return;
    }
    const double c = root_cos(R, k), s = DIR * root_sin(R, k);
    const bool cdom = (c < 0 ? -c : c) >= (s < 0 ? -s : s);
    const T f = (T)(cdom ? c : s);                 // common factor
    const T t = (T)(cdom ? s / c : c / s);         // tangent or cotangent
    T u, w;
    if (cdom) {
        u = fma(-t, o.y, o.x);
        w = fma(t, o.x, o.y);
    } else {
        u = fma(t, o.x, -o.y);
        w = fma(t, o.y, o.x);
    }
    a = cmk<CT>(fma(f, u, e.x), fma(f, w, e.y));
    b = cmk<CT>(fma(-f, u, e.x), fma(-f, w, e.y));
}

// In-register DFT of length R (1,2,4,8,16,32), natural order in and out, sign DIR.
template <int R, int DIR>
struct RegDFT {
    template <class CT>
    __device__ __forceinline__ static void run(CT* v) {
        CT e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
        RegDFT<R / 2, DIR>::run(e);
        RegDFT<R / 2, DIR>::run(o);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) {
            CT x = e[k], y = o[k];
            bfly<R, DIR>(x, y, k);
            v[k] = x;
            v[k + R / 2] = y;
        }
    }
};
template <int DIR>
struct RegDFT<1, DIR> {
    template <class CT>
    __device__ __forceinline__ static void run(CT*) {}
};
template <int DIR>
struct RegDFT<2, DIR> {
    template <class CT>
    __device__ __forceinline__ static void run(CT* v) {
        CT a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int N, int TP = 16>
struct FFTShape {
    static constexpr int T = N < TP ? N : TP;   // elements per thread
    static constexpr int G = N / T;             // threads per transform
};

// Inter-pass twiddles of one radix-R butterfly: v[r] *= w^r, w = exp(DIR 2 pi i k/(NS R)).
// w^(2^q) come from the table tw[m] = exp(-2 pi i m/N) (conjugated for DIR=+1); the other
// powers are products of at most three table values, formed just before use.
template <int N, int NS, int R, int DIR, class CT>
__device__ __forceinline__ void apply_twiddles(CT* v, int k, const CT* __restrict__ tw) {
    if constexpr (NS > 1) {
        constexpr int S = N / (NS * R);
        const int kS = k * S;
        auto ldw = [&](int r) {
            const CT t = __ldg(&tw[r * kS]);
            return DIR > 0 ? cconj(t) : t;
        };
        const CT w1 = ldw(1);
        v[1] = cmul(v[1], w1);
        if constexpr (R > 2) {
            const CT w2 = ldw(2);
            const CT w3 = cmul(w2, w1);
            v[2] = cmul(v[2], w2);
            v[3] = cmul(v[3], w3);
            if constexpr (R > 4) {
                const CT w4 = ldw(4);
                const CT w5 = cmul(w4, w1), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
                v[4] = cmul(v[4], w4);
                v[5] = cmul(v[5], w5);
                v[6] = cmul(v[6], w6);
                v[7] = cmul(v[7], w7);
                if constexpr (R > 8) {
                    const CT w8 = ldw(8);
                    v[8] = cmul(v[8], w8);
                    v[9] = cmul(v[9], cmul(w8, w1));
                    v[10] = cmul(v[10], cmul(w8, w2));
                    v[11] = cmul(v[11], cmul(w8, w3));
                    v[12] = cmul(v[12], cmul(w8, w4));
                    v[13] = cmul(v[13], cmul(w8, w5));
                    v[14] = cmul(v[14], cmul(w8, w6));
                    v[15] = cmul(v[15], cmul(w8, w7));
                    if constexpr (R > 16) {
                        // w^(16+r) = w16 * w^r; the low powers are formed again from the table
                        const CT w16 = ldw(16);
                        const CT u[8] = {w16, cmul(w16, w1), cmul(w16, w2), cmul(w16, w3),
                                         cmul(w16, w4), cmul(w16, w5), cmul(w16, w6), cmul(w16, w7)};
#pragma unroll
                        for (int r = 0; r < 8; ++r) {
                            v[16 + r] = cmul(v[16 + r], u[r]);
                            v[24 + r] = cmul(v[24 + r], cmul(u[r], w8));
                        }
                    }
                }
            }
        }
    }
}

// Where a pass takes its input from / puts its output to.
enum FftSrc { SRC_SMEM = 0, SRC_FN = 1, SRC_FN_SMEM = 2 };   // SRC_FN_SMEM: a functor that reads this smem
// DST_SMEM_MAP: the last pass writes x[st(idx)] (st maps an output index to a shared-memory
// offset) with the barriers of DST_SMEM
// DST_SMEM_STORE: the last pass hands each output to st(idx, value), which stores it in the
// transform's own shared buffer in a layout of its choice, with the barriers of DST_SMEM
enum FftDst { DST_SMEM = 0, DST_FN = 1, DST_SMEM_MAP = 2, DST_SMEM_STORE = 3 };

// One Stockham DIT pass (sub-length NS, radix R) of an N-point transform whose
// intermediate lives padded at x.  Pass 0 may read through ld(idx), the last pass may
// write through st(idx, value); every other access goes to x.  Barriers: a pass that reads
// the shared buffer it overwrites syncs between its reads and writes, and a pass that
// writes the shared buffer syncs after its writes.  With SRC_FN the caller guarantees
// that no thread still reads x when the pass starts writing it.  WS (warp-synchronous):
// the G threads of a transform lie in one warp and share it with no thread that touches
// another transform's buffer, so the barriers that only order accesses to x are __syncwarp;
// the barrier after a loader that reads other buffers (SRC_FN_SMEM) and the barrier that
// ends a transform written to shared memory (the caller may read across transforms) stay
// block-wide.
template <bool BLOCK, bool WS>
__device__ __forceinline__ void fft_sync() {
    if constexpr (WS && !BLOCK) __syncwarp();
    else __syncthreads();
}

template <int N, int NS, int DIR, int SRC, int DST, int TP, bool WS, class CT, class Ld, class St>
__device__ __forceinline__ void fft_pass_io(CT* x, int lane, bool active, const CT* __restrict__ tw, Ld& ld, St& st) {
    constexpr int T = FFTShape<N, TP>::T;
    constexpr int G = FFTShape<N, TP>::G;
    constexpr int R = (N / NS >= TP) ? TP : N / NS;
    constexpr int BPT = T / R;
    constexpr int STRIDE = N / R;
    constexpr bool LAST = (NS * R == N);
    CT v[T];
    if (active) {
#pragma unroll
        for (int b = 0; b < BPT; ++b) {
            const int j = lane + b * G;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int idx = j + r * STRIDE;
                if constexpr (SRC == SRC_SMEM) v[b * R + r] = x[fpad<TP>(idx)];
                else v[b * R + r] = ld(idx);
            }
        }
    }
    constexpr bool TO_SMEM = (DST == DST_SMEM || DST == DST_SMEM_MAP || DST == DST_SMEM_STORE);
    if constexpr (TO_SMEM && SRC != SRC_FN) fft_sync<SRC == SRC_FN_SMEM, WS>();
    if (active) {
#pragma unroll
        for (int b = 0; b < BPT; ++b) {
            const int j = lane + b * G;
            const int k = j & (NS - 1);
            apply_twiddles<N, NS, R, DIR>(&v[b * R], k, tw);
            RegDFT<R, DIR>::run(&v[b * R]);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int idx = base + r * NS;
                if constexpr (DST == DST_SMEM) x[fpad<TP>(idx)] = v[b * R + r];
                else if constexpr (DST == DST_SMEM_MAP) x[st(idx)] = v[b * R + r];
                else st(idx, v[b * R + r]);
            }
        }
    }
    if constexpr (TO_SMEM) fft_sync<LAST, WS>();
}

template <int N, int NS, int DIR, int SRC0, int DSTL, int TP, bool WS, class CT, class Ld, class St>
__device__ __forceinline__ void fft_rec(CT* x, int lane, bool active, const CT* __restrict__ tw, Ld& ld, St& st) {
    constexpr int R = (N / NS >= TP) ? TP : N / NS;
    constexpr bool FIRST = (NS == 1);
    constexpr bool LAST = (NS * R == N);
    constexpr int SRC = FIRST ? SRC0 : SRC_SMEM;
    constexpr int DST = LAST ? DSTL : DST_SMEM;
    fft_pass_io<N, NS, DIR, SRC, DST, TP, WS>(x, lane, active, tw, ld, st);
    if constexpr (!LAST) fft_rec<N, NS * R, DIR, SRC0, DSTL, TP, WS>(x, lane, active, tw, ld, st);
}

template <class CT>
struct NoIOT {
    __device__ CT operator()(int) const { return czero<CT>(); }
    __device__ void operator()(int, CT) const {}
};
using NoIO = NoIOT<double2>;

// N-point transform of one slot by the G = FFTShape<N, TP>::G threads with lane in [0,G),
// reading its input through ld (SRC0 = SRC_FN / SRC_FN_SMEM) or from x (SRC_SMEM, written and
// synced by the caller) and delivering its output through st (DSTL = DST_FN) or into x
// (DST_SMEM, synced block-wide on return).  Every thread of the block calls this (it may
// contain __syncthreads).  WS as for fft_pass_io.
template <int N, int DIR, int SRC0, int DSTL, int TP = 16, bool WS = false, class CT, class Ld, class St>
__device__ __forceinline__ void fft_fused(CT* x, int lane, bool active, const CT* __restrict__ tw, Ld ld, St st) {
    fft_rec<N, 1, DIR, SRC0, DSTL, TP, WS>(x, lane, active, tw, ld, st);
}

// In-place N-point transform of the padded array x (caller syncs before; ends with a barrier).
template <int N, int DIR, int TP = 16, class CT>
__device__ __forceinline__ void fft_block(CT* x, int lane, bool active, const CT* __restrict__ tw) {
    NoIOT<CT> io;
    fft_rec<N, 1, DIR, SRC_SMEM, DST_SMEM, TP, false>(x, lane, active, tw, io, io);
}

}  // namespace qgn
