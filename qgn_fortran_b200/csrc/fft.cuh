// fft.cuh -- FP64 shared-memory FFT building blocks for sm_100a.
//
// A transform of length N (power of two, 16..2048) is carried out by G = N/T threads
// (T = TP elements per thread, TP = 16 or 32, fewer for N < TP) as a sequence of Stockham
// decimation-in-time radix passes: radix TP for every pass except the last, which
// takes the remaining factor.  Each pass reads T values from shared memory into
// registers, applies the inter-pass twiddles (folded into the first radix-2 stage), performs register-resident radix-R
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

// In-register DFT of length R (1,2,4,8,16,32), natural order in and out, sign DIR.  With S1 the
// first radix-2 stage -- the sums and differences of elements i and i + R/2 -- has been done
// by the caller (twiddled_dft): the recursion's length-2 base cases are then the identity.
template <int R, int DIR, bool S1 = false>
struct RegDFT {
    template <class CT>
    __device__ __forceinline__ static void run(CT* v) {
        CT e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
        RegDFT<R / 2, DIR, S1>::run(e);
        RegDFT<R / 2, DIR, S1>::run(o);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) {
            CT x = e[k], y = o[k];
            bfly<R, DIR>(x, y, k);
            v[k] = x;
            v[k + R / 2] = y;
        }
    }
};
template <int DIR, bool S1>
struct RegDFT<1, DIR, S1> {
    template <class CT>
    __device__ __forceinline__ static void run(CT*) {}
};
template <int DIR, bool S1>
struct RegDFT<2, DIR, S1> {
    template <class CT>
    __device__ __forceinline__ static void run(CT* v) {
        if constexpr (!S1) {
            CT a = v[0], b = v[1];
            v[0] = cadd(a, b);
            v[1] = csub(a, b);
        }
    }
};

template <int N, int TP = 16>
struct FFTShape {
    static constexpr int T = N < TP ? N : TP;   // elements per thread
    static constexpr int G = N / T;             // threads per transform
};

// First radix-2 stage with the inter-pass twiddle of its second element folded in: given a
// (already multiplied by its own twiddle), (a + W b, a - W b) as a + W b by four FMAs and
// a - W b = 2 a - (a + W b) by two, against a complex product and four additions.
template <class CT>
__device__ __forceinline__ void fold2(CT& a, CT& b, CT W) {
    using T = typename CTraits<CT>::R;
    const CT y0 = cmk<CT>(fma(b.x, W.x, fma(-b.y, W.y, a.x)), fma(b.x, W.y, fma(b.y, W.x, a.y)));
    b = cmk<CT>(fma((T)2, a.x, -y0.x), fma((T)2, a.y, -y0.y));
    a = y0;
}

// The radix-R DFT of v[r] w^r, w = exp(DIR 2 pi i k/(NS R)) (the inter-pass twiddles of a
// Stockham pass): the powers w^(2^q) come from the table, the others are products of at most
// three of them, formed pair by pair (j, j + R/2) of the first radix-2 stage, which fold2
// performs; RegDFT does the rest.
template <int N, int NS, int R, int DIR, class CT>
__device__ __forceinline__ void twiddled_dft(CT* v, int k, const CT* __restrict__ tw) {
    if constexpr (NS == 1 || R < 2) {
        RegDFT<R, DIR>::run(v);
    } else {
        constexpr int S = N / (NS * R);
        const int kS = k * S;
        auto ldw = [&](int r) {
            const CT t = __ldg(&tw[r * kS]);
            return DIR > 0 ? cconj(t) : t;
        };
        constexpr int H = R / 2;
        const CT wH = ldw(H);                   // w^(R/2), the second element's extra factor
        const CT w1 = ldw(1);
        CT w2 = w1, w3 = w1, w4 = w1;
        if constexpr (R >= 8) w2 = ldw(2);
        if constexpr (R >= 8) w3 = cmul(w2, w1);
        if constexpr (R >= 16) w4 = ldw(4);
        // w^j for 0 < j < 8 (j < R/2): one product at most beyond the loads
        auto lowpow = [&](int j) -> CT {
            switch (j) {
                case 1: return w1;
                case 2: return w2;
                case 3: return w3;
                case 4: return w4;
                case 5: return cmul(w4, w1);
                case 6: return cmul(w4, w2);
                default: return cmul(w4, w3);   // 7
            }
        };
        if constexpr (R <= 16) {
#pragma unroll
            for (int j = 0; j < H; ++j) {
                if (j == 0) {
                    fold2(v[0], v[H], wH);
                } else {
                    const CT Wj = lowpow(j);
                    v[j] = cmul(v[j], Wj);
                    fold2(v[j], v[j + H], cmul(wH, Wj));
                }
            }
        } else {   // R = 32: j and j + 8 share w^j; w^(j+8) = w8 w^j, and w^16 is wH
            const CT w8 = ldw(8);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const CT Wj = j == 0 ? w8 : lowpow(j);   // (w8 unused as Wj when j == 0)
                if (j == 0) {
                    fold2(v[0], v[16], wH);
                } else {
                    v[j] = cmul(v[j], Wj);
                    fold2(v[j], v[j + 16], cmul(wH, Wj));
                }
                const CT W8 = j == 0 ? w8 : cmul(w8, Wj);
                v[j + 8] = cmul(v[j + 8], W8);
                fold2(v[j + 8], v[j + 24], cmul(W8, wH));
            }
        }
        RegDFT<R, DIR, true>::run(v);
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
            twiddled_dft<N, NS, R, DIR>(&v[b * R], k, tw);
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

// The last two passes of an N = RL TP NS point transform (a radix-TP pass at sub-length NS, then
// the final radix-RL pass, RL = 2, 4 or 8), fused, with the exchange between them done by warp
// shuffles instead of shared memory.  Final butterfly j' (< N/RL) takes the elements
// j' + m N/RL, m < RL, which are outputs r of the first pass's butterflies j + m NS
// (j' = j + NS r, j < NS).  The first pass assigns its butterflies to the transform's threads
// so that these RL sit in one warp: the transform's thread l is block thread l IL + slot (IL
// threads of other transforms interleaved, LPW = 32/IL of its threads per warp), and takes
// butterfly
//   j(l) = H (l / LPW) + l % H + NS q,  q = (l % LPW) / H,  H = LPW / RL,
// so that partner q ^ m is block thread ^ (32/RL) m.  Thread q finishes the final butterflies of
// its outputs r in [q TP/RL, (q+1) TP/RL): in round m = 1 .. RL-1 it sends partner p = q ^ m its
// block of outputs p and receives the partner's block q into the registers of the block just
// sent, after which register block m holds the inputs from partner m.  One read of shared
// memory, one write and two barriers in place of two of each and four.  Every thread of the
// warp executes the shuffles (a transform's threads share `active`; inactive ones exchange
// unused registers).
template <int N, int NS, int DIR, int SRC, int DST, int TP, bool WS, int IL, class CT, class Ld, class St>
__device__ __forceinline__ void fft_pass_tail2(CT* x, int lane, bool active, const CT* __restrict__ tw, Ld& ld, St& st) {
    constexpr int R = TP;
    constexpr int RL = N / (TP * NS);
    constexpr int B = R / RL;                    // outputs per block
    constexpr int LPW = 32 / IL, H = LPW / RL;
    constexpr int STRIDE = N / R;
    static_assert((RL == 2 || RL == 4 || RL == 8) && RL * R * NS == N && H >= 1, "fused radix-RL tail");
    static_assert(FFTShape<N, TP>::T == R && FFTShape<N, TP>::G % LPW == 0, "whole warp rows per transform");
    const int q = (lane % LPW) / H;
    const int jl = H * (lane / LPW) + lane % H;
    const int j = jl + NS * q;
    CT v[R];
    if (active) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int idx = j + r * STRIDE;
            if constexpr (SRC == SRC_SMEM) v[r] = x[fpad<TP>(idx)];
            else v[r] = ld(idx);
        }
    }
    constexpr bool TO_SMEM = (DST == DST_SMEM || DST == DST_SMEM_MAP || DST == DST_SMEM_STORE);
    if constexpr (TO_SMEM && SRC != SRC_FN) fft_sync<SRC == SRC_FN_SMEM, WS>();
    if (active) twiddled_dft<N, NS, R, DIR>(v, j & (NS - 1), tw);
#pragma unroll
    for (int m = 1; m < RL; ++m) {
        const int p = q ^ m;
#pragma unroll
        for (int i = 0; i < B; ++i) {
            CT send = v[i];
#pragma unroll
            for (int b = 1; b < RL; ++b)
                if (b == p) send = v[b * B + i];
            CT recv;
            recv.x = __shfl_xor_sync(0xffffffffu, send.x, (32 / RL) * m);
            recv.y = __shfl_xor_sync(0xffffffffu, send.y, (32 / RL) * m);
#pragma unroll
            for (int b = 0; b < RL; ++b)
                if (b == p) v[b * B + i] = recv;
        }
    }
    if (active) {
#pragma unroll
        for (int i = 0; i < B; ++i) {
            CT u[RL];
#pragma unroll
            for (int m = 0; m < RL; ++m) u[m] = v[m * B + i];
            const int jp = jl + NS * (q * B + i);   // final butterfly: outputs jp + m N/RL
            twiddled_dft<N, N / RL, RL, DIR>(u, jp, tw);
#pragma unroll
            for (int m = 0; m < RL; ++m) {
                const int idx = jp + m * (N / RL);
                if constexpr (DST == DST_SMEM) x[fpad<TP>(idx)] = u[m];
                else if constexpr (DST == DST_SMEM_MAP) x[st(idx)] = u[m];
                else st(idx, u[m]);
            }
        }
    }
    if constexpr (TO_SMEM) fft_sync<true, WS>();
}

// Largest final radix whose pass fft_pass_tail2 fuses (build-time knob, default 2).  Measured on
// B200: with radix-4 tails too, the FP32 1024-point y transforms (16 x 16 x 4) ran slower --
// y-inverse 38.4 -> 41.2 us, y-forward 43.6 -> 46.2 us, mixed 1024^2 x 8 step 1.021 -> 1.058
// ms: FP32 values are cheap to exchange through shared memory, and the rounds' selects are not
#ifndef QGN_TAIL_RADIX_MAX
#define QGN_TAIL_RADIX_MAX 2
#endif

// whether fft_pass_tail2 takes the pass at sub-length NS and the last one
template <int N, int NS, int TP, int IL>
__host__ __device__ constexpr bool tail2_applies() {
    if (IL <= 0 || IL > 16 || 32 % IL != 0) return false;
    if (N / NS < TP || N % (TP * NS) != 0) return false;
    const int rl = N / (TP * NS);                         // a radix-TP pass, then the radix-rl one
    if ((rl != 2 && rl != 4 && rl != 8) || rl > QGN_TAIL_RADIX_MAX) return false;
    if ((32 / IL) % rl != 0) return false;                // the rl partners in one warp row
    if (FFTShape<N, TP>::T != TP) return false;
    return FFTShape<N, TP>::G % (32 / IL) == 0;           // the transform's threads fill whole warp rows
}

// IL: 0, or the interleave of the caller's threads (see fft_pass_tail2), which fuses the last
// two passes when the last one is radix 2 and its partners sit in one warp
template <int N, int NS, int DIR, int SRC0, int DSTL, int TP, bool WS, int IL, class CT, class Ld, class St>
__device__ __forceinline__ void fft_rec(CT* x, int lane, bool active, const CT* __restrict__ tw, Ld& ld, St& st) {
    constexpr int R = (N / NS >= TP) ? TP : N / NS;
    constexpr bool FIRST = (NS == 1);
    constexpr bool LAST = (NS * R == N);
    constexpr int SRC = FIRST ? SRC0 : SRC_SMEM;
    constexpr int DST = LAST ? DSTL : DST_SMEM;
    constexpr bool TAIL2 = tail2_applies<N, NS, TP, IL>();
    if constexpr (TAIL2) {
        fft_pass_tail2<N, NS, DIR, SRC, DSTL, TP, WS, IL>(x, lane, active, tw, ld, st);
    } else {
        fft_pass_io<N, NS, DIR, SRC, DST, TP, WS>(x, lane, active, tw, ld, st);
        if constexpr (!LAST) fft_rec<N, NS * R, DIR, SRC0, DSTL, TP, WS, IL>(x, lane, active, tw, ld, st);
    }
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
template <int N, int DIR, int SRC0, int DSTL, int TP = 16, bool WS = false, int IL = 0, class CT, class Ld, class St>
__device__ __forceinline__ void fft_fused(CT* x, int lane, bool active, const CT* __restrict__ tw, Ld ld, St st) {
    fft_rec<N, 1, DIR, SRC0, DSTL, TP, WS, IL>(x, lane, active, tw, ld, st);
}

// In-place N-point transform of the padded array x (caller syncs before; ends with a barrier).
template <int N, int DIR, int TP = 16, class CT>
__device__ __forceinline__ void fft_block(CT* x, int lane, bool active, const CT* __restrict__ tw) {
    NoIOT<CT> io;
    fft_rec<N, 1, DIR, SRC_SMEM, DST_SMEM, TP, false, 0>(x, lane, active, tw, io, io);
}

}  // namespace qgn
