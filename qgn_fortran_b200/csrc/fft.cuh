// fft.cuh -- FP64 shared-memory FFT building blocks for sm_100a.
//
// A transform of length N (power of two, 16..2048) is carried out by G = N/T threads
// (T = 16 elements per thread, fewer for N < 16) as a sequence of Stockham
// decimation-in-time radix passes: radix 16 for every pass except the last, which
// takes the remaining factor.  Each pass reads T values from shared memory into
// registers, applies the inter-pass twiddles, performs register-resident radix-R
// DFTs and writes the results back in place (the load and store halves of a pass
// are separated by a block barrier).  Indices are padded by one element per 16
// (p -> p + p/16) so that both the strided stores of the first pass and the
// contiguous accesses of later passes are free of 16-byte bank-group conflicts.
//
// Twiddles come from a per-length table tw[m] = exp(-2*pi*i*m/N) computed on the
// host in long double; DIR=-1 is the forward (exp(-i...)) transform of MKL's
// DftiComputeForward, DIR=+1 the unnormalised backward transform.
#pragma once
#include <cuda_runtime.h>

namespace qgn {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// (i * s) * a for real s
__device__ __forceinline__ double2 cmul_i(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

// padded shared-memory index of element p of a transform
__device__ __forceinline__ int fpad(int p) { return p + (p >> 4); }
// padded length of one transform of length N
__host__ __device__ constexpr int fpadlen(int N) { return N + (N >> 4); }

// Multiply by exp(DIR * 2*pi*i * m/16); m is a compile-time constant after unrolling.
template <int DIR>
__device__ __forceinline__ double2 rot16(double2 a, int m) {
    constexpr double C1 = 0.92387953251128675613;  // cos(pi/8)
    constexpr double S1 = 0.38268343236508977173;  // sin(pi/8)
    constexpr double HH = 0.70710678118654752440;  // sqrt(2)/2
    switch (m & 15) {
        case 0: return a;
        case 4: return DIR > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
        case 8: return make_double2(-a.x, -a.y);
        case 12: return DIR > 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
        case 2: { double s = DIR * HH; return make_double2(HH * a.x - s * a.y, s * a.x + HH * a.y); }
        case 6: { double s = DIR * HH; return make_double2(-HH * a.x - s * a.y, s * a.x - HH * a.y); }
        case 10: { double s = -DIR * HH; return make_double2(-HH * a.x - s * a.y, s * a.x - HH * a.y); }
        case 14: { double s = -DIR * HH; return make_double2(HH * a.x - s * a.y, s * a.x + HH * a.y); }
        default: break;
    }
    double c, s;
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
    return make_double2(a.x * c - a.y * s, a.x * s + a.y * c);
}

// In-register DFT of length R (1,2,4,8,16), natural order in and out, sign DIR.
template <int R, int DIR>
struct RegDFT {
    __device__ __forceinline__ static void run(double2* v) {
        double2 e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
        RegDFT<R / 2, DIR>::run(e);
        RegDFT<R / 2, DIR>::run(o);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) {
            double2 t = rot16<DIR>(o[k], k * (16 / R));
            v[k] = cadd(e[k], t);
            v[k + R / 2] = csub(e[k], t);
        }
    }
};
template <int DIR>
struct RegDFT<1, DIR> {
    __device__ __forceinline__ static void run(double2*) {}
};
template <int DIR>
struct RegDFT<2, DIR> {
    __device__ __forceinline__ static void run(double2* v) {
        double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int N>
struct FFTShape {
    static constexpr int T = N < 16 ? N : 16;   // elements per thread
    static constexpr int G = N / T;             // threads per transform
};

// twiddle w^r for r = 1..R-1 with w = table[k*S] (conjugated for DIR=+1);
// powers of two are read from the table, the rest formed by at most 3 products.
template <int R, int DIR>
__device__ __forceinline__ void load_twiddles(double2* w, const double2* __restrict__ tw, int kS) {
    w[0] = make_double2(1.0, 0.0);
#pragma unroll
    for (int r = 1; r < R; ++r) {
        if ((r & (r - 1)) == 0) {
            double2 t = __ldg(&tw[r * kS]);
            w[r] = DIR > 0 ? cconj(t) : t;
        }
    }
#pragma unroll
    for (int r = 3; r < R; ++r) {
        if ((r & (r - 1)) != 0) {
            const int hi = r >= 8 ? 8 : (r >= 4 ? 4 : 2);
            w[r] = cmul(w[hi], w[r - hi]);
        }
    }
}

// One Stockham DIT pass (current sub-transform length NS, radix R) of an N-point
// transform stored padded at x.  lane in [0,G).
template <int N, int NS, int DIR>
__device__ __forceinline__ void fft_pass(double2* x, int lane, bool active, const double2* __restrict__ tw) {
    constexpr int T = FFTShape<N>::T;
    constexpr int G = FFTShape<N>::G;
    constexpr int R = (N / NS >= 16) ? 16 : N / NS;
    constexpr int BPT = T / R;           // butterflies per thread
    constexpr int STRIDE = N / R;
    double2 v[T];
    if (active) {
#pragma unroll
        for (int b = 0; b < BPT; ++b) {
            int j = lane + b * G;
#pragma unroll
            for (int r = 0; r < R; ++r) v[b * R + r] = x[fpad(j + r * STRIDE)];
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int b = 0; b < BPT; ++b) {
            int j = lane + b * G;
            int k = j & (NS - 1);
            if (NS > 1) {
                double2 w[R];
                load_twiddles<R, DIR>(w, tw, k * (N / (NS * R)));
#pragma unroll
                for (int r = 1; r < R; ++r) v[b * R + r] = cmul(v[b * R + r], w[r]);
            }
            RegDFT<R, DIR>::run(&v[b * R]);
            int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) x[fpad(base + r * NS)] = v[b * R + r];
        }
    }
    __syncthreads();
}

template <int N, int NS, int DIR>
__device__ __forceinline__ void fft_passes(double2* x, int lane, bool active, const double2* __restrict__ tw) {
    if constexpr (NS < N) {
        constexpr int R = (N / NS >= 16) ? 16 : N / NS;
        fft_pass<N, NS, DIR>(x, lane, active, tw);
        fft_passes<N, NS * R, DIR>(x, lane, active, tw);
    }
}

// In-place N-point transform of the padded array x by the G threads with lane in [0,G).
// Every thread of the block must call this (it contains __syncthreads); threads that
// own no transform pass active=false and only take part in the barriers.  The caller
// syncs before (data ready); the function ends with a barrier.
template <int N, int DIR>
__device__ __forceinline__ void fft_block(double2* x, int lane, bool active, const double2* __restrict__ tw) {
    fft_passes<N, 1, DIR>(x, lane, active, tw);
}

}  // namespace qgn
