// cnn.cu -- the learned subgrid closure's convolutional network on the tensor cores.
//
// Network: L periodic 3x3 convolutions (stride 1, "same" with periodic wrap, as the doubly
// periodic QG domain), GELU after every layer but the last.  Activations are NHWC BF16 with
// the channel count padded to a multiple of 16; weights are FP32 masters with BF16 copies in
// two layouts (forward: [tap][cout][cin], backward-data: [tap'][cin][cout] with the taps
// mirrored); products run on the BF16 tensor cores with FP32 accumulation: tcgen05.mma with
// the accumulator tile in TMEM (default; forward, backward-data and weight gradients), or the
// warp-level mma.m16n8k16 path (selectable with qgn_cnn_set_engine or QGN_CNN_MMA=sync).  An inference
// whose tiles fit one CTA each runs all layers in one cooperative launch (k_cnn_fused);
// QGN_CNN_MMA=layers keeps one tcgen05 launch per layer.
//
// Kernels (one CTA = 8 warps = 128 consecutive pixels of one image row, persistent over rows):
//   k_conv<CIN,COUT,EPI>  implicit GEMM  out[p, n] = sum_{tap, k} in[p + tap, k] w[tap, n, k]
//                         EPI_GELU:      Z = acc + bias (FP32), A = bf16(GELU(Z))
//                         EPI_LINEAR:    Y = acc + bias (FP32)
//                         EPI_GELU_GRAD: G = bf16(acc * GELU'(Z))   (backward through a layer)
//   k_wgrad<CIN,COUT>     dW[tap, n, k] partials = sum_p G[p, n] in[p + tap, k] per row chunk
//   k_reduce_*            deterministic chunk sums of dW and the bias gradient
//   k_mse                 loss and dL/dY = 2 (Y - T)/count, as BF16 G of the last layer
//   k_adam                Adam on the FP32 masters, refreshing both BF16 layouts
//   k_conv_tc<CIN,COUT,EPI>  the implicit GEMM on tcgen05 (TMEM accumulators)
//   k_wgrad_tc<CIN,COUT>  the weight-gradient partials on tcgen05 (M = 64, MN-major operands)
//   k_cnn_fused           every layer of a small-batch inference, rows exchanged through L2
#include "qgn_internal.cuh"
#include "cnn.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

namespace qgn {
namespace cnn {

constexpr int kTileP = 128;          // pixels per CTA tile (one row segment)
constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
// Warps of the tcgen05 convolutions (one CTA per SM either way: shared memory).  The fused
// small-batch inference has one tile per CTA and per layer, with nothing to overlap its epilogue
// (TMEM loads, bias, GELU, BF16 packing, staged stores), so 16 warps each drain 16 accumulator
// columns: the 128^2 batch-1 inference ran 58.2 -> 53.7 us on B200.  The persistent layer kernel
// overlaps each tile's epilogue with the next tile's MMAs and stays at 8 warps (16 made the
// batch-32 forward 231 -> 228 TFLOP/s and a training step 3.92 -> 4.06 ms).
constexpr int kTcWarps = 8;
constexpr int kTcThreads = kTcWarps * 32;
constexpr int kFusedWarps = 16;
constexpr int kFusedThreads = kFusedWarps * 32;
constexpr int kWChunkRows = 16;      // image rows per weight-gradient partial

// EPI_PLANAR: as EPI_LINEAR but the FP32 output is planar, out[n][pixel] (the closure's input
// to its forward transform)
// EPI_GELU_ACT: as EPI_GELU without the FP32 pre-activation (inference: only the BF16
// activation feeds the next layer)
enum { EPI_GELU = 0, EPI_LINEAR = 1, EPI_GELU_GRAD = 2, EPI_PLANAR = 3, EPI_GELU_ACT = 4 };

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

// D += A(16x16, row) * B(16x8, col), BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <int C>
struct RowPad {
    static constexpr int LD = C + 8;   // bf16 elements per pixel in shared memory (16-byte skew)
};

// copy pixels [w0-1, w0+128] (periodic) of image row (b, h) into smem rows of LD elements
template <int C>
__device__ __forceinline__ void load_row(const __nv_bfloat16* __restrict__ src, int b, int h, int H, int W, int w0,
                                         int halo, __nv_bfloat16* dst) {
    constexpr int V = C / 8;   // 16-byte vectors per pixel
    const int npix = kTileP + 2 * halo;
    const size_t rowbase = ((size_t)b * H + h) * W;
    for (int i = threadIdx.x; i < npix * V; i += kThreads) {
        const int px = i / V, v = i % V;
        int w = w0 - halo + px;
        w = (w % W + W) % W;
        const uint4 val = *reinterpret_cast<const uint4*>(src + (rowbase + w) * C + v * 8);
        *reinterpret_cast<uint4*>(dst + px * RowPad<C>::LD + v * 8) = val;
    }
}

// ---- implicit-GEMM periodic 3x3 convolution -------------------------------------------------
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kThreads, 1)
    k_conv(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ wt, const float* __restrict__ bias,
           int B, int H, int W, float* __restrict__ outf, __nv_bfloat16* __restrict__ outb,
           const float* __restrict__ zin) {
    QGN_PDL_ENTRY();
    static_assert(CIN % 16 == 0 && COUT % 16 == 0, "channel counts are padded to 16");
    constexpr int LDI = RowPad<CIN>::LD;
    constexpr int NT = COUT / 8;       // n-tiles of 8 output channels per warp
    extern __shared__ __align__(16) unsigned char smraw[];
    __nv_bfloat16* ws = reinterpret_cast<__nv_bfloat16*>(smraw);           // [9][COUT][LDI]
    __nv_bfloat16* xs = ws + 9 * COUT * LDI;                                 // [3][130][LDI]
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    // weights once per CTA
    for (int i = threadIdx.x; i < 9 * COUT * (CIN / 8); i += kThreads) {
        const int row = i / (CIN / 8), v = i % (CIN / 8);
        *reinterpret_cast<uint4*>(ws + row * LDI + v * 8) = *reinterpret_cast<const uint4*>(wt + (size_t)row * CIN + v * 8);
    }
    const int segs = W / kTileP;
    const int ntiles = B * H * segs;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int seg = tile % segs;
        const int h = (tile / segs) % H;
        const int b = tile / (segs * H);
        const int w0 = seg * kTileP;
        __syncthreads();   // previous tile's readers of xs are done (and the weights are in)
        for (int r = 0; r < 3; ++r)
            load_row<CIN>(x, b, (h + r - 1 + H) % H, H, W, w0, 1, xs + r * (kTileP + 2) * LDI);
        __syncthreads();
        float acc[NT][4];
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
        const int pbase = warp * 16;
#pragma unroll 1
        for (int tap = 0; tap < 9; ++tap) {
            const int dh = tap / 3, dw = tap % 3;      // offsets +1 (halo included)
            const __nv_bfloat16* xr = xs + dh * (kTileP + 2) * LDI;
            const __nv_bfloat16* wr = ws + tap * COUT * LDI;
#pragma unroll
            for (int kc = 0; kc < CIN / 16; ++kc) {
                uint32_t a0, a1, a2, a3;
                {
                    const int prow = pbase + (lane % 8) + 8 * ((lane / 8) % 2);
                    const int kcol = kc * 16 + 8 * (lane / 16);
                    ldsm_x4(smem_u32(xr + (prow + dw) * LDI + kcol), a0, a1, a2, a3);
                }
#pragma unroll
                for (int j = 0; j < NT; j += 2) {
                    uint32_t b0, b1, b2, b3;
                    const int n = j * 8 + (lane % 8) + 8 * (lane / 16);
                    const int kcol = kc * 16 + 8 * ((lane / 8) % 2);
                    ldsm_x4(smem_u32(wr + n * LDI + kcol), b0, b1, b2, b3);
                    mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
                    mma_bf16(acc[j + 1], a0, a1, a2, a3, b2, b3);
                }
            }
        }
        // epilogue: thread holds pixels g, g+8 of the warp's 16 and channels 2t, 2t+1 of each n-tile
        const int g = lane / 4, t = lane % 4;
        const size_t prow0 = ((size_t)b * H + h) * W + w0 + pbase;
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int n = j * 8 + 2 * t;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const size_t p = prow0 + g + 8 * half;
                float v0 = acc[j][2 * half], v1 = acc[j][2 * half + 1];
                if (EPI == EPI_PLANAR) {
                    const size_t np = (size_t)B * H * W;
                    outf[(size_t)n * np + p] = v0 + bias[n];
                    outf[(size_t)(n + 1) * np + p] = v1 + bias[n + 1];
                } else if (EPI == EPI_GELU || EPI == EPI_LINEAR) {
                    v0 += bias[n];
                    v1 += bias[n + 1];
                    *reinterpret_cast<float2*>(outf + p * COUT + n) = make_float2(v0, v1);
                    if (EPI == EPI_GELU)
                        *reinterpret_cast<__nv_bfloat162*>(outb + p * COUT + n) =
                            __floats2bfloat162_rn(gelu(v0), gelu(v1));
                } else {
                    const float2 z = *reinterpret_cast<const float2*>(zin + p * COUT + n);
                    *reinterpret_cast<__nv_bfloat162*>(outb + p * COUT + n) =
                        __floats2bfloat162_rn(v0 * gelu_grad(z.x), v1 * gelu_grad(z.y));
                }
            }
        }
    }
}

// ---- weight gradient: partial[chunk][tap][n][k] = sum over the chunk's pixels of G[p,n] in[p+tap,k]
template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreads, 1)
    k_wgrad(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ gr, int B, int H, int W,
            float* __restrict__ part) {
    QGN_PDL_ENTRY();
    constexpr int LDI = RowPad<CIN>::LD, LDG = RowPad<COUT>::LD;
    constexpr int MT = CIN / 16, NT = COUT / 8;
    constexpr int TILES = MT * NT;                  // 16x8 output tiles of dW[tap]
    constexpr int PERW = (TILES + kWarps - 1) / kWarps;
    static_assert(TILES % kWarps == 0 || TILES < kWarps, "tiles split evenly over warps");
    extern __shared__ __align__(16) unsigned char smraw[];
    __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smraw);    // [130][LDI]
    __nv_bfloat16* gs = xs + (kTileP + 2) * LDI;                      // [128][LDG]
    const int tap = blockIdx.y;
    const int dh = tap / 3 - 1, dw = tap % 3 - 1;
    const int chunk = blockIdx.x;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int segs = W / kTileP;
    const int rows_total = B * H;
    const int r0 = chunk * kWChunkRows, r1 = min(rows_total, r0 + kWChunkRows);
    float acc[PERW][4];
#pragma unroll
    for (int i = 0; i < PERW; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    for (int row = r0; row < r1; ++row) {
        const int b = row / H, h = row % H;
        for (int seg = 0; seg < segs; ++seg) {
            const int w0 = seg * kTileP;
            __syncthreads();
            load_row<CIN>(x, b, (h + dh + H) % H, H, W, w0, 1, xs);
            load_row<COUT>(gr, b, h, H, W, w0, 0, gs);
            __syncthreads();
#pragma unroll 1
            for (int kp = 0; kp < kTileP / 16; ++kp) {
#pragma unroll
                for (int i = 0; i < PERW; ++i) {
                    const int tt = warp * PERW + i;
                    if (tt >= TILES) break;
                    const int mt = tt / NT, nt = tt % NT;
                    uint32_t a0, a1, a2, a3, b0, b1, b2, b3;
                    {
                        // A = in^T (rows k = input channel, cols = pixel): transposed 8x8 loads
                        const int mj = lane / 8, r = lane % 8;
                        const int p = kp * 16 + r + 8 * (mj / 2) + 1 + dw;     // +1: halo offset
                        const int k = mt * 16 + 8 * (mj % 2);
                        ldsm_x4_t(smem_u32(xs + p * LDI + k), a0, a1, a2, a3);
                    }
                    {
                        // B = G (rows = pixel, cols n): b0 = pixels 0-7, b1 = pixels 8-15 (transposed)
                        const int mj = lane / 8, r = lane % 8;
                        const int p = kp * 16 + r + 8 * (mj % 2);
                        const int n = (nt & ~1) * 8 + 8 * (mj / 2);
                        ldsm_x4_t(smem_u32(gs + p * LDG + n), b0, b1, b2, b3);
                    }
                    if (nt % 2 == 0) mma_bf16(acc[i], a0, a1, a2, a3, b0, b1);
                    else mma_bf16(acc[i], a0, a1, a2, a3, b2, b3);
                }
            }
        }
    }
    // acc[i]: rows k = mt*16 + g (+8), cols n = nt*8 + 2t (+1)
    const int g = lane / 4, t = lane % 4;
    float* out = part + ((size_t)chunk * 9 + tap) * COUT * CIN;
#pragma unroll
    for (int i = 0; i < PERW; ++i) {
        const int tt = warp * PERW + i;
        if (tt >= TILES) break;
        const int mt = tt / NT, nt = tt % NT;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int k = mt * 16 + g + 8 * half;
            const int n = nt * 8 + 2 * t;
            out[(size_t)n * CIN + k] = acc[i][2 * half];
            out[(size_t)(n + 1) * CIN + k] = acc[i][2 * half + 1];
        }
    }
}

__global__ void k_reduce_wgrad(const float* __restrict__ part, int nchunks, int n, float* __restrict__ dw) {
    QGN_PDL_ENTRY();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int c = 0; c < nchunks; ++c) s += part[(size_t)c * n + i];
        dw[i] = s;
    }
}

// bias gradient: per-block column sums of G, then a chunk reduction
__global__ void k_bias_part(const __nv_bfloat16* __restrict__ gr, long long npix, int C, int pix_per_block,
                            float* __restrict__ part) {
    QGN_PDL_ENTRY();
    const long long p0 = (long long)blockIdx.x * pix_per_block;
    const long long p1 = min(npix, p0 + pix_per_block);
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        float s = 0.f;
        for (long long p = p0; p < p1; ++p) s += __bfloat162float(gr[p * C + c]);
        part[(size_t)blockIdx.x * C + c] = s;
    }
}

// MSE over the real output channels; G = bf16(2 (Y - T) / count), zero in padded channels
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ tgt, long long npix, int C, int creal,
                      double inv_count, __nv_bfloat16* __restrict__ g, double* __restrict__ loss_part) {
    QGN_PDL_ENTRY();
    __shared__ double red[kThreads / 32];
    double s = 0.0;
    const long long n = npix * C;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        float gv = 0.f;
        if (c < creal) {
            const float d = y[i] - tgt[i];
            s += (double)d * (double)d;
            gv = (float)(2.0 * inv_count) * d;
        }
        g[i] = __float2bfloat16_rn(gv);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) tot += red[i];
        loss_part[blockIdx.x] = tot * inv_count;
    }
}

// Adam (bias-corrected) on FP32 masters [9][cout][cin]; refreshes the forward ([tap][cout][cin])
// and backward-data ([8-tap][cin][cout]) BF16 copies
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, int n, int cout, int cin, float lr, float b1, float b2, float eps,
                       float c1, float c2, __nv_bfloat16* __restrict__ wf, __nv_bfloat16* __restrict__ wb) {
    QGN_PDL_ENTRY();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wf) {
            const int tap = i / (cout * cin), r = i % (cout * cin);
            const int co = r / cin, ci = r % cin;
            const __nv_bfloat16 bv = __float2bfloat16_rn(wi);
            wf[i] = bv;
            wb[((size_t)(8 - tap) * cin + ci) * cout + co] = bv;
        }
    }
}

__global__ void k_adam_bias(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    QGN_PDL_ENTRY();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_weights_bf16(const float* __restrict__ w, int n, int cout, int cin, __nv_bfloat16* __restrict__ wf,
                               __nv_bfloat16* __restrict__ wb) {
    QGN_PDL_ENTRY();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int tap = i / (cout * cin), r = i % (cout * cin);
        const int co = r / cin, ci = r % cin;
        const __nv_bfloat16 bv = __float2bfloat16_rn(w[i]);
        wf[i] = bv;
        wb[((size_t)(8 - tap) * cin + ci) * cout + co] = bv;
    }
}

// gather batch samples: dst[b] = src[idx[b]] (rows of `bytes` bytes, 16-byte multiples)
__global__ void k_gather(const unsigned char* __restrict__ src, const int* __restrict__ idx, int nb, size_t bytes,
                         unsigned char* __restrict__ dst) {
    QGN_PDL_ENTRY();
    const size_t vec = bytes / 16;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vec * nb; i += (size_t)gridDim.x * blockDim.x) {
        const size_t b = i / vec, o = i % vec;
        reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src + (size_t)idx[b] * bytes)[o];
    }
}

// ---- the same convolution on the 5th-generation tensor cores (tcgen05, accumulator in TMEM) ----
// One tile = 128 consecutive pixels of an image row (GEMM M = 128) x all COUT output channels
// (N = COUT) with K = 9 taps x CIN, issued as 9*CIN/16 tcgen05.mma (kind::f16, BF16 in, FP32
// accumulate) by one thread; the FP32 tile lives in TMEM (COUT columns, one lane per pixel) and
// the epilogue reads it back with tcgen05.ld.  Operands sit in shared memory in the canonical
// K-major no-swizzle layout (core matrices of 8 rows x 16 bytes):
//   input rows  ring of 4 slots [CIN/8 chunks][130 pixels][8 channels]; the A tile of tap
//               (dh, dw) starts at pixel dw of the slot holding row h+dh-1: rows (pixels) 16 B
//               apart, 8-row groups 128 B apart (SBO), the two halves of a K step 130*16 B apart (LBO);
//   weights     [9 taps][CIN/8 chunks][COUT][8]: SBO 128 B, LBO COUT*16 B.
// Each CTA takes a contiguous range of tiles ordered row-fastest, so consecutive tiles share two
// of their three input rows: one new row per tile, fetched with cp.async into the free ring slot
// while the current tile's MMAs run.  Completion is signalled by tcgen05.commit on an mbarrier;
// every wait is bounded, and a wait that runs out records an error, waits once more, frees the
// TMEM and returns.
namespace tc {

constexpr int kPixS = kTileP + 2;        // staged pixels per input row (periodic halo)
constexpr int kSlots = 6;                // input-row ring: rows of the tile in flight and the next
constexpr long long kWaitLimit = 1LL << 22;

constexpr int imax(int a, int b) { return a > b ? a : b; }

// Shared-memory plan.  SMEM also covers the bytes an MMA would read if the hardware took the
// two descriptor strides the other way round (8-row groups LBO apart, K halves SBO apart):
// every operand read of the kernel stays inside the CTA's allocation under either reading.
template <int CIN, int COUT>
struct Lay {
    static constexpr int SLOT_BYTES = (CIN / 8) * kPixS * 16;
    static constexpr int IN_BYTES = kSlots * SLOT_BYTES;
    static constexpr int W_OFF = (IN_BYTES + 1023) / 1024 * 1024;
    static constexpr int W_BYTES = 9 * (CIN / 8) * COUT * 16;
    static constexpr int BAR_OFF = (W_OFF + W_BYTES + 1023) / 1024 * 1024;
    static constexpr int A_LAST = (kSlots - 1) * SLOT_BYTES + ((CIN / 8 - 2) * kPixS + 2) * 16;
    static constexpr int B_LAST = W_OFF + (8 * (CIN / 8) + CIN / 8 - 2) * COUT * 16;
    static constexpr int A_END = A_LAST + imax(kPixS * 16 + 15 * 128, 15 * kPixS * 16 + 128) + 128;
    static constexpr int B_END = B_LAST + imax(COUT * 16 + (COUT / 8 - 1) * 128, (COUT / 8 - 1) * COUT * 16 + 128) + 128;
    static constexpr int OPS_END = (imax(BAR_OFF + 64, imax(A_END, B_END)) + 1023) / 1024 * 1024;
    static constexpr int STF_OFF = OPS_END;                         // FP32 output staging [128][COUT]
    static constexpr int STB_OFF = STF_OFF + kTileP * COUT * 4;     // BF16 output staging [128][COUT]
    static constexpr int SMEM = STB_OFF + kTileP * COUT * 2;
    static constexpr int TMEM_COLS = COUT < 32 ? 64 : 2 * COUT;   // two accumulator tiles, power of two
};

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);   // version 1, no swizzle
}

// M = 128, N = COUT, BF16 x BF16 -> F32, both operands K-major
template <int N>
__host__ __device__ constexpr uint32_t idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(id), "r"(accumulate));
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void cp16(uint32_t saddr, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int NC>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float* v);
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float* v) {
    tmem_ld<16>(taddr, v);
    tmem_ld<16>(taddr + 16, v + 16);
}

// The 9*CIN/16 MMAs of one tile into the accumulator at TMEM address dacc, then a commit that
// arrives on the mbarrier at bar when they have completed.  ra: shared addresses of the ring
// slots holding input rows h-1, h, h+1; w: the layer's weights.  One thread issues.
template <int CIN, int COUT>
__device__ __forceinline__ void issue_tile(uint32_t dacc, const uint32_t* ra, uint32_t w, uint32_t bar) {
    // descriptors without their start address; per MMA the address is added in
    const uint64_t da0 = sdesc(0u, kPixS * 16, 128), db0 = sdesc(0u, COUT * 16, 128);
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
#pragma unroll
        for (int kc = 0; kc < CIN / 16; ++kc) {
            const uint32_t a_addr = ra[tap / 3] + (uint32_t)((2 * kc * kPixS + tap % 3) * 16);
            const uint32_t b_addr = w + (uint32_t)((tap * (CIN / 8) + 2 * kc) * COUT * 16);
            mma(dacc, da0 | (uint64_t)((a_addr >> 4) & 0x3FFFu), db0 | (uint64_t)((b_addr >> 4) & 0x3FFFu),
                idesc<COUT>(), (tap | kc) ? 1u : 0u);
        }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}

// a layer's weights [9][COUT][CIN] (BF16) into the K-major operand layout [9][CIN/8][COUT][8];
// cin and cout are powers of two (16 or 64), so the index split is shifts and masks
template <int NT>
__device__ __forceinline__ void fetch_weights(const __nv_bfloat16* __restrict__ wt, int cin, int cout, uint32_t w) {
    const int c8n = cin >> 3;
    const int lc8 = __ffs(c8n) - 1, lco = __ffs(cout) - 1;
    for (int i = threadIdx.x; i < 9 * cout * c8n; i += NT) {
        const int c8 = i & (c8n - 1), n = (i >> lc8) & (cout - 1), tap = i >> (lc8 + lco);
        cp16(w + (uint32_t)(((tap * c8n + c8) * cout + n) * 16), wt + ((size_t)tap * cout + n) * cin + c8 * 8);
    }
}

// one input row (image b, row hh, pixels w0-1 .. w0+128 periodic) into a ring slot, asynchronously
template <int CIN, int NT>
__device__ __forceinline__ void fetch_row(const __nv_bfloat16* __restrict__ x, int b, int hh, int H, int W, int w0,
                                         uint32_t slot_addr) {
    const size_t row = ((size_t)b * H + hh) * W;
    for (int i = threadIdx.x; i < kPixS * (CIN / 8); i += NT) {
        const int c8 = i % (CIN / 8), px = i / (CIN / 8);
        int ww = w0 - 1 + px;   // in [-1, W]: one periodic wrap at either end
        ww = ww < 0 ? ww + W : (ww >= W ? ww - W : ww);
        cp16(slot_addr + (uint32_t)((c8 * kPixS + px) * 16), x + (row + ww) * CIN + c8 * 8);
    }
}

}  // namespace tc

// Epilogue of one tile: warp w reads TMEM lanes 32 (w % 4).. (one pixel per thread) and a block
// of columns, applies bias + GELU (or GELU' for the backward pass), and writes the tile through
// XOR-swizzled shared-memory staging so that the global stores are contiguous 16-byte pieces.
// The tile's outputs are contiguous in global memory: pixels p0 .. p0+127, COUT channels each.
// Columns of the accumulator each epilogue thread drains (NW warps: four TMEM sub-partitions,
// NW/4 column blocks each when COUT = 64; four warps when COUT = 16) and the first of them.
template <int COUT, int NW>
__host__ __device__ constexpr int epi_ncol() { return COUT == 64 ? 64 / (NW / 4) : 16; }
template <int COUT, int NW>
__device__ __forceinline__ int epi_n0(int warp) { return COUT == 64 ? epi_ncol<COUT, NW>() * (warp / 4) : 0; }

template <int CIN, int COUT, int EPI, int NW>
__device__ __forceinline__ void conv_tc_epilogue(uint32_t tacc, size_t p0, const float* breg,
                                                 float* __restrict__ outf, __nv_bfloat16* __restrict__ outb,
                                                 const float* __restrict__ zin, unsigned char* stf, unsigned char* stb,
                                                 size_t npix) {
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    constexpr int NCOL = epi_ncol<COUT, NW>();
    constexpr int NT = NW * 32;
    constexpr int CF = COUT / 4;        // 16-byte pieces per staged FP32 row
    constexpr int CB = COUT / 8;        // 16-byte pieces per staged BF16 row
    const bool reads = COUT == 64 || warp < 4;
    const int px = 32 * (warp % 4) + lane;
    const int n0 = epi_n0<COUT, NW>(warp);
    if (EPI == EPI_GELU_GRAD) {   // the tile's pre-activations, read contiguously
        for (int i = threadIdx.x; i < kTileP * CF; i += NT) {
            const int r = i / CF, c = i % CF;
            *reinterpret_cast<float4*>(stf + (r * CF + (c ^ (r % CF))) * 16) =
                *reinterpret_cast<const float4*>(zin + (p0 + r) * COUT + c * 4);
        }
        __syncthreads();
    }
    if (reads) {
        float v[NCOL];
        tc::tmem_ld<NCOL>(tacc + ((uint32_t)(32 * (warp % 4)) << 16) + (uint32_t)n0, v);
#pragma unroll
        for (int j = 0; j < NCOL; j += 4) {
            const int c = (n0 + j) / 4;
            float4* fz = reinterpret_cast<float4*>(stf + (px * CF + (c ^ (px % CF))) * 16);
            uint2* fb = reinterpret_cast<uint2*>(stb + (px * CB + (((n0 + j) / 8) ^ (px % CB))) * 16 + ((n0 + j) % 8) * 2);
            if (EPI == EPI_GELU || EPI == EPI_LINEAR || EPI == EPI_PLANAR || EPI == EPI_GELU_ACT) {
                const float4 z = make_float4(v[j] + breg[j], v[j + 1] + breg[j + 1], v[j + 2] + breg[j + 2],
                                             v[j + 3] + breg[j + 3]);
                if (EPI != EPI_GELU_ACT) *fz = z;
                if (EPI == EPI_GELU || EPI == EPI_GELU_ACT) {
                    __nv_bfloat162 g2[2] = {__floats2bfloat162_rn(gelu(z.x), gelu(z.y)),
                                            __floats2bfloat162_rn(gelu(z.z), gelu(z.w))};
                    *fb = *reinterpret_cast<const uint2*>(g2);
                }
            } else {
                const float4 z = *fz;
                __nv_bfloat162 g2[2] = {__floats2bfloat162_rn(v[j] * gelu_grad(z.x), v[j + 1] * gelu_grad(z.y)),
                                        __floats2bfloat162_rn(v[j + 2] * gelu_grad(z.z), v[j + 3] * gelu_grad(z.w))};
                *fb = *reinterpret_cast<const uint2*>(g2);
            }
        }
    }
    __syncthreads();
    if (EPI == EPI_GELU || EPI == EPI_LINEAR) {
        for (int i = threadIdx.x; i < kTileP * CF; i += NT) {
            const int r = i / CF, c = i % CF;
            *reinterpret_cast<float4*>(outf + (p0 + r) * COUT + c * 4) =
                *reinterpret_cast<const float4*>(stf + (r * CF + (c ^ (r % CF))) * 16);
        }
    }
    if (EPI == EPI_PLANAR) {   // out[n][p0 + r]: each channel's 128 pixels are contiguous
        for (int i = threadIdx.x; i < COUT * kTileP; i += NT) {
            const int n = i / kTileP, r = i % kTileP;
            const int c = n / 4;
            outf[(size_t)n * npix + p0 + r] =
                reinterpret_cast<const float*>(stf + (r * CF + (c ^ (r % CF))) * 16)[n % 4];
        }
    }
    if (EPI == EPI_GELU || EPI == EPI_GELU_GRAD || EPI == EPI_GELU_ACT) {
        for (int i = threadIdx.x; i < kTileP * CB; i += NT) {
            const int r = i / CB, c = i % CB;
            *reinterpret_cast<uint4*>(outb + (p0 + r) * COUT + c * 8) =
                *reinterpret_cast<const uint4*>(stb + (r * CB + (c ^ (r % CB))) * 16);
        }
    }
}

// Pipelined over the CTA's tiles: the MMAs of tile t run into TMEM buffer t&1 while the
// epilogue drains tile t-1 from the other buffer, and the next tile's new input row is fetched
// meanwhile.  Input rows live in a 6-slot ring.
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_conv_tc(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ wt, const float* __restrict__ bias,
              int B, int H, int W, float* __restrict__ outf, __nv_bfloat16* __restrict__ outb,
              const float* __restrict__ zin, int* __restrict__ err) {
    QGN_PDL_ENTRY();
    using L = tc::Lay<CIN, COUT>;
    static_assert(COUT == 16 || COUT == 64, "N of the MMA");
    constexpr int NACC = COUT < 32 ? 32 : COUT;           // TMEM columns per accumulator tile
    extern __shared__ __align__(1024) unsigned char smtc[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smtc + L::BAR_OFF);   // bar[0], bar[1]
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smtc + L::BAR_OFF + 32);
    const int warp = threadIdx.x / 32;
    const uint32_t bar_a = smem_u32(bar), in_a = smem_u32(smtc), w_a = smem_u32(smtc + L::W_OFF);

    // this CTA's tiles: a contiguous range of t = ((b * segs + seg) * H + h), rows fastest
    const int segs = W / kTileP;
    const int ntiles = B * H * segs;
    const int per = (ntiles + gridDim.x - 1) / gridDim.x;
    const int t0 = blockIdx.x * per, t1 = min(ntiles, t0 + per);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"((uint32_t)L::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_a));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_a + 8));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc::fetch_weights<kTcThreads>(wt, CIN, COUT, w_a);
    tc::cp_commit();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;
    unsigned char* stf = smtc + L::STF_OFF;
    unsigned char* stb = smtc + L::STB_OFF;
    // this thread's bias values (its columns are the same in every tile)
    constexpr int NCOL = epi_ncol<COUT, kTcWarps>();
    float breg[NCOL];
    {
        const int n0 = epi_n0<COUT, kTcWarps>(warp);
#pragma unroll
        for (int j = 0; j < NCOL; ++j) breg[j] = (EPI == EPI_GELU_GRAD) ? 0.f : bias[n0 + j];
    }
    // Ring slots are handed out round-robin, so the last six rows fetched sit in distinct slots.
    // A tile that continues the previous one (same image and segment, next row) reuses two of
    // its rows and needs one new row, usually prefetched during the previous tile; otherwise
    // all three rows are fetched.  Live rows (previous tile, this tile, the prefetch) are at
    // most the last five fetched, so no slot that an MMA in flight reads is overwritten.
    int next_slot = 0;
    int sl[3] = {0, 0, 0};                  // this tile's slots (rows h-1, h, h+1)
    int pre_slot = -1;                      // slot of the row prefetched for this tile, or -1
    int pbs = -1;
    uint32_t phase[2] = {0u, 0u};
    int pb = 0, ph = 0, pw0 = 0;            // coordinates of the previous tile
    bool failed = false;
    for (int t = t0; t < t1 && !failed; ++t) {
        const int h = t % H, bs = t / H;
        const int seg = bs % segs, b = bs / segs;
        const int w0 = seg * kTileP;
        const bool cont = t > t0 && bs == pbs && h == ph + 1 && H >= 3;
        if (cont) {
            sl[0] = sl[1];
            sl[1] = sl[2];
            if (pre_slot >= 0) {
                sl[2] = pre_slot;
            } else {
                sl[2] = next_slot;
                next_slot = (next_slot + 1) % tc::kSlots;
                tc::fetch_row<CIN, kTcThreads>(x, b, (h + 1) % H, H, W, w0, in_a + (uint32_t)(sl[2] * L::SLOT_BYTES));
            }
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sl[k] = next_slot;
                next_slot = (next_slot + 1) % tc::kSlots;
                tc::fetch_row<CIN, kTcThreads>(x, b, (h + k - 1 + H) % H, H, W, w0, in_a + (uint32_t)(sl[k] * L::SLOT_BYTES));
            }
        }
        pre_slot = -1;
        tc::cp_commit();
        tc::cp_wait_all();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        const int buf = (t - t0) & 1;
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t ra[3] = {in_a + (uint32_t)(sl[0] * L::SLOT_BYTES), in_a + (uint32_t)(sl[1] * L::SLOT_BYTES),
                                    in_a + (uint32_t)(sl[2] * L::SLOT_BYTES)};
            tc::issue_tile<CIN, COUT>(tmem + (uint32_t)(buf * NACC), ra, w_a, bar_a + 8u * (uint32_t)buf);
        }
        // the next tile's new row, if it continues this one.  Only when this tile continued the
        // previous one (or is the first): after a fresh three-row fetch the six slots hold the
        // previous tile's rows, whose MMAs may still be running, and this tile's.
        if ((cont || t == t0) && t + 1 < t1 && (t + 1) / H == bs && h + 1 < H && H >= 3) {
            pre_slot = next_slot;
            next_slot = (next_slot + 1) % tc::kSlots;
            tc::fetch_row<CIN, kTcThreads>(x, b, (h + 2) % H, H, W, w0, in_a + (uint32_t)(pre_slot * L::SLOT_BYTES));
            tc::cp_commit();
        }
        // drain the previous tile while this one's MMAs run
        if (t > t0) {
            const int pbuf = buf ^ 1;
            const bool ok = tc::bar_wait(bar_a + 8u * (uint32_t)pbuf, phase[pbuf]);
            phase[pbuf] ^= 1u;
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0) atomicOr(err, 1);
                failed = true;
            } else {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                conv_tc_epilogue<CIN, COUT, EPI, kTcWarps>(tmem + (uint32_t)(pbuf * NACC), ((size_t)pb * H + ph) * W + pw0, breg,
                                                 outf, outb, zin, stf, stb, (size_t)B * H * W);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();   // the drained buffer and the previous tile's slots are free again
        pbs = bs;
        pb = b;
        ph = h;
        pw0 = w0;
    }
    // the last tile
    if (t1 > t0 && !failed) {
        const int lbuf = (t1 - 1 - t0) & 1;
        const bool ok = tc::bar_wait(bar_a + 8u * (uint32_t)lbuf, phase[lbuf]);
        phase[lbuf] ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(err, 1);
            failed = true;
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            conv_tc_epilogue<CIN, COUT, EPI, kTcWarps>(tmem + (uint32_t)(lbuf * NACC), ((size_t)pb * H + ph) * W + pw0, breg,
                                             outf, outb, zin, stf, stb, (size_t)B * H * W);
        }
    }
    if (failed) {   // once more, bounded, for MMAs still in flight, before the TMEM is freed
        tc::bar_wait(bar_a, phase[0]);
        tc::bar_wait(bar_a + 8u, phase[1]);
    }
    tc::cp_wait_all();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)L::TMEM_COLS));
    }
}

// ---- all layers of an inference in one launch (small batches) --------------------------------
// When every tile (one image row segment) of a batch has a CTA of its own, the network runs as a
// single cooperative launch: CTA t computes tile t of every layer in turn.  Layer l of tile
// (b, h) needs layer l-1 of rows h-1, h, h+1: its own row is its own previous output, the other
// two come from the CTAs of the neighbouring rows, which publish each finished layer by
// incrementing their flag (release after a device-scope fence; the reader polls with an acquire
// load, bounded).  Flags count up across launches: a CTA reads its own flag at entry (every flag
// holds the same value between launches, since each launch adds L-1 to each) and waits for its
// neighbours' flags to reach that base + l.  Each layer writes its own activation buffer, so no
// row is overwritten while a neighbour may still read it.  The next layer's weights are fetched
// while the epilogue drains the accumulator.  A wait that runs out sets bit 2 of the error word
// and the CTA skips its remaining layers; its neighbours then run out too, so the launch ends.
constexpr int kMaxFusedLayers = 8;
constexpr long long kFlagLimit = 1LL << 21;

struct FusedArgs {
    const __nv_bfloat16* x;                       // input [B][H][W][ci[0]]
    __nv_bfloat16* act[kMaxFusedLayers];          // act[l]: input of layer l (l >= 1), [B][H][W][ci[l]]
    const __nv_bfloat16* wt[kMaxFusedLayers];     // [9][co][ci] BF16
    const float* bias[kMaxFusedLayers];
    int ci[kMaxFusedLayers], co[kMaxFusedLayers];
    int L, B, H, W, planar;
    float* y;                                     // last layer: planar [co][B*H*W] or [B][H][W][co]
    unsigned int* flags;                          // one per tile
    int* err;
};

namespace tc {
// shared-memory plan of the fused kernel: three row slots (rows h-1, h, h+1) of up to 64
// channels, one weight block, the accumulator barrier, FP32 and BF16 output staging; the
// operand region also covers reads under the swapped reading of the descriptor strides
struct FusedLay {
    static constexpr int SLOT_BYTES = 8 * kPixS * 16;
    static constexpr int IN_BYTES = 3 * SLOT_BYTES;
    static constexpr int W_OFF = (IN_BYTES + 1023) / 1024 * 1024;
    static constexpr int W_BYTES = 9 * 8 * 64 * 16;
    static constexpr int BAR_OFF = (W_OFF + W_BYTES + 1023) / 1024 * 1024;
    static constexpr int A_LAST = 2 * SLOT_BYTES + (6 * kPixS + 2) * 16;
    static constexpr int B_LAST = W_OFF + (8 * 8 + 8 - 2) * 64 * 16;
    static constexpr int A_END = A_LAST + imax(kPixS * 16 + 15 * 128, 15 * kPixS * 16 + 128) + 128;
    static constexpr int B_END = B_LAST + imax(64 * 16 + 7 * 128, 7 * 64 * 16 + 128) + 128;
    static constexpr int OPS_END = (imax(BAR_OFF + 64, imax(A_END, B_END)) + 1023) / 1024 * 1024;
    static constexpr int STF_OFF = OPS_END;
    static constexpr int STB_OFF = STF_OFF + kTileP * 64 * 4;
    static constexpr int SMEM = STB_OFF + kTileP * 64 * 2;
    static constexpr int TMEM_COLS = 64;
};

__device__ __forceinline__ bool wait_flag(const unsigned int* f, unsigned int target) {
    for (long long i = 0; i < kFlagLimit; ++i) {
        unsigned int v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(f) : "memory");
        if ((int)(v - target) >= 0) return true;
        __nanosleep(64);
    }
    return false;
}
}  // namespace tc

// One layer of the fused inference for this CTA's tile.  Returns false if a wait ran out.
template <int CIN, int COUT, int EPI>
__device__ __forceinline__ bool fused_layer(const FusedArgs& a, int l, int t, int tup, int tdn, int b, int h, int w0,
                                            unsigned int base, uint32_t in_a, uint32_t w_a, uint32_t bar_a,
                                            uint32_t& phase, uint32_t tmem, unsigned char* stf, unsigned char* stb) {
    using FL = tc::FusedLay;
    const int H = a.H, W = a.W;
    const __nv_bfloat16* src = l == 0 ? a.x : a.act[l];
    // the own row needs no wait: it is this CTA's previous output (or the input)
    tc::fetch_row<CIN, kFusedThreads>(src, b, h, H, W, w0, in_a + (uint32_t)FL::SLOT_BYTES);
    tc::cp_commit();
    // the epilogue's bias columns, loaded while the rows and the MMAs are in flight
    const int warp = threadIdx.x / 32;
    constexpr int NCOL = epi_ncol<COUT, kFusedWarps>();
    float breg[NCOL];
    {
        const int n0 = epi_n0<COUT, kFusedWarps>(warp);
#pragma unroll
        for (int j = 0; j < NCOL; ++j) breg[j] = a.bias[l][n0 + j];
    }
    bool ok = true;
    if (l > 0 && threadIdx.x == 0)
        ok = tc::wait_flag(a.flags + tup, base + (unsigned)l) && tc::wait_flag(a.flags + tdn, base + (unsigned)l);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(a.err, 2);
        tc::cp_wait_all();
        return false;
    }
    tc::fetch_row<CIN, kFusedThreads>(src, b, (h - 1 + H) % H, H, W, w0, in_a);
    tc::fetch_row<CIN, kFusedThreads>(src, b, (h + 1) % H, H, W, w0, in_a + 2u * (uint32_t)FL::SLOT_BYTES);
    tc::cp_commit();
    tc::cp_wait_all();   // the rows and this layer's weights
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t ra[3] = {in_a, in_a + (uint32_t)FL::SLOT_BYTES, in_a + 2u * (uint32_t)FL::SLOT_BYTES};
        tc::issue_tile<CIN, COUT>(tmem, ra, w_a, bar_a);
    }
    ok = tc::bar_wait(bar_a, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(a.err, 1);
        tc::bar_wait(bar_a, phase ^ 1u);   // once more, bounded, before the caller frees the TMEM
        return false;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // the MMAs have read the weights: fetch the next layer's while the accumulator drains
    if (l + 1 < a.L) {
        tc::fetch_weights<kFusedThreads>(a.wt[l + 1], a.ci[l + 1], a.co[l + 1], w_a);
        tc::cp_commit();
    }
    const size_t p0 = ((size_t)b * H + h) * W + w0;
    conv_tc_epilogue<CIN, COUT, EPI, kFusedWarps>(tmem, p0, breg, a.y, EPI == EPI_GELU_ACT ? a.act[l + 1] : nullptr,
                                               nullptr, stf, stb, (size_t)a.B * H * W);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    if (l + 1 < a.L) {   // publish the row
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(a.flags + t, 1u);
    } else {
        __syncthreads();
    }
    return true;
}

template <int EPI>
__device__ __forceinline__ bool fused_dispatch(const FusedArgs& a, int l, int t, int tup, int tdn, int b, int h,
                                               int w0, unsigned int base, uint32_t in_a, uint32_t w_a, uint32_t bar_a,
                                               uint32_t& phase, uint32_t tmem, unsigned char* stf, unsigned char* stb) {
    const int ci = a.ci[l], co = a.co[l];
    if (ci == 16 && co == 64)
        return fused_layer<16, 64, EPI>(a, l, t, tup, tdn, b, h, w0, base, in_a, w_a, bar_a, phase, tmem, stf, stb);
    if (ci == 64 && co == 64)
        return fused_layer<64, 64, EPI>(a, l, t, tup, tdn, b, h, w0, base, in_a, w_a, bar_a, phase, tmem, stf, stb);
    if (ci == 64 && co == 16)
        return fused_layer<64, 16, EPI>(a, l, t, tup, tdn, b, h, w0, base, in_a, w_a, bar_a, phase, tmem, stf, stb);
    return fused_layer<16, 16, EPI>(a, l, t, tup, tdn, b, h, w0, base, in_a, w_a, bar_a, phase, tmem, stf, stb);
}

__global__ void __launch_bounds__(kFusedThreads, 1) k_cnn_fused(FusedArgs a) {
    QGN_PDL_ENTRY();
    using FL = tc::FusedLay;
    extern __shared__ __align__(1024) unsigned char smtc[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smtc + FL::BAR_OFF);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smtc + FL::BAR_OFF + 32);
    unsigned int* sbase = reinterpret_cast<unsigned int*>(smtc + FL::BAR_OFF + 40);
    const int warp = threadIdx.x / 32;
    const uint32_t bar_a = smem_u32(bar), in_a = smem_u32(smtc), w_a = smem_u32(smtc + FL::W_OFF);
    const int H = a.H, segs = a.W / kTileP;
    const int t = blockIdx.x;
    const int h = t % H, bs = t / H;
    const int w0 = (bs % segs) * kTileP, b = bs / segs;
    const int tup = t - h + (h - 1 + H) % H, tdn = t - h + (h + 1) % H;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"((uint32_t)FL::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_a));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        unsigned int v;
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(a.flags + t) : "memory");
        *sbase = v;
    }
    tc::fetch_weights<kFusedThreads>(a.wt[0], a.ci[0], a.co[0], w_a);
    tc::cp_commit();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;
    const unsigned int base = *sbase;
    unsigned char* stf = smtc + FL::STF_OFF;
    unsigned char* stb = smtc + FL::STB_OFF;
    uint32_t phase = 0u;
    for (int l = 0; l < a.L; ++l) {
        bool ok;
        if (l + 1 < a.L)
            ok = fused_dispatch<EPI_GELU_ACT>(a, l, t, tup, tdn, b, h, w0, base, in_a, w_a, bar_a, phase, tmem, stf, stb);
        else if (a.planar)
            ok = fused_dispatch<EPI_PLANAR>(a, l, t, tup, tdn, b, h, w0, base, in_a, w_a, bar_a, phase, tmem, stf, stb);
        else
            ok = fused_dispatch<EPI_LINEAR>(a, l, t, tup, tdn, b, h, w0, base, in_a, w_a, bar_a, phase, tmem, stf, stb);
        if (!ok) break;
    }
    tc::cp_wait_all();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)FL::TMEM_COLS));
    }
}

// ---- weight gradient on tcgen05 -------------------------------------------------------------
// dW[tap][n][k] = sum_p G[p][n] X[p + tap][k] as MMAs with M = 64 (the 64-channel side: G when
// COUT = 64, else X, whose channels are then padded to 64 with zero rows), N = the other side's
// channels and K = 16 pixels.  Both operands are read MN-major (channels contiguous), straight
// from the NHWC rows staged in the [channel group][pixel][16 B] layout of the forward pass, so a
// tap's horizontal shift is a 16-byte offset of the descriptor's start address.  One CTA covers
// a chunk of image rows for one tap row dh and keeps the three taps dw in TMEM; each stage (one
// image row segment of 128 pixels: X row h + dh with its periodic halo, G row h) is fetched into
// a three-buffer ring while the previous stage's 24 MMAs run.  On B200 an M = 64 accumulator
// holds row m in TMEM lane 32 (m / 16) + m % 16, and an MN-major no-swizzle descriptor takes the
// stride between 8-pixel (K) groups as its leading byte offset and the stride between 8-channel
// groups as its stride byte offset (both measured with known operands).
namespace tc {
template <int CIN, int COUT>
struct WgLay {
    static constexpr bool A_IS_G = COUT == 64;
    static constexpr int N = A_IS_G ? CIN : COUT;           // MMA N
    static constexpr int XG = A_IS_G ? CIN / 8 : 8;        // channel groups of an X slot
    static constexpr int GG = A_IS_G ? 8 : COUT / 8;       // channel groups of a G slot
    static constexpr int X_BYTES = XG * kPixS * 16;
    static constexpr int G_BYTES = GG * kTileP * 16;
    static constexpr int STAGE = (X_BYTES + G_BYTES + 1023) / 1024 * 1024;
    static constexpr int NST = 3;                          // ring buffers
    static constexpr int BAR_OFF = NST * STAGE;
    static constexpr int SMEM = BAR_OFF + 64;
    static constexpr int TMEM_COLS = 3 * N <= 64 ? 64 : (3 * N <= 128 ? 128 : 256);
    // every byte an MMA reads lies inside its stage, under either reading of LBO/SBO: the
    // furthest is the last pixel group of the last channel group at the largest start offset
    static_assert((16 * 7 + 2) * 16 + (XG - 1) * kPixS * 16 + 2 * 128 <= X_BYTES, "X reads stay in the slot");
    static_assert(16 * 7 * 16 + (GG - 1) * kTileP * 16 + 2 * 128 <= G_BYTES, "G reads stay in the slot");
};

// M = 64, N, BF16 x BF16 -> F32, both operands MN-major
template <int N>
__host__ __device__ constexpr uint32_t idesc_mn() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(64 >> 4) << 24);
}

// one G row segment (image b, row h, pixels w0 .. w0+127) into a slot [C/8][128][16 B]
template <int C, int NT>
__device__ __forceinline__ void fetch_grow(const __nv_bfloat16* __restrict__ g, int b, int h, int H, int W, int w0,
                                          uint32_t slot_addr) {
    const size_t row = ((size_t)b * H + h) * W + w0;
    for (int i = threadIdx.x; i < kTileP * (C / 8); i += NT) {
        const int c8 = i % (C / 8), px = i / (C / 8);
        cp16(slot_addr + (uint32_t)((c8 * kTileP + px) * 16), g + (row + px) * C + c8 * 8);
    }
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
}  // namespace tc

// partial[chunk][tap][n][k] over the chunk's rows for taps 3 dh' + 0..2 (dh' = blockIdx.y)
template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreads, 1)
    k_wgrad_tc(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ gr, int B, int H, int W,
               float* __restrict__ part, int* __restrict__ err) {
    QGN_PDL_ENTRY();
    using L = tc::WgLay<CIN, COUT>;
    constexpr int N = L::N;
    extern __shared__ __align__(1024) unsigned char smw[];
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smw + L::BAR_OFF + 32);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t base_a = smem_u32(smw), bar_a = smem_u32(smw + L::BAR_OFF);
    const int dhi = blockIdx.y, dh = dhi - 1;
    const int chunk = blockIdx.x;
    const int segs = W / kTileP;
    const int r0 = chunk * kWChunkRows, r1 = min(B * H, r0 + kWChunkRows);
    const int S = (r1 - r0) * segs;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"((uint32_t)L::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < L::NST; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_a + 8u * i));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if constexpr (!L::A_IS_G && CIN < 64) {   // X as M: channel groups CIN/8 .. 7 are zero rows
        constexpr int P = tc::kPixS;
        for (int i = threadIdx.x; i < L::NST * (8 - CIN / 8) * P; i += kThreads) {
            const int st = i / ((8 - CIN / 8) * P), r = i % ((8 - CIN / 8) * P);
            *reinterpret_cast<uint4*>(smw + st * L::STAGE + (CIN / 8) * P * 16 + r * 16) = make_uint4(0, 0, 0, 0);
        }
    }
    auto fetch = [&](int s, int buf) {
        const int row = r0 + s / segs, w0 = (s % segs) * kTileP;
        const int b = row / H, h = row % H;
        const uint32_t xs = base_a + (uint32_t)(buf * L::STAGE), gs = xs + (uint32_t)L::X_BYTES;
        tc::fetch_row<CIN, kThreads>(x, b, (h + dh + H) % H, H, W, w0, xs);
        tc::fetch_grow<COUT, kThreads>(gr, b, h, H, W, w0, gs);
        tc::cp_commit();
    };
    fetch(0, 0);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    bool failed = false;
    int issued = 0;   // stages whose MMAs were issued
    for (int s = 0; s < S; ++s) {
        const int buf = s % L::NST;
        if (s + 1 < S) {
            const int nb = (s + 1) % L::NST;
            if (s + 1 >= L::NST) {   // the MMAs of stage s+1-NST read buffer nb
                const bool ok = tc::bar_wait(bar_a + 8u * (uint32_t)nb, (uint32_t)(((s + 1 - L::NST) / L::NST) & 1));
                if (__syncthreads_or(!ok)) {
                    failed = true;
                    break;
                }
            }
            fetch(s + 1, nb);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");   // stage s has landed
        } else {
            tc::cp_wait_all();
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t xs = base_a + (uint32_t)(buf * L::STAGE), gs = xs + (uint32_t)L::X_BYTES;
#pragma unroll
            for (int dw = 0; dw < 3; ++dw) {
#pragma unroll
                for (int kc = 0; kc < kTileP / 16; ++kc) {
                    const uint32_t xa = xs + (uint32_t)((16 * kc + dw) * 16);   // slot pixel 0 is w0 - 1
                    const uint32_t ga = gs + (uint32_t)(16 * kc * 16);
                    const uint64_t xd = tc::sdesc(xa, 128, tc::kPixS * 16), gd = tc::sdesc(ga, 128, kTileP * 16);
                    tc::mma(tmem + (uint32_t)(dw * N), L::A_IS_G ? gd : xd, L::A_IS_G ? xd : gd, tc::idesc_mn<N>(),
                            (s > 0 || kc > 0) ? 1u : 0u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             bar_a + 8u * (uint32_t)buf)
                         : "memory");
        }
        issued = s + 1;
    }
    // the last issued stage's commit covers every earlier MMA of this thread
    bool ok = true;
    if (issued > 0) {
        const int ls = issued - 1;
        ok = tc::bar_wait(bar_a + 8u * (uint32_t)(ls % L::NST), (uint32_t)((ls / L::NST) & 1));
    }
    if (__syncthreads_or(!ok) || failed) {
        if (threadIdx.x == 0) atomicOr(err, 4);
        failed = true;
    }
    if (!failed) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        // warp w reads TMEM lanes 32 (w % 4) ..; its threads 0..15 hold rows m = 16 (w % 4) + lane,
        // and the two warps of a sub-partition split the N columns
        const int m = 16 * (warp % 4) + lane;
        const int c0 = (warp / 4) * (N / 2);
#pragma unroll
        for (int dw = 0; dw < 3; ++dw) {
            const int tap = 3 * dhi + dw;
            float* out = part + ((size_t)chunk * 9 + tap) * COUT * CIN;
#pragma unroll
            for (int c = 0; c < N / 2; c += 8) {
                float v[8];
                tc::tmem_ld8(tmem + ((uint32_t)(32 * (warp % 4)) << 16) + (uint32_t)(dw * N + c0 + c), v);
                if (lane < 16) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int col = c0 + c + j;
                        if constexpr (L::A_IS_G) out[(size_t)m * CIN + col] = v[j];          // D[n][k]
                        else if (m < CIN) out[(size_t)col * CIN + m] = v[j];                 // D[k][n]
                    }
                }
            }
        }
    }
    tc::cp_wait_all();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)L::TMEM_COLS));
    }
}

template <int CIN, int COUT>
constexpr int conv_smem() {
    return (9 * COUT + 3 * (kTileP + 2)) * RowPad<CIN>::LD * 2;
}
template <int CIN, int COUT>
constexpr int wgrad_smem() {
    return ((kTileP + 2) * RowPad<CIN>::LD + kTileP * RowPad<COUT>::LD) * 2;
}

}  // namespace cnn
}  // namespace qgn

using namespace qgn;
using namespace qgn::cnn;

struct qgn_cnn {
    int cin = 0, width = 0, cout = 0, layers = 0;   // real channel counts
    int H = 0, W = 0, max_batch = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<int> ci, co;                         // padded channel counts per layer
    std::vector<float*> w, bias, mw, vw, mb, vb, gw, gb;
    std::vector<__nv_bfloat16*> wf, wb;
    std::vector<float*> z;                           // pre-activations (FP32) per layer
    std::vector<__nv_bfloat16*> act;                 // act[0] = input batch, act[l+1] = GELU(z[l])
    __nv_bfloat16* gA = nullptr;                     // backward: G of the current layer
    __nv_bfloat16* gB = nullptr;
    float* part = nullptr;                           // weight-gradient partials
    size_t part_elems = 0;
    double* loss_part = nullptr;
    double* loss_host = nullptr;
    float* ytgt = nullptr;                           // gathered targets
    long long adam_t = 0;
    int engine = 0;                                  // 0: tcgen05, all layers in one launch when the
                                                     // tiles fit one CTA each; 1: mma.sync; 2: tcgen05
                                                     // one launch per layer
    int* d_err = nullptr;                            // device error word of the tcgen05 kernels
    unsigned int* flags = nullptr;                   // per-tile layer counters of the fused inference
    int fused_tiles = -1;                            // tile count the flags were last used with
    int fused_max_tiles = 0;                         // co-resident CTAs of the fused kernel
    std::vector<void*> owned;
    std::string last_error;
};

namespace {

int cnn_err(qgn_cnn* n, int code, const std::string& m) {
    if (n) n->last_error = m;
    return code;
}

#define NCK(call)                                                                                      \
    do {                                                                                               \
        cudaError_t _e = (call);                                                                       \
        if (_e != cudaSuccess) return cnn_err(net, QGN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

int pad16(int c) { return (c + 15) / 16 * 16; }

template <class T>
cudaError_t nalloc(qgn_cnn* net, T** p, size_t count) {
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
    if (e == cudaSuccess) {
        net->owned.push_back(*p);
        cudaMemsetAsync(*p, 0, sizeof(T) * (count ? count : 1), net->stream);
    }
    return e;
}

size_t npix(const qgn_cnn* n, int batch) { return (size_t)batch * n->H * n->W; }

int conv_grid(const qgn_cnn* n, int batch) {
    const int tiles = batch * n->H * (n->W / kTileP);
    return std::max(1, std::min(tiles, 148));
}

template <int CIN, int COUT, int EPI>
cudaError_t launch_conv_t(qgn_cnn* n, const __nv_bfloat16* x, const __nv_bfloat16* wt, const float* bias, int batch,
                          float* outf, __nv_bfloat16* outb, const float* zin) {
    if (n->engine == 0) {
        constexpr int SM = tc::Lay<CIN, COUT>::SMEM;
        if (cudaError_t e = smem_opt_in(k_conv_tc<CIN, COUT, EPI>, SM); e != cudaSuccess) return e;
        ::qgn::launch(k_conv_tc<CIN, COUT, EPI>, conv_grid(n, batch), kTcThreads, SM, n->stream, x, wt, bias, batch, n->H, n->W,
                                                                                    outf, outb, zin, n->d_err);
        return cudaGetLastError();
    }
    constexpr int SM = conv_smem<CIN, COUT>();
    if (cudaError_t e = smem_opt_in(k_conv<CIN, COUT, EPI>, SM); e != cudaSuccess) return e;
    ::qgn::launch(k_conv<CIN, COUT, EPI>, conv_grid(n, batch), kThreads, SM, n->stream, x, wt, bias, batch, n->H, n->W, outf,
                                                                             outb, zin);
    return cudaGetLastError();
}

template <int EPI>
cudaError_t launch_conv(qgn_cnn* n, int cin, int cout, const __nv_bfloat16* x, const __nv_bfloat16* wt,
                        const float* bias, int batch, float* outf, __nv_bfloat16* outb, const float* zin) {
    if (cin == 16 && cout == 64) return launch_conv_t<16, 64, EPI>(n, x, wt, bias, batch, outf, outb, zin);
    if (cin == 64 && cout == 64) return launch_conv_t<64, 64, EPI>(n, x, wt, bias, batch, outf, outb, zin);
    if (cin == 64 && cout == 16) return launch_conv_t<64, 16, EPI>(n, x, wt, bias, batch, outf, outb, zin);
    if (cin == 16 && cout == 16) return launch_conv_t<16, 16, EPI>(n, x, wt, bias, batch, outf, outb, zin);
    return cudaErrorInvalidValue;
}

template <int CIN, int COUT>
cudaError_t launch_wgrad_t(qgn_cnn* n, const __nv_bfloat16* x, const __nv_bfloat16* g, int batch, float* part,
                           int* nchunks) {
    const int chunks = (batch * n->H + kWChunkRows - 1) / kWChunkRows;
    *nchunks = chunks;
    if (n->engine != 1) {   // tcgen05: one CTA per (row chunk, tap row), the three taps in TMEM
        constexpr int SM = tc::WgLay<CIN, COUT>::SMEM;
        if (cudaError_t e = smem_opt_in(k_wgrad_tc<CIN, COUT>, SM); e != cudaSuccess) return e;
        ::qgn::launch(k_wgrad_tc<CIN, COUT>, dim3(chunks, 3), kThreads, SM, n->stream, x, g, batch, n->H, n->W, part,
                      n->d_err);
        return cudaGetLastError();
    }
    constexpr int SM = wgrad_smem<CIN, COUT>();
    if (cudaError_t e = smem_opt_in(k_wgrad<CIN, COUT>, SM); e != cudaSuccess) return e;
    ::qgn::launch(k_wgrad<CIN, COUT>, dim3(chunks, 9), kThreads, SM, n->stream, x, g, batch, n->H, n->W, part);
    return cudaGetLastError();
}

cudaError_t launch_wgrad(qgn_cnn* n, int cin, int cout, const __nv_bfloat16* x, const __nv_bfloat16* g, int batch,
                         float* part, int* nchunks) {
    if (cin == 16 && cout == 64) return launch_wgrad_t<16, 64>(n, x, g, batch, part, nchunks);
    if (cin == 64 && cout == 64) return launch_wgrad_t<64, 64>(n, x, g, batch, part, nchunks);
    if (cin == 64 && cout == 16) return launch_wgrad_t<64, 16>(n, x, g, batch, part, nchunks);
    if (cin == 16 && cout == 16) return launch_wgrad_t<16, 16>(n, x, g, batch, part, nchunks);
    return cudaErrorInvalidValue;
}

// forward of a batch: layer 0 reads x0 (default act[0]); the last layer's FP32 output goes
// to ylast (default z[L-1])
int forward(qgn_cnn* net, int batch, const __nv_bfloat16* x0 = nullptr, float* ylast = nullptr, bool planar = false) {
    const int L = net->layers;
    for (int l = 0; l < L; ++l) {
        const bool last = l == L - 1;
        const __nv_bfloat16* in = (l == 0 && x0) ? x0 : net->act[l];
        cudaError_t e = (last && planar)
                            ? launch_conv<EPI_PLANAR>(net, net->ci[l], net->co[l], in, net->wf[l], net->bias[l], batch,
                                                      ylast ? ylast : net->z[l], nullptr, nullptr)
                        : last ? launch_conv<EPI_LINEAR>(net, net->ci[l], net->co[l], in, net->wf[l], net->bias[l],
                                                       batch, ylast ? ylast : net->z[l], nullptr, nullptr)
                             : launch_conv<EPI_GELU>(net, net->ci[l], net->co[l], in, net->wf[l], net->bias[l],
                                                     batch, net->z[l], net->act[l + 1], nullptr);
        NCK(e);
    }
    return QGN_OK;
}

// backward from the BF16 output gradient in gA; fills gw/gb of every layer
int backward(qgn_cnn* net, int batch) {
    const int L = net->layers;
    __nv_bfloat16* gcur = net->gA;
    __nv_bfloat16* gnext = net->gB;
    const long long np = (long long)npix(net, batch);
    for (int l = L - 1; l >= 0; --l) {
        int chunks = 0;
        NCK(launch_wgrad(net, net->ci[l], net->co[l], net->act[l], gcur, batch, net->part, &chunks));
        const int nw = 9 * net->co[l] * net->ci[l];
        ::qgn::launch(k_reduce_wgrad, (nw + 255) / 256, 256, 0, net->stream, net->part, chunks, nw, net->gw[l]);
        NCK(cudaGetLastError());
        const int ppb = 1024;
        const int nbp = (int)((np + ppb - 1) / ppb);
        ::qgn::launch(k_bias_part, nbp, 64, 0, net->stream, gcur, np, net->co[l], ppb, net->part);
        NCK(cudaGetLastError());
        ::qgn::launch(k_reduce_wgrad, 1, 64, 0, net->stream, net->part, nbp, net->co[l], net->gb[l]);
        NCK(cudaGetLastError());
        if (l > 0) {
            NCK(launch_conv<EPI_GELU_GRAD>(net, net->co[l], net->ci[l], gcur, net->wb[l], nullptr, batch, nullptr,
                                           gnext, net->z[l - 1]));
            std::swap(gcur, gnext);
        }
    }
    return QGN_OK;
}

int mse(qgn_cnn* net, int batch, const float* tgt) {
    const int L = net->layers;
    const long long np = (long long)npix(net, batch);
    const int C = net->co[L - 1];
    const double inv = 1.0 / ((double)np * net->cout);
    ::qgn::launch(k_mse, 148, kThreads, 0, net->stream, net->z[L - 1], tgt, np, C, net->cout, inv, net->gA, net->loss_part);
    NCK(cudaGetLastError());
    return QGN_OK;
}

int check_err(qgn_cnn* net) {
    int h = 0;
    NCK(cudaMemcpyAsync(&h, net->d_err, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
    NCK(cudaStreamSynchronize(net->stream));
    if (h) {
        net->fused_tiles = -1;   // the layer counters may be uneven: the next fused launch clears them
        NCK(cudaMemsetAsync(net->d_err, 0, sizeof(int), net->stream));   // reported once
        return cnn_err(net, QGN_ERR_CUDA,
                       (h & 2)   ? "the fused inference timed out waiting for a neighbouring row"
                       : (h & 4) ? "a tensor-core weight gradient timed out waiting for its MMAs"
                                 : "a tensor-core convolution timed out waiting for its MMAs");
    }
    return QGN_OK;
}

// the fused single-launch inference applies: tcgen05 engine, at most kMaxFusedLayers layers,
// 128-pixel row segments, at least 3 rows, and one co-resident CTA per tile
bool fused_ok(qgn_cnn* net, int batch) {
    if (net->engine != 0 || net->layers > kMaxFusedLayers || net->H < 3 || net->W % kTileP != 0) return false;
    if (net->fused_max_tiles == 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (smem_opt_in(k_cnn_fused, tc::FusedLay::SMEM) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cnn_fused, kFusedThreads, tc::FusedLay::SMEM) !=
                cudaSuccess)
            per = 0;
        net->fused_max_tiles = per > 0 ? sms * per : -1;
    }
    return (long long)batch * net->H * (net->W / kTileP) <= net->fused_max_tiles;
}

int forward_fused(qgn_cnn* net, int batch, const __nv_bfloat16* x, float* y, bool planar) {
    const int L = net->layers;
    const int tiles = batch * net->H * (net->W / kTileP);
    if (tiles != net->fused_tiles) {
        NCK(cudaMemsetAsync(net->flags, 0, sizeof(unsigned int) * tiles, net->stream));
        net->fused_tiles = tiles;
    }
    FusedArgs a = {};
    a.x = x;
    for (int l = 0; l < L; ++l) {
        a.act[l] = net->act[l];
        a.wt[l] = net->wf[l];
        a.bias[l] = net->bias[l];
        a.ci[l] = net->ci[l];
        a.co[l] = net->co[l];
    }
    a.L = L;
    a.B = batch;
    a.H = net->H;
    a.W = net->W;
    a.planar = planar ? 1 : 0;
    a.y = y;
    a.flags = net->flags;
    a.err = net->d_err;
    // cooperative: every CTA is resident at once, which the waits on neighbouring rows need
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(tiles);
    cfg.blockDim = dim3(kFusedThreads);
    cfg.dynamicSmemBytes = tc::FusedLay::SMEM;
    cfg.stream = net->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    NCK(smem_opt_in(k_cnn_fused, tc::FusedLay::SMEM));   // per device: a no-op after the first
    NCK(cudaLaunchKernelEx(&cfg, k_cnn_fused, a));
    return QGN_OK;
}

int read_loss(qgn_cnn* net, double* loss) {
    NCK(cudaMemcpyAsync(net->loss_host, net->loss_part, sizeof(double) * 148, cudaMemcpyDeviceToHost, net->stream));
    NCK(cudaStreamSynchronize(net->stream));
    if (int rc = check_err(net)) return rc;
    double s = 0.0;
    for (int i = 0; i < 148; ++i) s += net->loss_host[i];
    if (loss) *loss = s;
    return QGN_OK;
}

}  // namespace

namespace qgn {
namespace cnn {
int padded_in(const qgn_cnn* net) { return net->ci[0]; }
int padded_out(const qgn_cnn* net) { return net->co[net->layers - 1]; }
int height(const qgn_cnn* net) { return net->H; }
int width(const qgn_cnn* net) { return net->W; }
int real_out(const qgn_cnn* net) { return net->cout; }
int infer(qgn_cnn* net, const void* x, float* y, int batch, cudaStream_t stream, bool planar) {
    if (batch < 1 || batch > net->max_batch) return QGN_ERR_ARG;
    cudaStream_t own = net->stream;
    net->stream = stream;
    const __nv_bfloat16* xb = static_cast<const __nv_bfloat16*>(x);
    const int rc = fused_ok(net, batch) ? forward_fused(net, batch, xb, y, planar) : forward(net, batch, xb, y, planar);
    net->stream = own;
    return rc;
}
}  // namespace cnn
}  // namespace qgn

extern "C" {

int qgn_cnn_create(int cin, int width, int cout, int layers, int H, int W, int max_batch, unsigned long long seed,
                   qgn_cnn** out) {
    if (!out) return QGN_ERR_ARG;
    *out = nullptr;
    if (cin < 1 || cin > 16 || cout < 1 || cout > 16 || width != 64 || layers < 2 || layers > 16) return QGN_ERR_CONFIG;
    if (H < 1 || W < kTileP || W % kTileP != 0 || max_batch < 1) return QGN_ERR_CONFIG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return QGN_ERR_NO_DEVICE;
    qgn_cnn* net = new (std::nothrow) qgn_cnn();
    if (!net) return QGN_ERR_CUDA;
    net->cin = cin;
    net->width = width;
    net->cout = cout;
    net->layers = layers;
    net->H = H;
    net->W = W;
    net->max_batch = max_batch;
    cudaGetDevice(&net->device);
    auto fail = [&](int code) {
        qgn_cnn_destroy(net);
        return code;
    };
    if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(QGN_ERR_CUDA);
    for (int l = 0; l < layers; ++l) {
        net->ci.push_back(l == 0 ? pad16(cin) : width);
        net->co.push_back(l == layers - 1 ? pad16(cout) : width);
    }
    const size_t NP = npix(net, max_batch);
    net->w.resize(layers); net->bias.resize(layers); net->mw.resize(layers); net->vw.resize(layers);
    net->mb.resize(layers); net->vb.resize(layers); net->gw.resize(layers); net->gb.resize(layers);
    net->wf.resize(layers); net->wb.resize(layers); net->z.resize(layers); net->act.resize(layers + 1);
    size_t part = 0;
    std::mt19937_64 rng(seed);
    for (int l = 0; l < layers; ++l) {
        const int nw = 9 * net->co[l] * net->ci[l];
        if (nalloc(net, &net->w[l], nw) || nalloc(net, &net->mw[l], nw) || nalloc(net, &net->vw[l], nw) ||
            nalloc(net, &net->gw[l], nw) || nalloc(net, &net->wf[l], nw) || nalloc(net, &net->wb[l], nw) ||
            nalloc(net, &net->bias[l], net->co[l]) || nalloc(net, &net->mb[l], net->co[l]) ||
            nalloc(net, &net->vb[l], net->co[l]) || nalloc(net, &net->gb[l], net->co[l]) ||
            nalloc(net, &net->z[l], NP * net->co[l]) || nalloc(net, &net->act[l], NP * net->ci[l]))
            return fail(QGN_ERR_CUDA);
        // He initialisation over the real fan-in, zeros in padded channels
        const int real_in = l == 0 ? cin : width, real_out = l == layers - 1 ? cout : width;
        std::normal_distribution<float> nd(0.f, std::sqrt(2.0f / (9.0f * real_in)) * (l == layers - 1 ? 0.1f : 1.0f));
        std::vector<float> hw(nw, 0.f);
        for (int tap = 0; tap < 9; ++tap)
            for (int o = 0; o < real_out; ++o)
                for (int i = 0; i < real_in; ++i) hw[((size_t)tap * net->co[l] + o) * net->ci[l] + i] = nd(rng);
        if (cudaMemcpyAsync(net->w[l], hw.data(), sizeof(float) * nw, cudaMemcpyHostToDevice, net->stream) !=
            cudaSuccess)
            return fail(QGN_ERR_CUDA);
        cudaStreamSynchronize(net->stream);
        ::qgn::launch(k_weights_bf16, (nw + 255) / 256, 256, 0, net->stream, net->w[l], nw, net->co[l], net->ci[l], net->wf[l],
                                                                  net->wb[l]);
        const size_t chunks = (size_t)((max_batch * H + kWChunkRows - 1) / kWChunkRows);
        part = std::max(part, chunks * nw);
        part = std::max(part, ((NP + 1023) / 1024) * (size_t)net->co[l]);
    }
    if (nalloc(net, &net->act[layers], 16) || nalloc(net, &net->gA, NP * net->width) ||
        nalloc(net, &net->gB, NP * net->width) || nalloc(net, &net->part, part) ||
        nalloc(net, &net->loss_part, 148) || nalloc(net, &net->ytgt, NP * pad16(cout)) ||
        nalloc(net, &net->d_err, 1) || nalloc(net, &net->flags, 1024))
        return fail(QGN_ERR_CUDA);
    net->part_elems = part;
    if (const char* e = std::getenv("QGN_CNN_MMA"))
        net->engine = (std::string(e) == "sync") ? 1 : (std::string(e) == "layers") ? 2 : 0;
    if (cudaMallocHost((void**)&net->loss_host, sizeof(double) * 148) != cudaSuccess) return fail(QGN_ERR_CUDA);
    if (cudaStreamSynchronize(net->stream) != cudaSuccess) return fail(QGN_ERR_CUDA);
    *out = net;
    return QGN_OK;
}

int qgn_cnn_padded_channels(const qgn_cnn* net, int* cin_padded, int* cout_padded) {
    if (!net) return QGN_ERR_ARG;
    if (cin_padded) *cin_padded = net->ci[0];
    if (cout_padded) *cout_padded = net->co[net->layers - 1];
    return QGN_OK;
}

// weights: per layer [9][cout_p][cin_p] FP32 then bias [cout_p], layers in order
long long qgn_cnn_num_params(const qgn_cnn* net) {
    if (!net) return -1;
    long long n = 0;
    for (int l = 0; l < net->layers; ++l) n += 9LL * net->co[l] * net->ci[l] + net->co[l];
    return n;
}

int qgn_cnn_get_weights(qgn_cnn* net, float* host) {
    if (!net || !host) return QGN_ERR_ARG;
    size_t off = 0;
    for (int l = 0; l < net->layers; ++l) {
        const size_t nw = 9ull * net->co[l] * net->ci[l];
        NCK(cudaMemcpyAsync(host + off, net->w[l], sizeof(float) * nw, cudaMemcpyDeviceToHost, net->stream));
        off += nw;
        NCK(cudaMemcpyAsync(host + off, net->bias[l], sizeof(float) * net->co[l], cudaMemcpyDeviceToHost, net->stream));
        off += net->co[l];
    }
    NCK(cudaStreamSynchronize(net->stream));
    return QGN_OK;
}

int qgn_cnn_set_weights(qgn_cnn* net, const float* host) {
    if (!net || !host) return QGN_ERR_ARG;
    size_t off = 0;
    for (int l = 0; l < net->layers; ++l) {
        const int nw = 9 * net->co[l] * net->ci[l];
        NCK(cudaMemcpyAsync(net->w[l], host + off, sizeof(float) * nw, cudaMemcpyHostToDevice, net->stream));
        off += nw;
        NCK(cudaMemcpyAsync(net->bias[l], host + off, sizeof(float) * net->co[l], cudaMemcpyHostToDevice, net->stream));
        off += net->co[l];
        ::qgn::launch(k_weights_bf16, (nw + 255) / 256, 256, 0, net->stream, net->w[l], nw, net->co[l], net->ci[l], net->wf[l],
                                                                  net->wb[l]);
        NCK(cudaGetLastError());
    }
    NCK(cudaStreamSynchronize(net->stream));
    net->adam_t = 0;
    for (int l = 0; l < net->layers; ++l) {
        const int nw = 9 * net->co[l] * net->ci[l];
        NCK(cudaMemsetAsync(net->mw[l], 0, sizeof(float) * nw, net->stream));
        NCK(cudaMemsetAsync(net->vw[l], 0, sizeof(float) * nw, net->stream));
        NCK(cudaMemsetAsync(net->mb[l], 0, sizeof(float) * net->co[l], net->stream));
        NCK(cudaMemsetAsync(net->vb[l], 0, sizeof(float) * net->co[l], net->stream));
    }
    NCK(cudaStreamSynchronize(net->stream));
    return QGN_OK;
}

// inference: x = BF16 [batch][H][W][cin_p] (device), y = FP32 [batch][H][W][cout_p] (device).
// Runs on `stream` (NULL: the network's own stream), ordered after the caller's work there.
int qgn_cnn_forward(qgn_cnn* net, const void* x, float* y, int batch, void* stream) {
    QGN_NVTX("qgn_cnn_forward");
    if (!net || !x || !y || batch < 1 || batch > net->max_batch) return QGN_ERR_ARG;
    return qgn::cnn::infer(net, x, y, batch, stream ? static_cast<cudaStream_t>(stream) : net->stream, false);
}

// gradients of the MSE loss at the current weights for x (BF16 [batch][H][W][cin_p]) and
// targets y (FP32 [batch][H][W][cout_p]); host output in the get_weights layout
int qgn_cnn_gradients(qgn_cnn* net, const void* x, const float* y, int batch, float* grads_host, double* loss) {
    if (!net || !x || !y || batch < 1 || batch > net->max_batch) return QGN_ERR_ARG;
    const size_t xb = npix(net, batch) * net->ci[0] * sizeof(__nv_bfloat16);
    NCK(cudaMemcpyAsync(net->act[0], x, xb, cudaMemcpyDeviceToDevice, net->stream));
    int rc = forward(net, batch);
    if (rc == QGN_OK) rc = mse(net, batch, y);
    if (rc == QGN_OK) rc = backward(net, batch);
    if (rc == QGN_OK) rc = read_loss(net, loss);
    if (rc != QGN_OK) return rc;
    if (grads_host) {
        size_t off = 0;
        for (int l = 0; l < net->layers; ++l) {
            const size_t nw = 9ull * net->co[l] * net->ci[l];
            NCK(cudaMemcpyAsync(grads_host + off, net->gw[l], sizeof(float) * nw, cudaMemcpyDeviceToHost, net->stream));
            off += nw;
            NCK(cudaMemcpyAsync(grads_host + off, net->gb[l], sizeof(float) * net->co[l], cudaMemcpyDeviceToHost,
                                net->stream));
            off += net->co[l];
        }
        NCK(cudaStreamSynchronize(net->stream));
    }
    return QGN_OK;
}

// one Adam step on the batch idx[0..batch) (device int32) of a dataset: x_all BF16
// [n][H][W][cin_p], y_all FP32 [n][H][W][cout_p]; loss (before the update) optional
int qgn_cnn_train_step(qgn_cnn* net, const void* x_all, const float* y_all, const int* idx, int batch, float lr,
                       double* loss) {
    QGN_NVTX("qgn_cnn_train_step");
    if (!net || !x_all || !y_all || !idx || batch < 1 || batch > net->max_batch || !(lr > 0)) return QGN_ERR_ARG;
    const int L = net->layers;
    const size_t xs = (size_t)net->H * net->W * net->ci[0] * sizeof(__nv_bfloat16);
    const size_t ys = (size_t)net->H * net->W * net->co[L - 1] * sizeof(float);
    ::qgn::launch(k_gather, 148 * 4, 256, 0, net->stream, static_cast<const unsigned char*>(x_all), idx, batch, xs,
                                              reinterpret_cast<unsigned char*>(net->act[0]));
    NCK(cudaGetLastError());
    ::qgn::launch(k_gather, 148 * 4, 256, 0, net->stream, reinterpret_cast<const unsigned char*>(y_all), idx, batch, ys,
                                              reinterpret_cast<unsigned char*>(net->ytgt));
    NCK(cudaGetLastError());
    int rc = forward(net, batch);
    if (rc == QGN_OK) rc = mse(net, batch, net->ytgt);
    if (rc == QGN_OK) rc = backward(net, batch);
    if (rc != QGN_OK) return rc;
    net->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)net->adam_t), c2 = 1.f - std::pow(b2, (float)net->adam_t);
    for (int l = 0; l < L; ++l) {
        const int nw = 9 * net->co[l] * net->ci[l];
        ::qgn::launch(k_adam, (nw + 255) / 256, 256, 0, net->stream, net->w[l], net->mw[l], net->vw[l], net->gw[l], nw, net->co[l],
                                                          net->ci[l], lr, b1, b2, eps, c1, c2, net->wf[l], net->wb[l]);
        NCK(cudaGetLastError());
        ::qgn::launch(k_adam_bias, 1, 64, 0, net->stream, net->bias[l], net->mb[l], net->vb[l], net->gb[l], net->co[l], lr, b1, b2,
                                               eps, c1, c2);
        NCK(cudaGetLastError());
    }
    if (loss) return read_loss(net, loss);
    return QGN_OK;
}

int qgn_cnn_set_engine(qgn_cnn* net, int engine) {
    if (!net || engine < 0 || engine > 2) return QGN_ERR_ARG;
    if (cudaStreamSynchronize(net->stream) != cudaSuccess) return QGN_ERR_CUDA;
    net->engine = engine;
    return QGN_OK;
}

// failure injection for tests: set the fused inference's layer counter of one tile.  A large
// value makes that tile's CTA wait, in the next fused launch, for neighbour counters that
// never reach it; the bounded wait runs out and qgn_cnn_check reports it.
int qgn_cnn_debug_set_counter(qgn_cnn* net, int tile, unsigned int value) {
    if (!net || tile < 0 || tile >= 1024) return QGN_ERR_ARG;
    NCK(cudaMemcpyAsync(net->flags + tile, &value, sizeof(value), cudaMemcpyHostToDevice, net->stream));
    NCK(cudaStreamSynchronize(net->stream));
    return QGN_OK;
}

int qgn_cnn_check(qgn_cnn* net) {
    if (!net) return QGN_ERR_ARG;
    return check_err(net);
}

int qgn_cnn_stream(qgn_cnn* net, void** stream) {
    if (!net || !stream) return QGN_ERR_ARG;
    *stream = net->stream;
    return QGN_OK;
}

const char* qgn_cnn_last_error(const qgn_cnn* net) { return net ? net->last_error.c_str() : "NULL network"; }

int qgn_cnn_destroy(qgn_cnn* net) {
    if (!net) return QGN_OK;
    if (net->stream) cudaStreamSynchronize(net->stream);
    for (void* p : net->owned) cudaFree(p);
    if (net->loss_host) cudaFreeHost(net->loss_host);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
    return QGN_OK;
}

}  // extern "C"
