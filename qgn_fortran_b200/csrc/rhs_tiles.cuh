// rhs_tiles.cuh -- per-tile bodies of the spectral right-hand side passes (see rhs_kernels.cu).
//
// Each body transforms one tile (a group of kx columns or of row pairs of one layer) whose
// coordinates the caller passes, so the same code serves the single-field launches
// (tile = blockIdx) and the ensemble launches, where a table maps a CTA to a member and tile.
// Bodies synchronise the whole CTA: every thread of the CTA must call them.
#pragma once
#include "qgn_internal.cuh"
#include "fft.cuh"

#include <cuda_bf16.h>

namespace qgn {

// ------------------------------------------------------------------------------------
// Tile shapes
// ------------------------------------------------------------------------------------
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }

// slot stride (in elements) of a padded transform such that slot*stride spreads the bank
// groups of one shared-memory wavefront: W = 128 bytes / element size elements per wavefront
// (8 for double2, 16 for float2); target is the stride's residue mod W.
__host__ __device__ constexpr int slot_stride(int N, int target, int elem_bytes = 16, int tp = 16) {
    return (N + N / tp) + ((target - ((N + N / tp) % (128 / elem_bytes))) + (128 / elem_bytes)) % (128 / elem_bytes);
}
// residue for `slots` lane-interleaved slots: consecutive threads hit different slots
__host__ __device__ constexpr int interleave_target(int slots, int elem_bytes) {
    return slots >= 128 / elem_bytes ? 1 : (128 / elem_bytes) / slots;
}

// minimum resident CTAs for __launch_bounds__ such that a thread keeps up to maxregs registers
__host__ __device__ constexpr int minb(int threads, int maxregs = 128) {
    return cmax(1, cmin(8, 65536 / (threads * maxregs)));
}
// register budget per thread: an FP32 transform holds half the register bytes of an FP64 one
template <class CT>
__host__ __device__ constexpr int regcap(int fp64 = 128, int fp32 = 64) { return sizeof(CT) == 16 ? fp64 : fp32; }

// y-pass tiles: TKX kx columns per CTA, lane-interleaved (slot = tid % TKX) so that one
// warp touches 8 consecutive y rows of TKX adjacent columns: 16*TKX-byte segments in the
// half-transformed row layout, 128-byte segments in the compact column layout.
// The last parameter of each config selects a tile-width variant: 0 is the tuned default of
// the single-field launches; a non-zero value is the CTA size in threads (per slot group for
// the x pass), the same for every transform length, which lets one launch cover fields of
// different sizes (ensembles).
// elements per thread of an x transform (fft.cuh): 32 for the 512- and 1024-point transforms of
// the single-field x pass (two radix passes instead of three, each transform in one warp: the
// FP32 x pass ran 9 % faster, the FP64 one cut the 1024^2 x 8 step by 2 % despite 168
// registers), 16 otherwise.  The y passes keep 16 in FP32: their CTAs interleave columns
// across warps, and at 32 elements they had half the threads per column and ran 1.3-1.7x
// slower on B200.
// A non-zero tile-variant code carries the CTA width in its low 16 bits and, above them, the
// elements per thread of its transforms (8, 16 or 32; 0 there means 16): the ensemble's
// autotuner searches both.
__host__ __device__ constexpr int tv_width(int tv) { return tv & 0xFFFF; }
__host__ __device__ constexpr int tv_radix(int tv) { return tv >> 16; }
__host__ __device__ constexpr int tv_make(int width, int radix) { return width | (radix << 16); }
template <class CT, int N, int TV>
__host__ __device__ constexpr int fft_tp() {
    return TV == 0 ? ((N == 512 || N == 1024) ? 32 : 16) : (tv_radix(TV) ? tv_radix(TV) : 16);
}
// elements per thread of a y transform: 8 for the FP64 512- and 1024-point columns of the
// single-field launches, 16 otherwise.  Half the registers per thread (64, two 512-thread CTAs
// per SM) doubles the resident warps of these latency-bound kernels at the price of a fourth
// radix pass at 1024 points: on B200 the 512^2 step ran 11 % and the 1024^2 step 1 % faster.
// QGN_Y_TP64 (build-time tuning knob, default 8) overrides the FP64 value.
#ifndef QGN_Y_TP64
#define QGN_Y_TP64 8
#endif
template <class CT, int N, int TV>
__host__ __device__ constexpr int fft_tp_y() {
    return TV == 0 ? ((sizeof(CT) == 16 && N >= 512) ? QGN_Y_TP64 : 16) : (tv_radix(TV) ? tv_radix(TV) : 16);
}
// Row pairs per CTA of the single-field x pass with one warp per transform (a build-time tuning
// knob).  One row pair (three warps, 96 threads, four CTAs per SM at 168 registers) couples only
// the three warps of a pair at the barrier between the inverse and forward transforms: the
// FP64 1024^2 x 8 x pass ran 7 % faster on B200 than with two row pairs per CTA.
#ifndef QGN_X_ROWPAIRS
#define QGN_X_ROWPAIRS 1
#endif

template <int NY, class CT = double2, int TV = 0>
struct YInvCfg {
    static constexpr int TP = fft_tp_y<CT, NY, TV>();
    static constexpr int G = FFTShape<NY, TP>::G;
    static constexpr int TKX = TV == 0 ? cmin(cmax(4, 128 / G), 16) : cmax(1, tv_width(TV) / G);
    static constexpr int THREADS = TKX * G;
    static constexpr int TS = slot_stride(NY, interleave_target(TKX, (int)sizeof(CT)), (int)sizeof(CT), TP);
    static constexpr int SMEM = TKX * TS * (int)sizeof(CT);
    // de-interleaved output rows (yinv_tile): odd rows start at HY.  A wavefront holds W
    // elements, LP = W/TKX consecutive rows of each slot; HY = NY/2 + LP/2 puts their even and
    // odd halves on distinct bank groups.
    static constexpr int LP = cmax(1, (128 / (int)sizeof(CT)) / TKX);
    static constexpr int HY = NY / 2 + LP / 2;
    static_assert(2 * HY <= TS, "de-interleaved rows fit the slot");
};

template <int NX, bool DRAG, class CT = double2, int TV = 0>
struct XCfg {
    static constexpr int TP = fft_tp<CT, NX, TV>();
    static constexpr int G = FFTShape<NX, TP>::G;
    static constexpr int RP = (TV == 0 && G == 32) ? QGN_X_ROWPAIRS : cmax(1, (TV == 0 ? 64 : tv_width(TV)) / G);   // row pairs per CTA
    static constexpr int SP = DRAG ? 4 : 3;             // slots per row pair
    static constexpr int THREADS = SP * RP * G;
    static constexpr int TS = slot_stride(NX, 2, (int)sizeof(CT), TP);
    static constexpr int SMEM = SP * RP * TS * (int)sizeof(CT);
};

template <int NY, bool DRAG, class CT = double2, int TV = 0>
struct YFwdCfg {
    static constexpr int TP = fft_tp_y<CT, NY, TV>();
    static constexpr int G = FFTShape<NY, TP>::G;
    // tid ^ TKX stays in the warp
    static constexpr int TKX = TV == 0 ? cmin(cmax(2, 64 / G), 16) : cmin(cmax(1, tv_width(TV) / (2 * G)), 16);
    static constexpr int SLOTS = 2 * TKX;
    static constexpr int THREADS = SLOTS * G;
    static constexpr int TS = slot_stride(NY, interleave_target(SLOTS, (int)sizeof(CT)), (int)sizeof(CT), TP);
    static constexpr int SMEM = SLOTS * TS * (int)sizeof(CT);
};

// ------------------------------------------------------------------------------------
// Modal inversion: GetPsi (QGN_Module.f90:315-341) at every kept mode, all layers per thread
// ------------------------------------------------------------------------------------
template <int NZ>
__device__ __forceinline__ void modal_invert(const double* __restrict__ proj, const double* __restrict__ back,
                                             const double* __restrict__ ev, double Htot, int nz, double k2,
                                             bool mean_mode, const double2* qv, double2* pv) {
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    const int n = NZ > 0 ? NZ : nz;
    double2 pm[NZC];
#pragma unroll
    for (int k = 0; k < NZC; ++k) {
        if (k < n) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int kk = 0; kk < NZC; ++kk) {
                if (kk < n) {
                    double c = proj[k * n + kk];
                    acc.x += c * qv[kk].x;
                    acc.y += c * qv[kk].y;
                }
            }
            const double rden = 1.0 / ((-k2 + ev[k]) * Htot);
            pm[k] = mean_mode ? make_double2(0.0, 0.0) : make_double2(acc.x * rden, acc.y * rden);
        }
    }
#pragma unroll
    for (int k = 0; k < NZC; ++k) {
        if (k < n) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int kk = 0; kk < NZC; ++kk) {
                if (kk < n) {
                    double c = back[k * n + kk];
                    acc.x += pm[kk].x * c;
                    acc.y += pm[kk].y * c;
                }
            }
            pv[k] = acc;
        }
    }
}

// ------------------------------------------------------------------------------------
// Packed row pairs.  The x pass transforms rows y1 = 2p and y2 = 2p+1 of one field as one
// complex signal f1 + i f2 whose Hermitian extension is
//     A[k]      = F1[k] + i F2[k]               (0 <= k < nkx; Re parts only at k = 0)
//     A[nx - k] = conj(F1[k]) + i conj(F2[k])   (1 <= k < nkx)
// The y passes store exactly these two arrays per row pair: [nz][ny/2][2][nkxp] with slot
// 0 = A[k] and slot 1 = A[nx-k] (same bytes as two plain rows).  The x pass reads one value
// per element, and its forward transform writes P[k] and P[nx-k] of every row the same
// way, which the forward y pass splits into (uq)^ = (P[k] + conj P[nx-k])/2 and
// (vq)^ = (P[k] - conj P[nx-k])/(2i).
// ------------------------------------------------------------------------------------
template <class CT>
__device__ __forceinline__ CT pack_lo(CT f1, CT f2, bool k0) {
    return k0 ? cmk<CT>(f1.x, f2.x) : cmk<CT>(f1.x - f2.y, f1.y + f2.x);
}
template <class CT>
__device__ __forceinline__ CT pack_hi(CT f1, CT f2) {
    return cmk<CT>(f1.x + f2.y, f2.x - f1.y);
}

// Layout of the forward x transforms P[k] (part 0) and P[nx-k] (part 1) of every row y: the x
// pass's output, the forward y pass's input.  QGN_P_TILED (default 1): tiles of two kx columns,
// [nz][nkxp/2][ny][2 parts][2 columns], so that the rows of one column pair are contiguous and a
// warp of the y-forward pass (8 rows x 2 columns x 2 parts) reads 512 contiguous bytes; the
// x pass's stores of one row scatter over the tiles instead (stores are not waited for).
// QGN_P_TILED 0: rows [nz][ny][2 parts][nkxp].  Both hold 2 nz ny nkxp elements.
#ifndef QGN_P_TILED
#define QGN_P_TILED 0
#endif
__host__ __device__ __forceinline__ size_t p_index(const Geom& g, int l, int y, int part, int k) {
#if QGN_P_TILED
    return ((size_t)(l * (g.nkxp >> 1) + (k >> 1)) * g.ny + y) * 4 + part * 2 + (k & 1);
#else
    return ((size_t)l * g.ny + y) * 2 * g.nkxp + (size_t)part * g.nkxp + k;
#endif
}

// ------------------------------------------------------------------------------------
// Bulk-copy staging (cp.async.bulk, the untiled TMA copy) of contiguous global spans into shared
// memory, completing on an mbarrier.  Source and destination are 16-byte aligned and the sizes
// multiples of 16 bytes; a CTA copies from this GPU's own memory only, with no multicast.
// QGN_Y_BULK (build-time knob, default 1): the FP64 y-inverse stages its compact columns this way.
// ------------------------------------------------------------------------------------
#ifndef QGN_Y_BULK
#define QGN_Y_BULK 1
#endif
constexpr long long kBulkWaitLimit = 1LL << 22;   // polls of the mbarrier before the wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
    // the initialised barrier becomes visible to the async (bulk-copy) proxy
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void bar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// bounded wait for phase `parity` of the barrier; false when it ran out
__device__ __forceinline__ bool bar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kBulkWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// ------------------------------------------------------------------------------------
// yinv: inverse y transforms of kept columns into packed row pairs.
// NF = 3: (q -> pq, -i ky psi -> pu, i kx psi -> pv);  NF = 2: (q -> pq, psi -> pu);  NF = 1: (f -> pq).
// The first radix pass reads the compact column (zeros in the dealiased band) straight from HBM,
// or, in FP64 with a wait-flag in the geometry (QGN_Y_BULK), from the column's own shared-memory
// slot, where one bulk copy per column has staged it; the transformed column stays in shared
// memory, where a packing loop pairs rows y and y+1 and writes the two packed arrays with
// TKX-wide coalesced stores.
// ------------------------------------------------------------------------------------
template <int NY, int NF, class CT, int TV = 0>
// f_begin/f_end: the fields this CTA transforms (all NF by default; one each when a launch
// spreads the fields over CTAs)
__device__ __forceinline__ void yinv_tile(const Geom g, int bx, int l, const CT* __restrict__ q,
                                          const CT* __restrict__ psi, CT* __restrict__ pq, CT* __restrict__ pv,
                                          CT* __restrict__ pu, const CT* __restrict__ twy, int f_begin = 0,
                                          int f_end = NF) {
    using C = YInvCfg<NY, CT, TV>;
    using RT = typename CTraits<CT>::R;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    CT* sm = reinterpret_cast<CT*>(sm_raw);
    const int tid = threadIdx.x;
    const int kx0 = bx * C::TKX;
    const int slot = tid % C::TKX, lane = tid / C::TKX;
    const int kx = kx0 + slot;
    const bool colok = kx < g.nkx;
    const size_t colbase = ((size_t)l * g.nkx + kx) * g.nky;
    const RT kxv = (RT)(g.dkx * kx);
    CT* xs = sm + slot * C::TS;
    NoIOT<CT> none;
#pragma unroll
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        if (f < f_begin || f >= f_end) continue;
        const CT* src = (f == 0) ? q : psi;
        CT* dst = (f == 0) ? pq : (f == 1 ? pu : pv);
        // the spectral derivative of field f at ky index j (QGN_Module.f90:223-224)
        auto deriv = [&](CT v, int j) -> CT {
            if (f == 1 && NF == 3) {   // u_hat = -i ky psi_hat
                const RT kyv = (RT)g.kyval(j);
                return cmk<CT>(kyv * v.y, -kyv * v.x);
            } else if (f == 2) {   // v_hat = i kx psi_hat
                return cmk<CT>(-kxv * v.y, kxv * v.x);
            }
            return v;
        };
        // the last pass writes rows y de-interleaved: even y at y/2, odd y at HY + y/2, so the
        // packing loop below reads consecutive offsets (free of bank-group conflicts; HY
        // offsets the odd half so that the last pass's stores are conflict-free too)
        auto omap = [](int y) { return (y & 1) * C::HY + (y >> 1); };
        bool staged = false;
        if constexpr (QGN_Y_BULK && sizeof(CT) == 16) {
            const int ncol = cmin(C::TKX, g.nkx - kx0);   // kept columns of this tile (>= 1)
            const size_t last = ((size_t)l * g.nkx + kx0 + ncol - 1) * g.nky + g.nky - 1;
            if (g.wait_err && in_bounds(g, last, g.csize())) {
                // one bulk copy per kept column into its slot (nky <= TS elements), thread 0 issues
                __shared__ __align__(8) uint64_t ybar;
                // this thread's earlier accesses to the slots are ordered before the copies' writes
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                if (tid == 0) bar_init(&ybar);
                __syncthreads();   // the barrier is initialised before anyone waits on it
                if (tid == 0) {
                    bar_expect_tx(&ybar, (uint32_t)(ncol * g.nky * (int)sizeof(CT)));
                    for (int c = 0; c < ncol; ++c)
                        bulk_g2s(sm + c * C::TS, src + ((size_t)l * g.nkx + kx0 + c) * g.nky,
                                 (uint32_t)(g.nky * (int)sizeof(CT)), &ybar);
                }
                if (!bar_wait_bounded(&ybar, 0)) {
                    atomicExch(g.wait_err, 1);            // the controller halts the run on it
                    bar_wait_bounded(&ybar, 0);           // once more for the copies still in flight
                }
                const CT* stage = xs;
                auto lds = [&](int j) -> CT {
                    const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
                    if (!colok || !kept) return cmk<CT>(0.0, 0.0);
                    return deriv(stage[j < g.kylo ? j : j - g.kyshift], j);
                };
                // SRC_FN_SMEM: every thread has read the staged column before the first pass
                // overwrites the slot (block-wide barrier inside the pass)
                fft_fused<NY, +1, SRC_FN_SMEM, DST_SMEM_MAP, C::TP, false, C::TKX>(xs, lane, true, twy, lds, omap);
                if (tid == 0) bar_inval(&ybar);           // every waiter has passed the barrier
                staged = true;
            }
        }
        if (!staged) {
            auto ld = [&](int j) -> CT {
                const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
                if (!colok || !kept) return cmk<CT>(0.0, 0.0);
                const size_t ci = colbase + (j < g.kylo ? j : j - g.kyshift);
                if (!in_bounds(g, ci, g.csize())) return cmk<CT>(0.0, 0.0);
                return deriv(src[ci], j);
            };
            fft_fused<NY, +1, SRC_FN, DST_SMEM_MAP, C::TP, false, C::TKX>(xs, lane, true, twy, ld, omap);
        }
        // pack rows (2p, 2p+1): e -> (pair p, column c); both arrays of a pair row per thread
        CT* dl = dst + (size_t)l * (NY / 2) * 2 * g.nkxp;
        for (int e = tid; e < (NY / 2) * C::TKX; e += C::THREADS) {
            const int p = e / C::TKX, c = e % C::TKX;
            const int k = kx0 + c;
            if (k >= g.nkxp) continue;
            const CT f1 = sm[c * C::TS + p], f2 = sm[c * C::TS + C::HY + p];
            const bool ok = k < g.nkx;
            const size_t ro = ((size_t)l * (NY / 2) + p) * 2 * g.nkxp;   // row pair p of layer l
            if (!in_bounds(g, ro + g.nkxp + k, g.hsize())) continue;
            CT* row = dl + (size_t)p * 2 * g.nkxp;
            // Re parts at kx = 0 and at the kx Nyquist column (kept only in the full-spectrum geometry)
            row[k] = ok ? pack_lo(f1, f2, k == 0 || 2 * k == g.nx) : cmk<CT>(0.0, 0.0);
            row[g.nkxp + k] = (ok && k > 0) ? pack_hi(f1, f2) : cmk<CT>(0.0, 0.0);
        }
        if (f + 1 < f_end) __syncthreads();   // the next field's first pass reuses the slots
    }
}

// ------------------------------------------------------------------------------------
// xpass: x transforms of row pairs.  c2r of the packed q1 + i q2, u1 + i u2, v1 + i v2
// (pairing two rows of one field keeps roundoff relative to that field; q and u differ by
// ~1e4 in these units), physical products formed inside the first pass of the forward
// transforms, r2c of p = uq + i vq per row, whose last pass writes P[k] and P[nx-k] for the
// kept kx straight to HBM.
// ------------------------------------------------------------------------------------
template <int NX, bool DRAG, class CT, int TV = 0>
__device__ __forceinline__ void xpass_tile(const Geom g, int bx, int l, const CT* __restrict__ pq,
                                           const CT* __restrict__ pv, const CT* __restrict__ pu,
                                           CT* __restrict__ pp, CT* __restrict__ pd, const CT* __restrict__ twx) {
    using C = XCfg<NX, DRAG, CT, TV>;
    using RT = typename CTraits<CT>::R;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    CT* sm = reinterpret_cast<CT*>(sm_raw);
    const int tid = threadIdx.x;
    const int npairs = g.ny / 2;
    const int nkx = g.nkx;
    const int slot = tid / C::G, lane = tid % C::G;
    const int r_of = slot / C::SP, s_of = slot % C::SP;
    const int rp = bx * C::RP + r_of;
    const bool pair_ok = rp < npairs;
    CT* base = sm + (r_of * C::SP) * C::TS;
    CT* xs = sm + slot * C::TS;

    // ---- inverse: slot 0 = q1+iq2, 1 = u1+iu2, 2 = v1+iv2
    const size_t fo = ((size_t)l * npairs + rp) * 2 * g.nkxp;   // row pair rp of layer l
    const CT* F = (s_of == 0 ? pq : (s_of == 1 ? pu : pv)) + fo;
    auto ld_inv = [&](int k) -> CT {
        if (k < nkx) return in_bounds(g, fo + k, g.hsize()) ? F[k] : cmk<CT>(0.0, 0.0);
        if (k > NX - nkx) return in_bounds(g, fo + g.nkxp + (NX - k), g.hsize()) ? F[g.nkxp + (NX - k)] : cmk<CT>(0.0, 0.0);
        return cmk<CT>(0.0, 0.0);
    };
    // the last pass stores the two rows apart, as real planes: row 2p at RT offset 0 of the
    // slot, row 2p+1 at RT offset TS, so that each forward transform below reads only its
    // own row (half the bytes of reading the packed complex values)
    RT* plane = reinterpret_cast<RT*>(xs);
    auto st_inv = [&](int x, CT v) {
        plane[x] = v.x;
        plane[C::TS + x] = v.y;
    };
    fft_fused<NX, +1, SRC_FN, DST_SMEM_STORE, C::TP, (C::G <= 32)>(xs, lane, pair_ok && s_of < 3, twx, ld_inv,
                                                                     st_inv);

    // ---- forward: slot 0 = u1 q1 + i v1 q1, 1 = u2 q2 + i v2 q2 (grid/(nx*ny) scaling as in
    //      QGN_Module.f90:229-235); with drag 2 = |u1|u1 + i|u1|v1, 3 = |u2|u2 + i|u2|v2
    const RT sc = (RT)g.inv_nxny;
    const RT sc2 = sc * sc;   // nx, ny are powers of two: u (q sc^2) == (u sc)(q sc) exactly
    // this slot's row in the planes of the q, u, v slots (RT offsets 0, 2 TS, 4 TS)
    const RT* rows = reinterpret_cast<const RT*>(base) + ((s_of & 1) ? C::TS : 0);
    auto ld_fwd = [&](int x) -> CT {
        if (s_of < 2) {
            const RT qs = rows[x] * sc2;
            return cmk<CT>(rows[2 * C::TS + x] * qs, rows[4 * C::TS + x] * qs);
        }
        const RT uv = rows[2 * C::TS + x] * sc;
        const RT vv = rows[4 * C::TS + x] * sc;
        const RT m = sqrt(uv * uv + vv * vv);   // URMS, QGN_Module.f90:285
        return cmk<CT>(m * uv, m * vv);
    };
    const int y = 2 * rp + (s_of & 1);
    const int ol = (s_of < 2) ? l : 0;                                              // pd holds one layer
    const size_t olen = (s_of < 2) ? 2 * g.hsize() : (size_t)g.ny * 2 * g.nkxp;   // pp, or pd
    CT* out = (s_of < 2) ? pp : pd;
    auto st_fwd = [&](int k, CT v) {
        if (k < nkx) {
            const size_t i = p_index(g, ol, y, 0, k);
            if (in_bounds(g, i, olen)) out[i] = v;
        } else if (k > NX - nkx) {
            const size_t i = p_index(g, ol, y, 1, NX - k);
            if (in_bounds(g, i, olen)) out[i] = v;
        }
    };
#if QGN_P_TILED
    // Tiled layout: the last radix pass leaves the kept outputs in the transform's own slot
    // (P[k] at k, P[nx-k] at nkxp + k; the dealiased band's outputs on the slot's last element),
    // and the whole CTA then writes each kx column pair's values of its rows as one contiguous
    // run: with one row pair per CTA, rows 2p and 2p+1 of a tile are adjacent, 8 values = 128 B.
    if (2 * g.nkxp < C::TS - 1) {   // the kept outputs fit below the spare element (uniform)
        auto omap = [&](int k) -> int {
            if (k < nkx) return k;
            if (k > NX - nkx) return g.nkxp + (NX - k);
            return C::TS - 1;
        };
        fft_fused<NX, -1, SRC_FN_SMEM, DST_SMEM_MAP, C::TP, (C::G <= 32)>(xs, lane, pair_ok && s_of < (DRAG ? 4 : 2),
                                                                             twx, ld_fwd, omap);
        // fft_fused ended with a block-wide barrier: every slot holds its row's outputs
        const int T = g.nkxp >> 1;
        for (int dr = 0; dr < (DRAG ? 2 : 1); ++dr) {   // dr 0: uq + i vq into pp; 1: drag fields into pd
            CT* o = dr == 0 ? pp : pd;
            const int ol2 = dr == 0 ? l : 0;
            const size_t olen2 = dr == 0 ? 2 * g.hsize() : (size_t)g.ny * 2 * g.nkxp;
            for (int e = tid; e < C::RP * T * 8; e += C::THREADS) {
                const int r = e / (T * 8), rem = e % (T * 8);
                const int t = rem >> 3, w = rem & 7;
                const int rr = w >> 2, part = (w >> 1) & 1, k = 2 * t + (w & 1);
                const int rpp = bx * C::RP + r;
                if (rpp >= npairs || k >= nkx || (part == 1 && k == 0)) continue;
                const CT* src = sm + (r * C::SP + 2 * dr + rr) * C::TS;
                const size_t i = p_index(g, ol2, 2 * rpp + rr, part, k);
                if (in_bounds(g, i, olen2)) o[i] = src[part * g.nkxp + k];
            }
        }
        return;
    }
#endif
    fft_fused<NX, -1, SRC_FN_SMEM, DST_FN, C::TP, (C::G <= 32)>(xs, lane, pair_ok && s_of < (DRAG ? 4 : 2), twx, ld_fwd,
                                                                   st_fwd);
}

// ------------------------------------------------------------------------------------
// yfwd: forward y transforms of uq, vq columns and assembly of the right-hand side.
// Slots are lane-interleaved: slot = tid % (2 TKX), slot = field*TKX + column.  The first
// radix pass reads the half-transformed rows straight from HBM.
// ------------------------------------------------------------------------------------
// split of the packed forward x transform of row y at kx: fld 0 -> (uq)^, fld 1 -> (vq)^
__device__ __forceinline__ double2 unpack_p(const double2* __restrict__ P, const Geom& g, int l, int y, int kx,
                                            int fld) {
    const double2 X = P[p_index(g, l, y, 0, kx)];
    const double2 Y = kx == 0 ? cconj(X) : cconj(P[p_index(g, l, y, 1, kx)]);
    return fld == 0 ? make_double2(0.5 * (X.x + Y.x), 0.5 * (X.y + Y.y))
                    : make_double2(0.5 * (X.y - Y.y), -0.5 * (X.x - Y.x));
}

// the thread of field fld loads part fld (P[k] for fld 0, P[nx-k] for fld 1) at index i and
// swaps it with its partner's, so each value is read once
template <class CT>
__device__ __forceinline__ CT unpack_pair(const CT* __restrict__ P, size_t i, int kx, int fld, bool ok, int partner) {
    CT mine = cmk<CT>(0.0, 0.0);
    if (ok && (fld == 0 || kx > 0)) mine = P[i];
    CT other;
    other.x = __shfl_xor_sync(0xffffffffu, mine.x, partner);
    other.y = __shfl_xor_sync(0xffffffffu, mine.y, partner);
    const CT X = fld == 0 ? mine : other;
    const CT Y = kx == 0 ? cconj(X) : cconj(fld == 0 ? other : mine);
    return fld == 0 ? cmk<CT>((typename CTraits<CT>::R)0.5 * (X.x + Y.x), (typename CTraits<CT>::R)0.5 * (X.y + Y.y))
                    : cmk<CT>((typename CTraits<CT>::R)0.5 * (X.y - Y.y), -(typename CTraits<CT>::R)0.5 * (X.x - Y.x));
}

template <int NY, bool DRAG, class CT, int TV = 0>
__device__ __forceinline__ void yfwd_tile(const Geom g, int bx, int l, const LayerConst* __restrict__ lc,
                                          const CT* __restrict__ q, const CT* __restrict__ psi,
                                          const CT* __restrict__ pp, const CT* __restrict__ pd,
                                          CT* __restrict__ out, const CT* __restrict__ twy,
                                          const CT* __restrict__ extra = nullptr) {
    using C = YFwdCfg<NY, DRAG, CT, TV>;
    using RT = typename CTraits<CT>::R;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    CT* sm = reinterpret_cast<CT*>(sm_raw);
    const int tid = threadIdx.x;
    const int kx0 = bx * C::TKX;
    const int slot = tid % C::SLOTS, lane = tid / C::SLOTS;
    const int fld = slot / C::TKX, c = slot % C::TKX;
    const bool colok = kx0 + c < g.nkx;
    const int nky = g.nky;
    const size_t colbase = (size_t)l * g.nkx;
    const bool bottom = (l == g.nz - 1);
    CT* xs = sm + slot * C::TS;
    // the last radix pass writes the transformed column unpadded (row y at y): the assembly
    // loops below read 8-16 consecutive rows per wavefront, which a pad element every TP rows
    // would split across one bank group twice
    auto omap = [](int y) { return y; };

    if (DRAG) {
        // drag_hat = i ky (|u|u)^ - i kx (|u|v)^ on the bottom layer (QGN_Module.f90:284-292)
        auto ldd = [&](int y) -> CT {
            const size_t i = p_index(g, 0, y, fld, kx0 + c);
            const bool ok = colok && in_bounds(g, i, (size_t)g.ny * 2 * g.nkxp);
            return unpack_pair(pd, i, kx0 + c, fld, ok, C::TKX);
        };
        fft_fused<NY, -1, SRC_FN, DST_SMEM_MAP, C::TP, false, C::SLOTS>(xs, lane, true, twy, ldd, omap);
        const RT dc = (RT)lc->dragc;
        for (int e = tid; e < C::TKX * nky; e += C::THREADS) {
            const int cc = e / nky, m = e % nky;
            const int kx = kx0 + cc;
            if (kx >= g.nkx) continue;
            const int j = g.jfull(m);
            const RT kxv = (RT)(g.dkx * kx), kyv = (RT)g.kyval(j);
            const CT fu = sm[cc * C::TS + j], fv = sm[(C::TKX + cc) * C::TS + j];
            CT d = cmk<CT>(-kyv * fu.y, kyv * fu.x);        // i ky (|u|u)^
            d = cmk<CT>(d.x + kxv * fv.y, d.y - kxv * fv.x);      // - i kx (|u|v)^
            if (in_bounds(g, (colbase + kx) * nky + m, g.csize())) out[(colbase + kx) * nky + m] = cmk<CT>(dc * d.x, dc * d.y);
        }
        __syncthreads();
    }

    // the (uq)^ and (vq)^ slots of one column load P[k] and P[nx-k] respectively and swap
    // them with a shuffle (partner tid ^ TKX, same warp), so each value is read once
    auto ld = [&](int y) -> CT {
        const size_t i = p_index(g, l, y, fld, kx0 + c);
        const bool ok = colok && in_bounds(g, i, 2 * g.hsize());
        return unpack_pair(pp, i, kx0 + c, fld, ok, C::TKX);
    };
    fft_fused<NY, -1, SRC_FN, DST_SMEM_MAP, C::TP, false, C::SLOTS>(xs, lane, true, twy, ld, omap);

    const RT ub = (RT)lc->uBar[l], bq = (RT)lc->betaq[l];
    const RT ek = (RT)lc->ekman;
    const bool expl = lc->explicit_diss != 0;
    for (int e = tid; e < C::TKX * nky; e += C::THREADS) {
        const int cc = e / nky, m = e % nky;
        const int kx = kx0 + cc;
        if (kx >= g.nkx) continue;
        const int j = g.jfull(m);
        const RT kxv = (RT)(g.dkx * kx), kyv = (RT)g.kyval(j);
        const size_t idx = (colbase + kx) * nky + m;
        if (!in_bounds(g, idx, g.csize())) continue;
        const CT fuq = sm[cc * C::TS + j], fvq = sm[(C::TKX + cc) * C::TS + j];
        const CT qv = q[idx], pv = psi[idx];
        // jaco_hat = i kx uq_hat + i ky vq_hat  (QGN_Module.f90:244-247)
        const CT jac = cmk<CT>(-kxv * fuq.y - kyv * fvq.y, kxv * fuq.x + kyv * fvq.x);
        CT r = cmk<CT>(-jac.x, -jac.y);
        // - uBar i kx q_hat - (beta+qyBar) v_hat   (QGN_Module.f90:270-273)
        const RT uk = ub * kxv;
        const CT vh = cmk<CT>(-kxv * pv.y, kxv * pv.x);
        r = cmk<CT>(r.x + uk * qv.y, r.y - uk * qv.x);
        r = cmk<CT>(r.x - bq * vh.x, r.y - bq * vh.y);
        const RT k2 = kxv * kxv + kyv * kyv;
        if (expl) {   // QGN_Module.f90:275-280
            const RT k4 = k2 * k2, k8 = k4 * k4;
            const RT dcoef = (RT)lc->A2 * k2 + (RT)lc->A8 * k8;
            r = cmk<CT>(r.x - dcoef * qv.x, r.y - dcoef * qv.y);
        }
        if (bottom) {   // Ekman, QGN_Module.f90:282
            const RT ekk = ek * k2;
            r = cmk<CT>(r.x + ekk * pv.x, r.y + ekk * pv.y);
            if (DRAG) {
                const CT d = out[idx];
                r = cmk<CT>(r.x + d.x, r.y + d.y);
            }
        }
        if (extra) {   // an extra tendency on the kept modes (the learned closure's)
            const CT x = extra[idx];
            r = cmk<CT>(r.x + x.x, r.y + x.y);
        }
        if (kx == 0 && m == 0) r = cmk<CT>(0.0, 0.0);
        out[idx] = r;
    }
}

// ------------------------------------------------------------------------------------
// Single-field inverse 2-D transform: x c2r of row pairs with an epilogue
//   EPI 0: max |grid| (unnormalised) into sc->maxbits
//   EPI 1: physical field grid/(nx*ny) into out[nz][ny][nx]
// ------------------------------------------------------------------------------------
template <int NX, int TV = 0, class CT = double2>
struct X1Cfg {
    static constexpr int TP = 16;
    static constexpr int G = FFTShape<NX, TP>::G;
    static constexpr int RP = cmax(1, (TV == 0 ? 128 : TV) / G);
    static constexpr int THREADS = RP * G;
    static constexpr int TS = slot_stride(NX, 2, (int)sizeof(CT));
    static constexpr int SMEM = RP * TS * (int)sizeof(CT);
};

// CT = float2 (the mixed mode's error norm) supports EPI 0 only
template <int NX, int EPI, int TV = 0, class CT = double2>
// EPI 2 (the learned closure's input): channel chan of the NHWC BF16 tensor xout with
// cin_p channels per pixel, grid/(nx*ny) * scale[chan]
__device__ __forceinline__ void xinv1_tile(const Geom g, int bx, int l, const CT* __restrict__ hq,
                                           DevScalars* __restrict__ sc, double* __restrict__ outp,
                                           const CT* __restrict__ twx, const float* __restrict__ scale = nullptr,
                                           __nv_bfloat16* __restrict__ xout = nullptr, int cin_p = 0,
                                           int chan = 0) {
    static_assert(EPI == 0 || sizeof(CT) == 16, "FP32 rows: max only");
    using C = X1Cfg<NX, TV, CT>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    CT* sm = reinterpret_cast<CT*>(sm_raw);
    __shared__ double smax[32];
    const int tid = threadIdx.x;
    const int npairs = g.ny / 2;
    const int nkx = g.nkx;
    const int slot = tid / C::G, lane = tid % C::G;
    const int rp = bx * C::RP + slot;
    const bool ok = rp < npairs;
    const CT* F = hq + ((size_t)l * npairs + rp) * 2 * g.nkxp;   // packed row pair
    auto ld = [&](int k) -> CT {
        if (k < nkx) return F[k];
        if (k > NX - nkx) return F[g.nkxp + (NX - k)];
        return cmk<CT>(0.0, 0.0);
    };
    double mx = 0.0;
    const size_t prow = ((size_t)l * g.ny + 2 * rp) * NX;
    auto st = [&](int x, CT a) {
        if constexpr (EPI == 0) {
            // NaN is kept as the largest value
            const double m1 = fabs((double)a.x), m2 = fabs((double)a.y);
            if (!(m1 == m1) || !(m2 == m2)) mx = __longlong_as_double(0x7ff8000000000000LL);
            else if (mx == mx) mx = fmax(mx, fmax(m1, m2));
        } else if constexpr (EPI == 1) {
            outp[prow + x] = a.x * g.inv_nxny;
            outp[prow + NX + x] = a.y * g.inv_nxny;
        } else {
            const size_t pix = (size_t)(2 * rp) * NX + x;
            const float sf = scale[chan];
            xout[pix * cin_p + chan] = __float2bfloat16_rn((float)(a.x * g.inv_nxny) * sf);
            xout[(pix + NX) * cin_p + chan] = __float2bfloat16_rn((float)(a.y * g.inv_nxny) * sf);
        }
    };
    fft_fused<NX, +1, SRC_FN, DST_FN, C::TP, (C::G <= 32)>(sm + slot * C::TS, lane, ok, twx, ld, st);
    if (EPI == 0) {
        // block max of non-negative doubles (NaN as the largest bit pattern)
        unsigned long long bits = (unsigned long long)__double_as_longlong(mx);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long ob = __shfl_xor_sync(0xffffffffu, bits, o);
            bits = ob > bits ? ob : bits;
        }
        if ((tid & 31) == 0) smax[tid >> 5] = __longlong_as_double((long long)bits);
        __syncthreads();
        if (tid < 32) {
            unsigned long long b2 = (tid < (C::THREADS + 31) / 32)
                                        ? (unsigned long long)__double_as_longlong(smax[tid]) : 0ULL;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                unsigned long long ob = __shfl_xor_sync(0xffffffffu, b2, o);
                b2 = ob > b2 ? ob : b2;
            }
            if (tid == 0) atomicMax(&sc->maxbits, b2);
        }
    }
}

}  // namespace qgn
