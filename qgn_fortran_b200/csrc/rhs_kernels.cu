// rhs_kernels.cu -- the spectral right-hand side of QGN on sm_100a (FP64, and FP32 for the mixed mode).
//
// One GetRHS (QGN_Module.f90:258-296) = GetPsi + Jacobian + linear terms + drag +
// DeAlias is evaluated as three streaming passes over HBM plus the modal inversion
// that the stage kernels fuse into their epilogue:
//
//   yinv  (per layer, per tile of kx columns)  compact q, psi -> y-inverse of q, u = -i ky psi,
//         v = i kx psi, written as packed row pairs [nz][ny/2][2][nkxp]     (3 inverse y FFTs)
//   xpass (per layer, per pair of rows y)       c2r of q1+iq2, u1+iu2, v1+iv2, products uq, vq
//         (and |u|u, |u|v in the bottom layer), r2c of uq+ivq per row; keeps kx < nx/3
//   yfwd  (per layer, per tile of kx columns)  forward y FFT of uq, vq (and drag fields), then
//         J = i kx (uq)^ + i ky (vq)^ and RHS = -J - U i kx q - (beta+Qy) v + Ekman + drag,
//         written for the kept modes only (DeAlias is the storage format).
//
// The dealiased band (kx >= nx/3, ny/3 <= j <= 2(ny/3)) is never stored: inverse
// transforms see zeros there and forward transforms do not write it.
#include "qgn_internal.cuh"
#include "fft.cuh"
#include "prof.cuh"
#include "rhs_tiles.cuh"

#include <cuda_bf16.h>

#include <mutex>
#include <type_traits>
#include <unordered_set>

namespace qgn {

template <int NZ>
__global__ void __launch_bounds__(256, 2) k_modal(Geom g, const __grid_constant__ ModalArg<NZ> ma,
                                               const double2* __restrict__ q, double2* __restrict__ psi) {
    QGN_PDL_ENTRY();
    QGN_MODAL_SHARED(NZ);
    const int nz = g.nz;
    const ModalView mv = modal_view<NZ>(ma, s_proj, s_back, s_ev, nz);
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int kx = (int)(p / g.nky), m = (int)(p % g.nky);
    const double kxv = g.dkx * kx, kyv = g.kyval(g.jfull(m));
    const double k2 = kxv * kxv + kyv * kyv;
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    double2 qv[NZC], pv[NZC];
#pragma unroll
    for (int k = 0; k < NZC; ++k)
        if (k < nz) qv[k] = in_bounds(g, (size_t)k * P + p, g.csize()) ? q[(size_t)k * P + p] : make_double2(0.0, 0.0);
    modal_invert<NZ>(mv.proj, mv.back, mv.ev, mv.Htot, nz, k2, p == 0, qv, pv);
#pragma unroll
    for (int k = 0; k < NZC; ++k)
        if (k < nz && in_bounds(g, (size_t)k * P + p, g.csize())) psi[(size_t)k * P + p] = pv[k];
}

// ------------------------------------------------------------------------------------
// Single-field launches of the tile bodies (rhs_tiles.cuh): one CTA per tile, tile = blockIdx
// ------------------------------------------------------------------------------------
// TV selects a tile width (0: the default; see the configs in rhs_tiles.cuh)
// with more than one field, the narrow variants and the 512- and 1024-point launches spread the
// fields over CTAs (blockIdx.z): 688 CTAs of one FP64 1024^2 x 8 launch filled 2.3 waves of the
// 296 resident slots, three times as many fill 7 (the 1024^2 x 8 step ran 3 % faster, 512^2 x 4
// 8 %); in FP32 the same spread cut the mixed-precision 1024^2 x 8 step by 4 %
template <int NY, class CT, int TV>
constexpr bool yinv_spread() { return TV != 0 || NY >= 512; }

template <int NY, int NF, class CT, int TV = 0>
__global__ void __launch_bounds__(YInvCfg<NY, CT, TV>::THREADS, minb(YInvCfg<NY, CT, TV>::THREADS, YInvCfg<NY, CT, TV>::TP == 8 ? 64 : regcap<CT>()))
    k_yinv(Geom g, const CT* __restrict__ q, const CT* __restrict__ psi, CT* __restrict__ pq,
           CT* __restrict__ pv, CT* __restrict__ pu, const CT* __restrict__ twy) {
    QGN_PDL_ENTRY();
    if constexpr (yinv_spread<NY, CT, TV>() && NF > 1)
        yinv_tile<NY, NF, CT, TV>(g, blockIdx.x, blockIdx.y, q, psi, pq, pv, pu, twy, blockIdx.z, blockIdx.z + 1);
    else
        yinv_tile<NY, NF, CT, TV>(g, blockIdx.x, blockIdx.y, q, psi, pq, pv, pu, twy);
}

template <int NX, bool DRAG, class CT, int TV = 0>
__global__ void __launch_bounds__(XCfg<NX, DRAG, CT, TV>::THREADS,
                                  minb(XCfg<NX, DRAG, CT, TV>::THREADS,
                                       XCfg<NX, DRAG, CT, TV>::TP == 32 ? (sizeof(CT) == 16 ? 168 : 112) : regcap<CT>(NX >= 1024 ? 112 : 128, 80)))
    k_xpass(Geom g, int layer0, const CT* __restrict__ pq, const CT* __restrict__ pv,
            const CT* __restrict__ pu, CT* __restrict__ pp, CT* __restrict__ pd,
            const CT* __restrict__ twx) {
    QGN_PDL_ENTRY();
    xpass_tile<NX, DRAG, CT, TV>(g, blockIdx.x, layer0 + blockIdx.y, pq, pv, pu, pp, pd, twx);
}

template <int NY, bool DRAG, class CT, int TV = 0>
__global__ void __launch_bounds__(YFwdCfg<NY, DRAG, CT, TV>::THREADS,
                                  minb(YFwdCfg<NY, DRAG, CT, TV>::THREADS, YFwdCfg<NY, DRAG, CT, TV>::TP == 8 ? 64 : regcap<CT>()))
    k_yfwd(Geom g, int layer0, const LayerConst* __restrict__ lc, const CT* __restrict__ q,
           const CT* __restrict__ psi, const CT* __restrict__ pp, const CT* __restrict__ pd,
           CT* __restrict__ out, const CT* __restrict__ twy, const CT* __restrict__ extra) {
    QGN_PDL_ENTRY();
    yfwd_tile<NY, DRAG, CT, TV>(g, blockIdx.x, layer0 + blockIdx.y, lc, q, psi, pp, pd, out, twy, extra);
}

template <int NX, int EPI, int TV = 0, class CT = double2>
__global__ void __launch_bounds__(X1Cfg<NX, TV, CT>::THREADS, minb(X1Cfg<NX, TV, CT>::THREADS))
    k_xinv1(Geom g, const CT* __restrict__ hq, DevScalars* __restrict__ sc, double* __restrict__ outp,
            const CT* __restrict__ twx) {
    QGN_PDL_ENTRY();
    xinv1_tile<NX, EPI, TV, CT>(g, blockIdx.x, blockIdx.y, hq, sc, outp, twx);
}

// Small grids launch few CTAs with the default tiles (at 128^2 x 4: 12 for the y-inverse),
// so each CTA's serial transform work sets the kernel's duration.  For transform lengths
// 64..256 a narrow variant (fewer columns or rows per CTA) is used when the default gives
// fewer than two CTAs per SM and the narrow one gives more.  Tile width changes no arithmetic.
constexpr int kNarrowY = 32, kNarrowX = 16, kNarrowX1 = 32;
template <int N>
constexpr bool has_narrow() { return N >= 64 && N <= 256; }
static bool narrow_better(long long ctas_default, long long ctas_narrow) {
    return ctas_default < 2 * 148 && ctas_narrow > ctas_default;
}

// ------------------------------------------------------------------------------------
// Forward 2-D transform of a physical field (DftiComputeForward + DeAlias of Initialize,
// QGN_Module.f90:179-183): r2c of row pairs packed as r1 + i r2, then forward y columns
// keeping the dealiased modes only.
// ------------------------------------------------------------------------------------
// SRC 0: physical field phys[nz][ny][nx]; SRC 1: channel l of the planar FP32 tensor
// y[channel][ny*nx] divided by osc[l] (the learned closure's output)
template <int NX, int SRC = 0, int TV = 0>
__global__ void __launch_bounds__(X1Cfg<NX, TV>::THREADS, minb(X1Cfg<NX, TV>::THREADS))
    k_xfwd1(Geom g, const double* __restrict__ phys, double2* __restrict__ hq, const double2* __restrict__ twx,
            const float* __restrict__ y = nullptr, int cout_p = 0, const float* __restrict__ osc = nullptr) {
    QGN_PDL_ENTRY();
    using C = X1Cfg<NX, TV>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = reinterpret_cast<double2*>(sm_raw);
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int npairs = g.ny / 2;
    const int slot = tid / C::G, lane = tid % C::G;
    const int rp = blockIdx.x * C::RP + slot;
    const size_t prow = ((size_t)l * g.ny + 2 * rp) * NX;
    const double rsc = SRC == 0 ? 1.0 : 1.0 / (double)osc[l];   // one division per thread
    auto ld = [&](int x) -> double2 {
        if constexpr (SRC == 0) return make_double2(phys[prow + x], phys[prow + NX + x]);
        const size_t pix = (size_t)(2 * rp) * NX + x;
        const float* yl = y + (size_t)l * g.ny * NX;
        return make_double2((double)yl[pix] * rsc, (double)yl[pix + NX] * rsc);
    };
    NoIO none;
    fft_fused<NX, -1, SRC_FN, DST_SMEM, C::TP, (C::G <= 32)>(sm + slot * C::TS, lane, rp < npairs, twx, ld, none);
    const int nkx = g.nkx;
    for (int e = tid; e < C::RP * nkx; e += C::THREADS) {
        const int r = e / nkx, k = e % nkx;
        const int rq = blockIdx.x * C::RP + r;
        if (rq >= npairs) continue;
        const double2 X = sm[r * C::TS + fpad<C::TP>(k)];
        const double2 Y = cconj(sm[r * C::TS + fpad<C::TP>((NX - k) & (NX - 1))]);
        const size_t row = ((size_t)l * g.ny + 2 * rq) * g.nkxp + k;
        hq[row] = make_double2(0.5 * (X.x + Y.x), 0.5 * (X.y + Y.y));
        hq[row + g.nkxp] = make_double2(0.5 * (X.y - Y.y), -0.5 * (X.x - Y.x));
    }
}

template <int NY>
__global__ void __launch_bounds__(YInvCfg<NY>::THREADS, minb(YInvCfg<NY>::THREADS))
    k_yfwd1(Geom g, const double2* __restrict__ hq, double2* __restrict__ out, const double2* __restrict__ twy) {
    QGN_PDL_ENTRY();
    using C = YInvCfg<NY>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = reinterpret_cast<double2*>(sm_raw);
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int slot = tid % C::TKX, lane = tid / C::TKX;
    const int kx = blockIdx.x * C::TKX + slot;
    const bool colok = kx < g.nkx;
    const size_t colbase = ((size_t)l * g.nkx + kx) * g.nky;
    auto ld = [&](int y) -> double2 {
        return colok ? hq[((size_t)l * NY + y) * g.nkxp + kx] : make_double2(0.0, 0.0);
    };
    auto st = [&](int j, double2 v) {
        const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
        if (!colok || !kept) return;
        const int m = j < g.kylo ? j : j - g.kyshift;
        if (kx == 0 && m == 0) v = make_double2(0.0, 0.0);
        out[colbase + m] = v;
    };
    fft_fused<NY, -1, SRC_FN, DST_FN, C::TP>(sm + slot * C::TS, lane, true, twy, ld, st);
}

// ------------------------------------------------------------------------------------
// Dispatch
// ------------------------------------------------------------------------------------
template <class F>
static cudaError_t dispatch_n(int n, F&& f) {
    switch (n) {
        case 16: return f(std::integral_constant<int, 16>{});
        case 32: return f(std::integral_constant<int, 32>{});
        case 64: return f(std::integral_constant<int, 64>{});
        case 128: return f(std::integral_constant<int, 128>{});
        case 256: return f(std::integral_constant<int, 256>{});
        case 512: return f(std::integral_constant<int, 512>{});
        case 1024: return f(std::integral_constant<int, 1024>{});
        case 2048: return f(std::integral_constant<int, 2048>{});
        default: return cudaErrorInvalidValue;
    }
}

// dynamic shared memory above 48 KB, opted into once per (device, kernel) (launch.cuh)
template <class K>
static cudaError_t set_smem(K kernel, int bytes) {
    return smem_opt_in(kernel, bytes);
}

cudaError_t launch_modal(const Geom& g, const Buffers& b, const double2* q, double2* psi, cudaStream_t s) {
    const size_t P = (size_t)g.nkx * g.nky;
    dim3 grid((unsigned)((P + 255) / 256));
    const double nb = 2.0 * 16.0 * (double)g.csize();
    switch (b.mc_h ? g.nz : 0) {
        case 2: QGN_LAUNCH(KID_MODAL, nb, s, ::qgn::launch(k_modal<2>, grid, 256, 0, s, g, modal_arg<2>(b), q, psi)); break;
        case 4: QGN_LAUNCH(KID_MODAL, nb, s, ::qgn::launch(k_modal<4>, grid, 256, 0, s, g, modal_arg<4>(b), q, psi)); break;
        case 8: QGN_LAUNCH(KID_MODAL, nb, s, ::qgn::launch(k_modal<8>, grid, 256, 0, s, g, modal_arg<8>(b), q, psi)); break;
        case 16: QGN_LAUNCH(KID_MODAL, nb, s, ::qgn::launch(k_modal<16>, grid, 256, 0, s, g, modal_arg<16>(b), q, psi)); break;
        default: QGN_LAUNCH(KID_MODAL, nb, s, ::qgn::launch(k_modal<0>, grid, 256, 0, s, g, modal_arg<0>(b), q, psi)); break;
    }
    return cudaGetLastError();
}

template <int NY, int NF, class CT, int TV>
static cudaError_t yinv_go(const Geom& g, const CT* q, const CT* psi, CT* hq, CT* hp, CT* hu, const CT* twy,
                           cudaStream_t s) {
    using C = YInvCfg<NY, CT, TV>;
    cudaError_t e;
    if ((e = set_smem(k_yinv<NY, NF, CT, TV>, C::SMEM)) != cudaSuccess) return e;
    dim3 grid((g.nkx + C::TKX - 1) / C::TKX, g.nz, (yinv_spread<NY, CT, TV>() && NF > 1) ? NF : 1);
    const double es = (double)sizeof(CT);
    const double Cb = es * (double)g.csize(), Hb = es * (double)g.nz * NY * g.nkx;
    QGN_LAUNCH(KID_YINV, NF == 3 ? 2.0 * Cb + 3.0 * Hb : NF * (Cb + Hb), s,
               ::qgn::launch(k_yinv<NY, NF, CT, TV>, grid, C::THREADS, C::SMEM, s, g, q, psi, hq, hp, hu, twy));
    return cudaGetLastError();
}

template <class CT>
static cudaError_t launch_yinv(const Geom& g, int nf, const CT* q, const CT* psi, CT* hq, CT* hp, CT* hu, const CT* twy,
                               cudaStream_t s) {
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        if constexpr (has_narrow<NY>()) {
            const long long cd = (long long)((g.nkx + YInvCfg<NY, CT>::TKX - 1) / YInvCfg<NY, CT>::TKX) * g.nz;
            const long long cn =
                (long long)((g.nkx + YInvCfg<NY, CT, kNarrowY>::TKX - 1) / YInvCfg<NY, CT, kNarrowY>::TKX) * g.nz;
            if (narrow_better(cd, cn)) {
                if constexpr (std::is_same<CT, double2>::value) {
                    if (nf == 2) return yinv_go<NY, 2, CT, kNarrowY>(g, q, psi, hq, hp, hu, twy, s);
                }
                return nf == 3 ? yinv_go<NY, 3, CT, kNarrowY>(g, q, psi, hq, hp, hu, twy, s)
                               : yinv_go<NY, 1, CT, kNarrowY>(g, q, psi, hq, hp, hu, twy, s);
            }
        }
        if constexpr (std::is_same<CT, double2>::value) {
            if (nf == 2) return yinv_go<NY, 2, CT, 0>(g, q, psi, hq, hp, hu, twy, s);
        }
        return nf == 3 ? yinv_go<NY, 3, CT, 0>(g, q, psi, hq, hp, hu, twy, s)
                       : yinv_go<NY, 1, CT, 0>(g, q, psi, hq, hp, hu, twy, s);
    });
}

template <int NX, bool DRAG, class CT, int TV>
static cudaError_t xpass_go(const Geom& g, int layer0, int layers, const CT* hq, const CT* hp, const CT* hu, CT* hpp,
                            CT* hpd, const CT* twx, cudaStream_t s) {
    using C = XCfg<NX, DRAG, CT, TV>;
    cudaError_t e;
    if ((e = set_smem(k_xpass<NX, DRAG, CT, TV>, C::SMEM)) != cudaSuccess) return e;
    dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, layers);
    const double es = (double)sizeof(CT);
    QGN_LAUNCH(KID_XPASS, (DRAG ? 7.0 : 5.0) * es * (double)layers * g.ny * g.nkx, s,
               ::qgn::launch(k_xpass<NX, DRAG, CT, TV>, grid, C::THREADS, C::SMEM, s, g, layer0, hq, hp, hu, hpp, hpd, twx));
    return cudaGetLastError();
}

template <class CT>
static cudaError_t launch_xpass(const Geom& g, const CT* hq, const CT* hp, const CT* hu, CT* hpp, CT* hpd, const CT* twx,
                                bool drag, cudaStream_t s) {
    return dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        cudaError_t e;
        const int nplain = drag ? g.nz - 1 : g.nz;
        bool narrow = false;
        if constexpr (has_narrow<NX>()) {
            const long long cd = (long long)((g.ny / 2 + XCfg<NX, false, CT>::RP - 1) / XCfg<NX, false, CT>::RP) * g.nz;
            const long long cn =
                (long long)((g.ny / 2 + XCfg<NX, false, CT, kNarrowX>::RP - 1) / XCfg<NX, false, CT, kNarrowX>::RP) *
                g.nz;
            narrow = narrow_better(cd, cn);
        }
        if (nplain > 0) {
            if constexpr (has_narrow<NX>())
                e = narrow ? xpass_go<NX, false, CT, kNarrowX>(g, 0, nplain, hq, hp, hu, hpp, hpd, twx, s)
                           : xpass_go<NX, false, CT, 0>(g, 0, nplain, hq, hp, hu, hpp, hpd, twx, s);
            else
                e = xpass_go<NX, false, CT, 0>(g, 0, nplain, hq, hp, hu, hpp, hpd, twx, s);
            if (e != cudaSuccess) return e;
        }
        if (drag) {
            if constexpr (has_narrow<NX>())
                e = narrow ? xpass_go<NX, true, CT, kNarrowX>(g, g.nz - 1, 1, hq, hp, hu, hpp, hpd, twx, s)
                           : xpass_go<NX, true, CT, 0>(g, g.nz - 1, 1, hq, hp, hu, hpp, hpd, twx, s);
            else
                e = xpass_go<NX, true, CT, 0>(g, g.nz - 1, 1, hq, hp, hu, hpp, hpd, twx, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    });
}

template <int NY, bool DRAG, class CT, int TV>
static cudaError_t yfwd_go(const Geom& g, int layer0, int layers, const LayerConst* lc, const CT* q, const CT* psi,
                           const CT* hpp, const CT* hpd, CT* out, const CT* twy, const CT* extra, cudaStream_t s) {
    using C = YFwdCfg<NY, DRAG, CT, TV>;
    cudaError_t e;
    if ((e = set_smem(k_yfwd<NY, DRAG, CT, TV>, C::SMEM)) != cudaSuccess) return e;
    dim3 grid((g.nkx + C::TKX - 1) / C::TKX, layers);
    const double lb = (double)sizeof(CT) * (double)layers * g.nkx;
    QGN_LAUNCH(KID_YFWD, lb * ((DRAG ? 4.0 : 2.0) * NY + 3.0 * g.nky), s,
               ::qgn::launch(k_yfwd<NY, DRAG, CT, TV>, grid, C::THREADS, C::SMEM, s, g, layer0, lc, q, psi, hpp, hpd, out, twy,
                                                                          extra));
    return cudaGetLastError();
}

template <class CT>
static cudaError_t launch_yfwd(const Geom& g, const LayerConst* lc, const CT* q, const CT* psi, const CT* hpp,
                               const CT* hpd, CT* out, const CT* twy, bool drag, cudaStream_t s,
                               const CT* extra = nullptr) {
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        cudaError_t e;
        const int nplain = drag ? g.nz - 1 : g.nz;
        bool narrow = false;
        if constexpr (has_narrow<NY>()) {
            using D = YFwdCfg<NY, false, CT>;
            using Nn = YFwdCfg<NY, false, CT, kNarrowY>;
            narrow = narrow_better((long long)((g.nkx + D::TKX - 1) / D::TKX) * g.nz,
                                   (long long)((g.nkx + Nn::TKX - 1) / Nn::TKX) * g.nz);
        }
        if (nplain > 0) {
            if constexpr (has_narrow<NY>())
                e = narrow ? yfwd_go<NY, false, CT, kNarrowY>(g, 0, nplain, lc, q, psi, hpp, hpd, out, twy, extra, s)
                           : yfwd_go<NY, false, CT, 0>(g, 0, nplain, lc, q, psi, hpp, hpd, out, twy, extra, s);
            else
                e = yfwd_go<NY, false, CT, 0>(g, 0, nplain, lc, q, psi, hpp, hpd, out, twy, extra, s);
            if (e != cudaSuccess) return e;
        }
        if (drag) {
            if constexpr (has_narrow<NY>())
                e = narrow ? yfwd_go<NY, true, CT, kNarrowY>(g, g.nz - 1, 1, lc, q, psi, hpp, hpd, out, twy, extra, s)
                           : yfwd_go<NY, true, CT, 0>(g, g.nz - 1, 1, lc, q, psi, hpp, hpd, out, twy, extra, s);
            else
                e = yfwd_go<NY, true, CT, 0>(g, g.nz - 1, 1, lc, q, psi, hpp, hpd, out, twy, extra, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    });
}

cudaError_t launch_rhs(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                       bool do_drag, cudaStream_t s, const double2* extra) {
    cudaError_t e;
    if ((e = launch_yinv<double2>(g, 3, q, psi, b.hq, b.hp, b.hu, b.twy, s)) != cudaSuccess) return e;
    return launch_rhs_tail(g, b, q, psi, out, do_drag, s, extra);
}

cudaError_t launch_rhs_tail(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                            bool do_drag, cudaStream_t s, const double2* extra) {
    cudaError_t e;
    if ((e = launch_rhs_x(g, b, do_drag, s)) != cudaSuccess) return e;
    return launch_rhs_yfwd(g, b, q, psi, out, do_drag, s, extra);
}

cudaError_t launch_rhs_x(const Geom& g, const Buffers& b, bool do_drag, cudaStream_t s) {
    return launch_xpass<double2>(g, b.hq, b.hp, b.hu, b.hpp, b.hpd, b.twx, do_drag, s);
}

cudaError_t launch_rhs_yfwd(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                            bool do_drag, cudaStream_t s, const double2* extra) {
    return launch_yfwd<double2>(g, b.lc, q, psi, b.hpp, b.hpd, out, b.twy, do_drag, s, extra);
}

// FP32 right-hand side of the mixed mode: compact FP32 q, psi in, compact FP32 RHS out; the
// half-transformed fields live in the (larger) FP64 buffers.
cudaError_t launch_rhs32(const Geom& g, const Buffers& b, const float2* q, const float2* psi, float2* out, bool do_drag,
                         cudaStream_t s) {
    float2* hq = reinterpret_cast<float2*>(b.hq);
    float2* hp = reinterpret_cast<float2*>(b.hp);
    float2* hu = reinterpret_cast<float2*>(b.hu);
    float2* hpp = reinterpret_cast<float2*>(b.hpp);
    float2* hpd = reinterpret_cast<float2*>(b.hpd);
    cudaError_t e;
    if ((e = launch_yinv<float2>(g, 3, q, psi, hq, hp, hu, b.twy32, s)) != cudaSuccess) return e;
    if ((e = launch_xpass<float2>(g, hq, hp, hu, hpp, hpd, b.twx32, do_drag, s)) != cudaSuccess) return e;
    return launch_yfwd<float2>(g, b.lc, q, psi, hpp, hpd, out, b.twy32, do_drag, s);
}

template <int NX, int EPI, int TV, class CT>
static cudaError_t xinv1_go(const Geom& g, const CT* hq, const CT* twx, DevScalars* sc, double* outp, cudaStream_t s) {
    using C = X1Cfg<NX, TV, CT>;
    cudaError_t e;
    if ((e = set_smem(k_xinv1<NX, EPI, TV, CT>, C::SMEM)) != cudaSuccess) return e;
    dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, g.nz);
    const double hb = (double)sizeof(CT) * (double)g.nz * g.ny * g.nkx;
    QGN_LAUNCH(KID_XINV1, hb + (EPI == 1 ? 8.0 * (double)g.nz * g.ny * NX : 0.0), s,
               ::qgn::launch(k_xinv1<NX, EPI, TV, CT>, grid, C::THREADS, C::SMEM, s, g, hq, sc, outp, twx));
    return cudaGetLastError();
}

template <int EPI, class CT = double2>
static cudaError_t launch_xinv1(const Geom& g, const CT* hq, const CT* twx, DevScalars* sc, double* outp,
                                cudaStream_t s) {
    return dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        if constexpr (has_narrow<NX>()) {
            using CD = X1Cfg<NX, 0, CT>;
            using CN = X1Cfg<NX, kNarrowX1, CT>;
            const long long cd = (long long)((g.ny / 2 + CD::RP - 1) / CD::RP) * g.nz;
            const long long cn = (long long)((g.ny / 2 + CN::RP - 1) / CN::RP) * g.nz;
            if (narrow_better(cd, cn)) return xinv1_go<NX, EPI, kNarrowX1, CT>(g, hq, twx, sc, outp, s);
        }
        return xinv1_go<NX, EPI, 0, CT>(g, hq, twx, sc, outp, s);
    });
}

cudaError_t launch_maxabs_phys(const Geom& g, const Buffers& b, const double2* f, DevScalars* sc, cudaStream_t s) {
    cudaError_t e;
    if ((e = launch_yinv<double2>(g, 1, f, nullptr, b.hq, nullptr, nullptr, b.twy, s)) != cudaSuccess) return e;
    return launch_xinv1<0>(g, b.hq, b.twx, sc, nullptr, s);
}

// the same from an FP32 spectrum with FP32 transforms (the mixed mode's error norm)
cudaError_t launch_maxabs_phys32(const Geom& g, const Buffers& b, const float2* f, DevScalars* sc, cudaStream_t s) {
    cudaError_t e;
    float2* hq = reinterpret_cast<float2*>(b.hq);
    if ((e = launch_yinv<float2>(g, 1, f, nullptr, hq, nullptr, nullptr, b.twy32, s)) != cudaSuccess) return e;
    return launch_xinv1<0, float2>(g, hq, b.twx32, sc, nullptr, s);
}

template <int NX, int SRC, int TV>
static cudaError_t xfwd1_go(const Geom& g, const Buffers& b, const double* phys, const float* y, int cout_p,
                            const float* osc, double2* dst, cudaStream_t s) {
    using C = X1Cfg<NX, TV>;
    cudaError_t e;
    if ((e = set_smem(k_xfwd1<NX, SRC, TV>, C::SMEM)) != cudaSuccess) return e;
    dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, g.nz);
    QGN_LAUNCH(KID_XFWD1, (SRC ? 4.0 : 8.0) * (double)g.nz * g.ny * NX + 16.0 * (double)g.nz * g.ny * g.nkx, s,
               ::qgn::launch(k_xfwd1<NX, SRC, TV>, grid, C::THREADS, C::SMEM, s, g, phys, dst, b.twx, y, cout_p, osc));
    return cudaGetLastError();
}

// forward x transform of a physical field (SRC 0) or of the closure's NHWC output (SRC 1)
// into packed rows at dst
template <int SRC>
static cudaError_t launch_xfwd1(const Geom& g, const Buffers& b, const double* phys, const float* y, int cout_p,
                                const float* osc, double2* dst, cudaStream_t s) {
    return dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        if constexpr (has_narrow<NX>()) {
            const long long cd = (long long)((g.ny / 2 + X1Cfg<NX>::RP - 1) / X1Cfg<NX>::RP) * g.nz;
            const long long cn = (long long)((g.ny / 2 + X1Cfg<NX, kNarrowX1>::RP - 1) / X1Cfg<NX, kNarrowX1>::RP) * g.nz;
            if (narrow_better(cd, cn)) return xfwd1_go<NX, SRC, kNarrowX1>(g, b, phys, y, cout_p, osc, dst, s);
        }
        return xfwd1_go<NX, SRC, 0>(g, b, phys, y, cout_p, osc, dst, s);
    });
}

cudaError_t launch_from_phys(const Geom& g, const Buffers& b, const double* phys, double2* out, cudaStream_t s) {
    cudaError_t e = launch_xfwd1<0>(g, b, phys, nullptr, 0, nullptr, b.hq, s);
    if (e != cudaSuccess) return e;
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        using C = YInvCfg<NY>;
        cudaError_t e2;
        if ((e2 = set_smem(k_yfwd1<NY>, C::SMEM)) != cudaSuccess) return e2;
        dim3 grid((g.nkx + C::TKX - 1) / C::TKX, g.nz);
        QGN_LAUNCH(KID_YFWD1, 16.0 * (double)g.nz * g.nkx * (NY + g.nky), s,
                   ::qgn::launch(k_yfwd1<NY>, grid, C::THREADS, C::SMEM, s, g, b.hq, out, b.twy));
        return cudaGetLastError();
    });
}

cudaError_t launch_to_phys(const Geom& g, const Buffers& b, const double2* f, double* out, cudaStream_t s) {
    cudaError_t e;
    if ((e = launch_yinv<double2>(g, 1, f, nullptr, b.hq, nullptr, nullptr, b.twy, s)) != cudaSuccess) return e;
    return launch_xinv1<1>(g, b.hq, b.twx, nullptr, out, s);
}


// ------------------------------------------------------------------------------------
// The learned closure's tensors: the network input (scaled physical q, psi as NHWC BF16)
// straight from the y-inverse's packed rows, and the forward transform of its NHWC output.
// ------------------------------------------------------------------------------------
template <int NX, int TV>
__global__ void __launch_bounds__(X1Cfg<NX, TV>::THREADS, minb(X1Cfg<NX, TV>::THREADS))
    k_xpack(Geom g, const double2* __restrict__ hq_q, const double2* __restrict__ hq_psi,
            const double2* __restrict__ twx, const float* __restrict__ scale, __nv_bfloat16* __restrict__ xout,
            int cin_p) {
    QGN_PDL_ENTRY();
    const int field = blockIdx.y / g.nz, l = blockIdx.y % g.nz;
    xinv1_tile<NX, 2, TV>(g, blockIdx.x, l, field ? hq_psi : hq_q, nullptr, nullptr, twx, scale, xout, cin_p,
                          field * g.nz + l);
}

template <int NX, int TV>
static cudaError_t xpack_go(const Geom& g, const Buffers& b, const double2* hq, const double2* hu, const float* scale,
                            __nv_bfloat16* xout, int cin_p, cudaStream_t s) {
    using C = X1Cfg<NX, TV>;
    cudaError_t e;
    if ((e = set_smem(k_xpack<NX, TV>, C::SMEM)) != cudaSuccess) return e;
    dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, 2 * g.nz);
    QGN_LAUNCH(KID_XINV1, 2.0 * (16.0 * g.nz * g.ny * g.nkx + 2.0 * g.nz * g.ny * NX), s,
               ::qgn::launch(k_xpack<NX, TV>, grid, C::THREADS, C::SMEM, s, g, hq, hu, b.twx, scale, xout, cin_p));
    return cudaGetLastError();
}

cudaError_t launch_closure_input(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* hq,
                                 double2* hu, const float* scale, void* xout, int cin_p, cudaStream_t s) {
    cudaError_t e = launch_yinv<double2>(g, 2, q, psi, hq, nullptr, hu, b.twy, s);
    if (e != cudaSuccess) return e;
    __nv_bfloat16* x = static_cast<__nv_bfloat16*>(xout);
    return dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        if constexpr (has_narrow<NX>()) {
            const long long cd = (long long)((g.ny / 2 + X1Cfg<NX>::RP - 1) / X1Cfg<NX>::RP) * 2 * g.nz;
            const long long cn =
                (long long)((g.ny / 2 + X1Cfg<NX, kNarrowX1>::RP - 1) / X1Cfg<NX, kNarrowX1>::RP) * 2 * g.nz;
            if (narrow_better(cd, cn)) return xpack_go<NX, kNarrowX1>(g, b, hq, hu, scale, x, cin_p, s);
        }
        return xpack_go<NX, 0>(g, b, hq, hu, scale, x, cin_p, s);
    });
}

cudaError_t launch_closure_output(const Geom& g, const Buffers& b, const float* y, int cout_p, const float* osc,
                                  double2* h, double2* out, cudaStream_t s) {
    cudaError_t e = launch_xfwd1<1>(g, b, nullptr, y, cout_p, osc, h, s);
    if (e != cudaSuccess) return e;
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        using C = YInvCfg<NY>;
        cudaError_t e2;
        if ((e2 = set_smem(k_yfwd1<NY>, C::SMEM)) != cudaSuccess) return e2;
        dim3 grid((g.nkx + C::TKX - 1) / C::TKX, g.nz);
        QGN_LAUNCH(KID_YFWD1, 16.0 * (double)g.nz * g.nkx * (NY + g.nky), s,
                   ::qgn::launch(k_yfwd1<NY>, grid, C::THREADS, C::SMEM, s, g, h, out, b.twy));
        return cudaGetLastError();
    });
}

// ------------------------------------------------------------------------------------
// WriteQPmodal support (QGN_Module.f90:381-440): the reference's Jacobian there is the full,
// undealiased spectrum of i kx (uq)^ + i ky (vq)^.  The transform kernels above run on it
// with a "full" geometry -- every kx up to Nyquist and every ky kept, compact index = ky index.
// ------------------------------------------------------------------------------------
Geom full_geom(const Geom& g) {
    Geom f = g;
    f.nkx = g.nxh;
    f.nkxp = (g.nxh + 3) / 4 * 4;
    f.kylo = g.ny;
    f.kyshift = 0;
    f.nky = g.ny;
    return f;
}

__global__ void k_uv_hat(Geom g, const double2* __restrict__ psi, double2* __restrict__ uh, double2* __restrict__ vh) {
    QGN_PDL_ENTRY();
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t total = P * g.nz;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t p = e % P;
        const int kx = (int)(p / g.nky), m = (int)(p % g.nky);
        const double kxv = g.dkx * kx, kyv = g.kyval(g.jfull(m));
        const double2 v = psi[e];
        uh[e] = make_double2(kyv * v.y, -kyv * v.x);      // -i ky psi_hat (QGN_Module.f90:223)
        vh[e] = make_double2(-kxv * v.y, kxv * v.x);      //  i kx psi_hat (QGN_Module.f90:224)
    }
}

__global__ void k_products(size_t n, const double* __restrict__ q, double* __restrict__ u, double* __restrict__ v) {
    QGN_PDL_ENTRY();
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const double qq = q[e];
        u[e] = u[e] * qq;     // u_phys*q_phys
        v[e] = v[e] * qq;     // v_phys*q_phys
    }
}

// jaco_hat = i kx uq_hat + i ky vq_hat on the full spectrum (QGN_Module.f90:244-247), in place into uq
__global__ void k_jac_full(Geom gf, double2* __restrict__ uq, const double2* __restrict__ vq) {
    QGN_PDL_ENTRY();
    const size_t P = (size_t)gf.nkx * gf.nky;
    const size_t total = P * gf.nz;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t p = e % P;
        const int kx = (int)(p / gf.nky), j = (int)(p % gf.nky);
        const double kxv = gf.dkx * kx, kyv = gf.kyval(j);
        const double2 a = uq[e], b = vq[e];
        uq[e] = make_double2(-kxv * a.y - kyv * b.y, kxv * a.x + kyv * b.x);
    }
}

// modal projection x_mode(k) = sum_kk H(kk) Modes(kk,k) x(kk) / Htot (QGN_Module.f90:392-398), and
// optionally psi_mode = q_mode / (-k^2 + EVals(k)) with psi_mode(1,1) = 0 (QGN_Module.f90:399-400)
__global__ void k_modal_proj(Geom g, const ModalConst* __restrict__ mc, const double2* __restrict__ x,
                             double2* __restrict__ xm, double2* __restrict__ pm) {
    QGN_PDL_ENTRY();
    const size_t P = (size_t)g.nkx * g.nky;
    const int nz = g.nz;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (size_t)gridDim.x * blockDim.x) {
        const int kx = (int)(p / g.nky), m = (int)(p % g.nky);
        const double kxv = g.dkx * kx, kyv = g.kyval(g.jfull(m));
        const double k2 = kxv * kxv + kyv * kyv;
        for (int k = 0; k < nz; ++k) {
            double2 acc = make_double2(0.0, 0.0);
            for (int kk = 0; kk < nz; ++kk) {
                const double c = mc->proj[k * nz + kk];
                const double2 v = x[(size_t)kk * P + p];
                acc.x += c * v.x;
                acc.y += c * v.y;
            }
            const double2 qm = make_double2(acc.x / mc->Htot, acc.y / mc->Htot);
            xm[(size_t)k * P + p] = qm;
            if (pm) {
                const double den = -k2 + mc->evals[k];
                pm[(size_t)k * P + p] = (p == 0) ? make_double2(0.0, 0.0) : make_double2(qm.x / den, qm.y / den);
            }
        }
    }
}

cudaError_t launch_modal_fields(const Geom& g, const Buffers& b, const double2* q, double* out_q, double* out_p,
                                double* out_j, double2* full_half, double2* fa, double2* fb, double* phys3,
                                cudaStream_t s) {
    // fa and fb (full spectra) are larger than a compact field: they hold u_hat, v_hat first and
    // the compact q_mode, psi_mode last; b.psi is overwritten, nothing else of b is touched
    cudaError_t e;
    const int blocks = 148 * 8;
    const size_t np = (size_t)g.nz * g.ny * g.nx;
    double* Pq = phys3;
    double* Pu = phys3 + np;
    double* Pv = phys3 + 2 * np;
    // GetPsi, u_hat, v_hat and the physical fields of the Jacobian (QGN_Module.f90:218-234)
    if ((e = launch_modal(g, b, q, b.psi, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_LAYOUT, 48.0 * (double)g.csize(), s, ::qgn::launch(k_uv_hat, blocks, 256, 0, s, g, b.psi, fa, fb));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, q, Pq, s)) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, fa, Pu, s)) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, fb, Pv, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_LAYOUT, 40.0 * (double)np, s, ::qgn::launch(k_products, blocks, 256, 0, s, np, Pq, Pu, Pv));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // full-spectrum r2c of u*q and v*q and the undealiased Jacobian (QGN_Module.f90:235-247)
    const Geom gf = full_geom(g);
    Buffers bf = b;
    bf.hq = full_half;
    if ((e = launch_from_phys(gf, bf, Pu, fa, s)) != cudaSuccess) return e;
    if ((e = launch_from_phys(gf, bf, Pv, fb, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_LAYOUT, 48.0 * (double)gf.csize(), s, ::qgn::launch(k_jac_full, blocks, 256, 0, s, gf, fa, fb));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // modal projections and their physical fields (QGN_Module.f90:390-415)
    QGN_LAUNCH(KID_MODAL, 32.0 * (double)gf.csize(), s, ::qgn::launch(k_modal_proj, blocks, 256, 0, s, gf, b.mc, fa, fb, nullptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_to_phys(gf, bf, fb, out_j, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_MODAL, 48.0 * (double)g.csize(), s, ::qgn::launch(k_modal_proj, blocks, 256, 0, s, g, b.mc, q, fa, fb));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, fa, out_q, s)) != cudaSuccess) return e;
    return launch_to_phys(g, b, fb, out_p, s);
}

}  // namespace qgn
