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

#include <mutex>
#include <type_traits>
#include <unordered_set>

namespace qgn {

// ------------------------------------------------------------------------------------
// Tile shapes
// ------------------------------------------------------------------------------------
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }

// slot stride (in elements) of a padded transform such that slot*stride spreads the bank
// groups of one shared-memory wavefront: W = 128 bytes / element size elements per wavefront
// (8 for double2, 16 for float2); target is the stride's residue mod W.
__host__ __device__ constexpr int slot_stride(int N, int target, int elem_bytes = 16) {
    return fpadlen(N) + ((target - (fpadlen(N) % (128 / elem_bytes))) + (128 / elem_bytes)) % (128 / elem_bytes);
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
template <int NY, class CT = double2>
struct YInvCfg {
    static constexpr int G = FFTShape<NY>::G;
    static constexpr int TKX = cmin(cmax(4, 128 / G), 16);
    static constexpr int THREADS = TKX * G;
    static constexpr int TS = slot_stride(NY, interleave_target(TKX, (int)sizeof(CT)), (int)sizeof(CT));
    static constexpr int SMEM = TKX * TS * (int)sizeof(CT);
};

template <int NX, bool DRAG, class CT = double2>
struct XCfg {
    static constexpr int G = FFTShape<NX>::G;
    static constexpr int RP = cmax(1, 64 / G);         // row pairs per CTA
    static constexpr int SP = DRAG ? 4 : 3;             // slots per row pair
    static constexpr int THREADS = SP * RP * G;
    static constexpr int TS = slot_stride(NX, 2);
    static constexpr int SMEM = SP * RP * TS * (int)sizeof(CT);
};

template <int NY, bool DRAG, class CT = double2>
struct YFwdCfg {
    static constexpr int G = FFTShape<NY>::G;
    static constexpr int TKX = cmin(cmax(2, 64 / G), 16);   // tid ^ TKX stays in the warp
    static constexpr int SLOTS = 2 * TKX;
    static constexpr int THREADS = SLOTS * G;
    static constexpr int TS = slot_stride(NY, interleave_target(SLOTS, (int)sizeof(CT)), (int)sizeof(CT));
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

template <int NZ>
__global__ void __launch_bounds__(256, 2) k_modal(Geom g, const ModalConst* __restrict__ mc,
                                               const double2* __restrict__ q, double2* __restrict__ psi) {
    __shared__ double s_proj[kMaxNZ * kMaxNZ], s_back[kMaxNZ * kMaxNZ], s_ev[kMaxNZ];
    const int nz = g.nz;
    for (int i = threadIdx.x; i < nz * nz; i += blockDim.x) { s_proj[i] = mc->proj[i]; s_back[i] = mc->back[i]; }
    for (int i = threadIdx.x; i < nz; i += blockDim.x) s_ev[i] = mc->evals[i];
    __syncthreads();
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
        if (k < nz) qv[k] = q[(size_t)k * P + p];
    modal_invert<NZ>(s_proj, s_back, s_ev, mc->Htot, nz, k2, p == 0, qv, pv);
#pragma unroll
    for (int k = 0; k < NZC; ++k)
        if (k < nz) psi[(size_t)k * P + p] = pv[k];
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

// ------------------------------------------------------------------------------------
// yinv: inverse y transforms of kept columns into packed row pairs.
// NF = 3: (q -> pq, -i ky psi -> pu, i kx psi -> pv);  NF = 1: (f -> pq).
// The first radix pass reads the compact column straight from HBM (zeros in the dealiased
// band); the transformed column stays in shared memory, where a packing loop pairs rows
// y and y+1 and writes the two packed arrays with TKX-wide coalesced stores.
// ------------------------------------------------------------------------------------
template <int NY, int NF, class CT>
__global__ void __launch_bounds__(YInvCfg<NY, CT>::THREADS, minb(YInvCfg<NY, CT>::THREADS, regcap<CT>()))
    k_yinv(Geom g, const CT* __restrict__ q, const CT* __restrict__ psi, CT* __restrict__ pq,
           CT* __restrict__ pv, CT* __restrict__ pu, const CT* __restrict__ twy) {
    using C = YInvCfg<NY, CT>;
    using RT = typename CTraits<CT>::R;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    CT* sm = reinterpret_cast<CT*>(sm_raw);
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int kx0 = blockIdx.x * C::TKX;
    const int slot = tid % C::TKX, lane = tid / C::TKX;
    const int kx = kx0 + slot;
    const bool colok = kx < g.nkx;
    const size_t colbase = ((size_t)l * g.nkx + kx) * g.nky;
    const RT kxv = (RT)(g.dkx * kx);
    CT* xs = sm + slot * C::TS;
    NoIOT<CT> none;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        const CT* src = (f == 0) ? q : psi;
        CT* dst = (f == 0) ? pq : (f == 1 ? pu : pv);
        auto ld = [&](int j) -> CT {
            const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
            if (!colok || !kept) return cmk<CT>(0.0, 0.0);
            CT v = src[colbase + (j < g.kylo ? j : j - g.kyshift)];
            if (f == 1) {   // u_hat = -i ky psi_hat  (QGN_Module.f90:223)
                const RT kyv = (RT)g.kyval(j);
                v = cmk<CT>(kyv * v.y, -kyv * v.x);
            } else if (f == 2) {   // v_hat = i kx psi_hat  (QGN_Module.f90:224)
                v = cmk<CT>(-kxv * v.y, kxv * v.x);
            }
            return v;
        };
        fft_fused<NY, +1, SRC_FN, DST_SMEM>(xs, lane, true, twy, ld, none);
        // pack rows (2p, 2p+1): e -> (pair p, column c); both arrays of a pair row per thread
        CT* dl = dst + (size_t)l * (NY / 2) * 2 * g.nkxp;
        for (int e = tid; e < (NY / 2) * C::TKX; e += C::THREADS) {
            const int p = e / C::TKX, c = e % C::TKX;
            const int k = kx0 + c;
            if (k >= g.nkxp) continue;
            const CT f1 = sm[c * C::TS + fpad(2 * p)], f2 = sm[c * C::TS + fpad(2 * p + 1)];
            const bool ok = k < g.nkx;
            CT* row = dl + (size_t)p * 2 * g.nkxp;
            // Re parts at kx = 0 and at the kx Nyquist column (kept only in the full-spectrum geometry)
            row[k] = ok ? pack_lo(f1, f2, k == 0 || 2 * k == g.nx) : cmk<CT>(0.0, 0.0);
            row[g.nkxp + k] = (ok && k > 0) ? pack_hi(f1, f2) : cmk<CT>(0.0, 0.0);
        }
        if (f + 1 < NF) __syncthreads();   // the next field's first pass reuses the slots
    }
}

// ------------------------------------------------------------------------------------
// xpass: x transforms of row pairs.  c2r of the packed q1 + i q2, u1 + i u2, v1 + i v2
// (pairing two rows of one field keeps roundoff relative to that field; q and u differ by
// ~1e4 in these units), physical products formed inside the first pass of the forward
// transforms, r2c of p = uq + i vq per row, whose last pass writes P[k] and P[nx-k] for the
// kept kx straight to HBM.
// ------------------------------------------------------------------------------------
template <int NX, bool DRAG, class CT>
__global__ void __launch_bounds__(XCfg<NX, DRAG, CT>::THREADS, minb(XCfg<NX, DRAG, CT>::THREADS, regcap<CT>(128, 80)))
    k_xpass(Geom g, int layer0, const CT* __restrict__ pq, const CT* __restrict__ pv,
            const CT* __restrict__ pu, CT* __restrict__ pp, CT* __restrict__ pd,
            const CT* __restrict__ twx) {
    using C = XCfg<NX, DRAG, CT>;
    using RT = typename CTraits<CT>::R;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    CT* sm = reinterpret_cast<CT*>(sm_raw);
    const int tid = threadIdx.x;
    const int l = layer0 + blockIdx.y;
    const int npairs = g.ny / 2;
    const int nkx = g.nkx;
    const int slot = tid / C::G, lane = tid % C::G;
    const int r_of = slot / C::SP, s_of = slot % C::SP;
    const int rp = blockIdx.x * C::RP + r_of;
    const bool pair_ok = rp < npairs;
    CT* base = sm + (r_of * C::SP) * C::TS;
    CT* xs = sm + slot * C::TS;

    // ---- inverse: slot 0 = q1+iq2, 1 = u1+iu2, 2 = v1+iv2
    const CT* F = (s_of == 0 ? pq : (s_of == 1 ? pu : pv)) + ((size_t)l * npairs + rp) * 2 * g.nkxp;
    auto ld_inv = [&](int k) -> CT {
        if (k < nkx) return F[k];
        if (k > NX - nkx) return F[g.nkxp + (NX - k)];
        return cmk<CT>(0.0, 0.0);
    };
    NoIOT<CT> none;
    fft_fused<NX, +1, SRC_FN, DST_SMEM>(xs, lane, pair_ok && s_of < 3, twx, ld_inv, none);

    // ---- forward: slot 0 = u1 q1 + i v1 q1, 1 = u2 q2 + i v2 q2 (grid/(nx*ny) scaling as in
    //      QGN_Module.f90:229-235); with drag 2 = |u1|u1 + i|u1|v1, 3 = |u2|u2 + i|u2|v2
    const RT sc = (RT)g.inv_nxny;
    auto ld_fwd = [&](int x) -> CT {
        const CT a = base[fpad(x)], bu = base[C::TS + fpad(x)], cv = base[2 * C::TS + fpad(x)];
        const bool second = (s_of & 1) != 0;
        const RT qv = (second ? a.y : a.x) * sc;
        const RT uv = (second ? bu.y : bu.x) * sc;
        const RT vv = (second ? cv.y : cv.x) * sc;
        if (s_of < 2) return cmk<CT>(uv * qv, vv * qv);
        const RT m = sqrt(uv * uv + vv * vv);   // URMS, QGN_Module.f90:285
        return cmk<CT>(m * uv, m * vv);
    };
    const int y = 2 * rp + (s_of & 1);
    CT* out = (s_of < 2) ? pp + ((size_t)l * g.ny + y) * 2 * g.nkxp : pd + (size_t)y * 2 * g.nkxp;
    auto st_fwd = [&](int k, CT v) {
        if (k < nkx) out[k] = v;
        else if (k > NX - nkx) out[g.nkxp + (NX - k)] = v;
    };
    fft_fused<NX, -1, SRC_FN_SMEM, DST_FN>(xs, lane, pair_ok && s_of < (DRAG ? 4 : 2), twx, ld_fwd, st_fwd);
}

// ------------------------------------------------------------------------------------
// yfwd: forward y transforms of uq, vq columns and assembly of the right-hand side.
// Slots are lane-interleaved: slot = tid % (2 TKX), slot = field*TKX + column.  The first
// radix pass reads the half-transformed rows straight from HBM.
// ------------------------------------------------------------------------------------
// split of the packed forward x transform of row y at kx: fld 0 -> (uq)^, fld 1 -> (vq)^
__device__ __forceinline__ double2 unpack_p(const double2* __restrict__ row, int nkxp, int kx, int fld) {
    const double2 X = row[kx];
    const double2 Y = kx == 0 ? cconj(X) : cconj(row[nkxp + kx]);
    return fld == 0 ? make_double2(0.5 * (X.x + Y.x), 0.5 * (X.y + Y.y))
                    : make_double2(0.5 * (X.y - Y.y), -0.5 * (X.x - Y.x));
}

template <class CT>
__device__ __forceinline__ CT unpack_pair(const CT* __restrict__ row, int nkxp, int kx, int fld, bool ok, int partner) {
    CT mine = cmk<CT>(0.0, 0.0);
    if (ok && (fld == 0 || kx > 0)) mine = row[fld == 0 ? kx : nkxp + kx];
    CT other;
    other.x = __shfl_xor_sync(0xffffffffu, mine.x, partner);
    other.y = __shfl_xor_sync(0xffffffffu, mine.y, partner);
    const CT X = fld == 0 ? mine : other;
    const CT Y = kx == 0 ? cconj(X) : cconj(fld == 0 ? other : mine);
    return fld == 0 ? cmk<CT>((typename CTraits<CT>::R)0.5 * (X.x + Y.x), (typename CTraits<CT>::R)0.5 * (X.y + Y.y))
                    : cmk<CT>((typename CTraits<CT>::R)0.5 * (X.y - Y.y), -(typename CTraits<CT>::R)0.5 * (X.x - Y.x));
}

template <int NY, bool DRAG, class CT>
__global__ void __launch_bounds__(YFwdCfg<NY, DRAG, CT>::THREADS, minb(YFwdCfg<NY, DRAG, CT>::THREADS, regcap<CT>()))
    k_yfwd(Geom g, int layer0, const LayerConst* __restrict__ lc, const CT* __restrict__ q,
           const CT* __restrict__ psi, const CT* __restrict__ pp, const CT* __restrict__ pd,
           CT* __restrict__ out, const CT* __restrict__ twy) {
    using C = YFwdCfg<NY, DRAG, CT>;
    using RT = typename CTraits<CT>::R;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    CT* sm = reinterpret_cast<CT*>(sm_raw);
    const int tid = threadIdx.x;
    const int l = layer0 + blockIdx.y;
    const int kx0 = blockIdx.x * C::TKX;
    const int slot = tid % C::SLOTS, lane = tid / C::SLOTS;
    const int fld = slot / C::TKX, c = slot % C::TKX;
    const bool colok = kx0 + c < g.nkx;
    const int nky = g.nky;
    const size_t colbase = (size_t)l * g.nkx;
    const bool bottom = (l == g.nz - 1);
    CT* xs = sm + slot * C::TS;
    NoIOT<CT> none;

    if (DRAG) {
        // drag_hat = i ky (|u|u)^ - i kx (|u|v)^ on the bottom layer (QGN_Module.f90:284-292)
        auto ldd = [&](int y) -> CT {
            return unpack_pair(pd + (size_t)y * 2 * g.nkxp, g.nkxp, kx0 + c, fld, colok, C::TKX);
        };
        fft_fused<NY, -1, SRC_FN, DST_SMEM>(xs, lane, true, twy, ldd, none);
        const RT dc = (RT)lc->dragc;
        for (int e = tid; e < C::TKX * nky; e += C::THREADS) {
            const int cc = e / nky, m = e % nky;
            const int kx = kx0 + cc;
            if (kx >= g.nkx) continue;
            const int j = g.jfull(m);
            const RT kxv = (RT)(g.dkx * kx), kyv = (RT)g.kyval(j);
            const CT fu = sm[cc * C::TS + fpad(j)], fv = sm[(C::TKX + cc) * C::TS + fpad(j)];
            CT d = cmk<CT>(-kyv * fu.y, kyv * fu.x);        // i ky (|u|u)^
            d = cmk<CT>(d.x + kxv * fv.y, d.y - kxv * fv.x);      // - i kx (|u|v)^
            out[(colbase + kx) * nky + m] = cmk<CT>(dc * d.x, dc * d.y);
        }
        __syncthreads();
    }

    // the (uq)^ and (vq)^ slots of one column load P[k] and P[nx-k] respectively and swap
    // them with a shuffle (partner tid ^ TKX, same warp), so each value is read once
    auto ld = [&](int y) -> CT { return unpack_pair(pp + ((size_t)l * NY + y) * 2 * g.nkxp, g.nkxp, kx0 + c,
                                                         fld, colok, C::TKX); };
    fft_fused<NY, -1, SRC_FN, DST_SMEM>(xs, lane, true, twy, ld, none);

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
        const CT fuq = sm[cc * C::TS + fpad(j)], fvq = sm[(C::TKX + cc) * C::TS + fpad(j)];
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
        if (kx == 0 && m == 0) r = cmk<CT>(0.0, 0.0);
        out[idx] = r;
    }
}

// ------------------------------------------------------------------------------------
// Single-field inverse 2-D transform: x c2r of row pairs with an epilogue
//   EPI 0: max |grid| (unnormalised) into sc->maxbits
//   EPI 1: physical field grid/(nx*ny) into out[nz][ny][nx]
// ------------------------------------------------------------------------------------
template <int NX>
struct X1Cfg {
    static constexpr int G = FFTShape<NX>::G;
    static constexpr int RP = cmax(1, 128 / G);
    static constexpr int THREADS = RP * G;
    static constexpr int TS = slot_stride(NX, 2);
    static constexpr int SMEM = RP * TS * (int)sizeof(double2);
};

template <int NX, int EPI>
__global__ void __launch_bounds__(X1Cfg<NX>::THREADS, minb(X1Cfg<NX>::THREADS))
    k_xinv1(Geom g, const double2* __restrict__ hq, DevScalars* __restrict__ sc, double* __restrict__ outp,
            const double2* __restrict__ twx) {
    using C = X1Cfg<NX>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = reinterpret_cast<double2*>(sm_raw);
    __shared__ double smax[32];
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int npairs = g.ny / 2;
    const int nkx = g.nkx;
    const int slot = tid / C::G, lane = tid % C::G;
    const int rp = blockIdx.x * C::RP + slot;
    const bool ok = rp < npairs;
    const double2* F = hq + ((size_t)l * npairs + rp) * 2 * g.nkxp;   // packed row pair
    auto ld = [&](int k) -> double2 {
        if (k < nkx) return F[k];
        if (k > NX - nkx) return F[g.nkxp + (NX - k)];
        return make_double2(0.0, 0.0);
    };
    double mx = 0.0;
    const size_t prow = ((size_t)l * g.ny + 2 * rp) * NX;
    auto st = [&](int x, double2 a) {
        if (EPI == 0) {
            // NaN is kept as the largest value
            const double m1 = fabs(a.x), m2 = fabs(a.y);
            if (!(m1 == m1) || !(m2 == m2)) mx = __longlong_as_double(0x7ff8000000000000LL);
            else if (mx == mx) mx = fmax(mx, fmax(m1, m2));
        } else {
            outp[prow + x] = a.x * g.inv_nxny;
            outp[prow + NX + x] = a.y * g.inv_nxny;
        }
    };
    fft_fused<NX, +1, SRC_FN, DST_FN>(sm + slot * C::TS, lane, ok, twx, ld, st);
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

// ------------------------------------------------------------------------------------
// Forward 2-D transform of a physical field (DftiComputeForward + DeAlias of Initialize,
// QGN_Module.f90:179-183): r2c of row pairs packed as r1 + i r2, then forward y columns
// keeping the dealiased modes only.
// ------------------------------------------------------------------------------------
template <int NX>
__global__ void __launch_bounds__(X1Cfg<NX>::THREADS, minb(X1Cfg<NX>::THREADS))
    k_xfwd1(Geom g, const double* __restrict__ phys, double2* __restrict__ hq, const double2* __restrict__ twx) {
    using C = X1Cfg<NX>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* sm = reinterpret_cast<double2*>(sm_raw);
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int npairs = g.ny / 2;
    const int slot = tid / C::G, lane = tid % C::G;
    const int rp = blockIdx.x * C::RP + slot;
    const size_t prow = ((size_t)l * g.ny + 2 * rp) * NX;
    auto ld = [&](int x) -> double2 { return make_double2(phys[prow + x], phys[prow + NX + x]); };
    NoIO none;
    fft_fused<NX, -1, SRC_FN, DST_SMEM>(sm + slot * C::TS, lane, rp < npairs, twx, ld, none);
    const int nkx = g.nkx;
    for (int e = tid; e < C::RP * nkx; e += C::THREADS) {
        const int r = e / nkx, k = e % nkx;
        const int rq = blockIdx.x * C::RP + r;
        if (rq >= npairs) continue;
        const double2 X = sm[r * C::TS + fpad(k)];
        const double2 Y = cconj(sm[r * C::TS + fpad((NX - k) & (NX - 1))]);
        const size_t row = ((size_t)l * g.ny + 2 * rq) * g.nkxp + k;
        hq[row] = make_double2(0.5 * (X.x + Y.x), 0.5 * (X.y + Y.y));
        hq[row + g.nkxp] = make_double2(0.5 * (X.y - Y.y), -0.5 * (X.x - Y.x));
    }
}

template <int NY>
__global__ void __launch_bounds__(YInvCfg<NY>::THREADS, minb(YInvCfg<NY>::THREADS))
    k_yfwd1(Geom g, const double2* __restrict__ hq, double2* __restrict__ out, const double2* __restrict__ twy) {
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
    fft_fused<NY, -1, SRC_FN, DST_FN>(sm + slot * C::TS, lane, true, twy, ld, st);
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

// Opt a kernel into more than 48 KB of dynamic shared memory once per process, so that
// later launches -- including those recorded into CUDA graphs -- issue no attribute calls.
static std::mutex g_attr_mu;
static std::unordered_set<const void*> g_attr_done;

template <class K>
static cudaError_t set_smem(K kernel, int bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    const void* key = reinterpret_cast<const void*>(kernel);
    if (g_attr_done.count(key)) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) g_attr_done.insert(key);
    return e;
}

cudaError_t launch_modal(const Geom& g, const ModalConst* mc, const double2* q, double2* psi, cudaStream_t s) {
    const size_t P = (size_t)g.nkx * g.nky;
    dim3 grid((unsigned)((P + 255) / 256));
    const double nb = 2.0 * 16.0 * (double)g.csize();
    switch (g.nz) {
        case 2: QGN_LAUNCH(KID_MODAL, nb, s, k_modal<2><<<grid, 256, 0, s>>>(g, mc, q, psi)); break;
        case 4: QGN_LAUNCH(KID_MODAL, nb, s, k_modal<4><<<grid, 256, 0, s>>>(g, mc, q, psi)); break;
        case 8: QGN_LAUNCH(KID_MODAL, nb, s, k_modal<8><<<grid, 256, 0, s>>>(g, mc, q, psi)); break;
        case 16: QGN_LAUNCH(KID_MODAL, nb, s, k_modal<16><<<grid, 256, 0, s>>>(g, mc, q, psi)); break;
        default: QGN_LAUNCH(KID_MODAL, nb, s, k_modal<0><<<grid, 256, 0, s>>>(g, mc, q, psi)); break;
    }
    return cudaGetLastError();
}

template <class CT>
static cudaError_t launch_yinv(const Geom& g, int nf, const CT* q, const CT* psi, CT* hq, CT* hp, CT* hu, const CT* twy,
                               cudaStream_t s) {
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        using C = YInvCfg<NY, CT>;
        dim3 grid((g.nkx + C::TKX - 1) / C::TKX, g.nz);
        cudaError_t e;
        const double es = (double)sizeof(CT);
        const double Cb = es * (double)g.csize(), Hb = es * (double)g.nz * NY * g.nkx;
        if (nf == 3) {
            if ((e = set_smem(k_yinv<NY, 3, CT>, C::SMEM)) != cudaSuccess) return e;
            QGN_LAUNCH(KID_YINV, 2.0 * Cb + 3.0 * Hb, s,
                       k_yinv<NY, 3, CT><<<grid, C::THREADS, C::SMEM, s>>>(g, q, psi, hq, hp, hu, twy));
        } else {
            if ((e = set_smem(k_yinv<NY, 1, CT>, C::SMEM)) != cudaSuccess) return e;
            QGN_LAUNCH(KID_YINV, Cb + Hb, s,
                       k_yinv<NY, 1, CT><<<grid, C::THREADS, C::SMEM, s>>>(g, q, psi, hq, hp, hu, twy));
        }
        return cudaGetLastError();
    });
}

template <class CT>
static cudaError_t launch_xpass(const Geom& g, const CT* hq, const CT* hp, const CT* hu, CT* hpp, CT* hpd, const CT* twx,
                                bool drag, cudaStream_t s) {
    return dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        cudaError_t e;
        const double es = (double)sizeof(CT);
        const int nplain = drag ? g.nz - 1 : g.nz;
        if (nplain > 0) {
            using C = XCfg<NX, false, CT>;
            if ((e = set_smem(k_xpass<NX, false, CT>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, nplain);
            QGN_LAUNCH(KID_XPASS, 5.0 * es * (double)nplain * g.ny * g.nkx, s,
                       k_xpass<NX, false, CT><<<grid, C::THREADS, C::SMEM, s>>>(g, 0, hq, hp, hu, hpp, hpd, twx));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (drag) {
            using C = XCfg<NX, true, CT>;
            if ((e = set_smem(k_xpass<NX, true, CT>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, 1);
            QGN_LAUNCH(KID_XPASS, 7.0 * es * (double)g.ny * g.nkx, s,
                       k_xpass<NX, true, CT><<<grid, C::THREADS, C::SMEM, s>>>(g, g.nz - 1, hq, hp, hu, hpp, hpd,
                                                                                twx));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        return cudaSuccess;
    });
}

template <class CT>
static cudaError_t launch_yfwd(const Geom& g, const LayerConst* lc, const CT* q, const CT* psi, const CT* hpp,
                               const CT* hpd, CT* out, const CT* twy, bool drag, cudaStream_t s) {
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        cudaError_t e;
        const double es = (double)sizeof(CT);
        const int nplain = drag ? g.nz - 1 : g.nz;
        if (nplain > 0) {
            using C = YFwdCfg<NY, false, CT>;
            if ((e = set_smem(k_yfwd<NY, false, CT>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.nkx + C::TKX - 1) / C::TKX, nplain);
            const double lb = es * (double)nplain * g.nkx;
            QGN_LAUNCH(KID_YFWD, lb * (2.0 * NY + 3.0 * g.nky), s,
                       k_yfwd<NY, false, CT><<<grid, C::THREADS, C::SMEM, s>>>(g, 0, lc, q, psi, hpp, hpd, out, twy));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (drag) {
            using C = YFwdCfg<NY, true, CT>;
            if ((e = set_smem(k_yfwd<NY, true, CT>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.nkx + C::TKX - 1) / C::TKX, 1);
            const double lb = es * (double)g.nkx;
            QGN_LAUNCH(KID_YFWD, lb * (4.0 * NY + 3.0 * g.nky), s,
                       k_yfwd<NY, true, CT><<<grid, C::THREADS, C::SMEM, s>>>(g, g.nz - 1, lc, q, psi, hpp, hpd, out,
                                                                               twy));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        return cudaSuccess;
    });
}

cudaError_t launch_rhs(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                       bool do_drag, cudaStream_t s) {
    cudaError_t e;
    if ((e = launch_yinv<double2>(g, 3, q, psi, b.hq, b.hp, b.hu, b.twy, s)) != cudaSuccess) return e;
    if ((e = launch_xpass<double2>(g, b.hq, b.hp, b.hu, b.hpp, b.hpd, b.twx, do_drag, s)) != cudaSuccess) return e;
    return launch_yfwd<double2>(g, b.lc, q, psi, b.hpp, b.hpd, out, b.twy, do_drag, s);
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

template <int EPI>
static cudaError_t launch_xinv1(const Geom& g, const Buffers& b, DevScalars* sc, double* outp, cudaStream_t s) {
    return dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        using C = X1Cfg<NX>;
        cudaError_t e;
        if ((e = set_smem(k_xinv1<NX, EPI>, C::SMEM)) != cudaSuccess) return e;
        dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, g.nz);
        const double hb = 16.0 * (double)g.nz * g.ny * g.nkx;
        QGN_LAUNCH(KID_XINV1, hb + (EPI == 1 ? 8.0 * (double)g.nz * g.ny * NX : 0.0), s,
                   k_xinv1<NX, EPI><<<grid, C::THREADS, C::SMEM, s>>>(g, b.hq, sc, outp, b.twx));
        return cudaGetLastError();
    });
}

cudaError_t launch_maxabs_phys(const Geom& g, const Buffers& b, const double2* f, DevScalars* sc, cudaStream_t s) {
    cudaError_t e;
    if ((e = launch_yinv<double2>(g, 1, f, nullptr, b.hq, nullptr, nullptr, b.twy, s)) != cudaSuccess) return e;
    return launch_xinv1<0>(g, b, sc, nullptr, s);
}

cudaError_t launch_from_phys(const Geom& g, const Buffers& b, const double* phys, double2* out, cudaStream_t s) {
    cudaError_t e = dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        using C = X1Cfg<NX>;
        cudaError_t e2;
        if ((e2 = set_smem(k_xfwd1<NX>, C::SMEM)) != cudaSuccess) return e2;
        dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, g.nz);
        QGN_LAUNCH(KID_XFWD1, 8.0 * (double)g.nz * g.ny * NX + 16.0 * (double)g.nz * g.ny * g.nkx, s,
                   k_xfwd1<NX><<<grid, C::THREADS, C::SMEM, s>>>(g, phys, b.hq, b.twx));
        return cudaGetLastError();
    });
    if (e != cudaSuccess) return e;
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        using C = YInvCfg<NY>;
        cudaError_t e2;
        if ((e2 = set_smem(k_yfwd1<NY>, C::SMEM)) != cudaSuccess) return e2;
        dim3 grid((g.nkx + C::TKX - 1) / C::TKX, g.nz);
        QGN_LAUNCH(KID_YFWD1, 16.0 * (double)g.nz * g.nkx * (NY + g.nky), s,
                   k_yfwd1<NY><<<grid, C::THREADS, C::SMEM, s>>>(g, b.hq, out, b.twy));
        return cudaGetLastError();
    });
}

cudaError_t launch_to_phys(const Geom& g, const Buffers& b, const double2* f, double* out, cudaStream_t s) {
    cudaError_t e;
    if ((e = launch_yinv<double2>(g, 1, f, nullptr, b.hq, nullptr, nullptr, b.twy, s)) != cudaSuccess) return e;
    return launch_xinv1<1>(g, b, nullptr, out, s);
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
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const double qq = q[e];
        u[e] = u[e] * qq;     // u_phys*q_phys
        v[e] = v[e] * qq;     // v_phys*q_phys
    }
}

// jaco_hat = i kx uq_hat + i ky vq_hat on the full spectrum (QGN_Module.f90:244-247), in place into uq
__global__ void k_jac_full(Geom gf, double2* __restrict__ uq, const double2* __restrict__ vq) {
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
    if ((e = launch_modal(g, b.mc, q, b.psi, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_LAYOUT, 48.0 * (double)g.csize(), s, k_uv_hat<<<blocks, 256, 0, s>>>(g, b.psi, fa, fb));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, q, Pq, s)) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, fa, Pu, s)) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, fb, Pv, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_LAYOUT, 40.0 * (double)np, s, k_products<<<blocks, 256, 0, s>>>(np, Pq, Pu, Pv));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // full-spectrum r2c of u*q and v*q and the undealiased Jacobian (QGN_Module.f90:235-247)
    const Geom gf = full_geom(g);
    Buffers bf = b;
    bf.hq = full_half;
    if ((e = launch_from_phys(gf, bf, Pu, fa, s)) != cudaSuccess) return e;
    if ((e = launch_from_phys(gf, bf, Pv, fb, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_LAYOUT, 48.0 * (double)gf.csize(), s, k_jac_full<<<blocks, 256, 0, s>>>(gf, fa, fb));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // modal projections and their physical fields (QGN_Module.f90:390-415)
    QGN_LAUNCH(KID_MODAL, 32.0 * (double)gf.csize(), s, k_modal_proj<<<blocks, 256, 0, s>>>(gf, b.mc, fa, fb, nullptr));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_to_phys(gf, bf, fb, out_j, s)) != cudaSuccess) return e;
    QGN_LAUNCH(KID_MODAL, 48.0 * (double)g.csize(), s, k_modal_proj<<<blocks, 256, 0, s>>>(g, b.mc, q, fa, fb));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_to_phys(g, b, fa, out_q, s)) != cudaSuccess) return e;
    return launch_to_phys(g, b, fb, out_p, s);
}

}  // namespace qgn
