// rhs_kernels.cu -- the spectral right-hand side of QGN on sm_100a (FP64).
//
// One GetRHS (QGN_Module.f90:258-296) = GetPsi + Jacobian + linear terms + drag +
// DeAlias is evaluated as three streaming passes over HBM plus the modal inversion
// that the stage kernels fuse into their epilogue:
//
//   yinv  (per layer, per tile of kx columns)  compact q, psi -> y-inverse of q, psi, u=-i ky psi
//         written as half-transformed rows [nz][ny][nkxp]                     (3 inverse y FFTs)
//   xpass (per layer, per pair of rows y)       c2r of q1+iq2, u1+iu2, v1+iv2 (v = i kx psi),
//         products uq, vq (and |u|u, |u|v in the bottom layer), r2c of uq+ivq; keeps kx < nx/3
//   yfwd  (per layer, per tile of kx columns)  forward y FFT of uq, vq (and drag fields), then
//         J = i kx (uq)^ + i ky (vq)^ and RHS = -J - U i kx q - (beta+Qy) v + Ekman + drag,
//         written for the kept modes only (DeAlias is the storage format).
//
// The dealiased band (kx >= nx/3, ny/3 <= j <= 2(ny/3)) is never stored: inverse
// transforms see zeros there and forward transforms do not write it.
#include "qgn_internal.cuh"
#include "fft.cuh"
#include "prof.cuh"

#include <type_traits>

namespace qgn {

// ------------------------------------------------------------------------------------
// Tile shapes
// ------------------------------------------------------------------------------------
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }

// slot stride of a padded transform such that slot*stride spreads 16-byte bank groups
__host__ __device__ constexpr int slot_stride(int N, int target_mod8) {
    return fpadlen(N) + ((target_mod8 - (fpadlen(N) % 8)) + 8) % 8;
}

template <int NY>
struct YInvCfg {
    static constexpr int G = FFTShape<NY>::G;
    static constexpr int TKX = cmin(cmax(4, 128 / G), 64);
    static constexpr int THREADS = TKX * G;
    static constexpr int TS = slot_stride(NY, TKX >= 8 ? 1 : 8 / TKX);
    static constexpr int SMEM = TKX * TS * (int)sizeof(double2);
};

template <int NX, bool DRAG>
struct XCfg {
    static constexpr int G = FFTShape<NX>::G;
    static constexpr int RP = cmax(1, 64 / G);         // row pairs per CTA
    static constexpr int SP = DRAG ? 4 : 3;             // slots per row pair
    static constexpr int THREADS = SP * RP * G;
    static constexpr int TS = slot_stride(NX, 2);
    static constexpr int SMEM = SP * RP * TS * (int)sizeof(double2);
};

template <int NY, bool DRAG>
struct YFwdCfg {
    static constexpr int G = FFTShape<NY>::G;
    static constexpr int TKX = cmin(cmax(2, 64 / G), 32);
    static constexpr int SLOTS = 2 * TKX;
    static constexpr int THREADS = SLOTS * G;
    static constexpr int TS = slot_stride(NY, TKX >= 8 ? 1 : 8 / TKX);
    static constexpr int SMEM = SLOTS * TS * (int)sizeof(double2);
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
            double2 qm = make_double2(acc.x / Htot, acc.y / Htot);
            double den = -k2 + ev[k];
            pm[k] = mean_mode ? make_double2(0.0, 0.0) : make_double2(qm.x / den, qm.y / den);
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
__global__ void __launch_bounds__(256) k_modal(Geom g, const ModalConst* __restrict__ mc,
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
// yinv: inverse y transforms of kept columns into half-transformed rows.
// NF = 3: (q -> hq, psi -> hp, -i ky psi -> hu);  NF = 1: (f -> hq).
// ------------------------------------------------------------------------------------
template <int NY, int NF>
__global__ void __launch_bounds__(YInvCfg<NY>::THREADS) k_yinv(Geom g, const double2* __restrict__ q,
                                                               const double2* __restrict__ psi,
                                                               double2* __restrict__ hq, double2* __restrict__ hp,
                                                               double2* __restrict__ hu,
                                                               const double2* __restrict__ twy) {
    using C = YInvCfg<NY>;
    extern __shared__ double2 sm[];
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int kx0 = blockIdx.x * C::TKX;
    const int slot = tid / C::G, lane = tid % C::G;
    const size_t colbase = (size_t)l * g.nkx;
#pragma unroll 1
    for (int f = 0; f < NF; ++f) {
        const double2* src = (f == 0) ? q : psi;
        double2* dst = (f == 0) ? hq : (f == 1 ? hp : hu);
        for (int e = tid; e < C::TKX * NY; e += C::THREADS) {
            const int c = e / NY, j = e % NY;
            const int kx = kx0 + c;
            double2 v = make_double2(0.0, 0.0);
            const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
            if (kx < g.nkx && kept) {
                const int m = j < g.kylo ? j : j - g.kyshift;
                v = src[(colbase + kx) * g.nky + m];
                if (f == 2) {   // u_hat = -i ky psi_hat  (QGN_Module.f90:223)
                    const double kyv = g.kyval(j);
                    v = make_double2(kyv * v.y, -kyv * v.x);
                }
            }
            sm[c * C::TS + fpad(j)] = v;
        }
        __syncthreads();
        fft_block<NY, +1>(sm + slot * C::TS, lane, true, twy);
        for (int e = tid; e < C::TKX * NY; e += C::THREADS) {
            const int y = e / C::TKX, c = e % C::TKX;
            const int kx = kx0 + c;
            if (kx < g.nkxp) dst[((size_t)l * NY + y) * g.nkxp + kx] = sm[c * C::TS + fpad(y)];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------
// xpass: x transforms of row pairs.  c2r of q1 + i q2, u1 + i u2 and v1 + i v2 (Hermitian
// extension of the kept kx, Re of kx=0 as the c2r Hermitian projection), physical products,
// r2c of p = uq + i vq, split and truncated to kx < nx/3.
// ------------------------------------------------------------------------------------
template <int NX, bool DRAG>
__global__ void __launch_bounds__(XCfg<NX, DRAG>::THREADS) k_xpass(Geom g, int layer0,
                                                                   const double2* __restrict__ hq,
                                                                   const double2* __restrict__ hp,
                                                                   const double2* __restrict__ hu,
                                                                   double2* __restrict__ huq,
                                                                   double2* __restrict__ hvq,
                                                                   double2* __restrict__ hdu,
                                                                   double2* __restrict__ hdv,
                                                                   const double2* __restrict__ twx) {
    using C = XCfg<NX, DRAG>;
    extern __shared__ double2 sm[];
    const int tid = threadIdx.x;
    const int l = layer0 + blockIdx.y;
    const int rp0 = blockIdx.x * C::RP;
    const int npairs = g.ny / 2;
    const int nkx = g.nkx;
    // ---- load: Hermitian-extended spectra of the three complex signals per row pair
    for (int e = tid; e < C::RP * NX; e += C::THREADS) {
        const int r = e / NX, k = e % NX;
        const int rp = rp0 + r;
        if (rp >= npairs) continue;
        double2* base = sm + (r * C::SP) * C::TS;
        double2 a1 = make_double2(0.0, 0.0), a2 = a1, b = a1;
        const bool lo = k < nkx, hi = k > NX - nkx;
        if (lo || hi) {
            const int kk = lo ? k : NX - k;
            const size_t r1 = ((size_t)l * g.ny + 2 * rp) * g.nkxp + kk;
            const size_t r2 = r1 + g.nkxp;
            const double2 Q1 = hq[r1], Q2 = hq[r2], U1 = hu[r1], U2 = hu[r2];
            const double2 P1 = hp[r1], P2 = hp[r2];
            const double kxv = g.dkx * kk;
            const double2 V1 = make_double2(-kxv * P1.y, kxv * P1.x);   // v_hat = i kx psi_hat
            const double2 V2 = make_double2(-kxv * P2.y, kxv * P2.x);
            // pack two rows of the same field per complex transform: q1+iq2, u1+iu2, v1+iv2
            // (pairing fields of very different magnitude, e.g. q+iu, would leak the roundoff
            // of the larger one into the smaller one)
            if (k == 0) {
                a1 = make_double2(Q1.x, Q2.x);
                a2 = make_double2(U1.x, U2.x);
                b = make_double2(V1.x, V2.x);
            } else if (lo) {
                a1 = make_double2(Q1.x - Q2.y, Q1.y + Q2.x);
                a2 = make_double2(U1.x - U2.y, U1.y + U2.x);
                b = make_double2(V1.x - V2.y, V1.y + V2.x);
            } else {
                a1 = make_double2(Q1.x + Q2.y, Q2.x - Q1.y);
                a2 = make_double2(U1.x + U2.y, U2.x - U1.y);
                b = make_double2(V1.x + V2.y, V2.x - V1.y);
            }
        }
        base[fpad(k)] = a1;
        base[C::TS + fpad(k)] = a2;
        base[2 * C::TS + fpad(k)] = b;
    }
    __syncthreads();
    const int slot = tid / C::G, lane = tid % C::G;
    const int r_of = slot / C::SP, s_of = slot % C::SP;
    const bool pair_ok = (rp0 + r_of) < npairs;
    fft_block<NX, +1>(sm + slot * C::TS, lane, pair_ok && s_of < 3, twx);
    // ---- physical products (grid/(nx*ny) as in QGN_Module.f90:229-235)
    const double s = g.inv_nxny;
    for (int e = tid; e < C::RP * NX; e += C::THREADS) {
        const int r = e / NX, x = e % NX;
        if (rp0 + r >= npairs) continue;
        double2* base = sm + (r * C::SP) * C::TS;
        const double2 a1 = base[fpad(x)], a2 = base[C::TS + fpad(x)], b = base[2 * C::TS + fpad(x)];
        const double q1 = a1.x * s, q2 = a1.y * s, u1 = a2.x * s, u2 = a2.y * s;
        const double v1 = b.x * s, v2 = b.y * s;
        base[fpad(x)] = make_double2(u1 * q1, v1 * q1);
        base[C::TS + fpad(x)] = make_double2(u2 * q2, v2 * q2);
        if (DRAG) {   // URMS = sqrt(u^2+v^2), QGN_Module.f90:285
            const double m1 = sqrt(u1 * u1 + v1 * v1), m2 = sqrt(u2 * u2 + v2 * v2);
            base[2 * C::TS + fpad(x)] = make_double2(m1 * u1, m1 * v1);
            base[3 * C::TS + fpad(x)] = make_double2(m2 * u2, m2 * v2);
        }
    }
    __syncthreads();
    fft_block<NX, -1>(sm + slot * C::TS, lane, pair_ok && s_of < (DRAG ? 4 : 2), twx);
    // ---- split the packed real transforms and keep kx < nx/3
    for (int e = tid; e < C::RP * nkx; e += C::THREADS) {
        const int r = e / nkx, k = e % nkx;
        const int rp = rp0 + r;
        if (rp >= npairs) continue;
        const double2* base = sm + (r * C::SP) * C::TS;
        const int km = (NX - k) & (NX - 1);
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            const size_t row = ((size_t)l * g.ny + 2 * rp + w) * g.nkxp + k;
            const double2 X = base[w * C::TS + fpad(k)];
            const double2 Y = cconj(base[w * C::TS + fpad(km)]);
            huq[row] = make_double2(0.5 * (X.x + Y.x), 0.5 * (X.y + Y.y));
            hvq[row] = make_double2(0.5 * (X.y - Y.y), -0.5 * (X.x - Y.x));
            if (DRAG) {
                const size_t drow = (size_t)(2 * rp + w) * g.nkxp + k;
                const double2 Xd = base[(2 + w) * C::TS + fpad(k)];
                const double2 Yd = cconj(base[(2 + w) * C::TS + fpad(km)]);
                hdu[drow] = make_double2(0.5 * (Xd.x + Yd.x), 0.5 * (Xd.y + Yd.y));
                hdv[drow] = make_double2(0.5 * (Xd.y - Yd.y), -0.5 * (Xd.x - Yd.x));
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// yfwd: forward y transforms of uq, vq columns and assembly of the right-hand side.
// ------------------------------------------------------------------------------------
template <int NY, bool DRAG>
__global__ void __launch_bounds__(YFwdCfg<NY, DRAG>::THREADS) k_yfwd(Geom g, int layer0,
                                                                     const LayerConst* __restrict__ lc,
                                                                     const double2* __restrict__ q,
                                                                     const double2* __restrict__ psi,
                                                                     const double2* __restrict__ huq,
                                                                     const double2* __restrict__ hvq,
                                                                     const double2* __restrict__ hdu,
                                                                     const double2* __restrict__ hdv,
                                                                     double2* __restrict__ out,
                                                                     const double2* __restrict__ twy) {
    using C = YFwdCfg<NY, DRAG>;
    extern __shared__ double2 sm[];
    const int tid = threadIdx.x;
    const int l = layer0 + blockIdx.y;
    const int kx0 = blockIdx.x * C::TKX;
    const int slot = tid / C::G, lane = tid % C::G;
    const int nky = g.nky;
    const size_t colbase = (size_t)l * g.nkx;
    const bool bottom = (l == g.nz - 1);

    if (DRAG) {
        // drag_hat = i ky (|u|u)^ - i kx (|u|v)^ on the bottom layer (QGN_Module.f90:284-292)
        for (int e = tid; e < C::TKX * NY; e += C::THREADS) {
            const int y = e / C::TKX, c = e % C::TKX;
            const size_t src = (size_t)y * g.nkxp + kx0 + c;
            const bool ok = kx0 + c < g.nkx;
            sm[c * C::TS + fpad(y)] = ok ? hdu[src] : make_double2(0.0, 0.0);
            sm[(C::TKX + c) * C::TS + fpad(y)] = ok ? hdv[src] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        fft_block<NY, -1>(sm + slot * C::TS, lane, true, twy);
        const double dc = lc->dragc;
        for (int e = tid; e < C::TKX * nky; e += C::THREADS) {
            const int c = e / nky, m = e % nky;
            const int kx = kx0 + c;
            if (kx >= g.nkx) continue;
            const int j = g.jfull(m);
            const double kxv = g.dkx * kx, kyv = g.kyval(j);
            const double2 fu = sm[c * C::TS + fpad(j)], fv = sm[(C::TKX + c) * C::TS + fpad(j)];
            double2 d = make_double2(-kyv * fu.y, kyv * fu.x);        // i ky (|u|u)^
            d = make_double2(d.x + kxv * fv.y, d.y - kxv * fv.x);      // - i kx (|u|v)^
            out[(colbase + kx) * nky + m] = make_double2(dc * d.x, dc * d.y);
        }
        __syncthreads();
    }

    for (int e = tid; e < C::TKX * NY; e += C::THREADS) {
        const int y = e / C::TKX, c = e % C::TKX;
        const size_t src = ((size_t)l * NY + y) * g.nkxp + kx0 + c;
        const bool ok = kx0 + c < g.nkx;
        sm[c * C::TS + fpad(y)] = ok ? huq[src] : make_double2(0.0, 0.0);
        sm[(C::TKX + c) * C::TS + fpad(y)] = ok ? hvq[src] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    fft_block<NY, -1>(sm + slot * C::TS, lane, true, twy);

    const double ub = lc->uBar[l], bq = lc->betaq[l];
    const double ek = lc->ekman;
    const bool expl = lc->explicit_diss != 0;
    for (int e = tid; e < C::TKX * nky; e += C::THREADS) {
        const int c = e / nky, m = e % nky;
        const int kx = kx0 + c;
        if (kx >= g.nkx) continue;
        const int j = g.jfull(m);
        const double kxv = g.dkx * kx, kyv = g.kyval(j);
        const size_t idx = (colbase + kx) * nky + m;
        const double2 fuq = sm[c * C::TS + fpad(j)], fvq = sm[(C::TKX + c) * C::TS + fpad(j)];
        const double2 qv = q[idx], pv = psi[idx];
        // jaco_hat = i kx uq_hat + i ky vq_hat  (QGN_Module.f90:244-247)
        const double2 jac = make_double2(-kxv * fuq.y - kyv * fvq.y, kxv * fuq.x + kyv * fvq.x);
        double2 r = make_double2(-jac.x, -jac.y);
        // - uBar i kx q_hat - (beta+qyBar) v_hat   (QGN_Module.f90:270-273)
        const double uk = ub * kxv;
        const double2 vh = make_double2(-kxv * pv.y, kxv * pv.x);
        r = make_double2(r.x + uk * qv.y, r.y - uk * qv.x);
        r = make_double2(r.x - bq * vh.x, r.y - bq * vh.y);
        const double k2 = kxv * kxv + kyv * kyv;
        if (expl) {   // QGN_Module.f90:275-280
            const double k4 = k2 * k2, k8 = k4 * k4;
            const double dcoef = lc->A2 * k2 + lc->A8 * k8;
            r = make_double2(r.x - dcoef * qv.x, r.y - dcoef * qv.y);
        }
        if (bottom) {   // Ekman, QGN_Module.f90:282
            const double ekk = ek * k2;
            r = make_double2(r.x + ekk * pv.x, r.y + ekk * pv.y);
            if (DRAG) {
                const double2 d = out[idx];
                r = make_double2(r.x + d.x, r.y + d.y);
            }
        }
        if (kx == 0 && m == 0) r = make_double2(0.0, 0.0);
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
__global__ void __launch_bounds__(X1Cfg<NX>::THREADS) k_xinv1(Geom g, const double2* __restrict__ hq,
                                                              DevScalars* __restrict__ sc, double* __restrict__ outp,
                                                              const double2* __restrict__ twx) {
    using C = X1Cfg<NX>;
    extern __shared__ double2 sm[];
    __shared__ double smax[32];
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int rp0 = blockIdx.x * C::RP;
    const int npairs = g.ny / 2;
    const int nkx = g.nkx;
    for (int e = tid; e < C::RP * NX; e += C::THREADS) {
        const int r = e / NX, k = e % NX;
        const int rp = rp0 + r;
        if (rp >= npairs) continue;
        double2 a = make_double2(0.0, 0.0);
        const bool lo = k < nkx, hi = k > NX - nkx;
        if (lo || hi) {
            const int kk = lo ? k : NX - k;
            const size_t r1 = ((size_t)l * g.ny + 2 * rp) * g.nkxp + kk;
            const double2 F1 = hq[r1], F2 = hq[r1 + g.nkxp];
            if (k == 0) a = make_double2(F1.x, F2.x);
            else if (lo) a = make_double2(F1.x - F2.y, F1.y + F2.x);
            else a = make_double2(F1.x + F2.y, F2.x - F1.y);
        }
        sm[r * C::TS + fpad(k)] = a;
    }
    __syncthreads();
    const int slot = tid / C::G, lane = tid % C::G;
    fft_block<NX, +1>(sm + slot * C::TS, lane, (rp0 + slot) < npairs, twx);
    double mx = 0.0;
    for (int e = tid; e < C::RP * NX; e += C::THREADS) {
        const int r = e / NX, x = e % NX;
        const int rp = rp0 + r;
        if (rp >= npairs) continue;
        const double2 a = sm[r * C::TS + fpad(x)];
        if (EPI == 0) {
            // NaN propagates through fmax only if both are NaN; flag it explicitly
            const double m1 = fabs(a.x), m2 = fabs(a.y);
            if (!(m1 == m1) || !(m2 == m2)) mx = __longlong_as_double(0x7ff8000000000000ULL);
            else if (mx == mx) mx = fmax(mx, fmax(m1, m2));
        } else {
            const size_t row = ((size_t)l * g.ny + 2 * rp) * NX + x;
            outp[row] = a.x * g.inv_nxny;
            outp[row + NX] = a.y * g.inv_nxny;
        }
    }
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
__global__ void __launch_bounds__(X1Cfg<NX>::THREADS) k_xfwd1(Geom g, const double* __restrict__ phys,
                                                              double2* __restrict__ hq,
                                                              const double2* __restrict__ twx) {
    using C = X1Cfg<NX>;
    extern __shared__ double2 sm[];
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int rp0 = blockIdx.x * C::RP;
    const int npairs = g.ny / 2;
    for (int e = tid; e < C::RP * NX; e += C::THREADS) {
        const int r = e / NX, x = e % NX;
        const int rp = rp0 + r;
        if (rp >= npairs) continue;
        const size_t row = ((size_t)l * g.ny + 2 * rp) * NX + x;
        sm[r * C::TS + fpad(x)] = make_double2(phys[row], phys[row + NX]);
    }
    __syncthreads();
    const int slot = tid / C::G, lane = tid % C::G;
    fft_block<NX, -1>(sm + slot * C::TS, lane, (rp0 + slot) < npairs, twx);
    const int nkx = g.nkx;
    for (int e = tid; e < C::RP * nkx; e += C::THREADS) {
        const int r = e / nkx, k = e % nkx;
        const int rp = rp0 + r;
        if (rp >= npairs) continue;
        const double2 X = sm[r * C::TS + fpad(k)];
        const double2 Y = cconj(sm[r * C::TS + fpad((NX - k) & (NX - 1))]);
        const size_t row = ((size_t)l * g.ny + 2 * rp) * g.nkxp + k;
        hq[row] = make_double2(0.5 * (X.x + Y.x), 0.5 * (X.y + Y.y));
        hq[row + g.nkxp] = make_double2(0.5 * (X.y - Y.y), -0.5 * (X.x - Y.x));
    }
}

template <int NY>
__global__ void __launch_bounds__(YInvCfg<NY>::THREADS) k_yfwd1(Geom g, const double2* __restrict__ hq,
                                                                double2* __restrict__ out,
                                                                const double2* __restrict__ twy) {
    using C = YInvCfg<NY>;
    extern __shared__ double2 sm[];
    const int tid = threadIdx.x;
    const int l = blockIdx.y;
    const int kx0 = blockIdx.x * C::TKX;
    const int slot = tid / C::G, lane = tid % C::G;
    for (int e = tid; e < C::TKX * NY; e += C::THREADS) {
        const int y = e / C::TKX, c = e % C::TKX;
        const bool ok = kx0 + c < g.nkx;
        sm[c * C::TS + fpad(y)] = ok ? hq[((size_t)l * NY + y) * g.nkxp + kx0 + c] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    fft_block<NY, -1>(sm + slot * C::TS, lane, true, twy);
    const int nky = g.nky;
    for (int e = tid; e < C::TKX * nky; e += C::THREADS) {
        const int c = e / nky, m = e % nky;
        const int kx = kx0 + c;
        if (kx >= g.nkx) continue;
        double2 v = sm[c * C::TS + fpad(g.jfull(m))];
        if (kx == 0 && m == 0) v = make_double2(0.0, 0.0);
        out[((size_t)l * g.nkx + kx) * nky + m] = v;
    }
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

template <class K>
static cudaError_t set_smem(K kernel, int bytes) {
    if (bytes > 48 * 1024) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return cudaSuccess;
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

static cudaError_t launch_yinv(const Geom& g, int nf, const double2* q, const double2* psi, double2* hq,
                               double2* hp, double2* hu, const double2* twy, cudaStream_t s) {
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        using C = YInvCfg<NY>;
        dim3 grid((g.nkx + C::TKX - 1) / C::TKX, g.nz);
        cudaError_t e;
        const double Cb = 16.0 * (double)g.csize(), Hb = 16.0 * (double)g.nz * NY * g.nkx;
        if (nf == 3) {
            if ((e = set_smem(k_yinv<NY, 3>, C::SMEM)) != cudaSuccess) return e;
            QGN_LAUNCH(KID_YINV, 2.0 * Cb + 3.0 * Hb, s,
                       k_yinv<NY, 3><<<grid, C::THREADS, C::SMEM, s>>>(g, q, psi, hq, hp, hu, twy));
        } else {
            if ((e = set_smem(k_yinv<NY, 1>, C::SMEM)) != cudaSuccess) return e;
            QGN_LAUNCH(KID_YINV, Cb + Hb, s,
                       k_yinv<NY, 1><<<grid, C::THREADS, C::SMEM, s>>>(g, q, psi, hq, hp, hu, twy));
        }
        return cudaGetLastError();
    });
}

static cudaError_t launch_xpass(const Geom& g, const Buffers& b, bool drag, cudaStream_t s) {
    return dispatch_n(g.nx, [&](auto NXc) -> cudaError_t {
        constexpr int NX = decltype(NXc)::value;
        cudaError_t e;
        const int nplain = drag ? g.nz - 1 : g.nz;
        if (nplain > 0) {
            using C = XCfg<NX, false>;
            if ((e = set_smem(k_xpass<NX, false>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, nplain);
            QGN_LAUNCH(KID_XPASS, 5.0 * 16.0 * (double)nplain * g.ny * g.nkx, s,
                       k_xpass<NX, false><<<grid, C::THREADS, C::SMEM, s>>>(g, 0, b.hq, b.hp, b.hu, b.huq, b.hvq,
                                                                             b.hdu, b.hdv, b.twx));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (drag) {
            using C = XCfg<NX, true>;
            if ((e = set_smem(k_xpass<NX, true>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.ny / 2 + C::RP - 1) / C::RP, 1);
            QGN_LAUNCH(KID_XPASS, 7.0 * 16.0 * (double)g.ny * g.nkx, s,
                       k_xpass<NX, true><<<grid, C::THREADS, C::SMEM, s>>>(g, g.nz - 1, b.hq, b.hp, b.hu, b.huq,
                                                                            b.hvq, b.hdu, b.hdv, b.twx));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        return cudaSuccess;
    });
}

static cudaError_t launch_yfwd(const Geom& g, const Buffers& b, const double2* q, const double2* psi,
                               double2* out, bool drag, cudaStream_t s) {
    return dispatch_n(g.ny, [&](auto NYc) -> cudaError_t {
        constexpr int NY = decltype(NYc)::value;
        cudaError_t e;
        const int nplain = drag ? g.nz - 1 : g.nz;
        if (nplain > 0) {
            using C = YFwdCfg<NY, false>;
            if ((e = set_smem(k_yfwd<NY, false>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.nkx + C::TKX - 1) / C::TKX, nplain);
            const double lb = 16.0 * (double)nplain * g.nkx;
            QGN_LAUNCH(KID_YFWD, lb * (2.0 * NY + 3.0 * g.nky), s,
                       k_yfwd<NY, false><<<grid, C::THREADS, C::SMEM, s>>>(g, 0, b.lc, q, psi, b.huq, b.hvq, b.hdu,
                                                                            b.hdv, out, b.twy));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        if (drag) {
            using C = YFwdCfg<NY, true>;
            if ((e = set_smem(k_yfwd<NY, true>, C::SMEM)) != cudaSuccess) return e;
            dim3 grid((g.nkx + C::TKX - 1) / C::TKX, 1);
            const double lb = 16.0 * (double)g.nkx;
            QGN_LAUNCH(KID_YFWD, lb * (4.0 * NY + 3.0 * g.nky), s,
                       k_yfwd<NY, true><<<grid, C::THREADS, C::SMEM, s>>>(g, g.nz - 1, b.lc, q, psi, b.huq, b.hvq,
                                                                           b.hdu, b.hdv, out, b.twy));
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        return cudaSuccess;
    });
}

cudaError_t launch_rhs(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                       bool do_drag, cudaStream_t s) {
    cudaError_t e;
    if ((e = launch_yinv(g, 3, q, psi, b.hq, b.hp, b.hu, b.twy, s)) != cudaSuccess) return e;
    if ((e = launch_xpass(g, b, do_drag, s)) != cudaSuccess) return e;
    return launch_yfwd(g, b, q, psi, out, do_drag, s);
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
    if ((e = launch_yinv(g, 1, f, nullptr, b.hq, nullptr, nullptr, b.twy, s)) != cudaSuccess) return e;
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
    if ((e = launch_yinv(g, 1, f, nullptr, b.hq, nullptr, nullptr, b.twy, s)) != cudaSuccess) return e;
    return launch_xinv1<1>(g, b, nullptr, out, s);
}

}  // namespace qgn
