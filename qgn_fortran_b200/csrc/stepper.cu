// stepper.cu -- stage combinations, implicit solve, QG-Leith, error norm and PI controllers.
//
// The ARK4(3)6L[2]SA stage kernel fuses, per kept mode and for all layers at once:
//   L_j = -(A2 k^2 + A8L_k k^8) q_j                        (ARK43_QGLeith.f90:77-118)
//   q_s = Mq (q + dt (sum_j ae_sj N_j + sum_j ai_sj L_j)),  Mq = 1/(1 + dt/4 (A2 k^2 + A8L_k k^8))
//   psi_s = GetPsi(q_s)                                     (QGN_Module.f90:315-341)
// so the next RHS starts from q_s and psi_s without another pass.  L_j is recomputed from
// the stored stage state q_j instead of being stored.  dt, t and the controller memory live
// in device scalars so a whole step can be replayed without host round trips.
#include "qgn_internal.cuh"
#include "prof.cuh"
#include "ctrl.cuh"
#include "rhs_tiles.cuh"

#include <cstdlib>
#include <mutex>
#include <unordered_set>

namespace qgn {

// ARK4(3)6L[2]SA tableau, ARK43_QGLeith.f90:18-58 (exact rationals rounded once).
__constant__ double c_ae[36] = {
    0, 0, 0, 0, 0, 0,
    0.5, 0, 0, 0, 0, 0,
    13861.0 / 62500.0, 6889.0 / 62500.0, 0, 0, 0, 0,
    -116923316275.0 / 2393684061468.0, -2731218467317.0 / 15368042101831.0, 9408046702089.0 / 11113171139209.0, 0, 0, 0,
    -451086348788.0 / 2902428689909.0, -2682348792572.0 / 7519795681897.0, 12662868775082.0 / 11960479115383.0,
    3355817975965.0 / 11060851509271.0, 0, 0,
    647845179188.0 / 3216320057751.0, 73281519250.0 / 8382639484533.0, 552539513391.0 / 3454668386233.0,
    3354512671639.0 / 8306763924573.0, 4040.0 / 17871.0, 0};
__constant__ double c_ai[36] = {
    0, 0, 0, 0, 0, 0,
    0.25, 0.25, 0, 0, 0, 0,
    8611.0 / 62500.0, -1743.0 / 31250.0, 0, 0, 0, 0,
    5012029.0 / 34652500.0, -654441.0 / 2922500.0, 174375.0 / 388108.0, 0, 0, 0,
    15267082809.0 / 155376265600.0, -71443401.0 / 120774400.0, 730878875.0 / 902184768.0, 2285395.0 / 8070912.0, 0, 0,
    82889.0 / 524892.0, 0.0, 15625.0 / 83664.0, 69875.0 / 102672.0, -2260.0 / 8211.0, 0.25};
__constant__ double c_b[6] = {82889.0 / 524892.0, 0.0, 15625.0 / 83664.0, 69875.0 / 102672.0, -2260.0 / 8211.0, 0.25};
__constant__ double c_be[6] = {31666707.0 / 9881966720.0, 0.0, -256875.0 / 105007616.0, -2768025.0 / 128864768.0,
                               169839.0 / 3864644.0, -5247.0 / 225920.0};

template <int NZ>
__device__ __forceinline__ void modal_invert_s(const double* proj, const double* back, const double* ev, double Htot,
                                               int nz, double k2, bool mean_mode, const double2* qv, double2* pv) {
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    const int n = NZ > 0 ? NZ : nz;
    double2 pm[NZC];
#pragma unroll
    for (int k = 0; k < NZC; ++k) {
        if (k < n) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int kk = 0; kk < NZC; ++kk)
                if (kk < n) {
                    const double c = proj[k * n + kk];
                    acc.x += c * qv[kk].x;
                    acc.y += c * qv[kk].y;
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
            for (int kk = 0; kk < NZC; ++kk)
                if (kk < n) {
                    const double c = back[k * n + kk];
                    acc.x += pm[kk].x * c;
                    acc.y += pm[kk].y * c;
                }
            pv[k] = acc;
        }
    }
}

struct StagePtrs {
    const double2* N[6];
    const double2* Qs[6];
};

__device__ __forceinline__ void point_k(const Geom& g, size_t p, int& kx, int& m, double& k2) {
    kx = (int)(p / g.nky);
    m = (int)(p % g.nky);
    const double kxv = g.dkx * kx, kyv = g.kyval(g.jfull(m));
    k2 = kxv * kxv + kyv * kyv;
}

// ---- ARK update + embedded error combination (ARK43_QGLeith.f90:120-134) ---------------------
// It also clears the scalars of the error transform's max reduction that follows it.
__global__ void __launch_bounds__(256) k_ark_update(Geom g, StagePtrs sp, const double2* __restrict__ q,
                                                    double2* __restrict__ qnew, double2* __restrict__ err,
                                                    const LayerConst* __restrict__ lc,
                                                    DevScalars* __restrict__ sc) {
    QGN_PDL_ENTRY();
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t total = P * g.nz;
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e == 0) {
        sc->maxbits = 0ULL;
        sc->accept = 0;
    }
    if (e >= total) return;
    const int l = (int)(e / P);
    const size_t p = e % P;
    int kx, m;
    double k2;
    point_k(g, p, kx, m, k2);
    const double k8 = (k2 * k2) * (k2 * k2);
    const double D = lc->A2 * k2 + sc->A8L[l] * k8;
    const double dt = sc->dt;
    double2 ec = make_double2(0.0, 0.0), uc = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        if (i == 1) continue;   // b(2) = be(2) = 0
        const double2 n = sp.N[i][e];
        const double2 qi = sp.Qs[i][e];
        const double2 nl = make_double2(n.x + (-D * qi.x), n.y + (-D * qi.y));
        ec.x += c_be[i] * nl.x;
        ec.y += c_be[i] * nl.y;
        uc.x += c_b[i] * nl.x;
        uc.y += c_b[i] * nl.y;
    }
    err[e] = ec;
    const double2 q0 = q[e];
    qnew[e] = (p == 0) ? make_double2(0.0, 0.0) : make_double2(q0.x + dt * uc.x, q0.y + dt * uc.y);
}

// ---- mixed precision (QGN_PREC_MIXED) ----------------------------------------------------------
// Stage values N_j and q_j are stored in FP32.  The stage sums
//   sum_j ae_sj N_j + sum_j ai_sj L_j
// are formed in FP32 with Kahan-compensated summation (tableau coefficients rounded to FP32);
// the FP64 term L_1 = -D q_hat enters as its FP32 head plus its FP32 remainder.
// q_s = Mq (q_hat + dt * sum) is formed in FP64 from the compensated sum, GetPsi runs in FP64,
// and q_s, psi_s are stored in FP32.
struct Comp32 {
    float s = 0.f, c = 0.f;     // running sum and the negated lost low part
    __device__ __forceinline__ void add(float x) {
        const float y = __fsub_rn(x, c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

__device__ __forceinline__ void comp_add_prod(Comp32& acc, double a, float v) { acc.add(__fmul_rn((float)a, v)); }
__device__ __forceinline__ void comp_add_double(Comp32& acc, double x) {
    const float hi = (float)x;
    acc.add(hi);
    acc.add((float)(x - (double)hi));
}

// ---- ARK stage s as two streaming kernels ------------------------------------------------------
// k_ark_comb: one thread per (layer, mode): q_s = Mq (q + dt (sum ae N_j + sum ai L_j)), the
// sums in FP64 (FP64 storage) or Kahan-compensated FP32 (FP32 storage, mixed mode), q in FP64.
// GetPsi of q_s follows as a separate all-layers kernel (k_modal / k_modal_f32).
template <class T> struct StoreT;
template <> struct StoreT<double2> {
    __device__ static double2 put(double x, double y) { return make_double2(x, y); }
};
template <> struct StoreT<float2> {
    __device__ static float2 put(double x, double y) { return make_float2((float)x, (float)y); }
};

template <class T>
struct CombPtrs {
    const T* N[6];
    const T* Q[6];
};

// sum_j ae_sj N_j + sum_j ai_sj L_j with L_j = -D q_j, in FP64 (stage S of ARK43_QGLeith.f90:87-118)
template <int S>
__device__ __forceinline__ void comb_sum64(const double2* nn, const double2* qq, double2 q0, double D, double& ax,
                                           double& ay) {
    ax = 0.0;
    ay = 0.0;
#pragma unroll
    for (int j = 0; j < S; ++j) {
        ax += c_ae[S * 6 + j] * nn[j].x;
        ay += c_ae[S * 6 + j] * nn[j].y;
    }
    ax += c_ai[S * 6] * (-D * q0.x);
    ay += c_ai[S * 6] * (-D * q0.y);
#pragma unroll
    for (int j = 1; j < S; ++j) {
        ax += c_ai[S * 6 + j] * (-D * qq[j].x);
        ay += c_ai[S * 6 + j] * (-D * qq[j].y);
    }
}

template <int S, class T>
__global__ void __launch_bounds__(256) k_ark_comb(Geom g, CombPtrs<T> cp, const double2* __restrict__ q,
                                                  T* __restrict__ qout, const LayerConst* __restrict__ lc,
                                                  const DevScalars* __restrict__ sc) {
    QGN_PDL_ENTRY();
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t total = P * g.nz;
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int l = (int)(e / P);
    const size_t p = e % P;
    int kx, m;
    double k2;
    point_k(g, p, kx, m, k2);
    const double k8 = (k2 * k2) * (k2 * k2);
    const double D = lc->A2 * k2 + sc->A8L[l] * k8;
    const double dt = sc->dt;
    T nn[S], qq[S];
#pragma unroll
    for (int j = 0; j < S; ++j) nn[j] = cp.N[j][e];
#pragma unroll
    for (int j = 1; j < S; ++j) qq[j] = cp.Q[j][e];
    const double2 q0 = q[e];
    double ax, ay;
    if constexpr (sizeof(T) == 16) {
        comb_sum64<S>(nn, qq, q0, D, ax, ay);
    } else {
        Comp32 cx, cy;
        const float Df = (float)D;
#pragma unroll
        for (int j = 0; j < S; ++j) {
            comp_add_prod(cx, c_ae[S * 6 + j], nn[j].x);
            comp_add_prod(cy, c_ae[S * 6 + j], nn[j].y);
        }
        comp_add_double(cx, c_ai[S * 6] * (-D * q0.x));   // L_1 from the FP64 state
        comp_add_double(cy, c_ai[S * 6] * (-D * q0.y));
#pragma unroll
        for (int j = 1; j < S; ++j) {
            comp_add_prod(cx, c_ai[S * 6 + j], -Df * qq[j].x);
            comp_add_prod(cy, c_ai[S * 6 + j], -Df * qq[j].y);
        }
        ax = cx.value();
        ay = cy.value();
    }
    const double Mq = 1.0 / (1.0 + 0.25 * dt * D);
    qout[e] = StoreT<T>::put(Mq * (q0.x + dt * ax), Mq * (q0.y + dt * ay));
}

// GetPsi of an FP32 field with FP64 arithmetic (mixed mode)
template <int NZ>
__global__ void __launch_bounds__(256, 2) k_modal_f32(Geom g, const __grid_constant__ ModalArg<NZ> ma,
                                                      const float2* __restrict__ q, float2* __restrict__ psi) {
    QGN_PDL_ENTRY();
    QGN_MODAL_SHARED(NZ);
    const int nz = g.nz;
    const ModalView mv = modal_view<NZ>(ma, s_proj, s_back, s_ev, nz);
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    int kx, m;
    double k2;
    point_k(g, p, kx, m, k2);
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    double2 qv[NZC], pv[NZC];
#pragma unroll
    for (int l = 0; l < NZC; ++l)
        if (l < nz) {
            const float2 v = q[(size_t)l * P + p];
            qv[l] = make_double2(v.x, v.y);
        }
    modal_invert_s<NZ>(mv.proj, mv.back, mv.ev, mv.Htot, nz, k2, p == 0, qv, pv);
#pragma unroll
    for (int l = 0; l < NZC; ++l)
        if (l < nz) psi[(size_t)l * P + p] = make_float2((float)pv[l].x, (float)pv[l].y);
}


struct StagePtrs32 {
    const float2* N[6];
    const float2* Qs[6];
};

// update + embedded error in FP64 from FP32 stage values (ARK43_QGLeith.f90:120-134)
__global__ void __launch_bounds__(256) k_ark_update_mixed(Geom g, StagePtrs32 sp, const double2* __restrict__ q,
                                                          double2* __restrict__ qnew, float2* __restrict__ err,
                                                          const LayerConst* __restrict__ lc,
                                                          DevScalars* __restrict__ sc) {
    QGN_PDL_ENTRY();
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t total = P * g.nz;
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e == 0) {   // clears the max reduction of the error transform that follows
        sc->maxbits = 0ULL;
        sc->accept = 0;
    }
    if (e >= total) return;
    const int l = (int)(e / P);
    const size_t p = e % P;
    int kx, m;
    double k2;
    point_k(g, p, kx, m, k2);
    const double k8 = (k2 * k2) * (k2 * k2);
    const double D = lc->A2 * k2 + sc->A8L[l] * k8;
    const double dt = sc->dt;
    const double2 q0 = q[e];
    double2 ec = make_double2(0.0, 0.0), uc = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        if (i == 1) continue;   // b(2) = be(2) = 0
        const float2 n = sp.N[i][e];
        double qx, qy;
        if (i == 0) { qx = q0.x; qy = q0.y; }
        else { const float2 qi = sp.Qs[i][e]; qx = qi.x; qy = qi.y; }
        const double nlx = (double)n.x + (-D * qx), nly = (double)n.y + (-D * qy);
        ec.x += c_be[i] * nlx;
        ec.y += c_be[i] * nly;
        uc.x += c_b[i] * nlx;
        uc.y += c_b[i] * nly;
    }
    err[e] = make_float2((float)ec.x, (float)ec.y);   // its norm is taken with FP32 transforms
    qnew[e] = (p == 0) ? make_double2(0.0, 0.0) : make_double2(q0.x + dt * uc.x, q0.y + dt * uc.y);
}

// FP32 copy of the FP64 state and its GetPsi (FP64 arithmetic, FP32 result)
template <int NZ>
__global__ void __launch_bounds__(256, 2) k_modal_mixed(Geom g, const __grid_constant__ ModalArg<NZ> ma,
                                                     const double2* __restrict__ q, float2* __restrict__ q32,
                                                     float2* __restrict__ psi32) {
    QGN_PDL_ENTRY();
    QGN_MODAL_SHARED(NZ);
    const int nz = g.nz;
    const ModalView mv = modal_view<NZ>(ma, s_proj, s_back, s_ev, nz);
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    int kx, m;
    double k2;
    point_k(g, p, kx, m, k2);
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    double2 qv[NZC], pv[NZC];
#pragma unroll
    for (int l = 0; l < NZC; ++l)
        if (l < nz) qv[l] = q[(size_t)l * P + p];
    modal_invert_s<NZ>(mv.proj, mv.back, mv.ev, mv.Htot, nz, k2, p == 0, qv, pv);
#pragma unroll
    for (int l = 0; l < NZC; ++l) {
        if (l < nz) {
            q32[(size_t)l * P + p] = make_float2((float)qv[l].x, (float)qv[l].y);
            psi32[(size_t)l * P + p] = make_float2((float)pv[l].x, (float)pv[l].y);
        }
    }
}

__global__ void k_f2d(size_t n, const float2* __restrict__ a, double2* __restrict__ b) {
    QGN_PDL_ENTRY();
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) b[e] = make_double2(a[e].x, a[e].y);
}

// ---- explicit combinations: out = q + sum_j (a_j dt) R_j, then optionally psi = GetPsi(out) ---
template <int NZ>
__global__ void __launch_bounds__(256, 2) k_combo(Geom g, Combo cb, const double2* __restrict__ q,
                                               double2* __restrict__ out, double2* __restrict__ psi,
                                               const __grid_constant__ ModalArg<NZ> ma,
                                               const DevScalars* __restrict__ sc, int want_psi) {
    QGN_PDL_ENTRY();
    QGN_MODAL_SHARED(NZ);
    const int nz = g.nz;
    const ModalView mv = modal_view<NZ>(ma, s_proj, s_back, s_ev, nz);
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    int kx, m;
    double k2;
    point_k(g, p, kx, m, k2);
    const double dt = sc->dt;
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    double2 qv[NZC], pv[NZC];
#pragma unroll
    for (int l = 0; l < NZC; ++l) {
        if (l < nz) {
            const size_t idx = (size_t)l * P + p;
            double2 v = q[idx];
            for (int j = 0; j < cb.n; ++j) {
                const double c = cb.a[j] * dt;
                const double2 r = cb.R[j][idx];
                v.x += c * r.x;
                v.y += c * r.y;
            }
            qv[l] = v;
        }
    }
    if (want_psi) modal_invert_s<NZ>(mv.proj, mv.back, mv.ev, mv.Htot, nz, k2, p == 0, qv, pv);
#pragma unroll
    for (int l = 0; l < NZC; ++l) {
        if (l < nz) {
            out[(size_t)l * P + p] = qv[l];
            if (want_psi) psi[(size_t)l * P + p] = pv[l];
        }
    }
}

// ---- linear combination without q: out = sum_j a_j R_j (error spectra) --------------------
__global__ void k_lincomb(size_t n, Combo cb, double2* __restrict__ out) {
    QGN_PDL_ENTRY();
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double2 v = make_double2(0.0, 0.0);
    for (int j = 0; j < cb.n; ++j) {
        const double2 r = cb.R[j][e];
        v.x += cb.a[j] * r.x;
        v.y += cb.a[j] * r.y;
    }
    out[e] = v;
}

// ---- weighted Parseval sums over the full plane, per layer ------------------------------------
// sum_k w(k) |F_k|^2 with the Hermitian extension of the kept half plane; the kx=0 column
// uses the Hermitian projection (f(ky) + conj f(-ky))/2 that the reference's c2r applies.
// POW selects the weight (k^2)^POW.
template <int POW>
__device__ __forceinline__ double kpow(double k2) {
    if (POW == 1) return k2;
    const double k4 = k2 * k2;
    return k4 * k4;
}

template <int POW>
__device__ __forceinline__ double parseval_block(const Geom& g, const double2* __restrict__ f, int l);

template <int POW>
__global__ void __launch_bounds__(256) k_parseval(Geom g, const double2* __restrict__ f, double* __restrict__ partial) {
    QGN_PDL_ENTRY();
    const double t = parseval_block<POW>(g, f, blockIdx.y);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
}

// this block's share of sum_k w(k)|F_k|^2 for layer l (valid in thread 0)
template <int POW>
__device__ __forceinline__ double parseval_block(const Geom& g, const double2* __restrict__ f, int l) {
    __shared__ double red[8];
    const size_t P = (size_t)g.nkx * g.nky;
    double acc = 0.0;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (size_t)gridDim.x * blockDim.x) {
        int kx, m;
        double k2;
        point_k(g, p, kx, m, k2);
        const double w = kpow<POW>(k2);
        const double2 v = f[(size_t)l * P + p];
        if (kx > 0) {
            acc += 2.0 * w * (v.x * v.x + v.y * v.y);
        } else {
            const int j = g.jfull(m);
            const int jp = (g.ny - j) % g.ny;
            const bool pk = (jp < g.kylo) || (jp >= g.kylo + g.kyshift);
            double2 fp = make_double2(0.0, 0.0);
            if (pk) fp = f[(size_t)l * P + (jp < g.kylo ? jp : jp - g.kyshift)];
            const double hx = 0.5 * (v.x + fp.x), hy = 0.5 * (v.y - fp.y);
            acc += (pk ? 1.0 : 2.0) * w * (hx * hx + hy * hy);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    return t;
}

// warp-parallel fixed-order sum of one layer's partials (deterministic)
__device__ __forceinline__ double layer_sum(const double* __restrict__ partial, int l, int nblocks) {
    double s = 0.0;
    for (int b = threadIdx.x & 31; b < nblocks; b += 32) s += partial[(size_t)l * nblocks + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// QG-Leith in one launch, A8L(k) = (1.3*Lx/(nx*pi))**12 * sqrt(mean(q*d)) with
// mean(q*d) = S/(nx ny)^2 (ARK43_QGLeith.f90:71-73): each block writes its Parseval partial;
// the block that finishes last (counted in sc->red_count, reset to 0 after) sums the
// partials of every layer in a fixed order (deterministic) and writes A8L.
__global__ void __launch_bounds__(256) k_leith(Geom g, const double2* __restrict__ f, double* __restrict__ partial,
                                               double c12, DevScalars* __restrict__ sc) {
    QGN_PDL_ENTRY();
    __shared__ unsigned s_last;
    const int nb = gridDim.x;
    const double t = parseval_block<4>(g, f, blockIdx.y);
    if (threadIdx.x == 0) {
        partial[(size_t)blockIdx.y * nb + blockIdx.x] = t;
        __threadfence();
        const unsigned prev = atomicAdd(&sc->red_count, 1u);
        s_last = (prev + 1 == gridDim.x * gridDim.y) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const double N = (double)g.nx * (double)g.ny;
    for (int l = threadIdx.x >> 5; l < g.nz; l += blockDim.x >> 5) {
        double s = 0.0;
        for (int b = threadIdx.x & 31; b < nb; b += 32) s += __ldcg(&partial[(size_t)l * nb + b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) sc->A8L[l] = c12 * sqrt((s / N) / N);
    }
    if (threadIdx.x == 0) sc->red_count = 0u;
}


// layer KE = 0.5 * S/(nx ny)^2 * H_k/Htot with S the k^2-weighted Parseval sum of psi
__global__ void k_ke_final(Geom g, const double* __restrict__ partial, int nblocks, const double* __restrict__ Hw,
                           double* __restrict__ ke) {
    QGN_PDL_ENTRY();
    const int l = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (l >= g.nz) return;
    const double s = layer_sum(partial, l, nblocks);
    const double N = (double)g.nx * (double)g.ny;
    if ((threadIdx.x & 31) == 0) ke[l] = 0.5 * ((s / N) / N) * Hw[l];
}

// Energetics of the state, per layer (block partials, one (block, layer) per CTA): Parseval sums
// over the full plane of 0: k^2 |psi|^2 (kinetic energy), 1: -Re(conj(psi) (q + k^2 psi)) (the
// available potential energy: q_hat + k^2 psi_hat is the stretching term (L psi)^ of
// [Del + L] psi = q, QGN_Module.f90:100-112), 2: |q|^2 (enstrophy).  The kx = 0 column uses the
// Hermitian projections of both fields, as the reference's c2r does.
__global__ void __launch_bounds__(256) k_energetics(Geom g, const double2* __restrict__ q,
                                                    const double2* __restrict__ psi, double* __restrict__ partial) {
    QGN_PDL_ENTRY();
    __shared__ double red[3][8];
    const size_t P = (size_t)g.nkx * g.nky;
    const int l = blockIdx.y;
    double a[3] = {0.0, 0.0, 0.0};
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (size_t)gridDim.x * blockDim.x) {
        int kx, m;
        double k2;
        point_k(g, p, kx, m, k2);
        double2 hp = psi[(size_t)l * P + p], hq = q[(size_t)l * P + p];
        double w = 2.0;
        if (kx == 0) {
            const int j = g.jfull(m);
            const int jp = (g.ny - j) % g.ny;
            const bool pk = (jp < g.kylo) || (jp >= g.kylo + g.kyshift);
            double2 fp = make_double2(0.0, 0.0), fq = make_double2(0.0, 0.0);
            if (pk) {
                const size_t pp = (size_t)l * P + (jp < g.kylo ? jp : jp - g.kyshift);
                fp = psi[pp];
                fq = q[pp];
            }
            hp = make_double2(0.5 * (hp.x + fp.x), 0.5 * (hp.y - fp.y));
            hq = make_double2(0.5 * (hq.x + fq.x), 0.5 * (hq.y - fq.y));
            w = pk ? 1.0 : 2.0;
        }
        a[0] += w * k2 * (hp.x * hp.x + hp.y * hp.y);
        a[1] -= w * (hp.x * (hq.x + k2 * hp.x) + hp.y * (hq.y + k2 * hp.y));
        a[2] += w * (hq.x * hq.x + hq.y * hq.y);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[c] += __shfl_xor_sync(0xffffffffu, a[c], o);
        if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = a[c];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int w8 = 0; w8 < (int)(blockDim.x >> 5); ++w8) t += red[threadIdx.x][w8];
        partial[((size_t)threadIdx.x * g.nz + l) * gridDim.x + blockIdx.x] = t;
    }
}

// out[c*nz + l] = 0.5 * S_c(l)/(nx ny)^2 * H_l/Htot, one warp per (quantity, layer), fixed order
__global__ void k_energetics_final(Geom g, const double* __restrict__ partial, int nblocks,
                                   const double* __restrict__ Hw, double* __restrict__ out) {
    QGN_PDL_ENTRY();
    const int cl = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (cl >= 3 * g.nz) return;
    const double s = layer_sum(partial, cl, nblocks);
    const double N = (double)g.nx * (double)g.ny;
    if ((threadIdx.x & 31) == 0) out[cl] = 0.5 * ((s / N) / N) * Hw[cl % g.nz];
}

// isotropic KE spectrum per layer in integer shells round(sqrt(i^2 + jj^2))
__global__ void k_ke_spectrum(Geom g, const double2* __restrict__ psi, const double* __restrict__ Hw, int nbins,
                              double* __restrict__ spec) {
    QGN_PDL_ENTRY();
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t total = P * g.nz;
    const double N = (double)g.nx * (double)g.ny;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int l = (int)(e / P);
        const size_t p = e % P;
        int kx, m;
        double k2;
        point_k(g, p, kx, m, k2);
        const int j = g.jfull(m);
        const int jj = j <= g.ny / 2 ? j : j - g.ny;
        const int bin = (int)floor(sqrt((double)kx * kx + (double)jj * jj) + 0.5);
        if (bin >= nbins) continue;
        const double2 v = psi[e];
        double c;
        if (kx > 0) {
            c = 2.0 * k2 * (v.x * v.x + v.y * v.y);
        } else {
            const int jp = (g.ny - j) % g.ny;
            const bool pk = (jp < g.kylo) || (jp >= g.kylo + g.kyshift);
            double2 fp = make_double2(0.0, 0.0);
            if (pk) fp = psi[(size_t)l * P + (jp < g.kylo ? jp : jp - g.kyshift)];
            const double hx = 0.5 * (v.x + fp.x), hy = 0.5 * (v.y - fp.y);
            c = (pk ? 1.0 : 2.0) * k2 * (hx * hx + hy * hy);
        }
        atomicAdd(&spec[(size_t)l * nbins + bin], 0.5 * c / N / N * Hw[l]);
    }
}

// ---- PI controllers (ctrl.cuh); with a loop handle the kernel also sets the condition of
// the graph's retry loop ---------------------------------------------------------------------
__global__ void k_controller(int kind, double inv_n, double TOL, double dt_max, int max_rejects,
                             cudaGraphConditionalHandle loop, int has_loop, DevScalars* sc) {
    QGN_PDL_ENTRY();
    const unsigned again = ctrl_decide(kind, inv_n, TOL, dt_max, max_rejects, sc);
    if (has_loop) cudaGraphSetConditional(loop, again);
}

// start of a step: clears the per-step reject count; with a gate handle it also opens the
// graph's step body only while the run is not halted
__global__ void k_step_gate(DevScalars* sc, cudaGraphConditionalHandle gate, int has_gate) {
    QGN_PDL_ENTRY();
    sc->rejects_step = 0;
    if (has_gate) cudaGraphSetConditional(gate, sc->halt == 0 ? 1u : 0u);
}

__global__ void k_set_cond(cudaGraphConditionalHandle h, unsigned int v) {
    QGN_PDL_ENTRY(); cudaGraphSetConditional(h, v); }

__global__ void k_zero_max(DevScalars* sc) {
    QGN_PDL_ENTRY();
    sc->maxbits = 0ULL;
    sc->accept = 0;
}

__global__ void k_advance_time(DevScalars* sc) {
    QGN_PDL_ENTRY(); sc->t = sc->t + sc->dt; }

// a new state from the host: set t and dt and clear a previous failure
__global__ void k_set_time(DevScalars* sc, double t, double dt) {
    QGN_PDL_ENTRY();
    sc->t = t;
    sc->dt = dt;
    sc->nonfinite = 0;
    sc->halt = 0;
    sc->status = 0;
    sc->rejects_step = 0;
    sc->wait_timeout = 0;
}

// ------------------------------------------------------------------------------------------
// launch wrappers
// ------------------------------------------------------------------------------------------
static inline unsigned blocks_for(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

template <class T>
static CombPtrs<T> comb_ptrs(const Buffers& b) {
    CombPtrs<T> cp{};
    for (int j = 0; j < 6; ++j) {
        cp.N[j] = reinterpret_cast<const T*>(b.N[j]);
        cp.Q[j] = reinterpret_cast<const T*>(b.Qs[j]);
    }
    return cp;
}

template <class T>
static cudaError_t launch_comb(const Geom& g, const Buffers& b, int s, cudaStream_t st) {
    const CombPtrs<T> cp = comb_ptrs<T>(b);
    T* qout = reinterpret_cast<T*>(b.Qs[s]);
    const double es = (double)sizeof(T), C = (double)g.csize();
    const double nb = 16.0 * C + es * C * (2.0 * s - 1.0 + 1.0);
    const unsigned nbk = blocks_for(g.csize(), 256);
    switch (s) {
        case 1: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_comb<1, T>, nbk, 256, 0, st, g, cp, b.q, qout, b.lc, b.sc))); break;
        case 2: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_comb<2, T>, nbk, 256, 0, st, g, cp, b.q, qout, b.lc, b.sc))); break;
        case 3: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_comb<3, T>, nbk, 256, 0, st, g, cp, b.q, qout, b.lc, b.sc))); break;
        case 4: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_comb<4, T>, nbk, 256, 0, st, g, cp, b.q, qout, b.lc, b.sc))); break;
        case 5: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_comb<5, T>, nbk, 256, 0, st, g, cp, b.q, qout, b.lc, b.sc))); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// Stage S on a small grid in one kernel: one thread per kept mode combines every layer (the
// arithmetic of k_ark_comb) and runs GetPsi on the result, saving the second launch that
// dominates when the grid is only a few thousand modes per layer.
template <int S, int NZ>
__global__ void __launch_bounds__(256, 2) k_ark_stage_small(Geom g, CombPtrs<double2> cp, const double2* __restrict__ q,
                                                           double2* __restrict__ qout, double2* __restrict__ psi,
                                                           const LayerConst* __restrict__ lc,
                                                           const __grid_constant__ ModalArg<NZ> ma,
                                                           const DevScalars* __restrict__ sc) {
    QGN_PDL_ENTRY();
    QGN_MODAL_SHARED(NZ);
    const int nz = g.nz;
    const ModalView mv = modal_view<NZ>(ma, s_proj, s_back, s_ev, nz);
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    int kx, m;
    double k2;
    point_k(g, p, kx, m, k2);
    const double k8 = (k2 * k2) * (k2 * k2);
    const double dt = sc->dt;
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    double2 qv[NZC], pv[NZC];
#pragma unroll
    for (int l = 0; l < NZC; ++l) {
        if (l < nz) {
            const size_t e = (size_t)l * P + p;
            const double D = lc->A2 * k2 + sc->A8L[l] * k8;
            double2 nn[S], qq[S];
#pragma unroll
            for (int j = 0; j < S; ++j) nn[j] = cp.N[j][e];
#pragma unroll
            for (int j = 1; j < S; ++j) qq[j] = cp.Q[j][e];
            const double2 q0 = q[e];
            double ax, ay;
            comb_sum64<S>(nn, qq, q0, D, ax, ay);
            const double Mq = 1.0 / (1.0 + 0.25 * dt * D);
            qv[l] = make_double2(Mq * (q0.x + dt * ax), Mq * (q0.y + dt * ay));
            qout[e] = qv[l];
        }
    }
    modal_invert_s<NZ>(mv.proj, mv.back, mv.ev, mv.Htot, nz, k2, p == 0, qv, pv);
#pragma unroll
    for (int l = 0; l < NZC; ++l)
        if (l < nz) psi[(size_t)l * P + p] = pv[l];
}

// grids of at most this many kept mode-layers take the fused stage kernel and the column kernels
constexpr size_t kSmallStage = (size_t)1 << 17;
// the fused stage kernel (combination and GetPsi of all layers per mode) up to this many kept
// mode-layers (build-time tuning knob; beyond it the stage is a streaming combination per
// element followed by GetPsi)
#ifndef QGN_FUSED_STAGE_MAX
#define QGN_FUSED_STAGE_MAX kSmallStage
#endif

template <int NZ>
static cudaError_t launch_stage_small_nz(const Geom& g, const Buffers& b, int s, cudaStream_t st) {
    const CombPtrs<double2> cp = comb_ptrs<double2>(b);
    const size_t P = (size_t)g.nkx * g.nky;
    const unsigned nbk = blocks_for(P, 256);
    const double C = (double)g.csize(), nb = 16.0 * C * (2.0 * s + 2.0);
    double2* qo = b.Qs[s];
    switch (s) {
        case 1: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_stage_small<1, NZ>, nbk, 256, 0, st, g, cp, b.q, qo, b.psi, b.lc, modal_arg<NZ>(b), b.sc))); break;
        case 2: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_stage_small<2, NZ>, nbk, 256, 0, st, g, cp, b.q, qo, b.psi, b.lc, modal_arg<NZ>(b), b.sc))); break;
        case 3: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_stage_small<3, NZ>, nbk, 256, 0, st, g, cp, b.q, qo, b.psi, b.lc, modal_arg<NZ>(b), b.sc))); break;
        case 4: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_stage_small<4, NZ>, nbk, 256, 0, st, g, cp, b.q, qo, b.psi, b.lc, modal_arg<NZ>(b), b.sc))); break;
        case 5: QGN_LAUNCH(KID_STAGE, nb, st, (::qgn::launch(k_ark_stage_small<5, NZ>, nbk, 256, 0, st, g, cp, b.q, qo, b.psi, b.lc, modal_arg<NZ>(b), b.sc))); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// ---- small grids: the stage, GetPsi and the y passes of one kx column in one CTA -------------
// On a grid of at most kSmallStage kept mode-layers every kernel of a step is a few
// microseconds of latency, so launches are what a step costs.  A stage's combination and
// GetPsi work per mode (all layers of one (kx, ky)), and the y transforms per kx column, so one
// CTA per column can do both without waiting for other CTAs.
template <int NY, int NZ>
struct StageYinvCfg {
    static constexpr int G = FFTShape<NY, 16>::G;
    static constexpr int SLOTS = 3 * NZ;   // (q, u, v) x layers
    static constexpr int THREADS = SLOTS * G;
    static constexpr int TS = slot_stride(NY, 2, 16, 16);
    // rows are written de-interleaved (even y at y/2, odd y at HY + y/2): the 8 lanes of a
    // quarter-warp hold 4 even and 4 odd rows, so HY = 4 mod 8 keeps their stores on distinct
    // bank groups, and the packing reads are consecutive
    static constexpr int HY = NY / 2 + 4;
    static_assert(2 * HY <= TS, "de-interleaved rows fit the slot");
    static_assert(G >= 8 && G <= 32, "one slot per 8..32 lanes");
    static constexpr int SLOT_BYTES = SLOTS * TS * 16;
};

// Stage S (S = 0: the state itself) of column kx: q_S at every kept mode of the column for all
// layers (the arithmetic of k_ark_stage_small), GetPsi of it, both kept in shared memory;
// then the 3*NZ inverse y transforms of q, u = -i ky psi, v = i kx psi of the column, one per
// slot of G threads, packed into row pairs for the x pass (the arithmetic of yinv_tile).
template <int S, int NZ, int NY>
__device__ __forceinline__ void stage_yinv_col(const Geom& g, int kx, const CombPtrs<double2>& cp,
                                               const double2* __restrict__ q, double2* __restrict__ qout,
                                               double2* __restrict__ psi, const LayerConst* __restrict__ lc,
                                               const ModalView& mv, const DevScalars* __restrict__ sc,
                                               double2* __restrict__ pq, double2* __restrict__ pv,
                                               double2* __restrict__ pu, const double2* __restrict__ twy,
                                               unsigned char* sm_raw) {
    using C = StageYinvCfg<NY, NZ>;
    double2* slots = reinterpret_cast<double2*>(sm_raw);
    const int nky = g.nky;
    double2* qcol = reinterpret_cast<double2*>(sm_raw + C::SLOT_BYTES);   // [NZ][nky]
    double2* pcol = qcol + NZ * nky;
    const int tid = threadIdx.x;
    const size_t P = (size_t)g.nkx * nky;
    const double kxv = g.dkx * kx;
    const double dt = sc->dt;
    for (int m = tid; m < nky; m += C::THREADS) {
        const size_t p = (size_t)kx * nky + m;
        const double kyv = g.kyval(g.jfull(m));
        const double k2 = kxv * kxv + kyv * kyv;
        const double k8 = (k2 * k2) * (k2 * k2);
        double2 qv[NZ], pvv[NZ];
#pragma unroll
        for (int l = 0; l < NZ; ++l) {
            const size_t e = (size_t)l * P + p;
            if constexpr (S == 0) {
                qv[l] = q[e];
            } else {
                const double D = lc->A2 * k2 + sc->A8L[l] * k8;
                double2 nn[S], qq[S];
#pragma unroll
                for (int j = 0; j < S; ++j) nn[j] = cp.N[j][e];
#pragma unroll
                for (int j = 1; j < S; ++j) qq[j] = cp.Q[j][e];
                const double2 q0 = q[e];
                double ax, ay;
                comb_sum64<S>(nn, qq, q0, D, ax, ay);
                const double Mq = 1.0 / (1.0 + 0.25 * dt * D);
                qv[l] = make_double2(Mq * (q0.x + dt * ax), Mq * (q0.y + dt * ay));
                qout[e] = qv[l];
            }
            qcol[l * nky + m] = qv[l];
        }
        modal_invert_s<NZ>(mv.proj, mv.back, mv.ev, mv.Htot, NZ, k2, p == 0, qv, pvv);
#pragma unroll
        for (int l = 0; l < NZ; ++l) {
            psi[(size_t)l * P + p] = pvv[l];
            pcol[l * nky + m] = pvv[l];
        }
    }
    __syncthreads();
    const int slot = tid / C::G, lane = tid % C::G;
    const int f = slot / NZ, l = slot % NZ;
    double2* xs = slots + slot * C::TS;
    const double2* col = (f == 0 ? qcol : pcol) + l * nky;
    auto ld = [&](int j) -> double2 {
        const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
        if (!kept) return make_double2(0.0, 0.0);
        double2 v = col[j < g.kylo ? j : j - g.kyshift];
        if (f == 1) {   // u_hat = -i ky psi_hat  (QGN_Module.f90:223)
            const double kyv = g.kyval(j);
            v = make_double2(kyv * v.y, -kyv * v.x);
        } else if (f == 2) {   // v_hat = i kx psi_hat  (QGN_Module.f90:224)
            v = make_double2(-kxv * v.y, kxv * v.x);
        }
        return v;
    };
    auto omap = [](int y) { return (y & 1) * C::HY + (y >> 1); };
    fft_fused<NY, +1, SRC_FN, DST_SMEM_MAP, 16, true>(xs, lane, true, twy, ld, omap);
    double2* dst = (f == 0 ? pq : (f == 1 ? pu : pv)) + (size_t)l * (NY / 2) * 2 * g.nkxp;
    for (int pr = lane; pr < NY / 2; pr += C::G) {
        const double2 f1 = xs[pr], f2 = xs[C::HY + pr];
        double2* row = dst + (size_t)pr * 2 * g.nkxp;
        row[kx] = pack_lo(f1, f2, kx == 0 || 2 * kx == g.nx);
        row[g.nkxp + kx] = kx > 0 ? pack_hi(f1, f2) : make_double2(0.0, 0.0);
    }
}

template <int S, int NZ, int NY>
__global__ void __launch_bounds__(StageYinvCfg<NY, NZ>::THREADS)
    k_stage_yinv(Geom g, CombPtrs<double2> cp, const double2* __restrict__ q, double2* __restrict__ qout,
                 double2* __restrict__ psi, const LayerConst* __restrict__ lc, const __grid_constant__ ModalArg<NZ> ma,
                 const DevScalars* __restrict__ sc, double2* __restrict__ pq, double2* __restrict__ pv,
                 double2* __restrict__ pu, const double2* __restrict__ twy) {
    QGN_PDL_ENTRY();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const ModalView mv = modal_view<NZ>(ma, nullptr, nullptr, nullptr, NZ);
    stage_yinv_col<S, NZ, NY>(g, blockIdx.x, cp, q, qout, psi, lc, mv, sc, pq, pv, pu, twy, sm_raw);
}

// Stages 2..5 without quadratic drag: the y-forward pass that finishes N_{S-1} for column kx
// (all layers; the assembly of yfwd_tile), then stage S and its y-inverse for the same column.
// N_{S-1} of the column is complete before stage S reads it, so no other CTA's output is
// needed: the y-forward, stage and y-inverse launches become one.
template <int S, int NZ, int NY>
__global__ void __launch_bounds__(StageYinvCfg<NY, NZ>::THREADS)
    k_yfwd_stage_yinv(Geom g, const double2* __restrict__ pp, const double2* __restrict__ qprev,
                      double2* __restrict__ nout, const double2* __restrict__ extra, CombPtrs<double2> cp,
                      const double2* __restrict__ q, double2* __restrict__ qout, double2* __restrict__ psi,
                      const LayerConst* __restrict__ lc, const __grid_constant__ ModalArg<NZ> ma,
                      const DevScalars* __restrict__ sc, double2* __restrict__ pq, double2* __restrict__ pv,
                      double2* __restrict__ pu, const double2* __restrict__ twy) {
    QGN_PDL_ENTRY();
    using C = StageYinvCfg<NY, NZ>;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* slots = reinterpret_cast<double2*>(sm_raw);
    const ModalView mv = modal_view<NZ>(ma, nullptr, nullptr, nullptr, NZ);
    const int tid = threadIdx.x;
    const int kx = blockIdx.x;
    const int nky = g.nky;
    {   // forward y transforms of (uq)^ (slots 0..NZ-1) and (vq)^ (slots NZ..2NZ-1), unpadded
        const int slot = tid / C::G, lane = tid % C::G;
        const int f = slot / NZ, l = slot % NZ;
        const bool act = slot < 2 * NZ;
        double2* xs = slots + slot * C::TS;
        auto ld = [&](int y) -> double2 { return unpack_p(pp, g, act ? l : 0, y, kx, f); };
        auto omap = [](int y) { return y; };
        fft_fused<NY, -1, SRC_FN, DST_SMEM_MAP, 16, true>(xs, lane, act, twy, ld, omap);
    }
    const double kxv = g.dkx * kx;
    const bool expl = lc->explicit_diss != 0;
    for (int m = tid; m < nky; m += C::THREADS) {
        const int j = g.jfull(m);
        const double kyv = g.kyval(j);
#pragma unroll
        for (int l = 0; l < NZ; ++l) {
            const size_t idx = ((size_t)l * g.nkx + kx) * nky + m;
            const double2 fuq = slots[l * C::TS + j], fvq = slots[(NZ + l) * C::TS + j];
            const double2 qv = qprev[idx], pvv = psi[idx];
            // jaco_hat = i kx uq_hat + i ky vq_hat  (QGN_Module.f90:244-247)
            const double2 jac = make_double2(-kxv * fuq.y - kyv * fvq.y, kxv * fuq.x + kyv * fvq.x);
            double2 r = make_double2(-jac.x, -jac.y);
            // - uBar i kx q_hat - (beta+qyBar) v_hat   (QGN_Module.f90:270-273)
            const double uk = lc->uBar[l] * kxv;
            const double2 vh = make_double2(-kxv * pvv.y, kxv * pvv.x);
            const double bq = lc->betaq[l];
            r = make_double2(r.x + uk * qv.y, r.y - uk * qv.x);
            r = make_double2(r.x - bq * vh.x, r.y - bq * vh.y);
            const double k2 = kxv * kxv + kyv * kyv;
            if (expl) {   // QGN_Module.f90:275-280
                const double k4 = k2 * k2, k8 = k4 * k4;
                const double dcoef = lc->A2 * k2 + lc->A8 * k8;
                r = make_double2(r.x - dcoef * qv.x, r.y - dcoef * qv.y);
            }
            if (l == NZ - 1) {   // Ekman, QGN_Module.f90:282
                const double ekk = lc->ekman * k2;
                r = make_double2(r.x + ekk * pvv.x, r.y + ekk * pvv.y);
            }
            if (extra) {
                const double2 x = extra[idx];
                r = make_double2(r.x + x.x, r.y + x.y);
            }
            if (kx == 0 && m == 0) r = make_double2(0.0, 0.0);
            nout[idx] = r;
        }
    }
    __syncthreads();   // N_{S-1} of the column is written; the slots are free
    stage_yinv_col<S, NZ, NY>(g, kx, cp, q, qout, psi, lc, mv, sc, pq, pv, pu, twy, sm_raw);
}

// the (ny, nz) pairs built: a CTA keeps its registers without spilling
constexpr bool stage_yinv_built(int ny, int nz) {
    return (ny == 128 && nz <= 16) || (ny == 256 && nz <= 8) || (ny == 512 && nz <= 4);
}

// the dynamic shared-memory limit of each column kernel, raised once per (device, kernel)
static cudaError_t column_smem(const void* kern, int bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return smem_opt_in(kern, 227 * 1024);
}

template <int NZ, int NY, class Kern, class... Args>
static cudaError_t stage_yinv_launch(const Geom& g, Kern kern, int kid, double nb, cudaStream_t st, Args... args) {
    using C = StageYinvCfg<NY, NZ>;
    const int smem = C::SLOT_BYTES + 2 * NZ * g.nky * 16;
    cudaError_t e = column_smem(reinterpret_cast<const void*>(kern), smem);
    if (e != cudaSuccess) return e;
    QGN_LAUNCH(kid, nb, st, ::qgn::launch(kern, g.nkx, C::THREADS, smem, st, args...));
    return cudaGetLastError();
}

template <int S, int NZ, int NY>
static cudaError_t stage_yinv_s(const Geom& g, const Buffers& b, cudaStream_t st) {
    const double Cb = 16.0 * (double)g.csize(), Hb = 16.0 * (double)g.nz * NY * g.nkx;
    const double nb = Cb * (S == 0 ? 2.0 : 2.0 * S + 2.0) + 3.0 * Hb;
    return stage_yinv_launch<NZ, NY>(g, k_stage_yinv<S, NZ, NY>, KID_STAGE, nb, st, g, comb_ptrs<double2>(b), b.q,
                                     b.Qs[S], b.psi, b.lc, modal_arg<NZ>(b), b.sc, b.hq, b.hp, b.hu, b.twy);
}

template <int S, int NZ, int NY>
static cudaError_t yfwd_stage_yinv_s(const Geom& g, const Buffers& b, const double2* extra, cudaStream_t st) {
    const double Cb = 16.0 * (double)g.csize(), Hb = 16.0 * (double)g.nz * NY * g.nkx;
    const double nb = 2.0 * Hb + 3.0 * Cb + Cb * (2.0 * S + 2.0) + 3.0 * Hb;
    return stage_yinv_launch<NZ, NY>(g, k_yfwd_stage_yinv<S, NZ, NY>, KID_YFWD, nb, st, g, b.hpp, b.Qs[S - 1],
                                     b.N[S - 1], extra, comb_ptrs<double2>(b), b.q, b.Qs[S], b.psi, b.lc,
                                     modal_arg<NZ>(b), b.sc, b.hq, b.hp, b.hu, b.twy);
}

// fused = false: stage s and its y-inverse; true: the y-forward of RHS s-1 as well (s = 2..5)
template <int NZ, int NY>
static cudaError_t stage_yinv_go(const Geom& g, const Buffers& b, int s, bool fused, const double2* extra,
                                 cudaStream_t st) {
    if (!fused) {
        switch (s) {
            case 0: return stage_yinv_s<0, NZ, NY>(g, b, st);
            case 1: return stage_yinv_s<1, NZ, NY>(g, b, st);
            case 2: return stage_yinv_s<2, NZ, NY>(g, b, st);
            case 3: return stage_yinv_s<3, NZ, NY>(g, b, st);
            case 4: return stage_yinv_s<4, NZ, NY>(g, b, st);
            case 5: return stage_yinv_s<5, NZ, NY>(g, b, st);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (s) {
        case 2: return yfwd_stage_yinv_s<2, NZ, NY>(g, b, extra, st);
        case 3: return yfwd_stage_yinv_s<3, NZ, NY>(g, b, extra, st);
        case 4: return yfwd_stage_yinv_s<4, NZ, NY>(g, b, extra, st);
        case 5: return yfwd_stage_yinv_s<5, NZ, NY>(g, b, extra, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int NZ>
static cudaError_t stage_yinv_nz(const Geom& g, const Buffers& b, int s, bool fused, const double2* extra,
                                 cudaStream_t st) {
    switch (g.ny) {
        case 128: return stage_yinv_go<NZ, 128>(g, b, s, fused, extra, st);
        case 256:
            if constexpr (stage_yinv_built(256, NZ)) return stage_yinv_go<NZ, 256>(g, b, s, fused, extra, st);
            return cudaErrorInvalidValue;
        case 512:
            if constexpr (stage_yinv_built(512, NZ)) return stage_yinv_go<NZ, 512>(g, b, s, fused, extra, st);
            return cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
}

static cudaError_t stage_yinv_dispatch(const Geom& g, const Buffers& b, int s, bool fused, const double2* extra,
                                       cudaStream_t st) {
    switch (g.nz) {
        case 2: return stage_yinv_nz<2>(g, b, s, fused, extra, st);
        case 4: return stage_yinv_nz<4>(g, b, s, fused, extra, st);
        case 8: return stage_yinv_nz<8>(g, b, s, fused, extra, st);
        case 16: return stage_yinv_nz<16>(g, b, s, fused, extra, st);
        default: return cudaErrorInvalidValue;
    }
}

// small grids (at most kSmallStage kept mode-layers, a built (ny, nz) pair, the shared memory
// fits) take the column kernels; QGN_NO_FUSED_STAGE=1 keeps the separate kernels
bool stage_yinv_ok(const Geom& g, const Buffers& b) {
    if (!b.mc_h || g.csize() > kSmallStage || std::getenv("QGN_NO_FUSED_STAGE")) return false;
    if (g.nz != 2 && g.nz != 4 && g.nz != 8 && g.nz != 16) return false;
    if (!stage_yinv_built(g.ny, g.nz)) return false;
    const int TS = g.ny + g.ny / 16 + 8;
    const size_t smem = (size_t)3 * g.nz * TS * 16 + (size_t)2 * g.nz * g.nky * 16;
    return smem <= 220 * 1024;
}

cudaError_t launch_ark_stage_yinv(const Geom& g, const Buffers& b, int s, cudaStream_t st) {
    return stage_yinv_dispatch(g, b, s, false, nullptr, st);
}

cudaError_t launch_yfwd_stage_yinv(const Geom& g, const Buffers& b, int s, const double2* extra, cudaStream_t st) {
    return stage_yinv_dispatch(g, b, s, true, extra, st);
}

cudaError_t launch_modal_f32(const Geom& g, const Buffers& b, const float2* q, float2* psi, cudaStream_t st) {
    const size_t P = (size_t)g.nkx * g.nky;
    dim3 grid(blocks_for(P, 256));
    const double nb = 16.0 * (double)g.csize();
    switch (b.mc_h ? g.nz : 0) {
        case 2: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_f32<2>, grid, 256, 0, st, g, modal_arg<2>(b), q, psi)); break;
        case 4: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_f32<4>, grid, 256, 0, st, g, modal_arg<4>(b), q, psi)); break;
        case 8: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_f32<8>, grid, 256, 0, st, g, modal_arg<8>(b), q, psi)); break;
        case 16: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_f32<16>, grid, 256, 0, st, g, modal_arg<16>(b), q, psi)); break;
        default: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_f32<0>, grid, 256, 0, st, g, modal_arg<0>(b), q, psi)); break;
    }
    return cudaGetLastError();
}

// stage s of ARK4(3)6L[2]SA: q_s (streaming combination), then psi_s = GetPsi(q_s)
cudaError_t launch_ark_stage(const Geom& g, const Buffers& b, int s, cudaStream_t st) {
    if (g.csize() <= (size_t)(QGN_FUSED_STAGE_MAX) && b.mc_h) {
        switch (g.nz) {
            case 2: return launch_stage_small_nz<2>(g, b, s, st);
            case 4: return launch_stage_small_nz<4>(g, b, s, st);
            case 8: return launch_stage_small_nz<8>(g, b, s, st);
            case 16: return launch_stage_small_nz<16>(g, b, s, st);
            default: break;   // other layer counts: the two streaming kernels
        }
    }
    cudaError_t e = launch_comb<double2>(g, b, s, st);
    if (e != cudaSuccess) return e;
    return launch_modal(g, b, b.Qs[s], b.psi, st);
}

static StagePtrs32 stage_ptrs32(const Buffers& b) {
    StagePtrs32 sp{};
    for (int j = 0; j < 6; ++j) {
        sp.N[j] = reinterpret_cast<const float2*>(b.N[j]);
        sp.Qs[j] = reinterpret_cast<const float2*>(b.Qs[j]);
    }
    return sp;
}

cudaError_t launch_ark_stage_mixed(const Geom& g, const Buffers& b, int s, cudaStream_t st) {
    cudaError_t e = launch_comb<float2>(g, b, s, st);
    if (e != cudaSuccess) return e;
    return launch_modal_f32(g, b, reinterpret_cast<const float2*>(b.Qs[s]), reinterpret_cast<float2*>(b.psi), st);
}

cudaError_t launch_ark_update_mixed(const Geom& g, const Buffers& b, cudaStream_t st) {
    const StagePtrs32 sp = stage_ptrs32(b);
    const double C = (double)g.csize();
    QGN_LAUNCH(KID_UPDATE, 16.0 * C * 2.0 + 8.0 * C * 10.0, st,
               ::qgn::launch(k_ark_update_mixed, blocks_for(g.csize(), 256), 256, 0, st, g, sp, b.q, b.qnew,
                             reinterpret_cast<float2*>(b.err), b.lc, b.sc));
    return cudaGetLastError();
}

cudaError_t launch_modal_mixed(const Geom& g, const Buffers& b, const double2* q, float2* q32, float2* psi32,
                               cudaStream_t st) {
    const size_t P = (size_t)g.nkx * g.nky;
    dim3 grid(blocks_for(P, 256));
    const double nb = 32.0 * (double)g.csize();
    switch (b.mc_h ? g.nz : 0) {
        case 2: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_mixed<2>, grid, 256, 0, st, g, modal_arg<2>(b), q, q32, psi32)); break;
        case 4: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_mixed<4>, grid, 256, 0, st, g, modal_arg<4>(b), q, q32, psi32)); break;
        case 8: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_mixed<8>, grid, 256, 0, st, g, modal_arg<8>(b), q, q32, psi32)); break;
        case 16: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_mixed<16>, grid, 256, 0, st, g, modal_arg<16>(b), q, q32, psi32)); break;
        default: QGN_LAUNCH(KID_MODAL, nb, st, ::qgn::launch(k_modal_mixed<0>, grid, 256, 0, st, g, modal_arg<0>(b), q, q32, psi32)); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_f2d(size_t n, const float2* a, double2* b, cudaStream_t st) {
    QGN_LAUNCH(KID_LAYOUT, 24.0 * (double)n, st, ::qgn::launch(k_f2d, blocks_for(n, 256), 256, 0, st, n, a, b));
    return cudaGetLastError();
}

cudaError_t launch_ark_update(const Geom& g, const Buffers& b, cudaStream_t st) {
    StagePtrs sp{};
    for (int j = 0; j < 6; ++j) { sp.N[j] = b.N[j]; sp.Qs[j] = b.Qs[j]; }
    QGN_LAUNCH(KID_UPDATE, 12.0 * 16.0 * (double)g.csize(), st,
               ::qgn::launch(k_ark_update, blocks_for(g.csize(), 256), 256, 0, st, g, sp, b.q, b.qnew, b.err, b.lc, b.sc));
    return cudaGetLastError();
}

cudaError_t launch_combo(const Geom& g, const Buffers& b, const Combo& cb, const double2* q, double2* out,
                         double2* psi, bool want_psi, cudaStream_t st) {
    const size_t P = (size_t)g.nkx * g.nky;
    dim3 grid(blocks_for(P, 256));
    const int wp = want_psi ? 1 : 0;
    const double nb = 16.0 * (double)g.csize() * (1.0 + cb.n + 1.0 + wp);
    switch (b.mc_h ? g.nz : 0) {
        case 2: QGN_LAUNCH(KID_COMBO, nb, st, ::qgn::launch(k_combo<2>, grid, 256, 0, st, g, cb, q, out, psi, modal_arg<2>(b), b.sc, wp)); break;
        case 4: QGN_LAUNCH(KID_COMBO, nb, st, ::qgn::launch(k_combo<4>, grid, 256, 0, st, g, cb, q, out, psi, modal_arg<4>(b), b.sc, wp)); break;
        case 8: QGN_LAUNCH(KID_COMBO, nb, st, ::qgn::launch(k_combo<8>, grid, 256, 0, st, g, cb, q, out, psi, modal_arg<8>(b), b.sc, wp)); break;
        case 16: QGN_LAUNCH(KID_COMBO, nb, st, ::qgn::launch(k_combo<16>, grid, 256, 0, st, g, cb, q, out, psi, modal_arg<16>(b), b.sc, wp)); break;
        default: QGN_LAUNCH(KID_COMBO, nb, st, ::qgn::launch(k_combo<0>, grid, 256, 0, st, g, cb, q, out, psi, modal_arg<0>(b), b.sc, wp)); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_lincomb(const Geom& g, const Combo& cb, double2* out, cudaStream_t st) {
    QGN_LAUNCH(KID_LINCOMB, 16.0 * (double)g.csize() * (cb.n + 1.0), st,
               ::qgn::launch(k_lincomb, blocks_for(g.csize(), 256), 256, 0, st, g.csize(), cb, out));
    return cudaGetLastError();
}

// blocks per layer of the Parseval reductions: about 8 per SM over all layers, so each thread
// streams only a few dozen modes (with 2 per SM the Leith reduction of 1024^2 x 8 read its
// 29.8 MB at 1.1 TB/s); the partials buffer holds 512 x kMaxNZ doubles, 3 x nz x nb at most here
static int parseval_blocks(const Geom& g) {
    const size_t P = (size_t)g.nkx * g.nky;
    const size_t want = (size_t)(8 * 148 + g.nz - 1) / g.nz;
    size_t nb = (P + 255) / 256;
    if (nb > want) nb = want;
    if (nb > 512) nb = 512;
    return (int)(nb > 0 ? nb : 1);
}

cudaError_t launch_leith(const Geom& g, const Buffers& b, const double2* q, double c12, cudaStream_t st) {
    const int nb = parseval_blocks(g);
    QGN_LAUNCH(KID_PARSEVAL, 16.0 * (double)g.csize(), st,
               ::qgn::launch(k_leith, dim3(nb, g.nz), 256, 0, st, g, q, b.red, c12, b.sc));
    return cudaGetLastError();
}

cudaError_t launch_ke(const Geom& g, const Buffers& b, const double2* psi, const double* Hw, double* ke, cudaStream_t st) {
    const int nb = parseval_blocks(g);
    QGN_LAUNCH(KID_PARSEVAL, 16.0 * (double)g.csize(), st,
               ::qgn::launch(k_parseval<1>, dim3(nb, g.nz), 256, 0, st, g, psi, b.red));
    QGN_LAUNCH(KID_SCALAR, 0.0, st, ::qgn::launch(k_ke_final, (g.nz + 7) / 8, 256, 0, st, g, b.red, nb, Hw, ke));
    return cudaGetLastError();
}

cudaError_t launch_energetics(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double* out,
                              cudaStream_t st) {
    const int nb = parseval_blocks(g);
    QGN_LAUNCH(KID_PARSEVAL, 32.0 * (double)g.csize(), st,
               ::qgn::launch(k_energetics, dim3(nb, g.nz), 256, 0, st, g, q, psi, b.red));
    QGN_LAUNCH(KID_SCALAR, 0.0, st,
               ::qgn::launch(k_energetics_final, (3 * g.nz + 7) / 8, 256, 0, st, g, b.red, nb, b.Hw, out));
    return cudaGetLastError();
}

cudaError_t launch_ke_spectrum(const Geom& g, const double2* psi, const double* Hw, int nbins, double* spec,
                               cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(spec, 0, sizeof(double) * (size_t)nbins * g.nz, st);
    if (e != cudaSuccess) return e;
    QGN_LAUNCH(KID_PARSEVAL, 16.0 * (double)g.csize(), st,
               ::qgn::launch(k_ke_spectrum, 148 * 8, 256, 0, st, g, psi, Hw, nbins, spec));
    return cudaGetLastError();
}

cudaError_t launch_controller(const Geom& g, const Buffers& b, int kind, double TOL, double dt_max, int max_rejects,
                              const cudaGraphConditionalHandle* loop, cudaStream_t st) {
    QGN_LAUNCH(KID_SCALAR, 0.0, st,
               ::qgn::launch(k_controller, 1, 1, 0, st, kind, g.inv_nxny, TOL, dt_max, max_rejects, loop ? *loop : 0,
                                             loop ? 1 : 0, b.sc));
    return cudaGetLastError();
}

cudaError_t launch_step_gate(DevScalars* sc, const cudaGraphConditionalHandle* gate, cudaStream_t st) {
    QGN_LAUNCH(KID_SCALAR, 0.0, st, ::qgn::launch(k_step_gate, 1, 1, 0, st, sc, gate ? *gate : 0, gate ? 1 : 0));
    return cudaGetLastError();
}

cudaError_t launch_set_cond(cudaGraphConditionalHandle h, unsigned int v, cudaStream_t st) {
    QGN_LAUNCH(KID_SCALAR, 0.0, st, ::qgn::launch(k_set_cond, 1, 1, 0, st, h, v));
    return cudaGetLastError();
}

cudaError_t launch_zero_scalar_max(DevScalars* sc, cudaStream_t st) {
    QGN_LAUNCH(KID_SCALAR, 0.0, st, ::qgn::launch(k_zero_max, 1, 1, 0, st, sc));
    return cudaGetLastError();
}

cudaError_t launch_set_time(DevScalars* sc, double t, double dt, cudaStream_t st) {
    QGN_LAUNCH(KID_SCALAR, 0.0, st, ::qgn::launch(k_set_time, 1, 1, 0, st, sc, t, dt));
    return cudaGetLastError();
}

cudaError_t launch_advance_time(DevScalars* sc, cudaStream_t st) {
    QGN_LAUNCH(KID_SCALAR, 0.0, st, ::qgn::launch(k_advance_time, 1, 1, 0, st, sc));
    return cudaGetLastError();
}

}  // namespace qgn
