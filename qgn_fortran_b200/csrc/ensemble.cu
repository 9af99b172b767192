// ensemble.cu -- independent QGN members with different grid sizes and layer counts,
// advanced together with BSRK3 (BSRK3.f90) in FP64 or in the mixed mode.
//
// Every pass of an attempt -- stage combination + GetPsi, the three right-hand-side passes,
// the error combination, the error transform and the controller -- is ONE launch for the
// whole ensemble: a table of tile counts maps each CTA of a persistent grid-stride loop to
// a member and a tile, and the tile bodies of the single-field kernels (rhs_tiles.cuh) run
// on it with the member's geometry.  All members take their attempts in lockstep; members
// that have taken their steps (or halted) drop out of the tile loops.  The attempts of an
// advance run as the body of a CUDA graph WHILE node whose condition the controller kernel
// sets on the device ("any member still active"), so an advance is one graph launch.  An
// autotuner times each pass's tile-width variants and grid sizes on the ensemble at hand
// the first time it advances and keeps the fastest.
//
// Members are ordinary contexts (qgn_create, scheme BSRK3) that the ensemble borrows: their
// buffers, constants and device scalars are used in place, so qgn_get_state, qgn_rhs,
// qgn_physical and the diagnostics keep working on each member.  In the mixed mode the
// stage right-hand sides, stage inputs and psi are FP32 and the transforms run in FP32; the
// state, the stage sums (accumulated in FP64), GetPsi's arithmetic, the error combination,
// its transform and the controller are FP64.
#include "qgn_internal.cuh"
#include "fft.cuh"
#include "prof.cuh"
#include "rhs_tiles.cuh"
#include "ctrl.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <utility>
#include <string>
#include <unordered_set>
#include <vector>

namespace qgn {
namespace {

// one row of the device member table
struct EnsMember {
    Geom g;
    double2* q;           // accepted state (FP64)
    double2* qc;          // fourth-stage state q_tmp, the candidate solution (FP64)
    double2* err;         // embedded error spectrum (FP64)
    void* N[4];           // RHS0..RHS3 in the stage precision
    void* Qs;             // stage input in the stage precision
    void* psi;            // GetPsi of the stage input
    void* hq;             // half-transformed fields (stage precision; FP64 for the error transform)
    void* hp;
    void* hu;
    void* hpp;
    void* hpd;
    const void* twx;      // twiddles in the stage precision
    const void* twy;
    const double2* twx64;
    const double2* twy64;
    const LayerConst* lc;
    const ModalConst* mc;
    DevScalars* sc;
    double TOL, dt_max;
    int max_rejects;
    int steps_left;       // accepted steps still to take in this advance
    int active;           // 1 while steps_left > 0 and the member has not halted
    int need_fsal;        // RHS0 of the current state is still to be computed
};

// passes with their own tile tables
enum { EP_POINT = 0, EP_ELEM, EP_YINV, EP_XPASS, EP_YFWD, EP_YINV1, EP_XINV1, EP_COUNT };
// passes the autotuner chooses for
enum { TP_YINV = 0, TP_XPASS, TP_YFWD, TP_COUNT };
// Tile variants the autotuner searches per pass: CTA width (threads of a y pass, threads per
// slot group of the x pass) and elements per thread of the transforms (tv_make, rhs_tiles.cuh).
// Every listed pair gives whole tiles for 128-, 256- and 512-point transforms (the y-forward
// needs a width of at least two transforms, the others one); 32 elements per thread only in
// FP32, where they take 64 registers (FP64 would spill under the 128-register cap).  Index 1 is
// the default before tuning (16 elements per thread).
template <class CT>
struct EnsVariants;
template <>
struct EnsVariants<double2> {
    static constexpr int yinv[] = {tv_make(64, 16), tv_make(128, 16), tv_make(256, 16),
                                   tv_make(64, 8),  tv_make(128, 8),  tv_make(256, 8)};
    static constexpr int xpass[] = {tv_make(32, 16), tv_make(64, 16), tv_make(128, 16), tv_make(64, 8),
                                    tv_make(128, 8)};
    static constexpr int yfwd[] = {tv_make(64, 16), tv_make(128, 16), tv_make(256, 16), tv_make(128, 8),
                                   tv_make(256, 8)};
};
template <>
struct EnsVariants<float2> {
    static constexpr int yinv[] = {tv_make(64, 16), tv_make(128, 16), tv_make(256, 16), tv_make(64, 8),
                                   tv_make(128, 8),  tv_make(256, 8),  tv_make(64, 32),  tv_make(128, 32),
                                   tv_make(256, 32)};
    static constexpr int xpass[] = {tv_make(32, 16), tv_make(64, 16), tv_make(128, 16), tv_make(64, 8),
                                    tv_make(128, 8), tv_make(32, 32), tv_make(64, 32),  tv_make(128, 32)};
    static constexpr int yfwd[] = {tv_make(64, 16), tv_make(128, 16), tv_make(256, 16), tv_make(128, 8),
                                   tv_make(256, 8), tv_make(64, 32),  tv_make(128, 32)};
};
template <class CT>
constexpr int ens_variant_count(int tp) {
    return tp == 0 ? (int)(sizeof(EnsVariants<CT>::yinv) / sizeof(int))
                   : tp == 1 ? (int)(sizeof(EnsVariants<CT>::xpass) / sizeof(int))
                             : (int)(sizeof(EnsVariants<CT>::yfwd) / sizeof(int));
}
template <class CT>
constexpr int ens_variant(int tp, int v) {
    return tp == 0 ? EnsVariants<CT>::yinv[v] : tp == 1 ? EnsVariants<CT>::xpass[v] : EnsVariants<CT>::yfwd[v];
}
constexpr int kDefaultVariant = 1;
// register cap of an ensemble transform kernel: 32 FP32 elements per thread need 64 for data
template <class CT, int TV>
__host__ __device__ constexpr int ens_regcap() {
    return tv_radix(TV) == 32 ? 128 : regcap<CT>(128, 96);
}
constexpr int kPointTile = 256;

__device__ __forceinline__ int ens_find(const int* __restrict__ start, int nm, int t) {
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// stage 0 is the FSAL evaluation RHS0 = GetRHS(q_hat) (BSRK3.f90:12-17), stages 1..3 the
// attempt's stages; a member takes part in a pass when it needs that evaluation
__device__ __forceinline__ bool ens_runs(const EnsMember& M, int stage) {
    return stage == 0 ? (M.need_fsal != 0 && M.active != 0) : M.active != 0;
}

template <class CT>
__device__ __forceinline__ CT to_ct(double2 v);
template <>
__device__ __forceinline__ double2 to_ct<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 to_ct<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

template <class CT>
__device__ __forceinline__ void axpy(double2& v, double c, CT r) {
    v.x += c * (double)r.x;
    v.y += c * (double)r.y;
}

// the field the stage-s right-hand side reads: FP64 stage 3 reads q_tmp in place
template <class CT>
__device__ __forceinline__ const CT* stage_input(const EnsMember& M, int s) {
    return (sizeof(CT) == 16 && s == 3) ? reinterpret_cast<const CT*>(M.qc) : static_cast<const CT*>(M.Qs);
}

// ---- stage combination + GetPsi (BSRK3.f90:21-28, QGN_Module.f90:315-341) ------------------
template <int NZ, class CT>
__device__ __noinline__ void ens_stage_point(const EnsMember& M, const Geom& g, size_t p, int s,
                                                const double* proj, const double* back, const double* ev) {
    constexpr int NZC = NZ > 0 ? NZ : kMaxNZ;
    const int nz = NZ > 0 ? NZ : g.nz;
    const size_t P = (size_t)g.nkx * g.nky;
    const int kx = (int)(p / g.nky), m = (int)(p % g.nky);
    const double kxv = g.dkx * kx, kyv = g.kyval(g.jfull(m));
    const double k2 = kxv * kxv + kyv * kyv;
    const double dt = M.sc->dt;
    const CT* N0 = static_cast<const CT*>(M.N[0]);
    const CT* N1 = static_cast<const CT*>(M.N[1]);
    const CT* N2 = static_cast<const CT*>(M.N[2]);
    double2 qv[NZC], pv[NZC];
#pragma unroll
    for (int l = 0; l < NZC; ++l) {
        if (l < nz) {
            const size_t idx = (size_t)l * P + p;
            double2 v = M.q[idx];
            if (s == 1) {
                axpy(v, 0.5 * dt, N0[idx]);
            } else if (s == 2) {
                axpy(v, 0.75 * dt, N1[idx]);
            } else if (s == 3) {
                axpy(v, (2.0 / 9.0) * dt, N0[idx]);
                axpy(v, (1.0 / 3.0) * dt, N1[idx]);
                axpy(v, (4.0 / 9.0) * dt, N2[idx]);
            }
            qv[l] = v;
        }
    }
    modal_invert<NZ>(proj, back, ev, M.mc->Htot, nz, k2, p == 0, qv, pv);
    CT* Qs = const_cast<CT*>(stage_input<CT>(M, s));
    CT* psi = static_cast<CT*>(M.psi);
#pragma unroll
    for (int l = 0; l < NZC; ++l) {
        if (l < nz) {
            const size_t idx = (size_t)l * P + p;
            Qs[idx] = to_ct<CT>(qv[l]);
            psi[idx] = to_ct<CT>(pv[l]);
            if (sizeof(CT) == 8 && s == 3) M.qc[idx] = qv[l];
        }
    }
}

template <class CT>
__global__ void __launch_bounds__(256, 2) k_ens_stage(const EnsMember* __restrict__ mem, const int* __restrict__ start,
                                                   int nm, int s) {
    QGN_PDL_ENTRY();
    __shared__ double s_proj[kMaxNZ * kMaxNZ], s_back[kMaxNZ * kMaxNZ], s_ev[kMaxNZ];
    const int total = start[nm];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int mi = ens_find(start, nm, t);
        const EnsMember& M = mem[mi];
        if (!ens_runs(M, s)) continue;
        const Geom g = M.g;
        const int nz = g.nz;
        __syncthreads();   // the previous tile's readers of the mode tables are done
        for (int i = threadIdx.x; i < nz * nz; i += blockDim.x) {
            s_proj[i] = M.mc->proj[i];
            s_back[i] = M.mc->back[i];
        }
        for (int i = threadIdx.x; i < nz; i += blockDim.x) s_ev[i] = M.mc->evals[i];
        __syncthreads();
        const size_t p = (size_t)(t - start[mi]) * kPointTile + threadIdx.x;
        if (p >= (size_t)g.nkx * g.nky) continue;
        switch (nz) {
            case 2: ens_stage_point<2, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            case 3: ens_stage_point<3, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            case 4: ens_stage_point<4, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            case 5: ens_stage_point<5, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            case 6: ens_stage_point<6, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            case 7: ens_stage_point<7, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            case 8: ens_stage_point<8, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            case 16: ens_stage_point<16, CT>(M, g, p, s, s_proj, s_back, s_ev); break;
            default: break;   // qgn_ens_create admits these layer counts only
        }
    }
}

// ---- right-hand-side passes over all members ------------------------------------------------
template <int N, class CT, int TV>
__device__ __noinline__ void ens_yinv_one(const EnsMember& M, const Geom& g, int local, int s) {
    using C = YInvCfg<N, CT, TV>;
    static_assert(C::THREADS == tv_width(TV), "y-inverse tile width must give TV threads");
    const int nbx = (g.nkx + C::TKX - 1) / C::TKX;
    yinv_tile<N, 3, CT, TV>(g, local % nbx, local / nbx, stage_input<CT>(M, s), static_cast<const CT*>(M.psi),
                            static_cast<CT*>(M.hq), static_cast<CT*>(M.hp), static_cast<CT*>(M.hu),
                            static_cast<const CT*>(M.twy));
}

template <class CT, int TV>
__global__ void __launch_bounds__(tv_width(TV), minb(tv_width(TV), ens_regcap<CT, TV>()))
    k_ens_yinv(const EnsMember* __restrict__ mem, const int* __restrict__ start, int nm, int s) {
    QGN_PDL_ENTRY();
    const int total = start[nm];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int mi = ens_find(start, nm, t);
        const EnsMember& M = mem[mi];
        if (!ens_runs(M, s)) continue;
        const Geom g = M.g;
        const int local = t - start[mi];
        switch (g.ny) {
            case 128: ens_yinv_one<128, CT, TV>(M, g, local, s); break;
            case 256: ens_yinv_one<256, CT, TV>(M, g, local, s); break;
            case 512: ens_yinv_one<512, CT, TV>(M, g, local, s); break;
            default: break;
        }
        __syncthreads();   // shared memory is reused by the next tile
    }
}

template <int N, class CT, int TV>
__device__ __noinline__ void ens_xpass_one(const EnsMember& M, const Geom& g, int local) {
    using C = XCfg<N, false, CT, TV>;
    static_assert(C::THREADS == 3 * tv_width(TV), "x-pass tile width must give 3 TV threads");
    const int nbx = (g.ny / 2 + C::RP - 1) / C::RP;
    xpass_tile<N, false, CT, TV>(g, local % nbx, local / nbx, static_cast<const CT*>(M.hq),
                                 static_cast<const CT*>(M.hp), static_cast<const CT*>(M.hu), static_cast<CT*>(M.hpp),
                                 static_cast<CT*>(M.hpd), static_cast<const CT*>(M.twx));
}

template <class CT, int TV>
__global__ void __launch_bounds__(3 * tv_width(TV), minb(3 * tv_width(TV), ens_regcap<CT, TV>()))
    k_ens_xpass(const EnsMember* __restrict__ mem, const int* __restrict__ start, int nm, int s) {
    QGN_PDL_ENTRY();
    const int total = start[nm];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int mi = ens_find(start, nm, t);
        const EnsMember& M = mem[mi];
        if (!ens_runs(M, s)) continue;
        const Geom g = M.g;
        const int local = t - start[mi];
        switch (g.nx) {
            case 128: ens_xpass_one<128, CT, TV>(M, g, local); break;
            case 256: ens_xpass_one<256, CT, TV>(M, g, local); break;
            case 512: ens_xpass_one<512, CT, TV>(M, g, local); break;
            default: break;
        }
        __syncthreads();
    }
}

template <int N, class CT, int TV>
__device__ __noinline__ void ens_yfwd_one(const EnsMember& M, const Geom& g, int local, int s) {
    using C = YFwdCfg<N, false, CT, TV>;
    static_assert(C::THREADS == tv_width(TV), "y-forward tile width must give TV threads");
    const int nbx = (g.nkx + C::TKX - 1) / C::TKX;
    yfwd_tile<N, false, CT, TV>(g, local % nbx, local / nbx, M.lc, stage_input<CT>(M, s),
                                static_cast<const CT*>(M.psi), static_cast<const CT*>(M.hpp),
                                static_cast<const CT*>(M.hpd), static_cast<CT*>(M.N[s]),
                                static_cast<const CT*>(M.twy));
}

template <class CT, int TV>
__global__ void __launch_bounds__(tv_width(TV), minb(tv_width(TV), ens_regcap<CT, TV>()))
    k_ens_yfwd(const EnsMember* __restrict__ mem, const int* __restrict__ start, int nm, int s) {
    QGN_PDL_ENTRY();
    const int total = start[nm];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int mi = ens_find(start, nm, t);
        const EnsMember& M = mem[mi];
        if (!ens_runs(M, s)) continue;
        const Geom g = M.g;
        const int local = t - start[mi];
        switch (g.ny) {
            case 128: ens_yfwd_one<128, CT, TV>(M, g, local, s); break;
            case 256: ens_yfwd_one<256, CT, TV>(M, g, local, s); break;
            case 512: ens_yfwd_one<512, CT, TV>(M, g, local, s); break;
            default: break;
        }
        __syncthreads();
    }
}

// ---- embedded error (BSRK3.f90:30-34), FP64 -------------------------------------------------
template <class CT>
__global__ void __launch_bounds__(256) k_ens_err(EnsMember* __restrict__ mem, const int* __restrict__ start, int nm) {
    QGN_PDL_ENTRY();
    const int total = start[nm];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int mi = ens_find(start, nm, t);
        const EnsMember& M = mem[mi];
        if (!M.active) continue;
        const int local = t - start[mi];
        if (local == 0 && threadIdx.x == 0) {
            M.sc->maxbits = 0ULL;
            M.sc->accept = 0;
        }
        const size_t e = (size_t)local * kPointTile + threadIdx.x;
        if (e >= M.g.csize()) continue;
        double2 v = make_double2(0.0, 0.0);
        axpy(v, 5.0 / 72.0, static_cast<const CT*>(M.N[0])[e]);
        axpy(v, -1.0 / 12.0, static_cast<const CT*>(M.N[1])[e]);
        axpy(v, -1.0 / 9.0, static_cast<const CT*>(M.N[2])[e]);
        axpy(v, 1.0 / 8.0, static_cast<const CT*>(M.N[3])[e]);
        M.err[e] = v;
    }
}

// FP64 y-inverse of the error spectrum, then the x c2r with max|.| (err_phys, BSRK3.f90:35-37)
template <int N>
__device__ __noinline__ void ens_yinv1_one(const EnsMember& M, const Geom& g, int local) {
    using C = YInvCfg<N, double2, 128>;
    static_assert(C::THREADS == 128, "");
    const int nbx = (g.nkx + C::TKX - 1) / C::TKX;
    yinv_tile<N, 1, double2, 128>(g, local % nbx, local / nbx, M.err, nullptr, static_cast<double2*>(M.hq), nullptr,
                                  nullptr, M.twy64);
}

__global__ void __launch_bounds__(128, minb(128)) k_ens_yinv1(const EnsMember* __restrict__ mem,
                                                              const int* __restrict__ start, int nm) {
    QGN_PDL_ENTRY();
    const int total = start[nm];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int mi = ens_find(start, nm, t);
        const EnsMember& M = mem[mi];
        if (!M.active) continue;
        const Geom g = M.g;
        const int local = t - start[mi];
        switch (g.ny) {
            case 128: ens_yinv1_one<128>(M, g, local); break;
            case 256: ens_yinv1_one<256>(M, g, local); break;
            case 512: ens_yinv1_one<512>(M, g, local); break;
            default: break;
        }
        __syncthreads();
    }
}

template <int N>
__device__ __noinline__ void ens_xinv1_one(const EnsMember& M, const Geom& g, int local) {
    using C = X1Cfg<N, 128>;
    static_assert(C::THREADS == 128, "");
    const int nbx = (g.ny / 2 + C::RP - 1) / C::RP;
    xinv1_tile<N, 0, 128>(g, local % nbx, local / nbx, static_cast<const double2*>(M.hq), M.sc, nullptr, M.twx64);
}

__global__ void __launch_bounds__(128, minb(128)) k_ens_xinv1(const EnsMember* __restrict__ mem,
                                                              const int* __restrict__ start, int nm) {
    QGN_PDL_ENTRY();
    const int total = start[nm];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int mi = ens_find(start, nm, t);
        const EnsMember& M = mem[mi];
        if (!M.active) continue;
        const Geom g = M.g;
        const int local = t - start[mi];
        switch (g.nx) {
            case 128: ens_xinv1_one<128>(M, g, local); break;
            case 256: ens_xinv1_one<256>(M, g, local); break;
            case 512: ens_xinv1_one<512>(M, g, local); break;
            default: break;
        }
        __syncthreads();
    }
}

// ---- controller, arming and FSAL bookkeeping ------------------------------------------------
// BSRK3's accept/reject and PI update per member (BSRK3.f90:38-48); an accepted member
// takes q_tmp as its state and RHS3 as RHS0 by swapping table pointers.  The WHILE
// condition of the graph (and *any) says whether a member is still active.
__global__ void __launch_bounds__(256) k_ens_ctrl(EnsMember* __restrict__ mem, int nm,
                                                  cudaGraphConditionalHandle loop, int has_loop, int* __restrict__ any) {
    QGN_PDL_ENTRY();
    int act = 0;
    for (int i = threadIdx.x; i < nm; i += blockDim.x) {
        EnsMember& M = mem[i];
        if (M.active) {
            DevScalars* sc = M.sc;
            ctrl_decide(2, M.g.inv_nxny, M.TOL, M.dt_max, M.max_rejects, sc);
            if (sc->halt) {
                M.active = 0;
            } else if (sc->accept) {
                double2* tq = M.q;
                M.q = M.qc;
                M.qc = tq;
                void* tn = M.N[0];
                M.N[0] = M.N[3];
                M.N[3] = tn;
                sc->rejects_step = 0;
                if (--M.steps_left <= 0) M.active = 0;
            }
        }
        act |= M.active;
    }
    act = __syncthreads_or(act);
    if (threadIdx.x == 0) {
        *any = act;
        if (has_loop) cudaGraphSetConditional(loop, act ? 1u : 0u);
    }
}

__global__ void k_ens_arm(EnsMember* __restrict__ mem, int nm, int nsteps) {
    QGN_PDL_ENTRY();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
        EnsMember& M = mem[i];
        const bool go = nsteps > 0 && M.sc->halt == 0;
        M.steps_left = nsteps;
        M.active = go ? 1 : 0;
        if (go) M.sc->rejects_step = 0;
    }
}

__global__ void k_ens_fsal_done(EnsMember* __restrict__ mem, int nm) {
    QGN_PDL_ENTRY();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x)
        if (mem[i].active) mem[i].need_fsal = 0;
}

// ---- host side --------------------------------------------------------------------------------
// opt a kernel into more than 48 KB of dynamic shared memory once per process, so that no
// attribute call happens while a graph is being captured
template <class K>
cudaError_t smem_attr(K kernel, int bytes) {
    return smem_opt_in(kernel, bytes);
}

template <class CT, int TV>
constexpr int yinv_smem() {
    return cmax(YInvCfg<128, CT, TV>::SMEM, cmax(YInvCfg<256, CT, TV>::SMEM, YInvCfg<512, CT, TV>::SMEM));
}
template <class CT, int TV>
constexpr int xpass_smem() {
    return cmax(XCfg<128, false, CT, TV>::SMEM, cmax(XCfg<256, false, CT, TV>::SMEM, XCfg<512, false, CT, TV>::SMEM));
}
template <class CT, int TV>
constexpr int yfwd_smem() {
    return cmax(YFwdCfg<128, false, CT, TV>::SMEM,
                cmax(YFwdCfg<256, false, CT, TV>::SMEM, YFwdCfg<512, false, CT, TV>::SMEM));
}
constexpr int yinv1_smem() {
    return cmax(YInvCfg<128, double2, 128>::SMEM,
                cmax(YInvCfg<256, double2, 128>::SMEM, YInvCfg<512, double2, 128>::SMEM));
}
constexpr int xinv1_smem() {
    return cmax(X1Cfg<128, 128>::SMEM, cmax(X1Cfg<256, 128>::SMEM, X1Cfg<512, 128>::SMEM));
}

int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// threads per transform of n points at t elements per thread (FFTShape)
int fft_threads(int n, int t) { return n / std::min(n, t); }

// tiles of one member for a pass and tile variant (the tile shapes of YInvCfg, XCfg, YFwdCfg)
int member_tiles(const Geom& g, int pass, int tv) {
    const int w = tv_width(tv), r = tv_radix(tv) ? tv_radix(tv) : 16;
    const int Gx = fft_threads(g.nx, r), Gy = fft_threads(g.ny, r);
    const int G1x = g.nx / 16, G1y = g.ny / 16;   // the error transforms: 16 elements per thread
    switch (pass) {
        case EP_POINT: return ceil_div((long long)g.nkx * g.nky, kPointTile);
        case EP_ELEM: return ceil_div((long long)g.csize(), kPointTile);
        case EP_YINV: return ceil_div(g.nkx, std::max(1, w / Gy)) * g.nz;
        case EP_XPASS: return ceil_div(g.ny / 2, std::max(1, w / Gx)) * g.nz;
        case EP_YFWD: return ceil_div(g.nkx, std::min(std::max(1, w / (2 * Gy)), 16)) * g.nz;
        case EP_YINV1: return ceil_div(g.nkx, 128 / G1y) * g.nz;
        case EP_XINV1: return ceil_div(g.ny / 2, 128 / G1x) * g.nz;
        default: return 0;
    }
}

}  // namespace
}  // namespace qgn

using namespace qgn;

struct qgn_ens {
    std::vector<qgn_ctx*> mem;
    std::vector<long long> seen_version;
    int precision = QGN_PREC_FP64;
    int device = 0;
    cudaStream_t stream = nullptr;
    EnsMember* d_mem = nullptr;
    std::vector<EnsMember> h_mem;
    int* d_start = nullptr;          // EP_COUNT tables of nm+1 prefix sums
    std::vector<int> h_start;
    int* d_any = nullptr;
    int* h_any = nullptr;            // pinned
    int variant[TP_COUNT] = {kDefaultVariant, kDefaultVariant, kDefaultVariant};
    int grid_mode[TP_COUNT] = {0, 0, 0};   // 0: one CTA per tile; k > 0: k CTAs per SM, persistent
    float tuned_ms[TP_COUNT] = {0.f, 0.f, 0.f};
    bool pinned[TP_COUNT] = {false, false, false};   // set by qgn_ens_set_tiles: not tuned
    bool tuned = false;
    bool graphs_off = false;
    cudaGraphExec_t gexec = nullptr;
    long long g_body[KID_COUNT] = {};
    long long g_root[KID_COUNT] = {};
    Prof prof;
    std::string last_error;
    int sms = 148;
};

namespace {

struct EnsProfScope {
    Prof* prev;
    explicit EnsProfScope(qgn_ens* e) : prev(current_prof()) { current_prof() = &e->prof; }
    ~EnsProfScope() { current_prof() = prev; }
};

int ens_err(qgn_ens* e, int code, const std::string& msg) {
    e->last_error = msg;
    return code;
}

#define ECK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t _e = (call);                                                                    \
        if (_e != cudaSuccess) {                                                                    \
            char _b[512];                                                                           \
            std::snprintf(_b, sizeof(_b), "%s: %s (%s)", #call, cudaGetErrorString(_e), cudaGetErrorName(_e)); \
            return ens_err(e, QGN_ERR_CUDA, _b);                                                    \
        }                                                                                           \
    } while (0)

bool fp32(const qgn_ens* e) { return e->precision == QGN_PREC_MIXED; }

int tv_of(const qgn_ens* e, int tp) {
    return fp32(e) ? ens_variant<float2>(tp, e->variant[tp]) : ens_variant<double2>(tp, e->variant[tp]);
}
int variant_count(const qgn_ens* e, int tp) {
    return fp32(e) ? ens_variant_count<float2>(tp) : ens_variant_count<double2>(tp);
}

const int* start_of(const qgn_ens* e, int pass) { return e->d_start + (size_t)pass * (e->mem.size() + 1); }

int total_of(const qgn_ens* e, int pass) { return e->h_start[(size_t)pass * (e->mem.size() + 1) + e->mem.size()]; }

int grid_for(const qgn_ens* e, int pass, int tp) {
    const int total = total_of(e, pass);
    if (tp < 0 || e->grid_mode[tp] == 0) return std::max(1, total);
    return std::max(1, std::min(total, e->sms * e->grid_mode[tp]));
}

void build_tables(qgn_ens* e) {
    const size_t nm = e->mem.size();
    e->h_start.assign((size_t)EP_COUNT * (nm + 1), 0);
    for (int pass = 0; pass < EP_COUNT; ++pass) {
        int tv = 0;
        if (pass == EP_YINV) tv = tv_of(e, TP_YINV);
        if (pass == EP_XPASS) tv = tv_of(e, TP_XPASS);
        if (pass == EP_YFWD) tv = tv_of(e, TP_YFWD);
        int* st = &e->h_start[(size_t)pass * (nm + 1)];
        for (size_t m = 0; m < nm; ++m) st[m + 1] = st[m] + member_tiles(e->mem[m]->g, pass, tv);
    }
}

int upload_tables(qgn_ens* e) {
    ECK(cudaMemcpyAsync(e->d_start, e->h_start.data(), sizeof(int) * e->h_start.size(), cudaMemcpyHostToDevice,
                        e->stream));
    return QGN_OK;
}

// member table from the contexts' current buffers
void fill_members(qgn_ens* e) {
    const bool f = fp32(e);
    for (size_t m = 0; m < e->mem.size(); ++m) {
        qgn_ctx* c = e->mem[m];
        Buffers& b = c->b;
        EnsMember& M = e->h_mem[m];
        std::memset(&M, 0, sizeof(M));
        M.g = c->g;
        M.q = b.q;
        M.qc = b.qnew;
        M.err = b.err;
        for (int j = 0; j < 4; ++j) M.N[j] = b.N[j];
        M.Qs = b.Qs[1];
        M.psi = b.psi;
        M.hq = b.hq;
        M.hp = b.hp;
        M.hu = b.hu;
        M.hpp = b.hpp;
        M.hpd = b.hpd;
        M.twx = f ? (const void*)b.twx32 : (const void*)b.twx;
        M.twy = f ? (const void*)b.twy32 : (const void*)b.twy;
        M.twx64 = b.twx;
        M.twy64 = b.twy;
        M.lc = b.lc;
        M.mc = b.mc;
        M.sc = b.sc;
        M.TOL = c->p.TOL;
        M.dt_max = c->p.dt_max;
        M.max_rejects = c->p.max_rejects > 0 ? c->p.max_rejects : 64;
        M.need_fsal = (e->seen_version[m] != c->state_version) ? 1 : 0;
    }
}

// ---- launches -------------------------------------------------------------------------------------
template <class CT>
int launch_stage(qgn_ens* e, int s) {
    double bytes = 0.0;
    for (qgn_ctx* c : e->mem) bytes += (double)c->g.csize() * (16.0 + 2.0 * sizeof(CT) + (s == 3 ? 3 : (s ? 1 : 0)) * sizeof(CT));
    QGN_LAUNCH(KID_STAGE, bytes, e->stream,
               ::qgn::launch(k_ens_stage<CT>, grid_for(e, EP_POINT, -1), kPointTile, 0, e->stream, e->d_mem, start_of(e, EP_POINT),
                                                                                        (int)e->mem.size(), s));
    ECK(cudaGetLastError());
    return QGN_OK;
}

template <class CT, int TV>
int launch_yinv_tv(qgn_ens* e, int s, int grid) {
    constexpr int SM = yinv_smem<CT, TV>();
    ECK(smem_attr(k_ens_yinv<CT, TV>, SM));
    double bytes = 0.0;
    for (qgn_ctx* c : e->mem) bytes += sizeof(CT) * (2.0 * c->g.csize() + 3.0 * c->g.nz * c->g.ny * c->g.nkx);
    QGN_LAUNCH(KID_YINV, bytes, e->stream,
               ::qgn::launch(k_ens_yinv<CT, TV>, grid, tv_width(TV), SM, e->stream, e->d_mem, start_of(e, EP_YINV),
                             (int)e->mem.size(), s));
    ECK(cudaGetLastError());
    return QGN_OK;
}

template <class CT, int TV>
int launch_xpass_tv(qgn_ens* e, int s, int grid) {
    constexpr int SM = xpass_smem<CT, TV>();
    ECK(smem_attr(k_ens_xpass<CT, TV>, SM));
    double bytes = 0.0;
    for (qgn_ctx* c : e->mem) bytes += 5.0 * sizeof(CT) * c->g.nz * c->g.ny * c->g.nkx;
    QGN_LAUNCH(KID_XPASS, bytes, e->stream,
               ::qgn::launch(k_ens_xpass<CT, TV>, grid, 3 * tv_width(TV), SM, e->stream, e->d_mem, start_of(e, EP_XPASS),
                                                                   (int)e->mem.size(), s));
    ECK(cudaGetLastError());
    return QGN_OK;
}

template <class CT, int TV>
int launch_yfwd_tv(qgn_ens* e, int s, int grid) {
    constexpr int SM = yfwd_smem<CT, TV>();
    ECK(smem_attr(k_ens_yfwd<CT, TV>, SM));
    double bytes = 0.0;
    for (qgn_ctx* c : e->mem) bytes += sizeof(CT) * c->g.nz * c->g.nkx * (2.0 * c->g.ny + 3.0 * c->g.nky);
    QGN_LAUNCH(KID_YFWD, bytes, e->stream,
               ::qgn::launch(k_ens_yfwd<CT, TV>, grid, tv_width(TV), SM, e->stream, e->d_mem, start_of(e, EP_YFWD),
                             (int)e->mem.size(), s));
    ECK(cudaGetLastError());
    return QGN_OK;
}

// variant v of a pass: the I-th instantiation of the pass's list for I == v
template <class CT, size_t... I>
int launch_yinv_v(qgn_ens* e, int v, int s, std::index_sequence<I...>) {
    int r = QGN_ERR_CONFIG;
    const int grid = grid_for(e, EP_YINV, TP_YINV);
    (void)((v == (int)I ? (r = launch_yinv_tv<CT, ens_variant<CT>(TP_YINV, (int)I)>(e, s, grid), true) : false) || ...);
    return r;
}
template <class CT, size_t... I>
int launch_xpass_v(qgn_ens* e, int v, int s, std::index_sequence<I...>) {
    int r = QGN_ERR_CONFIG;
    const int grid = grid_for(e, EP_XPASS, TP_XPASS);
    (void)((v == (int)I ? (r = launch_xpass_tv<CT, ens_variant<CT>(TP_XPASS, (int)I)>(e, s, grid), true) : false) || ...);
    return r;
}
template <class CT, size_t... I>
int launch_yfwd_v(qgn_ens* e, int v, int s, std::index_sequence<I...>) {
    int r = QGN_ERR_CONFIG;
    const int grid = grid_for(e, EP_YFWD, TP_YFWD);
    (void)((v == (int)I ? (r = launch_yfwd_tv<CT, ens_variant<CT>(TP_YFWD, (int)I)>(e, s, grid), true) : false) || ...);
    return r;
}

template <class CT>
int launch_pass(qgn_ens* e, int tp, int s) {
    const int v = e->variant[tp];
    if (tp == TP_YINV) return launch_yinv_v<CT>(e, v, s, std::make_index_sequence<ens_variant_count<CT>(TP_YINV)>{});
    if (tp == TP_XPASS) return launch_xpass_v<CT>(e, v, s, std::make_index_sequence<ens_variant_count<CT>(TP_XPASS)>{});
    return launch_yfwd_v<CT>(e, v, s, std::make_index_sequence<ens_variant_count<CT>(TP_YFWD)>{});
}

template <class CT>
int launch_rhs_all(qgn_ens* e, int s) {
    for (int tp = 0; tp < TP_COUNT; ++tp) {
        int r = launch_pass<CT>(e, tp, s);
        if (r != QGN_OK) return r;
    }
    return QGN_OK;
}

template <class CT>
int launch_fsal(qgn_ens* e) {
    int r = launch_stage<CT>(e, 0);
    if (r == QGN_OK) r = launch_rhs_all<CT>(e, 0);
    if (r != QGN_OK) return r;
    QGN_LAUNCH(KID_SCALAR, 0.0, e->stream, ::qgn::launch(k_ens_fsal_done, 1, 256, 0, e->stream, e->d_mem, (int)e->mem.size()));
    ECK(cudaGetLastError());
    return QGN_OK;
}

template <class CT>
int launch_attempt(qgn_ens* e, const cudaGraphConditionalHandle* loop) {
    for (int s = 1; s <= 3; ++s) {
        int r = launch_stage<CT>(e, s);
        if (r == QGN_OK) r = launch_rhs_all<CT>(e, s);
        if (r != QGN_OK) return r;
    }
    double eb = 0.0, yb = 0.0, xb = 0.0;
    for (qgn_ctx* c : e->mem) {
        eb += (double)c->g.csize() * (4.0 * sizeof(CT) + 16.0);
        yb += 16.0 * ((double)c->g.csize() + (double)c->g.nz * c->g.ny * c->g.nkx);
        xb += 16.0 * (double)c->g.nz * c->g.ny * c->g.nkx;
    }
    const int nm = (int)e->mem.size();
    QGN_LAUNCH(KID_LINCOMB, eb, e->stream,
               ::qgn::launch(k_ens_err<CT>, grid_for(e, EP_ELEM, -1), kPointTile, 0, e->stream, e->d_mem, start_of(e, EP_ELEM), nm));
    ECK(cudaGetLastError());
    ECK(smem_attr(k_ens_yinv1, yinv1_smem()));
    QGN_LAUNCH(KID_YINV, yb, e->stream,
               ::qgn::launch(k_ens_yinv1, grid_for(e, EP_YINV1, -1), 128, yinv1_smem(), e->stream, e->d_mem, start_of(e, EP_YINV1),
                                                                                      nm));
    ECK(cudaGetLastError());
    ECK(smem_attr(k_ens_xinv1, xinv1_smem()));
    QGN_LAUNCH(KID_XINV1, xb, e->stream,
               ::qgn::launch(k_ens_xinv1, grid_for(e, EP_XINV1, -1), 128, xinv1_smem(), e->stream, e->d_mem, start_of(e, EP_XINV1),
                                                                                      nm));
    ECK(cudaGetLastError());
    QGN_LAUNCH(KID_SCALAR, 0.0, e->stream,
               ::qgn::launch(k_ens_ctrl, 1, 256, 0, e->stream, e->d_mem, nm, loop ? *loop : 0, loop ? 1 : 0, e->d_any));
    ECK(cudaGetLastError());
    return QGN_OK;
}

int attempt(qgn_ens* e, const cudaGraphConditionalHandle* loop) {
    QGN_NVTX("ensemble attempt");
    return fp32(e) ? launch_attempt<float2>(e, loop) : launch_attempt<double2>(e, loop);
}
int fsal(qgn_ens* e) { return fp32(e) ? launch_fsal<float2>(e) : launch_fsal<double2>(e); }

// ---- autotuner: per right-hand-side pass, the tile-width variant and grid size with the
// shortest event-timed launch on this ensemble (outputs are scratch: stage 1's RHS1 and
// half-transformed fields, which the first attempt overwrites) ------------------------------
int autotune(qgn_ens* e) {
    cudaEvent_t a, b;
    ECK(cudaEventCreate(&a));
    ECK(cudaEventCreate(&b));
    const bool timing = e->prof.timing;
    e->prof.timing = false;
    long long launches0[KID_COUNT];
    for (int k = 0; k < KID_COUNT; ++k) launches0[k] = e->prof.launches[k];
    int rc = QGN_OK;
    const int grid_modes[4] = {0, 2, 4, 8};
    for (int tp = 0; tp < TP_COUNT && rc == QGN_OK; ++tp) {
        if (e->pinned[tp]) continue;
        float best = 1e30f;
        int bv = kDefaultVariant, bg = 0;
        for (int v = 0; v < variant_count(e, tp) && rc == QGN_OK; ++v) {
            e->variant[tp] = v;
            build_tables(e);
            rc = upload_tables(e);
            for (int gm = 0; gm < 4 && rc == QGN_OK; ++gm) {
                e->grid_mode[tp] = grid_modes[gm];
                const int reps = 5;
                rc = fp32(e) ? launch_pass<float2>(e, tp, 1) : launch_pass<double2>(e, tp, 1);   // warm-up
                if (rc != QGN_OK) break;
                if (cudaEventRecord(a, e->stream) != cudaSuccess) { rc = QGN_ERR_CUDA; break; }
                for (int r = 0; r < reps && rc == QGN_OK; ++r)
                    rc = fp32(e) ? launch_pass<float2>(e, tp, 1) : launch_pass<double2>(e, tp, 1);
                if (rc != QGN_OK) break;
                if (cudaEventRecord(b, e->stream) != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess) {
                    rc = QGN_ERR_CUDA;
                    break;
                }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, a, b);
                ms /= reps;
                if (ms < best) {
                    best = ms;
                    bv = v;
                    bg = grid_modes[gm];
                }
            }
        }
        e->variant[tp] = bv;
        e->grid_mode[tp] = bg;
        e->tuned_ms[tp] = best;
    }
    e->prof.timing = timing;
    for (int k = 0; k < KID_COUNT; ++k) e->prof.launches[k] = launches0[k];
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc != QGN_OK) return rc == QGN_ERR_CUDA && e->last_error.empty() ? ens_err(e, rc, "autotune failed") : rc;
    build_tables(e);
    return upload_tables(e);
}

int add_while(qgn_ens* e, cudaGraphConditionalHandle h, cudaGraph_t* body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    ECK(cudaStreamGetCaptureInfo(e->stream, &cs, nullptr, &graph, &deps, &nd));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    ECK(cudaGraphAddNode(&node, graph, deps, nd, &np));
    ECK(cudaStreamUpdateCaptureDependencies(e->stream, &node, 1, cudaStreamSetCaptureDependencies));
    *body = np.conditional.phGraph_out[0];
    return QGN_OK;
}

// root: FSAL pass (members that need RHS0) -> WHILE(any active) { attempt }
int capture(qgn_ens* e) {
    cudaGraph_t root = nullptr;
    long long c0[KID_COUNT], c1[KID_COUNT], c2[KID_COUNT];
    const bool timing = e->prof.timing;
    e->prof.timing = false;
    auto run = [&]() -> int {
        ECK(cudaGraphCreate(&root, 0));
        cudaGraphConditionalHandle hloop;
        ECK(cudaGraphConditionalHandleCreate(&hloop, root, 1u, cudaGraphCondAssignDefault));
        for (int k = 0; k < KID_COUNT; ++k) c0[k] = e->prof.launches[k];
        ECK(cudaStreamBeginCaptureToGraph(e->stream, root, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        int r = fsal(e);
        cudaGraph_t wbody = nullptr;
        if (r == QGN_OK) r = add_while(e, hloop, &wbody);
        cudaGraph_t tmp = nullptr;
        ECK(cudaStreamEndCapture(e->stream, &tmp));
        if (r != QGN_OK) return r;
        for (int k = 0; k < KID_COUNT; ++k) c1[k] = e->prof.launches[k];
        ECK(cudaStreamBeginCaptureToGraph(e->stream, wbody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        r = attempt(e, &hloop);
        ECK(cudaStreamEndCapture(e->stream, &tmp));
        if (r != QGN_OK) return r;
        for (int k = 0; k < KID_COUNT; ++k) c2[k] = e->prof.launches[k];
        ECK(cudaGraphInstantiate(&e->gexec, root, 0));
        return QGN_OK;
    };
    const int rc = run();
    e->prof.timing = timing;
    if (root) cudaGraphDestroy(root);
    for (int k = 0; k < KID_COUNT; ++k) {
        e->g_root[k] = c1[k] - c0[k];
        e->g_body[k] = c2[k] - c1[k];
        e->prof.launches[k] = c0[k];
    }
    return rc;
}

int read_member_scalars(qgn_ens* e, std::vector<DevScalars>& out) {
    out.resize(e->mem.size());
    for (size_t m = 0; m < e->mem.size(); ++m)
        ECK(cudaMemcpyAsync(&out[m], e->mem[m]->b.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, e->stream));
    ECK(cudaStreamSynchronize(e->stream));
    return QGN_OK;
}

}  // namespace

extern "C" {

int qgn_ens_create(qgn_ctx* const* members, int nmembers, int precision, qgn_ens** out) {
    if (!out) return QGN_ERR_ARG;
    *out = nullptr;
    if (!members || nmembers < 1 || nmembers > 4096) return QGN_ERR_ARG;
    if (precision != QGN_PREC_FP64 && precision != QGN_PREC_MIXED) return QGN_ERR_CONFIG;
    for (int m = 0; m < nmembers; ++m) {
        const qgn_ctx* c = members[m];
        if (!c) return QGN_ERR_ARG;
        if (c->scheme != QGN_SCHEME_BSRK3 || c->precision != QGN_PREC_FP64) return QGN_ERR_CONFIG;
        const int nx = c->g.nx, ny = c->g.ny;
        auto ok = [](int n) { return n == 128 || n == 256 || n == 512; };
        if (!ok(nx) || !ok(ny) || c->p.C_d != 0.0) return QGN_ERR_CONFIG;
        if (!(c->g.nz >= 2 && c->g.nz <= 8) && c->g.nz != 16) return QGN_ERR_CONFIG;
        if (c->device != members[0]->device) return QGN_ERR_CONFIG;
        for (int k = 0; k < m; ++k)
            if (members[k] == c) return QGN_ERR_ARG;
    }
    qgn_ens* e = new (std::nothrow) qgn_ens();
    if (!e) return QGN_ERR_CUDA;
    e->mem.assign(members, members + nmembers);
    e->seen_version.assign(nmembers, -1);
    e->precision = precision;
    e->device = members[0]->device;
    e->h_mem.resize(nmembers);
    e->graphs_off = std::getenv("QGN_NO_GRAPHS") != nullptr;
    auto fail = [&](int code) {
        qgn_ens_destroy(e);
        return code;
    };
    if (cudaSetDevice(e->device) != cudaSuccess) return fail(QGN_ERR_CUDA);
    cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->device);
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(QGN_ERR_CUDA);
    if (cudaMalloc((void**)&e->d_mem, sizeof(EnsMember) * nmembers) != cudaSuccess) return fail(QGN_ERR_CUDA);
    if (cudaMalloc((void**)&e->d_start, sizeof(int) * (size_t)EP_COUNT * (nmembers + 1)) != cudaSuccess)
        return fail(QGN_ERR_CUDA);
    if (cudaMalloc((void**)&e->d_any, sizeof(int)) != cudaSuccess) return fail(QGN_ERR_CUDA);
    if (cudaMallocHost((void**)&e->h_any, sizeof(int)) != cudaSuccess) return fail(QGN_ERR_CUDA);
    build_tables(e);
    *out = e;
    return QGN_OK;
}

int qgn_ens_advance(qgn_ens* e, int nsteps) {
    QGN_NVTX("qgn_ens_advance");
    if (!e) return QGN_ERR_ARG;
    if (nsteps < 0) return ens_err(e, QGN_ERR_ARG, "nsteps < 0");
    EnsProfScope ps_(e);
    ECK(cudaSetDevice(e->device));
    const int nm = (int)e->mem.size();
    // members' own work (state uploads) precedes the ensemble's
    for (qgn_ctx* c : e->mem) ECK(cudaStreamSynchronize(c->stream));
    fill_members(e);
    ECK(cudaMemcpyAsync(e->d_mem, e->h_mem.data(), sizeof(EnsMember) * nm, cudaMemcpyHostToDevice, e->stream));
    int rc = upload_tables(e);
    if (rc != QGN_OK) return rc;
    QGN_LAUNCH(KID_SCALAR, 0.0, e->stream, ::qgn::launch(k_ens_arm, (nm + 255) / 256, 256, 0, e->stream, e->d_mem, nm, nsteps));
    ECK(cudaGetLastError());
    std::vector<DevScalars> s0, s1;
    if (!e->tuned && nsteps > 0) {
        // RHS0 with the default tiles, then tune on real fields
        rc = fsal(e);
        if (rc != QGN_OK) return rc;
        if (!std::getenv("QGN_NO_AUTOTUNE")) {
            rc = autotune(e);
            if (rc != QGN_OK) return rc;
        }
        e->tuned = true;
    }
    const bool use_graph = !e->graphs_off && !e->prof.timing;
    if (use_graph && !e->gexec) {
        rc = capture(e);
        if (rc != QGN_OK) {
            if (e->gexec) {
                cudaGraphExecDestroy(e->gexec);
                e->gexec = nullptr;
            }
            cudaGetLastError();
            e->graphs_off = true;
        }
    }
    rc = read_member_scalars(e, s0);
    if (rc != QGN_OK) return rc;
    if (nsteps > 0) {
        if (use_graph && e->gexec) {
            ECK(cudaGraphLaunch(e->gexec, e->stream));
        } else {
            rc = fsal(e);
            if (rc != QGN_OK) return rc;
            // bounded: every member halts after max_rejects consecutive rejections
            long long guard = 0;
            long long limit = 0;
            for (const EnsMember& M : e->h_mem) limit += (long long)nsteps * (M.max_rejects + 1);
            for (;;) {
                rc = attempt(e, nullptr);
                if (rc != QGN_OK) return rc;
                ECK(cudaMemcpyAsync(e->h_any, e->d_any, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
                ECK(cudaStreamSynchronize(e->stream));
                e->prof.harvest();
                if (!*e->h_any || ++guard > limit) break;
            }
        }
    }
    rc = read_member_scalars(e, s1);
    if (rc != QGN_OK) return rc;
    if (use_graph && e->gexec && nsteps > 0) {
        // every attempt covers all members: the body ran as often as the busiest member attempted
        long long body_runs = 0;
        for (int m = 0; m < nm; ++m) body_runs = std::max(body_runs, s1[m].attempts - s0[m].attempts);
        for (int k = 0; k < KID_COUNT; ++k) e->prof.launches[k] += e->g_root[k] + body_runs * e->g_body[k];
    }
    // the device table holds the swapped state / RHS0 pointers: hand them back to the members
    ECK(cudaMemcpyAsync(e->h_mem.data(), e->d_mem, sizeof(EnsMember) * nm, cudaMemcpyDeviceToHost, e->stream));
    ECK(cudaStreamSynchronize(e->stream));
    e->prof.harvest();
    int first_bad = -1;
    for (int m = 0; m < nm; ++m) {
        qgn_ctx* c = e->mem[m];
        const EnsMember& M = e->h_mem[m];
        c->b.q = M.q;
        c->b.qnew = M.qc;
        c->b.N[0] = static_cast<double2*>(M.N[0]);
        c->b.N[3] = static_cast<double2*>(M.N[3]);
        c->b.Qs[0] = c->b.q;
        // an FP64 ensemble leaves a valid FP64 RHS0 for the member's own BSRK3 steps
        c->first_call = fp32(e) || M.need_fsal != 0;
        e->seen_version[m] = c->state_version;
        if (s1[m].halt) {
            c->halted = true;
            if (first_bad < 0) first_bad = m;
        }
    }
    if (first_bad >= 0) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "member %d halted: %s", first_bad,
                      s1[first_bad].status == QGN_ERR_NONFINITE ? "non-finite embedded error estimate"
                                                                : "adaptive step rejected max_rejects times in a row");
        return ens_err(e, s1[first_bad].status ? s1[first_bad].status : QGN_ERR_CUDA, buf);
    }
    return QGN_OK;
}

int qgn_ens_tuning(qgn_ens* e, int pass, int* threads, int* ctas_per_sm, float* ms) {
    if (!e || pass < 0 || pass >= TP_COUNT) return QGN_ERR_ARG;
    const int w = tv_width(tv_of(e, pass));
    if (threads) *threads = pass == TP_XPASS ? 3 * w : w;
    if (ctas_per_sm) *ctas_per_sm = e->grid_mode[pass];
    if (ms) *ms = e->tuned_ms[pass];
    return QGN_OK;
}

int qgn_ens_fft_radix(qgn_ens* e, int pass, int* elements_per_thread) {
    if (!e || !elements_per_thread || pass < 0 || pass >= TP_COUNT) return QGN_ERR_ARG;
    const int r = tv_radix(tv_of(e, pass));
    *elements_per_thread = r ? r : 16;
    return QGN_OK;
}

int qgn_ens_set_tiles(qgn_ens* e, int pass, int threads, int elements_per_thread, int ctas_per_sm) {
    if (!e || pass < 0 || pass >= TP_COUNT || ctas_per_sm < 0 || ctas_per_sm > 64) return QGN_ERR_ARG;
    const int w = pass == TP_XPASS ? threads / 3 : threads;
    if (pass == TP_XPASS && threads % 3 != 0) return ens_err(e, QGN_ERR_CONFIG, "x-pass threads: three slot groups");
    for (int v = 0; v < variant_count(e, pass); ++v) {
        const int tv = fp32(e) ? ens_variant<float2>(pass, v) : ens_variant<double2>(pass, v);
        if (tv_width(tv) == w && (tv_radix(tv) ? tv_radix(tv) : 16) == elements_per_thread) {
            e->variant[pass] = v;
            e->grid_mode[pass] = ctas_per_sm;
            e->pinned[pass] = true;
            e->tuned_ms[pass] = 0.f;
            build_tables(e);
            if (e->gexec) {   // the captured graph holds the old launches
                ECK(cudaStreamSynchronize(e->stream));
                cudaGraphExecDestroy(e->gexec);
                e->gexec = nullptr;
            }
            return QGN_OK;
        }
    }
    return ens_err(e, QGN_ERR_CONFIG, "no tile variant with these threads and elements per thread");
}

int qgn_ens_profile_enable(qgn_ens* e, int on) {
    if (!e) return QGN_ERR_ARG;
    e->prof.reset();
    e->prof.timing = on != 0;
    return QGN_OK;
}

int qgn_ens_profile_read(qgn_ens* e, int kernel, double* ms, double* bytes, long long* timed, long long* launches) {
    if (!e || kernel < 0 || kernel >= KID_COUNT) return QGN_ERR_ARG;
    e->prof.harvest();
    if (ms) *ms = e->prof.total_ms[kernel];
    if (bytes) *bytes = e->prof.bytes[kernel];
    if (timed) *timed = e->prof.timed[kernel];
    if (launches) *launches = e->prof.launches[kernel];
    return QGN_OK;
}

int qgn_ens_stream(qgn_ens* e, void** stream) {
    if (!e || !stream) return QGN_ERR_ARG;
    *stream = e->stream;
    return QGN_OK;
}

const char* qgn_ens_last_error(qgn_ens* e) { return e ? e->last_error.c_str() : "NULL ensemble"; }

int qgn_ens_destroy(qgn_ens* e) {
    if (!e) return QGN_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    e->prof.release();
    if (e->d_mem) cudaFree(e->d_mem);
    if (e->d_start) cudaFree(e->d_start);
    if (e->d_any) cudaFree(e->d_any);
    if (e->h_any) cudaFreeHost(e->h_any);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return QGN_OK;
}

}  // extern "C"
