// closure.cu -- the learned subgrid closure of a coarse QGN model and its training data.
//
// Training data: the high-resolution model's state is coarse-grained by a sharp spectral
// cutoff onto the coarse grid's kept modes (qgn_coarse_grain); the subgrid PV tendency is the
// coarse-grained high-resolution right-hand side minus the coarse model's right-hand side of
// the coarse-grained state,
//     S = trunc(GetRHS_fine(q)) - GetRHS_coarse(trunc(q)),
// in which every linear term cancels and the difference of the Jacobians remains.  A sample
// is the network input (q, psi of every layer, physical, scaled, BF16) and target (S,
// physical, scaled, FP32) on the coarse grid.
//
// Closure: in the ARK43_QGLeith prologue of a context with an attached network, the network
// maps the state's physical q, psi to S; S (forward-transformed, dealiased) is added to every
// stage right-hand side inside the y-forward assembly.  An energy-budget check on the applied
// tendency, in FP64,
//     dZ = sum_l H_l/Htot <q_l S_l> <= 0            (the closure removes enstrophy)
//     dE = -sum_l H_l/Htot <psi_l S_l> <= limit * E / day,  E = -1/2 sum_l H_l/Htot <psi_l q_l>,
// decides per step: passing, the step uses S with the background hyperviscosity A8_background;
// failing, S is dropped and the step is plain QG-Leith (ARK43_QGLeith.f90:62-73).  The
// averages are Parseval sums over the kept modes, so the check costs one launch.
#include "qgn_internal.cuh"
#include "cnn.cuh"
#include "prof.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

namespace qgn {

struct ClosureStats {
    long long evaluations;
    long long fallbacks;
    double dE, dZ, E;
    int pass;
    unsigned int red_count;     // blocks done in the budget kernel's last-block reduction
};

struct Closure {
    qgn_cnn* net = nullptr;
    float* scales = nullptr;          // device: in [2 nz], out [nz]
    __nv_bfloat16* x = nullptr;       // [ny][nx][cin_p]
    float* y = nullptr;               // [cout_p][ny*nx] (planar network output)
    double2* S = nullptr;             // compact closure tendency
    double2* psi = nullptr;           // GetPsi of the state (compact), the closure's own copy
    double2* hq = nullptr;            // packed-row scratch of the input and output transforms
    double2* hu = nullptr;
    cudaStream_t side = nullptr;      // the closure's stream when it runs beside the first RHS
    cudaEvent_t fork = nullptr, join = nullptr;
    double* red = nullptr;            // 3 x nblocks partial sums
    double* flag = nullptr;           // 1 passing, 0 fallback
    ClosureStats* stats = nullptr;
    double A8bg = 0.0, elimit = 0.0;
    int nblocks = 0, cin_p = 0, cout_p = 0;
};

namespace {

constexpr int kBudgetBlocks = 148;

// sharp spectral cutoff: coarse compact <- fine compact on the coarse grid's kept modes,
// rescaled for the unnormalised transforms
__global__ void k_truncate(Geom gf, Geom gc, const double2* __restrict__ src, double2* __restrict__ dst, double scale) {
    QGN_PDL_ENTRY();
    const size_t n = gc.csize();
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(e % gc.nky);
        const size_t r = e / gc.nky;
        const int kx = (int)(r % gc.nkx);
        const int l = (int)(r / gc.nkx);
        const int jc = gc.jfull(m);
        const int jf = jc <= gc.ny / 2 ? jc : jc - gc.ny + gf.ny;
        const int mf = jf < gf.kylo ? jf : jf - gf.kyshift;
        const double2 v = src[((size_t)l * gf.nkx + kx) * gf.nky + mf];
        dst[e] = (kx == 0 && m == 0) ? make_double2(0.0, 0.0) : make_double2(v.x * scale, v.y * scale);
    }
}

__global__ void k_copy_time(const DevScalars* __restrict__ a, DevScalars* __restrict__ b) {
    QGN_PDL_ENTRY();
    b->t = a->t;
    b->dt = a->dt;
    b->halt = 0;
    b->status = 0;
    b->nonfinite = 0;
}

__global__ void k_sub(size_t n, const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ o) {
    QGN_PDL_ENTRY();
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        o[e] = make_double2(a[e].x - b[e].x, a[e].y - b[e].y);
}

// network input x[p][c]: c < nz -> q_c, nz <= c < 2 nz -> psi_{c-nz}, scaled; zeros beyond
__global__ void k_pack_in(int nz, size_t npix, const double* __restrict__ q, const double* __restrict__ psi,
                          const float* __restrict__ sc, int cin_p, __nv_bfloat16* __restrict__ x) {
    QGN_PDL_ENTRY();
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
        __nv_bfloat16* xp = x + p * cin_p;
        for (int c = 0; c < cin_p; ++c) {
            float v = 0.f;
            if (c < nz) v = (float)q[(size_t)c * npix + p] * sc[c];
            else if (c < 2 * nz) v = (float)psi[(size_t)(c - nz) * npix + p] * sc[c];
            xp[c] = __float2bfloat16_rn(v);
        }
    }
}

// training target y[p][c] = S_c * out_scale_c (c < nz), zeros beyond
__global__ void k_pack_out(int nz, size_t npix, const double* __restrict__ s, const float* __restrict__ osc, int cout_p,
                           float* __restrict__ y) {
    QGN_PDL_ENTRY();
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x)
        for (int c = 0; c < cout_p; ++c) y[p * cout_p + c] = c < nz ? (float)s[(size_t)c * npix + p] * osc[c] : 0.f;
}

// The energy-budget check of the applied tendency S (compact, dealiased) in one launch, by
// Parseval on the kept modes (the kx = 0 column in the Hermitian projection that the
// inverse transform applies):
//   <a b> = sum over the full plane of Re(conj(a_k) b_k) / (nx ny)^2,
//   dE = -sum_l w_l <psi_l S_l>,  dZ = sum_l w_l <q_l S_l>,  E = -1/2 sum_l w_l <psi_l q_l>.
// Each block writes its partial sums; the block that finishes last (counted in st->red_count)
// adds them in a fixed order, decides, updates the statistics, and keeps S with the
// background A8 or zeroes S (plain QG-Leith for the step).
__device__ __forceinline__ double2 herm_proj(const Geom& g, const double2* __restrict__ f, size_t lP, int m, bool& pk) {
    const int j = g.jfull(m);
    const int jp = (g.ny - j) % g.ny;
    pk = (jp < g.kylo) || (jp >= g.kylo + g.kyshift);
    const double2 v = f[lP + m];
    double2 fp = make_double2(0.0, 0.0);
    if (pk) fp = f[lP + (jp < g.kylo ? jp : jp - g.kyshift)];
    return make_double2(0.5 * (v.x + fp.x), 0.5 * (v.y - fp.y));
}

__global__ void __launch_bounds__(256) k_budget_spec(Geom g, const double2* __restrict__ q,
                                                     const double2* __restrict__ psi, double2* __restrict__ S,
                                                     const double* __restrict__ Hw, double* __restrict__ red,
                                                     double A8bg, double elimit, DevScalars* __restrict__ sc,
                                                     ClosureStats* __restrict__ st, double* __restrict__ flag) {
    QGN_PDL_ENTRY();
    __shared__ double sm[3][8];
    __shared__ unsigned s_last;
    const size_t P = (size_t)g.nkx * g.nky;
    const int nb = gridDim.x;
    double a = 0.0, b = 0.0, c = 0.0;
    const size_t ne = (size_t)g.nz * P;   // one (layer, mode) per thread and pass
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (size_t)gridDim.x * blockDim.x) {
        const int l = (int)(e / P);
        const size_t p = e - (size_t)l * P;
        const int kx = (int)(p / g.nky), m = (int)(p % g.nky);
        {
            const size_t lP = (size_t)l * P;
            double2 hq, hp, hs;
            double f;
            if (kx > 0) {
                hq = q[lP + p];
                hp = psi[lP + p];
                hs = S[lP + p];
                f = 2.0;
            } else {
                bool pk;
                hq = herm_proj(g, q, lP, m, pk);
                hp = herm_proj(g, psi, lP, m, pk);
                hs = herm_proj(g, S, lP, m, pk);
                f = pk ? 1.0 : 2.0;
            }
            const double w = Hw[l] * f;
            a += w * (hp.x * hs.x + hp.y * hs.y);
            b += w * (hq.x * hs.x + hq.y * hs.y);
            c += w * (hp.x * hq.x + hp.y * hq.y);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (threadIdx.x % 32 == 0) {
        sm[0][threadIdx.x / 32] = a;
        sm[1][threadIdx.x / 32] = b;
        sm[2][threadIdx.x / 32] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) {
            t0 += sm[0][i];
            t1 += sm[1][i];
            t2 += sm[2][i];
        }
        red[blockIdx.x] = t0;
        red[nb + blockIdx.x] = t1;
        red[2 * nb + blockIdx.x] = t2;
        __threadfence();
        const unsigned prev = atomicAdd(&st->red_count, 1u);
        s_last = (prev + 1 == (unsigned)nb) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __shared__ int s_pass;
    // the last block sums the partials with all its threads (a fixed order: per thread, then
    // the warp's butterfly, then the warps in order)
    __threadfence();
    a = b = c = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        a += __ldcg(&red[i]);
        b += __ldcg(&red[nb + i]);
        c += __ldcg(&red[2 * nb + i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (threadIdx.x % 32 == 0) {
        sm[0][threadIdx.x / 32] = a;
        sm[1][threadIdx.x / 32] = b;
        sm[2][threadIdx.x / 32] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0, sc2 = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) {
            sa += sm[0][i];
            sb += sm[1][i];
            sc2 += sm[2][i];
        }
        const double N = (double)g.nx * (double)g.ny, inv = 1.0 / (N * N);
        const double dE = -sa * inv, dZ = sb * inv, E = -0.5 * sc2 * inv;
        const bool pass = (dZ <= 0.0) && (dE <= elimit * E / 86400.0) && (dE == dE) && (dZ == dZ);
        st->evaluations += 1;
        st->fallbacks += pass ? 0 : 1;
        st->dE = dE;
        st->dZ = dZ;
        st->E = E;
        st->pass = pass ? 1 : 0;
        st->red_count = 0u;
        *flag = pass ? 1.0 : 0.0;
        if (pass)
            for (int l = 0; l < g.nz; ++l) sc->A8L[l] = A8bg;
        s_pass = pass ? 1 : 0;
    }
    __syncthreads();
    if (!s_pass) {   // a dropped tendency is exactly zero (not S * 0: S may hold Inf)
        const size_t n = g.csize();
        for (size_t e = threadIdx.x; e < n; e += blockDim.x) S[e] = make_double2(0.0, 0.0);
    }
}

int grid_of(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

cudaError_t coarse_grain_on(const qgn_ctx* fine, qgn_ctx* coarse, const double2* src, double2* dst, cudaStream_t s) {
    const double scale = ((double)coarse->g.nx * coarse->g.ny) / ((double)fine->g.nx * fine->g.ny);
    QGN_LAUNCH(KID_LAYOUT, 32.0 * (double)coarse->g.csize(), s,
               ::qgn::launch(k_truncate, grid_of(coarse->g.csize()), 256, 0, s, fine->g, coarse->g, src, dst, scale));
    return cudaGetLastError();
}

bool compatible(const qgn_ctx* f, const qgn_ctx* c) {
    return f->g.nz == c->g.nz && c->g.nx <= f->g.nx && c->g.ny <= f->g.ny && f->p.Lx == c->p.Lx && f->p.Ly == c->p.Ly;
}

}  // namespace

// the closure's tendency (compact) for the stage right-hand sides, or NULL
const double2* closure_tendency(const qgn_ctx* ctx) { return ctx->closure ? ctx->closure->S : nullptr; }

// evaluate the network on the state (b.q, with psi = GetPsi(b.q)) on stream st and run the
// budget check: y-inverse of (q, psi) and an x-inverse that writes the network input, the
// network, the forward transform of its output, the budget kernel.  It writes only the
// closure's own buffers and, when the check passes, the layers' A8 in the device scalars.
int closure_eval(qgn_ctx* ctx, const double2* psi, cudaStream_t st) {
    QGN_NVTX("closure evaluation");
    Closure* c = ctx->closure;
    const Geom& g = ctx->g;
    const Buffers& b = ctx->b;
    if (launch_closure_input(g, b, b.q, psi, c->hq, c->hu, c->scales, c->x, c->cin_p, st) != cudaSuccess)
        return QGN_ERR_CUDA;
    if (cnn::infer(c->net, c->x, c->y, 1, st, true) != QGN_OK) return QGN_ERR_CUDA;   // planar output
    if (launch_closure_output(g, b, c->y, c->cout_p, c->scales + 2 * g.nz, c->hq, c->S, st) != cudaSuccess)
        return QGN_ERR_CUDA;
    const int nb = (int)std::min<size_t>((g.csize() + 255) / 256, (size_t)c->nblocks);
    QGN_LAUNCH(KID_PARSEVAL, 48.0 * g.csize(), st,
               ::qgn::launch(k_budget_spec, nb, 256, 0, st, g, b.q, psi, c->S, b.Hw, c->red, c->A8bg, c->elimit, b.sc,
                                                  c->stats, c->flag));
    if (cudaGetLastError() != cudaSuccess) return QGN_ERR_CUDA;
    return QGN_OK;
}

// The closure on its own stream, forked from the context's stream: GetPsi into the closure's
// copy, then closure_eval.  The context's stream may meanwhile run work that reads b.q and
// writes none of the closure's buffers, S, or the A8 of the device scalars (the first RHS's
// y-inverse and x pass); closure_join makes it wait for the closure before anything reads S.
int closure_fork(qgn_ctx* ctx) {
    Closure* c = ctx->closure;
    if (cudaEventRecord(c->fork, ctx->stream) != cudaSuccess || cudaStreamWaitEvent(c->side, c->fork, 0) != cudaSuccess)
        return QGN_ERR_CUDA;
    if (launch_modal(ctx->g, ctx->b, ctx->b.q, c->psi, c->side) != cudaSuccess) return QGN_ERR_CUDA;
    const int rc = closure_eval(ctx, c->psi, c->side);
    if (rc != QGN_OK) return rc;
    return cudaEventRecord(c->join, c->side) == cudaSuccess ? QGN_OK : QGN_ERR_CUDA;
}

int closure_join(qgn_ctx* ctx) {
    return cudaStreamWaitEvent(ctx->stream, ctx->closure->join, 0) == cudaSuccess ? QGN_OK : QGN_ERR_CUDA;
}

void closure_free(qgn_ctx* ctx) {
    Closure* c = ctx->closure;
    if (!c) return;
    if (c->side) cudaStreamSynchronize(c->side);
    cudaFree(c->psi);
    cudaFree(c->hq);
    cudaFree(c->hu);
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->join) cudaEventDestroy(c->join);
    if (c->side) cudaStreamDestroy(c->side);
    cudaFree(c->scales);
    cudaFree(c->x);
    cudaFree(c->y);
    cudaFree(c->S);
    cudaFree(c->red);
    cudaFree(c->flag);
    cudaFree(c->stats);
    delete c;
    ctx->closure = nullptr;
}

}  // namespace qgn

using namespace qgn;

namespace {

int snap_scratch(qgn_ctx* c, double** out) {
    const size_t np = (size_t)c->g.nx * c->g.ny * c->g.nz;
    if (!c->b.snap) {
        if (cudaMalloc((void**)&c->b.snap, sizeof(double) * (3 * np + 64)) != cudaSuccess) return QGN_ERR_CUDA;
    }
    *out = c->b.snap;
    return QGN_OK;
}

}  // namespace

extern "C" {

int qgn_coarse_grain(qgn_ctx* fine, qgn_ctx* coarse) {
    QGN_NVTX("qgn_coarse_grain");
    if (!fine || !coarse || fine == coarse) return QGN_ERR_ARG;
    if (!compatible(fine, coarse)) return QGN_ERR_CONFIG;
    if (cudaSetDevice(fine->device) != cudaSuccess) return QGN_ERR_CUDA;
    if (cudaStreamSynchronize(coarse->stream) != cudaSuccess) return QGN_ERR_CUDA;
    cudaStream_t s = fine->stream;
    if (coarse_grain_on(fine, coarse, fine->b.q, coarse->b.q, s) != cudaSuccess) return QGN_ERR_CUDA;
    ::qgn::launch(k_copy_time, 1, 1, 0, s, fine->b.sc, coarse->b.sc);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return QGN_ERR_CUDA;
    coarse->b.Qs[0] = coarse->b.q;
    coarse->halted = false;
    ++coarse->state_version;
    return QGN_OK;
}

int qgn_closure_snapshot(qgn_ctx* fine, qgn_ctx* coarse, const float* in_scale, const float* out_scale, void* x_dev,
                         float* y_dev, int cin_p, int cout_p) {
    QGN_NVTX("qgn_closure_snapshot");
    if (!fine || !coarse || !in_scale || !out_scale || !x_dev || !y_dev) return QGN_ERR_ARG;
    const int nz = coarse->g.nz;
    if (cin_p < 2 * nz || cin_p % 16 || cout_p < nz || cout_p % 16) return QGN_ERR_CONFIG;
    int rc = qgn_coarse_grain(fine, coarse);
    if (rc != QGN_OK) return rc;
    double* P0 = nullptr;
    if ((rc = snap_scratch(coarse, &P0)) != QGN_OK) return rc;
    const Geom& gf = fine->g;
    const Geom& gc = coarse->g;
    const Buffers& bf = fine->b;
    const Buffers& bc = coarse->b;
    cudaStream_t s = fine->stream;
    const size_t npix = (size_t)gc.nx * gc.ny, np = npix * nz;
    double* P1 = P0 + np;
    double* P2 = P1 + np;
    float* sc = reinterpret_cast<float*>(P2 + np);
    if (cudaMemcpyAsync(sc, in_scale, sizeof(float) * 2 * nz, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(sc + 2 * nz, out_scale, sizeof(float) * nz, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return QGN_ERR_CUDA;
    // high-resolution GetRHS (no hyperviscosity for implicit schemes: is_explicit as configured)
    if (launch_modal(gf, bf, bf.q, bf.psi, s) != cudaSuccess) return QGN_ERR_CUDA;
    if (launch_rhs(gf, bf, bf.q, bf.psi, bf.N[5], fine->p.C_d != 0.0, s) != cudaSuccess) return QGN_ERR_CUDA;
    if (coarse_grain_on(fine, coarse, bf.N[5], bc.N[4], s) != cudaSuccess) return QGN_ERR_CUDA;
    // coarse GetRHS of the coarse-grained state
    if (launch_modal(gc, bc, bc.q, bc.psi, s) != cudaSuccess) return QGN_ERR_CUDA;
    if (launch_rhs(gc, bc, bc.q, bc.psi, bc.N[5], coarse->p.C_d != 0.0, s) != cudaSuccess) return QGN_ERR_CUDA;
    ::qgn::launch(k_sub, grid_of(gc.csize()), 256, 0, s, gc.csize(), bc.N[4], bc.N[5], bc.err);
    if (cudaGetLastError() != cudaSuccess) return QGN_ERR_CUDA;
    if (launch_to_phys(gc, bc, bc.q, P0, s) != cudaSuccess) return QGN_ERR_CUDA;
    if (launch_to_phys(gc, bc, bc.psi, P1, s) != cudaSuccess) return QGN_ERR_CUDA;
    if (launch_to_phys(gc, bc, bc.err, P2, s) != cudaSuccess) return QGN_ERR_CUDA;
    ::qgn::launch(k_pack_in, grid_of(npix), 256, 0, s, nz, npix, P0, P1, sc, cin_p, static_cast<__nv_bfloat16*>(x_dev));
    ::qgn::launch(k_pack_out, grid_of(npix), 256, 0, s, nz, npix, P2, sc + 2 * nz, cout_p, y_dev);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return QGN_ERR_CUDA;
    return QGN_OK;
}

int qgn_closure_attach(qgn_ctx* ctx, qgn_cnn* net, const float* in_scale, const float* out_scale, double A8_background,
                       double energy_limit) {
    if (!ctx) return QGN_ERR_ARG;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return QGN_ERR_CUDA;
    cudaStreamSynchronize(ctx->stream);
    closure_free(ctx);
    drop_graphs(ctx);
    if (!net) return QGN_OK;
    if (!in_scale || !out_scale) return QGN_ERR_ARG;
    if (ctx->scheme != QGN_SCHEME_ARK43_QGLEITH || ctx->precision != QGN_PREC_FP64) return QGN_ERR_CONFIG;
    const Geom& g = ctx->g;
    if (cnn::height(net) != g.ny || cnn::width(net) != g.nx || cnn::padded_in(net) < 2 * g.nz ||
        cnn::real_out(net) != g.nz)
        return QGN_ERR_CONFIG;
    Closure* c = new (std::nothrow) Closure();
    if (!c) return QGN_ERR_CUDA;
    ctx->closure = c;
    c->net = net;
    c->A8bg = A8_background;
    c->elimit = energy_limit;
    c->cin_p = cnn::padded_in(net);
    c->cout_p = cnn::padded_out(net);
    c->nblocks = kBudgetBlocks;
    const size_t npix = (size_t)g.nx * g.ny;
    bool ok = cudaMalloc((void**)&c->scales, sizeof(float) * 3 * g.nz) == cudaSuccess &&
              cudaMalloc((void**)&c->x, sizeof(__nv_bfloat16) * npix * c->cin_p) == cudaSuccess &&
              cudaMalloc((void**)&c->y, sizeof(float) * npix * c->cout_p) == cudaSuccess &&
              cudaMalloc((void**)&c->S, sizeof(double2) * g.csize()) == cudaSuccess &&
              cudaMalloc((void**)&c->psi, sizeof(double2) * g.csize()) == cudaSuccess &&
              cudaMalloc((void**)&c->hq, sizeof(double2) * g.hsize()) == cudaSuccess &&
              cudaMalloc((void**)&c->hu, sizeof(double2) * g.hsize()) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming) == cudaSuccess &&
              cudaMalloc((void**)&c->red, sizeof(double) * 3 * c->nblocks) == cudaSuccess &&
              cudaMalloc((void**)&c->flag, sizeof(double)) == cudaSuccess &&
              cudaMalloc((void**)&c->stats, sizeof(ClosureStats)) == cudaSuccess;
    ok = ok && cudaMemcpy(c->scales, in_scale, sizeof(float) * 2 * g.nz, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(c->scales + 2 * g.nz, out_scale, sizeof(float) * g.nz, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(c->stats, 0, sizeof(ClosureStats)) == cudaSuccess &&
         cudaMemset(c->x, 0, sizeof(__nv_bfloat16) * npix * c->cin_p) == cudaSuccess &&
         cudaMemset(c->S, 0, sizeof(double2) * g.csize()) == cudaSuccess;
    if (!ok) {
        closure_free(ctx);
        return QGN_ERR_CUDA;
    }
    return QGN_OK;
}

int qgn_closure_stats(qgn_ctx* ctx, long long* evaluations, long long* fallbacks, double* last_budget) {
    if (!ctx) return QGN_ERR_ARG;
    if (!ctx->closure) return QGN_ERR_CONFIG;
    ClosureStats s;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess ||
        cudaMemcpy(&s, ctx->closure->stats, sizeof(s), cudaMemcpyDeviceToHost) != cudaSuccess)
        return QGN_ERR_CUDA;
    if (evaluations) *evaluations = s.evaluations;
    if (fallbacks) *fallbacks = s.fallbacks;
    if (last_budget) {
        last_budget[0] = s.dE;
        last_budget[1] = s.dZ;
        last_budget[2] = s.E;
    }
    return QGN_OK;
}

}  // extern "C"
