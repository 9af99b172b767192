// capi.cu -- extern "C" boundary (include/qgn_gpu.h) and the host-side scheme drivers.
//
// The scheme drivers issue, per TimeStep, the same sequence of RHS evaluations, stage
// combinations, error norms and controller updates as the reference include files
// (ARK43_QGLeith.f90, ARK43.f90, BSRK3.f90, RK4.f90, AB3.f90).  Adaptive schemes read one
// small scalar block back per attempt to decide accept/reject; the reject loop is bounded
// by qgn_params.max_rejects (the reference loops forever and silently accepts NaN errors).
#include "qgn_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <utility>

using namespace qgn;

namespace qgn {
Prof*& current_prof() {
    thread_local Prof* p = nullptr;
    return p;
}

// forget the recorded step graphs (their prologue changes); the next advance records anew
void drop_graphs(qgn_ctx* ctx) {
    for (int w = 0; w < 2; ++w)
        if (ctx->gexec[w]) {
            cudaGraphExecDestroy(ctx->gexec[w]);
            ctx->gexec[w] = nullptr;
        }
    ctx->graphs_ready = false;
}
}  // namespace qgn

namespace {

// Makes the context's profiler the current one for the duration of an API call.
struct ProfScope {
    Prof* prev;
    NvtxRange range;
    ProfScope(qgn_ctx* ctx, const char* api) : prev(current_prof()), range(api) {
        current_prof() = ctx ? &ctx->prof : nullptr;
    }
    ~ProfScope() { current_prof() = prev; }
};

int set_err(qgn_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

int cuda_err(qgn_ctx* ctx, const char* what, cudaError_t e) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return set_err(ctx, QGN_ERR_CUDA, buf);
}

#define CK(call)                                                    \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_err(ctx, #call, _e);     \
    } while (0)

#define RET(call)                        \
    do {                                 \
        int _r = (call);                 \
        if (_r != QGN_OK) return _r;     \
    } while (0)

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// twiddles exp(-2 pi i m/n), m in [0,n), in long double with octant reduction
void make_twiddles(int n, std::vector<double2>& tw) {
    tw.resize(n);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < n; ++m) {
        long double a = 2.0L * PI * (long double)m / (long double)n;
        tw[m] = make_double2((double)cosl(a), (double)(-sinl(a)));
    }
    // exact values at the quadrant points
    for (int m = 0; m < n; m += (n >= 4 ? n / 4 : n)) {
        const int qd = (n >= 4) ? (4 * m / n) : 0;
        const double c[4] = {1.0, 0.0, -1.0, 0.0}, s[4] = {0.0, -1.0, 0.0, 1.0};
        tw[m] = make_double2(c[qd], s[qd]);
    }
}

template <class T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

int copy_kept(qgn_ctx* ctx, double* host, bool h2d) {
    const Geom& g = ctx->g;
    for (int part = 0; part < 2; ++part) {
        const int j0 = part == 0 ? 0 : g.kylo + g.kyshift;
        const int m0 = part == 0 ? 0 : g.kylo;
        const int rows = part == 0 ? g.kylo : g.nky - g.kylo;
        if (rows <= 0) continue;
        cudaMemcpy3DParms prm;
        std::memset(&prm, 0, sizeof(prm));
        cudaPitchedPtr hp = make_cudaPitchedPtr(host, (size_t)g.nxh * 16, (size_t)g.nxh * 16, (size_t)g.ny);
        cudaPitchedPtr dp = make_cudaPitchedPtr(ctx->b.xfer, (size_t)g.nkx * 16, (size_t)g.nkx * 16, (size_t)g.nky);
        cudaPos hpos = make_cudaPos(0, (size_t)j0, 0), dpos = make_cudaPos(0, (size_t)m0, 0);
        prm.extent = make_cudaExtent((size_t)g.nkx * 16, (size_t)rows, (size_t)g.nz);
        if (h2d) {
            prm.srcPtr = hp; prm.srcPos = hpos; prm.dstPtr = dp; prm.dstPos = dpos;
            prm.kind = cudaMemcpyHostToDevice;
        } else {
            prm.srcPtr = dp; prm.srcPos = dpos; prm.dstPtr = hp; prm.dstPos = hpos;
            prm.kind = cudaMemcpyDeviceToHost;
        }
        CK(cudaMemcpy3DAsync(&prm, ctx->stream));
    }
    return QGN_OK;
}

// host q_hat (kept modes) -> compact device field
int upload_kept(qgn_ctx* ctx, const double* host, double2* dst) {
    RET(copy_kept(ctx, const_cast<double*>(host), true));
    CK(launch_xfer_to_compact(ctx->g, ctx->b.xfer, dst, ctx->stream));
    return QGN_OK;
}

int ensure_full(qgn_ctx* ctx) {
    if (!ctx->b.full) CK(dalloc(&ctx->b.full, (size_t)ctx->g.nz * ctx->g.ny * ctx->g.nxh));
    return QGN_OK;
}

int download_full(qgn_ctx* ctx, const double2* src, double* host);

// compact device field -> host q_hat of TimeStep.  By default only the modes DeAlias keeps
// cross the link (the same two pitched copies as the upload): the reference's TimeStep ends
// with `call DeAlias(q_hat)` (QGN_Module.f90:307), which zeroes the others on the host, and
// they are zero already in a dealiased input.  QGN_OUTPUT_FULL writes the whole array with
// zeros in the dealiased band instead (one contiguous copy of 2.25x the bytes).
int download_kept(qgn_ctx* ctx, const double2* src, double* host) {
    if (ctx->output_mode == QGN_OUTPUT_FULL) return download_full(ctx, src, host);
    CK(launch_compact_to_xfer(ctx->g, src, ctx->b.xfer, ctx->stream));
    return copy_kept(ctx, host, false);
}

// compact device field -> whole host q_hat (zeros in the dealiased band)
int download_full(qgn_ctx* ctx, const double2* src, double* host) {
    RET(ensure_full(ctx));
    const Geom& g = ctx->g;
    CK(launch_compact_to_xfer(g, src, ctx->b.xfer, ctx->stream));
    CK(launch_xfer_to_full(g, ctx->b.xfer, ctx->b.full, ctx->stream));
    CK(cudaMemcpyAsync(host, ctx->b.full, sizeof(double2) * (size_t)g.nz * g.ny * g.nxh, cudaMemcpyDeviceToHost,
                       ctx->stream));
    return QGN_OK;
}

int read_scalars(qgn_ctx* ctx, DevScalars* out) {
    CK(cudaMemcpyAsync(ctx->host_pin, ctx->b.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->prof.harvest();
    std::memcpy(out, ctx->host_pin, sizeof(DevScalars));
    return QGN_OK;
}

// new state from the host: set t, dt and clear a previous failure (halt, status); stream-ordered
int write_time(qgn_ctx* ctx, double t, double dt) {
    CK(launch_set_time(ctx->b.sc, t, dt, ctx->stream));
    return QGN_OK;
}

const char* status_text(int st) {
    switch (st) {
        case QGN_ERR_NONFINITE: return "non-finite embedded error estimate";
        case QGN_ERR_REJECT_LIMIT: return "adaptive step rejected max_rejects times in a row";
        case QGN_ERR_CUDA: return "a bounded device wait ran out";
        default: return "step failed";
    }
}

bool drag_on(const qgn_ctx* ctx) { return ctx->p.C_d != 0.0; }

double leith_c12(const qgn_params& p) {
    const double pi = 4.0 * std::atan(1.0);
    const double x = (double)1.3f * p.Lx / ((double)p.nx * pi);   // default-REAL 1.3 (ARK43_QGLeith.f90:72)
    const double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
    return x4 * x8;
}

// a stage right-hand side of the schemes: GetRHS plus the learned closure's tendency if attached
int rhs_of(qgn_ctx* ctx, const double2* q, const double2* psi, double2* out) {
    CK(launch_rhs(ctx->g, ctx->b, q, psi, out, drag_on(ctx), ctx->stream, closure_tendency(ctx)));
    return QGN_OK;
}

int max_rejects(const qgn_ctx* ctx) { return ctx->p.max_rejects > 0 ? ctx->p.max_rejects : 64; }

// ---- ARK4(3)6L[2]SA, ARK43_QGLeith.f90 / ARK43.f90 ------------------------------------------
// Kernel sequence of one attempt (stages 2..6 with their RHS, update + error combination,
// error transform, controller).  Shared by the eager path and the graph capture.
bool mixed(const qgn_ctx* ctx) { return ctx->precision == QGN_PREC_MIXED; }

template <class T>
float2* f32(T* p) { return reinterpret_cast<float2*>(p); }

static const char* const kStageRange[6] = {"stage 0", "stage 1", "stage 2", "stage 3", "stage 4", "stage 5"};

int ark_attempt(qgn_ctx* ctx, bool leith, const cudaGraphConditionalHandle* loop) {
    QGN_NVTX("ARK attempt");
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    cudaStream_t st = ctx->stream;
    const bool columns = !mixed(ctx) && stage_yinv_ok(g, b);
    if (columns && !drag_on(ctx)) {
        // small grids: stage s with the y-inverse of its RHS, and the y-forward of RHS s-1
        // with both, in one launch per column (two launches per stage instead of four)
        const double2* extra = closure_tendency(ctx);
        CK(launch_ark_stage_yinv(g, b, 1, st));
        for (int s = 1; s < 6; ++s) {
            CK(launch_rhs_x(g, b, false, st));
            if (s < 5) CK(launch_yfwd_stage_yinv(g, b, s + 1, extra, st));
            else CK(launch_rhs_yfwd(g, b, b.Qs[5], b.psi, b.N[5], false, st, extra));
        }
    } else for (int s = 1; s < 6; ++s) {
        QGN_NVTX(kStageRange[s]);
        if (mixed(ctx)) {
            CK(launch_ark_stage_mixed(g, b, s, st));
            CK(launch_rhs32(g, b, f32(b.Qs[s]), f32(b.psi), f32(b.N[s]), drag_on(ctx), st));
        } else if (columns) {   // small grids with quadratic drag: the stage with the y-inverse
            CK(launch_ark_stage_yinv(g, b, s, st));
            CK(launch_rhs_tail(g, b, b.Qs[s], b.psi, b.N[s], true, st, closure_tendency(ctx)));
        } else {
            CK(launch_ark_stage(g, b, s, st));
            RET(rhs_of(ctx, b.Qs[s], b.psi, b.N[s]));
        }
    }
    // the update kernels also clear the max reduction of the error transform
    if (mixed(ctx)) {
        CK(launch_ark_update_mixed(g, b, st));
        CK(launch_maxabs_phys32(g, b, f32(b.err), b.sc, st));
    } else {
        CK(launch_ark_update(g, b, st));
        CK(launch_maxabs_phys(g, b, b.err, b.sc, st));
    }
    CK(launch_controller(g, b, leith ? 0 : 1, ctx->p.TOL, ctx->p.dt_max, max_rejects(ctx), loop, st));
    return QGN_OK;
}

int ark_prologue(qgn_ctx* ctx, bool leith) {
    QGN_NVTX("ARK prologue");
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    cudaStream_t st = ctx->stream;
    if (leith) CK(launch_leith(g, b, b.q, leith_c12(ctx->p), st));
    b.Qs[0] = b.q;
    if (mixed(ctx)) {
        // FP32 copy of q_hat for the FP32 RHS lives in the error buffer until the update
        CK(launch_modal_mixed(g, b, b.q, f32(b.err), f32(b.psi), st));
        CK(launch_rhs32(g, b, f32(b.err), f32(b.psi), f32(b.N[0]), drag_on(ctx), st));
    } else if (stage_yinv_ok(g, b)) {
        // small grids: GetPsi and the y-inverse of the first RHS in one launch per column.  An
        // attached closure (its own GetPsi, the network, the budget check) runs on its own
        // stream beside that launch and the x pass, which read none of its outputs; the
        // y-forward pass that adds S waits for it.
        if (ctx->closure && !drag_on(ctx)) {
            RET(closure_fork(ctx));
            CK(launch_ark_stage_yinv(g, b, 0, st));
            CK(launch_rhs_x(g, b, false, st));
            RET(closure_join(ctx));
            CK(launch_rhs_yfwd(g, b, b.q, b.psi, b.N[0], false, st, closure_tendency(ctx)));
            return QGN_OK;
        }
        if (ctx->closure) {
            CK(launch_modal(g, b, b.q, b.psi, st));
            RET(closure_eval(ctx, b.psi, st));
        }
        CK(launch_ark_stage_yinv(g, b, 0, st));
        CK(launch_rhs_tail(g, b, b.q, b.psi, b.N[0], drag_on(ctx), st, closure_tendency(ctx)));
    } else {
        CK(launch_modal(g, b, b.q, b.psi, st));
        // the learned closure (if attached): S of this step's state and the budget check that
        // keeps it (background A8) or falls back to the Leith A8L just computed
        if (ctx->closure) RET(closure_eval(ctx, b.psi, st));
        RET(rhs_of(ctx, b.q, b.psi, b.N[0]));
    }
    return QGN_OK;
}

int step_ark(qgn_ctx* ctx, bool leith) {
    Buffers& b = ctx->b;
    CK(launch_step_gate(b.sc, nullptr, ctx->stream));
    RET(ark_prologue(ctx, leith));
    for (;;) {
        RET(ark_attempt(ctx, leith, nullptr));
        DevScalars s;
        RET(read_scalars(ctx, &s));
        if (s.halt) {
            ctx->halted = true;
            return set_err(ctx, s.status, status_text(s.status));
        }
        if (s.accept) {
            std::swap(b.q, b.qnew);
            b.Qs[0] = b.q;
            return QGN_OK;
        }
    }
}

// ---- CUDA-graph steps for the ARK schemes ------------------------------------------------
// One executable graph = one TimeStep: a gate kernel opens an IF node while the run is not
// halted; its body is the prologue (Leith, GetPsi, N1) and a WHILE node whose body is one
// attempt; the controller kernel sets the WHILE condition (1 = rejected, retry).  The two
// executables differ only in which state buffer holds q_hat and which receives the update,
// so consecutive steps alternate between them and no buffer is copied.
int add_conditional(qgn_ctx* ctx, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(ctx->stream, &cs, nullptr, &graph, &deps, &nd));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, graph, deps, nd, &np));
    CK(cudaStreamUpdateCaptureDependencies(ctx->stream, &node, 1, cudaStreamSetCaptureDependencies));
    *body = np.conditional.phGraph_out[0];
    return QGN_OK;
}

void snapshot(const qgn_ctx* ctx, long long* out) {
    for (int k = 0; k < KID_COUNT; ++k) out[k] = ctx->prof.launches[k];
}

int capture_ark(qgn_ctx* ctx, bool leith, int variant, cudaGraphExec_t* out) {
    Buffers& b = ctx->b;
    const Buffers saved = b;
    b.q = ctx->gbuf[variant];
    b.qnew = ctx->gbuf[variant ^ 1];
    b.Qs[0] = b.q;
    cudaStream_t st = ctx->stream;
    long long c0[KID_COUNT], c1[KID_COUNT], c2[KID_COUNT], c3[KID_COUNT];
    int rc = QGN_OK;
    cudaGraph_t root = nullptr;
    auto run = [&]() -> int {
        CK(cudaGraphCreate(&root, 0));
        cudaGraphConditionalHandle hgate, hloop;
        CK(cudaGraphConditionalHandleCreate(&hgate, root, 0, 0));
        snapshot(ctx, c0);
        CK(cudaStreamBeginCaptureToGraph(st, root, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        CK(launch_step_gate(b.sc, &hgate, st));
        cudaGraph_t ifbody = nullptr;
        int r = add_conditional(ctx, hgate, cudaGraphCondTypeIf, &ifbody);
        cudaGraph_t tmp = nullptr;
        CK(cudaStreamEndCapture(st, &tmp));
        if (r != QGN_OK) return r;
        snapshot(ctx, c1);
        CK(cudaGraphConditionalHandleCreate(&hloop, ifbody, 0, 0));
        CK(cudaStreamBeginCaptureToGraph(st, ifbody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        r = ark_prologue(ctx, leith);
        if (r == QGN_OK) {
            cudaError_t e = launch_set_cond(hloop, 1u, st);
            if (e != cudaSuccess) r = cuda_err(ctx, "launch_set_cond", e);
        }
        cudaGraph_t wbody = nullptr;
        if (r == QGN_OK) r = add_conditional(ctx, hloop, cudaGraphCondTypeWhile, &wbody);
        CK(cudaStreamEndCapture(st, &tmp));
        if (r != QGN_OK) return r;
        snapshot(ctx, c2);
        CK(cudaStreamBeginCaptureToGraph(st, wbody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        r = ark_attempt(ctx, leith, &hloop);
        CK(cudaStreamEndCapture(st, &tmp));
        if (r != QGN_OK) return r;
        snapshot(ctx, c3);
        CK(cudaGraphInstantiate(out, root, 0));
        return QGN_OK;
    };
    const bool timing = ctx->prof.timing;
    ctx->prof.timing = false;
    rc = run();
    ctx->prof.timing = timing;
    if (root) cudaGraphDestroy(root);
    // captured launches did not run: take them out of the counters, keep them per graph part
    for (int k = 0; k < KID_COUNT; ++k) {
        ctx->g_pro[k] = c2[k] - c1[k] + (c1[k] - c0[k]);   // gate + prologue, once per executed step
        ctx->g_body[k] = c3[k] - c2[k];                     // once per attempt
        ctx->prof.launches[k] = c0[k];
    }
    b = saved;
    return rc;
}

int ensure_ark_graphs(qgn_ctx* ctx, bool leith) {
    if (ctx->graphs_ready) return QGN_OK;
    ctx->gbuf[0] = ctx->b.q;
    ctx->gbuf[1] = ctx->b.qnew;
    for (int v = 0; v < 2; ++v) {
        int rc = capture_ark(ctx, leith, v, &ctx->gexec[v]);
        if (rc != QGN_OK) {
            for (int w = 0; w < 2; ++w)
                if (ctx->gexec[w]) { cudaGraphExecDestroy(ctx->gexec[w]); ctx->gexec[w] = nullptr; }
            cudaGetLastError();
            ctx->graphs_off = true;
            return rc;
        }
    }
    ctx->graphs_ready = true;
    return QGN_OK;
}

int advance_ark_graph(qgn_ctx* ctx, bool leith, int nsteps) {
    Buffers& b = ctx->b;
    DevScalars s0, s1;
    RET(read_scalars(ctx, &s0));
    if (s0.halt) {
        ctx->halted = true;
        return set_err(ctx, s0.status, status_text(s0.status));
    }
    const int par0 = (b.q == ctx->gbuf[0]) ? 0 : 1;
    int par = par0;
    for (int i = 0; i < nsteps; ++i) {
        CK(cudaGraphLaunch(ctx->gexec[par], ctx->stream));
        par ^= 1;
    }
    RET(read_scalars(ctx, &s1));
    const long long acc = s1.accepted - s0.accepted;
    const long long att = s1.attempts - s0.attempts;
    const long long runs = acc + (s1.halt ? 1 : 0);
    for (int k = 0; k < KID_COUNT; ++k) ctx->prof.launches[k] += runs * ctx->g_pro[k] + att * ctx->g_body[k];
    ctx->prof.launches[KID_SCALAR] += nsteps - runs;   // gate kernels of skipped steps
    b.q = ctx->gbuf[par0 ^ (int)(acc & 1)];
    b.qnew = ctx->gbuf[par0 ^ 1 ^ (int)(acc & 1)];
    b.Qs[0] = b.q;
    if (s1.halt) {
        ctx->halted = true;
        return set_err(ctx, s1.status, status_text(s1.status));
    }
    return QGN_OK;
}

// ---- Bogacki-Shampine 3(2), BSRK3.f90 -----------------------------------------------------
int step_bsrk3(qgn_ctx* ctx) {
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    cudaStream_t st = ctx->stream;
    if (ctx->first_call) {
        CK(launch_modal(g, b, b.q, b.psi, st));
        RET(rhs_of(ctx, b.q, b.psi, b.N[0]));     // RHS0 (kept between calls, FSAL)
        ctx->first_call = false;
    }
    CK(launch_step_gate(b.sc, nullptr, st));
    for (;;) {
        Combo c1{{b.N[0]}, {0.5}, 1};
        CK(launch_combo(g, b, c1, b.q, b.Qs[1], b.psi, true, st));
        RET(rhs_of(ctx, b.Qs[1], b.psi, b.N[1]));
        Combo c2{{b.N[1]}, {0.75}, 1};
        CK(launch_combo(g, b, c2, b.q, b.Qs[2], b.psi, true, st));
        RET(rhs_of(ctx, b.Qs[2], b.psi, b.N[2]));
        Combo c3{{b.N[0], b.N[1], b.N[2]}, {2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0}, 3};
        CK(launch_combo(g, b, c3, b.q, b.Qs[3], b.psi, true, st));
        RET(rhs_of(ctx, b.Qs[3], b.psi, b.N[3]));
        Combo ce{{b.N[0], b.N[1], b.N[2], b.N[3]}, {5.0 / 72.0, -1.0 / 12.0, -1.0 / 9.0, 1.0 / 8.0}, 4};
        CK(launch_lincomb(g, ce, b.err, st));
        CK(launch_zero_scalar_max(b.sc, st));
        CK(launch_maxabs_phys(g, b, b.err, b.sc, st));
        CK(launch_controller(g, b, 2, ctx->p.TOL, ctx->p.dt_max, max_rejects(ctx), nullptr, st));
        DevScalars s;
        RET(read_scalars(ctx, &s));
        if (s.halt) {
            ctx->halted = true;
            return set_err(ctx, s.status, status_text(s.status));
        }
        if (s.accept) {
            std::swap(b.q, b.Qs[3]);      // q_hat = q_tmp
            std::swap(b.N[0], b.N[3]);    // RHS0 = RHS3
            return QGN_OK;
        }
    }
}

// ---- classic RK4, RK4.f90 -------------------------------------------------------------------
int step_rk4(qgn_ctx* ctx) {
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    cudaStream_t st = ctx->stream;
    CK(launch_modal(g, b, b.q, b.psi, st));
    RET(rhs_of(ctx, b.q, b.psi, b.N[0]));
    Combo c1{{b.N[0]}, {0.5}, 1};
    CK(launch_combo(g, b, c1, b.q, b.Qs[1], b.psi, true, st));
    RET(rhs_of(ctx, b.Qs[1], b.psi, b.N[1]));
    Combo c2{{b.N[1]}, {0.5}, 1};
    CK(launch_combo(g, b, c2, b.q, b.Qs[2], b.psi, true, st));
    RET(rhs_of(ctx, b.Qs[2], b.psi, b.N[2]));
    Combo c3{{b.N[2]}, {1.0}, 1};
    CK(launch_combo(g, b, c3, b.q, b.Qs[3], b.psi, true, st));
    RET(rhs_of(ctx, b.Qs[3], b.psi, b.N[3]));
    Combo cu{{b.N[0], b.N[1], b.N[2], b.N[3]}, {1.0 / 6.0, 2.0 / 6.0, 2.0 / 6.0, 1.0 / 6.0}, 4};
    CK(launch_combo(g, b, cu, b.q, b.qnew, nullptr, false, st));
    std::swap(b.q, b.qnew);
    CK(launch_advance_time(b.sc, st));
    return QGN_OK;
}

// ---- AB3 with Euler / AB2 start-up, AB3.f90 -------------------------------------------------
int step_ab3(qgn_ctx* ctx) {
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    cudaStream_t st = ctx->stream;
    CK(launch_modal(g, b, b.q, b.psi, st));
    if (ctx->ab_calls == 0) {
        RET(rhs_of(ctx, b.q, b.psi, b.N[0]));
        Combo c{{b.N[0]}, {1.0}, 1};
        CK(launch_combo(g, b, c, b.q, b.qnew, nullptr, false, st));
    } else if (ctx->ab_calls == 1) {
        RET(rhs_of(ctx, b.q, b.psi, b.N[1]));
        Combo c{{b.N[1], b.N[0]}, {1.5, -0.5}, 2};
        CK(launch_combo(g, b, c, b.q, b.qnew, nullptr, false, st));
    } else {
        RET(rhs_of(ctx, b.q, b.psi, b.N[2]));
        Combo c{{b.N[2], b.N[1], b.N[0]}, {23.0 / 12.0, -16.0 / 12.0, 5.0 / 12.0}, 3};
        CK(launch_combo(g, b, c, b.q, b.qnew, nullptr, false, st));
        double2* old0 = b.N[0];
        b.N[0] = b.N[1];
        b.N[1] = b.N[2];
        b.N[2] = old0;
    }
    ++ctx->ab_calls;
    std::swap(b.q, b.qnew);
    CK(launch_advance_time(b.sc, st));
    return QGN_OK;
}

int step_once(qgn_ctx* ctx) {
    switch (ctx->scheme) {
        case QGN_SCHEME_ARK43_QGLEITH: return step_ark(ctx, true);
        case QGN_SCHEME_ARK43: return step_ark(ctx, false);
        case QGN_SCHEME_BSRK3: return step_bsrk3(ctx);
        case QGN_SCHEME_RK4: return step_rk4(ctx);
        case QGN_SCHEME_AB3: return step_ab3(ctx);
        default: return set_err(ctx, QGN_ERR_CONFIG, "unknown scheme");
    }
}

int check_state(qgn_ctx* ctx) {
    DevScalars s;
    CK(launch_nonfinite_check(ctx->g, ctx->b.q, ctx->b.sc, ctx->stream));
    RET(read_scalars(ctx, &s));
    if (s.wait_timeout) return set_err(ctx, QGN_ERR_CUDA, "a bounded device wait ran out");
    if (s.nonfinite) return set_err(ctx, QGN_ERR_NONFINITE, "non-finite values in the state q_hat");
    return QGN_OK;
}

bool use_graphs(const qgn_ctx* ctx) {
    if (ctx->graphs_off || ctx->prof.timing) return false;
    if (ctx->scheme != QGN_SCHEME_ARK43_QGLEITH && ctx->scheme != QGN_SCHEME_ARK43) return false;
    const char* env = std::getenv("QGN_NO_GRAPHS");
    return !(env && env[0] && env[0] != '0');
}

int advance_n(qgn_ctx* ctx, int nsteps) {
    if (ctx->halted) return set_err(ctx, QGN_ERR_CONFIG, "a previous step failed; upload a new state first");
    if (nsteps > 0 && use_graphs(ctx)) {
        const bool leith = ctx->scheme == QGN_SCHEME_ARK43_QGLEITH;
        if (!ctx->graphs_ready) {
            // one eager step first: it sets kernel attributes and loads every module function
            RET(step_once(ctx));
            --nsteps;
            if (nsteps == 0) return QGN_OK;
            if (ensure_ark_graphs(ctx, leith) != QGN_OK) {
                ctx->last_error.clear();
                for (int i = 0; i < nsteps; ++i) RET(step_once(ctx));
                return QGN_OK;
            }
        }
        return advance_ark_graph(ctx, leith, nsteps);
    }
    for (int i = 0; i < nsteps; ++i) RET(step_once(ctx));
    return QGN_OK;
}

bool finite_all(const double* a, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(a[i])) return false;
    return true;
}

void free_all(qgn_ctx* ctx) {
    ctx->prof.release();
    for (int w = 0; w < 2; ++w)
        if (ctx->gexec[w]) { cudaGraphExecDestroy(ctx->gexec[w]); ctx->gexec[w] = nullptr; }
    // stage buffers are swapped between roles while stepping, so memory is released
    // through the ownership list recorded at creation, never through the role pointers
    for (void* p : ctx->owned) cudaFree(p);
    ctx->owned.clear();
    Buffers& b = ctx->b;
    if (b.full) cudaFree(b.full);
    if (b.phys) cudaFree(b.phys);
    if (b.diag) cudaFree(b.diag);
    if (b.modal_scratch) cudaFree(b.modal_scratch);
    if (b.snap) cudaFree(b.snap);
    b = Buffers{};
    if (ctx->host_pin) cudaFreeHost(ctx->host_pin);
    ctx->host_pin = nullptr;
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = nullptr;
}

}  // namespace

// ============================================================================================
extern "C" {

int qgn_create(const qgn_params* p, const double* H, const double* S, const double* uBar, const double* qyBar,
               const double* Modes, const double* EVals, int scheme, int precision, qgn_ctx** out) {
    if (!out) return QGN_ERR_ARG;
    *out = nullptr;
    if (!p || !H || !uBar || !qyBar || !Modes || !EVals) return QGN_ERR_ARG;
    if (!is_pow2(p->nx) || !is_pow2(p->ny) || p->nx < 16 || p->ny < 16 || p->nx > 2048 || p->ny > 2048)
        return QGN_ERR_CONFIG;
    if (p->nz < 2 || p->nz > kMaxNZ) return QGN_ERR_CONFIG;
    if (scheme < 0 || scheme > 4) return QGN_ERR_CONFIG;
    if (precision != QGN_PREC_FP64 && precision != QGN_PREC_MIXED) return QGN_ERR_CONFIG;
    // the mixed mode is built for the ARK4(3)6L[2]SA schemes
    if (precision == QGN_PREC_MIXED && scheme != QGN_SCHEME_ARK43_QGLEITH && scheme != QGN_SCHEME_ARK43)
        return QGN_ERR_CONFIG;
    if (!(p->Lx > 0) || !(p->Ly > 0) || !(p->Htot > 0)) return QGN_ERR_CONFIG;
    const int nz = p->nz;
    if (!finite_all(H, nz) || !finite_all(uBar, nz) || !finite_all(qyBar, nz) || !finite_all(Modes, (size_t)nz * nz) ||
        !finite_all(EVals, nz) || (S && !finite_all(S, nz + 1)))
        return QGN_ERR_CONFIG;
    for (int k = 0; k < nz; ++k)
        if (!(H[k] > 0)) return QGN_ERR_CONFIG;

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return QGN_ERR_NO_DEVICE;
    }
    qgn_ctx* ctx = new (std::nothrow) qgn_ctx();
    if (!ctx) return QGN_ERR_CUDA;
    ctx->p = *p;
    ctx->scheme = scheme;
    ctx->precision = precision;
    cudaGetDevice(&ctx->device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess || prop.major != 10) {
        delete ctx;
        return QGN_ERR_NO_DEVICE;
    }
    ctx->H.assign(H, H + nz);
    ctx->uBar.assign(uBar, uBar + nz);
    ctx->qyBar.assign(qyBar, qyBar + nz);
    ctx->Modes.assign(Modes, Modes + (size_t)nz * nz);
    ctx->EVals.assign(EVals, EVals + nz);

    Geom& g = ctx->g;
    g.nx = p->nx; g.ny = p->ny; g.nz = nz; g.nxh = p->nx / 2 + 1;
    g.nkx = p->nx / 3;
    g.kylo = p->ny / 3;
    g.kyshift = p->ny / 3 + 1;
    g.nky = p->ny - p->ny / 3 - 1;
    g.nkxp = (g.nkx + 3) / 4 * 4;
    const double pi = 4.0 * std::atan(1.0);
    g.dkx = 2.0 * pi / p->Lx;
    g.dky = 2.0 * pi / p->Ly;
    g.inv_nxny = 1.0 / ((double)p->nx * (double)p->ny);

    Buffers& b = ctx->b;
    int rc = QGN_OK;
    auto fail = [&](const char* what, cudaError_t e) {
        rc = cuda_err(ctx, what, e);
    };
#define AL(ptr, n)                                   \
    if (rc == QGN_OK) {                              \
        cudaError_t _e = dalloc(&(ptr), (n));        \
        if (_e != cudaSuccess) fail(#ptr, _e);       \
        else ctx->owned.push_back((void*)(ptr));     \
    }
    const size_t C = g.csize(), Hh = g.hsize();
    AL(b.q, C); AL(b.qnew, C); AL(b.psi, C); AL(b.err, C);
    for (int j = 0; j < 6; ++j) AL(b.N[j], C);
    for (int j = 1; j < 6; ++j) AL(b.Qs[j], C);
    AL(b.hq, Hh); AL(b.hp, Hh); AL(b.hu, Hh); AL(b.hpp, 2 * Hh);
    AL(b.hpd, (size_t)2 * g.ny * g.nkxp);
    AL(b.xfer, C);
    AL(b.twx, (size_t)g.nx); AL(b.twy, (size_t)g.ny);
    AL(b.twx32, (size_t)g.nx); AL(b.twy32, (size_t)g.ny);
    AL(b.red, (size_t)512 * kMaxNZ);
    AL(b.Hw, (size_t)kMaxNZ);
    AL(b.lc, 1); AL(b.mc, 1); AL(b.sc, 1);
    if (rc == QGN_OK)   // the sticky flag a bounded device wait sets when it runs out
        g.wait_err = reinterpret_cast<int*>(reinterpret_cast<char*>(b.sc) + offsetof(DevScalars, wait_timeout));
#ifdef QGN_CHECK
    AL(ctx->chk, 1);
    if (rc == QGN_OK) {
        cudaError_t e = cudaMemset(ctx->chk, 0, sizeof(unsigned long long));
        if (e != cudaSuccess) fail("cudaMemset(chk)", e);
        g.chk = ctx->chk;
    }
#endif
#undef AL
    if (rc == QGN_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) fail("cudaStreamCreate", e);
    }
    if (rc == QGN_OK) {
        cudaError_t e = cudaMallocHost((void**)&ctx->host_pin, sizeof(DevScalars) + 64);
        if (e != cudaSuccess) fail("cudaMallocHost", e);
    }
    if (rc == QGN_OK) {
        // zero everything once: padding columns of the half fields stay zero forever
        double2* zs[] = {b.q, b.qnew, b.psi, b.err, b.hq, b.hp, b.hu, b.hpp};
        for (double2* z : zs) {
            const size_t n = (z == b.hpp) ? 2 * Hh : ((z == b.hq || z == b.hp || z == b.hu) ? Hh : C);
            cudaError_t e = cudaMemset(z, 0, sizeof(double2) * n);
            if (e != cudaSuccess) { fail("cudaMemset", e); break; }
        }
        for (int j = 0; j < 6 && rc == QGN_OK; ++j) {
            cudaError_t e = cudaMemset(b.N[j], 0, sizeof(double2) * C);
            if (e == cudaSuccess && j > 0) e = cudaMemset(b.Qs[j], 0, sizeof(double2) * C);
            if (e != cudaSuccess) fail("cudaMemset", e);
        }
        if (rc == QGN_OK) {
            cudaError_t e = cudaMemset(b.hpd, 0, sizeof(double2) * 2 * g.ny * g.nkxp);
            if (e != cudaSuccess) fail("cudaMemset", e);
        }
    }
    if (rc == QGN_OK) {
        std::vector<double2> tw;
        std::vector<float2> tw32;
        auto to32 = [&]() {
            tw32.resize(tw.size());
            for (size_t i = 0; i < tw.size(); ++i) tw32[i] = make_float2((float)tw[i].x, (float)tw[i].y);
        };
        make_twiddles(g.nx, tw);
        to32();
        cudaError_t e = cudaMemcpy(b.twx, tw.data(), sizeof(double2) * g.nx, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b.twx32, tw32.data(), sizeof(float2) * g.nx, cudaMemcpyHostToDevice);
        make_twiddles(g.ny, tw);
        to32();
        if (e == cudaSuccess) e = cudaMemcpy(b.twy, tw.data(), sizeof(double2) * g.ny, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b.twy32, tw32.data(), sizeof(float2) * g.ny, cudaMemcpyHostToDevice);
        LayerConst lc;
        std::memset(&lc, 0, sizeof(lc));
        for (int k = 0; k < nz; ++k) {
            lc.uBar[k] = uBar[k];
            lc.betaq[k] = p->beta + qyBar[k];
        }
        lc.ekman = p->r0 * p->Htot / H[nz - 1];
        lc.dragc = p->C_d * p->Htot / H[nz - 1];
        lc.A2 = p->A2;
        lc.A8 = p->A8;
        lc.explicit_diss = p->is_explicit ? 1 : 0;
        ModalConst mc;
        std::memset(&mc, 0, sizeof(mc));
        for (int k = 0; k < nz; ++k) {
            for (int kk = 0; kk < nz; ++kk) {
                mc.proj[k * nz + kk] = H[kk] * Modes[kk + (size_t)k * nz];   // H(kk)*Modes(kk,k)
                mc.back[k * nz + kk] = Modes[k + (size_t)kk * nz];          // Modes(k,kk)
            }
            mc.evals[k] = EVals[k];
        }
        mc.Htot = p->Htot;
        DevScalars sc;
        std::memset(&sc, 0, sizeof(sc));
        sc.err0 = p->TOL;   // FirstCall: err0 = TOL (ARK43*.f90:17), r0 = TOL (BSRK3.f90:15)
        for (int k = 0; k < nz; ++k) sc.A8L[k] = p->A8;
        double Hw[kMaxNZ] = {0};
        for (int k = 0; k < nz; ++k) Hw[k] = H[k] / p->Htot;
        if (e == cudaSuccess) e = cudaMemcpy(b.lc, &lc, sizeof(lc), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b.mc, &mc, sizeof(mc), cudaMemcpyHostToDevice);
        ctx->mc_host = mc;
        b.mc_h = &ctx->mc_host;
        if (e == cudaSuccess) e = cudaMemcpy(b.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b.Hw, Hw, sizeof(Hw), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) fail("constant upload", e);
    }
    if (rc != QGN_OK) {
        free_all(ctx);
        delete ctx;
        return rc;
    }
    b.Qs[0] = b.q;
    *out = ctx;
    return QGN_OK;
}

int qgn_set_state(qgn_ctx* ctx, const double* q_hat, double t, double dt) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    ++ctx->state_version;
    if (!q_hat) return set_err(ctx, QGN_ERR_ARG, "q_hat is NULL");
    CK(cudaSetDevice(ctx->device));
    RET(upload_kept(ctx, q_hat, ctx->b.q));
    ctx->b.Qs[0] = ctx->b.q;
    RET(write_time(ctx, t, dt));
    ctx->halted = false;
    return QGN_OK;
}

int qgn_get_time(qgn_ctx* ctx, double* t, double* dt) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    DevScalars s;
    RET(read_scalars(ctx, &s));
    if (t) *t = s.t;
    if (dt) *dt = s.dt;
    return QGN_OK;
}

int qgn_get_state(qgn_ctx* ctx, double* q_hat, double* t, double* dt) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    CK(cudaSetDevice(ctx->device));
    if (q_hat) RET(download_full(ctx, ctx->b.q, q_hat));
    return qgn_get_time(ctx, t, dt);
}

int qgn_advance_resident(qgn_ctx* ctx, int nsteps) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    ++ctx->state_version;
    if (nsteps < 0) return set_err(ctx, QGN_ERR_ARG, "nsteps < 0");
    CK(cudaSetDevice(ctx->device));
    RET(advance_n(ctx, nsteps));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->prof.harvest();
    return QGN_OK;
}

int qgn_advance(qgn_ctx* ctx, double* q_hat, double* t, double* dt, int nsteps) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    ++ctx->state_version;
    if (!q_hat || !t || !dt) return set_err(ctx, QGN_ERR_ARG, "NULL argument");
    if (nsteps < 0) return set_err(ctx, QGN_ERR_ARG, "nsteps < 0");
    RET(qgn_set_state(ctx, q_hat, *t, *dt));
    RET(advance_n(ctx, nsteps));
    // the adaptive schemes' controller already halts on a non-finite error estimate
    const bool adaptive = ctx->scheme == QGN_SCHEME_ARK43_QGLEITH || ctx->scheme == QGN_SCHEME_ARK43 ||
                          ctx->scheme == QGN_SCHEME_BSRK3;
    if (!adaptive) RET(check_state(ctx));
    RET(download_kept(ctx, ctx->b.q, q_hat));
    DevScalars s;
    RET(read_scalars(ctx, &s));
    *t = s.t;
    *dt = s.dt;
    return QGN_OK;
}

int qgn_step(qgn_ctx* ctx, double* q_hat, double* t, double* dt) { return qgn_advance(ctx, q_hat, t, dt, 1); }

int qgn_set_output(qgn_ctx* ctx, int mode) {
    if (!ctx) return QGN_ERR_ARG;
    if (mode != QGN_OUTPUT_KEPT && mode != QGN_OUTPUT_FULL) return set_err(ctx, QGN_ERR_ARG, "unknown output mode");
    ctx->output_mode = mode;
    return QGN_OK;
}

int qgn_rhs(qgn_ctx* ctx, const double* q_hat, double* rhs) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    ++ctx->state_version;
    if (!q_hat || !rhs) return set_err(ctx, QGN_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(ctx->device));
    Buffers& b = ctx->b;
    RET(upload_kept(ctx, q_hat, b.err));
    if (mixed(ctx)) {
        // FP32 RHS: the FP32 state copy goes to N[5], the FP32 result to qnew, widened into err
        CK(launch_modal_mixed(ctx->g, b, b.err, f32(b.N[5]), f32(b.psi), ctx->stream));
        CK(launch_rhs32(ctx->g, b, f32(b.N[5]), f32(b.psi), f32(b.qnew), drag_on(ctx), ctx->stream));
        CK(launch_f2d(ctx->g.csize(), f32(b.qnew), b.err, ctx->stream));
        RET(download_full(ctx, b.err, rhs));
        CK(cudaStreamSynchronize(ctx->stream));
        return QGN_OK;
    }
    CK(launch_modal(ctx->g, b, b.err, b.psi, ctx->stream));
    CK(launch_rhs(ctx->g, b, b.err, b.psi, b.qnew, drag_on(ctx), ctx->stream));
    RET(download_full(ctx, b.qnew, rhs));
    CK(cudaStreamSynchronize(ctx->stream));
    return QGN_OK;
}

int qgn_psi(qgn_ctx* ctx, const double* q_hat, double* psi_hat) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    if (!q_hat || !psi_hat) return set_err(ctx, QGN_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(ctx->device));
    Buffers& b = ctx->b;
    RET(upload_kept(ctx, q_hat, b.err));
    CK(launch_modal(ctx->g, b, b.err, b.psi, ctx->stream));
    RET(download_full(ctx, b.psi, psi_hat));
    CK(cudaStreamSynchronize(ctx->stream));
    return QGN_OK;
}

int qgn_leith(qgn_ctx* ctx, double* A8L) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    if (!A8L) return set_err(ctx, QGN_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(ctx->device));
    CK(launch_leith(ctx->g, ctx->b, ctx->b.q, leith_c12(ctx->p), ctx->stream));
    DevScalars s;
    RET(read_scalars(ctx, &s));
    std::memcpy(A8L, s.A8L, sizeof(double) * ctx->g.nz);
    return QGN_OK;
}

int qgn_diagnostics(qgn_ctx* ctx, double* ke_layer, double* spectrum, int nbins) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    if (!ke_layer) return set_err(ctx, QGN_ERR_ARG, "NULL argument");
    if (spectrum && nbins <= 0) return set_err(ctx, QGN_ERR_ARG, "nbins <= 0");
    CK(cudaSetDevice(ctx->device));
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    const size_t need = (size_t)g.nz * (1 + (spectrum ? nbins : 0));
    if (b.diag) { cudaFree(b.diag); b.diag = nullptr; }
    CK(dalloc(&b.diag, need));
    CK(launch_modal(g, b, b.q, b.psi, ctx->stream));
    CK(launch_ke(g, b, b.psi, b.Hw, b.diag, ctx->stream));
    if (spectrum) CK(launch_ke_spectrum(g, b.psi, b.Hw, nbins, b.diag + g.nz, ctx->stream));
    CK(cudaMemcpyAsync(ke_layer, b.diag, sizeof(double) * g.nz, cudaMemcpyDeviceToHost, ctx->stream));
    if (spectrum)
        CK(cudaMemcpyAsync(spectrum, b.diag + g.nz, sizeof(double) * (size_t)g.nz * nbins, cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return QGN_OK;
}

int qgn_energetics(qgn_ctx* ctx, double* ke_layer, double* ape_layer, double* enstrophy_layer) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    if (!ke_layer && !ape_layer && !enstrophy_layer) return set_err(ctx, QGN_ERR_ARG, "all outputs NULL");
    CK(cudaSetDevice(ctx->device));
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    if (b.diag) { cudaFree(b.diag); b.diag = nullptr; }
    CK(dalloc(&b.diag, (size_t)3 * g.nz));
    CK(launch_modal(g, b, b.q, b.psi, ctx->stream));
    CK(launch_energetics(g, b, b.q, b.psi, b.diag, ctx->stream));
    double* outs[3] = {ke_layer, ape_layer, enstrophy_layer};
    for (int c = 0; c < 3; ++c)
        if (outs[c])
            CK(cudaMemcpyAsync(outs[c], b.diag + (size_t)c * g.nz, sizeof(double) * g.nz, cudaMemcpyDeviceToHost,
                               ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return QGN_OK;
}

int qgn_physical(qgn_ctx* ctx, const double* q_hat, double* q_phys, double* psi_phys) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    CK(cudaSetDevice(ctx->device));
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    const size_t np = (size_t)g.nz * g.ny * g.nx;
    if (!b.phys) CK(dalloc(&b.phys, np));
    const double2* src = b.q;
    if (q_hat) {
        RET(upload_kept(ctx, q_hat, b.err));
        src = b.err;
    }
    if (q_phys) {
        CK(launch_to_phys(g, b, src, b.phys, ctx->stream));
        CK(cudaMemcpyAsync(q_phys, b.phys, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (psi_phys) {
        CK(launch_modal(g, b, src, b.psi, ctx->stream));
        CK(launch_to_phys(g, b, b.psi, b.phys, ctx->stream));
        CK(cudaMemcpyAsync(psi_phys, b.phys, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return QGN_OK;
}

int qgn_physical_modal(qgn_ctx* ctx, const double* q_hat, double* q_mode, double* p_mode, double* J_mode) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    if (!q_mode || !p_mode || !J_mode) return set_err(ctx, QGN_ERR_ARG, "NULL output");
    CK(cudaSetDevice(ctx->device));
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    const Geom gf = full_geom(g);
    const size_t np = (size_t)g.nz * g.ny * g.nx;
    const size_t half = gf.hsize(), fc = gf.csize();
    // scratch: 3 outputs + 3 physical work fields (doubles), full half field + 2 full spectra (double2)
    const size_t need = 6 * np + 2 * (half + 2 * fc);
    if (!b.modal_scratch) CK(dalloc(&b.modal_scratch, need));
    double* outs = b.modal_scratch;
    double* phys3 = outs + 3 * np;
    double2* full_half = reinterpret_cast<double2*>(outs + 6 * np);
    double2* fa = full_half + half;
    double2* fb = fa + fc;
    const double2* src = b.q;
    if (q_hat) {
        RET(upload_kept(ctx, q_hat, b.err));
        src = b.err;
    }
    CK(launch_modal_fields(g, b, src, outs, outs + np, outs + 2 * np, full_half, fa, fb, phys3, ctx->stream));
    CK(cudaMemcpyAsync(q_mode, outs, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(p_mode, outs + np, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(J_mode, outs + 2 * np, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return QGN_OK;
}

int qgn_set_state_physical(qgn_ctx* ctx, const double* q_phys, double t, double dt) {
    if (!ctx) return QGN_ERR_ARG;
    ProfScope ps_(ctx, __func__);
    ++ctx->state_version;
    if (!q_phys) return set_err(ctx, QGN_ERR_ARG, "q_phys is NULL");
    CK(cudaSetDevice(ctx->device));
    const Geom& g = ctx->g;
    Buffers& b = ctx->b;
    const size_t np = (size_t)g.nz * g.ny * g.nx;
    if (!b.phys) CK(dalloc(&b.phys, np));
    CK(cudaMemcpyAsync(b.phys, q_phys, sizeof(double) * np, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_from_phys(g, b, b.phys, b.q, ctx->stream));
    b.Qs[0] = b.q;
    RET(write_time(ctx, t, dt));
    ctx->halted = false;
    return QGN_OK;
}

int qgn_profile_enable(qgn_ctx* ctx, int enable) {
    if (!ctx) return QGN_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->prof.reset();
    ctx->prof.timing = enable != 0;
    return QGN_OK;
}

int qgn_profile_read(qgn_ctx* ctx, int kernel, double* total_ms, double* bytes, long long* timed,
                     long long* launches) {
    if (!ctx) return QGN_ERR_ARG;
    if (kernel < 0 || kernel >= KID_COUNT) return set_err(ctx, QGN_ERR_ARG, "kernel id out of range");
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->prof.harvest();
    if (total_ms) *total_ms = ctx->prof.total_ms[kernel];
    if (bytes) *bytes = ctx->prof.bytes[kernel];
    if (timed) *timed = ctx->prof.timed[kernel];
    if (launches) *launches = ctx->prof.launches[kernel];
    return QGN_OK;
}

const char* qgn_kernel_name(int kernel) {
    static const char* names[KID_COUNT] = {"modal", "yinv", "xpass", "yfwd", "xinv1", "xfwd1", "yfwd1",
                                           "ark_stage", "ark_update", "combo", "lincomb", "parseval",
                                           "scalar", "layout"};
    if (kernel < 0 || kernel >= KID_COUNT) return "";
    return names[kernel];
}

int qgn_debug_read(qgn_ctx* ctx, int which, double* out, long long count) {
    if (!ctx || !out) return QGN_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    const Buffers& b = ctx->b;
    const double2* src = nullptr;
    size_t n = 0;
    switch (which) {
        case 0: src = b.q; n = ctx->g.csize(); break;
        case 1: src = b.psi; n = ctx->g.csize(); break;
        case 2: src = b.hq; n = ctx->g.hsize(); break;
        case 3: src = b.hp; n = ctx->g.hsize(); break;
        case 4: src = b.hu; n = ctx->g.hsize(); break;
        case 5: src = b.hpp; n = 2 * ctx->g.hsize(); break;
        default: return set_err(ctx, QGN_ERR_ARG, "unknown buffer");
    }
    if ((size_t)count < 2 * n) return set_err(ctx, QGN_ERR_ARG, "output too small");
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(out, src, sizeof(double2) * n, cudaMemcpyDeviceToHost));
    return QGN_OK;
}

int qgn_stream(qgn_ctx* ctx, void** stream) {
    if (!ctx || !stream) return QGN_ERR_ARG;
    *stream = (void*)ctx->stream;
    return QGN_OK;
}

int qgn_rejects(qgn_ctx* ctx, long long* count) {
    if (!ctx || !count) return QGN_ERR_ARG;
    DevScalars s;
    RET(read_scalars(ctx, &s));
    *count = s.rejected;
    return QGN_OK;
}

const char* qgn_last_error(const qgn_ctx* ctx) {
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

int qgn_check_failures(qgn_ctx* ctx, long long* failures) {
    if (!ctx || !failures) return QGN_ERR_ARG;
#ifdef QGN_CHECK
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long n = 0;
    CK(cudaMemcpy(&n, ctx->chk, sizeof(n), cudaMemcpyDeviceToHost));
    *failures = (long long)n;
#else
    *failures = -1;
#endif
    return QGN_OK;
}

int qgn_destroy(qgn_ctx* ctx) {
    if (!ctx) return QGN_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    closure_free(ctx);
    free_all(ctx);
    delete ctx;
    return QGN_OK;
}

}  // extern "C"
