// qgn_internal.cuh -- device data layout, context and launch wrappers of the QGN path.
//
// HBM layout (all FP64 complex = double2):
//   compact spectral field  [nz][nkx][nky]   -- only the modes DeAlias keeps
//       (QGN_Module.f90:194-204): kx index i in [0, nx/3), ky index j in
//       [0, ny/3) U [2(ny/3)+1, ny); compact m < ny/3 -> j = m, else j = m + ny/3 + 1.
//       ky is the contiguous axis so the y transforms stream whole columns.
//   half-transformed field  [nz][ny][nkxp]   -- x still spectral (kept kx only), y physical;
//       the row layout the x pass streams, stored as packed row pairs (see rhs_kernels.cu).
//       nkxp = nkx rounded up to a multiple of 4.
//   Mode (0,0) of every compact field is held at zero, as DeAlias does.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/qgn_gpu.h"
#include "../../include/qgn_gpu_debug.h"
#include "prof.cuh"
#include "launch.cuh"

namespace qgn {

constexpr int kMaxNZ = 32;
constexpr int kTKX = 4;   // kx columns per CTA in the y-pass kernels

struct Geom {
    int nx, ny, nz, nxh;
    int nkx, nky, kylo, kyshift, nkxp;
    double dkx, dky, inv_nxny;
    unsigned long long* chk = nullptr;   // failed-check counter of the bounds-checked build (device)
    int* wait_err = nullptr;             // set to 1 when a bounded device wait runs out (device);
                                         // null: the kernels take no path that waits
    __host__ __device__ size_t csize() const { return (size_t)nz * nkx * nky; }
    __host__ __device__ size_t hsize() const { return (size_t)nz * ny * nkxp; }
    __host__ __device__ int jfull(int m) const { return m < kylo ? m : m + kyshift; }
    __host__ __device__ double kyval(int j) const { return dky * (double)(j <= ny / 2 ? j : j - ny); }
};

// Bounds-checked build (compile every source with -DQGN_CHECK; qgn_fortran_b200.build(check=True)
// makes libqgn_b200_check.so).  The right-hand-side tile bodies, GetPsi and the stage
// combinations test each global index against the length of the array it addresses -- compact
// fields g.csize(), packed row pairs g.hsize(), forward x transforms 2 g.hsize() -- before the
// access.  An index out of range is not accessed (a load yields zero) and increments the
// context's counter, which qgn_check_failures reads: no trap, no fault, the context stays
// usable.  In the normal build in_bounds is the constant true and the checks compile away.
#ifdef QGN_CHECK
__device__ __forceinline__ bool in_bounds(const Geom& g, size_t i, size_t n) {
    if (i < n) return true;
    if (g.chk) atomicAdd(g.chk, 1ull);
    return false;
}
#else
__device__ __forceinline__ constexpr bool in_bounds(const Geom&, size_t, size_t) { return true; }
#endif

// Per-layer physical constants of the RHS (QGN_Module.f90:268-292).
struct LayerConst {
    double uBar[kMaxNZ];
    double betaq[kMaxNZ];   // beta + qyBar(k)
    double ekman;           // r0*Htot/H(nz)
    double dragc;           // C_d*Htot/H(nz)
    double A2, A8;
    int explicit_diss;
};

// Modal-inversion coefficients (GetPsi, QGN_Module.f90:315-341).
struct ModalConst {
    double proj[kMaxNZ * kMaxNZ];   // proj[k*nz+kk] = H(kk)*Modes(kk,k)
    double back[kMaxNZ * kMaxNZ];   // back[k*nz+kk] = Modes(k,kk)
    double evals[kMaxNZ];
    double Htot;
};

// GetPsi constants of a fixed layer count (2, 4, 8, 16) passed by value as a kernel parameter:
// the unrolled arithmetic reads the matrix entries straight from the constant bank, with no
// shared-memory staging and no load instructions
template <int NZ>
struct ModalParams {
    double proj[NZ * NZ];
    double back[NZ * NZ];
    double ev[NZ];
    double Htot;
};
template <int NZ>
inline ModalParams<NZ> modal_params(const ModalConst& mc) {
    ModalParams<NZ> m;
    for (int i = 0; i < NZ * NZ; ++i) {
        m.proj[i] = mc.proj[i];
        m.back[i] = mc.back[i];
    }
    for (int i = 0; i < NZ; ++i) m.ev[i] = mc.evals[i];
    m.Htot = mc.Htot;
    return m;
}

// The GetPsi constants as a kernel argument: by value for a fixed layer count, else the device
// copy, which the kernel stages in shared memory (modal_view)
template <int NZ>
struct ModalArg {
    ModalParams<NZ> m;
};
template <>
struct ModalArg<0> {
    const ModalConst* mc;
};

// shared-memory staging arrays of a GetPsi kernel (used only for NZ = 0)
#define QGN_MODAL_SHARED(NZ)                                                      \
    __shared__ double s_proj[(NZ) > 0 ? 1 : kMaxNZ * kMaxNZ];                     \
    __shared__ double s_back[(NZ) > 0 ? 1 : kMaxNZ * kMaxNZ];                     \
    __shared__ double s_ev[(NZ) > 0 ? 1 : kMaxNZ]

struct ModalView {
    const double* proj;
    const double* back;
    const double* ev;
    double Htot;
};

// where the kernel reads the constants from; for NZ = 0 every thread of the block must call
// this (it stages the device copy and synchronises)
template <int NZ>
__device__ __forceinline__ ModalView modal_view(const ModalArg<NZ>& a, double* s_proj, double* s_back, double* s_ev,
                                                int nz) {
    if constexpr (NZ > 0) {
        return ModalView{a.m.proj, a.m.back, a.m.ev, a.m.Htot};
    } else {
        for (int i = threadIdx.x; i < nz * nz; i += blockDim.x) {
            s_proj[i] = a.mc->proj[i];
            s_back[i] = a.mc->back[i];
        }
        for (int i = threadIdx.x; i < nz; i += blockDim.x) s_ev[i] = a.mc->evals[i];
        __syncthreads();
        return ModalView{s_proj, s_back, s_ev, a.mc->Htot};
    }
}

// Device scalars of the adaptive controllers.  The controller kernel makes every
// accept/reject/halt decision on the device, so a step can run without host round trips.
struct DevScalars {
    double t, dt, err0, err1;
    unsigned long long maxbits;   // bit pattern of max|err_phys| (non-negative doubles)
    int accept;                   // 1 accepted, 0 rejected
    int nonfinite;
    int halt;                     // sticky: set with status, cleared by a state upload
    int status;                   // QGN_ERR_* of the failure that set halt
    int rejects_step;             // consecutive rejections in the current step
    unsigned int red_count;       // blocks done in a last-block reduction (0 between launches)
    long long accepted;           // accepted steps since creation
    long long attempts;           // attempts (accepted + rejected) since creation
    long long rejected;           // rejected attempts since creation
    int wait_timeout;             // a bounded device wait (bulk-copy completion) ran out; sticky
    double A8L[kMaxNZ];
};

struct Buffers {
    double2* q = nullptr;        // state q_hat (compact)
    double2* qnew = nullptr;     // candidate update
    double2* N[6] = {};          // stage right-hand sides
    double2* Qs[6] = {};         // stage states (Qs[0] aliases q for the ARK schemes)
    double2* psi = nullptr;      // psi of the field being evaluated
    double2* err = nullptr;      // error combination (compact)
    double2* hq = nullptr;       // packed row pairs of q (and of single fields) [nz][ny/2][2][nkxp]
    double2* hp = nullptr;       // packed row pairs of v = i kx psi
    double2* hu = nullptr;       // packed row pairs of u = -i ky psi
    double2* hpp = nullptr;      // forward x transforms P[k], P[nx-k] of u*q + i v*q [nz][ny][2][nkxp]
    double2* hpd = nullptr;      // same for |u|u + i |u|v of the bottom layer [ny][2][nkxp]
    double2* xfer = nullptr;     // host-order kept modes [nz][nky][nkx]
    double2* full = nullptr;     // full CCE field [nz][ny][nxh] (lazy)
    double* phys = nullptr;      // physical field [nz][ny][nx] (lazy)
    double2* twx = nullptr;      // twiddles exp(-2 pi i m/nx)
    double2* twy = nullptr;      // twiddles exp(-2 pi i m/ny)
    float2* twx32 = nullptr;     // the same rounded to FP32 (mixed mode)
    float2* twy32 = nullptr;
    double* red = nullptr;       // reduction partials
    double* Hw = nullptr;        // H(k)/Htot per layer
    double* diag = nullptr;      // diagnostics output (lazy)
    double* modal_scratch = nullptr;  // WriteQPmodal work space (lazy)
    double* snap = nullptr;           // closure training-sample work space (lazy)
    LayerConst* lc = nullptr;
    ModalConst* mc = nullptr;
    const ModalConst* mc_h = nullptr;   // host copy of *mc, the source of ModalParams
    DevScalars* sc = nullptr;
};

// the kernel argument of the GetPsi constants (NZ = 0, or no host copy: the device copy)
template <int NZ>
inline ModalArg<NZ> modal_arg(const Buffers& b) {
    if constexpr (NZ > 0) return ModalArg<NZ>{modal_params<NZ>(*b.mc_h)};
    else return ModalArg<0>{b.mc};
}

}  // namespace qgn

namespace qgn {
struct Closure;
}

struct qgn_ctx {
    qgn_params p{};
    int scheme = 0, precision = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    qgn::Geom g{};
    qgn::Buffers b{};
    std::vector<double> H, uBar, qyBar, Modes, EVals;
    // stepper memory (the reference's `save` variables); BSRK3's RHS0 and AB3's history
    // live in b.N[0..1], err0 / r0 in the device scalars
    int output_mode = QGN_OUTPUT_KEPT;   // what qgn_step / qgn_advance write back (qgn_set_output)
    unsigned long long* chk = nullptr;   // device failed-check counter (bounds-checked build only)
    bool first_call = true;
    int ab_calls = 0;
    bool halted = false;           // a step failed; cleared by the next state upload
    long long state_version = 0;   // bumped by every call that changes the state outside an ensemble
    qgn::Closure* closure = nullptr;   // learned closure of a coarse ARK43_QGLeith model (closure.cu)
    qgn::ModalConst mc_host{};     // host copy of b.mc (b.mc_h points here)
    double* host_pin = nullptr;    // pinned scalar readback
    std::vector<void*> owned;      // every device allocation made at creation
    std::string last_error;
    qgn::Prof prof;                // launch counts and per-kernel event timing
    // graph-launched steps (ARK schemes): one executable per role of the two state buffers
    bool graphs_ready = false;
    bool graphs_off = false;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    double2* gbuf[2] = {nullptr, nullptr};
    cudaStream_t body_stream = nullptr;
    long long g_pro[qgn::KID_COUNT] = {};   // kernel launches per executed step prologue
    long long g_body[qgn::KID_COUNT] = {};  // kernel launches per attempt
};

namespace qgn {

// the learned closure's tensors (rhs_kernels.cu): xout = NHWC BF16 [ny][nx][cin_p] with
// channels (q_0..q_nz-1, psi_0..psi_nz-1) * scale; out = forward transform (compact, dealiased)
// of channel l of the planar FP32 y[channel][ny*nx] divided by osc[l].  hq, hu and h are
// packed-row scratch of g.hsize() elements each (h may be hq).
cudaError_t launch_closure_input(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* hq,
                                 double2* hu, const float* scale, void* xout, int cin_p, cudaStream_t s);
cudaError_t launch_closure_output(const Geom& g, const Buffers& b, const float* y, int cout_p, const float* osc,
                                  double2* h, double2* out, cudaStream_t s);

// ---- learned closure (closure.cu) and graph invalidation (capi.cu) -----------------------
int closure_eval(qgn_ctx* ctx, const double2* psi, cudaStream_t st);
int closure_fork(qgn_ctx* ctx);
int closure_join(qgn_ctx* ctx);
void closure_free(qgn_ctx* ctx);
const double2* closure_tendency(const qgn_ctx* ctx);
void drop_graphs(qgn_ctx* ctx);

// ---- launch wrappers (rhs_kernels.cu) -------------------------------------------------
cudaError_t launch_modal(const Geom& g, const Buffers& b, const double2* q, double2* psi, cudaStream_t s);
// extra (optional, compact): a tendency added to the RHS on the kept modes (learned closure)
cudaError_t launch_rhs(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                       bool do_drag, cudaStream_t s, const double2* extra = nullptr);
// the x and y-forward passes of launch_rhs, when the y-inverse already ran, and each alone
cudaError_t launch_rhs_tail(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                            bool do_drag, cudaStream_t s, const double2* extra = nullptr);
cudaError_t launch_rhs_x(const Geom& g, const Buffers& b, bool do_drag, cudaStream_t s);
cudaError_t launch_rhs_yfwd(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double2* out,
                            bool do_drag, cudaStream_t s, const double2* extra = nullptr);
cudaError_t launch_rhs32(const Geom& g, const Buffers& b, const float2* q, const float2* psi, float2* out, bool do_drag,
                         cudaStream_t s);
// y-inverse + x-pass of one compact field with a max|.| reduction into sc->maxbits
cudaError_t launch_maxabs_phys(const Geom& g, const Buffers& b, const double2* f, DevScalars* sc, cudaStream_t s);
cudaError_t launch_maxabs_phys32(const Geom& g, const Buffers& b, const float2* f, DevScalars* sc, cudaStream_t s);
// physical field (c2r/(nx*ny)) of a compact field into b.phys ([nz][ny][nx])
cudaError_t launch_to_phys(const Geom& g, const Buffers& b, const double2* f, double* out, cudaStream_t s);
// the fields of WriteQPmodal (QGN_Module.f90:381-440): q_mode, psi_mode and J_mode in physical
// space (out_* [nz][ny][nx]); scratch: full_half [nz][ny][round4(nxh)], fa/fb full compact
// [nz][nxh][ny], phys3 three physical fields
Geom full_geom(const Geom& g);
cudaError_t launch_modal_fields(const Geom& g, const Buffers& b, const double2* q, double* out_q, double* out_p,
                                double* out_j, double2* full_half, double2* fa, double2* fb, double* phys3,
                                cudaStream_t s);
// forward transform + dealias of a physical field [nz][ny][nx] into a compact field
cudaError_t launch_from_phys(const Geom& g, const Buffers& b, const double* phys, double2* out, cudaStream_t s);

// ---- layout kernels (layout.cu) -------------------------------------------------------
cudaError_t launch_xfer_to_compact(const Geom& g, const double2* xfer, double2* c, cudaStream_t s);
cudaError_t launch_compact_to_xfer(const Geom& g, const double2* c, double2* xfer, cudaStream_t s);
cudaError_t launch_xfer_to_full(const Geom& g, const double2* xfer, double2* full, cudaStream_t s);
cudaError_t launch_nonfinite_check(const Geom& g, const double2* c, DevScalars* sc, cudaStream_t s);

// ---- stepper kernels (stepper.cu) -----------------------------------------------------
struct Combo {
    const double2* R[4];
    double a[4];
    int n;
};
cudaError_t launch_leith(const Geom& g, const Buffers& b, const double2* q, double c12, cudaStream_t s);
cudaError_t launch_ark_stage(const Geom& g, const Buffers& b, int stage, cudaStream_t s);
bool stage_yinv_ok(const Geom& g, const Buffers& b);
cudaError_t launch_ark_stage_yinv(const Geom& g, const Buffers& b, int stage, cudaStream_t s);
cudaError_t launch_yfwd_stage_yinv(const Geom& g, const Buffers& b, int stage, const double2* extra, cudaStream_t s);
cudaError_t launch_ark_update(const Geom& g, const Buffers& b, cudaStream_t s);
cudaError_t launch_ark_stage_mixed(const Geom& g, const Buffers& b, int stage, cudaStream_t s);
cudaError_t launch_ark_update_mixed(const Geom& g, const Buffers& b, cudaStream_t s);
cudaError_t launch_modal_mixed(const Geom& g, const Buffers& b, const double2* q, float2* q32, float2* psi32,
                               cudaStream_t s);
cudaError_t launch_f2d(size_t n, const float2* a, double2* b, cudaStream_t s);
cudaError_t launch_combo(const Geom& g, const Buffers& b, const Combo& cb, const double2* q, double2* out,
                         double2* psi, bool want_psi, cudaStream_t s);
cudaError_t launch_lincomb(const Geom& g, const Combo& cb, double2* out, cudaStream_t s);
cudaError_t launch_controller(const Geom& g, const Buffers& b, int kind, double TOL, double dt_max, int max_rejects,
                              const cudaGraphConditionalHandle* loop, cudaStream_t s);
cudaError_t launch_step_gate(DevScalars* sc, const cudaGraphConditionalHandle* gate, cudaStream_t s);
cudaError_t launch_set_cond(cudaGraphConditionalHandle h, unsigned int v, cudaStream_t s);
cudaError_t launch_zero_scalar_max(DevScalars* sc, cudaStream_t s);
cudaError_t launch_advance_time(DevScalars* sc, cudaStream_t s);
cudaError_t launch_set_time(DevScalars* sc, double t, double dt, cudaStream_t s);
cudaError_t launch_ke(const Geom& g, const Buffers& b, const double2* psi, const double* Hw, double* ke, cudaStream_t s);
// per-layer kinetic energy, available potential energy and enstrophy of (q, psi): out[3*nz]
cudaError_t launch_energetics(const Geom& g, const Buffers& b, const double2* q, const double2* psi, double* out,
                              cudaStream_t s);
cudaError_t launch_ke_spectrum(const Geom& g, const double2* psi, const double* Hw, int nbins, double* spec,
                               cudaStream_t s);

}  // namespace qgn
