// rhs_static.cu -- one GetRHS evaluation that allocates no device memory.
//
// For hosts that cannot call cudaMalloc from the code that evaluates the model: a
// component coupled into a larger application whose device memory is owned by the
// application (an OpenACC/OpenMP-offload data region, or a pool carved up at start-up),
// or a time loop that must not take cudaMalloc's implicit device synchronisation.  The
// caller passes device pointers for q_hat and the result; every intermediate lives in
// one file-scope __device__ array of QGN_STATIC_SCRATCH_BYTES.
//
// The array belongs to the library's module: every GPU on which the library is used
// holds it until the process exits.  All calls share it and it keeps the contents of the
// last call, so calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race.  Nothing in it needs to start at zero: each stage
// writes every element a later stage reads.
#include "qgn_internal.cuh"
#include "fft.cuh"

#include <cmath>
#include <cstring>
#include <mutex>

namespace qgn {

constexpr size_t kStaticScratchBytes = (size_t)QGN_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// device address of the scratch array on the current device (looked up once per device)
cudaError_t scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

// the reference's q_hat(nx/2+1,ny,nz) in device memory -> compact kept modes, (0,0) zeroed
__global__ void k_full_to_compact_dev(Geom g, const double2* __restrict__ full, double2* __restrict__ c) {
    QGN_PDL_ENTRY();
    const size_t n = g.csize();
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(e % g.nky);
        const size_t r = e / g.nky;
        const int kx = (int)(r % g.nkx);
        const int l = (int)(r / g.nkx);
        const int j = g.jfull(m);
        double2 v = full[((size_t)l * g.ny + j) * g.nxh + kx];
        if (kx == 0 && m == 0) v = make_double2(0.0, 0.0);
        c[e] = v;
    }
}

// compact -> the reference's layout with zeros in the dealiased band
__global__ void k_compact_to_full_dev(Geom g, const double2* __restrict__ c, double2* __restrict__ full) {
    QGN_PDL_ENTRY();
    const size_t total = (size_t)g.nz * g.ny * g.nxh;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % g.nxh);
        const size_t r = e / g.nxh;
        const int j = (int)(r % g.ny);
        const int l = (int)(r / g.ny);
        double2 v = make_double2(0.0, 0.0);
        const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
        if (i < g.nkx && kept) v = c[((size_t)l * g.nkx + i) * g.nky + (j < g.kylo ? j : j - g.kyshift)];
        full[e] = v;
    }
}

// exp(-2 pi i m/n) for m in [0,n)
__global__ void k_twiddle_table(int n, double2* __restrict__ tw) {
    QGN_PDL_ENTRY();
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_double2(c, -s);
}

bool pow2_in(int n, int lo, int hi) { return n >= lo && n <= hi && (n & (n - 1)) == 0; }

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace qgn

using namespace qgn;

extern "C" int qgn_rhs_static(const qgn_params* p, const double* H, const double* uBar, const double* qyBar,
                              const double* Modes, const double* EVals, const double* q_hat_dev, double* rhs_dev,
                              void* stream) {
    if (!p || !H || !uBar || !qyBar || !Modes || !EVals || !q_hat_dev || !rhs_dev) return QGN_ERR_ARG;
    if (!pow2_in(p->nx, 16, 2048) || !pow2_in(p->ny, 16, 2048) || p->nz < 2 || p->nz > kMaxNZ) return QGN_ERR_CONFIG;
    if (!(p->Lx > 0) || !(p->Ly > 0) || !(p->Htot > 0)) return QGN_ERR_CONFIG;
    const int nz = p->nz;
    for (int k = 0; k < nz; ++k)
        if (!(H[k] > 0) || !std::isfinite(H[k]) || !std::isfinite(uBar[k]) || !std::isfinite(qyBar[k]) ||
            !std::isfinite(EVals[k]))
            return QGN_ERR_CONFIG;
    // the same checks qgn_create makes on the mode matrix and the scalar parameters
    for (int i = 0; i < nz * nz; ++i)
        if (!std::isfinite(Modes[i])) return QGN_ERR_CONFIG;
    const double scal[] = {p->Lx, p->Ly, p->Htot, p->beta, p->A2, p->A8, p->r0, p->C_d};
    for (double v : scal)
        if (!std::isfinite(v)) return QGN_ERR_CONFIG;

    int ndev = 0, dev = 0, major = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10) {
        cudaGetLastError();
        return QGN_ERR_NO_DEVICE;
    }
    // the constant blocks are copied from this call's stack: a capture would record copies
    // from a frame that is gone when the graph runs, so the call refuses to be captured
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap) != cudaSuccess) return QGN_ERR_CUDA;
    if (cap != cudaStreamCaptureStatusNone) return QGN_ERR_CONFIG;

    Geom g;
    g.nx = p->nx; g.ny = p->ny; g.nz = nz; g.nxh = p->nx / 2 + 1;
    g.nkx = p->nx / 3; g.kylo = p->ny / 3; g.kyshift = p->ny / 3 + 1; g.nky = p->ny - p->ny / 3 - 1;
    g.nkxp = (g.nkx + 3) / 4 * 4;
    const double pi = 4.0 * std::atan(1.0);
    g.dkx = 2.0 * pi / p->Lx;
    g.dky = 2.0 * pi / p->Ly;
    g.inv_nxny = 1.0 / ((double)p->nx * (double)p->ny);

    // carve the scratch array: half-transformed fields, drag rows, compact q/psi/out,
    // twiddles and the constant blocks, each aligned to 256 bytes
    const size_t hb = sizeof(double2) * g.hsize(), db = sizeof(double2) * (size_t)g.ny * g.nkxp;
    const size_t cb = sizeof(double2) * g.csize();
    size_t off[16];
    size_t total = 0;
    const size_t sizes[13] = {hb, hb, hb, 2 * hb, 0, 2 * db, 0, cb, cb, cb, sizeof(double2) * (size_t)g.nx,
                              sizeof(double2) * (size_t)g.ny, sizeof(LayerConst) + sizeof(ModalConst) + 256};
    for (int i = 0; i < 13; ++i) {
        off[i] = total;
        total += align256(sizes[i]);
    }
    if (total > kStaticScratchBytes) return QGN_ERR_TOO_LARGE;

    unsigned char* base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return QGN_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    Buffers b;
    b.hq = reinterpret_cast<double2*>(base + off[0]);
    b.hp = reinterpret_cast<double2*>(base + off[1]);
    b.hu = reinterpret_cast<double2*>(base + off[2]);
    b.hpp = reinterpret_cast<double2*>(base + off[3]);
    b.hpd = reinterpret_cast<double2*>(base + off[5]);
    double2* qc = reinterpret_cast<double2*>(base + off[7]);
    double2* pc = reinterpret_cast<double2*>(base + off[8]);
    double2* oc = reinterpret_cast<double2*>(base + off[9]);
    b.twx = reinterpret_cast<double2*>(base + off[10]);
    b.twy = reinterpret_cast<double2*>(base + off[11]);
    b.lc = reinterpret_cast<LayerConst*>(base + off[12]);
    b.mc = reinterpret_cast<ModalConst*>(base + off[12] + align256(sizeof(LayerConst)));

    // constants of the RHS and of GetPsi (QGN_Module.f90:268-292, 315-341); the host blocks
    // are copied from pageable memory, which the runtime stages before returning
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
            mc.proj[k * nz + kk] = H[kk] * Modes[kk + (size_t)k * nz];
            mc.back[k * nz + kk] = Modes[k + (size_t)kk * nz];
        }
        mc.evals[k] = EVals[k];
    }
    mc.Htot = p->Htot;
    if (cudaMemcpyAsync(b.lc, &lc, sizeof(lc), cudaMemcpyHostToDevice, s) != cudaSuccess) return QGN_ERR_CUDA;
    if (cudaMemcpyAsync(b.mc, &mc, sizeof(mc), cudaMemcpyHostToDevice, s) != cudaSuccess) return QGN_ERR_CUDA;
    b.mc_h = &mc;   // read while this call launches its kernels

    ::qgn::launch(k_twiddle_table, (g.nx + 255) / 256, 256, 0, s, g.nx, b.twx);
    ::qgn::launch(k_twiddle_table, (g.ny + 255) / 256, 256, 0, s, g.ny, b.twy);
    const int blocks = 148 * 8;
    ::qgn::launch(k_full_to_compact_dev, blocks, 256, 0, s, g, reinterpret_cast<const double2*>(q_hat_dev), qc);
    if (cudaGetLastError() != cudaSuccess) return QGN_ERR_CUDA;
    if (launch_modal(g, b, qc, pc, s) != cudaSuccess) return QGN_ERR_CUDA;
    if (launch_rhs(g, b, qc, pc, oc, p->C_d != 0.0, s) != cudaSuccess) return QGN_ERR_CUDA;
    ::qgn::launch(k_compact_to_full_dev, blocks, 256, 0, s, g, oc, reinterpret_cast<double2*>(rhs_dev));
    if (cudaGetLastError() != cudaSuccess) return QGN_ERR_CUDA;
    return QGN_OK;
}
