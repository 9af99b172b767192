// layout.cu -- conversions between the reference's CCE spectral layout and the compact
// column layout of the device, and state checks.
//
//   xfer     [nz][nky][nkx]  the kept modes in the reference's order (kx fastest); this is what
//            crosses PCIe (two pitched 3-D copies per direction pick them out of q_hat(nx/2+1,ny,nz))
//   compact  [nz][nkx][nky]  device working layout (ky fastest)
//   full     [nz][ny][nx/2+1] the reference's q_hat with the dealiased band as zeros
#include "qgn_internal.cuh"
#include "prof.cuh"

namespace qgn {

// 32x32 tiled transpose per layer: in [nz][R][C] -> out [nz][C][R]
__global__ void __launch_bounds__(256) k_transpose(const double2* __restrict__ in, double2* __restrict__ out,
                                                   int R, int Cc, int zero_first) {
    QGN_PDL_ENTRY();
    __shared__ double2 tile[32][33];
    const int l = blockIdx.z;
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const size_t lbase = (size_t)l * R * Cc;
    for (int dy = threadIdx.y; dy < 32; dy += 8) {
        const int r = r0 + dy, c = c0 + threadIdx.x;
        if (r < R && c < Cc) tile[dy][threadIdx.x] = in[lbase + (size_t)r * Cc + c];
    }
    __syncthreads();
    for (int dy = threadIdx.y; dy < 32; dy += 8) {
        const int c = c0 + dy, r = r0 + threadIdx.x;
        if (r < R && c < Cc) {
            double2 v = tile[threadIdx.x][dy];
            if (zero_first && r == 0 && c == 0) v = make_double2(0.0, 0.0);   // DeAlias: field(1,1,:)=0
            out[lbase + (size_t)c * R + r] = v;
        }
    }
}

// xfer [nz][nky][nkx] -> full [nz][ny][nxh] with zeros in the dealiased band
__global__ void k_xfer_to_full(Geom g, const double2* __restrict__ xfer, double2* __restrict__ full) {
    QGN_PDL_ENTRY();
    const size_t total = (size_t)g.nz * g.ny * g.nxh;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % g.nxh);
        const size_t rest = e / g.nxh;
        const int j = (int)(rest % g.ny);
        const int l = (int)(rest / g.ny);
        double2 v = make_double2(0.0, 0.0);
        const bool kept = (j < g.kylo) || (j >= g.kylo + g.kyshift);
        if (i < g.nkx && kept) {
            const int m = j < g.kylo ? j : j - g.kyshift;
            v = xfer[((size_t)l * g.nky + m) * g.nkx + i];
        }
        full[e] = v;
    }
}

// sets sc->nonfinite if any entry of a compact field is NaN or Inf
__global__ void k_nonfinite(const double2* __restrict__ c, size_t n, DevScalars* sc) {
    QGN_PDL_ENTRY();
    int bad = 0;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const double2 v = c[e];
        if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
    }
    bad = __syncthreads_or(bad);
    if (bad && threadIdx.x == 0) atomicExch(&sc->nonfinite, 1);
}

cudaError_t launch_xfer_to_compact(const Geom& g, const double2* xfer, double2* c, cudaStream_t s) {
    dim3 grid((g.nkx + 31) / 32, (g.nky + 31) / 32, g.nz);
    QGN_LAUNCH(KID_LAYOUT, 32.0 * (double)g.csize(), s, ::qgn::launch(k_transpose, grid, dim3(32, 8), 0, s, xfer, c, g.nky, g.nkx, 1));
    return cudaGetLastError();
}

cudaError_t launch_compact_to_xfer(const Geom& g, const double2* c, double2* xfer, cudaStream_t s) {
    dim3 grid((g.nky + 31) / 32, (g.nkx + 31) / 32, g.nz);
    QGN_LAUNCH(KID_LAYOUT, 32.0 * (double)g.csize(), s, ::qgn::launch(k_transpose, grid, dim3(32, 8), 0, s, c, xfer, g.nkx, g.nky, 0));
    return cudaGetLastError();
}

cudaError_t launch_xfer_to_full(const Geom& g, const double2* xfer, double2* full, cudaStream_t s) {
    const size_t total = (size_t)g.nz * g.ny * g.nxh;
    const int blocks = (int)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
    QGN_LAUNCH(KID_LAYOUT, 16.0 * ((double)g.csize() + (double)g.nz * g.ny * g.nxh), s,
               ::qgn::launch(k_xfer_to_full, blocks, 256, 0, s, g, xfer, full));
    return cudaGetLastError();
}

cudaError_t launch_nonfinite_check(const Geom& g, const double2* c, DevScalars* sc, cudaStream_t s) {
    const size_t n = g.csize();
    const int blocks = (int)((n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8);
    QGN_LAUNCH(KID_LAYOUT, 16.0 * (double)n, s, ::qgn::launch(k_nonfinite, blocks, 256, 0, s, c, n, sc));
    return cudaGetLastError();
}

}  // namespace qgn
