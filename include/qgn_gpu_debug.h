/*
 * qgn_gpu_debug.h -- test and debugging hooks of libqgn_b200.
 *
 * Not part of the drop-in boundary (include/qgn_gpu.h): a host that replaces the reference's
 * TimeStep never needs these.  The library exports them so that its own tests can read
 * intermediate device buffers and make a bounded device wait run out on purpose.  Both have
 * no counterpart in the reference.
 */
#ifndef QGN_GPU_DEBUG_H
#define QGN_GPU_DEBUG_H

#include "qgn_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Copy one device work buffer to the host as interleaved doubles (count = capacity in
 * doubles).  which: 0 state q (compact [nz][nx/3][nky]), 1 psi of the last evaluation
 * (compact), 2..6 the half-transformed fields [nz][ny][nkxp] of the last RHS as packed row
 * pairs [nz][ny/2][2][nkxp]: 2 q, 3 v = i kx psi, 4 u = -i ky psi; 5 the forward x transforms
 * P of u*q + i v*q row by row, [nz][ny][2][nkxp] (P[k] at k and P[nx-k] at nkxp + k, for
 * k < nkx; a build with -DQGN_P_TILED=1 stores them in tiles of two kx columns instead,
 * [nz][nkxp/2][ny][2][2]).  nkxp = nx/3 rounded up to a multiple of 4.
 */
int qgn_debug_read(qgn_ctx* ctx, int which, double* out, long long count);

/*
 * Failure injection: set the fused network inference's layer counter of one tile.  A large
 * value makes that tile's bounded wait run out in the next fused launch, which then reports
 * a timeout through qgn_cnn_check without faulting or hanging the GPU.
 */
int qgn_cnn_debug_set_counter(qgn_cnn* net, int tile, unsigned int value);

/*
 * Bounds-checked build (libqgn_b200_check.so, every source compiled with -DQGN_CHECK): the
 * right-hand-side transforms and GetPsi test each global index against the length of the
 * array it addresses and skip, and count, an access out of range instead of making it.
 * failures receives the count of this context since creation (its kernels are waited for
 * first), or -1 from the normal build, which compiles no checks.  It stands in for a memory
 * checker: the checks fault nothing and leave the context usable.
 */
int qgn_check_failures(qgn_ctx* ctx, long long* failures);

#ifdef __cplusplus
}
#endif
#endif /* QGN_GPU_DEBUG_H */
