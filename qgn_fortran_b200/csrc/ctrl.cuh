// ctrl.cuh -- the PI step-size controllers of the adaptive schemes, shared by the
// single-context controller kernel and the ensemble controller.
#pragma once
#include "qgn_internal.cuh"

namespace qgn {

// One accept/reject decision (ARK43_QGLeith.f90:124-138, ARK43.f90:108-124, BSRK3.f90:35-48).
// kind 0: ARK43_QGLeith (reject x0.5, safety 0.2); 1: ARK43 (x0.75, 0.75); 2: BSRK3.
// err1 = dt * max|err_phys| from sc->maxbits (the unnormalised maximum) times inv_n = 1/(nx*ny).
// Besides the reference's accept/reject, the device keeps the bounded-retry and NaN checks:
// a non-finite error estimate or max_rejects consecutive rejections halt the run with a
// status.  Returns 1 when the attempt is to be repeated.
__device__ __forceinline__ unsigned ctrl_decide(int kind, double inv_n, double TOL, double dt_max, int max_rejects,
                                                DevScalars* sc) {
    const double M = __longlong_as_double((long long)sc->maxbits);
    const double dt = sc->dt;
    double err1;
    if (kind == 2) err1 = dt * (M * inv_n);
    else err1 = dt * M * inv_n;
    sc->err1 = err1;
    sc->attempts += 1;
    unsigned again = 0;
    if (sc->wait_timeout) {   // a transform of this attempt ran on data it never received
        sc->accept = 0;
        sc->halt = 1;
        sc->status = QGN_ERR_CUDA;
    } else if (!(err1 == err1) || isinf(err1)) {
        sc->nonfinite = 1;
        sc->accept = 0;
        sc->halt = 1;
        sc->status = QGN_ERR_NONFINITE;
    } else if (err1 > TOL) {
        sc->dt = (kind == 0 ? 0.5 : 0.75) * dt;
        sc->accept = 0;
        sc->rejected += 1;
        sc->rejects_step += 1;
        if (sc->rejects_step >= max_rejects) {
            sc->halt = 1;
            sc->status = QGN_ERR_REJECT_LIMIT;
        } else {
            again = 1;
        }
    } else {
        sc->accept = 1;
        sc->accepted += 1;
        sc->t = sc->t + dt;
        const double err0 = sc->err0;
        double nd;
        if (kind == 0) nd = dt * pow(0.2 * TOL / err1, 0.075) * pow(err0 / err1, 0.1);
        else if (kind == 1) nd = dt * pow(0.75 * TOL / err1, 0.075) * pow(err0 / err1, 0.1);
        else nd = dt * pow(0.75 * TOL / err1, 0.1) * pow(err0 / err1, 0.4 / 3.0);
        sc->dt = nd < dt_max ? nd : dt_max;
        sc->err0 = err1;
    }
    return again;
}

}  // namespace qgn
