/*
 * qgn_probe.h -- throughput probe of libqgn_b200 for the FP64 roofline.
 *
 * Not part of the drop-in boundary (include/qgn_gpu.h) and without a counterpart in the
 * reference: the transforms of the right-hand side run near the FP64 ridge of the GPU, so
 * their FLOP fraction is reported beside the HBM one, and its denominator is measured on the
 * device that runs them rather than taken from a data sheet.
 */
#ifndef QGN_PROBE_H
#define QGN_PROBE_H

#ifdef __cplusplus
extern "C" {
#endif

/*
 * FP64 fused multiply-add throughput of the current device: a grid of 8 CTAs of 256 threads
 * per SM, each thread running 32 independent FMA chains per iteration, timed with CUDA events
 * on a private stream (two untimed launches, then the best of `reps` launches, reps <= 0 -> 5).
 * tflops receives 2 x FMAs / seconds / 1e12 of the best launch and ms (if not null) its
 * duration.  QGN_ERR_NO_DEVICE without an sm_100 device, QGN_ERR_CUDA if a CUDA call fails.
 */
int qgn_probe_fp64_fma(int reps, double* tflops, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* QGN_PROBE_H */
