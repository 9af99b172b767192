// cnn.cuh -- internal interface of the closure network (cnn.cu) for the closure driver.
#pragma once
#include "qgn_internal.cuh"

namespace qgn {
namespace cnn {
// channel counts of the network's input and output tensors, padded to multiples of 16
int padded_in(const qgn_cnn* net);
int padded_out(const qgn_cnn* net);
int height(const qgn_cnn* net);
int width(const qgn_cnn* net);
int real_out(const qgn_cnn* net);
// inference of `batch` samples on `stream`: x BF16 [batch][H][W][padded_in] (device), y FP32
// [batch][H][W][padded_out] or, planar, [padded_out][batch*H*W] (device); kernel launches only
int infer(qgn_cnn* net, const void* x, float* y, int batch, cudaStream_t stream, bool planar);
}  // namespace cnn
}  // namespace qgn
