// launch.cuh -- every kernel of the library is launched as a programmatic dependent of the
// kernel before it in the stream (CUDA programmatic dependent launch).
//
// A step of a small grid (128^2) is 30-45 short kernels whose device time is a few
// microseconds each, so the gap between one kernel's end and the next one's start is a large
// share of the step.  Launching with cudaLaunchAttributeProgrammaticStreamSerialization lets
// the next grid be scheduled while the current one finishes; stream capture turns the
// attribute into programmatic edges of the CUDA graph.  Correctness rests on one rule: the
// first statement of every kernel is QGN_PDL_ENTRY(), whose griddepcontrol.wait blocks until
// the grids this one depends on have completed and their writes are visible (a no-op when the
// kernel was not launched as a dependent).  No kernel triggers its dependents early
// (griddepcontrol.launch_dependents): the next grid is scheduled when every block of this one
// has exited, which removes the completion-to-launch gap without letting waiting blocks of
// the next grid crowd the SMs of a running one (an early trigger made 256^2 steps 20 % slower
// on B200 while saving 0.6 % at 1024^2).  tests/test_launch_rules.py checks the rule over the
// sources.  QGN_NO_PDL=1 launches without the attribute.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>

#define QGN_PDL_ENTRY() asm volatile("griddepcontrol.wait;" ::: "memory")

namespace qgn {

inline bool pdl_allowed() { return std::getenv("QGN_NO_PDL") == nullptr; }

// Opt a kernel into `bytes` of dynamic shared memory (above the 48 KB default) on the current
// device.  The attribute belongs to the device, so the opt-in is remembered per (device,
// kernel) and made again for a larger size; later launches, including those recorded into CUDA
// graphs, issue no attribute calls.
inline cudaError_t smem_opt_in(const void* kernel, int bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> done;
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_pair(dev, kernel);
    const auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done[key] = bytes;
    return e;
}
template <class... KArgs>
inline cudaError_t smem_opt_in(void (*kernel)(KArgs...), int bytes) {
    return smem_opt_in(reinterpret_cast<const void*>(kernel), bytes);
}

// kernel<<<grid, block, smem, stream>>>(args...) with the programmatic-serialization attribute;
// the error, if any, is left for cudaGetLastError like a <<<>>> launch.
template <class... KArgs, class... Args>
inline cudaError_t launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                          Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_allowed() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace qgn
