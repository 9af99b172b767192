// prof.cuh -- launch counting and CUDA-event timing of every kernel the library issues.
//
// Each launch site brackets its kernel with prof_begin/prof_end.  Launches are always
// counted; when timing is enabled (qgn_profile_enable) the bracket also records a pair of
// CUDA events on the launching stream, harvested at the next host synchronisation, so the
// per-kernel device time and the algorithmic bytes each launch must move are available
// to the caller (qgn_profile_read) without a profiler attached.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <vector>

namespace qgn {

enum KernelId {
    KID_MODAL = 0,
    KID_YINV,
    KID_XPASS,
    KID_YFWD,
    KID_XINV1,
    KID_XFWD1,
    KID_YFWD1,
    KID_STAGE,
    KID_UPDATE,
    KID_COMBO,
    KID_LINCOMB,
    KID_PARSEVAL,
    KID_SCALAR,
    KID_LAYOUT,
    KID_COUNT
};

struct Prof {
    bool timing = false;
    struct Rec {
        int id;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<cudaEvent_t> pool;
    std::vector<Rec> pending;
    double total_ms[KID_COUNT] = {};
    double bytes[KID_COUNT] = {};   // sum of algorithmic bytes over timed launches
    long long timed[KID_COUNT] = {};
    long long launches[KID_COUNT] = {};
    cudaEvent_t cur_a = nullptr;
    int cur_id = -1;

    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int id, cudaStream_t s) {
        ++launches[id];
        if (!timing) return;
        cur_a = get();
        cur_id = id;
        cudaEventRecord(cur_a, s);
    }
    void end(int id, cudaStream_t s, double nbytes) {
        if (!timing || cur_id != id || !cur_a) return;
        cudaEvent_t b = get();
        cudaEventRecord(b, s);
        pending.push_back(Rec{id, cur_a, b, nbytes});
        cur_a = nullptr;
        cur_id = -1;
    }
    // call after the stream has been synchronised
    void harvest() {
        for (const Rec& r : pending) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
                total_ms[r.id] += ms;
                bytes[r.id] += r.bytes;
                ++timed[r.id];
            }
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    void reset() {
        harvest();
        for (int i = 0; i < KID_COUNT; ++i) {
            total_ms[i] = 0.0;
            bytes[i] = 0.0;
            timed[i] = 0;
            launches[i] = 0;
        }
    }
    void release() {
        harvest();
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
        pool.clear();
    }
};

// The profiler of the context whose API call is running on this host thread.
Prof*& current_prof();

inline void prof_begin(int id, cudaStream_t s) {
    if (Prof* p = current_prof()) p->begin(id, s);
}
inline void prof_end(int id, cudaStream_t s, double nbytes) {
    if (Prof* p = current_prof()) p->end(id, s, nbytes);
}

// An NVTX range (Nsight Systems timelines) for the scope: every C-ABI call opens one named after
// itself, and the scheme drivers one per prologue, attempt and stage (with graph-launched steps
// the ranges mark the graph launches).  NVTX3 is header-only: without an attached tool a push or
// pop is a check of a null function pointer.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace qgn

#define QGN_NVTX_CAT2(a, b) a##b
#define QGN_NVTX_CAT(a, b) QGN_NVTX_CAT2(a, b)
#define QGN_NVTX(name) ::qgn::NvtxRange QGN_NVTX_CAT(qgn_nvtx_, __LINE__)(name)

// bracket one kernel launch: QGN_LAUNCH(id, algorithmic_bytes, stream, kernel<<<...>>>(...))
#define QGN_LAUNCH(id, nbytes, stream, ...)          \
    do {                                             \
        ::qgn::prof_begin((id), (stream));           \
        __VA_ARGS__;                                 \
        ::qgn::prof_end((id), (stream), (nbytes));   \
    } while (0)
