// context.cuh -- the evaluator context shared by the C ABI's source files.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/galop_b200.h"
#include "interp.cuh"

namespace galop {

// Reference constant pools (src/LGPConfig.h:159-168).
inline const float kRefPool8[8] = {0.0f, 1.0f, -1.0f, 3.14159f, 0.5f, 2.0f, 10.0f, 100.0f};
inline const float kRefPool16[16] = {0.0f, 1.0f, -1.0f, 3.14159f, 0.5f, 2.0f, 10.0f, 100.0f,
                              0.1f, -0.5f, 0.25f, 5.0f, 20.0f, -2.0f, 0.01f, 1000.0f};

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;  // elements
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        size_t want = std::max<size_t>(n, cap + cap / 4);
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, want * sizeof(T));
        if (e != cudaSuccess) { p = nullptr; return e; }
        cap = want;
        return cudaSuccess;
    }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

enum Ev { kEvStart = 0, kEvH2D, kEvPrepass, kEvInterp, kEvFinalize, kEvD2H, kEvCount };

}  // namespace galop

using galop::DevBuf;
using galop::kEvCount;
using galop::ConstPool;
using galop::IsaParams;
using galop::Objective;

// Total sum of squares of the targets, two passes in double in case order
// (the reference caches it per dataset: compute_ss_tot, src/Dataset.cpp:35-47).
inline double targets_ss_tot(const float* y, int64_t n) {
    if (n <= 0) return 0.0;
    double mean = 0.0;
    for (int64_t i = 0; i < n; ++i) mean += (double)y[i];
    mean /= (double)n;
    double ss = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double d = (double)y[i] - mean;
        const double d2 = d * d;
        ss += d2;
    }
    return ss;
}

// Device counters of a context: [0] work-queue head, [1..5] instruction
// totals of the call (raw, effective, interpreted, dedup copies and their
// instructions), [6] set when caller-stated device offsets are inconsistent,
// [7] size of the first register-file class in the order.
constexpr int kCounters = 8;
constexpr int kCounterBadOffsets = 6;
constexpr int kCounterClassSplit = 7;   // programs of the 8-slot class at the head of the order
constexpr int kSplitSlots = 8;          // register-file slots of the smaller interpreter

struct galop_ctx {
    galop_options opt{};
    IsaParams isa{};
    ConstPool pool{};
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;   // host-to-device copies overlapped with compute (lazy)
    cudaEvent_t seg_ev[8 * 5] = {};        // per segment: copied, pre-pass start/end, interp end, finalize end
    cudaEvent_t ev[kEvCount] = {};
    cudaEvent_t timers[8] = {};
    std::string err;

    // resident dataset (feature-major, padded)
    DevBuf<float> X, y;
    DevBuf<float> stage_aos, stage_y;
    int64_t N = -1, Np = 0;
    double ss_tot = 0.0;          // sum of squared target deviations (R^2)
    int num_inputs = 0;

    // population buffers (high-water)
    DevBuf<uint32_t> raw_words, uops, eff_raw;
    DevBuf<uint8_t> raw_lens8;
    DevBuf<int64_t> raw_off, eff_off, tiles;
    DevBuf<int32_t> eff_len, order;
    DevBuf<uint32_t> livein;      // registers each program reads before writing them (fold.cuh)
    DevBuf<float> fitness, outputs, trace;
    DevBuf<double> sse, partial;
    DevBuf<unsigned long long> counters;   // kCounters entries; layout in run_prepass
    DevBuf<unsigned int> hist;
    std::vector<int64_t> host_tmp;

    galop_stats stats{};
    int launches = 0;
    bool stats_pending = false;   // device-path call whose timings are not read yet
    bool flagged = false;         // the last pre-pass marked forwarding and live-in registers
    bool folded = false;          // the last pre-pass folded constants (interp lengths in eff_len)
    bool deduped = false;         // ... and left identical programs out (representatives in rep)
    bool class_split = false;     // ... and ordered the programs by register-file class
    DevBuf<unsigned long long> dkeys, dkeys_sorted;
    DevBuf<int32_t> dvals, dvals_sorted, rep, dhead;
    DevBuf<unsigned char> dsort_tmp;

    int fail(int code, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        err = buf;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        cudaGetLastError();   // a non-sticky error must not resurface in a later call
        return fail(e == cudaErrorMemoryAllocation ? GALOP_E_NOMEM : GALOP_E_CUDA,
                    "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    }
};

#define GALOP_CK(call, what)                                   \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return ctx->cuda_fail(_e, what); \
    } while (0)


namespace galop {
// Interpreter configuration shared by the single-population and batched paths.
int pick_k(const galop_ctx* ctx);
int pick_wpb(const galop_ctx* ctx);
const void* kernel_for(const galop_ctx* ctx, int k, int mode);
const void* kernel_for_slots(const galop_ctx* ctx, int k, int mode, int nslot);
int pick_dispatch(const galop_ctx* ctx);
UopFormat uop_format(const galop_ctx* ctx);
size_t interp_smem_bytes(const galop_ctx* ctx, int k, int wpb);
int evaluate_dense_device(galop_ctx* ctx, const uint32_t* d_words, const uint8_t* d_lens, int64_t stride,
                          int64_t n, float* d_fitness);
const void* interp_kernel_nr8(int k, int dispatch, int profile, int reduce, int mode);
const void* interp_kernel_nr16(int k, int dispatch, int profile, int reduce, int mode);
}  // namespace galop

// The fitness definition of this context for a dataset with this ss_tot.
inline Objective objective_for(const galop_ctx* ctx, double ss_tot) {
    Objective o{};
    o.kind = ctx->opt.objective == GALOP_OBJECTIVE_R2 ? galop::kObjectiveR2 : galop::kObjectiveMse;
    o.ss_tot = ss_tot;
    return o;
}
