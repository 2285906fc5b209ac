// runtime.cu -- evaluator context and the C ABI (include/galop_b200.h).
//
// Replaces CudaEvaluator (src/EvaluatorCuda.{h,cu}):
//   - dataset uploaded once and kept resident (src/EvaluatorCuda.cu:96-110),
//     transposed to feature-major on the device;
//   - population buffers grow to a high-water mark and are reused
//     (src/EvaluatorCuda.cu:69-81);
//   - the host pack + intron strip (src/EvaluatorCuda.cu:335-422) becomes
//     the device pre-pass of prepass.cuh;
//   - one stream, CUDA-event timings, status codes instead of exit().
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/galop_b200.h"
#include "interp.cuh"
#include "prepass.cuh"
#include "interp_wide.cuh"
#include "fold.cuh"
#include "dedup.cuh"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace galop {
const void* interp_kernel_nr8(int k, int dispatch, int profile, int reduce, int mode);
const void* interp_kernel_nr16(int k, int dispatch, int profile, int reduce, int mode);
}  // namespace galop

using namespace galop;

#include "context.cuh"

namespace galop {

// Cases per lane: the option, else 8 for the 16-byte micro-op interpreter
// (its loop's dispatch work spread over 8 cases) and 4 for the 32-bit one,
// whose register file holds all NR registers per lane in shared memory.
int pick_k(const galop_ctx* ctx) {
    const int k = ctx->opt.cases_per_lane;
    if (k == 1 || k == 2 || k == 4 || k == 8) return k;
    return ctx->opt.dispatch == 2 ? 4 : 8;
}

int pick_wpb(const galop_ctx* ctx) {
    const int w = ctx->opt.warps_per_block;
    return (w >= 1 && w <= 8) ? w : 4;
}

int pick_dispatch(const galop_ctx* ctx) {
    return ctx->opt.dispatch == 2 ? 2 : 3;
}

// Micro-op form the pre-pass writes for the chosen interpreter.
UopFormat uop_format(const galop_ctx* ctx) {
    UopFormat f{};
    f.wide = pick_dispatch(ctx) == 3 ? 1 : 0;
    f.stride = 128u * (uint32_t)pick_k(ctx);
    f.consts = ctx->pool;
    return f;
}

// Dynamic shared memory of one interpreter block.
size_t interp_smem_bytes(const galop_ctx* ctx, int k, int wpb) {
    const int d = pick_dispatch(ctx);
    if (d == 3) return wide_smem_bytes(ctx->isa.num_registers, k, wpb);
    // Register file of every lane plus one block-shared copy of the constant
    // pool laid out the same way.
    return (size_t)(32 * wpb + 32) * ctx->isa.num_registers * k * sizeof(float);
}

// The wide interpreter with an NSLOT-slot register file (8 or 16): the
// same kernels serve both ISAs, since renamed micro-ops address slots.
const void* kernel_for_slots(const galop_ctx* ctx, int k, int mode, int nslot) {
    if (nslot == 8) return interp_kernel_nr8(k, 3, ctx->isa.profile, ctx->opt.reduce, mode);
    return interp_kernel_nr16(k, 3, ctx->isa.profile, ctx->opt.reduce, mode);
}

const void* kernel_for(const galop_ctx* ctx, int k, int mode) {
    const int reduce = ctx->opt.reduce;
    const int dispatch = pick_dispatch(ctx);
    if (ctx->isa.num_registers == 8) return interp_kernel_nr8(k, dispatch, ctx->isa.profile, reduce, mode);
    if (ctx->isa.num_registers == 16) return interp_kernel_nr16(k, dispatch, ctx->isa.profile, reduce, mode);
    return nullptr;
}

}  // namespace galop

namespace {

float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return 0.0f;
    return ms;
}

// Pre-pass over `src` into ctx->uops / eff_off (and order when sched).
//
// `bad` (device, may be null): the flag check_offsets_kernel sets for
// caller-stated device offsets that are inconsistent; when it is set the
// count and compact kernels treat every program as empty.  With `bad`, the
// micro-op buffer is sized for raw_words_total instructions (the effective
// total is not known on the host without waiting for the device).
template <class Src>
int run_prepass(galop_ctx* ctx, const Src& src, int64_t n, int64_t raw_words_total,
                bool strip, bool sched, uint32_t* raw_out, bool reset_totals = true, bool fitness_mode = false,
                const unsigned long long* bad = nullptr) {
    cudaStream_t s = ctx->stream;
    GALOP_CK(ctx->eff_len.ensure((size_t)std::max<int64_t>(n, 1)), "alloc eff_len");
    GALOP_CK(ctx->livein.ensure((size_t)std::max<int64_t>(n, 1)), "alloc livein");
    GALOP_CK(ctx->eff_off.ensure((size_t)n + 1), "alloc eff_off");
    const int64_t n_tiles = (n + kScanTile - 1) / kScanTile;
    GALOP_CK(ctx->tiles.ensure((size_t)n_tiles + 1), "alloc scan tiles");
    // counters: [0] work queue, [1] raw, [2] effective, [3] interpreted
    // instructions, [4] copies left out by dedup (this pre-pass), [5] their
    // interpreted instructions, [6] bad device offsets (check_offsets_kernel),
    // [7] register-file class split (order_scan_kernel)
    GALOP_CK(ctx->counters.ensure(kCounters), "alloc counters");
    if (reset_totals)
        GALOP_CK(cudaMemsetAsync(ctx->counters.p, 0, kCounters * sizeof(unsigned long long), s), "memset");
    else
        GALOP_CK(cudaMemsetAsync(ctx->counters.p + 4, 0, sizeof(unsigned long long), s), "memset");

    const int tpb = 256;
    const unsigned blocks = (unsigned)((n + tpb - 1) / tpb);
    if (n > 0) {
        prepass_count_kernel<Src><<<blocks, tpb, 0, s>>>(src, n, ctx->isa, strip ? 1 : 0,
                                                         ctx->eff_len.p, ctx->counters.p + 1, bad);
        scan_tile_sums_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(ctx->eff_len.p, n, ctx->tiles.p);
        scan_tile_offsets_kernel<<<1, kScanThreads, 0, s>>>(ctx->tiles.p, n_tiles);
        scan_apply_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(ctx->eff_len.p, n, ctx->tiles.p,
                                                                     n_tiles, ctx->eff_off.p);
        ctx->launches += 4;
    } else {
        GALOP_CK(cudaMemsetAsync(ctx->eff_off.p, 0, sizeof(int64_t), s), "memset eff_off");
    }
    GALOP_CK(cudaGetLastError(), "pre-pass count/scan launch");
    // Device buffer for the micro-ops.  The raw total bounds the effective
    // total; when the buffer is smaller than that bound, read the effective
    // total (the scan's last offset) and size the buffer for exactly that, so
    // the footprint follows the interpreted instructions, not the raw ones.
    const UopFormat fmt = uop_format(ctx);
    const size_t per = fmt.wide ? 4 : 1;
    if (ctx->uops.cap < (size_t)std::max<int64_t>(raw_words_total, 1) * per) {
        bool exact = strip && n > 0 && bad == nullptr;
        if (!exact && strip && n > 0) {
            // A buffer for the raw total that would take more than half the
            // free device memory is sized exactly instead (one wait), so
            // that very large populations still fit.
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
                (size_t)raw_words_total * per * sizeof(uint32_t) > free_b / 2)
                exact = true;
            cudaGetLastError();
        }
        if (!exact) {
            // Sized for the raw total without waiting; only when that does
            // not fit is the effective total read back after all.
            const cudaError_t e = ctx->uops.ensure((size_t)std::max<int64_t>(raw_words_total, 1) * per);
            if (e == cudaErrorMemoryAllocation && strip && n > 0) {
                cudaGetLastError();
                exact = true;
            } else {
                GALOP_CK(e, "alloc uops");
            }
        }
        if (exact) {
            int64_t eff_total = raw_words_total;
            GALOP_CK(cudaMemcpyAsync(&eff_total, ctx->eff_off.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s),
                     "D2H effective total");
            GALOP_CK(cudaStreamSynchronize(s), "effective total");
            GALOP_CK(ctx->uops.ensure((size_t)std::max<int64_t>(eff_total, 1) * per), "alloc uops");
        }
    }
    if (n > 0) {
        prepass_compact_kernel<Src><<<blocks, tpb, 0, s>>>(src, n, ctx->isa, strip ? 1 : 0,
                                                           ctx->eff_off.p, ctx->uops.p, raw_out, fmt, bad);
        ctx->launches += 1;
    }
    // Constant folding (wide micro-ops of effective code only; the raw-word
    // output of galop_effective_csr keeps the intron pass's result as is),
    // and the forwarding flags every wide stream carries (fold.cuh).
    ctx->folded = fmt.wide && strip && raw_out == nullptr && n > 0;
    ctx->flagged = fmt.wide && raw_out == nullptr && n > 0;
    if (ctx->flagged) {
        FoldParams fp{ctx->isa.profile, ctx->isa.num_registers, ctx->isa.output_reg,
                      7u + (uint32_t)__builtin_ctz((unsigned)pick_k(ctx)), ctx->num_inputs, nullptr, nullptr,
                      ctx->folded ? 1 : 0, sched ? 1 : 0};
        fold_kernel<<<blocks, tpb, 0, s>>>(reinterpret_cast<uint4*>(ctx->uops.p), ctx->eff_off.p, n, fp,
                                           ctx->eff_len.p, ctx->livein.p, ctx->counters.p + 3);
        ctx->launches += 1;
    }
    // Identical interpreted programs: one representative each (dedup.cuh).
    ctx->deduped = fitness_mode && ctx->folded && ctx->opt.dedup && sched && n > 1;
    if (ctx->deduped) {
        const size_t N1 = (size_t)n;
        GALOP_CK(ctx->dkeys.ensure(N1), "alloc dedup keys");
        GALOP_CK(ctx->dkeys_sorted.ensure(N1), "alloc dedup keys");
        GALOP_CK(ctx->dvals.ensure(N1), "alloc dedup values");
        GALOP_CK(ctx->dvals_sorted.ensure(N1), "alloc dedup values");
        GALOP_CK(ctx->rep.ensure(N1), "alloc representatives");
        GALOP_CK(ctx->dhead.ensure(N1), "alloc dedup runs");
        size_t tsort = 0, tscan = 0;
        GALOP_CK(cub::DeviceRadixSort::SortPairs(nullptr, tsort, ctx->dkeys.p, ctx->dkeys_sorted.p, ctx->dvals.p,
                                                 ctx->dvals_sorted.p, (int)n, 0, 64, s), "dedup sort size");
        GALOP_CK(cub::DeviceScan::InclusiveScan(nullptr, tscan, ctx->dhead.p, ctx->dvals.p, cub::Max(), (int)n, s),
                 "dedup scan size");
        GALOP_CK(ctx->dsort_tmp.ensure(std::max<size_t>(std::max(tsort, tscan), 1)), "alloc dedup sort");
        size_t tmp = ctx->dsort_tmp.cap;
        const uint4* u4 = reinterpret_cast<const uint4*>(ctx->uops.p);
        dedup_hash_kernel<<<blocks, tpb, 0, s>>>(u4, ctx->eff_off.p, ctx->eff_len.p, n, ctx->dkeys.p, ctx->dvals.p,
                                                 ctx->rep.p, nullptr, ctx->livein.p);
        GALOP_CK(cub::DeviceRadixSort::SortPairs(ctx->dsort_tmp.p, tmp, ctx->dkeys.p, ctx->dkeys_sorted.p,
                                                 ctx->dvals.p, ctx->dvals_sorted.p, (int)n, 0, 64, s), "dedup sort");
        dedup_run_start_kernel<<<blocks, tpb, 0, s>>>(ctx->dkeys_sorted.p, n, ctx->dhead.p);
        tmp = ctx->dsort_tmp.cap;
        GALOP_CK(cub::DeviceScan::InclusiveScan(ctx->dsort_tmp.p, tmp, ctx->dhead.p, ctx->dvals.p, cub::Max(), (int)n,
                                                s), "dedup scan");
        dedup_rep_kernel<<<blocks, tpb, 0, s>>>(ctx->dvals.p, ctx->dvals_sorted.p, n, u4, ctx->eff_off.p,
                                                ctx->eff_len.p, ctx->rep.p, ctx->counters.p + 4, nullptr,
                                                ctx->livein.p);
        ctx->launches += 5;
        GALOP_CK(cudaGetLastError(), "dedup launch");
    }
    GALOP_CK(cudaGetLastError(), "pre-pass compact launch");
    // Register-file classes: with a 16-register ISA, programs whose values
    // fit in 8 slots lead the order and run on the 8-slot interpreter (half
    // the shared memory per warp), the rest after them on the 16-slot one.
    ctx->class_split = sched && n > 1 && ctx->flagged && ctx->isa.num_registers > kSplitSlots &&
                       ctx->opt.schedule == GALOP_SCHEDULE_PERSISTENT;
    if (sched && n > 1) {
        const uint32_t* lv = ctx->class_split ? ctx->livein.p : nullptr;
        GALOP_CK(ctx->order.ensure((size_t)n), "alloc order");
        GALOP_CK(ctx->hist.ensure(kOrderBins), "alloc hist");
        GALOP_CK(cudaMemsetAsync(ctx->hist.p, 0, kOrderBins * sizeof(unsigned int), s), "memset hist");
        order_hist_kernel<<<blocks, tpb, 0, s>>>(ctx->eff_len.p, n, ctx->hist.p, lv, kSplitSlots);
        order_scan_kernel<<<1, 1024, 0, s>>>(ctx->hist.p, ctx->class_split ? ctx->counters.p + kCounterClassSplit
                                                                           : nullptr);
        order_scatter_kernel<<<blocks, tpb, 0, s>>>(ctx->eff_len.p, n, ctx->hist.p, ctx->order.p, lv, kSplitSlots);
        ctx->launches += 3;
        GALOP_CK(cudaGetLastError(), "order launch");
    }
    return GALOP_OK;
}

// Interpreter launch over the pre-passed population.
int run_interp(galop_ctx* ctx, int64_t n, int mode, bool sched, float* d_fitness, double* d_sse,
               float* d_outputs, float* d_trace, int32_t* chunks_out, int64_t policy_n = -1) {
    cudaStream_t s = ctx->stream;
    const int k = pick_k(ctx);
    const int wpb = pick_wpb(ctx);
    const int threads = 32 * wpb;
    const void* fn = kernel_for(ctx, k, mode);
    if (!fn) return ctx->fail(GALOP_E_INVALID, "no interpreter kernel for NR=%d K=%d",
                              ctx->isa.num_registers, k);
    const size_t smem = interp_smem_bytes(ctx, k, wpb);
    if (smem) {
        GALOP_CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
        GALOP_CK(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared), "smem carveout");
    }
    int per_sm = 0;
    GALOP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem), "occupancy");
    if (per_sm < 1) per_sm = 1;
    const int64_t resident_warps = (int64_t)ctx->sm_count * per_sm * wpb;

    // Case chunking: enough work items to keep every resident warp busy, and
    // no item longer than kMaxItemCases cases, so that the longest programs
    // of a population with uneven lengths do not leave a tail of one warp.
    const int64_t pass = 32LL * k;
    const int64_t passes = std::max<int64_t>(1, (ctx->N + pass - 1) / pass);
    int64_t n_chunks = 1;
    // policy_n: the population size the chunking is decided for (a segment
    // of a larger call is chunked as the whole call would be)
    const int64_t pn = policy_n >= 0 ? policy_n : n;
    if (mode == kModeFitness && ctx->opt.reduce != GALOP_REDUCE_ORDERED && n > 0) {
        if (pn < 4 * resident_warps) n_chunks = std::min<int64_t>(passes, (4 * resident_warps + pn - 1) / pn);
        n_chunks = std::max<int64_t>(n_chunks, std::min<int64_t>(passes, (ctx->N + kMaxItemCases - 1) / kMaxItemCases));
    }
    const bool plain = ctx->opt.schedule == GALOP_SCHEDULE_PLAIN && mode != kModeTrace;
    if (mode != kModeFitness || plain) n_chunks = 1;
    const int64_t chunk_passes = (passes + n_chunks - 1) / n_chunks;
    const int64_t chunk_cases = chunk_passes * pass;
    n_chunks = std::max<int64_t>(1, (std::max<int64_t>(ctx->N, 1) + chunk_cases - 1) / chunk_cases);

    InterpArgs a{};
    a.uops = ctx->uops.p;
    a.eff_off = ctx->eff_off.p;
    a.interp_len = ctx->folded ? ctx->eff_len.p : nullptr;
    a.livein = ctx->flagged ? ctx->livein.p : nullptr;
    a.n_skipped = ctx->deduped ? ctx->counters.p + 4 : nullptr;
    a.order = (sched && n > 1 && !plain) ? ctx->order.p : nullptr;
    a.plain = plain ? 1 : 0;
    a.n_programs = n;
    a.n_chunks = (int32_t)n_chunks;
    a.chunk_cases = chunk_cases;
    a.X = ctx->X.p;
    a.y = ctx->y.p;
    a.N = ctx->N;
    a.Np = ctx->Np;
    a.num_inputs = ctx->num_inputs;
    a.output_reg = ctx->isa.output_reg;
    a.consts = ctx->pool;
    a.obj = objective_for(ctx, ctx->ss_tot);
    a.counter = ctx->counters.p;
    a.fitness = d_fitness;
    a.sse = d_sse;
    a.outputs = d_outputs;
    a.trace = d_trace;
    if (n_chunks > 1) {
        GALOP_CK(ctx->partial.ensure((size_t)(n * n_chunks)), "alloc partial");
        a.partial = ctx->partial.p;
    }
    const int64_t items = n * n_chunks;
    const int64_t need = (items + wpb - 1) / wpb;
    // One launch per register-file class (the 8-slot programs first, then
    // the rest), or one launch over the whole order.
    const bool split = ctx->class_split && sched && n > 1 && mode != kModeTrace && pick_dispatch(ctx) == 3;
    const int parts = split ? 2 : 1;
    int64_t blocks = 0;
    for (int part = 0; part < parts && n > 0; ++part) {
        const void* f = fn;
        size_t sm = smem;
        int psm = per_sm;
        if (split && part == 0) {
            f = kernel_for_slots(ctx, k, mode, kSplitSlots);
            sm = wide_smem_bytes(kSplitSlots, k, wpb);
            GALOP_CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), "smem attribute");
            GALOP_CK(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared), "smem carveout");
            GALOP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&psm, f, threads, sm), "occupancy");
            if (psm < 1) psm = 1;
        }
        a.class_split = split ? ctx->counters.p + kCounterClassSplit : nullptr;
        a.class_part = part;
        int64_t b = (int64_t)ctx->sm_count * psm;
        if (b > need || plain) b = std::max<int64_t>(need, 1);   // plain: one warp per program
        GALOP_CK(cudaMemsetAsync(ctx->counters.p, 0, sizeof(unsigned long long), s), "memset queue");
        void* params[] = {&a};
        GALOP_CK(cudaLaunchKernel(f, dim3((unsigned)b), dim3(threads), params, sm, s), "interpreter launch");
        ctx->launches += 1;
        blocks = std::max(blocks, b);
    }
    ctx->stats.cases_per_lane = k;
    ctx->stats.warps_per_block = wpb;
    ctx->stats.blocks = (int32_t)blocks;
    ctx->stats.case_chunks = (int32_t)n_chunks;
    if (chunks_out) *chunks_out = (int32_t)n_chunks;
    return GALOP_OK;
}

int finalize(galop_ctx* ctx, int64_t n, int32_t n_chunks, float* d_fitness, double* d_sse) {
    if (ctx->deduped && n > 0) {
        // chunk sums first (copies get garbage there), then the copies' results
        if (n_chunks > 1)
            finalize_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
                ctx->partial.p, n, n_chunks, ctx->N, objective_for(ctx, ctx->ss_tot), d_fitness, d_sse);
        dedup_scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(ctx->rep.p, n, d_fitness, d_sse);
        ctx->launches += n_chunks > 1 ? 2 : 1;
        GALOP_CK(cudaGetLastError(), "finalize launch");
        return GALOP_OK;
    }
    if (n_chunks <= 1 || n == 0) return GALOP_OK;
    finalize_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        ctx->partial.p, n, n_chunks, ctx->N, objective_for(ctx, ctx->ss_tot), d_fitness, d_sse);
    ctx->launches += 1;
    GALOP_CK(cudaGetLastError(), "finalize launch");
    return GALOP_OK;
}

int check_ready(galop_ctx* ctx) {
    if (!ctx) return GALOP_E_INVALID;
    if (ctx->N < 0) return ctx->fail(GALOP_E_NO_DATASET, "no dataset: call galop_set_dataset first");
    return GALOP_OK;
}

void begin_call(galop_ctx* ctx, int64_t n) {
    cudaGetLastError();   // a stale error of an earlier call must not be reported as ours
    ctx->stats_pending = false;
    ctx->stats = galop_stats{};
    ctx->stats.n_programs = n;
    ctx->stats.n_cases = ctx->N;
    ctx->launches = 0;
}

// Timings and instruction counts of the last call, once its work is done.
int finish_stats(galop_ctx* ctx) {
    galop_stats& st = ctx->stats;
    st.h2d_ms = ev_ms(ctx->ev[kEvStart], ctx->ev[kEvH2D]);
    st.prepass_ms = ev_ms(ctx->ev[kEvH2D], ctx->ev[kEvPrepass]);
    st.interp_ms = ev_ms(ctx->ev[kEvPrepass], ctx->ev[kEvInterp]);
    st.finalize_ms = ev_ms(ctx->ev[kEvInterp], ctx->ev[kEvFinalize]);
    st.d2h_ms = ev_ms(ctx->ev[kEvFinalize], ctx->ev[kEvD2H]);
    st.total_ms = ev_ms(ctx->ev[kEvStart], ctx->ev[kEvD2H]);
    unsigned long long tot[kCounters - 1] = {};
    if (ctx->counters.p)
        GALOP_CK(cudaMemcpy(tot, ctx->counters.p + 1, sizeof tot, cudaMemcpyDeviceToHost), "stats D2H");
    st.raw_instructions = (int64_t)tot[0];
    st.eff_instructions = (int64_t)tot[1];
    st.interp_instructions = ctx->folded ? (int64_t)(tot[2] - tot[4]) : (int64_t)tot[1];
    st.kernels_launched = ctx->launches;
    ctx->stats_pending = false;
    if (tot[kCounterBadOffsets - 1])
        return ctx->fail(GALOP_E_INVALID, "device offsets disagree with total_words (offsets[0] != 0, a "
                                          "decreasing offset or a program over 2^30 words, or offsets[n] != "
                                          "total_words): nothing was read, every fitness is NaN");
    return GALOP_OK;
}

int end_call(galop_ctx* ctx) {
    GALOP_CK(cudaStreamSynchronize(ctx->stream), "evaluate (device execution)");
    return finish_stats(ctx);
}

}  // namespace

namespace galop {

// n device-resident programs in the dense layout (program i at
// d_words + i*stride, d_lens[i] instructions) into d_fitness, on the
// context's stream, synchronously; stats as the other evaluate calls.
int evaluate_dense_device(galop_ctx* ctx, const uint32_t* d_words, const uint8_t* d_lens, int64_t stride,
                          int64_t n, float* d_fitness) {
    if (int rc = check_ready(ctx)) return rc;
    begin_call(ctx, n);
    cudaStream_t s = ctx->stream;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], s), "event");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvH2D], s), "event");
    DenseSource src{d_words, d_lens, stride};
    if (int rc = run_prepass(ctx, src, n, n * stride, ctx->opt.intron_prepass != 0, true, nullptr, true, true))
        return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvPrepass], s), "event");
    int32_t chunks = 1;
    if (int rc = run_interp(ctx, n, kModeFitness, true, d_fitness, nullptr, nullptr, nullptr, &chunks)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvInterp], s), "event");
    if (int rc = finalize(ctx, n, chunks, d_fitness, nullptr)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvFinalize], s), "event");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvD2H], s), "event");
    return end_call(ctx);
}

}  // namespace galop

namespace {

int validate_offsets(galop_ctx* ctx, const int64_t* off, int64_t n) {
    if (off[0] != 0) return ctx->fail(GALOP_E_INVALID, "offsets[0] must be 0 (got %lld)", (long long)off[0]);
    for (int64_t i = 0; i < n; ++i) {
        const int64_t l = off[i + 1] - off[i];
        if (l < 0) return ctx->fail(GALOP_E_INVALID, "offsets not non-decreasing at program %lld", (long long)i);
        if (l > (int64_t)1 << 30) return ctx->fail(GALOP_E_CAPACITY, "program %lld longer than 2^30", (long long)i);
    }
    return GALOP_OK;
}

// Upload a host CSR population into raw_words/raw_off.
int upload_csr(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets, int64_t n) {
    if (!offsets || (n > 0 && !words && offsets[n] > 0))
        return ctx->fail(GALOP_E_INVALID, "null words/offsets");
    if (int rc = validate_offsets(ctx, offsets, n)) return rc;
    const int64_t total = offsets[n];
    GALOP_CK(ctx->raw_words.ensure((size_t)std::max<int64_t>(total, 1)), "alloc raw words");
    GALOP_CK(ctx->raw_off.ensure((size_t)n + 1), "alloc raw offsets");
    if (total > 0)
        GALOP_CK(cudaMemcpyAsync(ctx->raw_words.p, words, (size_t)total * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, ctx->stream), "H2D words");
    GALOP_CK(cudaMemcpyAsync(ctx->raw_off.p, offsets, (size_t)(n + 1) * sizeof(int64_t),
                             cudaMemcpyHostToDevice, ctx->stream), "H2D offsets");
    return GALOP_OK;
}

}  // namespace

extern "C" {

int galop_abi_version(void) { return GALOP_ABI_VERSION; }

const char* galop_status_string(int s) {
    switch (s) {
        case GALOP_OK: return "ok";
        case GALOP_E_INVALID: return "invalid argument";
        case GALOP_E_CUDA: return "CUDA error";
        case GALOP_E_NOMEM: return "out of memory";
        case GALOP_E_NO_DATASET: return "no dataset";
        case GALOP_E_TIMEOUT: return "device wait timed out";
        case GALOP_E_CAPACITY: return "capacity exceeded";
        case GALOP_E_NO_DEVICE: return "no suitable device";
        case GALOP_E_STATE: return "invalid state";
        default: return "unknown status";
    }
}

int galop_options_init(galop_options* opt) {
    if (!opt) return GALOP_E_INVALID;
    std::memset(opt, 0, sizeof *opt);
    opt->profile = GALOP_PROFILE_REF;
    opt->num_registers = 8;
    opt->input_protect = 0;
    opt->reduce = GALOP_REDUCE_KAHAN32;
    opt->constants = nullptr;
    opt->device = 0;
    opt->intron_prepass = 1;
    opt->cases_per_lane = 0;
    opt->warps_per_block = 0;
    opt->dispatch = 3;
    opt->dedup = 1;
    return GALOP_OK;
}

int galop_create(const galop_options* opt, galop_ctx** out) {
    if (!opt || !out) return GALOP_E_INVALID;
    *out = nullptr;
    if (opt->num_registers != 8 && opt->num_registers != 16) return GALOP_E_INVALID;
    if (opt->profile != GALOP_PROFILE_REF && opt->profile != GALOP_PROFILE_BJ) return GALOP_E_INVALID;
    if (opt->reduce < GALOP_REDUCE_KAHAN32 || opt->reduce > GALOP_REDUCE_ORDERED) return GALOP_E_INVALID;
    if (opt->objective != GALOP_OBJECTIVE_MSE && opt->objective != GALOP_OBJECTIVE_R2) return GALOP_E_INVALID;
    if (opt->dispatch != 2 && opt->dispatch != 3) return GALOP_E_INVALID;
    if (opt->schedule != GALOP_SCHEDULE_PERSISTENT && opt->schedule != GALOP_SCHEDULE_PLAIN) return GALOP_E_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return GALOP_E_NO_DEVICE;
    }
    if (opt->device < 0 || opt->device >= ndev) return GALOP_E_NO_DEVICE;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, opt->device) != cudaSuccess) return GALOP_E_NO_DEVICE;
    if (prop.major != 10) return GALOP_E_NO_DEVICE;   // built for sm_100a only

    galop_ctx* ctx = new galop_ctx();
    ctx->opt = *opt;
    ctx->opt.constants = nullptr;
    ctx->device = opt->device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->isa.profile = opt->profile;
    ctx->isa.num_registers = opt->num_registers;
    ctx->isa.input_protect = opt->input_protect ? 1 : 0;
    ctx->isa.output_reg = opt->input_protect ? opt->num_registers / 2 : 0;
    const float* pool = opt->constants ? opt->constants
                                       : (opt->num_registers == 16 ? kRefPool16 : kRefPool8);
    for (int i = 0; i < kMaxRegisters; ++i) ctx->pool.c[i] = i < opt->num_registers ? pool[i] : 0.0f;

    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    for (int i = 0; e == cudaSuccess && i < kEvCount; ++i) e = cudaEventCreate(&ctx->ev[i]);
    for (int i = 0; e == cudaSuccess && i < 8; ++i) e = cudaEventCreate(&ctx->timers[i]);
    if (e == cudaSuccess) e = ctx->counters.ensure(kCounters);
    if (e != cudaSuccess) {
        galop_destroy(ctx);
        return e == cudaErrorMemoryAllocation ? GALOP_E_NOMEM : GALOP_E_CUDA;
    }
    *out = ctx;
    return GALOP_OK;
}

void galop_destroy(galop_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->X.release(); ctx->y.release(); ctx->stage_aos.release(); ctx->stage_y.release();
    ctx->raw_words.release(); ctx->uops.release(); ctx->eff_raw.release(); ctx->raw_lens8.release();
    ctx->raw_off.release(); ctx->eff_off.release(); ctx->tiles.release();
    ctx->eff_len.release(); ctx->order.release(); ctx->livein.release();
    ctx->fitness.release(); ctx->outputs.release(); ctx->trace.release();
    ctx->sse.release(); ctx->partial.release(); ctx->counters.release(); ctx->hist.release();
    ctx->dkeys.release(); ctx->dkeys_sorted.release(); ctx->dvals.release(); ctx->dvals_sorted.release();
    ctx->rep.release(); ctx->dsort_tmp.release(); ctx->dhead.release();
    for (auto& e : ctx->ev) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->timers) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->seg_ev) if (e) cudaEventDestroy(e);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* galop_last_error(const galop_ctx* ctx) {
    if (!ctx) return "null context";
    return ctx->err.c_str();
}

int galop_last_stats(galop_ctx* ctx, galop_stats* out) {
    if (!ctx || !out) return GALOP_E_INVALID;
    if (ctx->stats_pending) {
        GALOP_CK(cudaSetDevice(ctx->device), "set device");
        GALOP_CK(cudaEventSynchronize(ctx->ev[kEvD2H]), "wait for last call");
        if (int rc = finish_stats(ctx)) return rc;
    }
    *out = ctx->stats;
    return GALOP_OK;
}

int galop_synchronize(galop_ctx* ctx) {
    if (!ctx) return GALOP_E_INVALID;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    GALOP_CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return GALOP_OK;
}

int galop_timer_record(galop_ctx* ctx, int32_t slot) {
    if (!ctx || slot < 0 || slot >= 8) return GALOP_E_INVALID;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    GALOP_CK(cudaEventRecord(ctx->timers[slot], ctx->stream), "timer record");
    return GALOP_OK;
}

int galop_timer_elapsed(galop_ctx* ctx, int32_t a, int32_t b, double* ms) {
    if (!ctx || !ms || a < 0 || a >= 8 || b < 0 || b >= 8) return GALOP_E_INVALID;
    GALOP_CK(cudaEventSynchronize(ctx->timers[b]), "timer sync");
    float f = 0.0f;
    GALOP_CK(cudaEventElapsedTime(&f, ctx->timers[a], ctx->timers[b]), "timer elapsed");
    *ms = f;
    return GALOP_OK;
}

int galop_host_alloc(int64_t bytes, void** out) {
    if (!out || bytes < 0) return GALOP_E_INVALID;
    *out = nullptr;
    cudaError_t e = cudaMallocHost(out, (size_t)std::max<int64_t>(bytes, 1));
    if (e != cudaSuccess) { cudaGetLastError(); *out = nullptr; return GALOP_E_NOMEM; }
    return GALOP_OK;
}

int galop_host_free(void* p) {
    if (p && cudaFreeHost(p) != cudaSuccess) return GALOP_E_CUDA;
    return GALOP_OK;
}

int galop_device_alloc(galop_ctx* ctx, int64_t bytes, void** out) {
    if (!ctx || !out || bytes < 0) return GALOP_E_INVALID;
    *out = nullptr;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    GALOP_CK(cudaMalloc(out, (size_t)std::max<int64_t>(bytes, 1)), "device alloc");
    return GALOP_OK;
}

int galop_device_free(galop_ctx* ctx, void* p) {
    if (!ctx) return GALOP_E_INVALID;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    if (p) GALOP_CK(cudaFree(p), "device free");
    return GALOP_OK;
}

int galop_memcpy_h2d(galop_ctx* ctx, void* dst, const void* src, int64_t bytes) {
    if (!ctx || bytes < 0) return GALOP_E_INVALID;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    if (bytes) GALOP_CK(cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    GALOP_CK(cudaStreamSynchronize(ctx->stream), "H2D sync");
    return GALOP_OK;
}

int galop_memcpy_d2h(galop_ctx* ctx, void* dst, const void* src, int64_t bytes) {
    if (!ctx || bytes < 0) return GALOP_E_INVALID;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    if (bytes) GALOP_CK(cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    GALOP_CK(cudaStreamSynchronize(ctx->stream), "D2H sync");
    return GALOP_OK;
}

static int set_dataset_common(galop_ctx* ctx, const float* src_aos, const float* src_y,
                              int64_t n_cases, int32_t num_inputs) {
    cudaGetLastError();   // a stale error of an earlier call must not be reported as ours
    const int64_t np = std::max<int64_t>(1024, (n_cases + 1023) / 1024 * 1024);
    GALOP_CK(ctx->X.ensure((size_t)(np * std::max(num_inputs, 1))), "alloc dataset X");
    GALOP_CK(ctx->y.ensure((size_t)np), "alloc dataset y");
    const unsigned blocks = (unsigned)((np + 255) / 256);
    dataset_transpose_kernel<<<blocks, 256, 0, ctx->stream>>>(src_aos, src_y, n_cases, num_inputs, np,
                                                              ctx->X.p, ctx->y.p);
    GALOP_CK(cudaGetLastError(), "dataset transpose launch");
    GALOP_CK(cudaStreamSynchronize(ctx->stream), "dataset upload");
    ctx->N = n_cases;
    ctx->Np = np;
    ctx->num_inputs = num_inputs;
    return GALOP_OK;
}

// ss_tot of targets already on the device (one copy to the host).
static int device_ss_tot(galop_ctx* ctx, const float* d_targets, int64_t n_cases, double* out) {
    *out = 0.0;
    if (n_cases <= 0) return GALOP_OK;
    std::vector<float> y((size_t)n_cases);
    GALOP_CK(cudaMemcpyAsync(y.data(), d_targets, (size_t)n_cases * sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->stream), "D2H targets");
    GALOP_CK(cudaStreamSynchronize(ctx->stream), "D2H targets");
    *out = targets_ss_tot(y.data(), n_cases);
    return GALOP_OK;
}

int galop_set_dataset(galop_ctx* ctx, const float* inputs, const float* targets, int64_t n_cases,
                      int32_t num_inputs) {
    if (!ctx) return GALOP_E_INVALID;
    if (n_cases < 0 || num_inputs < 0 || num_inputs > ctx->isa.num_registers)
        return ctx->fail(GALOP_E_INVALID, "bad dataset shape: n_cases=%lld num_inputs=%d (NR=%d)",
                         (long long)n_cases, num_inputs, ctx->isa.num_registers);
    if (n_cases > 0 && (!targets || (num_inputs > 0 && !inputs)))
        return ctx->fail(GALOP_E_INVALID, "null dataset pointer");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    const size_t nx = (size_t)n_cases * (size_t)num_inputs;
    GALOP_CK(ctx->stage_aos.ensure(std::max<size_t>(nx, 1)), "alloc dataset staging");
    GALOP_CK(ctx->stage_y.ensure(std::max<size_t>((size_t)n_cases, 1)), "alloc dataset staging");
    if (nx) GALOP_CK(cudaMemcpyAsync(ctx->stage_aos.p, inputs, nx * sizeof(float), cudaMemcpyHostToDevice,
                                     ctx->stream), "H2D dataset inputs");
    if (n_cases) GALOP_CK(cudaMemcpyAsync(ctx->stage_y.p, targets, (size_t)n_cases * sizeof(float),
                                          cudaMemcpyHostToDevice, ctx->stream), "H2D dataset targets");
    int rc = set_dataset_common(ctx, ctx->stage_aos.p, ctx->stage_y.p, n_cases, num_inputs);
    ctx->stage_aos.release();
    ctx->stage_y.release();
    if (rc == GALOP_OK) ctx->ss_tot = targets_ss_tot(targets, n_cases);
    return rc;
}

int galop_set_dataset_device(galop_ctx* ctx, const float* d_inputs, const float* d_targets,
                             int64_t n_cases, int32_t num_inputs) {
    if (!ctx) return GALOP_E_INVALID;
    if (n_cases < 0 || num_inputs < 0 || num_inputs > ctx->isa.num_registers)
        return ctx->fail(GALOP_E_INVALID, "bad dataset shape");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    double ss = 0.0;
    if (ctx->opt.objective == GALOP_OBJECTIVE_R2)
        if (int rc = device_ss_tot(ctx, d_targets, n_cases, &ss)) return rc;
    if (int rc = set_dataset_common(ctx, d_inputs, d_targets, n_cases, num_inputs)) return rc;
    ctx->ss_tot = ss;
    return GALOP_OK;
}

}  // extern "C"

// Shared body of the host-pointer evaluate calls, after the raw population
// is on the device (in raw_words/raw_off or raw_words/raw_lens8).
template <class Src>
static int evaluate_uploaded(galop_ctx* ctx, const Src& src, int64_t n, int64_t raw_total,
                             float* fitness_out, double* sse_out) {
    cudaStream_t s = ctx->stream;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvH2D], s), "event");
    if (int rc = run_prepass(ctx, src, n, raw_total, ctx->opt.intron_prepass != 0, true, nullptr, true, true))
        return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvPrepass], s), "event");
    GALOP_CK(ctx->fitness.ensure((size_t)std::max<int64_t>(n, 1)), "alloc fitness");
    GALOP_CK(ctx->sse.ensure((size_t)std::max<int64_t>(n, 1)), "alloc sse");
    int32_t chunks = 1;
    if (int rc = run_interp(ctx, n, kModeFitness, true, ctx->fitness.p, ctx->sse.p, nullptr, nullptr, &chunks))
        return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvInterp], s), "event");
    if (int rc = finalize(ctx, n, chunks, ctx->fitness.p, ctx->sse.p)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvFinalize], s), "event");
    if (n > 0) {
        GALOP_CK(cudaMemcpyAsync(fitness_out, ctx->fitness.p, (size_t)n * sizeof(float),
                                 cudaMemcpyDeviceToHost, s), "D2H fitness");
        if (sse_out)
            GALOP_CK(cudaMemcpyAsync(sse_out, ctx->sse.p, (size_t)n * sizeof(double),
                                     cudaMemcpyDeviceToHost, s), "D2H sse");
    }
    GALOP_CK(cudaEventRecord(ctx->ev[kEvD2H], s), "event");
    return end_call(ctx);
}

// Host-pointer CSR evaluation in segments of programs: the words of segment
// k+1 are copied on a second stream while segment k is pre-passed and
// interpreted, so most of the host-to-device copy hides behind compute.
// Segment k ends at program n * kSegEnd[k] / 32: the first segment is
// small, so only its short copy is exposed, and each later one is copied
// while the previous (at least as large) computes.  The offsets are
// checked while the copies run (only the segment boundaries, which size
// the copies, before).  Every segment is chunked as the whole call would
// be, so the fitness is the unsegmented call's bit for bit.
constexpr int kSegs = 5;
constexpr int64_t kSegEnd[kSegs] = {1, 4, 8, 16, 32};

static int evaluate_csr_segmented(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets, int64_t n,
                                  float* fitness_out, double* sse_out) {
    const int segs = kSegs;
    std::vector<int64_t> b(segs + 1);
    b[0] = 0;
    for (int k = 0; k < segs; ++k) b[k + 1] = n * kSegEnd[k] / 32;
    bool bounds_ok = offsets[0] == 0;
    for (int k = 0; k < segs; ++k) bounds_ok = bounds_ok && offsets[b[k + 1]] >= offsets[b[k]];
    if (!bounds_ok) return validate_offsets(ctx, offsets, n);
    cudaStream_t s = ctx->stream;
    if (!ctx->copy_stream) {
        GALOP_CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream");
        for (auto& e : ctx->seg_ev) GALOP_CK(cudaEventCreate(&e), "segment events");
    }
    cudaStream_t cs = ctx->copy_stream;
    const int64_t total = offsets[n];
    GALOP_CK(ctx->raw_words.ensure((size_t)std::max<int64_t>(total, 1)), "alloc raw words");
    GALOP_CK(ctx->raw_off.ensure((size_t)n + 1), "alloc raw offsets");
    GALOP_CK(ctx->fitness.ensure((size_t)std::max<int64_t>(n, 1)), "alloc fitness");
    GALOP_CK(ctx->sse.ensure((size_t)std::max<int64_t>(n, 1)), "alloc sse");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], s), "event");
    GALOP_CK(cudaStreamWaitEvent(cs, ctx->ev[kEvStart], 0), "stream wait");
    GALOP_CK(cudaMemcpyAsync(ctx->raw_off.p, offsets, (size_t)(n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, cs),
             "H2D offsets");
    for (int k = 0; k < segs; ++k) {
        const int64_t w0 = offsets[b[k]], w1 = offsets[b[k + 1]];
        if (w1 > w0)
            GALOP_CK(cudaMemcpyAsync(ctx->raw_words.p + w0, words + w0, (size_t)(w1 - w0) * sizeof(uint32_t),
                                     cudaMemcpyHostToDevice, cs), "H2D words");
        GALOP_CK(cudaEventRecord(ctx->seg_ev[5 * k], cs), "event");
    }
    if (int rc = validate_offsets(ctx, offsets, n)) {
        cudaStreamSynchronize(cs);   // the copies read the caller's buffers
        return rc;
    }
    GALOP_CK(ctx->counters.ensure(kCounters), "alloc counters");
    GALOP_CK(cudaMemsetAsync(ctx->counters.p, 0, kCounters * sizeof(unsigned long long), s), "memset");
    for (int k = 0; k < segs; ++k) {
        const int64_t nk = b[k + 1] - b[k];
        GALOP_CK(cudaStreamWaitEvent(s, ctx->seg_ev[5 * k], 0), "stream wait");
        GALOP_CK(cudaEventRecord(ctx->seg_ev[5 * k + 1], s), "event");
        CsrSource src{ctx->raw_words.p, ctx->raw_off.p + b[k]};
        if (int rc = run_prepass(ctx, src, nk, offsets[b[k + 1]] - offsets[b[k]], ctx->opt.intron_prepass != 0,
                                 true, nullptr, false, true))
            return rc;
        GALOP_CK(cudaEventRecord(ctx->seg_ev[5 * k + 2], s), "event");
        int32_t chunks = 1;
        if (int rc = run_interp(ctx, nk, kModeFitness, true, ctx->fitness.p + b[k], ctx->sse.p + b[k], nullptr,
                                nullptr, &chunks, n))
            return rc;
        GALOP_CK(cudaEventRecord(ctx->seg_ev[5 * k + 3], s), "event");
        if (int rc = finalize(ctx, nk, chunks, ctx->fitness.p + b[k], ctx->sse.p + b[k])) return rc;
        GALOP_CK(cudaEventRecord(ctx->seg_ev[5 * k + 4], s), "event");
    }
    if (n > 0) {
        GALOP_CK(cudaMemcpyAsync(fitness_out, ctx->fitness.p, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, s),
                 "D2H fitness");
        if (sse_out)
            GALOP_CK(cudaMemcpyAsync(sse_out, ctx->sse.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s),
                     "D2H sse");
    }
    GALOP_CK(cudaEventRecord(ctx->ev[kEvD2H], s), "event");
    GALOP_CK(cudaStreamSynchronize(s), "evaluate (device execution)");
    if (int rc = finish_stats(ctx)) return rc;
    galop_stats& st = ctx->stats;
    st.h2d_ms = ev_ms(ctx->ev[kEvStart], ctx->seg_ev[5 * (segs - 1)]);
    st.prepass_ms = st.interp_ms = st.finalize_ms = 0.0;
    for (int k = 0; k < segs; ++k) {
        st.prepass_ms += ev_ms(ctx->seg_ev[5 * k + 1], ctx->seg_ev[5 * k + 2]);
        st.interp_ms += ev_ms(ctx->seg_ev[5 * k + 2], ctx->seg_ev[5 * k + 3]);
        st.finalize_ms += ev_ms(ctx->seg_ev[5 * k + 3], ctx->seg_ev[5 * k + 4]);
    }
    st.d2h_ms = ev_ms(ctx->seg_ev[5 * (segs - 1) + 4], ctx->ev[kEvD2H]);
    st.total_ms = ev_ms(ctx->ev[kEvStart], ctx->ev[kEvD2H]);
    st.n_programs = n;
    return GALOP_OK;
}

extern "C" {

int galop_evaluate_csr(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets, int64_t n_programs,
                       float* fitness_out, double* sse_out) {
    if (int rc = check_ready(ctx)) return rc;
    if (n_programs < 0) return ctx->fail(GALOP_E_INVALID, "n_programs < 0");
    if (n_programs > INT32_MAX) return ctx->fail(GALOP_E_CAPACITY, "n_programs > 2^31-1");
    if (n_programs > 0 && !fitness_out) return ctx->fail(GALOP_E_INVALID, "null fitness_out");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    begin_call(ctx, n_programs);
    // Large populations: copy and compute overlapped in segments.
    if (n_programs >= 65536 && offsets && offsets[n_programs] >= (int64_t)(32ll << 20)) {
        if (!words) return ctx->fail(GALOP_E_INVALID, "null words/offsets");
        return evaluate_csr_segmented(ctx, words, offsets, n_programs, fitness_out, sse_out);
    }
    GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], ctx->stream), "event");
    if (int rc = upload_csr(ctx, words, offsets, n_programs)) return rc;
    CsrSource src{ctx->raw_words.p, ctx->raw_off.p};
    return evaluate_uploaded(ctx, src, n_programs, offsets[n_programs], fitness_out, sse_out);
}

int galop_evaluate_population(galop_ctx* ctx, const uint32_t* instructions, const uint8_t* lengths,
                              int64_t stride, int64_t n_programs, float* fitness_out) {
    if (int rc = check_ready(ctx)) return rc;
    if (n_programs < 0 || stride < 0) return ctx->fail(GALOP_E_INVALID, "negative size");
    if (n_programs > INT32_MAX) return ctx->fail(GALOP_E_CAPACITY, "n_programs > 2^31-1");
    if (n_programs > 0 && (!instructions || !lengths || !fitness_out))
        return ctx->fail(GALOP_E_INVALID, "null pointer");
    for (int64_t i = 0; i < n_programs; ++i)
        if ((int64_t)lengths[i] > stride)
            return ctx->fail(GALOP_E_INVALID, "lengths[%lld]=%d exceeds stride %lld", (long long)i,
                             (int)lengths[i], (long long)stride);
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    begin_call(ctx, n_programs);
    cudaStream_t s = ctx->stream;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], s), "event");
    const int64_t total = n_programs * stride;
    GALOP_CK(ctx->raw_words.ensure((size_t)std::max<int64_t>(total, 1)), "alloc raw words");
    GALOP_CK(ctx->raw_lens8.ensure((size_t)std::max<int64_t>(n_programs, 1)), "alloc lengths");
    if (total > 0)
        GALOP_CK(cudaMemcpyAsync(ctx->raw_words.p, instructions, (size_t)total * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, s), "H2D instructions");
    if (n_programs > 0)
        GALOP_CK(cudaMemcpyAsync(ctx->raw_lens8.p, lengths, (size_t)n_programs, cudaMemcpyHostToDevice, s),
                 "H2D lengths");
    DenseSource src{ctx->raw_words.p, ctx->raw_lens8.p, stride};
    return evaluate_uploaded(ctx, src, n_programs, total, fitness_out, nullptr);
}

int galop_evaluate_csr_device(galop_ctx* ctx, const uint32_t* d_words, const int64_t* d_offsets,
                              int64_t n_programs, int64_t total_words, float* d_fitness, double* d_sse,
                              void* stream) {
    if (int rc = check_ready(ctx)) return rc;
    if (n_programs < 0 || total_words < 0 || !d_offsets) return ctx->fail(GALOP_E_INVALID, "bad arguments");
    if (n_programs > INT32_MAX) return ctx->fail(GALOP_E_CAPACITY, "n_programs > 2^31-1");
    if (n_programs > 0 && (!d_fitness || (!d_words && total_words > 0)))
        return ctx->fail(GALOP_E_INVALID, "null pointer");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    begin_call(ctx, n_programs);
    cudaStream_t user = (cudaStream_t)stream;
    cudaStream_t s = ctx->stream;
    if (user && user != s) {
        GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], user), "event");
        GALOP_CK(cudaStreamWaitEvent(s, ctx->ev[kEvStart], 0), "stream wait");
    } else {
        GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], s), "event");
    }
    // The caller's offsets are checked on the device against total_words
    // before any word is read (prepass.cuh); nothing waits for the device.
    GALOP_CK(ctx->counters.ensure(kCounters), "alloc counters");
    GALOP_CK(cudaMemsetAsync(ctx->counters.p, 0, kCounters * sizeof(unsigned long long), s), "memset");
    unsigned long long* bad = ctx->counters.p + kCounterBadOffsets;
    check_offsets_kernel<<<(unsigned)((n_programs + 256) / 256), 256, 0, s>>>(d_offsets, n_programs, total_words,
                                                                            bad);
    ctx->launches += 1;
    GALOP_CK(cudaGetLastError(), "offset check launch");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvH2D], s), "event");
    CsrSource src{d_words, d_offsets};
    if (int rc = run_prepass(ctx, src, n_programs, total_words, ctx->opt.intron_prepass != 0, true, nullptr, false,
                             true, bad))
        return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvPrepass], s), "event");
    int32_t chunks = 1;
    if (int rc = run_interp(ctx, n_programs, kModeFitness, true, d_fitness, d_sse, nullptr, nullptr, &chunks))
        return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvInterp], s), "event");
    if (int rc = finalize(ctx, n_programs, chunks, d_fitness, d_sse)) return rc;
    if (n_programs > 0) {
        poison_results_kernel<<<(unsigned)((n_programs + 255) / 256), 256, 0, s>>>(bad, n_programs, d_fitness, d_sse);
        ctx->launches += 1;
        GALOP_CK(cudaGetLastError(), "result check launch");
    }
    GALOP_CK(cudaEventRecord(ctx->ev[kEvFinalize], s), "event");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvD2H], s), "event");
    if (user && user != s) GALOP_CK(cudaStreamWaitEvent(user, ctx->ev[kEvD2H], 0), "stream wait");
    ctx->stats.kernels_launched = ctx->launches;
    ctx->stats_pending = true;
    return GALOP_OK;
}

int galop_case_outputs_csr(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets,
                           int64_t n_programs, float* outputs) {
    if (int rc = check_ready(ctx)) return rc;
    if (n_programs < 0) return ctx->fail(GALOP_E_INVALID, "n_programs < 0");
    if (n_programs > 0 && !outputs) return ctx->fail(GALOP_E_INVALID, "null outputs");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    begin_call(ctx, n_programs);
    cudaStream_t s = ctx->stream;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], s), "event");
    if (int rc = upload_csr(ctx, words, offsets, n_programs)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvH2D], s), "event");
    CsrSource src{ctx->raw_words.p, ctx->raw_off.p};
    if (int rc = run_prepass(ctx, src, n_programs, offsets[n_programs], ctx->opt.intron_prepass != 0, true,
                             nullptr)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvPrepass], s), "event");
    const size_t total = (size_t)n_programs * (size_t)std::max<int64_t>(ctx->N, 0);
    GALOP_CK(ctx->outputs.ensure(std::max<size_t>(total, 1)), "alloc outputs");
    if (int rc = run_interp(ctx, n_programs, kModeOutputs, true, nullptr, nullptr, ctx->outputs.p, nullptr,
                            nullptr)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvInterp], s), "event");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvFinalize], s), "event");
    if (total)
        GALOP_CK(cudaMemcpyAsync(outputs, ctx->outputs.p, total * sizeof(float), cudaMemcpyDeviceToHost, s),
                 "D2H outputs");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvD2H], s), "event");
    return end_call(ctx);
}

int galop_trace_program(galop_ctx* ctx, const uint32_t* words, int64_t len, float* state, int64_t* n_traced) {
    if (int rc = check_ready(ctx)) return rc;
    if (len < 0 || (len > 0 && !words) || !state) return ctx->fail(GALOP_E_INVALID, "bad arguments");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    const int k = pick_k(ctx);
    const int64_t pass = 32LL * k;
    const int64_t nt = std::min<int64_t>(pass, ctx->N);
    if (n_traced) *n_traced = nt;
    if (nt <= 0) return GALOP_OK;
    begin_call(ctx, 1);
    cudaStream_t s = ctx->stream;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], s), "event");
    int64_t off[2] = {0, len};
    if (int rc = upload_csr(ctx, words, off, 1)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvH2D], s), "event");
    CsrSource src{ctx->raw_words.p, ctx->raw_off.p};
    if (int rc = run_prepass(ctx, src, 1, len, false, false, nullptr)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvPrepass], s), "event");
    const int nr = ctx->isa.num_registers;
    const size_t cells = (size_t)(len + 1) * nr * pass;
    GALOP_CK(ctx->trace.ensure(cells), "alloc trace");
    if (int rc = run_interp(ctx, 1, kModeTrace, false, nullptr, nullptr, nullptr, ctx->trace.p, nullptr))
        return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvInterp], s), "event");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvFinalize], s), "event");
    std::vector<float> tmp(cells);
    GALOP_CK(cudaMemcpyAsync(tmp.data(), ctx->trace.p, cells * sizeof(float), cudaMemcpyDeviceToHost, s),
             "D2H trace");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvD2H], s), "event");
    if (int rc = end_call(ctx)) return rc;
    for (int64_t row = 0; row < (len + 1) * nr; ++row)
        std::memcpy(state + row * nt, tmp.data() + row * pass, (size_t)nt * sizeof(float));
    return GALOP_OK;
}

int galop_effective_csr(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets, int64_t n_programs,
                        int64_t* eff_len, uint32_t* eff_words) {
    if (!ctx || !eff_len) return GALOP_E_INVALID;
    if (n_programs < 0) return ctx->fail(GALOP_E_INVALID, "n_programs < 0");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    begin_call(ctx, n_programs);
    cudaStream_t s = ctx->stream;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvStart], s), "event");
    if (int rc = upload_csr(ctx, words, offsets, n_programs)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvH2D], s), "event");
    GALOP_CK(ctx->eff_raw.ensure((size_t)std::max<int64_t>(offsets[n_programs], 1)), "alloc eff words");
    CsrSource src{ctx->raw_words.p, ctx->raw_off.p};
    if (int rc = run_prepass(ctx, src, n_programs, offsets[n_programs], true, false, ctx->eff_raw.p)) return rc;
    GALOP_CK(cudaEventRecord(ctx->ev[kEvPrepass], s), "event");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvInterp], s), "event");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvFinalize], s), "event");
    std::vector<int64_t> off((size_t)n_programs + 1);
    GALOP_CK(cudaMemcpyAsync(off.data(), ctx->eff_off.p, off.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, s),
             "D2H eff offsets");
    GALOP_CK(cudaStreamSynchronize(s), "sync");
    for (int64_t i = 0; i < n_programs; ++i) eff_len[i] = off[i + 1] - off[i];
    if (eff_words && off[n_programs] > 0)
        GALOP_CK(cudaMemcpyAsync(eff_words, ctx->eff_raw.p, (size_t)off[n_programs] * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, s), "D2H eff words");
    GALOP_CK(cudaEventRecord(ctx->ev[kEvD2H], s), "event");
    return end_call(ctx);
}

}  // extern "C"
