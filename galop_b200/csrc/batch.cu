// batch.cu -- resident datasets and batched evaluation of many populations.
//
// Populations of uneven sizes, program lengths and datasets are evaluated
// together: one persistent interpreter launch per register-file class (the
// programs whose renamed values fit 8 slots, then the rest) pulls (program,
// case chunk) items from a device queue, largest work first.  Each
// generation's device work (intron pass, ordering, item list, interpreter,
// chunk reduction) can be captured once as a CUDA graph and replayed.  Each
// batch has its own stream, so several batches overlap on the device (the
// serving loop in serve.cu relies on this).
//
// Case chunking depends only on a population's own case count (at most
// kChunkCases cases per work item), never on what else is in the batch, so a
// population's fitness is bit-identical whichever batch it is evaluated in.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <vector>

#include "batch.cuh"
#include "context.cuh"
#include "prepass.cuh"
#include "interp_wide.cuh"
#include "fold.cuh"
#include "dedup.cuh"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

using namespace galop;

namespace {

constexpr int64_t kChunkCases = kMaxItemCases;

int64_t chunk_cases_for(int64_t n_cases) {
    const int64_t padded = std::max<int64_t>(1024, (n_cases + 1023) / 1024 * 1024);
    return std::min<int64_t>(padded, kChunkCases);
}

int64_t chunks_for(int64_t n_cases) {
    const int64_t c = chunk_cases_for(n_cases);
    return std::max<int64_t>(1, (n_cases + c - 1) / c);
}

}  // namespace

// Dataset buffers come from the stream-ordered allocator (cudaMallocAsync):
// admitting a new dataset while batches run does not synchronise the device.
struct galop_dataset {
    galop_ctx* ctx = nullptr;
    int device = 0;                 // kept so destruction never reads the context
    struct Buf { float* p = nullptr; size_t cap = 0; } X, y;
    int64_t N = 0, Np = 0;
    int32_t k = 0;
    double ss_tot = 0.0;            // of the targets, for the R^2 objective
};

struct BatchPop {
    const galop_dataset* ds = nullptr;
    int64_t max_programs = 0, max_words = 0;
    int64_t n = 0;                  // programs set for this generation
    int64_t word_base = 0, off_base = 0, out_base = 0;
    int64_t n_chunks = 1, chunk_cases = 1024;
};

struct galop_batch {
    galop_ctx* ctx = nullptr;
    int device = 0;                 // kept so destruction never reads the context
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    std::vector<BatchPop> pops;
    int64_t total_max_programs = 0, total_max_words = 0, total_max_items = 0;
    // pooled mode (galop_batch_create_pool): populations are appended per
    // generation into shared capacity; cursors of the current composition
    bool pooled = false;
    int32_t max_pops = 0;
    int64_t cur_words = 0, cur_offs = 0, cur_progs = 0, cur_items = 0;
    // device buffers (fixed capacities: nothing is reallocated after creation)
    DevBuf<uint32_t> arena, uops;
    DevBuf<int64_t> local_off, starts, eff_off, item_off, first_item, tiles;
    DevBuf<int32_t> lens, prog_pop, eff_len, key, order, cnt, chunks_of_pop;
    DevBuf<uint32_t> livein;
    // dedup within each population (dedup.cuh)
    DevBuf<unsigned long long> dkeys, dkeys_sorted;
    DevBuf<int32_t> dvals, dvals_sorted, rep, dhead;
    DevBuf<unsigned char> dtmp;
    bool dedup = false;
    DevBuf<unsigned long long> items, counters;
    DevBuf<unsigned int> hist;
    DevBuf<float> fitness;
    DevBuf<double> sse, partial;
    DevBuf<PopLayout> layout;
    DevBuf<PopDesc> descs;
    // launch plan of the current generation shape
    std::vector<int64_t> planned_n;
    int64_t G = 0, n_items = 0;
    const void* interp_fn = nullptr;
    int threads = 0, grid = 0;
    size_t smem = 0;
    // register-file classes: programs whose renamed values fit kSplitSlots
    // slots run first in the smaller-footprint interpreter, the rest after
    bool split = false;
    const void* interp_fn8 = nullptr;
    int grid8 = 0;
    size_t smem8 = 0;
    UopFormat fmt{};                  // micro-op form of the chosen interpreter
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    galop_stats stats{};
    int launches = 0;
    bool pending = false;
};

// Batch counters: [0] work queue, [1..5] the pre-pass totals the
// statistics read, [6] programs of the first register-file class, [7] the
// first work item of the second class.
constexpr int kBatchCounters = 8;

#define B_CK(call, what)                                              \
    do {                                                              \
        cudaError_t _e = (call);                                      \
        if (_e != cudaSuccess) return b->ctx->cuda_fail(_e, what);    \
    } while (0)

namespace {

void drop_graph(galop_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// Layout, descriptors and launch configuration for the current shape.
int plan(galop_batch* b) {
    galop_ctx* ctx = b->ctx;
    const int n_pops = (int)b->pops.size();
    std::vector<PopLayout> lay(n_pops);
    std::vector<PopDesc> desc(n_pops);
    std::vector<int32_t> chunks(n_pops);
    int64_t base = 0, items = 0;
    for (int p = 0; p < n_pops; ++p) {
        BatchPop& P = b->pops[p];
        lay[p] = PopLayout{base, P.n, P.word_base, P.off_base, P.ds->N};
        desc[p] = PopDesc{P.ds->X.p, P.ds->y.p, P.ds->N, P.ds->Np, b->fitness.p + P.out_base,
                          b->sse.p + P.out_base, base, P.chunk_cases, (int32_t)P.n_chunks, P.ds->k,
                          objective_for(ctx, P.ds->ss_tot)};
        chunks[p] = (int32_t)P.n_chunks;
        base += P.n;
        items += P.n * P.n_chunks;
    }
    b->G = base;
    b->n_items = items;
    B_CK(cudaMemcpyAsync(b->layout.p, lay.data(), n_pops * sizeof(PopLayout), cudaMemcpyHostToDevice, b->stream),
         "H2D batch layout");
    B_CK(cudaMemcpyAsync(b->descs.p, desc.data(), n_pops * sizeof(PopDesc), cudaMemcpyHostToDevice, b->stream),
         "H2D batch descriptors");
    B_CK(cudaMemcpyAsync(b->chunks_of_pop.p, chunks.data(), n_pops * sizeof(int32_t), cudaMemcpyHostToDevice,
                         b->stream), "H2D batch chunks");
    B_CK(cudaStreamSynchronize(b->stream), "batch plan");   // host vectors go out of scope

    const int k = pick_k(ctx);
    const int wpb = pick_wpb(ctx);
    b->threads = 32 * wpb;
    // Batched work items need a shared-memory interpreter (2 or 3).
    const int dispatch = pick_dispatch(ctx) == 3 ? 3 : 2;
    b->interp_fn = ctx->isa.num_registers == 8
                       ? interp_kernel_nr8(k, dispatch, ctx->isa.profile, ctx->opt.reduce, kModeFitness)
                       : interp_kernel_nr16(k, dispatch, ctx->isa.profile, ctx->opt.reduce, kModeFitness);
    if (!b->interp_fn) return ctx->fail(GALOP_E_INVALID, "no batched interpreter for this configuration");
    b->smem = dispatch == 3 ? wide_smem_bytes(ctx->isa.num_registers, k, wpb)
                            : (size_t)(b->threads + 32) * ctx->isa.num_registers * k * sizeof(float);
    B_CK(cudaFuncSetAttribute(b->interp_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem), "smem attr");
    B_CK(cudaFuncSetAttribute(b->interp_fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                              cudaSharedmemCarveoutMaxShared), "carveout");
    int per_sm = 0;
    B_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->interp_fn, b->threads, b->smem), "occupancy");
    per_sm = std::max(per_sm, 1);
    const int64_t need = (b->n_items + wpb - 1) / wpb;
    b->grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->sm_count * per_sm, need));
    b->split = dispatch == 3 && b->fmt.wide && ctx->opt.intron_prepass && ctx->isa.num_registers > kSplitSlots;
    if (b->split) {
        b->interp_fn8 = kernel_for_slots(ctx, k, kModeFitness, kSplitSlots);
        if (!b->interp_fn8) return ctx->fail(GALOP_E_INVALID, "no batched interpreter for this configuration");
        b->smem8 = wide_smem_bytes(kSplitSlots, k, wpb);
        B_CK(cudaFuncSetAttribute(b->interp_fn8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem8),
             "smem attr");
        B_CK(cudaFuncSetAttribute(b->interp_fn8, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared), "carveout");
        int per_sm8 = 0;
        B_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm8, b->interp_fn8, b->threads, b->smem8),
             "occupancy");
        per_sm8 = std::max(per_sm8, 1);
        b->grid8 = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->sm_count * per_sm8, need));
    }
    b->planned_n.resize(n_pops);
    for (int p = 0; p < n_pops; ++p) b->planned_n[p] = b->pops[p].n;
    b->stats.cases_per_lane = k;
    b->stats.warps_per_block = wpb;
    b->stats.blocks = b->grid;
    return GALOP_OK;
}

// The device work of one generation, on b->stream (capturable: no
// allocation, no synchronisation, no host reads).
int enqueue(galop_batch* b) {
    galop_ctx* ctx = b->ctx;
    cudaStream_t s = b->stream;
    const int64_t G = b->G;
    b->launches = 0;
    B_CK(cudaMemsetAsync(b->counters.p, 0, kBatchCounters * sizeof(unsigned long long), s), "memset counters");
    B_CK(cudaMemsetAsync(b->hist.p, 0, kOrderBins * sizeof(unsigned int), s), "memset hist");
    if (G == 0) return GALOP_OK;
    const int tpb = 256;
    const unsigned blocks = (unsigned)((G + tpb - 1) / tpb);
    const int64_t n_tiles = (G + kScanTile - 1) / kScanTile;
    const int n_pops = (int)b->pops.size();
    const bool strip = ctx->opt.intron_prepass != 0;
    batch_rebase_kernel<<<blocks, tpb, 0, s>>>(b->layout.p, n_pops, G, b->local_off.p, b->starts.p, b->lens.p,
                                               b->prog_pop.p);
    SpanSource src{b->arena.p, b->starts.p, b->lens.p};
    prepass_count_kernel<SpanSource><<<blocks, tpb, 0, s>>>(src, G, ctx->isa, strip ? 1 : 0, b->eff_len.p,
                                                            b->counters.p + 1, nullptr);
    scan_tile_sums_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(b->eff_len.p, G, b->tiles.p);
    scan_tile_offsets_kernel<<<1, kScanThreads, 0, s>>>(b->tiles.p, n_tiles);
    scan_apply_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(b->eff_len.p, G, b->tiles.p, n_tiles, b->eff_off.p);
    prepass_compact_kernel<SpanSource><<<blocks, tpb, 0, s>>>(src, G, ctx->isa, strip ? 1 : 0, b->eff_off.p,
                                                              b->uops.p, nullptr, b->fmt, nullptr);
    const bool fold = b->fmt.wide && strip;
    if (b->fmt.wide) {
        // constants folded per program with its own population's input count
        // (intron pass on), forwarding flags on every wide stream
        FoldParams fp{ctx->isa.profile, ctx->isa.num_registers, ctx->isa.output_reg,
                      7u + (uint32_t)__builtin_ctz(b->fmt.stride / 128u), 0, b->descs.p, b->prog_pop.p,
                      fold ? 1 : 0, 1};
        fold_kernel<<<blocks, tpb, 0, s>>>(reinterpret_cast<uint4*>(b->uops.p), b->eff_off.p, G, fp, b->eff_len.p,
                                           b->livein.p,
                                           b->counters.p + 3);
        b->launches += 1;
    }
    const bool dedup = fold && b->dedup && G > 1;
    if (dedup) {
        // copies within a population share the representative's fitness
        const uint4* u4 = reinterpret_cast<const uint4*>(b->uops.p);
        size_t tmp = b->dtmp.cap;
        dedup_hash_kernel<<<blocks, tpb, 0, s>>>(u4, b->eff_off.p, b->eff_len.p, G, b->dkeys.p, b->dvals.p, b->rep.p,
                                                 b->prog_pop.p, b->livein.p);
        B_CK(cub::DeviceRadixSort::SortPairs(b->dtmp.p, tmp, b->dkeys.p, b->dkeys_sorted.p, b->dvals.p,
                                             b->dvals_sorted.p, (int)G, 0, 64, s), "dedup sort");
        dedup_run_start_kernel<<<blocks, tpb, 0, s>>>(b->dkeys_sorted.p, G, b->dhead.p);
        tmp = b->dtmp.cap;
        B_CK(cub::DeviceScan::InclusiveScan(b->dtmp.p, tmp, b->dhead.p, b->dvals.p, cub::Max(), (int)G, s),
             "dedup scan");
        dedup_rep_kernel<<<blocks, tpb, 0, s>>>(b->dvals.p, b->dvals_sorted.p, G, u4, b->eff_off.p, b->eff_len.p,
                                                b->rep.p, b->counters.p + 4, b->prog_pop.p, b->livein.p);
        b->launches += 5;
    }
    batch_key_kernel<<<blocks, tpb, 0, s>>>(b->layout.p, b->prog_pop.p, b->eff_len.p, G, b->key.p);
    // longest first; with the class split, the first register-file class
    // before the second (counters[6] = its program count)
    const uint32_t* cls = b->split ? b->livein.p : nullptr;
    order_hist_kernel<<<blocks, tpb, 0, s>>>(b->key.p, G, b->hist.p, cls, kSplitSlots);
    order_scan_kernel<<<1, 1024, 0, s>>>(b->hist.p, b->split ? b->counters.p + 6 : nullptr);
    order_scatter_kernel<<<blocks, tpb, 0, s>>>(b->key.p, G, b->hist.p, b->order.p, cls, kSplitSlots);
    batch_item_count_kernel<<<blocks, tpb, 0, s>>>(b->order.p, b->prog_pop.p, b->chunks_of_pop.p, b->key.p, G,
                                                   b->cnt.p);
    scan_tile_sums_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(b->cnt.p, G, b->tiles.p);
    scan_tile_offsets_kernel<<<1, kScanThreads, 0, s>>>(b->tiles.p, n_tiles);
    scan_apply_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(b->cnt.p, G, b->tiles.p, n_tiles, b->item_off.p);
    batch_item_fill_kernel<<<blocks, tpb, 0, s>>>(b->order.p, b->cnt.p, b->item_off.p, G, b->items.p,
                                                  b->first_item.p);
    b->launches += 16;
    if (b->split) {
        batch_split_items_kernel<<<1, 1, 0, s>>>(b->counters.p + 6, b->item_off.p, b->counters.p + 7);
        b->launches += 1;
    }
    B_CK(cudaGetLastError(), "batch pre-pass launch");

    InterpArgs a{};
    a.uops = b->uops.p;
    a.eff_off = b->eff_off.p;
    a.interp_len = fold ? b->eff_len.p : nullptr;
    a.livein = b->fmt.wide ? b->livein.p : nullptr;
    a.n_programs = G;
    a.n_chunks = 1;
    a.output_reg = ctx->isa.output_reg;
    a.consts = ctx->pool;
    a.counter = b->counters.p;
    a.partial = b->partial.p;
    a.pops = b->descs.p;
    a.prog_pop = b->prog_pop.p;
    a.items = b->items.p;
    a.n_items = b->n_items;
    a.n_items_dev = dedup ? b->item_off.p + G : nullptr;
    void* params[] = {&a};
    if (b->split) {
        // items [0, counters[7]) in the kSplitSlots-slot interpreter, then the
        // rest, each launch with its own work-queue counter reset
        a.class_split = b->counters.p + 7;
        a.class_part = 0;
        B_CK(cudaLaunchKernel(b->interp_fn8, dim3((unsigned)b->grid8), dim3(b->threads), params, b->smem8, s),
             "batched interpreter launch");
        B_CK(cudaMemsetAsync(b->counters.p, 0, sizeof(unsigned long long), s), "memset queue");
        a.class_part = 1;
        b->launches += 1;
    }
    B_CK(cudaLaunchKernel(b->interp_fn, dim3((unsigned)b->grid), dim3(b->threads), params, b->smem, s),
         "batched interpreter launch");
    batch_finalize_kernel<<<blocks, tpb, 0, s>>>(b->descs.p, b->prog_pop.p, b->first_item.p, b->partial.p, G);
    b->launches += 2;
    if (dedup) {
        batch_dedup_scatter_kernel<<<blocks, tpb, 0, s>>>(b->descs.p, b->prog_pop.p, b->rep.p, G);
        b->launches += 1;
    }
    B_CK(cudaGetLastError(), "batch finalize launch");
    return GALOP_OK;
}

}  // namespace

extern "C" {

int galop_dataset_create(galop_ctx* ctx, const float* inputs, const float* targets, int64_t n_cases,
                         int32_t num_inputs, galop_dataset** out) {
    if (!ctx || !out) return GALOP_E_INVALID;
    *out = nullptr;
    if (n_cases < 0 || num_inputs < 0 || num_inputs > ctx->isa.num_registers)
        return ctx->fail(GALOP_E_INVALID, "bad dataset shape: n_cases=%lld num_inputs=%d", (long long)n_cases,
                         num_inputs);
    if (n_cases > 0 && (!targets || (num_inputs > 0 && !inputs)))
        return ctx->fail(GALOP_E_INVALID, "null dataset pointer");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    cudaGetLastError();   // a stale error of an earlier call must not be reported as ours
    galop_dataset* ds = new galop_dataset();
    ds->ctx = ctx;
    ds->device = ctx->device;
    ds->N = n_cases;
    ds->k = num_inputs;
    ds->ss_tot = targets_ss_tot(targets, n_cases);
    ds->Np = std::max<int64_t>(1024, (n_cases + 1023) / 1024 * 1024);
    ds->X.cap = (size_t)ds->Np * std::max(num_inputs, 1);
    ds->y.cap = (size_t)ds->Np;
    cudaStream_t s = ctx->stream;
    float* aos = nullptr;
    float* yin = nullptr;
    const size_t nx = std::max<size_t>((size_t)n_cases * num_inputs, 1);
    const size_t ny = std::max<size_t>((size_t)n_cases, 1);
    cudaError_t e = cudaMallocAsync(&ds->X.p, ds->X.cap * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&ds->y.p, ds->y.cap * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&aos, nx * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&yin, ny * sizeof(float), s);
    if (e == cudaSuccess && n_cases * num_inputs > 0)
        e = cudaMemcpyAsync(aos, inputs, (size_t)n_cases * num_inputs * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && n_cases > 0)
        e = cudaMemcpyAsync(yin, targets, (size_t)n_cases * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        dataset_transpose_kernel<<<(unsigned)((ds->Np + 255) / 256), 256, 0, s>>>(aos, yin, n_cases, num_inputs,
                                                                                ds->Np, ds->X.p, ds->y.p);
        e = cudaGetLastError();
    }
    if (aos) cudaFreeAsync(aos, s);
    if (yin) cudaFreeAsync(yin, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // this stream only, not the device
    if (e != cudaSuccess) {
        if (ds->X.p) cudaFreeAsync(ds->X.p, s);
        if (ds->y.p) cudaFreeAsync(ds->y.p, s);
        delete ds;
        return ctx->cuda_fail(e, "dataset upload");
    }
    *out = ds;
    return GALOP_OK;
}

int galop_dataset_destroy(galop_dataset* ds) {
    if (!ds) return GALOP_OK;
    cudaSetDevice(ds->device);
    // stream-ordered release; no kernel may still be reading the dataset
    if (ds->X.p) cudaFreeAsync(ds->X.p, 0);
    if (ds->y.p) cudaFreeAsync(ds->y.p, 0);
    delete ds;
    return GALOP_OK;
}

int64_t galop_dataset_device_bytes(const galop_dataset* ds) {
    if (!ds) return 0;
    return (int64_t)((ds->X.cap + ds->y.cap) * sizeof(float));
}

}  // extern "C"

namespace {

void chunk_policy(const galop_ctx* ctx, BatchPop& P) {
    if (ctx->opt.reduce == GALOP_REDUCE_ORDERED) {   // strict case order: one item per program
        P.chunk_cases = std::max<int64_t>(1024, (P.ds->N + 1023) / 1024 * 1024);
        P.n_chunks = 1;
    } else {
        P.chunk_cases = chunk_cases_for(P.ds->N);
        P.n_chunks = chunks_for(P.ds->N);
    }
}

// Streams, events and every device buffer, sized once.
int allocate(galop_batch* b, int64_t words, int64_t offs, int64_t progs, int64_t items, int n_pops) {
    galop_ctx* ctx = b->ctx;
    b->total_max_programs = progs;
    b->total_max_words = words;
    b->total_max_items = items;
    const size_t G1 = (size_t)std::max<int64_t>(progs, 1);
    const size_t W1 = (size_t)std::max<int64_t>(words, 1);
    const size_t I1 = (size_t)std::max<int64_t>(items, 1);
    const size_t T1 = (size_t)((progs + kScanTile - 1) / kScanTile + 1);
    const size_t P1 = (size_t)std::max(n_pops, 1);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev2);
    if (e == cudaSuccess) e = b->arena.ensure(W1);
    b->fmt = uop_format(ctx);
    if (e == cudaSuccess) e = b->uops.ensure(W1 * (b->fmt.wide ? 4 : 1));
    if (e == cudaSuccess) e = b->local_off.ensure((size_t)std::max<int64_t>(offs, 1));
    if (e == cudaSuccess) e = b->starts.ensure(G1);
    if (e == cudaSuccess) e = b->lens.ensure(G1);
    if (e == cudaSuccess) e = b->prog_pop.ensure(G1);
    if (e == cudaSuccess) e = b->eff_len.ensure(G1);
    if (e == cudaSuccess) e = b->livein.ensure(G1);
    if (e == cudaSuccess) e = b->eff_off.ensure(G1 + 1);
    if (e == cudaSuccess) e = b->key.ensure(G1);
    if (e == cudaSuccess) e = b->order.ensure(G1);
    if (e == cudaSuccess) e = b->cnt.ensure(G1);
    if (e == cudaSuccess) e = b->item_off.ensure(G1 + 1);
    if (e == cudaSuccess) e = b->first_item.ensure(G1);
    if (e == cudaSuccess) e = b->tiles.ensure(T1);
    if (e == cudaSuccess) e = b->items.ensure(I1);
    if (e == cudaSuccess) e = b->partial.ensure(I1);
    if (e == cudaSuccess) e = b->counters.ensure(kBatchCounters);
    b->dedup = ctx->opt.dedup && b->fmt.wide && ctx->opt.intron_prepass && progs > 1;
    if (b->dedup) {
        if (e == cudaSuccess) e = b->dkeys.ensure(G1);
        if (e == cudaSuccess) e = b->dkeys_sorted.ensure(G1);
        if (e == cudaSuccess) e = b->dvals.ensure(G1);
        if (e == cudaSuccess) e = b->dvals_sorted.ensure(G1);
        if (e == cudaSuccess) e = b->rep.ensure(G1);
        if (e == cudaSuccess) e = b->dhead.ensure(G1);
        size_t tsort = 0, tscan = 0;
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortPairs(nullptr, tsort, b->dkeys.p, b->dkeys_sorted.p, b->dvals.p,
                                                b->dvals_sorted.p, (int)G1, 0, 64);
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveScan(nullptr, tscan, b->dhead.p, b->dvals.p, cub::Max(), (int)G1);
        if (e == cudaSuccess) e = b->dtmp.ensure(std::max<size_t>(std::max(tsort, tscan), 1));
    }
    if (e == cudaSuccess) e = b->hist.ensure(kOrderBins);
    if (e == cudaSuccess) e = b->fitness.ensure(G1);
    if (e == cudaSuccess) e = b->sse.ensure(G1);
    if (e == cudaSuccess) e = b->layout.ensure(P1);
    if (e == cudaSuccess) e = b->descs.ensure(P1);
    if (e == cudaSuccess) e = b->chunks_of_pop.ensure(P1);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "batch allocation");
    return GALOP_OK;
}

}  // namespace

extern "C" {

int galop_batch_create(galop_ctx* ctx, const galop_population_spec* specs, int32_t n_pops, galop_batch** out) {
    if (!ctx || !out || n_pops <= 0 || !specs) return GALOP_E_INVALID;
    *out = nullptr;
    for (int p = 0; p < n_pops; ++p)
        if (!specs[p].dataset || specs[p].dataset->ctx != ctx || specs[p].max_programs < 0 || specs[p].max_words < 0)
            return ctx->fail(GALOP_E_INVALID, "bad population spec %d", p);
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    galop_batch* b = new galop_batch();
    b->ctx = ctx;
    b->device = ctx->device;
    b->pops.resize(n_pops);
    int64_t words = 0, offs = 0, progs = 0, items = 0;
    for (int p = 0; p < n_pops; ++p) {
        BatchPop& P = b->pops[p];
        P.ds = specs[p].dataset;
        P.max_programs = specs[p].max_programs;
        P.max_words = specs[p].max_words;
        P.word_base = words;
        P.off_base = offs;
        P.out_base = progs;
        chunk_policy(ctx, P);
        words += P.max_words;
        offs += P.max_programs + 1;
        progs += P.max_programs;
        items += P.max_programs * P.n_chunks;
    }
    if (int rc = allocate(b, words, offs, progs, items, n_pops)) {
        galop_batch_destroy(b);
        return rc;
    }
    *out = b;
    return GALOP_OK;
}

int galop_batch_create_pool(galop_ctx* ctx, int32_t max_pops, int64_t max_programs, int64_t max_words,
                            int64_t max_items, galop_batch** out) {
    if (!ctx || !out || max_pops <= 0 || max_programs < 0 || max_words < 0 || max_items < 0)
        return GALOP_E_INVALID;
    *out = nullptr;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    galop_batch* b = new galop_batch();
    b->ctx = ctx;
    b->device = ctx->device;
    b->pooled = true;
    b->max_pops = max_pops;
    if (int rc = allocate(b, max_words, max_programs + max_pops, max_programs, max_items, max_pops)) {
        galop_batch_destroy(b);
        return rc;
    }
    *out = b;
    return GALOP_OK;
}

int galop_batch_clear(galop_batch* b) {
    if (!b) return GALOP_E_INVALID;
    if (!b->pooled) return b->ctx->fail(GALOP_E_STATE, "galop_batch_clear needs a pooled batch");
    b->pops.clear();
    b->cur_words = b->cur_offs = b->cur_progs = b->cur_items = 0;
    return GALOP_OK;
}

int galop_batch_append(galop_batch* b, const galop_dataset* ds, const uint32_t* words, const int64_t* offsets,
                       int64_t n_programs, int32_t* pop_out) {
    if (!b || !ds || !offsets || n_programs < 0) return GALOP_E_INVALID;
    galop_ctx* ctx = b->ctx;
    if (!b->pooled) return ctx->fail(GALOP_E_STATE, "galop_batch_append needs a pooled batch");
    if (ds->ctx != ctx) return ctx->fail(GALOP_E_INVALID, "dataset belongs to another context");
    BatchPop P;
    P.ds = ds;
    chunk_policy(ctx, P);
    const int64_t total = offsets[n_programs];
    if ((int32_t)b->pops.size() >= b->max_pops || b->cur_progs + n_programs > b->total_max_programs ||
        b->cur_words + total > b->total_max_words || b->cur_items + n_programs * P.n_chunks > b->total_max_items)
        return GALOP_E_CAPACITY;
    P.max_programs = n_programs;
    P.max_words = total;
    P.word_base = b->cur_words;
    P.off_base = b->cur_offs;
    P.out_base = b->cur_progs;
    b->pops.push_back(P);
    const int32_t pop = (int32_t)b->pops.size() - 1;
    const int rc = galop_batch_set_population(b, pop, words, offsets, n_programs);
    if (rc) {
        b->pops.pop_back();
        return rc;
    }
    b->cur_words += total;
    b->cur_offs += n_programs + 1;
    b->cur_progs += n_programs;
    b->cur_items += n_programs * P.n_chunks;
    b->planned_n.clear();      // composition changed: plan again
    if (pop_out) *pop_out = pop;
    return GALOP_OK;
}

int galop_batch_destroy(galop_batch* b) {
    if (!b) return GALOP_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    b->arena.release(); b->uops.release(); b->local_off.release(); b->starts.release();
    b->eff_off.release(); b->item_off.release(); b->first_item.release(); b->tiles.release();
    b->lens.release(); b->prog_pop.release(); b->eff_len.release(); b->livein.release(); b->key.release(); b->order.release();
    b->cnt.release(); b->chunks_of_pop.release(); b->items.release(); b->counters.release(); b->hist.release();
    b->dkeys.release(); b->dkeys_sorted.release(); b->dvals.release(); b->dvals_sorted.release(); b->rep.release();
    b->dhead.release(); b->dtmp.release();
    b->fitness.release(); b->sse.release(); b->partial.release(); b->layout.release(); b->descs.release();
    for (cudaEvent_t e : {b->ev0, b->ev1, b->ev2}) if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return GALOP_OK;
}

int64_t galop_batch_device_bytes(const galop_batch* b) {
    if (!b) return 0;
    int64_t s = 0;
    s += (b->arena.cap + b->uops.cap) * 4;
    s += (b->local_off.cap + b->starts.cap + b->eff_off.cap + b->item_off.cap + b->first_item.cap + b->tiles.cap) * 8;
    s += (b->lens.cap + b->prog_pop.cap + b->eff_len.cap + b->livein.cap + b->key.cap + b->order.cap + b->cnt.cap) * 4;
    s += (b->items.cap + b->partial.cap + b->sse.cap) * 8 + b->fitness.cap * 4;
    s += (b->dkeys.cap + b->dkeys_sorted.cap) * 8 + (b->dvals.cap + b->dvals_sorted.cap + b->rep.cap + b->dhead.cap) * 4;
    s += b->dtmp.cap;
    return s;
}

int galop_batch_set_population(galop_batch* b, int32_t pop, const uint32_t* words, const int64_t* offsets,
                               int64_t n_programs) {
    if (!b) return GALOP_E_INVALID;
    galop_ctx* ctx = b->ctx;
    if (pop < 0 || pop >= (int)b->pops.size()) return ctx->fail(GALOP_E_INVALID, "population %d out of range", pop);
    BatchPop& P = b->pops[pop];
    if (n_programs < 0 || !offsets) return ctx->fail(GALOP_E_INVALID, "bad population arguments");
    if (n_programs > P.max_programs)
        return ctx->fail(GALOP_E_CAPACITY, "population %d: %lld programs > capacity %lld", pop,
                         (long long)n_programs, (long long)P.max_programs);
    if (offsets[0] != 0) return ctx->fail(GALOP_E_INVALID, "offsets[0] must be 0");
    for (int64_t i = 0; i < n_programs; ++i)
        if (offsets[i + 1] < offsets[i]) return ctx->fail(GALOP_E_INVALID, "offsets decrease at %lld", (long long)i);
    const int64_t total = offsets[n_programs];
    if (total > P.max_words)
        return ctx->fail(GALOP_E_CAPACITY, "population %d: %lld instructions > capacity %lld", pop,
                         (long long)total, (long long)P.max_words);
    if (total > 0 && !words) return ctx->fail(GALOP_E_INVALID, "null words");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    if (total > 0)
        B_CK(cudaMemcpyAsync(b->arena.p + P.word_base, words, (size_t)total * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, b->stream), "H2D population words");
    B_CK(cudaMemcpyAsync(b->local_off.p + P.off_base, offsets, (size_t)(n_programs + 1) * sizeof(int64_t),
                         cudaMemcpyHostToDevice, b->stream), "H2D population offsets");
    P.n = n_programs;
    return GALOP_OK;
}

int galop_batch_evaluate(galop_batch* b, int32_t use_graph) {
    if (!b) return GALOP_E_INVALID;
    galop_ctx* ctx = b->ctx;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    cudaGetLastError();   // a stale error of an earlier call must not be reported as ours
    bool same = b->planned_n.size() == b->pops.size();
    for (size_t p = 0; same && p < b->pops.size(); ++p) same = b->planned_n[p] == b->pops[p].n;
    if (!same) {
        drop_graph(b);
        if (int rc = plan(b)) return rc;
    }
    b->stats = galop_stats{};
    b->stats.n_programs = b->G;
    B_CK(cudaEventRecord(b->ev0, b->stream), "event");
    if (use_graph) {
        if (!b->exec) {
            B_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            const int rc = enqueue(b);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
            if (rc) { if (g) cudaGraphDestroy(g); return rc; }
            B_CK(ce, "end capture");
            b->graph = g;
            B_CK(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
        }
        B_CK(cudaGraphLaunch(b->exec, b->stream), "graph launch");
    } else {
        if (int rc = enqueue(b)) return rc;
    }
    B_CK(cudaEventRecord(b->ev1, b->stream), "event");
    b->pending = true;
    return GALOP_OK;
}

int galop_batch_synchronize(galop_batch* b) {
    if (!b) return GALOP_E_INVALID;
    galop_ctx* ctx = b->ctx;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    B_CK(cudaStreamSynchronize(b->stream), "batch synchronize");
    if (b->pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) b->stats.total_ms = ms;
        b->stats.interp_ms = b->stats.total_ms;
        unsigned long long tot[5] = {0, 0, 0, 0, 0};
        B_CK(cudaMemcpy(tot, b->counters.p + 1, sizeof tot, cudaMemcpyDeviceToHost), "batch stats");
        b->stats.raw_instructions = (int64_t)tot[0];
        b->stats.eff_instructions = (int64_t)tot[1];
        b->stats.interp_instructions =
            (b->fmt.wide && ctx->opt.intron_prepass) ? (int64_t)(tot[2] - tot[4]) : (int64_t)tot[1];
        b->stats.kernels_launched = b->launches;
        b->stats.case_chunks = (int32_t)(b->G ? b->n_items / b->G : 0);
        b->pending = false;
    }
    return GALOP_OK;
}

int galop_batch_get_fitness(galop_batch* b, int32_t pop, float* fitness_out, double* sse_out) {
    if (!b) return GALOP_E_INVALID;
    galop_ctx* ctx = b->ctx;
    if (pop < 0 || pop >= (int)b->pops.size()) return ctx->fail(GALOP_E_INVALID, "population out of range");
    const BatchPop& P = b->pops[pop];
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    if (P.n > 0 && fitness_out)
        B_CK(cudaMemcpyAsync(fitness_out, b->fitness.p + P.out_base, (size_t)P.n * sizeof(float),
                             cudaMemcpyDeviceToHost, b->stream), "D2H fitness");
    if (P.n > 0 && sse_out)
        B_CK(cudaMemcpyAsync(sse_out, b->sse.p + P.out_base, (size_t)P.n * sizeof(double), cudaMemcpyDeviceToHost,
                             b->stream), "D2H sse");
    return galop_batch_synchronize(b);
}

int galop_batch_last_stats(galop_batch* b, galop_stats* out) {
    if (!b || !out) return GALOP_E_INVALID;
    if (b->pending)
        if (int rc = galop_batch_synchronize(b)) return rc;
    *out = b->stats;
    return GALOP_OK;
}

void* galop_batch_stream(galop_batch* b) { return b ? (void*)b->stream : nullptr; }

int galop_batch_get_fitness_all(galop_batch* b, float* fitness_out, int64_t* eff_per_pop) {
    if (!b) return GALOP_E_INVALID;
    galop_ctx* ctx = b->ctx;
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    // Populations occupy consecutive output slots in pooled batches; fixed
    // batches have per-population regions, copied one by one.
    int64_t base = 0;
    std::vector<int64_t> gb(b->pops.size());
    for (size_t p = 0; p < b->pops.size(); ++p) { gb[p] = base; base += b->pops[p].n; }
    std::vector<int64_t> eo;
    if (eff_per_pop) {
        eo.resize((size_t)base + 1);
        B_CK(cudaMemcpyAsync(eo.data(), b->eff_off.p, eo.size() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                             b->stream), "D2H effective offsets");
    }
    int64_t o = 0;
    for (size_t p = 0; p < b->pops.size(); ++p) {
        const BatchPop& P = b->pops[p];
        if (P.n && fitness_out)
            B_CK(cudaMemcpyAsync(fitness_out + o, b->fitness.p + P.out_base, (size_t)P.n * sizeof(float),
                                 cudaMemcpyDeviceToHost, b->stream), "D2H fitness");
        o += P.n;
    }
    if (int rc = galop_batch_synchronize(b)) return rc;
    if (eff_per_pop)
        for (size_t p = 0; p < b->pops.size(); ++p) eff_per_pop[p] = eo[gb[p] + b->pops[p].n] - eo[gb[p]];
    return GALOP_OK;
}

int galop_batch_population_work(galop_batch* b, int32_t pop, int64_t* eff_instructions) {
    if (!b || !eff_instructions) return GALOP_E_INVALID;
    galop_ctx* ctx = b->ctx;
    if (pop < 0 || pop >= (int)b->pops.size()) return ctx->fail(GALOP_E_INVALID, "population out of range");
    int64_t base = 0;
    for (int p = 0; p < pop; ++p) base += b->pops[p].n;
    const int64_t n = b->pops[pop].n;
    *eff_instructions = 0;
    if (n == 0) return GALOP_OK;
    std::vector<int64_t> off(2);
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    B_CK(cudaStreamSynchronize(b->stream), "batch synchronize");
    B_CK(cudaMemcpy(&off[0], b->eff_off.p + base, sizeof(int64_t), cudaMemcpyDeviceToHost), "D2H offsets");
    B_CK(cudaMemcpy(&off[1], b->eff_off.p + base + n, sizeof(int64_t), cudaMemcpyDeviceToHost), "D2H offsets");
    *eff_instructions = off[1] - off[0];
    return GALOP_OK;
}

}  // extern "C"
