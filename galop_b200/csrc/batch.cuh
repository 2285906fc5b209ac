// batch.cuh -- device kernels of the batched evaluation (galop_batch_*).
//
// Many populations, each with its own resident dataset, are evaluated by one
// persistent interpreter launch.  Programs of all populations are numbered
// globally (population p owns [prog_base_p, prog_base_p + n_p)).  The raw
// words of population p live in its region of one arena; its CSR offsets are
// copied into its region of a staging array and rebased here into a
// (start, length) span table that the intron pass reads like one population
// (SpanSource).  Work items are (program, case chunk) pairs ordered by
// interpreted work (effective length x cases), largest first.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "isa.cuh"
#include "interp.cuh"

namespace galop {

// Programs given by explicit start offsets into one words array and lengths.
struct SpanSource {
    const uint32_t* words;
    const int64_t* starts;
    const int32_t* lens;
    __device__ __forceinline__ int64_t start(int64_t i) const { return starts[i]; }
    __device__ __forceinline__ int64_t length(int64_t i) const { return (int64_t)lens[i]; }
};

struct PopLayout {
    int64_t prog_base;     // first global program
    int64_t n_programs;
    int64_t word_base;     // region of the arena
    int64_t off_base;      // region of the offset staging array (n_programs + 1 entries)
    int64_t n_cases;
};

// Population of global program g (binary search over prog_base).
__device__ __forceinline__ int pop_of(const PopLayout* pops, int n_pops, int64_t g) {
    int lo = 0, hi = n_pops - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pops[mid].prog_base <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

static __global__ void batch_rebase_kernel(const PopLayout* __restrict__ pops, int n_pops, int64_t n_total,
                                           const int64_t* __restrict__ local_off, int64_t* __restrict__ start,
                                           int32_t* __restrict__ len, int32_t* __restrict__ prog_pop) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_total) return;
    const int p = pop_of(pops, n_pops, g);
    const PopLayout L = pops[p];
    const int64_t j = g - L.prog_base;
    const int64_t a = local_off[L.off_base + j];
    const int64_t b = local_off[L.off_base + j + 1];
    start[g] = L.word_base + a;
    len[g] = (int32_t)(b - a);
    prog_pop[g] = p;
}

// Sort key: log-scale bin of interpreted work (effective length x cases),
// larger key = more work.  Bins of width 2^(1/48): keys up to 2046 cover
// work below 2^42, and each register-file class of the order holds 2047.
static __global__ void batch_key_kernel(const PopLayout* __restrict__ pops, const int32_t* __restrict__ prog_pop,
                                        const int32_t* __restrict__ eff_len, int64_t n_total,
                                        int32_t* __restrict__ key) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_total) return;
    if (eff_len[g] < 0) {            // a copy left out by dedup: last in the order, no work items
        key[g] = -1;
        return;
    }
    const double work = (double)eff_len[g] * (double)pops[prog_pop[g]].n_cases;
    int k = work >= 1.0 ? (int)(log2(work) * 48.0) + 1 : 0;
    key[g] = k < 2046 ? k : 2046;
}

// Work items per program, by position in the order.
static __global__ void batch_item_count_kernel(const int32_t* __restrict__ order,
                                               const int32_t* __restrict__ prog_pop,
                                               const int32_t* __restrict__ chunks_of_pop,
                                               const int32_t* __restrict__ key, int64_t n_total,
                                               int32_t* __restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total) return;
    const int32_t g = order[i];
    cnt[i] = key[g] < 0 ? 0 : chunks_of_pop[prog_pop[g]];
}

static __global__ void batch_item_fill_kernel(const int32_t* __restrict__ order,
                                              const int32_t* __restrict__ cnt,
                                              const int64_t* __restrict__ item_off, int64_t n_total,
                                              unsigned long long* __restrict__ items,
                                              int64_t* __restrict__ first_item) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total) return;
    const int64_t g = order[i];
    const int64_t o = item_off[i];
    for (int c = 0; c < cnt[i]; ++c) items[o + c] = ((unsigned long long)g << 20) | (unsigned long long)c;
    first_item[g] = o;
}

// The first work item of the second register-file class: the order holds
// the n0 = *class0 programs of the first class first, so their items are
// items [0, item_off[n0]).  One thread.
static __global__ void batch_split_items_kernel(const unsigned long long* __restrict__ class0,
                                                const int64_t* __restrict__ item_off,
                                                unsigned long long* __restrict__ split_item) {
    *split_item = (unsigned long long)item_off[*class0];
}

// Copies left out by dedup take their representative's results (same
// population, so the same output arrays).
static __global__ void batch_dedup_scatter_kernel(const PopDesc* __restrict__ descs,
                                                  const int32_t* __restrict__ prog_pop,
                                                  const int32_t* __restrict__ rep, int64_t n_total) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_total) return;
    const int32_t r = rep[g];
    if (r == (int32_t)g) return;
    const PopDesc d = descs[prog_pop[g]];
    d.fitness[g - d.prog_base] = d.fitness[r - d.prog_base];
    if (d.sse) d.sse[g - d.prog_base] = d.sse[r - d.prog_base];
}

// Programs split into case chunks: sum the chunk partials in chunk order.
static __global__ void batch_finalize_kernel(const PopDesc* __restrict__ descs, const int32_t* __restrict__ prog_pop,
                                             const int64_t* __restrict__ first_item,
                                             const double* __restrict__ partial, int64_t n_total) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_total) return;
    const PopDesc d = descs[prog_pop[g]];
    if (d.n_chunks <= 1) return;
    const int64_t o = first_item[g];
    double s = 0.0;
    for (int c = 0; c < d.n_chunks; ++c) s += partial[o + c];
    d.fitness[g - d.prog_base] = fitness_of(s, d.N, d.obj);
    if (d.sse) d.sse[g - d.prog_base] = s;
}

}  // namespace galop
