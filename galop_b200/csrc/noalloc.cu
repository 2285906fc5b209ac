// noalloc.cu -- population evaluation for callers that cannot allocate.
//
// Every other entry point keeps its working buffers (micro-ops, offsets,
// evaluation order, work-queue counters, per-chunk partial sums) in device
// memory that it obtains with cudaMalloc and grows as populations grow.
// Some callers cannot let a library do that:
//   - hosts that own all device memory through their own pool allocator
//     (a framework's caching allocator, a serving process with a fixed
//     per-model budget) and must never see an out-of-memory failure, or
//     memory they did not account for, in the middle of a run;
//   - loops that must not stall: cudaMalloc and cudaFree can synchronise
//     the whole device.
//
// galop_evaluate_csr_noalloc runs the same pre-pass and the compact
// interpreter (dispatch 2: one 32-bit micro-op per instruction) on the
// caller's device buffers, with its working buffers in one file-scope
// __device__ array of fixed size (about 11 MiB) that every GPU loading this
// library holds until the process exits.  It allocates nothing: no
// cudaMalloc, no cudaFree, no allocating library routine.
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>

#include "../../include/galop_b200.h"
#include "interp.cuh"
#include "prepass.cuh"

namespace galop {
const void* interp_kernel_nr8(int k, int dispatch, int profile, int reduce, int mode);
const void* interp_kernel_nr16(int k, int dispatch, int profile, int reduce, int mode);
}  // namespace galop

using namespace galop;

namespace {

constexpr int64_t kNaMaxPrograms = GALOP_NOALLOC_MAX_PROGRAMS;
constexpr int64_t kNaMaxWords = GALOP_NOALLOC_MAX_WORDS;
constexpr int64_t kNaMaxPartials = 4 * GALOP_NOALLOC_MAX_PROGRAMS;
constexpr int64_t kNaMaxTiles = (kNaMaxPrograms + kScanTile - 1) / kScanTile;
constexpr int kNaDispatch = 2;   // 32-bit micro-ops: one scratch word per instruction

struct NoAllocScratch {
    uint32_t uops[kNaMaxWords];
    int64_t eff_off[kNaMaxPrograms + 1];
    int64_t tiles[kNaMaxTiles + 1];
    double partial[kNaMaxPartials];
    int32_t eff_len[kNaMaxPrograms];
    int32_t order[kNaMaxPrograms];
    unsigned int hist[kOrderBins];
    // [0] work-queue head, [1..2] length totals, [3] set by
    // check_offsets_kernel when the caller's offsets are inconsistent
    unsigned long long counters[4];
};

// The scratch itself.  Host code must not pass `g_noalloc_scratch` to a
// kernel: in host code the name is a host-side stand-in, not a device
// address.  The device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_addr[kMaxDevices] = {};

// Every kernel this entry point can launch, loaded on the current device
// (cudaFuncGetAttributes makes the runtime load a kernel's code), so that
// no later call, whatever its options, loads code on the device.
cudaError_t preload_kernels() {
    cudaFuncAttributes fa{};
    const void* fixed[] = {
        (const void*)&check_offsets_kernel,
        (const void*)&prepass_count_kernel<CsrSource>,
        (const void*)&scan_tile_sums_kernel,
        (const void*)&scan_tile_offsets_kernel,
        (const void*)&scan_apply_kernel,
        (const void*)&prepass_compact_kernel<CsrSource>,
        (const void*)&order_hist_kernel,
        (const void*)&order_scan_kernel,
        (const void*)&order_scatter_kernel,
        (const void*)&finalize_kernel,
        (const void*)&poison_results_kernel,
    };
    for (const void* f : fixed)
        if (cudaError_t e = cudaFuncGetAttributes(&fa, f)) return e;
    for (int nr : {8, 16})
        for (int k : {1, 2, 4, 8})
            for (int profile : {kProfileRef, kProfileBj})
                for (int reduce : {kReduceKahan32, kReduceFp64, kReduceOrdered}) {
                    const void* f = nr == 8 ? interp_kernel_nr8(k, kNaDispatch, profile, reduce, kModeFitness)
                                            : interp_kernel_nr16(k, kNaDispatch, profile, reduce, kModeFitness);
                    if (!f) return cudaErrorInvalidDeviceFunction;
                    if (cudaError_t e = cudaFuncGetAttributes(&fa, f)) return e;
                }
    return cudaSuccess;
}

// Once per device, with that device current: the scratch's device address
// (checked return code) and the kernels' code.
cudaError_t scratch_for_device(int device, NoAllocScratch** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess) e = preload_kernels();
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

// Reference constant pools (src/LGPConfig.h:159-168).
const float kPool8[8] = {0.0f, 1.0f, -1.0f, 3.14159f, 0.5f, 2.0f, 10.0f, 100.0f};
const float kPool16[16] = {0.0f, 1.0f, -1.0f, 3.14159f, 0.5f, 2.0f, 10.0f, 100.0f,
                           0.1f, -0.5f, 0.25f, 5.0f, 20.0f, -2.0f, 0.01f, 1000.0f};

}  // namespace

extern "C" int galop_evaluate_csr_noalloc(const galop_options* opt, const uint32_t* d_words,
                                          const int64_t* d_offsets, int64_t n_programs, int64_t total_words,
                                          const float* d_inputs, const float* d_targets, int64_t n_cases,
                                          int64_t padded_cases, int32_t num_inputs, float* d_fitness,
                                          double* d_sse, void* stream) {
    if (!opt || !d_offsets || n_programs < 0 || total_words < 0 || n_cases < 0) return GALOP_E_INVALID;
    if (opt->num_registers != 8 && opt->num_registers != 16) return GALOP_E_INVALID;
    if (opt->profile != GALOP_PROFILE_REF && opt->profile != GALOP_PROFILE_BJ) return GALOP_E_INVALID;
    if (opt->reduce < GALOP_REDUCE_KAHAN32 || opt->reduce > GALOP_REDUCE_ORDERED) return GALOP_E_INVALID;
    if (opt->objective != GALOP_OBJECTIVE_MSE) return GALOP_E_INVALID;   // R^2 needs the targets' ss_tot
    if (num_inputs < 0 || num_inputs > opt->num_registers) return GALOP_E_INVALID;
    if (padded_cases < n_cases || padded_cases % 1024 != 0 || padded_cases == 0) return GALOP_E_INVALID;
    if (n_programs > kNaMaxPrograms || total_words > kNaMaxWords) return GALOP_E_CAPACITY;
    if (n_programs > 0 && (!d_words && total_words > 0)) return GALOP_E_INVALID;
    if (n_programs > 0 && (!d_fitness || !d_targets || (num_inputs > 0 && !d_inputs))) return GALOP_E_INVALID;
    if (n_programs == 0) return GALOP_OK;

    // An error that an earlier CUDA call of the caller left pending is the
    // caller's to read: report it without clearing it.
    if (cudaPeekAtLastError() != cudaSuccess) return GALOP_E_CUDA;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return GALOP_E_NO_DEVICE; }
    NoAllocScratch* sc = nullptr;
    if (scratch_for_device(device, &sc) != cudaSuccess) { cudaGetLastError(); return GALOP_E_CUDA; }
    int sm_count = 0;
    if (cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return GALOP_E_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    IsaParams isa{opt->profile, opt->num_registers, opt->input_protect ? 1 : 0,
                  opt->input_protect ? opt->num_registers / 2 : 0};
    ConstPool pool{};
    const float* src_pool = opt->constants ? opt->constants : (opt->num_registers == 16 ? kPool16 : kPool8);
    for (int i = 0; i < kMaxRegisters; ++i) pool.c[i] = i < opt->num_registers ? src_pool[i] : 0.0f;
    const bool strip = opt->intron_prepass != 0;
    const int k = (opt->cases_per_lane == 1 || opt->cases_per_lane == 2 || opt->cases_per_lane == 4 ||
                   opt->cases_per_lane == 8) ? opt->cases_per_lane : 4;
    const int wpb = (opt->warps_per_block >= 1 && opt->warps_per_block <= 8) ? opt->warps_per_block : 4;

    // The scratch keeps the previous call's contents: the work-queue head,
    // the length totals, the order histogram and the offset-check flag
    // must start at zero.
    cudaError_t e = cudaMemsetAsync(sc->counters, 0, sizeof(sc->counters), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(sc->hist, 0, sizeof(sc->hist), s);
    if (e != cudaSuccess) { cudaGetLastError(); return GALOP_E_CUDA; }

    // The caller's offsets are checked against total_words on the device
    // before any word is read: with inconsistent offsets every program is
    // treated as empty (nothing beyond total_words is read, nothing beyond
    // the scratch written) and every result becomes NaN.
    const int64_t n = n_programs;
    unsigned long long* bad = sc->counters + 3;
    check_offsets_kernel<<<(unsigned)((n + 256) / 256), 256, 0, s>>>(d_offsets, n, total_words, bad);

    // Intron pass, scan, compaction, longest-first order (prepass.cuh).
    CsrSource src{d_words, d_offsets};
    const int tpb = 256;
    const unsigned blocks = (unsigned)((n + tpb - 1) / tpb);
    const int64_t n_tiles = (n + kScanTile - 1) / kScanTile;
    prepass_count_kernel<CsrSource><<<blocks, tpb, 0, s>>>(src, n, isa, strip ? 1 : 0, sc->eff_len,
                                                           sc->counters + 1, bad);
    scan_tile_sums_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(sc->eff_len, n, sc->tiles);
    scan_tile_offsets_kernel<<<1, kScanThreads, 0, s>>>(sc->tiles, n_tiles);
    scan_apply_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s>>>(sc->eff_len, n, sc->tiles, n_tiles, sc->eff_off);
    prepass_compact_kernel<CsrSource><<<blocks, tpb, 0, s>>>(src, n, isa, strip ? 1 : 0, sc->eff_off, sc->uops,
                                                             nullptr, UopFormat{}, bad);
    const bool sched = n > 1;
    if (sched) {
        order_hist_kernel<<<blocks, tpb, 0, s>>>(sc->eff_len, n, sc->hist, nullptr, 0);
        order_scan_kernel<<<1, 1024, 0, s>>>(sc->hist, nullptr);
        order_scatter_kernel<<<blocks, tpb, 0, s>>>(sc->eff_len, n, sc->hist, sc->order, nullptr, 0);
    }
    if (cudaGetLastError() != cudaSuccess) return GALOP_E_CUDA;

    // Interpreter: the kernel selection and case chunking of the other
    // entry points (enough work items for every resident warp, none longer
    // than kMaxItemCases cases), within the scratch's partial sums.
    const void* fn = opt->num_registers == 8
                         ? interp_kernel_nr8(k, kNaDispatch, opt->profile, opt->reduce, kModeFitness)
                         : interp_kernel_nr16(k, kNaDispatch, opt->profile, opt->reduce, kModeFitness);
    if (!fn) return GALOP_E_INVALID;
    const int threads = 32 * wpb;
    const size_t smem = (size_t)(threads + 32) * opt->num_registers * k * sizeof(float);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) { cudaGetLastError(); return GALOP_E_CUDA; }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return GALOP_E_CUDA;
    }
    per_sm = std::max(per_sm, 1);
    const int64_t resident_warps = (int64_t)sm_count * per_sm * wpb;
    const int64_t pass = 32LL * k;
    const int64_t passes = std::max<int64_t>(1, (n_cases + pass - 1) / pass);
    int64_t n_chunks = 1;
    if (opt->reduce != GALOP_REDUCE_ORDERED) {
        if (n < 4 * resident_warps) n_chunks = std::min<int64_t>(passes, (4 * resident_warps + n - 1) / n);
        n_chunks = std::max<int64_t>(n_chunks, std::min<int64_t>(passes, (n_cases + kMaxItemCases - 1) / kMaxItemCases));
    }
    n_chunks = std::max<int64_t>(1, std::min<int64_t>(n_chunks, kNaMaxPartials / n));
    const int64_t chunk_cases = ((passes + n_chunks - 1) / n_chunks) * pass;
    n_chunks = std::max<int64_t>(1, (std::max<int64_t>(n_cases, 1) + chunk_cases - 1) / chunk_cases);

    InterpArgs a{};
    a.uops = sc->uops;
    a.eff_off = sc->eff_off;
    a.order = sched ? sc->order : nullptr;
    a.n_programs = n;
    a.n_chunks = (int32_t)n_chunks;
    a.chunk_cases = chunk_cases;
    a.X = d_inputs;
    a.y = d_targets;
    a.N = n_cases;
    a.Np = padded_cases;
    a.num_inputs = num_inputs;
    a.output_reg = isa.output_reg;
    a.consts = pool;
    a.counter = sc->counters;
    a.fitness = d_fitness;
    a.sse = d_sse;
    a.partial = n_chunks > 1 ? sc->partial : nullptr;
    const int64_t need = (n * n_chunks + wpb - 1) / wpb;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((int64_t)sm_count * per_sm, need));
    void* params[] = {&a};
    if (cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(threads), params, smem, s) != cudaSuccess) {
        cudaGetLastError();
        return GALOP_E_CUDA;
    }
    if (n_chunks > 1)
        finalize_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(sc->partial, n, (int)n_chunks, n_cases,
                                                                  Objective{}, d_fitness, d_sse);
    poison_results_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(bad, n, d_fitness, d_sse);
    if (cudaGetLastError() != cudaSuccess) return GALOP_E_CUDA;
    return GALOP_OK;
}
