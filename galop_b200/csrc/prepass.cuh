// prepass.cuh -- GPU intron removal, compaction and scheduling.
//
// Structural introns (src/Introns.h:28-46): one backward liveness pass over
// straight-line code is exact, so interpreting only the effective
// instructions yields bit-identical outputs.  The reference runs it on the
// host with OpenMP at the H2D boundary (src/EvaluatorCuda.cu:374-422); here
// it runs on the device, one thread per program, with the live set as a
// bitmask in a register:
//
//   count    eff_len[i] = number of effective instructions (or the raw
//            length when the pass is off)
//   scan     eff_off = exclusive prefix sum (int64), three phases
//   compact  write the micro-ops of the effective instructions, program
//            order preserved, at eff_off[i]
//   order    counting sort of program indices by interpreted length,
//            longest first, for longest-processing-time-first scheduling
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "isa.cuh"
#include "fitness.cuh"

namespace galop {

// Programs as the reference packs them (src/eval_kernels.cuh:292-303).
struct CsrSource {
    const uint32_t* words;
    const int64_t* off;
    __device__ __forceinline__ int64_t start(int64_t i) const { return off[i]; }
    __device__ __forceinline__ int64_t length(int64_t i) const { return off[i + 1] - off[i]; }
};

// The engine's dense layout (src/EvalBackend.h:10-17): stride words per
// program, uint8 lengths.
struct DenseSource {
    const uint32_t* words;
    const uint8_t* lens;
    int64_t stride;
    __device__ __forceinline__ int64_t start(int64_t i) const { return i * stride; }
    __device__ __forceinline__ int64_t length(int64_t i) const { return (int64_t)lens[i]; }
};

constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;                       // per thread
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kOrderBins = 4096;                    // lengths >= kOrderBins-1 share a bin

// Device-side check of CSR offsets that a caller states for a
// device-resident population, before anything reads the program words:
// offsets[0] == 0, every program length in [0, 2^30], offsets[n] ==
// total_words.  A violation sets *bad.  The count and compact kernels given
// `bad` then treat every program as empty (no word is read, no micro-op
// written), so no access leaves the buffers the caller stated, and
// poison_results_kernel turns every fitness and SSE of the call into NaN.
// One thread per offset: grid ceil((n + 1) / 256) x 256.
static __global__ void check_offsets_kernel(const int64_t* __restrict__ off, int64_t n, int64_t total_words,
                                            unsigned long long* __restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    bool ok;
    if (i == n) {
        ok = off[n] == total_words;
    } else {
        const int64_t l = off[i + 1] - off[i];
        ok = l >= 0 && l <= ((int64_t)1 << 30) && (i != 0 || off[0] == 0);
    }
    if (!ok) atomicOr(bad, 1ull);
}

static __global__ void poison_results_kernel(const unsigned long long* __restrict__ bad, int64_t n,
                                             float* __restrict__ fitness, double* __restrict__ sse) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || *bad == 0ull) return;
    fitness[i] = __int_as_float(0x7fc00000);
    if (sse) sse[i] = __longlong_as_double(0x7ff8000000000000ll);
}

template <class Src>
__global__ void prepass_count_kernel(Src src, int64_t n, IsaParams isa, int strip,
                                     int32_t* __restrict__ eff_len,
                                     unsigned long long* __restrict__ totals,
                                     const unsigned long long* __restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t raw = 0, cnt = 0;
    if (i < n && bad != nullptr && *bad != 0ull) {
        eff_len[i] = 0;
    } else if (i < n) {
        const int64_t s = src.start(i);
        raw = src.length(i);
        if (!strip) {
            cnt = raw;
        } else {
            uint32_t live = 1u << isa.output_reg;
#pragma unroll 4
            for (int64_t pc = raw - 1; pc >= 0; --pc) {
                const Decoded d = decode_raw(isa, __ldg(src.words + s + pc));
                if (!((live >> d.dest) & 1u)) continue;
                ++cnt;
                live &= ~(1u << d.dest);
                if (!d.unary) live |= 1u << d.src1;
                if (!d.is_const) live |= 1u << d.src2;
            }
        }
        eff_len[i] = (int32_t)cnt;
    }
    // Block totals of raw and effective lengths (for the stats).
    __shared__ unsigned long long sraw, seff;
    if (threadIdx.x == 0) { sraw = 0; seff = 0; }
    __syncthreads();
    if (raw) atomicAdd(&sraw, (unsigned long long)raw);
    if (cnt) atomicAdd(&seff, (unsigned long long)cnt);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (sraw) atomicAdd(&totals[0], sraw);
        if (seff) atomicAdd(&totals[1], seff);
    }
}

// Phase 1: per-tile sums.
static __global__ void scan_tile_sums_kernel(const int32_t* __restrict__ in, int64_t n,
                                      int64_t* __restrict__ tile_sums) {
    __shared__ int64_t warp_sums[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int64_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        int64_t v = threadIdx.x < kScanThreads / 32 ? warp_sums[threadIdx.x] : 0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (threadIdx.x == 0) tile_sums[blockIdx.x] = v;
    }
}

// Phase 2: exclusive scan of the tile sums in one block (serial over chunks
// of kScanThreads), total written at tile_sums[n_tiles].
static __global__ void scan_tile_offsets_kernel(int64_t* __restrict__ tile_sums, int64_t n_tiles) {
    __shared__ int64_t buf[kScanThreads];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t b = 0; b < n_tiles; b += kScanThreads) {
        const int64_t i = b + threadIdx.x;
        const int64_t v = i < n_tiles ? tile_sums[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < kScanThreads; off <<= 1) {
            const int64_t t = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        const int64_t incl = buf[threadIdx.x];
        const int64_t c = carry;
        if (i < n_tiles) tile_sums[i] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = c + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_sums[n_tiles] = carry;
}

// Phase 3: exclusive scan inside each tile plus the tile offset; out[n] = total.
static __global__ void scan_apply_kernel(const int32_t* __restrict__ in, int64_t n,
                                  const int64_t* __restrict__ tile_offsets, int64_t n_tiles,
                                  int64_t* __restrict__ out) {
    __shared__ int64_t warp_tot[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const int64_t i = base + j;
        v[j] = i < n ? in[i] : 0;
        s += v[j];
    }
    // Inclusive warp scan of per-thread sums.
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t incl = s;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int64_t t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += t;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        int64_t x = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += t;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = x;  // inclusive
    }
    __syncthreads();
    int64_t run = tile_offsets[blockIdx.x] + (w ? warp_tot[w - 1] : 0) + (incl - s);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const int64_t i = base + j;
        if (i < n) out[i] = run;
        run += v[j];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_offsets[n_tiles];
}

__device__ __forceinline__ void put_uop(uint32_t* __restrict__ uops, int64_t pos, const Decoded& d,
                                        const UopFormat& fmt) {
    if (fmt.wide) reinterpret_cast<uint4*>(uops)[pos] = encode_wide(d, fmt.stride, fmt.consts);
    else uops[pos] = encode_uop(d);
}

// Write micro-ops of the interpreted instructions of program i at eff_off[i]
// (one word each, or four in the wide format).  raw_out (optional) receives
// the raw words of the same instructions.
template <class Src>
__global__ void prepass_compact_kernel(Src src, int64_t n, IsaParams isa, int strip,
                                       const int64_t* __restrict__ eff_off,
                                       uint32_t* __restrict__ uops,
                                       uint32_t* __restrict__ raw_out, UopFormat fmt,
                                       const unsigned long long* __restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (bad != nullptr && *bad != 0ull)) return;
    const int64_t s = src.start(i);
    const int64_t raw = src.length(i);
    const int64_t o = eff_off[i];
    if (!strip) {
        for (int64_t pc = 0; pc < raw; ++pc) {
            const uint32_t w = __ldg(src.words + s + pc);
            put_uop(uops, o + pc, decode_raw(isa, w), fmt);
            if (raw_out) raw_out[o + pc] = w;
        }
        return;
    }
    int64_t pos = eff_off[i + 1];   // fill backwards
    uint32_t live = 1u << isa.output_reg;
#pragma unroll 4
    for (int64_t pc = raw - 1; pc >= 0; --pc) {
        const uint32_t w = __ldg(src.words + s + pc);
        const Decoded d = decode_raw(isa, w);
        if (!((live >> d.dest) & 1u)) continue;
        --pos;
        put_uop(uops, pos, d, fmt);
        if (raw_out) raw_out[pos] = w;
        live &= ~(1u << d.dest);
        if (!d.unary) live |= 1u << d.src1;
        if (!d.is_const) live |= 1u << d.src2;
    }
}

// Longest-first order: histogram of bins (bin 0 = longest), scan, scatter.
// A negative length (a copy left out by dedup.cuh) goes to the last bin,
// after every program that is interpreted.
//
// With per-program live-in words (fold.cuh), programs are also grouped by
// register-file class: those whose values fit in split_slots slots come
// first (bins [0, kClassBins)), the others after them (bins [kClassBins,
// 2 kClassBins)), each group longest first; the scan reports the size of
// the first group, where the interpreter's launches split the order.
constexpr int kClassBins = 2047;

__device__ __forceinline__ int order_bin(int l, int cls) {
    if (l < 0) return kOrderBins - 1;
    if (cls < 0) {
        if (l > kOrderBins - 2) l = kOrderBins - 2;
        return kOrderBins - 2 - l;
    }
    if (l > kClassBins - 1) l = kClassBins - 1;
    return cls * kClassBins + (kClassBins - 1 - l);
}

__device__ __forceinline__ int order_class(const uint32_t* livein, int64_t i, int split_slots) {
    if (livein == nullptr) return -1;
    return (int)livein_slots(livein[i]) > split_slots ? 1 : 0;
}

static __global__ void order_hist_kernel(const int32_t* __restrict__ len, int64_t n,
                                  unsigned int* __restrict__ hist, const uint32_t* __restrict__ livein,
                                  int split_slots) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    atomicAdd(&hist[order_bin(len[i], order_class(livein, i, split_slots))], 1u);
}

// split_out (may be null): programs in bins below kClassBins (the first
// register-file class).
static __global__ void order_scan_kernel(unsigned int* __restrict__ hist, unsigned long long* __restrict__ split_out) {
    // Single block of 1024 threads, 4 bins per thread, exclusive in place.
    __shared__ unsigned int buf[1024];
    const int t = threadIdx.x;
    unsigned int v[4], s = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) { v[j] = hist[t * 4 + j]; s += v[j]; }
    buf[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const unsigned int x = t >= off ? buf[t - off] : 0u;
        __syncthreads();
        buf[t] += x;
        __syncthreads();
    }
    unsigned int run = buf[t] - s;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (split_out != nullptr && t * 4 + j == kClassBins) *split_out = run;
        hist[t * 4 + j] = run;
        run += v[j];
    }
}

static __global__ void order_scatter_kernel(const int32_t* __restrict__ len, int64_t n,
                                     unsigned int* __restrict__ cursor,
                                     int32_t* __restrict__ order, const uint32_t* __restrict__ livein,
                                     int split_slots) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned int pos = atomicAdd(&cursor[order_bin(len[i], order_class(livein, i, split_slots))], 1u);
    order[pos] = (int32_t)i;
}

// Case-major (AoS) dataset to feature-major (SoA) with zero padding to Np.
static __global__ void dataset_transpose_kernel(const float* __restrict__ aos, const float* __restrict__ y_in,
                                         int64_t n, int k, int64_t np,
                                         float* __restrict__ X, float* __restrict__ y) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= np) return;
    const bool in = c < n;
    for (int f = 0; f < k; ++f) X[(int64_t)f * np + c] = in ? aos[c * k + f] : 0.0f;
    y[c] = in ? y_in[c] : 0.0f;
}

// Sum of chunk partials in chunk order, then fitness.
static __global__ void finalize_kernel(const double* __restrict__ partial, int64_t n_programs,
                                int n_chunks, int64_t n_cases, Objective obj, float* __restrict__ fitness,
                                double* __restrict__ sse_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_programs) return;
    double s = 0.0;
    for (int c = 0; c < n_chunks; ++c) s += partial[i * n_chunks + c];
    fitness[i] = fitness_of(s, n_cases, obj);
    if (sse_out) sse_out[i] = s;
}

}  // namespace galop
