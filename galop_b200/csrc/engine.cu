// engine.cu -- the evolution loop with the population resident on the GPU
// (galop_engine_*).  Each generation: top-k elites by a radix sort of
// (fitness bits, index) keys, one thread per child pair for tournament
// selection, crossover and mutation, evaluation of the non-elites, and the
// generation statistics in 256 fixed chunks.  Every random draw is the one
// the reference engine makes (engine_rng.cuh), so the run equals
// LGPEngine::evolve_sr with this evaluator as backend.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/galop_b200.h"
#include "context.cuh"
#include "engine_rng.cuh"
#include "isa.cuh"

using namespace galop;

namespace {

constexpr int kStatChunks = 256;          // src/LGPEngine.cpp:486 (fixed chunk count)

struct EngineCfg {
    int64_t P;
    int maxp, start_len, elites, tsize, macro_inserts;
    int effmut, random_pos;
    float crossover_rate, micro_rate, micro_per_instr, effmut_rate, insert_rate, delete_rate;
    IsaParams isa;
    uint32_t reg_mask;
};

// src/ISA.h:106-136 (encode_from_random): every field masked from one draw.
GALOP_HD uint32_t encode_random(uint32_t raw, uint32_t reg_mask) {
    return (raw & 7u) | (raw & (reg_mask << 8)) | (raw & (reg_mask << 16)) | (raw & (reg_mask << 24)) |
           (raw & (0x80u << 24));
}

// src/Introns.h:28-46 with the engine's ISA (SIN/COS are its unary ops).
__device__ int engine_effective_mask(const uint32_t* prog, int len, char* mask, const EngineCfg& c) {
    uint32_t live = 1u << c.isa.output_reg;
    int cnt = 0;
    for (int i = len - 1; i >= 0; --i) {
        const uint32_t w = prog[i];
        const Decoded d = decode_raw(c.isa, w);
        if (!((live >> d.dest) & 1u)) {
            mask[i] = 0;
            continue;
        }
        mask[i] = 1;
        ++cnt;
        live &= ~(1u << d.dest);
        const bool unary = d.op == kSin || d.op == kCos;
        if (!unary) live |= 1u << d.src1;
        if (!d.is_const) live |= 1u << d.src2;
    }
    return cnt;
}

// src/LGPEngine.cpp:148-167 (tournament_t).
__device__ int tournament(Pcg32& r, const float* __restrict__ fit, const EngineCfg& c) {
    int best = uniform_int(r, 0, (int)c.P - 1);
    float best_fit = fit[best];
    for (int a = 1; a < c.tsize; ++a) {
        const int cand = uniform_int(r, 0, (int)c.P - 1);
        const float f = fit[cand];
        if (f > best_fit) {
            best_fit = f;
            best = cand;
        }
    }
    return best;
}

// src/LGPEngine.cpp:293-331 (micro_mutate_instruction_t).
__device__ uint32_t micro_mutate(uint32_t instr, Pcg32& r, const EngineCfg& c) {
    const int field = uniform_int(r, 0, 4);
    const uint32_t bits = uniform_u32(r, 0u, 0xFFFFFFFFu);
    switch (field) {
        case 0: return (instr & ~7u) | (bits & 7u);
        case 1: return (instr & ~(c.reg_mask << 8)) | ((bits & c.reg_mask) << 8);
        case 2: return (instr & ~(c.reg_mask << 16)) | ((bits & c.reg_mask) << 16);
        case 3: return (instr & ~(c.reg_mask << 24)) | ((bits & c.reg_mask) << 24);
        default: return instr ^ (0x80u << 24);
    }
}

// k-th effective position of the mask taken before any insertion
// (src/LGPEngine.cpp:226-231).
__device__ int eff_at(const char* mask, int n, int k) {
    int seen = 0;
    for (int i = 0; i < n; ++i)
        if (mask[i] && seen++ == k) return i;
    return n - 1;
}

// src/LGPEngine.cpp:213-281 (mutate_t), in place on a child slot.
__device__ void mutate(uint32_t* prog, uint8_t& length_io, Pcg32& r, const EngineCfg& c, char* effm) {
    int length = length_io;
    if (length == 0) return;
    const int mask_len = length;
    const int neff = c.effmut ? engine_effective_mask(prog, length, effm, c) : 0;

    if (c.micro_per_instr > 0.0f) {
        for (int i = 0; i < length; ++i)
            if (unit_float(r) < c.micro_per_instr) prog[i] = micro_mutate(prog[i], r, c);
    } else if (unit_float(r) < c.micro_rate) {
        int idx;
        if (c.effmut && neff > 0 && unit_float(r) < c.effmut_rate) idx = eff_at(effm, mask_len, uniform_int(r, 0, neff - 1));
        else idx = uniform_int(r, 0, length - 1);
        prog[idx] = micro_mutate(prog[idx], r, c);
    }

    for (int ins = 0; ins < c.macro_inserts; ++ins) {
        if (unit_float(r) < c.insert_rate) {
            if (length < c.maxp) {
                if (c.random_pos) {
                    int pos;
                    if (c.effmut && neff > 0 && unit_float(r) < c.effmut_rate)
                        pos = eff_at(effm, mask_len, uniform_int(r, 0, neff - 1));
                    else
                        pos = uniform_int(r, 0, length);
                    for (int i = length - 1; i >= pos; --i) prog[i + 1] = prog[i];
                    prog[pos] = encode_random(uniform_u32(r, 0u, 0xFFFFFFFFu), c.reg_mask);
                } else {
                    prog[length] = encode_random(uniform_u32(r, 0u, 0xFFFFFFFFu), c.reg_mask);
                }
                ++length;
            }
        }
    }

    if (unit_float(r) < c.delete_rate) {
        if (length > 1) {
            if (c.random_pos) {
                const int pos = uniform_int(r, 0, length - 1);
                for (int i = pos; i < length - 1; ++i) prog[i] = prog[i + 1];
            }
            --length;
        }
    }
    length_io = (uint8_t)length;
}

// One thread per pair: src/LGPEngine.cpp:442-453 (selection) and :344-373
// (vary_children_t: clone or crossover_t, then mutate both children).
__global__ void vary_kernel(EngineCfg c, uint64_t stream_base, const uint32_t* __restrict__ cur_w,
                            const uint8_t* __restrict__ cur_len, const float* __restrict__ cur_fit,
                            uint32_t* __restrict__ next_w, uint8_t* __restrict__ next_len,
                            float* __restrict__ next_fit, int64_t n_pairs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pairs) return;
    Pcg32 r(stream_base, (uint64_t)i);
    const int pa = tournament(r, cur_fit, c);
    const int pb = tournament(r, cur_fit, c);
    const int64_t da = c.elites + 2 * i, db = da + 1;
    const uint32_t* a = cur_w + (int64_t)pa * c.maxp;
    const uint32_t* b = cur_w + (int64_t)pb * c.maxp;
    const int la = cur_len[pa], lb = cur_len[pb];
    uint32_t* ca = next_w + da * c.maxp;
    uint32_t* cb = next_w + db * c.maxp;
    uint8_t len_a, len_b;
    const bool cross = unit_float(r) < c.crossover_rate;
    const int min_len = la < lb ? la : lb;
    if (!cross || min_len < 2) {
        // clone (no crossover drawn, or src/LGPEngine.cpp:184-191)
        for (int k = 0; k < la; ++k) ca[k] = a[k];
        for (int k = 0; k < lb; ++k) cb[k] = b[k];
        len_a = (uint8_t)la;
        len_b = (uint8_t)lb;
    } else {
        // src/LGPEngine.cpp:193-206: child A = a[:cut] + b[cut:], child B = b[:cut] + a[cut:]
        const int cut = uniform_int(r, 1, min_len - 1);
        for (int k = 0; k < cut; ++k) ca[k] = a[k];
        for (int k = cut; k < lb; ++k) ca[k] = b[k];
        for (int k = 0; k < cut; ++k) cb[k] = b[k];
        for (int k = cut; k < la; ++k) cb[k] = a[k];
        len_a = (uint8_t)lb;
        len_b = (uint8_t)la;
    }
    char effm[256];
    mutate(ca, len_a, r, c, effm);
    mutate(cb, len_b, r, c, effm);
    next_len[da] = len_a;
    next_len[db] = len_b;
    next_fit[da] = __int_as_float(0x7fc00000);
    next_fit[db] = __int_as_float(0x7fc00000);
}

// Keys for the elite selection: fitness bits above the index
// (src/LGPEngine.cpp:383-392), descending order = best first, ties by index.
__global__ void keys_kernel(const float* __restrict__ fit, int64_t P, unsigned long long* __restrict__ keys) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) keys[i] = ((unsigned long long)__float_as_uint(fit[i]) << 32) | (unsigned long long)(uint32_t)i;
}

// src/LGPEngine.cpp:413-421 (copy_elite_to_next), elite e into slot e.
__global__ void elites_kernel(EngineCfg c, const unsigned long long* __restrict__ sorted,
                              const uint32_t* __restrict__ cur_w, const uint8_t* __restrict__ cur_len,
                              const float* __restrict__ cur_fit, uint32_t* __restrict__ next_w,
                              uint8_t* __restrict__ next_len, float* __restrict__ next_fit) {
    const int e = blockIdx.x;
    if (e >= c.elites) return;
    const int64_t src = (int64_t)(uint32_t)sorted[e];
    const int len = cur_len[src];
    for (int k = threadIdx.x; k < len; k += blockDim.x) next_w[(int64_t)e * c.maxp + k] = cur_w[src * c.maxp + k];
    if (threadIdx.x == 0) {
        next_len[e] = (uint8_t)len;
        next_fit[e] = cur_fit[src];
    }
}

// src/LGPEngine.cpp:476-516 (compute_stats), one thread per fixed chunk.
__global__ void stats_kernel(const float* __restrict__ fit, const uint8_t* __restrict__ len, int64_t P,
                             double* __restrict__ csum, long long* __restrict__ clen, float* __restrict__ cbest,
                             int* __restrict__ cidx) {
    const int ch = threadIdx.x;
    if (ch >= kStatChunks) return;
    const int64_t lo = P * ch / kStatChunks, hi = P * (ch + 1) / kStatChunks;
    double s = 0.0;
    long long ls = 0;
    float b = -1.0f;
    int bi = (int)lo;
    for (int64_t i = lo; i < hi; ++i) {
        ls += len[i];
        s = __dadd_rn(s, (double)fit[i]);
        if (fit[i] > b) {
            b = fit[i];
            bi = (int)i;
        }
    }
    csum[ch] = s;
    clen[ch] = ls;
    cbest[ch] = b;
    cidx[ch] = bi;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct galop_engine {
    galop_ctx* ctx = nullptr;
    int device = 0;
    EngineCfg cfg{};
    galop_engine_options opt{};
    DevBuf<uint32_t> words[2];
    DevBuf<uint8_t> lens[2];
    DevBuf<float> fit[2];
    DevBuf<unsigned long long> keys, keys_sorted;
    DevBuf<unsigned char> sort_tmp;
    DevBuf<double> csum;
    DevBuf<long long> clen;
    DevBuf<float> cbest;
    DevBuf<int> cidx;
    int cur = 0;
    galop_engine_times times{};
};

namespace {

#define E_CK(call, what)                                                  \
    do {                                                                  \
        cudaError_t _e = (call);                                          \
        if (_e != cudaSuccess) return e->ctx->cuda_fail(_e, what);        \
    } while (0)

int stats_of(galop_engine* e, int generation, galop_generation_stats* out) {
    const EngineCfg& c = e->cfg;
    cudaStream_t s = e->ctx->stream;
    stats_kernel<<<1, kStatChunks, 0, s>>>(e->fit[e->cur].p, e->lens[e->cur].p, c.P, e->csum.p, e->clen.p,
                                          e->cbest.p, e->cidx.p);
    E_CK(cudaGetLastError(), "stats launch");
    double cs[kStatChunks];
    long long cl[kStatChunks];
    float cb[kStatChunks];
    int ci[kStatChunks];
    E_CK(cudaMemcpyAsync(cs, e->csum.p, sizeof cs, cudaMemcpyDeviceToHost, s), "D2H stats");
    E_CK(cudaMemcpyAsync(cl, e->clen.p, sizeof cl, cudaMemcpyDeviceToHost, s), "D2H stats");
    E_CK(cudaMemcpyAsync(cb, e->cbest.p, sizeof cb, cudaMemcpyDeviceToHost, s), "D2H stats");
    E_CK(cudaMemcpyAsync(ci, e->cidx.p, sizeof ci, cudaMemcpyDeviceToHost, s), "D2H stats");
    E_CK(cudaStreamSynchronize(s), "stats");
    double sum = 0.0;
    long long len_sum = 0;
    float best = -1.0f;
    int best_idx = 0;
    for (int k = 0; k < kStatChunks; ++k) {   // fixed combine order, strict > (lowest index on ties)
        sum += cs[k];
        len_sum += cl[k];
        if (cb[k] > best) {
            best = cb[k];
            best_idx = ci[k];
        }
    }
    uint8_t best_len = 0;
    E_CK(cudaMemcpy(&best_len, e->lens[e->cur].p + best_idx, 1, cudaMemcpyDeviceToHost), "D2H best length");
    out->generation = generation;
    out->best_fitness = best;
    out->mean_fitness = (float)(sum / (double)c.P);
    out->best_length = best_len;
    out->mean_length = (float)((double)len_sum / (double)c.P);
    out->best_index = best_idx;
    return GALOP_OK;
}

int evaluate(galop_engine* e, int64_t first, int64_t count, double* seconds, int64_t* eff) {
    const EngineCfg& c = e->cfg;
    const double t0 = now_s();
    int rc = evaluate_dense_device(e->ctx, e->words[e->cur].p + first * c.maxp, e->lens[e->cur].p + first,
                                   c.maxp, count, e->fit[e->cur].p + first);
    *seconds += now_s() - t0;
    *eff += e->ctx->stats.eff_instructions;
    return rc;
}

}  // namespace

extern "C" {

int galop_engine_options_init(galop_engine_options* o) {
    if (!o) return GALOP_E_INVALID;
    std::memset(o, 0, sizeof *o);
    o->population = 1000;
    o->max_program_size = 50;
    o->starting_program_size = 8;
    o->max_generations = 1000;
    o->elite_count = (int32_t)(1000 * 0.1f);
    o->tournament_size = 3;
    o->macro_inserts = 1;
    o->effmut = 0;
    o->macro_random_pos = 1;
    o->crossover_rate = 1.0f;
    o->micro_rate = 0.8f;
    o->micro_per_instr = 0.0f;
    o->effmut_rate = 1.0f;
    o->insert_tail_rate = 0.8f;
    o->delete_tail_rate = 0.75f;
    o->seed = 42;
    return GALOP_OK;
}

int galop_engine_create(galop_ctx* ctx, const galop_engine_options* o, galop_engine** out) {
    if (!ctx || !o || !out) return GALOP_E_INVALID;
    *out = nullptr;
    if (o->population < 2 || o->population > INT32_MAX || o->elite_count < 0 ||
        o->elite_count > o->population || ((o->population - o->elite_count) & 1) ||
        o->max_program_size < 1 || o->max_program_size > 254 || o->starting_program_size < 1 ||
        o->starting_program_size > o->max_program_size || o->max_generations < 1 || o->tournament_size < 1 ||
        o->macro_inserts < 0)
        return ctx->fail(GALOP_E_INVALID, "bad engine options");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    galop_engine* e = new galop_engine();
    e->ctx = ctx;
    e->device = ctx->device;
    e->opt = *o;
    EngineCfg& c = e->cfg;
    c.P = o->population;
    c.maxp = o->max_program_size;
    c.start_len = o->starting_program_size;
    c.elites = o->elite_count;
    c.tsize = o->tournament_size;
    c.macro_inserts = o->macro_inserts;
    c.effmut = o->effmut ? 1 : 0;
    c.random_pos = o->macro_random_pos ? 1 : 0;
    c.crossover_rate = o->crossover_rate;
    c.micro_rate = o->micro_rate;
    c.micro_per_instr = o->micro_per_instr;
    c.effmut_rate = o->effmut_rate;
    c.insert_rate = o->insert_tail_rate;
    c.delete_rate = o->delete_tail_rate;
    c.isa = ctx->isa;
    c.reg_mask = (uint32_t)ctx->isa.num_registers - 1u;
    const size_t P = (size_t)c.P;
    cudaError_t err = cudaSuccess;
    for (int b = 0; b < 2 && err == cudaSuccess; ++b) {
        err = e->words[b].ensure(P * (size_t)c.maxp);
        if (err == cudaSuccess) err = e->lens[b].ensure(P);
        if (err == cudaSuccess) err = e->fit[b].ensure(P);
    }
    if (err == cudaSuccess) err = e->keys.ensure(P);
    if (err == cudaSuccess) err = e->keys_sorted.ensure(P);
    size_t tmp = 0;
    if (err == cudaSuccess)
        err = cub::DeviceRadixSort::SortKeysDescending(nullptr, tmp, e->keys.p, e->keys_sorted.p, (int)P);
    if (err == cudaSuccess) err = e->sort_tmp.ensure(std::max<size_t>(tmp, 1));
    if (err == cudaSuccess) err = e->csum.ensure(kStatChunks);
    if (err == cudaSuccess) err = e->clen.ensure(kStatChunks);
    if (err == cudaSuccess) err = e->cbest.ensure(kStatChunks);
    if (err == cudaSuccess) err = e->cidx.ensure(kStatChunks);
    if (err != cudaSuccess) {
        galop_engine_destroy(e);
        return ctx->cuda_fail(err, "engine buffers");
    }
    *out = e;
    return GALOP_OK;
}

int galop_engine_destroy(galop_engine* e) {
    if (!e) return GALOP_OK;
    cudaSetDevice(e->device);
    for (int b = 0; b < 2; ++b) {
        e->words[b].release();
        e->lens[b].release();
        e->fit[b].release();
    }
    e->keys.release();
    e->keys_sorted.release();
    e->sort_tmp.release();
    e->csum.release();
    e->clen.release();
    e->cbest.release();
    e->cidx.release();
    delete e;
    return GALOP_OK;
}

int galop_engine_evolve(galop_engine* e, galop_generation_stats* history, int32_t capacity) {
    if (!e) return GALOP_E_INVALID;
    galop_ctx* ctx = e->ctx;
    const EngineCfg& c = e->cfg;
    if (!history || capacity < e->opt.max_generations)
        return ctx->fail(GALOP_E_INVALID, "history needs max_generations rows");
    if (ctx->N < 0) return ctx->fail(GALOP_E_NO_DATASET, "no dataset: call galop_set_dataset first");
    GALOP_CK(cudaSetDevice(ctx->device), "set device");
    cudaStream_t s = ctx->stream;
    e->times = galop_engine_times{};
    const double t_start = now_s();

    // src/LGPEngine.cpp:42-81: sentinels, then one mt19937 draw per
    // instruction slot of buffer 0, lengths = STARTING_PROGRAM_SIZE.
    Mt19937 rng(e->opt.seed);
    const size_t P = (size_t)c.P;
    {
        std::vector<uint32_t> w(P * (size_t)c.maxp);
        for (size_t i = 0; i < w.size(); ++i) w[i] = encode_random(rng.next(), c.reg_mask);
        std::vector<uint8_t> len(P, (uint8_t)c.start_len);
        e->cur = 0;
        E_CK(cudaMemcpyAsync(e->words[0].p, w.data(), w.size() * 4, cudaMemcpyHostToDevice, s), "H2D population");
        E_CK(cudaMemcpyAsync(e->lens[0].p, len.data(), P, cudaMemcpyHostToDevice, s), "H2D lengths");
        E_CK(cudaMemsetAsync(e->lens[1].p, 0xFF, P, s), "sentinel lengths");
        E_CK(cudaStreamSynchronize(s), "H2D population");
    }
    e->times.init_s = now_s() - t_start;

    if (int rc = evaluate(e, 0, c.P, &e->times.evaluate_s, &e->times.eff_instructions)) return rc;
    double t = now_s();
    if (int rc = stats_of(e, 0, &history[0])) return rc;
    e->times.stats_s += now_s() - t;

    const int64_t n_pairs = (c.P - c.elites) / 2;
    size_t tmp_bytes = e->sort_tmp.cap;
    for (int gen = 1; gen < e->opt.max_generations; ++gen) {
        t = now_s();
        const int nx = 1 - e->cur;
        // elites: keys, descending radix sort, copy the first elite_count
        keys_kernel<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(e->fit[e->cur].p, c.P, e->keys.p);
        E_CK(cub::DeviceRadixSort::SortKeysDescending(e->sort_tmp.p, tmp_bytes, e->keys.p, e->keys_sorted.p,
                                                      (int)P, 0, 64, s), "elite sort");
        if (c.elites > 0)
            elites_kernel<<<(unsigned)c.elites, 64, 0, s>>>(c, e->keys_sorted.p, e->words[e->cur].p,
                                                            e->lens[e->cur].p, e->fit[e->cur].p, e->words[nx].p,
                                                            e->lens[nx].p, e->fit[nx].p);
        // two master draws per generation seed the pair streams (src/LGPEngine.cpp:433-436)
        const uint64_t hi = rng.next();
        const uint64_t lo = rng.next();
        const uint64_t base = (hi << 32) | lo;
        if (n_pairs > 0)
            vary_kernel<<<(unsigned)((n_pairs + 127) / 128), 128, 0, s>>>(
                c, base, e->words[e->cur].p, e->lens[e->cur].p, e->fit[e->cur].p, e->words[nx].p, e->lens[nx].p,
                e->fit[nx].p, n_pairs);
        E_CK(cudaGetLastError(), "variation launch");
        E_CK(cudaStreamSynchronize(s), "variation");
        e->cur = nx;
        e->times.select_vary_s += now_s() - t;
        if (int rc = evaluate(e, c.elites, c.P - c.elites, &e->times.evaluate_s, &e->times.eff_instructions))
            return rc;
        t = now_s();
        if (int rc = stats_of(e, gen, &history[gen])) return rc;
        e->times.stats_s += now_s() - t;
    }
    e->times.total_s = now_s() - t_start;
    return GALOP_OK;
}

int galop_engine_population(galop_engine* e, uint32_t* words, uint8_t* lengths, float* fitness) {
    if (!e) return GALOP_E_INVALID;
    galop_ctx* ctx = e->ctx;
    GALOP_CK(cudaSetDevice(e->device), "set device");
    const size_t P = (size_t)e->cfg.P;
    if (words)
        GALOP_CK(cudaMemcpy(words, e->words[e->cur].p, P * (size_t)e->cfg.maxp * 4, cudaMemcpyDeviceToHost),
                 "D2H words");
    if (lengths) GALOP_CK(cudaMemcpy(lengths, e->lens[e->cur].p, P, cudaMemcpyDeviceToHost), "D2H lengths");
    if (fitness) GALOP_CK(cudaMemcpy(fitness, e->fit[e->cur].p, P * 4, cudaMemcpyDeviceToHost), "D2H fitness");
    return GALOP_OK;
}

int galop_engine_times_get(const galop_engine* e, galop_engine_times* out) {
    if (!e || !out) return GALOP_E_INVALID;
    *out = e->times;
    return GALOP_OK;
}

}  // extern "C"
