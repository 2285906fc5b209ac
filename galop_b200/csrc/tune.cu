// tune.cu -- the interpreter autotuner (galop_autotune).
//
// Chooses dispatch, cases per lane and warps per block by timing each
// candidate on a sample of the caller's population over the resident
// dataset, and remembers the choice in a JSON-lines cache keyed by the
// device, the ISA, the reduction and the workload's size class.  The
// reference has no tuner: its kernel shape is fixed at compile time
// (src/EvaluatorCuda.cu:28-31, one thread per program, 32 programs per block).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/galop_b200.h"
#include "interp.cuh"
#include "prepass.cuh"

using namespace galop;

#include "context.cuh"

namespace {

int log2_class(double v) {
    return v < 1.0 ? 0 : (int)std::lround(std::log2(v));
}

std::string tune_key(const galop_ctx* ctx, int64_t n_programs, double mean_len) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) {
        cudaGetLastError();
        std::snprintf(prop.name, sizeof prop.name, "device%d", ctx->device);
    }
    std::string name = prop.name;
    for (char& c : name)
        if (c == '"' || c == '\\' || c == '|') c = '_';
    char buf[320];
    std::snprintf(buf, sizeof buf, "%s|sm%d|nr%d|prof%d|ip%d|red%d|intron%d|cases2^%d|len2^%d|progs2^%d",
                  name.c_str(), ctx->sm_count, ctx->isa.num_registers, ctx->isa.profile, ctx->isa.input_protect,
                  ctx->opt.reduce, ctx->opt.intron_prepass ? 1 : 0, log2_class((double)ctx->N),
                  log2_class(mean_len), log2_class((double)n_programs));
    return buf;
}

// Value of "field": <number> in a line of our own cache format.
bool field_num(const std::string& line, const char* field, double* out) {
    const std::string pat = std::string("\"") + field + "\":";
    size_t p = line.find(pat);
    if (p == std::string::npos) return false;
    p += pat.size();
    while (p < line.size() && line[p] == ' ') ++p;
    char* end = nullptr;
    const double v = std::strtod(line.c_str() + p, &end);
    if (end == line.c_str() + p) return false;
    *out = v;
    return true;
}

bool valid_tile(int d, int k, int w) {
    return (d == 2 || d == 3) && (k == 1 || k == 2 || k == 4 || k == 8) && (w >= 1 && w <= 8);
}

// Last cache line with this key, if any.
bool cache_lookup(const char* path, const std::string& key, galop_tune_result* r) {
    std::ifstream f(path);
    if (!f) return false;
    const std::string kpat = "\"key\": \"" + key + "\"";
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        if (line.find(kpat) == std::string::npos) continue;
        double d, k, w, gops = 0.0;
        if (!field_num(line, "dispatch", &d) || !field_num(line, "cases_per_lane", &k) ||
            !field_num(line, "warps_per_block", &w))
            continue;
        if (!valid_tile((int)d, (int)k, (int)w)) continue;
        field_num(line, "gpops", &gops);
        r->dispatch = (int32_t)d;
        r->cases_per_lane = (int32_t)k;
        r->warps_per_block = (int32_t)w;
        r->gpops = gops;
        found = true;
    }
    return found;
}

bool cache_append(const char* path, const std::string& key, const galop_tune_result& r) {
    FILE* f = std::fopen(path, "a");
    if (!f) return false;
    char line[768];
    const int n = std::snprintf(line, sizeof line,
                                "{\"key\": \"%s\", \"dispatch\": %d, \"cases_per_lane\": %d, \"warps_per_block\": %d, "
                                "\"gpops\": %.1f, \"default_gpops\": %.1f, \"candidates\": %d}\n",
                                key.c_str(), r.dispatch, r.cases_per_lane, r.warps_per_block, r.gpops,
                                r.default_gpops, r.candidates);
    const bool ok = n > 0 && n < (int)sizeof line && std::fwrite(line, 1, (size_t)n, f) == (size_t)n;
    return std::fclose(f) == 0 && ok;
}

}  // namespace

extern "C" {

int galop_autotune(galop_ctx* ctx, const uint32_t* words, const int64_t* offsets, int64_t n_programs,
                   int64_t sample_programs, int32_t reps, const char* cache_path, galop_tune_result* out) {
    if (!ctx) return GALOP_E_INVALID;
    if (!out) return ctx->fail(GALOP_E_INVALID, "null result pointer");
    std::memset(out, 0, sizeof *out);
    if (ctx->N < 0) return ctx->fail(GALOP_E_NO_DATASET, "no dataset: call galop_set_dataset first");
    if (n_programs <= 0 || !words || !offsets) return ctx->fail(GALOP_E_INVALID, "empty population");
    if (offsets[0] != 0) return ctx->fail(GALOP_E_INVALID, "offsets[0] != 0");
    for (int64_t i = 0; i < n_programs; ++i)
        if (offsets[i + 1] < offsets[i])
            return ctx->fail(GALOP_E_INVALID, "offsets not non-decreasing at %lld", (long long)i);
    if (sample_programs <= 0) sample_programs = 16384;
    if (reps <= 0) reps = 2;

    const double mean_len = (double)offsets[n_programs] / (double)n_programs;
    const std::string key = tune_key(ctx, n_programs, mean_len);
    std::snprintf(out->key, sizeof out->key, "%s", key.c_str());
    if (cache_path && cache_lookup(cache_path, key, out)) {
        ctx->opt.dispatch = out->dispatch;
        ctx->opt.cases_per_lane = out->cases_per_lane;
        ctx->opt.warps_per_block = out->warps_per_block;
        out->from_cache = 1;
        return GALOP_OK;
    }

    // Every s-th program: the sample keeps the population's length mix.
    const int64_t m = std::min(n_programs, sample_programs);
    const int64_t stride = n_programs / m;
    std::vector<int64_t> so(m + 1, 0);
    std::vector<uint32_t> sw;
    sw.reserve((size_t)(mean_len * m) + 16);
    for (int64_t i = 0; i < m; ++i) {
        const int64_t p = i * stride;
        sw.insert(sw.end(), words + offsets[p], words + offsets[p + 1]);
        so[i + 1] = (int64_t)sw.size();
    }
    std::vector<float> fit((size_t)m);

    const galop_options saved = ctx->opt;
    auto time_tile = [&](int d, int k, int w, double* gops) -> int {
        ctx->opt.dispatch = d;
        ctx->opt.cases_per_lane = k;
        ctx->opt.warps_per_block = w;
        if (int rc = galop_evaluate_csr(ctx, sw.data(), so.data(), m, fit.data(), nullptr)) return rc;
        double best_ms = 1e300;
        for (int r = 0; r < reps; ++r) {
            if (int rc = galop_evaluate_csr(ctx, sw.data(), so.data(), m, fit.data(), nullptr)) return rc;
            best_ms = std::min(best_ms, ctx->stats.interp_ms);
        }
        if (!(best_ms > 0.0)) return ctx->fail(GALOP_E_CUDA, "autotune: no interpreter time measured");
        *gops = (double)ctx->stats.eff_instructions * (double)std::max<int64_t>(ctx->N, 1) / (best_ms * 1e-3) / 1e9;
        return GALOP_OK;
    };

    double def_gops = 0.0;
    if (int rc = time_tile(3, 8, 4, &def_gops)) {
        ctx->opt = saved;
        return rc;
    }
    out->default_gpops = def_gops;
    int best_d = 3, best_k = 8, best_w = 4;
    double best = def_gops;
    int measured = 1;
    const int dispatches[] = {3, 2};
    const int ks[] = {1, 2, 4, 8};
    const int ws[] = {2, 4, 8};
    for (int d : dispatches)
        for (int k : ks)
            for (int w : ws) {
                if (d == 3 && k == 8 && w == 4) continue;
                double g = 0.0;
                if (time_tile(d, k, w, &g) != GALOP_OK) {
                    ctx->err.clear();   // a tile this device cannot run is skipped
                    continue;
                }
                ++measured;
                if (g > best) {
                    best = g;
                    best_d = d;
                    best_k = k;
                    best_w = w;
                }
            }
    ctx->opt = saved;
    ctx->opt.dispatch = best_d;
    ctx->opt.cases_per_lane = best_k;
    ctx->opt.warps_per_block = best_w;
    out->dispatch = best_d;
    out->cases_per_lane = best_k;
    out->warps_per_block = best_w;
    out->gpops = best;
    out->candidates = measured;
    out->sample_programs = m;
    if (cache_path && !cache_append(cache_path, key, *out))
        return ctx->fail(GALOP_E_INVALID, "autotune: cannot append to cache file %s", cache_path);
    return GALOP_OK;
}

}  // extern "C"
