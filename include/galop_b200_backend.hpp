// galop_b200_backend.hpp -- drop-in EvalBackend for Galop's LGPEngine.
//
// Header-only C++ adapter over the C ABI in galop_b200.h.  It derives from
// the reference's interface (src/EvalBackend.h:8-19), so it is compiled inside
// the reference's build: the reference's src/ directory must be on the
// include path, and its compile-time LGPConfig (register count, constant
// pool, INPUT_PROTECT, MAX_PROGRAM_SIZE) is read from there.
//
//   auto eval = std::make_unique<galop::B200Evaluator>();
//   LGPEngine engine(seed, std::move(eval));        // src/LGPEngine.cpp:94-99
//
// Behaviour of evaluate_population matches CudaEvaluator
// (src/EvaluatorCuda.cu:298-469): synchronous, fitness_out filled on return,
// pointers pre-offset by the caller (src/LGPEngine.cpp:132-139), program i at
// instructions + i*MAX_PROGRAM_SIZE.  The dataset is uploaded when first seen
// and stays resident; residency is keyed on the Dataset's address, case count,
// feature count and a hash of its contents (the reference keys on the address
// alone, src/EvaluatorCuda.cu:309-312, which misses a new Dataset reusing an
// old address).  Errors throw std::runtime_error with the library's message
// instead of exit() (src/cuda_errors.h:3-15).
#pragma once
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "Dataset.h"
#include "EvalBackend.h"
#include "LGPConfig.h"
#include "galop_b200.h"

namespace galop {

class B200Evaluator : public EvalBackend {
public:
    // Options matching the build's LGPConfig: REF profile, NUM_REGISTERS,
    // CONSTANTS, INPUT_PROTECT.  Fitness reduction ORDERED (the CPU's
    // case-order double sum, src/Evaluator.cpp:23-42) unless overridden.
    static galop_options options_from_config(int reduce = GALOP_REDUCE_ORDERED, int device = 0) {
        galop_options o;
        galop_options_init(&o);
        o.profile = GALOP_PROFILE_REF;
        o.num_registers = LGPConfig::NUM_REGISTERS;
        o.input_protect = LGPConfig::INPUT_PROTECT ? 1 : 0;
        o.constants = LGPConfig::CONSTANTS.data();
        o.reduce = reduce;
        o.device = device;
        return o;
    }

    explicit B200Evaluator(const galop_options& opt = options_from_config()) {
        const int rc = galop_create(&opt, &ctx_);
        if (rc != GALOP_OK)
            throw std::runtime_error(std::string("galop_create: ") + galop_status_string(rc));
    }
    B200Evaluator(const B200Evaluator&) = delete;
    B200Evaluator& operator=(const B200Evaluator&) = delete;
    ~B200Evaluator() override { galop_destroy(ctx_); }

    void evaluate_population(const uint32_t* instructions, const uint8_t* lengths, float* fitness_out,
                             int n_programs, const Dataset& ds) override {
        ensure_dataset(ds);
        check(galop_evaluate_population(ctx_, instructions, lengths, LGPConfig::MAX_PROGRAM_SIZE,
                                        n_programs, fitness_out));
    }

    galop_stats last_stats() const {
        galop_stats s;
        galop_last_stats(ctx_, &s);
        return s;
    }
    galop_ctx* context() const { return ctx_; }

private:
    static uint64_t fnv1a(const void* p, size_t n, uint64_t h) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ULL; }
        return h;
    }

    void ensure_dataset(const Dataset& ds) {
        uint64_t h = 1469598103934665603ULL;
        h = fnv1a(ds.inputs.data(), (size_t)ds.N * ds.num_inputs * sizeof(float), h);
        h = fnv1a(ds.targets.data(), (size_t)ds.N * sizeof(float), h);
        if (&ds == ds_ptr_ && ds.N == ds_n_ && ds.num_inputs == ds_k_ && h == ds_hash_) return;
        check(galop_set_dataset(ctx_, ds.inputs.data(), ds.targets.data(), ds.N, ds.num_inputs));
        ds_ptr_ = &ds;
        ds_n_ = ds.N;
        ds_k_ = ds.num_inputs;
        ds_hash_ = h;
    }

    void check(int rc) const {
        if (rc != GALOP_OK)
            throw std::runtime_error(std::string("galop: ") + galop_status_string(rc) + ": " +
                                     galop_last_error(ctx_));
    }

    galop_ctx* ctx_ = nullptr;
    const Dataset* ds_ptr_ = nullptr;
    int ds_n_ = -1, ds_k_ = -1;
    uint64_t ds_hash_ = 0;
};

}  // namespace galop
